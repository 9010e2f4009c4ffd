/*
 * scc_b200.h -- C ABI of the B200 SCC engine (libscc_b200.so).
 *
 * Plain C types only: pointers, sizes, integer codes.  No function crosses
 * the ABI with an exception or a process exit; every entry point returns an
 * scc_status code.
 *
 * Graph layout is the reference's (load.cpp:49-113): vertices are 1..V;
 * Fr and Br hold V+2 offsets with Fr[0] = Fr[1] = 0 and Fr[V+1] = E; vertex v
 * owns Fc[Fr[v] .. Fr[v+1]); (Br, Bc) is the transpose.  RSize in the
 * reference's signatures is V and CSize is E (load.cpp:133-134).
 */
#ifndef SCC_B200_H
#define SCC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
typedef enum {
    SCC_OK = 0,
    SCC_ERR_INVALID_ARG = 1,    /* bad algorithm, warp width, null pointer */
    SCC_ERR_CUDA = 2,           /* a CUDA runtime call failed */
    SCC_ERR_OOM = 3,            /* device allocation failed */
    SCC_ERR_TOO_LARGE = 4,      /* V or E above SCC_MAX_VERTICES / SCC_MAX_EDGES */
    SCC_ERR_NO_DEVICE = 5,      /* no CUDA device / wrong architecture */
    SCC_ERR_BUDGET = 6,         /* batch or serving memory budget exceeded */
    SCC_ERR_IO = 7,             /* graph file could not be read */
    SCC_ERR_OVERFLOW = 20,      /* an internal work list overflowed (bug guard) */
    SCC_ERR_NOT_CONVERGED = 21, /* a convergence loop hit its iteration cap */
    SCC_ERR_TIMEOUT = 22,       /* a grid barrier wait timed out */
    SCC_ERR_BAD_GRAPH = 23      /* offsets not monotone / ids outside [1, V] */
} scc_status;

/* ---- algorithms: the reference's -a letters (scc.cu:78-102) ------------- */
typedef enum {
    SCC_ALGO_VHONG = 'g',  /* vHong  scc_WCC.cu:573       */
    SCC_ALGO_VSLOTA = 'h', /* vSlota scc_Coloring.cu:403  */
    SCC_ALGO_WHONG = 'x',  /* wHong  scc_WCC.cu:53        */
    SCC_ALGO_WSLOTA = 'y'  /* wSlota scc_Coloring.cu:6    */
} scc_algo;

/* ---- flags ------------------------------------------------------------- */
#define SCC_FLAG_TRIM1 0x1u          /* -p 1 */
#define SCC_FLAG_TRIM2 0x2u          /* -q 1 (used by Hong; Slota ignores it, as the reference does) */
#define SCC_FLAG_DEVICE 0x4u         /* CSR arrays and labels_out are device pointers */
#define SCC_FLAG_INSTRUMENT 0x8u     /* count adjacency entries / vertex visits (slower) */
#define SCC_FLAG_FORCE_GRID 0x10u    /* always use the whole-GPU persistent launch */
#define SCC_FLAG_FORCE_BLOCK 0x20u   /* always use the single-CTA launch */
#define SCC_FLAG_BATCH_SEQUENTIAL 0x40u /* scc_batch_run: one plain scc_run per graph (the baseline) */
#define SCC_FLAG_DERIVE_REVERSE 0x80u /* scc_run: Br/Bc are not read (may be NULL); the reverse CSR is built on
                                         the device from Fr/Fc, in the reference loader's layout (in-lists in
                                         ascending source order), so only the forward CSR crosses PCIe.  No
                                         counterpart in the reference, whose loader builds both on the host. */

#define SCC_MAX_VERTICES 268435454u  /* 2^28 - 2 */
#define SCC_MAX_EDGES 4294967040u     /* 2^32 - 256 */

typedef struct {
    uint32_t num_vertices;  /* V  (RSize) */
    uint32_t num_edges;     /* E  (CSize) */
    const uint32_t *Fr;     /* V+2 forward offsets  */
    const uint32_t *Fc;     /* E forward columns    */
    const uint32_t *Br;     /* V+2 reverse offsets  */
    const uint32_t *Bc;     /* E reverse columns    */
} scc_csr_view;

typedef struct {
    uint64_t num_sccs;       /* trim1 + trim2 + pivot SCCs: the reference's "Number Of Sccs" */
    uint64_t num_trim1;      /* the reference's numberOf1Sccs (scc_WCC.cu:948) */
    uint64_t num_trim2;      /* trim-2 pairs */
    uint64_t num_pivot;      /* SCCs found from a pivot / colouring root */
    uint64_t edges_scanned;  /* adjacency entries read (SCC_FLAG_INSTRUMENT) */
    uint64_t vertex_visits;  /* vertex visits (SCC_FLAG_INSTRUMENT) */
    uint32_t passes;         /* device passes (barrier-separated steps) */
    uint32_t outer_iters;    /* Hong main-loop iterations / Slota colouring peels */
    uint32_t tail_pass;      /* pass at which one CTA took over (0 = never) */
    uint32_t gpu_launches;   /* kernels this call launched */
    uint32_t grid_blocks;    /* CTAs of the main launch */
    uint32_t used_block_path;/* 1 when the single-CTA launch ran the graph */
    float kernel_ms;         /* main SCC kernel, CUDA events on the call's stream */
    float total_ms;          /* whole call on the device, copies included */
    int32_t error_where;     /* internal location of a device-side error */
} scc_stats;

typedef struct scc_context scc_context;

/* Create a context on CUDA device `device` (owns a stream and a device
 * workspace that grows to the largest graph it has run). */
int scc_create(int device, scc_context **out);
int scc_destroy(scc_context *ctx);

/* Run one SCC decomposition.
 *   algo        one of scc_algo ('g', 'h', 'x', 'y')
 *   flags       SCC_FLAG_*
 *   warp_width  virtual-warp width W for 'x' / 'y' (1, 2, 4, 8, 16, 32);
 *               ignored for 'g' / 'h'
 *   labels_out  V entries or NULL: labels_out[i] = smallest vertex id of
 *               the SCC of vertex i+1 (1-based ids, canonical labels)
 *   stats       optional
 *   stream      cudaStream_t to run on; NULL is the legacy default stream.
 *               Device inputs must be complete in that stream's order.
 * With SCC_FLAG_DEVICE the CSR arrays and labels_out are device pointers;
 * otherwise they are host pointers and the call copies them.  Synchronous:
 * returns after the result (and the labels) are complete.
 * Replaces the bodies of vHong / vSlota / wHong / wSlota (scc.h:49-52,
 * scc_WCC.cu:53,573, scc_Coloring.cu:6,403), which return nothing and
 * print their count. */
int scc_run(scc_context *ctx, const scc_csr_view *g, int algo, uint32_t flags, int warp_width,
            uint32_t *labels_out, scc_stats *stats, void *stream);

/* scc_run without the wait, for device-resident pipelines: the same work is
 * enqueued on `stream` (SCC_FLAG_DEVICE required: inputs and labels_out are
 * device pointers) and the call returns; labels_out is complete in the
 * stream's order.  scc_finish waits for the last run enqueued on the
 * context and returns its status and stats (the same as scc_run's).  Until
 * then the context's workspace belongs to that run: the next run on the
 * context must be on the same stream or after scc_finish.  No counterpart in
 * the reference, whose drivers block on the host after every BFS level. */
int scc_run_async(scc_context *ctx, const scc_csr_view *g, int algo, uint32_t flags, int warp_width,
                  uint32_t *labels_out, void *stream);
int scc_finish(scc_context *ctx, scc_stats *stats);

/* The reverse CSR built on the device from the forward one, in the reference
 * loader's layout (load.cpp:47-113: Br[0] = Br[1] = 0, in-lists in ascending
 * source order).  All pointers are device pointers; Br has V+2 entries, Bc E.
 * Synchronous on `stream`.  Ids outside [1, V] or malformed offsets give
 * SCC_ERR_BAD_GRAPH.  No counterpart in the reference, which builds both
 * CSRs on the host.  Uses (and keeps) temporaries of about 12 B per edge. */
int scc_derive_reverse(scc_context *ctx, const uint32_t *Fr, const uint32_t *Fc, uint32_t V, uint32_t E,
                       uint32_t *Br, uint32_t *Bc, void *stream);

/* Tuning knobs (used by tests and the batch autotuner):
 *   "tail_vertices"       live-vertex count under which CTA 0 finishes alone
 *   "block_max_vertices"  graphs up to this V run on the single-CTA path
 *   "block_max_edges"     ... and up to this E
 *   "timeout_ms"          bound on any grid-barrier wait (default 4000)
 *   "max_blocks_per_sm"   cap on CTAs per SM of the persistent launch
 *   "trace"               record a per-pass trace of up to `value` passes
 *   "bu_k"                bottom-up BFS step when the frontier's edges exceed
 *                         bu_k * (vertices the search can reach) (default 2,
 *                         0 = never)
 *   "warp_schedule"       wHong / wSlota top-down expansion: 0 = the
 *                         virtual-warp schedule (W lanes per vertex, the
 *                         reference's fwd_warp<W>) when W > 1 and
 *                         E >= W * V, else the warp walk of the vertex
 *                         drivers (default); 1 =
 *                         always virtual warps; 2 = always the warp walk.
 *                         Results do not depend on it.
 *   "pull_lane"           bottom-up step: adjacency lists up to this length
 *                         are tested by their lane alone; of a longer list
 *                         the lane tests the first min(8, pull_lane) entries
 *                         and the whole warp the rest (1..1024, default 4)
 *   "qcap"                entries of each warp's shared-memory staging slice
 *                         (32..576; 3 queues x 32 warps x qcap x 4 bytes on
 *                         the whole-GPU kernel, 2 queues on one CTA)
 *   "cluster_check"       batched launches with clusters use a software
 *                         barrier in global memory whose waits end after
 *                         timeout_ms with SCC_ERR_TIMEOUT (a check mode;
 *                         default 0: the hardware cluster barrier)
 *   "max_passes"          a run stops with SCC_ERR_NOT_CONVERGED once it has
 *                         made this many device passes (0, the default: no
 *                         cap beyond the V + 2 passes of every loop)
 *   "test_withhold_arrival"  failure-detection test hook: with k + 1, one CTA
 *                         of a whole-GPU launch (or of a cluster in check
 *                         mode) withholds its barrier arrival at pass k, so
 *                         every wait of that barrier runs out after
 *                         timeout_ms and the run ends with SCC_ERR_TIMEOUT;
 *                         0 (the default) turns it off */
int scc_set_tuning(scc_context *ctx, const char *key, long long value);

/* Per-pass trace of the last run (enable with scc_set_tuning(ctx, "trace",
 * max_passes)): two words per pass, [2i] = %globaltimer (ns) at the end of
 * pass i, [2i+1] = phase id | (items pushed << 8).  *n_out = passes
 * recorded, *t_start = %globaltimer at kernel entry.  The reference keeps
 * per-phase CUDA-event timers behind #define _DEBUG (scc_WCC.cu:650-672). */
int scc_get_trace(scc_context *ctx, uint64_t *out, uint32_t cap, uint32_t *n_out, uint64_t *t_start);

/* Human-readable text for a status code. */
const char *scc_status_string(int status);

/* Library version string. */
const char *scc_version(void);

/* ---- run without device allocation ------------------------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory when they need an SCC -- a process whose GPU memory is reserved up
 * front by another allocator (a framework's caching pool, a serving process
 * with a fixed budget), or a plugin whose host forbids allocations outside
 * its own pool.  Runs the single-CTA SCC kernel on a scratch area that is a
 * static __device__ array inside the library (about 1.2 MiB, held by every
 * GPU that loads the library until the process exits); the caller passes
 * device CSR arrays (SCC_FLAG_DEVICE is required) and a device buffer of V
 * labels.  Graphs above SCC_NOALLOC_MAX_VERTICES / SCC_NOALLOC_MAX_EDGES
 * are rejected with SCC_ERR_TOO_LARGE.  Accepted flags: SCC_FLAG_DEVICE
 * (required), SCC_FLAG_TRIM1, SCC_FLAG_TRIM2; any other flag is rejected with
 * SCC_ERR_INVALID_ARG.  The first call on a device (with that device
 * current) looks up the array's device address; make it before any stream
 * capture.  The address is kept per CUDA context, so a call in a context
 * created later (after cudaDeviceReset, say) looks it up again.  All calls
 * share the array: calls that overlap on the GPU race.  Calls no cudaMalloc,
 * cudaFree or allocating library routine.  Synchronous; `stream` as in
 * scc_run. */
#define SCC_NOALLOC_MAX_VERTICES 16384u
#define SCC_NOALLOC_MAX_EDGES 262144u
int scc_run_noalloc(const scc_csr_view *g, int algo, uint32_t flags, int warp_width, uint32_t *labels_out,
                    scc_stats *stats, void *stream);

/* ---- serving form: continuous batching under a device-memory budget ---- */
/* No counterpart in the reference.  A request is one host CSR plus a host
 * buffer for its V labels; both stay owned by the caller and must remain
 * valid until the request's result is polled.  `lanes` worker threads, each
 * with its own stream, take whatever has arrived: a graph above
 * large_vertices alone, on one thread-block cluster of large_cluster CTAs;
 * otherwise every waiting small graph (up to max_graphs_per_batch) in one
 * batched launch, graphs of at least big_vertices vertices on clusters of
 * `cluster` CTAs and the rest one per CTA.  Lanes run concurrently: copies
 * and kernels of later arrivals overlap on the device with earlier work,
 * and no launch needs the whole GPU.  CSR arrays in page-locked memory are
 * copied by DMA directly; pageable ones go through the lane's page-locked
 * staging.  All device memory the server holds stays within budget_bytes;
 * a request that cannot fit even alone gets SCC_ERR_BUDGET.  Zero fields
 * take the defaults shown. */
typedef struct {
    uint64_t budget_bytes;          /* 120e9 */
    uint32_t lanes;                 /* 8 */
    uint32_t max_graphs_per_batch;  /* 512 */
    uint32_t large_vertices;        /* 65536 */
    int32_t batch_threads;          /* 1024 (128, 256, 512, 1024) */
    uint32_t qcap;                  /* 256 (32..768) */
    int32_t algo;                   /* SCC_ALGO_VSLOTA */
    uint32_t flags;                 /* SCC_FLAG_TRIM1 | SCC_FLAG_TRIM2 as wanted (host inputs only) */
    int32_t warp_width;             /* 1 */
    uint32_t cluster;               /* 4 (1, 2, 4, 8, 16) */
    uint32_t big_vertices;          /* 16384 */
    uint32_t large_cluster;         /* 16, or the largest cluster the device holds */
} scc_server_config;

typedef struct {
    uint64_t ticket;
    int32_t status;
    uint32_t num_vertices;
    uint64_t num_sccs;
    uint64_t num_trim1;
    double latency_ms;              /* submit -> labels in the caller's buffer */
    double queue_ms;                /* submit -> a lane started it */
    int32_t lane;
    uint32_t reserved;
} scc_server_result;

typedef struct scc_server scc_server;
int scc_server_create(int device, const scc_server_config *cfg, scc_server **out);
/* Thread-safe.  *ticket identifies the request in its result. */
int scc_server_submit(scc_server *s, const scc_csr_view *host_graph, uint32_t *labels_out, uint64_t *ticket);
/* Returns up to cap finished results (waits up to wait_ms for one). */
int scc_server_poll(scc_server *s, scc_server_result *out, uint32_t cap, uint32_t *n, int wait_ms);
int scc_server_info(scc_server *s, uint64_t *pending, uint64_t *completed, uint64_t *held_bytes, uint64_t *rejected);
/* Kernel launches the server has made so far. */
int scc_server_launches(scc_server *s, uint64_t *launches);
/* Finishes every submitted request, then frees everything. */
int scc_server_destroy(scc_server *s);

/* ---- graph files ------------------------------------------------------ */
/* A host CSR owned by the library (arrays allocated with new[], as the
 * reference loader does, load.cpp:52-115). */
typedef struct {
    uint32_t V, E;
    uint32_t *Fr, *Fc, *Br, *Bc;
    uint32_t *Pr;           /* METIS partition ids (detectSCC only): read from the file named by the
                               environment variable SCC_METIS_PARTITION when it is set, else zero-filled */
} scc_host_graph;

/* Read a GTgraph text file (load.cpp:12-140 semantics) or a binary CSR file
 * ("SCCBIN01", u64 V, u64 E, Fr[V+2], Fc[E], Br[V+2], Bc[E], uint32 LE). */
int scc_load_graph(const char *path, scc_host_graph *out);
/* Write the binary CSR format. */
int scc_save_binary(const char *path, const scc_host_graph *g);
/* Write GTgraph text that loadFullGraph reads back as g: seven comment
 * lines, "p sp V E", then one "a u v 1" line per arc in forward order. */
int scc_save_gtgraph(const char *path, const scc_host_graph *g);
/* Read a GTgraph text file (or the binary CSR format) and build both CSRs
 * on the device (load.cpp:12-113 semantics): the host reads the bytes and
 * the header, the device parses the arc lines -- one arc "a u v w" per line,
 * as GTgraph writes them; a line that does not parse, fewer arcs than the
 * header announces, or an id outside [1, V] gives SCC_ERR_BAD_GRAPH --
 * orders the arcs by (u, v) and builds the reverse CSR.  *out receives
 * device pointers into the context's CSR arrays, valid until the next call
 * of this function or of scc_run with host inputs on the same context. */
int scc_load_graph_device(scc_context *ctx, const char *path, scc_csr_view *out, void *stream);
/* Build forward + reverse CSR from E arcs (1-based ids in [1, V]). */
int scc_graph_from_arcs(uint32_t V, uint64_t E, const uint32_t *src, const uint32_t *dst,
                        scc_host_graph *out);
void scc_free_host_graph(scc_host_graph *g);

/* ---- METIS input converter and partitions ------------------------------ */
/* Replaces the reference's converter tool (MetisInput.cpp:12-141, its
 * loadFullGraph + writer): writes g in that tool's layout -- a line "V E",
 * then for every vertex 1..V one line with its out-neighbours (forward list
 * order) followed by its in-neighbours (reverse list order), each number
 * followed by one space (MetisInput.cpp:114-131).  Duplicate arcs appear as
 * often as they occur, as there. */
int scc_save_metis(const char *path, const scc_host_graph *g);
/* Reads a METIS partition file (one partition id per vertex, whitespace
 * separated, load.cpp:115-130) into Pr[1..V]; Pr[0] and Pr[V+1] are set to
 * 0.  Pr must hold V+2 entries. */
int scc_load_partition(const char *path, uint32_t V, uint32_t *Pr);

/* ---- detectSCC (-a d) -------------------------------------------------- */
/* The reference's METIS-partitioned driver (scc_WCC.cu:1000-1617): SCCs
 * inside every partition (Pr[v], V + 2 entries, host), then pairwise merges
 * of partitions 2k and 2k+1 through the edges that cross them, with the
 * reference's own range arithmetic.  num_sccs is what the reference prints
 * (trim-1 tags + trim-2 tags + distinct range values of the other vertices),
 * which is not always the number of SCCs: values that coincide count once.
 * Host CSR only; flags: SCC_FLAG_TRIM1, SCC_FLAG_TRIM2.  Partition ids may
 * be any uint32 (the reference indexes 10 fixed pivot tables with them,
 * scc_WCC.cu:1035).  The merge tests every pair of crossing edges, as the
 * reference does: meant for the small graphs that driver was written for. */
typedef struct {
    uint64_t num_sccs;      /* the reference's "Number Of Sccs" */
    uint64_t num_trim1, num_trim2, num_ranges;
    uint32_t merge_rounds;  /* the reference's "Iterations k" lines */
    uint32_t nospace_mask;  /* bit r-1: round r printed "No space!" */
} scc_detect_result;
int scc_detect(scc_context *ctx, const scc_csr_view *host_graph, const uint32_t *Pr, uint32_t flags,
               scc_detect_result *out);
/* detectSCC with the reference's stdout (scc_WCC.cu:1264-1561): its progress
 * lines, "Iterations k" per merge round, then "\nNumber Of Sccs : N" and
 * "\nTime : T\n".  The C++ shim detectSCC (include/scc_compat.h) calls it. */
int scc_reference_detect(uint32_t CSize, uint32_t RSize, const uint32_t *Fc, const uint32_t *Fr, const uint32_t *Bc,
                         const uint32_t *Br, const uint32_t *Pr, int t1, int t2, uint64_t *num_sccs_out);

/* ---- reference-compatible driver call ----------------------------------- */
/* Runs one of the reference drivers with its exact stdout: for 'g' the line
 * "numberOf1Sccs: N\n", then "\nNumber Of Sccs : N" and "\nTime : T" (ms,
 * from entry to the count, scc_WCC.cu:577-581,948-967).  Returns a status
 * instead of exiting.  The C++ shims vHong / vSlota / wHong / wSlota
 * (include/scc_compat.h) call it. */
int scc_reference_call(int algo, uint32_t CSize, uint32_t RSize, const uint32_t *Fc, const uint32_t *Fr,
                       const uint32_t *Bc, const uint32_t *Br, int t1, int t2, int warp_width,
                       uint64_t *num_sccs_out);

/* ---- batched form: many independent graphs, one persistent launch ------ */
/* No counterpart in the reference, which runs one graph per process.  The
 * graphs are uploaded once (host CSR views) into one device arena and stay
 * resident until scc_batch_destroy.  scc_batch_run runs all of them in one
 * launch (captured once into a CUDA graph and replayed): every CTA takes the
 * next graph, largest first, and runs the same driver code as scc_run on a
 * private scratch slice.  With SCC_FLAG_BATCH_SEQUENTIAL it instead calls
 * scc_run once per graph, in order, on one stream (the baseline). */
typedef struct scc_batch scc_batch;

typedef struct {
    uint64_t num_sccs;
    uint64_t num_trim1;
    int32_t status;     /* SCC_OK or the graph's own error; other graphs are unaffected */
    uint32_t reserved;
} scc_batch_result;

int scc_batch_create(scc_context *ctx, const scc_csr_view *graphs, uint32_t n, scc_batch **out);
/* labels_out (host, optional): the concatenation of every graph's V labels in
 * batch order; results (host, optional): n entries.  Returns SCC_OK or the
 * first graph error. */
int scc_batch_run(scc_batch *b, int algo, uint32_t flags, int warp_width, uint32_t *labels_out,
                  scc_batch_result *results, scc_stats *stats);
/* Schedule of the batched launch: CTA size (128, 256, 512, 1024) and the
 * per-warp staging slice (32..768 entries). */
int scc_batch_set_schedule(scc_batch *b, int threads, uint32_t qcap);
int scc_batch_get_schedule(scc_batch *b, int *threads, uint32_t *qcap);
/* Thread-block clusters: with cluster > 1 (2, 4, 8, 16) the launch is made of
 * clusters of that many CTAs, and every graph with at least big_vertices
 * vertices runs on a whole cluster (the CTAs share one scratch slice and
 * meet at the hardware cluster barrier), before the remaining graphs run
 * one per CTA.  cluster 1 (the default) runs every graph on one CTA. */
int scc_batch_set_cluster(scc_batch *b, int cluster, uint32_t big_vertices);
int scc_batch_get_cluster(scc_batch *b, int *cluster, uint32_t *big_vertices, uint32_t *num_cluster_graphs);
/* Times every candidate schedule on the batch and keeps the fastest: CTA
 * size and staging slice first, then cluster size and big_vertices, then
 * the processing order (largest first by size, or longest first by each
 * graph's own time in a run with the chosen schedule). */
int scc_batch_autotune(scc_batch *b, int algo, uint32_t flags, int warp_width, int *best_threads,
                       uint32_t *best_qcap, float *best_ms);
int scc_batch_info(scc_batch *b, uint64_t *num_vertices, uint64_t *num_edges, uint32_t *num_graphs);
int scc_batch_destroy(scc_batch *b);

#ifdef __cplusplus
}
#endif

#endif /* SCC_B200_H */
