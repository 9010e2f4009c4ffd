// The reference's driver entry points (scc.h:49-52) on top of the C ABI.
//
// Each shim keeps the reference's observable behaviour:
//   * output: vHong prints "numberOf1Sccs: N\n" (scc_WCC.cu:948); every
//     driver prints "\nNumber Of Sccs : N" and "\nTime : T" with T in ms
//     from function entry to the end of the count (scc_WCC.cu:577-581,
//     951-967; scc_Coloring.cu:407-411, 654-670);
//   * errors: out of device memory throws the reference's const char*
//     (scc_WCC.cu:618-623, caught in scc.cu:104-108); any other failure
//     prints a GPUassert-style line and exits with the code (scc.h:12-20).
// The device work itself is scc_run (scc_engine.cu).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "../../include/scc_compat.h"
#include "scc_host.h"

namespace {

std::mutex g_mu;
scc_context *g_ctx = nullptr;
int g_ctx_status = SCC_OK;

scc_context *shared_context(int *status)
{
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_ctx && g_ctx_status == SCC_OK) {
        const char *dev = getenv("SCC_DEVICE");
        g_ctx_status = scc_create(dev ? atoi(dev) : 0, &g_ctx);
    }
    *status = g_ctx_status;
    return g_ctx;
}

}  // namespace

extern "C" int scc_reference_call(int algo, uint32_t CSize, uint32_t RSize, const uint32_t *Fc, const uint32_t *Fr,
                                  const uint32_t *Bc, const uint32_t *Br, int t1, int t2, int warp_width,
                                  uint64_t *num_sccs_out)
{
    auto t0 = std::chrono::steady_clock::now();
    int status = SCC_OK;
    scc_context *ctx = shared_context(&status);
    if (!ctx) return status;
    scc_csr_view g{RSize, CSize, Fr, Fc, Br, Bc};
    uint32_t flags = (t1 ? SCC_FLAG_TRIM1 : 0u) | (t2 ? SCC_FLAG_TRIM2 : 0u);
    scc_stats st;
    int rc = scc_run(ctx, &g, algo, flags, warp_width, nullptr, &st, nullptr);
    if (rc != SCC_OK) return rc;
    if (algo == SCC_ALGO_VHONG) printf("numberOf1Sccs: %d\n", (int)st.num_trim1);
    double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    printf("\nNumber Of Sccs : %d", (int)st.num_sccs);
    printf("\nTime : %f", ms);
    if (num_sccs_out) *num_sccs_out = st.num_sccs;
    return SCC_OK;
}

static void run_or_die(int algo, uint32_t CSize, uint32_t RSize, uint32_t *Fc, uint32_t *Fr, uint32_t *Bc,
                       uint32_t *Br, bool t1, bool t2, int warpSize)
{
    int rc = scc_reference_call(algo, CSize, RSize, Fc, Fr, Bc, Br, t1, t2, warpSize, nullptr);
    if (rc == SCC_OK) return;
    if (rc == SCC_ERR_OOM) throw "Error: Not enough memory on GPU\n";
    fprintf(stderr, "GPUassert: %s %s %d\n", scc_status_string(rc), __FILE__, __LINE__);
    exit(rc);
}

void vHong(uint32_t CSize, uint32_t RSize, uint32_t *Fc, uint32_t *Fr, uint32_t *Bc, uint32_t *Br, bool t1, bool t2)
{
    run_or_die(SCC_ALGO_VHONG, CSize, RSize, Fc, Fr, Bc, Br, t1, t2, 1);
}

void vSlota(uint32_t CSize, uint32_t RSize, uint32_t *Fc, uint32_t *Fr, uint32_t *Bc, uint32_t *Br, bool t1, bool t2)
{
    run_or_die(SCC_ALGO_VSLOTA, CSize, RSize, Fc, Fr, Bc, Br, t1, t2, 1);
}

void wHong(uint32_t CSize, uint32_t RSize, uint32_t *Fc, uint32_t *Fr, uint32_t *Bc, uint32_t *Br, bool t1, bool t2,
           int warpSize)
{
    run_or_die(SCC_ALGO_WHONG, CSize, RSize, Fc, Fr, Bc, Br, t1, t2, warpSize);
}

void wSlota(uint32_t CSize, uint32_t RSize, uint32_t *Fc, uint32_t *Fr, uint32_t *Bc, uint32_t *Br, bool t1, bool t2,
            int warpSize)
{
    run_or_die(SCC_ALGO_WSLOTA, CSize, RSize, Fc, Fr, Bc, Br, t1, t2, warpSize);
}

extern "C" int scc_reference_detect(uint32_t CSize, uint32_t RSize, const uint32_t *Fc, const uint32_t *Fr,
                                    const uint32_t *Bc, const uint32_t *Br, const uint32_t *Pr, int t1, int t2,
                                    uint64_t *num_sccs_out)
{
    auto t0 = std::chrono::steady_clock::now();
    int status = SCC_OK;
    scc_context *ctx = shared_context(&status);
    if (!ctx) return status;
    scc_csr_view g{RSize, CSize, Fr, Fc, Br, Bc};
    scc_detect_result r;
    const int rc = scc_detect(ctx, &g, Pr, (t1 ? SCC_FLAG_TRIM1 : 0u) | (t2 ? SCC_FLAG_TRIM2 : 0u), &r);
    if (rc != SCC_OK) return rc;
    printf("LOCAL SCC's IDENTIFIED! NODES WITH SAME RANGE VALUES BELONG TO THE SAME SCC!!\n");
    printf("Fs AND Bs ARE POPULATED!!\n");
    printf("STARTING MERGE!\n");
    for (uint32_t k = 1; k <= r.merge_rounds; k++) {
        printf("Iterations %u\n", k);
        if (k <= 32 && ((r.nospace_mask >> (k - 1)) & 1u)) printf("No space!\n");
    }
    printf("MERGING DONE! ^_^\n");
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    printf("\nNumber Of Sccs : %d", (int)r.num_sccs);
    printf("\nTime : %f\n", ms);
    if (num_sccs_out) *num_sccs_out = r.num_sccs;
    return SCC_OK;
}

// detectSCC (scc.h:53, scc_WCC.cu:1000-1617), the METIS-partitioned
// driver: same stdout, same error policy as the other shims.
void detectSCC(uint32_t CSize, uint32_t RSize, uint32_t *Fc, uint32_t *Fr, uint32_t *Bc, uint32_t *Br, uint32_t *Pr,
               bool t1, bool t2)
{
    int rc = scc_reference_detect(CSize, RSize, Fc, Fr, Bc, Br, Pr, t1, t2, nullptr);
    if (rc == SCC_OK) return;
    if (rc == SCC_ERR_OOM) throw "Error: Not enough memory on GPU\n";
    fprintf(stderr, "GPUassert: %s %s %d\n", scc_status_string(rc), __FILE__, __LINE__);
    exit(rc);
}
