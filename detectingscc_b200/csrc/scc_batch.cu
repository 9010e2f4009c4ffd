// Batched form (placeholder until the batch kernel lands).
#include "../../include/scc_b200.h"

extern "C" int scc_batch_create(scc_context *, const scc_csr_view *, uint32_t, scc_batch **out)
{
    if (out) *out = nullptr;
    return SCC_ERR_INVALID_ARG;
}
extern "C" int scc_batch_run(scc_batch *, int, uint32_t, int, uint32_t *, scc_batch_result *, scc_stats *)
{
    return SCC_ERR_INVALID_ARG;
}
extern "C" int scc_batch_destroy(scc_batch *) { return SCC_OK; }
