// dpmm_tc.cu -- tensor-core (tcgen05) form of the Gaussian label phase.
#include "dpmm_internal.h"

namespace dpmm {

bool tc_supported(const dpmm_ctx* c, int K)
{
    (void)c;
    (void)K;
    return false;
}

dpmm_status launch_cluster_labels_tc(dpmm_ctx* c, int K, int final_, const float* d_u, float* d_rout)
{
    (void)c; (void)K; (void)final_; (void)d_u; (void)d_rout;
    return fail(DPMM_ERR_INVALID_ARG, "tensor-core label kernel not available");
}

}  // namespace dpmm
