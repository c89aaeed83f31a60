// Chebyshev time evolution (KuboChebyshevEvolve / KuboEvol): placeholder until the kernels land.
#include "gbn_internal.cuh"

namespace gbn {

int cheb_evolve(gbn_ctx* c, int32_t, const double*, int32_t, double, double, double*)
{
    return fail(c, GBN_ERR_STATE, "Chebyshev evolution is not built yet");
}

int kubo_evol(gbn_ctx* c, int32_t, const double*, int32_t, double, double, int32_t, double*, double*)
{
    return fail(c, GBN_ERR_STATE, "Kubo time evolution is not built yet");
}

}  // namespace gbn
