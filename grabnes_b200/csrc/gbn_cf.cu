// Continued-fraction density of states (KuboFrac, lanczosKuboCode/Src/kubosubs.F90:222-288), one
// thread per (right-hand side, energy), FP64 throughout.  g(z) starts from the square-root
// terminator of the last coefficients and is folded back to the first level; complex quotients use
// Smith's method, as GNU Fortran evaluates them.
#include <cuda_runtime.h>
#include <math.h>

#include "gbn_internal.cuh"

namespace gbn {

__device__ __forceinline__ double2 csqrt_principal(double x, double y)
{
    if (x == 0.0 && y == 0.0) return make_double2(0.0, y);
    const double r = hypot(x, y);
    if (x >= 0.0) {
        const double t = sqrt(0.5 * (r + x));
        return make_double2(t, y / (2.0 * t));
    }
    const double t = sqrt(0.5 * (r - x));
    return make_double2(fabs(y) / (2.0 * t), copysign(t, y));
}

__device__ __forceinline__ double2 recip_smith(double c, double d)
{
    if (fabs(c) >= fabs(d)) {
        const double r = d / c, den = c + d * r;
        return make_double2(1.0 / den, -r / den);
    }
    const double r = c / d, den = c * r + d;
    return make_double2(r / den, -1.0 / den);
}

__global__ void k_cf_dos(const double* a, const double* b, const int32_t* nsteps, int32_t nmax, int32_t nrhs,
                         double eta, int32_t n_en, double emin, double de, const double* norm, double* dos)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t ne = (int64_t)n_en + 1;
    if (t >= ne * nrhs) return;
    const int r = (int)(t / ne);
    const int k = (int)(t % ne);
    const int n = nsteps ? nsteps[r] : nmax;
    const double* ar = a + (int64_t)r * nmax;
    const double* br = b + (int64_t)r * nmax;
    const double E = emin + (double)k * de;
    const double ainf = ar[n - 1], binf = br[n - 1];
    const double wr = E - ainf, wi = eta;
    const double w2r = wr * wr - wi * wi, w2i = wr * wi + wi * wr;
    const double bb = binf * binf;
    const double2 s = csqrt_principal(w2r - 4.0 * bb, w2i);
    const double tb = 2.0 * bb;
    double gr = (wr - s.x) / tb, gi = (wi - s.y) / tb;
    if (gi >= 0.0) {
        gr = (wr + s.x) / tb;
        gi = (wi + s.y) / tb;
    }
    for (int i = n - 2; i >= 0; --i) {
        const double b2 = br[i] * br[i];
        const double2 g = recip_smith((E - ar[i]) - b2 * gr, eta - b2 * gi);
        gr = g.x;
        gi = g.y;
    }
    dos[t] = (-gi / 3.14159265358979323846) * (norm ? norm[r] : 1.0);
}

int cf_dos(gbn_ctx* c, int32_t nrhs, const double* d_a, const double* d_b, const int32_t* d_nsteps, int32_t nmax,
           double eta, int32_t n_en, double emin, double emax, const double* d_norm, double* d_dos)
{
    const int64_t tot = ((int64_t)n_en + 1) * nrhs;
    const double de = (emax - emin) / n_en;
    k_cf_dos<<<(unsigned)((tot + 127) / 128), 128, 0, c->stream>>>(d_a, d_b, d_nsteps, nmax, nrhs, eta, n_en, emin,
                                                                    de, d_norm, d_dos);
    GBN_CK_LAUNCH(c);
    return GBN_OK;
}

}  // namespace gbn
