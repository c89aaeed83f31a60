// Host-side set-up of the Chebyshev propagator: the spectral centre and scale (KuboInterval,
// lanczosKuboCode/Src/kubosubs.F90:290-350) and the expansion coefficients (KuboCn, kubosubs.F90:352-433).
//
// KuboInterval takes the extreme eigenvalues of the recursion's tridiagonal matrix (diagonal a,
// off-diagonal b) and returns ac = (emax + emin)/2, bc = 1.2 (emax - emin)/4.  Only the two extreme
// eigenvalues are needed, so they are found by bisection on Sturm counts (the number of negative
// pivots of T - x I in its LDL^T factorisation equals the number of eigenvalues below x), from the
// Gershgorin interval down to the resolution of double precision.
//
// KuboCn diagonalises the Jacobi matrix of the scaled Chebyshev recurrence (diagonal ac, off-diagonal
// bc, the first one sqrt(2) bc) and forms c_n = sum_j v_j(0) v_j(n) exp(-i lambda_j dT), i.e. the
// elements <0| exp(-i J dT) |n>.  Those are known in closed form: the Chebyshev expansion of
// exp(-i x t) has Bessel-function coefficients, so
//     c_0 = exp(-i ac dT) J_0(2 bc dT),   c_n = sqrt(2) (-i)^n exp(-i ac dT) J_n(2 bc dT)   (n >= 1),
// and the J_n are computed here by Miller's backward recurrence J_{k-1} = (2k/x) J_k - J_{k+1} from a
// start well above max(n, x), normalised with J_0 + 2 sum_{k>=1} J_{2k} = 1 (J. C. P. Miller, 1952).
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

#include "../../include/grabnes_gpu.h"

namespace {

// eigenvalues of T strictly below x
int sturm_below(const double* a, const double* b, int n, double x)
{
    int cnt = 0;
    double q = 1.0;
    for (int i = 0; i < n; ++i) {
        const double off = (i > 0) ? b[i - 1] * b[i - 1] : 0.0;
        if (q == 0.0) q = 1e-300;   // a zero pivot is perturbed to the positive side
        q = (a[i] - x) - (i > 0 ? off / q : 0.0);
        if (q < 0.0) ++cnt;
    }
    return cnt;
}

// the k-th smallest eigenvalue (k = 1..n) by bisection of the Sturm count
double kth_eigenvalue(const double* a, const double* b, int n, int k, double lo, double hi)
{
    for (int it = 0; it < 2000; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break;   // the interval is down to adjacent doubles
        if (sturm_below(a, b, n, mid) >= k) hi = mid;
        else lo = mid;
    }
    return 0.5 * (lo + hi);
}

}  // namespace

extern "C" {

int gbn_cheb_interval(const double* a, const double* b, int32_t nrecurs, double* ac, double* bc)
{
    if (!a || !b || !ac || !bc || nrecurs < 1) return GBN_ERR_ARG;
    const int n = nrecurs;
    double lo = a[0], hi = a[0];
    for (int i = 0; i < n; ++i) {
        if (!isfinite(a[i]) || (i + 1 < n && !isfinite(b[i]))) return GBN_ERR_NUMERIC;
        const double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i + 1 < n ? fabs(b[i]) : 0.0);
        lo = std::min(lo, a[i] - r);
        hi = std::max(hi, a[i] + r);
    }
    const double pad = 1e-12 * std::max(1.0, std::max(fabs(lo), fabs(hi)));
    lo -= pad;
    hi += pad;
    const double emin = kth_eigenvalue(a, b, n, 1, lo, hi);
    const double emax = kth_eigenvalue(a, b, n, n, lo, hi);
    *ac = (emax + emin) / 2.0;
    *bc = 1.2 * (emax - emin) / 4.0;
    return GBN_OK;
}

int gbn_cheb_coef(double dt, double ac, double bc, int32_t npol, double* c)
{
    if (!c || npol < 1 || !isfinite(dt) || !isfinite(ac) || !isfinite(bc) || bc < 0.0) return GBN_ERR_ARG;
    const double x = 2.0 * bc * fabs(dt);
    std::vector<double> J((size_t)npol, 0.0);
    if (x < 1e-300) {
        J[0] = 1.0;
    } else {
        const double m = std::max((double)npol, x);
        int top = (int)(m + 10.0 * sqrt(m) + 40.0);
        top += top & 1;   // even start, so that the normalisation sum ends on J_0
        std::vector<double> w((size_t)top + 2, 0.0);
        w[(size_t)top + 1] = 0.0;
        w[(size_t)top] = 1e-30;
        for (int k = top; k >= 1; --k) {
            w[(size_t)k - 1] = (2.0 * k / x) * w[(size_t)k] - w[(size_t)k + 1];
            if (fabs(w[(size_t)k - 1]) > 1e250) {   // rescale to stay in range
                for (int i = k - 1; i <= top + 1; ++i) w[(size_t)i] *= 1e-250;
            }
        }
        double norm = w[0];
        for (int k = 2; k <= top; k += 2) norm += 2.0 * w[(size_t)k];
        for (int k = 0; k < npol; ++k) J[(size_t)k] = w[(size_t)k] / norm;
    }
    if (dt < 0.0)   // J_n(-x) = (-1)^n J_n(x)
        for (int k = 1; k < npol; k += 2) J[(size_t)k] = -J[(size_t)k];
    const double ph = -ac * dt;   // exp(-i ac dT)
    const double er = cos(ph), ei = sin(ph);
    for (int k = 0; k < npol; ++k) {
        // (-i)^k: 1, -i, -1, i
        double ur = 0.0, ui = 0.0;
        switch (k & 3) {
            case 0: ur = 1.0; break;
            case 1: ui = -1.0; break;
            case 2: ur = -1.0; break;
            default: ui = 1.0; break;
        }
        const double s = (k == 0 ? 1.0 : 1.4142135623730951) * J[(size_t)k];
        c[2 * k] = s * (ur * er - ui * ei);
        c[2 * k + 1] = s * (ur * ei + ui * er);
    }
    return GBN_OK;
}

// Spread and diffusivity of the time evolution (no counterpart in the reference, which writes only the
// norms, kubo.F90:376-385).  The norm |ZUPsi_r|^2 = <psi_r| [X, U(t)]^+ [X, U(t)] |psi_r> of KuboTEvol is
// the spread <(X(t) - X(0))^2> of the start vector psi_r; for random-phase vectors it estimates the
// trace over the states per atom, so the mean over the vectors is the mean-square displacement
// MSD(t) = <Delta X^2>(t) [Ang^2].  The diffusivity is written both ways: D(t) = MSD(t) / t and
// D'(t) = d MSD / dt, the latter by central differences between write steps (MSD(0) = 0 at the start,
// one-sided at the last step).  Sums in FP64, vectors in order.
int gbn_kubo_msd(int32_t nrhs, int32_t nw, int32_t nwr, double dt_fs, const double* norms, double* t_fs,
                 double* msd, double* d_ratio, double* d_slope)
{
    if (nrhs < 1 || nw < 1 || nwr < 1 || !(dt_fs > 0.0) || !norms || !t_fs || !msd) return GBN_ERR_ARG;
    for (int w = 0; w < nw; ++w) {
        double s = 0.0;
        for (int r = 0; r < nrhs; ++r) s += norms[(size_t)r * nw + w];
        msd[w] = s / nrhs;
        t_fs[w] = (double)(w + 1) * nwr * dt_fs;
        if (d_ratio) d_ratio[w] = msd[w] / t_fs[w];
    }
    if (d_slope) {
        for (int w = 0; w < nw; ++w) {
            const double t0 = w > 0 ? t_fs[w - 1] : 0.0, m0 = w > 0 ? msd[w - 1] : 0.0;
            if (w + 1 < nw) d_slope[w] = (msd[w + 1] - m0) / (t_fs[w + 1] - t0);
            else d_slope[w] = (msd[w] - m0) / (t_fs[w] - t0);
        }
    }
    return GBN_OK;
}

}  // extern "C"
