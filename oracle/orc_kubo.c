/*
 * Oracle (test infrastructure only): the recursion solver of the reference --
 * start vector, Lanczos recursion, continued-fraction DOS, spectral interval,
 * Chebyshev coefficients and Chebyshev time evolution.  Complex numbers are
 * interleaved (re, im) doubles; complex products and quotients are written out
 * in the form GNU Fortran evaluates them (no NaN recovery; Smith's division).
 */
#include "oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846264338327950288

typedef struct { double re, im; } cpx;

static inline cpx cmul(cpx a, cpx b) { return (cpx){a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
static inline cpx csub(cpx a, cpx b) { return (cpx){a.re - b.re, a.im - b.im}; }
static inline cpx cadd(cpx a, cpx b) { return (cpx){a.re + b.re, a.im + b.im}; }
static inline cpx rmul(double r, cpx a) { return (cpx){r * a.re, r * a.im}; }
static inline cpx rdiv(cpx a, double r) { return (cpx){a.re / r, a.im / r}; }
/* (a)/(b) by Smith's method */
static inline cpx cdiv(cpx a, cpx b)
{
    if (fabs(b.re) >= fabs(b.im)) {
        const double r = b.im / b.re, den = b.re + b.im * r;
        return (cpx){(a.re + a.im * r) / den, (a.im - a.re * r) / den};
    }
    const double r = b.re / b.im, den = b.re * r + b.im;
    return (cpx){(a.re * r + a.im) / den, (a.im * r - a.re) / den};
}
static inline cpx ld(const double* p, size_t i) { return (cpx){p[2 * i], p[2 * i + 1]}; }
static inline void st(double* p, size_t i, cpx v) { p[2 * i] = v.re; p[2 * i + 1] = v.im; }

/* KuboInitWF, kubo.F90:24-85: psi_i = exp(2 pi i r_i)/sqrt(N) */
void orc_init_wf(int64_t n, int32_t seed, double* psi)
{
    orc_rng r;
    orc_rng_put(&r, seed);
    const double twopi = 2.0 * ORC_PI, sn = sqrt((double)n);
    for (int64_t i = 0; i < n; ++i) {
        const double y = twopi * orc_rng_r8(&r);
        psi[2 * i] = cos(y) / sn;
        psi[2 * i + 1] = sin(y) / sn;
    }
}

/* H psi at row i: H0(i) psi(i) - sum_j hopp(j,i) psi(NList(j,i)) (kubosubs.F90:69-72) */
static inline cpx hrow(int64_t i, int32_t maxNeigh, const int32_t* Nneigh, const int32_t* NList,
                       const double* hopp, const double* H0, const double* x)
{
    cpx c = rmul(H0[i], ld(x, i));
    const size_t base = (size_t)i * maxNeigh;
    for (int32_t j = 0; j < Nneigh[i]; ++j)
        c = csub(c, cmul(ld(hopp, base + j), ld(x, (size_t)NList[base + j] - 1)));
    return c;
}

/* KuboRecursion, kubosubs.F90:26-138 (three passes per step, as the reference). */
void orc_recursion(int64_t n, int32_t maxNeigh, const int32_t* Nneigh, const int32_t* NList,
                   const double* hopp, const double* H0, const double* psi, int32_t nrecurs,
                   double* a, double* b, int32_t nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    double* Psin = (double*)malloc(sizeof(double) * 2 * n);
    double* Psinm1 = (double*)malloc(sizeof(double) * 2 * n);
    double* H = (double*)malloc(sizeof(double) * 2 * n);
    double sr = 0.0, si = 0.0;
#pragma omp parallel for reduction(+ : sr, si) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const cpx p = ld(psi, i);
        st(Psinm1, i, p);
        const cpx c = hrow(i, maxNeigh, Nneigh, NList, hopp, H0, psi);
        sr += c.re * p.re + c.im * p.im; /* c * conjg(p) */
        si += c.im * p.re - c.re * p.im;
        st(H, i, c);
    }
    a[0] = sr;
    sr = 0.0; si = 0.0;
#pragma omp parallel for reduction(+ : sr, si) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const cpx c = csub(ld(H, i), rmul(a[0], ld(Psinm1, i)));
        st(Psin, i, c);
        sr += c.re * c.re + c.im * c.im;
    }
    b[0] = sqrt(fabs(sr));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) st(Psin, i, rdiv(ld(Psin, i), b[0]));
    for (int32_t it = 1; it < nrecurs; ++it) {
        sr = 0.0; si = 0.0;
#pragma omp parallel for reduction(+ : sr, si) schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            const cpx p = ld(Psin, i);
            const cpx c = hrow(i, maxNeigh, Nneigh, NList, hopp, H0, Psin);
            sr += c.re * p.re + c.im * p.im;
            si += c.im * p.re - c.re * p.im;
            st(H, i, c);
        }
        a[it] = sr;
        sr = 0.0;
#pragma omp parallel for reduction(+ : sr) schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            const cpx c = csub(csub(ld(H, i), rmul(a[it], ld(Psin, i))), rmul(b[it - 1], ld(Psinm1, i)));
            sr += c.re * c.re + c.im * c.im;
            st(H, i, c);
        }
        b[it] = sqrt(fabs(sr));
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            st(Psinm1, i, ld(Psin, i));
            st(Psin, i, rdiv(ld(H, i), b[it]));
        }
    }
    free(Psin); free(Psinm1); free(H);
}

/* KuboFrac, kubosubs.F90:222-288 */
void orc_frac(const double* a, const double* b, int32_t nrecurs, double norm, double eps, int32_t nEn,
              double Emin, double Emax, double* energy, double* dos)
{
    const double dE = (Emax - Emin) / nEn;
    const double ainf = a[nrecurs - 1], binf = b[nrecurs - 1];
    for (int32_t iE = 0; iE <= nEn; ++iE) {
        const double E = Emin + (double)iE * dE;
        const cpx z = {E, eps};
        const cpx w = {z.re - ainf, z.im};
        const cpx w2 = cmul(w, w);
        const double fb = 4.0 * (binf * binf), tb = 2.0 * (binf * binf);
        const double complex s = csqrt(CMPLX(w2.re - fb, w2.im));
        cpx g = rdiv((cpx){w.re - creal(s), w.im - cimag(s)}, tb);
        if (g.im >= 0.0) g = rdiv((cpx){w.re + creal(s), w.im + cimag(s)}, tb);
        for (int32_t iR = nrecurs - 2; iR >= 0; --iR) {
            const cpx den = csub((cpx){z.re - a[iR], z.im}, rmul(b[iR] * b[iR], g));
            g = cdiv((cpx){1.0, 0.0}, den);
        }
        energy[iE] = E;
        dos[iE] = (-g.im / ORC_PI) * norm;
    }
}

/* TQL2, kubosubs.F90:725-868 (Wilkinson & Reinsch, Handbook vol. 2): QL with
 * implicit shifts on a symmetric tridiagonal matrix; d diagonal, e sub-diagonal
 * in e[1..n-1] on entry (e[0] unused), z (n x n, column-major) accumulates. */
static int tql2(int n, double* d, double* e, double* z, int want_vectors)
{
    double eps = 1.0;
    do { eps = eps / 2.0; } while (1.0 + eps > 1.0);
    if (n == 1) return 0;
    for (int i = 1; i < n; ++i) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    double f = 0.0, bnd = 0.0;
    for (int l = 0; l < n; ++l) {
        int j = 0;
        double h = eps * (fabs(d[l]) + fabs(e[l]));
        if (bnd < h) bnd = h;
        int m;
        for (m = l; m < n; ++m)
            if (fabs(e[m]) <= bnd) break;
        if (m == n) m = n - 1;
        if (m != l) {
            do {
                if (j == 30) return l + 1;
                ++j;
                double g = d[l];
                double p = (d[l + 1] - g) / (2.0 * e[l]);
                double r = sqrt(p * p + 1.0);
                d[l] = e[l] / (p + copysign(r, p));
                h = g - d[l];
                for (int i = l + 1; i < n; ++i) d[i] = d[i] - h;
                f = f + h;
                p = d[m];
                double c = 1.0, s = 0.0;
                for (int i = m - 1; i >= l; --i) {
                    g = c * e[i];
                    h = c * p;
                    if (fabs(p) >= fabs(e[i])) {
                        c = e[i] / p;
                        r = sqrt(c * c + 1.0);
                        e[i + 1] = s * p * r;
                        s = c / r;
                        c = 1.0 / r;
                    } else {
                        c = p / e[i];
                        r = sqrt(c * c + 1.0);
                        e[i + 1] = s * e[i] * r;
                        s = 1.0 / r;
                        c = c * s;
                    }
                    p = c * d[i] - s * g;
                    d[i + 1] = h + s * (c * g + s * d[i]);
                    if (want_vectors)
                        for (int k = 0; k < n; ++k) {
                            h = z[(size_t)(i + 1) * n + k];
                            z[(size_t)(i + 1) * n + k] = s * z[(size_t)i * n + k] + c * h;
                            z[(size_t)i * n + k] = z[(size_t)i * n + k] * c - s * h;
                        }
                }
                e[l] = s * p;
                d[l] = c * p;
            } while (fabs(e[l]) > bnd);
        }
        d[l] = d[l] + f;
    }
    for (int l = 1; l < n; ++l) { /* ascending order */
        int i = l - 1, k = i;
        double p = d[i];
        for (int jj = l; jj < n; ++jj)
            if (!(d[jj] >= p)) { k = jj; p = d[jj]; }
        if (k != i) {
            d[k] = d[i];
            d[i] = p;
            if (want_vectors)
                for (int jj = 0; jj < n; ++jj) {
                    const double t = z[(size_t)i * n + jj];
                    z[(size_t)i * n + jj] = z[(size_t)k * n + jj];
                    z[(size_t)k * n + jj] = t;
                }
        }
    }
    return 0;
}

/* KuboInterval, kubosubs.F90:290-350.  The reference calls LAPACK DSTERF for the
 * eigenvalues of the Lanczos matrix; the same eigenvalues are taken here from the
 * QL iteration above (values only). */
int orc_interval(const double* a, const double* b, int32_t nrecurs, double* ac, double* bc)
{
    double* d = (double*)malloc(sizeof(double) * nrecurs);
    double* e = (double*)malloc(sizeof(double) * nrecurs);
    memcpy(d, a, sizeof(double) * nrecurs);
    e[0] = 0.0;
    for (int i = 1; i < nrecurs; ++i) e[i] = b[i - 1];
    const int info = tql2(nrecurs, d, e, NULL, 0);
    if (info == 0) {
        double emin = d[0], emax = d[0];
        for (int i = 1; i < nrecurs; ++i) { emin = fmin(emin, d[i]); emax = fmax(emax, d[i]); }
        *ac = (emax + emin) / 2.0;
        *bc = 1.2 * (emax - emin) / 4.0;
    }
    free(d); free(e);
    return info;
}

/* KuboCn, kubosubs.F90:352-433 */
int orc_cheb_coef(double dT, double ac, double bc, int32_t nPol, double* c)
{
    double* d = (double*)malloc(sizeof(double) * nPol);
    double* e = (double*)malloc(sizeof(double) * nPol);
    double* z = (double*)calloc((size_t)nPol * nPol, sizeof(double));
    for (int i = 0; i < nPol; ++i) { d[i] = ac; e[i] = bc; z[(size_t)i * nPol + i] = 1.0; }
    if (nPol > 1) e[1] = sqrt(2.0) * bc;
    const int info = tql2(nPol, d, e, z, 1);
    if (info == 0)
        for (int i = 0; i < nPol; ++i) {
            cpx sc = {0.0, 0.0};
            for (int j = 0; j < nPol; ++j) {
                const double w = z[(size_t)j * nPol + 0] * z[(size_t)j * nPol + i];
                const double ph = d[j] * dT;
                sc = cadd(sc, rmul(w, (cpx){cos(ph), -sin(ph)}));
            }
            c[2 * i] = sc.re;
            c[2 * i + 1] = sc.im;
        }
    free(d); free(e); free(z);
    return info;
}

/* KuboChebyshevEvolve, kubosubs.F90:557-619: Z <- sum_n c_n T_n Z */
void orc_cheb_evolve(int64_t n, int32_t maxNeigh, const int32_t* Nneigh, const int32_t* NList,
                     const double* hopp, const double* H0, const double* c, int32_t nPol, double ac,
                     double bc, double* Z)
{
    double* Psin = (double*)malloc(sizeof(double) * 2 * n);
    double* Psinm1 = (double*)malloc(sizeof(double) * 2 * n);
    const cpx c0 = {c[0], c[1]};
    for (int64_t i = 0; i < n; ++i) st(Psinm1, i, rmul(sqrt(2.0), ld(Z, i)));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        cpx cn = rmul(H0[i] - ac, ld(Psinm1, i));
        const size_t base = (size_t)i * maxNeigh;
        for (int32_t j = 0; j < Nneigh[i]; ++j)
            cn = csub(cn, cmul(ld(hopp, base + j), ld(Psinm1, (size_t)NList[base + j] - 1)));
        st(Psin, i, rdiv(cn, 2.0 * bc));
        st(Z, i, cmul(ld(Z, i), c0));
    }
    for (int32_t ip = 1; ip < nPol; ++ip) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            cpx cn = rmul(H0[i] - ac, ld(Psin, i));
            const size_t base = (size_t)i * maxNeigh;
            for (int32_t j = 0; j < Nneigh[i]; ++j)
                cn = csub(cn, cmul(ld(hopp, base + j), ld(Psin, (size_t)NList[base + j] - 1)));
            st(Psinm1, i, rdiv(csub(cn, rmul(bc, ld(Psinm1, i))), bc));
        }
        const cpx ci = {c[2 * ip], c[2 * ip + 1]};
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            st(Z, i, cadd(ld(Z, i), cmul(ci, ld(Psin, i))));
            const cpx t = ld(Psin, i);
            st(Psin, i, ld(Psinm1, i));
            st(Psinm1, i, t);
        }
    }
    free(Psin); free(Psinm1);
}

/* KuboEvol, kubosubs.F90:438-553: psi <- U psi; zupsi <- U zupsi + [U, X] psi */
void orc_evol(int64_t n, int32_t maxNeigh, const int32_t* Nneigh, const int32_t* NList,
              const double* NeighD, const double* hopp, const double* H0, const double* c, int32_t nPol,
              double ac, double bc, int32_t dir, double* psi, double* zupsi)
{
    orc_cheb_evolve(n, maxNeigh, Nneigh, NList, hopp, H0, c, nPol, ac, bc, zupsi);
    double* Psin = (double*)malloc(sizeof(double) * 2 * n);
    double* Psinm1 = (double*)malloc(sizeof(double) * 2 * n);
    double* X = (double*)malloc(sizeof(double) * 2 * n);
    double* Xm1 = (double*)malloc(sizeof(double) * 2 * n);
    const int k = (dir == 2) ? 1 : 0;
    const cpx c0 = {c[0], c[1]};
    for (int64_t i = 0; i < n; ++i) {
        st(Psinm1, i, rmul(sqrt(2.0), ld(psi, i)));
        st(Xm1, i, (cpx){0.0, 0.0});
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        cpx cn = rmul(H0[i] - ac, ld(Psinm1, i));
        cpx cn2 = {0.0, 0.0};
        const size_t base = (size_t)i * maxNeigh;
        for (int32_t j = 0; j < Nneigh[i]; ++j) {
            const cpx h = ld(hopp, base + j);
            const cpx xj = ld(Psinm1, (size_t)NList[base + j] - 1);
            cn = csub(cn, cmul(h, xj));
            cn2 = csub(cn2, cmul(rmul(NeighD[3 * (base + j) + k], h), xj));
        }
        st(Psin, i, rdiv(cn, 2.0 * bc));
        st(X, i, rdiv(cn2, 2.0 * bc));
        st(psi, i, cmul(c0, ld(psi, i)));
    }
    for (int32_t ip = 1; ip < nPol; ++ip) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            cpx cn = rmul(H0[i] - ac, ld(Psin, i));
            cpx cn2 = rmul(H0[i] - ac, ld(X, i));
            const size_t base = (size_t)i * maxNeigh;
            for (int32_t j = 0; j < Nneigh[i]; ++j) {
                const cpx h = ld(hopp, base + j);
                const size_t col = (size_t)NList[base + j] - 1;
                const cpx pj = ld(Psin, col);
                cn = csub(cn, cmul(h, pj));
                cn2 = csub(csub(cn2, cmul(rmul(NeighD[3 * (base + j) + k], h), pj)), cmul(h, ld(X, col)));
            }
            st(Psinm1, i, rdiv(csub(cn, rmul(bc, ld(Psinm1, i))), bc));
            st(Xm1, i, rdiv(csub(cn2, rmul(bc, ld(Xm1, i))), bc));
        }
        const cpx ci = {c[2 * ip], c[2 * ip + 1]};
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            st(psi, i, cadd(ld(psi, i), cmul(ci, ld(Psin, i))));
            st(zupsi, i, cadd(ld(zupsi, i), cmul(ci, ld(X, i))));
            const cpx t = ld(Psin, i), t2 = ld(X, i);
            st(Psin, i, ld(Psinm1, i));
            st(X, i, ld(Xm1, i));
            st(Psinm1, i, t);
            st(Xm1, i, t2);
        }
    }
    free(Psin); free(Psinm1); free(X); free(Xm1);
}
