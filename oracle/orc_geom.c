/*
 * Oracle (test infrastructure only): random numbers, cell and atom geometry,
 * neighbour search.  See oracle.h for the rules that apply to this directory.
 * Compiled with -O2 -ffp-contract=off and without -march, like the reference's
 * GNU build (lanczosKuboCode/make.sys.example: -O3, no FMA contraction on
 * x86-64), so that every expression below rounds as the Fortran one does.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.14159265358979323846264338327950288

/* ======================================================================
 * libgfortran intrinsic RNG (GNU Fortran >= 8), as used by the reference
 * through random_seed(PUT=...) / random_number(r) with r real(8):
 *   state: xoshiro256** (Blackman & Vigna, 2018), 4 x uint64;
 *   PUT:   the 8 default-integer seed words are copied in reverse order into
 *          the 32-byte state and XORed with a fixed 4-word key (the library's
 *          scrambling of user seeds); the calling thread starts from it;
 *   real(8) draw: top 53 bits of the 64-bit output times 2^-53.
 * Third-party dependency of the reference (libgfortran, GCC 11.4 / 12.2 per
 * .github/workflows/regression.yml and lanczosKuboCode/README.md); its call
 * sites are kubo.F90:46-64, random.F90:31-52, ham.F90:1245.
 * ====================================================================== */
static const uint64_t kGfortranSeedKey[4] = {
    0xbd0c5b6e50c2df49ULL, 0xd46061cd46e1df38ULL,
    0xbb4f4d4ed6103544ULL, 0x114a583d0756ad39ULL};

static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

void orc_rng_put(orc_rng* r, int32_t seed_value)
{
    uint32_t words[8];
    for (int i = 0; i < 8; ++i) words[i] = (uint32_t)seed_value; /* reversed copy of equal words */
    memcpy(r->s, words, sizeof(words));
    for (int i = 0; i < 4; ++i) r->s[i] ^= kGfortranSeedKey[i];
}

static inline uint64_t xoshiro_next(orc_rng* r)
{
    const uint64_t result = rotl64(r->s[1] * 5, 7) * 9;
    const uint64_t t = r->s[1] << 17;
    r->s[2] ^= r->s[0];
    r->s[3] ^= r->s[1];
    r->s[1] ^= r->s[2];
    r->s[0] ^= r->s[3];
    r->s[2] ^= t;
    r->s[3] = rotl64(r->s[3], 45);
    return result;
}

double orc_rng_r8(orc_rng* r)
{
    uint64_t v = xoshiro_next(r);
    v &= ~(uint64_t)0 << 11;
    return (double)v * 0x1p-64;
}

void orc_rng_fill(int32_t seed_value, int64_t n, double* out)
{
    orc_rng r;
    orc_rng_put(&r, seed_value);
    for (int64_t i = 0; i < n; ++i) out[i] = orc_rng_r8(&r);
}

/* ====================================================================== geometry */

static int gcd_ref(int i1, int i2) /* atoms.F90:2063-2092 */
{
    int a = abs(i1), b = abs(i2), g;
    if (a > b) { g = a; a = b; b = g; }
    if (a == 0) return b;
    for (;;) {
        g = a % b;
        if (g == 0) break;
        a = b;
        b = g;
    }
    return b;
}

/* Swap of the moire indices and twist of TwistedBilayerBasedOnMoireCell:
 * cell.F90:207-240 and atoms.F90:330-350. */
static void moire_indices(const int32_t m_in[4], int n_out[4], double* phi)
{
    int n[4] = {m_in[0], m_in[1], m_in[2], m_in[3]};
    double g = (double)(n[0] * n[0] + n[1] * n[1] + n[0] * n[1]);
    double delta = sqrt((double)(float)(n[2] * n[2] + n[3] * n[3] + n[2] * n[3]) / g);
    *phi = acos((2.0 * n[0] * n[2] + 2.0 * n[1] * n[3] + (double)(n[0] * n[3]) + (double)(n[1] * n[2]))
                / (2.0 * delta * g));
    if (!(delta < 1.0)) {
        int t = n[0]; n[0] = n[2]; n[2] = t;
        t = n[1]; n[1] = n[3]; n[3] = t;
    }
    memcpy(n_out, n, sizeof(n));
}

int64_t orc_geom_natoms(const orc_geom_params* p)
{
    if (p->kind == ORC_GRAPHENE) {
        int64_t n = (int64_t)p->cell_size * p->super_cell;
        return 2 * n * n;
    }
    int n[4];
    double phi;
    moire_indices(p->m, n, &phi);
    int64_t s = p->super_cell;
    int64_t a0 = n[0] * s, a1 = n[1] * s, a2 = n[2] * s, a3 = n[3] * s;
    return 2 * (a0 * a0 + a0 * a1 + a1 * a1) + 2 * (a2 * a2 + a2 * a3 + a3 * a3);
}

/* AtomsConstruct, atoms.F90:1506-1607: fractional coordinates X[k][3]. */
static void atoms_construct(int mm0, int mm1, double angle, double d, double yshift, double* X)
{
    const int64_t ncell = (int64_t)mm0 * mm0 + (int64_t)mm0 * mm1 + (int64_t)mm1 * mm1;
    const double a = angle * ORC_PI / 180.0;
    const double u[2][2] = {{cos(a), sin(a)}, {cos(a + ORC_PI / 3.0), sin(a + ORC_PI / 3.0)}}; /* u[k][r] */
    const double m[2][2] = {{(double)mm0, (double)mm1}, {(double)(-mm1), (double)(mm0 + mm1)}}; /* m[c][k] */
    double R[2][2]; /* R[r][c] = sum_k u(r,k) m(k,c) */
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 2; ++c) R[r][c] = u[0][r] * m[c][0] + u[1][r] * m[c][1];
    const double bss[2][2] = {{1.0 / 3.0, 1.0 / 3.0}, {2.0 / 3.0, 2.0 / 3.0}}; /* bss[j][k] */
    double basis[2][2];                                                       /* basis[j][r] */
    for (int j = 0; j < 2; ++j)
        for (int r = 0; r < 2; ++r) basis[j][r] = u[0][r] * bss[j][0] + u[1][r] * bss[j][1];
    int64_t n1 = gcd_ref(mm0, mm1);
    int64_t n2 = ncell / n1;
    if (n2 > n1) { int64_t t = n1; n1 = n2; n2 = t; }
    for (int64_t i2 = 0; i2 < n2; ++i2)
        for (int64_t i1 = 0; i1 < n1; ++i1)
            for (int j = 0; j < 2; ++j) {
                double* x = X + 3 * (2 * (n1 * i2 + i1) + j);
                x[0] = (double)i1 * u[0][0] + (double)i2 * u[1][0] + basis[j][0];
                x[1] = (double)i1 * u[0][1] + (double)i2 * u[1][1] + basis[j][1];
                x[2] = 0.0;
            }
    const double det = R[1][1] * R[0][0] - R[0][1] * R[1][0];
    for (int64_t k = 0; k < 2 * ncell; ++k) {
        double* x = X + 3 * k;
        double f1, f2;
        if (fabs(R[0][0]) > 1.0e-6 * fabs(R[1][0])) {
            f2 = R[0][0] * (x[1] - x[0] * R[1][0] / R[0][0]) / det;
            f1 = (x[0] - f2 * R[0][1]) / R[0][0];
        } else {
            const double dc = R[0][0] * R[1][1] - R[0][1] * R[1][0];
            f1 = (x[0] * R[1][1] - x[1] * R[0][1]) / dc;
            f2 = (x[1] * R[0][0] - x[0] * R[1][0]) / dc;
        }
        x[0] = fmod(f1, 1.0) + yshift;
        x[1] = fmod(f2, 1.0) + yshift;
        x[2] = 0.5 + d;
        if (x[0] < 0.0) x[0] = fmod(x[0] + 1.0, 1.0);
        if (x[1] < 0.0) x[1] = fmod(x[1] + 1.0, 1.0);
        if (x[0] > 1.0) x[0] = fmod(x[0] - 1.0, 1.0);
        if (x[1] > 1.0) x[1] = fmod(x[1] - 1.0, 1.0);
    }
}

/* AtomsSetCart, atoms.F90:1768-1794 */
static void set_cart(int64_t n, const double* uc, double* Rat)
{
    for (int64_t i = 0; i < n; ++i) {
        double* r = Rat + 3 * i;
        const double f1 = r[0], f2 = r[1], f3 = r[2];
        for (int k = 0; k < 3; ++k) r[k] = f1 * uc[k] + f2 * uc[3 + k] + f3 * uc[6 + k];
    }
}

/* AtomsSetFrac, atoms.F90:1796-1830 */
static void set_frac(int64_t n, const double* uc, double* Rat)
{
    const double u11 = uc[0], u21 = uc[1], u12 = uc[3], u22 = uc[4], u33 = uc[8];
    for (int64_t i = 0; i < n; ++i) {
        double* r = Rat + 3 * i;
        if (u11 != 0.0) {
            r[1] = u11 * (r[1] - r[0] * u21 / u11) / (u22 * u11 - u12 * u21);
            r[0] = (r[0] - r[1] * u12) / u11;
        } else {
            const double x = r[0], y = r[1], dc = u11 * u22 - u12 * u21;
            r[0] = (u22 * x - u12 * y) / dc;
            r[1] = (u11 * y - u21 * x) / dc;
        }
        r[2] = r[2] / u33;
    }
}

void orc_geom_roundtrip(int64_t n, const double* ucell, double* Rat)
{
    set_frac(n, ucell, Rat);
    set_cart(n, ucell, Rat);
}

double orc_cell_area(const double* u) /* cell.F90:396-403 */
{
    const double v1 = u[1] * u[5] - u[2] * u[4];
    const double v2 = u[2] * u[3] - u[0] * u[5];
    const double v3 = u[0] * u[4] - u[1] * u[3];
    return sqrt(v1 * v1 + v2 * v2 + v3 * v3);
}

int orc_geom_build(const orc_geom_params* p, double* ucell, double* Rat, int32_t* species,
                   int32_t* layer, double* twist_rad)
{
    const double aG = p->aG, h = p->height;
    memset(ucell, 0, 9 * sizeof(double));
    if (p->kind == ORC_GRAPHENE) {
        /* cell.F90:108-140; atoms.F90:168-208 */
        const int n = p->cell_size * p->super_cell;
        const double dn = (double)n;
        ucell[0] = aG * dn;
        ucell[1] = 0.0 * dn;
        ucell[3] = aG / 2.0 * dn;
        ucell[4] = sqrt(3.0) * aG / 2.0 * dn;
        ucell[8] = h;
        atoms_construct(n, 0, 0.0, 0.0, 0.0, Rat);
        const int64_t nat = 2 * (int64_t)n * n;
        for (int64_t i = 0; i < nat; ++i) {
            species[i] = (int32_t)(((i + 2) % 2) + 1); /* mod(i+1,2)+1 with 1-based i */
            layer[i] = 1;
        }
        set_cart(nat, ucell, Rat);
        *twist_rad = 0.0;
        return 0;
    }
    if (p->kind != ORC_TBG_MOIRE_CELL) return -1;
    /* cell.F90:207-240 */
    int n[4];
    double phi;
    moire_indices(p->m, n, &phi);
    const double uc[2][2] = {{aG, 0.0}, {aG / 2.0, sqrt(3.0) * aG / 2.0}}; /* uc[k][r] */
    const int m1[2][2] = {{n[0], n[1]}, {-n[1], n[0] + n[1]}};             /* m1[c][k] */
    for (int c = 0; c < 2; ++c)
        for (int r = 0; r < 2; ++r)
            ucell[3 * c + r] = (uc[0][r] * (double)m1[c][0] + uc[1][r] * (double)m1[c][1]) * (double)p->super_cell;
    ucell[8] = h;
    /* atoms.F90:330-380 and :1391-1397 */
    const int s = p->super_cell;
    int nn[4] = {n[0] * s, n[1] * s, n[2] * s, n[3] * s};
    const double g = p->d_interlayer / (2.0 * h);
    const int64_t natc = 2 * ((int64_t)nn[0] * nn[0] + (int64_t)nn[0] * nn[1] + (int64_t)nn[1] * nn[1]);
    const int64_t natb = 2 * ((int64_t)nn[2] * nn[2] + (int64_t)nn[2] * nn[3] + (int64_t)nn[3] * nn[3]);
    /* atoms.F90:352-366: the second layer's offset, from the indices after the swap and the super cell */
    double yshift = 0.0;
    if (p->add_shift == 1 || p->add_shift == 2) {
        const double frac = p->shift_factor /
                            (sqrt(3.0) * aG * sqrt((double)(nn[0] * nn[0] + nn[0] * nn[1] + nn[1] * nn[1])));
        yshift = (p->add_shift == 1) ? (aG / 3.0) / ((double)nn[0] * aG) + frac
                                     : (aG / 3.0 / 2.0) / ((double)nn[0] * aG) + frac;
    }
    atoms_construct(nn[0], nn[1], 0.0, g, 0.0, Rat);
    atoms_construct(nn[2], nn[3], -phi * 180.0 / ORC_PI, -g, yshift, Rat + 3 * natc);
    const int64_t nat = natc + natb;
    for (int64_t i = 0; i < nat; ++i) species[i] = (int32_t)(((i + 2) % 2) + 1);
    set_cart(nat, ucell, Rat);
    for (int64_t i = 0; i < nat; ++i) layer[i] = (Rat[3 * i + 2] < 20.0) ? 1 : 2;
    *twist_rad = phi;
    return 0;
}

/* ====================================================================== neighbours */

struct orc_nbr {
    int64_t n;
    int32_t max_neigh;
    int32_t* nneigh;
    int32_t* nlist;   /* [n][max] */
    double* neighd;   /* [n][max][3] */
    int32_t* ncell;   /* [n][max][3] */
};

/* NeighSearchLayered, neigh.F90:117-316, with periodicZ = .false. (A3 = 0). */
orc_nbr* orc_neigh_search(int64_t natoms, const double* Rat, const double* ucell,
                          double cut2intra, double cut2inter, int32_t second_layer)
{
    const double dzIntra = 1.5, dzInter = 4.5, dzSecond = 7.5;
    const double A1[2] = {ucell[0], ucell[1]}, A2[2] = {ucell[3], ucell[4]};
    const double det = A1[0] * A2[1] - A1[1] * A2[0];
    if (fabs(det) < 2.2250738585072014e-308) return NULL;
    const double rmax = sqrt(fmax(cut2intra, cut2inter));
    const double dzmax = second_layer ? dzSecond : dzInter;
    double s1min = HUGE_VAL, s1max = -HUGE_VAL, s2min = HUGE_VAL, s2max = -HUGE_VAL;
    double xmin = HUGE_VAL, xmax = -HUGE_VAL, ymin = HUGE_VAL, ymax = -HUGE_VAL, zmin = HUGE_VAL, zmax = -HUGE_VAL;
    for (int64_t i = 0; i < natoms; ++i) {
        const double x = Rat[3 * i], y = Rat[3 * i + 1], z = Rat[3 * i + 2];
        const double s1 = (x * A2[1] - y * A2[0]) / det;
        const double s2 = (-(x * A1[1]) + y * A1[0]) / det;
        s1min = fmin(s1min, s1); s1max = fmax(s1max, s1);
        s2min = fmin(s2min, s2); s2max = fmax(s2max, s2);
        xmin = fmin(xmin, x); xmax = fmax(xmax, x);
        ymin = fmin(ymin, y); ymax = fmax(ymax, y);
        zmin = fmin(zmin, z); zmax = fmax(zmax, z);
    }
    const double h1 = fabs(det) / sqrt(A2[0] * A2[0] + A2[1] * A2[1]);
    const double h2 = fabs(det) / sqrt(A1[0] * A1[0] + A1[1] * A1[1]);
    const int n1 = (int)ceil(rmax / h1 + (s1max - s1min));
    const int n2 = (int)ceil(rmax / h2 + (s2max - s2min));
    const double xlo = xmin - rmax, xhi = xmax + rmax;
    const double ylo = ymin - rmax, yhi = ymax + rmax;
    const double zlo = zmin - dzmax, zhi = zmax + dzmax;

    /* candidates in the order u1, u2, m (u3 = 0) */
    int64_t ncand = 0, cap = natoms + 16;
    int32_t* cidx = (int32_t*)malloc(sizeof(int32_t) * cap);
    int32_t* cu = (int32_t*)malloc(sizeof(int32_t) * 2 * cap);
    for (int u1 = -n1; u1 <= n1; ++u1)
        for (int u2 = -n2; u2 <= n2; ++u2) {
            const double tx = (double)u1 * A1[0] + (double)u2 * A2[0];
            const double ty = (double)u1 * A1[1] + (double)u2 * A2[1];
            for (int64_t m = 0; m < natoms; ++m) {
                const double px = Rat[3 * m] + tx;
                if (px < xlo || px > xhi) continue;
                const double py = Rat[3 * m + 1] + ty;
                if (py < ylo || py > yhi) continue;
                const double pz = Rat[3 * m + 2] + 0.0;
                if (pz < zlo || pz > zhi) continue;
                if (ncand == cap) {
                    cap *= 2;
                    cidx = (int32_t*)realloc(cidx, sizeof(int32_t) * cap);
                    cu = (int32_t*)realloc(cu, sizeof(int32_t) * 2 * cap);
                }
                cidx[ncand] = (int32_t)m;
                cu[2 * ncand] = u1;
                cu[2 * ncand + 1] = u2;
                ++ncand;
            }
        }
    /* bins with head-inserted linked lists */
    int nbx = (int)((xhi - xlo) / rmax); if (nbx < 1) nbx = 1;
    int nby = (int)((yhi - ylo) / rmax); if (nby < 1) nby = 1;
    const double wx = (xhi - xlo) / nbx, wy = (yhi - ylo) / nby;
    int64_t* head = (int64_t*)malloc(sizeof(int64_t) * (size_t)nbx * nby);
    int64_t* next = (int64_t*)malloc(sizeof(int64_t) * (ncand + 1));
    for (int64_t k = 0; k < (int64_t)nbx * nby; ++k) head[k] = -1;
    for (int64_t c = 0; c < ncand; ++c) {
        const int64_t m = cidx[c];
        const double px = Rat[3 * m] + (double)cu[2 * c] * A1[0] + (double)cu[2 * c + 1] * A2[0];
        const double py = Rat[3 * m + 1] + (double)cu[2 * c] * A1[1] + (double)cu[2 * c + 1] * A2[1];
        int ibx = 1 + (int)((px - xlo) / wx); if (ibx < 1) ibx = 1; if (ibx > nbx) ibx = nbx;
        int iby = 1 + (int)((py - ylo) / wy); if (iby < 1) iby = 1; if (iby > nby) iby = nby;
        const int64_t b = (int64_t)(iby - 1) * nbx + (ibx - 1);
        next[c] = head[b];
        head[b] = c;
    }
    orc_nbr* out = (orc_nbr*)calloc(1, sizeof(orc_nbr));
    out->n = natoms;
    out->nneigh = (int32_t*)calloc(natoms, sizeof(int32_t));
    for (int pass = 1; pass <= 2; ++pass) {
        if (pass == 2) {
            int32_t mx = 0;
            for (int64_t i = 0; i < natoms; ++i) if (out->nneigh[i] > mx) mx = out->nneigh[i];
            out->max_neigh = mx < 1 ? 1 : mx;
            const size_t e = (size_t)natoms * out->max_neigh;
            out->nlist = (int32_t*)calloc(e, sizeof(int32_t));
            out->neighd = (double*)calloc(3 * e, sizeof(double));
            out->ncell = (int32_t*)calloc(3 * e, sizeof(int32_t));
        }
        for (int64_t nn = 0; nn < natoms; ++nn) {
            int32_t cnt = 0;
            const double xn = Rat[3 * nn], yn = Rat[3 * nn + 1], zn = Rat[3 * nn + 2];
            int ibx = 1 + (int)((xn - xlo) / wx); if (ibx < 1) ibx = 1; if (ibx > nbx) ibx = nbx;
            int iby = 1 + (int)((yn - ylo) / wy); if (iby < 1) iby = 1; if (iby > nby) iby = nby;
            for (int ax = (ibx - 1 > 1 ? ibx - 1 : 1); ax <= (ibx + 1 < nbx ? ibx + 1 : nbx); ++ax)
                for (int ay = (iby - 1 > 1 ? iby - 1 : 1); ay <= (iby + 1 < nby ? iby + 1 : nby); ++ay) {
                    int64_t c = head[(int64_t)(ay - 1) * nbx + (ax - 1)];
                    while (c >= 0) {
                        const int64_t m = cidx[c];
                        const int c1 = cu[2 * c], c2 = cu[2 * c + 1];
                        if (!(m == nn && c1 == 0 && c2 == 0)) {
                            const double tx = (double)c1 * A1[0] + (double)c2 * A2[0];
                            const double ty = (double)c1 * A1[1] + (double)c2 * A2[1];
                            const double tz = 0.0 * 0.0;
                            const double ddx = (Rat[3 * m] - xn) + tx;
                            const double ddy = (Rat[3 * m + 1] - yn) + ty;
                            const double ddz = (Rat[3 * m + 2] - zn) + tz;
                            const double adz = fabs(ddz);
                            const double d2 = ddx * ddx + ddy * ddy;
                            int keep;
                            if (adz < dzIntra) keep = d2 < cut2intra;
                            else if (adz > dzIntra && adz < dzInter) keep = d2 < cut2inter;
                            else if (second_layer && adz > dzInter && adz < dzSecond) keep = d2 < cut2inter;
                            else keep = 0;
                            if (keep) {
                                if (pass == 2) {
                                    const size_t e = (size_t)nn * out->max_neigh + cnt;
                                    out->nlist[e] = (int32_t)(m + 1);
                                    out->neighd[3 * e] = ddx;
                                    out->neighd[3 * e + 1] = ddy;
                                    out->neighd[3 * e + 2] = ddz;
                                    out->ncell[3 * e] = c1;
                                    out->ncell[3 * e + 1] = c2;
                                    out->ncell[3 * e + 2] = 0;
                                }
                                ++cnt;
                            }
                        }
                        c = next[c];
                    }
                }
            out->nneigh[nn] = cnt;
        }
    }
    free(cidx); free(cu); free(head); free(next);
    return out;
}

int32_t orc_nbr_max(const orc_nbr* b) { return b->max_neigh; }
int64_t orc_nbr_total(const orc_nbr* b)
{
    int64_t t = 0;
    for (int64_t i = 0; i < b->n; ++i) t += b->nneigh[i];
    return t;
}
void orc_nbr_copy(const orc_nbr* b, int32_t* Nneigh, int32_t* NList, double* NeighD, int32_t* neighCell)
{
    const size_t e = (size_t)b->n * b->max_neigh;
    if (Nneigh) memcpy(Nneigh, b->nneigh, sizeof(int32_t) * b->n);
    if (NList) memcpy(NList, b->nlist, sizeof(int32_t) * e);
    if (NeighD) memcpy(NeighD, b->neighd, sizeof(double) * 3 * e);
    if (neighCell) memcpy(neighCell, b->ncell, sizeof(int32_t) * 3 * e);
}
void orc_nbr_free(orc_nbr* b)
{
    if (!b) return;
    free(b->nneigh); free(b->nlist); free(b->neighd); free(b->ncell); free(b);
}
