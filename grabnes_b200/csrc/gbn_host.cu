// Host-side parts of the hot path that are O(N) and sequential by definition:
//   - cell vectors and atom positions of the Graphene and TwistedBilayerBasedOnMoireCell systems
//     (lanczosKuboCode/Src/cell.F90:108-140, 207-240; atoms.F90:124-230, 330-380, 1506-1607, 1768-1830),
//     in the reference's atom order and floating-point operation order (this file is compiled without
//     FMA contraction), so that the device neighbour search sees bit-identical positions;
//   - the uniform random numbers of GNU Fortran's intrinsic random_number after random_seed(PUT=...),
//     which the reference uses for its random-phase start vectors (kubo.F90:46-64) and Anderson
//     disorder (ham.F90:1237-1248, seeded by random.F90:31-52).  The generator is libgfortran's
//     (GCC >= 8): xoshiro256** (Blackman & Vigna) whose 256-bit state is the 8 seed words copied in
//     reverse order and XORed with a fixed key; a real(8) draw keeps the top 53 bits of the output.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <cstdlib>

#include "../../include/grabnes_gpu.h"

namespace {

const double kPi = 3.14159265358979323846264338327950288;

struct Xoshiro {
    uint64_t s[4];
    void put(int32_t seed) {
        static const uint64_t key[4] = {0xbd0c5b6e50c2df49ULL, 0xd46061cd46e1df38ULL, 0xbb4f4d4ed6103544ULL,
                                        0x114a583d0756ad39ULL};
        uint32_t w[8];
        for (int i = 0; i < 8; ++i) w[i] = (uint32_t)seed;
        memcpy(s, w, sizeof(s));
        for (int i = 0; i < 4; ++i) s[i] ^= key[i];
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double r8() { return (double)(next() & (~(uint64_t)0 << 11)) * 0x1p-64; }
};

int gcd_abs(int a, int b)
{
    a = abs(a);
    b = abs(b);
    if (a > b) { int t = a; a = b; b = t; }
    if (a == 0) return b;
    for (;;) {
        const int g = a % b;
        if (g == 0) return b;
        a = b;
        b = g;
    }
}

// Hermann indices as used for the layers (swap when the second set is not the smaller cell)
void moire_order(const int32_t m[4], int out[4], double* phi)
{
    int n[4] = {m[0], m[1], m[2], m[3]};
    const double g = (double)(n[0] * n[0] + n[1] * n[1] + n[0] * n[1]);
    const double delta = sqrt((double)(float)(n[2] * n[2] + n[3] * n[3] + n[2] * n[3]) / g);
    *phi = acos((2.0 * n[0] * n[2] + 2.0 * n[1] * n[3] + (double)(n[0] * n[3]) + (double)(n[1] * n[2])) /
                (2.0 * delta * g));
    if (!(delta < 1.0)) {
        int t = n[0]; n[0] = n[2]; n[2] = t;
        t = n[1]; n[1] = n[3]; n[3] = t;
    }
    memcpy(out, n, sizeof(n));
}

// one honeycomb layer of the supercell spanned by (mm0, mm1): fractional coordinates X[k][3]
void honeycomb_layer(int mm0, int mm1, double angle_deg, double dz, double yshift, double* X)
{
    const int64_t ncell = (int64_t)mm0 * mm0 + (int64_t)mm0 * mm1 + (int64_t)mm1 * mm1;
    const double a = angle_deg * kPi / 180.0;
    const double u[2][2] = {{cos(a), sin(a)}, {cos(a + kPi / 3.0), sin(a + kPi / 3.0)}};
    const double m[2][2] = {{(double)mm0, (double)mm1}, {(double)(-mm1), (double)(mm0 + mm1)}};
    double R[2][2];
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 2; ++c) R[r][c] = u[0][r] * m[c][0] + u[1][r] * m[c][1];
    double basis[2][2];
    const double third[2] = {1.0 / 3.0, 2.0 / 3.0};
    for (int j = 0; j < 2; ++j)
        for (int r = 0; r < 2; ++r) basis[j][r] = u[0][r] * third[j] + u[1][r] * third[j];
    int64_t n1 = gcd_abs(mm0, mm1), n2 = ncell / n1;
    if (n2 > n1) { const int64_t t = n1; n1 = n2; n2 = t; }
    for (int64_t i2 = 0; i2 < n2; ++i2)
        for (int64_t i1 = 0; i1 < n1; ++i1)
            for (int j = 0; j < 2; ++j) {
                double* x = X + 3 * (2 * (n1 * i2 + i1) + j);
                x[0] = (double)i1 * u[0][0] + (double)i2 * u[1][0] + basis[j][0];
                x[1] = (double)i1 * u[0][1] + (double)i2 * u[1][1] + basis[j][1];
            }
    const double det = R[1][1] * R[0][0] - R[0][1] * R[1][0];
    const bool generic = fabs(R[0][0]) > 1.0e-6 * fabs(R[1][0]);
    for (int64_t k = 0; k < 2 * ncell; ++k) {
        double* x = X + 3 * k;
        double f1, f2;
        if (generic) {
            f2 = R[0][0] * (x[1] - x[0] * R[1][0] / R[0][0]) / det;
            f1 = (x[0] - f2 * R[0][1]) / R[0][0];
        } else {
            const double dc = R[0][0] * R[1][1] - R[0][1] * R[1][0];
            f1 = (x[0] * R[1][1] - x[1] * R[0][1]) / dc;
            f2 = (x[1] * R[0][0] - x[0] * R[1][0]) / dc;
        }
        x[0] = fmod(f1, 1.0) + yshift;
        x[1] = fmod(f2, 1.0) + yshift;
        x[2] = 0.5 + dz;
        if (x[0] < 0.0) x[0] = fmod(x[0] + 1.0, 1.0);
        if (x[1] < 0.0) x[1] = fmod(x[1] + 1.0, 1.0);
        if (x[0] > 1.0) x[0] = fmod(x[0] - 1.0, 1.0);
        if (x[1] > 1.0) x[1] = fmod(x[1] - 1.0, 1.0);
    }
}

void frac_to_cart(int64_t n, const double* u, double* r)
{
    for (int64_t i = 0; i < n; ++i) {
        double* p = r + 3 * i;
        const double f1 = p[0], f2 = p[1], f3 = p[2];
        for (int k = 0; k < 3; ++k) p[k] = f1 * u[k] + f2 * u[3 + k] + f3 * u[6 + k];
    }
}

void cart_to_frac(int64_t n, const double* u, double* r)
{
    const double u11 = u[0], u21 = u[1], u12 = u[3], u22 = u[4], u33 = u[8];
    for (int64_t i = 0; i < n; ++i) {
        double* p = r + 3 * i;
        if (u11 != 0.0) {
            p[1] = u11 * (p[1] - p[0] * u21 / u11) / (u22 * u11 - u12 * u21);
            p[0] = (p[0] - p[1] * u12) / u11;
        } else {
            const double x = p[0], y = p[1], dc = u11 * u22 - u12 * u21;
            p[0] = (u22 * x - u12 * y) / dc;
            p[1] = (u11 * y - u21 * x) / dc;
        }
        p[2] = p[2] / u33;
    }
}


// One Cartesian -> fractional -> Cartesian conversion of a single position (AtomsSetFrac followed by
// AtomsSetCart, atoms.F90:1768-1830).
void roundtrip1(const double* u, double* p)
{
    cart_to_frac(1, u, p);
    frac_to_cart(1, u, p);
}

// The position of one atom after k roundtrips.  The map reaches a fixed point (or, rarely, a 2-cycle)
// within a few applications, so k is cut short once it does.
void roundtrip_k(const double* u, const double* c0, int64_t k, double* p)
{
    p[0] = c0[0]; p[1] = c0[1]; p[2] = c0[2];
    double prev[3] = {p[0], p[1], p[2]};
    for (int64_t it = 0; it < k; ++it) {
        const double before[3] = {p[0], p[1], p[2]};
        roundtrip1(u, p);
        if (p[0] == before[0] && p[1] == before[1] && p[2] == before[2]) return;   // fixed point
        if (it >= 1 && p[0] == prev[0] && p[1] == prev[1] && p[2] == prev[2]) {  // 2-cycle: parity decides
            if (((k - 1 - it) & 1) != 0) { p[0] = before[0]; p[1] = before[1]; p[2] = before[2]; }
            return;
        }
        prev[0] = before[0]; prev[1] = before[1]; prev[2] = before[2];
    }
}

}  // namespace

extern "C" {

int gbn_cell_atoms(const gbn_cell* p, int64_t* n)
{
    if (!p || !n) return GBN_ERR_ARG;
    if (p->super_cell < 1) return GBN_ERR_ARG;
    if (p->kind == GBN_CELL_GRAPHENE) {
        if (p->cell_size < 1) return GBN_ERR_ARG;
        const int64_t k = (int64_t)p->cell_size * p->super_cell;
        *n = 2 * k * k;
        return GBN_OK;
    }
    if (p->kind != GBN_CELL_TBG_MOIRE) return GBN_ERR_ARG;
    if ((p->m[0] == 0 && p->m[1] == 0) || (p->m[2] == 0 && p->m[3] == 0)) return GBN_ERR_ARG;
    int o[4];
    double phi;
    moire_order(p->m, o, &phi);
    int64_t s = p->super_cell, a = o[0] * s, b = o[1] * s, c = o[2] * s, d = o[3] * s;
    *n = 2 * (a * a + a * b + b * b) + 2 * (c * c + c * d + d * d);
    return GBN_OK;
}

int gbn_build_cell(const gbn_cell* p, double* ucell, double* rat, int32_t* species, int32_t* layer, double* twist)
{
    int64_t n;
    const int rc = gbn_cell_atoms(p, &n);
    if (rc) return rc;
    if (!ucell || !rat || !species || !layer) return GBN_ERR_ARG;
    const double aG = p->aG, h = p->height;
    memset(ucell, 0, 9 * sizeof(double));
    if (p->kind == GBN_CELL_GRAPHENE) {
        const int k = p->cell_size * p->super_cell;
        const double dk = (double)k;
        ucell[0] = aG * dk;
        ucell[1] = 0.0 * dk;
        ucell[3] = aG / 2.0 * dk;
        ucell[4] = sqrt(3.0) * aG / 2.0 * dk;
        ucell[8] = h;
        honeycomb_layer(k, 0, 0.0, 0.0, 0.0, rat);
        for (int64_t i = 0; i < n; ++i) {
            species[i] = (int32_t)((i % 2) + 1);
            layer[i] = 1;
        }
        frac_to_cart(n, ucell, rat);
        if (twist) *twist = 0.0;
        return GBN_OK;
    }
    int o[4];
    double phi;
    moire_order(p->m, o, &phi);
    const double uc[2][2] = {{aG, 0.0}, {aG / 2.0, sqrt(3.0) * aG / 2.0}};
    const int m1[2][2] = {{o[0], o[1]}, {-o[1], o[0] + o[1]}};
    for (int c = 0; c < 2; ++c)
        for (int r = 0; r < 2; ++r)
            ucell[3 * c + r] = (uc[0][r] * (double)m1[c][0] + uc[1][r] * (double)m1[c][1]) * (double)p->super_cell;
    ucell[8] = h;
    const int s = p->super_cell;
    const double g = p->d_interlayer / (2.0 * h);
    const int64_t nc = 2 * ((int64_t)o[0] * s * o[0] * s + (int64_t)o[0] * s * o[1] * s + (int64_t)o[1] * s * o[1] * s);
    // the second layer's offset (atoms.F90:352-366), from the indices after the swap and the super cell
    double yshift = 0.0;
    if (p->add_shift == 1 || p->add_shift == 2) {
        const int a = o[0] * s, b = o[1] * s;
        const double frac = p->shift_factor / (sqrt(3.0) * aG * sqrt((double)(a * a + a * b + b * b)));
        yshift = (p->add_shift == 1) ? (aG / 3.0) / ((double)a * aG) + frac : (aG / 3.0 / 2.0) / ((double)a * aG) + frac;
    }
    honeycomb_layer(o[0] * s, o[1] * s, 0.0, g, 0.0, rat);
    honeycomb_layer(o[2] * s, o[3] * s, -phi * 180.0 / kPi, -g, yshift, rat + 3 * nc);
    for (int64_t i = 0; i < n; ++i) species[i] = (int32_t)((i % 2) + 1);
    frac_to_cart(n, ucell, rat);
    for (int64_t i = 0; i < n; ++i) layer[i] = (rat[3 * i + 2] < 20.0) ? 1 : 2;
    if (twist) *twist = phi;
    return GBN_OK;
}

int gbn_cart_roundtrip(int64_t n, const double* ucell, double* rat)
{
    if (n < 0 || !ucell || !rat) return GBN_ERR_ARG;
    cart_to_frac(n, ucell, rat);
    frac_to_cart(n, ucell, rat);
    return GBN_OK;
}

int gbn_rng_uniform(int32_t seed, int64_t n, double* out)
{
    if (n < 0 || (!out && n > 0)) return GBN_ERR_ARG;
    Xoshiro x;
    x.put(seed);
    for (int64_t i = 0; i < n; ++i) out[i] = x.r8();
    return GBN_OK;
}

// Kubo.PDOS atom selections of CalcKubo (lanczosKuboCode/Src/calc.F90:362-541).  The reference's loops
// switch the module positions between fractional and Cartesian coordinates: the moire selections
// convert to fractional before testing an atom and back to Cartesian after each selected atom, so an
// atom is tested at F(R^k(r0)) with k the atoms selected before it (R = Cartesian->fractional->Cartesian)
// and its coords line holds R^(k+1)(r0).  The positions enter in Cartesian form.
int gbn_pdos_atoms(const gbn_pdos* p, int64_t n, const double* rat, const int32_t* species, const int32_t* layer,
                   const double* ucell, int64_t cap, int64_t* count, int64_t* atoms, double* coords)
{
    if (!p || n < 0 || !rat || !species || !layer || !ucell || !count || cap < 0 || (cap > 0 && (!atoms || !coords)))
        return GBN_ERR_ARG;
    int64_t cnt = 0;
    auto take = [&](int64_t i, const double* pos) {
        if (cnt < cap) {
            atoms[cnt] = i + 1;
            coords[3 * cnt] = pos[0]; coords[3 * cnt + 1] = pos[1]; coords[3 * cnt + 2] = pos[2];
        }
        ++cnt;
    };
    switch (p->mode) {
    case GBN_PDOS_DIST:   // calc.F90:362-380, Cartesian positions, open bounds
        for (int64_t i = 0; i < n; ++i) {
            const double* r = rat + 3 * i;
            if (r[0] > p->xmin && r[0] < p->xmax && r[1] > p->ymin && r[1] < p->ymax && i + 1 >= p->min_value)
                take(i, r);
        }
        break;
    case GBN_PDOS_MOIRE_SC1:
    case GBN_PDOS_SUPERMOIRE:
    case GBN_PDOS_SUPERMOIRE2:
    case GBN_PDOS_SUPERMOIRE3: {   // calc.F90:381-467
        const double len = p->supermoire_length / p->aG;
        const double sc = (double)p->super_cell, cs = (double)p->cell_size;
        const double t1 = 1.0 / sc / cs * len, t2 = 2.0 / sc / cs * len, t3 = 3.0 / sc / cs * len;
        const double sc1 = 1.0 / sc;
        int64_t k = 0;
        double pos[3], f[3];
        for (int64_t i = 0; i < n; ++i) {
            roundtrip_k(ucell, rat + 3 * i, k, pos);
            f[0] = pos[0]; f[1] = pos[1]; f[2] = pos[2];
            cart_to_frac(1, ucell, f);
            bool sel = false;
            if (p->mode == GBN_PDOS_MOIRE_SC1) {
                sel = f[0] < sc1 && f[1] < sc1 && i + 1 >= p->min_value;
                if (sel && p->ignore_layers_1_4 && (layer[i] == 1 || layer[i] == 4)) sel = false;
            } else {
                const double lo = p->mode == GBN_PDOS_SUPERMOIRE ? -INFINITY : (p->mode == GBN_PDOS_SUPERMOIRE2 ? t1 : t2);
                const double hi = p->mode == GBN_PDOS_SUPERMOIRE ? t1 : (p->mode == GBN_PDOS_SUPERMOIRE2 ? t2 : t3);
                sel = f[0] >= lo && f[1] >= lo && f[0] < hi && f[1] < hi && species[i] == 1 && i + 1 >= p->min_value;
            }
            if (!sel) continue;
            frac_to_cart(1, ucell, f);
            take(i, f);
            ++k;
        }
        break;
    }
    case GBN_PDOS_ATOM_LIST:   // calc.F90:471-487
        for (int j = 0; j < 6; ++j) {
            const int64_t i = (int64_t)p->atom_list[j] - 1;
            if (i < 0 || i >= n) return GBN_ERR_ARG;
            take(i, rat + 3 * i);
        }
        break;
    case GBN_PDOS_BY_NUMBER: {   // calc.F90:489-493
        const int64_t i = (int64_t)p->atom_number - 1;
        if (i < 0 || i >= n) return GBN_ERR_ARG;
        take(i, rat + 3 * i);
        break;
    }
    case GBN_PDOS_PNP: {   // calc.F90:494-541: the first atom past L/4 and the first past L/4 + 2 delta
        const double acc = p->aG / sqrt(3.0);
        const double limit1 = ((double)(p->cell_size * p->super_cell) * p->aG) * 1.0 / 4.0;
        const double lo2 = limit1 + p->pnp_delta * 2.0;
        bool f1 = false, f2 = false;
        for (int64_t i = 0; i < n; ++i) {
            const double* r = rat + 3 * i;
            if (r[0] > limit1 && r[0] < limit1 + acc && !f1) { f1 = true; take(i, r); }
            if (r[0] > lo2 && r[0] < lo2 + acc && !f2) { f2 = true; take(i, r); }
        }
        break;
    }
    default:
        return GBN_ERR_ARG;
    }
    *count = cnt;
    return GBN_OK;
}

// The sets of Kubo.PDOSLayer and Kubo.PDOSLayerAndSpecies (calc.F90:300-361) with the atom counts the
// reference assumes when it scales their start vectors.
int gbn_pdos_sets(const gbn_pdos* p, int64_t n, const int32_t* species, const int32_t* layer, int32_t cap,
                  int32_t* nsets, int32_t* set_of_atom, int32_t* set_layer, int32_t* set_species, double* assumed)
{
    if (!p || n < 0 || !species || !layer || !nsets || !set_of_atom || cap < 0 ||
        (cap > 0 && (!set_layer || !set_species || !assumed)))
        return GBN_ERR_ARG;
    const int32_t L = p->number_of_layers;
    if (L < 1) return GBN_ERR_ARG;
    const int64_t s2 = (int64_t)p->super_cell * p->super_cell;
    int32_t ns = 0;
    for (int64_t i = 0; i < n; ++i) set_of_atom[i] = -1;
    if (p->mode == GBN_PDOS_LAYER) {
        if (L > cap) return GBN_ERR_ARG;
        for (int32_t l = 1; l <= L; ++l) {
            int64_t m;
            const bool t3 = p->stack == GBN_STACK_T3BG, e4 = p->stack == GBN_STACK_ENCAPSULATED_FOUR;
            if (t3 && l >= 1 && l <= 6) m = (int64_t)p->n_c * s2;
            else if (e4 && l == 1) m = (int64_t)p->n_bn1 * s2;
            else if (e4 && l == 4) m = (int64_t)p->n_bn2 * s2;
            else if (e4 && (l == 2 || l == 3)) m = (int64_t)p->n_c * s2;
            else m = n / L;
            set_layer[l - 1] = l;
            set_species[l - 1] = 0;
            assumed[l - 1] = (double)m;
        }
        for (int64_t i = 0; i < n; ++i)
            if (layer[i] >= 1 && layer[i] <= L) set_of_atom[i] = layer[i] - 1;
        ns = L;
    } else if (p->mode == GBN_PDOS_LAYER_SPECIES) {
        int32_t maxs = 1;
        for (int64_t i = 0; i < n; ++i) maxs = species[i] > maxs ? species[i] : maxs;
        for (int32_t l = 1; l <= L; ++l)
            for (int32_t s = 1; s <= maxs; ++s) {
                int64_t m = 0;
                for (int64_t i = 0; i < n; ++i)
                    if (layer[i] == l && species[i] == s) ++m;
                if (m == 0) continue;   // combinations without atoms are skipped
                if (ns >= cap) return GBN_ERR_ARG;
                for (int64_t i = 0; i < n; ++i)
                    if (layer[i] == l && species[i] == s) set_of_atom[i] = ns;
                set_layer[ns] = l;
                set_species[ns] = s;
                assumed[ns] = (double)m;
                ++ns;
            }
    } else {
        return GBN_ERR_ARG;
    }
    *nsets = ns;
    return GBN_OK;
}

}  // extern "C"
