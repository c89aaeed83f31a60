/*
 * Oracle (test infrastructure only): on-site energies, hoppings and Peierls
 * phases of the models on the recursion hot path.  Restates the reference's
 * arithmetic in the same operation order (see oracle.h for the rules).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.14159265358979323846264338327950288

/* diago, ham.F90:4696-4716:
 * 2 C Re[(e^{-i G dy} + 2 e^{i G dy/2} cos(sqrt3 G dx/2)) e^{i phi}] */
static double diago(double dx, double dy, double C, double phi, double aG)
{
    const double G1 = 4.0 * ORC_PI / sqrt(3.0) / aG;
    const double e1r = cos(G1 * dy), e1i = -sin(G1 * dy);
    const double hh = G1 * dy / 2.0;
    const double k = cos(sqrt(3.0) * G1 * dx / 2.0);
    const double e2r = 2.0 * cos(hh) * k, e2i = 2.0 * sin(hh) * k;
    const double sr = e1r + e2r, si = e1i + e2i;
    const double pr = cos(phi), pi_ = sin(phi);
    return 2.0 * C * (sr * pr - si * pi_);
}

/* offdiago, ham.F90:4752-4776 */
static void offdiago(double dx, double dy, double C, double phi, double aG, double* re, double* im)
{
    const double G1 = 4.0 * ORC_PI / sqrt(3.0) / aG;
    const double ax = sqrt(3.0) * G1 * dx / 2.0;
    const double p = cos(G1 * dy / 2.0 - phi);
    const double q = sin(G1 * dy / 2.0 - phi - ORC_PI / 6.0);
    *re = 2.0 * C * cos(ax) * (p + q) + 2.0 * C * sin(G1 * dy + phi - ORC_PI / 6.0);
    *im = 2.0 * C * sin(ax) * (p - q);
}

/* del(1..3) of one atom or bond: ham.F90:12666-12678, :4862-4868 */
static void bond_deltas(int spec, double re, double im, double del[3])
{
    del[0] = 2.0 * re / 3.0;
    if (spec == 1) {
        del[1] = -(re + sqrt(3.0) * im) / 3.0;
        del[2] = (-re + sqrt(3.0) * im) / 3.0;
    } else {
        del[1] = (-re + sqrt(3.0) * im) / 3.0;
        del[2] = -(re + sqrt(3.0) * im) / 3.0;
    }
}

/* moire displacement map d = ((1+eps) R(theta) - 1) r (ham.F90:12610-12617, :3452-3458) */
static void moire_disp(const orc_model* m, double x, double y, int integer_one, double* dx, double* dy)
{
    (void)integer_one;
    if (m->moire_twisted) {
        const double t = m->twist_rad;
        *dx = x * ((1.0 + m->eps) * cos(t) - 1.0) - y * (1.0 + m->eps) * sin(t);
        *dy = y * ((1.0 + m->eps) * cos(t) - 1.0) + x * (1.0 + m->eps) * sin(t);
    } else {
        *dx = x * m->eps;
        *dy = y * m->eps;
    }
}

/* Displacement of the second moire before its shift and flip (HamOnSiteSecondMoireTerms, ham.F90:3573-3590;
 * the Structure.BasedOnMoireCellParameters branch is not restated: it reads eps2, which is never set) */
static void second_moire_disp(const orc_model* m, double x, double y, double* dx, double* dy)
{
    const double e = m->eps * m->eps_factor;
    const double t = m->twist2_rad;
    if (m->twisted2) {
        if (m->rotate_first) {
            *dx = x * ((1.0 + e) * cos(t) - 1.0) - y * (1.0 + e) * sin(t);
            *dy = y * ((1.0 + e) * cos(t) - 1.0) + x * (1.0 + e) * sin(t);
        } else {
            const double ys = y - m->shift2 / m->eps;
            *dx = x * ((1.0 + e) * cos(t) - 1.0) - ys * (1.0 + e) * sin(t);
            *dy = ys * ((1.0 + e) * cos(t) - 1.0) + x * (1.0 + e) * sin(t);
        }
    } else {
        *dx = x * e;
        *dy = y * e;
    }
}

/* Displacement of the encapsulated bilayer's moire at atom (x, y) of layer L (HamOnSiteMoireEffectiveBilayer,
 * ham.F90:3318-3376, and the same lines of the bond terms, :12564-12585): layer 1 from the bottom hBN angle
 * plus (tauX1, tauY1), the other layer from the top angle with (tauX2, tauY2) added after the rotation, or,
 * without rotate_first, tauY2 / eps taken off y before it. */
static void bilayer_disp(const orc_model* m, int L, double x, double y, double* dx, double* dy)
{
    const double e1 = 1.0 + m->eps;
    if (L == 1) {
        const double a = m->bl_bottom_rad;
        *dx = (e1 * cos(a) - 1.0) * x - (e1 * sin(a) * y);
        *dy = (e1 * cos(a) - 1.0) * y + (e1 * sin(a) * x);
        *dx = *dx + m->tau[0];
        *dy = *dy + m->tau[1];
    } else if (m->rotate_first) {
        const double a = m->bl_top_rad;
        *dx = (e1 * cos(a) - 1.0) * x - (e1 * sin(a) * y);
        *dy = (e1 * cos(a) - 1.0) * y + (e1 * sin(a) * x);
        *dx = *dx + m->tau[2];
        *dy = *dy + m->tau[3];
    } else {
        const double a = m->bl_top_rad, ys = y - m->tau[3] / m->eps;
        *dx = (e1 * cos(a) - 1.0) * x - (e1 * sin(a) * ys);
        *dy = (e1 * cos(a) - 1.0) * ys + (e1 * sin(a) * x);
    }
}

/* Moire.BLDeactivateUpperLayer / TDBLDeactivateUpperLayers: no moire term on layer 2 / above layer 1 */
static int deactivated(const orc_model* m, int L)
{
    return (L == 2 && m->deact_upper) || (L != 1 && m->deact_uppers);
}

static void moire_terms(const orc_model* m, double dx, double dy, double* Hz, double* Hd)
{
    *Hz = 0.0;
    *Hd = 0.0;
    switch (m->moire_onsite) {
    case ORC_ONSITE_ONLY_H0: *Hd = diago(dx, dy, m->C0, m->Phi0, m->aG); break;
    case ORC_ONSITE_ONLY_HZ: *Hz = diago(dx, dy, m->Cz, m->Phiz, m->aG); break;
    case ORC_ONSITE_NO_H0_AND_HZ: break;
    case ORC_ONSITE_H0_AND_HZ:
        *Hz = diago(dx, dy, m->Cz, m->Phiz, m->aG);
        *Hd = diago(dx, dy, m->C0, m->Phi0, m->aG);
        break;
    }
}

void orc_onsite_layers(const orc_model* m, int64_t n, const double* Rat, const int32_t* species,
                       const int32_t* layer, double* H0, double* H0Bottom)
{
    /* ham.F90:846-850 and HamOnSiteSpeciesEnergies :3703-4014 (carbon), called at :947 */
    for (int64_t i = 0; i < n; ++i) H0[i] = m->e0_c;
    /* Anderson disorder, ham.F90:1237-1248 (before the moire terms), seeded by RandSeedFromInput
     * (random.F90:31-52) */
    if (m->anderson) {
        orc_rng r;
        orc_rng_put(&r, m->seed);
        for (int64_t i = 0; i < n; ++i) {
            const double rnd = orc_rng_r8(&r);
            H0[i] = H0[i] + (rnd - 0.5) * m->anderson_w;
        }
    }
    if (H0Bottom)
        for (int64_t i = 0; i < n; ++i) H0Bottom[i] = 0.0;
    if (m->moire_onsite == ORC_ONSITE_NONE) return;
    if (m->encapsulated) {
        /* HamOnSiteMoireEffectiveBilayer, ham.F90:3303-3434 (H0Bottom stays 0 on this branch) */
        for (int64_t i = 0; i < n; ++i) {
            double dx, dy, Hz = 0.0, Hd = 0.0;
            bilayer_disp(m, layer[i], Rat[3 * i], Rat[3 * i + 1], &dx, &dy);
            if (layer[i] == 1 || !deactivated(m, layer[i])) moire_terms(m, dx, dy, &Hz, &Hd);
            const double sgn = (species[i] % 2 == 1) ? -1.0 : 1.0;
            H0[i] = H0[i] + sgn * Hz + Hd;   /* (H0 + (-1)**S Hz) + H0jj, left to right */
        }
        return;
    }
    /* HamOnSiteMoireEffective, ham.F90:3437-3544 */
    for (int64_t i = 0; i < n; ++i) {
        double dx, dy, Hz, Hd;
        moire_disp(m, Rat[3 * i], Rat[3 * i + 1], 1, &dx, &dy);
        dy = dy + m->shift1;
        if ((layer[i] == 1 && m->sign1 < 0.0) || (layer[i] == 2 && m->sign2 < 0.0)) {
            dx = -dx;
            dy = -dy;
        }
        moire_terms(m, dx, dy, &Hz, &Hd);
        const double sgn = (species[i] % 2 == 1) ? -1.0 : 1.0; /* (-1)**Species */
        if (layer[i] == 1) H0[i] = H0[i] + sgn * Hz * m->sign1 + Hd;
        else if (layer[i] == 2) H0[i] = H0[i] + sgn * Hz * m->sign2 + Hd;
    }
    /* H0Bottom = H0, ham.F90:2703 */
    if (H0Bottom)
        for (int64_t i = 0; i < n; ++i) H0Bottom[i] = H0[i];
    if (!m->second_moire) return;
    /* HamOnSiteSecondMoireTerms, ham.F90:3546-3642: every atom, whatever its layer */
    for (int64_t i = 0; i < n; ++i) {
        double dx, dy, Hz, Hd;
        second_moire_disp(m, Rat[3 * i], Rat[3 * i + 1], &dx, &dy);
        if (m->rotate_first) {
            dy = dy + m->shift2_y;
            dx = dx + m->shift2_x;
        }
        if (m->sign2 < 0.0) {
            dx = -dx;
            dy = -dy;
        }
        moire_terms(m, dx, dy, &Hz, &Hd);
        const double sgn = (species[i] % 2 == 1) ? -1.0 : 1.0;
        H0[i] = H0[i] + sgn * Hz * m->sign2 + Hd;
    }
}

void orc_onsite(const orc_model* m, int64_t n, const double* Rat, const int32_t* species,
                const int32_t* layer, double* H0)
{
    orc_onsite_layers(m, n, Rat, species, layer, H0, NULL);
}

/* MoireBondDeltaMidpoint, ham.F90:4822-4883: the bond term of one bond from the moire displacement at the
 * bond's midpoint.  First moire: its own mismatch and twist, shift1 before the flip, no post shift, no flip
 * of Im, no swap; second moire (ham.F90:7866-7869): eps * eps_factor, TwistAngle2, the flip, shift2 after
 * it, and the flip of Im and the swap of del(2) and del(3) with the mass factor's sign. */
static double mid_delta(const double* ri, const double* bond, int spec, double epsM, double thM, double pre_y,
                        int flip, double post_x, double post_y, int flip_imag, int swap23, double Cab, double Phi,
                        double aG)
{
    if (spec != 1 && spec != 2) return 0.0;
    const double rm0 = ri[0] + 0.5 * bond[0], rm1 = ri[1] + 0.5 * bond[1];
    double ddx = rm0 * ((1.0 + epsM) * cos(thM) - 1.0) - rm1 * (1.0 + epsM) * sin(thM);
    double ddy = rm1 * ((1.0 + epsM) * cos(thM) - 1.0) + rm0 * (1.0 + epsM) * sin(thM);
    ddy = ddy + pre_y;
    if (flip) {
        ddx = -ddx;
        ddy = -ddy;
    }
    ddx = ddx + post_x;
    ddy = ddy + post_y;
    double re, im, del[3];
    offdiago(ddx, ddy, Cab, Phi, aG, &re, &im);
    if (flip_imag) im = -im;
    bond_deltas(spec, re, im, del);
    if (fabs(bond[0]) < aG / 4.0) return del[0];
    if (bond[0] < 0.0) return swap23 ? del[1] : del[2];
    return swap23 ? del[2] : del[1];
}

static double moire_mid_delta(const orc_model* m, const double* ri, const double* bond, int spec, int flip)
{
    const double th = m->moire_twisted ? m->twist_rad : 0.0;
    return mid_delta(ri, bond, spec, m->eps, th, m->shift1, flip, 0.0, 0.0, 0, 0, m->Cab, m->Phiab, m->aG);
}

/* F2G2 single-layer shell terms of HamHopIntralayerGraphene, ham.F90:10660-10925 (twoLayers/oneLayer). */
static double f2g2_shell(const orc_model* m, double dist)
{
    const double aG = m->aG, aCC = m->aCC;
    if (dist > aCC * 0.9 && dist < aCC * 1.1) return 0.0;
    if (dist > aG * 0.9 && dist < aG * 1.1) return m->tksl[2];
    if (dist > 2.0 * aCC * 0.9 && dist < aCC * 2.0 * 1.1) return m->tksl[3];
    if (dist > 2.0 * aCC * 1.1 && dist < 4.0) return m->tksl[4];
    if (dist > (aCC * 3.0) * 0.9 && dist < (aCC * 3.0) * 1.1) return m->tksl[5];
    if (dist > 2.0 * aG * 0.97 && dist < 2.0 * aG * 1.03) return m->tksl[6];
    const double r7 = sqrt((2.0 * aG) * (2.0 * aG) + aCC * aCC);
    if (dist > r7 * 0.9 && dist < r7 * 1.1) return m->tksl[7];
    return 0.0; /* shell 8 is zero in every configuration used here */
}

/* HamHopping bond loop, ham.F90:6517-6846, for carbon layers (Species 1, 2):
 * intralayer HamHopIntralayerDefault (:10177-10194) or HamHopIntralayerGraphene
 * (:10616-10931); interlayer HamHopInterlayerTwoCenter (:9620-9838) with
 * interlayerTwoCenter (:4094-4110), or the gIntLay term (:6837-6840). */
/* HamHopSecondMoire, ham.F90:7745-7880: a second pass over the bonds of each layer, after every other
 * term, that subtracts the second moire's bond term from the first-shell bonds.  Its displacement is
 * always rotated by Moire.TwistAngle2 (Moire.Twisted2 is not read here), flipped before the shift
 * (the on-site term shifts first), and Im of the bond amplitude changes sign with the mass factor.
 * delta carries over between the bonds of one atom, as in the reference (bonds with 0.01 <= |dx| <= 0.02
 * keep the previous one).  The reference leaves del unset for species other than 1 and 2; the library's
 * cells have only those two, and 0 stands there.  With Moire.OffDiagMidpoint the term of each bond comes
 * from its midpoint (MoireBondDeltaMidpoint with the second moire's arguments, ham.F90:7866-7869). */
static void second_moire_bonds(const orc_model* m, int64_t n, const double* Rat, const int32_t* species,
                               const int32_t* layer, int32_t maxNeigh, const int32_t* Nneigh,
                               const int32_t* NList, const double* NeighD, double* hopp)
{
    for (int64_t i = 0; i < n; ++i) {
        double delta = 0.0;
        double del[3] = {0.0, 0.0, 0.0};
        const double x = Rat[3 * i], y = Rat[3 * i + 1], t = m->twist2_rad, e = m->eps * m->eps_factor;
        double dx, dy;
        if (m->rotate_first) {
            dx = x * ((1.0 + e) * cos(t) - 1.0) - y * (1.0 + e) * sin(t);
            dy = y * ((1.0 + e) * cos(t) - 1.0) + x * (1.0 + e) * sin(t);
        } else {
            const double ys = y - m->shift2 / m->eps / m->eps_factor;
            dx = x * ((1.0 + e) * cos(t) - 1.0) - ys * (1.0 + m->eps) * sin(t);
            dy = ys * ((1.0 + m->eps) * cos(t) - 1.0) + x * (1.0 + m->eps / m->eps_factor) * sin(t);
        }
        if (m->sign2 < 0.0) {
            dx = -dx;
            dy = -dy;
        }
        if (m->rotate_first) {
            dx = dx + m->shift2_x;
            dy = dy + m->shift2_y;
        }
        double re, im;
        offdiago(dx, dy, m->Cab, m->Phiab, m->aG, &re, &im);
        if (m->sign2 < 0.0) im = -im;
        if (species[i] == 1 || species[i] == 2) bond_deltas(species[i], re, im, del);   /* ham.F90:7817-7833 */
        for (int32_t j = 0; j < Nneigh[i]; ++j) {
            const size_t e2 = (size_t)i * maxNeigh + j;
            const int64_t jj = NList[e2] - 1;
            if (layer[i] != layer[jj]) continue;
            const double* D = NeighD + 3 * e2;
            const double d = sqrt(D[0] * D[0] + D[1] * D[1]);
            for (int lv = 0; lv < m->tbnn; ++lv) {
                if (d < m->nradii[lv]) {
                    if (fabs(D[0]) < 0.01) delta = del[0];
                    else if (D[0] < -0.02) delta = (m->sign2 < 0.0) ? del[1] : del[2];
                    else if (D[0] > 0.02) delta = (m->sign2 < 0.0) ? del[2] : del[1];
                    if (m->moire_mid) {
                        const int neg = m->sign2 < 0.0;
                        delta = mid_delta(Rat + 3 * i, D, species[i], m->eps * m->eps_factor, m->twist2_rad, 0.0, neg,
                                          m->shift2_x, m->shift2_y, neg, neg, m->Cab, m->Phiab, m->aG);
                    }
                    if (d > 1.7) delta = 0.0;
                    hopp[2 * e2] = hopp[2 * e2] - 1.0 * delta;
                    break;
                }
            }
        }
    }
}

void orc_hopping(const orc_model* m, int64_t n, const double* Rat, const int32_t* species,
                 const int32_t* layer, int32_t maxNeigh, const int32_t* Nneigh, const int32_t* NList,
                 const double* NeighD, double* hopp)
{
    memset(hopp, 0, sizeof(double) * 2 * (size_t)n * maxNeigh);
    int bernal = 0;
    int8_t* dimer = NULL;
    if (m->encapsulated) {
        bernal = m->bernal;
        if (bernal == 2) {
            dimer = (int8_t*)calloc((size_t)n, 1);
            if (!dimer) return;
            const int64_t cnt = orc_bernal_dimers(n, layer, maxNeigh, Nneigh, NList, NeighD, dimer);
            if (llabs(2 * cnt - n) > n / 10) bernal = 1; /* not AB stacked: the former coupling, ham.F90:6488-6495 */
        }
    }
    for (int64_t i = 0; i < n; ++i) {
        double delta = 0.0;
        double del[3] = {0.0, 0.0, 0.0};
        if (m->moire_offdiag) { /* HamHopBondTermsMoire, ham.F90:12542-12680 */
            double dx, dy, re = 0.0, im = 0.0;
            if (m->encapsulated) bilayer_disp(m, layer[i], Rat[3 * i], Rat[3 * i + 1], &dx, &dy);
            else moire_disp(m, Rat[3 * i], Rat[3 * i + 1], 0, &dx, &dy);
            dy = dy + m->shift1;
            if ((layer[i] == 1 && m->sign1 < 0.0) || (layer[i] == 2 && m->sign2 < 0.0)) {
                dx = -dx;
                dy = -dy;
            }
            if (!deactivated(m, layer[i])) offdiago(dx, dy, m->Cab, m->Phiab, m->aG, &re, &im);
            if (species[i] == 1 || species[i] == 2) bond_deltas(species[i], re, im, del);
        }
        const int flip = (layer[i] == 1 && m->sign1 < 0.0) || (layer[i] == 2 && m->sign2 < 0.0);
        for (int32_t j = 0; j < Nneigh[i]; ++j) {
            const size_t e = (size_t)i * maxNeigh + j;
            const int64_t jj = NList[e] - 1;
            const double* D = NeighD + 3 * e;
            double* h = hopp + 2 * e;
            if (layer[i] == layer[jj]) {
                const double d = sqrt(D[0] * D[0] + D[1] * D[1]);
                for (int lv = 0; lv < m->tbnn; ++lv) {
                    if (d < m->nradii[lv]) {
                        if (d < 1.7) {
                            if (fabs(D[0]) < m->aG / 4.0) delta = del[0];
                            else if (D[0] < -m->aG / 4.0) delta = del[2];
                            else if (D[0] > m->aG / 4.0) delta = del[1];
                            if (m->moire_mid) delta = moire_mid_delta(m, Rat + 3 * i, D, species[i], flip);
                        }
                        if (m->intralayer == ORC_INTRA_F2G2_SL) {
                            const double dist = sqrt(D[0] * D[0] + D[1] * D[1]);
                            h[0] = h[0] + f2g2_shell(m, dist);
                        }
                        if (d > 1.5) delta = 0.0;
                        h[0] = h[0] + (m->gn_cc[lv] - 1.0 * delta);
                        break;
                    }
                }
            } else if (layer[i] == layer[jj] + 1 || layer[i] == layer[jj] - 1) {
                if (m->encapsulated) {
                    /* the encapsulated bilayer's interlayer branch, ham.F90:6721-6745 */
                    if (bernal == 2) { /* HamHopInterlayerBernalF2G2, ham.F90:12800-12827 */
                        const int mixed = dimer[i] != dimer[jj];
                        const double dxy = sqrt(D[0] * D[0] + D[1] * D[1]), aCC = m->aCC, aG = m->aG;
                        const double* t = m->tbl; /* tAA1 tAA2 tAB1 tAB2 tBA0 tBA2 tBA5 */
                        if (dxy < 0.2) h[0] = h[0] + t[4];
                        else if (dxy > aCC * 0.9 && dxy < aCC * 1.1) h[0] = h[0] + (mixed ? t[0] : t[2]);
                        else if (dxy > aG * 0.9 && dxy < aG * 1.1) h[0] = h[0] + t[5];
                        else if (dxy > aCC * 2.0 * 0.9 && dxy < aCC * 2.0 * 1.1) h[0] = h[0] + (mixed ? t[1] : t[3]);
                        else if (dxy > (aCC * 3.0) * 0.9 && dxy < (aCC * 3.0) * 1.1 && !mixed) h[0] = h[0] + t[6];
                    } else if (fabs(D[0]) < 0.01 && fabs(D[1]) < 0.01) {
                        h[0] = h[0] - m->tbl[2];
                    }
                } else if (m->interlayer == ORC_INTER_TWO_CENTRE) {
                    /* ham.F90:9810-9830: renormalizeHoppingFactorAAp of KoshinoSR (aval 1.34, bval 3.25) */
                    const double dist = sqrt(D[0] * D[0] + D[1] * D[1] + D[2] * D[2]);
                    const double renorm = m->koshino_sr ? exp((fabs(D[2]) - 3.25) / 1.34) : 1.0;
                    const double vsig = m->vppsigma0 * exp(-(dist - m->d_interlayer) / m->bl_delta) * renorm;
                    const double vpi = m->vpppi0 * exp(-(dist - m->aCC) / m->bl_delta) * renorm;
                    const double q = D[2] / dist;
                    double sc = 1.0;   /* smooth cutoff of the differentiable model (1 without one) */
                    if (m->inter_smooth_w > 0.0) {
                        const double rho = sqrt(D[0] * D[0] + D[1] * D[1]);
                        const double r0 = m->inter_cut_rho - m->inter_smooth_w;
                        if (rho >= m->inter_cut_rho) sc = 0.0;
                        else if (rho > r0) sc = 0.5 * (1.0 + cos(ORC_PI * (rho - r0) / m->inter_smooth_w));
                    }
                    h[0] = h[0] + (vpi * (1.0 - q * q) + vsig * (q * q)) * sc;
                    /* ham.F90:6807-6838 without Interlayer.DifferentCouplings */
                    if (m->renormalize_coupling) h[0] = m->coupling_factor * h[0];
                } else {
                    const double d = sqrt(D[0] * D[0] + D[1] * D[1]);
                    h[0] = h[0] + m->g_intlay * exp(-d / m->d_interlayer);
                }
            }
        }
    }
    free(dimer);
    if (m->second_moire && m->moire_offdiag) second_moire_bonds(m, n, Rat, species, layer, maxNeigh, Nneigh, NList,
                                                                NeighD, hopp);
}

/* Dimer sites of the Bernal interlayer branch, ham.F90:6475-6484: an atom with a neighbour of an adjacent
 * layer within 0.2 A in plane.  Returns their number. */
int64_t orc_bernal_dimers(int64_t n, const int32_t* layer, int32_t maxNeigh, const int32_t* Nneigh,
                          const int32_t* NList, const double* NeighD, int8_t* dimer)
{
    int64_t cnt = 0;
    for (int64_t i = 0; i < n; ++i) {
        dimer[i] = 0;
        for (int32_t j = 0; j < Nneigh[i]; ++j) {
            const size_t e = (size_t)i * maxNeigh + j;
            const int64_t jj = NList[e] - 1;
            if (layer[i] != layer[jj] + 1 && layer[i] != layer[jj] - 1) continue;
            const double* D = NeighD + 3 * e;
            if (sqrt(D[0] * D[0] + D[1] * D[1]) < 0.2) dimer[i] = 1;
        }
        cnt += dimer[i];
    }
    return cnt;
}

/* HamPeierlsPeriodicGauge, ham.F90:12834-12882 (with the corner term). */
void orc_peierls(int64_t n, const double* Rat, const double* ucell, int32_t maxNeigh,
                 const int32_t* Nneigh, const int32_t* NList, const int32_t* neighCell,
                 double flux, double* hopp)
{
    const double cellArea = fabs(ucell[0] * ucell[4] - ucell[1] * ucell[3]);
    const double fluxQuanta = flux * cellArea / (ORC_PI * 1.0e20);
    const double mq = (double)lround(fluxQuanta);
    for (int64_t i = 0; i < n; ++i) {
        const double* ri = Rat + 3 * i;
        for (int32_t j = 0; j < Nneigh[i]; ++j) {
            const size_t e = (size_t)i * maxNeigh + j;
            const double* rj = Rat + 3 * (size_t)(NList[e] - 1);
            const int n1 = neighCell[3 * e], n2 = neighCell[3 * e + 1];
            double v1[3] = {ri[0] + rj[0], ri[1] + rj[1], ri[2] + rj[2]};
            double v2[3];
            for (int k = 0; k < 3; ++k) v2[k] = (double)n1 * ucell[k] + (double)n2 * ucell[3 + k];
            const double c3 = v1[0] * v2[1] - v1[1] * v2[0];             /* (v1 x v2)_z */
            const double r3 = ri[0] * rj[1] - ri[1] * rj[0];             /* (ri x rj)_z */
            double phase = flux * (r3 + c3) / 1.0e20;
            if (n1 != 0 && n2 != 0) phase = phase + ORC_PI * mq * (double)n1 * (double)n2;
            const double c = cos(phase), s = sin(phase);
            double* h = hopp + 2 * e;
            const double hr = h[0], hi = h[1];
            h[0] = hr * c - hi * s;
            h[1] = hr * s + hi * c;
        }
    }
}

/* HamHaldaneChirality, ham.F90:13063-13100: +1 if the path i -> k -> j through a common nearest
 * neighbour turns clockwise, -1 if anticlockwise, 0 if there is none. */
static int haldane_chirality(const int32_t* layer, int32_t maxNeigh, const int32_t* Nneigh, const int32_t* NList,
                             const double* NeighD, double aG, int64_t i, int jn)
{
    const double* dij = NeighD + 3 * ((size_t)i * maxNeigh + jn);
    const double acc = aG / sqrt(3.0);
    for (int k1 = 0; k1 < Nneigh[i]; ++k1) {
        const int64_t k = NList[(size_t)i * maxNeigh + k1] - 1;
        if (layer[k] != layer[i]) continue;
        const double* d1 = NeighD + 3 * ((size_t)i * maxNeigh + k1);
        if (fabs(sqrt(d1[0] * d1[0] + d1[1] * d1[1]) - acc) > 0.1) continue;
        for (int k2 = 0; k2 < Nneigh[k]; ++k2) {
            if (NList[(size_t)k * maxNeigh + k2] != NList[(size_t)i * maxNeigh + jn]) continue;
            const double* d2 = NeighD + 3 * ((size_t)k * maxNeigh + k2);
            if (fabs(sqrt(d2[0] * d2[0] + d2[1] * d2[1]) - acc) > 0.1) continue;
            const double ex = d1[0] + d2[0] - dij[0], ey = d1[1] + d2[1] - dij[1];
            if (sqrt(ex * ex + ey * ey) > 0.1) continue;
            const double cr = d1[0] * d2[1] - d1[1] * d2[0];
            return cr < 0.0 ? 1 : -1;
        }
    }
    return 0;
}

int64_t orc_haldane(int64_t n, const int32_t* species, const int32_t* layer, int32_t maxNeigh,
                    const int32_t* Nneigh, const int32_t* NList, const double* NeighD, double aG, double t2,
                    double phase, int32_t paper, uint32_t layer_mask, double* hopp)
{
    int64_t missing = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (layer_mask != 0u && (layer[i] < 1 || layer[i] > 32 || !((layer_mask >> (layer[i] - 1)) & 1u))) continue;
        for (int j = 0; j < Nneigh[i]; ++j) {
            const size_t e = (size_t)i * maxNeigh + j;
            const int64_t jj = NList[e] - 1;
            if (layer[jj] != layer[i]) continue;
            const double* D = NeighD + 3 * e;
            const double d = sqrt(D[0] * D[0] + D[1] * D[1]);
            if (!((d - 0.1) < aG && (d + 0.1) > aG && species[i] <= 2)) continue;
            const int nu = haldane_chirality(layer, maxNeigh, Nneigh, NList, NeighD, aG, i, j);
            if (nu == 0) {
                ++missing;
                continue;
            }
            const double c = cos(nu * phase), s = sin(nu * phase);
            double* h = hopp + 2 * e;
            if (paper) {
                const double re = h[0] * c - h[1] * s, im = h[0] * s + h[1] * c;
                h[0] = re;
                h[1] = im;
            } else {
                h[0] = h[0] + t2 * c;
                h[1] = h[1] + t2 * s;
            }
        }
    }
    return missing;
}

void orc_check_hamiltonian(int64_t n, int32_t maxNeigh, const int32_t* Nneigh, const int32_t* NList,
                           const int32_t* neighCell, const double* hopp, const double* H0, int64_t* out,
                           double* max_asym)
{
    int64_t nhop = 0, nons = 0, first = 0, missing = 0, pairs = 0;
    double mx = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        if (!isfinite(H0[i])) {
            ++nons;
            if (first == 0) first = i + 1;
        }
        for (int j = 0; j < Nneigh[i]; ++j) {
            const double* h = hopp + 2 * ((size_t)i * maxNeigh + j);
            if (!(isfinite(h[0]) && isfinite(h[1]))) {
                ++nhop;
                if (first == 0) first = i + 1;
            }
        }
    }
    for (int64_t i = 0; i < n; ++i)
        for (int j = 0; j < Nneigh[i]; ++j) {
            const size_t e = (size_t)i * maxNeigh + j;
            const int64_t m = NList[e] - 1;
            if (m < i) continue;
            int j2 = 0;
            for (; j2 < Nneigh[m]; ++j2) {
                const size_t e2 = (size_t)m * maxNeigh + j2;
                if (NList[e2] - 1 == i && neighCell[3 * e2] == -neighCell[3 * e] &&
                    neighCell[3 * e2 + 1] == -neighCell[3 * e + 1] && neighCell[3 * e2 + 2] == -neighCell[3 * e + 2])
                    break;
            }
            if (j2 >= Nneigh[m]) {
                ++missing;
                continue;
            }
            if (m == i && j2 <= j) continue;
            ++pairs;
            const double* a = hopp + 2 * e;
            const double* b = hopp + 2 * ((size_t)m * maxNeigh + j2);
            const double asym = hypot(a[0] - b[0], a[1] + b[1]);
            if (asym > mx) mx = asym;
        }
    out[0] = nhop;
    out[1] = nons;
    out[2] = first;
    out[3] = missing;
    out[4] = pairs;
    *max_asym = mx;
}
