// Hamiltonian assembly on the device: on-site energies (HamOnSite), hoppings of the bond loop
// (HamHopping) and Peierls phases (HamPeierlsPeriodicGauge) for the models on the recursion path:
//   - carbon shells with gn(C,C,shell) and, for the Koshino/HTC bilayers, the single-layer F2G2
//     shell terms (ham.F90:10177-10194, 10616-10931);
//   - the effective moire model of Jung et al. (PRB 89, 205414): on-site H0/Hz harmonics
//     (ham.F90:3437-3544, diago :4696-4716) and the bond term del(1..3) per atom (:12542-12680) or at
//     the bond midpoint (:4822-4883, offdiago :4752-4776), with or without twist;
//   - the two-centre interlayer hopping Vpp_pi/Vpp_sigma (ham.F90:9620-9838, :4094-4110);
//   - Anderson disorder (ham.F90:1237-1248) from host-drawn uniform numbers.
// One thread per atom, FP64; results are in the reference layout hopp(maxNeigh,N).
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include "gbn_internal.cuh"

namespace gbn {

#define GBN_PI 3.14159265358979323846

__device__ double d_diago(double dx, double dy, double C, double phi, double aG)
{
    const double G1 = 4.0 * GBN_PI / sqrt(3.0) / aG;
    const double e1r = cos(G1 * dy), e1i = -sin(G1 * dy);
    const double hh = G1 * dy / 2.0;
    const double k = cos(sqrt(3.0) * G1 * dx / 2.0);
    double sh, ch;
    sincos(hh, &sh, &ch);
    const double sr = e1r + 2.0 * ch * k, si = e1i + 2.0 * sh * k;
    double sp, cp;
    sincos(phi, &sp, &cp);
    return 2.0 * C * (sr * cp - si * sp);
}

__device__ void d_offdiago(double dx, double dy, double C, double phi, double aG, double* re, double* im)
{
    const double G1 = 4.0 * GBN_PI / sqrt(3.0) / aG;
    const double ax = sqrt(3.0) * G1 * dx / 2.0;
    const double p = cos(G1 * dy / 2.0 - phi);
    const double q = sin(G1 * dy / 2.0 - phi - GBN_PI / 6.0);
    double sa, ca;
    sincos(ax, &sa, &ca);
    *re = 2.0 * C * ca * (p + q) + 2.0 * C * sin(G1 * dy + phi - GBN_PI / 6.0);
    *im = 2.0 * C * sa * (p - q);
}

__device__ void d_bond_deltas(int spec, double re, double im, double del[3])
{
    del[0] = 2.0 * re / 3.0;
    const double u = -(re + sqrt(3.0) * im) / 3.0, w = (-re + sqrt(3.0) * im) / 3.0;
    if (spec == 1) { del[1] = u; del[2] = w; }
    else { del[1] = w; del[2] = u; }
}

__device__ void d_moire_disp(const gbn_model& m, double x, double y, double* dx, double* dy)
{
    if (m.moire_twisted) {
        double st, ct;
        sincos(m.twist_rad, &st, &ct);
        *dx = x * ((1.0 + m.eps) * ct - 1.0) - y * (1.0 + m.eps) * st;
        *dy = y * ((1.0 + m.eps) * ct - 1.0) + x * (1.0 + m.eps) * st;
    } else {
        *dx = x * m.eps;
        *dy = y * m.eps;
    }
}

// Displacement of the second moire before its shift and flip (HamOnSiteSecondMoireTerms, ham.F90:3573-3590)
__device__ void d_second_moire_disp(const gbn_model& m, double x, double y, double* dx, double* dy)
{
    const double e = m.eps * m.eps_factor;
    if (m.twisted2) {
        double st, ct;
        sincos(m.twist2_rad, &st, &ct);
        const double ys = m.rotate_first ? y : y - m.shift2 / m.eps;
        *dx = x * ((1.0 + e) * ct - 1.0) - ys * (1.0 + e) * st;
        *dy = ys * ((1.0 + e) * ct - 1.0) + x * (1.0 + e) * st;
    } else {
        *dx = x * e;
        *dy = y * e;
    }
}

// Displacement of the encapsulated bilayer's moire at (x, y) of layer L (HamOnSiteMoireEffectiveBilayer,
// ham.F90:3318-3376, and the bond terms' copy, :12564-12585): layer 1 from the bottom hBN angle plus
// (tauX1, tauY1); the other layer from the top angle plus (tauX2, tauY2), or, without rotate_first, with
// tauY2 / eps taken off y before the rotation.
__device__ void d_bilayer_disp(const gbn_model& m, int L, double x, double y, double* dx, double* dy)
{
    const double e1 = 1.0 + m.eps;
    double st, ct;
    sincos(L == 1 ? m.bl_bottom_rad : m.bl_top_rad, &st, &ct);
    const double A = e1 * ct - 1.0, B = e1 * st;
    if (L == 1 || m.rotate_first) {
        *dx = A * x - (B * y);
        *dy = A * y + (B * x);
        *dx = *dx + (L == 1 ? m.tau[0] : m.tau[2]);
        *dy = *dy + (L == 1 ? m.tau[1] : m.tau[3]);
    } else {
        const double ys = y - m.tau[3] / m.eps;
        *dx = A * x - (B * ys);
        *dy = A * ys + (B * x);
    }
}

// Moire.BLDeactivateUpperLayer / TDBLDeactivateUpperLayers: no moire term on layer 2 / above layer 1
__device__ __forceinline__ bool d_deactivated(const gbn_model& m, int L)
{
    return (L == 2 && m.deact_upper) || (L != 1 && m.deact_uppers);
}

__device__ __forceinline__ void d_moire_terms(const gbn_model& m, double dx, double dy, double* hz, double* hd)
{
    *hz = 0.0;
    *hd = 0.0;
    if (m.moire_onsite == 2) *hd = d_diago(dx, dy, m.C0, m.Phi0, m.aG);
    else if (m.moire_onsite == 3) *hz = d_diago(dx, dy, m.Cz, m.Phiz, m.aG);
    else if (m.moire_onsite == 1) {
        *hz = d_diago(dx, dy, m.Cz, m.Phiz, m.aG);
        *hd = d_diago(dx, dy, m.C0, m.Phi0, m.aG);
    }
}

// HamOnSite in its order: the carbon site energy (:947), Anderson disorder (:1237-1248), the first moire's
// terms (HamOnSiteMoireEffective, :3437-3544), H0Bottom = H0 (:2703, into h0b when given), then the second
// moire's terms on every atom (HamOnSiteSecondMoireTerms, :3546-3642).
__global__ void k_onsite(gbn_model m, int64_t n, const double* rat, const int32_t* species, const int32_t* layer,
                         const double* uniform, double* h0, double* h0b)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double h = m.e0_c;
    if (m.anderson) h = h + (uniform[i] - 0.5) * m.anderson_w;
    const double sgn = (species[i] % 2 == 1) ? -1.0 : 1.0;
    if (m.moire_onsite != 0 && m.encapsulated) {
        // HamOnSiteMoireEffectiveBilayer (ham.F90:3303-3434): no mass factors, H0Bottom not set
        double dx, dy, hz = 0.0, hd = 0.0;
        const int L = layer[i];
        d_bilayer_disp(m, L, rat[3 * i], rat[3 * i + 1], &dx, &dy);
        if (L == 1 || !d_deactivated(m, L)) d_moire_terms(m, dx, dy, &hz, &hd);
        h = h + sgn * hz + hd;
    } else if (m.moire_onsite != 0) {
        double dx, dy, hz, hd;
        d_moire_disp(m, rat[3 * i], rat[3 * i + 1], &dx, &dy);
        dy = dy + m.shift1;
        const int L = layer[i];
        if ((L == 1 && m.sign1 < 0.0) || (L == 2 && m.sign2 < 0.0)) { dx = -dx; dy = -dy; }
        d_moire_terms(m, dx, dy, &hz, &hd);
        if (L == 1) h = h + sgn * hz * m.sign1 + hd;
        else if (L == 2) h = h + sgn * hz * m.sign2 + hd;
        if (h0b) h0b[i] = h;
        if (m.second_moire) {
            d_second_moire_disp(m, rat[3 * i], rat[3 * i + 1], &dx, &dy);
            if (m.rotate_first) {
                dy = dy + m.shift2_y;
                dx = dx + m.shift2_x;
            }
            if (m.sign2 < 0.0) { dx = -dx; dy = -dy; }
            d_moire_terms(m, dx, dy, &hz, &hd);
            h = h + sgn * hz * m.sign2 + hd;
        }
    } else if (h0b) {
        h0b[i] = 0.0;
    }
    h0[i] = h;
}

// del(1..3) of the second moire's bond term of atom i (HamHopSecondMoire, ham.F90:7772-7833): the
// displacement is rotated by TwistAngle2 whether or not Twisted2 is set, flipped before the shift, and Im of
// the amplitude changes sign with the mass factor.
__device__ void d_second_moire_deltas(const gbn_model& m, double x, double y, int spec, double del[3])
{
    const double e = m.eps * m.eps_factor;
    double st, ct, dx, dy;
    sincos(m.twist2_rad, &st, &ct);
    if (m.rotate_first) {
        dx = x * ((1.0 + e) * ct - 1.0) - y * (1.0 + e) * st;
        dy = y * ((1.0 + e) * ct - 1.0) + x * (1.0 + e) * st;
    } else {
        const double ys = y - m.shift2 / m.eps / m.eps_factor;
        dx = x * ((1.0 + e) * ct - 1.0) - ys * (1.0 + m.eps) * st;
        dy = ys * ((1.0 + m.eps) * ct - 1.0) + x * (1.0 + m.eps / m.eps_factor) * st;
    }
    if (m.sign2 < 0.0) { dx = -dx; dy = -dy; }
    if (m.rotate_first) {
        dx = dx + m.shift2_x;
        dy = dy + m.shift2_y;
    }
    double re, im;
    d_offdiago(dx, dy, m.Cab, m.Phiab, m.aG, &re, &im);
    if (m.sign2 < 0.0) im = -im;
    if (spec == 1 || spec == 2) d_bond_deltas(spec, re, im, del);
}

// MoireBondDeltaMidpoint (ham.F90:4822-4883): the bond term of one bond from the moire displacement at its
// midpoint.  First moire: eps, its twist, shift1 before the flip; second moire: eps * eps_factor, TwistAngle2,
// shift2 after the flip, Im flipped and del(2), del(3) swapped with the mass factor's sign.
__device__ double d_mid_delta(double rix, double riy, double bx, double by, int spec, double epsM, double thM,
                              double pre_y, bool flip, double post_x, double post_y, bool flip_imag, bool swap23,
                              double Cab, double Phi, double aG)
{
    if (spec != 1 && spec != 2) return 0.0;
    const double rm0 = rix + 0.5 * bx, rm1 = riy + 0.5 * by;
    double st, ct;
    sincos(thM, &st, &ct);
    double ddx = rm0 * ((1.0 + epsM) * ct - 1.0) - rm1 * (1.0 + epsM) * st;
    double ddy = rm1 * ((1.0 + epsM) * ct - 1.0) + rm0 * (1.0 + epsM) * st;
    ddy = ddy + pre_y;
    if (flip) { ddx = -ddx; ddy = -ddy; }
    ddx = ddx + post_x;
    ddy = ddy + post_y;
    double re, im, del[3];
    d_offdiago(ddx, ddy, Cab, Phi, aG, &re, &im);
    if (flip_imag) im = -im;
    d_bond_deltas(spec, re, im, del);
    if (fabs(bx) < aG / 4.0) return del[0];
    if (bx < 0.0) return swap23 ? del[1] : del[2];
    return swap23 ? del[2] : del[1];
}

__device__ double d_moire_mid_delta(const gbn_model& m, double rix, double riy, double bx, double by, int spec, bool flip)
{
    const double th = m.moire_twisted ? m.twist_rad : 0.0;
    return d_mid_delta(rix, riy, bx, by, spec, m.eps, th, m.shift1, flip, 0.0, 0.0, false, false, m.Cab, m.Phiab, m.aG);
}

__device__ double d_f2g2_shell(const gbn_model& m, double dist)
{
    const double aG = m.aG, aCC = m.aCC;
    if (dist > aCC * 0.9 && dist < aCC * 1.1) return 0.0;
    if (dist > aG * 0.9 && dist < aG * 1.1) return m.tksl[2];
    if (dist > 2.0 * aCC * 0.9 && dist < aCC * 2.0 * 1.1) return m.tksl[3];
    if (dist > 2.0 * aCC * 1.1 && dist < 4.0) return m.tksl[4];
    if (dist > (aCC * 3.0) * 0.9 && dist < (aCC * 3.0) * 1.1) return m.tksl[5];
    if (dist > 2.0 * aG * 0.97 && dist < 2.0 * aG * 1.03) return m.tksl[6];
    const double r7 = sqrt((2.0 * aG) * (2.0 * aG) + aCC * aCC);
    if (dist > r7 * 0.9 && dist < r7 * 1.1) return m.tksl[7];
    return 0.0;
}

// smooth interlayer cutoff factor (1 when the model has none)
__device__ __forceinline__ double smooth_cut(const gbn_model& m, double rho)
{
    if (!(m.inter_smooth_w > 0.0)) return 1.0;
    const double w = m.inter_smooth_w, r0 = m.inter_cut_rho - w;
    if (rho <= r0) return 1.0;
    if (rho >= m.inter_cut_rho) return 0.0;
    return 0.5 * (1.0 + cospi((rho - r0) / w));
}

// Dimer sites of the Bernal interlayer branch (ham.F90:6475-6484): an atom with a neighbour of an adjacent
// layer within 0.2 A in plane; count gets their number.
__global__ void k_dimer(int64_t n, const int32_t* layer, int32_t max_neigh, const int32_t* nneigh,
                        const int32_t* nlist, const double* neighd, int8_t* dimer, unsigned long long* count)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int8_t d = 0;
    for (int j = 0; j < nneigh[i]; ++j) {
        const int64_t e = i * max_neigh + j;
        const int Lj = layer[nlist[e] - 1];
        if (layer[i] != Lj + 1 && layer[i] != Lj - 1) continue;
        const double Dx = neighd[3 * e], Dy = neighd[3 * e + 1];
        if (sqrt(Dx * Dx + Dy * Dy) < 0.2) d = 1;
    }
    dimer[i] = d;
    if (d) atomicAdd(count, 1ULL);
}

__global__ void k_hopping(gbn_model m, int64_t n, const double* rat, const int32_t* species, const int32_t* layer,
                          int32_t max_neigh, const int32_t* nneigh, const int32_t* nlist, const double* neighd,
                          int bernal, const int8_t* dimer, double2* hopp)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double delta = 0.0;
    double del[3] = {0.0, 0.0, 0.0};
    const int Li = layer[i], si = species[i];
    const bool flip = (Li == 1 && m.sign1 < 0.0) || (Li == 2 && m.sign2 < 0.0);
    const double rix = rat[3 * i], riy = rat[3 * i + 1];
    if (m.moire_offdiag) {
        double dx, dy, re = 0.0, im = 0.0;
        if (m.encapsulated) d_bilayer_disp(m, Li, rix, riy, &dx, &dy);
        else d_moire_disp(m, rix, riy, &dx, &dy);
        dy = dy + m.shift1;
        if (flip) { dx = -dx; dy = -dy; }
        if (!d_deactivated(m, Li)) d_offdiago(dx, dy, m.Cab, m.Phiab, m.aG, &re, &im);
        if (si == 1 || si == 2) d_bond_deltas(si, re, im, del);
    }
    // the second moire's bond term (HamHopSecondMoire, ham.F90:7745-7880), a pass of its own in the
    // reference after every other term and before the Peierls phases: subtracted here from the same
    // entry, with its own delta carried over between the bonds of the atom as there
    const bool second = m.second_moire && m.moire_offdiag;
    double delta2 = 0.0;
    double del2[3] = {0.0, 0.0, 0.0};
    if (second) d_second_moire_deltas(m, rix, riy, si, del2);
    const int k = nneigh[i];
    for (int j = 0; j < max_neigh; ++j) {
        const int64_t e = i * max_neigh + j;
        double hr = 0.0;
        if (j < k) {
            const int64_t jj = nlist[e] - 1;
            const double Dx = neighd[3 * e], Dy = neighd[3 * e + 1], Dz = neighd[3 * e + 2];
            const int Lj = layer[jj];
            if (Li == Lj) {
                const double d = sqrt(Dx * Dx + Dy * Dy);
                for (int lv = 0; lv < m.tbnn; ++lv) {
                    if (d < m.nradii[lv]) {
                        if (d < 1.7) {
                            if (fabs(Dx) < m.aG / 4.0) delta = del[0];
                            else if (Dx < -m.aG / 4.0) delta = del[2];
                            else if (Dx > m.aG / 4.0) delta = del[1];
                            if (m.moire_mid) delta = d_moire_mid_delta(m, rix, riy, Dx, Dy, si, flip);
                        }
                        if (m.intralayer == 1) hr = hr + d_f2g2_shell(m, d);
                        if (d > 1.5) delta = 0.0;
                        hr = hr + (m.gn_cc[lv] - delta);
                        if (second) {
                            if (fabs(Dx) < 0.01) delta2 = del2[0];
                            else if (Dx < -0.02) delta2 = (m.sign2 < 0.0) ? del2[1] : del2[2];
                            else if (Dx > 0.02) delta2 = (m.sign2 < 0.0) ? del2[2] : del2[1];
                            if (m.moire_mid) {
                                const bool neg = m.sign2 < 0.0;
                                delta2 = d_mid_delta(rix, riy, Dx, Dy, si, m.eps * m.eps_factor, m.twist2_rad, 0.0, neg,
                                                     m.shift2_x, m.shift2_y, neg, neg, m.Cab, m.Phiab, m.aG);
                            }
                            if (d > 1.7) delta2 = 0.0;
                            hr = hr - delta2;
                        }
                        break;
                    }
                }
            } else if (Li == Lj + 1 || Li == Lj - 1) {
                if (m.encapsulated) {
                    // the encapsulated bilayer's interlayer branch (ham.F90:6721-6745)
                    if (bernal == 2) {   // HamHopInterlayerBernalF2G2 (ham.F90:12800-12827)
                        const bool mixed = dimer[i] != dimer[jj];
                        const double dxy = sqrt(Dx * Dx + Dy * Dy), aCC = m.aCC, aG = m.aG;
                        if (dxy < 0.2) hr = hr + m.tbl[4];
                        else if (dxy > aCC * 0.9 && dxy < aCC * 1.1) hr = hr + (mixed ? m.tbl[0] : m.tbl[2]);
                        else if (dxy > aG * 0.9 && dxy < aG * 1.1) hr = hr + m.tbl[5];
                        else if (dxy > aCC * 2.0 * 0.9 && dxy < aCC * 2.0 * 1.1) hr = hr + (mixed ? m.tbl[1] : m.tbl[3]);
                        else if (dxy > (aCC * 3.0) * 0.9 && dxy < (aCC * 3.0) * 1.1 && !mixed) hr = hr + m.tbl[6];
                    } else if (fabs(Dx) < 0.01 && fabs(Dy) < 0.01) {
                        hr = hr - m.tbl[2];
                    }
                } else if (m.interlayer == 1) {
                    const double dist = sqrt(Dx * Dx + Dy * Dy + Dz * Dz);
                    const double sr = m.koshino_sr ? exp((fabs(Dz) - 3.25) / 1.34) : 1.0;
                    const double vsig = m.vppsigma0 * exp(-(dist - m.d_interlayer) / m.bl_delta) * sr;
                    const double vpi = m.vpppi0 * exp(-(dist - m.aCC) / m.bl_delta) * sr;
                    const double q = Dz / dist;
                    hr = hr + (vpi * (1.0 - q * q) + vsig * (q * q)) * smooth_cut(m, sqrt(Dx * Dx + Dy * Dy));
                    if (m.renormalize_coupling) hr = m.coupling_factor * hr;
                } else {
                    const double d = sqrt(Dx * Dx + Dy * Dy);
                    hr = hr + m.g_intlay * exp(-d / m.d_interlayer);
                }
            }
        }
        hopp[e] = make_double2(hr, 0.0);
    }
}

__global__ void k_peierls(int64_t n, const double* rat, double u0, double u1, double u3, double u4, int32_t max_neigh,
                          const int32_t* nneigh, const int32_t* nlist, const int32_t* ncell, double flux, double mq,
                          double2* hopp)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double rix = rat[3 * i], riy = rat[3 * i + 1];
    for (int j = 0; j < nneigh[i]; ++j) {
        const int64_t e = i * max_neigh + j;
        const int64_t jj = nlist[e] - 1;
        const double rjx = rat[3 * jj], rjy = rat[3 * jj + 1];
        const int n1 = ncell[3 * e], n2 = ncell[3 * e + 1];
        const double v1x = rix + rjx, v1y = riy + rjy;
        const double v2x = (double)n1 * u0 + (double)n2 * u3, v2y = (double)n1 * u1 + (double)n2 * u4;
        const double c3 = v1x * v2y - v1y * v2x;
        const double r3 = rix * rjy - riy * rjx;
        double ph = flux * (r3 + c3) / 1.0e20;
        if (n1 != 0 && n2 != 0) ph = ph + GBN_PI * mq * (double)n1 * (double)n2;
        double s, co;
        sincos(ph, &s, &co);
        const double2 h = hopp[e];
        hopp[e] = make_double2(h.x * co - h.y * s, h.x * s + h.y * co);
    }
}

// The phase of k_peierls per flux quantum as a fraction of a turn, in 64-bit fixed point: for m quanta
// the phase is m * pi [(r_i x r_j + (r_i + r_j) x T) / A + n1 n2] (flux = m pi 1e20 / A), i.e. m turns
// times (r_i x r_j + (r_i + r_j) x T) / (2 A) + n1 n2 / 2, taken modulo one turn.
__global__ void k_peierls_turns(int64_t n, const double* rat, double u0, double u1, double u3, double u4,
                                double area, int32_t max_neigh, const int32_t* nneigh, const int32_t* nlist,
                                const int32_t* ncell, uint64_t* tau)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double rix = rat[3 * i], riy = rat[3 * i + 1];
    for (int j = 0; j < nneigh[i]; ++j) {
        const int64_t e = i * max_neigh + j;
        const int64_t jj = nlist[e] - 1;
        const double rjx = rat[3 * jj], rjy = rat[3 * jj + 1];
        const int n1 = ncell[3 * e], n2 = ncell[3 * e + 1];
        const double v1x = rix + rjx, v1y = riy + rjy;
        const double v2x = (double)n1 * u0 + (double)n2 * u3, v2y = (double)n1 * u1 + (double)n2 * u4;
        const double c3 = v1x * v2y - v1y * v2x;
        const double r3 = rix * rjy - riy * rjx;
        double t = (r3 + c3) / (2.0 * area);
        t -= floor(t);
        if (n1 != 0 && n2 != 0 && (((long long)n1 * (long long)n2) & 1LL)) t += 0.5;
        if (t >= 1.0) t -= 1.0;
        // t * 2^64 in [0, 2^64): the high and the low 32 bits separately (exact for t's 53 bits)
        const double hi = floor(t * 4294967296.0);
        const double lo = (t * 4294967296.0 - hi) * 4294967296.0;
        uint64_t q = ((uint64_t)hi << 32) + (uint64_t)llrint(lo);
        tau[e] = q;
    }
}

int peierls_turns(gbn_ctx* c)
{
    if (!c->rat_hop.p || !c->ncell.p) return fail(c, GBN_ERR_STATE, "batched fields need the device geometry and neighbour search");
    const double* u = c->ucell;
    const double area = fabs(u[0] * u[4] - u[1] * u[3]);
    GBN_CK(c, c->ptau.ensure(sizeof(uint64_t) * (size_t)c->n * c->max_neigh));
    GBN_CK(c, cudaMemsetAsync(c->ptau.p, 0, sizeof(uint64_t) * (size_t)c->n * c->max_neigh, c->stream));
    const unsigned grd = (unsigned)((c->n + 127) / 128);
    k_peierls_turns<<<grd, 128, 0, c->stream>>>(c->n, c->rat_hop.as<double>(), u[0], u[1], u[3], u[4], area,
                                                c->max_neigh, c->nneigh.as<int32_t>(), c->nlist.as<int32_t>(),
                                                c->ncell.as<int32_t>(), c->ptau.as<uint64_t>());
    GBN_CK_LAUNCH(c);
    return GBN_OK;
}

int assemble(gbn_ctx* c, const gbn_model* m, const double* d_rat_on, const double* d_rat_hop, const double* d_uniform)
{
    const int64_t n = c->n;
    GBN_CK(c, c->h0.ensure(sizeof(double) * n));
    GBN_CK(c, c->hopp.ensure(sizeof(double2) * (size_t)n * c->max_neigh));
    const unsigned grd = (unsigned)((n + 127) / 128);
    // H0Bottom is kept only for the moire branch (elsewhere it is 0 and nothing is stored)
    double* h0b = nullptr;
    if (m->moire_onsite != 0 && !m->encapsulated) {
        GBN_CK(c, c->h0_bottom.ensure(sizeof(double) * n));
        h0b = c->h0_bottom.as<double>();
    }
    k_onsite<<<grd, 128, 0, c->stream>>>(*m, n, d_rat_on, c->species.as<int32_t>(), c->layer.as<int32_t>(), d_uniform,
                                         c->h0.as<double>(), h0b);
    GBN_CK_LAUNCH(c);
    // the Bernal interlayer set needs an AB-stacked cell: half of the atoms dimer sites (to 10 %), else the
    // vertical pairs only, as the reference decides (ham.F90:6473-6495)
    int bernal = m->encapsulated ? m->bernal : 0;
    const int8_t* dimer = nullptr;
    if (bernal == 2) {
        GBN_CK(c, c->dimer.ensure((size_t)n + sizeof(unsigned long long) + 8));
        int8_t* dm = c->dimer.as<int8_t>();
        unsigned long long* cnt = reinterpret_cast<unsigned long long*>(dm + ((n + 7) / 8) * 8);
        GBN_CK(c, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), c->stream));
        k_dimer<<<grd, 128, 0, c->stream>>>(n, c->layer.as<int32_t>(), c->max_neigh, c->nneigh.as<int32_t>(),
                                            c->nlist.as<int32_t>(), c->neighd.as<double>(), dm, cnt);
        GBN_CK_LAUNCH(c);
        unsigned long long h_cnt = 0;
        GBN_CK(c, cudaMemcpyAsync(&h_cnt, cnt, sizeof h_cnt, cudaMemcpyDeviceToHost, c->stream));
        GBN_CK(c, cudaStreamSynchronize(c->stream));
        const long long diff = 2LL * (long long)h_cnt - (long long)n;
        if ((diff < 0 ? -diff : diff) > (long long)(n / 10)) bernal = 1;
        dimer = dm;
    }
    c->bernal_used = bernal;
    k_hopping<<<grd, 128, 0, c->stream>>>(*m, n, d_rat_hop, c->species.as<int32_t>(), c->layer.as<int32_t>(),
                                          c->max_neigh, c->nneigh.as<int32_t>(), c->nlist.as<int32_t>(),
                                          c->neighd.as<double>(), bernal, dimer, c->hopp.as<double2>());
    GBN_CK_LAUNCH(c);
    c->have_ham = true;
    c->ham_complex = false;
    c->has_field = false;
    c->ell.valid = false;
    c->have_bottom = h0b != nullptr;
    c->have_top = h0b != nullptr && m->second_moire != 0;
    return GBN_OK;
}

int peierls(gbn_ctx* c, double flux)
{
    const double* u = c->ucell;
    const double area = fabs(u[0] * u[4] - u[1] * u[3]);
    const double fq = flux * area / (GBN_PI * 1.0e20);
    const double mq = (double)llround(fq);
    if (fabs(fq - mq) > 1.0e-6)
        return fail(c, GBN_ERR_NUMERIC, "the number of flux quanta through the cell is not an integer");
    const unsigned grd = (unsigned)((c->n + 127) / 128);
    k_peierls<<<grd, 128, 0, c->stream>>>(c->n, c->rat_hop.as<double>(), u[0], u[1], u[3], u[4], c->max_neigh,
                                          c->nneigh.as<int32_t>(), c->nlist.as<int32_t>(), c->ncell.as<int32_t>(), flux,
                                          mq, c->hopp.as<double2>());
    GBN_CK_LAUNCH(c);
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    c->ham_complex = true;
    c->has_field = true;
    c->ell.valid = false;
    return GBN_OK;
}

// HamHaldaneChirality (ham.F90:13063-13100): +1 if the path i -> k -> j through a common nearest neighbour
// turns clockwise, -1 if anticlockwise, 0 if no such neighbour exists.
__device__ int haldane_chirality(const int32_t* layer, int32_t mn, const int32_t* nneigh, const int32_t* nlist,
                                 const double* neighd, double aG, int64_t i, int jn)
{
    const double* dij = neighd + 3 * (i * mn + jn);
    const double acc = aG / sqrt(3.0);
    const int32_t target = nlist[i * mn + jn];
    for (int k1 = 0; k1 < nneigh[i]; ++k1) {
        const int64_t k = nlist[i * mn + k1] - 1;
        if (layer[k] != layer[i]) continue;
        const double* d1 = neighd + 3 * (i * mn + k1);
        if (fabs(sqrt(d1[0] * d1[0] + d1[1] * d1[1]) - acc) > 0.1) continue;
        for (int k2 = 0; k2 < nneigh[k]; ++k2) {
            if (nlist[k * mn + k2] != target) continue;
            const double* d2 = neighd + 3 * (k * mn + k2);
            if (fabs(sqrt(d2[0] * d2[0] + d2[1] * d2[1]) - acc) > 0.1) continue;
            const double ex = d1[0] + d2[0] - dij[0], ey = d1[1] + d2[1] - dij[1];
            if (sqrt(ex * ex + ey * ey) > 0.1) continue;
            const double cr = d1[0] * d2[1] - d1[1] * d2[0];
            return cr < 0.0 ? 1 : -1;
        }
    }
    return 0;
}

// HamHopHaldane (ham.F90:7043-7142): second-neighbour bonds (|d - aG| < 0.1 Ang, same layer, graphene
// species) get + t2 exp(i nu phase), or with the paper orientation are multiplied by exp(i nu phase).
__global__ void k_haldane(int64_t n, const int32_t* species, const int32_t* layer, int32_t mn, const int32_t* nneigh,
                          const int32_t* nlist, const double* neighd, double aG, double t2, double phase, int paper,
                          uint32_t mask, double2* hopp, unsigned long long* missing)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (mask != 0u && (layer[i] < 1 || layer[i] > 32 || !((mask >> (layer[i] - 1)) & 1u))) return;
    for (int j = 0; j < nneigh[i]; ++j) {
        const int64_t e = i * mn + j;
        const int64_t jj = nlist[e] - 1;
        if (layer[jj] != layer[i]) continue;
        const double dx = neighd[3 * e], dy = neighd[3 * e + 1];
        const double d = sqrt(dx * dx + dy * dy);
        if (!((d - 0.1) < aG && (d + 0.1) > aG && species[i] <= 2)) continue;
        const int nu = haldane_chirality(layer, mn, nneigh, nlist, neighd, aG, i, j);
        if (nu == 0) {
            atomicAdd(missing, 1ull);
            continue;
        }
        double sn, cs;
        sincos(nu * phase, &sn, &cs);
        const double2 h = hopp[e];
        hopp[e] = paper ? make_double2(h.x * cs - h.y * sn, h.x * sn + h.y * cs)
                        : make_double2(h.x + t2 * cs, h.y + t2 * sn);
    }
}

int haldane(gbn_ctx* c, double aG, double t2, double phase, int32_t paper, uint32_t layer_mask)
{
    if (!c->have_ham || !c->have_neighd || !c->have_geometry)
        return fail(c, GBN_ERR_STATE, "the Haldane term needs the geometry, NeighD and a Hamiltonian");
    DevBuf cnt;
    GBN_CK(c, cnt.ensure(sizeof(unsigned long long)));
    GBN_CK(c, cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long), c->stream));
    const unsigned grd = (unsigned)((c->n + 127) / 128);
    k_haldane<<<grd, 128, 0, c->stream>>>(c->n, c->species.as<int32_t>(), c->layer.as<int32_t>(), c->max_neigh,
                                          c->nneigh.as<int32_t>(), c->nlist.as<int32_t>(), c->neighd.as<double>(), aG,
                                          t2, phase, paper, layer_mask, c->hopp.as<double2>(),
                                          cnt.as<unsigned long long>());
    GBN_CK_LAUNCH(c);
    unsigned long long missing = 0;
    GBN_CK(c, cudaMemcpyAsync(&missing, cnt.p, sizeof missing, cudaMemcpyDeviceToHost, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    c->ham_complex = true;
    c->has_field = true;   // not a field-free Hamiltonian any more (batched fields would drop the term)
    c->ell.valid = false;
    if (missing)
        return fail(c, GBN_ERR_NUMERIC, std::to_string(missing) + " second-neighbour bonds have no common nearest "
                                        "neighbour: their chirality is undefined (not a honeycomb lattice?)");
    return GBN_OK;
}

// HamCheckFinite (ham.F90:4432-4477) and the pair scan of HamCheckHermiticity (ham.F90:4491-4571), one
// thread per atom: cnt[0] non-finite hoppings, [1] non-finite on-site energies, [2] first offending
// atom (0-based, via min), [3] entries without a reverse entry (same pair, opposite lattice translation),
// [4] pairs compared, [5] the largest |hopp(j,i) - conj(hopp(j2,m))| as the bits of a non-negative double.
__global__ void k_check(int64_t n, int32_t mn, const int32_t* nneigh, const int32_t* nlist, const int32_t* ncell,
                        const double2* hopp, const double* h0, unsigned long long* cnt)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned long long nhop = 0, missing = 0, pairs = 0;
    double mx = 0.0;
    bool bad = !isfinite(h0[i]);
    if (bad) atomicAdd(&cnt[1], 1ull);
    for (int j = 0; j < nneigh[i]; ++j) {
        const int64_t e = i * mn + j;
        const double2 a = hopp[e];
        if (!(isfinite(a.x) && isfinite(a.y))) {
            ++nhop;
            bad = true;
        }
        const int64_t m = nlist[e] - 1;
        if (m < i) continue;
        int j2 = 0;
        for (; j2 < nneigh[m]; ++j2) {
            const int64_t e2 = m * mn + j2;
            if (nlist[e2] - 1 == i && ncell[3 * e2] == -ncell[3 * e] && ncell[3 * e2 + 1] == -ncell[3 * e + 1] &&
                ncell[3 * e2 + 2] == -ncell[3 * e + 2])
                break;
        }
        if (j2 >= nneigh[m]) {
            ++missing;
            continue;
        }
        if (m == i && j2 <= j) continue;
        ++pairs;
        const double2 b = hopp[m * mn + j2];
        const double asym = hypot(a.x - b.x, a.y + b.y);
        mx = asym > mx ? asym : mx;   // a NaN asymmetry is counted by the finiteness check
    }
    if (nhop) atomicAdd(&cnt[0], nhop);
    if (missing) atomicAdd(&cnt[3], missing);
    if (pairs) atomicAdd(&cnt[4], pairs);
    if (bad) atomicMin(&cnt[2], (unsigned long long)i);
    if (mx > 0.0) atomicMax(&cnt[5], (unsigned long long)__double_as_longlong(mx));
}

int check_hamiltonian(gbn_ctx* c, int64_t* out, double* max_asym)
{
    if (!c->have_ham || !c->ncell.p) return fail(c, GBN_ERR_STATE, "the checks need a Hamiltonian and the neighbour images");
    DevBuf cnt;
    GBN_CK(c, cnt.ensure(sizeof(unsigned long long) * 6));
    unsigned long long init[6] = {0ull, 0ull, ~0ull, 0ull, 0ull, 0ull};
    GBN_CK(c, cudaMemcpyAsync(cnt.p, init, sizeof init, cudaMemcpyHostToDevice, c->stream));
    const unsigned grd = (unsigned)((c->n + 127) / 128);
    k_check<<<grd, 128, 0, c->stream>>>(c->n, c->max_neigh, c->nneigh.as<int32_t>(), c->nlist.as<int32_t>(),
                                        c->ncell.as<int32_t>(), c->hopp.as<double2>(), c->h0.as<double>(),
                                        cnt.as<unsigned long long>());
    GBN_CK_LAUNCH(c);
    unsigned long long h[6];
    GBN_CK(c, cudaMemcpyAsync(h, cnt.p, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    out[0] = (int64_t)h[0];
    out[1] = (int64_t)h[1];
    out[2] = h[2] == ~0ull ? 0 : (int64_t)h[2] + 1;
    out[3] = (int64_t)h[3];
    out[4] = (int64_t)h[4];
    double mx;
    memcpy(&mx, &h[5], sizeof mx);
    *max_asym = mx;
    return GBN_OK;
}

}  // namespace gbn
