/*
 * CPU oracle for the GRABNES recursion hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference algorithms (gjung-group/grabnes,
 * Fortran 90) that the CUDA library is checked against.  Only the tests, the
 * smoke check and the CPU-baseline leg of bench.py may load it; the product
 * (grabnes_b200/) never links or calls it.
 *
 * Every function cites the reference routine (path:line inside the reference
 * project) whose floating-point operation order it follows.  Arrays use the
 * reference's memory layout: Rat(3,N), NList(maxNeigh,N), NeighD(3,maxNeigh,N),
 * neighCell(3,maxNeigh,N), hopp(maxNeigh,N) (complex, interleaved re/im), all
 * column-major, i.e. C arrays indexed [i][j][k]; neighbour indices are 1-based.
 */
#ifndef GRABNES_ORACLE_H
#define GRABNES_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- RNG ---- */
/* GNU Fortran (libgfortran >= 8) intrinsic random_seed / random_number:
 * xoshiro256** state, PUT copies the 8 int32 seed words in reverse order and
 * XORs the state with a fixed key; random_number(real(8)) keeps the top 53
 * bits.  Called at lanczosKuboCode/Src/kubo.F90:46-64, random.F90:31-52. */
typedef struct { uint64_t s[4]; } orc_rng;
void   orc_rng_put(orc_rng* r, int32_t seed_value);
double orc_rng_r8(orc_rng* r);
/* n draws after random_seed(PUT=[seed]*8) */
void   orc_rng_fill(int32_t seed_value, int64_t n, double* out);

/* ----------------------------------------------------------- geometry ---- */
enum { ORC_GRAPHENE = 0, ORC_TBG_MOIRE_CELL = 1 };
typedef struct {
    int32_t kind;          /* ORC_GRAPHENE | ORC_TBG_MOIRE_CELL           */
    int32_t cell_size;     /* Structure.CellSize                          */
    int32_t super_cell;    /* Structure.SuperCell                         */
    int32_t m[4];          /* Structure.MoireCellParameters               */
    double  aG;            /* Structure.LatticeParameter [Ang]            */
    double  height;        /* Structure.CellHeight [Ang]                  */
    double  d_interlayer;  /* Structure.InterlayerDistance [Ang]          */
    /* Structure.TwistedBLAddShift of the moire cell's second layer (atoms.F90:352-366): 0 none, 1 the
     * Bernal offset (Structure.BernalShift), 2 the bridge offset (Structure.BridgeShift); plus
     * Structure.BilayerShiftFactor [Ang] along a1+a2 (AtomsShiftFrac, atoms.F90:1490-1504) */
    int32_t add_shift;
    double  shift_factor;
} orc_geom_params;

int64_t orc_geom_natoms(const orc_geom_params* p);
/* ucell: 9 doubles, column c at ucell[3c..3c+2]; Rat: Cartesian [N][3]. */
int orc_geom_build(const orc_geom_params* p, double* ucell, double* Rat,
                   int32_t* species, int32_t* layer, double* twist_rad);
/* AtomsSetFrac followed by AtomsSetCart (atoms.F90:1768-1830) */
void orc_geom_roundtrip(int64_t n, const double* ucell, double* Rat);
double orc_cell_area(const double* ucell);

/* --------------------------------------------------- neighbour search ---- */
typedef struct orc_nbr orc_nbr;
/* NeighSearchLayered, neigh.F90:117-316 (periodicZ=.false.) */
orc_nbr* orc_neigh_search(int64_t n, const double* Rat, const double* ucell,
                          double cut2intra, double cut2inter, int32_t second_layer);
int32_t orc_nbr_max(const orc_nbr* b);
int64_t orc_nbr_total(const orc_nbr* b);
void    orc_nbr_copy(const orc_nbr* b, int32_t* Nneigh, int32_t* NList,
                     double* NeighD, int32_t* neighCell);
void    orc_nbr_free(orc_nbr* b);

/* -------------------------------------------------------- Hamiltonian ---- */
enum { ORC_INTRA_DEFAULT = 0, ORC_INTRA_F2G2_SL = 1 };
enum { ORC_INTER_NONE = 0, ORC_INTER_TWO_CENTRE = 1 };
enum { ORC_ONSITE_NONE = 0, ORC_ONSITE_H0_AND_HZ = 1, ORC_ONSITE_ONLY_H0 = 2,
       ORC_ONSITE_ONLY_HZ = 3, ORC_ONSITE_NO_H0_AND_HZ = 4 };
typedef struct {
    double  aG;
    int32_t tbnn;              /* TB.NeighLevels                                   */
    double  gn_cc[8];          /* gn(C,C,shell)/g0 for carbon pairs                */
    double  nradii[8];         /* Nradii(shell,1) [Ang]                            */
    int32_t intralayer;        /* ORC_INTRA_*                                      */
    double  tksl[8];           /* F2G2 single layer t2..t8 (index 2..7 used) /g0   */
    /* effective moire model (Jung et al. PRB 89 205414) */
    int32_t moire_offdiag;     /* Moire.OffDiag                                    */
    int32_t moire_mid;         /* Moire.OffDiagMidpoint                            */
    int32_t moire_twisted;     /* Moire.Twisted                                    */
    int32_t moire_onsite;      /* ORC_ONSITE_*                                     */
    double  eps;               /* Moire.LatticePercent                             */
    double  twist_rad;         /* Moire.TwistAngle [rad]                           */
    double  shift1;            /* Moire.LayerShift1                                */
    double  sign1, sign2;      /* Moire.FirstMoireMassFactor / SecondMoireMassFactor */
    double  C0, Cz, Cab;       /* /g0                                              */
    double  Phi0, Phiz, Phiab;
    /* interlayer */
    int32_t interlayer;        /* ORC_INTER_*                                      */
    double  vpppi0, vppsigma0; /* already /g0, sign convention of ham.F90:5931-5936 */
    double  bl_delta, d_interlayer, aCC;
    double  g_intlay;          /* TB.InterLayerHopping/g0 (ORC_INTER_NONE)         */
    /* disorder */
    int32_t anderson;          /* Disorder.Anderson                                */
    double  anderson_w;        /* /g0                                              */
    int32_t seed;              /* Kubo.SeedValue                                   */
    double  e0_c;              /* TB.OnSiteC/g0                                    */
    /* Interlayer.KoshinoSR (ham.F90:9817-9823) and RenormalizeCoupling (ham.F90:6807-6838) */
    int32_t koshino_sr;
    int32_t renormalize_coupling;
    double  coupling_factor;
    /* Smooth interlayer cutoff of the differentiable model (no counterpart in the reference, whose cutoff
     * is hard, neigh.F90:269-276): the two-centre term times s(rho) of the in-plane distance rho,
     * s = 1 up to rho_c - w, (1 + cos(pi (rho - rho_c + w) / w)) / 2 up to rho_c, 0 beyond; w = 0: none. */
    double  inter_smooth_w;
    double  inter_cut_rho;
    /* Moire.AddSecondMoire (HamOnSiteSecondMoireTerms, ham.F90:3546-3642; HamHopSecondMoire,
     * ham.F90:7745-7880, with Moire.OffDiag): a second moire pattern on the same graphene */
    int32_t second_moire;
    double  eps_factor;        /* Moire.LatticePercentFactor                       */
    int32_t twisted2;          /* Moire.Twisted2                                   */
    double  twist2_rad;        /* Moire.TwistAngle2 [rad]                          */
    int32_t rotate_first;      /* Moire.SecondMoireRotateFirst                     */
    double  shift2;            /* Moire.LayerShift2 [Ang]                          */
    double  shift2_x, shift2_y; /* shift2 (cos, sin) phi2M, ham.F90:2688-2690      */
    /* MoireEncapsulatedBilayerBasedOnMoireCell: HamOnSiteMoireEffectiveBilayer (ham.F90:3303-3434), its bond
     * displacement (ham.F90:12561-12590) and its interlayer branch (ham.F90:6455-6500, 6721-6745, 12800-12827) */
    int32_t encapsulated;
    double  bl_bottom_rad, bl_top_rad; /* Moire.BilayerBottomAngle / TopAngle [rad]       */
    double  tau[4];            /* tauX1, tauY1, tauX2, tauY2 (moireBLShift) [Ang]      */
    int32_t deact_upper;       /* Moire.BLDeactivateUpperLayer                     */
    int32_t deact_uppers;      /* Moire.TDBLDeactivateUpperLayers                  */
    int32_t bernal;            /* 1 vertical pairs (-tAB1), 2 bilayer F2G2 set      */
    double  tbl[7];            /* tAA1 tAA2 tAB1 tAB2 tBA0 tBA2 tBA5 (-t/g0)          */
} orc_model;

void orc_onsite(const orc_model* m, int64_t n, const double* Rat,
                const int32_t* species, const int32_t* layer, double* H0);
/* orc_onsite, and H0Bottom (ham.F90:2703): the on-site energies after the first moire's terms when the
 * moire branch runs, else 0.  H0Top = H0 - H0Bottom when the second moire runs (ham.F90:3639), else 0. */
void orc_onsite_layers(const orc_model* m, int64_t n, const double* Rat, const int32_t* species,
                       const int32_t* layer, double* H0, double* H0Bottom);
int64_t orc_bernal_dimers(int64_t n, const int32_t* layer, int32_t maxNeigh, const int32_t* Nneigh,
                          const int32_t* NList, const double* NeighD, int8_t* dimer);
void orc_hopping(const orc_model* m, int64_t n, const double* Rat,
                 const int32_t* species, const int32_t* layer,
                 int32_t maxNeigh, const int32_t* Nneigh, const int32_t* NList,
                 const double* NeighD, double* hopp);
/* HamHopHaldane (ham.F90:7043-7142) with HamHaldaneChirality (ham.F90:13063-13100), after the
 * Peierls phases: second-neighbour bonds within a layer get + t2 exp(i nu phase) (paper: times
 * exp(i nu phase)); layer_mask bit l-1 enables layer l (0 = every layer).  Returns the number of
 * bonds without a common nearest neighbour (the reference stops on any). */
int64_t orc_haldane(int64_t n, const int32_t* species, const int32_t* layer, int32_t maxNeigh,
                    const int32_t* Nneigh, const int32_t* NList, const double* NeighD, double aG, double t2,
                    double phase, int32_t paper, uint32_t layer_mask, double* hopp);
/* HamCheckFinite (ham.F90:4432-4477) and the pair scan of HamCheckHermiticity (ham.F90:4491-4571):
 * out[0] non-finite hoppings, out[1] non-finite on-site energies, out[2] first offending atom (1-based,
 * 0 if none), out[3] entries without a reverse entry, out[4] pairs compared; *max_asym the largest
 * |hopp(j,i) - conj(hopp(j2,m))| (g0 units). */
void orc_check_hamiltonian(int64_t n, int32_t maxNeigh, const int32_t* Nneigh, const int32_t* NList,
                           const int32_t* neighCell, const double* hopp, const double* H0, int64_t* out,
                           double* max_asym);
void orc_peierls(int64_t n, const double* Rat, const double* ucell,
                 int32_t maxNeigh, const int32_t* Nneigh, const int32_t* NList,
                 const int32_t* neighCell, double flux, double* hopp);

/* ------------------------------------------------------------ solver ---- */
/* KuboInitWF, kubo.F90:24-85 */
void orc_init_wf(int64_t n, int32_t seed, double* psi);
/* KuboRecursion, kubosubs.F90:26-138.  psi is not modified. */
void orc_recursion(int64_t n, int32_t maxNeigh, const int32_t* Nneigh,
                   const int32_t* NList, const double* hopp, const double* H0,
                   const double* psi, int32_t nrecurs, double* a, double* b,
                   int32_t nthreads);
/* KuboFrac, kubosubs.F90:222-288 -> energies[nEn+1], dos[nEn+1] */
void orc_frac(const double* a, const double* b, int32_t nrecurs, double norm,
              double eps, int32_t nEn, double Emin, double Emax,
              double* energy, double* dos);
/* KuboInterval, kubosubs.F90:290-350 (eigenvalues by QL, in place of DSTERF) */
int  orc_interval(const double* a, const double* b, int32_t nrecurs, double* ac, double* bc);
/* KuboCn, kubosubs.F90:352-433 (TQL2 :725-868) -> c[2*nPol] */
int  orc_cheb_coef(double dT, double ac, double bc, int32_t nPol, double* c);
/* KuboChebyshevEvolve, kubosubs.F90:557-619 */
void orc_cheb_evolve(int64_t n, int32_t maxNeigh, const int32_t* Nneigh,
                     const int32_t* NList, const double* hopp, const double* H0,
                     const double* c, int32_t nPol, double ac, double bc, double* Z);
/* KuboEvol, kubosubs.F90:438-553; dir 1 = x, 2 = y */
void orc_evol(int64_t n, int32_t maxNeigh, const int32_t* Nneigh,
              const int32_t* NList, const double* NeighD, const double* hopp,
              const double* H0, const double* c, int32_t nPol, double ac,
              double bc, int32_t dir, double* psi, double* zupsi);

#ifdef __cplusplus
}
#endif
#endif
