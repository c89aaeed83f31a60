/*
 * grabnes_gpu.h -- C ABI of the B200 (sm_100a) library for the large-cell
 * recursion hot path of GRABNES: neighbour search, Hamiltonian assembly,
 * Lanczos recursion, continued-fraction DOS and Chebyshev time evolution.
 *
 * Conventions of the reference solver (gjung-group/grabnes, Fortran) are kept
 * at this boundary so that a Fortran host can bind every entry point with
 * iso_c_binding and pass its module arrays unchanged:
 *   - arrays are the Fortran arrays in memory order: Rat(3,N) -> rat[3*i+k],
 *     NList(maxNeigh,N) -> nlist[maxNeigh*i+j] (1-based atom numbers),
 *     NeighD(3,maxNeigh,N), neighCell(3,maxNeigh,N), hopp(maxNeigh,N) complex
 *     (interleaved re, im), H0(N); energies in units of g0 (TB.Hopping);
 *   - hopp stores MINUS the hopping: (H x)_i = H0_i x_i - sum_j hopp(j,i) x(NList(j,i)).
 * Every function returns GBN_OK (0) or a negative GBN_ERR_* code; the text of
 * the last error is gbn_last_error().  Nothing in the library aborts, traps or
 * exits.  A context owns device memory and one CUDA stream; calls on one
 * context must not overlap (one context per host thread).  Host buffers are
 * owned by the caller; the library copies them in and writes results into
 * caller buffers.
 */
#ifndef GRABNES_GPU_H
#define GRABNES_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GBN_OK 0
#define GBN_ERR_ARG (-1)     /* invalid argument (the message names it)            */
#define GBN_ERR_CUDA (-2)    /* CUDA runtime error                                  */
#define GBN_ERR_STATE (-3)   /* call out of order (e.g. no Hamiltonian loaded)      */
#define GBN_ERR_NUMERIC (-4) /* non-finite or non-positive b_n, non-integer flux ... */
#define GBN_ERR_ALLOC (-5)   /* device or host allocation failed                    */
#define GBN_ERR_TIMEOUT (-6) /* a bounded device wait ran out                       */

#define GBN_FP64 0  /* complex128 vectors and hoppings, FP64 everything              */
#define GBN_MIXED 1 /* complex64 vectors, FP32 hoppings, FP64 a_n/b_n reductions      */

typedef struct gbn_ctx gbn_ctx;

/* Model of the hot path (units: g0 unless stated; see grabnes_b200/model.py for
 * the mapping from Gendata.in keys).  Mirrors the variables the reference's
 * HamOnSite / HamHopping read (lanczosKuboCode/Src/ham.F90:756-4016, 5373-12829). */
typedef struct gbn_model {
    double  aG;            /* Structure.LatticeParameter [Ang]                        */
    int32_t tbnn;          /* TB.NeighLevels (1..8)                                   */
    double  gn_cc[8];      /* gn(C,C,shell)/g0                                        */
    double  nradii[8];     /* Nradii(shell,1) [Ang]                                   */
    int32_t intralayer;    /* 0 HamHopIntralayerDefault, 1 F2G2 single layer          */
    double  tksl[8];       /* F2G2 shell terms t2..t7 at index 2..7 (/g0)             */
    int32_t moire_offdiag; /* Moire.OffDiag                                           */
    int32_t moire_mid;     /* Moire.OffDiagMidpoint                                   */
    int32_t moire_twisted; /* Moire.Twisted                                           */
    int32_t moire_onsite;  /* 0 none, 1 H0AndHZ, 2 OnlyH0, 3 OnlyHZ, 4 NoH0AndHZ       */
    double  eps, twist_rad, shift1, sign1, sign2;
    double  C0, Cz, Cab, Phi0, Phiz, Phiab;
    int32_t interlayer;    /* 0 gIntLay*exp(-d/dIntLay), 1 two-centre (Koshino/HTC)   */
    double  vpppi0, vppsigma0, bl_delta, d_interlayer, aCC, g_intlay;
    int32_t anderson;      /* Disorder.Anderson: add (u_i - 0.5) * anderson_w         */
    double  anderson_w;
    double  e0_c;          /* TB.OnSiteC/g0                                           */
    /* Smooth interlayer cutoff (no counterpart in the reference, whose cutoff is the hard edge of the
     * neighbour table): with inter_smooth_w > 0 the interlayer hoppings are multiplied by
     * s(rho) = 1 for rho <= rho_c - w, (1 + cos(pi (rho - rho_c + w) / w)) / 2 up to rho_c, 0 beyond,
     * rho the in-plane distance [Ang] and rho_c = inter_cut_rho.  0 = the reference's hard cutoff. */
    double  inter_cut_rho;
    double  inter_smooth_w;
    /* Interlayer.KoshinoSR: both two-centre terms scaled per bond by exp((|dz| - 3.25)/1.34); and
     * Interlayer.RenormalizeCoupling: every interlayer hopping times coupling_factor
     * (Interlayer.CouplingFactor) (ham.F90:6247-6260, 6807-6838, 9817-9823). */
    int32_t koshino_sr;
    int32_t renormalize_coupling;
    double  coupling_factor;
    /* Moire.AddSecondMoire: a second moire pattern on the same graphene (HamOnSiteSecondMoireTerms,
     * ham.F90:3546-3642, and, with moire_offdiag, HamHopSecondMoire, ham.F90:7745-7880): lattice mismatch
     * eps * eps_factor (Moire.LatticePercentFactor), Moire.Twisted2 / TwistAngle2 [rad], Moire.LayerShift2
     * [Ang] with its components along phi2M = atan((1+eps) sin t2 / ((1+eps) cos t2 - 1)),
     * Moire.SecondMoireRotateFirst; its mass term scaled by sign2 (Moire.SecondMoireMassFactor). */
    int32_t second_moire;
    double  eps_factor;
    int32_t twisted2;
    double  twist2_rad;
    int32_t rotate_first;
    double  shift2;
    double  shift2_x, shift2_y;
    /* Run.TypeOfSystem MoireEncapsulatedBilayerBasedOnMoireCell: the effective moire on-site model of the
     * encapsulated bilayer (HamOnSiteMoireEffectiveBilayer, ham.F90:3303-3434) and its bond displacement
     * (ham.F90:12561-12590): bottom / top hBN angles (Moire.BilayerBottomAngle, TopAngle) [rad] and the rigid
     * layer shifts tauX1, tauY1, tauX2, tauY2 of moireBLShift [Ang]; the top layer's displacement takes the
     * rotation first with rotate_first.  deact_upper / deact_uppers: Moire.BLDeactivateUpperLayer /
     * TDBLDeactivateUpperLayers (no moire term on layer 2 / above layer 1; the bond terms of every system).
     * bernal: its interlayer branch (ham.F90:6455-6500, 6721-6745): 1 the vertical pairs only (-tAB1),
     * 2 the bilayer F2G2 set of HamHopInterlayerBernalF2G2 (ham.F90:12800-12827) on an AB-stacked cell (dimer
     * sites found from the structure; a cell that is not AB stacked falls back to 1 as in the reference).
     * tbl: tAA1, tAA2, tAB1, tAB2, tBA0, tBA2, tBA5 as the reference stores them (-t/g0). */
    int32_t encapsulated;
    double  bl_bottom_rad, bl_top_rad;
    double  tau[4];
    int32_t deact_upper, deact_uppers;
    int32_t bernal;
    double  tbl[7];
} gbn_model;

/* ---- host-side cell construction and random numbers (no context, no GPU needed) ------ */
#define GBN_CELL_GRAPHENE 0  /* Run.TypeOfSystem Graphene                       */
#define GBN_CELL_TBG_MOIRE 1 /* Run.TypeOfSystem TwistedBilayerBasedOnMoireCell, and the same cell of
                                MoireEncapsulatedBilayerBasedOnMoireCell (atoms.F90:455-512) */
typedef struct gbn_cell {
    int32_t kind;         /* GBN_CELL_*                                   */
    int32_t cell_size;    /* Structure.CellSize (graphene)                */
    int32_t super_cell;   /* Structure.SuperCell                          */
    int32_t m[4];         /* Structure.MoireCellParameters (bilayer)      */
    double  aG;           /* Structure.LatticeParameter [Ang]             */
    double  height;       /* Structure.CellHeight [Ang]                   */
    double  d_interlayer; /* Structure.InterlayerDistance [Ang]           */
    /* Structure.TwistedBLAddShift (atoms.F90:352-366): the moire cell's second layer offset by 1 the
     * Bernal (Structure.BernalShift) or 2 the bridge (Structure.BridgeShift) offset, plus
     * Structure.BilayerShiftFactor [Ang] along a1+a2 (AtomsShiftFrac, atoms.F90:1490-1504); 0: none */
    int32_t add_shift;
    double  shift_factor;
} gbn_cell;
/* Number of atoms of the cell (CellGet/AtomsPos, lanczosKuboCode/Src/cell.F90:108-140, 207-240). */
int gbn_cell_atoms(const gbn_cell* cell, int64_t* n);
/* ucell(3,3), Rat(3,N) Cartesian, Species(N), layerIndex(N) and the twist [rad] in the reference's
 * atom order and rounding (atoms.F90:124-230, 330-380, 1506-1607, 1768-1794). */
int gbn_build_cell(const gbn_cell* cell, double* ucell, double* rat, int32_t* species, int32_t* layer, double* twist);
/* AtomsSetFrac followed by AtomsSetCart (atoms.F90:1768-1830), in place: the positions the reference's
 * moire on-site and hopping routines see after their own conversions. */
int gbn_cart_roundtrip(int64_t n, const double* ucell, double* rat);
/* n draws of GNU Fortran's random_number(real(8)) after random_seed(PUT=[seed]*n_seed)
 * (the start vectors of KuboInitWF, kubo.F90:46-64, and Anderson disorder, ham.F90:1237-1248). */
int gbn_rng_uniform(int32_t seed, int64_t n, double* out);

/* ---- context ------------------------------------------------------------------------ */
/* No counterpart in the reference (module state); device = CUDA ordinal. */
int         gbn_create(gbn_ctx** out, int32_t device);
int         gbn_destroy(gbn_ctx* ctx);
const char* gbn_last_error(const gbn_ctx* ctx);
const char* gbn_version(void);
/* Use the caller's CUDA stream (a cudaStream_t) for all work of the context; NULL = own stream. */
int         gbn_set_stream(gbn_ctx* ctx, void* cuda_stream);
/* Tuning of the recursion kernels: right-hand sides per thread (1, 2, 4; 0 = widest load), a cap on
 * resident blocks per SM (0 = occupancy limit), the rows per group of the matrix layout (1 = plain
 * sliced ELL; 2, 4 = neighbouring rows share one gather per union column; 0 = chosen from the mean
 * entries per row), the matrix path of the sparse product (1 = each warp stages its next slice
 * records in shared memory with bulk asynchronous copies, 0 = records read from global memory,
 * -1 = staged when two records per warp fit in shared memory) and, for the staged path, a prefetch of
 * the vector rows each slice gathers (0 = none, 1 = into L2, 2 = into L1) or of the rows its epilogue
 * reads (3 = into L1, 4 = into L2; 5, 6, 7 = as 4, and one bulk prefetch into L2 of the rows of the
 * warp's slice 1, 2 or 4 sweeps ahead; -1 = the default, 4).  Used by the autotuner
 * (grabnes_b200/tune.py). */
int         gbn_set_tuning(gbn_ctx* ctx, int32_t rhs_per_thread, int32_t blocks_per_sm, int32_t rows_per_group,
                           int32_t staged, int32_t prefetch);
/* Variant of the recursion's sparse-product kernel: union columns whose gathers are in flight together
 * per batch (4 or 8; 0 = the default), for the staged path whether the staged slice records carry the
 * values (1) or only the column indices, with the values prefetched into L2 and streamed beside the
 * gathers (0; -1 = the default), and the resident blocks per SM the kernel's registers are bounded for
 * (1, 2 or 3; 2 and 3 only with unroll 8 on the staged path, 2 only with whole records staged; 0 = 1); for gbn_lanczos_fields, whether each tile's
 * Peierls rotations are tabulated once before its steps (1) or done on the fly by every thread at every
 * step (0, -1 = the default); and the tile-local product (1: mixed precision, real hoppings; each tile of
 * slices copies the rows it gathers into shared memory first; 0, -1 = the default: no); and the fused step
 * (1: real hoppings or batched fields, staged records, the widest loads per thread, unroll 8 in mixed
 * precision and 4 in FP64; the update
 * folded into the product: every gathered column forms u_k = v_k - alpha u_{k-1} from two stored vectors,
 * and b_k comes from three sums of the previous product, so a step is one launch; 0: two launches; -1 =
 * the default: fused where the rows hold at most 8 entries on average and the shape has a fused kernel,
 * two launches otherwise).
 * No counterpart in the reference.  Used by the autotuner (grabnes_b200/tune.py). */
int         gbn_set_kernel_variant(gbn_ctx* ctx, int32_t col_unroll, int32_t stage_values, int32_t min_blocks,
                                   int32_t field_table, int32_t tiled, int32_t fused);
/* Kernels launched by this context since creation (for launch accounting). */
int64_t     gbn_launch_count(const gbn_ctx* ctx);
/* Device time of the recursion loop of the last gbn_lanczos* / gbn_run_staged call and its number of
 * recursion steps (each step launches one update and one sparse-product kernel, or one kernel with the
 * fused step of gbn_set_kernel_variant). */
int         gbn_last_timing(const gbn_ctx* ctx, double* step_ms_total, int64_t* step_launches);
/* Average per-launch device time of the sparse-product and the update kernels over the first (up to 64)
 * steps of the last call, measured with CUDA events on the context's stream. */
int         gbn_last_kernel_timing(const gbn_ctx* ctx, double* spmm_ms, double* update_ms);

/* ---- geometry and neighbour search ---------------------------------------------------- */
/* Atoms of the cell: Rat(3,N) Cartesian [Ang], Species(N), layerIndex(N), ucell(3,3).
 * Replaces the module arrays of lanczosKuboCode/Src/atoms.F90 and cell.F90 (AtomsPos, CellGet). */
int gbn_set_geometry(gbn_ctx* ctx, int64_t n, const double* rat, const int32_t* species,
                     const int32_t* layer, const double* ucell);
/* NeighSearchLayered (lanczosKuboCode/Src/neigh.F90:117-316, periodicZ = .false.) on the device:
 * same entries, same order within each atom, NeighD bit-identical. */
int gbn_neighbours(gbn_ctx* ctx, double cut2intra, double cut2inter, int32_t second_layer,
                   int32_t* max_neigh, int64_t* total);
/* Copy Nneigh(N), NList(maxNeigh,N), NeighD(3,maxNeigh,N), neighCell(3,maxNeigh,N) out (any may be NULL). */
int gbn_get_neighbours(gbn_ctx* ctx, int32_t* nneigh, int32_t* nlist, double* neighd, int32_t* neigh_cell);

/* ---- Hamiltonian ----------------------------------------------------------------------- */
/* HamOnSite + HamHopping bond loop (ham.F90:846-1248, 6517-6846) on the device.  rat_onsite and
 * rat_hop are the positions HamOnSite and HamHopping see (they may differ in the last bit after
 * the reference's fractional/Cartesian round trips); uniform holds the N Anderson draws (or NULL). */
int gbn_assemble(gbn_ctx* ctx, const gbn_model* model, const double* rat_onsite,
                 const double* rat_hop, const double* uniform);
/* HamCheckFinite (ham.F90:4432-4477) and the pair scan of HamCheckHermiticity (ham.F90:4491-4571) on the
 * current Hamiltonian: counts[0] non-finite hoppings, [1] non-finite on-site energies, [2] the first
 * atom with either (1-based, 0 if none), [3] entries without a reverse entry (the same pair with the
 * opposite lattice translation), [4] pairs compared; *max_asym = max |hopp(j,i) - conj(hopp(j2,m))| in
 * g0.  The reference stops on non-finite values and prints or warns about the asymmetry; the caller
 * decides here.  Needs the neighbour images (gbn_neighbours, or gbn_set_images after loading). */
int gbn_check_hamiltonian(gbn_ctx* ctx, int64_t* counts, double* max_asym);
/* HamHopHaldane (ham.F90:7043-7142, chirality HamHaldaneChirality ham.F90:13063-13100), after
 * gbn_peierls as in HamHopping: every second-neighbour bond within a layer (|d - aG| < 0.1 Ang,
 * Species 1 or 2) gets + t2 exp(i nu phase), or, with paper != 0, is multiplied by exp(i nu phase);
 * nu = +1 / -1 for a clockwise / anticlockwise path through the common nearest neighbour.  t2 in g0,
 * phase in rad (Haldane.OppositePhase already applied); layer_mask bit l-1 selects layer l
 * (Haldane.LayerControl), 0 = every layer.  Needs NeighD (gbn_neighbours or gbn_set_neighd).
 * GBN_ERR_NUMERIC if a bond has no common nearest neighbour (the reference stops there too). */
int gbn_haldane(gbn_ctx* ctx, double aG, double t2, double phase, int32_t paper, uint32_t layer_mask);
/* neighCell(3,maxNeigh,N) of a neighbour list loaded with gbn_load_hamiltonian, so that gbn_peierls can
 * act on loaded hoppings, with the positions of gbn_set_geometry (the Output.ReadDataFiles path of
 * CalcKubo, calc.F90:86-104: hoppings read from a file, then HamPeierlsPeriodicGauge). */
int gbn_set_images(gbn_ctx* ctx, const int32_t* ncell);
/* HamPeierlsPeriodicGauge (ham.F90:12834-12882): multiply the assembled hoppings by the phases of
 * flux (= B pi / Phi0, in 1/Ang^2 * 1e20) including the corner term; positions from gbn_assemble. */
int gbn_peierls(gbn_ctx* ctx, double flux);
/* Copy H0(N) and hopp(maxNeigh,N) (complex) of the current Hamiltonian out (either may be NULL). */
int gbn_get_hamiltonian(gbn_ctx* ctx, double* h0, double* hopp);
/* H0Bottom and H0Top of HamOnSite (ham.F90:44-45, 2703, 3639), written by HamHopWriteTables to
 * <prefix>.bottom.e and <prefix>.top.e (ham.F90:7020-7034): bottom = the on-site energies after the first
 * moire's terms when the assembled model ran the moire branch (moire_onsite != 0), else 0; top = H0 - H0Bottom
 * when it also ran the second moire (second_moire), else 0.  g0 units, reference atom order; either
 * pointer may be NULL.  Replaces the H0Bottom / H0Top arrays of the ham module. */
int gbn_get_onsite_layers(gbn_ctx* ctx, double* bottom, double* top);
/* Minimal drop-in for a Fortran host: the arrays KuboRecursion receives
 * (lanczosKuboCode/Src/kubosubs.F90:26-43: H0, hopp, NList2 and the module's Nneigh, nAt). */
int gbn_load_hamiltonian(gbn_ctx* ctx, int64_t n, int32_t max_neigh, const int32_t* nneigh,
                         const int32_t* nlist, const double* hopp, const double* h0);

/* ---- recursion ------------------------------------------------------------------------- */
/* KuboRecursion (kubosubs.F90:26-138) for nrhs start vectors at once.  psi0: complex [nrhs][N]
 * (reference atom order, normalised by the caller); nsteps[r] <= nmax recursion steps of vector r;
 * a, b: [nrhs][nmax] (entries beyond nsteps[r] are left as computed for nmax).  precision:
 * GBN_FP64 or GBN_MIXED.  Host buffers; copies in and out are part of the call. */
int gbn_lanczos(gbn_ctx* ctx, int32_t precision, int32_t nrhs, const double* psi0,
                const int32_t* nsteps, int32_t nmax, double* a, double* b);
/* Same with random-phase start vectors built on the device from host uniform draws
 * u[nrhs][N]: psi_i = exp(2 pi i u_i)/sqrt(N) (KuboInitWF, kubo.F90:61-64). */
int gbn_lanczos_phases(gbn_ctx* ctx, int32_t precision, int32_t nrhs, const double* u,
                       const int32_t* nsteps, int32_t nmax, double* a, double* b);
/* Many perpendicular fields in one batch (the MagField sweep of magf.F90:100-146 with KuboInitWF +
 * KuboRecursion per field): field f has m[f] flux quanta through the cell and nvec random-phase start
 * vectors, u[f][v][N] their uniform draws as for gbn_lanczos_phases; nsteps[f][v] (or NULL = nmax) their
 * recursion lengths; a, b: [f][v][nmax].  The hoppings must come from gbn_assemble without gbn_peierls:
 * the entries keep the field-free hopping and the Peierls phase per flux quantum, and each field's phase
 * is applied on the fly, so that one matrix serves all fields.  Vectors of similar length share tiles.
 * A cell so small that a row holds two periodic images of one neighbour is rejected (GBN_ERR_ARG). */
int gbn_lanczos_fields(gbn_ctx* ctx, int32_t precision, int32_t nfields, const int32_t* m, int32_t nvec,
                       const double* u, const int32_t* nsteps, int32_t nmax, double* a, double* b);
/* Local DOS of single atoms (KuboInitWFPDOS, kubo.F90:87-138): start vector r is the unit vector
 * on atom sites[r] (1-based), built on the device; all sites run as one batch of right-hand sides. */
int gbn_lanczos_sites(gbn_ctx* ctx, int32_t precision, int32_t nsites, const int64_t* sites,
                      const int32_t* nsteps, int32_t nmax, double* a, double* b);
/* Layer (and species) DOS (KuboInitWFLayerDOS / KuboInitWFLayerAndSpeciesDOS, kubo.F90:140-274):
 * set_of_atom[N] gives each atom's set (0..nsets-1, or -1); the k-th atom of a set, in atom order,
 * takes psi = exp(2 pi i u[k])/sqrt(assumed[set]), and a set whose norm then differs from 1 by more
 * than 1e-6 is normalised.  All sets run as one batch of right-hand sides; a set without atoms has a
 * zero start vector and no DOS, and its a, b are NaN (the reference divides by the zero norm). */
int gbn_lanczos_sets(gbn_ctx* ctx, int32_t precision, int32_t nsets, const int32_t* set_of_atom,
                     const double* u, const double* assumed, const int32_t* nsteps, int32_t nmax,
                     double* a, double* b);

/* ---- Kubo.PDOS selections (CalcKubo, calc.F90:214-541) ------------------------------------ */
enum {
    GBN_PDOS_LAYER = 1,           /* Kubo.PDOSLayer */
    GBN_PDOS_LAYER_SPECIES = 2,   /* Kubo.PDOSLayerAndSpecies */
    GBN_PDOS_DIST = 3,            /* Kubo.PDOSDist */
    GBN_PDOS_MOIRE_SC1 = 4,       /* Kubo.PDOSMoireSC1 */
    GBN_PDOS_SUPERMOIRE = 5,      /* Kubo.PDOSMoireSuperMoire */
    GBN_PDOS_SUPERMOIRE2 = 6,     /* Kubo.PDOSMoireSuperMoire2 */
    GBN_PDOS_SUPERMOIRE3 = 7,     /* Kubo.PDOSMoireSuperMoire3 */
    GBN_PDOS_ATOM_LIST = 8,       /* Kubo.PDOSAtomList */
    GBN_PDOS_BY_NUMBER = 9,       /* Kubo.PDOSByNumber */
    GBN_PDOS_PNP = 10             /* Kubo.PDOSPNP */
};
enum { GBN_STACK_NONE = 0, GBN_STACK_ENCAPSULATED_FOUR = 1, GBN_STACK_T3BG = 2 };
typedef struct gbn_pdos {
    int32_t mode;                 /* GBN_PDOS_*: the first selection flag that is set */
    double xmin, xmax, ymin, ymax;   /* Kubo.PDOSxmin.. [Ang] */
    int32_t min_value;            /* Kubo.PDOSMinValue */
    int32_t super_cell;           /* Structure.SuperCell */
    int32_t cell_size;            /* Structure.CellSize */
    double supermoire_length;     /* Kubo.PDOSMoireSuperMoireLength [Ang] */
    double aG;                    /* lattice parameter [Ang] */
    int32_t ignore_layers_1_4;    /* Kubo.PDOSIgnoreLayer1and4 */
    int32_t atom_list[6];         /* Kubo.PDOSList */
    int32_t atom_number;          /* Kubo.PDOSNumber */
    double pnp_delta;             /* Potential.PNPDelta [Ang] */
    int32_t number_of_layers;     /* Kubo.NumberOfLayers */
    int32_t stack;                /* GBN_STACK_*: Stack.EncapsulatedFourLayers / Stack.T3BG */
    int32_t n_bn1, n_bn2, n_c;    /* Kubo.NumberOfBNAtoms1/2, Kubo.NumberOfCAtoms */
} gbn_pdos;
/* The atoms of the single-atom modes (3..10), in the order the reference visits them: atoms[k]
 * (1-based) and coords[k][3], the position the reference writes to the folder's coords file (after
 * the fractional/Cartesian conversions the selection loop makes).  rat: Cartesian positions as the
 * Hamiltonian left them.  At most cap atoms are written; *count is the full count. */
int gbn_pdos_atoms(const gbn_pdos* p, int64_t n, const double* rat, const int32_t* species,
                   const int32_t* layer, const double* ucell, int64_t cap, int64_t* count,
                   int64_t* atoms, double* coords);
/* The sets of the layer modes (1, 2): set_of_atom[N] for gbn_lanczos_sets, and per set (at most cap)
 * its layer, species (0 for GBN_PDOS_LAYER) and the reference's assumed atom count. */
int gbn_pdos_sets(const gbn_pdos* p, int64_t n, const int32_t* species, const int32_t* layer,
                  int32_t cap, int32_t* nsets, int32_t* set_of_atom, int32_t* set_layer,
                  int32_t* set_species, double* assumed);
/* Split form used for timing with device-resident inputs: gbn_stage_phases uploads and builds the
 * start vectors; gbn_run_staged runs nmax steps and leaves a, b on the device unless a, b are
 * non-NULL (then they are copied out). */
int gbn_stage_phases(gbn_ctx* ctx, int32_t precision, int32_t nrhs, const double* u);
int gbn_run_staged(gbn_ctx* ctx, int32_t nmax, double* a, double* b);

/* ---- continued fraction ------------------------------------------------------------------ */
/* KuboFrac (kubosubs.F90:222-288) for nrhs coefficient sets a, b [nrhs][nmax] of lengths
 * nsteps[r]; energies E_k = emin + k (emax - emin)/n_en, k = 0..n_en; dos [nrhs][n_en+1] =
 * -Im g(E + i eta)/pi * norm[r] (norm may be NULL: 1). energy [n_en+1] may be NULL. */
int gbn_cf_dos(gbn_ctx* ctx, int32_t nrhs, const double* a, const double* b, const int32_t* nsteps,
               int32_t nmax, double eta, int32_t n_en, double emin, double emax, const double* norm,
               double* energy, double* dos);

/* ---- Chebyshev time evolution --------------------------------------------------------------- */
/* KuboInterval (kubosubs.F90:290-350) on the host: from the recursion coefficients a, b [nrecurs]
 * (b[i] couples levels i and i+1), ac = (emax + emin)/2 and bc = 1.2 (emax - emin)/4 of the extreme
 * eigenvalues of the tridiagonal matrix.  No context, no GPU. */
int gbn_cheb_interval(const double* a, const double* b, int32_t nrecurs, double* ac, double* bc);
/* KuboCn (kubosubs.F90:352-433) on the host: the npol complex coefficients c [npol] of the propagator
 * exp(-i H dt) in the scaled Chebyshev basis of gbn_cheb_evolve, c_0 = exp(-i ac dt) J_0(2 bc dt),
 * c_n = sqrt(2) (-i)^n exp(-i ac dt) J_n(2 bc dt) (the reference's Jacobi-matrix quadrature gives the
 * same values).  No context, no GPU. */
int gbn_cheb_coef(double dt, double ac, double bc, int32_t npol, double* c);
/* KuboChebyshevEvolve (kubosubs.F90:557-619) for nrhs complex vectors z [nrhs][N] (host, reference atom
 * order, in place): with x = (H - ac)/(2 bc), psi_0 = sqrt(2) z, psi_1 = x psi_0,
 * psi_{n+1} = 2 x psi_n - psi_{n-1}, z <- c_0 z + sum_{n=1}^{npol-1} c_n psi_n; c complex [npol] (the
 * coefficients of KuboCn).  precision: GBN_FP64, or GBN_MIXED (complex FP32 psi_n, FP64 step
 * arithmetic and FP64 accumulation of z). */
int gbn_cheb_evolve(gbn_ctx* ctx, int32_t precision, int32_t nrhs, const double* c, int32_t npol, double ac,
                    double bc, double* z);
/* KuboEvol (kubosubs.F90:438-553): psi <- U psi and zupsi <- U zupsi + [U, X] psi for nrhs vectors
 * psi, zupsi [nrhs][N] (host, in place), U the propagator of gbn_cheb_evolve (same c, ac, bc) and X
 * the position along dir (1 = x, 2 = y) through NeighD: the commutator recurrence
 * X_0 = 0, X_{n+1} = 2 x X_n + D psi_n / bc - X_{n-1} with D = NeighD(dir) * (-hopp).  Needs
 * gbn_neighbours or NeighD through gbn_set_neighd.  precision as for gbn_cheb_evolve. */
int gbn_kubo_evol(gbn_ctx* ctx, int32_t precision, int32_t nrhs, const double* c, int32_t npol, double ac,
                  double bc, int32_t dir, double* psi, double* zupsi);
/* KuboTEvol (kubo.F90:321-397) with psi and zupsi kept on the device: nt steps of gbn_kubo_evol; after
 * every nwr-th step, norms[r][w] = |zupsi_r|^2 and a, b [r][w][nrecurs] = the FP64-reduced recursion of
 * zupsi_r / |zupsi_r| (w = 0 .. nt/nwr - 1; NaN where a norm is 0).  psi, zupsi [nrhs][N] complex are
 * read at the start and hold the evolved states on return.  Host traffic: the states once each way and
 * the coefficients, instead of both states every step. */
int gbn_kubo_tevol(gbn_ctx* ctx, int32_t precision, int32_t nrhs, const double* c, int32_t npol, double ac,
                   double bc, int32_t dir, int32_t nt, int32_t nwr, int32_t nrecurs, double* psi, double* zupsi,
                   double* norms, double* a, double* b);
/* Mean-square displacement and diffusivity from the norms of gbn_kubo_tevol (no counterpart in the
 * reference, which writes only the norms |ZUPsi|^2 of KuboTEvol, kubo.F90:376-385, in its .Z2_ files).
 * norms [nrhs][nw] as gbn_kubo_tevol returns them, for write steps every nwr time steps of dt_fs
 * femtoseconds (dt_fs = Kubo.TimeStep * hbar / g0).  Out [nw]: t_fs = (w + 1) nwr dt_fs; msd = the mean
 * over the vectors of |ZUPsi_r|^2, the spread <(X(t) - X(0))^2> [Ang^2] along the evolution's
 * direction; d_ratio = msd / t and d_slope = d msd / dt (central differences between write steps, from
 * msd = 0 at t = 0; one-sided at the last step) [Ang^2 / fs = 0.1 cm^2 / s]; d_ratio, d_slope may be
 * NULL.  Host arithmetic in FP64 (no device, no context). */
int gbn_kubo_msd(int32_t nrhs, int32_t nw, int32_t nwr, double dt_fs, const double* norms, double* t_fs,
                 double* msd, double* d_ratio, double* d_slope);
/* NeighD(3,maxNeigh,N) for gbn_kubo_evol after gbn_load_hamiltonian. */
int gbn_set_neighd(gbn_ctx* ctx, const double* neighd);

/* ---- gradient of a DOS loss ------------------------------------------------------------------ */
/* No counterpart in the reference.  Loss L = sum_E (DOS(E) - target(E))^2, DOS from one start vector
 * (phases from the uniform draws u [N]) by an FP64 recursion of nrecurs steps and the continued
 * fraction (eta, n_en, emin, emax as for gbn_cf_dos, units of g0; target [n_en+1]).  grad [4] =
 * dL/d(t, Vpp_sigma0, delta, w): the intralayer nearest-neighbour hopping [eV], the sigma two-centre
 * amplitude [eV], the two-centre decay length [Ang] and the width of the smooth interlayer cutoff
 * [Ang], for the Hamiltonian last assembled with `model` (gbn_assemble; real hoppings, geometry and
 * NeighD on the context; g0 [eV] the energy unit).  Reverse sweep through the same sparse product
 * (the adjoint of the three-term recurrence), with the recursion vectors checkpointed every
 * `checkpoint` steps and recomputed in between.  dos [n_en+1], a, b [nrecurs] may be NULL. */
int gbn_dos_gradient(gbn_ctx* ctx, const gbn_model* model, double g0, const double* u, int32_t nrecurs,
                     int32_t checkpoint, double eta, int32_t n_en, double emin, double emax, const double* target,
                     double* loss, double* grad, double* dos, double* a, double* b);
/* The same with a precision: GBN_FP64 (= gbn_dos_gradient) or GBN_MIXED, the FP32 variant: complex64
 * recursion and adjoint vectors (checkpoints included) and FP32 hoppings, with FP64 arithmetic in every
 * kernel, FP64 dot products, scalars, continued fraction and dL/dH accumulation.  No counterpart in
 * the reference. */
int gbn_dos_gradient_prec(gbn_ctx* ctx, int32_t precision, const gbn_model* model, double g0, const double* u,
                          int32_t nrecurs, int32_t checkpoint, double eta, int32_t n_en, double emin, double emax,
                          const double* target, double* loss, double* grad, double* dos, double* a, double* b);

/* ---- recursion without device allocation ------------------------------------------------------ */
/* No counterpart in the reference: an addition for hosts that cannot allocate device memory.
 *
 * A host that gives all of a GPU's memory to its own pool allocator, or that must not call cudaMalloc
 * and cudaFree because they synchronise the whole device while the host has other work in flight
 * there, cannot create a gbn_ctx (a context allocates per-context device buffers).  This call needs
 * no context and allocates nothing: its three recursion vectors, reduction partials and counter sit
 * in one fixed array inside the library, sized for GBN_NOALLOC_MAX_ATOMS atoms (about 48 MiB), which
 * every GPU that loads the library holds until the process exits.
 *
 * It runs the KuboRecursion of one start vector in FP64 on the CURRENT device, on `stream` (NULL:
 * the default stream), and returns when the stream has finished it.  All pointers are device memory
 * of the current device, in the layouts of gbn_load_hamiltonian: nneigh(N), nlist(maxNeigh,N)
 * (1-based), hopp(maxNeigh,N) complex, h0(N), psi(N) complex (normalised by the caller; hopp and psi
 * 16-byte aligned); a, b: nrecurs doubles each, written by the call.
 * The first call on a device, and the first after that device's context was reset, looks up the
 * array's device address (cudaGetSymbolAddress); make that call before any stream capture on that
 * device.  All calls on a device share the array, so
 * calls that overlap on the GPU (other host threads, other streams) race: serialise them.
 * Returns GBN_ERR_LIMIT when n > GBN_NOALLOC_MAX_ATOMS, GBN_ERR_ARG for other bad arguments
 * (including Nneigh/NList entries out of range, found on the device), GBN_ERR_NUMERIC for a b_n that
 * is not finite or not positive, GBN_ERR_CUDA for a failed launch or copy.  gbn_last_error() does not
 * apply (there is no context). */
#define GBN_NOALLOC_MAX_ATOMS 1048576
#define GBN_ERR_LIMIT (-7) /* a size beyond the stated maximum of the call */
int gbn_lanczos_noalloc(int64_t n, int32_t max_neigh, const int32_t* nneigh, const int32_t* nlist,
                        const double* hopp, const double* h0, const double* psi, int32_t nrecurs,
                        double* a, double* b, void* stream);

#ifdef __cplusplus
}
#endif
#endif
