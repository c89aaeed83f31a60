"""grabnes_b200 -- B200 (sm_100a) implementation of the GRABNES large-cell recursion hot path.

The work is done by libgrabnes_gpu.so (CUDA kernels behind the C ABI of include/grabnes_gpu.h);
this module is a thin ctypes binding that mirrors that ABI for Python callers and tests.  There is
no CPU fallback: importing works without a GPU, but every call that needs the library raises if the
shared object is missing or no CUDA device is present.
"""

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgrabnes_gpu.so")

GBN_FP64, GBN_MIXED = 0, 1
ERRORS = {-1: "argument", -2: "cuda", -3: "state", -4: "numeric", -5: "alloc", -6: "timeout", -7: "limit"}
GBN_ERR_ARG, GBN_ERR_CUDA, GBN_ERR_STATE, GBN_ERR_NUMERIC, GBN_ERR_ALLOC, GBN_ERR_TIMEOUT = -1, -2, -3, -4, -5, -6
GBN_ERR_LIMIT = -7
NOALLOC_MAX_ATOMS = 1048576   # GBN_NOALLOC_MAX_ATOMS


class GbnError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"grabnes_gpu error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class Model(C.Structure):
    """gbn_model of include/grabnes_gpu.h"""
    _fields_ = [
        ("aG", C.c_double), ("tbnn", C.c_int32), ("gn_cc", C.c_double * 8), ("nradii", C.c_double * 8),
        ("intralayer", C.c_int32), ("tksl", C.c_double * 8),
        ("moire_offdiag", C.c_int32), ("moire_mid", C.c_int32), ("moire_twisted", C.c_int32),
        ("moire_onsite", C.c_int32), ("eps", C.c_double), ("twist_rad", C.c_double), ("shift1", C.c_double),
        ("sign1", C.c_double), ("sign2", C.c_double), ("C0", C.c_double), ("Cz", C.c_double), ("Cab", C.c_double),
        ("Phi0", C.c_double), ("Phiz", C.c_double), ("Phiab", C.c_double),
        ("interlayer", C.c_int32), ("vpppi0", C.c_double), ("vppsigma0", C.c_double), ("bl_delta", C.c_double),
        ("d_interlayer", C.c_double), ("aCC", C.c_double), ("g_intlay", C.c_double),
        ("anderson", C.c_int32), ("anderson_w", C.c_double), ("e0_c", C.c_double),
        ("inter_cut_rho", C.c_double), ("inter_smooth_w", C.c_double),
        ("koshino_sr", C.c_int32), ("renormalize_coupling", C.c_int32), ("coupling_factor", C.c_double),
        ("second_moire", C.c_int32), ("eps_factor", C.c_double), ("twisted2", C.c_int32), ("twist2_rad", C.c_double),
        ("rotate_first", C.c_int32), ("shift2", C.c_double), ("shift2_x", C.c_double), ("shift2_y", C.c_double),
        ("encapsulated", C.c_int32), ("bl_bottom_rad", C.c_double), ("bl_top_rad", C.c_double),
        ("tau", C.c_double * 4), ("deact_upper", C.c_int32), ("deact_uppers", C.c_int32), ("bernal", C.c_int32),
        ("tbl", C.c_double * 7),
    ]


class Cell(C.Structure):
    """gbn_cell of include/grabnes_gpu.h"""
    _fields_ = [("kind", C.c_int32), ("cell_size", C.c_int32), ("super_cell", C.c_int32), ("m", C.c_int32 * 4),
                ("aG", C.c_double), ("height", C.c_double), ("d_interlayer", C.c_double), ("add_shift", C.c_int32),
                ("shift_factor", C.c_double)]


CELL_GRAPHENE, CELL_TBG_MOIRE = 0, 1


class Pdos(C.Structure):
    """gbn_pdos of include/grabnes_gpu.h: a Kubo.PDOS selection"""
    _fields_ = [("mode", C.c_int32), ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
                ("ymax", C.c_double), ("min_value", C.c_int32), ("super_cell", C.c_int32), ("cell_size", C.c_int32),
                ("supermoire_length", C.c_double), ("aG", C.c_double), ("ignore_layers_1_4", C.c_int32),
                ("atom_list", C.c_int32 * 6), ("atom_number", C.c_int32), ("pnp_delta", C.c_double),
                ("number_of_layers", C.c_int32), ("stack", C.c_int32), ("n_bn1", C.c_int32), ("n_bn2", C.c_int32),
                ("n_c", C.c_int32)]


(PDOS_LAYER, PDOS_LAYER_SPECIES, PDOS_DIST, PDOS_MOIRE_SC1, PDOS_SUPERMOIRE, PDOS_SUPERMOIRE2, PDOS_SUPERMOIRE3,
 PDOS_ATOM_LIST, PDOS_BY_NUMBER, PDOS_PNP) = range(1, 11)
STACK_NONE, STACK_ENCAPSULATED_FOUR, STACK_T3BG = 0, 1, 2

_lib = None


def lib():
    """Load libgrabnes_gpu.so; raise (never fall back) if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m grabnes_b200.build`")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _p(dtype):
    return np.ctypeslib.ndpointer(dtype=dtype, flags="C_CONTIGUOUS")


def _opt(dtype):
    """pointer argument that also accepts None"""
    base = _p(dtype)

    class Opt(base):
        @classmethod
        def from_param(cls, obj):
            return None if obj is None else base.from_param(obj)
    return Opt


EXPORTS = ["gbn_cell_atoms", "gbn_build_cell", "gbn_cart_roundtrip", "gbn_rng_uniform", "gbn_create", "gbn_destroy", "gbn_last_error", "gbn_version", "gbn_set_stream", "gbn_set_tuning", "gbn_set_kernel_variant", "gbn_launch_count",
           "gbn_last_timing", "gbn_last_kernel_timing", "gbn_set_geometry", "gbn_neighbours", "gbn_get_neighbours", "gbn_assemble",
           "gbn_peierls", "gbn_get_hamiltonian", "gbn_load_hamiltonian", "gbn_lanczos", "gbn_lanczos_phases",
           "gbn_stage_phases", "gbn_run_staged", "gbn_cf_dos", "gbn_cheb_evolve", "gbn_kubo_evol", "gbn_set_neighd", "gbn_lanczos_noalloc",
           "gbn_cheb_interval", "gbn_cheb_coef", "gbn_dos_gradient", "gbn_dos_gradient_prec", "gbn_lanczos_sites", "gbn_lanczos_sets",
           "gbn_pdos_atoms", "gbn_pdos_sets", "gbn_lanczos_fields", "gbn_set_images", "gbn_haldane", "gbn_kubo_tevol", "gbn_check_hamiltonian", "gbn_kubo_msd",
           "gbn_get_onsite_layers"]


def _declare(L):
    d, i32, i64, vp = C.c_double, C.c_int32, C.c_int64, C.c_void_p
    L.gbn_cell_atoms.argtypes = [C.POINTER(Cell), C.POINTER(i64)]
    L.gbn_build_cell.argtypes = [C.POINTER(Cell), _p(np.float64), _p(np.float64), _p(np.int32), _p(np.int32),
                                 C.POINTER(d)]
    L.gbn_cart_roundtrip.argtypes = [i64, _p(np.float64), _p(np.float64)]
    L.gbn_rng_uniform.argtypes = [i32, i64, _p(np.float64)]
    L.gbn_create.argtypes = [C.POINTER(vp), i32]
    L.gbn_destroy.argtypes = [vp]
    L.gbn_last_error.argtypes = [vp]
    L.gbn_last_error.restype = C.c_char_p
    L.gbn_version.restype = C.c_char_p
    L.gbn_set_stream.argtypes = [vp, vp]
    L.gbn_set_tuning.argtypes = [vp, i32, i32, i32, i32, i32]
    L.gbn_set_kernel_variant.argtypes = [vp, i32, i32, i32, i32, i32, i32]
    L.gbn_launch_count.argtypes = [vp]
    L.gbn_launch_count.restype = i64
    L.gbn_last_timing.argtypes = [vp, C.POINTER(d), C.POINTER(i64)]
    L.gbn_last_kernel_timing.argtypes = [vp, C.POINTER(d), C.POINTER(d)]
    L.gbn_set_geometry.argtypes = [vp, i64, _p(np.float64), _p(np.int32), _p(np.int32), _p(np.float64)]
    L.gbn_neighbours.argtypes = [vp, d, d, i32, C.POINTER(i32), C.POINTER(i64)]
    L.gbn_get_neighbours.argtypes = [vp, _opt(np.int32), _opt(np.int32), _opt(np.float64), _opt(np.int32)]
    L.gbn_assemble.argtypes = [vp, C.POINTER(Model), _opt(np.float64), _opt(np.float64), _opt(np.float64)]
    L.gbn_peierls.argtypes = [vp, d]
    L.gbn_set_images.argtypes = [vp, _p(np.int32)]
    L.gbn_haldane.argtypes = [vp, d, d, d, i32, C.c_uint32]
    L.gbn_check_hamiltonian.argtypes = [vp, _p(np.int64), C.POINTER(d)]
    L.gbn_get_hamiltonian.argtypes = [vp, _opt(np.float64), _opt(np.complex128)]
    L.gbn_get_onsite_layers.argtypes = [vp, _opt(np.float64), _opt(np.float64)]
    L.gbn_load_hamiltonian.argtypes = [vp, i64, i32, _p(np.int32), _p(np.int32), _p(np.complex128), _p(np.float64)]
    L.gbn_lanczos.argtypes = [vp, i32, i32, _p(np.complex128), _opt(np.int32), i32, _p(np.float64), _p(np.float64)]
    L.gbn_lanczos_phases.argtypes = [vp, i32, i32, _p(np.float64), _opt(np.int32), i32, _p(np.float64),
                                     _p(np.float64)]
    L.gbn_lanczos_fields.argtypes = [vp, i32, i32, _p(np.int32), i32, _p(np.float64), _opt(np.int32), i32,
                                     _p(np.float64), _p(np.float64)]
    L.gbn_lanczos_sites.argtypes = [vp, i32, i32, _p(np.int64), _opt(np.int32), i32, _p(np.float64), _p(np.float64)]
    L.gbn_lanczos_sets.argtypes = [vp, i32, i32, _p(np.int32), _p(np.float64), _p(np.float64), _opt(np.int32), i32,
                                   _p(np.float64), _p(np.float64)]
    L.gbn_pdos_atoms.argtypes = [C.POINTER(Pdos), i64, _p(np.float64), _p(np.int32), _p(np.int32), _p(np.float64), i64,
                                 C.POINTER(i64), _opt(np.int64), _opt(np.float64)]
    L.gbn_pdos_sets.argtypes = [C.POINTER(Pdos), i64, _p(np.int32), _p(np.int32), i32, C.POINTER(i32), _p(np.int32),
                                _p(np.int32), _p(np.int32), _p(np.float64)]
    L.gbn_stage_phases.argtypes = [vp, i32, i32, _p(np.float64)]
    L.gbn_run_staged.argtypes = [vp, i32, _opt(np.float64), _opt(np.float64)]
    L.gbn_cf_dos.argtypes = [vp, i32, _p(np.float64), _p(np.float64), _opt(np.int32), i32, d, i32, d, d,
                             _opt(np.float64), _opt(np.float64), _p(np.float64)]
    L.gbn_cheb_evolve.argtypes = [vp, i32, i32, _p(np.complex128), i32, d, d, _p(np.complex128)]
    L.gbn_kubo_evol.argtypes = [vp, i32, i32, _p(np.complex128), i32, d, d, i32, _p(np.complex128),
                                _p(np.complex128)]
    L.gbn_set_neighd.argtypes = [vp, _p(np.float64)]
    L.gbn_kubo_tevol.argtypes = [vp, i32, i32, _p(np.complex128), i32, d, d, i32, i32, i32, i32, _p(np.complex128),
                                 _p(np.complex128), _opt(np.float64), _opt(np.float64), _opt(np.float64)]
    L.gbn_cheb_interval.argtypes = [_p(np.float64), _p(np.float64), i32, C.POINTER(d), C.POINTER(d)]
    L.gbn_dos_gradient.argtypes = [vp, C.POINTER(Model), d, _p(np.float64), i32, i32, d, i32, d, d, _p(np.float64),
                                   C.POINTER(d), _p(np.float64), _opt(np.float64), _opt(np.float64), _opt(np.float64)]
    L.gbn_dos_gradient_prec.argtypes = [vp, i32, C.POINTER(Model), d, _p(np.float64), i32, i32, d, i32, d, d,
                                        _p(np.float64), C.POINTER(d), _p(np.float64), _opt(np.float64),
                                        _opt(np.float64), _opt(np.float64)]
    L.gbn_cheb_coef.argtypes = [d, d, d, i32, _p(np.complex128)]
    L.gbn_kubo_msd.argtypes = [i32, i32, i32, d, _p(np.float64), _p(np.float64), _p(np.float64), _opt(np.float64),
                               _opt(np.float64)]
    # device pointers (ints from tensor.data_ptr()), no context
    L.gbn_lanczos_noalloc.argtypes = [i64, i32, vp, vp, vp, vp, vp, i32, vp, vp, vp]


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype).reshape(-1)


class Context:
    """One library context on one CUDA device (owns device memory and a stream)."""

    def __init__(self, device=0):
        self._L = lib()
        h = C.c_void_p()
        rc = self._L.gbn_create(C.byref(h), device)
        if rc != 0:
            raise GbnError(rc, "gbn_create failed (no CUDA device?)")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._L.gbn_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _ck(self, rc):
        if rc != 0:
            raise GbnError(rc, self._L.gbn_last_error(self._h).decode())

    # ---------------------------------------------------------------- plumbing
    def set_stream(self, stream_handle):
        self._ck(self._L.gbn_set_stream(self._h, C.c_void_p(stream_handle)))

    def set_tuning(self, rhs_per_thread=0, blocks_per_sm=0, rows_per_group=0, staged=-1, prefetch=-1):
        self._ck(self._L.gbn_set_tuning(self._h, rhs_per_thread, blocks_per_sm, rows_per_group, staged, prefetch))

    def set_kernel_variant(self, col_unroll=0, stage_values=-1, min_blocks=0, field_table=-1, tiled=-1, fused=-1):
        """Columns in flight per batch of the sparse product (4, 8; 0 = default), whether staged slice
        records carry the values (1) or only the column indices (0; -1 = default), the resident blocks per
        SM its registers are bounded for (1, 2, 3; 0 = 1), and for batched fields the per-tile rotation table
        (1) or rotations on the fly (0, -1 = default), the tile-local product (1; 0, -1 = default: no), and
        the fused step, the update folded into the product (1; 0 two launches; -1 = default: fused on cells
        of at most 8 entries per row)."""
        self._ck(self._L.gbn_set_kernel_variant(self._h, col_unroll, stage_values, min_blocks, field_table, tiled,
                                                fused))

    @property
    def launches(self):
        return self._L.gbn_launch_count(self._h)

    def last_timing(self):
        ms, n = C.c_double(), C.c_int64()
        self._ck(self._L.gbn_last_timing(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def kernel_timing(self):
        """(sparse-product ms, update ms) per launch, averaged over the first steps of the last call."""
        a, b = C.c_double(), C.c_double()
        self._ck(self._L.gbn_last_kernel_timing(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    # ---------------------------------------------------------------- geometry / search
    def set_geometry(self, rat, species, layer, ucell):
        n = len(species)
        self._ck(self._L.gbn_set_geometry(self._h, n, _c(rat, np.float64), _c(species, np.int32),
                                          _c(layer, np.int32), _c(ucell, np.float64)))
        self.n = n

    def neighbours(self, cut2intra, cut2inter, second_layer=False, tables=True):
        mx, tot = C.c_int32(), C.c_int64()
        self._ck(self._L.gbn_neighbours(self._h, cut2intra, cut2inter, int(second_layer), C.byref(mx), C.byref(tot)))
        self.max_neigh = mx.value
        self.neighbours_total = tot.value
        if not tables:
            return dict(max_neigh=mx.value, total=tot.value)
        n = self.n
        nn = np.zeros(n, np.int32)
        nl = np.zeros(n * mx.value, np.int32)
        nd = np.zeros(n * mx.value * 3, np.float64)
        nc = np.zeros(n * mx.value * 3, np.int32)
        self._ck(self._L.gbn_get_neighbours(self._h, nn, nl, nd, nc))
        return dict(max_neigh=mx.value, total=tot.value, nneigh=nn, nlist=nl.reshape(n, -1),
                    neighd=nd.reshape(n, -1, 3), ncell=nc.reshape(n, -1, 3))

    def tables(self):
        """Nneigh(N) and NList(maxNeigh,N) of the current neighbour list (reference layout)."""
        nn = np.zeros(self.n, np.int32)
        nl = np.zeros(self.n * self.max_neigh, np.int32)
        self._ck(self._L.gbn_get_neighbours(self._h, nn, nl, None, None))
        return dict(max_neigh=self.max_neigh, nneigh=nn, nlist=nl.reshape(self.n, -1))

    # ---------------------------------------------------------------- Hamiltonian
    def assemble(self, model, rat_onsite=None, rat_hop=None, uniform=None):
        self._ck(self._L.gbn_assemble(self._h, C.byref(model),
                                      None if rat_onsite is None else _c(rat_onsite, np.float64),
                                      None if rat_hop is None else _c(rat_hop, np.float64),
                                      None if uniform is None else _c(uniform, np.float64)))

    def peierls(self, flux):
        self._ck(self._L.gbn_peierls(self._h, flux))

    def hamiltonian(self):
        h0 = np.zeros(self.n, np.float64)
        hop = np.zeros(self.n * self.max_neigh, np.complex128)
        self._ck(self._L.gbn_get_hamiltonian(self._h, h0, hop))
        return h0, hop.reshape(self.n, -1)

    def onsite_layers(self):
        """(H0Bottom, H0Top) of the assembled model: the on-site energies after the first moire's terms
        (0 without the moire branch) and H0 - H0Bottom with the second moire (0 without it)."""
        bottom = np.zeros(self.n, np.float64)
        top = np.zeros(self.n, np.float64)
        self._ck(self._L.gbn_get_onsite_layers(self._h, bottom, top))
        return bottom, top

    def load_hamiltonian(self, nneigh, nlist, hopp, h0):
        n = len(h0)
        mx = np.asarray(nlist).reshape(n, -1).shape[1]
        self._ck(self._L.gbn_load_hamiltonian(self._h, n, mx, _c(nneigh, np.int32), _c(nlist, np.int32),
                                              _c(hopp, np.complex128), _c(h0, np.float64)))
        self.n, self.max_neigh = n, mx

    def check_hamiltonian(self):
        """(non-finite hoppings, non-finite on-site, first atom, entries without reverse, pairs, max asymmetry)"""
        out = np.zeros(5, np.int64)
        mx = C.c_double()
        self._ck(self._L.gbn_check_hamiltonian(self._h, out, C.byref(mx)))
        return tuple(int(x) for x in out) + (mx.value,)

    def haldane(self, aG, t2, phase, paper=False, layer_mask=0):
        """HamHopHaldane on the current hoppings (after peierls): t2 in g0, phase in rad."""
        self._ck(self._L.gbn_haldane(self._h, aG, t2, phase, int(paper), layer_mask))

    def kubo_tevol(self, c, ac, bc, psi, zupsi, nt, nwr, nrecurs, direction=1, precision=GBN_FP64):
        """KuboTEvol on the device: returns (psi, zupsi, norms [nrhs, nt//nwr], a, b [nrhs, nt//nwr, nrecurs])."""
        p = np.ascontiguousarray(np.atleast_2d(psi), np.complex128).copy()
        z = np.ascontiguousarray(np.atleast_2d(zupsi), np.complex128).copy()
        nrhs, nw = p.shape[0], nt // nwr
        norms = np.zeros((nrhs, max(nw, 1)))
        a = np.zeros((nrhs, max(nw, 1), nrecurs))
        b = np.zeros((nrhs, max(nw, 1), nrecurs))
        cc = _c(c, np.complex128)
        self._ck(self._L.gbn_kubo_tevol(self._h, precision, nrhs, cc, len(cc), ac, bc, direction, nt, nwr, nrecurs,
                                        p.reshape(-1), z.reshape(-1), norms.reshape(-1), a.reshape(-1), b.reshape(-1)))
        return p, z, norms[:, :nw], a[:, :nw], b[:, :nw]

    def set_images(self, ncell):
        """neighCell of the loaded neighbour list (for peierls after load_hamiltonian)."""
        self._ck(self._L.gbn_set_images(self._h, _c(ncell, np.int32)))

    def set_neighd(self, neighd):
        self._ck(self._L.gbn_set_neighd(self._h, _c(neighd, np.float64)))

    # ---------------------------------------------------------------- recursion
    def lanczos(self, psi0, nsteps, precision=GBN_FP64):
        """psi0: complex [nrhs, N] start vectors; nsteps: int or [nrhs]; returns a, b [nrhs, nmax]."""
        psi = np.ascontiguousarray(np.atleast_2d(psi0), np.complex128)
        nrhs = psi.shape[0]
        ns = np.broadcast_to(np.asarray(nsteps, np.int32), (nrhs,)).copy()
        nmax = int(ns.max())
        a = np.zeros((nrhs, nmax))
        b = np.zeros((nrhs, nmax))
        self._ck(self._L.gbn_lanczos(self._h, precision, nrhs, psi.reshape(-1), ns, nmax, a.reshape(-1), b.reshape(-1)))
        return a, b

    def lanczos_phases(self, u, nsteps, precision=GBN_FP64):
        """u: uniform draws [nrhs, N]: start vectors exp(2 pi i u)/sqrt(N)."""
        uu = np.ascontiguousarray(np.atleast_2d(u), np.float64)
        nrhs = uu.shape[0]
        ns = np.broadcast_to(np.asarray(nsteps, np.int32), (nrhs,)).copy()
        nmax = int(ns.max())
        a = np.zeros((nrhs, nmax))
        b = np.zeros((nrhs, nmax))
        self._ck(self._L.gbn_lanczos_phases(self._h, precision, nrhs, uu.reshape(-1), ns, nmax, a.reshape(-1),
                                            b.reshape(-1)))
        return a, b

    def lanczos_fields(self, m, u, nsteps, precision=GBN_MIXED):
        """Random-phase recursions of many fields in one batch from the field-free assembled Hamiltonian:
        m[nfields] flux quanta, u[nfields, nvec, N] draws, nsteps int or [nfields, nvec];
        returns a, b [nfields, nvec, nmax]."""
        mm = _c(m, np.int32)
        uu = np.ascontiguousarray(u, np.float64)
        nf, nv = uu.shape[0], uu.shape[1]
        assert len(mm) == nf
        ns = np.broadcast_to(np.asarray(nsteps, np.int32), (nf, nv)).copy()
        nmax = int(ns.max())
        a = np.zeros((nf, nv, nmax))
        b = np.zeros((nf, nv, nmax))
        self._ck(self._L.gbn_lanczos_fields(self._h, precision, nf, mm, nv, uu.reshape(-1), ns.reshape(-1), nmax,
                                            a.reshape(-1), b.reshape(-1)))
        return a, b

    def lanczos_sites(self, sites, nsteps, precision=GBN_FP64):
        """Local DOS recursion of single atoms: unit start vectors on sites (1-based), one per vector."""
        st = np.ascontiguousarray(np.atleast_1d(sites), np.int64)
        ns = np.broadcast_to(np.asarray(nsteps, np.int32), (len(st),)).copy()
        nmax = int(ns.max())
        a = np.zeros((len(st), nmax))
        b = np.zeros((len(st), nmax))
        self._ck(self._L.gbn_lanczos_sites(self._h, precision, len(st), st, ns, nmax, a.reshape(-1), b.reshape(-1)))
        return a, b

    def lanczos_sets(self, set_of_atom, u, assumed, nsteps, precision=GBN_FP64):
        """Layer / layer-and-species DOS recursion: random phases on each set of atoms (gbn_lanczos_sets)."""
        so = _c(set_of_atom, np.int32)
        asm = np.ascontiguousarray(np.atleast_1d(assumed), np.float64)
        ns = np.broadcast_to(np.asarray(nsteps, np.int32), (len(asm),)).copy()
        nmax = int(ns.max())
        a = np.zeros((len(asm), nmax))
        b = np.zeros((len(asm), nmax))
        self._ck(self._L.gbn_lanczos_sets(self._h, precision, len(asm), so, _c(u, np.float64), asm, ns, nmax,
                                          a.reshape(-1), b.reshape(-1)))
        return a, b

    def stage_phases(self, u, precision=GBN_MIXED):
        uu = np.ascontiguousarray(np.atleast_2d(u), np.float64)
        self._staged = uu.shape[0]
        self._ck(self._L.gbn_stage_phases(self._h, precision, uu.shape[0], uu.reshape(-1)))

    def run_staged(self, nmax, a=None, b=None):
        self._ck(self._L.gbn_run_staged(self._h, nmax, None if a is None else a.reshape(-1),
                                        None if b is None else b.reshape(-1)))

    def cf_dos(self, a, b, eta, n_en, emin, emax, nsteps=None, norm=None):
        a = np.ascontiguousarray(np.atleast_2d(a), np.float64)
        b = np.ascontiguousarray(np.atleast_2d(b), np.float64)
        nrhs, nmax = a.shape
        ns = None if nsteps is None else np.broadcast_to(np.asarray(nsteps, np.int32), (nrhs,)).copy()
        nm = None if norm is None else np.broadcast_to(np.asarray(norm, np.float64), (nrhs,)).copy()
        e = np.zeros(n_en + 1)
        dos = np.zeros((nrhs, n_en + 1))
        self._ck(self._L.gbn_cf_dos(self._h, nrhs, a.reshape(-1), b.reshape(-1), ns, nmax, eta, n_en, emin, emax, nm,
                                    e, dos.reshape(-1)))
        return e, dos

    # ---------------------------------------------------------------- gradient
    def dos_gradient(self, model, g0, u, nrecurs, eta, n_en, emin, emax, target, checkpoint=32,
                     precision=GBN_FP64):
        """Loss, dL/d(t, Vpp_sigma0, delta, w) and the DOS of the assembled Hamiltonian (see gbn_dos_gradient;
        precision GBN_MIXED: the FP32-vector variant, gbn_dos_gradient_prec)."""
        loss = C.c_double()
        grad = np.zeros(4)
        dos = np.zeros(n_en + 1)
        a = np.zeros(nrecurs)
        b = np.zeros(nrecurs)
        self._ck(self._L.gbn_dos_gradient_prec(self._h, precision, C.byref(model), g0, _c(u, np.float64), nrecurs,
                                               checkpoint, eta, n_en, emin, emax, _c(target, np.float64),
                                               C.byref(loss), grad, dos, a, b))
        return loss.value, grad, dos, a, b

    # ---------------------------------------------------------------- Chebyshev
    def cheb_evolve(self, c, ac, bc, z, precision=GBN_FP64):
        zz = np.ascontiguousarray(np.atleast_2d(z), np.complex128).copy()
        cc = _c(c, np.complex128)
        self._ck(self._L.gbn_cheb_evolve(self._h, precision, zz.shape[0], cc, len(cc), ac, bc, zz.reshape(-1)))
        return zz

    def kubo_evol(self, c, ac, bc, psi, zupsi, direction=1, precision=GBN_FP64):
        p = np.ascontiguousarray(np.atleast_2d(psi), np.complex128).copy()
        z = np.ascontiguousarray(np.atleast_2d(zupsi), np.complex128).copy()
        cc = _c(c, np.complex128)
        self._ck(self._L.gbn_kubo_evol(self._h, precision, p.shape[0], cc, len(cc), ac, bc, direction, p.reshape(-1),
                                       z.reshape(-1)))
        return p, z


def cheb_interval(a, b):
    """KuboInterval: spectral centre ac and scale bc from recursion coefficients a, b (host)."""
    a = _c(a, np.float64)
    b = _c(b, np.float64)
    ac, bc = C.c_double(), C.c_double()
    rc = lib().gbn_cheb_interval(a, b, len(a), C.byref(ac), C.byref(bc))
    if rc != 0:
        raise GbnError(rc, "gbn_cheb_interval failed")
    return ac.value, bc.value


def cheb_coef(dt, ac, bc, npol):
    """KuboCn: the npol complex propagator coefficients for the time step dt (host)."""
    c = np.zeros(npol, np.complex128)
    rc = lib().gbn_cheb_coef(dt, ac, bc, npol, c)
    if rc != 0:
        raise GbnError(rc, "gbn_cheb_coef failed")
    return c


def pdos_atoms(p, rat, species, layer, ucell):
    """Atoms (1-based) of a single-atom Kubo.PDOS selection and the positions written to their coords files."""
    r = _c(rat, np.float64).reshape(-1)
    n = len(r) // 3
    sp, ly, uc = _c(species, np.int32), _c(layer, np.int32), _c(ucell, np.float64)
    cnt = C.c_int64()
    rc = lib().gbn_pdos_atoms(C.byref(p), n, r, sp, ly, uc, 0, C.byref(cnt), None, None)
    if rc:
        raise GbnError(rc, "bad PDOS selection")
    atoms = np.zeros(max(cnt.value, 1), np.int64)
    coords = np.zeros(3 * max(cnt.value, 1))
    rc = lib().gbn_pdos_atoms(C.byref(p), n, r, sp, ly, uc, cnt.value, C.byref(cnt), atoms, coords)
    if rc:
        raise GbnError(rc, "bad PDOS selection")
    return atoms[:cnt.value], coords.reshape(-1, 3)[:cnt.value]


def pdos_sets(p, species, layer, cap=4096):
    """Sets of a layer Kubo.PDOS selection: (set_of_atom, layers, species, assumed counts)."""
    sp, ly = _c(species, np.int32), _c(layer, np.int32)
    so = np.zeros(len(sp), np.int32)
    sl, ss, asm = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap)
    ns = C.c_int32()
    rc = lib().gbn_pdos_sets(C.byref(p), len(sp), sp, ly, cap, C.byref(ns), so, sl, ss, asm)
    if rc:
        raise GbnError(rc, "bad PDOS selection")
    k = ns.value
    return so, sl[:k], ss[:k], asm[:k]


def build_cell(kind, aG=2.46, cell_size=50, super_cell=1, m=(0, 0, 0, 0), height=40.0, d_interlayer=3.35,
               add_shift=0, shift_factor=0.0):
    """Atoms of a Graphene or moire bilayer cell (TwistedBilayerBasedOnMoireCell,
    MoireEncapsulatedBilayerBasedOnMoireCell), in the reference's order; add_shift 1 / 2 offsets the second
    layer by the Bernal / bridge offset plus shift_factor [Ang] along a1+a2."""
    p = Cell(kind, cell_size, super_cell, (C.c_int32 * 4)(*m), aG, height, d_interlayer, add_shift, shift_factor)
    n = C.c_int64()
    rc = lib().gbn_cell_atoms(C.byref(p), C.byref(n))
    if rc:
        raise GbnError(rc, "invalid cell")
    n = n.value
    ucell = np.zeros(9)
    rat = np.zeros(3 * n)
    species = np.zeros(n, np.int32)
    layer = np.zeros(n, np.int32)
    tw = C.c_double()
    rc = lib().gbn_build_cell(C.byref(p), ucell, rat, species, layer, C.byref(tw))
    if rc:
        raise GbnError(rc, "invalid cell")
    return dict(n=n, ucell=ucell, rat=rat.reshape(n, 3), species=species, layer=layer, twist=tw.value)


def cart_roundtrip(rat, ucell):
    r = np.ascontiguousarray(rat, np.float64).reshape(-1).copy()
    rc = lib().gbn_cart_roundtrip(len(r) // 3, np.ascontiguousarray(ucell, np.float64), r)
    if rc:
        raise GbnError(rc, "bad arguments")
    return r.reshape(-1, 3)


def rng_uniform(seed, n):
    """GNU Fortran random_number draws after random_seed(PUT=[seed]*8)."""
    out = np.zeros(n)
    rc = lib().gbn_rng_uniform(seed, n, out)
    if rc:
        raise GbnError(rc, "bad arguments")
    return out


def version():
    return lib().gbn_version().decode()


def kubo_msd(norms, nwr, dt_fs):
    """Mean-square displacement and diffusivity from the norms [nrhs][nw] of Context.kubo_tevol (see
    gbn_kubo_msd): (t [fs], MSD [Ang^2], MSD / t, d MSD / dt [Ang^2 / fs])."""
    nr = np.ascontiguousarray(np.atleast_2d(norms), np.float64)
    nrhs, nw = nr.shape
    t, msd, dr, ds = (np.zeros(nw) for _ in range(4))
    rc = lib().gbn_kubo_msd(nrhs, nw, nwr, dt_fs, nr.reshape(-1), t, msd, dr, ds)
    if rc:
        raise GbnError(rc, "bad arguments")
    return t, msd, dr, ds
