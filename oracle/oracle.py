"""ctypes binding of the CPU oracle (oracle/liboracle.so) -- TEST INFRASTRUCTURE ONLY.

The oracle restates the reference's Fortran algorithms in C (see oracle.h).  It is the
checker of the CUDA library: only tests/, __graft_entry__.smoke() and the CPU-baseline leg
of bench.py import this module.  Build it with `make -C oracle`.

Parity status: pinned against the reference's own golden data -- the Hamiltonian
fingerprints of tests/regression/model_survey_reference.json and the recursion DOS tables
of examples/06 and examples/07 (see tests/golden/).
"""

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

GRAPHENE, TBG_MOIRE_CELL = 0, 1
INTRA_DEFAULT, INTRA_F2G2_SL = 0, 1
INTER_NONE, INTER_TWO_CENTRE = 0, 1
ONSITE_NONE, ONSITE_H0_AND_HZ, ONSITE_ONLY_H0, ONSITE_ONLY_HZ, ONSITE_NO_H0_AND_HZ = range(5)


class GeomParams(C.Structure):
    _fields_ = [("kind", C.c_int32), ("cell_size", C.c_int32), ("super_cell", C.c_int32),
                ("m", C.c_int32 * 4), ("aG", C.c_double), ("height", C.c_double),
                ("d_interlayer", C.c_double), ("add_shift", C.c_int32), ("shift_factor", C.c_double)]


class Model(C.Structure):
    _fields_ = [
        ("aG", C.c_double), ("tbnn", C.c_int32), ("gn_cc", C.c_double * 8), ("nradii", C.c_double * 8),
        ("intralayer", C.c_int32), ("tksl", C.c_double * 8),
        ("moire_offdiag", C.c_int32), ("moire_mid", C.c_int32), ("moire_twisted", C.c_int32),
        ("moire_onsite", C.c_int32), ("eps", C.c_double), ("twist_rad", C.c_double), ("shift1", C.c_double),
        ("sign1", C.c_double), ("sign2", C.c_double), ("C0", C.c_double), ("Cz", C.c_double), ("Cab", C.c_double),
        ("Phi0", C.c_double), ("Phiz", C.c_double), ("Phiab", C.c_double),
        ("interlayer", C.c_int32), ("vpppi0", C.c_double), ("vppsigma0", C.c_double), ("bl_delta", C.c_double),
        ("d_interlayer", C.c_double), ("aCC", C.c_double), ("g_intlay", C.c_double),
        ("anderson", C.c_int32), ("anderson_w", C.c_double), ("seed", C.c_int32), ("e0_c", C.c_double),
        ("koshino_sr", C.c_int32), ("renormalize_coupling", C.c_int32), ("coupling_factor", C.c_double),
        ("inter_smooth_w", C.c_double), ("inter_cut_rho", C.c_double),
        ("second_moire", C.c_int32), ("eps_factor", C.c_double), ("twisted2", C.c_int32), ("twist2_rad", C.c_double),
        ("rotate_first", C.c_int32), ("shift2", C.c_double), ("shift2_x", C.c_double), ("shift2_y", C.c_double),
        ("encapsulated", C.c_int32), ("bl_bottom_rad", C.c_double), ("bl_top_rad", C.c_double),
        ("tau", C.c_double * 4), ("deact_upper", C.c_int32), ("deact_uppers", C.c_int32), ("bernal", C.c_int32),
        ("tbl", C.c_double * 7),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: run `make -C {HERE}`")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _p(dtype):
    return np.ctypeslib.ndpointer(dtype=dtype, flags="C_CONTIGUOUS")


def _declare(L):
    d, i32, i64 = C.c_double, C.c_int32, C.c_int64
    L.orc_rng_fill.argtypes = [i32, i64, _p(np.float64)]
    L.orc_geom_natoms.argtypes = [C.POINTER(GeomParams)]
    L.orc_geom_natoms.restype = i64
    L.orc_geom_build.argtypes = [C.POINTER(GeomParams), _p(np.float64), _p(np.float64), _p(np.int32),
                                 _p(np.int32), C.POINTER(d)]
    L.orc_geom_roundtrip.argtypes = [i64, _p(np.float64), _p(np.float64)]
    L.orc_cell_area.argtypes = [_p(np.float64)]
    L.orc_cell_area.restype = d
    L.orc_neigh_search.argtypes = [i64, _p(np.float64), _p(np.float64), d, d, i32]
    L.orc_neigh_search.restype = C.c_void_p
    L.orc_nbr_max.argtypes = [C.c_void_p]
    L.orc_nbr_max.restype = i32
    L.orc_nbr_copy.argtypes = [C.c_void_p, _p(np.int32), _p(np.int32), _p(np.float64), _p(np.int32)]
    L.orc_nbr_free.argtypes = [C.c_void_p]
    L.orc_onsite.argtypes = [C.POINTER(Model), i64, _p(np.float64), _p(np.int32), _p(np.int32), _p(np.float64)]
    L.orc_onsite_layers.argtypes = [C.POINTER(Model), i64, _p(np.float64), _p(np.int32), _p(np.int32), _p(np.float64),
                                    _p(np.float64)]
    L.orc_hopping.argtypes = [C.POINTER(Model), i64, _p(np.float64), _p(np.int32), _p(np.int32), i32,
                              _p(np.int32), _p(np.int32), _p(np.float64), _p(np.complex128)]
    L.orc_haldane.argtypes = [i64, _p(np.int32), _p(np.int32), i32, _p(np.int32), _p(np.int32), _p(np.float64), C.c_double,
                              C.c_double, C.c_double, i32, C.c_uint32, _p(np.float64)]
    L.orc_haldane.restype = i64
    L.orc_check_hamiltonian.argtypes = [i64, i32, _p(np.int32), _p(np.int32), _p(np.int32), _p(np.float64),
                                        _p(np.float64), _p(np.int64), C.POINTER(C.c_double)]
    L.orc_peierls.argtypes = [i64, _p(np.float64), _p(np.float64), i32, _p(np.int32), _p(np.int32),
                              _p(np.int32), d, _p(np.complex128)]
    L.orc_init_wf.argtypes = [i64, i32, _p(np.complex128)]
    L.orc_recursion.argtypes = [i64, i32, _p(np.int32), _p(np.int32), _p(np.complex128), _p(np.float64),
                                _p(np.complex128), i32, _p(np.float64), _p(np.float64), i32]
    L.orc_frac.argtypes = [_p(np.float64), _p(np.float64), i32, d, d, i32, d, d, _p(np.float64), _p(np.float64)]
    L.orc_interval.argtypes = [_p(np.float64), _p(np.float64), i32, C.POINTER(d), C.POINTER(d)]
    L.orc_interval.restype = C.c_int
    L.orc_cheb_coef.argtypes = [d, d, d, i32, _p(np.complex128)]
    L.orc_cheb_coef.restype = C.c_int
    L.orc_cheb_evolve.argtypes = [i64, i32, _p(np.int32), _p(np.int32), _p(np.complex128), _p(np.float64),
                                  _p(np.complex128), i32, d, d, _p(np.complex128)]
    L.orc_evol.argtypes = [i64, i32, _p(np.int32), _p(np.int32), _p(np.float64), _p(np.complex128),
                           _p(np.float64), _p(np.complex128), i32, d, d, i32, _p(np.complex128),
                           _p(np.complex128)]


# ----------------------------------------------------------------------------- wrappers

def rng_draws(seed, n):
    out = np.empty(n, np.float64)
    lib().orc_rng_fill(seed, n, out)
    return out


def geometry(kind, aG=2.46, cell_size=50, super_cell=1, m=(0, 0, 0, 0), height=40.0, d_interlayer=3.35,
             add_shift=0, shift_factor=0.0):
    p = GeomParams(kind, cell_size, super_cell, (C.c_int32 * 4)(*m), aG, height, d_interlayer, add_shift, shift_factor)
    n = lib().orc_geom_natoms(C.byref(p))
    ucell = np.zeros(9, np.float64)
    rat = np.zeros(3 * n, np.float64)
    species = np.zeros(n, np.int32)
    layer = np.zeros(n, np.int32)
    tw = C.c_double(0.0)
    if lib().orc_geom_build(C.byref(p), ucell, rat, species, layer, C.byref(tw)) != 0:
        raise ValueError("unsupported geometry")
    return dict(n=n, ucell=ucell, rat=rat.reshape(n, 3), species=species, layer=layer, twist=tw.value)


def roundtrip(rat, ucell):
    r = np.ascontiguousarray(rat, np.float64).reshape(-1).copy()
    lib().orc_geom_roundtrip(len(r) // 3, np.ascontiguousarray(ucell), r)
    return r.reshape(-1, 3)


def cell_area(ucell):
    return lib().orc_cell_area(np.ascontiguousarray(ucell, np.float64))


def neighbours(rat, ucell, cut2intra, cut2inter, second_layer=False):
    r = np.ascontiguousarray(rat, np.float64).reshape(-1)
    n = len(r) // 3
    h = lib().orc_neigh_search(n, r, np.ascontiguousarray(ucell), cut2intra, cut2inter, int(second_layer))
    if not h:
        raise ValueError("neighbour search refused the cell")
    try:
        mx = lib().orc_nbr_max(h)
        nn = np.zeros(n, np.int32)
        nl = np.zeros(n * mx, np.int32)
        nd = np.zeros(n * mx * 3, np.float64)
        nc = np.zeros(n * mx * 3, np.int32)
        lib().orc_nbr_copy(h, nn, nl, nd, nc)
    finally:
        lib().orc_nbr_free(h)
    return dict(max_neigh=mx, nneigh=nn, nlist=nl.reshape(n, mx), neighd=nd.reshape(n, mx, 3),
                ncell=nc.reshape(n, mx, 3))


def onsite(model, rat, species, layer):
    n = len(species)
    h0 = np.zeros(n, np.float64)
    lib().orc_onsite(C.byref(model), n, np.ascontiguousarray(rat, np.float64).reshape(-1), species, layer, h0)
    return h0


def onsite_layers(model, rat, species, layer):
    """(H0, H0Bottom, H0Top) of HamOnSite (ham.F90:2703, 3639): H0Bottom is H0 after the first moire's
    terms when the moire branch runs (0 otherwise), H0Top = H0 - H0Bottom when the second moire runs."""
    n = len(species)
    h0, bottom = np.zeros(n, np.float64), np.zeros(n, np.float64)
    lib().orc_onsite_layers(C.byref(model), n, np.ascontiguousarray(rat, np.float64).reshape(-1), species, layer,
                            h0, bottom)
    top = h0 - bottom if model.second_moire else np.zeros(n, np.float64)
    return h0, bottom, top


def hopping(model, rat, species, layer, nb):
    n = len(species)
    mx = nb["max_neigh"]
    hop = np.zeros(n * mx, np.complex128)
    lib().orc_hopping(C.byref(model), n, np.ascontiguousarray(rat, np.float64).reshape(-1), species, layer, mx,
                      nb["nneigh"], np.ascontiguousarray(nb["nlist"]).reshape(-1),
                      np.ascontiguousarray(nb["neighd"]).reshape(-1), hop)
    return hop.reshape(n, mx)


def haldane(species, layer, nb, aG, t2, phase, hop, paper=False, layer_mask=0):
    """HamHopHaldane on the hoppings (returns the new hoppings and the bonds without a chirality)."""
    n = len(nb["nneigh"])
    h = np.ascontiguousarray(hop, np.complex128).reshape(-1).copy()
    miss = lib().orc_haldane(n, np.ascontiguousarray(species, np.int32), np.ascontiguousarray(layer, np.int32),
                             nb["max_neigh"], nb["nneigh"], np.ascontiguousarray(nb["nlist"]).reshape(-1),
                             np.ascontiguousarray(nb["neighd"]).reshape(-1), aG, t2, phase, int(paper), layer_mask,
                             h.view(np.float64))
    return h.reshape(n, nb["max_neigh"]), miss


def check_hamiltonian(nb, hop, h0):
    """(non-finite hoppings, non-finite on-site, first atom, entries without reverse, pairs, max asymmetry)"""
    n = len(h0)
    out = np.zeros(5, np.int64)
    mx = C.c_double()
    h = np.ascontiguousarray(hop, np.complex128).reshape(-1)
    lib().orc_check_hamiltonian(n, nb["max_neigh"], nb["nneigh"], np.ascontiguousarray(nb["nlist"]).reshape(-1),
                                np.ascontiguousarray(nb["ncell"]).reshape(-1), h.view(np.float64),
                                np.ascontiguousarray(h0, np.float64), out, C.byref(mx))
    return tuple(int(x) for x in out) + (mx.value,)


def peierls(rat, ucell, nb, flux, hop):
    n = len(nb["nneigh"])
    h = np.ascontiguousarray(hop, np.complex128).reshape(-1).copy()
    lib().orc_peierls(n, np.ascontiguousarray(rat, np.float64).reshape(-1), np.ascontiguousarray(ucell),
                      nb["max_neigh"], nb["nneigh"], np.ascontiguousarray(nb["nlist"]).reshape(-1),
                      np.ascontiguousarray(nb["ncell"]).reshape(-1), flux, h)
    return h.reshape(n, nb["max_neigh"])


def init_wf(n, seed):
    psi = np.zeros(n, np.complex128)
    lib().orc_init_wf(n, seed, psi)
    return psi


def recursion(nb, hop, h0, psi, nrecurs, nthreads=0):
    n = len(h0)
    a = np.zeros(nrecurs, np.float64)
    b = np.zeros(nrecurs, np.float64)
    lib().orc_recursion(n, nb["max_neigh"], nb["nneigh"], np.ascontiguousarray(nb["nlist"]).reshape(-1),
                        np.ascontiguousarray(hop, np.complex128).reshape(-1), np.ascontiguousarray(h0, np.float64),
                        np.ascontiguousarray(psi, np.complex128), nrecurs, a, b, nthreads)
    return a, b


def frac(a, b, eps, n_en, emin, emax, norm=1.0):
    e = np.zeros(n_en + 1, np.float64)
    dos = np.zeros(n_en + 1, np.float64)
    lib().orc_frac(np.ascontiguousarray(a), np.ascontiguousarray(b), len(a), norm, eps, n_en, emin, emax, e, dos)
    return e, dos


def interval(a, b):
    ac, bc = C.c_double(), C.c_double()
    if lib().orc_interval(np.ascontiguousarray(a), np.ascontiguousarray(b), len(a), C.byref(ac), C.byref(bc)):
        raise RuntimeError("tridiagonal eigenvalues did not converge")
    return ac.value, bc.value


def cheb_coef(dt, ac, bc, npol):
    c = np.zeros(npol, np.complex128)
    if lib().orc_cheb_coef(dt, ac, bc, npol, c):
        raise RuntimeError("Chebyshev coefficients: QL did not converge")
    return c


def cheb_evolve(nb, hop, h0, c, ac, bc, z):
    zz = np.ascontiguousarray(z, np.complex128).copy()
    lib().orc_cheb_evolve(len(h0), nb["max_neigh"], nb["nneigh"], np.ascontiguousarray(nb["nlist"]).reshape(-1),
                          np.ascontiguousarray(hop, np.complex128).reshape(-1), np.ascontiguousarray(h0),
                          np.ascontiguousarray(c, np.complex128), len(c), ac, bc, zz)
    return zz


def evol(nb, hop, h0, c, ac, bc, psi, zupsi, direction=1):
    p = np.ascontiguousarray(psi, np.complex128).copy()
    z = np.ascontiguousarray(zupsi, np.complex128).copy()
    lib().orc_evol(len(h0), nb["max_neigh"], nb["nneigh"], np.ascontiguousarray(nb["nlist"]).reshape(-1),
                   np.ascontiguousarray(nb["neighd"]).reshape(-1), np.ascontiguousarray(hop, np.complex128).reshape(-1),
                   np.ascontiguousarray(h0), np.ascontiguousarray(c, np.complex128), len(c), ac, bc, direction, p, z)
    return p, z


def dos_loss(model, rat_hop, species, layer, nb, h0, u, nrecurs, eta, n_en, emin, emax, target, nthreads=0):
    """L = sum_E (DOS(E) - target(E))^2 of the DOS-fitting problem, all in the oracle: hoppings of `model`
    (orc_hopping, with the smooth interlayer cutoff), the FP64 three-pass recursion (KuboRecursion) of the
    random-phase state exp(2 pi i u) / sqrt(N), and the continued fraction (KuboFrac).  Returns (L, DOS)."""
    hop = hopping(model, rat_hop, species, layer, nb)
    n = len(species)
    psi = np.exp(2j * np.pi * np.asarray(u, np.float64)) / np.sqrt(n)
    a, b = recursion(nb, hop, h0, psi, nrecurs, nthreads)
    _, dos = frac(a, b, eta, n_en, emin, emax)
    t = np.asarray(target, np.float64)
    return float(((dos - t) ** 2).sum()), dos
