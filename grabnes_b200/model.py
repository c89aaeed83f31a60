"""Gendata.in keys -> inputs of the C ABI (cell, search radii, gbn_model, fields, Kubo parameters).

Defaults and unit conversions follow the readers of the reference (gjung-group/grabnes):
  cell / atoms      lanczosKuboCode/Src/cell.F90:16-140, 207-240; atoms.F90:124-230, 330-380
  TB parameters     tbpar.f90:20-130 (g0 = TB.Hopping, default -3.72 aG + 12.14 eV)
  search radii      ham.F90:542-606 (NeighShellCutoff2, Neigh.LayerDistFactor), neigh.F90:27-31, 348-381
  hopping keys      ham.F90:5720-5941 (Moire.PotCab, Interlayer.Vpppi0/Vppsigma0/BLdelta, ...)
  on-site keys      ham.F90:2099-2140, 2646-2690 (Moire.*), 1237-1248 and 13260-13283 (Anderson, eV)
  fields            magf.F90:20-146 (B = m Phi0 / A), ham.F90:5657 (flux = B pi / Phi0)
  Kubo              calc.F90:161-188 (energies and broadening in eV, divided by g0)
Keys are given here in their short (former) form without section, matching case-insensitively
with '_' and '-' ignored, as the reference's input library does.
"""

import math

from . import CELL_GRAPHENE, CELL_TBG_MOIRE, Model

def _shared_table():
    """The key aliases, shell radii and constants shared with the drop-in driver
    (grabnes_b200/driver/gendata_keys.inc, the one list of them)."""
    import os
    import re
    text = open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "driver", "gendata_keys.inc")).read()
    text = re.sub(r"//[^\n]*", "", text)
    aliases = dict(re.findall(r'GBN_ALIAS\("([^"]+)",\s*"([^"]+)"\)', text))
    radii = [float(x) for x in re.findall(r"GBN_SHELL_RADIUS\(([^)]+)\)", text)]
    consts = {k: float(v) for k, v in re.findall(r"GBN_CONST\((\w+),\s*([^)]+)\)", text)}
    return aliases, radii, consts


_ALIASES, SHELL_RADIUS, _CONSTS = _shared_table()
FLUXQ = _CONSTS["HPLANCK"] / _CONSTS["QE"]   # h/e of constants.f90
F2G2_SINGLE_LAYER = {2: -0.2354, 3: 0.1877, 4: 0.0, 5: -0.0633, 6: 0.0, 7: 0.0}   # ham.F90:8331-8350 [eV]


# former (section-less) names of the keys read here: lanczosKuboCode/Src/MIO/input_aliases.inc
FORMER = dict(_ALIASES)


def _norm(k):
    return k.lower().replace("_", "").replace("-", "")


class Keys:
    """Input keys; a key is found by its present Section.Name or by its former name."""

    def __init__(self, keys):
        self._k = {}
        for k, v in keys.items():
            self._k.setdefault(_norm(k), v)   # the first occurrence wins

    def has(self, name):
        return _norm(name) in self._k or _norm(FORMER.get(name, "\0")) in self._k

    def get(self, name, default):
        for cand in (name, FORMER.get(name)):
            if cand is not None and _norm(cand) in self._k:
                return self._k[_norm(cand)]
        return default


def job_from_keys(keys):
    k = Keys(keys)
    g = k.get
    aG = g("Structure.LatticeParameter", 2.46)
    system = g("Run.TypeOfSystem", "Graphene")
    kind = {"graphene": CELL_GRAPHENE, "twistedbilayerbasedonmoirecell": CELL_TBG_MOIRE,
            "moireencapsulatedbilayerbasedonmoirecell": CELL_TBG_MOIRE}.get(system.lower())
    if kind is None:
        raise ValueError(f"Run.TypeOfSystem {system} is not on the recursion path of this library")
    encapsulated = system.lower() == "moireencapsulatedbilayerbasedonmoirecell"
    add_shift, shift_factor = 0, 0.0
    if g("Structure.TwistedBLAddShift", False):   # atoms.F90:352-366
        if g("Structure.BernalShift", False):
            add_shift = 1
        elif g("Structure.BridgeShift", False):
            add_shift = 2
        else:
            raise ValueError("TwistedBLAddShift needs BernalShift or BridgeShift to say which shift is added")
        shift_factor = g("Structure.BilayerShiftFactor", 0.0)
    cell = dict(kind=kind, aG=aG, cell_size=g("Structure.CellSize", 50), super_cell=g("Structure.SuperCell", 1),
                m=tuple(g("Structure.MoireCellParameters", (0, 0, 0, 0))), height=g("Structure.CellHeight", 40.0),
                d_interlayer=g("Structure.InterlayerDistance", 3.35), add_shift=add_shift, shift_factor=shift_factor)
    g0 = g("TB.Hopping", -3.72 * aG + 12.14)
    tbnn = g("TB.NeighLevels", 1)
    if not 1 <= tbnn <= 8:
        raise ValueError("TB.NeighLevels must be between 1 and 8")
    acc = aG / math.sqrt(3.0)
    r = 0.5 * (SHELL_RADIUS[tbnn - 1] + SHELL_RADIUS[tbnn]) * acc
    cut2intra = r * r
    if g("Neigh.LayerNeighbors", 0) != 0:
        x = aG / math.sqrt(3.0) * 1.1 * g("Neigh.LayerDistFactor", 1.0)
        cut2inter = x * x
    else:
        cut2inter = 1.0
    m = Model()
    m.aG = aG
    m.tbnn = tbnn
    for i in range(tbnn):
        m.nradii[i] = SHELL_RADIUS[i] * aG / math.sqrt(3.0) * 1.1
        m.gn_cc[i] = (g0 / g0) if i == 0 else 0.0
    bl = g("Interlayer.TypeOfBL", "None")
    koshino_intra = g("Intralayer.KoshinoIntralayer", False)
    if bl in ("Koshino", "Mayou", "HTC") and not koshino_intra:
        m.intralayer = 1
        for i, v in F2G2_SINGLE_LAYER.items():
            m.tksl[i] = v / g0
    moire = bool(g("Moire.Potential", False) and g("Moire.Jeil", False))
    if moire:
        sel = [("Moire.OnlyH0", 2), ("Moire.OnlyHZ", 3), ("Moire.NoH0AndHZ", 4), ("Moire.H0AndHZ", 1)]
        chosen = [v for key, v in sel if g(key, False)]
        if not chosen:
            raise ValueError("the moire potential needs one of MoireH0AndHZ, MoireOnlyH0, MoireOnlyHZ, MoireNoH0AndHZ")
        m.moire_onsite = chosen[0]
    pref = g("Moire.PreFactor", 1.0)
    m.C0 = g("Moire.PotC0", -0.01013) / g0 * pref
    m.Cz = g("Moire.PotCz", -0.00901) / g0 * pref
    m.Phi0 = g("Moire.PotPhi0", 1.510233401750693)
    m.Phiz = g("Moire.PotPhiz", 0.147131255943122)
    m.Cab = g("Moire.PotCab", 0.01134) / g0
    m.Phiab = g("Moire.PotPhiab", 0.342084533390889)
    m.eps = g("Moire.LatticePercent", -0.018181818181818)
    m.moire_twisted = int(bool(g("Moire.Twisted", False)))
    m.twist_rad = g("Moire.TwistAngle", 0.0) * math.pi / 180.0
    m.moire_offdiag = int(bool(g("Moire.OffDiag", False)))
    m.moire_mid = int(bool(g("Moire.OffDiagMidpoint", False)) and m.moire_offdiag)
    m.shift1 = g("Moire.LayerShift1", 0.0)
    m.sign1 = g("Moire.FirstMoireMassFactor", 1.0)
    m.sign2 = g("Moire.SecondMoireMassFactor", 1.0)
    # Moire.AddSecondMoire (ham.F90:2652-2704 on-site, 5859-5888 and 7745-7880 bonds)
    m.second_moire = int(bool(g("Moire.AddSecondMoire", False)))
    if m.second_moire:
        if g("Structure.BasedOnMoireCellParameters", False):
            raise ValueError("Moire.AddSecondMoire with Structure.BasedOnMoireCellParameters: the reference's "
                             "second moire then reads a lattice mismatch it never sets")
    m.eps_factor = g("Moire.LatticePercentFactor", 1.0)
    m.twisted2 = int(bool(g("Moire.Twisted2", False)))
    m.twist2_rad = g("Moire.TwistAngle2", 0.0) * math.pi / 180.0
    m.rotate_first = int(bool(g("Moire.SecondMoireRotateFirst", True)))
    m.shift2 = g("Moire.LayerShift2", 0.0)
    phi2m = math.atan((1.0 + m.eps) * math.sin(m.twist2_rad) / ((1.0 + m.eps) * math.cos(m.twist2_rad) - 1.0))
    m.shift2_x = m.shift2 * math.cos(phi2m)
    m.shift2_y = m.shift2 * math.sin(phi2m)
    # MoireEncapsulatedBilayerBasedOnMoireCell (ham.F90:2607-2640, 5729-5780, 6455-6500)
    m.encapsulated = int(encapsulated)
    m.bl_bottom_rad = g("Moire.BilayerBottomAngle", 0.0) * math.pi / 180.0
    m.bl_top_rad = g("Moire.BilayerTopAngle", 0.0) * math.pi / 180.0
    m.deact_upper = int(bool(g("Moire.BLDeactivateUpperLayer", False)))
    m.deact_uppers = int(bool(g("Moire.TDBLDeactivateUpperLayers", False)))
    if encapsulated:
        f2g2 = g("Intralayer.F2G2Model", True) and not g("Intralayer.RemoveF2G2Flag", False)
        one = g("Interlayer.BilayerOneParameter", False)
        if g("Intralayer.BilayerThreeParameters", False) or not (f2g2 or one):
            raise ValueError("encapsulated bilayer: BilayerThreeParameters, or neither F2G2Model nor "
                             "BilayerOneParameter, is not on the recursion path of this library")
        if one:
            m.bernal = 1
            m.tbl[2] = -g("Intralayer.BilayertAB1", 0.361) / g0
        else:
            m.bernal = 1 if g("Interlayer.LegacyBernalTAB1", False) else 2
            for t, (key, dflt) in enumerate(BERNAL_F2G2):
                m.tbl[t] = -g(key, dflt) / g0
    shifts = blshift_units(k)
    for i in range(4):
        m.tau[i] = shifts[0][0][i]
    if bl in ("Koshino", "HTC"):
        m.interlayer = 1
    m.vpppi0 = g("Interlayer.Vpppi0", 2.7 if koshino_intra else 3.5) / g0
    m.vppsigma0 = -g("Interlayer.Vppsigma0", 0.48) / g0
    m.bl_delta = g("Interlayer.BLdelta", 0.184 * aG)
    m.d_interlayer = g("Structure.InterlayerDistance", 3.35)
    m.aCC = acc
    m.g_intlay = g("TB.InterLayerHopping", 0.39) / g0
    m.anderson = int(bool(g("Disorder.Anderson", False)))
    amp = g("Disorder.AndersonAmp", None)
    m.anderson_w = 1.0 if amp is None else amp / g0
    m.e0_c = g("TB.OnSiteC", 0.0) / g0
    m.koshino_sr = int(bool(g("Interlayer.KoshinoSR", False)))
    m.renormalize_coupling = int(bool(g("Interlayer.RenormalizeCoupling", False)))
    m.coupling_factor = g("Interlayer.CouplingFactor", 1.0)
    seed = g("Kubo.SeedValue", 123456)
    kubo = dict(nrecurs=g("Kubo.RecursionNumber", 700), eta=g("Kubo.Epsilon", 0.01) / g0, n_en=g("Kubo.NumberofEnergyPoints", 1000),
                emin=g("Kubo.EnergyMin", -4.0) / g0, emax=g("Kubo.EnergyMax", 4.0) / g0, seed=seed,
                npol=g("Kubo.NumberofPolynomials", 100), dt=g("Kubo.TimeStep", 5.0), nt=g("Kubo.NumberofTimeSteps", 500),
                nwr=g("Kubo.WriteNumberofSteps", 10))
    return dict(cell=cell, g0=g0, cut2intra=cut2intra, cut2inter=cut2inter,
                second_layer=bool(g("Interlayer.AddSecondLayerInteractions", False)), model=m, moire=moire, kubo=kubo)


# the bilayer F2G2 interlayer set (ham.F90:5756-5779): tAA1, tAA2 (key BilayertAA3), tAB1, tAB2 (key
# BilayertAB3), tBA0, tBA2, tBA5 [eV]
BERNAL_F2G2 = (("Intralayer.BilayertAA1", 0.09244), ("Intralayer.BilayertAA3", -0.02299),
               ("Intralayer.BilayertAB1", 0.1391), ("Intralayer.BilayertAB3", -0.07211),
               ("Intralayer.BilayertBA0", 0.331), ("Intralayer.BilayertBA2", -0.01016),
               ("Intralayer.BilayertBA5", 0.0001))


def blshift_units(keys):
    """The layer shifts (tauX1, tauY1, tauX2, tauY2) [Ang] of each calculation of a moireBLShift.Calc sweep
    (calc.F90:40-60, moireBLShift.F90:17-110) with its folder name, or None for the run's own prefix:
    Moire.BLShiftRange gives tau = min + mS (max - min) / steps for mS = 0 .. Moire.BLShiftRangeSteps, in
    folders X1_<tauX1>_Y1_<tauY1>_X2_<tauX2>_Y2_<tauY2>; Moire.BLShiftDefinedValues one calculation with
    the Moire.Bilayer{Bottom,Top}{X,Y}Shift values; otherwise one calculation with no shift."""
    k = keys if isinstance(keys, Keys) else Keys(keys)
    g = k.get
    if not g("moireBLShift.Calc", False):
        return [((0.0, 0.0, 0.0, 0.0), None)]
    names = ("Moire.BilayerBottomX", "Moire.BilayerBottomY", "Moire.BilayerTopX", "Moire.BilayerTopY")
    if g("Moire.BLShiftDefinedValues", False):
        return [(tuple(g(n + "Shift", 0.0) for n in names), None)]
    if not g("Moire.BLShiftRange", False):
        return [((0.0, 0.0, 0.0, 0.0), None)]
    steps = g("Moire.BLShiftRangeSteps", 10)
    if steps < 1:
        raise ValueError("Moire.BLShiftRangeSteps must be at least 1")
    out = []
    for ms in range(steps + 1):
        tau = tuple(g(n + "Min", 0.0) + ms * (g(n + "Max", 0.0) - g(n + "Min", 0.0)) / steps for n in names)
        out.append((tau, "X1_%.4f_Y1_%.4f_X2_%.4f_Y2_%.4f" % tau))
    return out


def flux_of(m_quanta, area):
    """Peierls flux parameter of HamHopping for m flux quanta through a cell of area [Ang^2]."""
    bmag = m_quanta * FLUXQ / (area * 1.0e-20)
    return bmag * math.pi / FLUXQ


def cell_area(ucell):
    u = ucell
    v1 = u[1] * u[5] - u[2] * u[4]
    v2 = u[2] * u[3] - u[0] * u[5]
    v3 = u[0] * u[4] - u[1] * u[3]
    return math.sqrt(v1 * v1 + v2 * v2 + v3 * v3)


def setup(ctx, job):
    """Cell, device neighbour search and device assembly for a job; returns the cell dict."""
    from . import build_cell, cart_roundtrip, rng_uniform
    cell = build_cell(**job["cell"])
    ctx.set_geometry(cell["rat"], cell["species"], cell["layer"], cell["ucell"])
    ctx.neighbours(job["cut2intra"], job["cut2inter"], job["second_layer"], tables=False)
    rat_on = rat_hop = None
    if job["moire"]:
        rat_on = cart_roundtrip(cell["rat"], cell["ucell"])
        rat_hop = cart_roundtrip(rat_on, cell["ucell"])
    m = job["model"]
    uniform = rng_uniform(job["kubo"]["seed"], cell["n"]) if m.anderson else None
    ctx.assemble(m, rat_on, rat_hop, uniform)
    return cell
