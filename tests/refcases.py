"""Test helpers: build the oracle's inputs from reference-style input keys, and the
Hamiltonian fingerprint of the reference's model survey.

The defaults and unit conversions restate the reference's readers:
  cell / atoms      lanczosKuboCode/Src/cell.F90:16-140, 207-240; atoms.F90:124-230, 330-380
  TB parameters     tbpar.f90:20-130
  search radii      ham.F90:542-606, neigh.F90:27-31, 63-80, 348-381
  hopping keys      ham.F90:5720-5941, 6092-6122
  on-site keys      ham.F90:2099-2140, 2646-2690, 1237-1248
  field             magf.F90:20-146, ham.F90:5657
The fingerprint restates tests/regression/model_survey.py:209-229 (classify): a SHA-1 of the
sorted (atom, neighbour, image, hopping) rows and of the on-site energies, rounded to 1e-6 g0.
"""

import hashlib
import math

import numpy as np

from oracle import oracle as orc

SHELL_RADIUS = [1.0, 1.7320508075688772, 2.0, 2.6457513110645906, 3.0,
                3.4641016151377544, 3.6055512754639891, 4.0, 4.3588989435406740]
HPLANCK, QE = 6.62606896e-34, 1.602176565e-19
FLUXQ = HPLANCK / QE

# case inputs of tests/regression/model_cases.py (only the keys that matter on this path)
COMMON = {"SuperCell": 1, "LayerNeighbors": 100, "LayerDistFactor": 6.2, "NeighLevels": 5}
BILAYER = {"TypeOfBL": "Koshino", "MoireCellParameters": (3, 2, 2, 3), "twoLayers": True,
           "InterlayerDistance": 3.34, "CellHeight": 40.0}
EFFECTIVE = {"TypeOfSystem": "Graphene", "CellSize": 11, "MoirePotential": True, "MoireJeil": True,
             "MoirePotC0": -0.01013, "MoirePotCz": -0.00901, "MoirePotCab": 0.01134,
             "MoirePotPhi0": 1.510233401750693, "MoirePotPhiz": 0.147131255943122,
             "MoirePotPhiab": 0.342084533390889, "LatticePercent": -0.0909090909090909,
             "MoireH0AndHZ": True}
BASES = {
    "graphene": dict(TypeOfSystem="Graphene", CellSize=6, **COMMON),
    "tbg": dict(TypeOfSystem="TwistedBilayerBasedOnMoireCell", **BILAYER, **COMMON),
    "eff": dict(EFFECTIVE, **COMMON),
    "encmc": dict(TypeOfSystem="MoireEncapsulatedBilayerBasedOnMoireCell", **BILAYER, **COMMON),
}
CASES = {
    "graphene": ("graphene", {}),
    "graphene+NeighLevels1": ("graphene", {"NeighLevels": 1}),
    "graphene+NeighLevels2": ("graphene", {"NeighLevels": 2}),
    "graphene+NeighLevels3": ("graphene", {"NeighLevels": 3}),
    "graphene+MagField1": ("graphene", {"MagFieldInteger": 1}),
    "eff": ("eff", {}),
    "eff+MoireOffDiag": ("eff", {"MoireOffDiag": True, "MoireTwistAngle": 0.5}),
    "eff+MoireOffDiagMidpoint": ("eff", {"MoireOffDiag": True, "MoireOffDiagMidpoint": True}),
    "eff+MoireTwisted": ("eff", {"MoireTwisted": True, "MoireTwistAngle": 0.5}),
    "eff+MoireAddSecondMoire": ("eff", {"MoireAddSecondMoire": True, "MoireOffDiag": True}),
    "eff+MoireAddSecondMoire+Midpoint": ("eff", {"MoireAddSecondMoire": True, "MoireOffDiag": True,
                                                 "MoireOffDiagMidpoint": True}),
    "eff+MoireAddSecondMoire+Twisted2": ("eff", {"MoireAddSecondMoire": True, "MoireTwisted2": True,
                                                 "MoireTwistAngle2": 0.5}),
    "eff+MoireSecondMoireRotateFirst_off": ("eff", {"MoireAddSecondMoire": True, "MoireSecondMoireRotateFirst": False}),
    "tbg": ("tbg", {}),
    "sys_MoireEncapsulatedBilayerMC": ("encmc", {}),
    "sys_MoireEncapsulatedBilayerMC+MoirePotential": ("encmc", {"MoirePotential": True, "MoireJeil": True,
                                                                "MoireH0AndHZ": True}),
    "sys_MoireEncapsulatedBilayerMC+MoireOffDiag": ("encmc", {"MoirePotential": True, "MoireJeil": True,
                                                              "MoireH0AndHZ": True, "MoireOffDiag": True}),
    "tbg+MagField1": ("tbg", {"MagFieldInteger": 1}),
}


def case_keys(name):
    base, changes = CASES[name]
    k = dict(BASES[base])
    k.update(changes)
    return k


def build(keys):
    """Geometry, neighbours, on-site energies and hoppings (complex, g0 units) for input keys."""
    g = lambda k, d: keys.get(k, d)
    aG = g("LatticeParameter", 2.46)
    system = g("TypeOfSystem", "Graphene")
    kind = {"Graphene": orc.GRAPHENE, "TwistedBilayerBasedOnMoireCell": orc.TBG_MOIRE_CELL,
            "MoireEncapsulatedBilayerBasedOnMoireCell": orc.TBG_MOIRE_CELL}[system]
    encapsulated = system == "MoireEncapsulatedBilayerBasedOnMoireCell"
    add_shift = 0
    if g("TwistedBLAddShift", False):
        add_shift = 1 if g("BernalShift", False) else 2 if g("BridgeShift", False) else None
        if add_shift is None:
            raise ValueError("TwistedBLAddShift needs BernalShift or BridgeShift")
    geo = orc.geometry(kind, aG=aG, cell_size=g("CellSize", 50), super_cell=g("SuperCell", 1),
                       m=g("MoireCellParameters", (0, 0, 0, 0)), height=g("CellHeight", 40.0),
                       d_interlayer=g("InterlayerDistance", 3.35), add_shift=add_shift,
                       shift_factor=g("BilayerShiftFactor", 0.0))
    g0 = g("Hopping", -3.72 * aG + 12.14)
    tbnn = g("NeighLevels", 1)
    acc = aG / math.sqrt(3.0)
    r = 0.5 * (SHELL_RADIUS[tbnn - 1] + SHELL_RADIUS[tbnn]) * acc
    cut2intra = r * r
    if g("LayerNeighbors", 0) != 0:
        x = aG / math.sqrt(3.0) * 1.1 * g("LayerDistFactor", 1.0)
        cut2inter = x * x
    else:
        cut2inter = 1.0
    nb = orc.neighbours(geo["rat"], geo["ucell"], cut2intra, cut2inter, g("AddSecondLayerInteractions", False))

    m = orc.Model()
    m.aG = aG
    m.tbnn = tbnn
    for i in range(min(tbnn, 8)):
        m.nradii[i] = SHELL_RADIUS[i] * aG / math.sqrt(3.0) * 1.1
        m.gn_cc[i] = (g0 / g0) if i == 0 else 0.0
    bl = g("TypeOfBL", "None")
    koshino_intra = g("KoshinoIntralayer", False)
    if bl in ("Koshino", "Mayou", "HTC") and not koshino_intra:
        m.intralayer = orc.INTRA_F2G2_SL
        # single-layer F2G2 set of HamHopF2G2sParameters (ham.F90:8253-8395), twoLayers/oneLayer stacks
        for k, v in F2G2_SINGLE_LAYER.items():
            m.tksl[k] = v / g0
    moire = g("MoirePotential", False) and g("MoireJeil", False)
    if moire:
        if g("MoireOnlyH0", False):
            m.moire_onsite = orc.ONSITE_ONLY_H0
        elif g("MoireOnlyHZ", False):
            m.moire_onsite = orc.ONSITE_ONLY_HZ
        elif g("MoireNoH0AndHZ", False):
            m.moire_onsite = orc.ONSITE_NO_H0_AND_HZ
        elif g("MoireH0AndHZ", False):
            m.moire_onsite = orc.ONSITE_H0_AND_HZ
        else:
            raise ValueError("moire potential without an on-site selector")
    pref = g("MoirePreFactor", 1.0)
    m.C0 = g("MoirePotC0", -0.01013) / g0 * pref
    m.Cz = g("MoirePotCz", -0.00901) / g0 * pref
    m.Phi0 = g("MoirePotPhi0", 1.510233401750693)
    m.Phiz = g("MoirePotPhiz", 0.147131255943122)
    m.Cab = g("MoirePotCab", 0.01134) / g0
    m.Phiab = g("MoirePotPhiab", 0.342084533390889)
    m.eps = g("LatticePercent", -0.018181818181818)
    m.moire_twisted = int(g("MoireTwisted", False))
    m.twist_rad = g("MoireTwistAngle", 0.0) * math.pi / 180.0
    m.moire_offdiag = int(g("MoireOffDiag", False))
    m.moire_mid = int(g("MoireOffDiagMidpoint", False) and m.moire_offdiag)
    m.shift1 = g("MoireLayerShift1", 0.0)
    m.sign1 = g("MoireFirstMoireMassFactor", 1.0)
    m.sign2 = g("MoireSecondMoireMassFactor", 1.0)
    # Moire.AddSecondMoire (ham.F90:2652-2704, 5859-5888)
    m.second_moire = int(g("MoireAddSecondMoire", False))
    m.eps_factor = g("LatticepercentFactor", 1.0)
    m.twisted2 = int(g("MoireTwisted2", False))
    m.twist2_rad = g("MoireTwistAngle2", 0.0) * math.pi / 180.0
    m.rotate_first = int(g("MoireSecondMoireRotateFirst", True))
    m.shift2 = g("MoireLayerShift2", 0.0)
    phi2m = math.atan((1.0 + m.eps) * math.sin(m.twist2_rad) / ((1.0 + m.eps) * math.cos(m.twist2_rad) - 1.0))
    m.shift2_x = m.shift2 * math.cos(phi2m)
    m.shift2_y = m.shift2 * math.sin(phi2m)
    # MoireEncapsulatedBilayerBasedOnMoireCell (ham.F90:2607-2640, 5729-5780, 6455-6500)
    m.encapsulated = int(encapsulated)
    m.bl_bottom_rad = g("MoireBilayerBottomAngle", 0.0) * math.pi / 180.0
    m.bl_top_rad = g("MoireBilayerTopAngle", 0.0) * math.pi / 180.0
    for k, key in enumerate(("MoireBilayerBottomXShift", "MoireBilayerBottomYShift", "MoireBilayerTopXShift",
                              "MoireBilayerTopYShift")):
        m.tau[k] = g(key, 0.0)
    m.deact_upper = int(g("MoireBLDeactivateUpperLayer", False))
    m.deact_uppers = int(g("MoiretDBLDeactivateUpperLayers", False))
    f2g2 = g("F2G2Model", True) and not g("RemoveF2G2Flag", False)
    one, three = g("BilayerOneParameter", False), g("BilayerThreeParameters", False)
    if encapsulated:
        if three or not (f2g2 or one):
            raise ValueError("encapsulated bilayer: BilayerThreeParameters, or neither F2G2Model nor "
                             "BilayerOneParameter, is not on this path")
        if one:
            m.bernal, m.tbl[2] = 1, -g("BilayertAB1", 0.361) / g0
        else:
            m.bernal = 1 if g("LegacyBernalTAB1", False) else 2
            for k, (key, dflt) in enumerate((("BilayertAA1", 0.09244), ("BilayertAA3", -0.02299),
                                             ("BilayertAB1", 0.1391), ("BilayertAB3", -0.07211),
                                             ("BilayertBA0", 0.331), ("BilayertBA2", -0.01016),
                                             ("BilayertBA5", 0.0001))):
                m.tbl[k] = -g(key, dflt) / g0
    if bl in ("Koshino", "HTC"):
        m.interlayer = orc.INTER_TWO_CENTRE
    vpppi0 = g("Vpppi0", 2.7 if koshino_intra else 3.5)
    m.vpppi0 = vpppi0 / g0
    m.vppsigma0 = -g("Vppsigma0", 0.48) / g0
    m.bl_delta = g("BLdelta", 0.184 * aG)
    m.d_interlayer = g("InterlayerDistance", 3.35)
    m.aCC = acc
    m.g_intlay = g("InterLayerHopping", 0.39) / g0
    m.anderson = int(g("Anderson", False))
    m.anderson_w = g("AndersonAmp", 1.0 * g0) / g0
    m.seed = g("SeedValue", 123456)
    m.e0_c = g("OnSiteC", 0.0) / g0
    m.koshino_sr = int(g("KoshinoSR", False))
    m.renormalize_coupling = int(g("RenormalizeCoupling", False))
    m.coupling_factor = g("CouplingFactor", 1.0)

    rat = geo["rat"]
    rat_on = orc.roundtrip(rat, geo["ucell"]) if moire else rat
    rat_hop = orc.roundtrip(rat_on, geo["ucell"]) if moire else rat
    h0, h0_bottom, h0_top = orc.onsite_layers(m, rat_on, geo["species"], geo["layer"])
    hop = orc.hopping(m, rat_hop, geo["species"], geo["layer"], nb)
    area = orc.cell_area(geo["ucell"])
    mb = g("MagFieldInteger", 0)
    if mb != 0:
        bmag = mb * FLUXQ / (area * 1.0e-20)
        flux = bmag * math.pi / FLUXQ
        hop = orc.peierls(rat_hop, geo["ucell"], nb, flux, hop)
    flux = 0.0
    if mb != 0:
        flux = mb * FLUXQ / (area * 1.0e-20) * math.pi / FLUXQ
    return dict(geo=geo, nb=nb, h0=h0, h0_bottom=h0_bottom, h0_top=h0_top, hop=hop, g0=g0, model=m, area=area,
                rat_on=rat_on, rat_hop=rat_hop,
                cut2intra=cut2intra, cut2inter=cut2inter, flux=flux, second_layer=g("AddSecondLayerInteractions", False))


def gpu_model(m):
    """The same model as the library's gbn_model structure.  Fields the oracle does not have (the smooth
    interlayer cutoff, which the reference lacks) stay 0: the reference's hard cutoff."""
    import grabnes_b200 as G
    out = G.Model()
    for name, _ in G.Model._fields_:
        if not hasattr(m, name):
            continue
        v = getattr(m, name)
        if hasattr(v, "__len__"):
            arr = getattr(out, name)
            for i in range(len(arr)):
                arr[i] = v[i]
        else:
            setattr(out, name, v)
    return out


# F2G2 single-layer graphene intralayer terms [eV] of HamHopF2G2sParameters (ham.F90:8253-8395)
F2G2_SINGLE_LAYER = {2: -0.2354, 3: 0.1877, 4: 0.0, 5: -0.0633, 6: 0.0, 7: 0.0}


def fingerprint(nb, hop, h0, digits=6):
    """tests/regression/model_survey.py:209-229"""
    n = len(h0)
    bonds = {}
    for i in range(n):
        for j in range(int(nb["nneigh"][i])):
            key = (i, int(nb["nlist"][i, j]) - 1, tuple(int(x) for x in nb["ncell"][i, j]))
            bonds[key] = bonds.get(key, 0.0) + complex(hop[i, j])
    rows = sorted((i, m) + r + (round(v.real, digits) + 0.0, round(v.imag, digits) + 0.0)
                  for (i, m, r), v in bonds.items())
    h = hashlib.sha1()
    h.update(repr(rows).encode())
    h.update(repr([round(float(x), digits) + 0.0 for x in h0]).encode())
    return h.hexdigest()[:16]
