"""The `grabnes Gendata.in` driver: its reading of the input against the package's key mapping (CPU),
and its output files against the oracle for a field sweep (GPU)."""
import json
import math
import os
import subprocess

import numpy as np
import pytest

import refcases as R
from oracle import oracle as orc

G = pytest.importorskip("grabnes_b200")
from grabnes_b200 import model as M  # noqa: E402

DRIVER = os.path.join(os.path.dirname(G.__file__), "grabnes")

INPUTS = {
    "moire_sweep": {
        "Run.Prefix": "generate", "Run.TypeOfSystem": "Graphene", "Structure.CellSize": 11, "Structure.SuperCell": 4,
        "Moire.LatticePercent": -1.0 / 11.0, "Moire.Potential": True, "Moire.Jeil": True, "Moire.H0AndHZ": True,
        "Moire.OffDiag": True, "Moire.OffDiagMidpoint": True, "Kubo.RecursionNumber": 120,
        "Kubo.Epsilon": 0.004, "Kubo.EnergyMin": -0.3, "Kubo.EnergyMax": 0.3, "Kubo.SeedValue": 123456,
        "Calculate.OnlyDOS": True,
    },
    "tbg_former_names": {
        "TypeOfSystem": "TwistedBilayerBasedOnMoireCell", "MoireCellParameters": (31, 30, 30, 31),
        "TypeOfBL": "Koshino", "vpppi0": 2.7, "vppsigma0": 0.48, "BLdelta": 0.319, "InterlayerDistance": 3.35,
        "Neigh.LayerNeighbors": 100, "Neigh.LayerDistFactor": 3.2005, "TB.Hopping": 2.7, "RecursionNumber": 150,
    },
    "example08_model": {
        "Run.TypeOfSystem": "TwistedBilayerBasedOnMoireCell", "Structure.MoireCellParameters": (31, 30, 30, 31),
        "Stack.TwoLayers": True, "Structure.InterlayerDistance": 3.35, "Intralayer.F2G2Model": True,
        "TB.NeighLevels": 5, "TB.Hopping": 3.5, "TB.OnSiteC": 0.4914, "Interlayer.TypeOfBL": "Koshino",
        "Interlayer.KoshinoSR": True, "Interlayer.RenormalizeCoupling": True, "Interlayer.CouplingFactor": 1.008,
        "Neigh.LayerNeighbors": 400, "Neigh.LayerDistFactor": 4.0, "Kubo.RecursionNumber": 100,
    },
    "anderson": {"Run.TypeOfSystem": "Graphene", "Structure.CellSize": 30, "Disorder.Anderson": True,
                 "Disorder.AndersonAmp": 1.0, "Kubo.SeedValue": 5, "TB.NeighLevels": 2},
    "encapsulated_bilayer_former_names": {
        "TypeOfSystem": "MoireEncapsulatedBilayerBasedOnMoireCell", "MoireCellParameters": (6, 0, 6, 0),
        "twistedBLAddShift": True, "BernalShift": True, "BilayerShiftFactor": 0.2, "MoirePotential": True,
        "MoireJeil": True, "MoireH0AndHZ": True, "MoireOffDiag": True, "MoireBilayerBottomAngle": 0.3,
        "MoireBilayerTopAngle": -0.7, "MoireBLDeactivateUpperLayer": True, "BilayertBA0": 0.35, "TypeOfBL": "Koshino",
        "moireBLShift.Calc": True, "moireBLShiftDefinedValues": True, "MoireBilayerTopXShift": 0.4, "RecursionNumber": 30,
    },
    "encapsulated_shift_sweep": {
        "Run.Prefix": "generate", "Run.TypeOfSystem": "MoireEncapsulatedBilayerBasedOnMoireCell",
        "Structure.MoireCellParameters": (6, 0, 6, 0), "Structure.SuperCell": 4, "Structure.TwistedBLAddShift": True,
        "Structure.BernalShift": True, "Structure.InterlayerDistance": 3.34, "Interlayer.TypeOfBL": "Koshino",
        "TB.NeighLevels": 5, "Neigh.LayerNeighbors": 100, "Neigh.LayerDistFactor": 3.2, "Moire.Potential": True,
        "Moire.Jeil": True, "Moire.H0AndHZ": True, "Moire.OffDiag": True, "Moire.LatticePercent": -0.0166,
        "Moire.BilayerBottomAngle": 0.4, "Moire.BilayerTopAngle": -0.9, "moireBLShift.Calc": True,
        "Moire.BLShiftRange": True, "Moire.BLShiftRangeSteps": 2, "Moire.BilayerBottomXMax": 0.6,
        "Moire.BilayerTopYMin": -0.3, "Moire.BilayerTopYMax": 0.9, "Kubo.RecursionNumber": 100,
        "Kubo.Epsilon": 0.01, "Kubo.EnergyMin": -1.0, "Kubo.EnergyMax": 1.0, "Kubo.SeedValue": 11,
        "Calculate.OnlyDOS": True,
    },
    "second_moire_former_names": {
        "TypeOfSystem": "Graphene", "CellSize": 11, "SuperCell": 2, "Latticepercent": -1.0 / 11.0,
        "MoirePotential": True, "MoireJeil": True, "MoireH0AndHZ": True, "MoireOffDiag": True,
        "MoireAddSecondMoire": True, "LatticepercentFactor": 1.3, "MoireTwisted2": True, "MoireTwistAngle2": 0.7,
        "MoireLayerShift2": 0.9, "MoireSecondMoireRotateFirst": False, "MoireSecondMoireMassFactor": -1.0,
        "RecursionNumber": 50,
    },
}


def _fmt(v):
    if isinstance(v, bool):
        return ".true." if v else ".false."
    if isinstance(v, tuple):
        return " ".join(str(x) for x in v)
    if isinstance(v, float) and v < 0:
        return f"0-{-v!r}"   # the reference's way of writing a negative number
    return repr(v) if isinstance(v, float) else str(v)


def _write(path, keys, extra=""):
    with open(path, "w") as f:
        f.write("# written by the test\n")
        for k, v in keys.items():
            f.write(f"{k} {_fmt(v)}   # a comment\n")
        f.write(extra)


def _print_job(path, env=None):
    """The job the driver reads (its last line) and, with env, the sweep units of that rank (its first)."""
    out = subprocess.run([DRIVER, "--print-job", path], check=True, capture_output=True, text=True,
                         env=env).stdout.strip().splitlines()
    return json.loads(out[-1]) if env is None else (json.loads(out[-1]), json.loads(out[0]))


pytestmark_cpu = pytest.mark.skipif(not os.path.exists(DRIVER), reason="driver not built")


@pytestmark_cpu
@pytest.mark.parametrize("name", sorted(INPUTS))
def test_driver_reads_input_like_the_package(tmp_path, name):
    keys = INPUTS[name]
    path = str(tmp_path / "Gendata.in")
    _write(path, keys)
    got = _print_job(path)
    job = M.job_from_keys(keys)
    assert got["g0"] == job["g0"]
    assert got["cut2intra"] == job["cut2intra"] and got["cut2inter"] == job["cut2inter"]
    assert got["moire"] == int(job["moire"])
    assert got["nrecurs"] == job["kubo"]["nrecurs"] and got["seed"] == job["kubo"]["seed"]
    assert math.isclose(got["eta"], job["kubo"]["eta"], rel_tol=1e-15)
    assert math.isclose(got["emin"], job["kubo"]["emin"], rel_tol=1e-15)
    m = job["model"]
    for f in ("tbnn", "intralayer", "moire_onsite", "moire_offdiag", "moire_mid", "moire_twisted", "interlayer",
              "anderson", "koshino_sr", "renormalize_coupling", "second_moire", "twisted2", "rotate_first"):
        assert got["model"][f] == getattr(m, f), f
    for f in ("eps", "C0", "Cz", "Cab", "vpppi0", "vppsigma0", "bl_delta", "anderson_w", "coupling_factor",
              "eps_factor", "twist2_rad", "shift2_x", "shift2_y", "sign2", "bl_bottom_rad", "bl_top_rad"):
        assert math.isclose(got["model"][f], getattr(m, f), rel_tol=1e-15, abs_tol=1e-300), f
    for f in ("encapsulated", "deact_upper", "deact_uppers", "bernal"):
        assert got["model"][f] == getattr(m, f), f
    assert got["model"]["tbl"] == list(m.tbl)
    assert got["add_shift"] == job["cell"]["add_shift"] and got["shift_factor"] == job["cell"]["shift_factor"]
    assert got["cell_size"] == job["cell"]["cell_size"] and got["super_cell"] == job["cell"]["super_cell"]
    assert tuple(got["m"]) == tuple(job["cell"]["m"])


@pytestmark_cpu
@pytest.mark.parametrize("nranks", [1, 2, 3])
def test_driver_sweep_shards(tmp_path, nranks):
    """GRABNES_RANK / GRABNES_NRANKS: every (field, Haldane phase) unit of a sweep runs on exactly one rank,
    unit u on rank u % NRANKS, in the reference's loop order (fields outer, phases inner)."""
    from grabnes_b200 import replicas
    path = str(tmp_path / "Gendata.in")
    _write(path, {"Run.TypeOfSystem": "Graphene", "Structure.CellSize": 10}, "MagField.InitialInteger 0\n"
           "MagField.FinalInteger 8\nMagField.IntegerStep 2\nHaldane.NNN .true.\nHaldane.SpecifyRange .true.\n"
           "HaldPhase.InitialInteger 0\nHaldPhase.FinalInteger 2\n")
    everything = [[mb, ph] for mb in range(0, 9, 2) for ph in range(0, 3)]
    got = []
    for rank in range(nranks):
        env = dict(os.environ, GRABNES_RANK=str(rank), GRABNES_NRANKS=str(nranks))
        _, units = _print_job(path, env)
        assert units["rank"] == rank and units["nranks"] == nranks
        assert units["units"] == [everything[k] for k in replicas.shard_units(len(everything), rank, nranks)]
        got += units["units"]
    assert sorted(got) == sorted(everything)


@pytestmark_cpu
def test_driver_expressions(tmp_path):
    path = str(tmp_path / "Gendata.in")
    _write(path, {"TB.Hopping": "2*1.35", "Kubo.Epsilon": "1.0d-2", "Kubo.EnergyMin": "-(1+2)*sqrt(4)",
                  "Kubo.EnergyMax": "2**3", "Kubo.RecursionNumber": "10*10"})
    got = _print_job(path)
    assert got["g0"] == 2.7 and got["nrecurs"] == 100
    assert math.isclose(got["eta"] * 2.7, 0.01, rel_tol=1e-15)
    assert math.isclose(got["emin"] * 2.7, -6.0, rel_tol=1e-15) and math.isclose(got["emax"] * 2.7, 8.0, rel_tol=1e-15)


@pytest.mark.gpu
def test_driver_field_sweep_against_oracle(tmp_path):
    """A three-field sweep of the moire model: one folder per field with the reference's files; a_n, b_n
    and the DOS of every field against the oracle's recursion and continued fraction.  120 steps: this
    3872-atom cell is small and symmetric, and beyond about 150 steps two FP64 recursions that differ
    only in summation order part ways (the recursion's own parity is tested on larger cells)."""
    keys = dict(INPUTS["moire_sweep"])
    path = str(tmp_path / "Gendata.in")
    _write(path, keys, "MagField.InitialInteger 0\nMagField.FinalInteger 4\nMagField.IntegerStep 2\n")
    subprocess.run([DRIVER, path], check=True, cwd=str(tmp_path), capture_output=True, text=True)
    folders = sorted(d for d in os.listdir(tmp_path) if d.startswith("m0"))
    assert [f[:6] for f in folders] == ["m00000", "m00002", "m00004"]
    base = dict(TypeOfSystem="Graphene", CellSize=11, SuperCell=4, LatticePercent=-1.0 / 11.0, MoirePotential=True,
                MoireJeil=True, MoireH0AndHZ=True, MoireOffDiag=True, MoireOffDiagMidpoint=True)
    for folder, mb in zip(folders, (0, 2, 4)):
        r = R.build(dict(base, MagFieldInteger=mb))
        n, g0 = r["geo"]["n"], r["g0"]
        a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], orc.init_wf(n, 123456), 120, 0)
        a = np.loadtxt(tmp_path / folder / "generate.a0.dat")
        b = np.loadtxt(tmp_path / folder / "generate.b0.dat")
        assert np.abs(a - a0).max() <= 1e-10 * np.abs(a0).max() and np.abs(b - b0).max() <= 1e-10 * np.abs(b0).max()
        e0, d0 = orc.frac(a0, b0, 0.004 / g0, 1000, -0.3 / g0, 0.3 / g0)
        dos = np.loadtxt(tmp_path / folder / "generate.DOS")
        assert np.abs(dos[:, 0] - e0).max() == 0.0
        assert np.abs(dos[:, 1] - d0).sum() <= 1e-6 * np.abs(d0).sum()   # normalised L1, the DOS bar
        ab = np.loadtxt(tmp_path / folder / "generate.AB", skiprows=1)
        assert np.array_equal(ab[:, 0], a) and np.array_equal(ab[:, 1], b)


@pytest.mark.gpu
def test_launcher_two_ranks_match_one_process(tmp_path):
    """The three-field sweep through grabnes_b200.launch with two ranks (both on this GPU: each is its own
    process and CUDA context, and no kernel of one waits on the other) against one driver process: the
    same folders, a_n and b_n within 1e-10 of their scale and the DOS within 1e-6 (normalised L1) -- the
    ranks batch different sets of fields, so their tiles differ."""
    import sys
    keys = dict(INPUTS["moire_sweep"])
    sweep = "MagField.InitialInteger 0\nMagField.FinalInteger 4\nMagField.IntegerStep 2\n"
    one, two = tmp_path / "one", tmp_path / "two"
    one.mkdir()
    two.mkdir()
    for d in (one, two):
        _write(str(d / "Gendata.in"), keys, sweep)
    subprocess.run([DRIVER, "Gendata.in"], check=True, cwd=str(one), capture_output=True, text=True)
    env = dict(os.environ, PYTHONPATH=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    p = subprocess.run([sys.executable, "-m", "grabnes_b200.launch", "--gpus", "2", "Gendata.in"], cwd=str(two),
                       env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    f1 = sorted(d for d in os.listdir(one) if d.startswith("m0"))
    f2 = sorted(d for d in os.listdir(two) if d.startswith("m0"))
    assert f1 == f2 and len(f1) == 3
    for folder in f1:
        for name in ("generate.a0.dat", "generate.b0.dat"):
            x, y = np.loadtxt(one / folder / name), np.loadtxt(two / folder / name)
            assert np.abs(x - y).max() <= 1e-10 * np.abs(x).max()
        d1, d2 = np.loadtxt(one / folder / "generate.DOS"), np.loadtxt(two / folder / "generate.DOS")
        assert np.array_equal(d1[:, 0], d2[:, 0])
        assert np.abs(d1[:, 1] - d2[:, 1]).sum() <= 1e-6 * np.abs(d1[:, 1]).sum()
    logs = [(two / f"grabnes.rank{r}.log").read_text() for r in range(2)]
    assert "rank 0 of 2" in logs[0] and "rank 1 of 2" in logs[1]


@pytest.mark.gpu
def test_driver_time_evolution_against_oracle(tmp_path):
    """Without Calculate.OnlyDOS: KuboInterval and KuboCn (<prefix>.cn.dat), then four steps of KuboEvol in
    a field, writing the recursion of the commutator term every two steps (.AB_0002/.Z2_0002, ...),
    against the oracle's KuboEvol loop."""
    keys = {"Run.Prefix": "tev", "Run.TypeOfSystem": "Graphene", "Structure.CellSize": 60, "TB.Hopping": 2.7,
            "MagField.Integer": 3, "Kubo.RecursionNumber": 80, "Kubo.NumberofEnergyPoints": 200,
            "Kubo.Epsilon": 0.05, "Kubo.EnergyMin": -8.0, "Kubo.EnergyMax": 8.0, "Kubo.SeedValue": 11,
            "Kubo.NumberofPolynomials": 40, "Kubo.TimeStep": 2.0, "Kubo.NumberofTimeSteps": 4,
            "Kubo.WriteNumberofSteps": 2}
    path = str(tmp_path / "Gendata.in")
    _write(path, keys)
    subprocess.run([DRIVER, path], check=True, cwd=str(tmp_path), capture_output=True, text=True)
    r = R.build(dict(TypeOfSystem="Graphene", CellSize=60, Hopping=2.7, MagFieldInteger=3))
    n, g0 = r["geo"]["n"], r["g0"]
    psi = orc.init_wf(n, 11)
    a, b = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 80, 0)
    ac, bc = orc.interval(a, b)
    c = orc.cheb_coef(2.0, ac, bc, 40)
    cn = np.loadtxt(tmp_path / "tev.cn.dat")
    assert np.abs(cn[:, 0] - c.real).max() <= 1e-11 and np.abs(cn[:, 1] - np.abs(c)).max() <= 1e-11
    zu = np.zeros(n, np.complex128)
    for it in range(1, 5):
        psi, zu = orc.evol(r["nb"], r["hop"], r["h0"], c, ac, bc, psi, zu, 1)
        if it % 2:
            continue
        norm = float(np.vdot(zu, zu).real)
        az, bz = orc.recursion(r["nb"], r["hop"], r["h0"], zu / np.sqrt(norm), 80, 0)
        tag = f"{it:04d}"
        ab = np.loadtxt(tmp_path / f"tev.AB_{tag}.dat", skiprows=1)
        with open(tmp_path / f"tev.AB_{tag}.dat") as f:
            assert abs(float(f.readline()) - norm) <= 1e-9 * norm
        assert np.abs(ab[:, 0] - az).max() <= 1e-9 * np.abs(az).max()
        assert np.abs(ab[:, 1] - bz).max() <= 1e-9 * np.abs(bz).max()
        e0, d0 = orc.frac(az, bz, 0.05 / g0, 200, -8.0 / g0, 8.0 / g0, norm)
        z2 = np.loadtxt(tmp_path / f"tev.Z2_{tag}.dat")
        assert np.abs(z2[:, 1] - d0).sum() <= 1e-6 * np.abs(d0).sum()


@pytest.mark.gpu
def test_driver_msd_against_oracle(tmp_path):
    """Kubo.TEvolVectors 3 on disordered graphene: the reference's files from vector 0, and
    <prefix>.MSD.dat, the spread <(X(t) - X(0))^2> averaged over the three vectors (|ZUPsi_r|^2 of
    KuboTEvol, kubo.F90:376-385) with its diffusivity, against the oracle's KuboEvol loop of the same
    vectors (vector r: draws r N .. (r + 1) N - 1 of the seeded stream): 1e-9 relative."""
    keys = {"Run.Prefix": "msd", "Run.TypeOfSystem": "Graphene", "Structure.CellSize": 50, "TB.Hopping": 2.7,
            "Disorder.Anderson": True, "Disorder.AndersonAmp": 1.0, "Kubo.RecursionNumber": 60,
            "Kubo.NumberofEnergyPoints": 100, "Kubo.Epsilon": 0.05, "Kubo.EnergyMin": -8.0,
            "Kubo.EnergyMax": 8.0, "Kubo.SeedValue": 5, "Kubo.NumberofPolynomials": 40, "Kubo.TimeStep": 2.0,
            "Kubo.NumberofTimeSteps": 6, "Kubo.WriteNumberofSteps": 2, "Kubo.TEvolVectors": 3}
    path = str(tmp_path / "Gendata.in")
    _write(path, keys)
    subprocess.run([DRIVER, path], check=True, cwd=str(tmp_path), capture_output=True, text=True)
    r = R.build(dict(TypeOfSystem="Graphene", CellSize=50, Hopping=2.7, Anderson=True, AndersonAmp=1.0, SeedValue=5))
    n, g0 = r["geo"]["n"], r["g0"]
    u = orc.rng_draws(5, 3 * n).reshape(3, n)
    psis = [np.exp(2j * np.pi * u[k]) / np.sqrt(n) for k in range(3)]
    a, b = orc.recursion(r["nb"], r["hop"], r["h0"], psis[0], 60, 0)
    ac, bc = orc.interval(a, b)
    c = orc.cheb_coef(2.0, ac, bc, 40)
    norms = np.zeros((3, 3))
    for k in range(3):
        psi, zu = psis[k], np.zeros(n, np.complex128)
        for it in range(1, 7):
            psi, zu = orc.evol(r["nb"], r["hop"], r["h0"], c, ac, bc, psi, zu, 1)
            if it % 2 == 0:
                norms[k, it // 2 - 1] = float(np.vdot(zu, zu).real)
    msd = norms.mean(axis=0)
    dt_fs = 2.0 * (6.62606896e-34 / (2 * np.pi)) / 1.602176565e-19 / g0 * 1e15
    t = dt_fs * 2 * np.arange(1, 4)
    slope = np.array([(msd[1] - 0.0) / (t[1] - 0.0), (msd[2] - msd[0]) / (t[2] - t[0]), (msd[2] - msd[1]) / (t[2] - t[1])])
    got = np.loadtxt(tmp_path / "msd.MSD.dat")
    assert got.shape == (3, 4)
    assert np.abs(got[:, 0] - t).max() <= 1e-12 * t.max()
    assert np.abs(got[:, 1] - msd).max() <= 1e-9 * msd.max()
    assert np.abs(got[:, 2] - msd / t).max() <= 1e-9 * (msd / t).max()
    assert np.abs(got[:, 3] - slope).max() <= 1e-9 * np.abs(slope).max()
    with open(tmp_path / "msd.AB_0002.dat") as f:   # the reference's file, from vector 0
        assert abs(float(f.readline()) - norms[0, 0]) <= 1e-9 * norms[0, 0]


@pytest.mark.gpu
def test_driver_layer_pdos_against_oracle(tmp_path):
    """Kubo.PDOSLayer: one folder per layer with the reference's files, from random phases on the layer's
    atoms (Kubo.SeedSet stream), against the oracle's recursion and continued fraction."""
    from oracle import pdos as OP
    keys = dict(INPUTS["tbg_former_names"], **{"Run.Prefix": "tbg", "Kubo.PDOS": True, "Kubo.PDOSLayer": True,
                                                "Kubo.SeedSet": 77, "Kubo.EnergyMin": -1.0, "Kubo.EnergyMax": 1.0,
                                                "Kubo.Epsilon": 0.01, "Calculate.OnlyDOS": True})
    path = str(tmp_path / "Gendata.in")
    _write(path, keys)
    subprocess.run([DRIVER, path], check=True, cwd=str(tmp_path), capture_output=True, text=True)
    r = R.build(dict(TypeOfSystem="TwistedBilayerBasedOnMoireCell", MoireCellParameters=(31, 30, 30, 31),
                     TypeOfBL="Koshino", Vpppi0=2.7, Vppsigma0=0.48, BLdelta=0.319, InterlayerDistance=3.35,
                     LayerNeighbors=100, LayerDistFactor=3.2005, Hopping=2.7))
    geo, g0 = r["geo"], r["g0"]
    n = geo["n"]
    u = orc.rng_draws(77, n)
    for lay, _, m, mask in OP.layer_sets(OP.LAYER, geo["species"], geo["layer"], number_of_layers=2):
        psi = OP.layer_start_vector(mask, m, u)
        a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 150, 0)
        folder = tmp_path / f"PDOS_layer{lay:02d}"
        a = np.loadtxt(folder / "tbg.a0.dat")
        b = np.loadtxt(folder / "tbg.b0.dat")
        assert np.abs(a - a0).max() <= 1e-10 * np.abs(a0).max() and np.abs(b - b0).max() <= 1e-10 * np.abs(b0).max()
        _, d0 = orc.frac(a0, b0, 0.01 / g0, 1000, -1.0 / g0, 1.0 / g0)
        dos = np.loadtxt(folder / "tbg.DOS")
        assert np.abs(dos[:, 1] - d0).sum() <= 1e-6 * np.abs(d0).sum()


@pytest.mark.gpu
def test_driver_atom_pdos_and_time_evolution(tmp_path):
    """Kubo.PDOSDist: one folder per atom in the window (coords file and DOS files), then the time
    evolution continuing from the last atom's start vector, as the reference's CalcKubo does."""
    from oracle import pdos as OP
    keys = {"Run.Prefix": "gr", "Run.TypeOfSystem": "Graphene", "Structure.CellSize": 60, "TB.Hopping": 2.7,
            "MagField.Integer": 2, "Kubo.RecursionNumber": 120, "Kubo.NumberofEnergyPoints": 300,
            "Kubo.Epsilon": 0.05, "Kubo.EnergyMin": -8.0, "Kubo.EnergyMax": 8.0, "Kubo.PDOS": True,
            "Kubo.PDOSDist": True, "Kubo.PDOSxmin": 10.0, "Kubo.PDOSxmax": 14.0, "Kubo.PDOSymin": 5.0,
            "Kubo.PDOSymax": 9.0, "Kubo.NumberofPolynomials": 30, "Kubo.TimeStep": 1.5,
            "Kubo.NumberofTimeSteps": 2, "Kubo.WriteNumberofSteps": 2}
    path = str(tmp_path / "Gendata.in")
    _write(path, keys)
    subprocess.run([DRIVER, path], check=True, cwd=str(tmp_path), capture_output=True, text=True)
    r = R.build(dict(TypeOfSystem="Graphene", CellSize=60, Hopping=2.7, MagFieldInteger=2))
    geo, g0 = r["geo"], r["g0"]
    n = geo["n"]
    sel = OP.select_atoms(OP.DIST, geo["rat"], geo["species"], geo["layer"], geo["ucell"], xmin=10.0, xmax=14.0,
                          ymin=5.0, ymax=9.0)
    assert len(sel) >= 2
    folders = sorted(d for d in os.listdir(tmp_path) if d.startswith("PDOS_atom"))
    assert folders == [f"PDOS_atom{i:08d}" for i, _ in sel]
    for i, xyz in sel:
        folder = tmp_path / f"PDOS_atom{i:08d}"
        line = np.loadtxt(folder / "coords")
        assert int(line[0]) == i and np.abs(line[1:] - np.asarray(xyz)).max() <= 1e-15 * 200
        a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], OP.site_start_vector(n, i), 120, 0)
        a = np.loadtxt(folder / "gr.a0.dat")
        b = np.loadtxt(folder / "gr.b0.dat")
        assert np.abs(a - a0).max() <= 1e-10 * np.abs(a0).max() and np.abs(b - b0).max() <= 1e-10 * np.abs(b0).max()
    # KuboTEvol from the last atom's start vector, files under the last atom's prefix
    last = sel[-1][0]
    psi = OP.site_start_vector(n, last)
    a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 120, 0)
    ac, bc = orc.interval(a0, b0)
    c = orc.cheb_coef(1.5, ac, bc, 30)
    zu = np.zeros(n, np.complex128)
    for _ in range(2):
        psi, zu = orc.evol(r["nb"], r["hop"], r["h0"], c, ac, bc, psi, zu, 1)
    norm = float(np.vdot(zu, zu).real)
    az, bz = orc.recursion(r["nb"], r["hop"], r["h0"], zu / np.sqrt(norm), 120, 0)
    folder = tmp_path / f"PDOS_atom{last:08d}"
    ab = np.loadtxt(folder / "gr.AB_0002.dat", skiprows=1)
    assert np.abs(ab[:, 0] - az).max() <= 1e-9 * np.abs(az).max()
    assert np.abs(ab[:, 1] - bz).max() <= 1e-9 * np.abs(bz).max()


def _parse_v(path):
    tok = open(path).read().split()
    out, p = [], 0
    while p < len(tok):
        k = int(tok[p]); p += 1
        out.append([int(x) for x in tok[p:p + k]]); p += k
    return out


@pytest.mark.gpu
def test_driver_write_data_files(tmp_path):
    """Output.WriteDataFiles: the neighbour files (v, dx, dy, dz, pos, neighCell.dat, neighD.dat) and the
    Hamiltonian files (<prefix>.s.mag with the field's phases, .e, .pos, .cell) against the oracle's
    tables, read the way the reference's tools/hamiltonian/verify_tables.py reads them."""
    import re
    keys = dict(INPUTS["moire_sweep"], **{"Output.WriteDataFiles": True, "MagField.Integer": 2, "Kubo.RecursionNumber": 20})
    path = str(tmp_path / "Gendata.in")
    _write(path, keys)
    subprocess.run([DRIVER, path], check=True, cwd=str(tmp_path), capture_output=True, text=True)
    base = dict(TypeOfSystem="Graphene", CellSize=11, SuperCell=4, LatticePercent=-1.0 / 11.0, MoirePotential=True,
                MoireJeil=True, MoireH0AndHZ=True, MoireOffDiag=True, MoireOffDiagMidpoint=True, MagFieldInteger=2)
    r = R.build(base)
    nb, geo = r["nb"], r["geo"]
    n = geo["n"]
    rows = _parse_v(tmp_path / "v")
    assert [len(x) for x in rows] == list(nb["nneigh"])
    assert all(row == list(nb["nlist"][i, :len(row)]) for i, row in enumerate(rows))
    mask = np.arange(nb["max_neigh"])[None, :] < nb["nneigh"][:, None]
    cells = np.loadtxt(tmp_path / "neighCell.dat", dtype=np.int64).reshape(-1, 3)
    assert np.array_equal(cells, nb["ncell"][mask])
    disp = np.loadtxt(tmp_path / "neighD.dat").reshape(-1, 3)
    assert np.array_equal(disp.view(np.int64), nb["neighd"][mask].view(np.int64))   # 17 digits: bitwise
    dx = np.concatenate([np.array(line.split(), float) for line in open(tmp_path / "dx") if line.strip()])
    assert np.abs(dx - nb["neighd"][mask][:, 0]).max() <= 5e-6
    pair = re.compile(r"\(\s*([-+0-9.Ee]+)\s*,\s*([-+0-9.Ee]+)\s*\)")
    hop = [complex(float(a), float(b)) for line in open(tmp_path / "generate.s.mag") for a, b in pair.findall(line)]
    assert np.abs(np.array(hop) - r["hop"][mask]).max() <= 1e-13
    e = np.loadtxt(tmp_path / "generate.e")
    assert np.abs(e[:, 0] - r["h0"]).max() <= 1e-13
    assert np.array_equal(e[:, 1].astype(int), geo["species"]) and np.array_equal(e[:, 2].astype(int), geo["layer"])
    pos = np.loadtxt(tmp_path / "generate.pos")
    assert np.array_equal(pos, r["rat_hop"])
    cell = np.loadtxt(tmp_path / "generate.cell")
    u = geo["ucell"].reshape(3, 3)
    assert np.array_equal(cell[:3], u)
    assert np.abs(cell[3:] @ u.T - 2 * np.pi * np.eye(3)).max() <= 1e-12
    labels = [line.split()[0] for line in open(tmp_path / "pos")]
    assert labels == ["C"] * n
    bottom = np.loadtxt(tmp_path / "generate.bottom.e")
    assert np.abs(bottom[:, 0] - r["h0_bottom"]).max() <= 1e-13
    assert np.array_equal(bottom[:, 1].astype(int), geo["species"])
    assert not (tmp_path / "generate.top.e").exists()


@pytest.mark.gpu
def test_driver_second_moire_files(tmp_path):
    """Moire.AddSecondMoire with Output.WriteDataFiles: <prefix>.e, .bottom.e (H0 after the first moire) and
    .top.e (the second moire's term, H0 - H0Bottom), ham.F90:7020-7034, and the hoppings with the second
    moire's bond terms, against the oracle."""
    import re
    keys = dict(INPUTS["moire_sweep"], **{"Output.WriteDataFiles": True, "Kubo.RecursionNumber": 20,
                                          "Moire.AddSecondMoire": True, "Moire.Twisted2": True,
                                          "Moire.TwistAngle2": 0.7, "Moire.LatticePercentFactor": 1.3,
                                          "Moire.LayerShift2": 0.9, "Moire.SecondMoireMassFactor": -1.0})
    path = str(tmp_path / "Gendata.in")
    _write(path, keys)
    subprocess.run([DRIVER, path], check=True, cwd=str(tmp_path), capture_output=True, text=True)
    r = R.build(dict(TypeOfSystem="Graphene", CellSize=11, SuperCell=4, LatticePercent=-1.0 / 11.0,
                     MoirePotential=True, MoireJeil=True, MoireH0AndHZ=True, MoireOffDiag=True,
                     MoireOffDiagMidpoint=True, MoireAddSecondMoire=True, MoireTwisted2=True, MoireTwistAngle2=0.7,
                     LatticepercentFactor=1.3, MoireLayerShift2=0.9, MoireSecondMoireMassFactor=-1.0))
    nb, geo = r["nb"], r["geo"]
    mask = np.arange(nb["max_neigh"])[None, :] < nb["nneigh"][:, None]
    pair = re.compile(r"\(\s*([-+0-9.Ee]+)\s*,\s*([-+0-9.Ee]+)\s*\)")
    hop = [complex(float(a), float(b)) for line in open(tmp_path / "generate.s.mag") for a, b in pair.findall(line)]
    assert np.abs(np.array(hop) - r["hop"][mask]).max() <= 1e-13
    e = np.loadtxt(tmp_path / "generate.e")
    assert np.abs(e[:, 0] - r["h0"]).max() <= 1e-13
    bottom = np.loadtxt(tmp_path / "generate.bottom.e")
    top = np.loadtxt(tmp_path / "generate.top.e")
    assert np.abs(bottom[:, 0] - r["h0_bottom"]).max() <= 1e-13
    assert np.abs(top[:, 0] - r["h0_top"]).max() <= 1e-13 and np.abs(top[:, 0]).max() > 1e-4
    assert np.array_equal(top[:, 1].astype(int), geo["species"])


@pytest.mark.gpu
@pytest.mark.parametrize("details", [True, False])
def test_driver_read_data_files(tmp_path, details):
    """Output.ReadDataFiles: neighbour list from v (images from neighCell.dat / neighD.dat with
    Neigh.ReadDetails, else the nearest in-plane image), H0 from generate.e, field-free hoppings from
    generate.s, then the Peierls phases of MagField.Integer 3: a_n, b_n against the oracle."""
    r0 = R.build(dict(TypeOfSystem="Graphene", CellSize=40, Hopping=2.7))
    nb = r0["nb"]
    mask = np.arange(nb["max_neigh"])[None, :] < nb["nneigh"][:, None]
    with open(tmp_path / "v", "w") as f:
        for i in range(len(nb["nneigh"])):
            f.write(f"{nb['nneigh'][i]:12d}\n" + " ".join(f"{x:8d}" for x in nb["nlist"][i, :nb["nneigh"][i]]) + "\n")
    if details:
        np.savetxt(tmp_path / "neighCell.dat", nb["ncell"][mask], fmt="%6d")
        np.savetxt(tmp_path / "neighD.dat", nb["neighd"][mask], fmt="%24.16E")
    np.savetxt(tmp_path / "generate.e", np.c_[r0["h0"], r0["geo"]["species"], r0["geo"]["layer"]], fmt="%.17g")
    hop = r0["hop"][mask]
    np.savetxt(tmp_path / "generate.s", np.c_[hop.real, hop.imag], fmt="%.17g")
    keys = {"Run.Prefix": "rd", "Run.TypeOfSystem": "Graphene", "Structure.CellSize": 40, "TB.Hopping": 2.7,
            "Output.ReadDataFiles": True, "Neigh.ReadDetails": details, "MagField.Integer": 3,
            "Kubo.RecursionNumber": 150, "Kubo.SeedValue": 9, "Calculate.OnlyDOS": True}
    path = str(tmp_path / "Gendata.in")
    _write(path, keys)
    subprocess.run([DRIVER, path], check=True, cwd=str(tmp_path), capture_output=True, text=True)
    r = R.build(dict(TypeOfSystem="Graphene", CellSize=40, Hopping=2.7, MagFieldInteger=3))
    n = r["geo"]["n"]
    a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], orc.init_wf(n, 9), 150, 0)
    a = np.loadtxt(tmp_path / "rd.a0.dat")
    b = np.loadtxt(tmp_path / "rd.b0.dat")
    scale = max(np.abs(a0).max(), np.abs(b0).max())
    assert np.abs(a - a0).max() <= 1e-10 * scale and np.abs(b - b0).max() <= 1e-10 * scale


@pytestmark_cpu
def test_driver_reads_pdos_and_haldane_keys(tmp_path):
    """The first PDOS flag that is set wins, PDOSMoireSuperMoire defaulting to .true. (calc.F90:214-300);
    Haldane.T2 is read in eV; HaldPhase bounds only with Haldane.SpecifyRange (magf.F90:148-211)."""
    path = str(tmp_path / "Gendata.in")
    _write(path, {"Kubo.PDOS": True, "Kubo.PDOSAtomList": True, "TB.Hopping": 2.7})
    got = _print_job(path)
    assert got["pdos_mode"] == G.PDOS_SUPERMOIRE   # the default-true SuperMoire flag comes before AtomList
    _write(path, {"Kubo.PDOS": True, "Kubo.PDOSMoireSuperMoire": False, "Kubo.PDOSMoireSuperMoire2": False,
                  "Kubo.PDOSMoireSuperMoire3": False, "Kubo.PDOSAtomList": True, "Kubo.PDOSLayer": True})
    assert _print_job(path)["pdos_mode"] == G.PDOS_LAYER
    _write(path, {"TB.Hopping": 2.7, "Haldane.NNN": True, "Haldane.T2": 0.27, "Haldane.SpecifyRange": True,
                  "HaldPhase.InitialInteger": 0, "HaldPhase.FinalInteger": 6, "HaldPhase.Step": 3})
    got = _print_job(path)
    assert got["haldane"] == 1 and got["hal_mode"] == 3 and got["mphi"] == [0, 6, 3]
    assert math.isclose(got["hal_t2"], 0.1, rel_tol=1e-15)
    _write(path, {"Haldane.NNN": True, "Haldane.SpecifyPhase": True, "Haldane.Phase": 1.0,
                  "HaldPhase.InitialInteger": 0, "HaldPhase.FinalInteger": 6})
    got = _print_job(path)
    assert got["hal_mode"] == 2 and got["mphi"][:2] == [0, 0]   # no sweep without SpecifyRange


@pytest.mark.gpu
def test_driver_layer_shift_sweep(tmp_path):
    """moireBLShift.Calc with Moire.BLShiftRange (calc.F90:40-60, moireBLShift.F90): the encapsulated AB
    bilayer at three layer shifts, one folder X1_.._Y1_.._X2_.._Y2_.. per shift; a_n, b_n and the DOS of each
    against the oracle's Hamiltonian with those shifts.  The same sweep through grabnes_b200.launch with two
    ranks (each its own process; no kernel waits on another) writes the same folders with the same numbers."""
    import sys
    keys = dict(INPUTS["encapsulated_shift_sweep"])
    one, two = tmp_path / "one", tmp_path / "two"
    one.mkdir()
    two.mkdir()
    for d in (one, two):
        _write(str(d / "Gendata.in"), keys)
    subprocess.run([DRIVER, "Gendata.in"], check=True, cwd=str(one), capture_output=True, text=True)
    units = M.blshift_units(keys)
    folders = sorted(d for d in os.listdir(one) if d.startswith("X1_"))
    assert folders == sorted(f for _, f in units)
    base = dict(TypeOfSystem="MoireEncapsulatedBilayerBasedOnMoireCell", MoireCellParameters=(6, 0, 6, 0),
                SuperCell=4, TwistedBLAddShift=True, BernalShift=True, InterlayerDistance=3.34, TypeOfBL="Koshino",
                NeighLevels=5, LayerNeighbors=100, LayerDistFactor=3.2, MoirePotential=True, MoireJeil=True,
                MoireH0AndHZ=True, MoireOffDiag=True, LatticePercent=-0.0166, MoireBilayerBottomAngle=0.4,
                MoireBilayerTopAngle=-0.9)
    for tau, folder in units:
        r = R.build(dict(base, MoireBilayerBottomXShift=tau[0], MoireBilayerBottomYShift=tau[1],
                         MoireBilayerTopXShift=tau[2], MoireBilayerTopYShift=tau[3]))
        n, g0 = r["geo"]["n"], r["g0"]
        a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], orc.init_wf(n, 11), 100, 0)
        a = np.loadtxt(one / folder / "generate.a0.dat")
        b = np.loadtxt(one / folder / "generate.b0.dat")
        assert np.abs(a - a0).max() <= 1e-10 * np.abs(a0).max() and np.abs(b - b0).max() <= 1e-10 * np.abs(b0).max()
        _, d0 = orc.frac(a0, b0, 0.01 / g0, 1000, -1.0 / g0, 1.0 / g0)
        dos = np.loadtxt(one / folder / "generate.DOS")
        assert np.abs(dos[:, 1] - d0).sum() <= 1e-6 * np.abs(d0).sum()
    env = dict(os.environ, PYTHONPATH=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    p = subprocess.run([sys.executable, "-m", "grabnes_b200.launch", "--gpus", "2", "Gendata.in"], cwd=str(two),
                       env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert sorted(d for d in os.listdir(two) if d.startswith("X1_")) == folders
    for folder in folders:
        for name in ("generate.a0.dat", "generate.b0.dat"):
            x, y = np.loadtxt(one / folder / name), np.loadtxt(two / folder / name)
            assert np.abs(x - y).max() <= 1e-10 * np.abs(y).max()


@pytestmark_cpu
def test_driver_layer_shift_units(tmp_path):
    """The driver's shift units (its --print-job units line with GRABNES_RANK / NRANKS) follow the
    package's blshift_units: three shifts, on ranks 0, 1, 0."""
    keys = dict(INPUTS["encapsulated_shift_sweep"])
    path = str(tmp_path / "Gendata.in")
    _write(path, keys)
    assert len(M.blshift_units(keys)) == 3
    for rank in (0, 1):
        env = dict(os.environ, GRABNES_RANK=str(rank), GRABNES_NRANKS="2")
        _, units = _print_job(path, env)
        assert units["units"] == [[u, 0] for u in range(3) if u % 2 == rank]
