"""CPU tests of the oracle (pinning it to the reference) and of the engine's host-side reader.

* the Python restatement of the ffield reader reproduces the reference's canonical table dump byte for byte;
* the C restatement of the cpu64 engine reproduces the reference's golden vectors (generated from the reference
  itself, tests/golden/make_golden.py) and, where the reference oracle is built, the reference live;
* the oracle's charge solve satisfies the equalisation conditions and its matrix equals an independent brute-force
  construction over periodic images;
* the engine's own C++ reader (librxcuda.so, host-only context) reproduces the same dump.
"""
from pathlib import Path

import numpy as np
import pytest

from helpers import ffield_text, fixed_charges, small_systems

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def coracle():
    from oracle.oracle import COracle
    return COracle(ffield_text(), shell=15.0)


def _golden_system(path):
    z = np.load(path)
    s = {k: z[k] for k in ["x", "type", "tag", "box", "origin", "periodic"]}
    s["name"] = path.stem
    return s, z


def test_python_reader_matches_reference_dump():
    from oracle import ffield
    assert ffield.canonical_dump(ffield.parse(ffield_text())) == (GOLDEN / "ffield_synthetic.dump.txt").read_text()


@pytest.mark.parametrize("name", ["water192", "cho3_108", "cho7_78", "cho11_141", "carbon200",
                                  "water192_vdw1", "water192_vdw2", "water192_lg", "water192_acks2"])
def test_oracle_matches_golden(name):
    """The C restatement against the reference's own outputs (energies, gradient, census, counts and the fdotr
    virial), including the force-field variants that switch the non-bonded branches (vdW types 1 and 2, lgvdw) and the
    pair side of the ACKS2 charge model."""
    from oracle.oracle import COracle
    import make_synthetic_ffield
    s, z = _golden_system(GOLDEN / (name + ".npz"))
    variant = name.rsplit("_", 1)[-1]
    variant = variant if variant in make_synthetic_ffield.VARIANTS else "vdw3"
    orc = COracle(make_synthetic_ffield.render(variant), shell=15.0, lgvdw=(variant == "lg"))
    r = orc.single_point(s, z["q"], s_kin=z["s_kin"] if "s_kin" in z.files else None)
    assert np.array_equal(r["census"], z["census"])
    assert np.array_equal(r["counts"], z["counts"])
    assert np.abs(r["e"] - z["e"]).max() <= 1e-9 * max(1.0, np.abs(z["e"]).max())
    assert np.abs(r["grad"] - z["grad"]).max() <= 1e-9
    assert np.abs(r["virial"] - z["virial"]).max() <= 1e-9 * max(1.0, np.abs(z["virial"]).max())


@pytest.mark.parametrize("idx", [0, 1, 4])
def test_oracle_virial_is_the_strain_derivative(coracle, idx):
    """An independent check of the virial's definition (every periodic image counted at its own position): under the
    affine strain x_b -> x_b + eps x_a of the atoms and the lattice, dE/deps = -W_ab. Central differences of the
    oracle's energy (charges held fixed) against its fdotr virial, within 1e-6 of the largest component."""
    s = small_systems()[idx]
    q = fixed_charges(s)
    w = coracle.single_point(s, q)["virial"]

    def energy(a, b, eps):
        F = np.eye(3)
        F[b, a] += eps
        st = dict(s)
        st["x"] = s["x"] @ F.T
        st["box"] = np.asarray(s["box"]) @ F.T
        st["origin"] = np.asarray(s["origin"]) @ F.T
        return coracle.single_point(st, q)["e"].sum()

    h = 1e-6
    fd = np.array([-(energy(a, b, h) - energy(a, b, -h)) / (2 * h)
                   for a, b in [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]])
    assert np.abs(fd - w).max() <= 1e-6 * np.abs(w).max(), (fd, w)


def test_oracle_variants_match_reference_live():
    from oracle.oracle import COracle, RefOracle
    import make_synthetic_ffield
    import systems
    if not RefOracle.available():
        pytest.skip("reference oracle not built here")
    s = systems.random_cho(7)
    q = fixed_charges(s)
    for v in make_synthetic_ffield.VARIANTS:
        text = make_synthetic_ffield.render(v)
        a = COracle(text, shell=15.0, lgvdw=(v == "lg")).single_point(s, q)
        b = RefOracle(text, shell=15.0, lgvdw=(v == "lg")).single_point(s, q)
        assert np.array_equal(a["census"], b["census"]), v
        assert np.abs(a["e"] - b["e"]).max() <= 1e-9 * max(1.0, np.abs(b["e"]).max()), v
        assert np.abs(a["grad"] - b["grad"]).max() <= 1e-9, v
        assert np.abs(a["virial"] - b["virial"]).max() <= 1e-9 * max(1.0, np.abs(b["virial"]).max()), v


def test_golden_fixtures_are_current():
    """The fixtures were generated from the systems the GPU tests use (same seeds)."""
    for s in small_systems():
        z = np.load(GOLDEN / (s["name"] + ".npz"))
        assert np.array_equal(z["x"], s["x"]) and np.array_equal(z["q"], fixed_charges(s))


def test_oracle_matches_reference_live(coracle):
    from oracle.oracle import RefOracle
    if not RefOracle.available():
        pytest.skip("reference oracle not built here")
    ref = RefOracle(ffield_text(), shell=15.0)
    for s in small_systems()[:3]:
        q = fixed_charges(s)
        a, b = coracle.single_point(s, q), ref.single_point(s, q)
        assert np.array_equal(a["census"], b["census"])
        assert np.abs(a["e"] - b["e"]).max() <= 1e-9 * max(1.0, np.abs(b["e"]).max())


def test_oracle_enobonds_and_shell(coracle):
    """Edge cases the reference tests: an isolated atom (no bonds; enobonds on/off) and a larger ghost shell."""
    from oracle.oracle import COracle
    import systems
    s = systems.random_cho(3)
    s["x"] = s["x"].copy()
    s["x"][0] = s["x"][0] + 0.0   # unchanged geometry; the shell must not change owned results
    a = coracle.single_point(s, fixed_charges(s))
    wide = COracle(ffield_text(), shell=20.0).single_point(s, fixed_charges(s))
    assert np.array_equal(a["census"], wide["census"])
    assert np.abs(a["e"] - wide["e"]).max() <= 1e-9 * max(1.0, np.abs(a["e"]).max())
    lone = {"origin": np.zeros(3), "box": np.eye(3) * 30.0, "periodic": np.ones(3, dtype=np.int32),
            "x": np.array([[1.0, 1.0, 1.0], [15.0, 15.0, 15.0]]), "type": np.array([0, 2], dtype=np.int32),
            "tag": np.array([1, 2], dtype=np.int64)}
    on = coracle.single_point(lone, np.zeros(2))
    off = COracle(ffield_text(), enobonds=False, shell=15.0).single_point(lone, np.zeros(2))
    assert on["census"][0].sum() == 0
    assert off["e"][3] == 0.0 and off["e"][2] == 0.0      # no lone-pair / under-coordination without bonds
    assert on["e"][3] != 0.0


def _brute_force_h(s, tables, swb=10.0, swa=0.0):
    """Independent charge matrix: all periodic images within swb, both directions, by direct enumeration."""
    x, t = s["x"], s["type"]
    L = np.asarray(s["box"])
    n = len(t)
    from oracle.ffield import parse  # noqa: F401  (tables come from the same restated reader)
    d1 = swb - swa
    d7 = d1 ** 7
    c = np.zeros(8)
    swa2, swa3, swb2, swb3 = swa * swa, swa ** 3, swb * swb, swb ** 3
    c[7] = 20.0 / d7
    c[6] = -70.0 * (swa + swb) / d7
    c[5] = 84.0 * (swa2 + 3.0 * swa * swb + swb2) / d7
    c[4] = -35.0 * (swa3 + 9.0 * swa2 * swb + 9.0 * swa * swb2 + swb3) / d7
    c[3] = 140.0 * (swa3 * swb + 3.0 * swa2 * swb2 + swa * swb3) / d7
    c[2] = -210.0 * (swa3 * swb2 + swa2 * swb3) / d7
    c[1] = 140.0 * swa3 * swb3 / d7
    c[0] = (-35.0 * swa3 * swb2 * swb2 + 21.0 * swa2 * swb3 * swb2 - 7.0 * swa * swb3 * swb3 + swb3 * swb3 * swb) / d7
    gam = np.array([sb["gamma"] for sb in tables["sbp"]])
    H = np.zeros((n, n))
    rng = range(-2, 3)
    for a in rng:
        for b in rng:
            for cc in rng:
                sh = a * L[0] + b * L[1] + cc * L[2]
                dv = x[None, :, :] + sh - x[:, None, :]
                r = np.sqrt((dv ** 2).sum(-1))
                mask = (r <= swb) & (r > 1e-9)
                rr = np.where(mask, r, 1.0)
                tap = np.polyval(c[::-1], rr)
                shld = (gam[t][:, None] * gam[t][None, :]) ** -1.5
                H += np.where(mask, tap * 14.4 / np.cbrt(rr ** 3 + shld), 0.0)
    return H


def test_oracle_charge_matrix_brute_force(coracle):
    import systems
    s = systems.random_cho(7)
    H = _brute_force_h(s, coracle.tables)
    eta = np.array([coracle.tables["sbp"][t]["eta"] for t in s["type"]])
    v = np.random.default_rng(3).normal(size=len(s["type"]))
    y = coracle.qeq_matvec(s, v)
    assert np.abs(y - (eta * v + H @ v)).max() <= 1e-10 * np.abs(y).max()


def test_oracle_qeq_equalisation(coracle):
    """Solved charges are neutral and equalise the chemical potential (the reference's independent EEM residual)."""
    s = small_systems()[0]
    r = coracle.qeq(s, tol=1e-12, imax=500)
    q = r["q"]
    assert abs(q.sum()) <= 1e-10
    eta = np.array([coracle.tables["sbp"][t]["eta"] for t in s["type"]])
    chi = coracle.chi(s["type"])
    mu = coracle.qeq_matvec(s, q) + chi
    assert np.ptp(mu) <= 1e-8          # tolerances.json C3 equalization_residual_eV = 0.002
    assert r["rel"].max() <= 1e-12


def test_engine_reader_matches_reference_dump():
    """The engine's own C++ reader, through the C ABI on a host-only context (no GPU needed)."""
    import rxcuda
    if not rxcuda.LIB_PATH.exists():
        pytest.skip("librxcuda.so not built")
    e = rxcuda.Engine(-1)
    e.set_forcefield(ffield_text())
    assert e.forcefield_dump() == (GOLDEN / "ffield_synthetic.dump.txt").read_text()
    p = e.forcefield_params()
    assert p["eta"][2] == 2 * 8.3 and p["eta"][1] == 2 * 9.6 and p["chi"][0] == 5.9
    with pytest.raises(rxcuda.RxError):
        e.set_systems([small_systems()[1]])
    e.close()


def test_engine_reader_rejects_bad_files():
    import rxcuda
    if not rxcuda.LIB_PATH.exists():
        pytest.skip("librxcuda.so not built")
    e = rxcuda.Engine(-1)
    text = ffield_text()
    bad = text.replace(" 39       ! Number of general parameters", " 30       ! Number of general parameters", 1)
    with pytest.raises(rxcuda.RxError) as ei:
        e.set_forcefield(bad)
    assert ei.value.code == 2
    with pytest.raises(rxcuda.RxError):
        e.set_forcefield(text[: len(text) // 2])     # truncated file (strict mode rejects)
    e.close()


def test_oracle_matches_reference_triclinic(coracle):
    """General triclinic box (system.hpp Box: lattice rows a, b, c with tilts): the restatement against the reference."""
    from oracle.oracle import RefOracle
    import systems
    if not RefOracle.available():
        pytest.skip("reference oracle not built here")
    s = systems.triclinic(systems.water_box(4))
    q = fixed_charges(s)
    a, b = coracle.single_point(s, q), RefOracle(ffield_text(), shell=15.0).single_point(s, q)
    assert np.array_equal(a["census"], b["census"])
    assert np.abs(a["e"] - b["e"]).max() <= 1e-9 * max(1.0, np.abs(b["e"]).max())
    assert np.abs(a["grad"] - b["grad"]).max() <= 1e-9
