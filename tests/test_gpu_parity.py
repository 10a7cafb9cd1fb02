"""GPU parity: the CUDA engine (through its C ABI) against the CPU oracle (the C restatement of the reference's cpu64
engine, pinned against the reference itself in test_oracle.py).

Bars (the reference's own acceptance of an FP32 GPU engine against cpu64, tolerances/tolerances.json "C3"):
  energy  |dE_total| / N <= 1e-3 kcal/mol/atom
  force   max |dF| <= 0.05, RMS <= 5e-3 kcal/mol/A
  census  every discrete decision (bonds, angle sets, torsions, H-bonds, non-bonded pairs, SBO branch, lone-pair
          truncation) identical atom by atom
Tighter bars for the terms computed in FP64 (bond, over/under, lone pair, valence, penalty, coalition, torsion,
conjugation): within 1e-7 relative (max(1, |E|)); the FP32 H-bond term within 2e-5 relative.
"""
import numpy as np
import pytest

from helpers import (C3_ENERGY_PER_ATOM, C3_FORCE_MAX, C3_FORCE_RMS, fixed_charges, ffield_text, force_metrics,
                     small_systems)

pytestmark = pytest.mark.gpu

FP64_TERMS = [0, 1, 2, 3, 4, 5, 6, 8, 9]
HBOND = 7


@pytest.fixture(scope="module")
def oracle():
    from oracle.oracle import COracle
    return COracle(ffield_text(), shell=15.0)


@pytest.fixture(scope="module")
def engine():
    import rxcuda
    e = rxcuda.Engine(0)
    e.set_forcefield(ffield_text())
    e.set_control()
    yield e
    e.close()


@pytest.mark.parametrize("idx", range(5))
def test_single_point_matches_oracle(engine, oracle, idx):
    s = small_systems()[idx]
    q = fixed_charges(s)
    ref = oracle.single_point(s, q)
    engine.set_systems([s])
    engine.set_charges(q)
    out = engine.compute(census=True, counts=True)
    e, e_ref = out["e"][0], ref["e"]
    n = len(s["type"])
    # FP64 bond-order terms: tight; FP32 H-bonds: FP32 level
    rel = np.abs(e[FP64_TERMS] - e_ref[FP64_TERMS]) / np.maximum(1.0, np.abs(e_ref[FP64_TERMS]))
    assert rel.max() <= 1e-7, (s["name"], e[FP64_TERMS], e_ref[FP64_TERMS])
    assert abs(e[HBOND] - e_ref[HBOND]) <= 2e-5 * max(1.0, abs(e_ref[HBOND])), (s["name"], e[HBOND], e_ref[HBOND])
    # total energy per atom (C3)
    assert abs(e.sum() - e_ref.sum()) / n <= C3_ENERGY_PER_ATOM, (s["name"], e, e_ref)
    fmax, frms = force_metrics(ref["grad"], out["grad"])
    assert fmax <= C3_FORCE_MAX and frms <= C3_FORCE_RMS, (s["name"], fmax, frms)
    # every discrete decision identical
    for k, name in enumerate(["bonds", "angle_sets", "torsions", "hbonds", "nonbonded", "sbo_region", "lp_trunc"]):
        assert np.array_equal(out["census"][k], ref["census"][k]), (s["name"], name)


def test_bonded_gradient_tight(engine, oracle):
    """Without charges the gradient is the FP64 bonded chain alone plus FP32 van der Waals: compare tightly."""
    s = small_systems()[1]
    q = np.zeros(len(s["type"]))
    ref = oracle.single_point(s, q)
    engine.set_systems([s])
    engine.set_charges(q)
    out = engine.compute()
    fmax, frms = force_metrics(ref["grad"], out["grad"])
    assert fmax <= 5e-3 and frms <= 1e-3, (fmax, frms)


def test_bitwise_rerun(engine):
    """FORCE-2 of the reference (tests/python/test_gpu_fixtures.py:58): two runs give identical bits."""
    s = small_systems()[0]
    engine.set_systems([s])
    engine.set_charges(fixed_charges(s))
    a = engine.compute()
    engine.set_systems([s])
    engine.set_charges(fixed_charges(s))
    b = engine.compute()
    assert np.array_equal(a["e"], b["e"]) and np.array_equal(a["grad"], b["grad"])


def test_qeq_charges_match_oracle(engine, oracle):
    s = small_systems()[0]
    engine.set_systems([s])
    engine.set_qeq(0.0, 10.0, 1e-12, 400)
    got = engine.qeq_solve()
    ref = oracle.qeq(s, tol=1e-12, imax=400)
    assert np.abs(got["q"] - ref["q"]).max() <= 1e-10
    assert abs(got["q"].sum()) <= 1e-9
    engine.set_qeq()


def test_qeq_tol_1e6_within_c3(engine, oracle):
    s = small_systems()[0]
    engine.set_systems([s])
    engine.qeq_reset()
    engine.set_qeq(0.0, 10.0, 1e-6, 200)
    got = engine.qeq_solve()
    ref = oracle.qeq(s, tol=1e-6, imax=200)
    assert np.abs(got["q"] - ref["q"]).max() <= 1e-4
    assert tuple(got["iters"][0]) == tuple(ref["iters"])


def test_qeq_matvec_matches_oracle(engine, oracle):
    s = small_systems()[2]
    engine.set_systems([s])
    v = np.random.default_rng(5).normal(size=len(s["type"]))
    y = engine.qeq_matvec(v)
    y_ref = oracle.qeq_matvec(s, v)
    assert np.abs(y - y_ref).max() <= 1e-10 * max(1.0, np.abs(y_ref).max())


def test_batch_equals_alone(engine):
    """Each system's result is the same alone and inside a batch (per-system reductions in fixed order)."""
    ss = small_systems()[1:4]
    alone = []
    for s in ss:
        engine.set_systems([s])
        engine.set_charges(fixed_charges(s))
        alone.append(engine.compute())
    engine.set_systems(ss)
    engine.set_charges(np.concatenate([fixed_charges(s) for s in ss]))
    both = engine.compute()
    off = 0
    for k, s in enumerate(ss):
        n = len(s["type"])
        assert np.array_equal(both["e"][k], alone[k]["e"][0])
        assert np.array_equal(both["grad"][off:off + n], alone[k]["grad"])
        off += n


def test_batched_charges_equal_alone_and_oracle(engine, oracle):
    """Batching form: the charge solve of a batch gives every system the same bits as its solve alone (per-system
    fixed-order reductions), and the oracle's charges within 1e-10 e at tol 1e-12."""
    import systems
    ss = [systems.random_cho(k) for k in (0, 4, 9, 21, 33, 40)]
    engine.set_qeq(0.0, 10.0, 1e-12, 400)
    engine.set_systems(ss)
    engine.qeq_reset()
    both = engine.qeq_solve()
    off = 0
    for k, s in enumerate(ss):
        n = len(s["type"])
        engine.set_systems([s])
        engine.qeq_reset()
        alone = engine.qeq_solve()
        assert np.array_equal(alone["q"], both["q"][off:off + n]), s["name"]
        assert np.array_equal(alone["iters"][0], both["iters"][k])
        ref = oracle.qeq(s, tol=1e-12, imax=400)
        assert np.abs(alone["q"] - ref["q"]).max() <= 1e-10, s["name"]
        assert abs(alone["q"].sum()) <= 1e-9
        off += n
    engine.set_qeq()


def test_batch_of_mixed_systems_matches_oracle(engine, oracle):
    """Eight systems of the 512-system batching workload (uneven sizes and compositions) in one batch, each against
    the oracle under the same bars as the single-system test."""
    import systems
    ss = [systems.random_cho(k) for k in (1, 5, 12, 77, 130, 256, 300, 511)]
    qs = [fixed_charges(s) for s in ss]
    engine.set_systems(ss)
    engine.set_charges(np.concatenate(qs))
    out = engine.compute(census=True)
    off = 0
    for k, s in enumerate(ss):
        n = len(s["type"])
        ref = oracle.single_point(s, qs[k])
        e = out["e"][k]
        assert abs(e.sum() - ref["e"].sum()) / n <= C3_ENERGY_PER_ATOM, s["name"]
        fmax, frms = force_metrics(ref["grad"], out["grad"][off:off + n])
        assert fmax <= C3_FORCE_MAX and frms <= C3_FORCE_RMS, (s["name"], fmax, frms)
        for c in range(7):
            assert np.array_equal(out["census"][c][off:off + n], ref["census"][c]), (s["name"], c)
        off += n


def test_capacity_regrowth_gives_same_bits(engine):
    """Failure detection on the host: lists started far too small overflow, the engine grows them from the counts the
    kernels report and repeats the evaluation; the result is bitwise the one with ample capacities."""
    s = small_systems()[2]
    engine.set_systems([s])
    engine.set_charges(fixed_charges(s))
    ref = engine.compute()
    ample = engine.capacities()
    engine.set_capacities(32, 1, 32)
    assert engine.capacities() == (32, 1, 32)
    out = engine.compute()
    grown = engine.capacities()
    assert grown[0] > 32 and grown[1] > 1
    assert np.array_equal(out["e"], ref["e"]) and np.array_equal(out["grad"], ref["grad"])
    assert ample[0] >= 32


def test_strict_qeq_reports_non_convergence(engine):
    """fix qeq/reaxff/metal strict mode (fix_qeq_reaxff_metal.cpp:79-80): hitting imax is an error; otherwise the
    iteration counts and residuals report it."""
    import rxcuda
    s = small_systems()[0]
    engine.set_systems([s])
    engine.set_qeq(0.0, 10.0, 1e-14, 3, strict=True)
    with pytest.raises(rxcuda.RxError) as ei:
        engine.qeq_solve()
    assert ei.value.code == 5
    engine.set_qeq(0.0, 10.0, 1e-14, 3, strict=False)
    r = engine.qeq_solve()
    assert r["iters"].max() <= 3 and r["rel"].max() > 1e-14
    engine.set_qeq()


def test_nvt_batch_equals_alone_and_reruns_bitwise():
    """NVT with charge equilibration every step: a system advanced inside a batch follows bitwise the trajectory it
    follows alone (per-system thermostat sums in fixed chunks, per-system CG reductions), and a rerun repeats it."""
    import rxcuda
    import systems
    mass = [12.0, 1.008, 15.999]
    ss = [systems.random_cho(3), systems.water_box(4)]
    vs = [systems.maxwell_velocities(s, 300.0, seed=7 + k) for k, s in enumerate(ss)]

    def run(group, vel):
        e = rxcuda.Engine(0)
        e.set_forcefield(ffield_text())
        e.set_control()
        e.set_qeq(0.0, 10.0, 1e-6, 200)
        e.set_systems(group)
        e.md_setup(mass, dt=0.25, t_start=300.0, t_damp=25.0, chain=3)
        e.set_velocities(np.concatenate(vel))
        out = e.md_run(20)
        x = e.get_positions()
        e.close()
        return out, x

    alone = [run([s], [v]) for s, v in zip(ss, vs)]
    both, xb = run(ss, vs)
    again, xa = run(ss, vs)
    assert np.array_equal(xb, xa)
    n0 = len(ss[0]["type"])
    assert np.array_equal(alone[0][1], xb[:n0]) and np.array_equal(alone[1][1], xb[n0:])
    for k in range(2):
        assert np.all(np.isfinite(alone[k][1]))


def _check_against_oracle(engine, oracle, s, q):
    ref = oracle.single_point(s, q)
    engine.set_systems([s])
    engine.set_charges(q)
    out = engine.compute(census=True)
    e, e_ref = out["e"][0], ref["e"]
    rel = np.abs(e[FP64_TERMS] - e_ref[FP64_TERMS]) / np.maximum(1.0, np.abs(e_ref[FP64_TERMS]))
    assert rel.max() <= 1e-7, (s["name"], e, e_ref)
    assert abs(e.sum() - e_ref.sum()) / len(s["type"]) <= C3_ENERGY_PER_ATOM
    fmax, frms = force_metrics(ref["grad"], out["grad"])
    assert fmax <= C3_FORCE_MAX and frms <= C3_FORCE_RMS, (s["name"], fmax, frms)
    for k in range(7):
        assert np.array_equal(out["census"][k], ref["census"][k]), (s["name"], k)


def test_triclinic_box_matches_oracle(engine, oracle):
    """A general triclinic cell (tilted lattice rows): images, cut-off pruning by face distances and the lattice-shift
    table on a non-orthogonal box."""
    import systems
    s = systems.triclinic(systems.water_box(4))
    _check_against_oracle(engine, oracle, s, fixed_charges(s))


def test_sparse_system_matches_oracle(engine, oracle):
    """Two far-apart atoms in a large periodic box (no bonds, only images beyond the bond cut-off): every term of the
    empty-list path, and the charge solve of a 2-atom system."""
    s = {"name": "lone2", "origin": np.zeros(3), "box": np.eye(3) * 30.0, "periodic": np.ones(3, dtype=np.int32),
         "x": np.array([[1.0, 1.0, 1.0], [15.0, 15.0, 15.0]]), "type": np.array([0, 2], dtype=np.int32),
         "tag": np.array([1, 2], dtype=np.int64)}
    _check_against_oracle(engine, oracle, s, np.array([0.1, -0.1]))
    engine.set_qeq(0.0, 10.0, 1e-12, 100)
    got = engine.qeq_solve()
    ref = oracle.qeq(s, tol=1e-12, imax=100)
    assert np.abs(got["q"] - ref["q"]).max() <= 1e-10
    engine.set_qeq()


@pytest.mark.parametrize("idx", range(5))
def test_virial_matches_oracle(engine, oracle, idx):
    """The per-system virial (LAMMPS fdotr order xx yy zz xy xz yz) against the oracle's sum of x f over owned and
    ghost atoms. Bars: each component within the C3 energy bar per atom (1e-3 kcal/mol/atom), and within 1e-6 of the
    largest component (FP32 non-bonded and H-bond terms, FP64 elsewhere)."""
    s = small_systems()[idx]
    q = fixed_charges(s)
    ref = oracle.single_point(s, q)
    engine.set_systems([s])
    engine.set_charges(q)
    engine.compute()
    w = engine.virial()[0]
    n = len(s["type"])
    dv = np.abs(w - ref["virial"])
    assert dv.max() / n <= C3_ENERGY_PER_ATOM, (s["name"], w, ref["virial"])
    assert dv.max() <= 1e-6 * np.abs(ref["virial"]).max(), (s["name"], w, ref["virial"])


def test_virial_of_a_batch_is_per_system(engine):
    """Each system's virial is the same alone and inside a batch."""
    ss = small_systems()[1:4]
    alone = []
    for s in ss:
        engine.set_systems([s])
        engine.set_charges(fixed_charges(s))
        engine.compute()
        alone.append(engine.virial()[0])
    engine.set_systems(ss)
    engine.set_charges(np.concatenate([fixed_charges(s) for s in ss]))
    engine.compute()
    both = engine.virial()
    for k in range(len(ss)):
        assert np.array_equal(both[k], alone[k])


@pytest.mark.parametrize("variant", ["vdw1", "vdw2", "lg"])
def test_vdw_variants_match_oracle(variant):
    """The non-bonded branches the default force field does not take: van der Waals with shielding only (type 1), inner
    wall only (type 2), and the lg dispersion of `lgvdw yes` (include/reaxmetal/terms.hpp:280-323). Same bars as the
    single-point test, on the water box and a mixed CHO system."""
    import make_synthetic_ffield
    import rxcuda
    import systems
    from oracle.oracle import COracle
    text = make_synthetic_ffield.render(variant)
    lg = variant == "lg"
    orc = COracle(text, shell=15.0, lgvdw=lg)
    eng = rxcuda.Engine(0)
    eng.set_forcefield(text, lgvdw=lg)
    eng.set_control()
    for s in (systems.water_box(4), systems.random_cho(7)):
        q = fixed_charges(s)
        ref = orc.single_point(s, q)
        eng.set_systems([s])
        eng.set_charges(q)
        out = eng.compute(census=True)
        n = len(s["type"])
        e, e_ref = out["e"][0], ref["e"]
        rel = np.abs(e[FP64_TERMS] - e_ref[FP64_TERMS]) / np.maximum(1.0, np.abs(e_ref[FP64_TERMS]))
        assert rel.max() <= 1e-7, (variant, s["name"])
        assert abs(e[10] - e_ref[10]) <= 1e-5 * max(1.0, abs(e_ref[10])), (variant, s["name"], e[10], e_ref[10])
        assert abs(e.sum() - e_ref.sum()) / n <= C3_ENERGY_PER_ATOM, (variant, s["name"])
        fmax, frms = force_metrics(ref["grad"], out["grad"])
        assert fmax <= C3_FORCE_MAX and frms <= C3_FORCE_RMS, (variant, s["name"], fmax, frms)
        for k in range(7):
            assert np.array_equal(out["census"][k], ref["census"][k]), (variant, s["name"], k)
        assert np.abs(eng.virial()[0] - ref["virial"]).max() / n <= C3_ENERGY_PER_ATOM
    eng.close()


def test_qeq_cg_given_rhs_and_guesses(engine, oracle):
    """mtl::Context::qeq_solve (metal_backend.hpp:84-86) through rx_qeq_cg: the stock right-hand sides (-chi, -1) from
    the oracle's own guesses give the oracle's s and t; iteration limit reported as status 3; the charges are left
    alone."""
    s = small_systems()[0]
    n = len(s["type"])
    engine.set_systems([s])
    engine.set_charges(np.zeros(n))
    engine.set_qeq(0.0, 10.0, 1e-12, 400)
    rng = np.random.default_rng(9)
    s0, t0 = rng.normal(scale=0.1, size=n), rng.normal(scale=0.1, size=n)
    ref = oracle.qeq(s, tol=1e-12, imax=400, s0=s0, t0=t0)
    b = np.stack([-oracle.chi(s["type"]), -np.ones(n)])
    got = engine.qeq_cg(b, np.stack([s0, t0]))
    assert np.abs(got["x"][0] - ref["s"]).max() <= 1e-10 and np.abs(got["x"][1] - ref["t"]).max() <= 1e-10
    assert got["status"].tolist() == [[1, 1]] and got["rel"].max() <= 1e-12
    assert np.abs(engine.get_charges()).max() == 0.0
    engine.set_qeq(0.0, 10.0, 1e-12, 3)
    lim = engine.qeq_cg(b)
    assert lim["status"].tolist() == [[3, 3]] and lim["iters"].max() <= 3
    engine.set_qeq()


def test_set_systems_keeps_charge_history_by_tag(engine):
    """Re-neighbouring (the same atoms handed over again, in another order) keeps each atom's charge history, so the
    next solve starts warm: it takes no more iterations than a solve that was never interrupted, and far fewer than
    a cold one."""
    s = small_systems()[0]
    engine.set_qeq(0.0, 10.0, 1e-8, 200)
    engine.set_systems([s])
    for _ in range(3):
        engine.compute(qeq=True)
    engine.compute(qeq=True)
    warm = engine.qeq_last()["iters"].max()
    perm = np.random.default_rng(3).permutation(len(s["type"]))
    sp = dict(s, x=s["x"][perm], type=s["type"][perm], tag=s["tag"][perm])
    engine.set_systems([sp])
    engine.compute(qeq=True)
    after = engine.qeq_last()["iters"].max()
    engine.compute(qeq=True, cold=True)
    cold = engine.qeq_last()["iters"].max()
    assert after <= warm + 1 and after < cold, (warm, after, cold)
    engine.set_qeq()


def test_acks2_pair_terms_match_oracle():
    """The pair side of fix acks2/reaxff (src/cpu/acks2.cpp:11-63) through rx_set_acks2: with kinetic potentials set,
    the Coulomb and polarization energies, forces and virial match the oracle's under the same bars as the
    single-point test; switched off again, the plain evaluation returns."""
    import make_synthetic_ffield
    import rxcuda
    import systems
    from helpers import acks2_potentials
    from oracle.oracle import COracle
    text = make_synthetic_ffield.render("acks2")
    orc = COracle(text, shell=15.0)
    eng = rxcuda.Engine(0)
    eng.set_forcefield(text)
    eng.set_control()
    for s in (systems.water_box(4), systems.random_cho(7)):
        n = len(s["type"])
        q = fixed_charges(s)
        sk = acks2_potentials(n)
        ref = orc.single_point(s, q, s_kin=sk)
        plain = orc.single_point(s, q)
        eng.set_systems([s])
        eng.set_charges(q)
        eng.set_acks2(sk)
        out = eng.compute(census=True)
        e = out["e"][0]
        assert abs(e[12] - ref["e"][12]) <= 1e-9 * max(1.0, abs(ref["e"][12])), s["name"]
        assert abs(e[11] - ref["e"][11]) <= 1e-5 * max(1.0, abs(ref["e"][11])), s["name"]
        assert abs(e.sum() - ref["e"].sum()) / n <= C3_ENERGY_PER_ATOM
        fmax, frms = force_metrics(ref["grad"], out["grad"])
        assert fmax <= C3_FORCE_MAX and frms <= C3_FORCE_RMS, (s["name"], fmax, frms)
        assert np.abs(eng.virial()[0] - ref["virial"]).max() / n <= C3_ENERGY_PER_ATOM
        eng.set_acks2(None)
        off = eng.compute()
        assert abs(off["e"][0][12] - plain["e"][12]) <= 1e-9 * max(1.0, abs(plain["e"][12]))
    eng.close()


@pytest.mark.parametrize("periodic", [(1, 1, 0), (0, 0, 0)], ids=["slab", "cluster"])
def test_nonperiodic_directions_match_oracle(engine, oracle, periodic):
    """Box::periodic (include/reaxmetal/system.hpp:29): a water slab periodic in x and y only, and a water cluster with
    no periodic direction - no image along a non-periodic direction, atoms never wrapped along it. Same bars as the
    single-point test, virial included."""
    import systems
    s = systems.water_box(4)
    s = dict(s, periodic=np.array(periodic, dtype=np.int32), name="water192_" + "".join(map(str, periodic)))
    _check_against_oracle(engine, oracle, s, fixed_charges(s))
    ref = oracle.single_point(s, fixed_charges(s))
    assert np.abs(engine.virial()[0] - ref["virial"]).max() / len(s["type"]) <= C3_ENERGY_PER_ATOM


def test_peratom_energies_and_bond_table_match_reference(engine):
    """RX_COMPUTE_PERATOM and rx_get_bonds against the reference's own per-atom tallies and bond table (cpu64 with
    BondedOptions::per_atom / bond_table, ghosts folded onto owners): per-atom energies within the reference's C3
    energy bar of each atom (1e-3 kcal/mol: an atom's tally holds half of each of its few hundred FP32 pair energies,
    whose rounding leaves 1e-4-2.5e-4 kcal/mol per atom on these cases, as the per-term totals suggest), summing to the
    total; per-atom virials summing to the global virial; every atom's bonds (partner, corrected bond order to 1e-9),
    total bond order and lone pairs the same."""
    from oracle.oracle import RefOracle
    if not RefOracle.available():
        pytest.skip("reference oracle not built here")
    for s in small_systems()[:3]:
        q = fixed_charges(s)
        ref = RefOracle(ffield_text(), shell=15.0).peratom(s, q)
        engine.set_systems([s])
        engine.set_charges(q)
        out = engine.compute(peratom=True)
        ea, va = engine.peratom()
        assert np.abs(ea - ref["eatom"]).max() <= C3_ENERGY_PER_ATOM, (s["name"], np.abs(ea - ref["eatom"]).max())
        assert abs(ea.sum() - out["e"][0].sum()) <= 1e-6 * max(1.0, abs(out["e"][0].sum()))
        assert np.abs(va.sum(0) - engine.virial()[0]).max() <= 1e-6 * max(1.0, np.abs(engine.virial()[0]).max())
        b = engine.bonds()
        n = len(s["type"])
        assert np.abs(b["total_bo"] - ref["total_bo"]).max() <= 1e-9 and np.abs(b["nlp"] - ref["nlp"]).max() <= 1e-9
        for a in range(n):
            mine = sorted(zip(b["partner"][b["start"][a]:b["start"][a + 1]], b["bo"][b["start"][a]:b["start"][a + 1]]))
            theirs = sorted(zip(ref["partner"][ref["start"][a]:ref["start"][a + 1]], ref["bo"][ref["start"][a]:ref["start"][a + 1]]))
            assert [p for p, _ in mine] == [p for p, _ in theirs], (s["name"], a)
            assert np.allclose([v for _, v in mine], [v for _, v in theirs], rtol=0, atol=1e-9), (s["name"], a)


def test_pinned_arrays_give_the_same_bits(engine):
    """rx_set_positions from page-locked memory and the gradient copied straight into page-locked memory (the device
    does the layout change) give bitwise the results of the pageable path."""
    import rxcuda
    s = small_systems()[0]
    q = fixed_charges(s)
    engine.set_systems([s])
    engine.set_charges(q)
    engine.set_positions(s["x"])
    ref = engine.compute()
    n = len(s["type"])
    x = rxcuda.pinned_array((n, 3))
    x[:] = s["x"]
    g = rxcuda.pinned_array((n, 3))
    engine.set_systems([s])
    engine.set_charges(q)
    engine.set_positions(x)
    out = engine.compute(grad_out=g)
    assert np.array_equal(out["e"], ref["e"])
    assert np.array_equal(g, ref["grad"])


def test_cg_block_size_changes_only_rounding():
    """The single-system CG's threads per SM (RX_TUNE_CG_BLOCKS_PER_SM, one block per SM of 256 x value threads)
    changes the order of its sums and nothing else: at tolerance 1e-12 every size gives the same charges to 1e-10 e,
    each size is bitwise reproducible, and a size outside 0-4 is rejected."""
    import rxcuda
    import systems
    s = systems.water_box(12)   # 5,184 atoms: above the lone-system size, so the single-system CG
    e = rxcuda.Engine(0)
    try:
        e.set_forcefield(ffield_text())
        e.set_control()
        e.set_qeq(0.0, 10.0, 1e-12, 400)
        e.set_systems([s])
        q = {}
        for units in (2, 1, 3, 4, 0, 2):
            e.set_tuning("cg_blocks_per_sm", units)
            e.qeq_reset()
            e.qeq_solve()
            got = e.get_charges()
            if units in q:
                assert np.array_equal(got, q[units]), units
            q[units] = got
        for units, qq in q.items():
            assert np.abs(qq - q[2]).max() <= 1e-10, units
        with pytest.raises(rxcuda.RxError):
            e.set_tuning("cg_blocks_per_sm", 5)
    finally:
        e.close()


def test_half_pair_nonbonded_matches_full_rows(engine):
    """The step's non-bonded kernel computes each pair once and hands the partner its share through the fixed-point
    accumulator; the full-row kernel (taken for per-atom tallies) computes every pair from both ends. Same pairs and the
    same FP32 terms, so energies agree to summation order and the census is identical; the gradients agree to FP32
    rounding (1e-6 of the largest component), because the two ends of a pair round the charge product and the type-pair
    constants in their own order, so the full-row kernel's two shares of a pair differ in their last bits."""
    for s in small_systems()[:3] + [__import__("systems").water_box(8)]:
        q = fixed_charges(s)
        engine.set_systems([s])
        engine.set_charges(q)
        half = engine.compute(census=True)
        full = engine.compute(census=True, peratom=True)
        assert np.abs(half["e"] - full["e"]).max() <= 1e-9 * max(1.0, np.abs(full["e"]).max()), s.get("name")
        assert np.abs(half["grad"] - full["grad"]).max() <= 1e-6 * max(1.0, np.abs(full["grad"]).max()), s.get("name")
        assert np.array_equal(half["census"], full["census"]), s.get("name")
