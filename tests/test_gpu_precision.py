"""GPU parity on the precision-form workload: 30,000 carbon atoms uniformly random at 1.0 g/cm3 (84.265 A periodic box,
pairs closer than 1.2 A rejected) with the 2013 C force field, charges zero (one element, no charge fix, as the
reference's graphitization example), against the reference's cpu64 engine on the same geometry: at step 0 and at the
frame reached after 200 NVT steps at 4000 K on the GPU.

The force field is extracted from the reference's Supporting Information PDF by metal-reax_b200/data/decode_c2013.py
into a git-ignored directory (its parameters are not redistributable); without it these tests are skipped.

Bars: the reference's C3 acceptance (energy 1e-3 kcal/mol/atom in total and per term, force max 0.05 and RMS 5e-3
kcal/mol/A, virial per component 1e-3 kcal/mol/atom), the decision census identical atom by atom. With RX_REPORT_DIR
set, the per-term errors are written there as JSON.
"""
import json
import os
from pathlib import Path

import numpy as np
import pytest

from helpers import C3_ENERGY_PER_ATOM, C3_FORCE_MAX, C3_FORCE_RMS, force_metrics

pytestmark = pytest.mark.gpu

C2013 = Path(__file__).resolve().parents[1] / "metal-reax_b200" / "data" / "_c2013" / "ffield.reax.C2013"
TERMS = ["bond", "over", "under", "lone_pair", "valence", "penalty", "coalition", "hbond", "torsion", "conjugation", "vdw",
         "coulomb", "polarization"]


def _cpu(text, s, q):
    from oracle.oracle import COracle, RefOracle
    if RefOracle.available():
        return RefOracle(text, shell=15.0).single_point(s, q), "reference cpu64"
    return COracle(text, shell=15.0).single_point(s, q), "C restatement"


@pytest.mark.skipif(not C2013.exists(), reason="2013 C force field not extracted (metal-reax_b200/data/decode_c2013.py)")
def test_carbon30k_c2013_step0_and_nvt_frame():
    import rxcuda
    import systems
    text = C2013.read_text()
    s = systems.random_carbon(30000, density=1.0, seed=4000, amu=12.011)
    n = len(s["type"])
    q = np.zeros(n)
    eng = rxcuda.Engine(0)
    eng.set_forcefield(text)
    eng.set_control()
    eng.set_systems([s])
    eng.set_charges(q)
    report = []

    def compare(tag, frame):
        out = eng.compute(census=True)
        ref, kind = _cpu(text, frame, q)
        de = np.abs(out["e"][0] - ref["e"])
        fmax, frms = force_metrics(ref["grad"], out["grad"])
        dv = np.abs(eng.virial()[0] - ref["virial"])
        rep = {"frame": tag, "atoms": n, "cpu": kind, "term_abs_error_kcal": dict(zip(TERMS, de.tolist())),
               "term_ref_kcal": dict(zip(TERMS, ref["e"].tolist())),
               "total_error_per_atom": float(abs(out["e"][0].sum() - ref["e"].sum()) / n), "force_max": fmax,
               "force_rms": frms, "virial_abs_error": dv.tolist()}
        report.append(rep)
        assert rep["total_error_per_atom"] <= C3_ENERGY_PER_ATOM, rep
        assert (de / n).max() <= C3_ENERGY_PER_ATOM, rep
        assert fmax <= C3_FORCE_MAX and frms <= C3_FORCE_RMS, rep
        assert (dv / n).max() <= C3_ENERGY_PER_ATOM, rep
        for k in range(7):
            assert np.array_equal(out["census"][k], ref["census"][k]), (tag, k)

    compare("step0", s)
    eng.md_setup([12.011], dt=0.25, t_start=4000.0, t_damp=25.0, chain=3)
    eng.md_charges(False)
    eng.set_velocities(systems.maxwell_velocities(dict(s, mass=np.full(n, 12.011)), 4000.0, seed=4001))
    md = eng.md_run(200)
    assert np.all(np.isfinite(md["e"]))
    frame = dict(s)
    frame["x"] = eng.get_positions()
    compare("step200", frame)
    eng.close()
    d = os.environ.get("RX_REPORT_DIR")
    if d:
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, "parity_carbon30k_c2013.json"), "w") as f:
            json.dump(report, f, indent=1)
