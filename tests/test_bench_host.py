"""bench.py's measurement bookkeeping on the CPU: the fixed algorithmic byte model and its split over the timed phases,
the DRAM traffic read from the committed ncu summary, the roofline denominator, and the phase-to-kernel map against
the engine's own phase names."""
import json
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO))
import bench  # noqa: E402


def test_step_byte_model_is_the_scope_table_formula():
    N, P, D, I, R = 24000, 5045742, 83570, 12, 2
    assert bench.model_bytes(N, P, D, I, R) == 128 * N + 8 * P + P * (4 + 8 * I) + 12 * P * R + 256 * D
    # the per-phase split covers the pair and bond terms of the step model (the N-proportional terms stay with the step)
    phases = ("neighbors", "qeq", "nonbonded", "bond_orders", "bonded_terms", "torsion", "gather")
    split = sum(bench.phase_model_bytes(p, N, P, D, I) for p in phases)
    assert split + 12 * P * R + 128 * N == bench.model_bytes(N, P, D, I, R)


def test_traffic_from_the_committed_summary():
    text = (REPO / "profiles" / "dram_traffic_water24k.txt").read_text()
    per_pass = next(float(l.split()[2]) for l in text.splitlines() if l.startswith("k_cg_grid dram_bytes_per_pass"))
    assert bench.profiled_traffic("k_cg_grid", 12) == pytest.approx(12 * per_pass)
    per_launch = next(float(l.split()[2]) for l in text.splitlines() if l.startswith("k_pairs dram_bytes_per_launch"))
    assert bench.profiled_traffic("k_pairs", 12) == per_launch
    assert bench.profiled_traffic("no_such_kernel", 12) is None


def test_roofline_denominator():
    peak, kind = bench.measured_peak()
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        assert kind == "measured" and peak == float(json.loads(p.read_text())["hbm_gbs"])
    else:
        assert kind == "fallback" and peak > 0


def test_every_engine_phase_names_its_kernel():
    src = (REPO / "metal-reax_b200" / "csrc" / "engine.cu").read_text()
    import re
    names = set(re.findall(r'tic\(\d+, "([a-z_]+)"\)', src))
    assert names and names <= set(bench.PHASE_KERNEL), names - set(bench.PHASE_KERNEL)
    kernels = (REPO / "metal-reax_b200" / "csrc" / "kernels_nb.cu").read_text() + \
        (REPO / "metal-reax_b200" / "csrc" / "kernels_bonded.cu").read_text()
    for k in bench.PHASE_KERNEL.values():
        assert re.search(r"__global__ void (__launch_bounds__\([^)]*\) )?%s\(" % k, kernels), k
