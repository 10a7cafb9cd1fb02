"""GPU tests of the serving form: continuous batching keeps the state of the systems that stay, and every request's
result is the same served alone and served in a mix of concurrent requests.

Bars: single points (one force evaluation of a system frozen in place) are bitwise the same alone and in the mix
(per-system fixed-order reductions, per-system charge solves, fixed-point H-bond scatter). NVT requests follow their
own trajectory alone and in the mix; rounds of the mix end at other requests' completions, which restarts the force
evaluation and the charge warm start at different steps, so their final energies agree within the reference's C3
energy bar (1e-3 kcal/mol/atom) after a run of 40 steps.
"""
import numpy as np
import pytest

from helpers import C3_ENERGY_PER_ATOM, ffield_text

pytestmark = pytest.mark.gpu

MASS = [12.0, 1.008, 15.999]


def _engine(systems_):
    import rxcuda
    e = rxcuda.Engine(0)
    e.set_forcefield(ffield_text())
    e.set_control()
    e.set_qeq(0.0, 10.0, 1e-6, 200)
    e.set_systems(systems_)
    e.md_setup(MASS, dt=0.25, t_start=300.0, t_damp=25.0, chain=3)
    return e


def test_update_systems_carries_device_state():
    """rx_update_systems: a kept system's positions, velocities and charges are carried bitwise; a new system joins with
    the caller's positions; the batch then runs on."""
    import systems
    a, b, c = systems.random_cho(2), systems.random_cho(5), systems.random_cho(8)
    e = _engine([a, b])
    e.set_velocities(np.concatenate([systems.maxwell_velocities(s, 600.0, seed=k) for k, s in enumerate((a, b))]))
    e.md_run(15)
    na = len(a["type"])
    x0, v0, q0 = e.get_positions()[na:], e.get_velocities()[na:], e.get_charges()[na:]
    e.update_systems([1], [c], [systems.maxwell_velocities(c, 600.0, seed=9)])
    assert e.nsys == 2
    nb = len(b["type"])
    assert np.array_equal(e.get_positions()[:nb], x0)
    assert np.array_equal(e.get_velocities()[:nb], v0)
    assert np.array_equal(e.get_charges()[:nb], q0)
    assert np.array_equal(e.get_positions()[nb:], c["x"])
    out = e.md_run(10)
    assert np.all(np.isfinite(out["e"])) and np.all(out["T"] > 0)
    e.close()


def _requests(specs):
    from serving import Request
    import systems
    out = []
    for rid, (k, t_arr, kind, steps, T) in enumerate(specs):
        s = systems.random_cho(k)
        v = systems.maxwell_velocities(s, T, seed=100 + k) if kind == "md" else None
        out.append(Request(rid=rid, arrival=t_arr, system=s, kind=kind, steps=steps, T=T, velocities=v))
    return out


def _late_clock():
    """A clock that reads 0 when the loop starts and 10 s ever after: every request (arrivals <= 0.003 s) has arrived
    at the first round, and no round waits for an arrival."""
    calls = []

    def clock():
        calls.append(None)
        return 0.0 if len(calls) == 1 else 10.0
    return clock


def test_served_results_same_alone_and_in_mix():
    from serving import Server
    specs = [(3, 0.0, "md", 40, 600.0), (11, 0.0, "sp", 0, 300.0), (21, 0.001, "md", 25, 1500.0),
             (7, 0.002, "sp", 0, 300.0), (40, 0.003, "md", 40, 900.0)]
    srv = Server(ffield_text(), budget_bytes=1 << 34, bytes_per_atom=20000.0, chunk=10)
    # the mix: all requests at once (every request has arrived at the first round)
    mix = _requests(specs)
    st = srv.run(mix, clock=_late_clock())
    assert st["requests"] == len(specs)
    for k, spec in enumerate(specs):
        alone = _requests([spec])
        srv.run(alone, clock=_late_clock())
        r_mix, r_alone = mix[k], alone[0]
        n = r_alone.natoms
        if spec[2] == "sp":
            assert np.array_equal(r_mix.result["e"], r_alone.result["e"]), spec
            assert np.array_equal(r_mix.result["grad"], r_alone.result["grad"]), spec
            assert np.array_equal(r_mix.result["q"], r_alone.result["q"]), spec
        else:
            de = abs(r_mix.result["e"].sum() - r_alone.result["e"].sum()) / n
            assert de <= C3_ENERGY_PER_ATOM, (spec, de)
            assert abs(r_mix.result["T"] - r_alone.result["T"]) <= 0.05 * r_alone.result["T"], spec


def test_admission_respects_the_memory_budget():
    """With a budget of about two systems, the loop never holds more than the budget admits, and still serves every
    request (the queue drains as requests complete)."""
    from serving import Server
    specs = [(k, 0.0, "md", 10, 500.0) for k in (1, 2, 3, 4, 5)]
    reqs = _requests(specs)
    bpa = 20000.0
    budget = bpa * (sum(r.natoms for r in reqs[:2]) + 1)
    peak = []
    srv = Server(ffield_text(), budget_bytes=budget, bytes_per_atom=bpa, chunk=5)
    st = srv.run(reqs, clock=_late_clock(), on_round=lambda s, act: peak.append(sum(r.natoms for r in act) * bpa))
    assert st["requests"] == len(specs)
    assert max(peak) <= budget
