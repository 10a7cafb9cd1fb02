"""The serving loop's host logic on the CPU, with a stand-in for the engine context: admission in arrival order within
the device-memory budget, continuous batching (finished systems leave, waiting ones join, kept systems keep their
identity and state), MD requests advanced by exactly their step counts, single points answered in the round they
join, and the latency bookkeeping. The engine itself is covered by the GPU serving test."""
import numpy as np
import pytest

import serving


class FakeEngine:
    """Records what the serving loop asks of an engine context (systems held, per-system targets, steps run)."""

    instances = []

    def __init__(self):
        self.ids = []            # identity of each held system, in context order
        self.sizes = {}          # system id -> atoms
        self.steps = {}          # system id -> MD steps advanced while active
        self.active = None
        self.batches = []        # atoms held at every md_run
        self.closed = False
        FakeEngine.instances.append(self)

    def set_systems(self, systems):
        self.ids = [id(s) for s in systems]
        for s in systems:
            self.sizes[id(s)] = len(s["type"])

    def md_setup(self, *a, **k):
        pass

    def set_velocities(self, v):
        assert v.shape == (sum(self.sizes[i] for i in self.ids), 3)

    def update_systems(self, keep, new_systems, new_velocities=None):
        assert len(set(keep)) == len(keep) and all(0 <= k < len(self.ids) for k in keep)
        assert list(keep) == sorted(keep)   # kept systems stay in their order
        self.ids = [self.ids[k] for k in keep] + [id(s) for s in new_systems]
        for s in new_systems:
            self.sizes[id(s)] = len(s["type"])

    def md_targets(self, t_target=None, active=None):
        assert len(t_target) == len(self.ids) and len(active) == len(self.ids)
        self.active = list(active)

    def md_run(self, nsteps):
        self.batches.append([self.sizes[i] for i in self.ids])
        for i, on in zip(self.ids, self.active):
            if on:
                self.steps[i] = self.steps.get(i, 0) + nsteps
        n = len(self.ids)
        return {"e": np.zeros((n, 13)), "T": np.full(n, 300.0)}

    def get_charges(self):
        return np.zeros(sum(self.sizes[i] for i in self.ids))

    def gradient(self):
        return np.zeros((sum(self.sizes[i] for i in self.ids), 3))

    def close(self):
        self.closed = True


def _requests(n, seed=7):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(0.0003, n))
    out = []
    for k in range(n):
        natoms = int(rng.integers(20, 400))
        md = rng.random() < 0.6
        out.append(serving.Request(rid=k, arrival=float(t[k]), system={"type": np.zeros(natoms, dtype=np.int32)},
                                   kind="md" if md else "sp", steps=int(rng.integers(3, 60)) if md else 0,
                                   T=float(rng.uniform(250, 900)),
                                   velocities=np.zeros((natoms, 3)) if md else None))
    return out


@pytest.mark.parametrize("budget_atoms,max_systems", [(1500, 64), (400, 64), (100000, 5)])
def test_admission_batching_and_step_counts(monkeypatch, budget_atoms, max_systems):
    FakeEngine.instances.clear()
    monkeypatch.setattr(serving.Server, "_engine", lambda self: FakeEngine())
    monkeypatch.setattr(serving.time, "sleep", lambda s: None)
    ticks = {"t": 0.0}

    def clock():   # each reading advances the clock by 0.5 ms, so arrivals come due while the loop runs
        ticks["t"] += 5e-4
        return ticks["t"]

    bpa = 1000.0
    srv = serving.Server("", bytes_per_atom=bpa, budget_bytes=budget_atoms * bpa, chunk=10, max_systems=max_systems)
    reqs = _requests(80)
    stats = srv.run(reqs, clock=clock)
    assert stats["requests"] == len(reqs)
    steps = {}
    for e in FakeEngine.instances:
        assert e.closed
        for i, n in e.steps.items():
            steps[i] = steps.get(i, 0) + n
        for batch in e.batches:
            # within the budget, or one request larger than the budget admitted alone
            assert sum(batch) * bpa <= budget_atoms * bpa or len(batch) == 1
            assert len(batch) <= max_systems
    sizes = [len(b) for e in FakeEngine.instances for b in e.batches]
    assert max(sizes) >= min(max_systems, 4)   # requests overlap: the batch holds several systems at once
    admitted = [r.admitted for r in reqs]
    assert all(a <= b for a, b in zip(admitted, admitted[1:]))   # admission in arrival order
    for r in reqs:
        assert r.arrival <= r.admitted <= r.done
        if r.kind == "md":
            assert steps[id(r.system)] == r.steps, (r.rid, steps.get(id(r.system)), r.steps)
            assert set(r.result) == {"e", "T"}
        else:
            assert steps.get(id(r.system), 0) == 0   # single points stay frozen
            assert set(r.result) == {"e", "q", "grad"} and r.result["grad"].shape == (r.natoms, 3)
    lat = np.array([r.done - r.arrival for r in reqs]) * 1e3
    assert stats["latency_ms"]["p50"] == pytest.approx(float(np.percentile(lat, 50)))
