"""Serving form: a request loop with continuous batching over one engine context.

Requests (one fresh periodic system each) arrive over time. Each asks either for a single point (energy, forces and
charges) or for an NVT run of a given number of steps at its own temperature. The loop keeps every admitted system's
state resident on the device (positions, velocities, charges, neighbor rows, charge-equilibration warm starts, chain
state) and advances all of them together:

* admission: requests that have arrived join in arrival order while the device memory they need, at the measured
  bytes per atom of this engine, fits the budget;
* continuous batching: at every round, finished requests leave and waiting ones join the running batch
  (rx_update_systems carries the state of the systems that stay), so new work overlaps with work in flight;
* one round advances the batch by a chunk of steps (rx_md_run): MD requests at their own target temperature
  (rx_md_targets), single points frozen in place (they need one evaluation, which the round's first step provides);
* results per request: energies, charges and forces (single points), energies and temperature after the last step
  (MD); latency = completion time - arrival time.

The reference has no serving layer (it runs one system inside LAMMPS); this is the serving pattern of the workload
this project measures, built on the engine's C ABI.
"""
import time
from dataclasses import dataclass, field

import numpy as np

import rxcuda


@dataclass
class Request:
    rid: int
    arrival: float
    system: dict
    kind: str            # "sp" single point, "md" NVT run
    steps: int = 0
    T: float = 300.0
    velocities: np.ndarray = None
    remaining: int = 0
    admitted: float = None
    done: float = None
    result: dict = field(default_factory=dict)

    @property
    def natoms(self):
        return len(self.system["type"])


class Server:
    """Continuous-batching request loop on one GPU context.

    budget_bytes: device memory the admitted systems may take, at bytes_per_atom (measured by measure_bytes_per_atom,
    or given); chunk: MD steps per round (a round ends early at the next completion of an MD request)."""

    def __init__(self, ffield_text, device=0, budget_bytes=None, bytes_per_atom=None, chunk=10, dt=0.25, t_damp=25.0,
                 qeq_tol=1e-6, mass=(12.0, 1.008, 15.999), max_systems=1024):
        self.text = ffield_text
        self.device = device
        self.chunk = chunk
        self.dt, self.t_damp, self.qeq_tol, self.mass = dt, t_damp, qeq_tol, list(mass)
        self.bytes_per_atom = bytes_per_atom or self.measure_bytes_per_atom()
        if budget_bytes is None:
            import torch
            budget_bytes = int(0.5 * torch.cuda.mem_get_info(device)[0])
        self.budget = budget_bytes
        self.max_systems = max_systems
        self.eng = None

    def _engine(self):
        e = rxcuda.Engine(self.device)
        e.set_forcefield(self.text)
        e.set_control()
        e.set_qeq(0.0, 10.0, self.qeq_tol, 200)
        return e

    def measure_bytes_per_atom(self, n_probe=3):
        """Device bytes per atom of a context holding a few serving systems, evaluated once (lists at their grown
        capacities), from the device's free memory before and after."""
        import torch
        import systems
        ss = [systems.serving_request(10 ** 6 + k)[0] for k in range(n_probe)]
        torch.cuda.synchronize(self.device)
        free0 = torch.cuda.mem_get_info(self.device)[0]
        e = self._engine()
        e.set_systems(ss)
        e.md_setup(self.mass, dt=self.dt, t_start=300.0, t_damp=self.t_damp, chain=3)
        e.compute(qeq=True)
        torch.cuda.synchronize(self.device)
        used = free0 - torch.cuda.mem_get_info(self.device)[0]
        e.close()
        na = sum(len(s["type"]) for s in ss)
        return max(1.0, used / na) * 1.25   # headroom for list growth on denser systems

    def run(self, requests, clock=time.perf_counter, on_round=None):
        """Serve `requests` (sorted by arrival, arrival times in seconds from the start). Returns a stats dict."""
        pending = list(requests)
        waiting, active = [], []
        finished = []
        t0 = clock()
        used_bytes = 0.0
        atom_steps = 0.0
        self.eng = None
        rounds = 0
        while pending or waiting or active:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.pop(0))
            # completed requests leave, waiting ones join while the budget allows (arrival order)
            keep = [k for k, r in enumerate(active) if r.done is None]
            for r in active:
                if r.done is not None:
                    used_bytes -= r.natoms * self.bytes_per_atom
            joining = []
            while waiting and len(keep) + len(joining) < self.max_systems:
                r = waiting[0]
                need = r.natoms * self.bytes_per_atom
                if used_bytes + need > self.budget and (keep or joining):
                    break
                waiting.pop(0)
                r.admitted = now
                r.remaining = r.steps
                used_bytes += need
                joining.append(r)
            if len(keep) != len(active) or joining:
                newv = [r.velocities if r.velocities is not None else np.zeros((r.natoms, 3)) for r in joining]
                if not keep and not joining:
                    active = []
                elif self.eng is None or not keep:
                    if self.eng is not None:
                        self.eng.close()
                    self.eng = self._engine()
                    self.eng.set_systems([r.system for r in joining])
                    self.eng.md_setup(self.mass, dt=self.dt, t_start=300.0, t_damp=self.t_damp, chain=3)
                    self.eng.set_velocities(np.concatenate(newv))
                    active = joining
                else:
                    self.eng.update_systems(keep, [r.system for r in joining], newv)
                    active = [active[k] for k in keep] + joining
            if not active:
                if pending:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - (clock() - t0))))
                continue
            # one round: the batch's force evaluation of its new configuration (single points are answered from it),
            # then the MD requests advance while single points stay frozen
            self.eng.md_targets([r.T if r.kind == "md" else 300.0 for r in active],
                                [1 if (r.kind == "md" and r.remaining > 0) else 0 for r in active])
            if any(r.kind == "sp" and r.done is None for r in active):
                out0 = self.eng.md_run(0)
                t_sp = clock() - t0
                q = self.eng.get_charges()
                g = self.eng.gradient()
                off = 0
                for k, r in enumerate(active):
                    n = r.natoms
                    if r.kind == "sp" and r.done is None:
                        r.result = {"e": out0["e"][k].copy(), "q": q[off:off + n].copy(), "grad": g[off:off + n].copy()}
                        r.done = t_sp
                        atom_steps += n
                        finished.append(r)
                    off += n
            md_left = [r.remaining for r in active if r.kind == "md" and r.remaining > 0]
            nsteps = min([self.chunk] + md_left) if md_left else 0
            rounds += 1
            if nsteps > 0:
                out = self.eng.md_run(nsteps)
                tdone = clock() - t0
                for k, r in enumerate(active):
                    if r.done is None and r.kind == "md":
                        r.remaining -= nsteps
                        atom_steps += r.natoms * nsteps
                        if r.remaining <= 0:
                            r.result = {"e": out["e"][k].copy(), "T": float(out["T"][k])}
                            r.done = tdone
                            finished.append(r)
            if on_round:
                on_round(self, active)
        wall = clock() - t0
        if self.eng is not None:
            self.eng.close()
            self.eng = None
        lat = np.array([r.done - r.arrival for r in finished]) * 1e3
        return {"requests": len(finished), "wall_s": wall, "rounds": rounds, "atom_steps": atom_steps,
                "atom_steps_per_s": atom_steps / wall if wall > 0 else 0.0,
                "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                               "mean": float(lat.mean())} if len(lat) else None,
                "bytes_per_atom": self.bytes_per_atom, "budget_bytes": self.budget}


def make_requests(nreq, rate=200.0, seed=4242, workers=8):
    """The serving workload's first nreq requests (arrival times, systems, kinds, steps, temperatures, Maxwell
    velocities at the request's temperature), generated in a spawned process pool."""
    import multiprocessing as mp
    import systems
    arr = systems.poisson_arrivals(nreq, rate, seed)
    if workers > 1:
        with mp.get_context("spawn").Pool(workers) as pool:
            specs = pool.map(_request_spec, [(k, seed) for k in range(nreq)], chunksize=16)
    else:
        specs = [_request_spec((k, seed)) for k in range(nreq)]
    out = []
    for k, (s, kind, steps, T, v) in enumerate(specs):
        out.append(Request(rid=k, arrival=float(arr[k]), system=s, kind=kind, steps=steps, T=T if T > 0 else 300.0,
                           velocities=v))
    return out


def _request_spec(args):
    import sys
    from pathlib import Path
    here = str(Path(__file__).resolve().parent)
    if here not in sys.path:
        sys.path.insert(0, here)
    import systems
    k, seed = args
    s, kind, steps, T = systems.serving_request(k, seed=seed)
    v = systems.maxwell_velocities(s, T, seed=seed * 7919 + k) if kind == "md" else None
    return s, kind, steps, T, v
