#!/usr/bin/env python3
"""Benchmark of the ReaxFF force + charge-equilibration step on B200 (one JSON line on rank 0).

Workload (the single-GPU configuration the headline metric is quoted on): 8000 H2O = 24,000 atoms in a 62.07 A
periodic box (lattice of molecules, +-0.3 A jitter, random orientations, O-H 0.96 A, 104.5 deg), synthetic CHO
force field (metal-reax_b200/data/ffield.synthetic.cho), NVT at 300 K, dt 0.25 fs, Tdamp 25 fs, chain 3, charge
equilibration every step (taper 0-10 A, tol 1e-6, maxiter 200). One step = QEq + energy/forces + velocity Verlet.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

value: atom-steps/s of the whole job with the state resident in HBM (device-timed with CUDA events on the engine's
stream, max over ranks). e2e: the same metric through the C ABI with host buffers (positions in, gradient and
energies out every step, integration on the host, as the LAMMPS plugin drives the engine). N > 1: N independent
replicas (one per GPU, no collective on the data path; the single-system step does not shard).
batch: the batching form on the same GPU, 512 mixed CHO systems evaluated as one batch versus one context per
system (atom-evals/s of each, their ratio, p50/p99 latency of the batched evaluation).
--impl reference: the reference's own CPU engine (oracle/_ref, cpu64) plus the C restatement of the stock QEq CG on
the host, same workload and metric.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
PKG = REPO / "metal-reax_b200"
for p in (str(REPO), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)

import systems  # noqa: E402

METRIC = "atom-steps/s"
UNIT = "atom-steps/s"
WORKLOAD = "water24k_nvt_qeq"
DT, TEMP, TDAMP, CHAIN = 0.25, 300.0, 25.0, 3
QEQ = dict(swa=0.0, swb=10.0, tol=1e-6, imax=200)
MASS = [12.0, 1.008, 15.999]
KTERMS = 13


def ffield_text():
    return (PKG / "data" / "ffield.synthetic.cho").read_text()


def workload(n_side=20):
    s = systems.water_box(n_side)
    v = systems.maxwell_velocities(s, TEMP, seed=20261203)
    return s, v


# ---------------------------------------------------------------------------------------------------- clocks
class Clocks:
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = Path("/tmp/rx_clocks_%d_%d.csv" % (os.getpid(), device))

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits", "-lms", "200",
                                          "-i", str(self.device)], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if parts[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        self.path.unlink(missing_ok=True)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------------------- byte model
def model_bytes(N, P, D, I, R=0):
    """Algorithmic HBM bytes of one MD step, the fixed model of the hot-path scope table (independent of the
    implementation): 128 N + 8 P + P (4 + 8 I) + 12 P R + 256 D, with N atoms, P counted half pairs within the
    non-bonded cut-off, D directed bonds, I fused s/t CG iterations, R FP64 residual passes of the solve (the CG
    iterates on the single-precision matrix and checks / refines with the FP64 one)."""
    return 128 * N + 8 * P + P * (4 + 8 * I) + 12 * P * R + 256 * D


def phase_model_bytes(name, N, P, D, I):
    """The same model split over the timed phases (N-proportional terms stay with the step)."""
    return {
        "neighbors": 4 * P + 4 * P,                 # pair list written (4 B) + H value written once (4 B)
        "qeq": 8 * P * I,                           # H value + index read once per fused s/t iteration (+ 12 P R below)
        "nonbonded": 4 * P,                         # pair list read
        "bond_orders": 128 * D,
        "bonded_terms": 64 * D,
        "torsion": 32 * D,
        "gather": 32 * D,
    }.get(name, 0)


def phase_impl_bytes(name, N, E, D, I, R=1, EV=None):
    """Bytes this implementation moves per phase: E neighbor-row entries (both directions) filtered every step from EV
    Verlet-row entries; the charge matrix as single-precision hi + lo parts."""
    EV = EV if EV is not None else E
    return {
        "neighbors": 4 * EV + 12 * E + 64 * N,      # Verlet codes read; row code + hi + lo written; positions
        "qeq": I * (8 * E + 112 * N) + R * (12 * E + 64 * N),   # code + hi per iteration; code + hi + lo per FP64 pass
        "nonbonded": 4 * E + 64 * N,
    }.get(name, phase_model_bytes(name, N, E // 2, D, I))


# the dominant kernel of each timed phase (the neighbor phase's every-step kernel is the row filter; the Verlet build
# runs only on rebuild steps)
PHASE_KERNEL = {"neighbors": "k_pairs", "qeq": "k_cg_grid", "bond_orders": "k_bonds", "bonded_terms": "k_bonded_atom",
                "torsion": "k_torsion", "nonbonded": "k_nonbonded_half", "gather": "k_fold", "force_final": "k_force_final"}


def profiled_traffic(kernel, passes):
    """DRAM bytes (read + write) per launch of `kernel` on this workload, from the committed ncu summary: a per-launch
    figure, or a per-matrix-pass figure scaled by the passes of the measured launch. None without a summary."""
    p = REPO / "profiles" / "dram_traffic_water24k.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        f = line.split()
        if len(f) >= 3 and f[0] == kernel and f[1] == "dram_bytes_per_launch":
            return float(f[2])
        if len(f) >= 3 and f[0] == kernel and f[1] == "dram_bytes_per_pass":
            return float(f[2]) * passes
    return None


def measured_peak():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            v = json.loads(p.read_text()).get("hbm_gbs")
            if v:
                return float(v), "measured"
        except (ValueError, OSError):
            pass
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------------------------------- engine arm
def make_engine(device, s, v):
    import rxcuda
    e = rxcuda.Engine(device)
    e.set_forcefield(ffield_text())
    e.set_control()
    e.set_qeq(QEQ["swa"], QEQ["swb"], QEQ["tol"], QEQ["imax"])
    e.set_systems([s])
    e.md_setup(MASS, dt=DT, t_start=TEMP, t_damp=TDAMP, chain=CHAIN)
    e.set_velocities(v)
    return e


def host_cpu():
    """Model name and logical core count of this host."""
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return model, os.cpu_count()


def cpu_baseline_sample(seconds=15.0):
    """The reference's own cpu64 engine (oracle/_ref) + the C restatement of the stock QEq CG (warm-started from the
    previous step's solution, as the fix does), one core, on MD steps of the 24,000-atom water workload repeated for
    about `seconds` (the cpu64 engine is single-threaded by design)."""
    from oracle.oracle import COracle, RefOracle
    text = ffield_text()
    s, v = workload()
    n = len(s["type"])
    co = COracle(text, shell=12.0)
    kind = "reference" if RefOracle.available() else "port"
    ref = RefOracle(text, shell=12.0) if kind == "reference" else co
    m = np.asarray(MASS)[s["type"]][:, None]
    ftm2v = 1.0 / 48.88821291 / 48.88821291
    x, vel = s["x"].copy(), v.copy()
    sq, tq = np.zeros(n), np.zeros(n)

    def grad(xx):
        nonlocal sq, tq
        qr = co.qeq(dict(s, x=xx), tol=QEQ["tol"], imax=QEQ["imax"], s0=sq, t0=tq)
        sq, tq = qr["s"], qr["t"]
        return ref.single_point(dict(s, x=xx), qr["q"])["grad"]

    g = grad(x)
    count = 0
    t0 = time.perf_counter()
    while True:
        vel -= 0.5 * DT * ftm2v * g / m
        x = x + DT * vel
        g = grad(x)
        vel -= 0.5 * DT * ftm2v * g / m
        count += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    model, ncpu = host_cpu()
    return {"value": n * count / dt, "unit": UNIT, "cores": 1, "kind": kind,
            "host": {"cpu": model, "logical_cores": ncpu},
            "sample": "%d MD steps of the 24,000-atom water workload (QEq + energy/forces + velocity Verlet), %.1f s, %s" % (
                count, dt, "reference cpu64 engine + C restatement of the stock QEq CG" if kind == "reference" else "C restatement")}


def e2e_run(device, s, v, steps, warmup):
    """Plugin-style loop through the C ABI: positions from host memory in, gradient + energies out, host integration."""
    import torch
    import rxcuda
    e = rxcuda.Engine(device)
    e.set_forcefield(ffield_text())
    e.set_control()
    e.set_qeq(QEQ["swa"], QEQ["swb"], QEQ["tol"], QEQ["imax"])
    e.set_systems([s])
    n = len(s["type"])
    m = np.asarray(MASS)[s["type"]][:, None]
    ftm2v = 1.0 / 48.88821291 / 48.88821291
    # positions in and gradient out live in page-locked host memory, copied from and into directly each step
    x = rxcuda.pinned_array((n, 3))
    x[:] = s["x"]
    g = rxcuda.pinned_array((n, 3))
    vel = v.copy()
    stream = torch.cuda.ExternalStream(e.stream(), device=torch.device("cuda", device))
    e.set_positions(x)
    e.compute(qeq=True, grad_out=g)
    # velocity Verlet in its leapfrog form, in place: u is the half-step velocity times dt (the displacement of the
    # next drift), so a step is one drift and one full kick, u -= 2 k dt g with k the per-atom half-kick factor
    # (host arithmetic through torch's multithreaded CPU kernels on views of the same arrays)
    kick = np.ascontiguousarray(np.repeat(0.5 * DT * ftm2v / m, 3, axis=1))
    fullkick_dt = torch.from_numpy(2.0 * kick * DT)
    u = torch.from_numpy((vel - kick * g) * DT)
    xt, gt = torch.from_numpy(x), torch.from_numpy(g)

    def step():
        xt.add_(u)
        e.set_positions(x)
        e.compute(qeq=True, grad_out=g)
        u.addcmul_(gt, fullkick_dt, value=-1.0)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize(device)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        step()
    b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b)
    e.close()
    # positions in and gradient out: 24 B per atom each way (3 doubles), plus the energies
    return n * steps / (ms * 1e-3), {"h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 24 * n + 8 * KTERMS}


def run_engine(args, rank, world, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local_rank))
    s, v = workload()
    n = len(s["type"])
    eng = make_engine(local_rank, s, v)
    stream = torch.cuda.ExternalStream(eng.stream(), device=torch.device("cuda", local_rank))
    if args.rebuild_evals > 0:
        eng.set_timing(True)   # eager launches, each phase timed alone
        ms = []
        for k in range(args.rebuild_evals):
            if k > 0:
                eng.set_capacities(*eng.capacities())   # same capacities: flags every system for a rebuild
            t0 = eng.phase_times().get("neighbors", 0.0)
            eng.compute(qeq=True)
            ms.append(eng.phase_times()["neighbors"] - t0)
        print(json.dumps({"rebuild_evals": args.rebuild_evals, "neighbors_ms": ms, "atoms": n}), flush=True)
        eng.close()
        if dist:
            dist.destroy_process_group()
        return
    eng.md_run(max(args.warmup, 3))
    if args.qeq_passes > 0:
        eng.set_qeq(QEQ["swa"], QEQ["swb"], 1e-300, args.qeq_passes)
        r = eng.qeq_solve()
        print(json.dumps({"qeq_passes": int(r["iters"].max()), "atoms": n}), flush=True)
        eng.close()
        if dist:
            dist.destroy_process_group()
        return
    clocks = Clocks(local_rank) if rank == 0 else None
    if dist:
        dist.barrier()
    torch.cuda.synchronize(local_rank)
    if clocks:
        clocks.start()
    launches0 = eng.kernel_launches()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    eng.md_run(args.steps)
    b.record(stream)
    b.synchronize()
    torch.cuda.synchronize(local_rank)
    launches = eng.kernel_launches() - launches0
    ck = clocks.stop() if clocks else None
    ms = a.elapsed_time(b)
    if dist:
        dist.barrier()
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    value = world * n * args.steps / (ms * 1e-3)

    # per-phase device times (a separate short run with phase events on), sizes for the byte model
    eng.set_timing(True)
    prof_steps = 3
    eng.md_run(prof_steps)
    phases = {k: v_ / prof_steps for k, v_ in eng.phase_times().items()}
    eng.set_timing(False)
    I = int(eng.qeq_last()["iters"].max())       # fused s/t CG iterations of the last MD step's solve
    R = max(1, eng.qeq_refinements())            # its FP64 residual passes
    out = eng.compute(counts=True)
    P = int(out["counts"][1])
    E = int(out["counts"][2])
    D = int(out["counts"][0]) * 2
    peak, peak_kind = measured_peak()
    dom = max(phases, key=phases.get) if phases else "qeq"
    t_dom = phases.get(dom)
    dom_bytes = phase_model_bytes(dom, n, P, D, I) + (12 * P * R if dom == "qeq" else 0)
    impl_bytes = phase_impl_bytes(dom, n, E, D, I, R)
    achieved = dom_bytes / (t_dom * 1e-3) / 1e9 if t_dom else None
    achieved_impl = impl_bytes / (t_dom * 1e-3) / 1e9 if t_dom else None
    step_bytes = model_bytes(n, P, D, I, R)
    step_achieved = step_bytes / (ms_step * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
        "data": "synthetic (seeded water box, synthetic CHO force field)",
        "config": {"workload": WORKLOAD, "atoms_per_gpu": n, "systems_per_gpu": 1, "qeq_tol": QEQ["tol"], "dt_fs": DT,
                   "T_K": TEMP, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "per-step working set larger than L2 (Verlet + neighbor rows + charge matrix ~230 MB)",
                   "neighbor_skin_A": 1.0},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": PHASE_KERNEL.get(dom, dom), "phase": dom, "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                     "traffic": profiled_traffic(PHASE_KERNEL.get(dom, dom), I), "bytes_alg": dom_bytes,
                     "bytes_model": "scope-table model: 8 B per counted half pair per fused CG iteration",
                     "impl": {"bytes": impl_bytes, "achieved": achieved_impl,
                              "frac": (achieved_impl / peak) if achieved_impl else None,
                              "note": "full rows (both directions); charge matrix as single-precision hi + lo"},
                     "peak_kind": peak_kind, "phase_ms_per_step": phases},
        "step_roofline": {"bytes_alg": step_bytes, "achieved": step_achieved, "peak": peak, "unit": "GB/s",
                          "frac": step_achieved / peak, "frac_of_nominal_8TBs": step_achieved / 8000.0,
                          "N": n, "P": P, "E": E, "D": D, "I": I, "R": R},
        "clocks": ck,
    }
    eng.close()
    if world == 1 and rank == 0:
        if not args.no_e2e:
            # the same untimed warm-up as the device-resident run (the first steps' charge solves start from an
            # empty history and take several times the iterations of the later ones)
            e2e_value, e2e_bytes = e2e_run(local_rank, s, v, max(2, args.steps // 2), args.warmup)
            line["e2e"] = {"value": e2e_value, "unit": UNIT, **e2e_bytes}
        if not args.no_batch:
            line["batch"] = batch_run(local_rank)
        if args.serve_requests > 0:
            try:
                line["serve"] = serve_run(local_rank, args.serve_requests)
            except Exception as exc:   # the serving sample is reported beside the headline; its failure is recorded
                line["serve"] = {"error": "%s: %s" % (type(exc).__name__, exc)}
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_sample(args.cpu_seconds)
    elif rank == 0:
        line["e2e"] = None
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------------- batching form
BATCH_SYSTEMS = 512


def batch_run(device, reps=20, world=1, rank=0):
    """512 independent periodic CHO systems (log-uniform 64-1024 atoms, Dirichlet C/H/O, 0.5-1.2 g/cm3, seed per
    system): one energy + forces + charges evaluation of all of them, as a fresh single point (CG from zero), through
    the C ABI with host buffers out (energies, gradient). Batched: every system in one context and one launch sequence;
    per-system: one context per system, evaluated one after the other. Latency percentiles are over `reps` batched
    evaluations (host wall clock around the synchronous call). Under N ranks each rank takes its shard of the systems."""
    import rxcuda
    import batching
    ss_all = [systems.random_cho(k) for k in range(BATCH_SYSTEMS)]
    mine = batching.shard_systems([len(s["type"]) for s in ss_all], world, rank)
    ss = [ss_all[k] for k in mine]
    na = sum(len(s["type"]) for s in ss)
    text = ffield_text()

    def engine_for(group):
        e = rxcuda.Engine(device)
        e.set_forcefield(text)
        e.set_control()
        e.set_qeq(QEQ["swa"], QEQ["swb"], QEQ["tol"], QEQ["imax"])
        e.set_systems(group)
        return e

    eng = engine_for(ss)
    tuned = eng.autotune()
    for _ in range(3):
        eng.compute(qeq=True, cold=True)
    lat = []
    for _ in range(reps):
        t = time.perf_counter()
        eng.compute(qeq=True, cold=True)
        lat.append(time.perf_counter() - t)
    it = np.asarray(eng.qeq_solve()["iters"])
    eng.close()
    lat_ms = np.array(lat) * 1e3
    batched = na / (np.median(lat_ms) * 1e-3)
    singles = [engine_for([s]) for s in ss]
    for e in singles:
        e.set_tuning("lone_grid_min", 0)   # a lone system on its fastest charge solve (all SMs on its rows)
        e.compute(qeq=True, cold=True)
    best = None
    for _ in range(2):
        t = time.perf_counter()
        for e in singles:
            e.compute(qeq=True, cold=True)
        dt = time.perf_counter() - t
        best = dt if best is None else min(best, dt)
    for e in singles:
        e.close()
    per_system = na / best
    return {"workload": "cho512_single_point_qeq", "systems": len(ss), "atoms": na, "qeq_tol": QEQ["tol"],
            "unit": "atom-evals/s", "batched": batched, "per_system": per_system, "speedup": batched / per_system,
            "latency_ms": {"p50": float(np.percentile(lat_ms, 50)), "p99": float(np.percentile(lat_ms, 99)),
                           "reps": reps},
            "qeq_iters_max": int(it.max()), "per_system_pass_ms": best * 1e3, "autotuned": tuned,
            "note": "host wall clock through the C ABI (D2H of energies and gradient each evaluation); batched: one "
                    "captured evaluation graph over all systems; per system: one context each, lone-system CG"}


def serve_run(device, nreq=400, rate=200.0, chunk=10):
    """The serving form on a bounded sample: the first `nreq` requests of the Poisson stream (200 req/s, seed 4242;
    fresh CHO systems of 100-5000 atoms; half single points, half NVT runs of 10-1000 steps at 300-3000 K), served
    with continuous batching and HBM-budget admission. Requests are generated before the clock starts."""
    import serving
    reqs = serving.make_requests(nreq, rate=rate)
    srv = serving.Server(ffield_text(), device=device, chunk=chunk)
    st = srv.run(reqs)
    st.update({"workload": "serve_cho_poisson%d" % int(rate), "requests_total": nreq, "rate_per_s": rate, "chunk_steps": chunk,
               "unit": "atom-steps/s (MD atom-steps + single-point atoms)"})
    return st


def precision_run(device, nvt_steps=10000, nve_ps=20.0, sample=100):
    """The precision form: 30,000 carbon atoms uniformly random at 1.0 g/cm3 (84.265 A box, pairs closer than 1.2 A
    rejected) with the 2013 C force field and zero charges (one element: no charge solve), Maxwell velocities at 4000 K,
    `nvt_steps` Nose-Hoover steps at 4000 K (Tdamp 25 fs), then `nve_ps` of NVE, dt 0.25 fs. Returns the step times of
    both phases (CUDA events on the engine stream) and the NVE total-energy drift (slope of a linear fit of E_tot/N
    against time) and the RMS of E_tot/N about that line, sampled every `sample` steps. None when the force field has
    not been extracted (metal-reax_b200/data/decode_c2013.py)."""
    import torch
    import rxcuda
    path = PKG / "data" / "_c2013" / "ffield.reax.C2013"
    if not path.exists():
        return None
    s = systems.random_carbon(30000, density=1.0, seed=4000, amu=12.011)
    n = len(s["type"])
    mass = 12.011
    eng = rxcuda.Engine(device)
    eng.set_forcefield(path.read_text())
    eng.set_control()
    eng.set_systems([s])
    eng.set_charges(np.zeros(n))
    eng.md_setup([mass], dt=0.25, t_start=4000.0, t_damp=25.0, chain=3)
    eng.md_charges(False)
    eng.set_velocities(systems.maxwell_velocities(dict(s, mass=np.full(n, mass)), 4000.0, seed=4001))
    st = torch.cuda.ExternalStream(eng.stream(), device=torch.device("cuda", device))

    def timed(nsteps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        out = eng.md_run(nsteps)
        b.record(st)
        b.synchronize()
        return out, a.elapsed_time(b)

    ms_nvt = 0.0
    done = 0
    while done < nvt_steps:
        k = min(1000, nvt_steps - done)
        out, ms = timed(k)
        ms_nvt += ms
        done += k
    t_nvt = float(out["T"][0])
    v = eng.get_velocities()
    eng.md_setup([mass], dt=0.25, t_start=4000.0, t_damp=25.0, chain=0)   # chain 0: plain velocity Verlet (NVE)
    eng.set_velocities(v)
    nve_steps = int(round(nve_ps * 1000.0 / 0.25))
    kcal = 1.0 / 4.184e-4    # g/mol A^2/fs^2 -> kcal/mol
    times, etot, temps = [], [], []
    ms_nve = 0.0
    for k in range(0, nve_steps, sample):
        out, ms = timed(sample)
        ms_nve += ms
        vv = eng.get_velocities()
        ke = 0.5 * mass * float((vv * vv).sum()) * kcal
        etot.append((float(out["e"][0].sum()) + ke) / n)
        times.append((k + sample) * 0.25e-3)
        temps.append(float(out["T"][0]))
    eng.close()
    t_ps = np.asarray(times)
    e = np.asarray(etot)
    slope, icpt = np.polyfit(t_ps, e, 1)
    rms = float(np.sqrt(np.mean((e - (slope * t_ps + icpt)) ** 2)))
    return {"workload": "carbon30k_c2013_precision", "atoms": n, "dt_fs": 0.25, "nvt_steps": nvt_steps,
            "nvt_T_end_K": t_nvt, "nve_ps": nve_ps, "nve_steps": nve_steps, "sample_every": sample,
            "ms_per_step_nvt": ms_nvt / nvt_steps, "ms_per_step_nve": ms_nve / nve_steps,
            "atom_steps_per_s_nvt": n * nvt_steps / (ms_nvt * 1e-3),
            "nve_drift_kcal_per_atom_ps": float(slope), "nve_rms_kcal_per_atom": rms,
            "nve_T_mean_K": float(np.mean(temps)), "nve_etot_first_last": [float(e[0]), float(e[-1])],
            "reference_published": "VO oxide, 512 atoms, 20 ps NVE (docs/make_figures.py): drift stock 3.7e-6, "
                                   "all-FP32 GPU 4.0e-4, mixed 3.4e-6 kcal/mol/atom/ps; RMS 1.1e-4 / 1.24e-3 / 1.07e-4"}


# ---------------------------------------------------------------------------------------------------- reference arm
def run_reference(args, rank):
    if rank != 0:
        return
    from oracle.oracle import COracle, RefOracle
    text = ffield_text()
    s, v = workload()
    n = len(s["type"])
    co = COracle(text, shell=12.0)
    kind = "reference" if RefOracle.available() else "port"
    ref = RefOracle(text, shell=12.0) if kind == "reference" else co
    m = np.asarray(MASS)[s["type"]][:, None]
    ftm2v = 1.0 / 48.88821291 / 48.88821291
    x = s["x"].copy()
    vel = v.copy()
    sq, tq = np.zeros(n), np.zeros(n)

    def forces(xx):
        nonlocal sq, tq
        sys_ = dict(s, x=xx)
        qr = co.qeq(sys_, tol=QEQ["tol"], imax=QEQ["imax"], s0=sq, t0=tq)
        sq, tq = qr["s"], qr["t"]
        return ref.single_point(sys_, qr["q"])["grad"]

    g = forces(x)

    def step():
        nonlocal x, vel, g
        vel -= 0.5 * DT * ftm2v * g / m
        x = x + DT * vel
        g = forces(x)
        vel -= 0.5 * DT * ftm2v * g / m

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    value = n * args.steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded water box, synthetic CHO force field)",
            "config": {"workload": WORKLOAD, "atoms_per_gpu": n, "systems_per_gpu": 1, "qeq_tol": QEQ["tol"], "dt_fs": DT,
                       "T_K": TEMP},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": kind,
                             "sample": "full 24,000-atom steps (QEq + energy/forces + host velocity Verlet); the cpu64 engine is "
                                       "single-threaded by design"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer (C ABI) run")
    ap.add_argument("--no-batch", action="store_true", help="skip the 512-system batching measurement")
    ap.add_argument("--serve-requests", type=int, default=300,
                    help="requests of the serving sample (0 skips it; the full serving workload is 10000)")
    ap.add_argument("--qeq-passes", type=int, default=0,
                    help="profiling case: after the warm-up steps, one charge solve of exactly this many matrix passes "
                         "(tolerance 0), then print the counts and exit")
    ap.add_argument("--rebuild-evals", type=int, default=0,
                    help="profiling case: evaluations launched one kernel at a time (no graph), each with every "
                         "system's Verlet rows rebuilt (the first is the initial build); print the neighbor-phase "
                         "times and exit")
    ap.add_argument("--precision-form", action="store_true",
                    help="run only the precision form (30k carbon, 2013 C force field: NVT at 4000 K, then NVE drift) "
                         "and print its JSON line")
    ap.add_argument("--nvt-steps", type=int, default=10000)
    ap.add_argument("--nve-ps", type=float, default=20.0)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.precision_form:
        out = precision_run(int(os.environ.get("LOCAL_RANK", "0")), args.nvt_steps, args.nve_ps)
        print(json.dumps(out if out is not None else {"workload": "carbon30k_c2013_precision",
                                                      "unavailable": "2013 C force field not extracted"}), flush=True)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.gpus != world:
        print("bench.py: --gpus %d but %d rank(s) were launched; start N > 1 under torchrun with --nproc-per-node N"
              % (args.gpus, world), file=sys.stderr)
        sys.exit(2)
    if args.impl == "reference":
        run_reference(args, rank)
        return
    run_engine(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
