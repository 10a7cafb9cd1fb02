"""TEST INFRASTRUCTURE ONLY: the NVE energy drift of the reference's own cpu64 engine on the precision-form protocol.

The precision form runs random carbon at 1.0 g/cm3 with the 2013 C force field at 4000 K, then NVE (dt 0.25 fs).
ReaxFF's bond-order, angle and torsion gates make the energy only piecewise smooth, and at 4000 K bonds form and break
all the time, so the NVE total energy of that protocol drifts whatever the arithmetic. This script measures the drift
the reference's FP64 engine itself gives on a small box of the same material and temperature, as the yardstick for
the GPU's figure: velocity Verlet driven by RefOracle (the reference compiled from its sources; COracle, its C
restatement, where that is not built), velocity rescaling to the target every 10 steps during equilibration, then
plain NVE; the drift is the slope of a linear fit of E_tot/N (kcal/mol/atom) against time (ps).

    python -m oracle.nve_drift [--atoms 300] [--equil 2000] [--nve 4000] [--temp 4000]

The force field is read from metal-reax_b200/data/_c2013/ffield.reax.C2013 (metal-reax_b200/data/decode_c2013.py).
"""
import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO / "metal-reax_b200"))

import systems  # noqa: E402

from .oracle import COracle, RefOracle  # noqa: E402

FTM2V = 1.0 / 48.88821291 ** 2   # (kcal/mol/A)/(g/mol) -> A/fs^2 (LAMMPS real units)
MVV2E = 48.88821291 ** 2         # (g/mol) A^2/fs^2 -> kcal/mol
KB = 0.0019872067                # kcal/mol/K


def run(atoms=300, equil=2000, nve=4000, temp=4000.0, dt=0.25, sample=50, seed=77, log=None):
    text = (REPO / "metal-reax_b200" / "data" / "_c2013" / "ffield.reax.C2013").read_text()
    engine = RefOracle(text, shell=15.0) if RefOracle.available() else COracle(text, shell=15.0)
    s = systems.random_carbon(n=atoms, density=1.0, seed=seed, amu=12.011)
    n = len(s["type"])
    m = 12.011
    q = np.zeros(n)
    v = systems.maxwell_velocities(dict(s, mass=np.full(n, m)), temp, seed=seed + 1)
    x = s["x"].copy()
    g = engine.single_point(dict(s, x=x), q)["grad"]
    times, etot, temps = [], [], []
    t0 = time.time()
    for k in range(equil + nve):
        v -= 0.5 * dt * FTM2V / m * g
        x += dt * v
        r = engine.single_point(dict(s, x=x), q)
        g = r["grad"]
        v -= 0.5 * dt * FTM2V / m * g
        ke = 0.5 * m * float((v * v).sum()) * MVV2E
        T = 2.0 * ke / ((3 * n - 3) * KB)
        if k < equil and (k + 1) % 10 == 0:
            v *= np.sqrt(temp / T)
        if k >= equil and (k + 1 - equil) % sample == 0:
            times.append((k + 1 - equil) * dt * 1e-3)
            etot.append((float(r["e"].sum()) + ke) / n)
            temps.append(T)
            if log:
                print("%.4f ps  E_tot/N %.6f  T %.1f  (%.0f s)" % (times[-1], etot[-1], T, time.time() - t0), file=log, flush=True)
    t = np.asarray(times)
    e = np.asarray(etot)
    slope, icpt = np.polyfit(t, e, 1)
    return {"engine": "reference cpu64" if isinstance(engine, RefOracle) else "C restatement", "atoms": n,
            "temperature_K": temp, "dt_fs": dt, "equil_steps": equil, "nve_steps": nve,
            "drift_kcal_per_atom_ps": float(slope), "rms_kcal_per_atom": float(np.sqrt(np.mean((e - (slope * t + icpt)) ** 2))),
            "T_mean_K": float(np.mean(temps))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--atoms", type=int, default=300)
    ap.add_argument("--equil", type=int, default=2000)
    ap.add_argument("--nve", type=int, default=4000)
    ap.add_argument("--temp", type=float, default=4000.0)
    a = ap.parse_args()
    print(json.dumps(run(a.atoms, a.equil, a.nve, a.temp, log=sys.stderr)))


if __name__ == "__main__":
    main()
