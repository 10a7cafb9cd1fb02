"""GPU tests of the NVT integrator against a CPU restatement of the same update, and of its temperature control.

The CPU restatement below advances velocity Verlet with the Martyna-Tuckerman-Klein Nose-Hoover chain (Mol. Phys. 87,
1117 (1996); the Trotter splitting of Tuckerman et al., J. Phys. A 39, 5629 (2006)): chain half-step, half kick, drift,
force evaluation, half kick, chain half-step, with chain masses Q_1 = Nf kT tau^2 and Q_k = kT tau^2 and Nf = 3N - 3.
Its forces come from the oracle (charges equilibrated at tol 1e-10 at every force evaluation, on both sides, so the
charge guesses do not matter), so this pins the device integrator and its coupling to the force evaluation.
"""
import numpy as np
import pytest

from helpers import ffield_text, small_systems

pytestmark = pytest.mark.gpu

MASS = np.array([12.0, 1.008, 15.999])
FTM2V = 1.0 / 48.88821291 ** 2
MVV2E = 48.88821291 ** 2
KB = 0.0019872067


def _chain_half(v, m, xi, vxi, T, tdamp, dt):
    """One dt/2 application of the chain; returns the velocity scale and updates xi, vxi in place."""
    M = len(xi)
    nf = 3.0 * len(m) - 3.0
    kT = KB * T
    Q = np.array([nf * kT * tdamp ** 2] + [kT * tdamp ** 2] * (M - 1))
    ke2 = MVV2E * (m[:, None] * v ** 2).sum()

    def G(k):
        return (ke2 - nf * kT) / Q[0] if k == 0 else (Q[k - 1] * vxi[k - 1] ** 2 - kT) / Q[k]

    dt2, dt4, dt8 = 0.5 * dt, 0.25 * dt, 0.125 * dt
    vxi[M - 1] += G(M - 1) * dt4
    for k in range(M - 2, -1, -1):
        e = np.exp(-vxi[k + 1] * dt8)
        vxi[k] = (vxi[k] * e + G(k) * dt4) * e
    scale = np.exp(-vxi[0] * dt2)
    ke2 *= scale * scale
    xi += vxi * dt2
    for k in range(M - 1):
        e = np.exp(-vxi[k + 1] * dt8)
        vxi[k] = (vxi[k] * e + G(k) * dt4) * e
    vxi[M - 1] += G(M - 1) * dt4
    return scale


def _min_image(d, box):
    f = d @ np.linalg.inv(box)
    return (f - np.round(f)) @ box


def test_nvt_matches_cpu_restatement():
    import rxcuda
    import systems
    from oracle.oracle import COracle
    s = small_systems()[0]
    n = len(s["type"])
    m = MASS[s["type"]]
    dt, T, tdamp, nsteps = 0.25, 300.0, 25.0, 5
    v0 = systems.maxwell_velocities(s, 450.0, seed=21)     # away from the target, so the chain acts
    eng = rxcuda.Engine(0)
    eng.set_forcefield(ffield_text())
    eng.set_control()
    eng.set_qeq(0.0, 10.0, 1e-10, 400)
    eng.set_systems([s])
    eng.md_setup(MASS, dt=dt, t_start=T, t_damp=tdamp, chain=3)
    eng.set_velocities(v0)
    out = eng.md_run(nsteps)
    xg, vg = eng.get_positions(), eng.get_velocities()
    eng.close()

    orc = COracle(ffield_text(), shell=15.0)

    def grad(x):
        sx = dict(s)
        sx["x"] = x
        q = orc.qeq(sx, tol=1e-10, imax=400)["q"]
        return orc.single_point(sx, q)["grad"]

    x, v = s["x"].copy(), v0.copy()
    xi, vxi = np.zeros(3), np.zeros(3)
    g = grad(x)
    for _ in range(nsteps):
        v *= _chain_half(v, m, xi, vxi, T, tdamp, dt)
        v -= 0.5 * dt * FTM2V * g / m[:, None]
        x = x + dt * v
        g = grad(x)
        v -= 0.5 * dt * FTM2V * g / m[:, None]
        v *= _chain_half(v, m, xi, vxi, T, tdamp, dt)
    dx = np.abs(_min_image(xg - x, np.asarray(s["box"]))).max()
    dv = np.abs(vg - v).max()
    t_cpu = MVV2E * (m[:, None] * v ** 2).sum() / ((3 * n - 3) * KB)
    assert dx <= 1e-6 and dv <= 1e-6, (dx, dv)
    assert abs(out["T"][0] - t_cpu) <= 1e-4 * t_cpu, (out["T"][0], t_cpu)


def test_nvt_relaxes_to_target_temperature():
    """Started at twice the target, the chain brings the 648-atom water box to the target: the mean temperature over
    the last third of 1500 steps (dt 0.25 fs, Tdamp 10 fs) is within 15 % of 300 K."""
    import rxcuda
    import systems
    s = systems.water_box(6)
    eng = rxcuda.Engine(0)
    eng.set_forcefield(ffield_text())
    eng.set_control()
    eng.set_qeq(0.0, 10.0, 1e-6, 200)
    eng.set_systems([s])
    eng.md_setup(MASS, dt=0.25, t_start=300.0, t_damp=10.0, chain=3)
    eng.set_velocities(systems.maxwell_velocities(s, 600.0, seed=5))
    temps = [eng.md_run(50)["T"][0] for _ in range(30)]
    eng.close()
    tail = np.mean(temps[20:])
    assert abs(tail - 300.0) <= 45.0, temps
