"""Shared fixtures of the test suite: force field text, seeded systems, oracle handles and the parity metrics."""
from pathlib import Path

import numpy as np

import systems

REPO = Path(__file__).resolve().parents[1]
FFIELD = REPO / "metal-reax_b200" / "data" / "ffield.synthetic.cho"
# tolerances/tolerances.json "C3" of the reference (Metal-32 vs CPU-64 acceptance)
C3_ENERGY_PER_ATOM = 1e-3      # kcal/mol/atom
C3_FORCE_MAX = 0.05            # kcal/mol/A
C3_FORCE_RMS = 5e-3            # kcal/mol/A
C3_CHARGE_MAX = 1e-4           # e


def ffield_text():
    return FFIELD.read_text()


def fixed_charges(sys_):
    """Deterministic neutral test charges (the non-bonded terms take charges as input)."""
    t = sys_["type"]
    q = np.where(t == 2, -0.6, np.where(t == 1, 0.3, 0.05)).astype(np.float64)
    rng = np.random.default_rng(len(t))
    q += rng.uniform(-0.05, 0.05, size=len(t))
    return q - q.mean()


def small_systems():
    """Parity cases the oracle finishes in about a second each."""
    out = [systems.water_box(4), systems.random_cho(3), systems.random_cho(7), systems.random_cho(11)]
    c = systems.random_carbon(n=200, density=1.0, seed=77)
    c["name"] = "carbon200"
    out.append(c)
    return out


def force_metrics(g_ref, g):
    d = np.asarray(g) - np.asarray(g_ref)
    return float(np.abs(d).max()), float(np.sqrt((d ** 2).sum(axis=1).mean()))


def acks2_potentials(n, seed=17):
    """Seeded stand-ins for the kinetic potentials of fix acks2/reaxff (its s[N + i]), one per atom."""
    return np.random.default_rng(seed).normal(scale=0.5, size=n)
