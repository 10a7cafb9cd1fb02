"""Seeded synthetic input systems for the ReaxFF step (the reference ships no dataset; all of its inputs are generated).

Every generator returns a dict with
    origin (3,), box (3, 3) lattice vectors as rows, periodic (3,) int,
    x (n, 3) float64 positions [Angstrom], type (n,) int32 force-field type index (0 = C, 1 = H, 2 = O in
    ffield.synthetic.cho), tag (n,) int64 atom ids (1-based), mass (n,) float64 [g/mol], name.

Workloads:
  water_box(n_side)      216 H2O (n_side 6, 18.62 A) or 8000 H2O (n_side 20, 62.07 A): molecule centres on a cubic
                         lattice with +-0.3 A jitter, uniformly random orientation, O-H 0.96 A, H-O-H 104.5 deg.
  random_carbon(n, rho)  uniform random carbon with a 1.2 A minimum separation (random sequential addition, as
                         the reference's examples/graphitization/make_box.py:14-26 builds its 30k box).
  random_cho(k)          one of the 512 batched systems: n log-uniform in [64, 1024], C/H/O fractions from a
                         Dirichlet(1,1,1) with largest-remainder counts, density U(0.5, 1.2) g/cm3, positions uniform
                         with a 0.9 A minimum separation, seed 1000 + k.
"""
import math

import numpy as np

AMU_G = 1.66053906660e-24  # g per amu
MASS = np.array([12.0, 1.008, 15.999])
KB_KCAL = 0.0019872067      # kcal/mol/K


def _cubic(L):
    return np.eye(3) * L


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([
        [a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
        [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
        [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d],
    ])


def water_box(n_side=6, seed=20261203, density=1.0):
    """(n_side^3) H2O molecules in a cubic periodic box at `density` g/cm3."""
    nmol = n_side ** 3
    mol_mass = 2 * 1.008 + 15.999
    L = (nmol * mol_mass * AMU_G / density) ** (1.0 / 3.0) * 1e8
    rng = np.random.default_rng(seed)
    h = L / n_side
    half = math.radians(104.5) / 2
    local = np.array([[0.0, 0.0, 0.0],
                      [0.96 * math.sin(half), 0.0, 0.96 * math.cos(half)],
                      [-0.96 * math.sin(half), 0.0, 0.96 * math.cos(half)]])
    xs, ts = [], []
    for ix in range(n_side):
        for iy in range(n_side):
            for iz in range(n_side):
                centre = (np.array([ix, iy, iz]) + 0.5) * h + rng.uniform(-0.3, 0.3, size=3)
                rot = _random_rotation(rng)
                xs.append(centre + local @ rot.T)
                ts.append([2, 1, 1])
    x = np.concatenate(xs).reshape(-1, 3)
    t = np.array(ts, dtype=np.int32).reshape(-1)
    return _finish("water%d" % (3 * nmol), L, x, t)


def _rsa(n, L, dmin, rng, max_tries=200000):
    """Random sequential addition in a periodic cube with a cell grid (minimum separation dmin)."""
    nc = max(1, int(L // dmin))
    cw = L / nc
    cells = {}
    out = np.empty((n, 3))
    k = 0
    d2 = dmin * dmin
    tries = 0
    while k < n:
        tries += 1
        if tries > max_tries * max(1, n):
            raise RuntimeError("random packing failed")
        p = rng.uniform(0.0, L, size=3)
        c = tuple((p // cw).astype(int) % nc)
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in cells.get(((c[0] + dx) % nc, (c[1] + dy) % nc, (c[2] + dz) % nc), ()):
                        d = out[j] - p
                        d -= L * np.round(d / L)
                        if d @ d < d2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            out[k] = p
            cells.setdefault(c, []).append(k)
            k += 1
    return out


def _rsa_batched(n, L, dmin, rng, max_rounds=10000):
    """Random sequential addition in a periodic cube (minimum separation dmin), accepting candidates in batches: a
    candidate is kept when no accepted atom and no earlier candidate of its batch lies within dmin (k-d tree with
    periodic bounds). The same acceptance rule as _rsa, vectorised for the large serving systems."""
    from scipy.spatial import cKDTree
    out = np.empty((0, 3))
    for _ in range(max_rounds):
        need = n - len(out)
        if need <= 0:
            break
        cand = rng.uniform(0.0, L, size=(max(8, need + need // 4), 3)) % L
        ok = np.ones(len(cand), dtype=bool)
        if len(out):
            ok &= np.isinf(cKDTree(out, boxsize=L).query(cand, k=1, distance_upper_bound=dmin)[0])
        for a, b in sorted(cKDTree(cand, boxsize=L).query_pairs(dmin)):
            if ok[a]:
                ok[b] = False
        out = np.concatenate([out, cand[ok][:need]])
    if len(out) < n:
        raise RuntimeError("random packing failed")
    return out


def serving_request(k, seed=4242, nmin=100, nmax=5000, dmin=0.9):
    """The k-th request of the serving workload: a fresh CHO system built as random_cho but with n log-uniform in
    [nmin, nmax]; half the requests are single points (energy, forces, charges), half NVT runs of 10-1000 steps at
    300-3000 K. Returns (system, kind, steps, T)."""
    rng = np.random.default_rng([seed, k])
    n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
    frac = rng.dirichlet([1.0, 1.0, 1.0])
    raw = frac * n
    cnt = np.floor(raw).astype(int)
    for idx in np.argsort(-(raw - cnt), kind="stable")[: n - cnt.sum()]:
        cnt[idx] += 1
    types = np.repeat(np.arange(3, dtype=np.int32), cnt)
    rng.shuffle(types)
    density = rng.uniform(0.5, 1.2)
    L = (MASS[types].sum() * AMU_G / density) ** (1.0 / 3.0) * 1e8
    x = _rsa_batched(n, L, dmin, rng)
    kind = "sp" if rng.uniform() < 0.5 else "md"
    steps = int(rng.integers(10, 1001)) if kind == "md" else 0
    T = float(rng.uniform(300.0, 3000.0)) if kind == "md" else 0.0
    return _finish("req%d_%d" % (k, n), L, x, types), kind, steps, T


def poisson_arrivals(nreq, rate=200.0, seed=4242):
    """Arrival times [s] of a Poisson request stream."""
    return np.cumsum(np.random.default_rng([seed, 1 << 20]).exponential(1.0 / rate, size=nreq))


def random_carbon(n=30000, density=1.0, seed=4000, dmin=1.2, amu=12.0):
    """n carbon atoms uniformly random at `density` g/cm3 with RSA rejection of pairs closer than dmin (the algorithm of
    the reference's examples/graphitization/make_box.py:14-26; with amu = 12.011, 30,000 atoms at 1.0 g/cm3 give its
    84.265 A box). Large boxes use the batched acceptance of _rsa_batched."""
    L = (n * amu * AMU_G / density) ** (1.0 / 3.0) * 1e8
    rng = np.random.default_rng(seed)
    x = _rsa(n, L, dmin, rng) if n <= 2000 else _rsa_batched(n, L, dmin, rng)
    s = _finish("carbon%d" % n, L, x, np.zeros(n, dtype=np.int32))
    return s


def random_cho(k, nmin=64, nmax=1024, dmin=0.9):
    rng = np.random.default_rng(1000 + k)
    n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
    frac = rng.dirichlet([1.0, 1.0, 1.0])
    raw = frac * n
    cnt = np.floor(raw).astype(int)
    for idx in np.argsort(-(raw - cnt), kind="stable")[: n - cnt.sum()]:
        cnt[idx] += 1
    types = np.repeat(np.arange(3, dtype=np.int32), cnt)
    rng.shuffle(types)
    density = rng.uniform(0.5, 1.2)
    mass = MASS[types].sum()
    L = (mass * AMU_G / density) ** (1.0 / 3.0) * 1e8
    x = _rsa(n, L, dmin, rng)
    return _finish("cho%d_%d" % (k, n), L, x, types)


def _finish(name, L, x, t):
    x = np.ascontiguousarray(x, dtype=np.float64)
    x -= L * np.floor(x / L)
    return {
        "name": name,
        "origin": np.zeros(3),
        "box": _cubic(L),
        "periodic": np.ones(3, dtype=np.int32),
        "x": x,
        "type": np.ascontiguousarray(t, dtype=np.int32),
        "tag": np.arange(1, len(t) + 1, dtype=np.int64),
        "mass": MASS[t].astype(np.float64),
    }


def maxwell_velocities(sys_, T, seed):
    """Maxwell-Boltzmann velocities [A/fs] at temperature T with zero net momentum."""
    rng = np.random.default_rng(seed)
    m = sys_["mass"]
    # sqrt(kT/m) in A/fs: kT [kcal/mol] / m [g/mol] -> (kcal/g) ; 1 kcal/g = 4.184e6 m^2/s^2 = 4.184e-4 A^2/fs^2
    sig = np.sqrt(KB_KCAL * T / m * 4.184e-4)
    v = rng.normal(size=(len(m), 3)) * sig[:, None]
    p = (v * m[:, None]).sum(0) / m.sum()
    v -= p
    return v


def triclinic(s, tilts=(0.12, -0.08, 0.05), name=None):
    """A general triclinic version of a cubic system: box rows a = (L,0,0), b = (xy, L, 0), c = (xz, yz, L) with the
    tilts given as fractions of L; atoms keep their fractional coordinates (molecules are sheared slightly)."""
    L = float(s["box"][0][0])
    xy, xz, yz = (t * L for t in tilts)
    box = np.array([[L, 0.0, 0.0], [xy, L, 0.0], [xz, yz, L]])
    f = s["x"] / L
    out = dict(s)
    out["box"] = box
    out["x"] = np.ascontiguousarray(f @ box)
    out["name"] = name or (s["name"] + "_tri")
    return out
