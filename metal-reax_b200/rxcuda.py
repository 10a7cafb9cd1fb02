"""Python front end of librxcuda.so, the C ABI of the B200 ReaxFF engine (include/rxcuda.h).

Mirrors the reference's plugin surface for the hot path:
  ``Engine.set_forcefield``   pair_coeff * * ffield ... (parse_force_field, src/io/ffield_parser.cpp:91)
  ``Engine.set_control``      ControlParams / pair_style keywords (bond_cut, hbond_cut, thb_cut, thb_cutsq, enobonds)
  ``Engine.set_qeq``          fix qeq/reaxff/metal <nevery> <swa> <swb> <tol> reaxff maxiter <imax> [strict]
  ``Engine.compute``          PairReaxFFMetal::compute (plugin/adapter/pair_reaxff_metal.cpp:412-524)
  ``Engine.qeq_solve``        FixQEqReaxFFMetal resident CG (plugin/adapter/fix_qeq_reaxff_metal.cpp:65-124)
  ``Engine.qeq_matvec``       FixQEqReaxFFMetal::sparse_matvec (:190-205)
  ``Engine.md_*``             an NVT driver (the reference delegates integration to LAMMPS `fix nvt`)

Errors are raised as ``RxError`` with the status code and the engine's message, as the reference's adapter turns
engine exceptions into LAMMPS errors. There is no CPU fallback: without the built library or without a GPU every
device call fails.
"""
import ctypes
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "librxcuda.so"
TERMS = ["bond", "over", "under", "lone_pair", "valence", "penalty", "coalition", "hbond", "torsion", "conjugation", "vdw",
         "coulomb", "polarization"]
CENSUS = ["bonds", "angle_sets", "torsions", "hbonds", "nonbonded", "sbo_region", "lp_trunc"]
RX_COMPUTE_QEQ = 1
RX_COMPUTE_CENSUS = 2
RX_COMPUTE_QEQ_COLD = 4
RX_COMPUTE_PERATOM = 8
TUNE = {"pairs_tpb": 1, "bonds_tpb": 2, "nonbonded_tpb": 3, "hbond_tpb": 4, "atom_tpb": 5, "lone_grid_min": 6, "overlap": 7, "cg_blocks_per_sm": 8}
STATUS = {0: "ok", 1: "invalid", 2: "ffield", 3: "capacity", 4: "cuda", 5: "not_converged", 6: "state", 7: "timeout"}
EXPORTS = ["rx_create", "rx_destroy", "rx_last_error", "rx_set_forcefield", "rx_forcefield_dump", "rx_forcefield_params",
           "rx_set_control", "rx_set_systems", "rx_num_atoms", "rx_set_positions", "rx_get_positions", "rx_set_charges",
           "rx_get_charges", "rx_set_qeq", "rx_qeq_solve", "rx_qeq_matvec", "rx_compute", "rx_md_setup", "rx_set_velocities",
           "rx_get_velocities", "rx_md_run", "rx_kernel_launches", "rx_stream", "rx_set_timing", "rx_phase_times",
           "rx_qeq_solve_static", "rx_set_capacities", "rx_get_capacities", "rx_qeq_last", "rx_get_virial", "rx_set_neighbor", "rx_qeq_cg", "rx_set_acks2", "rx_qeq_reset", "rx_update_systems", "rx_md_targets", "rx_get_gradient", "rx_md_charges", "rx_autotune", "rx_set_tuning", "rx_qeq_refinements", "rx_pvector", "rx_get_peratom",
           "rx_get_bonds", "rx_forcefield_element", "rx_host_alloc", "rx_host_free"]

_V = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int
_lib = None


class RxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%s): %s" % (STATUS.get(code, code), code, msg))
        self.code = code


def load():
    """Load librxcuda.so (built by metal-reax_b200/build.py). Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError("librxcuda.so is not built (%s); run metal-reax_b200/build.py" % LIB_PATH)
    lib = ctypes.CDLL(str(LIB_PATH))
    sig = {
        "rx_create": (_V, [_I]), "rx_destroy": (None, [_V]), "rx_last_error": (ctypes.c_char_p, [_V]),
        "rx_set_forcefield": (_I, [_V, ctypes.c_char_p, _I]),
        "rx_forcefield_dump": (ctypes.c_long, [_V, _I, ctypes.c_char_p, ctypes.c_long]),
        "rx_forcefield_params": (_I, [_V, _V, _V, _V, _V, _V]),
        "rx_set_control": (_I, [_V, _D, _D, _D, _D, _I]),
        "rx_set_systems": (_I, [_V, _I, _V, _V, _V, _V, _V, _V]), "rx_num_atoms": (_I, [_V]),
        "rx_set_positions": (_I, [_V, _V]), "rx_get_positions": (_I, [_V, _V]),
        "rx_set_charges": (_I, [_V, _V]), "rx_get_charges": (_I, [_V, _V]),
        "rx_set_qeq": (_I, [_V, _D, _D, _D, _I, _I]), "rx_qeq_solve": (_I, [_V, _V, _V]), "rx_qeq_matvec": (_I, [_V, _V, _V]),
        "rx_compute": (_I, [_V, _I, _V, _V, _V, _V]),
        "rx_md_setup": (_I, [_V, _V, _D, _D, _D, _D, _I]), "rx_set_velocities": (_I, [_V, _V]),
        "rx_get_velocities": (_I, [_V, _V]), "rx_md_run": (_I, [_V, _I, _V, _V]),
        "rx_stream": (_V, [_V]), "rx_set_timing": (_I, [_V, _I]), "rx_kernel_launches": (ctypes.c_int64, [_V]),
        "rx_phase_times": (_I, [_V, ctypes.c_char_p, ctypes.c_long, _V, _I]),
        "rx_qeq_solve_static": (_I, [_I, _V, _V, _V, _V, _V, _V, _V, _V, _D, _I, _V, _V, _V, ctypes.c_char_p, _I]),
        "rx_set_capacities": (_I, [_V, _I, _I, _I]), "rx_get_capacities": (_I, [_V, _V]),
        "rx_qeq_last": (_I, [_V, _V, _V]), "rx_get_virial": (_I, [_V, _V]), "rx_set_neighbor": (_I, [_V, _D]), "rx_qeq_cg": (_I, [_V, _V, _V, _V, _V, _V, _V]), "rx_set_acks2": (_I, [_V, _V]), "rx_qeq_reset": (_I, [_V]), "rx_md_targets": (_I, [_V, _V, _V]), "rx_get_gradient": (_I, [_V, _V]), "rx_md_charges": (_I, [_V, _I]), "rx_autotune": (_I, [_V, _I, _V]),
        "rx_set_tuning": (_I, [_V, _I, _I]), "rx_qeq_refinements": (_I, [_V]), "rx_pvector": (_I, [_V, _V, _V, _V]), "rx_get_peratom": (_I, [_V, _V, _V]), "rx_forcefield_element": (_I, [_V, ctypes.c_char_p]),
        "rx_get_bonds": (ctypes.c_longlong, [_V, _V, _V, _V, _V, _V, _V, ctypes.c_longlong]),
        "rx_update_systems": (_I, [_V, _I, _V, _I, _V, _V, _V, _V, _V, _V, _V, _V]),
        "rx_host_alloc": (_V, [ctypes.c_size_t]), "rx_host_free": (None, [_V]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data


class _PinnedBlock:
    """Owns one page-locked allocation (rx_host_alloc); freed with the last array that views it."""

    def __init__(self, nbytes):
        self.lib = load()
        self.ptr = self.lib.rx_host_alloc(nbytes)
        if not self.ptr:
            raise MemoryError("rx_host_alloc(%d) failed" % nbytes)

    def __del__(self):
        if getattr(self, "ptr", None):
            self.lib.rx_host_free(self.ptr)
            self.ptr = None


def pinned_array(shape, dtype=np.float64):
    """A numpy array in page-locked host memory: rx_set_positions and rx_compute copy from and into it directly."""
    dt = np.dtype(dtype)
    n = int(np.prod(shape))
    block = _PinnedBlock(max(1, n * dt.itemsize))
    buf = (ctypes.c_char * max(1, n * dt.itemsize)).from_address(block.ptr)
    buf.owner = block   # the array keeps the ctypes buffer alive (its base), the buffer the allocation
    return np.frombuffer(buf, dtype=dt, count=n).reshape(shape)


def pvector(e13):
    """LAMMPS's 14-slot pair energy vector and (eng_vdwl, eng_coul) of one system's 13 energies (rx_pvector)."""
    lib = load()
    e = np.ascontiguousarray(e13, dtype=np.float64)
    pv = np.zeros(14)
    vdwl, coul = ctypes.c_double(0.0), ctypes.c_double(0.0)
    rc = lib.rx_pvector(_p(e), _p(pv), ctypes.addressof(vdwl), ctypes.addressof(coul))
    if rc != 0:
        raise RxError(rc, "rx_pvector")
    return pv, vdwl.value, coul.value


class Engine:
    """One engine context: a force field and one or more independent periodic systems (a batch)."""

    def __init__(self, device=0):
        self.lib = load()
        self.h = self.lib.rx_create(device)
        if not self.h:
            raise RxError(4, self.lib.rx_last_error(None).decode())
        self.nsys = 0
        self.natoms = None
        self.na = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.rx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise RxError(rc, self.lib.rx_last_error(self.h).decode())

    # ---- configuration
    def set_forcefield(self, text, lgvdw=False):
        self._check(self.lib.rx_set_forcefield(self.h, text.encode(), 1 if lgvdw else 0))

    def forcefield_dump(self, portable=False):
        n = self.lib.rx_forcefield_dump(self.h, 1 if portable else 0, None, 0)
        if n < 0:
            raise RxError(6, self.lib.rx_last_error(self.h).decode())
        buf = ctypes.create_string_buffer(n + 1)
        self.lib.rx_forcefield_dump(self.h, 1 if portable else 0, buf, n + 1)
        return buf.value.decode()

    def forcefield_params(self):
        nt = ctypes.c_int(0)
        self._check(self.lib.rx_forcefield_params(self.h, ctypes.addressof(nt), None, None, None, None))
        chi, eta, gamma, mass = (np.zeros(nt.value) for _ in range(4))
        self._check(self.lib.rx_forcefield_params(self.h, ctypes.addressof(nt), _p(chi), _p(eta), _p(gamma), _p(mass)))
        return {"chi": chi, "eta": eta, "gamma": gamma, "mass": mass}

    def set_control(self, bond_cut=5.0, hbond_cut=7.5, thb_cut=0.001, thb_cutsq=0.00001, enobonds=True):
        self._check(self.lib.rx_set_control(self.h, bond_cut, hbond_cut, thb_cut, thb_cutsq, 1 if enobonds else 0))

    def set_neighbor(self, skin=1.0):
        self._check(self.lib.rx_set_neighbor(self.h, skin))

    def set_qeq(self, swa=0.0, swb=10.0, tol=1e-6, imax=200, strict=False):
        self._check(self.lib.rx_set_qeq(self.h, swa, swb, tol, imax, 1 if strict else 0))

    def set_systems(self, systems):
        """systems: list of dicts (origin, box, periodic, x, type, tag) as produced by systems.py."""
        natoms = np.array([len(s["type"]) for s in systems], dtype=np.int32)
        origin = np.ascontiguousarray(np.concatenate([np.asarray(s["origin"], dtype=np.float64) for s in systems]))
        box = np.ascontiguousarray(np.concatenate([np.asarray(s["box"], dtype=np.float64).reshape(9) for s in systems]))
        per = np.ascontiguousarray(np.concatenate([np.asarray(s["periodic"], dtype=np.int32) for s in systems]))
        ty = np.ascontiguousarray(np.concatenate([np.asarray(s["type"], dtype=np.int32) for s in systems]))
        tg = np.ascontiguousarray(np.concatenate([np.asarray(s["tag"], dtype=np.int64) for s in systems]))
        self._check(self.lib.rx_set_systems(self.h, len(systems), _p(natoms), _p(origin), _p(box), _p(per), _p(ty), _p(tg)))
        self.nsys = len(systems)
        self.natoms = natoms
        self.na = int(natoms.sum())
        self.offsets = np.concatenate([[0], np.cumsum(natoms)])
        x = np.ascontiguousarray(np.concatenate([np.asarray(s["x"], dtype=np.float64).reshape(-1, 3) for s in systems]))
        self.set_positions(x)

    def update_systems(self, keep, new_systems, new_velocities=None):
        """Continuous batching: keep the listed current systems (their device state carried, in this order) and append
        new ones (dicts as for set_systems, velocities per new system or None)."""
        keep = np.ascontiguousarray(keep, dtype=np.int32)
        nn = len(new_systems)
        if nn:
            natoms = np.array([len(s["type"]) for s in new_systems], dtype=np.int32)
            origin = np.ascontiguousarray(np.concatenate([np.asarray(s["origin"], dtype=np.float64) for s in new_systems]))
            box = np.ascontiguousarray(np.concatenate([np.asarray(s["box"], dtype=np.float64).reshape(9) for s in new_systems]))
            per = np.ascontiguousarray(np.concatenate([np.asarray(s["periodic"], dtype=np.int32) for s in new_systems]))
            ty = np.ascontiguousarray(np.concatenate([np.asarray(s["type"], dtype=np.int32) for s in new_systems]))
            tg = np.ascontiguousarray(np.concatenate([np.asarray(s["tag"], dtype=np.int64) for s in new_systems]))
            x = np.ascontiguousarray(np.concatenate([np.asarray(s["x"], dtype=np.float64).reshape(-1, 3) for s in new_systems]))
            v = None
            if new_velocities is not None:
                v = np.ascontiguousarray(np.concatenate([np.asarray(vv, dtype=np.float64).reshape(-1, 3) for vv in new_velocities]))
        else:
            natoms = origin = box = per = ty = tg = x = v = None
        self._check(self.lib.rx_update_systems(self.h, len(keep), _p(keep), nn, _p(natoms), _p(origin), _p(box), _p(per),
                                               _p(ty), _p(tg), _p(x), _p(v)))
        old = self.natoms
        kept = [int(old[k]) for k in keep]
        self.natoms = np.array(kept + ([] if not nn else list(natoms)), dtype=np.int32)
        self.nsys = len(self.natoms)
        self.na = int(self.natoms.sum())
        self.offsets = np.concatenate([[0], np.cumsum(self.natoms)])

    def autotune(self, reps=3):
        """Pick the fastest launch shapes on the current systems; returns them."""
        out = np.zeros(5, dtype=np.int32)
        self._check(self.lib.rx_autotune(self.h, reps, _p(out)))
        return dict(zip(["pairs_tpb", "bonds_tpb", "nonbonded_tpb", "hbond_tpb", "atom_tpb"], out.tolist()))

    def set_tuning(self, key, value):
        self._check(self.lib.rx_set_tuning(self.h, TUNE[key], int(value)))

    def md_charges(self, on=True):
        """False: MD keeps the charges as set (no charge fix)."""
        self._check(self.lib.rx_md_charges(self.h, 1 if on else 0))

    def md_targets(self, t_target=None, active=None):
        t = None if t_target is None else np.ascontiguousarray(t_target, dtype=np.float64)
        a = None if active is None else np.ascontiguousarray(active, dtype=np.int32)
        self._check(self.lib.rx_md_targets(self.h, _p(t), _p(a)))

    def set_positions(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        if x.size != 3 * self.na:
            raise ValueError("need 3 coordinates per atom")
        self._check(self.lib.rx_set_positions(self.h, _p(x)))

    def get_positions(self):
        x = np.zeros(3 * self.na)
        self._check(self.lib.rx_get_positions(self.h, _p(x)))
        return x.reshape(-1, 3)

    def set_charges(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64)
        self._check(self.lib.rx_set_charges(self.h, _p(q)))

    def get_charges(self):
        q = np.zeros(self.na)
        self._check(self.lib.rx_get_charges(self.h, _p(q)))
        return q

    # ---- evaluation
    def compute(self, qeq=False, census=False, counts=False, cold=False, peratom=False, grad_out=None):
        """grad_out: an (n, 3) float64 array to receive the gradient (page-locked, from pinned_array, for a direct copy)."""
        e = np.empty(13 * self.nsys)   # every entry is written by rx_compute
        if grad_out is not None:
            if grad_out.dtype != np.float64 or grad_out.size != 3 * self.na or not grad_out.flags.c_contiguous:
                raise ValueError("grad_out must be a contiguous float64 array of 3 entries per atom")
            g = grad_out.reshape(-1)
        else:
            g = np.empty(3 * self.na)
        cen = np.zeros(7 * self.na, dtype=np.int32) if census else None
        cnt = np.zeros(4, dtype=np.int64) if counts else None
        flags = (RX_COMPUTE_QEQ if qeq else 0) | (RX_COMPUTE_CENSUS if census else 0) | (RX_COMPUTE_QEQ_COLD if cold else 0) | \
            (RX_COMPUTE_PERATOM if peratom else 0)
        self._check(self.lib.rx_compute(self.h, flags, _p(e), _p(g), _p(cen), _p(cnt)))
        out = {"e": e.reshape(self.nsys, 13), "grad": g.reshape(-1, 3)}
        if census:
            out["census"] = cen.reshape(7, self.na)
        if counts:
            out["counts"] = cnt
        return out

    def set_acks2(self, s_kin):
        """Kinetic potentials of fix acks2/reaxff (one per atom), or None to switch the ACKS2 pair terms off."""
        sk = None if s_kin is None else np.ascontiguousarray(s_kin, dtype=np.float64)
        self._check(self.lib.rx_set_acks2(self.h, _p(sk)))
        self._s_kin = sk

    def peratom(self):
        """Per-atom energies (n,) and virials (n, 6) of the last compute(peratom=True)."""
        e = np.zeros(self.na)
        v = np.zeros(6 * self.na)
        self._check(self.lib.rx_get_peratom(self.h, _p(e), _p(v)))
        return e, v.reshape(-1, 6)

    def bonds(self):
        """The bond table of the last evaluation: start (n+1,), partner, shift (nb, 3), bo, total_bo, nlp."""
        nb = self.lib.rx_get_bonds(self.h, None, None, None, None, None, None, 0)
        if nb < 0:
            raise RxError(6, self.lib.rx_last_error(self.h).decode())
        start = np.zeros(self.na + 1, dtype=np.int32)
        partner = np.zeros(max(nb, 1), dtype=np.int32)
        shift = np.zeros(3 * max(nb, 1), dtype=np.int32)
        bo = np.zeros(max(nb, 1))
        tbo, nlp = np.zeros(self.na), np.zeros(self.na)
        got = self.lib.rx_get_bonds(self.h, _p(start), _p(partner), _p(shift), _p(bo), _p(tbo), _p(nlp), nb)
        if got != nb:
            raise RxError(6, self.lib.rx_last_error(self.h).decode())
        return {"start": start, "partner": partner[:nb], "shift": shift[:3 * nb].reshape(-1, 3), "bo": bo[:nb],
                "total_bo": tbo, "nlp": nlp}

    def gradient(self):
        """dE/dx of the last force evaluation (rx_compute or the last MD step)."""
        g = np.zeros(3 * self.na)
        self._check(self.lib.rx_get_gradient(self.h, _p(g)))
        return g.reshape(-1, 3)

    def virial(self):
        """LAMMPS-order virial (xx, yy, zz, xy, xz, yz) of the last force evaluation, per system."""
        v = np.zeros(6 * self.nsys)
        self._check(self.lib.rx_get_virial(self.h, _p(v)))
        return v.reshape(self.nsys, 6)

    def qeq_solve(self):
        it = np.zeros(2 * self.nsys, dtype=np.int32)
        rel = np.zeros(2 * self.nsys)
        self._check(self.lib.rx_qeq_solve(self.h, _p(it), _p(rel)))
        return {"q": self.get_charges(), "iters": it.reshape(-1, 2), "rel": rel.reshape(-1, 2)}

    def qeq_reset(self):
        """Zero the charge histories: the next solve starts cold."""
        self._check(self.lib.rx_qeq_reset(self.h))

    def qeq_cg(self, b, x0=None):
        """Both CG systems for given right-hand sides b (2, NA) and guesses x0 (2, NA) (mtl::Context::qeq_solve)."""
        b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1)
        x0 = None if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).reshape(-1)
        x = np.zeros(2 * self.na)
        it = np.zeros(2 * self.nsys, dtype=np.int32)
        rel = np.zeros(2 * self.nsys)
        st = np.zeros(2 * self.nsys, dtype=np.int32)
        self._check(self.lib.rx_qeq_cg(self.h, _p(b), _p(x0), _p(x), _p(it), _p(rel), _p(st)))
        return {"x": x.reshape(2, -1), "iters": it.reshape(-1, 2), "rel": rel.reshape(-1, 2), "status": st.reshape(-1, 2)}

    def qeq_matvec(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        y = np.zeros(self.na)
        self._check(self.lib.rx_qeq_matvec(self.h, _p(v), _p(y)))
        return y

    # ---- dynamics
    def md_setup(self, mass_per_type, dt=0.25, t_start=300.0, t_stop=None, t_damp=25.0, chain=3):
        m = np.ascontiguousarray(mass_per_type, dtype=np.float64)
        self._check(self.lib.rx_md_setup(self.h, _p(m), dt, t_start, t_start if t_stop is None else t_stop, t_damp, chain))

    def set_velocities(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        self._check(self.lib.rx_set_velocities(self.h, _p(v)))

    def get_velocities(self):
        v = np.zeros(3 * self.na)
        self._check(self.lib.rx_get_velocities(self.h, _p(v)))
        return v.reshape(-1, 3)

    def md_run(self, nsteps):
        e = np.zeros(13 * self.nsys)
        t = np.zeros(self.nsys)
        self._check(self.lib.rx_md_run(self.h, nsteps, _p(e), _p(t)))
        return {"e": e.reshape(self.nsys, 13), "T": t}

    def kernel_launches(self):
        return int(self.lib.rx_kernel_launches(self.h))

    def stream(self):
        return self.lib.rx_stream(self.h)

    def qeq_last(self):
        it = np.zeros(2 * self.nsys, dtype=np.int32)
        rel = np.zeros(2 * self.nsys)
        self._check(self.lib.rx_qeq_last(self.h, _p(it), _p(rel)))
        return {"iters": it.reshape(-1, 2), "rel": rel.reshape(-1, 2)}

    def qeq_refinements(self):
        return int(self.lib.rx_qeq_refinements(self.h))

    def set_capacities(self, nbr, bonds, near):
        self._check(self.lib.rx_set_capacities(self.h, int(nbr), int(bonds), int(near)))

    def capacities(self):
        out = np.zeros(3, dtype=np.int32)
        self._check(self.lib.rx_get_capacities(self.h, _p(out)))
        return tuple(int(v) for v in out)

    def set_timing(self, on=True):
        self._check(self.lib.rx_set_timing(self.h, 1 if on else 0))

    def phase_times(self):
        buf = ctypes.create_string_buffer(4096)
        ms = np.zeros(32)
        n = self.lib.rx_phase_times(self.h, buf, 4096, _p(ms), 32)
        names = buf.value.decode().split("\n")[:n]
        return dict(zip(names, ms[:n]))
