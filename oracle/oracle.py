"""TEST INFRASTRUCTURE ONLY: ctypes front end of the two CPU oracles.

* ``COracle``   the C restatement oracle/rx_oracle.c (built into oracle/_c/librxoracle.so by oracle/Makefile);
* ``RefOracle`` the reference's own cpu64 engine compiled from its sources (oracle/_ref/libreaxref.so), present
  wherever the reference tree was available at build time.

Both return the same dict: e (13 energies, kcal/mol, reference EnergyTerm order), grad (n, 3) dE/dx folded onto
owned atoms, census (7, n) int32, counts (bonds, pairs, nall, far entries).
Only tests/, the smoke check and the CPU-baseline leg of bench.py use this module.
"""
import ctypes
import os
from pathlib import Path

import numpy as np

from . import ffield as _ff

HERE = Path(__file__).resolve().parent
TERMS = ["bond", "over", "under", "lone_pair", "valence", "penalty", "coalition", "hbond", "torsion", "conjugation", "vdw",
         "coulomb", "polarization"]
CENSUS = ["bonds", "angle_sets", "torsions", "hbonds", "nonbonded", "sbo_region", "lp_trunc"]

_V = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int


def _ptr(a):
    return a.ctypes.data if a is not None else None


class _FF(ctypes.Structure):
    _fields_ = [("nt", _I), ("ngp", _I), ("gp", _V), ("vdw_type", _I), ("bo_cut", _D), ("nonb_low", _D), ("nonb_cut", _D),
                ("sbp", _V), ("tbp", _V), ("thb_n", _V), ("thb", _V), ("fbp_on", _V), ("fbp", _V), ("hbp_on", _V), ("hbp", _V),
                ("lgvdw", _I)]


class _Ctl(ctypes.Structure):
    _fields_ = [("bond_cut", _D), ("hbond_cut", _D), ("thb_cut", _D), ("thb_cutsq", _D), ("enobonds", _I), ("shell", _D)]


class _Box(ctypes.Structure):
    _fields_ = [("origin", _D * 3), ("vec", _D * 9), ("periodic", _I * 3)]


def reference_dir_default():
    """The reference checkout: $RX_REFERENCE_DIR, else a directory named `reference` beside this repository."""
    return os.environ.get("RX_REFERENCE_DIR", str(HERE.parent.parent / "reference"))


def build(reference_dir=None):
    """Compile the C restatement (always) and, when the reference tree exists, the reference oracle."""
    import subprocess
    subprocess.run(["make", "-s", "-C", str(HERE), "c"], check=True)
    ref = reference_dir or reference_dir_default()
    if Path(ref, "src", "cpu", "bonded.cpp").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", "REF=" + str(ref)], check=True)


def _box_struct(system):
    b = _Box()
    for c in range(3):
        b.origin[c] = float(system["origin"][c])
        b.periodic[c] = int(system["periodic"][c])
    vec = np.asarray(system["box"], dtype=np.float64).reshape(9)
    for c in range(9):
        b.vec[c] = float(vec[c])
    return b


class COracle:
    """The C restatement. `ffield_text` is parsed by the Python restatement of the reader (oracle/ffield.py)."""

    def __init__(self, ffield_text, bond_cut=5.0, hbond_cut=7.5, thb_cut=0.001, thb_cutsq=0.00001, enobonds=True, shell=12.0,
                 lgvdw=False):
        path = HERE / "_c" / "librxoracle.so"
        if not path.exists():
            build()
        self.lib = ctypes.CDLL(str(path))
        self.tables = _ff.parse(ffield_text, lgvdw=lgvdw)
        self.arr = _ff.oracle_arrays(self.tables)
        a = self.arr
        self.ff = _FF(self.tables["nt"], len(self.tables["gp"]), _ptr(a["gp"]), self.tables["vdw_type"], self.tables["bo_cut"],
                      self.tables["nonb_low"], self.tables["nonb_cut"], _ptr(a["sbp"]), _ptr(a["tbp"]), _ptr(a["thb_n"]),
                      _ptr(a["thb"]), _ptr(a["fbp_on"]), _ptr(a["fbp"]), _ptr(a["hbp_on"]), _ptr(a["hbp"]), 1 if lgvdw else 0)
        self.ctl = _Ctl(bond_cut, hbond_cut, thb_cut, thb_cutsq, 1 if enobonds else 0, shell)
        self.lib.rxo_single_point.argtypes = [_V, _V, _V, _I, _V, _V, _V, _V, _V, _V, _V, _V, _V, ctypes.c_char_p, _I]
        self.lib.rxo_single_point_acks2.argtypes = [_V, _V, _V, _I, _V, _V, _V, _V, _V, _V, _V, _V, _V, _V, ctypes.c_char_p,
                                                    _I]
        self.lib.rxo_qeq.argtypes = [_V, _V, _V, _I, _V, _V, _V, _D, _D, _D, _I, _V, _V, _V, _V, _V, _V, _V, ctypes.c_char_p, _I]
        self.lib.rxo_qeq_matvec.argtypes = [_V, _V, _V, _I, _V, _V, _V, _D, _D, _V, _V, ctypes.c_char_p, _I]

    def chi(self, types):
        return np.array([self.tables["sbp"][t]["chi"] for t in types])

    def single_point(self, system, q=None, s_kin=None):
        """Energies, gradient, census, counts and virial; with s_kin (the ACKS2 kinetic potentials, one per atom) the
        pair side of the ACKS2 charge model is added."""
        n = len(system["type"])
        x = np.ascontiguousarray(system["x"], dtype=np.float64)
        ty = np.ascontiguousarray(system["type"], dtype=np.int32)
        tg = np.ascontiguousarray(system["tag"], dtype=np.int64)
        qq = None if q is None else np.ascontiguousarray(q, dtype=np.float64)
        sk = None if s_kin is None else np.ascontiguousarray(s_kin, dtype=np.float64)
        e = np.zeros(13)
        g = np.zeros(3 * n)
        cen = np.zeros(7 * n, dtype=np.int32)
        cnt = np.zeros(4, dtype=np.int64)
        vir = np.zeros(6)
        err = ctypes.create_string_buffer(512)
        box = _box_struct(system)
        rc = self.lib.rxo_single_point_acks2(ctypes.byref(self.ff), ctypes.byref(self.ctl), ctypes.byref(box), n, _ptr(x),
                                             _ptr(ty), _ptr(tg), _ptr(qq), _ptr(sk), _ptr(e), _ptr(g), _ptr(cen), _ptr(cnt),
                                             _ptr(vir), err, 512)
        if rc:
            raise RuntimeError("oracle: " + err.value.decode())
        return {"e": e, "grad": g.reshape(n, 3), "census": cen.reshape(7, n), "counts": cnt, "virial": vir}

    def qeq(self, system, swa=0.0, swb=10.0, tol=1e-6, imax=200, s0=None, t0=None):
        n = len(system["type"])
        x = np.ascontiguousarray(system["x"], dtype=np.float64)
        ty = np.ascontiguousarray(system["type"], dtype=np.int32)
        tg = np.ascontiguousarray(system["tag"], dtype=np.int64)
        s0 = np.zeros(n) if s0 is None else np.ascontiguousarray(s0, dtype=np.float64)
        t0 = np.zeros(n) if t0 is None else np.ascontiguousarray(t0, dtype=np.float64)
        q, s, t = np.zeros(n), np.zeros(n), np.zeros(n)
        iters = np.zeros(2, dtype=np.int32)
        rel = np.zeros(2)
        err = ctypes.create_string_buffer(512)
        box = _box_struct(system)
        rc = self.lib.rxo_qeq(ctypes.byref(self.ff), ctypes.byref(self.ctl), ctypes.byref(box), n, _ptr(x), _ptr(ty), _ptr(tg),
                              swa, swb, tol, imax, _ptr(s0), _ptr(t0), _ptr(q), _ptr(s), _ptr(t), _ptr(iters), _ptr(rel), err, 512)
        if rc:
            raise RuntimeError("oracle: " + err.value.decode())
        return {"q": q, "s": s, "t": t, "iters": iters, "rel": rel}

    def qeq_matvec(self, system, v, swa=0.0, swb=10.0):
        n = len(system["type"])
        x = np.ascontiguousarray(system["x"], dtype=np.float64)
        ty = np.ascontiguousarray(system["type"], dtype=np.int32)
        tg = np.ascontiguousarray(system["tag"], dtype=np.int64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        y = np.zeros(n)
        err = ctypes.create_string_buffer(512)
        box = _box_struct(system)
        rc = self.lib.rxo_qeq_matvec(ctypes.byref(self.ff), ctypes.byref(self.ctl), ctypes.byref(box), n, _ptr(x), _ptr(ty),
                                     _ptr(tg), swa, swb, _ptr(v), _ptr(y), err, 512)
        if rc:
            raise RuntimeError("oracle: " + err.value.decode())
        return y


class RefOracle:
    """The reference's cpu64 engine itself (oracle/_ref/libreaxref.so)."""

    PATH = HERE / "_ref" / "libreaxref.so"

    @classmethod
    def available(cls):
        return cls.PATH.exists()

    def __init__(self, ffield_text, bond_cut=5.0, hbond_cut=7.5, enobonds=True, shell=12.0, lgvdw=False):
        self.lib = ctypes.CDLL(str(self.PATH))
        self.text = ffield_text.encode()
        self.bond_cut, self.hbond_cut, self.enobonds, self.shell = bond_cut, hbond_cut, enobonds, shell
        self.lgvdw = lgvdw
        self.lib.ref_single_point.argtypes = [ctypes.c_char_p, _V, _V, _V, _I, _V, _V, _V, _V, _D, _D, _D, _I, _I, _V, _V, _V,
                                              _V, _V, _V, ctypes.c_char_p, _I]
        self.lib.ref_table_dump.argtypes = [ctypes.c_char_p, _I, ctypes.c_char_p, ctypes.c_long]
        self.lib.ref_table_dump.restype = ctypes.c_long

    def peratom(self, system, q, cap=1 << 22):
        """Per-atom energies and virials (folded onto owners) and the bond table (partners as owner indices)."""
        n = len(system["type"])
        arrs = [np.ascontiguousarray(system[k], dtype=dt) for k, dt in
                (("origin", np.float64), ("box", np.float64), ("periodic", np.int32), ("x", np.float64), ("type", np.int32),
                 ("tag", np.int64))]
        qq = np.ascontiguousarray(q, dtype=np.float64)
        e, v = np.zeros(n), np.zeros(6 * n)
        start = np.zeros(n + 1, dtype=np.int32)
        partner = np.zeros(cap, dtype=np.int32)
        bo = np.zeros(cap)
        tbo, nlp = np.zeros(n), np.zeros(n)
        err = ctypes.create_string_buffer(512)
        f = self.lib.ref_peratom
        f.restype = ctypes.c_longlong
        f.argtypes = [ctypes.c_char_p] + [_V] * 3 + [_I] + [_V] * 4 + [_D] + [_V] * 5 + [ctypes.c_longlong] + [_V] * 2 + \
                     [ctypes.c_char_p, _I]
        nb = f(self.text, _ptr(arrs[0]), _ptr(arrs[1]), _ptr(arrs[2]), n, _ptr(arrs[3]), _ptr(arrs[4]), _ptr(arrs[5]),
               _ptr(qq), self.shell, _ptr(e), _ptr(v), _ptr(start), _ptr(partner), _ptr(bo), cap, _ptr(tbo), _ptr(nlp), err, 512)
        if nb < 0:
            raise RuntimeError("reference: " + err.value.decode())
        return {"eatom": e, "vatom": v.reshape(n, 6), "start": start, "partner": partner[:nb], "bo": bo[:nb],
                "total_bo": tbo, "nlp": nlp}

    def table_dump(self, portable=False):
        buf = ctypes.create_string_buffer(1 << 22)
        m = self.lib.ref_table_dump(self.text, 1 if portable else 0, buf, len(buf))
        if m < 0:
            raise RuntimeError(buf.value.decode())
        return buf.value.decode()

    def single_point(self, system, q=None, s_kin=None):
        n = len(system["type"])
        x = np.ascontiguousarray(system["x"], dtype=np.float64)
        ty = np.ascontiguousarray(system["type"], dtype=np.int32)
        tg = np.ascontiguousarray(system["tag"], dtype=np.int64)
        sk = None if s_kin is None else np.ascontiguousarray(s_kin, dtype=np.float64)
        org = np.ascontiguousarray(system["origin"], dtype=np.float64)
        box = np.ascontiguousarray(system["box"], dtype=np.float64)
        per = np.ascontiguousarray(system["periodic"], dtype=np.int32)
        qq = None if q is None else np.ascontiguousarray(q, dtype=np.float64)
        e = np.zeros(13)
        g = np.zeros(3 * n)
        cen = np.zeros(7 * n, dtype=np.int32)
        cnt = np.zeros(4, dtype=np.int64)
        vir = np.zeros(6)
        err = ctypes.create_string_buffer(512)
        rc = self.lib.ref_single_point(self.text, _ptr(org), _ptr(box), _ptr(per), n, _ptr(x), _ptr(ty), _ptr(tg), _ptr(qq),
                                       self.bond_cut, self.hbond_cut, self.shell, 1 if self.enobonds else 0,
                                       1 if self.lgvdw else 0, _ptr(sk), _ptr(e), _ptr(g),
                                       _ptr(cen), _ptr(cnt), _ptr(vir), err, 512)
        if rc:
            raise RuntimeError("reference: " + err.value.decode())
        return {"e": e, "grad": g.reshape(n, 3), "census": cen.reshape(7, n), "counts": cnt, "virial": vir}
