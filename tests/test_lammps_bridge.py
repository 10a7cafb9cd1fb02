"""The LAMMPS side of the CUDA backend (metal-reax_b200/lammps/rx_lammps.{hpp,cpp}, librxlammps.so): what the pair
style and the QEq fix of the reference's adapter do between LAMMPS's arrays and the engine
(plugin/adapter/pair_reaxff_metal.cpp:103-160,412-524; fix_qeq_reaxff_metal.cpp:65-124).

CPU: the pair_coeff element mapping (NULL types, case-insensitive symbols, unknown elements rejected as pair reaxff
does), and LAMMPS's box (boxlo/boxhi, xy/xz/yz tilts) as lattice vectors. GPU: forces, energy vector, virial and
charges through the bridge with LAMMPS-layout arrays (owned atoms in LAMMPS order, NULL-typed atoms skipped) equal the
engine's own for the same atoms.
"""
import ctypes
from pathlib import Path

import numpy as np
import pytest

from helpers import ffield_text

LIB = Path(__file__).resolve().parents[1] / "metal-reax_b200" / "librxlammps.so"


def _lib():
    if not LIB.exists():
        pytest.skip("librxlammps.so not built")
    lib = ctypes.CDLL(str(LIB))
    V, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.rxl_create.restype = V
    lib.rxl_create.argtypes = [I]
    lib.rxl_destroy.argtypes = [V]
    lib.rxl_last_error.restype = ctypes.c_char_p
    lib.rxl_coeff.argtypes = [V, ctypes.c_char_p, ctypes.c_char_p, I]
    lib.rxl_type_element.argtypes = [V, I]
    lib.rxl_lattice.argtypes = [V, V, D, D, D, V, V]
    lib.rxl_compute.argtypes = [V, I] + [V] * 13
    lib.rxl_equilibrate.argtypes = [V, I] + [V] * 9
    return lib


def test_pair_coeff_mapping_and_box():
    lib = _lib()
    h = lib.rxl_create(-1)   # a host-only engine context reads force fields without a GPU
    assert h, lib.rxl_last_error()
    assert lib.rxl_coeff(h, ffield_text().encode(), b"o NULL C h", 0) == 0, lib.rxl_last_error()
    assert [lib.rxl_type_element(h, t) for t in (1, 2, 3, 4)] == [2, -1, 0, 1]
    assert lib.rxl_coeff(h, ffield_text().encode(), b"C Xx", 0) == 1
    assert b"Non-existent ReaxFF type" in lib.rxl_last_error()
    assert lib.rxl_coeff(h, ffield_text().encode(), b"NULL NULL", 0) == 1
    lib.rxl_destroy(h)
    lo, hi = np.array([1.0, -2.0, 0.5]), np.array([11.0, 8.0, 12.5])
    origin, box = np.zeros(3), np.zeros(9)
    lib.rxl_lattice(lo.ctypes.data, hi.ctypes.data, 0.5, -1.0, 2.0, origin.ctypes.data, box.ctypes.data)
    assert np.array_equal(origin, lo)
    assert np.array_equal(box.reshape(3, 3), [[10.0, 0, 0], [0.5, 10.0, 0], [-1.0, 2.0, 12.0]])


def test_null_handle_is_an_error_not_a_crash():
    """Where rxl_create fails (no usable GPU, a bad device ordinal), the calls that take its NULL handle report an
    error through rxl_last_error instead of dereferencing it."""
    lib = _lib()
    assert lib.rxl_coeff(None, ffield_text().encode(), b"C H O", 0) == 1
    assert b"null bridge handle" in lib.rxl_last_error()
    assert lib.rxl_type_element(None, 1) == -2
    f = np.zeros((1, 3))
    zero3 = np.zeros(3)
    assert lib.rxl_compute(None, 1, zero3.ctypes.data, None, None, None, zero3.ctypes.data, zero3.ctypes.data, None,
                           None, f.ctypes.data, None, None, None, None) == 1
    lib.rxl_destroy(None)   # deleting nothing is allowed


@pytest.mark.gpu
def test_bridge_matches_engine():
    import rxcuda
    import systems
    lib = _lib()
    s = systems.water_box(4)
    n = len(s["type"])
    L = np.asarray(s["box"])
    # LAMMPS types: 1 = H, 2 = O, plus a NULL-typed probe atom (type 3) that the style must leave alone
    lmp_type = np.where(s["type"] == 1, 1, 2).astype(np.int32)
    x = np.vstack([s["x"], [[0.5, 0.5, 0.5]]])
    ltype = np.concatenate([lmp_type, [3]]).astype(np.int32)
    tag = np.concatenate([s["tag"], [10 ** 6]]).astype(np.int64)
    q = np.concatenate([np.where(s["type"] == 2, -0.6, 0.3), [0.9]])
    h = lib.rxl_create(0)
    assert lib.rxl_coeff(h, ffield_text().encode(), b"H O NULL", 0) == 0, lib.rxl_last_error()
    lo, hi = np.zeros(3), np.diag(L).copy()
    f = np.zeros((n + 1, 3))
    pv, e2, vir = np.zeros(14), np.zeros(2), np.zeros(6)
    rc = lib.rxl_compute(h, n + 1, x.ctypes.data, ltype.ctypes.data, tag.ctypes.data, q.ctypes.data, lo.ctypes.data,
                         hi.ctypes.data, None, None, f.ctypes.data, pv.ctypes.data, e2.ctypes.data, vir.ctypes.data, None)
    assert rc == 0, lib.rxl_last_error()
    e = rxcuda.Engine(0)
    e.set_forcefield(ffield_text())
    e.set_control()
    e.set_systems([s])
    e.set_charges(q[:n])
    out = e.compute()
    assert np.array_equal(f[:n], -out["grad"]) and np.all(f[n] == 0.0)
    ref_pv, vdwl, coul = rxcuda.pvector(out["e"][0])
    assert np.array_equal(pv, ref_pv) and e2[0] == vdwl and e2[1] == coul
    assert np.array_equal(vir, e.virial()[0])
    # the QEq fix: charges of the handled atoms from the engine's solve, the NULL atom's charge untouched
    e.set_qeq()
    it = np.zeros(2, dtype=np.int32)
    qq = q.copy()
    assert lib.rxl_equilibrate(h, n + 1, x.ctypes.data, ltype.ctypes.data, tag.ctypes.data, lo.ctypes.data, hi.ctypes.data,
                               None, None, qq.ctypes.data, it.ctypes.data) == 0, lib.rxl_last_error()
    e.qeq_reset()
    ref = e.qeq_solve()
    assert np.abs(qq[:n] - ref["q"]).max() <= 1e-12 and qq[n] == 0.9 and it.min() > 0
    lib.rxl_destroy(h)
    e.close()
