"""CPU tests of the host side: the C ABI surface of librxcuda.so against include/rxcuda.h, argument checking that
needs no GPU, and the sharding of independent systems over ranks (world_size 2 over gloo)."""
import ctypes
import os
import re
from pathlib import Path

import numpy as np
import pytest

from helpers import ffield_text, fixed_charges, small_systems

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    text = (ROOT / "include" / "rxcuda.h").read_text()
    return sorted(set(re.findall(r"\b(rx_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_exported_surface():
    import rxcuda
    assert sorted(rxcuda.EXPORTS) == _declared()


def test_library_exports_every_declared_symbol():
    import rxcuda
    if not rxcuda.LIB_PATH.exists():
        pytest.skip("librxcuda.so not built")
    lib = ctypes.CDLL(str(rxcuda.LIB_PATH))
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_host_only_context_rejects_device_work():
    import rxcuda
    if not rxcuda.LIB_PATH.exists():
        pytest.skip("librxcuda.so not built")
    e = rxcuda.Engine(-1)
    e.set_forcefield(ffield_text())
    with pytest.raises(rxcuda.RxError) as ei:
        e.set_systems([small_systems()[0]])
    assert ei.value.code == 6                      # RX_ERR_STATE
    assert e.lib.rx_num_atoms(e.h) == 0
    assert e.lib.rx_kernel_launches(e.h) == 0
    with pytest.raises(rxcuda.RxError) as ei:
        e.set_qeq(0.0, 10.0, 1e-6, 0)              # imax >= 1
    assert ei.value.code == 1
    with pytest.raises(rxcuda.RxError):
        e.set_qeq(10.0, 5.0, 1e-6, 10)             # swb > swa
    with pytest.raises(rxcuda.RxError):
        e.set_capacities(32, 4, 32)                # no systems
    e.close()


def test_null_context_and_static_solve_argument_checks():
    import rxcuda
    if not rxcuda.LIB_PATH.exists():
        pytest.skip("librxcuda.so not built")
    lib = rxcuda.load()
    assert lib.rx_num_atoms(None) == 0
    assert lib.rx_set_qeq(None, 0.0, 10.0, 1e-6, 10, 0) != 0
    out = np.zeros(3, dtype=np.int32)
    assert lib.rx_get_capacities(None, out.ctypes.data) == 1
    err = ctypes.create_string_buffer(256)
    for n in (-5, 32769):
        assert lib.rx_qeq_solve_static(n, None, None, None, None, None, None, None, None, 1e-6, 10, None, None, None,
                                       err, 256) == 1
    assert b"32768" in err.value
    # n = 0 is the set-up call: without a GPU it reports the CUDA error, with one it succeeds
    assert lib.rx_qeq_solve_static(0, None, None, None, None, None, None, None, None, 0.0, 0, None, None, None,
                                   err, 256) in (0, 4)
    dummy = ctypes.c_void_p(16)
    assert lib.rx_qeq_solve_static(10, None, dummy, dummy, dummy, dummy, dummy, dummy, dummy, 1e-6, 10, None, None,
                                   None, err, 256) == 1
    assert b"null" in err.value
    assert lib.rx_qeq_solve_static(10, dummy, dummy, dummy, dummy, dummy, dummy, dummy, dummy, 0.0, 10, None, None,
                                   None, err, 256) == 1


# ------------------------------------------------------------------------------------------------ sharding
def test_shard_systems_partition():
    import batching
    import systems
    sizes = [len(systems.random_cho(k)["type"]) for k in range(64)]
    for world in (1, 2, 3, 4, 8):
        parts = [batching.shard_systems(sizes, world, r) for r in range(world)]
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(64))
        loads = batching.shard_loads(sizes, world)
        assert max(loads) - min(loads) <= max(sizes)
    with pytest.raises(ValueError):
        batching.shard_systems(sizes, 2, 2)


def _gloo_worker(rank, world, port, q):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT)); sys.path.insert(0, str(ROOT / "metal-reax_b200")); sys.path.insert(0, str(ROOT / "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import batching
        import systems
        from oracle.oracle import COracle
        ss = [systems.random_cho(k) for k in range(6)]
        mine = batching.shard_systems([len(s["type"]) for s in ss], world, rank)
        orc = COracle(ffield_text(), shell=15.0)
        res = {k: float(orc.single_point(ss[k], fixed_charges(ss[k]))["e"].sum()) for k in mine}
        allres = [None] * world
        dist.all_gather_object(allres, res)
        if rank == 0:
            merged = {}
            for r in allres:
                assert not (set(r) & set(merged))
                merged.update(r)
            q.put(merged)
    finally:
        dist.destroy_process_group()


def test_sharded_batch_over_two_ranks_gloo():
    """Two ranks each evaluate their shard of six systems (the oracle stands in for the GPU evaluation); the gathered
    per-system energies equal a single-rank evaluation of all six."""
    import socket
    import torch.multiprocessing as mp
    import systems
    from oracle.oracle import COracle
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    orc = COracle(ffield_text(), shell=15.0)
    ss = [systems.random_cho(k) for k in range(6)]
    assert sorted(merged) == list(range(6))
    for k, s in enumerate(ss):
        assert merged[k] == float(orc.single_point(s, fixed_charges(s))["e"].sum())


def test_pvector_matches_reference_layout():
    """rx_pvector against the reference's own to_lammps_pvector (where the reference oracle is built), and the slot
    rules of the pair style's energy tally."""
    import rxcuda
    if not rxcuda.LIB_PATH.exists():
        pytest.skip("librxcuda.so not built")
    e = np.arange(1, 14, dtype=np.float64) * 1.5
    pv, vdwl, coul = rxcuda.pvector(e)
    assert pv[3] == 0.0 and pv[12] == 0.0 and pv[1] == e[1] + e[2] and pv[13] == e[12]
    assert vdwl == pytest.approx(e[:11].sum()) and coul == pytest.approx(e[11] + e[12])
    from oracle.oracle import RefOracle
    if RefOracle.available():
        lib = ctypes.CDLL(str(RefOracle.PATH))
        out = np.zeros(14)
        lib.ref_pvector(e.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p))
        assert np.array_equal(out, pv)
