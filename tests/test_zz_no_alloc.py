"""The allocation-free charge solve (rx_qeq_solve_static) against the engine's own charge solve (rx_qeq_solve).

rx_qeq_solve_static exists for callers that must not have a library allocate device memory behind their back (codes
with their own pooled allocator or a fixed memory budget, and codes running where an allocation and its implicit
synchronisation are not allowed): they hand it the charge matrix and every input and output as device arrays, and the
CG work vectors come from a fixed array the library reserves once per GPU.

The test builds the charge matrix of a small periodic system on the host (every image within the taper radius summed
into its entry), solves it twice in a row through the C ABI (the second call sees the work array exactly as the
first call left it), and compares both results with the charges of rx_qeq_solve for the same system and with the
oracle's, within the charge tolerance of the parity tests (1e-10 e at tol 1e-12); the device's free memory is
checked before and after each call. This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from helpers import ffield_text, small_systems

pytestmark = pytest.mark.gpu

TOL = 1e-12
IMAX = 400


def _taper(swa, swb):
    d7 = (swb - swa) ** 7
    swa2, swa3, swb2, swb3 = swa * swa, swa ** 3, swb * swb, swb ** 3
    c = np.zeros(8)
    c[7] = 20.0 / d7
    c[6] = -70.0 * (swa + swb) / d7
    c[5] = 84.0 * (swa2 + 3.0 * swa * swb + swb2) / d7
    c[4] = -35.0 * (swa3 + 9.0 * swa2 * swb + 9.0 * swa * swb2 + swb3) / d7
    c[3] = 140.0 * (swa3 * swb + 3.0 * swa2 * swb2 + swa * swb3) / d7
    c[2] = -210.0 * (swa3 * swb2 + swa2 * swb3) / d7
    c[1] = 140.0 * swa3 * swb3 / d7
    c[0] = (-35.0 * swa3 * swb2 * swb2 + 21.0 * swa2 * swb3 * swb2 - 7.0 * swa * swb3 * swb3 + swb3 * swb3 * swb) / d7
    return c


def _charge_matrix_csr(s, gamma, swa=0.0, swb=10.0):
    """H_ij = sum over images of 14.4 Tap(r) / cbrt(r^3 + (gamma_i gamma_j)^-1.5), r <= swb, as CSR."""
    x, t = s["x"], s["type"]
    L = np.asarray(s["box"])
    n = len(t)
    c = _taper(swa, swb)
    g = gamma[t]
    shld = (g[:, None] * g[None, :]) ** -1.5
    H = np.zeros((n, n))
    for a in range(-2, 3):
        for b in range(-2, 3):
            for cc in range(-2, 3):
                dv = x[None, :, :] + (a * L[0] + b * L[1] + cc * L[2]) - x[:, None, :]
                r = np.sqrt((dv ** 2).sum(-1))
                m = (r <= swb) & (r > 1e-9)
                rr = np.where(m, r, 1.0)
                H += np.where(m, np.polyval(c[::-1], rr) * 14.4 / np.cbrt(rr ** 3 + shld), 0.0)
    rows, cols = np.nonzero(H)
    row_start = np.zeros(n + 1, dtype=np.int32)
    np.add.at(row_start, rows + 1, 1)
    return np.cumsum(row_start).astype(np.int32), cols.astype(np.int32), H[rows, cols]


def test_static_solve_matches_engine_solve():
    import torch
    import rxcuda
    s = small_systems()[0]
    n = len(s["type"])
    eng = rxcuda.Engine(0)
    eng.set_forcefield(ffield_text())
    eng.set_control()
    eng.set_qeq(0.0, 10.0, TOL, IMAX)
    eng.set_systems([s])
    ref = eng.qeq_solve()
    prm = eng.forcefield_params()
    eng.close()

    rs, col, val = _charge_matrix_csr(s, prm["gamma"])
    dev = torch.device("cuda", 0)
    rs_d, col_d = torch.from_numpy(rs).to(dev), torch.from_numpy(col).to(dev)
    val_d = torch.from_numpy(val).to(dev)
    eta_d = torch.from_numpy(prm["eta"][s["type"]].copy()).to(dev)
    chi_d = torch.from_numpy(prm["chi"][s["type"]].copy()).to(dev)
    q_d = torch.empty(n, dtype=torch.float64, device=dev)
    it_d = torch.zeros(2, dtype=torch.int32, device=dev)
    rel_d = torch.zeros(2, dtype=torch.float64, device=dev)
    lib = rxcuda.load()
    err = ctypes.create_string_buffer(256)
    # the one-time set-up on this device (n = 0), as a caller would make it at start-up
    assert lib.rx_qeq_solve_static(0, None, None, None, None, None, None, None, None, 0.0, 0, None, None, None, err,
                                   256) == 0, err.value.decode()
    torch.cuda.synchronize(dev)
    results = []
    free_before = []
    for _ in range(2):     # two calls in a row: the second one starts from whatever the first left in the work array
        s_d = torch.zeros(n, dtype=torch.float64, device=dev)
        t_d = torch.zeros(n, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        free_before.append(torch.cuda.mem_get_info(dev)[0])
        rc = lib.rx_qeq_solve_static(n, rs_d.data_ptr(), col_d.data_ptr(), val_d.data_ptr(), eta_d.data_ptr(),
                                     chi_d.data_ptr(), s_d.data_ptr(), t_d.data_ptr(), q_d.data_ptr(), TOL, IMAX,
                                     it_d.data_ptr(), rel_d.data_ptr(), torch.cuda.current_stream(dev).cuda_stream, err, 256)
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize(dev)
        # the call allocated nothing: the device's free memory is what it was before the call
        assert torch.cuda.mem_get_info(dev)[0] == free_before[-1]
        results.append((q_d.cpu().numpy().copy(), it_d.cpu().numpy().copy(), rel_d.cpu().numpy().copy()))
    from oracle.oracle import COracle
    orc = COracle(ffield_text(), shell=15.0).qeq(s, tol=TOL, imax=IMAX)
    for q, it, rel in results:
        assert np.abs(q - ref["q"]).max() <= 1e-10
        assert np.abs(q - orc["q"]).max() <= 1e-10
        assert abs(q.sum()) <= 1e-9
        assert rel.max() <= TOL and 0 < it.min() and it.max() < IMAX
    assert np.array_equal(results[0][0], results[1][0])


def test_static_solve_reports_breakdown():
    """A singular matrix (eta = 1, H = -1 between two atoms) makes the first step length infinite: the call reports
    iters = -1 for that right-hand side instead of a count that looks like convergence."""
    import torch
    import rxcuda
    dev = torch.device("cuda", 0)
    lib = rxcuda.load()
    rs = torch.tensor([0, 1, 2], dtype=torch.int32, device=dev)
    col = torch.tensor([1, 0], dtype=torch.int32, device=dev)
    val = torch.tensor([-1.0, -1.0], dtype=torch.float64, device=dev)
    eta = torch.ones(2, dtype=torch.float64, device=dev)
    chi = torch.ones(2, dtype=torch.float64, device=dev)
    s_d = torch.zeros(2, dtype=torch.float64, device=dev)
    t_d = torch.zeros(2, dtype=torch.float64, device=dev)
    q_d = torch.zeros(2, dtype=torch.float64, device=dev)
    it_d = torch.zeros(2, dtype=torch.int32, device=dev)
    rel_d = torch.zeros(2, dtype=torch.float64, device=dev)
    err = ctypes.create_string_buffer(256)
    rc = lib.rx_qeq_solve_static(2, rs.data_ptr(), col.data_ptr(), val.data_ptr(), eta.data_ptr(), chi.data_ptr(),
                                 s_d.data_ptr(), t_d.data_ptr(), q_d.data_ptr(), 1e-10, 50, it_d.data_ptr(),
                                 rel_d.data_ptr(), torch.cuda.current_stream(dev).cuda_stream, err, 256)
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize(dev)
    assert it_d.cpu().numpy().tolist() == [-1, -1]


def test_static_solve_rejects_too_many_atoms():
    import rxcuda
    lib = rxcuda.load()
    err = ctypes.create_string_buffer(256)
    n = 32768 + 1
    rc = lib.rx_qeq_solve_static(n, None, None, None, None, None, None, None, None, TOL, IMAX, None, None, None, err, 256)
    assert rc == 1 and b"32768" in err.value
