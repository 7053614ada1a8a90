"""dpm_pcg_solve_noalloc, the allocation-free Jacobi-PCG entry point, against the allocating
drop-in solve fvm_petsc_solve_pressure on the same singular (pure-Neumann) pressure system.

Both run the same persistent PCG kernel, so the solutions must agree to the parity tolerance
used for the other device operators (relative 1e-12), over two calls in a row: the second call
starts from a non-zero guess and reuses the scratch array the first call left behind.  Before
them, a call with max_iterations = 0 does the per-device set-up a caller without allocation
rights makes up front (module load, kernels, the static array's address); around the second
solve the device's free memory must not change, which is the point of the entry point.  The
file is named so that pytest collects it last; it also passes when run alone."""
import ctypes as C

import numpy as np
import pytest

from dopamine_b200 import solver as S

RTOL_PARITY = 1e-12
MAX_CELLS = 131072  # DPM_NOALLOC_MAX_CELLS in include/dopamine_b200.h


def neumann_system(nx, ny, nz, seed):
    """Cell-centred 7-point operator on an nx*ny*nz box with seeded positive face coefficients and
    zero-flux walls: rows sum to zero, so the constant vector spans the null space."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    idx = np.arange(n).reshape(nz, ny, nx)
    owners, neigh = [], []
    for ax in (2, 1, 0):
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax] = slice(0, -1)
        hi[ax] = slice(1, None)
        owners.append(idx[tuple(lo)].ravel())
        neigh.append(idx[tuple(hi)].ravel())
    fo = np.concatenate(owners).astype(np.int64)
    fn = np.concatenate(neigh).astype(np.int64)
    coeff = rng.uniform(0.5, 2.0, fo.size)
    diag = np.zeros(n)
    np.add.at(diag, fo, coeff)
    np.add.at(diag, fn, coeff)
    return n, fo, fn, coeff, diag


def ell_from_faces(n, fo, fn, coeff, diag):
    """Padded ELL [width][n] with ascending columns per row and (own row, 0.0) padding."""
    rows = [[(i, diag[i])] for i in range(n)]
    for o, m, c in zip(fo.tolist(), fn.tolist(), coeff.tolist()):
        rows[o].append((m, -c))
        rows[m].append((o, -c))
    width = max(len(r) for r in rows)
    col = np.tile(np.arange(n, dtype=np.int32), (width, 1))
    val = np.zeros((width, n))
    for i, r in enumerate(rows):
        r.sort()
        for s, (j, v) in enumerate(r):
            col[s, i] = j
            val[s, i] = v
    return width, col, val, 1.0 / diag


def apply(n, fo, fn, coeff, diag, x):
    y = diag * x
    np.subtract.at(y, fo, coeff * x[fn])
    np.subtract.at(y, fn, coeff * x[fo])
    return y


def reference_solve(L, n, fo, fn, coeff, diag, rhs, guess, rtol, atol, maxit):
    """The allocating drop-in solve, host in/out, no Dirichlet rows (constant null space)."""
    ip, dp = C.POINTER(C.c_int), C.POINTER(C.c_double)
    l2g = np.arange(1, n + 1, dtype=np.int32)
    f_o = (fo + 1).astype(np.int32)
    f_n = (fn + 1).astype(np.int32)
    skip = np.zeros(fo.size, dtype=np.int32)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.ascontiguousarray(guess, dtype=np.float64).copy()
    its = C.c_int(0)
    res = C.c_double(0.0)
    L.fvm_petsc_set_io_on_device(0)
    rc = L.fvm_petsc_solve_pressure(n, n, fo.size, l2g.ctypes.data_as(ip), f_o.ctypes.data_as(ip),
                                    f_n.ctypes.data_as(ip), f_n.ctypes.data_as(ip), skip.ctypes.data_as(ip),
                                    diag.ctypes.data_as(dp), b.ctypes.data_as(dp), coeff.ctypes.data_as(dp), 1,
                                    maxit, rtol, atol, None, None, 0, x.ctypes.data_as(dp), C.byref(its),
                                    C.byref(res))
    assert rc == 0, rc
    return x, its.value, res.value


def test_noalloc_rejects_oversize_without_touching_the_gpu():
    L = S.lib()
    its, res = C.c_int(-7), C.c_double(-7.0)
    rc = L.dpm_pcg_solve_noalloc(MAX_CELLS + 1, 7, None, None, None, None, None, 1e-8, 0.0, 10, 1, None,
                                 C.byref(its), C.byref(res))
    assert rc == -1 and its.value == -7
    rc = L.dpm_pcg_solve_noalloc(64, 17, None, None, None, None, None, 1e-8, 0.0, 10, 1, None, C.byref(its),
                                 C.byref(res))
    assert rc == -1


@pytest.mark.gpu
def test_noalloc_matches_allocating_solve_on_two_calls():
    import torch

    L = S.lib()
    dev = torch.device("cuda:0")
    n, fo, fn, coeff, diag = neumann_system(44, 40, 36, seed=11)
    assert n <= MAX_CELLS
    width, col, val, dinv = ell_from_faces(n, fo, fn, coeff, diag)
    assert width == 7
    d_col = torch.from_numpy(col.ravel().copy()).to(dev)
    d_val = torch.from_numpy(val.ravel().copy()).to(dev)
    d_dinv = torch.from_numpy(dinv).to(dev)
    rtol, atol, maxit = 1e-10, 1e-50, 2000
    # per-device set-up call: no array argument is read
    its0, res0 = C.c_int(-1), C.c_double(-1.0)
    rc = L.dpm_pcg_solve_noalloc(n, width, None, None, None, None, None, rtol, atol, 0, 1, None, C.byref(its0),
                                 C.byref(res0))
    assert rc == 0 and its0.value == 0 and res0.value == 0.0
    rng = np.random.default_rng(5)
    guesses = [np.zeros(n), rng.standard_normal(n)]
    for call in range(2):
        rhs = rng.standard_normal(n) + 0.3  # non-zero mean: the null-space projection is exercised
        x_ref, its_ref, res_ref = reference_solve(L, n, fo, fn, coeff, diag, rhs, guesses[call], rtol, atol, maxit)
        d_rhs = torch.from_numpy(rhs).to(dev)
        d_x = torch.from_numpy(guesses[call].copy()).to(dev)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        its, res = C.c_int(0), C.c_double(0.0)
        rc = L.dpm_pcg_solve_noalloc(n, width, d_col.data_ptr(), d_val.data_ptr(), d_dinv.data_ptr(),
                                     d_rhs.data_ptr(), d_x.data_ptr(), rtol, atol, maxit, 1,
                                     torch.cuda.current_stream().cuda_stream, C.byref(its), C.byref(res))
        assert rc == 0, (call, rc)
        torch.cuda.synchronize()
        if call == 1:  # set-up done long before: the solve itself takes no device memory
            assert torch.cuda.mem_get_info(dev)[0] == free_before
        x = d_x.cpu().numpy()
        err = np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref)
        assert err <= RTOL_PARITY, (call, err)
        assert its.value == its_ref and 0 < its.value < maxit, (call, its.value, its_ref)
        assert abs(res.value - res_ref) <= RTOL_PARITY * max(res_ref, 1e-300) + 1e-300, (call, res.value, res_ref)
        # and it is a solution: the projected right-hand side is met to the requested tolerance
        bp = rhs - rhs.mean()
        true_res = np.linalg.norm(bp - apply(n, fo, fn, coeff, diag, x))
        assert true_res <= 10 * rtol * np.linalg.norm(bp), (call, true_res)
