"""Failure paths of the pressure solve, exercised without faulting or hanging the GPU.

* A grid-wide wait that runs out: the handle's poll limit is set to one poll
  (dpm_set_barrier_spin_limit), so the first wait of the Krylov kernel gives up; every block
  returns, the call reports DPM_ERR_BARRIER_TIMEOUT, and after the default limit is restored the
  same handle steps on and matches a fresh handle.
* The flexible-CG stall guard: a one-iteration window that asks for a 1e6-fold residual drop makes
  the guard fire, the solve is handed to plain Jacobi-PCG from the current iterate (the automatic
  fallback), and the step still matches the FP64 oracle.
* The drop-in solve (fvm_petsc_solve_pressure): non-finite right-hand-side entries are zeroed as
  the reference's caller scrubs them (src/solver/mod_pressure_solver.f90:721-727), and a solve that
  cannot converge within the forced cap, even after the retry, returns -(1000 + reason) as
  src/solver/pressure_backend_petsc.c:878-961 does.
"""
import ctypes as C

import numpy as np
import pytest

from dopamine_b200 import abi, cases
from dopamine_b200.solver import DopamineError, Solver, lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-3 * np.sqrt(b.size))


@pytest.mark.parametrize("form", [abi.PSOLVER_JACOBI_PCG, abi.PSOLVER_TWOLEVEL_FCG, abi.PSOLVER_MULTILEVEL_FCG])
def test_barrier_timeout_is_reported_and_the_handle_recovers(form):
    case = cases.tgv_config(n=32, n_steps=2)  # 32 k cells: every form launches dozens of blocks
    p = case.make_params()
    p.p_solver = form
    s = Solver(case, params=p)
    s.initialise()
    s.set_barrier_spin_limit(1)
    with pytest.raises(DopamineError) as err:
        s.advance()
    assert err.value.status == abi.ERR_BARRIER_TIMEOUT
    # default limit again: restart from the initial state and compare with a fresh handle
    s.set_barrier_spin_limit(0)
    lib().dpm_set_time(s.h, 0.0)
    s.initialise()
    ref = Solver(case, params=p)
    ref.initialise()
    for _ in range(2):
        s.advance()
        ref.advance()
    assert _rel(s.sync_host()["U"], ref.sync_host()["U"]) <= 1e-12
    assert s.stats()["max_abs_divU"] <= 1e-9
    s.close()
    ref.close()


@pytest.mark.parametrize("form", [abi.PSOLVER_TWOLEVEL_FCG, abi.PSOLVER_MULTILEVEL_FCG])
def test_stall_guard_hands_the_solve_to_plain_pcg(form):
    case = cases.channel_config(nx=16, ny=12, nz=8, n_steps=3)
    po = case.make_params()
    po.p_tol = 1e-13
    pg = case.make_params()
    pg.p_tol = 1e-13
    pg.p_solver = form
    pg.p_stall_window = 1
    pg.p_stall_ratio = 1e-6
    o = O.Oracle(case, params=po)
    s = Solver(case, params=pg)
    o.initialise()
    s.initialise()
    for _ in range(3):
        o.advance()
        s.advance()
    st = s.stats()
    assert st["p_fallbacks"] > 0, st
    assert _rel(s.sync_host()["U"], o.state()["U"]) <= 1e-8
    assert st["max_abs_divU"] <= 1e-8


def _neumann_faces(n1, seed):
    rng = np.random.default_rng(seed)
    n = n1 ** 3
    idx = np.arange(n).reshape(n1, n1, n1)
    fo, fn = [], []
    for ax in range(3):
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax] = slice(0, -1)
        hi[ax] = slice(1, None)
        fo.append(idx[tuple(lo)].ravel())
        fn.append(idx[tuple(hi)].ravel())
    fo = np.concatenate(fo)
    fn = np.concatenate(fn)
    coeff = rng.uniform(0.5, 2.0, fo.size)
    diag = np.zeros(n)
    np.add.at(diag, fo, coeff)
    np.add.at(diag, fn, coeff)
    return n, fo, fn, coeff, diag


def _drop_in_solve(n, fo, fn, coeff, diag, rhs, rtol=1e-10, atol=1e-50, maxit=1000):
    L = lib()
    ip, dp = C.POINTER(C.c_int), C.POINTER(C.c_double)
    l2g = np.arange(1, n + 1, dtype=np.int32)
    f_o = (fo + 1).astype(np.int32)
    f_n = (fn + 1).astype(np.int32)
    skip = np.zeros(fo.size, dtype=np.int32)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.zeros(n)
    its, res = C.c_int(0), C.c_double(0.0)
    L.fvm_petsc_set_io_on_device(0)
    rc = L.fvm_petsc_solve_pressure(n, n, fo.size, l2g.ctypes.data_as(ip), f_o.ctypes.data_as(ip),
                                    f_n.ctypes.data_as(ip), f_n.ctypes.data_as(ip), skip.ctypes.data_as(ip),
                                    diag.ctypes.data_as(dp), b.ctypes.data_as(dp), coeff.ctypes.data_as(dp), 1, maxit,
                                    rtol, atol, None, None, 0, x.ctypes.data_as(dp), C.byref(its), C.byref(res))
    return rc, x, its.value, res.value


def test_drop_in_zeroes_non_finite_rhs_entries():
    n, fo, fn, coeff, diag = _neumann_faces(20, seed=3)
    rng = np.random.default_rng(4)
    rhs = rng.standard_normal(n)
    bad = rng.choice(n, 7, replace=False)
    clean = rhs.copy()
    clean[bad] = 0.0
    dirty = rhs.copy()
    dirty[bad[:3]] = np.nan
    dirty[bad[3:5]] = np.inf
    dirty[bad[5:]] = -np.inf
    rc0, x0, its0, _ = _drop_in_solve(n, fo, fn, coeff, diag, clean)
    rc1, x1, its1, _ = _drop_in_solve(n, fo, fn, coeff, diag, dirty)
    assert rc0 == 0 and rc1 == 0
    assert np.all(np.isfinite(x1))
    assert its0 == its1
    np.testing.assert_array_equal(x0, x1)


def test_drop_in_reports_krylov_failure_after_the_retry():
    L = lib()
    n, fo, fn, coeff, diag = _neumann_faces(24, seed=5)
    rhs = np.random.default_rng(6).standard_normal(n)
    L.fvm_petsc_insert_option(b"-ksp_max_it 3")
    try:
        rc, x, its, res = _drop_in_solve(n, fo, fn, coeff, diag, rhs)
    finally:
        L.fvm_petsc_insert_option(b"-ksp_max_it 0")  # back to the default cap
    # cap 3, retry from zero with 12 iterations: still far from 1e-10, KSP_DIVERGED_ITS = -3
    assert rc == -(1000 - 3), rc
    assert its == 12 and res > 1e-6
    # the default cap converges on the same system
    rc2, _, its2, _ = _drop_in_solve(n, fo, fn, coeff, diag, rhs)
    assert rc2 == 0 and 12 < its2 < 1000
