"""GPU parity of the multilevel flexible-CG pressure solve (p_solver = DPM_PSOLVER_MULTILEVEL_FCG:
FP64 FCG preconditioned by an FP32 aggregation-multigrid V-cycle).

The preconditioner changes the Krylov path, not the system: at a tight Poisson tolerance the whole
step must agree with the FP64 oracle (which runs the reference's Jacobi-PCG) to 1e-8 on the
velocity, with divergence <= 1e-8; at the default tolerance the chosen-form gates (field error <=
1e-5, divergence <= 1e-8) hold.  On the channel operator it needs several times fewer iterations
than the two-level form."""
import numpy as np
import pytest

from dopamine_b200 import abi, cases
from dopamine_b200.solver import Solver
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-8
DIV_TOL = 1e-8


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-3 * np.sqrt(b.size))


def _case(name, steps):
    if name == "channel":
        return cases.channel_config(nx=16, ny=12, nz=8, n_steps=steps)
    if name in ("tet", "mixed"):
        return cases.hybrid_config(n=8, kind=name, n_steps=steps)
    return cases.regression_case(name)


@pytest.mark.parametrize("name,steps", [("tgv_skew", 4), ("pdrop", 4), ("hydrowall", 3), ("channel", 4),
                                        ("tet", 3), ("mixed", 3)])
def test_mlcg_step_parity(name, steps):
    case = _case(name, steps)
    po = case.make_params()
    po.p_tol = 1e-13
    pg = case.make_params()
    pg.p_tol = 1e-13
    pg.p_solver = abi.PSOLVER_MULTILEVEL_FCG
    o = O.Oracle(case, params=po)
    s = Solver(case, params=pg)
    o.initialise()
    s.initialise()
    for k in range(steps):
        o.advance()
        s.advance()
        so, sg = o.state(), s.sync_host()
        assert _rel(sg["U"], so["U"]) <= FIELD_TOL, (name, k, _rel(sg["U"], so["U"]))
    st = s.stats()
    assert st["max_abs_divU"] <= DIV_TOL, st["max_abs_divU"]
    assert st["p_solves"] > 0 and st["p_iters"] > 0 and st["p_fallbacks"] == 0


@pytest.mark.parametrize("name,steps", [("tgv_skew", 3), ("channel", 3)])
def test_mlcg_default_tolerance_against_fp64_oracle(name, steps):
    case = _case(name, steps)
    pg = case.make_params()
    pg.p_solver = abi.PSOLVER_MULTILEVEL_FCG
    o = O.Oracle(case)
    s = Solver(case, params=pg)
    o.initialise()
    s.initialise()
    for _ in range(steps):
        o.advance()
        s.advance()
    so, sg = o.state(), s.sync_host()
    eu = _rel(sg["U"], so["U"])
    ep = np.linalg.norm((sg["p"] - sg["p"].mean()) - (so["p"] - so["p"].mean())) / max(np.linalg.norm(so["p"]), 1e-30)
    st = s.stats()
    print(f"multilevel {name}: U rel {eu:.2e}, p rel {ep:.2e}, divU {st['max_abs_divU']:.2e}")
    assert eu <= 1e-5 and ep <= 1e-5
    assert st["max_abs_divU"] <= DIV_TOL


def test_mlcg_iterations_on_the_channel():
    """Same channel, same p_tol (1e-10): the multilevel form needs at most a third of the two-level
    form's iterations and at most a tenth of Jacobi-PCG's, with a divergence of the same order."""
    case = cases.channel_config(nx=48, ny=32, nz=32, n_steps=2)
    its, div = {}, {}
    for form in (abi.PSOLVER_JACOBI_PCG, abi.PSOLVER_TWOLEVEL_FCG, abi.PSOLVER_MULTILEVEL_FCG):
        p = case.make_params()
        p.p_solver = form
        s = Solver(case, params=p)
        s.initialise()
        s.advance()
        s.advance()
        st = s.stats()
        its[form] = st["p_iters"] / max(st["p_solves"], 1)
        div[form] = st["max_abs_divU"]
        s.close()
    print("iterations per solve", its)
    assert its[abi.PSOLVER_MULTILEVEL_FCG] * 3 <= its[abi.PSOLVER_TWOLEVEL_FCG], its
    assert its[abi.PSOLVER_MULTILEVEL_FCG] * 10 <= its[abi.PSOLVER_JACOBI_PCG], its
    assert div[abi.PSOLVER_MULTILEVEL_FCG] <= 10 * div[abi.PSOLVER_JACOBI_PCG] + 1e-12, div


def test_dropin_boomeramg_name_selects_the_multilevel_solve():
    """The drop-in pressure ABI: after fvm_petsc_set_pressure_solver("boomeramg") (what the
    reference's Fortran caller selects, src/solver/mod_pressure_solver.f90:136) the solve runs the
    multilevel form; it reaches the same solution as the Jacobi-PCG selection in far fewer
    iterations.  The selection is put back to Jacobi and the backend finalised afterwards."""
    from test_zz_no_alloc import neumann_system, reference_solve
    from dopamine_b200 import solver as S

    L = S.lib()
    n, fo, fn, coeff, diag = neumann_system(40, 36, 32, seed=12)
    rhs = np.random.default_rng(8).standard_normal(n) + 0.3
    try:
        L.fvm_petsc_set_pressure_solver(b"jacobi")
        x_j, its_j, _ = reference_solve(L, n, fo, fn, coeff, diag, rhs, np.zeros(n), 1e-10, 1e-50, 4000)
        L.fvm_petsc_set_pressure_solver(b"boomeramg")
        x_m, its_m, res_m = reference_solve(L, n, fo, fn, coeff, diag, rhs, np.zeros(n), 1e-10, 1e-50, 4000)
    finally:
        # the backend caches its operator by size, as the reference's does: drop it for later users
        L.fvm_petsc_set_pressure_solver(b"jacobi")
        L.fvm_petsc_backend_finalize()
    rel = np.linalg.norm((x_m - x_m.mean()) - (x_j - x_j.mean())) / np.linalg.norm(x_j - x_j.mean())
    print(f"drop-in: jacobi {its_j} its, multilevel {its_m} its, solution rel diff {rel:.2e}")
    assert rel <= 1e-6, rel  # both stop at ||r|| <= 1e-10 ||b'||; the operator's condition number is ~1e4
    assert 0 < its_m * 5 <= its_j, (its_m, its_j)
    from test_zz_no_alloc import apply
    bp = rhs - rhs.mean()
    assert np.linalg.norm(bp - apply(n, fo, fn, coeff, diag, x_m)) <= 10 * 1e-10 * np.linalg.norm(bp)


def test_auto_picks_the_form_that_fits():
    """p_solver = DPM_PSOLVER_AUTO takes the two-level form while the mesh has at most 4096 cells
    per SM and the multilevel form beyond; the stats report the form in use."""
    small = cases.channel_config(nx=16, ny=12, nz=8, n_steps=1)
    p = small.make_params()
    p.p_solver = abi.PSOLVER_AUTO
    s = Solver(small, params=p)
    s.initialise()
    s.advance()
    assert s.stats()["p_solver_used"] == abi.PSOLVER_TWOLEVEL_FCG
    s.close()
    big = cases.channel_config(nx=128, ny=96, nz=64, n_steps=1)  # 786 432 cells: > 4096 per SM
    div = {}
    for form in (abi.PSOLVER_AUTO, abi.PSOLVER_JACOBI_PCG):
        p = big.make_params()
        p.p_solver = form
        s = Solver(big, params=p)
        s.initialise()
        s.advance()
        st = s.stats()
        div[form] = st["max_abs_divU"]
        if form == abi.PSOLVER_AUTO:
            assert st["p_solver_used"] == abi.PSOLVER_MULTILEVEL_FCG
        s.close()
    # same relative stopping rule: the divergence left is of the plain form's order
    assert div[abi.PSOLVER_AUTO] <= 10 * div[abi.PSOLVER_JACOBI_PCG] + 1e-12, div


@pytest.mark.parametrize("bits", [32, 16])
def test_mlcg_multi_kernel_form_matches_plain_pcg(bits):
    """A mesh of 2^20 cells, large enough that the multilevel solve runs as standalone kernels
    (mlkern.cuh) instead of the persistent one: with the smoother's scaled off-diagonals in FP32
    and in binary16, against the plain FP64 Jacobi-PCG path (which the parity tests pin to the
    oracle) at a tight tolerance, with the same iteration count as the persistent form on a
    smaller copy of the operator family."""
    case = cases.channel_config(nx=128, ny=128, nz=64, n_steps=2)
    ref = None
    for form in (abi.PSOLVER_JACOBI_PCG, abi.PSOLVER_MULTILEVEL_FCG):
        p = case.make_params()
        p.p_tol = 1e-13
        p.p_solver = form
        p.p_ml_value_bits = bits
        s = Solver(case, params=p)
        s.initialise()
        s.advance()
        s.advance()
        U = s.sync_host()["U"]
        st = s.stats()
        s.close()
        if ref is None:
            ref = U
            continue
        err = np.linalg.norm(U - ref) / np.linalg.norm(ref)
        its = st["p_iters"] / st["p_solves"]
        print(f"multi-kernel multilevel ({bits}-bit smoother), 1.05M cells: U rel {err:.2e}, {its:.1f} its/solve")
        assert err <= 1e-9, err
        assert st["max_abs_divU"] <= 1e-8
        assert st["p_fallbacks"] == 0
        assert its <= 60, its
