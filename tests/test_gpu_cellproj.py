"""The exact cell projection on the GPU (cellproj.cuh) against the oracle.

* The operators B u and V^-1 B^T chi through the C ABI (dpm_cell_divergence,
  dpm_cell_adjoint_gradient) on meshes with interior, periodic, inlet, outlet and wall faces: 1e-12
  relative, the per-operator gate.
* The projection itself (dpm_cell_project) with the identity preconditioner and with the
  pressure-solve preconditioner: same iteration count as the oracle, velocity to 1e-10.
* Whole steps with cell_projection = EXACT (the reference's default) on the 45-degree skewed
  Taylor-Green box and on the inlet/outlet duct: the same outer iteration counts and divergence
  below 1e-9; velocity to 1e-9 relative of the oracle when every preconditioning solve took the
  oracle's iteration count.  A preconditioning solve stops at rtol 0.05, and FP64 sums taken in
  another order can move that stop by an iteration (the duct: 526 against 524 of 22 solves over
  3 steps), which moves the inexact projection (energy tolerance 0.1) by a few 1e-6: then the
  gate is 1e-5 and the counts must agree within 1 %.
* The hydrostatic column (hydro_exact), whose velocity is a start-up remainder that rounding
  differences move by about 1 % (two oracle runs with different thread counts already differ so),
  is held to what the case states: the fluid stays at rest near the reference's start-up value.
"""
import numpy as np
import pytest

from dopamine_b200 import abi, cases
from dopamine_b200.solver import Solver
from oracle import oracle as O
from tests.test_cell_projection import _adj, _div, _project, _unit_test_inputs, _walled_skewed_box

pytestmark = pytest.mark.gpu

MESHES = {
    "walled_box": _walled_skewed_box,
    "skewed_periodic": lambda: cases.regression_case("tgv_skew_exact"),
    "duct": lambda: cases.regression_case("duct_exact"),
}


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", sorted(MESHES))
def test_projection_operators_match_oracle(name):
    case = MESHES[name]()
    o = O.Oracle(case)
    s = Solver(case)
    u, chi = _unit_test_inputs(o.nc)
    assert _rel(s.cell_divergence(u), _div(o, u)) <= 1e-12
    assert _rel(s.cell_adjoint_gradient(chi), _adj(o, chi)) <= 1e-12
    s.close()


@pytest.mark.parametrize("identity", [True, False])
@pytest.mark.parametrize("name", ["walled_box", "duct"])
def test_projection_matches_oracle(name, identity):
    case = MESHES[name]()
    o = O.Oracle(case)
    s = Solver(case)
    rng = np.random.default_rng(11)
    u = rng.standard_normal((o.nc, 3))
    bconst = np.zeros(o.nc)
    if name == "duct":
        bconst[rng.choice(o.nc, 16, replace=False)] = 1e-3 * rng.standard_normal(16)
    tol, max_it = (1e-6, 400) if identity else (0.1, 100)
    want, n_o = _project(o, u, bconst, tol, max_it, identity)
    got, n_g = s.cell_project(u, bconst, tol, max_it, identity_precond=identity)
    print(f"{name} identity={identity}: iterations oracle {n_o} GPU {n_g}, rel {_rel(got, want):.2e}")
    assert n_g == n_o
    assert _rel(got, want) <= 1e-10
    s.close()


@pytest.mark.parametrize("name,steps", [("tgv_skew_exact", 5), ("duct_exact", 3)])
def test_exact_projection_steps_match_oracle(name, steps):
    case = cases.regression_case(name)
    assert case.make_params().cell_projection == abi.CELL_PROJECTION_EXACT
    o = O.Oracle(case)
    s = Solver(case)
    o.initialise()
    s.initialise()
    same = True
    for k in range(steps):
        o.advance()
        s.advance()
        so, sg = o.stats(), s.stats()
        assert sg["cp_iters"] == so["cp_iters"], (k, sg["cp_iters"], so["cp_iters"])
        assert abs(sg["cp_precond_iters"] - so["cp_precond_iters"]) <= 0.01 * so["cp_precond_iters"]
        same = same and sg["cp_precond_iters"] == so["cp_precond_iters"]
    Uo, Ug = o.state()["U"], s.sync_host()["U"]
    err = float(np.linalg.norm(Ug - Uo) / max(np.linalg.norm(Uo), 1e-300))
    st = s.stats()
    print(f"{name} {steps} steps: U rel {err:.2e}, cp {st['cp_iters']}/{st['cp_precond_iters']} "
          f"(oracle {so['cp_precond_iters']}), divU {st['max_abs_divU']:.2e}")
    assert err <= (1e-9 if same else 1e-5)
    assert st["max_abs_divU"] <= 1e-9
    s.close()


def test_hydrostatic_column_stays_at_rest():
    from tests.test_oracle_golden import load
    ref = load("hydro_exact")
    s = Solver(cases.regression_case("hydro_exact"))
    s.initialise()
    for step in range(1, max(ref) + 1):
        s.advance()
        if step in ref:
            st, r = s.stats(), ref[step]
            assert 0.8 * r["Umax"] <= st["Umax"] <= 1.2 * r["Umax"], (step, st["Umax"], r["Umax"])
            assert st["max_abs_divU"] <= 1e-9
    s.close()
