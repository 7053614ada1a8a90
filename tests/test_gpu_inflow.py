"""ABL inflow on the device (sem.cuh, the BC_ABL_INLET boundary): the synthetic-eddy method with
divergence-free and Jarrin eddies against the oracle, whose restatement tests/test_oracle_golden.py
pins to the reference's inflow and inflow_jarrin CSVs.

* 5 steps of each case: U within 1e-10 relative of the oracle.
* 20 steps against the reference's CSV under its own comparison (rtol 1e-6, divergence 1e-9): the
  eddies' random sequence is the reference's.
* A checkpoint carries the eddies (positions, signs, generator state): a restarted handle takes
  the next steps as the uninterrupted one does, up to the outlet's rebuilt boundary values.
"""
import numpy as np
import pytest

from dopamine_b200 import cases
from dopamine_b200.solver import Solver
from oracle import oracle as O
from tests.test_oracle_golden import COMPARED, load

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["inflow", "inflow_jarrin"])
def test_inflow_steps_match_oracle(name):
    case = cases.regression_case(name)
    o = O.Oracle(case)
    s = Solver(case)
    o.initialise()
    s.initialise()
    for _ in range(5):
        o.advance()
        s.advance()
    Uo, Ug = o.state()["U"], s.sync_host()["U"]
    e = float(np.linalg.norm(Ug - Uo) / np.linalg.norm(Uo))
    print(f"{name}: 5 steps, U rel {e:.2e}")
    assert e <= 1e-10
    s.close()


@pytest.mark.parametrize("name", ["inflow", "inflow_jarrin"])
def test_inflow_against_reference_csv(name):
    ref = load(name)
    s = Solver(cases.regression_case(name))
    s.initialise()
    worst = 0.0
    for step in range(1, max(ref) + 1):
        s.advance()
        if step in ref:
            st, r = s.stats(), ref[step]
            for col in COMPARED:
                e = abs(st[col] - r[col]) / max(abs(r[col]), 1e-6)
                worst = max(worst, e)
                assert e <= 1e-6, (step, col, st[col], r[col])
            assert st["max_abs_divU"] <= 1e-9
    print(f"{name}: worst rel {worst:.2e} over {len(ref)} rows")
    s.close()


def test_checkpoint_carries_the_eddies(tmp_path):
    case = cases.regression_case("inflow")
    a = Solver(case)
    a.initialise()
    for _ in range(4):
        a.advance()
    a.write_checkpoint(str(tmp_path), 4)
    for _ in range(3):
        a.advance()
    b = Solver(case)
    b.read_checkpoint(str(tmp_path))
    for _ in range(3):
        b.advance()
    ua, ub = a.sync_host()["U"], b.sync_host()["U"]
    e = float(np.linalg.norm(ub - ua) / np.linalg.norm(ua))
    print(f"inflow restart after 4 steps, 3 more: U rel {e:.2e}")
    # the restored eddies give the inlet the fluctuation the uninterrupted run had; the outlet's
    # extrapolated boundary velocity is rebuilt from the restored fields and fresh gradients, as the
    # reference's solver_refresh_after_restart rebuilds it (mod_fv_solver.f90:601-609), which moves
    # the continuation by O(h^2) there (the wall-bounded restarts in test_gpu_output.py, with no
    # outlet, continue to round-off)
    assert e <= 1e-4
    a.close()
    b.close()
