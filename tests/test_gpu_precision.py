"""The precision form (form = DPM_FORM_MIXED) with its FP32 explicit half - first gradient pass,
SGS, momentum flux assembly and scalar fluxes in FP32, FP64 state, projection and wall-model
Newton solve - against the FP64 oracle, on the configurations the north star names for it:

* the mixed-element box (hexes, prisms, pyramids, jittered vertices) with AMD SGS and Koren TVD
  momentum, the unstructured precision-form configuration;
* the reduced urban canopy (obstacles, MOST with per-patch roughness, AMD, KEP, van Leer
  temperature and tracer), the metric's configuration.

The chosen-form gates: each field within 1e-5 relative of the FP64 oracle and the divergence
below 1e-8.  Each field's error is printed.  The FP64 path is unchanged by this form (the same
handle without it is pinned to 1e-10 by the other parity tests)."""
import numpy as np
import pytest

from dopamine_b200 import abi, cases
from dopamine_b200.solver import DopamineError, Solver
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-5
DIV_TOL = 1e-8


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-3 * np.sqrt(b.size)))


def _run(case, steps, psolver, p_tol):
    po = case.make_params()
    po.p_tol = p_tol
    pg = case.make_params()
    pg.p_tol = p_tol
    pg.p_solver = psolver
    pg.form = abi.FORM_MIXED
    o = O.Oracle(case, params=po)
    s = Solver(case, params=pg)
    o.initialise()
    s.initialise()
    for _ in range(steps):
        o.advance()
        s.advance()
    return o, s


@pytest.mark.parametrize("psolver", [abi.PSOLVER_TWOLEVEL_FCG, abi.PSOLVER_MULTILEVEL_FCG])
def test_precision_form_mixed_element_box_koren(psolver):
    case = cases.hybrid_config(n=16, kind="mixed", n_steps=10)
    assert case.params["scheme"] == abi.SCHEME_KOREN_TVD and case.params["sgs_model"] == abi.SGS_AMD
    o, s = _run(case, 10, psolver, 1e-13)
    so, sg = o.state(), s.sync_host()
    errs = {"U": _rel(sg["U"], so["U"]), "nu_sgs": _rel(sg["nu_sgs"], so["nu_sgs"])}
    st = s.stats()
    print(f"precision form, mixed-element box, 10 steps, p_solver {psolver}: "
          + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()) + f", divU {st['max_abs_divU']:.2e}")
    for k, v in errs.items():
        assert v <= FIELD_TOL, (k, v)
    assert st["max_abs_divU"] <= DIV_TOL


def test_precision_form_urban_reduced():
    case = cases.urban_config(nx=24, ny=24, nz=12, n_blocks=4, lx=2.4, ly=2.4, lz=0.72, n_steps=5, scale=0.01)
    o, s = _run(case, 5, abi.PSOLVER_MULTILEVEL_FCG, 1e-13)
    so, sg = o.state(), s.sync_host()
    To, Co = o.scalars()
    Tg, Cg = s.scalars()
    errs = {"U": _rel(sg["U"], so["U"]), "T": _rel(Tg, To), "C": _rel(Cg, Co), "nu_sgs": _rel(sg["nu_sgs"], so["nu_sgs"])}
    info = _rel(Tg - 300.0, To - 300.0)
    st = s.stats()
    print("precision form, reduced urban, 5 steps: " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items())
          + f", T-T_ref {info:.2e}, divU {st['max_abs_divU']:.2e}")
    for k, v in errs.items():
        assert v <= FIELD_TOL, (k, v)
    assert st["max_abs_divU"] <= DIV_TOL


def test_precision_form_rejects_quick():
    case = cases.regression_case("tgv")  # QUICK momentum
    assert case.params["scheme"] == abi.SCHEME_QUICK
    p = case.make_params()
    p.p_solver = abi.PSOLVER_TWOLEVEL_FCG
    p.form = abi.FORM_MIXED
    with pytest.raises(DopamineError) as err:
        Solver(case, params=p)
    assert err.value.status == abi.ERR_UNSUPPORTED
