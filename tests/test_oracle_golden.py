"""The oracle against the reference's own regression statistics (golden vectors).

tests/golden/<case>_np1.csv are the reference's tests/regression/reference CSVs (made by the
gfortran CPU build), reduced to the compared columns by tests/golden/make_golden.py.  The check is
the reference's own (tests/regression/compare_stats.py): integral quantities within rtol 1e-6,
face-flux divergence below 1e-9; the dissipation and the cell-velocity divergence columns are held
to the same 1e-6.

Coverage: KEP / CDS / QUICK momentum advection, skewed and graded meshes, non-orthogonal
correctors, outlets and walls (tgv*, pdrop, hydro*); Vreman and AMD with the log-law wall model
and its filter (channel, amd, graded); temperature transport with van Leer TVD, fixed-temperature
walls and Boussinesq buoyancy (rb); the MOST surface layer with its heat flux into a
transported, buoyant temperature (channel_most); inlet, outlet and the synthetic-eddy inflow at an
ABL inlet, divergence-free (inflow) and Jarrin (inflow_jarrin) eddies.  The graded wall boxes are the reference's RB.geo meshes,
rebuilt with the closed-form "Bump" node distribution (dopamine_b200.cases.bump_nodes).
"""
import csv
import os

import pytest

from dopamine_b200 import cases
from oracle.oracle import Oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
RTOL, ATOL, DIV_MAX = 1.0e-6, 1.0e-12, 1.0e-9
COMPARED = ("time", "E", "Umax", "Ub", "tauw_mean", "nu_sgs_mean")
EXTRA = ("eps", "max_abs_divU_cell", "volavg_abs_divU_cell")


def load(case):
    with open(os.path.join(GOLDEN, f"{case}_np1.csv"), newline="") as fh:
        return {int(r["step"]): {k: float(v) for k, v in r.items() if k != "step"} for r in csv.DictReader(fh)}


def run_case(name, steps=None):
    case = cases.regression_case(name)
    o = Oracle(case)
    o.initialise()
    ref = load(name)
    last = max(ref) if steps is None else steps
    out = {}
    for step in range(1, last + 1):
        o.advance()
        if step in ref:
            out[step] = o.stats()
    return ref, out


@pytest.mark.parametrize("name", ["tgv_skew", "tgv_skew_chk", "pdrop", "hydro", "hydrowall", "tgv", "rb", "channel",
                                  "amd", "graded", "channel_most", "duct", "inflow", "inflow_jarrin"])
def test_oracle_matches_reference_csv(name):
    ref, got = run_case(name)
    for step, s in got.items():
        r = ref[step]
        for col in COMPARED:
            a, b = r[col], s[col]
            err = abs(a - b) / max(abs(a), ATOL / RTOL)
            assert err <= RTOL, f"{name} step {step} {col}: ref={a:.12e} oracle={b:.12e} rel={err:.2e}"
        assert s["max_abs_divU"] <= DIV_MAX, f"{name} step {step} divU {s['max_abs_divU']:.3e}"
        # beyond the reference's own comparison: the dissipation and the cell-velocity divergence
        for col in EXTRA:
            a, b = r[col], s[col]
            err = abs(a - b) / max(abs(a), ATOL / RTOL)
            assert err <= RTOL, f"{name} step {step} {col}: ref={a:.12e} oracle={b:.12e} rel={err:.2e}"


def test_oracle_dt_clamp_matches_reference():
    """tgv_skew requests dt=0.02 but the CFL clamp (solver_advance) shortens every step."""
    ref, got = run_case("tgv_skew", steps=3)
    t_prev = 0.0
    for step in (1, 2, 3):
        dt = ref[step]["time"] - t_prev
        t_prev = ref[step]["time"]
        assert dt < 0.02
        assert abs(got[step]["dt_used"] - dt) <= 1e-8 * dt + 1e-12
