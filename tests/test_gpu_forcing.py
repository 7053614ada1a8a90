"""Body forces, nudging and scalar sources on the device (forcing.cuh, the Coriolis term in the
momentum kernels) against the oracle, whose restatement tests/test_forcing_oracle.py pins to
closed forms:

* the closed-form box cases themselves on the GPU;
* whole steps of flows where these terms interact with transport, walls and the projection:
  the wall-modelled channel with rotation, harmonic forcing and the mass-flux force; Rayleigh-
  Benard with Davies nudging of U and T; the MOST channel with sphere, box, line and tag-point
  scalar sources, one harmonic.  U, T and C within 1e-10 relative of the oracle after 5 steps.
"""
import numpy as np
import pytest

from dopamine_b200 import abi, cases
from dopamine_b200.solver import DopamineError, Solver
from oracle import oracle as O
from tests import test_forcing_oracle as F

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-3 * np.sqrt(b.size)))


def test_closed_form_box_cases_on_the_device():
    # Coriolis: RK3 cubic of the rotation
    om, dt, steps = 0.7, 0.05, 5
    case = F._box(use_rotation=1, omega_rot=(0.0, 0.0, om), dt=dt)
    s = Solver(case)
    s.to_device(U=np.tile([1.0, 0.0, 0.0], (s.nc, 1)), p=np.zeros(s.nc))
    for _ in range(steps):
        s.advance()
    f = 2.0 * om
    M = np.array([[0.0, f], [-f, 0.0]]) * dt
    R = np.eye(2) + M + M @ M / 2.0 + M @ M @ M / 6.0
    uv = np.linalg.matrix_power(R, steps) @ np.array([1.0, 0.0])
    U = s.sync_host()["U"]
    assert np.abs(U[:, :2] - uv).max() <= 1e-13
    s.close()
    # mass-flux force: the target in one step
    case = F._box(constant_mass_flux_forcing=1, U_bulk_target=(1.0, 0.0, -0.25), dt=0.02)
    s = Solver(case)
    s.to_device(U=np.tile([0.5, 0.1, 0.0], (s.nc, 1)), p=np.zeros(s.nc))
    s.advance()
    assert np.abs(s.sync_host()["U"] - [1.0, 0.0, -0.25]).max() <= 1e-13
    s.close()


def _pair(case, steps, setup=None):
    o = O.Oracle(case)
    s = Solver(case)
    if setup:
        setup(o)
        setup(s)
    o.initialise()
    s.initialise()
    for _ in range(steps):
        o.advance()
        s.advance()
    return o, s


def test_channel_with_rotation_harmonic_and_mass_flux_forcing():
    case = cases.regression_case("channel")
    case.params.update(use_rotation=1, omega_rot=(0.05, 0.0, 0.3), use_harmonic_forcing=1, forcing_amp=0.4,
                       forcing_omega=5.0, forcing_phase=0.2, forcing_dir=(0.0, 1.0, 0.0),
                       constant_mass_flux_forcing=1, U_bulk_target=(0.9, 0.0, 0.0))
    o, s = _pair(case, 5)
    e = _rel(s.sync_host()["U"], o.state()["U"])
    print(f"channel + rotation + harmonic + mass flux: U rel {e:.2e}")
    assert e <= 1e-10


def test_rayleigh_benard_with_nudging():
    case = cases.regression_case("rb")
    case.params.update(use_nudging=1, nudging_tau=0.5, nudging_z_start=0.3, nudging_z_full=0.7,
                       nudging_horizontal_only=0)
    times = np.array([0.0, 0.1, 10.0])
    z = np.array([0.0, 0.4, 1.0])
    Up = np.stack([np.stack([[0.1 * (1 + k) * zz, -0.05 * zz, 0.02] for zz in z]) for k in range(3)])
    Tp = np.array([[1.0 - zz for zz in z] for _ in range(3)]) + 0.05 * np.arange(3)[:, None]

    def setup(h):
        h.set_nudging_profiles(times, z, Up, Tp)

    o, s = _pair(case, 5, setup)
    eU = _rel(s.sync_host()["U"], o.state()["U"])
    eT = _rel(s.scalars()[0], o.scalars()[0])
    print(f"Rayleigh-Benard + nudging: U rel {eU:.2e}, T rel {eT:.2e}")
    assert eU <= 1e-10 and eT <= 1e-10


def test_most_channel_with_scalar_sources():
    case = cases.regression_case("channel_most")
    L = 6.283185307179586
    defs = [dict(scalar_id=1, src_kind=abi.SRC_POINT, center=(L / 2, L / 2, 0.5), radius=0.6, magnitude=2.0),
            dict(scalar_id=1, src_kind=abi.SRC_VOLUME, shape=abi.SHAPE_BOX, box_min=(0.5, 0.5, 0.1),
                 box_max=(2.0, 3.0, 0.4), magnitude=-1.0, time_mode=abi.TIME_HARMONIC, omega=20.0, phase=0.3),
            dict(scalar_id=1, src_kind=abi.SRC_LINE, p0=(0.0, 1.0, 0.8), p1=(L, 4.0, 0.8), radius=0.15,
                 magnitude=0.5),
            dict(scalar_id=1, src_kind=abi.SRC_OBJ, tag_points=[(4.0, 1.0, 0.2), (5.0, 5.0, 0.7)], tag_radius=0.4,
                 magnitude=3.0),
            dict(scalar_id=2, src_kind=abi.SRC_POINT, center=(1.0, 1.0, 0.5), radius=0.5, magnitude=9.0)]  # no scalar 2

    def setup(h):
        h.set_scalar_sources(defs)

    o, s = _pair(case, 5, setup)
    eU = _rel(s.sync_host()["U"], o.state()["U"])
    eC = _rel(s.scalars()[1], o.scalars()[1])
    print(f"MOST channel + scalar sources: U rel {eU:.2e}, C rel {eC:.2e}")
    assert eU <= 1e-10 and eC <= 1e-10


def test_precision_form_refuses_nudging():
    case = cases.regression_case("tgv_skew")
    p = case.make_params()
    p.form = abi.FORM_MIXED
    p.p_solver = abi.PSOLVER_TWOLEVEL_FCG
    p.use_nudging = 1
    with pytest.raises(DopamineError) as e:
        Solver(case, params=p)
    assert e.value.status == abi.ERR_UNSUPPORTED
