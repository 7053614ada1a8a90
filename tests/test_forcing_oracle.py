"""Body forces, nudging and scalar sources in the oracle against closed forms.

On a periodic box at rest or in uniform motion (no advection, no viscous term, no pressure), the
RK3W step integrates these terms alone, so the result is known exactly:
* Coriolis, -2 Omega x U, is linear: three-stage third-order RK advances it by the cubic Taylor
  polynomial of the rotation (src/solver/mod_fv_solver.f90:1688-1692).
* Harmonic forcing is evaluated at the stage times t_n + c_k dt (compute_explicit_rhs receives
  self%time, :1309, :1667-1675), so one step adds dt [(a1 + b2) f(t1) + (a2 + b3) f(t2) + a3 f(t3)].
* The mass-flux force (U_bulk_target - <U>) / dt (:959-983) brings the mean velocity to the target
  in one step, the RK3W weights summing to one.
* Davies nudging relaxes u (not w, by default) and T towards the profile at the rate
  min(1/tau, 0.5/dt) above z_start with the linear ramp (src/abl/mod_abl_weather.f90:233-287).
* A box source adds magnitude x dt per step to the cells it covers (src/mod_scalar.f90:133-183);
  a harmonic one the stage-weighted cosines.
"""
import math

import numpy as np
import pytest

from dopamine_b200 import abi, cases
from oracle import oracle as O

A = (8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0)
B = (0.0, -17.0 / 60.0, -5.0 / 12.0)
CS = (0.0, 8.0 / 15.0, 2.0 / 3.0)


def _box(**prm):
    n = 6
    base = dict(scheme=abi.SCHEME_CDS, nu=0.0, dt=0.01, cfl_max=1e9, p_tol=1e-12, sgs_model=abi.SGS_NONE,
                wall_model=abi.WM_NONE)
    base.update(prm)
    return cases.Case("forcing_box", cases.uniform_box(n, n, n, 1.0, 1.0, 1.0), [{"bc": "periodic"}] * 6, base,
                      "uniform", 0.0)


def _run(case, U0, steps, setup=None, T0=None):
    o = O.Oracle(case)
    U = np.tile(np.asarray(U0, dtype=np.float64), (o.nc, 1))
    o.set_state(U=U, p=np.zeros(o.nc), T=None if T0 is None else np.full(o.nc, T0))
    if setup:
        setup(o)
    for _ in range(steps):
        o.advance()
    return o


def test_coriolis_is_the_rk3_cubic_of_the_rotation():
    om, dt, steps = 0.7, 0.05, 5
    case = _box(use_rotation=1, omega_rot=(0.0, 0.0, om), dt=dt)
    o = _run(case, (1.0, 0.0, 0.0), steps)
    f = 2.0 * om  # du/dt = f v, dv/dt = -f u
    M = np.array([[0.0, f], [-f, 0.0]]) * dt
    R = np.eye(2) + M + M @ M / 2.0 + M @ M @ M / 6.0
    uv = np.linalg.matrix_power(R, steps) @ np.array([1.0, 0.0])
    U = o.state()["U"]
    assert np.abs(U[:, 0] - uv[0]).max() <= 1e-13 and np.abs(U[:, 1] - uv[1]).max() <= 1e-13
    assert np.abs(U[:, 2]).max() <= 1e-15


def test_harmonic_forcing_at_the_stage_times():
    amp, w, ph, dt, steps = 0.3, 2.0, 0.4, 0.05, 4
    d = np.array([1.0, 2.0, 0.0]) / math.sqrt(5.0)
    case = _box(use_harmonic_forcing=1, forcing_amp=amp, forcing_omega=w, forcing_phase=ph,
                forcing_dir=(1.0, 2.0, 0.0), dt=dt)
    o = _run(case, (0.0, 0.0, 0.0), steps)
    f = lambda t: amp * math.cos(w * t + ph)
    s = 0.0
    for n in range(steps):
        t = n * dt
        s += dt * ((A[0] + B[1]) * f(t + CS[0] * dt) + (A[1] + B[2]) * f(t + CS[1] * dt) + A[2] * f(t + CS[2] * dt))
    U = o.state()["U"]
    assert np.abs(U - s * d).max() <= 1e-14


def test_mass_flux_forcing_reaches_the_target_in_one_step():
    case = _box(constant_mass_flux_forcing=1, U_bulk_target=(1.0, 0.0, -0.25), dt=0.02)
    o = _run(case, (0.5, 0.1, 0.0), 1)
    U = o.state()["U"]
    assert np.abs(U - np.array([1.0, 0.0, -0.25])).max() <= 1e-13


@pytest.mark.parametrize("horizontal", [1, 0])
def test_nudging_relaxes_towards_the_profile(horizontal):
    """u(z) stays divergence-free under the ramp; a nudged w must be uniform to stay so, so the
    vertical case nudges every cell."""
    dt, tau, steps = 0.05, 0.4, 3
    zs, zf = (0.5, 0.75) if horizontal else (-1.0, -1.0)
    case = _box(use_nudging=1, nudging_tau=tau, nudging_z_start=zs, nudging_z_full=zf,
                nudging_horizontal_only=horizontal, dt=dt)
    uref = np.array([2.0, -1.0, 0.5])
    prof_t = np.array([0.0, 10.0])
    prof_z = np.array([0.0, 1.0])
    Up = np.tile(uref, (2, 2, 1))
    Tp = np.full((2, 2), 310.0)
    o = _run(case, (0.0, 0.0, 0.0), steps, setup=lambda o: o.set_nudging_profiles(prof_t, prof_z, Up, Tp), T0=300.0)
    U = o.state()["U"]
    T, _ = o.scalars()
    z = o.centroid[:, 2]
    coeff = min(1.0 / tau, 0.5 / dt)
    for c in range(o.nc):
        ramp = 0.0 if z[c] < zs else (min(1.0, (z[c] - zs) / (zf - zs)) if zf > zs else 1.0)
        r = 1.0 - ramp * coeff * dt
        r3 = 1.0 + (r - 1.0) + (r - 1.0) ** 2 / 2.0 + (r - 1.0) ** 3 / 6.0
        g = r3 ** steps  # remaining fraction of the departure from the profile
        want = uref * (1.0 - g)
        if horizontal:
            want[2] = 0.0
        assert np.abs(U[c] - want).max() <= 1e-13, (c, U[c], want)
        assert abs(T[c] - (310.0 - 10.0 * g)) <= 1e-11


@pytest.mark.parametrize("mode", [abi.TIME_CONSTANT, abi.TIME_HARMONIC])
def test_box_source_adds_its_magnitude(mode):
    dt, steps, mag, w = 0.02, 3, 2.5, 3.0
    case = _box(n_scalars=1, scalar_scheme=abi.SCHEME_CDS, scalar_diffusivity=(0.0, 0, 0, 0), scalar_pr_t=(1.0, 0, 0, 0),
                dt=dt)
    src = dict(scalar_id=1, src_kind=abi.SRC_VOLUME, shape=abi.SHAPE_BOX, box_min=(0.2, 0.2, 0.2),
               box_max=(0.6, 0.7, 0.5), magnitude=mag, time_mode=mode, omega=w, phase=0.1)
    o = _run(case, (0.0, 0.0, 0.0), steps, setup=lambda o: o.set_scalar_sources([src]))
    _, C = o.scalars()
    x = o.centroid
    inside = np.all((x >= 0.2) & (x <= np.array([0.6, 0.7, 0.5])), axis=1)
    assert 0 < inside.sum() < o.nc
    if mode == abi.TIME_CONSTANT:
        want = mag * dt * steps
    else:
        f = lambda t: mag * math.cos(w * t + 0.1)
        want = sum(dt * ((A[0] + B[1]) * f(n * dt) + (A[1] + B[2]) * f((n + CS[1]) * dt) + A[2] * f((n + CS[2]) * dt))
                   for n in range(steps))
    assert np.abs(C[0][inside] - want).max() <= 1e-14
    assert np.abs(C[0][~inside]).max() == 0.0


def test_source_geometries():
    """Point, line, surface and tag-point sources mark the cells their geometry covers."""
    case = _box(n_scalars=1, scalar_scheme=abi.SCHEME_CDS, scalar_diffusivity=(0.0, 0, 0, 0), scalar_pr_t=(1.0, 0, 0, 0),
                dt=0.01)
    defs = [dict(src_kind=abi.SRC_POINT, center=(0.5, 0.5, 0.5), radius=0.2, magnitude=1.0),
            dict(src_kind=abi.SRC_LINE, p0=(0.0, 0.1, 0.1), p1=(1.0, 0.1, 0.1), radius=0.1, magnitude=10.0),
            dict(src_kind=abi.SRC_SURFACE, center=(0.5, 0.5, 0.9), normal=(0.0, 0.0, 2.0), half_thickness=0.05,
                 radius=0.3, magnitude=100.0),
            dict(src_kind=abi.SRC_OBJ, tag_points=[(0.9, 0.9, 0.1), (0.1, 0.9, 0.9)], tag_radius=0.12, magnitude=1000.0)]
    o = _run(case, (0.0, 0.0, 0.0), 1, setup=lambda o: o.set_scalar_sources(defs))
    _, C = o.scalars()
    x = o.centroid
    seg = np.clip(x[:, 0], 0.0, 1.0)
    in_pt = np.sum((x - 0.5) ** 2, axis=1) <= 0.04
    in_ln = np.sqrt((x[:, 0] - seg) ** 2 + (x[:, 1] - 0.1) ** 2 + (x[:, 2] - 0.1) ** 2) <= 0.1
    in_sf = (np.abs(x[:, 2] - 0.9) <= 0.05) & (np.sum((x - [0.5, 0.5, 0.9]) ** 2, axis=1) <= 0.09)
    dtag = np.minimum(np.linalg.norm(x - [0.9, 0.9, 0.1], axis=1), np.linalg.norm(x - [0.1, 0.9, 0.9], axis=1))
    in_ob = dtag <= 0.12
    want = 0.01 * (1.0 * in_pt + 10.0 * in_ln + 100.0 * in_sf + 1000.0 * in_ob)
    assert in_pt.any() and in_ln.any() and in_sf.any() and in_ob.any()
    assert np.abs(C[0] - want).max() <= 1e-12
