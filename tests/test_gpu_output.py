"""Output on the device: point sampling, checkpoints and the statistics CSV.

* Sampling (sampling.cuh) against the oracle's restatement of src/stats/mod_sampling.f90 after the
  two have taken the same steps: identical owner cells (nearest centroid, first in index order)
  and payloads within 1e-9 relative, on plane, line and scattered points; the NetCDF files the
  host writer makes from the device payload hold it unchanged.
* Checkpoints (dpm_write_checkpoint / dpm_read_checkpoint) in the reference's record format: the
  file is parsed here record by record (4-byte markers, header, time, global ids, U, p, T, nu_sgs,
  C, U_face, wall-model records) and checked against the handle's state; a handle restarted from
  it takes the next steps as the uninterrupted handle does, to 1e-10 (1e-5 with the exact cell
  projection, whose inexact solves amplify last-bit differences); another mesh is refused.
* The statistics CSV written from the device's dpm_stats on the reference's regression cases
  matches the reference's CSV under its own comparison (rtol 1e-6 on the compared columns, face
  divergence below 1e-9).
"""
import os
import struct

import numpy as np
import pytest

from dopamine_b200 import abi, cases
from dopamine_b200 import sampling as S
from dopamine_b200.solver import DopamineError, Solver
from oracle import oracle as O
from tests.test_oracle_golden import load

pytestmark = pytest.mark.gpu


def _points(case, o):
    lo, hi = case.mesh.vertex_bounds()
    lo, hi = np.asarray(lo), np.asarray(hi)
    mid = 0.5 * (lo + hi)
    span = hi - lo
    plane = S.plane_points(mid, (0, 0, 1), (1, 0, 0), 0.45 * span[0], 0.45 * span[1], 7, 5)
    line = S.line_points(lo + 0.05 * span, hi - 0.05 * span, 9)
    rng = np.random.default_rng(3)
    scat = lo + rng.uniform(0.02, 0.98, (16, 3)) * span
    return np.concatenate([plane, line, scat, o.centroid[:3]])  # centroids themselves: dx = 0


@pytest.mark.parametrize("name", ["rb", "channel_most", "duct"])
def test_sampling_matches_oracle(name, tmp_path):
    case = cases.regression_case(name)
    o = O.Oracle(case)
    s = Solver(case)
    o.initialise()
    s.initialise()
    for _ in range(2):
        o.advance()
        s.advance()
    o.stats()
    s.stats()  # both refresh the boundary velocity as the reference's divergence metrics do
    pts = _points(case, o)
    own_g = s.set_sample_points(pts)
    got = s.sample_points()
    want = np.zeros((len(pts), 6))
    own_o = np.zeros(len(pts), dtype=np.int32)
    import ctypes as C
    O.lib().orc_sample_points(o.h, len(pts), np.ascontiguousarray(pts).ctypes.data_as(C.POINTER(C.c_double)),
                              want.ctypes.data_as(C.POINTER(C.c_double)), own_o.ctypes.data_as(C.POINTER(C.c_int)))
    np.testing.assert_array_equal(own_g, own_o)
    scale = np.maximum(np.abs(want).max(axis=0), 1e-30)
    err = (np.abs(got - want) / scale).max()
    print(f"{name}: {len(pts)} points, payload max rel {err:.2e}")
    assert err <= 1e-9
    # the host writer stores the device payload unchanged
    objs = [S.SampleObject("points", "all", pts, 1)]
    samp = S.Sampler(s, str(tmp_path / name), objs)
    pay = samp.maybe_sample(0.5, 3)
    samp.close()
    from scipy.io import netcdf_file
    with netcdf_file(str(tmp_path / f"{name}_sample_points_all.nc"), "r", mmap=False) as f:
        np.testing.assert_array_equal(f.variables["U"][0], pay[:, 0:3])
        np.testing.assert_array_equal(f.variables["T"][0], pay[:, 4])
    s.close()


def _records(path):
    """The sequential unformatted records of a gfortran file (no subrecords at these sizes)."""
    out = []
    with open(path, "rb") as fh:
        data = fh.read()
    i = 0
    while i < len(data):
        (n,) = struct.unpack_from("<i", data, i)
        assert n >= 0
        payload = data[i + 4:i + 4 + n]
        (m,) = struct.unpack_from("<i", data, i + 4 + n)
        assert m == n
        out.append(payload)
        i += 8 + n
    return out


@pytest.mark.parametrize("name", ["amd", "channel_most", "duct_exact"])
def test_checkpoint_restart_continues_the_run(name, tmp_path):
    case = cases.regression_case(name)
    a = Solver(case)
    a.initialise()
    for _ in range(3):
        a.advance()
    d = str(tmp_path / "ckpt")
    a.write_checkpoint(d, 3)
    t_ck = a.time
    st = a.sync_host()
    T_a, C_a = a.scalars()
    for _ in range(2):
        a.advance()
    ua = a.sync_host()["U"]
    # the file, record by record
    assert open(os.path.join(d, "checkpoint_latest")).read().split() == ["3"]
    recs = _records(os.path.join(d, "processor0", "checkpoint_00000003.bin"))
    hdr = struct.unpack("<8i", recs[0])
    ns = int(case.make_params().n_scalars)
    p = case.make_params()
    mask = 1 + (6 if p.wall_model == abi.WM_MOST else 0) + (8 if (p.wall_model == abi.WM_LOGLAW and p.wall_model_filter_tf_fac > 0) else 0)
    assert hdr == (a.nc, ns, 0, 3, 1 if ns else 0, 0, 1, mask), hdr
    assert struct.unpack("<d", recs[1])[0] == t_ck
    np.testing.assert_array_equal(np.frombuffer(recs[2], dtype="<i8"), np.arange(1, a.nc + 1))
    np.testing.assert_array_equal(np.frombuffer(recs[3], dtype="<f8").reshape(-1, 3), st["U"])
    np.testing.assert_array_equal(np.frombuffer(recs[4], dtype="<f8"), st["p"])
    np.testing.assert_array_equal(np.frombuffer(recs[5], dtype="<f8"), T_a)
    k = 7
    if ns:
        np.testing.assert_array_equal(np.frombuffer(recs[7], dtype="<f8").reshape(-1, ns).T, C_a)
        k = 8
    assert len(recs[k]) == 8 * a.nf  # U_face
    expected_records = k + 1 + 1 + (2 if mask & 6 else 0) + (1 if mask & 8 else 0)
    assert len(recs) == expected_records
    # restart in a fresh handle and take the same steps
    b = Solver(case)
    b.read_checkpoint(d)  # the step checkpoint_latest names
    for _ in range(2):
        b.advance()
    ub = b.sync_host()["U"]
    err = float(np.linalg.norm(ub - ua) / np.linalg.norm(ua))
    print(f"{name}: restart after 3 steps, 2 more: U rel {err:.2e}, header {hdr}")
    # the exact projection's preconditioning solves stop at rtol 0.05; the restart's refreshed boundary
    # values and gradients can move one stop by an iteration, which moves the inexact projection by
    # ~1e-6 (the same sensitivity as its parity test); the other cases restart to round-off
    assert err <= (1e-5 if case.make_params().cell_projection == abi.CELL_PROJECTION_EXACT else 1e-10)
    assert b.time == pytest.approx(a.time, rel=1e-14)
    # another mesh is refused
    other = Solver(cases.regression_case("tgv_skew"))
    with pytest.raises(DopamineError) as e:
        other.read_checkpoint(d, 3)
    assert e.value.status == abi.ERR_MESH
    for h in (a, b, other):
        h.close()


@pytest.mark.parametrize("name", ["tgv_skew", "duct", "channel"])
def test_stats_csv_from_the_device_matches_reference(name, tmp_path):
    case = cases.regression_case(name)
    s = Solver(case)
    s.initialise()
    ref = load(name)
    w = S.StatsWriter(str(tmp_path / name), nu=case.make_params().nu)
    for step in range(1, max(ref) + 1):
        s.advance()
        if step in ref:
            st = s.stats()
            w.row(step, st, dt=st["dt_used"])
    got = S.load_stats_csv(w.path)
    for step, r in ref.items():
        for col in ("time", "E", "Umax", "Ub", "tauw_mean", "nu_sgs_mean"):
            a, b = r[col], got[step][col]
            assert abs(a - b) <= 1e-6 * max(abs(a), 1e-6), (step, col, a, b)
        assert got[step]["max_abs_divU"] <= 1e-9
    s.close()
