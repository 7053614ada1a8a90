"""Host side of the device output (dopamine_b200/sampling.py), on the CPU: the sample point sets
of the reference's plane and line objects (src/stats/mod_sampling.f90:252-321), its point-file
parser (:564-600, :1148-1178), the NetCDF layout of a sample file (:381-418, :470-490) and the
statistics CSV (src/stats/mod_stats.f90:33-254)."""
import numpy as np
import pytest

from dopamine_b200 import sampling as S


def test_plane_points_span_the_plane_in_the_reference_order():
    o, n = np.array([1.0, 2.0, 3.0]), np.array([0.0, 0.0, 2.0])
    pts = S.plane_points(o, n, (1.0, 1.0, 0.0), 0.5, 0.25, 5, 3)
    assert pts.shape == (15, 3)
    assert np.allclose((pts - o) @ (n / 2.0), 0.0, atol=1e-15)
    ex = np.array([1.0, 1.0, 0.0]) / np.sqrt(2.0)
    ey = np.cross([0.0, 0.0, 1.0], ex)
    # x index fastest: the first row runs along ex at ty = -half_height
    assert np.allclose(pts[0], o - 0.5 * ex - 0.25 * ey)
    assert np.allclose(pts[4], o + 0.5 * ex - 0.25 * ey)
    assert np.allclose(pts[-1], o + 0.5 * ex + 0.25 * ey)
    # a hint along the normal falls back to x (or y for a normal near x); at least 2 x 2 points
    q = S.plane_points(o, (0, 0, 1), (0, 0, 5), 1.0, 1.0, 1, 1)
    assert q.shape == (4, 3) and np.allclose(q[1] - q[0], [2.0, 0.0, 0.0])
    r = S.plane_points(o, (1, 0, 0), (3, 0, 0), 1.0, 1.0, 2, 2)
    assert np.allclose(r[1] - r[0], [0.0, 2.0, 0.0])


def test_line_points_include_both_ends():
    pts = S.line_points((0, 0, 0), (1, 2, 3), 4)
    assert np.allclose(pts[0], 0.0) and np.allclose(pts[-1], [1, 2, 3]) and len(pts) == 4
    assert len(S.line_points((0, 0, 0), (1, 0, 0), 1)) == 2


def test_point_file_parser(tmp_path):
    f = tmp_path / "pts.txt"
    f.write_text("# probes\n\n1 2 3\n4.5,5.5,6.5\nv 7 8 9\nvertex 1d0 2.0D1 -3e-1\nnot a point\n1 2\n")
    pts = S.read_points(str(f))
    assert np.allclose(pts, [[1, 2, 3], [4.5, 5.5, 6.5], [7, 8, 9], [1.0, 20.0, -0.3]])
    assert S.read_points(str(tmp_path / "missing.txt")).shape == (0, 3)


class _StubSolver:
    """Stands in for the device: owners are point indices, the payload a known function."""

    def set_sample_points(self, xyz):
        self.xyz = np.asarray(xyz)
        return np.arange(len(xyz), dtype=np.int32)

    def sample_points(self):
        x = self.xyz
        return np.stack([x[:, 0], x[:, 1], x[:, 2], x.sum(1), 2 * x[:, 0], 3 * x[:, 1]], axis=1)


def test_sample_files_have_the_reference_layout(tmp_path):
    from scipy.io import netcdf_file
    objs = [S.SampleObject("plane", "mid", S.plane_points((0, 0, 0), (0, 0, 1), (1, 0, 0), 1, 1, 3, 2), 2),
            S.SampleObject("line", "axis", S.line_points((0, 0, 0), (0, 0, 1), 5), 3)]
    samp = S.Sampler(_StubSolver(), str(tmp_path / "run"), objs)
    for step in range(1, 7):
        samp.maybe_sample(0.1 * step, step)
    samp.close()
    with netcdf_file(str(tmp_path / "run_sample_plane_mid.nc"), "r", mmap=False) as f:
        assert f.dimensions["time"] is None and f.dimensions["point"] == 6
        assert f.sampler_kind == b"plane" and f.sampler_name == b"mid"
        assert np.allclose(f.variables["time"][:], [0.2, 0.4, 0.6])
        assert f.variables["U"].shape == (3, 6, 3)
        assert np.allclose(f.variables["U"][1], objs[0].points)
        assert np.allclose(f.variables["p"][2], objs[0].points.sum(1))
        assert np.allclose(f.variables["coords"][:], objs[0].points)
    with netcdf_file(str(tmp_path / "run_sample_line_axis.nc"), "r", mmap=False) as f:
        assert np.allclose(f.variables["time"][:], [0.3, 0.6])
        assert np.allclose(f.variables["nu_sgs"][0], 3 * objs[1].points[:, 1])


def test_stats_csv_matches_the_reference_format(tmp_path):
    # a row of the reference's tests/regression/reference/tgv_skew_exact_np1.csv, as printed
    assert S._es18_9(1.125550134e-02) == "   1.125550134E-02"
    assert S._es18_9(4.166399705e-12) == "   4.166399705E-12"
    assert S._es18_9(0.0) == "   0.000000000E+00"
    assert S._es18_9(-2.5e-150) == "  -2.500000000-150"
    w = S.StatsWriter(str(tmp_path / "run"), nu=1e-3)
    st = dict(time=0.5, E=2.0, eps=0.1, Umax=1.5, max_abs_divU=1e-12, volavg_abs_divU=1e-13, max_abs_divU_cell=0.02,
              volavg_abs_divU_cell=0.001, Ub=1.0, tauw_mean=0.25, nu_sgs_mean=2e-4)
    w.row(1, st, dt=0.01)
    st["E"] = 1.0
    w.row(2, st, dt=0.01)
    lines = open(w.path).read().splitlines()
    assert lines[0] == S.STATS_HEADER
    rows = S.load_stats_csv(w.path)
    assert rows[2]["E_over_E0"] == pytest.approx(0.5) and rows[1]["Cf_bulk"] == pytest.approx(0.5)
    assert rows[1]["nu_sgs_over_nu"] == pytest.approx(0.2) and rows[1]["eps_ref"] == pytest.approx(0.1)
    assert lines[1].startswith("1,   5.000000000E-01,   2.000000000E+00,")
