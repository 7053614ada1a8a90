"""Host side of the device sampling and statistics output (src/stats/mod_sampling.f90,
src/stats/mod_stats.f90).

The samples themselves are taken on the device (dpm_sampling_set_points / dpm_sample_points:
owner search and gradient extrapolation there, only the (6, n) payload crosses PCIe); this module
builds the sample point sets the reference's namelists describe, decides when an object is due,
and writes the reference's files:

* ``<prefix>_sample_<kind>_<name>.nc`` - NetCDF classic, dimensions time (unlimited), point, xyz,
  vec; variables time, coords(point, xyz), U(time, point, vec), p, T, nu_sgs(time, point); global
  attributes sampler_kind and sampler_name (open_object_netcdf, :381-418; Fortran's column-major
  (vec, point, time) is C's (time, point, vec)).  Written with scipy's NetCDF-3 writer.
* ``<prefix>_stats.csv`` - the per-step statistics row of stats_sample (mod_stats.f90:162-254),
  every dpm_stats_t field the reference prints, in its column order and number format.
"""
import math

import numpy as np

SMALL = 1.0e-30


def plane_points(origin, normal, tangent_hint, half_width, half_height, nx, ny):
    """init_plane_object (mod_sampling.f90:252-299): an nx x ny grid (at least 2 x 2) spanning
    [-half_width, half_width] x [-half_height, half_height] about origin, in the plane with the given
    normal; the first axis is tangent_hint with its normal part removed (x, or y when the normal is
    nearly x, if the hint is parallel to the normal).  Points (nx*ny, 3), x index fastest."""
    nx, ny = max(2, int(nx)), max(2, int(ny))
    n = np.asarray(normal, dtype=np.float64)
    if math.sqrt(float(n @ n)) <= SMALL:
        n = np.array([0.0, 0.0, 1.0])
    n = n / max(math.sqrt(float(n @ n)), SMALL)
    hint = np.asarray(tangent_hint, dtype=np.float64)
    ex = hint - float(hint @ n) * n
    hmag = math.sqrt(float(ex @ ex))
    if hmag <= SMALL:
        ex = np.array([1.0, 0.0, 0.0]) if abs(n[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
        ex = ex - float(ex @ n) * n
        hmag = math.sqrt(float(ex @ ex))
    ex = ex / max(hmag, SMALL)
    ey = np.array([n[1] * ex[2] - n[2] * ex[1], n[2] * ex[0] - n[0] * ex[2], n[0] * ex[1] - n[1] * ex[0]])
    o = np.asarray(origin, dtype=np.float64)
    pts = np.empty((nx * ny, 3))
    k = 0
    for iy in range(ny):
        ty = (2.0 * (iy / max(1, ny - 1)) - 1.0) * half_height
        for ix in range(nx):
            tx = (2.0 * (ix / max(1, nx - 1)) - 1.0) * half_width
            pts[k] = o + tx * ex + ty * ey
            k += 1
    return pts


def line_points(p0, p1, npts):
    """init_line_object (:301-321): npts (at least 2) points from p0 to p1 inclusive."""
    npts = max(2, int(npts))
    p0 = np.asarray(p0, dtype=np.float64)
    p1 = np.asarray(p1, dtype=np.float64)
    s = np.arange(npts) / max(1, npts - 1)
    return (1.0 - s)[:, None] * p0 + s[:, None] * p1


def read_points(filename):
    """read_points_from_file / parse_point_line (:564-600, :1148-1178): one point per line as
    three numbers (list-directed: blanks or commas), or an OBJ 'v x y z' / STL 'vertex x y z'
    line; blank lines, '#' comments and unreadable lines are skipped.  A missing file gives no
    points (the reference warns and continues)."""
    pts = []
    try:
        fh = open(filename)
    except OSError:
        return np.zeros((0, 3))
    with fh:
        for line in fh:
            s = line.strip()
            if not s or s.startswith("#"):
                continue
            if s.startswith("vertex "):
                s = s[7:]
            elif s.startswith("v "):
                s = s[2:]
            toks = s.replace(",", " ").split()
            if len(toks) < 3:
                continue
            try:
                pts.append([float(t.replace("d", "e").replace("D", "e")) for t in toks[:3]])
            except ValueError:
                continue
    return np.array(pts, dtype=np.float64).reshape(-1, 3)


class SampleObject:
    def __init__(self, kind, name, points, write_frequency):
        self.kind, self.name = kind, name
        self.points = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        self.write_frequency = int(write_frequency)
        self.active = len(self.points) > 0
        self.samples_written = 0
        self._nc = None

    def due(self, step):
        return self.active and self.write_frequency > 0 and step % self.write_frequency == 0


class Sampler:
    """SamplingCollector: every object's points are given to the device once; a due step samples
    them all in one launch and appends each due object's slice to its NetCDF file."""

    def __init__(self, solver, prefix, objects):
        self.solver, self.prefix = solver, prefix
        self.objects = [o for o in objects if o.active]
        self.offsets = np.cumsum([0] + [len(o.points) for o in self.objects])
        allpts = np.concatenate([o.points for o in self.objects]) if self.objects else np.zeros((0, 3))
        self.owner = solver.set_sample_points(allpts) if len(allpts) else np.zeros(0, dtype=np.int32)
        for o in self.objects:
            self._open(o)

    def path(self, obj):
        return f"{self.prefix}_sample_{obj.kind}_{obj.name}.nc"

    def _open(self, obj):
        from scipy.io import netcdf_file
        f = netcdf_file(self.path(obj), "w", version=1)
        f.createDimension("time", None)
        f.createDimension("point", len(obj.points))
        f.createDimension("xyz", 3)
        f.createDimension("vec", 3)
        f.createVariable("time", "d", ("time",))
        f.createVariable("coords", "d", ("point", "xyz"))[:] = obj.points
        f.createVariable("U", "d", ("time", "point", "vec"))
        f.createVariable("p", "d", ("time", "point"))
        f.createVariable("T", "d", ("time", "point"))
        f.createVariable("nu_sgs", "d", ("time", "point"))
        f.sampler_kind = obj.kind
        f.sampler_name = obj.name
        f.flush()
        obj._nc = f

    def maybe_sample(self, time, step):
        """sampling_maybe_sample (:160-232); returns the payload when something was due."""
        due = [o.due(step) for o in self.objects]
        if not any(due):
            return None
        payload = self.solver.sample_points()
        for k, o in enumerate(self.objects):
            if not due[k]:
                continue
            sl = payload[self.offsets[k]:self.offsets[k + 1]]
            f, t = o._nc, o.samples_written
            f.variables["time"][t] = time
            f.variables["U"][t] = sl[:, 0:3]
            f.variables["p"][t] = sl[:, 3]
            f.variables["T"][t] = sl[:, 4]
            f.variables["nu_sgs"][t] = sl[:, 5]
            f.flush()
            o.samples_written = t + 1
        return payload

    def close(self):
        for o in self.objects:
            if o._nc is not None:
                o._nc.close()
                o._nc = None


STATS_HEADER = ("step,time,E,eps,E_over_E0,eps_ref,Umax,max_abs_divU,volavg_abs_divU,"
                "max_abs_divU_cell,volavg_abs_divU_cell,Ub,tauw_mean,Cf_bulk,nu_sgs_mean,nu_sgs_over_nu,dt")


def _es18_9(x):
    """Fortran ES18.9: one leading digit, 9 decimals and a signed exponent - 'E' and two digits,
    or three digits without the 'E' beyond +-99 - right-justified in 18 columns."""
    if x == 0.0:
        return f"{'0.000000000E+00':>18}"
    m, e = f"{x:.9E}".split("E")
    e = int(e)
    sign = "+" if e >= 0 else "-"
    tail = f"E{sign}{abs(e):02d}" if abs(e) <= 99 else f"{sign}{abs(e):03d}"
    return f"{m + tail:>18}"


class StatsWriter:
    """stats_init / stats_sample (mod_stats.f90:33-254): <prefix>_stats.csv, one row per call."""

    def __init__(self, prefix, nu):
        self.path = f"{prefix}_stats.csv"
        self.nu = nu
        self.E0 = 0.0
        with open(self.path, "w") as fh:
            fh.write(STATS_HEADER + "\n")

    def row(self, step, st, dt=None):
        E = st["E"]
        if self.E0 <= SMALL:
            self.E0 = E
        e_norm = E / self.E0 if self.E0 > SMALL else 1.0
        cf = st["tauw_mean"] / max(0.5 * st["Ub"] ** 2, SMALL)
        vals = [st["time"], E, st["eps"], e_norm, st["eps"], st["Umax"], st["max_abs_divU"], st["volavg_abs_divU"],
                st["max_abs_divU_cell"], st["volavg_abs_divU_cell"], st["Ub"], st["tauw_mean"], cf, st["nu_sgs_mean"],
                st["nu_sgs_mean"] / max(self.nu, SMALL), 0.0 if dt is None else dt]
        with open(self.path, "a") as fh:
            fh.write(str(int(step)) + "".join("," + _es18_9(float(v)) for v in vals) + "\n")
        return vals


def load_stats_csv(path):
    import csv
    with open(path, newline="") as fh:
        return {int(r["step"]): {k: float(v) for k, v in r.items() if k != "step"} for r in csv.DictReader(fh)}


__all__ = ["plane_points", "line_points", "read_points", "SampleObject", "Sampler", "StatsWriter", "STATS_HEADER",
           "load_stats_csv"]
