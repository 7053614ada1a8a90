"""ORACLE — test infrastructure only (the parity checker and the timed CPU baseline).

ctypes binding of oracle/oracle.cpp, the CPU restatement of the reference's RK3W time step.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from dopamine_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.POINTER(abi.RawMeshT), C.POINTER(abi.PatchCfgT), C.POINTER(abi.ParamsT), C.c_int]
        L.orc_destroy.argtypes = [vp]
        L.orc_sizes.argtypes = [vp, C.POINTER(C.c_int64)]
        L.orc_geometry.argtypes = [vp, dp, dp]
        L.orc_vertex_bounds.argtypes = [vp, dp, dp]
        L.orc_set_state.argtypes = [vp, dp, dp, dp]
        L.orc_get_state.argtypes = [vp, dp, dp, dp, dp, dp]
        L.orc_project_once.argtypes = [vp, C.c_double]
        L.orc_project_once.restype = C.c_int
        L.orc_advance.argtypes = [vp, C.c_double]
        L.orc_advance.restype = C.c_int
        L.orc_stats.argtypes = [vp, C.POINTER(abi.StatsT)]
        L.orc_time.argtypes = [vp]
        L.orc_time.restype = C.c_double
        L.orc_compute_dt.argtypes = [vp, dp]
        L.orc_compute_dt.restype = C.c_int
        L.orc_ls_gradient_vector.argtypes = [vp, dp, dp, dp]
        L.orc_gg_gradient_scalar.argtypes = [vp, dp, dp, dp, C.c_int]
        L.orc_face_centres.argtypes = [vp, dp]
        L.orc_advection.argtypes = [vp, C.c_int, dp, dp, dp, dp, dp]
        L.orc_viscous.argtypes = [vp, dp, dp, dp, dp, dp]
        L.orc_sgs.argtypes = [vp, C.c_int, dp, dp, C.c_double, dp]
        L.orc_wall_model.argtypes = [vp, dp, dp]
        L.orc_amd_point.argtypes = [dp, dp, C.c_double]
        L.orc_amd_point.restype = C.c_double
        L.orc_wall_stress_newton.argtypes = [C.c_double, C.c_double, C.c_double, dp, dp]
        L.orc_kfactor_limited.argtypes = [dp, dp, C.c_double, dp]
        L.orc_sample_points.argtypes = [vp, C.c_int, dp, dp, ip]
        L.orc_set_nudging_profiles.argtypes = [vp, C.c_int, C.c_int, dp, dp, dp, dp]
        L.orc_set_scalar_sources.argtypes = [vp, C.c_int, C.POINTER(abi.ScalarSourceT)]
        L.orc_cp_divergence.argtypes = [vp, dp, dp]
        L.orc_cp_adjoint.argtypes = [vp, dp, dp]
        L.orc_cp_project.argtypes = [vp, dp, dp, C.c_double, C.c_int, C.c_int, ip]
        L.orc_cp_project.restype = C.c_int
        L.orc_poisson_solve.argtypes = [vp, dp, dp, C.c_double, C.c_double, C.c_int, ip, dp]
        L.orc_poisson_solve.restype = C.c_int
        L.orc_poisson_matvec.argtypes = [vp, dp, dp]
        L.orc_poisson_csr.argtypes = [vp, C.POINTER(C.c_int64), ip, dp]
        L.orc_poisson_csr.restype = C.c_int64
        L.orc_record_poisson.argtypes = [vp, C.c_int]
        L.orc_get_scalars.argtypes = [vp, dp, dp]
        L.orc_lp_loss_grad.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, dp,
                                       C.c_int, dp, dp, dp, dp, C.c_void_p, dp, dp]
        L.orc_advection_scalar.argtypes = [vp, C.c_int, dp, dp, dp, dp, dp]
        L.orc_viscous_scalar.argtypes = [vp, dp, C.c_double, dp, C.c_double, dp, dp, dp]
        L.orc_set_scalars.argtypes = [vp, dp, dp]
        L.orc_recorded_poisson.argtypes = [vp, C.c_int, dp, dp, dp]
        L.orc_recorded_poisson.restype = C.c_int
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """CPU FVSolver restatement on one case (dopamine_b200.cases.Case)."""

    def __init__(self, case, nthreads=1, params=None):
        L = lib()
        self.case = case
        self._mesh = abi.RawMeshView(case.mesh)
        self._patches = abi.patch_cfgs(case.patches)
        self._params = params if params is not None else case.make_params()
        self.h = L.orc_create(C.byref(self._mesh.struct), self._patches, C.byref(self._params), nthreads)
        if not self.h:
            raise RuntimeError("oracle mesh set-up failed")
        sz = (C.c_int64 * 8)()
        L.orc_sizes(self.h, sz)
        self.nc, self.nf, self.nfi, self.nb, self.nfp = (int(sz[i]) for i in range(5))
        self.skip_nonortho, self.skip_grad_p, self.diag_interface = bool(sz[5]), bool(sz[6]), bool(sz[7])
        self.centroid = np.zeros((self.nc, 3))
        self.volume = np.zeros(self.nc)
        L.orc_geometry(self.h, _p(self.centroid), _p(self.volume))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def set_state(self, U=None, p=None, T=None):
        U = None if U is None else np.ascontiguousarray(U, dtype=np.float64)
        p = None if p is None else np.ascontiguousarray(p, dtype=np.float64)
        T = None if T is None else np.ascontiguousarray(T, dtype=np.float64)
        lib().orc_set_state(self.h, _p(U), _p(p), _p(T))

    def state(self):
        U = np.zeros((self.nc, 3)); p = np.zeros(self.nc); nu = np.zeros(self.nc)
        g = np.zeros((self.nc, 3, 3)); ff = np.zeros(self.nf)
        lib().orc_get_state(self.h, _p(U), _p(p), _p(nu), _p(g), _p(ff))
        return {"U": U, "p": p, "nu_sgs": nu, "grad_U": g, "face_flux": ff}

    def initialise(self):
        """apply_initial_conditions: profile (+ noise and an extra projection) + project_once."""
        U = self.case.initial_velocity(self.centroid)
        self.set_state(U=U, p=np.zeros(self.nc))
        dtp = 8.0 / 15.0 * self._params.dt
        if self.case.noise > 0.0:
            self._check(lib().orc_project_once(self.h, dtp))
        self._check(lib().orc_project_once(self.h, dtp))

    def advance(self, dt=None):
        self._check(lib().orc_advance(self.h, self._params.dt if dt is None else dt))

    def stats(self):
        s = abi.StatsT()
        lib().orc_stats(self.h, C.byref(s))
        return s.as_dict()

    def scalars(self):
        """(T [nc], C [n_scalars, nc])."""
        ns = max(0, min(int(self._params.n_scalars), 4))
        T = np.zeros(self.nc)
        Cs = np.zeros((ns, self.nc))
        lib().orc_get_scalars(self.h, _p(T), _p(Cs) if ns else None)
        return T, Cs

    def set_scalars(self, T=None, C=None):
        T = None if T is None else np.ascontiguousarray(T, dtype=np.float64)
        C = None if C is None else np.ascontiguousarray(C, dtype=np.float64)
        lib().orc_set_scalars(self.h, _p(T), _p(C))

    def poisson_csr(self):
        """The assembled pressure operator as (offsets, columns, values)."""
        L = lib()
        nnz = L.orc_poisson_csr(self.h, None, None, None)
        off = np.zeros(self.nc + 1, dtype=np.int64)
        col = np.zeros(nnz, dtype=np.int32)
        val = np.zeros(nnz)
        L.orc_poisson_csr(self.h, off.ctypes.data_as(C.POINTER(C.c_int64)), col.ctypes.data_as(C.POINTER(C.c_int)),
                          _p(val))
        return off, col, val

    def set_nudging_profiles(self, times, z_levels, U_profile, T_profile):
        """times (nt), z_levels (nz), U_profile (nt, nz, 3), T_profile (nt, nz)."""
        t = np.ascontiguousarray(times, dtype=np.float64)
        z = np.ascontiguousarray(z_levels, dtype=np.float64)
        Up = np.ascontiguousarray(U_profile, dtype=np.float64)
        Tp = np.ascontiguousarray(T_profile, dtype=np.float64)
        lib().orc_set_nudging_profiles(self.h, len(t), len(z), _p(t), _p(z), _p(Up), _p(Tp))

    def set_scalar_sources(self, defs):
        arr, self._src_keep = abi.scalar_sources(defs)
        lib().orc_set_scalar_sources(self.h, len(defs), arr)

    def record_poisson(self, on=True):
        lib().orc_record_poisson(self.h, 1 if on else 0)

    def recorded_poisson(self):
        """[(rhs, initial guess, atol)] of the pressure solves since record_poisson(True)."""
        L = lib()
        out = []
        n = L.orc_recorded_poisson(self.h, -1, None, None, None)
        for k in range(n):
            b, x0, at = np.zeros(self.nc), np.zeros(self.nc), C.c_double()
            L.orc_recorded_poisson(self.h, k, _p(b), _p(x0), C.byref(at))
            out.append((b, x0, at.value))
        return out

    @staticmethod
    def _check(rc):
        if rc != 0:
            raise RuntimeError(f"oracle status {rc}")
