"""ctypes binding of libdopamine_b200.so (C ABI in include/dopamine_b200.h).

`Solver` mirrors the reference's FVSolver (src/solver/mod_fv_solver.f90:270-285): init,
project_once, advance, compute_dt, stats, to_device / sync_host.  There is no CPU fallback: if the
library or a CUDA device is missing, construction raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libdopamine_b200.so")
_lib = None

EXPORTED = (
    "fvm_petsc_backend_available", "fvm_petsc_backend_initialize", "fvm_petsc_backend_finalize",
    "fvm_petsc_set_pressure_solver", "fvm_petsc_device_io_supported", "fvm_petsc_set_io_on_device",
    "fvm_petsc_insert_option", "fvm_petsc_set_device_local_rank", "fvm_petsc_solve_pressure",
    "dpm_create", "dpm_destroy", "dpm_n_cells", "dpm_upload_state", "dpm_download_state",
    "dpm_download_face_flux", "dpm_download_gradient", "dpm_cell_geometry", "dpm_project_once", "dpm_advance",
    "dpm_advance_n", "dpm_stats", "dpm_state_is_finite", "dpm_compute_dt", "dpm_get_time", "dpm_set_time",
    "dpm_last_timing", "dpm_kernel_launches", "dpm_ls_gradient_vector", "dpm_advection_rhs_vector",
    "dpm_viscous_rhs_vector", "dpm_sgs_viscosity", "dpm_wall_model", "dpm_pcg_solve_noalloc",
    "dpm_advection_rhs_scalar", "dpm_viscous_rhs_scalar", "dpm_upload_scalars", "dpm_download_scalars",
    "dpm_learn_collect", "dpm_learn_train", "dpm_learn_set_gamma", "dpm_learn_sizes", "dpm_learn_export",
    "dpm_learn_loss_grad", "dpm_multilevel_hierarchy", "dpm_set_barrier_spin_limit",
    "dpm_select_pressure_solver", "dpm_cell_divergence", "dpm_cell_adjoint_gradient", "dpm_cell_project",
    "dpm_write_checkpoint", "dpm_read_checkpoint", "dpm_sampling_set_points", "dpm_sample_points",
    "dpm_set_nudging_profiles", "dpm_set_scalar_sources", "dpm_setup_times", "dpm_setup_compare",
    "dpm_setup_array_name", "dpm_gmsh_read", "dpm_gmsh_sizes", "dpm_gmsh_fill", "dpm_gmsh_patch_name",
    "dpm_gmsh_free", "dpm_gmsh_write", "dpm_fcg_phase_times", "dpm_create_poly", "dpm_foam_read",
    "dpm_foam_sizes", "dpm_foam_fill", "dpm_foam_patch_name", "dpm_foam_patch_type", "dpm_foam_free",
    "dpm_poly_cell_geometry", "dpm_setup_compare_poly", "dpm_setup_host_digest", "dpm_setup_host_digest_poly",
    "dpm_multilevel_digest",
)


class DopamineError(RuntimeError):
    def __init__(self, msg, status=None):
        super().__init__(msg)
        self.status = status


def lib(build_if_missing=True):
    """Load the product library; builds it from source when it is missing and nvcc is present."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise DopamineError(f"{LIB_PATH} not built")
        from . import build as _build
        _build.build()
    L = C.CDLL(LIB_PATH)
    vp, dp, ip, lp = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int64)
    L.dpm_create.argtypes = [C.POINTER(abi.RawMeshT), C.POINTER(abi.PatchCfgT), C.POINTER(abi.ParamsT), C.c_int,
                             C.POINTER(vp)]
    L.dpm_destroy.argtypes = [vp]
    L.dpm_n_cells.argtypes = [vp, lp, lp, lp]
    L.dpm_cell_geometry.argtypes = [vp, dp, dp]
    L.dpm_upload_state.argtypes = [vp, dp, dp, dp]
    L.dpm_download_state.argtypes = [vp, dp, dp, dp, dp]
    L.dpm_download_face_flux.argtypes = [vp, dp]
    L.dpm_download_gradient.argtypes = [vp, dp]
    L.dpm_project_once.argtypes = [vp, C.c_double]
    L.dpm_advance.argtypes = [vp, C.c_double]
    L.dpm_advance_n.argtypes = [vp, C.c_double, C.c_int]
    L.dpm_stats.argtypes = [vp, C.POINTER(abi.StatsT)]
    L.dpm_state_is_finite.argtypes = [vp, ip]
    L.dpm_compute_dt.argtypes = [vp, dp]
    L.dpm_get_time.argtypes = [vp, dp]
    L.dpm_set_time.argtypes = [vp, C.c_double]
    L.dpm_last_timing.argtypes = [vp, dp, dp]
    L.dpm_kernel_launches.argtypes = [vp, lp]
    L.dpm_set_barrier_spin_limit.argtypes = [vp, C.c_longlong]
    L.dpm_select_pressure_solver.argtypes = [vp, C.c_int]
    L.dpm_ls_gradient_vector.argtypes = [vp, dp, dp, dp]
    L.dpm_advection_rhs_vector.argtypes = [vp, C.c_int, dp, dp, dp, dp, dp]
    L.dpm_viscous_rhs_vector.argtypes = [vp, dp, C.c_double, dp, dp, dp, dp]
    L.dpm_sgs_viscosity.argtypes = [vp, C.c_int, dp, dp, dp, C.c_double, dp]
    L.dpm_wall_model.argtypes = [vp, dp, C.c_double, dp]
    L.dpm_cell_divergence.argtypes = [vp, dp, dp]
    L.dpm_write_checkpoint.argtypes = [vp, C.c_char_p, C.c_int]
    L.dpm_read_checkpoint.argtypes = [vp, C.c_char_p, C.c_int]
    L.dpm_sampling_set_points.argtypes = [vp, C.c_int, dp, ip]
    L.dpm_sample_points.argtypes = [vp, dp]
    L.dpm_set_nudging_profiles.argtypes = [vp, C.c_int, C.c_int, dp, dp, dp, dp]
    L.dpm_set_scalar_sources.argtypes = [vp, C.c_int, C.POINTER(abi.ScalarSourceT)]
    L.dpm_cell_adjoint_gradient.argtypes = [vp, dp, dp]
    L.dpm_cell_project.argtypes = [vp, dp, dp, C.c_double, C.c_int, C.c_int, ip]
    L.dpm_advection_rhs_scalar.argtypes = [vp, C.c_int, dp, dp, dp, dp, dp]
    L.dpm_viscous_rhs_scalar.argtypes = [vp, dp, C.c_double, dp, C.c_double, dp, dp, dp]
    L.dpm_upload_scalars.argtypes = [vp, dp]
    fp = C.POINTER(C.c_float)
    L.dpm_learn_collect.argtypes = [vp, C.c_int, ip]
    L.dpm_learn_train.argtypes = [vp, C.c_int, C.c_double, C.POINTER(abi.LearnReportT)]
    L.dpm_learn_set_gamma.argtypes = [vp, C.c_double]
    L.dpm_learn_sizes.argtypes = [vp, ip]
    L.dpm_multilevel_hierarchy.argtypes = [C.c_int, C.c_int, ip, dp, C.c_int, C.c_int, ip, C.POINTER(C.c_longlong),
                                           C.c_int]
    L.dpm_multilevel_digest.argtypes = [C.c_int, C.c_int, ip, dp, C.c_int, C.c_int, C.POINTER(C.c_ulonglong)]
    L.dpm_learn_export.argtypes = [vp, fp, C.c_void_p, ip, dp, dp, dp, dp, dp, fp]
    L.dpm_learn_loss_grad.argtypes = [vp, fp, dp, fp]
    L.dpm_download_scalars.argtypes = [vp, dp]
    L.fvm_petsc_solve_pressure.argtypes = [C.c_int, C.c_int, C.c_int, ip, ip, ip, ip, ip, dp, dp, dp, C.c_int,
                                           C.c_int, C.c_double, C.c_double, ip, dp, C.c_int, dp, ip, dp]
    L.fvm_petsc_set_pressure_solver.argtypes = [C.c_char_p]
    L.fvm_petsc_insert_option.argtypes = [C.c_char_p]
    L.fvm_petsc_set_io_on_device.argtypes = [C.c_int]
    L.fvm_petsc_set_device_local_rank.argtypes = [C.c_int]
    L.dpm_pcg_solve_noalloc.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_int,
                                        C.c_int, vp, ip, dp]
    L.dpm_setup_times.argtypes = [vp, dp]
    L.dpm_create_poly.argtypes = [C.POINTER(abi.PolyMeshT), C.POINTER(abi.PatchCfgT), C.POINTER(abi.ParamsT), C.c_int,
                                  C.POINTER(vp)]
    L.dpm_fcg_phase_times.argtypes = [vp, C.c_int, dp]
    L.dpm_setup_compare.argtypes = [C.POINTER(abi.RawMeshT), C.POINTER(abi.PatchCfgT), C.POINTER(abi.ParamsT),
                                    C.c_int, C.POINTER(C.c_int64), dp, dp]
    L.dpm_setup_compare_poly.argtypes = [C.POINTER(abi.PolyMeshT), C.POINTER(abi.PatchCfgT), C.POINTER(abi.ParamsT),
                                         C.c_int, C.POINTER(C.c_int64), dp, dp]
    L.dpm_setup_array_name.argtypes = [C.c_int]
    L.dpm_setup_array_name.restype = C.c_char_p
    for name, mt in (("dpm_setup_host_digest", abi.RawMeshT), ("dpm_setup_host_digest_poly", abi.PolyMeshT)):
        getattr(L, name).argtypes = [C.POINTER(mt), C.POINTER(abi.PatchCfgT), C.POINTER(abi.ParamsT),
                                     C.POINTER(C.c_uint64), C.POINTER(C.c_int), C.POINTER(C.c_uint64), C.c_char_p,
                                     C.c_int]
    _lib = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _check(rc, what):
    if rc != 0:
        raise DopamineError(f"{what} failed with status {rc}", rc)


class Solver:
    """Device-resident RK3W solver on one GPU for a dopamine_b200.cases.Case."""

    def __init__(self, case, device=0, params=None):
        L = lib()
        self.case = case
        self._patches = abi.patch_cfgs(case.patches)
        self.params = params if params is not None else case.make_params()
        h = C.c_void_p()
        from .cases import PolyMesh
        if isinstance(case.mesh, PolyMesh):  # OpenFOAM-style face-based mesh
            self._mesh = abi.PolyMeshView(case.mesh)
            _check(L.dpm_create_poly(C.byref(self._mesh.struct), self._patches, C.byref(self.params), device,
                                     C.byref(h)), "dpm_create_poly")
        else:
            self._mesh = abi.RawMeshView(case.mesh)
            _check(L.dpm_create(C.byref(self._mesh.struct), self._patches, C.byref(self.params), device,
                                C.byref(h)), "dpm_create")
        self.h = h
        nc, nf, nb = C.c_int64(), C.c_int64(), C.c_int64()
        L.dpm_n_cells(self.h, C.byref(nc), C.byref(nf), C.byref(nb))
        self.nc, self.nf, self.nb = nc.value, nf.value, nb.value
        self.centroid = np.zeros((self.nc, 3))
        self.volume = np.zeros(self.nc)
        L.dpm_cell_geometry(self.h, _p(self.centroid), _p(self.volume))

    SETUP_KEYS = ("mesh_ms", "ops_ms", "upload_ms", "total_ms", "raw_upload_ms", "match_ms", "faces_ms",
                  "periodic_ms", "stencil_ms", "pressure_ops_ms", "cell_ops_ms", "psolver_ms")

    def setup_times(self):
        """Wall-clock milliseconds of this handle's set-up (dpm_setup_times)."""
        ms = np.zeros(len(self.SETUP_KEYS))
        _check(lib().dpm_setup_times(self.h, _p(ms)), "dpm_setup_times")
        return dict(zip(self.SETUP_KEYS, ms.tolist()))

    FCG_PHASES = ("coarse", "smoother", "publish_z_barrier", "w_Az_sums", "reduce_gather", "update")

    def fcg_phase_times(self, enable=True):
        """Two-level kernel phase times recorded since the last call (mean us per iteration by
        phase, and the iteration count); enable=False stops the recording."""
        us = np.zeros(8)
        _check(lib().dpm_fcg_phase_times(self.h, 1 if enable else 0, _p(us)), "dpm_fcg_phase_times")
        out = dict(zip(self.FCG_PHASES, us[:6].tolist()))
        out["iterations"] = int(us[7])
        return out

    def close(self):
        if getattr(self, "h", None):
            lib().dpm_destroy(self.h)
            self.h = None

    __del__ = close

    def to_device(self, U=None, p=None, T=None):
        U = None if U is None else np.ascontiguousarray(U, dtype=np.float64)
        p = None if p is None else np.ascontiguousarray(p, dtype=np.float64)
        T = None if T is None else np.ascontiguousarray(T, dtype=np.float64)
        _check(lib().dpm_upload_state(self.h, _p(U), _p(p), _p(T)), "dpm_upload_state")

    def sync_host(self):
        U = np.zeros((self.nc, 3)); p = np.zeros(self.nc); T = np.zeros(self.nc); nu = np.zeros(self.nc)
        _check(lib().dpm_download_state(self.h, _p(U), _p(p), _p(T), _p(nu)), "dpm_download_state")
        return {"U": U, "p": p, "T": T, "nu_sgs": nu}

    def face_flux(self):
        ff = np.zeros(self.nf)
        _check(lib().dpm_download_face_flux(self.h, _p(ff)), "dpm_download_face_flux")
        return ff

    def grad_U(self):
        g = np.zeros((self.nc, 3, 3))
        _check(lib().dpm_download_gradient(self.h, _p(g)), "dpm_download_gradient")
        return g

    def project_once(self, dt):
        _check(lib().dpm_project_once(self.h, dt), "dpm_project_once")

    def initialise(self):
        """apply_initial_conditions (src/init/mod_initconditions.f90:38-112): profile, optional noise
        with an extra projection, then project_once at dt_proj = gamma_1 dt."""
        U = self.case.initial_velocity(self.centroid)
        self.to_device(U=U, p=np.zeros(self.nc))
        dtp = 8.0 / 15.0 * self.params.dt
        if self.case.noise > 0.0:
            self.project_once(dtp)
        self.project_once(dtp)

    def advance(self, dt=None):
        _check(lib().dpm_advance(self.h, self.params.dt if dt is None else dt), "dpm_advance")

    def advance_n(self, n, dt=None):
        _check(lib().dpm_advance_n(self.h, self.params.dt if dt is None else dt, n), "dpm_advance_n")

    def compute_dt(self):
        v = C.c_double()
        _check(lib().dpm_compute_dt(self.h, C.byref(v)), "dpm_compute_dt")
        return v.value

    def state_is_finite(self):
        ok = C.c_int()
        _check(lib().dpm_state_is_finite(self.h, C.byref(ok)), "dpm_state_is_finite")
        return bool(ok.value)

    def stats(self):
        s = abi.StatsT()
        _check(lib().dpm_stats(self.h, C.byref(s)), "dpm_stats")
        return s.as_dict()

    def last_timing(self):
        a, b = C.c_double(), C.c_double()
        lib().dpm_last_timing(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def kernel_launches(self):
        n = C.c_int64()
        lib().dpm_kernel_launches(self.h, C.byref(n))
        return n.value

    def select_pressure_solver(self, p_solver):
        """Plain Jacobi-PCG (abi.PSOLVER_JACOBI_PCG) or back to the form the handle was created with."""
        _check(lib().dpm_select_pressure_solver(self.h, int(p_solver)), "dpm_select_pressure_solver")

    def set_barrier_spin_limit(self, spins):
        """Poll limit of the Krylov kernels' grid-wide waits (0: the default, about a second)."""
        _check(lib().dpm_set_barrier_spin_limit(self.h, int(spins)), "dpm_set_barrier_spin_limit")

    @property
    def time(self):
        v = C.c_double()
        lib().dpm_get_time(self.h, C.byref(v))
        return v.value

    # ---- per-operator entry points ----------------------------------------------------------
    def ls_gradient_vector(self, U, U_bnd):
        g = np.zeros((self.nc, 3, 3))
        _check(lib().dpm_ls_gradient_vector(self.h, _p(np.ascontiguousarray(U)), _p(np.ascontiguousarray(U_bnd)),
                                            _p(g)), "dpm_ls_gradient_vector")
        return g

    def advection_rhs_vector(self, scheme, U, U_bnd, face_flux, grad_U):
        r = np.zeros((self.nc, 3))
        _check(lib().dpm_advection_rhs_vector(self.h, scheme, _p(np.ascontiguousarray(U)),
                                              _p(np.ascontiguousarray(U_bnd)), _p(np.ascontiguousarray(face_flux)),
                                              _p(np.ascontiguousarray(grad_U)), _p(r)), "dpm_advection_rhs_vector")
        return r

    def viscous_rhs_vector(self, U, nu, nu_sgs, grad_U, U_bnd):
        r = np.zeros((self.nc, 3))
        _check(lib().dpm_viscous_rhs_vector(self.h, _p(np.ascontiguousarray(U)), nu, _p(np.ascontiguousarray(nu_sgs)),
                                            _p(np.ascontiguousarray(grad_U)), _p(np.ascontiguousarray(U_bnd)), _p(r)),
               "dpm_viscous_rhs_vector")
        return r

    def sgs_viscosity(self, model, U, grad_U, dt_stab):
        nu = np.zeros(self.nc)
        _check(lib().dpm_sgs_viscosity(self.h, model, _p(np.ascontiguousarray(U)), None,
                                       _p(np.ascontiguousarray(grad_U)), dt_stab, _p(nu)), "dpm_sgs_viscosity")
        return nu

    def advection_rhs_scalar(self, scheme, phi, phi_bnd, face_flux, grad_phi):
        rhs = np.zeros(self.nc)
        _check(lib().dpm_advection_rhs_scalar(self.h, scheme, _p(np.ascontiguousarray(phi)),
                                              _p(np.ascontiguousarray(phi_bnd)), _p(np.ascontiguousarray(face_flux)),
                                              _p(np.ascontiguousarray(grad_phi)), _p(rhs)), "dpm_advection_rhs_scalar")
        return rhs

    def viscous_rhs_scalar(self, phi, alpha, nu_sgs, pr_t, grad_phi, phi_bnd):
        rhs = np.zeros(self.nc)
        _check(lib().dpm_viscous_rhs_scalar(self.h, _p(np.ascontiguousarray(phi)), alpha,
                                            _p(np.ascontiguousarray(nu_sgs)), pr_t, _p(np.ascontiguousarray(grad_phi)),
                                            _p(np.ascontiguousarray(phi_bnd)), _p(rhs)), "dpm_viscous_rhs_scalar")
        return rhs

    def scalars(self):
        """(T [nc], C [n_scalars, nc])."""
        ns = max(0, min(int(self.params.n_scalars), 4))
        T = self.sync_host()["T"]
        Cf = np.zeros((self.nc, ns))
        if ns:
            _check(lib().dpm_download_scalars(self.h, _p(Cf)), "dpm_download_scalars")
        return T, np.ascontiguousarray(Cf.T)

    def set_scalars(self, C):
        """C [n_scalars, nc]."""
        Cf = np.ascontiguousarray(np.asarray(C, dtype=np.float64).T)
        _check(lib().dpm_upload_scalars(self.h, _p(Cf)), "dpm_upload_scalars")

    # ---- learned term of the two-level preconditioner
    def learn_collect(self, n_steps):
        k = C.c_int(0)
        _check(lib().dpm_learn_collect(self.h, n_steps, C.byref(k)), "dpm_learn_collect")
        return k.value

    def learn_train(self, epochs=100, lr=1e-2):
        rep = abi.LearnReportT()
        _check(lib().dpm_learn_train(self.h, epochs, lr, C.byref(rep)), "dpm_learn_train")
        return rep.as_dict()

    def learn_set_gamma(self, gamma):
        _check(lib().dpm_learn_set_gamma(self.h, gamma), "dpm_learn_set_gamma")

    def learn_export(self):
        sz = (C.c_int * 7)()
        _check(lib().dpm_learn_sizes(self.h, sz), "dpm_learn_sizes")
        n, Cp, WL, WA, S, F, NP = (int(v) for v in sz)
        out = dict(n=n, C=Cp, WL=WL, WA=WA, S=S, feat=np.zeros((F, n), dtype=np.float32),
                   lpk=np.zeros((WL, n), dtype=np.uint32), col=np.zeros((WA, n), dtype=np.int32),
                   val=np.zeros((WA, n)), R=np.zeros((S, n)), Z=np.zeros((S, n)), U=np.zeros((S, n)),
                   E=np.zeros((S, n)), params=np.zeros(NP, dtype=np.float32))
        fp = C.POINTER(C.c_float)
        _check(lib().dpm_learn_export(self.h, out["feat"].ctypes.data_as(fp), out["lpk"].ctypes.data_as(C.c_void_p),
                                      out["col"].ctypes.data_as(C.POINTER(C.c_int)), _p(out["val"]), _p(out["R"]),
                                      _p(out["Z"]), _p(out["U"]), _p(out["E"]), out["params"].ctypes.data_as(fp)),
               "dpm_learn_export")
        return out

    def learn_loss_grad(self, params=None):
        fp = C.POINTER(C.c_float)
        loss = C.c_double(0.0)
        grad = np.zeros(561, dtype=np.float32)
        pa = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        _check(lib().dpm_learn_loss_grad(self.h, None if pa is None else pa.ctypes.data_as(fp), C.byref(loss),
                                         grad.ctypes.data_as(fp)), "dpm_learn_loss_grad")
        return loss.value, grad

    def wall_model(self, U, nu):
        tau = np.zeros((self.nb, 3))
        _check(lib().dpm_wall_model(self.h, _p(np.ascontiguousarray(U)), nu, _p(tau)), "dpm_wall_model")
        return tau

    # right-hand-side sources (src/abl/mod_abl_weather.f90, src/mod_scalar.f90)
    def set_nudging_profiles(self, times, z_levels, U_profile, T_profile):
        """times (nt), z_levels (nz), U_profile (nt, nz, 3), T_profile (nt, nz)."""
        t = np.ascontiguousarray(times, dtype=np.float64)
        z = np.ascontiguousarray(z_levels, dtype=np.float64)
        Up = np.ascontiguousarray(U_profile, dtype=np.float64)  # C (nt, nz, 3) = Fortran (3, nz, nt)
        Tp = np.ascontiguousarray(T_profile, dtype=np.float64)
        _check(lib().dpm_set_nudging_profiles(self.h, len(t), len(z), _p(t), _p(z), _p(Up), _p(Tp)),
               "dpm_set_nudging_profiles")

    def set_scalar_sources(self, defs):
        arr, self._src_keep = abi.scalar_sources(defs)
        _check(lib().dpm_set_scalar_sources(self.h, len(defs), arr), "dpm_set_scalar_sources")

    # checkpoint and sampling (src/io/mod_checkpoint_io.f90, src/stats/mod_sampling.f90)
    def write_checkpoint(self, checkpoint_dir, step):
        _check(lib().dpm_write_checkpoint(self.h, os.fsencode(checkpoint_dir), int(step)), "dpm_write_checkpoint")

    def read_checkpoint(self, checkpoint_dir, step=-1):
        _check(lib().dpm_read_checkpoint(self.h, os.fsencode(checkpoint_dir), int(step)), "dpm_read_checkpoint")

    def set_sample_points(self, xyz):
        """xyz (n, 3); returns the 0-based owner cell of each point."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        owner = np.zeros(len(xyz), dtype=np.int32)
        _check(lib().dpm_sampling_set_points(self.h, len(xyz), _p(xyz), owner.ctypes.data_as(C.POINTER(C.c_int))),
               "dpm_sampling_set_points")
        self._n_samples = len(xyz)
        return owner

    def sample_points(self):
        """(n, 6): U(3), p, T, nu_sgs at the points given to set_sample_points."""
        out = np.zeros((getattr(self, "_n_samples", 0), 6))
        _check(lib().dpm_sample_points(self.h, _p(out)), "dpm_sample_points")
        return out

    # exact cell projection operators (src/numerics/mod_cell_projection.f90)
    def cell_divergence(self, u):
        out = np.zeros(self.nc)
        _check(lib().dpm_cell_divergence(self.h, _p(np.ascontiguousarray(u, dtype=np.float64)), _p(out)),
               "dpm_cell_divergence")
        return out

    def cell_adjoint_gradient(self, chi):
        v = np.zeros((self.nc, 3))
        _check(lib().dpm_cell_adjoint_gradient(self.h, _p(np.ascontiguousarray(chi, dtype=np.float64)), _p(v)),
               "dpm_cell_adjoint_gradient")
        return v

    def cell_project(self, u, bconst, tol, max_it, identity_precond=False):
        u = np.array(u, dtype=np.float64, order="C", copy=True)
        n_it = C.c_int(0)
        _check(lib().dpm_cell_project(self.h, _p(u), _p(np.ascontiguousarray(bconst, dtype=np.float64)), tol, max_it,
                                      1 if identity_precond else 0, C.byref(n_it)), "dpm_cell_project")
        return u, n_it.value


def compare_setups(case, device=0, params=None):
    """Builds the case's mesh and static operators with the device and the host builders
    (dpm_setup_compare).  Returns ({array name: entries whose bits differ}, largest relative
    difference of the SGS filter tensor, {stage: ms})."""
    from .cases import PolyMesh
    L = lib()
    patches = abi.patch_cfgs(case.patches)
    prm = params if params is not None else case.make_params()
    mism = (C.c_int64 * 64)()
    g = C.c_double()
    ms = np.zeros(4)
    if isinstance(case.mesh, PolyMesh):
        mesh = abi.PolyMeshView(case.mesh)
        _check(L.dpm_setup_compare_poly(C.byref(mesh.struct), patches, C.byref(prm), device, mism, C.byref(g),
                                        _p(ms)), "dpm_setup_compare_poly")
    else:
        mesh = abi.RawMeshView(case.mesh)
        _check(L.dpm_setup_compare(C.byref(mesh.struct), patches, C.byref(prm), device, mism, C.byref(g), _p(ms)),
               "dpm_setup_compare")
    out = {}
    for k in range(64):
        name = L.dpm_setup_array_name(k)
        if name is None:
            break
        out[name.decode()] = int(mism[k])
    times = dict(zip(("host_mesh_ms", "host_ops_ms", "device_mesh_ms", "device_ops_ms"), ms.tolist()))
    return out, g.value, times


def host_setup_digests(case, params=None):
    """Builds the case's mesh and static operators with the host builder alone (no device) and
    returns ({array name: 64-bit FNV-1a digest}, digest of the SGS filter tensor)
    (dpm_setup_host_digest)."""
    from .cases import PolyMesh
    L = lib()
    patches = abi.patch_cfgs(case.patches)
    prm = params if params is not None else case.make_params()
    dig = (C.c_uint64 * 64)()
    n = C.c_int()
    g = C.c_uint64()
    err = C.create_string_buffer(512)
    if isinstance(case.mesh, PolyMesh):
        mesh = abi.PolyMeshView(case.mesh)
        rc = L.dpm_setup_host_digest_poly(C.byref(mesh.struct), patches, C.byref(prm), dig, C.byref(n), C.byref(g),
                                          err, len(err))
    else:
        mesh = abi.RawMeshView(case.mesh)
        rc = L.dpm_setup_host_digest(C.byref(mesh.struct), patches, C.byref(prm), dig, C.byref(n), C.byref(g), err,
                                     len(err))
    if rc != 0:
        raise DopamineError(f"dpm_setup_host_digest: {err.value.decode()}", rc)
    return {L.dpm_setup_array_name(k).decode(): int(dig[k]) for k in range(n.value)}, int(g.value)
