"""ctypes mirrors of the plain-C structs in include/dopamine_b200.h.

These are the only types that cross the C ABI: a raw gmsh-like mesh, per-patch boundary
configurations and the solver parameters (src/solver/mod_fv_solver.f90:solver_params_t).
"""
import ctypes as C

import numpy as np

# Boundary-condition ids (src/mod_parameters.f90:41-51)
BC_INLET, BC_OUTLET, BC_WALL_NOSLIP, BC_WALL_MODEL, BC_SLIP, BC_PERIODIC = 1, 2, 3, 4, 5, 6
BC_SYMMETRY, BC_FIXEDTEMP, BC_ZEROGRADIENT, BC_WALL_VELOCITY, BC_ABL_INLET = 7, 8, 9, 10, 11
BC_BY_NAME = {
    "inlet": BC_INLET, "outlet": BC_OUTLET, "noSlip": BC_WALL_NOSLIP, "wallModel": BC_WALL_MODEL,
    "slip": BC_SLIP, "periodic": BC_PERIODIC, "symmetry": BC_SYMMETRY, "fixedTemp": BC_FIXEDTEMP,
    "zeroGradient": BC_ZEROGRADIENT, "wallVelocity": BC_WALL_VELOCITY, "ablInlet": BC_ABL_INLET,
}

SCHEME_VANLEER_TVD, SCHEME_KOREN_TVD, SCHEME_CDS, SCHEME_KEP, SCHEME_QUICK = 1, 2, 3, 4, 5
SCHEME_BY_NAME = {"VANLEER_TVD": 1, "KOREN_TVD": 2, "CDS": 3, "KEP": 4, "QUICK": 5}
SGS_NONE, SGS_VREMAN, SGS_SMAGORINSKY, SGS_AMD = 0, 1, 2, 3
WM_LOGLAW, WM_NONE, WM_MOST = 0, 1, 2
FORM_FP64, FORM_MIXED = 0, 1
PSOLVER_JACOBI_PCG, PSOLVER_TWOLEVEL_FCG, PSOLVER_MULTILEVEL_FCG, PSOLVER_AUTO = 0, 1, 2, 3
OK, ERR_ARG, ERR_CUDA, ERR_MESH, ERR_NOT_FINITE, ERR_DT_COLLAPSE, ERR_UNSUPPORTED, ERR_BARRIER_TIMEOUT = 0, -1, -2, -3, -4, -5, -6, -7
GRAD_LEAST_SQUARES, GRAD_GREEN_GAUSS = 0, 1
CELL_PROJECTION_LS, CELL_PROJECTION_EXACT = 0, 1
SEM_DFSEM, SEM_JARRIN = 0, 1
SEM_MEAN_LOG, SEM_MEAN_POWER = 0, 1

EL_TET4, EL_HEX8, EL_PRISM6, EL_PYR5 = 4, 5, 6, 7

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_int64)


class RawMeshT(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int64), ("xyz", _dp), ("n_cells", C.c_int64), ("cell_type", _ip),
        ("cell_off", _lp), ("cell_nodes", _ip), ("n_bfaces", C.c_int64), ("bface_off", _lp),
        ("bface_nodes", _ip), ("bface_patch", _ip), ("n_patches", C.c_int),
    ]


class PolyMeshT(C.Structure):
    _fields_ = [
        ("n_points", C.c_int64), ("xyz", _dp), ("n_faces", C.c_int64), ("face_off", _lp), ("face_nodes", _ip),
        ("owner", _ip), ("n_int_faces", C.c_int64), ("neighbour", _ip), ("n_patches", C.c_int),
        ("patch_start", _lp), ("patch_nfaces", _lp),
    ]


class PatchCfgT(C.Structure):
    _fields_ = [
        ("bc_id", C.c_int), ("U_val", C.c_double * 3), ("p_val", C.c_double), ("T_val", C.c_double),
        ("scalar_mode", C.c_int * 4), ("scalar_value", C.c_double * 4), ("abl_z0_m", C.c_double),
        ("abl_z0_h", C.c_double),
    ]


class ParamsT(C.Structure):
    _fields_ = [
        ("nu", C.c_double), ("dt", C.c_double), ("cfl_max", C.c_double), ("p_tol", C.c_double),
        ("p_max_iter", C.c_int), ("scheme", C.c_int), ("sgs_model", C.c_int), ("wall_model", C.c_int),
        ("n_nonortho_corr", C.c_int), ("rhie_chow_dual", C.c_int), ("nonortho_check", C.c_int),
        ("use_rotational_projection", C.c_int), ("adapt_dt", C.c_int),
        ("pressure_min_cos_theta", C.c_double), ("f_const", C.c_double * 3), ("g", C.c_double * 3),
        ("boussinesq", C.c_int), ("beta", C.c_double), ("T_ref", C.c_double), ("alpha_T", C.c_double),
        ("Pr_t", C.c_double), ("temperature_scheme", C.c_int), ("n_scalars", C.c_int),
        ("scalar_scheme", C.c_int), ("scalar_diffusivity", C.c_double * 4), ("scalar_pr_t", C.c_double * 4),
        ("c_amd", C.c_double), ("amd_wall_gradient", C.c_int), ("wall_model_height", C.c_double),
        ("wall_model_filter_time", C.c_double), ("wall_model_filter_tf_fac", C.c_double), ("form", C.c_int),
        ("p_solver", C.c_int), ("p_smooth_degree", C.c_int), ("p_smooth_lmin", C.c_double),
        ("p_smooth_lmax", C.c_double), ("abl_z0_m", C.c_double), ("abl_z0_h", C.c_double),
        ("abl_T_surface", C.c_double), ("abl_L_obukhov", C.c_double), ("abl_compute_L", C.c_int),
        ("p_ml_degree", C.c_int), ("p_ml_overcorrect", C.c_double), ("p_ml_passes", C.c_int),
        ("gradient_scheme", C.c_int), ("gg_iterations", C.c_int), ("p_stall_window", C.c_int),
        ("p_stall_ratio", C.c_double), ("p_ml_value_bits", C.c_int), ("cell_projection", C.c_int),
        ("cell_projection_tol", C.c_double), ("constant_mass_flux_forcing", C.c_int),
        ("U_bulk_target", C.c_double * 3), ("use_harmonic_forcing", C.c_int), ("forcing_amp", C.c_double),
        ("forcing_omega", C.c_double), ("forcing_phase", C.c_double), ("forcing_dir", C.c_double * 3),
        ("use_rotation", C.c_int), ("omega_rot", C.c_double * 3), ("use_nudging", C.c_int),
        ("nudging_tau", C.c_double), ("nudging_z_start", C.c_double), ("nudging_z_full", C.c_double),
        ("nudging_horizontal_only", C.c_int), ("abl_u_ref", C.c_double), ("abl_z_ref", C.c_double),
        ("abl_T_ref", C.c_double), ("abl_wind_dir_deg", C.c_double), ("use_sem", C.c_int), ("sem_type", C.c_int),
        ("sem_n_eddies", C.c_int), ("sem_seed", C.c_int), ("sem_mean_law", C.c_int), ("sem_sigma", C.c_double),
        ("sem_alpha", C.c_double), ("sem_Iu_ref", C.c_double), ("sem_Iv_ratio", C.c_double),
        ("sem_Iw_ratio", C.c_double), ("sem_rho_uw", C.c_double), ("host_setup", C.c_int),
    ]


class ScalarSourceT(C.Structure):
    _fields_ = [
        ("enabled", C.c_int), ("scalar_id", C.c_int), ("src_kind", C.c_int), ("shape", C.c_int),
        ("time_mode", C.c_int), ("magnitude", C.c_double), ("omega", C.c_double), ("phase", C.c_double),
        ("center", C.c_double * 3), ("p0", C.c_double * 3), ("p1", C.c_double * 3), ("normal", C.c_double * 3),
        ("half_thickness", C.c_double), ("radius", C.c_double), ("box_min", C.c_double * 3),
        ("box_max", C.c_double * 3), ("tag_radius", C.c_double), ("n_tag_points", C.c_int),
        ("tag_points", C.POINTER(C.c_double)),
    ]


SRC_POINT, SRC_LINE, SRC_SURFACE, SRC_VOLUME, SRC_OBJ = 1, 2, 3, 4, 5
SHAPE_SPHERE, SHAPE_BOX, SHAPE_PLANE = 1, 2, 3
TIME_CONSTANT, TIME_HARMONIC = 1, 2


def scalar_sources(defs):
    """dicts of ScalarSourceT fields -> (ctypes array, keep-alive list); the reference's defaults
    (mod_scalar.f90:ScalarSourceDef) for what a dict leaves out."""
    arr = (ScalarSourceT * max(1, len(defs)))()
    keep = []
    for i, dd in enumerate(defs):
        s = arr[i]
        s.enabled, s.scalar_id, s.src_kind, s.shape, s.time_mode = 1, 1, SRC_VOLUME, SHAPE_SPHERE, TIME_CONSTANT
        s.normal[2] = 1.0
        for k, v in dd.items():
            if k == "tag_points":
                pts = np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
                keep.append(pts)
                s.n_tag_points = len(pts)
                s.tag_points = pts.ctypes.data_as(C.POINTER(C.c_double))
            elif isinstance(getattr(s, k), C.Array):
                for j, x in enumerate(v):
                    getattr(s, k)[j] = x
            else:
                setattr(s, k, v)
    return arr, keep


class StatsT(C.Structure):
    _fields_ = [
        ("time", C.c_double), ("E", C.c_double), ("eps", C.c_double), ("Umax", C.c_double), ("Ub", C.c_double),
        ("tauw_mean", C.c_double), ("nu_sgs_mean", C.c_double), ("max_abs_divU", C.c_double),
        ("volavg_abs_divU", C.c_double), ("dt_used", C.c_double), ("p_solves", C.c_int), ("p_iters", C.c_int),
        ("p_resid_max", C.c_double), ("p_fallbacks", C.c_int), ("p_solver_used", C.c_int),
        ("p_bytes_per_iteration", C.c_double), ("cp_iters", C.c_int), ("cp_precond_iters", C.c_int),
        ("max_abs_divU_cell", C.c_double), ("volavg_abs_divU_cell", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LearnReportT(C.Structure):
    _fields_ = [
        ("samples", C.c_int), ("val_solves", C.c_int), ("loss_initial", C.c_double), ("loss_final", C.c_double),
        ("gamma", C.c_float), ("its_val_base", C.c_int), ("its_val_learned", C.c_int), ("train_ms", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def default_params(**kw):
    """solver_params_t defaults with the numerics the regression inputs pin
    (cell_projection='LS', rhie_chow_dual, rotational projection, least-squares gradients)."""
    p = ParamsT()
    p.nu = 1.0e-5
    p.dt = 1.0e-3
    p.cfl_max = 0.5
    p.p_tol = 1.0e-10
    p.p_max_iter = 1000
    p.scheme = SCHEME_KEP
    p.sgs_model = SGS_NONE
    p.wall_model = WM_LOGLAW
    p.n_nonortho_corr = 0
    p.rhie_chow_dual = 1
    p.nonortho_check = 0
    p.use_rotational_projection = 1
    p.adapt_dt = 0
    p.pressure_min_cos_theta = 0.0
    p.boussinesq = 0
    p.beta = 3.4e-3
    p.T_ref = 300.0
    p.alpha_T = 1.4e-5
    p.Pr_t = 0.85
    p.temperature_scheme = SCHEME_VANLEER_TVD
    p.n_scalars = 0
    p.scalar_scheme = SCHEME_VANLEER_TVD
    p.c_amd = 1.0 / 3.0
    p.amd_wall_gradient = 1
    p.form = FORM_FP64
    p.p_solver = PSOLVER_JACOBI_PCG
    p.p_smooth_degree = 7
    p.p_smooth_lmin = 0.05
    p.p_smooth_lmax = 2.0
    p.abl_z0_m = 0.1
    p.abl_z0_h = 0.01
    p.abl_T_surface = 300.0
    p.abl_L_obukhov = 0.0
    p.abl_compute_L = 1
    p.p_ml_degree = 0  # library default: 2 in the multi-kernel form (>= 2^20 cells), 3 in the persistent one
    p.p_ml_overcorrect = 1.6
    p.p_ml_passes = 3
    p.gradient_scheme = GRAD_LEAST_SQUARES
    p.gg_iterations = 2
    p.cell_projection = CELL_PROJECTION_LS
    p.cell_projection_tol = 0.1
    p.forcing_dir[0] = 1.0
    p.nudging_tau = 1800.0
    p.nudging_horizontal_only = 1
    p.abl_u_ref, p.abl_z_ref, p.abl_T_ref, p.abl_wind_dir_deg = 8.0, 100.0, 300.0, 270.0
    p.use_sem, p.sem_type, p.sem_n_eddies, p.sem_seed, p.sem_mean_law = 0, SEM_DFSEM, 500, 0, SEM_MEAN_LOG
    p.sem_sigma, p.sem_alpha, p.sem_Iu_ref, p.sem_Iv_ratio, p.sem_Iw_ratio, p.sem_rho_uw = 0.0, 0.2, 0.0, 0.75, 0.5, -0.3
    for k, v in kw.items():
        if k in ("f_const", "g", "scalar_diffusivity", "scalar_pr_t", "U_bulk_target", "forcing_dir", "omega_rot"):
            arr = getattr(p, k)
            for i in range(len(v)):
                arr[i] = v[i]
        else:
            setattr(p, k, v)
    return p


def patch_cfgs(patches):
    """patches: list of dicts {bc: name or id, U: (3,), p: float, T: float, scalar_mode, scalar_value,
    z0_m, z0_h (MOST roughness of the patch; 0 = the global value)}."""
    arr = (PatchCfgT * max(1, len(patches)))()
    for i, pd in enumerate(patches):
        bc = pd["bc"]
        arr[i].bc_id = BC_BY_NAME[bc] if isinstance(bc, str) else int(bc)
        for k, v in enumerate(pd.get("U", (0.0, 0.0, 0.0))):
            arr[i].U_val[k] = v
        arr[i].p_val = pd.get("p", 0.0)
        arr[i].T_val = pd.get("T", 0.0)
        for k, v in enumerate(pd.get("scalar_mode", (0, 0, 0, 0))):
            arr[i].scalar_mode[k] = v
        for k, v in enumerate(pd.get("scalar_value", (0.0, 0.0, 0.0, 0.0))):
            arr[i].scalar_value[k] = v
        arr[i].abl_z0_m = pd.get("z0_m", 0.0)
        arr[i].abl_z0_h = pd.get("z0_h", 0.0)
    return arr


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class RawMeshView:
    """Keeps the numpy buffers of a RawMesh alive while its C struct is in use."""

    def __init__(self, mesh):
        self._keep = [
            np.ascontiguousarray(mesh.xyz, dtype=np.float64),
            np.ascontiguousarray(mesh.cell_type, dtype=np.int32),
            np.ascontiguousarray(mesh.cell_off, dtype=np.int64),
            np.ascontiguousarray(mesh.cell_nodes, dtype=np.int32),
            np.ascontiguousarray(mesh.bface_off, dtype=np.int64),
            np.ascontiguousarray(mesh.bface_nodes, dtype=np.int32),
            np.ascontiguousarray(mesh.bface_patch, dtype=np.int32),
        ]
        xyz, ct, co, cn, bo, bn, bp = self._keep
        self.struct = RawMeshT(
            n_nodes=xyz.shape[0], xyz=_ptr(xyz, C.c_double), n_cells=ct.shape[0], cell_type=_ptr(ct, C.c_int),
            cell_off=_ptr(co, C.c_int64), cell_nodes=_ptr(cn, C.c_int), n_bfaces=bp.shape[0],
            bface_off=_ptr(bo, C.c_int64), bface_nodes=_ptr(bn, C.c_int), bface_patch=_ptr(bp, C.c_int),
            n_patches=len(mesh.patch_names),
        )


class PolyMeshView:
    """Keeps the numpy buffers of a cases.PolyMesh alive while its C struct is in use."""

    def __init__(self, mesh):
        self._keep = [
            np.ascontiguousarray(mesh.xyz, dtype=np.float64),
            np.ascontiguousarray(mesh.face_off, dtype=np.int64),
            np.ascontiguousarray(mesh.face_nodes, dtype=np.int32),
            np.ascontiguousarray(mesh.owner, dtype=np.int32),
            np.ascontiguousarray(mesh.neighbour, dtype=np.int32),
            np.ascontiguousarray(mesh.patch_start, dtype=np.int64),
            np.ascontiguousarray(mesh.patch_nfaces, dtype=np.int64),
        ]
        xyz, fo, fn, ow, nb, ps, pn = self._keep
        self.struct = PolyMeshT(
            n_points=xyz.shape[0], xyz=_ptr(xyz, C.c_double), n_faces=ow.shape[0], face_off=_ptr(fo, C.c_int64),
            face_nodes=_ptr(fn, C.c_int), owner=_ptr(ow, C.c_int), n_int_faces=nb.shape[0],
            neighbour=_ptr(nb, C.c_int), n_patches=len(mesh.patch_names), patch_start=_ptr(ps, C.c_int64),
            patch_nfaces=_ptr(pn, C.c_int64),
        )
