"""ctypes access to the FP64 oracle and the reference CPU builds.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, never by the product path.

  liboracle.so         FP64 restatement (oracle/pbf_oracle.c, sdf_oracle.c)
  liboracle32.so       the same sources with float32 storage (orc_real = float)
  _ref/libpbfref_cpu.so   reference src/fluid/Kernels.cpp + NeighborSearch.cpp
  _ref/libpbfref_glsl.so  reference compute shaders run on the CPU
  _ref/libpbfref_sdf.so   reference src/fluid/SDFBoundary.cpp (mesh SDF, BVH)
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
LIB32_PATH = os.path.join(HERE, "_build", "liboracle32.so")
REF_CPU_PATH = os.path.join(HERE, "_ref", "libpbfref_cpu.so")
REF_GLSL_PATH = os.path.join(HERE, "_ref", "libpbfref_glsl.so")
REF_SDF_PATH = os.path.join(HERE, "_ref", "libpbfref_sdf.so")

f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class FluidConfig(C.Structure):
    """pbf_fluid_config (include/pbf_b200.h)."""

    _fields_ = [
        ("dt", C.c_float), ("gravity", C.c_float * 3), ("h", C.c_float), ("rho0", C.c_float),
        ("solver_iterations", C.c_uint32), ("substep_iterations", C.c_uint32), ("eps", C.c_float),
        ("particle_count", C.c_uint32), ("spawn_min", C.c_float * 3), ("spawn_max", C.c_float * 3),
        ("spawn_random", C.c_uint32), ("spacing", C.c_float), ("initial_velocity", C.c_float * 3),
        ("bounds_min", C.c_float * 3), ("bounds_max", C.c_float * 3), ("bound_damping", C.c_float),
        ("hash_size", C.c_uint32), ("enable_scorr", C.c_uint32), ("k_corr", C.c_float),
        ("n_corr", C.c_float), ("delta_q", C.c_float), ("cohesion_strength", C.c_float),
        ("enable_viscosity", C.c_uint32), ("viscosity", C.c_float), ("interaction_radius", C.c_float),
        ("interaction_strength", C.c_float), ("enable_vorticity", C.c_uint32),
        ("vorticity_epsilon", C.c_float), ("enable_apbf", C.c_uint32), ("min_lod", C.c_uint32),
        ("max_lod", C.c_uint32), ("lod_max_dist", C.c_float),
    ]


class DerivedParams(C.Structure):
    """pbf_derived_params (include/pbf_b200.h) == FluidConfigUBO."""

    _fields_ = [
        ("bounds_min", C.c_float * 4), ("bounds_max", C.c_float * 4), ("gravity_dt", C.c_float * 4),
        ("h", C.c_float), ("rho0", C.c_float), ("eps", C.c_float), ("wq", C.c_float),
        ("k_corr", C.c_float), ("n_corr", C.c_float), ("viscosity", C.c_float), ("bound_damping", C.c_float),
        ("hash_size", C.c_uint32), ("particle_count", C.c_uint32), ("enable_scorr", C.c_uint32),
        ("enable_viscosity", C.c_uint32), ("cohesion_strength", C.c_float), ("interaction_radius", C.c_float),
        ("interaction_strength", C.c_float), ("w0_self", C.c_float), ("hash_mask", C.c_uint32),
        ("poly6_coeff", C.c_float), ("spiky_coeff", C.c_float), ("inv_rho0", C.c_float),
        ("min_lod", C.c_uint32), ("max_lod", C.c_uint32), ("lod_max_dist", C.c_float), ("enable_apbf", C.c_uint32),
    ]


def derive_f32(cfg, pad=0.0):
    """PBFluids::setParams in float32 arithmetic (src/fluid/PBFluids.cpp:39-109):
    the FluidConfigUBO the reference uploads for a FluidConfig-shaped `cfg`.
    `pad` is the collision padding that setBounds moves the walls in by (:299-306)."""
    d = DerivedParams()
    h = np.float32(cfg.h)
    PI = np.float32(3.14159265358979323846)
    for a in range(3):
        d.bounds_min[a] = np.float32(cfg.bounds_min[a]) + np.float32(pad)
        d.bounds_max[a] = np.float32(cfg.bounds_max[a]) - np.float32(pad)
        d.gravity_dt[a] = cfg.gravity[a]
    d.gravity_dt[3] = np.float32(cfg.dt) / np.float32(cfg.substep_iterations)
    dq = np.float32(cfg.delta_q) * h
    h2 = h * h
    r2 = dq * dq + np.float32(0) * np.float32(0) + np.float32(0) * np.float32(0)
    if r2 > h2:
        d.wq = 0.0
    else:
        h4 = h2 * h2
        h9k = h4 * h4 * h
        diff = h2 - r2
        d.wq = (np.float32(315.0) / (np.float32(64.0) * PI)) / h9k * (diff * diff * diff)
    d.h, d.rho0, d.eps = cfg.h, cfg.rho0, cfg.eps
    d.k_corr, d.n_corr, d.viscosity = cfg.k_corr, cfg.n_corr, cfg.viscosity
    d.bound_damping = min(max(np.float32(cfg.bound_damping), np.float32(0)), np.float32(1))
    d.hash_size, d.particle_count = cfg.hash_size, cfg.particle_count
    d.enable_scorr, d.enable_viscosity = cfg.enable_scorr, cfg.enable_viscosity
    d.cohesion_strength = cfg.cohesion_strength
    d.interaction_radius, d.interaction_strength = cfg.interaction_radius, cfg.interaction_strength
    h3 = h2 * h
    h6 = h3 * h3
    h9 = h6 * h3
    d.w0_self = (np.float32(315.0) / (np.float32(64.0) * PI)) / h3
    d.poly6_coeff = np.float32(315.0) / (np.float32(64.0) * PI * h9)
    d.spiky_coeff = np.float32(45.0) / (PI * h6)
    d.inv_rho0 = np.float32(1.0) / np.float32(cfg.rho0)
    d.hash_mask = cfg.hash_size - 1
    d.min_lod = cfg.min_lod if cfg.enable_apbf else cfg.solver_iterations
    d.max_lod = cfg.max_lod if cfg.enable_apbf else cfg.solver_iterations
    d.lod_max_dist = cfg.lod_max_dist
    d.enable_apbf = cfg.enable_apbf
    return d


class OrcParams(C.Structure):
    _fields_ = [
        ("bmin", C.c_double * 3), ("bmax", C.c_double * 3), ("g", C.c_double * 3), ("dt", C.c_double),
        ("h", C.c_double), ("h2", C.c_double), ("rho0", C.c_double), ("eps", C.c_double), ("wq", C.c_double),
        ("k_corr", C.c_double), ("n_corr", C.c_double), ("viscosity", C.c_double), ("damping", C.c_double),
        ("cohesion", C.c_double), ("i_radius", C.c_double), ("i_strength", C.c_double),
        ("w0_self", C.c_double), ("poly6", C.c_double), ("spiky", C.c_double), ("inv_rho0", C.c_double),
        ("vort_eps", C.c_double), ("lod_max_dist", C.c_double),
        ("hash_size", C.c_uint32), ("mask", C.c_uint32), ("scorr", C.c_uint32), ("visc_on", C.c_uint32),
        ("vort_on", C.c_uint32), ("apbf", C.c_uint32), ("min_lod", C.c_uint32), ("max_lod", C.c_uint32),
        ("iterations", C.c_uint32), ("substeps", C.c_uint32), ("interacting", C.c_uint32),
        ("i_pos", C.c_double * 3), ("camera", C.c_double * 3),
    ]


class OrcSdf(C.Structure):
    _fields_ = [
        ("enabled", C.c_int), ("dims", C.c_int * 3), ("origin", C.c_double * 3), ("cell", C.c_double),
        ("dist", C.POINTER(C.c_float)), ("padding", C.c_double), ("containment", C.c_int),
    ]


class ContactCandidate(C.Structure):
    _fields_ = [("pos", C.c_float * 4), ("vel", C.c_float * 4)]


def build():
    """Compile liboracle.so (and the reference builds when the tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    ref = os.environ.get("PBF_REFERENCE_TREE") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
    if os.path.isdir(ref):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref}"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_derive.argtypes = [C.POINTER(FluidConfig), C.c_double, C.POINTER(OrcParams)]
        L.orc_hash.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_uint32]
        L.orc_hash.restype = C.c_uint32
        L.orc_keys_f32.argtypes = [f32p, C.c_uint32, C.c_float, C.c_uint32, u32p]
        L.orc_stable_sort.argtypes = [u32p, C.c_uint32, C.c_uint32, u32p, u32p]
        L.orc_build_table.argtypes = [u32p, C.c_uint32, C.c_uint32, i32p]
        L.orc_sdf_query.argtypes = [C.POINTER(OrcSdf), f64p]
        L.orc_sdf_query.restype = C.c_double
        L.orc_sdf_gradient.argtypes = [C.POINTER(OrcSdf), f64p, f64p]
        L.orc_predict.argtypes = [C.POINTER(OrcParams), C.c_uint32, f64p, f64p, f64p, C.c_void_p]
        L.orc_lod.argtypes = [C.POINTER(OrcParams), C.c_uint32, f64p, u32p]
        L.orc_lambda.argtypes = [C.POINTER(OrcParams), C.c_uint32, f64p, u32p, i32p, C.c_void_p, C.c_uint32,
                                 f64p, C.c_void_p]
        L.orc_deltap_apply.argtypes = [C.POINTER(OrcParams), C.c_void_p, C.c_uint32, f64p, f64p, u32p, i32p,
                                       C.c_void_p, C.c_uint32, C.c_void_p]
        L.orc_integrate.argtypes = [C.POINTER(OrcParams), C.c_void_p, C.c_uint32, f64p, f64p, f64p, u32p, i32p,
                                    C.c_void_p]
        L.orc_vorticity.argtypes = [C.POINTER(OrcParams), C.c_uint32, f64p, f64p, f64p, u32p, i32p]
        L.orc_step.argtypes = [C.POINTER(OrcParams), C.c_void_p, C.c_uint32, f64p, f64p, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_adjoint_step.argtypes = [C.POINTER(OrcParams), C.c_void_p, C.c_uint32, f64p, f64p, C.c_void_p,
                                       C.c_void_p, f64p, f64p, f64p, C.c_void_p, C.c_void_p]
        L.orc_kernels.argtypes = [C.POINTER(OrcParams), f64p, C.POINTER(C.c_double), f64p]
        L.orc_neighbor_lists.argtypes = [C.POINTER(OrcParams), C.c_uint32, f64p, u32p, i32p, i32p, C.c_void_p,
                                         C.c_int32]
        L.orc_contact_filter.argtypes = [C.c_void_p, C.c_uint32, f64p, C.c_double, u32p]
        L.orc_contact_filter.restype = C.c_uint32
        L.orc_mesh_build.argtypes = [f64p, C.c_int32, i32p, C.c_int32, C.c_double]
        L.orc_mesh_build.restype = C.c_void_p
        L.orc_mesh_free.argtypes = [C.c_void_p]
        L.orc_mesh_refit.argtypes = [C.c_void_p, f64p]
        L.orc_mesh_grid_info.argtypes = [C.c_void_p, i32p, f64p, C.POINTER(C.c_double)]
        L.orc_mesh_grid.argtypes = [C.c_void_p, f32p]
        L.orc_mesh_signed_distance.argtypes = [C.c_void_p, f64p]
        L.orc_mesh_signed_distance.restype = C.c_double
        L.orc_mesh_closest.argtypes = [C.c_void_p, f64p, f64p, C.POINTER(C.c_double)]
        L.orc_mesh_closest.restype = C.c_int32
        L.orc_contact_forces.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_double, C.c_int, f64p]
        L.orc_contact_forces.restype = C.c_int32
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Params:
    """FP64 derived parameters of a FluidConfig (PBFluids::setParams)."""

    def __init__(self, cfg, collision_padding=0.0, camera=(0.0, 0.0, 0.0), interaction=None):
        self.p = OrcParams()
        lib().orc_derive(C.byref(cfg), float(collision_padding), C.byref(self.p))
        self.p.camera[:] = list(camera)
        if interaction is not None:
            self.p.interacting = 1
            self.p.i_pos[:] = list(interaction)
        self.cfg = cfg


class Sdf:
    """A sampled SDF grid for the oracle (keeps the array alive)."""

    def __init__(self, dist, origin, cell, padding=0.0, containment=False):
        self.dist = np.ascontiguousarray(dist, dtype=np.float32)
        assert self.dist.ndim == 3
        self.s = OrcSdf()
        self.s.enabled = 1
        self.s.dims[:] = list(self.dist.shape)
        self.s.origin[:] = [float(v) for v in origin]
        self.s.cell = float(cell)
        self.s.dist = self.dist.ctypes.data_as(C.POINTER(C.c_float))
        self.s.padding = float(padding)
        self.s.containment = 1 if containment else 0

    def ref(self):
        return C.byref(self.s)

    def query(self, pts):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        out = np.empty(len(pts))
        g = np.empty((len(pts), 3))
        for i, q in enumerate(pts):
            q = np.ascontiguousarray(q)
            out[i] = lib().orc_sdf_query(C.byref(self.s), q)
            gi = np.empty(3)
            lib().orc_sdf_gradient(C.byref(self.s), q, gi)
            g[i] = gi
        return out, g


def keys_f32(x4, h, mask):
    x4 = np.ascontiguousarray(x4, dtype=np.float32).reshape(-1, 4)
    keys = np.empty(len(x4), np.uint32)
    lib().orc_keys_f32(x4.reshape(-1), len(x4), float(h), int(mask), keys)
    return keys


def stable_sort(keys, hash_size):
    keys = np.ascontiguousarray(keys, dtype=np.uint32)
    sk = np.empty_like(keys)
    ids = np.empty_like(keys)
    lib().orc_stable_sort(keys, len(keys), int(hash_size), sk, ids)
    return sk, ids


def build_table(sorted_keys, hash_size):
    sk = np.ascontiguousarray(sorted_keys, dtype=np.uint32)
    t = np.empty(2 * int(hash_size), np.int32)
    lib().orc_build_table(sk, len(sk), int(hash_size), t)
    return t.reshape(-1, 2)


def step(params, pos, vel, sdf=None, want=False):
    """One PBFluids::step in FP64.  pos/vel (n,3) are updated in place."""
    n = len(pos)
    assert pos.dtype == np.float64 and vel.dtype == np.float64
    H = params.p.hash_size
    om = np.zeros((n, 3)) if want else None
    rho = np.zeros(n) if want else None
    sk = np.zeros(n, np.uint32) if want else None
    ids = np.zeros(n, np.uint32) if want else None
    tab = np.zeros(2 * H, np.int32) if want else None
    lib().orc_step(C.byref(params.p), sdf.ref() if sdf else None, n, pos.reshape(-1), vel.reshape(-1),
                   _ptr(om), _ptr(rho), _ptr(sk), _ptr(ids), _ptr(tab))
    if want:
        return dict(omega=om, rho=rho, sorted_keys=sk, sorted_ids=ids, table=tab.reshape(-1, 2))
    return None


def adjoint_step(params, pos0, vel0, gpos=None, gvel=None, sdf=None):
    """FP64 reverse-mode derivative of one step (orc_adjoint_step).  Returns
    (gpos0, gvel0, gt, pos_T, vel_T); gt is the adjoint of the SDF origin
    offset (translation)."""
    n = len(pos0)
    p0 = np.ascontiguousarray(pos0, dtype=np.float64).reshape(-1)
    v0 = np.ascontiguousarray(vel0, dtype=np.float64).reshape(-1)
    gp = None if gpos is None else np.ascontiguousarray(gpos, dtype=np.float64).reshape(-1)
    gv = None if gvel is None else np.ascontiguousarray(gvel, dtype=np.float64).reshape(-1)
    gp0 = np.zeros(3 * n)
    gv0 = np.zeros(3 * n)
    gt = np.zeros(3)
    pT = np.zeros(3 * n)
    vT = np.zeros(3 * n)
    lib().orc_adjoint_step(C.byref(params.p), sdf.ref() if sdf else None, n, p0, v0, _ptr(gp), _ptr(gv), gp0, gv0,
                           gt, _ptr(pT), _ptr(vT))
    return gp0.reshape(n, 3), gv0.reshape(n, 3), gt, pT.reshape(n, 3), vT.reshape(n, 3)


# ---- float32 build of the same restatement ------------------------------------
def _f32_fields(fields):
    return [(n, (C.c_float * t._length_) if (hasattr(t, "_length_") and t._type_ is C.c_double)
             else (C.c_float if t is C.c_double else t)) for n, t in fields]


class OrcParams32(C.Structure):
    _fields_ = _f32_fields(OrcParams._fields_)


class OrcSdf32(C.Structure):
    _fields_ = _f32_fields(OrcSdf._fields_)


_lib32 = None


def lib32():
    """liboracle32.so: the restatement with float32 storage and sequential
    sums (oracle/pbf_oracle.h, orc_real)."""
    global _lib32
    if _lib32 is None:
        if not os.path.exists(LIB32_PATH):
            build()
        L = C.CDLL(LIB32_PATH)
        L.orc_derive.argtypes = [C.POINTER(FluidConfig), C.c_float, C.POINTER(OrcParams32)]
        L.orc_step.argtypes = [C.POINTER(OrcParams32), C.c_void_p, C.c_uint32, f32p, f32p, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_adjoint_step.argtypes = [C.POINTER(OrcParams32), C.c_void_p, C.c_uint32, f32p, f32p, C.c_void_p,
                                       C.c_void_p, f32p, f32p, f32p, C.c_void_p, C.c_void_p]
        _lib32 = L
    return _lib32


class Params32:
    """Derived parameters of a FluidConfig for the float32 build."""

    def __init__(self, cfg):
        self.p = OrcParams32()
        lib32().orc_derive(C.byref(cfg), 0.0, C.byref(self.p))
        self.cfg = cfg


class Sdf32:
    def __init__(self, dist, origin, cell, padding=0.0, containment=False):
        self.dist = np.ascontiguousarray(dist, dtype=np.float32)
        self.s = OrcSdf32()
        self.s.enabled = 1
        self.s.dims[:] = list(self.dist.shape)
        self.s.origin[:] = [float(v) for v in origin]
        self.s.cell = float(cell)
        self.s.dist = self.dist.ctypes.data_as(C.POINTER(C.c_float))
        self.s.padding = float(padding)
        self.s.containment = 1 if containment else 0

    def ref(self):
        return C.byref(self.s)


def step32(params, pos, vel, sdf=None):
    """One step of the float32 build; pos/vel (n,3) float32, updated in place."""
    assert pos.dtype == np.float32 and vel.dtype == np.float32
    lib32().orc_step(C.byref(params.p), sdf.ref() if sdf else None, len(pos), pos.reshape(-1), vel.reshape(-1),
                     None, None, None, None, None)


def adjoint_step32(params, pos0, vel0, gpos=None, gvel=None, sdf=None):
    """adjoint_step in the float32 build: (gpos0, gvel0, gt) as float32."""
    n = len(pos0)
    p0 = np.ascontiguousarray(pos0, dtype=np.float32).reshape(-1)
    v0 = np.ascontiguousarray(vel0, dtype=np.float32).reshape(-1)
    gp = None if gpos is None else np.ascontiguousarray(gpos, dtype=np.float32).reshape(-1)
    gv = None if gvel is None else np.ascontiguousarray(gvel, dtype=np.float32).reshape(-1)
    gp0 = np.zeros(3 * n, np.float32)
    gv0 = np.zeros(3 * n, np.float32)
    gt = np.zeros(3, np.float32)
    lib32().orc_adjoint_step(C.byref(params.p), sdf.ref() if sdf else None, n, p0, v0, _ptr(gp), _ptr(gv), gp0, gv0,
                             gt, None, None)
    return gp0.reshape(n, 3), gv0.reshape(n, 3), gt


# ---- reference builds -------------------------------------------------------
class GlslCtx(C.Structure):
    """glsl_ref_ctx (oracle/glsl/harness.h)."""

    _fields_ = [
        ("ubo", DerivedParams), ("n", C.c_uint32), ("particles", C.c_void_p), ("solver", C.c_void_p),
        ("hash_grid", C.c_void_p), ("hash_grid_alt", C.c_void_p), ("histogram", C.c_void_p),
        ("offsets", C.c_void_p), ("lod", C.c_void_p), ("contact_count", C.c_void_p), ("contacts", C.c_void_p),
        ("is_interacting", C.c_uint32), ("interaction_pos", C.c_float * 3), ("camera_pos", C.c_float * 3),
        ("enable_vorticity", C.c_uint32), ("vorticity_epsilon", C.c_float), ("enable_sdf", C.c_uint32),
        ("sdf_mode", C.c_uint32), ("sdf_dist", C.c_void_p), ("sdf_dims", C.c_int32 * 3),
        ("sdf_origin", C.c_float * 3), ("sdf_cell", C.c_float), ("sdf_padding", C.c_float),
        ("contact_band", C.c_float), ("substeps", C.c_uint32), ("solver_iterations", C.c_uint32),
        ("sort_mode", C.c_int32), ("parallel", C.c_int32), ("pre_integrate", C.c_int32),
    ]


_ref_cpu = None
_ref_glsl = None


def ref_cpu():
    global _ref_cpu
    if _ref_cpu is None:
        L = C.CDLL(REF_CPU_PATH)
        L.ref_poly6.argtypes = [C.c_float] * 4
        L.ref_poly6.restype = C.c_float
        L.ref_grad_spiky.argtypes = [C.c_float] * 4 + [f32p]
        L.ref_scorr_kernel.argtypes = [C.c_float] * 4
        L.ref_scorr_kernel.restype = C.c_float
        L.ref_neighbor_build.argtypes = [f32p, C.c_int32, C.c_float, C.c_uint32, i32p, C.c_void_p, C.c_int32]
        L.ref_neighbor_build.restype = C.c_int64
        _ref_cpu = L
    return _ref_cpu


def ref_glsl():
    global _ref_glsl
    if _ref_glsl is None:
        L = C.CDLL(REF_GLSL_PATH)
        L.glsl_ref_stage.argtypes = [C.POINTER(GlslCtx), C.c_int, C.c_uint32]
        L.glsl_ref_step.argtypes = [C.POINTER(GlslCtx)]
        _ref_glsl = L
    return _ref_glsl


_ref_sdf = None


def ref_sdf():
    global _ref_sdf
    if _ref_sdf is None:
        L = C.CDLL(REF_SDF_PATH)
        L.sdfref_build.argtypes = [f64p, C.c_int, i32p, C.c_int, C.c_double]
        L.sdfref_build.restype = C.c_void_p
        L.sdfref_free.argtypes = [C.c_void_p]
        L.sdfref_grid_info.argtypes = [C.c_void_p, i32p, f64p, C.POINTER(C.c_double)]
        L.sdfref_grid.argtypes = [C.c_void_p, f32p]
        L.sdfref_refit.argtypes = [C.c_void_p, f64p, C.c_int]
        L.sdfref_refit_dirty.argtypes = [C.c_void_p, f64p, C.c_int, C.c_double, C.c_double]
        L.sdfref_refit_dirty.restype = C.c_int
        L.sdfref_closest.argtypes = [C.c_void_p, f32p, C.c_int, i32p, f32p]
        _ref_sdf = L
    return _ref_sdf


def have_ref_sdf():
    return os.path.exists(REF_SDF_PATH)


class RefSDF:
    """The reference's own SDFBoundary (buildFromMesh / refitFromMesh /
    refitDirty / closestTriangle) over a triangle mesh."""

    def __init__(self, verts, faces, cell):
        V = np.ascontiguousarray(verts, np.float64).reshape(-1, 3)
        F = np.ascontiguousarray(faces, np.int32).reshape(-1, 3)
        self.nv = len(V)
        self.h = ref_sdf().sdfref_build(V.reshape(-1), len(V), F.reshape(-1), len(F), float(cell))

    def __del__(self):
        if getattr(self, "h", None):
            ref_sdf().sdfref_free(self.h)
            self.h = None

    def info(self):
        dims = np.zeros(3, np.int32)
        org = np.zeros(3)
        c = C.c_double()
        ref_sdf().sdfref_grid_info(self.h, dims, org, C.byref(c))
        return dims, org, c.value

    def grid(self):
        dims = self.info()[0]
        out = np.zeros(int(np.prod(dims)), np.float32)
        ref_sdf().sdfref_grid(self.h, out)
        return out

    def refit(self, verts):
        V = np.ascontiguousarray(verts, np.float64).reshape(-1)
        ref_sdf().sdfref_refit(self.h, V, self.nv)

    def refit_dirty(self, verts, band, move_eps):
        V = np.ascontiguousarray(verts, np.float64).reshape(-1)
        return bool(ref_sdf().sdfref_refit_dirty(self.h, V, self.nv, float(band), float(move_eps)))

    def closest(self, pts):
        P = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
        face = np.zeros(len(P), np.int32)
        pt = np.zeros((len(P), 3), np.float32)
        ref_sdf().sdfref_closest(self.h, P.reshape(-1), len(P), face, pt.reshape(-1))
        return face, pt


def have_ref():
    return os.path.exists(REF_CPU_PATH) and os.path.exists(REF_GLSL_PATH)


class GlslScene:
    """Reference shaders on the CPU over GL-layout buffers."""

    def __init__(self, derived, cfg, pos, vel, sdf=None, sort_mode=0, parallel=True, pre_integrate=True,
                 interaction=None, camera=(0, 0, 0)):
        n = len(pos)
        self.n = n
        H = cfg.hash_size
        self.particles = np.zeros((n, 12), np.float32)
        self.particles[:, 0:3] = pos
        self.particles[:, 4:7] = pos
        self.particles[:, 8:11] = vel
        self.solver = np.zeros((n, 8), np.float32)
        self.hg = np.zeros((n, 2), np.uint32)
        self.hg_alt = np.zeros((n, 2), np.uint32)
        self.hist = np.zeros(256 * ((n + 255) // 256) + 1, np.uint32)
        self.offsets = np.full((H, 2), -1, np.int32)
        self.lod = np.full(n, cfg.solver_iterations, np.uint32)
        self.count = np.zeros(1, np.uint32)
        self.contacts = np.zeros((max(n, 1), 8), np.float32)
        c = GlslCtx()
        C.memmove(C.byref(c.ubo), C.byref(derived), C.sizeof(DerivedParams))
        c.ubo.particle_count = n
        c.n = n
        c.particles = _ptr(self.particles)
        c.solver = _ptr(self.solver)
        c.hash_grid = _ptr(self.hg)
        c.hash_grid_alt = _ptr(self.hg_alt)
        c.histogram = _ptr(self.hist)
        c.offsets = _ptr(self.offsets)
        c.lod = _ptr(self.lod)
        c.contact_count = _ptr(self.count)
        c.contacts = _ptr(self.contacts)
        if interaction is not None:
            c.is_interacting = 1
            c.interaction_pos[:] = list(interaction)
        c.camera_pos[:] = list(camera)
        c.enable_vorticity = cfg.enable_vorticity
        c.vorticity_epsilon = cfg.vorticity_epsilon
        if sdf is not None:
            self._sdf = sdf
            c.enable_sdf = 1
            c.sdf_mode = sdf.s.containment
            c.sdf_dist = sdf.dist.ctypes.data_as(C.c_void_p)
            c.sdf_dims[:] = list(sdf.dist.shape)
            c.sdf_origin[:] = list(sdf.s.origin)
            c.sdf_cell = sdf.s.cell
            c.sdf_padding = sdf.s.padding
        c.substeps = cfg.substep_iterations
        c.solver_iterations = cfg.solver_iterations
        c.sort_mode = sort_mode
        c.parallel = 1 if parallel else 0
        c.pre_integrate = 1 if pre_integrate else 0
        self.c = c

    def step(self):
        ref_glsl().glsl_ref_step(C.byref(self.c))

    def stage(self, stage, it=0):
        ref_glsl().glsl_ref_stage(C.byref(self.c), stage, it)

    @property
    def pos(self):
        return self.particles[:, 0:3]

    @property
    def vel(self):
        return self.particles[:, 8:11]
