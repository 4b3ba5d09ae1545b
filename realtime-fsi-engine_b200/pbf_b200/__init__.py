"""pbf_b200 — Python mirror of the reference's fluid-solver interface.

``PBFluids`` and ``SDFBoundary`` keep the member names, argument meaning and
silent no-op behaviour of the reference classes (include/fluid/PBFluids.h:88-163,
include/fluid/SDFBoundary.h:38-167); each call goes through the C ABI of
include/pbf_b200.h into the sm_100a kernels of ``libpbf_b200.so``.  Outputs that
the C++ reference returns through ``std::vector&`` out-parameters are returned
as numpy arrays here.
"""
import ctypes as C

import numpy as np

from ._capi import (BUF_KEYS, BUF_LOD, BUF_OMEGA, BUF_POS, BUF_RHO, BUF_SORTED_IDS, BUF_SORTED_KEYS, BUF_TABLE,
                    BUF_VEL, BUF_VPRED, BUF_XSTAR, NUM_PASS_SLOTS, PASS_NAMES, STAGE_DELTAP, STAGE_INTEGRATE,
                    STAGE_LAMBDA, STAGE_PREDICT, STAGE_REORDER, STAGE_SORT, STAGE_TABLE, STAGE_VORTICITY,
                    BATCH_ALL, BOPT_BLOCK, BOPT_BLOCKS_PER_SM, BOPT_NEIGHBOUR_MODE, BOPT_ORDER, BOPT_USE_GRAPH,
                    BatchTuning,
                    ContactCandidate, DerivedParams, FluidConfig, Particle, PBFError, SceneDesc, check, fvec, lib)

# numpy view of Particle (48 bytes: pos, pad0, predPos, pad1, vel, pad2)
PARTICLE_DTYPE = np.dtype([("pos", "<f4", 3), ("pad0", "<f4"), ("pred_pos", "<f4", 3), ("pad1", "<f4"),
                           ("vel", "<f4", 3), ("pad2", "<f4")])
CONTACT_DTYPE = np.dtype([("pos", "<f4", 4), ("vel", "<f4", 4)])
assert PARTICLE_DTYPE.itemsize == 48 and CONTACT_DTYPE.itemsize == 32


def default_config():
    """FluidConfig with the reference's in-class defaults (config.h:11-62)."""
    c = FluidConfig()
    check(lib().pbf_default_config(C.byref(c)))
    return c


def derive_params(cfg, collision_padding=0.0):
    """PBFluids::setParams constants (PBFluids.cpp:39-109) as the kernels use them."""
    d = DerivedParams()
    check(lib().pbf_derive_params(C.byref(cfg), float(collision_padding), C.byref(d)))
    return d


def make_particles(pos, vel=None):
    """Particle array from (n,3) positions (predPos = pos, as spawnParticles)."""
    pos = np.asarray(pos, dtype=np.float32).reshape(-1, 3)
    out = np.zeros(len(pos), PARTICLE_DTYPE)
    out["pos"] = pos
    out["pred_pos"] = pos
    if vel is not None:
        out["vel"] = np.asarray(vel, dtype=np.float32).reshape(-1, 3)
    return out


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class SDFBoundary:
    """Signed-distance boundary (include/fluid/SDFBoundary.h:38-167).

    The grid, the LBVH over the faces and the closest-triangle queries live on
    the GPU in a handle owned by this object.  ``uploadToGPU`` and
    ``uploadDirtyRegion`` are no-ops: the field is computed where it is used.
    """

    def __init__(self, device=0):
        self._h = C.c_void_p()
        check(lib().pbf_create(C.byref(default_config()), int(device), C.byref(self._h)))
        self._nv = 0
        self._faces = None
        self._resolution = None
        self._build_verts = None

    def __del__(self):
        try:
            if self._h:
                lib().pbf_destroy(self._h)
                self._h = C.c_void_p()
        except Exception:
            pass

    # ---- build / refit ------------------------------------------------------
    def buildFromMesh(self, verts, faces, resolution, verbose=False):
        """A build of the same faces at the same resolution as the last one (a
        deforming mesh's periodic rebuild) runs entirely on the GPU
        (pbf_rebuild_mesh); any other build starts from the face list."""
        v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
        f = np.ascontiguousarray(faces, dtype=np.int32).reshape(-1, 3)
        if (self._faces is not None and float(resolution) == self._resolution and len(v) == self._nv
                and np.array_equal(f, self._faces)):
            check(lib().pbf_rebuild_mesh(self._h, _ptr(v), len(v)))
        else:
            check(lib().pbf_set_sdf_mesh(self._h, _ptr(v), len(v), _ptr(f), len(f), float(resolution)))
            self._faces = f
            self._resolution = float(resolution)
        self._nv = len(v)
        self._build_verts = v.copy()
        if verbose:
            d = self.dimensions()
            print(f"SDF computed: {d[0]}x{d[1]}x{d[2]} ({int(np.prod(d))} voxels, {len(f)} triangles, LBVH)")

    def refitFromMesh(self, verts):
        if self._nv == 0:
            return
        v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
        check(lib().pbf_update_mesh_vertices(self._h, _ptr(v), len(v)))
        self._build_verts = v.copy()

    def refitDirty(self, newVerts, bandRadius, moveEps):
        """SDFBoundary::refitDirty (SDFBoundary.cpp:467-558).  The GPU recomputes
        the whole grid (the reference's authoritative full pass, which its
        debug verification compares the dirty voxels against); returns whether
        any vertex moved by more than moveEps."""
        v = np.ascontiguousarray(newVerts, dtype=np.float64).reshape(-1, 3)
        if self._nv == 0 or self._build_verts is None or len(v) != len(self._build_verts):
            self.refitFromMesh(v)
            return True
        moved = bool((((v - self._build_verts) ** 2).sum(1) > moveEps * moveEps).any())
        self.refitFromMesh(v)
        return moved

    def uploadToGPU(self):
        pass

    def uploadDirtyRegion(self):
        pass

    # ---- queries -------------------------------------------------------------
    def valid(self):
        return self._nv > 0

    def _info(self):
        dims = (C.c_int32 * 3)()
        org = (C.c_double * 3)()
        cell = C.c_double()
        check(lib().pbf_sdf_grid_info(self._h, dims, org, C.byref(cell)))
        return tuple(dims), tuple(org), cell.value

    def origin(self):
        return np.array(self._info()[1])

    def cellSize(self):
        return self._info()[2]

    def dimensions(self):
        return np.array(self._info()[0], dtype=np.int32)

    def distances(self):
        d = self.dimensions()
        out = np.empty(int(np.prod(d)), np.float32)
        check(lib().pbf_read_sdf_grid(self._h, _ptr(out), out.size))
        return out

    def index(self, x, y, z):
        d = self.dimensions()
        return int(x) * int(d[1]) * int(d[2]) + int(y) * int(d[2]) + int(z)

    def closestTriangle(self, p):
        """(face, point) of the nearest surface point; face = -1 without a mesh."""
        if self._nv == 0:
            return -1, np.zeros(3, np.float32)
        faces, pts = self.closest_many(np.asarray(p, np.float32).reshape(1, 3))
        return int(faces[0]), pts[0]

    def closest_many(self, pts):
        pts = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 3)
        face = np.empty(len(pts), np.int32)
        point = np.empty((len(pts), 3), np.float32)
        check(lib().pbf_closest_triangle(self._h, _ptr(pts), len(pts), _ptr(face), _ptr(point)))
        return face, point

    def sample(self, pts, grad=False):
        pts = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 3)
        d = np.empty(len(pts), np.float32)
        g = np.empty((len(pts), 3), np.float32) if grad else None
        check(lib().pbf_sample_sdf(self._h, _ptr(pts), len(pts), _ptr(d), _ptr(g) if grad else None))
        return (d, g) if grad else d


class GridSDF:
    """A pre-sampled SDF grid (reference CPU order index = x*dy*dz + y*dz + z)
    held on the GPU, for analytic obstacles such as the benchmark capsule."""

    def __init__(self, dist, origin, cell, device=0):
        self._h = C.c_void_p()
        check(lib().pbf_create(C.byref(default_config()), int(device), C.byref(self._h)))
        d = np.ascontiguousarray(dist, dtype=np.float32)
        dims = (C.c_int32 * 3)(*d.shape)
        check(lib().pbf_set_sdf_grid(self._h, _ptr(d), dims, fvec(origin), float(cell)))
        self._shape = d.shape

    def __del__(self):
        try:
            if self._h:
                lib().pbf_destroy(self._h)
                self._h = C.c_void_p()
        except Exception:
            pass

    def valid(self):
        return True


class PBFluids:
    """Position-based fluids solver (include/fluid/PBFluids.h:88-163)."""

    def __init__(self, p=None, device=0):
        self._h = C.c_void_p()
        self._cfg = p if p is not None else default_config()
        check(lib().pbf_create(C.byref(self._cfg), int(device), C.byref(self._h)))
        self._particles = np.zeros(0, PARTICLE_DTYPE)
        self._sdf = None
        self._n = 0

    def __del__(self):
        self.close()

    def close(self):
        try:
            if self._h:
                lib().pbf_destroy(self._h)
                self._h = C.c_void_p()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # ---- construction / parameters ------------------------------------------------
    def setParams(self, p):
        self._cfg = p
        check(lib().pbf_set_params(self._h, C.byref(p)))

    def params(self):
        c = FluidConfig()
        check(lib().pbf_get_params(self._h, C.byref(c)))
        return c

    def derived(self):
        d = DerivedParams()
        check(lib().pbf_get_derived(self._h, C.byref(d)))
        return d

    def setCameraPos(self, pos):
        check(lib().pbf_set_camera_pos(self._h, fvec(pos)))

    def setCollisionPadding(self, p):
        check(lib().pbf_set_collision_padding(self._h, float(p)))

    def setBounds(self, minBound, maxBound, damping=0.0):
        check(lib().pbf_set_bounds(self._h, fvec(minBound), fvec(maxBound), float(damping)))

    # ---- particles ---------------------------------------------------------------------
    def setParticles(self, particles):
        ps = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        self._particles = ps.copy()
        self._n = len(ps)
        check(lib().pbf_set_particles(self._h, _ptr(ps) if len(ps) else None, len(ps)))

    def particles(self):
        """Host copy from setParticles (stale after step(), as the reference)."""
        return self._particles

    def readbackParticles(self, out=None):
        """Current GPU state as a Particle array (fills `out` when given, e.g.
        a pinned host buffer of PARTICLE_DTYPE)."""
        if out is None:
            out = np.zeros(self._n, PARTICLE_DTYPE)
        if len(out) != self._n:
            raise PBFError(-1, f"readbackParticles: buffer holds {len(out)}, scene {self._n}")
        if self._n:
            check(lib().pbf_read_particles(self._h, _ptr(out), self._n))
        return out

    def uploadParticles(self, particles):
        """Refresh the state from host memory (same count; asynchronous)."""
        ps = particles if particles.dtype == PARTICLE_DTYPE else np.ascontiguousarray(particles, PARTICLE_DTYPE)
        check(lib().pbf_upload_particles(self._h, _ptr(ps), len(ps)))

    def bindParticlesForRendering(self):
        """Device pointers of the committed state (float4 pos, float4 vel)."""
        p, b = C.c_void_p(), C.c_size_t()
        check(lib().pbf_buffer_device_ptr(self._h, BUF_POS, C.byref(p), C.byref(b)))
        v = C.c_void_p()
        check(lib().pbf_buffer_device_ptr(self._h, BUF_VEL, C.byref(v), C.byref(b)))
        return {"pos4": p.value, "vel4": v.value, "count": self._n}

    # ---- SDF ----------------------------------------------------------------------------
    def setSDFBoundary(self, sdf):
        """Non-owning: the caller keeps `sdf` alive (PBFluids.h:117-120)."""
        self._sdf = sdf
        check(lib().pbf_attach_sdf(self._h, sdf._h if sdf is not None else None))

    def setSDFPadding(self, padding):
        self._sdf_padding = float(padding)
        check(lib().pbf_set_sdf_mode(self._h, float(padding), 1 if getattr(self, "_sdf_cont", False) else 0))

    def setSDFContainment(self, inside):
        self._sdf_cont = bool(inside)
        check(lib().pbf_set_sdf_mode(self._h, getattr(self, "_sdf_padding", 0.0), 1 if inside else 0))

    # ---- interaction / stepping ----------------------------------------------------------------
    def setInteraction(self, active, pos):
        check(lib().pbf_set_interaction(self._h, 1 if active else 0, fvec(pos)))

    def step(self):
        check(lib().pbf_step(self._h))

    def sync(self):
        check(lib().pbf_sync(self._h))

    # ---- contacts ---------------------------------------------------------------------------------
    def filterContactCandidates(self, contactBand):
        check(lib().pbf_filter_contacts(self._h, float(contactBand)))

    def readbackContactCandidates(self):
        cnt = C.c_uint32()
        check(lib().pbf_read_contacts(self._h, None, 0, C.byref(cnt)))
        out = np.zeros(cnt.value, CONTACT_DTYPE)
        if cnt.value:
            check(lib().pbf_read_contacts(self._h, _ptr(out), cnt.value, C.byref(cnt)))
        return out[: cnt.value]

    def computeContactForces(self, band, use_vel_magnitude=True):
        """Per-vertex push forces of the current candidates on the attached mesh
        (computeContactForces, src/main.cpp:604-710) -> (forces (nv,3), contacts)."""
        if self._sdf is None or not isinstance(self._sdf, SDFBoundary):
            raise PBFError(-3, "no mesh SDF attached")
        nv = self._sdf._nv
        out = np.zeros((nv, 3), np.float32)
        c = C.c_int32()
        check(lib().pbf_vertex_forces(self._h, float(band), 1 if use_vel_magnitude else 0, _ptr(out), nv,
                                      C.byref(c)))
        return out, c.value

    # ---- engine access (tests, benchmarks) -----------------------------------------------------------
    def run_stage(self, stage, it=0):
        check(lib().pbf_run_stage(self._h, int(stage), int(it)))

    def read_buffer(self, which, dtype, shape):
        a = np.empty(shape, dtype)
        check(lib().pbf_read_buffer(self._h, int(which), _ptr(a), a.nbytes))
        return a

    def set_profiling(self, on):
        check(lib().pbf_set_profiling(self._h, 1 if on else 0))

    def pass_times(self):
        ms = (C.c_double * NUM_PASS_SLOTS)()
        cnt = (C.c_uint64 * NUM_PASS_SLOTS)()
        check(lib().pbf_read_pass_times(self._h, ms, cnt))
        return {PASS_NAMES[i]: (ms[i], cnt[i]) for i in PASS_NAMES}

    def reset_pass_times(self):
        check(lib().pbf_reset_pass_times(self._h))

    def kernel_launches(self):
        v = C.c_uint64()
        check(lib().pbf_kernel_launches(self._h, C.byref(v)))
        return v.value

    def set_use_graph(self, on):
        check(lib().pbf_set_use_graph(self._h, 1 if on else 0))

    def set_option(self, option, value):
        check(lib().pbf_set_option(self._h, int(option), int(value)))

    def list_stats(self):
        """Mode 8: (particle passes that walked the hashed buckets, drift bound
        exceeded in the last substep, window cells with a hash collision
        nearby); zeros in mode 4."""
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(lib().pbf_list_stats(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def check_finite(self):
        bad = C.c_uint32()
        rc = lib().pbf_check_finite(self._h, C.byref(bad))
        return bad.value if rc in (0, -5) else check(rc)

    def stream(self):
        s = C.c_void_p()
        check(lib().pbf_get_stream(self._h, C.byref(s)))
        return s.value


class Batch:
    """Many independent scenes advanced by one launch per pass (pbf_batch_*).

    ``scenes`` is a list of dicts with ``n`` (particle count), ``bounds_min``,
    ``bounds_max`` and optionally ``hash_size``; the solver constants come
    from ``cfg`` and are shared.  Every scene evolves as a ``PBFluids`` with
    the same configuration would."""

    def __init__(self, cfg, scenes, device=0):
        self._b = C.c_void_p()
        self._cfg = cfg
        descs = (SceneDesc * len(scenes))()
        for k, s in enumerate(scenes):
            descs[k].num_particles = int(s["n"])
            descs[k].hash_size = int(s.get("hash_size", 0))
            descs[k].bounds_min[:] = [float(v) for v in s["bounds_min"]]
            descs[k].bounds_max[:] = [float(v) for v in s["bounds_max"]]
        check(lib().pbf_batch_create(C.byref(cfg), C.cast(descs, C.c_void_p), len(scenes), int(device),
                                     C.byref(self._b)))
        self.num_scenes, self.total = self.info()

    def __del__(self):
        self.close()

    def close(self):
        try:
            if self._b:
                lib().pbf_batch_destroy(self._b)
                self._b = C.c_void_p()
        except Exception:
            pass

    @property
    def handle(self):
        return self._b

    def info(self):
        ns, nt = C.c_uint32(), C.c_uint32()
        check(lib().pbf_batch_info(self._b, C.byref(ns), C.byref(nt)))
        return ns.value, nt.value

    def scene_range(self, k):
        off, cnt = C.c_uint32(), C.c_uint32()
        check(lib().pbf_batch_scene_range(self._b, int(k), C.byref(off), C.byref(cnt)))
        return off.value, cnt.value

    def _count(self, k):
        return self.total if k == BATCH_ALL else self.scene_range(k)[1]

    def set_collision_padding(self, pad):
        check(lib().pbf_batch_set_collision_padding(self._b, float(pad)))

    def set_particles(self, k, particles):
        ps = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        check(lib().pbf_batch_set_particles(self._b, int(k), _ptr(ps) if len(ps) else None, len(ps)))

    def read_particles(self, k=BATCH_ALL, out=None):
        n = self._count(k)
        if out is None:
            out = np.zeros(n, PARTICLE_DTYPE)
        check(lib().pbf_batch_read_particles(self._b, int(k), _ptr(out) if n else None, len(out)))
        return out

    def set_sdf_grid(self, k, dist, origin, cell):
        g = np.ascontiguousarray(dist, dtype=np.float32)
        dims = (C.c_int32 * 3)(*g.shape)
        check(lib().pbf_batch_set_sdf_grid(self._b, int(k), _ptr(g), dims, fvec(origin), float(cell)))

    def set_sdf_mode(self, k, padding, containment=False):
        check(lib().pbf_batch_set_sdf_mode(self._b, int(k), float(padding), 1 if containment else 0))

    def clear_sdf(self, k):
        check(lib().pbf_batch_clear_sdf(self._b, int(k)))

    def step(self):
        check(lib().pbf_batch_step(self._b))

    def sync(self):
        check(lib().pbf_batch_sync(self._b))

    def stream(self):
        s = C.c_void_p()
        check(lib().pbf_batch_get_stream(self._b, C.byref(s)))
        return s.value

    def device_ptrs(self):
        p, v = C.c_void_p(), C.c_void_p()
        check(lib().pbf_batch_device_ptrs(self._b, C.byref(p), C.byref(v)))
        return p.value, v.value

    def kernel_launches(self):
        c = C.c_uint64()
        check(lib().pbf_batch_kernel_launches(self._b, C.byref(c)))
        return c.value

    def set_option(self, option, value):
        check(lib().pbf_batch_set_option(self._b, int(option), int(value)))

    def get_option(self, option):
        v = C.c_int()
        check(lib().pbf_batch_get_option(self._b, int(option), C.byref(v)))
        return v.value

    def autotune(self, trial_steps=3):
        """Pick the neighbour mode (dense windows or hashed buckets) and, for
        the buckets, block size, cell order and persistence by timing; returns
        (best, [all candidates]) as dicts.  The particle state is restored."""
        best = BatchTuning()
        res = (BatchTuning * 32)()
        cnt = C.c_uint32()
        check(lib().pbf_batch_autotune(self._b, int(trial_steps), C.byref(best), C.cast(res, C.c_void_p), 32,
                                       C.byref(cnt)))

        def d(t):
            return dict(block=t.block, order=t.order, blocks_per_sm=t.blocks_per_sm, ms_per_step=t.ms_per_step,
                        neighbour_mode=t.neighbour_mode)

        return d(best), [d(res[i]) for i in range(cnt.value)]

    # ---- differentiable step (pbf_batch_forward_record / pbf_batch_backward) ----
    def set_sdf_offset(self, k, t):
        check(lib().pbf_batch_set_sdf_offset(self._b, int(k), fvec(t)))

    def set_state(self, pos4_ptr, vel4_ptr):
        """State from n float4 arrays (device or host addresses)."""
        check(lib().pbf_batch_set_state(self._b, C.c_void_p(pos4_ptr), C.c_void_p(vel4_ptr)))

    def get_state(self, pos4_ptr, vel4_ptr):
        check(lib().pbf_batch_get_state(self._b, C.c_void_p(pos4_ptr), C.c_void_p(vel4_ptr)))

    def forward_record(self):
        check(lib().pbf_batch_forward_record(self._b))

    def backward(self, gpos4_ptr, gvel4_ptr, out_gpos4_ptr, out_gvel4_ptr):
        """Adjoint of the recorded step; returns dL/d(SDF translation) as a
        (num_scenes, 3) float32 array."""
        gt = np.zeros((self.num_scenes, 3), np.float32)
        check(lib().pbf_batch_backward(self._b, C.c_void_p(gpos4_ptr), C.c_void_p(gvel4_ptr),
                                       C.c_void_p(out_gpos4_ptr), C.c_void_p(out_gvel4_ptr),
                                       gt.ctypes.data_as(C.POINTER(C.c_float))))
        return gt


def sort_keys(keys, key_bits):
    """Stable (key, id) radix sort on the GPU (the CS_Radix* contract)."""
    k = np.ascontiguousarray(keys, dtype=np.uint32)
    sk = np.empty_like(k)
    ids = np.empty_like(k)
    check(lib().pbf_sort_keys(_ptr(k), len(k), int(key_bits), _ptr(sk), _ptr(ids)))
    return sk, ids


def build_table(sorted_keys, hash_size):
    """CS_BuildOffsets on the GPU -> (hash_size, 2) int32 (start, end)."""
    k = np.ascontiguousarray(sorted_keys, dtype=np.uint32)
    t = np.empty((int(hash_size), 2), np.int32)
    check(lib().pbf_build_table(_ptr(k) if len(k) else None, len(k), int(hash_size), _ptr(t)))
    return t


__all__ = [
    "PBFluids", "SDFBoundary", "GridSDF", "FluidConfig", "DerivedParams", "Particle", "ContactCandidate",
    "PARTICLE_DTYPE", "CONTACT_DTYPE", "default_config", "derive_params", "make_particles", "sort_keys",
    "build_table", "PBFError", "lib", "Batch", "SceneDesc", "BATCH_ALL", "BOPT_BLOCK", "BOPT_ORDER",
    "BOPT_BLOCKS_PER_SM", "BOPT_USE_GRAPH", "BOPT_NEIGHBOUR_MODE",
    "STAGE_PREDICT", "STAGE_SORT", "STAGE_TABLE", "STAGE_REORDER", "STAGE_LAMBDA", "STAGE_DELTAP",
    "STAGE_INTEGRATE", "STAGE_VORTICITY", "BUF_KEYS", "BUF_SORTED_KEYS", "BUF_SORTED_IDS", "BUF_TABLE",
    "BUF_XSTAR", "BUF_VPRED", "BUF_RHO", "BUF_OMEGA", "BUF_POS", "BUF_VEL", "BUF_LOD",
]
