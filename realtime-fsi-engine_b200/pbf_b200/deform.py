"""Host deformation solver (pbf_deform_*): the reference's LaplacianDeformation
and its per-frame handle driver, the consumer of the fluid's vertex forces.

    d = Deformer(verts, faces)            # rest mesh (FP64)
    for v in anchors: d.add_anchor(v)
    moved = d.step(forces, dt, params)    # one frame (src/main.cpp:870-944)
    verts = d.vertices()
"""
import ctypes as C

import numpy as np

from ._capi import DeformParams, check, lib


def default_params(**kw):
    p = DeformParams()
    check(lib().pbf_deform_default_params(C.byref(p)))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Deformer:
    def __init__(self, verts, faces):
        v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
        f = np.ascontiguousarray(faces, dtype=np.int32).reshape(-1, 3)
        self._d = C.c_void_p()
        check(lib().pbf_deform_create(_p(v), len(v), _p(f), len(f), C.byref(self._d)))
        self.nv = len(v)

    def __del__(self):
        try:
            if self._d:
                lib().pbf_deform_destroy(self._d)
                self._d = C.c_void_p()
        except Exception:
            pass

    def set_mode(self, use_local=True, kring=3, use_incremental=False):
        check(lib().pbf_deform_set_mode(self._d, int(bool(use_local)), int(kring), int(bool(use_incremental))))

    def add_anchor(self, v):
        check(lib().pbf_deform_add_anchor(self._d, int(v)))

    def set_control_points(self, idx, targets):
        i = np.ascontiguousarray(idx, dtype=np.int32)
        t = np.ascontiguousarray(targets, dtype=np.float64).reshape(-1, 3)
        check(lib().pbf_deform_set_control_points(self._d, _p(i) if len(i) else None, _p(t) if len(t) else None,
                                                   len(i)))

    def precompute(self):
        check(lib().pbf_deform_precompute(self._d))

    def solve(self):
        check(lib().pbf_deform_solve(self._d))

    def vertices(self):
        out = np.empty((self.nv, 3))
        check(lib().pbf_deform_vertices(self._d, _p(out), self.nv))
        return out

    def set_vertices(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
        check(lib().pbf_deform_set_vertices(self._d, _p(v), len(v)))

    def step(self, forces, dt, params):
        """One frame; returns (handle count, refactored, moved)."""
        f = np.ascontiguousarray(forces, dtype=np.float32).reshape(-1, 3)
        hc, rf, mv = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().pbf_deform_step(self._d, _p(f), len(f), float(dt), C.byref(params), C.byref(hc), C.byref(rf),
                                    C.byref(mv)))
        return hc.value, bool(rf.value), bool(mv.value)

    def patch_size(self):
        s = C.c_int32()
        check(lib().pbf_deform_patch_size(self._d, C.byref(s)))
        return s.value

    def verify_incremental(self):
        m = C.c_double()
        check(lib().pbf_deform_verify_incremental(self._d, C.byref(m)))
        return m.value
