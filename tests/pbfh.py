"""Shared helpers for the test suite (fixtures -> oracle / engine inputs)."""
import ctypes as C
import os

import numpy as np

import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))


def oracle_cfg(z):
    c = O.FluidConfig()
    for k, _ in c._fields_:
        v = z["cfg_" + k]
        if v.shape == ():
            setattr(c, k, v.item())
        else:
            getattr(c, k)[:] = list(v)
    return c


def engine_cfg(z_or_cfg):
    from pbf_b200 import FluidConfig
    c = FluidConfig()
    if isinstance(z_or_cfg, dict):
        for k, _ in c._fields_:
            v = z_or_cfg["cfg_" + k]
            if v.shape == ():
                setattr(c, k, v.item())
            else:
                getattr(c, k)[:] = list(v)
    else:
        C.memmove(C.byref(c), C.byref(z_or_cfg), C.sizeof(c))
    return c


def oracle_sdf(z):
    if "sdf_dist" not in z:
        return None
    return O.Sdf(z["sdf_dist"], z["sdf_origin"], float(z["sdf_cell"]), padding=float(z["sdf_padding"]),
                 containment=bool(z["sdf_containment"]))


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def oracle_params(z, **kw):
    cfg = oracle_cfg(z)
    camera = tuple(z["camera"]) if "camera" in z else (0.0, 0.0, 0.0)
    inter = tuple(z["interaction"]) if "interaction" in z else None
    return O.Params(cfg, camera=camera, interaction=inter)


def rel_err(a, b, floor):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))
