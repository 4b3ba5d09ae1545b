"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, its structs have the reference layouts, and the host-side
parameter derivation equals PBFluids::setParams bit for bit."""
import ctypes as C
import os
import re

import numpy as np

import pbfh as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "pbf_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pbf_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from pbf_b200 import _capi
    L = _capi.lib()
    names = header_functions()
    assert len(names) >= 40
    for n in names:
        assert hasattr(L, n), n
    bound = {s[0] for s in _capi.SIGNATURES}
    assert set(names) == bound, set(names) ^ bound


def test_struct_layouts():
    from pbf_b200 import CONTACT_DTYPE, PARTICLE_DTYPE, ContactCandidate, DerivedParams, Particle
    assert C.sizeof(Particle) == 48          # Particle.h:8-12
    assert C.sizeof(ContactCandidate) == 32  # PBFluids.h:67-70
    assert C.sizeof(DerivedParams) == 144    # FluidConfigUBO, PBFluids.h:21-61
    assert PARTICLE_DTYPE.itemsize == 48 and CONTACT_DTYPE.itemsize == 32
    assert DerivedParams.w0_self.offset == 108 and DerivedParams.hash_mask.offset == 112


def test_batch_option_constants_and_tuning_layout_match_header():
    """The batch option numbers and pbf_batch_tuning's fields in the Python
    binding are the header's."""
    from pbf_b200 import _capi
    hdr = open(os.path.join(ROOT, "include", "pbf_b200.h")).read()
    for name in ("BLOCK", "ORDER", "BLOCKS_PER_SM", "USE_GRAPH", "NEIGHBOUR_MODE"):
        m = re.search(r"#define PBF_BOPT_%s (\d+)" % name, hdr)
        assert m and int(m.group(1)) == getattr(_capi, "BOPT_" + name), name
    body = re.search(r"typedef struct pbf_batch_tuning \{(.*?)\} pbf_batch_tuning;", hdr, re.S).group(1)
    fields = re.findall(r"(?:int32_t|float) (\w+);", body)
    assert fields == [f[0] for f in _capi.BatchTuning._fields_]
    assert C.sizeof(_capi.BatchTuning) == 4 * len(fields)


def test_default_config_matches_reference_defaults():
    import pbf_b200 as P
    c = P.default_config()
    assert abs(c.dt - 1 / 60) < 1e-9 and c.gravity[1] == np.float32(-3.81)
    assert c.h == np.float32(0.15) and c.rho0 == 1200 and c.solver_iterations == 3 and c.substep_iterations == 2
    assert c.hash_size == 1 << 17 and c.particle_count == 1 << 12 and c.k_corr == np.float32(0.001)
    assert c.enable_scorr and c.enable_viscosity and c.enable_vorticity and not c.enable_apbf
    assert (c.min_lod, c.max_lod) == (2, 7) and c.lod_max_dist == 15


def test_derive_params_bit_exact_with_setparams_float_arithmetic():
    import pbf_b200 as P
    from golden.make_golden import derive_f32
    for name in ["glsl_stages_plain.npz", "glsl_stages_apbf.npz", "glsl_step_radix.npz"]:
        z = H.load(name)
        cfg = H.engine_cfg(z)
        mine = P.derive_params(cfg, 0.0)
        ref = derive_f32(H.oracle_cfg(z))
        assert bytes(mine) == bytes(ref), name
    # collision padding shrinks the box (PBFluids.cpp:301-304)
    cfg = P.default_config()
    d = P.derive_params(cfg, 0.25)
    assert list(d.bounds_min)[:3] == [0.25] * 3 and list(d.bounds_max)[:3] == [5.75] * 3


def test_invalid_arguments_are_rejected_without_a_device():
    from pbf_b200 import _capi
    L = _capi.lib()
    assert L.pbf_default_config(None) == _capi.PBF_ERR_INVALID
    assert b"null" in L.pbf_last_error()
    assert L.pbf_derive_params(None, 0.0, None) == _capi.PBF_ERR_INVALID
    assert L.pbf_step(None) == _capi.PBF_ERR_INVALID
    assert L.pbf_destroy(None) == _capi.PBF_OK
    out = C.c_void_p()
    cfg = _capi.FluidConfig()
    L.pbf_default_config(C.byref(cfg))
    cfg.hash_size = 1000  # not a power of two
    assert L.pbf_create(C.byref(cfg), 0, C.byref(out)) == _capi.PBF_ERR_INVALID
    assert b"power of two" in L.pbf_last_error()
    assert L.pbf_abi_version() == 1
