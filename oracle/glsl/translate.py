#!/usr/bin/env python3
"""Rewrite the reference's GLSL compute shaders into C++ translation units.

TEST INFRASTRUCTURE ONLY.  Reads resources/shaders/compute/*.glsl from the
reference tree (path given on the command line) and writes one
``cs_<name>.inc`` per shader into the output directory (oracle/_ref/gen), to be
compiled by oracle/glsl/harness.cpp against oracle/glsl/glsl_shim.hpp.  The
rewrite is mechanical and keeps every shader statement as written:

  * ``#version`` and ``layout(local_size_x=...) in;`` lines are dropped;
  * the std140 uniform block becomes a struct plus one instance (``ubo``);
  * each std430 buffer block becomes a pointer per member (``T name[]`` ->
    ``T* name``; a scalar member ``T name`` -> pointer + macro);
  * ``uniform``/``shared`` declarations become namespace-scope statics;
  * ``vecN(...)``/``ivecN(...)``/``uvecN(...)`` constructors become
    ``make_vecN(...)`` calls; floating literals get an ``f`` suffix so the
    arithmetic stays single precision;
  * the shader is wrapped in ``namespace glsl::cs_<name>``.

One deliberate semantic edit, applied only when asked for
(``--pre-integrate-velocities``): in CS_Integrate the neighbour-velocity read
``particles[j].vel.xyz`` is redirected to a snapshot taken before the dispatch
(``particles_prev``).  The reference reads that buffer while other invocations
of the same dispatch write it (CS_Integrate.glsl:171 vs :277), a data race
whose outcome depends on GPU scheduling; the snapshot is the defined
semantics of this build.  The harness can also bind the snapshot to the live
buffer, which restores the racy read under a sequential schedule.
"""
import argparse
import os
import re
import sys

BARRIER_FREE = [
    "CS_PredictAndHash",
    "CS_BuildOffsets",
    "CS_ComputeLOD",
    "CS_ComputeLambdas",
    "CS_ComputeDeltaP",
    "CS_ApplyDeltaP",
    "CS_Integrate",
    "CS_VorticityConfinement",
    "CS_ContactFilter",
]
WORKGROUP = ["CS_RadixHistogram", "CS_RadixPrefixSum", "CS_RadixScatter"]

FLOAT_LIT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][-+]?\d+)?|\d+[eE][-+]?\d+)(?![\w.])")
CTOR = re.compile(r"\b(vec2|vec3|vec4|ivec2|ivec3|uvec2|uvec3)\s*\(")


def strip_line_comments(s):
    return re.sub(r"//[^\n]*", "", s)


def rewrite_buffer_block(m, macros):
    body = strip_line_comments(m.group(2))
    out = []
    for mem in re.finditer(r"(\w+)\s+(\w+)\s*(\[\s*\])?\s*;", body):
        typ, name, arr = mem.group(1), mem.group(2), mem.group(3)
        if arr:
            out.append(f"static {typ}* {name} = nullptr;")
        else:
            out.append(f"static {typ}* {name}__p = nullptr;")
            out.append(f"#define {name} (*{name}__p)")
            macros.append(name)
    return "\n".join(out)


def translate(src, name, pre_integrate):
    s = src
    s = re.sub(r"^\s*#version[^\n]*\n", "", s, flags=re.M)
    s = re.sub(r"layout\s*\(\s*local_size_x\s*=\s*\d+\s*\)\s*in\s*;", "", s)
    s = re.sub(
        r"layout\s*\(\s*std140[^)]*\)\s*uniform\s+(\w+)\s*\{(.*?)\}\s*(\w+)\s*;",
        lambda m: f"struct {m.group(1)} {{{m.group(2)}}};\nstatic {m.group(1)} {m.group(3)};",
        s,
        flags=re.S,
    )
    macros = []
    s = re.sub(
        r"layout\s*\(\s*std430[^)]*\)\s*(?:(?:readonly|writeonly|coherent|restrict)\s+)*buffer\s+(\w+)\s*\{(.*?)\}\s*;",
        lambda m: rewrite_buffer_block(m, macros),
        s,
        flags=re.S,
    )
    s = re.sub(r"layout\s*\(\s*binding\s*=\s*\d+\s*\)\s*uniform\s+sampler3D\s+(\w+)\s*;", r"static sampler3D \1;", s)
    s = re.sub(r"^(\s*)uniform\s+", r"\1static ", s, flags=re.M)
    s = re.sub(r"^(\s*)shared\s+", r"\1static ", s, flags=re.M)
    s = CTOR.sub(lambda m: f"make_{m.group(1)}(", s)
    s = FLOAT_LIT.sub(lambda m: m.group(1) + "f", s)
    if name == "CS_Integrate" and pre_integrate:
        target = "vec3 vj = particles[j].vel.xyz;"
        if s.count(target) != 1:
            sys.exit("translate.py: CS_Integrate neighbour-velocity read not found exactly once")
        s = s.replace(target, "vec3 vj = particles_prev[j].vel.xyz;")
        s = s.replace("static Particle* particles = nullptr;",
                      "static Particle* particles = nullptr;\nstatic Particle* particles_prev = nullptr;", 1)
    ns = "cs_" + re.sub(r"^CS_", "", name)
    head = (
        f"// generated by oracle/glsl/translate.py from {name}.glsl — do not edit\n"
        f"namespace glsl {{ namespace {ns} {{\n"
        "static thread_local uvec3 gl_GlobalInvocationID;\n"
        "static thread_local uvec3 gl_LocalInvocationID;\n"
        "static thread_local uvec3 gl_WorkGroupID;\n"
    )
    tail = "\n" + "".join(f"#undef {m}\n" for m in macros) + f"}} }} // namespace glsl::{ns}\n"
    return head + s + tail


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("shader_dir")
    ap.add_argument("out_dir")
    ap.add_argument("--pre-integrate-velocities", action="store_true")
    a = ap.parse_args()
    os.makedirs(a.out_dir, exist_ok=True)
    for name in BARRIER_FREE + WORKGROUP:
        with open(os.path.join(a.shader_dir, name + ".glsl")) as f:
            src = f.read()
        out = translate(src, name, a.pre_integrate_velocities)
        with open(os.path.join(a.out_dir, "cs_" + re.sub(r"^CS_", "", name) + ".inc"), "w") as f:
            f.write(out)


if __name__ == "__main__":
    main()
