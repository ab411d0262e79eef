"""Mechanical WGSL -> C++ translation of the reference's compute shaders.

TEST INFRASTRUCTURE ONLY (the recipe that builds ``oracle/_ref/``).

The reference's per-step pipeline is WGSL (``src/shaders/compute/lbvh.wgsl``
and ``barnes_hut.wgsl``) that needs a WebGPU device; none exists here.  This
script reads the two shader files where they lie in the reference checkout
and rewrites them, line by line, into C++ over ``wgsl_prelude.h`` (WGSL types
and builtins).  Nothing is edited by hand: the generated sources land in
``oracle/_ref/`` (git-ignored) and ``ref_harness.cpp`` dispatches their entry
points invocation by invocation in the reference's stage order
(``src/simulation.ts:393-420``).  The result is the reference's own shader
logic running on the CPU, used to pin the oracle restatement and to write the
golden fixtures in ``tests/golden/``.

Handled WGSL: struct declarations, uniform/storage bindings, ``fn``
declarations (entry points with ``@builtin(global_invocation_id)``),
``let``/``var``/``const``, ``while``/``if``/``else if``/``loop``/``for``
headers without parentheses, ``vec2<f32>``/``vec3<u32>``/``array<T, N>``
types and f32 literals.  Anything else raises, so a change in the shaders is
noticed instead of silently mistranslated.
"""
from __future__ import annotations

import os
import re
import struct
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))

TYPE_MAP = {
    "f32": "f32", "u32": "u32", "i32": "i32", "bool": "bool",
    "vec2<f32>": "vec2f", "vec3<u32>": "vec3u", "atomic<u32>": "u32",
    "vec3<f32>": "vec3f", "vec4<f32>": "vec4f",
}


def ctype(t: str) -> str:
    t = t.strip()
    if t in TYPE_MAP:
        return TYPE_MAP[t]
    if re.fullmatch(r"[A-Z]\w*", t):  # user struct
        return t
    raise ValueError(f"unsupported WGSL type: {t}")


def expr(s: str) -> str:
    s = s.replace("vec2<f32>(", "vec2f(").replace("vec3<u32>(", "vec3u(")
    s = s.replace("vec3<f32>(", "vec3f(").replace("vec4<f32>(", "vec4f(")
    s = s.replace(").r", ").x")  # the red channel of a sampled vec4
    # f32 literals (abstract floats concretised to f32 in these shaders)
    s = re.sub(r"(?<![\w.])(\d+\.\d*)(?![\w.])", r"\1f", s)
    return s


def split_comment(line: str):
    i = line.find("//")
    return (line, "") if i < 0 else (line[:i], line[i:])


def translate(src: str, namespace: str) -> str:
    out = [f"namespace {namespace} {{", "using namespace wgsl;"]
    in_struct = False
    for raw in src.splitlines():
        code, comment = split_comment(raw)
        s = code.rstrip()
        st = s.strip()
        ind = s[: len(s) - len(s.lstrip())]
        if not st:
            out.append(raw if comment else "")
            continue
        if in_struct:
            if st == "}" or st == "};":
                out.append("};")
                in_struct = False
                continue
            m = re.fullmatch(r"(\w+)\s*:\s*([^,]+),?", st)
            if not m:
                raise ValueError(f"struct field: {raw}")
            out.append(f"    {ctype(m.group(2))} {m.group(1)}; {comment}")
            continue
        m = re.fullmatch(r"struct\s+(\w+)\s*\{", st)
        if m:
            out.append(f"struct {m.group(1)} {{")
            in_struct = True
            continue
        m = re.fullmatch(r"@group\(\d+\)\s*@binding\(\d+\)\s*var<uniform>\s+(\w+)\s*:\s*(\w+)\s*;", st)
        if m:
            out.append(f"static {m.group(2)} {m.group(1)}; {comment}")
            continue
        m = re.fullmatch(r"@group\(\d+\)\s*@binding\(\d+\)\s*var<storage,\s*read_write>\s+(\w+)\s*:\s*array<(.+)>\s*;", st)
        if m:
            out.append(f"static {ctype(m.group(2))}* {m.group(1)} = nullptr; {comment}")
            continue
        if re.fullmatch(r"@compute\s+@workgroup_size\(\d+\)", st):
            out.append(f"// {st}")
            continue
        m = re.fullmatch(r"fn\s+(\w+)\(@builtin\(global_invocation_id\)\s*(\w+)\s*:\s*vec3<u32>\)\s*\{", st)
        if m:
            out.append(f"static void {m.group(1)}(vec3u {m.group(2)}) {{ {comment}")
            continue
        m = re.fullmatch(r"fn\s+(\w+)\((.*)\)\s*(->\s*(\S+))?\s*\{", st)
        if m:
            params = []
            for p in [x for x in m.group(2).split(",") if x.strip()]:
                nm, ty = [x.strip() for x in p.split(":")]
                params.append(f"{ctype(ty)} {nm}")
            ret = ctype(m.group(4)) if m.group(4) else "void"
            out.append(f"static {ret} {m.group(1)}({', '.join(params)}) {{ {comment}")
            continue
        m = re.fullmatch(r"const\s+(\w+)\s*=\s*(.+);", st)
        if m:
            out.append(f"{ind}constexpr int {m.group(1)} = {expr(m.group(2))}; {comment}")
            continue
        m = re.fullmatch(r"let\s+(\w+)\s*=\s*(.+);", st)
        if m:
            out.append(f"{ind}const auto {m.group(1)} = {expr(m.group(2))}; {comment}")
            continue
        m = re.fullmatch(r"var\s+(\w+)\s*:\s*array<(.+),\s*(\w+)>\s*;", st)
        if m:
            out.append(f"{ind}std::array<{ctype(m.group(2))}, {m.group(3)}> {m.group(1)}{{}}; {comment}")
            continue
        m = re.fullmatch(r"var\s+(\w+)\s*:\s*([\w<>]+)\s*=\s*(.+);", st)
        if m:
            out.append(f"{ind}{ctype(m.group(2))} {m.group(1)} = {expr(m.group(3))}; {comment}")
            continue
        m = re.fullmatch(r"var\s+(\w+)\s*=\s*(.+);", st)
        if m:
            out.append(f"{ind}auto {m.group(1)} = {expr(m.group(2))}; {comment}")
            continue
        m = re.fullmatch(r"(\}\s*else\s+if|if|while)\s+(.+)\s*\{", st)
        if m and not st.startswith(("if (", "while (")):
            out.append(f"{ind}{m.group(1)} ({expr(m.group(2))}) {{ {comment}")
            continue
        if st == "loop {":
            out.append(f"{ind}while (true) {{ {comment}")
            continue
        m = re.fullmatch(r"for\s*\(var\s+(.+)", st)
        if m:
            out.append(f"{ind}for (auto {expr(m.group(1))} {comment}")
            continue
        if re.search(r"\b(var|let|fn|struct|@\w+|loop)\b", st):
            raise ValueError(f"unhandled WGSL line: {raw}")
        out.append(f"{ind}{expr(st)} {comment}".rstrip())
    out.append(f"}}  // namespace {namespace}")
    return "\n".join(out) + "\n"


CONST_EXPR = re.compile(r"[0-9.\s+\-*/()]+")


def translate_render(src: str, namespace: str) -> str:
    """The render shaders (density.wgsl, tone_map.wgsl) without their vertex
    stages: structs (attributes dropped), bindings (textures and samplers as
    harness stubs), helper functions and the fragment entry point, whose
    `discard` sets wgsl::g_discarded.  A `let` of literals alone is a WGSL
    abstract-float constant expression: it is evaluated here in double
    precision and stored as the nearest f32, as WGSL does."""
    lines = []
    skip = 0
    it = iter(src.splitlines())
    for raw in it:
        st = split_comment(raw)[0].strip()
        if st == "@vertex":  # drop the whole vertex entry point
            depth = 0
            for body in it:
                code = split_comment(body)[0]
                depth += code.count("{") - code.count("}")
                if "{" in code and depth == 0:
                    break
                if depth == 0 and "}" in code:
                    break
            continue
        if st == "@fragment":
            lines.append("// @fragment")
            continue
        m = re.fullmatch(r"@group\(\d+\)\s*@binding\(\d+\)\s*var<storage,\s*read>\s+(\w+)\s*:\s*array<(.+)>\s*;", st)
        if m:
            lines.append(f"static {ctype(m.group(2))}* {m.group(1)} = nullptr;")
            continue
        m = re.fullmatch(r"@group\(\d+\)\s*@binding\(\d+\)\s*var\s+(\w+)\s*:\s*(texture_2d<f32>|sampler)\s*;", st)
        if m:
            ty = "texture_2d" if m.group(2).startswith("texture") else "sampler"
            lines.append(f"static {ty} {m.group(1)};")
            continue
        m = re.fullmatch(r"let\s+(\w+)\s*=\s*(.+);", st)
        if m and CONST_EXPR.fullmatch(m.group(2)):
            ind = raw[: len(raw) - len(raw.lstrip())]
            val = eval(m.group(2), {"__builtins__": {}})  # digits and + - * / ( ) only
            f32 = struct.unpack("f", struct.pack("f", float(val)))[0]  # nearest f32
            lines.append(f"{ind}const f32 {m.group(1)} = {f32!r};")
            continue
        raw = re.sub(r"@(builtin|location|interpolate)\([^)]*\)\s*", "", raw)
        raw = raw.replace("discard;", "{ g_discarded = true; return {}; }")
        lines.append(raw)
    return translate("\n".join(lines), namespace)


def build_render(shader_dir: str, out_dir: str, force: bool = False) -> str:
    """Translate density.wgsl and tone_map.wgsl and compile their harness."""
    os.makedirs(out_dir, exist_ok=True)
    lib = os.path.join(out_dir, "libref_render.so")
    srcs = [os.path.join(shader_dir, "density.wgsl"), os.path.join(shader_dir, "tone_map.wgsl")]
    deps = srcs + [os.path.abspath(__file__), os.path.join(HERE, "wgsl_prelude.h"),
                   os.path.join(HERE, "ref_render_harness.cpp")]
    if (not force and os.path.exists(lib)
            and all(os.path.getmtime(d) <= os.path.getmtime(lib) for d in deps)):
        return lib
    for path, ns, name in ((srcs[0], "ref_density", "ref_density.inc"),
                           (srcs[1], "ref_tone_map", "ref_tone_map.inc")):
        with open(path) as f:
            text = translate_render(f.read(), ns)
        with open(os.path.join(out_dir, name), "w") as f:
            f.write(f"// Generated from {os.path.basename(path)} by oracle/wgsl_to_cpp.py; do not edit.\n")
            f.write(text)
    cxx = shutil.which("g++") or "c++"
    tmp = lib + ".tmp"
    subprocess.run([cxx, "-O2", "-march=x86-64-v2", "-std=c++17", "-ffp-contract=off",
                    "-fno-fast-math", "-fPIC", "-shared", "-I", HERE, "-I", out_dir, "-o", tmp,
                    os.path.join(HERE, "ref_render_harness.cpp")], check=True)
    os.replace(tmp, lib)
    return lib


def build(shader_dir: str, out_dir: str, force: bool = False) -> str:
    """Translate lbvh.wgsl and barnes_hut.wgsl and compile the harness."""
    os.makedirs(out_dir, exist_ok=True)
    lib = os.path.join(out_dir, "libref_wgsl.so")
    srcs = [os.path.join(shader_dir, "lbvh.wgsl"), os.path.join(shader_dir, "barnes_hut.wgsl")]
    deps = srcs + [os.path.abspath(__file__), os.path.join(HERE, "wgsl_prelude.h"),
                   os.path.join(HERE, "ref_harness.cpp")]
    if (not force and os.path.exists(lib)
            and all(os.path.getmtime(d) <= os.path.getmtime(lib) for d in deps)):
        return lib
    for path, ns, name in ((srcs[0], "ref_lbvh", "ref_lbvh.inc"),
                           (srcs[1], "ref_barnes_hut", "ref_barnes_hut.inc")):
        with open(path) as f:
            text = translate(f.read(), ns)
        with open(os.path.join(out_dir, name), "w") as f:
            f.write(f"// Generated from {os.path.basename(path)} by oracle/wgsl_to_cpp.py; do not edit.\n")
            f.write(text)
    cxx = shutil.which("g++") or "c++"
    tmp = lib + ".tmp"
    subprocess.run([cxx, "-O2", "-march=x86-64-v2", "-fopenmp", "-std=c++17",
                    "-ffp-contract=off", "-fno-fast-math", "-fPIC",
                    "-shared", "-I", HERE, "-I", out_dir, "-o", tmp,
                    os.path.join(HERE, "ref_harness.cpp")], check=True)
    os.replace(tmp, lib)
    return lib
