"""Builds the reference-side checkers under oracle/_ref/ from the reference's own sources.

Test infrastructure only.  Two shared libraries are compiled, with outputs only under
oracle/_ref/ (git-ignored; they travel with the tree like the other built libraries):

* ``libref_shader.so``: the reference's ``msvc/Release/shaders/compute.hlsl`` compiled as C++
  and driven texel by texel by ``ref_engine.hpp`` through the oracle's C entry points
  (``orc_*``).  HLSL is not C++, so the source passes through a mechanical transform first,
  which changes no arithmetic:
    - ``cbuffer X : register(bN) { ... }`` -> ``namespace cb_X { ... } using namespace cb_X;``
    - ``Texture2D<T> name : register(tN);`` -> ``Texture2D<T> name{N};`` (the register slot)
    - semantics (``: SV_Target``, ``: TEX_IDX``) removed; ``out``/``inout`` parameters become
      references; ``(S) 0`` becomes ``S{}``
    - ``v.rg`` / ``v.rgb`` -> ``v.rg_()`` / ``v.rgb_()`` (hlsl_shim.hpp accessors)
    - unsuffixed floating literals get an ``f`` suffix (HLSL literals are single precision).
* ``libref_host.so``: the reference's ``terrain_heightfield.cpp`` and ``settings.cpp`` compiled
  unchanged (plus a small ``boost/scoped_array.hpp`` stand-in and ``ref_host.cpp``), giving the
  reference's own ``.cbf`` reader and bathymetry sampling (BY/BX/BA).

* ``libref_spectrum.so``: the reference's spectrum wave-maker, ``generateSpectrumWaves``
  (``engine.cpp:3559-3776``), cut out of ``engine.cpp`` by brace matching and turned into a free
  function by four textual substitutions (the engine's gravity setting, Boost's ``lgamma``, the log
  folder and the clock seed of ``srand``; see ``ref_spectrum.cpp``), then compiled with
  ``ref_spectrum.cpp``.  The rest of ``engine.cpp`` is never compiled.

It also copies the reference's example inputs (``msvc/Examples``: ``.cml`` settings, ``.cbf``
grids, wave and time-series files) to ``oracle/_ref/examples``, where the tests that parse and
run them look; nothing else reads the reference tree.

``engine.cpp`` itself is not buildable here (Direct3D 11, Windows headers, Boost), so the pass
schedule driving the shader is the oracle's restatement of it.

Usage: ``python oracle/ref_build.py [reference_root]`` (default: the ``CELERIS_REFERENCE``
environment variable, else ``/root/reference``).  Without the reference tree it does nothing.
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
FLAGS = ["-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", "-w"]


def transform_hlsl(src: str) -> str:
    s = src.replace("\r\n", "\n")
    # constant buffers -> namespaces whose members the shader functions see unqualified
    out = []
    pos = 0
    for m in re.finditer(r"cbuffer\s+(\w+)\s*:\s*register\s*\(\s*b\d+\s*\)\s*\{", s):
        name = m.group(1)
        close = s.index("}", m.end())
        out.append(s[pos:m.start()])
        out.append(f"namespace cb_{name} {{" + s[m.end():close] + f"}} using namespace cb_{name};")
        pos = close + 1
        if pos < len(s) and s[pos] == ";":
            pos += 1
    out.append(s[pos:])
    s = "".join(out)
    # textures bound to register slots
    s = re.sub(r"(Texture2D<\w+>\s+\w+)\s*:\s*register\s*\(\s*t(\d+)\s*\)\s*;", r"\1{\2};", s)
    # semantics on struct members and functions
    s = re.sub(r"\s*:\s*(SV_\w+|TEX_IDX)\b", "", s)
    # out / inout parameters
    s = re.sub(r"\b(?:inout|out)\s+(float[234]?|int[234]?)\s+(\w+)", r"\1& \2", s)
    # zero-initialising casts of output structs
    s = re.sub(r"\((\w+)\)\s*0\s*;", r"\1{};", s)
    # swizzles
    s = re.sub(r"\.(rgb|rg)\b", r".\1_()", s)
    # single-precision floating literals
    s = re.sub(r"(?<![\w.])(\d+\.\d*(?:[eE][+-]?\d+)?|\.\d+(?:[eE][+-]?\d+)?)(?![\w.])", r"\1f", s)
    return s


def extract_function(src: str, head: str) -> str:
    """The text of the function whose definition starts with `head`, through its closing brace."""
    i = src.index(head)
    k = src.index("{", i)
    depth = 0
    while True:
        if src[k] == "{":
            depth += 1
        elif src[k] == "}":
            depth -= 1
            if depth == 0:
                return src[i:k + 1]
        k += 1


def transform_spectrum(fn: str) -> str:
    subs = [
        (r"std::string\s+ShallowWaterEngine::generateSpectrumWaves\s*\(", "static std::string ref_generateSpectrumWaves("),
        (r"GetSetting\s*\(\s*\"gravity\"\s*\)", "ref_gravity"),
        (r"boost::math::lgamma\s*<\s*float\s*>\s*\(", "ref_lgammaf("),
        (r"initSetting\.logPath", "ref_log_path"),
        (r"srand\s*\(\s*time\s*\(\s*0\s*\)\s*\)", "srand(ref_seed)"),
    ]
    for pat, rep in subs:
        fn, n = re.subn(pat, rep, fn)
        if n == 0:
            raise RuntimeError("spectrum extraction: pattern not found: " + pat)
    return fn


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("reference-side build failed")


def build(ref_root: str | None = None) -> bool:
    ref_root = ref_root or os.environ.get("CELERIS_REFERENCE", "/root/reference")
    hlsl = os.path.join(ref_root, "msvc", "Release", "shaders", "compute.hlsl")
    if not os.path.exists(hlsl):
        return False
    os.makedirs(OUT, exist_ok=True)
    with open(hlsl, encoding="latin-1") as f:
        text = transform_hlsl(f.read())
    inc = os.path.join(OUT, "compute_hlsl.inc")
    with open(inc, "w") as f:
        f.write("// generated from the reference's compute.hlsl by oracle/ref_build.py\n" + text)
    inc_dir = os.path.join(HERE, "..", "include")
    run([CXX, *FLAGS, "-DORACLE_REAL=float", "-DORACLE_REF_SHADER", "-I", OUT, "-I", HERE, "-I", inc_dir,
         os.path.join(HERE, "oracle_capi.cpp"), "-o", os.path.join(OUT, "libref_shader.so")])
    # host side: terrain_heightfield.cpp + settings.cpp as they are, with a scoped_array stand-in
    shim = os.path.join(OUT, "shim", "boost")
    os.makedirs(shim, exist_ok=True)
    with open(os.path.join(shim, "scoped_array.hpp"), "w") as f:
        f.write(SCOPED_ARRAY)
    run([CXX, *FLAGS, "-include", "cstring", "-include", "string", "-I", os.path.join(OUT, "shim"), "-I", ref_root,
         os.path.join(ref_root, "terrain_heightfield.cpp"), os.path.join(ref_root, "settings.cpp"),
         os.path.join(HERE, "ref_host.cpp"), "-o", os.path.join(OUT, "libref_host.so")])
    # the spectrum wave-maker, cut out of engine.cpp
    with open(os.path.join(ref_root, "engine.cpp"), encoding="latin-1") as f:
        eng = f.read().replace("\r\n", "\n")
    fn = transform_spectrum(extract_function(eng, "std::string ShallowWaterEngine::generateSpectrumWaves("))
    with open(os.path.join(OUT, "spectrum_ref.inc"), "w") as f:
        f.write("// generated from the reference's engine.cpp (generateSpectrumWaves) by oracle/ref_build.py\n" + fn)
    run([CXX, *FLAGS, "-include", "cstring", "-include", "string", "-I", OUT, "-I", ref_root,
         os.path.join(HERE, "ref_spectrum.cpp"), "-o", os.path.join(OUT, "libref_spectrum.so")])
    examples = os.path.join(ref_root, "msvc", "Examples")
    if os.path.isdir(examples):
        shutil.copytree(examples, os.path.join(OUT, "examples"), dirs_exist_ok=True)
    return True


# A minimal owning array with the members terrain_heightfield.cpp uses (reset, operator[]).
SCOPED_ARRAY = """#pragma once
#include <cstddef>
namespace boost {
template <class T> class scoped_array {
    T* p_ = nullptr;
public:
    scoped_array() = default;
    explicit scoped_array(T* p) : p_(p) {}
    ~scoped_array() { delete[] p_; }
    scoped_array(const scoped_array&) = delete;
    scoped_array& operator=(const scoped_array&) = delete;
    void reset(T* p = nullptr) { delete[] p_; p_ = p; }
    T& operator[](std::ptrdiff_t i) const { return p_[i]; }
    T* get() const { return p_; }
};
}
"""

if __name__ == "__main__":
    ok = build(sys.argv[1] if len(sys.argv) > 1 else None)
    print("built" if ok else "reference tree not found; nothing built")
