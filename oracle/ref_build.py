"""Builds ``oracle/_ref/libref_host.so``: functions and per-element kernels of the reference
(StiffGIPC), compiled for the host CPU from the files of a reference checkout.

TEST INFRASTRUCTURE ONLY: ``tests/golden/make_golden.py`` runs the library once to write
golden vectors; nothing else loads it, and nothing of it is committed.

The reference as a whole does not build here (it needs Eigen 3.4, GLUT/GLEW and
nlohmann_json).  The functions named in ``ROOTS`` below use none of those: they work on
plain doubles, CUDA vector types and the reference's own ``__GEIGEN__`` helper structs.  This
recipe finds each definition in the checkout (and, by name, every helper function it calls,
transitively), writes them into one translation unit behind a prelude that maps the CUDA
qualifiers, vector types and the few device built-ins they use to host C++, and compiles it
with g++.  A kernel runs as a host loop with one "thread" per launch index.  The generated
source and the library go to ``oracle/_ref/`` (git-ignored); the repository keeps only this
recipe and the driver functions below, which are this project's own code.

Usage: python oracle/ref_build.py path/to/Stiff-GIPC     (the checkout's root directory)
       python oracle/ref_build.py --if-present           (the build container's checkout,
                                                          skipped where there is none)
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libref_host.so")

# files searched for definitions, in priority order (a name defined in several is taken
# from the first)
FILES = ["StiffGIPC/GIPC.cu", "StiffGIPC/femEnergy.cu", "StiffGIPC/ACCD.cu", "StiffGIPC/FrictionUtils.cuh",
         "StiffGIPC/mlbvh.cu", "StiffGIPC/GIPC_PDerivative.cuh", "StiffGIPC/gpu_eigen_libs.cu"]
TYPES = "StiffGIPC/eigen_data.h"

# (file, function) roots; their helpers are pulled in by name
ROOTS = [
    ("StiffGIPC/GIPC.cu", "__cal_Barrier_energy"),            # GIPC.cu:701-944
    ("StiffGIPC/GIPC.cu", "_calBarrierGradient"),             # GIPC.cu:5272-6337
    ("StiffGIPC/GIPC.cu", "_calFrictionGradient"),            # GIPC.cu:5087-5269
    ("StiffGIPC/GIPC.cu", "_calFrictionGradient_gd"),         # GIPC.cu:5047-5085
    ("StiffGIPC/GIPC.cu", "_computeGroundGradient"),          # GIPC.cu:6516-6545
    ("StiffGIPC/GIPC.cu", "_calFrictionLastH_gd"),            # GIPC.cu:8362-8386
    ("StiffGIPC/GIPC.cu", "_calFrictionLastH_DistAndTan"),    # GIPC.cu:8388-8499
    ("StiffGIPC/GIPC.cu", "_reduct_min_selfTimeStep_to_double"),  # GIPC.cu:7052-7155
    ("StiffGIPC/GIPC.cu", "_reduct_min_groundTimeStep_to_double"),  # GIPC.cu:6902-6977
    ("StiffGIPC/GIPC.cu", "_calKineticGradient"),             # GIPC.cu:6339-6350
    ("StiffGIPC/GIPC.cu", "_computeSoftConstraintGradient"),  # GIPC.cu:6409-6431
    ("StiffGIPC/GIPC.cu", "_computeXTilta"),                  # GIPC.cu:8073-8096
    ("StiffGIPC/GIPC.cu", "_stepForward"),                    # GIPC.cu:7937-7954
    ("StiffGIPC/femEnergy.cu", "__computePEPF_StableNHK3D1_double"),  # femEnergy.cu:432-459
    ("StiffGIPC/femEnergy.cu", "__cal_StabbleNHK_energy1_3D"),        # femEnergy.cu:1031-1050
    ("StiffGIPC/femEnergy.cu", "__calculateDms3D_double"),            # femEnergy.cu:324
    ("StiffGIPC/femEnergy.cu", "_calculate_fem_gradient"),            # femEnergy.cu:2264-2348 (USE_SNK1)
    ("StiffGIPC/femEnergy.cu", "_calculate_triangle_fem_gradient"),   # femEnergy.cu:2217-2262
    ("StiffGIPC/femEnergy.cu", "__cal_BaraffWitkinStretch_energy"),   # triangle energy
    ("StiffGIPC/femEnergy.cu", "__cal_quad_bending_energy"),          # hinge energy
    ("StiffGIPC/GIPC.cu", "__cal_Friction_energy"),                   # pair friction energy
    ("StiffGIPC/GIPC.cu", "__cal_Friction_gd_energy"),                # ground friction energy
    ("StiffGIPC/mlbvh.cu", "_checkPTintersection"),                   # mlbvh.cu:534-645
    ("StiffGIPC/mlbvh.cu", "_checkEEintersection"),                   # mlbvh.cu:685-1059
    ("StiffGIPC/GIPC.cu", "_GroundCollisionDetect"),                  # GIPC.cu:6433-6450
]

VOID_CHECKS = ("_checkPTintersection", "_checkEEintersection")

PRELUDE = r"""
// ---- host stand-ins for the CUDA qualifiers, vector types and built-ins -------------
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
// device code calls abs, sqrt, log, ... unqualified on doubles: make the floating overloads visible
using std::abs; using std::max; using std::min; using std::sqrt; using std::log; using std::fabs; using std::pow;
using std::exp;
#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __shared__
#define __constant__
#define __restrict__
#define RANK 2
#define NEWF
#define SFCLAMPING_ORDER 1
#define USE_SNK1 1
#define ADAPTIVE_KAPPA 1
#define USE_FRICTION 1
#define USE_QUADRATIC_BENDING 1
#define BANKSIZE 16
#define DEFAULT_BLOCKSIZE 256
#define DEFAULT_WARPNUM 16
using Precision_T = double;
using FloatP = float;
struct double2 { double x, y; };
struct double3 { double x, y, z; };
struct double4 { double x, y, z, w; };
struct float3 { float x, y, z; };
struct int2 { int x, y; };
struct int3 { int x, y, z; };
struct int4 { int x, y, z, w; };
struct uint2 { unsigned x, y; };
struct uint3 { unsigned x, y, z; };
struct uint4 { unsigned x, y, z, w; };
inline double2 make_double2(double a, double b) { return {a, b}; }
inline double3 make_double3(double a, double b, double c) { return {a, b, c}; }
inline int4 make_int4(int a, int b, int c, int d) { return {a, b, c, d}; }
inline int2 make_int2(int a, int b) { return {a, b}; }
inline uint2 make_uint2(unsigned a, unsigned b) { return {a, b}; }
inline uint4 make_uint4(unsigned a, unsigned b, unsigned c, unsigned d) { return {a, b, c, d}; }
struct HostDim3 { unsigned x, y, z; };
static HostDim3 threadIdx = {0, 0, 0}, blockIdx = {0, 0, 0}, blockDim = {1, 1, 1}, gridDim = {1, 1, 1};
inline double atomicAdd(double* a, double v) { double o = *a; *a += v; return o; }
inline int atomicAdd(int* a, int v) { int o = *a; *a += v; return o; }
inline unsigned atomicAdd(unsigned* a, unsigned v) { unsigned o = *a; *a += v; return o; }
template <class T> inline T __shfl_down_sync(unsigned, T v, int) { return v; }
inline void __syncthreads() {}
static double tep[1024];
"""


def strip_comments(src: str) -> str:
    out, i, n = [], 0, len(src)
    while i < n:
        if src.startswith("//", i):
            j = src.find("\n", i)
            i = n if j < 0 else j
        elif src.startswith("/*", i):
            j = src.find("*/", i + 2)
            out.append(" ")
            i = n if j < 0 else j + 2
        elif src[i] in "\"'":
            q, j = src[i], i + 1
            while j < n and src[j] != q:
                j += 2 if src[j] == "\\" else 1
            out.append(src[i:j + 1])
            i = j + 1
        else:
            out.append(src[i])
            i += 1
    return "".join(out)


def match_brace(s: str, i: int) -> int:
    """index one past the brace matching the '{' at i"""
    depth = 0
    while i < len(s):
        if s[i] == "{":
            depth += 1
        elif s[i] == "}":
            depth -= 1
            if depth == 0:
                return i + 1
        i += 1
    raise ValueError("unbalanced braces")


KEYWORDS = {"if", "for", "while", "switch", "return", "sizeof", "defined", "else", "do", "case"}


class Def:
    def __init__(self, name, ns, header, body, file):
        self.name, self.ns, self.header, self.body, self.file = name, ns, header, body, file

    def text(self):
        return self.header + "\n" + self.body


# the reference build's compile definitions (CMakeLists.txt:50-55) and the switches its
# sources set for themselves (GIPC.cu:28-29, FrictionUtils.cuh:13)
DEFINES = ["-DUSE_SNK1", "-DADAPTIVE_KAPPA", "-DUSE_FRICTION", "-DUSE_QUADRATIC_BENDING", "-DRANK=2", "-DNEWF",
           "-DSFCLAMPING_ORDER=1"]


def preprocess(path: str) -> str:
    """The file's text with its own #include lines dropped and its conditionals resolved
    under DEFINES (so that dead branches neither pull in helpers nor need Eigen)."""
    text = "".join(l for l in open(path) if not re.match(r"\s*#\s*include\b", l))
    return subprocess.run(["g++", "-E", "-P", "-x", "c++", "-w"] + DEFINES + ["-"], input=text, text=True,
                          capture_output=True, check=True).stdout


def index_file(path: str, rel: str):
    """Function definitions at namespace scope: name -> [Def]"""
    s = strip_comments(preprocess(path))
    defs = {}

    def scan(lo, hi, ns):
        i, seg = lo, lo
        while i < hi:
            c = s[i]
            if c == "#" and s[s.rfind("\n", 0, i) + 1:i].strip() == "":
                j = i
                while True:
                    j = s.find("\n", j)
                    if j < 0 or s[j - 1] != "\\":
                        break
                    j += 1
                i = hi if j < 0 else j + 1
                seg = i
                continue
            if c in "\"'":
                q, j = c, i + 1
                while j < hi and s[j] != q:
                    j += 2 if s[j] == "\\" else 1
                i = j + 1
                continue
            if c == ";":
                seg = i + 1
            elif c == "{":
                header = s[seg:i].strip()
                end = match_brace(s, i)
                m = re.fullmatch(r"namespace\s+(\w+)", header)
                if m:
                    scan(i + 1, end - 1, ns + [m.group(1)])
                elif header.startswith('extern "C"'):
                    scan(i + 1, end - 1, ns)
                elif ("(" in header and not re.match(r"(struct|class|enum|union|typedef)\b", header)
                      and "=" not in header.split("(")[0]):
                    pre = header[:header.index("(")]
                    nm = re.search(r"(\w+)\s*$", pre)
                    if nm and nm.group(1) not in KEYWORDS:
                        defs.setdefault(nm.group(1), []).append(Def(nm.group(1), tuple(ns), header, s[i:end], rel))
                i = end
                seg = end
                continue
            i += 1

    scan(0, len(s), [])
    return defs


def struct_defs(path: str):
    s = strip_comments(open(path).read())
    out = []
    for m in re.finditer(r"struct\s+(\w+)\s*\{", s):
        end = match_brace(s, m.end() - 1)
        body = s[m.start():end] + ";"
        if "Eigen" not in body:
            out.append(body)
    return out


def collect(root: str):
    index = {}
    for rel in FILES:
        for name, ds in index_file(os.path.join(root, rel), rel).items():
            index.setdefault(name, ds)  # first file wins
    chosen, order, todo = {}, [], [name for _, name in ROOTS]
    while todo:
        name = todo.pop()
        if name in chosen or name not in index:
            continue
        # helpers built on Eigen types sit only in preprocessor branches these builds leave
        # out (USE_SNK1 selects the Eigen-free stress); a root that needs one fails to compile
        ds = [d for d in index[name] if "Eigen" not in d.header + d.body]
        if not ds:
            continue
        # one definition per distinct signature (preprocessor alternatives keep the first)
        seen, keep = set(), []
        for d in ds:
            sig = re.sub(r"\s+", " ", d.header)
            if sig not in seen:
                seen.add(sig)
                keep.append(d)
        chosen[name] = keep
        order.append(name)
        for d in keep:
            for call in re.findall(r"\b([A-Za-z_]\w*)\s*\(", d.body):
                if call not in chosen and call in index:
                    todo.append(call)
    return [d for name in order for d in chosen[name]]


def strip_defaults(header: str) -> str:
    """drop default arguments from a parameter list (they stay in the prototype)"""
    lp = header.index("(")
    params, depth, cur, out = header[lp + 1:header.rindex(")")], 0, "", []
    for ch in params + ",":
        if ch in "(<":
            depth += 1
        elif ch in ")>":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.split("=")[0].rstrip())
            cur = ""
        else:
            cur += ch
    return header[:lp + 1] + ",".join(out) + header[header.rindex(")"):]


def generate(root: str) -> str:
    defs = collect(root)
    parts = [PRELUDE, "namespace __GEIGEN__ {"] + struct_defs(os.path.join(root, TYPES)) + ["}"]

    def wrap(ns, text):
        if not ns:
            return text
        inner = text
        if ns == ("Friction",):
            inner = "using namespace __GEIGEN__;\n" + inner
        return "".join("namespace %s {\n" % n for n in ns) + inner + "\n" + "}" * len(ns)

    # _checkPTintersection / _checkEEintersection are declared bool but end without returning a
    # value, and no caller reads one; g++ traps at such an end, nvcc lets it pass: give them the
    # void they behave as
    for d in defs:
        if d.name in VOID_CHECKS:
            d.header = re.sub(r"\bbool\s+(%s)\b" % d.name, r"void \1", d.header)
    parts.append("// ---- prototypes")
    for d in defs:
        if "template" in d.header:
            continue
        parts.append(wrap(d.ns, d.header + ";"))
    parts.append("// ---- definitions")
    for d in defs:
        header = d.header if "template" in d.header else strip_defaults(d.header)
        parts.append("// %s\n" % d.file + wrap(d.ns, header + "\n" + d.body))
    parts.append(open(os.path.join(HERE, "ref_drivers.inc")).read())
    # the reference writes `const const T*` in a few kernel signatures, which nvcc accepts
    # and g++ rejects as a duplicate qualifier
    return re.sub(r"\bconst\s+const\b", "const", "\n".join(parts))


def build(root: str) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    src = os.path.join(OUT_DIR, "ref_host.cpp")
    with open(src, "w") as f:
        f.write(generate(root))
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-w", "-o", LIB, src])
    return LIB


# where the build container keeps its read-only reference checkout
CHECKOUT = "/root/reference"

if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    if sys.argv[1] == "--if-present":
        if os.path.isdir(os.path.join(CHECKOUT, "StiffGIPC")):
            print(build(CHECKOUT))
    else:
        print(build(sys.argv[1]))
