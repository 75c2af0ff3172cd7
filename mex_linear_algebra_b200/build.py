"""Build recipe for the in-tree native libraries.

* ``libmela_b200.so`` -- the CUDA kernels (sm_100a only) and the C host layer
  behind ``include/mela.h``, compiled with nvcc and linked against the static
  CUDA runtime.
* ``mex/_build/mela_*.so`` -- the six MEX gateways compiled against the
  non-MATLAB MEX host (for use outside MATLAB; inside MATLAB the same
  gateway sources are compiled with ``mex`` against ``libmela_b200.so``).

Usage: ``python -m mex_linear_algebra_b200.build`` (or ``build()`` below).
Objects are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmela_b200.so")
MEXDIR = os.path.join(PKG, "mex")
MEXHOST = os.path.join(PKG, "mexhost")
MEXOUT = os.path.join(MEXDIR, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I" + CSRC, "-I" + INCLUDE, "-I" + OBJ]
GATEWAYS = ("mela_matmul_gf2", "mela_matmul_m4ri", "mela_rank_gf2", "mela_rank_m4ri",
            "mela_null_gf2", "mela_null_m4ri")


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cc() -> str:
    # an environment CC wrapper may lack OpenMP/spec files; the system gcc is used
    for cand in ("/usr/bin/gcc-13", "/usr/bin/gcc", shutil.which("gcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("gcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


MODEL_JSON = os.path.join(PKG, "costmodel.json")
MODEL_INC = os.path.join(OBJ, "costmodel_weights.inc")


def write_model_weights() -> None:
    """The trained cost model (costmodel.json) as a C initializer list that
    mlp.cu compiles in as the library's default dispatch model.  Without a
    model file of the network's size the include is empty and the library
    starts on its fixed rule."""
    import json
    import re
    params = []
    if os.path.exists(MODEL_JSON):
        with open(os.path.join(INCLUDE, "mela.h")) as f:
            want = int(re.search(r"#define MELA_MLP_PARAMS (\d+)", f.read()).group(1))
        with open(MODEL_JSON) as f:
            p = json.load(f)["params"]
        if len(p) == want:
            params = p
    text = "// generated from costmodel.json by build.py\n"
    if params:
        text += "#define MELA_DEFAULT_MODEL 1\n"
        text += "static const float kDefaultModel[] = {\n"
        text += ",\n".join(", ".join(f"{float(x)!r}f" for x in params[i:i + 8]) for i in range(0, len(params), 8))
        text += "\n};\n"
    old = open(MODEL_INC).read() if os.path.exists(MODEL_INC) else None
    if old != text:
        with open(MODEL_INC, "w") as f:
            f.write(text)


def build_library(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    write_model_weights()
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdrs = _headers() + [MODEL_INC]
    jobs = []
    for src in sources:
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        if ptxas_info or _newer(obj, [src] + hdrs):
            cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)
    logs = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            logs = list(ex.map(_run, jobs))
    objs = [os.path.join(OBJ, os.path.basename(s) + ".o") for s in sources]
    if _newer(LIB, objs):
        _run([nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda"])
    if verbose:
        for lg in logs:
            if lg.strip():
                print(lg)
    return LIB


def build_gateways() -> list:
    """Compile the MEX gateways against the non-MATLAB MEX host."""
    os.makedirs(MEXOUT, exist_ok=True)
    out = []
    for name in GATEWAYS:
        src = os.path.join(MEXDIR, name + ".c")
        if not os.path.exists(src):
            continue
        so = os.path.join(MEXOUT, name + ".so")
        deps = [src, os.path.join(MEXHOST, "mexhost.c"), os.path.join(MEXHOST, "mex.h"),
                os.path.join(MEXHOST, "matrix.h"), os.path.join(INCLUDE, "mela.h"),
                os.path.join(MEXDIR, "mela_gateway.h")]
        deps = [d for d in deps if os.path.exists(d)]
        if _newer(so, deps + [LIB]):
            _run([host_cc(), "-O2", "-fPIC", "-shared", "-std=gnu11", "-I" + MEXHOST, "-I" + INCLUDE,
                  "-I" + MEXDIR, "-o", so, src, os.path.join(MEXHOST, "mexhost.c"), LIB,
                  "-Wl,-rpath," + PKG])
        out.append(so)
    return out


def build(verbose: bool = False) -> None:
    build_library(verbose=verbose)
    build_gateways()


if __name__ == "__main__":
    import sys
    build(verbose=True)
    if "--ptxas" in sys.argv:
        build_library(verbose=True, ptxas_info=True)
    print(LIB)
