"""Build recipe for libphix_b200.so and libphix_cxx.so (sm_100a), in-tree.

    python -m phix_b200.build          # or phix_b200.build.build() / build_cxx()

Compiles every .cu under phix_b200/csrc with nvcc for sm_100a only and links
libphix_b200.so (the C ABI) next to this file, so it travels with the source
tree; build_cxx() then compiles phix_b200/cxx (the C++ API of include/phix)
into libphix_cxx.so on top of it.  Objects are cached under phix_b200/_build/
keyed by source and header mtimes.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libphix_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
CXX_SRC = os.path.join(HERE, "cxx")
CXX_LIB = os.path.join(HERE, "libphix_cxx.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-O3", f"-I{INCLUDE}"]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h")) + glob.glob(os.path.join(INCLUDE, "phix", "detail", "*"))


def json_include() -> str | None:
    """Directory holding nlohmann/json.hpp (a header-only dependency of the
    config / BC-factory / output API): $PHIX_JSON_INCLUDE, else the first copy
    found under the Python environment's site-packages."""
    env = os.environ.get("PHIX_JSON_INCLUDE")
    if env and os.path.exists(os.path.join(env, "nlohmann", "json.hpp")):
        return env
    import sysconfig
    for key in ("purelib", "platlib", "include"):
        root = sysconfig.get_paths().get(key)
        if root:
            hits = sorted(glob.glob(os.path.join(root, "**", "nlohmann", "json.hpp"), recursive=True))
            if hits:
                return os.path.dirname(os.path.dirname(hits[0]))
    return None


def _cxx_headers():
    return [p for p in glob.glob(os.path.join(INCLUDE, "phix", "**", "*"), recursive=True) if os.path.isfile(p)]


def build(verbose: bool = False, jobs: int = 8) -> str:
    return _compile_link(sorted(glob.glob(os.path.join(CSRC, "*.cu"))), "", FLAGS, _headers(), LIB, [], verbose, jobs)


def build_cxx(verbose: bool = False, jobs: int = 8) -> str:
    """libphix_cxx.so: the drop-in C++ API (Mesh, fields, BCs, Equation, Solver,
    IO) linked against libphix_b200.so."""
    build(verbose, jobs)
    inc = json_include()
    if inc is None:
        raise RuntimeError("nlohmann/json.hpp not found: set PHIX_JSON_INCLUDE")
    flags = FLAGS + ["--expt-extended-lambda", f"-I{os.path.join(INCLUDE, 'phix')}", f"-I{inc}"]
    srcs = sorted(glob.glob(os.path.join(CXX_SRC, "*.cu")) + glob.glob(os.path.join(CXX_SRC, "*.cpp")))
    link = [f"-L{HERE}", "-lphix_b200", "-Xlinker", "-rpath,$ORIGIN"]
    return _compile_link(srcs, "cxx_", flags, _headers() + _cxx_headers(), CXX_LIB, link, verbose, jobs)


def _compile_link(srcs, prefix, flags, headers, out, link, verbose, jobs) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr_mtime = max((os.path.getmtime(h) for h in headers), default=0.0)
    objs, procs = [], []
    for src in srcs:
        obj = os.path.join(BUILD, prefix + os.path.splitext(os.path.basename(src))[0] + ".o")
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime):
            continue
        cmd = [NVCC, *ARCH, *flags, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        if len(procs) >= jobs:
            _drain(procs)
    _drain(procs)
    if not os.path.exists(out) or any(os.path.getmtime(o) > os.path.getmtime(out) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", out, *objs, *link, "-lcudart"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}")
    return out


def _drain(procs):
    errs = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            errs.append(f"{src}:\n{out.decode(errors='replace')}")
    procs.clear()
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
    print(build_cxx(verbose="-v" in sys.argv))
