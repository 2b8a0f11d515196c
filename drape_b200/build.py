"""Builds libdrape_b200.so (CUDA sm_100a kernels + C++ host + C ABI) and the `drape` command line in-tree.

    python -m drape_b200.build            # incremental
    python -m drape_b200.build --clean

Objects go to drape_b200/_build/; the shared library to drape_b200/libdrape_b200.so and the CLI to
drape_b200/drape. nvcc cross-compiles for sm_100a without a GPU.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libdrape_b200.so")
CLI = os.path.join(PKG, "drape")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall", "-I", os.path.join(ROOT, "include")]
LIB_SOURCES = ["elem.cu", "pcg.cu", "mg.cu", "nn.cu", "checks.cu", "problem.cpp", "context.cpp", "capi.cpp",
               "noalloc.cu"]
CLI_SOURCES = ["cli.cpp"]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hs + [os.path.join(ROOT, "include", "drape_b200.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    path = os.path.join(CSRC, src)
    if _stale(obj, [path] + _headers()):
        cmd = [NVCC] + ARCH + COMMON + ["-x", "cu" if src.endswith(".cu") else "c++", "-c", path, "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        subprocess.run(cmd, check=True)
    return obj


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    objs = [_compile(s, verbose) for s in LIB_SOURCES]
    if _stale(LIB, objs):
        subprocess.run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs, check=True)
    cli_objs = [_compile(s, verbose) for s in CLI_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if cli_objs and _stale(CLI, cli_objs + objs):
        lib_objs = [o for o in objs if not o.endswith("capi.cpp.o")] + [os.path.join(BUILD, "capi.cpp.o")]
        subprocess.run([NVCC] + ARCH + ["-cudart", "static", "-o", CLI] + cli_objs + lib_objs, check=True)
    return LIB


def main(argv):
    if "--clean" in argv:
        shutil.rmtree(BUILD, ignore_errors=True)
        for f in (LIB, CLI):
            if os.path.exists(f):
                os.remove(f)
        return
    print(build(verbose="-v" in argv))


if __name__ == "__main__":
    main(sys.argv[1:])
