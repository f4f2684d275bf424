"""Build recipe for the CUDA library of the particle-mesh step.

Compiles every ``csrc/*.cu`` for sm_100a with nvcc and links them into
``libpm_b200.so`` next to this file (the C ABI of include/pm_b200.h), and the
C++ driver ``driver/pm_main.cpp`` into ``pm_main``.  nvcc cross-compiles, so
this runs on a machine without a GPU.  Objects go to ``_build/``.

    python particle-mesh_b200/build.py [--force] [--ptxas-v]
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libpm_b200.so")
DRIVER = os.path.join(HERE, "pm_main")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr"] + ARCH


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def _deps():
    return _sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [
        os.path.join(ROOT, "include", "pm_b200.h"), os.path.abspath(__file__)]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, ptxas_v: bool = False, verbose: bool = False) -> str:
    """Builds (if stale) and returns the path of libpm_b200.so."""
    os.makedirs(BUILD, exist_ok=True)
    deps = _deps()
    if force or ptxas_v or _stale(LIB, deps):
        cc = nvcc()
        objs = []

        headers = [d for d in deps if not d.endswith(".cu")]

        def compile_one(src):
            obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
            # an object is rebuilt when its source, a header or this recipe is newer
            if not (force or ptxas_v) and not _stale(obj, [src] + headers):
                return obj, ""
            cmd = [cc, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
            if ptxas_v:
                cmd += ["-Xptxas", "-v"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
            return obj, r.stderr

        with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
            for obj, err in ex.map(compile_one, _sources()):
                objs.append(obj)
                if (verbose or ptxas_v) and err:
                    print(err, file=sys.stderr)
        tmp = LIB + ".tmp"
        subprocess.run([cc, "-shared", *ARCH, "-o", tmp, *objs], check=True)
        os.replace(tmp, LIB)
    drv_src = os.path.join(HERE, "driver", "pm_main.cpp")
    if os.path.exists(drv_src) and (force or _stale(DRIVER, [drv_src, LIB, os.path.join(HERE, "driver", "pm_b200.hpp")])):
        subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                        "-I", "/usr/local/cuda/include", drv_src, "-o", DRIVER,
                        "-L", HERE, "-lpm_b200", "-Wl,-rpath,$ORIGIN",
                        "-L", "/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath,/usr/local/cuda/lib64"], check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, ptxas_v="--ptxas-v" in sys.argv, verbose=True))
