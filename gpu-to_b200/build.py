"""Build the gputo shared libraries in-tree with nvcc for sm_100a.

    python gpu-to_b200/build.py            # incremental
    python gpu-to_b200/build.py --force    # rebuild everything

Outputs (git-ignored, shipped with the tree):
  gpu-to_b200/lib/libgputo.so       the product: kernels + solver + C ABI
  gpu-to_b200/lib/libgputo_mex.so   the MEX gateway of mgcg1 (mexFunction) linked
                                    against libgputo.so.  It is compiled
                                    against MATLAB's mex.h when MATLAB_ROOT is
                                    set, else against the project's stand-in
                                    declarations (gpu-to_b200/mex_api/mex.h);
                                    the mx* symbols stay undefined and resolve
                                    from MATLAB's libmx (or a harness's own
                                    implementation) at load.
  gpu-to_b200/lib/libgputo_mex9.so  the same for the MEX mgcg9 (18 arguments)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
OBJ = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", f"-I{CSRC}",
          f"-I{os.path.join(ROOT, 'include')}"]

SOURCES = ["kernels_fine.cu", "kernels_mg.cu", "kernels_blas.cu", "kernels_design.cu", "solver.cu",
           "capi.cpp", "noalloc.cu", "kernels_quad.cu", "kernels_tc.cu", "kernels_tcsweep.cu",
           "kernels_learned.cu", "batch.cpp", "design_io.cpp",
           "kernels_hsweep.cu", "hostio.cpp", "homog.cu"]
HEADERS = ["gputo_internal.h", "solver.h", "tma.h", "hadamard.h"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "gputo.h")]
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            cmd = [NVCC, *ARCH, *COMMON, "-rdc=false", "-c", s, "-o", o]
            if src.endswith(".cu") and verbose:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd)
    so = os.path.join(LIB, "libgputo.so")
    if force or _newer(so, objs):
        _run([NVCC, *ARCH, "-shared", "-o", so, *objs, "-cudart", "static", "-lpthread"])
    # MEX gateway
    mex_inc = os.path.join(os.environ["MATLAB_ROOT"], "extern", "include") if os.environ.get(
        "MATLAB_ROOT") else os.path.join(HERE, "mex_api")
    for src, out in (("mex_gateway.cpp", "libgputo_mex.so"), ("mex_gateway9.cpp", "libgputo_mex9.so")):
        gw_src = os.path.join(CSRC, src)
        gw = os.path.join(LIB, out)
        if force or _newer(gw, [gw_src, so]):
            _run(["g++", "-O2", "-fPIC", "-shared", f"-I{mex_inc}", f"-I{os.path.join(ROOT, 'include')}",
                  gw_src, "-o", gw, f"-L{LIB}", "-lgputo", f"-Wl,-rpath,{LIB}", "-Wl,-rpath,$ORIGIN"])
    return so


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print("built", os.path.join(LIB, "libgputo.so"))
