"""Golden fixtures of the reference's CUDA MEX mgcg9 (Homogenization/QNC/mgcg9.cu).

TEST INFRASTRUCTURE.  Runs the reference's own mgcg9, compiled unmodified by
oracle/Makefile (target ref9) into oracle/_ref/libmgcg9_ref.so, on a GPU, and
stores its inputs and outputs.  The reference resets the CUDA device at the
start of every call, so this script must run in a process that uses CUDA for
nothing else (it imports no GPU framework), and it writes mgcg9.log, so it
runs in a scratch directory.

    python tests/golden/make_golden_mgcg9.py OUTDIR
"""
import ctypes
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

CASES = [
    # name, (nelx, nely, nelz), nl, density, nswp, tol, maxit
    ("mgcg9_16x8x8_rand_nl3", (16, 8, 8), 3, "rand", 2, 1e-8, 200),
    ("mgcg9_32x16x16_unif_nl4", (32, 16, 16), 4, "unif", 2, 1e-8, 200),
    ("mgcg9_24x16x8_rand_nl3_nswp3", (24, 16, 8), 3, "rand", 3, 1e-8, 200),
    ("mgcg9_16x8x8_maxit3_nl2", (16, 8, 8), 2, "rand", 2, 1e-12, 3),
]


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    outdir = os.path.abspath(outdir)
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libmgcg9_ref.so"))
    dp = ctypes.POINTER(ctypes.c_double)
    lib.ref_cuda_mgcg9.argtypes = [dp, dp, dp, dp, dp] + [ctypes.c_int] * 5 + [ctypes.c_double] + \
        [ctypes.c_int] * 3 + [ctypes.c_double] * 4 + [dp, ctypes.POINTER(ctypes.c_int)]
    lib.ref_cuda_mgcg9.restype = ctypes.c_int
    work = tempfile.mkdtemp()
    cwd = os.getcwd()
    os.chdir(work)
    try:
        for name, (nx, ny, nz), nl, dens, nswp, tol, maxit in CASES:
            p = oracle.cantilever(nx, ny, nz)
            if dens == "rand":
                CX = oracle.simp(oracle.random_density(nx, ny, nz, seed=nx + ny + nz))[0]
            else:
                CX = np.full(nx * ny * nz, 0.3 ** 3)
            Ke = np.ascontiguousarray(p.Ke0.reshape(-1))
            U = np.full(p.ndof, 5.0)   # input values are ignored by the reference
            rr, nit = ctypes.c_double(), ctypes.c_int()
            st = lib.ref_cuda_mgcg9(Ke.ctypes.data_as(dp), p.F.ctypes.data_as(dp), U.ctypes.data_as(dp),
                                    np.ascontiguousarray(CX).ctypes.data_as(dp), p.fixed.ctypes.data_as(dp),
                                    len(p.fixed), nx, ny, nz, nl, tol, maxit, nswp, 1, 0.3, 1.0, 1.0, 1.0,
                                    ctypes.byref(rr), ctypes.byref(nit))
            if st:
                raise SystemExit(f"{name}: reference mgcg9 returned cgiters {nit.value}")
            np.savez_compressed(os.path.join(outdir, name + ".npz"), nelx=nx, nely=ny, nelz=nz, nl=nl, nswp=nswp,
                                tol=tol, maxit=maxit, CX=CX, F=p.F, fixed=p.fixed, U=U, relres=rr.value,
                                nit=nit.value)
            print(name, "nit", nit.value, "relres", rr.value, flush=True)
    finally:
        os.chdir(cwd)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden"))
