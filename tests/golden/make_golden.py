"""Generate the golden fixtures in this directory from the reference itself.

Run here, where the reference tree is mounted:  python tests/golden/make_golden.py

* ``ke0_matlab.npy``: the driver's element matrix Ke0, evaluated from the
  packed lower-triangle table in Cantilever/TOP3D125MGCGCUDA/top3D125modCuda.m:50-77
  (read as text here; the numbers are stored, not the source).
* ``kem3_ref.npz``: Kem3 (Cantilever/omp/mgcg1.c:1370) from the compiled
  reference, h = 1 and 2.
* ``solve_*.npz``: known-answer solves of the reference's own, unmodified
  OpenMP MEX (Cantilever/omp/mgcg1.c), compiled into oracle/_ref (cantilevers,
  corner supports, and the bridge workload's supports and load).
* ``design_c1.npz``: the 64x32x32 cantilever (~215k DOF) design loop,
  50 OC iterations, with every solve done by that compiled reference and the
  MATLAB-side steps by the oracle's numpy restatement.

The fixtures are what the tests compare against on machines without the
reference tree.
"""
import ctypes
import os
import re
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

# Root of the reference checkout (read-only).  Set GPUTO_REFERENCE_ROOT to
# point at it; the fallback is where this build's recipe keeps it.
REFROOT = os.environ.get("GPUTO_REFERENCE_ROOT", "/root/reference")


def matlab_ke0():
    src = open(os.path.join(REFROOT, "Cantilever/TOP3D125MGCGCUDA/top3D125modCuda.m")).read()
    m = re.search(r"Ke = 1/\(1\+nu\)/\(2\*nu-1\)/144 \*\( \[(.*?)\]\+nu\*\[(.*?)\] \);", src, re.S)
    assert m, "Ke table not found"

    def nums(s):
        s = re.sub(r"\.\.\.", " ", s)
        return np.array([float(t) for t in re.split(r"[;\s]+", s) if t.strip()])

    a, b = nums(m.group(1)), nums(m.group(2))
    assert a.size == 300 and b.size == 300
    nu = 0.3
    v = 1 / (1 + nu) / (2 * nu - 1) / 144 * (a + nu * b)
    # Ke0(tril(ones(24))==1) = Ke': MATLAB fills the lower triangle column by column
    K = np.zeros((24, 24))
    idx = 0
    for col in range(24):
        for row in range(col, 24):
            K[row, col] = v[idx]
            idx += 1
    return K + K.T - np.diag(np.diag(K))


def kem3(h):
    L = ctypes.CDLL(O.REF_PATH)
    Ae = np.zeros(576)
    L.Kem3.argtypes = [ctypes.POINTER(ctypes.c_double)] + [ctypes.c_double] * 4
    L.Kem3(Ae.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0.3, h, h, h)
    return Ae.reshape(24, 24)


def corner_supports(nelx, nely, nelz):
    """A problem with sparse, asymmetric supports: the two bottom corner
    strips at x=0 and x=nelx (all dofs) plus a z-roller line, load on the
    top face centre line (exercises the coarse fixed-dof restriction and the
    coarsest penalty)."""
    p = O.cantilever(nelx, nely, nelz)
    fixed = []
    for i in (0, nelx):
        for j in range(nely + 1):
            n = O.node_id(nelx, nely, nelz, i, j, 0)
            fixed += [3 * n + 1, 3 * n + 2, 3 * n + 3]
    for i in range(nelx + 1):
        n = O.node_id(nelx, nely, nelz, i, 0, nelz)
        fixed.append(3 * n + 2)
    F = np.zeros(p.ndof)
    for i in range(nelx + 1):
        n = O.node_id(nelx, nely, nelz, i, nely // 2, nelz)
        F[3 * n + 2] = -1.0 / (nelx + 1)
    return O.Problem(nelx, nely, nelz, F, np.array(sorted(set(fixed)), dtype=np.float64))


def solve_cases():
    return [
        ("solve_16x8x8_rand_nl3", O.cantilever(16, 8, 8), lambda: O.simp(O.random_density(16, 8, 8, 1))[0], 3, 1e-8, 200),
        ("solve_32x16x16_unif_nl4", O.cantilever(32, 16, 16), lambda: O.simp(np.full(32 * 16 * 16, 0.12))[0], 4, 1e-8, 200),
        ("solve_16x8x8_corner_nl3", corner_supports(16, 8, 8), lambda: O.simp(O.random_density(16, 8, 8, 7))[0], 3, 1e-8, 200),
        ("solve_16x8x8_maxit3_nl2", O.cantilever(16, 8, 8), lambda: O.simp(O.random_density(16, 8, 8, 3))[0], 2, 1e-12, 3),
        # the bridge workload's supports and top-face load (oracle.bridge)
        ("solve_16x8x8_bridge_nl3", O.bridge(16, 8, 8), lambda: O.simp(O.random_density(16, 8, 8, 11))[0], 3, 1e-8, 200),
    ]


def solves(only=None):
    for name, p, cxf, nl, tol, maxit in solve_cases():
        if only and name not in only:
            continue
        CX = cxf()
        U, rr, nit = O.ref_mgcg1(p, CX, nl, tol, maxit)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), nelx=p.nelx, nely=p.nely, nelz=p.nelz,
                            F=p.F, fixed=p.fixed, CX=CX, nl=nl, tol=tol, maxit=maxit, U=U,
                            relres=rr, nit=nit)
        print(name, "relres", rr, "nit", nit)


def main(only_design=False, only=None):
    O.build()
    os.environ.setdefault("OMP_THREAD_LIMIT", str(os.cpu_count()))
    if only_design:
        return design()
    if only:
        return solves(only)
    np.save(os.path.join(HERE, "ke0_matlab.npy"), matlab_ke0())
    np.savez(os.path.join(HERE, "kem3_ref.npz"), h1=kem3(1.0), h2=kem3(2.0))
    solves()

    # 64x32x32 cantilever: first solve (uniform 0.12) + the 50-iteration design
    p = O.cantilever(64, 32, 32)
    CX = O.simp(np.full(p.nel, 0.12))[0]
    t = time.time()
    U, rr, nit = O.ref_mgcg1(p, CX, 4, 1e-8, 200)
    print("c1 first solve", rr, nit, f"{time.time() - t:.2f}s")
    sample = np.arange(0, p.ndof, 37)
    np.savez_compressed(os.path.join(HERE, "solve_c1_first.npz"), nelx=64, nely=32, nelz=32, nl=4,
                        tol=1e-8, maxit=200, relres=rr, nit=nit, sample=sample, U_sample=U[sample],
                        U_norm=np.linalg.norm(U), compliance=float(p.F @ U))
    design()


def design():
    p = O.cantilever(64, 32, 32)
    cfg = O.DesignConfig(nl=4, tol=1e-8, maxit=200, iters=50)
    t = time.time()
    hist = O.design_loop(p, cfg, solver=lambda CX: O.ref_mgcg1(p, CX, cfg.nl, cfg.tol, cfg.maxit))
    print("c1 design", f"{time.time() - t:.1f}s", "c[-1]", hist["c"][-1], "nit", hist["nit"][:5], "...")
    np.savez_compressed(os.path.join(HERE, "design_c1.npz"), c=np.array(hist["c"]),
                        nit=np.array(hist["nit"]), relres=np.array(hist["relres"]),
                        lmid=np.array(hist["lmid"]), ch=np.array(hist["ch"]),
                        xPhys=hist["xPhys"].astype(np.float32), x=hist["x"].astype(np.float32))


if __name__ == "__main__":
    # --design: only the design-loop history; --only NAME[,NAME]: only those solve fixtures
    only = sys.argv[sys.argv.index("--only") + 1].split(",") if "--only" in sys.argv else None
    main(only_design="--design" in sys.argv, only=only)
