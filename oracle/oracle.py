"""CPU oracle for GPU-TO's MGCG solve and the top3D125 design loop around it.

TEST INFRASTRUCTURE ONLY.  This module is the checker that the CUDA product
is compared against.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import it; the product never does.

Two CPU implementations live behind it:

* ``liboracle.so`` -- this project's C restatement (``topo_oracle.c``) of
  ``Cantilever/TOP3D125MGCGCUDA/mgcg1.cu`` plus the element-level design steps;
* ``_ref/libmgcg1_omp_ref.so`` -- the reference's own, unmodified
  ``Cantilever/omp/mgcg1.c`` compiled against a project-written MEX stand-in
  (built by ``oracle/Makefile`` where the reference tree exists).  It pins the
  restatement.

The numpy parts restate ``Cantilever/TOP3D125MGCGCUDA/top3D125modCuda.m``:
SIMP (``:124,130``), Heaviside projection with the eta Newton solve
(``:60-64,111-119``), the OC bisection (``:143-151``) and continuation (``:64,152``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libmgcg1_omp_ref.so")

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def build(force: bool = False) -> None:
    """Compile liboracle.so (and _ref when the reference tree is present)."""
    if force or not os.path.exists(LIB_PATH) or (
        os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "topo_oracle.c"))
    ):
        subprocess.run(["make", "-s", "-C", HERE, os.path.join(HERE, "liboracle.so")], check=True)
    if force or not os.path.exists(REF_PATH):
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


class _Opts(ctypes.Structure):
    _fields_ = [("nswp", ctypes.c_int), ("omega", ctypes.c_double),
                ("prerelax", ctypes.c_double), ("nu", ctypes.c_double), ("coarse", ctypes.c_int)]


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.or_hex8_stiffness.argtypes = [ctypes.c_double] * 4 + [_dp]
        L.or_hex8_gauss_parts.argtypes = [ctypes.c_double] * 4 + [_dp]
        L.or_apply_fine.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_mgcg1.argtypes = [_dp, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                               ctypes.POINTER(_Opts), _dp, ctypes.POINTER(ctypes.c_int), _dp]
        L.or_vcycle_apply.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, ctypes.POINTER(_Opts), _dp, _dp]
        L.or_element_energy.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_filter3d.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.or_filter3d.restype = ctypes.c_double
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref():
    global _ref
    if _ref is None:
        L = ctypes.CDLL(REF_PATH)
        L.ref_omp_workspace.argtypes = [ctypes.c_int] * 5
        L.ref_omp_workspace.restype = ctypes.c_int
        L.ref_omp_mgcg1.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_long, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_int)]
        L.ref_omp_mgcg1.restype = ctypes.c_int
        _ref = L
    return _ref


# --------------------------------------------------------------------------
# grid and problem helpers
# --------------------------------------------------------------------------

def ndof(nelx, nely, nelz):
    return 3 * (nelx + 1) * (nely + 1) * (nelz + 1)


def node_id(nelx, nely, nelz, i, j, k):
    return (nelz + 1) * (nely + 1) * i + (nely + 1) * k + j


def hex8_stiffness(nu=0.3, h=1.0):
    Ke = np.zeros(576)
    lib().or_hex8_stiffness(nu, h, h, h, _ptr(Ke))
    return Ke.reshape(24, 24)


def hex8_gauss_parts(nu=0.3, h=1.0):
    Kg = np.zeros(8 * 576)
    lib().or_hex8_gauss_parts(nu, h, h, h, _ptr(Kg))
    return Kg.reshape(8, 24, 24)


@dataclass
class Problem:
    """A hex8 voxel-grid elasticity problem in the MEX's argument layout."""
    nelx: int
    nely: int
    nelz: int
    F: np.ndarray            # ndof, MATLAB frame (no y loads, so same as solver frame)
    fixed: np.ndarray        # 1-based dof indices, float64 (as MATLAB passes them)
    Ke0: np.ndarray = field(default_factory=lambda: hex8_stiffness(0.3))

    @property
    def ndof(self):
        return ndof(self.nelx, self.nely, self.nelz)

    @property
    def nel(self):
        return self.nelx * self.nely * self.nelz


def cantilever(nelx, nely, nelz, load="edge"):
    """Cantilever of the benchmark configs: x=0 face clamped
    (``fixed = 1:3(nely+1)(nelz+1)``, top3D125modCuda.m:80) and a unit total
    downward (-z) load on the bottom edge (k=0) of the free end x=nelx.
    ``load="sin"`` uses the reference drivers' -sin profile (:82) instead."""
    n = ndof(nelx, nely, nelz)
    F = np.zeros(n)
    js = np.arange(nely + 1)
    nodes = node_id(nelx, nely, nelz, nelx, js, 0)
    if load == "edge":
        F[3 * nodes + 2] = -1.0 / (nely + 1)
    else:
        F[3 * nodes + 2] = -np.sin(js / nely * np.pi)
    fixed = np.arange(1, 3 * (nely + 1) * (nelz + 1) + 1, dtype=np.float64)
    return Problem(nelx, nely, nelz, F, fixed)


def random_density(nelx, nely, nelz, seed=0, lo=1e-3, hi=1.0, smooth=2):
    """Seeded smooth random density in [lo, hi] (element order)."""
    rng = np.random.default_rng(seed)
    x = rng.random((nelx, nelz, nely))
    for _ in range(smooth):
        x = (x + np.roll(x, 1, 0) + np.roll(x, -1, 0) + np.roll(x, 1, 1) + np.roll(x, -1, 1)
             + np.roll(x, 1, 2) + np.roll(x, -1, 2)) / 7.0
    x = (x - x.min()) / max(x.max() - x.min(), 1e-30)
    return (lo + (hi - lo) * x).reshape(-1).copy()


def simp(xphys, penal=3.0, E0=1.0, Emin=1e-9):
    """CX and dsK (top3D125modCuda.m:124,130)."""
    CX = Emin + xphys ** penal * (E0 - Emin)
    dsK = -penal * (E0 - Emin) * xphys ** (penal - 1)
    return CX, dsK


# --------------------------------------------------------------------------
# solver restatement and the compiled reference
# --------------------------------------------------------------------------

def bridge(nelx, nely, nelz):
    """Bridge supports and load, restated from ArchBridge/1/top3D125modCudaBridge1.m:79-99
    (fixed corner nodes at the bottom of both x ends, widened here to the two
    bottom edge lines; top-face pressure as -0.25 per element on each top
    node's z dof, :90-98), scaled to a unit total load.  Written as the
    per-element loop of the driver so it checks the vectorised product
    version independently."""
    n = ndof(nelx, nely, nelz)
    F = np.zeros(n)
    for i in range(nelx):
        for j in range(nely):
            for di in (0, 1):
                for dj in (0, 1):
                    nod = node_id(nelx, nely, nelz, i + di, j + dj, nelz)
                    F[3 * nod + 2] -= 0.25 / (nelx * nely)
    fixed = []
    for i in (0, nelx):
        for j in range(nely + 1):
            nod = node_id(nelx, nely, nelz, i, j, 0)
            fixed += [3 * nod + 1, 3 * nod + 2, 3 * nod + 3]
    fixed = np.array(sorted(fixed), dtype=np.float64)
    F[fixed.astype(np.int64) - 1] = 0.0
    return Problem(nelx, nely, nelz, F, fixed)


def mgcg1(p: Problem, CX, nl, tol, maxit, nswp=3, omega=0.48, prerelax=0.7, nu=0.3,
          history=False, coarse=0):
    """Restatement of the MEX: returns (U, relres, nit[, res_history]).
    coarse=1 gives the mgcg9 hierarchy (re-discretised levels)."""
    U = np.zeros(p.ndof)
    rr = ctypes.c_double(0.0)
    nit = ctypes.c_int(0)
    o = _Opts(nswp, omega, prerelax, nu, coarse)
    hist = np.zeros(max(maxit, 1) + 1)
    CX = np.ascontiguousarray(CX, dtype=np.float64)
    st = lib().or_mgcg1(_ptr(p.Ke0.reshape(-1).copy()), _ptr(p.F), _ptr(U), _ptr(CX),
                        _ptr(p.fixed), len(p.fixed), p.nelx, p.nely, p.nelz, nl, tol, maxit,
                        ctypes.byref(o), ctypes.byref(rr), ctypes.byref(nit), _ptr(hist))
    if st:
        raise RuntimeError(f"oracle mgcg1 failed with status {st}")
    if history:
        return U, rr.value, nit.value, hist[: nit.value + 1]
    return U, rr.value, nit.value


def vcycle(p: Problem, CX, nl, r, nswp=3, omega=0.48, prerelax=0.7, nu=0.3, coarse=0):
    z = np.zeros(p.ndof)
    o = _Opts(nswp, omega, prerelax, nu, coarse)
    st = lib().or_vcycle_apply(_ptr(p.Ke0.reshape(-1).copy()), _ptr(np.ascontiguousarray(CX)),
                               _ptr(p.fixed), len(p.fixed), p.nelx, p.nely, p.nelz, nl,
                               ctypes.byref(o), _ptr(np.ascontiguousarray(r)), _ptr(z))
    if st:
        raise RuntimeError(f"oracle vcycle failed with status {st}")
    return z


def apply_fine(p: Problem, CX, u):
    r = np.zeros(p.ndof)
    lib().or_apply_fine(_ptr(p.Ke0.reshape(-1).copy()), _ptr(np.ascontiguousarray(CX)),
                        _ptr(np.ascontiguousarray(u)), _ptr(r), p.nelx, p.nely, p.nelz)
    return r


def mgcg9(p: Problem, CX, nl, tol, maxit, nswp=2, history=False):
    """Restatement of the MEX mgcg9 (Homogenization/QNC/mgcg9.cu): the mgcg1
    PCG with re-discretised coarse levels and damped Jacobi omega = 0.33
    (mgcg9.cu:929-935), nswp from the call."""
    return mgcg1(p, CX, nl, tol, maxit, nswp=nswp, omega=0.33, prerelax=0.7, history=history, coarse=1)


def ref_mgcg1(p: Problem, CX, nl, tol, maxit, workdir=None):
    """Run the reference's own compiled OpenMP MEX.  Returns (U, relres, nit)."""
    L = ref()
    lenW = L.ref_omp_workspace(len(p.fixed), nl, p.nelx, p.nely, p.nelz)
    W = np.zeros(lenW)
    U = np.zeros(p.ndof)
    rr = ctypes.c_double(0.0)
    nit = ctypes.c_int(0)
    CX = np.ascontiguousarray(CX, dtype=np.float64)
    cwd = os.getcwd()
    tmp = workdir or tempfile.mkdtemp(prefix="mgcg1_ref_")
    os.chdir(tmp)  # the reference writes mgcg1.log into the working directory
    try:
        L.ref_omp_mgcg1(_ptr(p.Ke0.reshape(-1).copy()), _ptr(p.F), _ptr(U), _ptr(CX),
                        _ptr(p.fixed), _ptr(W), lenW, len(p.fixed), p.nelx, p.nely, p.nelz,
                        nl, tol, maxit, ctypes.byref(rr), ctypes.byref(nit))
    finally:
        os.chdir(cwd)
    return U, rr.value, nit.value


def element_energy(p: Problem, U):
    ce = np.zeros(p.nel)
    lib().or_element_energy(_ptr(p.Ke0.reshape(-1).copy()), _ptr(np.ascontiguousarray(U)),
                            _ptr(ce), p.nelx, p.nely, p.nelz)
    return ce


def filter3d(v, nelx, nely, nelz, rmin):
    """imfilter(reshape(v,nely,nelz,nelx), h, 'symmetric'); returns (out, Hs)."""
    out = np.zeros(nelx * nely * nelz)
    hs = lib().or_filter3d(_ptr(np.ascontiguousarray(v, dtype=np.float64)), _ptr(out),
                           nelx, nely, nelz, rmin)
    return out, hs


# --------------------------------------------------------------------------
# design loop (top3D125modCuda.m:105-166)
# --------------------------------------------------------------------------

def prj(v, eta, beta):
    return (np.tanh(beta * eta) + np.tanh(beta * (v - eta))) / (
        np.tanh(beta * eta) + np.tanh(beta * (1 - eta)))


def deta(v, eta, beta):
    return (-beta / np.sinh(beta) / np.cosh(beta * (v - eta)) ** 2
            * np.sinh(v * beta) * np.sinh((1 - v) * beta))


def dprj(v, eta, beta):
    return beta * (1 - np.tanh(beta * (v - eta)) ** 2) / (
        np.tanh(beta * eta) + np.tanh(beta * (1 - eta)))


def cnt(v, vcnt, loop):
    return v + (loop >= vcnt[0]) * (v < vcnt[1]) * (loop % vcnt[2] == 0) * vcnt[3]


def oc_update(x, dc, dv0, volfrac, move):
    """OC resizing with bisection on the multiplier (top3D125modCuda.m:143-151)."""
    xU, xL = x + move, x - move
    ocP = x * np.sqrt(-dc / dv0)
    l1, l2 = 0.0, ocP.mean() / volfrac
    xnew = x
    lmid = 0.5 * (l1 + l2)
    while (l2 - l1) / (l2 + l1) > 1e-4:
        lmid = 0.5 * (l1 + l2)
        xnew = np.maximum(np.maximum(np.minimum(np.minimum(ocP / lmid, xU), 1.0), xL), 0.0)
        if xnew.mean() > volfrac:
            l1 = lmid
        else:
            l2 = lmid
    return xnew, lmid


@dataclass
class DesignConfig:
    nl: int
    volfrac: float = 0.12
    penal: float = 3.0
    rmin: float = 3 ** 0.5
    ft: int = 1            # 1: density filter only; 3: plus Heaviside projection
    eta: float = 0.4
    beta: float = 2.0
    move: float = 0.2
    E0: float = 1.0
    Emin: float = 1e-9
    tol: float = 1e-8
    maxit: int = 200
    iters: int = 50


def design_loop(p: Problem, cfg: DesignConfig, solver=None, callback=None):
    """Run ``cfg.iters`` design iterations with the given MEX-like solver
    (defaults to the oracle restatement).  Returns a dict of the history."""
    solver = solver or (lambda CX: mgcg1(p, CX, cfg.nl, cfg.tol, cfg.maxit))
    nelx, nely, nelz = p.nelx, p.nely, p.nelz
    nel = p.nel
    x = np.full(nel, cfg.volfrac)
    dV = np.full(nel, 1.0 / nel / cfg.volfrac)
    _, hs = filter3d(np.ones(nel), nelx, nely, nelz, cfg.rmin)
    Hs = np.full(nel, hs)
    xPhys = x.copy()
    xOld = np.ones(nel)
    eta, beta, penal = cfg.eta, cfg.beta, cfg.penal
    hist = {"c": [], "nit": [], "relres": [], "ch": [], "lmid": []}
    for loop in range(1, cfg.iters + 1):
        xTilde = filter3d(x, nelx, nely, nelz, cfg.rmin)[0] / Hs
        xPhys = xTilde
        dHs = Hs
        if cfg.ft > 1:
            f = (prj(xPhys, eta, beta).mean() - cfg.volfrac) * (cfg.ft == 3)
            while abs(f) > 1e-6:
                eta = eta - f / deta(xPhys, eta, beta).mean()
                f = prj(xPhys, eta, beta).mean() - cfg.volfrac
            dHs = Hs / dprj(xPhys, eta, beta)
            xPhys = prj(xPhys, eta, beta)
        ch = np.linalg.norm(xPhys - xOld) / nel
        xOld = xPhys
        CX = cfg.Emin + xPhys ** penal * (cfg.E0 - cfg.Emin)
        dsK = -penal * (cfg.E0 - cfg.Emin) * xPhys ** (penal - 1)
        U, relres, nit = solver(CX)
        # the MEX returns U in the MATLAB frame (y negated); MATLAB's U(cMat)
        # gather is y-mirrored to match, so the C-order gather here needs the
        # solver frame back
        Uc = U.copy()
        Uc[1::3] *= -1.0
        ce = element_energy(p, Uc)
        dc = dsK * ce
        dc = filter3d(dc / dHs, nelx, nely, nelz, cfg.rmin)[0]
        dV0 = filter3d(dV / dHs, nelx, nely, nelz, cfg.rmin)[0]
        x, lmid = oc_update(x, dc, dV0, cfg.volfrac, cfg.move)
        penal = cnt(penal, (1, 1, 25, 0.25), loop)
        beta = cnt(beta, (1, 1, 25, 2), loop)
        c = float(p.F @ U)
        for k, v in (("c", c), ("nit", nit), ("relres", relres), ("ch", ch), ("lmid", lmid)):
            hist[k].append(v)
        if callback:
            callback(loop, x, xPhys, U, c)
    hist["x"] = x
    hist["xPhys"] = xPhys
    return hist
