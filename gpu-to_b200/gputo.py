"""Python host binding of the gputo C ABI (include/gputo.h).

``mgcg1`` mirrors the MATLAB MEX call of the top3D125 MGCG drivers argument
for argument (Cantilever/TOP3D125MGCGCUDA/top3D125modCuda.m:134):

    cgres, cgiters = mgcg1(Ke0, F1, U, CX, fixed, nfd, nelx, nely, nelz, nl, cgtol, cgmax[, printLev])

U is written in place (its input values are ignored, y components come back
negated, as the MEX returns them) and ``cgiters`` is -1 when device memory is
insufficient, like the reference (mgcg1.cu:166-174).

``Solver`` wraps the device-resident API for callers that keep their fields in
HBM (torch tensors or raw device pointers); ``compliance_sens`` and
``density_filter`` are the design-loop steps of the driver.

There is no CPU fallback: importing this module loads the CUDA library and
raises if it is missing, and every call fails with a ``GputoError`` when no
sm_100 device is present.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgputo.so")
MEX_PATH = os.path.join(HERE, "lib", "libgputo_mex.so")

GPUTO_OK = 0
GPUTO_ERR_ARG = 1
GPUTO_ERR_CUDA = 2
GPUTO_ERR_OOM = 3
GPUTO_ERR_NOT_SPD = 4
GPUTO_ERR_BREAKDOWN = 5
GPUTO_ERR_NO_DEVICE = 6
GPUTO_ERR_TIMEOUT = 7

PREC_FP64 = 0
PREC_MIXED = 1

# Every function the header declares, with (restype, argtypes).
_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int)
_i = ctypes.c_int
_d = ctypes.c_double


class Options(ctypes.Structure):
    _fields_ = [("precision", _i), ("nswp", _i), ("omega", _d), ("prerelax", _d), ("nu", _d),
                ("check_every", _i), ("use_graph", _i), ("max_coarse_dofs", _i)]


SIGNATURES = {
    "gputo_status_string": (ctypes.c_char_p, [_i]),
    "gputo_last_error": (ctypes.c_char_p, []),
    "gputo_version": (ctypes.c_char_p, []),
    "gputo_default_options": (None, [ctypes.POINTER(Options)]),
    "gputo_mgcg1": (_i, [_dp, _dp, _dp, _dp, _dp, _i, _i, _i, _i, _i, _d, _i, _i, _dp, _ip]),
    "gputo_mgcg1_ex": (_i, [_dp, _dp, _dp, _dp, _dp, _i, _i, _i, _i, _i, _d, _i, _i,
                            ctypes.POINTER(Options), _dp, _ip]),
    "gputo_solver_create": (_i, [ctypes.POINTER(_vp), _i, _i, _i, _i, ctypes.POINTER(Options)]),
    "gputo_solver_destroy": (None, [_vp]),
    "gputo_solver_device_bytes": (ctypes.c_size_t, [_vp]),
    "gputo_solver_set_problem": (_i, [_vp, _dp, _dp, _i]),
    "gputo_solver_setup_dev": (_i, [_vp, _vp, _vp]),
    "gputo_solver_solve_dev": (_i, [_vp, _vp, _vp, _d, _i, _dp, _ip, _vp]),
    "gputo_solver_vcycle_dev": (_i, [_vp, _vp, _vp, _vp]),
    "gputo_solver_apply_dev": (_i, [_vp, _vp, _vp, _vp]),
    "gputo_solver_launch_count": (ctypes.c_longlong, [_vp]),
    "gputo_compliance_sens_dev": (_i, [_dp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _dp, _vp]),
    "gputo_compliance_sens": (_i, [_dp, _dp, _dp, _dp, _i, _i, _i, _dp, _dp, _dp]),
    "gputo_density_filter_dev": (_i, [_vp, _vp, _vp, _i, _i, _i, _d, _i, _vp]),
    "gputo_density_filter": (_i, [_dp, _dp, _dp, _i, _i, _i, _d, _i]),
}


class GputoError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        msg = _lib.gputo_status_string(status).decode()
        detail = _lib.gputo_last_error().decode()
        super().__init__(f"{where}: {msg}" + (f" ({detail})" if detail else ""))


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"gputo CUDA library not built: {LIB_PATH} (run gpu-to_b200/build.py)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = _load()


def lib():
    return _lib


def _check(st: int, where: str):
    if st != GPUTO_OK:
        raise GputoError(st, where)


def _p(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_dp)


def default_options(**kw) -> Options:
    o = Options()
    _lib.gputo_default_options(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise AttributeError(k)
        setattr(o, k, v)
    return o


def version() -> str:
    return _lib.gputo_version().decode()


def mgcg1(Ke0, F1, U, CX, fixed, nfd, nelx, nely, nelz, nl, cgtol, cgmax, printLev=1,
          options: Options | None = None):
    """The MEX call.  Returns (cgres, cgiters); U (float64 ndarray) is written in place.
    Out-of-memory returns cgiters = -1 as the reference does; any other failure
    raises GputoError (the reference would exit the MATLAB process)."""
    Ke0 = np.ascontiguousarray(Ke0, dtype=np.float64)
    F1 = np.ascontiguousarray(F1, dtype=np.float64).reshape(-1)
    CX = np.ascontiguousarray(CX, dtype=np.float64).reshape(-1)
    fixed = np.ascontiguousarray(fixed, dtype=np.float64).reshape(-1)
    if not (isinstance(U, np.ndarray) and U.dtype == np.float64 and U.flags.c_contiguous):
        raise TypeError("U must be a C-contiguous float64 ndarray (written in place)")
    nelx, nely, nelz, nl, nfd = int(nelx), int(nely), int(nelz), int(nl), int(nfd)
    nd = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    if F1.size != nd or U.size != nd or CX.size != nelx * nely * nelz or Ke0.size != 576 \
            or fixed.size < nfd:
        raise ValueError("argument sizes do not match nelx/nely/nelz/nfd")
    rr = ctypes.c_double(0.0)
    nit = ctypes.c_int(-1)
    if options is None:
        st = _lib.gputo_mgcg1(_p(Ke0.reshape(-1)), _p(F1), _p(U.reshape(-1)), _p(CX), _p(fixed), nfd,
                              nelx, nely, nelz, nl, float(cgtol), int(cgmax), int(printLev),
                              ctypes.byref(rr), ctypes.byref(nit))
    else:
        st = _lib.gputo_mgcg1_ex(_p(Ke0.reshape(-1)), _p(F1), _p(U.reshape(-1)), _p(CX), _p(fixed),
                                 nfd, nelx, nely, nelz, nl, float(cgtol), int(cgmax), int(printLev),
                                 ctypes.byref(options), ctypes.byref(rr), ctypes.byref(nit))
    if st == GPUTO_ERR_OOM:
        return 0.0, -1
    if st not in (GPUTO_OK, GPUTO_ERR_BREAKDOWN):
        raise GputoError(st, "mgcg1")
    return rr.value, nit.value


def _ptr(t) -> int:
    """Device address of a torch tensor (or an int address)."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


class Solver:
    """Device-resident MGCG solver for one grid shape (gputo_solver_*)."""

    def __init__(self, nelx, nely, nelz, nl, options: Options | None = None):
        self._h = ctypes.c_void_p()
        self.shape = (int(nelx), int(nely), int(nelz))
        self.nl = int(nl)
        self.options = options or default_options()
        _check(_lib.gputo_solver_create(ctypes.byref(self._h), *self.shape, self.nl,
                                        ctypes.byref(self.options)), "gputo_solver_create")

    def close(self):
        if self._h:
            _lib.gputo_solver_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        return int(_lib.gputo_solver_device_bytes(self._h))

    def set_problem(self, Ke0, fixed):
        Ke0 = np.ascontiguousarray(Ke0, dtype=np.float64).reshape(-1)
        fixed = np.ascontiguousarray(fixed, dtype=np.float64).reshape(-1)
        _check(_lib.gputo_solver_set_problem(self._h, _p(Ke0), _p(fixed), fixed.size),
               "gputo_solver_set_problem")

    def setup(self, CX, stream=None):
        _check(_lib.gputo_solver_setup_dev(self._h, _ptr(CX), _ptr_stream(stream)),
               "gputo_solver_setup_dev")

    def solve(self, F, U, tol, maxit, stream=None):
        rr = ctypes.c_double(0.0)
        nit = ctypes.c_int(0)
        st = _lib.gputo_solver_solve_dev(self._h, _ptr(F), _ptr(U), float(tol), int(maxit),
                                         ctypes.byref(rr), ctypes.byref(nit), _ptr_stream(stream))
        _check(st, "gputo_solver_solve_dev")
        return rr.value, nit.value

    def vcycle(self, r, z, stream=None):
        _check(_lib.gputo_solver_vcycle_dev(self._h, _ptr(r), _ptr(z), _ptr_stream(stream)),
               "gputo_solver_vcycle_dev")

    def apply(self, u, r, stream=None):
        _check(_lib.gputo_solver_apply_dev(self._h, _ptr(u), _ptr(r), _ptr_stream(stream)),
               "gputo_solver_apply_dev")


def _ptr_stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream  # torch.cuda.Stream


def launch_count() -> int:
    return int(_lib.gputo_solver_launch_count(None))


def compliance_sens(Ke0, U, CX, dsK, nelx, nely, nelz):
    """Host-buffer form (U in the MATLAB frame): returns (ce, dc, compliance)."""
    Ke0 = np.ascontiguousarray(Ke0, dtype=np.float64).reshape(-1)
    U = np.ascontiguousarray(U, dtype=np.float64)
    CX = np.ascontiguousarray(CX, dtype=np.float64)
    dsK = np.ascontiguousarray(dsK, dtype=np.float64)
    ne = nelx * nely * nelz
    ce = np.zeros(ne)
    dc = np.zeros(ne)
    c = ctypes.c_double(0.0)
    _check(_lib.gputo_compliance_sens(_p(Ke0), _p(U), _p(CX), _p(dsK), nelx, nely, nelz, _p(ce),
                                      _p(dc), ctypes.byref(c)), "gputo_compliance_sens")
    return ce, dc, c.value


def compliance_sens_dev(Ke0, U, CX, dsK, nelx, nely, nelz, ce=None, dc=None, stream=None):
    """Device form on torch tensors (U in the solver frame); returns the compliance."""
    Ke0 = np.ascontiguousarray(Ke0, dtype=np.float64).reshape(-1)
    c = ctypes.c_double(0.0)
    _check(_lib.gputo_compliance_sens_dev(_p(Ke0), _ptr(U), _ptr(CX), _ptr(dsK), nelx, nely, nelz,
                                          _ptr(ce), _ptr(dc), ctypes.byref(c), _ptr_stream(stream)),
           "gputo_compliance_sens_dev")
    return c.value


def density_filter(x, nelx, nely, nelz, rmin, divisor=None, normalize=True):
    """Host-buffer form of the driver's imfilter calls."""
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    out = np.zeros_like(x)
    dv = None if divisor is None else np.ascontiguousarray(divisor, dtype=np.float64).reshape(-1)
    _check(_lib.gputo_density_filter(_p(x), None if dv is None else _p(dv), _p(out), nelx, nely,
                                     nelz, float(rmin), int(bool(normalize))), "gputo_density_filter")
    return out


def density_filter_dev(x, out, nelx, nely, nelz, rmin, divisor=None, normalize=True, stream=None):
    _check(_lib.gputo_density_filter_dev(_ptr(x), _ptr(divisor), _ptr(out), nelx, nely, nelz,
                                         float(rmin), int(bool(normalize)), _ptr_stream(stream)),
           "gputo_density_filter_dev")
