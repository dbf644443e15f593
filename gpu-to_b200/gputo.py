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
_fp = ctypes.POINTER(ctypes.c_float)


class Options(ctypes.Structure):
    _fields_ = [("precision", _i), ("nswp", _i), ("omega", _d), ("prerelax", _d), ("nu", _d),
                ("check_every", _i), ("use_graph", _i), ("max_coarse_dofs", _i), ("tc_parts", _i),
                ("tc_xchunk", _i), ("coarse", _i), ("fine_op", _i), ("nswp_fine", _i),
                ("fuse_prolong", _i), ("sweep_xchunk", _i), ("sweep_pairs", _i), ("nswp_coarse", _i),
                ("coarse_from", _i)]


SIGNATURES = {
    "gputo_status_string": (ctypes.c_char_p, [_i]),
    "gputo_last_error": (ctypes.c_char_p, []),
    "gputo_version": (ctypes.c_char_p, []),
    "gputo_default_options": (None, [ctypes.POINTER(Options)]),
    "gputo_hex8_stiffness": (_i, [_d, _d, _dp]),
    "gputo_fine_op_constants": (_i, [_dp, _dp]),
    "gputo_mgcg1": (_i, [_dp, _dp, _dp, _dp, _dp, _i, _i, _i, _i, _i, _d, _i, _i, _dp, _ip]),
    "gputo_mgcg1_ex": (_i, [_dp, _dp, _dp, _dp, _dp, _i, _i, _i, _i, _i, _d, _i, _i,
                            ctypes.POINTER(Options), _dp, _ip]),
    "gputo_design_save": (_i, [ctypes.c_char_p, _i, _i, _i, _i, _dp, _i, _dp, _dp]),
    "gputo_design_load": (_i, [ctypes.c_char_p, _ip, _ip, _ip, _ip, _dp, _ip, _dp, _dp]),
    "gputo_design_export_volume": (_i, [ctypes.c_char_p, _i, _i, _i, _dp]),
    "gputo_heaviside_dev": (_i, [_vp, ctypes.c_longlong, _d, _d, _dp, _vp, _vp, _vp]),
    "gputo_mul_dev": (_i, [_vp, _vp, _vp, ctypes.c_longlong, _vp]),
    "gputo_mgcg9": (_i, [_dp, _dp, _dp, _dp, _dp, _i, _i, _i, _i, _i, _d, _i, _i, _i, _d, _d, _d, _d, _dp, _ip]),
    "gputo_solver_create": (_i, [ctypes.POINTER(_vp), _i, _i, _i, _i, ctypes.POINTER(Options)]),
    "gputo_solver_destroy": (None, [_vp]),
    "gputo_solver_apply_fp32_dev": (_i, [_vp, _vp, _vp, _i, _vp]),
    "gputo_batch_create": (_i, [ctypes.POINTER(_vp), ctypes.POINTER(_vp), _i]),
    "gputo_batch_destroy": (None, [_vp]),
    "gputo_batch_solve_dev": (_i, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp), _d, _i, _i, _dp, _ip]),
    "gputo_solver_set_options": (_i, [_vp, ctypes.POINTER(Options)]),
    "gputo_autotune_dev": (_i, [_vp, _vp, _vp, _d, _i, ctypes.POINTER(Options), _dp, _dp, _ip, _i, _ip]),
    "gputo_net_num_params": (ctypes.c_longlong, []),
    "gputo_net_create": (_i, [ctypes.POINTER(_vp), ctypes.c_ulonglong]),
    "gputo_net_destroy": (None, [_vp]),
    "gputo_net_get_params": (_i, [_vp, _fp]),
    "gputo_net_set_params": (_i, [_vp, _fp]),
    "gputo_net_forward_dev": (_i, [_vp, _vp, _i, _i, _i, _vp, _vp]),
    "gputo_net_train_step_dev": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, _i, ctypes.c_float, _dp, _fp, _vp]),
    "gputo_solver_set_net": (_i, [_vp, _vp, _i]),
    "gputo_solver_net_state": (_i, [_vp, _ip, _ip, _ip]),
    "gputo_solver_net_dims": (_i, [_vp, _ip, _ip, _ip]),
    "gputo_solver_net_features_dev": (_i, [_vp, _vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_float), _vp]),
    "gputo_solver_level2_inject_dev": (_i, [_vp, _vp, _vp, _vp]),
    "gputo_solver_net_energy_rhs_dev": (_i, [_vp, _vp, ctypes.c_float, _vp, _vp]),
    "gputo_solver_net_train_step_dev": (_i, [_vp, _vp, _vp, _vp, _i, ctypes.c_float, _dp, _fp, _vp]),
    "gputo_solver_device_bytes": (ctypes.c_size_t, [_vp]),
    "gputo_solver_set_problem": (_i, [_vp, _dp, _dp, _i]),
    "gputo_solver_setup_dev": (_i, [_vp, _vp, _vp]),
    "gputo_solver_solve_dev": (_i, [_vp, _vp, _vp, _d, _i, _dp, _ip, _vp]),
    "gputo_solver_vcycle_dev": (_i, [_vp, _vp, _vp, _vp]),
    "gputo_solver_apply_dev": (_i, [_vp, _vp, _vp, _vp]),
    "gputo_solver_launch_count": (ctypes.c_longlong, [_vp]),
    "gputo_solver_time_kernel": (_i, [_vp, _i, _i, _dp, _vp]),
    "gputo_debug_set_sweep_fault": (_i, [_i, ctypes.c_uint]),
    "gputo_solver_energy_dev": (_i, [_vp, _vp, _vp, _vp, _dp, _dp, _vp]),
    "gputo_homog_create": (_i, [ctypes.POINTER(_vp), _i, _i, _i, _i, ctypes.POINTER(Options)]),
    "gputo_homog_destroy": (None, [_vp]),
    "gputo_homog_device_bytes": (ctypes.c_size_t, [_vp]),
    "gputo_homog_solve_dev": (_i, [_vp, _dp, _vp, _d, _i, _dp, _dp, ctypes.POINTER(_i), _vp, _vp]),
    "gputo_compliance_sens_dev": (_i, [_dp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _dp, _vp]),
    "gputo_compliance_sens": (_i, [_dp, _dp, _dp, _dp, _i, _i, _i, _dp, _dp, _dp]),
    "gputo_compliance_sens_tc_dev": (_i, [_dp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _dp, _vp]),
    "gputo_compliance_sens_noalloc_dev": (_i, [_dp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _dp, _vp]),
    "gputo_density_filter_dev": (_i, [_vp, _vp, _vp, _i, _i, _i, _d, _i, _vp]),
    "gputo_time_filter_dev": (_i, [_vp, _vp, _i, _i, _i, _i, _d, _i, _dp, _vp]),
    "gputo_density_filter": (_i, [_dp, _dp, _dp, _i, _i, _i, _d, _i]),
    "gputo_simp_dev": (_i, [_vp, ctypes.c_longlong, _d, _d, _d, _vp, _vp, _vp]),
    "gputo_simp": (_i, [_dp, ctypes.c_longlong, _d, _d, _d, _dp, _dp]),
    "gputo_oc_update_dev": (_i, [_vp, _vp, _vp, ctypes.c_longlong, _d, _d, _vp, _dp, _vp]),
    "gputo_oc_update": (_i, [_dp, _dp, _dp, ctypes.c_longlong, _d, _d, _dp, _dp]),
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


def hex8_stiffness(nu=0.3, h=1.0) -> np.ndarray:
    """The drivers' Ke0 (24x24) computed by the library (host only)."""
    Ke = np.zeros(576)
    _check(_lib.gputo_hex8_stiffness(float(nu), float(h), _p(Ke)), "gputo_hex8_stiffness")
    return Ke.reshape(24, 24)


def fine_op_constants(Ke):
    """The eight Hadamard-basis constants of Ke, or None when Ke lacks the
    pattern (then the fine sweeps use dense element rows)."""
    Ke = np.ascontiguousarray(Ke, dtype=np.float64).reshape(-1)
    c = np.zeros(8)
    st = _lib.gputo_fine_op_constants(_p(Ke), _p(c))
    return c if st == GPUTO_OK else None


def cantilever(nelx, nely, nelz):
    """Load and supports of the benchmark cantilever: x = 0 face clamped
    (fixed = 1:3(nely+1)(nelz+1), top3D125modCuda.m:80) and a unit total -z
    load spread over the bottom edge (k = 0) of the free end x = nelx.
    Returns (F, fixed) in the MEX's layout."""
    nd = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    F = np.zeros(nd)
    js = np.arange(nely + 1)
    nodes = (nelz + 1) * (nely + 1) * nelx + js
    F[3 * nodes + 2] = -1.0 / (nely + 1)
    fixed = np.arange(1, 3 * (nely + 1) * (nelz + 1) + 1, dtype=np.float64)
    return F, fixed


def bridge(nelx, nely, nelz):
    """Supports and load of the bridge workload (the ArchBridge drivers'
    layout, ArchBridge/1/top3D125modCudaBridge1.m:79-99, widened from its four
    corner nodes to the two bottom corner strips): every node of the bottom
    (k = 0) edge lines at x = 0 and x = nelx fixed in all three directions,
    and a uniform downward pressure of unit total on the top face (k = nelz),
    each top element giving a quarter of its share to the z dof of each of its
    four top nodes.  Returns (F, fixed) in the MEX's layout."""
    nd = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    F = np.zeros(nd)
    js = np.arange(nely + 1)
    plane = (nely + 1) * (nelz + 1)
    # nodal weight of the top face: 1, 2 or 4 elements touch a node
    wy = np.full(nely + 1, 2.0)
    wy[[0, -1]] = 1.0
    wx = np.full(nelx + 1, 2.0)
    wx[[0, -1]] = 1.0
    top = (np.arange(nelx + 1)[:, None] * plane + (nely + 1) * nelz + js[None, :]).reshape(-1)
    F[3 * top + 2] = -0.25 / (nelx * nely) * (wx[:, None] * wy[None, :]).reshape(-1)
    ends = np.concatenate([js, nelx * plane + js])   # k = 0 lines at i = 0 and i = nelx
    fixed = np.sort((3 * ends[:, None] + np.arange(3)[None, :]).reshape(-1)) + 1.0
    F[fixed.astype(np.int64) - 1] = 0.0
    return F, fixed


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
    if st == GPUTO_ERR_BREAKDOWN:   # as the MEX: U holds the last iterate, cgiters = -1
        return rr.value, -1
    if st != GPUTO_OK:
        raise GputoError(st, "mgcg1")
    return rr.value, nit.value


def mgcg9(Ae, F, U, CX, FDofs, nFD, nelx, nely, nelz, nl, tol, maxit, nswp, printLev=1, nu=0.3, hx=1.0,
          hy=1.0, hz=1.0):
    """The MEX mgcg9 call (18 arguments).  Returns (cgres, cgiters); U is written in place."""
    Ae = np.ascontiguousarray(Ae, dtype=np.float64).reshape(-1)
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(-1)
    CX = np.ascontiguousarray(CX, dtype=np.float64).reshape(-1)
    FDofs = np.ascontiguousarray(FDofs, dtype=np.float64).reshape(-1)
    if not (isinstance(U, np.ndarray) and U.dtype == np.float64 and U.flags.c_contiguous):
        raise TypeError("U must be a C-contiguous float64 ndarray (written in place)")
    nd = 3 * (int(nelx) + 1) * (int(nely) + 1) * (int(nelz) + 1)
    if F.size != nd or U.size != nd or CX.size != int(nelx) * int(nely) * int(nelz) or Ae.size != 576 \
            or FDofs.size < int(nFD):
        raise ValueError("argument sizes do not match nelx/nely/nelz/nFD")
    rr = ctypes.c_double(0.0)
    nit = ctypes.c_int(-1)
    st = _lib.gputo_mgcg9(_p(Ae), _p(F), _p(U.reshape(-1)), _p(CX), _p(FDofs), int(nFD), int(nelx), int(nely),
                          int(nelz), int(nl), float(tol), int(maxit), int(nswp), int(printLev), float(nu), float(hx),
                          float(hy), float(hz), ctypes.byref(rr), ctypes.byref(nit))
    if st == GPUTO_ERR_OOM:
        return 0.0, -1
    if st == GPUTO_ERR_BREAKDOWN:
        return rr.value, -1
    if st != GPUTO_OK:
        raise GputoError(st, "mgcg9")
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

    def energy(self, dsK=None, ce=None, dc=None, stream=None):
        """ce, dc = dsK ce, compliance and the true relative residual of the
        last solve's U, from one fused FP64 apply (gputo_solver_energy_dev).
        Returns (compliance, true_relres); true_relres is -1 when the dense
        fallback ran."""
        c, tr = ctypes.c_double(0.0), ctypes.c_double(0.0)
        _check(_lib.gputo_solver_energy_dev(self._h, _ptr(dsK), _ptr(ce), _ptr(dc), ctypes.byref(c),
                                            ctypes.byref(tr), _ptr_stream(stream)), "gputo_solver_energy_dev")
        return c.value, tr.value

    def vcycle(self, r, z, stream=None):
        _check(_lib.gputo_solver_vcycle_dev(self._h, _ptr(r), _ptr(z), _ptr_stream(stream)),
               "gputo_solver_vcycle_dev")

    def time_kernel(self, which, reps=20, stream=None):
        ms = ctypes.c_double(0.0)
        _check(_lib.gputo_solver_time_kernel(self._h, int(which), int(reps), ctypes.byref(ms),
                                             _ptr_stream(stream)), "gputo_solver_time_kernel")
        return ms.value

    def apply(self, u, r, stream=None):
        _check(_lib.gputo_solver_apply_dev(self._h, _ptr(u), _ptr(r), _ptr_stream(stream)),
               "gputo_solver_apply_dev")

    # learned coarse-grid correction -------------------------------------------------
    def set_options(self, options):
        """Change the options that need no new hierarchy (see gputo_solver_set_options)."""
        _check(_lib.gputo_solver_set_options(self._h, ctypes.byref(options)), "gputo_solver_set_options")
        self.options = options

    def set_net(self, net, mode=1):
        """Attach a Net (mode 1 always, 2 auto with plain-V-cycle fallback) or detach (None)."""
        self._net = net
        _check(_lib.gputo_solver_set_net(self._h, net._h if net is not None else None, int(mode)),
               "gputo_solver_set_net")

    def net_state(self):
        on, a, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(_lib.gputo_solver_net_state(self._h, ctypes.byref(on), ctypes.byref(a), ctypes.byref(b)),
               "gputo_solver_net_state")
        return bool(on.value), a.value, b.value

    def net_dims(self):
        X, Z, Y = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(_lib.gputo_solver_net_dims(self._h, ctypes.byref(X), ctypes.byref(Z), ctypes.byref(Y)),
               "gputo_solver_net_dims")
        return X.value, Z.value, Y.value

    def net_features(self, r, x, m=None, dsq=None, stream=None):
        s = ctypes.c_float()
        _check(_lib.gputo_solver_net_features_dev(self._h, _ptr(r), _ptr(x), _ptr(m), _ptr(dsq), ctypes.byref(s),
                                                  _ptr_stream(stream)), "gputo_solver_net_features_dev")
        return s.value

    def net_energy_rhs(self, w, scale, gt, stream=None):
        _check(_lib.gputo_solver_net_energy_rhs_dev(self._h, _ptr(w), float(scale), _ptr(gt), _ptr_stream(stream)),
               "gputo_solver_net_energy_rhs_dev")

    def net_train_step(self, net, x, gt, nsamples, lr, grads_out=None, stream=None):
        loss = ctypes.c_double()
        gp = grads_out.ctypes.data_as(_fp) if grads_out is not None else None
        _check(_lib.gputo_solver_net_train_step_dev(self._h, net._h, _ptr(x), _ptr(gt), int(nsamples), float(lr),
                                                    ctypes.byref(loss), gp, _ptr_stream(stream)),
               "gputo_solver_net_train_step_dev")
        return loss.value

    def level2_inject(self, v, out, stream=None):
        _check(_lib.gputo_solver_level2_inject_dev(self._h, _ptr(v), _ptr(out), _ptr_stream(stream)),
               "gputo_solver_level2_inject_dev")

    def apply_fp32(self, u, r, tc_parts=0, stream=None):
        """The mixed V-cycle's FP32 fine operator (0: CUDA cores, 1-3: tensor cores)."""
        _check(_lib.gputo_solver_apply_fp32_dev(self._h, _ptr(u), _ptr(r), int(tc_parts), _ptr_stream(stream)),
               "gputo_solver_apply_fp32_dev")


class Homog:
    """Periodic homogenization of a voxel unit cell (gputo_homog_*): the six
    unit-strain load cases as six right-hand sides of one MGCG solve."""

    def __init__(self, nx, ny, nz, nl, options: Options | None = None):
        self._h = ctypes.c_void_p()
        self.shape = (int(nx), int(ny), int(nz))
        self.options = options or default_options(precision=PREC_MIXED)
        _check(_lib.gputo_homog_create(ctypes.byref(self._h), *self.shape, int(nl), ctypes.byref(self.options)),
               "gputo_homog_create")

    def close(self):
        if self._h:
            _lib.gputo_homog_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        return int(_lib.gputo_homog_device_bytes(self._h))

    def solve(self, Ke0, CX, tol=1e-6, maxit=500, chi=None, stream=None):
        """Returns (Ceff [6, 6], relres [6], nit [6]); CX a device tensor of the
        element moduli; chi (optional device tensor of 18 N doubles) receives the
        fluctuations as [3 node + d][r]."""
        Ke0 = np.ascontiguousarray(Ke0, dtype=np.float64).reshape(-1)
        C = np.zeros(36)
        rr = np.zeros(6)
        nit = (ctypes.c_int * 6)()
        _check(_lib.gputo_homog_solve_dev(self._h, _p(Ke0), _ptr(CX), float(tol), int(maxit), _p(C), _p(rr), nit,
                                          _ptr(chi), _ptr_stream(stream)), "gputo_homog_solve_dev")
        return C.reshape(6, 6), rr, np.array(list(nit))


class Batch:
    """Several Solvers solved together, one CUDA graph launch per CG step (gputo_batch_*)."""

    def __init__(self, solvers):
        self.solvers = list(solvers)
        self._h = ctypes.c_void_p()
        arr = (_vp * len(self.solvers))(*[s._h.value for s in self.solvers])
        _check(_lib.gputo_batch_create(ctypes.byref(self._h), arr, len(self.solvers)), "gputo_batch_create")

    def close(self):
        if self._h:
            _lib.gputo_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, Fs, Us, tol, maxit, check_every=8):
        n = len(self.solvers)
        fa = (_vp * n)(*[_ptr(f) for f in Fs])
        ua = (_vp * n)(*[_ptr(u) for u in Us])
        rr = (_d * n)()
        it = (_i * n)()
        _check(_lib.gputo_batch_solve_dev(self._h, fa, ua, float(tol), int(maxit), int(check_every), rr, it),
               "gputo_batch_solve_dev")
        return list(rr), list(it)


def autotune(solver, F, U, tol, maxit):
    """Time complete solves over the tunable options and apply the fastest;
    returns (best Options, best ms, [(ms, nit)] per candidate)."""
    best = Options()
    bms = ctypes.c_double()
    cap = 64
    tms = (_d * cap)()
    tnit = (_i * cap)()
    nc = ctypes.c_int()
    _check(_lib.gputo_autotune_dev(solver._h, _ptr(F), _ptr(U), float(tol), int(maxit), ctypes.byref(best),
                                   ctypes.byref(bms), tms, tnit, cap, ctypes.byref(nc)), "gputo_autotune_dev")
    solver.options = best
    return best, bms.value, [(tms[i], tnit[i]) for i in range(min(nc.value, cap))]


class Net:
    """The learned coarse-grid correction network (gputo_net_*) on the current device."""

    def __init__(self, seed=0):
        self._h = ctypes.c_void_p()
        _check(_lib.gputo_net_create(ctypes.byref(self._h), int(seed)), "gputo_net_create")

    def close(self):
        if self._h:
            _lib.gputo_net_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def num_params() -> int:
        return int(_lib.gputo_net_num_params())

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.num_params(), dtype=np.float32)
        _check(_lib.gputo_net_get_params(self._h, p.ctypes.data_as(_fp)), "gputo_net_get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32).reshape(-1)
        if p.size != self.num_params():
            raise ValueError("wrong parameter count")
        _check(_lib.gputo_net_set_params(self._h, p.ctypes.data_as(_fp)), "gputo_net_set_params")

    def forward(self, x, dims, y, stream=None):
        _check(_lib.gputo_net_forward_dev(self._h, _ptr(x), *dims, _ptr(y), _ptr_stream(stream)),
               "gputo_net_forward_dev")

    def train_step(self, x, t, m, nsamples, dims, lr, grads_out=None, stream=None):
        """Summed loss/gradient over nsamples stacked samples, then one Adam step (lr > 0)."""
        loss = ctypes.c_double()
        gp = grads_out.ctypes.data_as(_fp) if grads_out is not None else None
        _check(_lib.gputo_net_train_step_dev(self._h, _ptr(x), _ptr(t), _ptr(m), int(nsamples), *dims,
                                             float(lr), ctypes.byref(loss), gp, _ptr_stream(stream)),
               "gputo_net_train_step_dev")
        return loss.value


def random_field_density(nelx, nely, nelz, seed=0, corr_len=8.0, lo=1e-3, hi=1.0):
    """Seeded Gaussian random field with correlation length corr_len (elements),
    mapped through a sigmoid to [lo, hi]; element order of the solver."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((nelx, nelz, nely))
    k = [np.fft.fftfreq(n) * 2 * np.pi for n in (nelx, nelz, nely)]
    kk = k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2
    f = np.real(np.fft.ifftn(np.fft.fftn(w) * np.exp(-0.5 * kk * corr_len ** 2)))
    f = (f - f.mean()) / (f.std() + 1e-30)
    x = lo + (hi - lo) / (1.0 + np.exp(-3.0 * f))
    return np.ascontiguousarray(x.reshape(-1))


def harvest_net_samples(solver, F, iters=40):
    """Training samples of the learned correction from one plain PCG solve
    with the solver's own V-cycle (network detached): at iteration k the input
    x_k is built from the residual r_k and the loss data from the residual the
    V-cycle leaves, g_k = D^-1/2 P'P'(r_k - A V(r_k)) / s_k.  F: device float64
    right-hand side (dense layout).  Returns [(x_k, g_k)]."""
    import torch

    X, Z, Y = solver.net_dims()
    n = X * Z * Y
    dev = F.device
    u = torch.zeros_like(F)
    r = F.clone()
    z = torch.empty_like(F)
    q = torch.empty_like(F)
    solver.vcycle(r, z)
    p = z.clone()
    rz = torch.dot(r, z)
    out = []
    for _ in range(iters):
        x = torch.empty(4 * n, dtype=torch.float32, device=dev)
        s = solver.net_features(r, x)
        solver.apply(z, q)
        g = torch.empty(3 * n, dtype=torch.float32, device=dev)
        solver.net_energy_rhs(r - q, s, g)
        out.append((x, g))
        solver.apply(p, q)
        alpha = rz / torch.dot(p, q)
        u += alpha * p
        r -= alpha * q
        if float(torch.linalg.norm(r)) <= 1e-10 * float(torch.linalg.norm(F)):
            break
        solver.vcycle(r, z)
        rz_new = torch.dot(r, z)
        p = z + (rz_new / rz) * p
        rz = rz_new
    return out


def train_net(solver, net, samples, epochs=20, lr=1e-3, batch=8, seed=0):
    """Adam on the energy loss of samples harvested with this solver's current
    hierarchy; returns the mean loss of every epoch (0 = the plain V-cycle)."""
    import torch

    rng = np.random.default_rng(seed)
    X = torch.stack([s[0] for s in samples])
    G = torch.stack([s[1] for s in samples])
    hist = []
    for _ in range(epochs):
        order = rng.permutation(len(samples))
        tot = 0.0
        for b0 in range(0, len(order), batch):
            idx = torch.as_tensor(order[b0:b0 + batch], device=X.device)
            tot += solver.net_train_step(net, X[idx].contiguous(), G[idx].contiguous(), len(idx), lr) * len(idx)
        hist.append(tot / len(samples))
    return hist


def _ptr_stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream  # torch.cuda.Stream


def debug_set_sweep_fault(skip_stage=-1, wait_us=0):
    """Test hook: Hadamard-basis sweeps launched afterwards leave ring stage
    skip_stage unissued and give up each wait after wait_us microseconds
    (gputo_debug_set_sweep_fault); (-1, 0) restores normal operation."""
    _check(_lib.gputo_debug_set_sweep_fault(int(skip_stage), int(wait_us)), "gputo_debug_set_sweep_fault")


def launch_count() -> int:
    return int(_lib.gputo_solver_launch_count(None))


def _host_out(a, n, name):
    """A caller's output array: float64, C-contiguous, writeable, n values."""
    if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous and a.flags.writeable
            and a.size == n):
        raise ValueError(f"{name} must be a writeable C-contiguous float64 array of {n} values")
    return a


def compliance_sens(Ke0, U, CX, dsK, nelx, nely, nelz, out=None):
    """Host-buffer form (U in the MATLAB frame): returns (ce, dc, compliance).
    out: optional (ce, dc) arrays to write into (a loop that keeps them skips
    the first-touch cost of fresh output pages)."""
    Ke0 = np.ascontiguousarray(Ke0, dtype=np.float64).reshape(-1)
    U = np.ascontiguousarray(U, dtype=np.float64)
    CX = np.ascontiguousarray(CX, dtype=np.float64)
    dsK = np.ascontiguousarray(dsK, dtype=np.float64)
    ne = nelx * nely * nelz
    if out is None:
        ce, dc = np.zeros(ne), np.zeros(ne)
    else:
        ce, dc = _host_out(out[0], ne, "ce"), _host_out(out[1], ne, "dc")
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


def compliance_sens_tc_dev(Ke0, U, CX, dsK, nelx, nely, nelz, ce=None, dc=None, stream=None):
    """Tensor-core form of compliance_sens_dev (U in the solver frame)."""
    Ke0 = np.ascontiguousarray(Ke0, dtype=np.float64).reshape(-1)
    c = ctypes.c_double(0.0)
    _check(_lib.gputo_compliance_sens_tc_dev(_p(Ke0), _ptr(U), _ptr(CX), _ptr(dsK), nelx, nely, nelz,
                                             _ptr(ce), _ptr(dc), ctypes.byref(c), _ptr_stream(stream)),
           "gputo_compliance_sens_tc_dev")
    return c.value


def density_filter(x, nelx, nely, nelz, rmin, divisor=None, normalize=True, out=None):
    """Host-buffer form of the driver's imfilter calls (out: optional array
    to write into; it may be x, which is copied to the device first)."""
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    out = np.zeros_like(x) if out is None else _host_out(out, x.size, "out")
    dv = None if divisor is None else np.ascontiguousarray(divisor, dtype=np.float64).reshape(-1)
    _check(_lib.gputo_density_filter(_p(x), None if dv is None else _p(dv), _p(out), nelx, nely,
                                     nelz, float(rmin), int(bool(normalize))), "gputo_density_filter")
    return out


def time_filter_dev(inputs, outputs, nelx, nely, nelz, rmin, reps=20, stream=None):
    """Profiling aid: mean ms of one normalised filter launch, launches back to
    back cycling through the (input, output) device-array pairs."""
    n = len(inputs)
    ins = (ctypes.c_void_p * n)(*[_ptr(x) for x in inputs])
    outs = (ctypes.c_void_p * n)(*[_ptr(x) for x in outputs])
    ms = ctypes.c_double(0.0)
    _check(_lib.gputo_time_filter_dev(ins, outs, n, nelx, nely, nelz, float(rmin), int(reps), ctypes.byref(ms),
                                      _ptr_stream(stream)), "gputo_time_filter_dev")
    return ms.value


def density_filter_dev(x, out, nelx, nely, nelz, rmin, divisor=None, normalize=True, stream=None):
    _check(_lib.gputo_density_filter_dev(_ptr(x), _ptr(divisor), _ptr(out), nelx, nely, nelz,
                                         float(rmin), int(bool(normalize)), _ptr_stream(stream)),
           "gputo_density_filter_dev")


def simp_dev(xphys, CX, dsK=None, penal=3.0, E0=1.0, Emin=1e-9, stream=None):
    _check(_lib.gputo_simp_dev(_ptr(xphys), xphys.numel(), float(penal), float(E0), float(Emin),
                               _ptr(CX), _ptr(dsK), _ptr_stream(stream)), "gputo_simp_dev")


def simp(xphys, penal=3.0, E0=1.0, Emin=1e-9, out=None):
    """Host-array SIMP (top3D125modCuda.m:124,130): returns (CX, dsK)
    (out: optional (CX, dsK) arrays to write into)."""
    xphys = np.ascontiguousarray(xphys, dtype=np.float64).reshape(-1)
    if out is None:
        CX, dsK = np.empty_like(xphys), np.empty_like(xphys)
    else:
        CX, dsK = _host_out(out[0], xphys.size, "CX"), _host_out(out[1], xphys.size, "dsK")
    _check(_lib.gputo_simp(_p(xphys), xphys.size, float(penal), float(E0), float(Emin), _p(CX), _p(dsK)),
           "gputo_simp")
    return CX, dsK


def oc_update_dev(x, dc, dv0, xnew, volfrac, move, stream=None):
    lm = ctypes.c_double(0.0)
    _check(_lib.gputo_oc_update_dev(_ptr(x), _ptr(dc), _ptr(dv0), x.numel(), float(volfrac),
                                    float(move), _ptr(xnew), ctypes.byref(lm), _ptr_stream(stream)),
           "gputo_oc_update_dev")
    return lm.value


def oc_update(x, dc, dv0, volfrac, move, out=None):
    """Host-buffer form: returns (xnew, lmid) (out: optional array for xnew)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    dc = np.ascontiguousarray(dc, dtype=np.float64)
    dv0 = np.ascontiguousarray(dv0, dtype=np.float64)
    xn = np.zeros_like(x) if out is None else _host_out(out, x.size, "out")
    lm = ctypes.c_double(0.0)
    _check(_lib.gputo_oc_update(_p(x), _p(dc), _p(dv0), x.size, float(volfrac), float(move),
                                _p(xn), ctypes.byref(lm)), "gputo_oc_update")
    return xn, lm.value


def design_save(path, shape, iteration, params, x, xPhys):
    """Write a design-state file (host arrays in element order)."""
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    xPhys = np.ascontiguousarray(xPhys, dtype=np.float64).reshape(-1)
    params = np.ascontiguousarray(params, dtype=np.float64).reshape(-1)
    _check(_lib.gputo_design_save(os.fsencode(path), *shape, int(iteration), _p(params) if params.size else None,
                                  params.size, _p(x), _p(xPhys)), "gputo_design_save")


def design_load(path):
    """Read a design-state file: (shape, iteration, params, x, xPhys)."""
    nx, ny, nz, it, npar = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int(0)
    _check(_lib.gputo_design_load(os.fsencode(path), ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(nz),
                                  ctypes.byref(it), None, ctypes.byref(npar), None, None), "gputo_design_load")
    nel = nx.value * ny.value * nz.value
    params = np.zeros(max(npar.value, 1))
    x, xp = np.zeros(nel), np.zeros(nel)
    cap = ctypes.c_int(params.size)
    _check(_lib.gputo_design_load(os.fsencode(path), ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(nz),
                                  ctypes.byref(it), _p(params), ctypes.byref(cap), _p(x), _p(xp)),
           "gputo_design_load")
    return (nx.value, ny.value, nz.value), it.value, params[:cap.value], x, xp


def design_export_volume(base, shape, xPhys):
    xPhys = np.ascontiguousarray(xPhys, dtype=np.float64).reshape(-1)
    _check(_lib.gputo_design_export_volume(os.fsencode(base), *shape, _p(xPhys)), "gputo_design_export_volume")


def heaviside_dev(xTilde, xPhys, volfrac, beta, eta, dprj=None, stream=None):
    """Volume-preserving Heaviside projection on device tensors; returns the final eta."""
    e = ctypes.c_double(float(eta))
    _check(_lib.gputo_heaviside_dev(_ptr(xTilde), xTilde.numel(), float(volfrac), float(beta), ctypes.byref(e),
                                    _ptr(xPhys), _ptr(dprj), _ptr_stream(stream)), "gputo_heaviside_dev")
    return e.value


def mul_dev(a, b, out, stream=None):
    _check(_lib.gputo_mul_dev(_ptr(a), _ptr(b), _ptr(out), a.numel(), _ptr_stream(stream)), "gputo_mul_dev")


class DesignLoop:
    """The top3D125 optimisation loop with every field resident on the GPU
    (Cantilever/TOP3D125MGCGCUDA/top3D125modCuda.m:105-166; ft=1 density filter,
    ft=3 density filter plus volume-preserving Heaviside projection):

        xPhys = imfilter(x, h, 'symmetric') ./ Hs          density filter
        CX, dsK = SIMP(xPhys)                               stiffness
        [cgres, cgiters] = mgcg1(...)                       MGCG solve
        dc = dsK .* ce;  c = sum(CX .* ce)                  sensitivity, compliance (one
                                                            FP64 apply of U, which also
                                                            gives the true residual)
        dc = imfilter(dc ./ Hs); dV0 = imfilter(dV ./ Hs)   filtered sensitivities
        x = OC(x, dc, dV0)                                  bisection update

    Every step is a C-ABI call on device buffers; the host sees only scalars.
    Under 'symmetric' padding Hs is the constant sum(h), so dividing by it
    before or after the filter is the same; the normalised filter is used.
    ``torch`` tensors provide the device memory.
    """

    def __init__(self, nelx, nely, nelz, nl, F, fixed, Ke0, volfrac=0.12, penal=3.0,
                 rmin=3 ** 0.5, move=0.2, tol=1e-6, maxit=200, E0=1.0, Emin=1e-9,
                 options: Options | None = None, x0=None, stream=None, ft=1, eta=0.4, beta=2.0):
        import torch
        self.torch = torch
        self.shape = (nelx, nely, nelz)
        self.nel = nelx * nely * nelz
        self.ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
        self.volfrac, self.penal, self.rmin, self.move = volfrac, penal, rmin, move
        self.tol, self.maxit, self.E0, self.Emin = tol, maxit, E0, Emin
        self.Ke0 = np.ascontiguousarray(Ke0, dtype=np.float64).reshape(-1)
        self.stream = stream
        dev = torch.device("cuda")
        f64 = dict(dtype=torch.float64, device=dev)
        self.F = torch.as_tensor(np.ascontiguousarray(F, dtype=np.float64), **f64)
        self.x = torch.full((self.nel,), float(volfrac), **f64) if x0 is None else \
            torch.as_tensor(np.ascontiguousarray(x0, dtype=np.float64), **f64).clone()
        self.xnew = torch.empty_like(self.x)
        self.xPhys = torch.empty_like(self.x)
        self.CX = torch.empty_like(self.x)
        self.dsK = torch.empty_like(self.x)
        self.ce = torch.empty_like(self.x)
        self.dc = torch.empty_like(self.x)
        self.dcf = torch.empty_like(self.x)
        self.dV = torch.full((self.nel,), 1.0 / self.nel / volfrac, **f64)
        self.dV0 = torch.empty_like(self.x)
        self.U = torch.zeros(self.ndof, **f64)
        if ft not in (1, 3):
            raise ValueError("ft must be 1 (density filter) or 3 (plus Heaviside projection)")
        self.ft, self.eta, self.beta = ft, eta, beta
        if ft == 3:
            self.xTilde = torch.empty_like(self.x)
            self.dprj = torch.empty_like(self.x)
            self.dVp = torch.empty_like(self.x)
        self.solver = Solver(nelx, nely, nelz, nl, options)
        self.solver.set_problem(self.Ke0, fixed)

    def save(self, path, iteration):
        """Design state (x, xPhys and the loop parameters) for a later resume."""
        params = [self.volfrac, self.penal, self.rmin, self.move, float(self.ft), self.eta, self.beta]
        design_save(path, self.shape, iteration, params, self.x.cpu().numpy(), self.xPhys.cpu().numpy())

    def resume(self, path):
        """Continue from a saved design state (the drivers' warm start); returns its iteration."""
        shape, it, params, x, xp = design_load(path)
        if tuple(shape) != tuple(self.shape):
            raise ValueError(f"saved design is {shape}, this loop is {self.shape}")
        if len(params) < 7 or int(params[4]) != self.ft:
            raise ValueError("saved design was not written by a loop with this filter type")
        self.volfrac, self.penal, self.rmin, self.move = (float(v) for v in params[:4])
        self.eta, self.beta = float(params[5]), float(params[6])
        self.dV.fill_(1.0 / self.nel / self.volfrac)
        self.x.copy_(self.torch.as_tensor(x, device=self.x.device))
        self.xPhys.copy_(self.torch.as_tensor(xp, device=self.x.device))
        return it

    def step(self):
        nelx, nely, nelz = self.shape
        s = self.stream
        if self.ft == 3:
            # xTilde = filtered x; eta keeps the volume; xPhys = prj(xTilde) (top3D125modCuda.m:109-119)
            density_filter_dev(self.x, self.xTilde, nelx, nely, nelz, self.rmin, stream=s)
            self.eta = heaviside_dev(self.xTilde, self.xPhys, self.volfrac, self.beta, self.eta, self.dprj,
                                     stream=s)
        else:
            density_filter_dev(self.x, self.xPhys, nelx, nely, nelz, self.rmin, stream=s)
        simp_dev(self.xPhys, self.CX, self.dsK, self.penal, self.E0, self.Emin, stream=s)
        self.solver.setup(self.CX, stream=s)
        relres, nit = self.solver.solve(self.F, self.U, self.tol, self.maxit, stream=s)
        # ce, dc and the compliance from the FP64 apply of U that also gives
        # the true residual of the solve (gputo_solver_energy_dev)
        c, true_relres = self.solver.energy(self.dsK, self.ce, self.dc, stream=s)
        if self.ft == 3:
            # dc ./ dHs with dHs = Hs ./ dprj: filter(dc .* dprj) / Hs (top3D125modCuda.m:117,140-141)
            mul_dev(self.dc, self.dprj, self.dc, stream=s)
            mul_dev(self.dV, self.dprj, self.dVp, stream=s)
            density_filter_dev(self.dc, self.dcf, nelx, nely, nelz, self.rmin, stream=s)
            density_filter_dev(self.dVp, self.dV0, nelx, nely, nelz, self.rmin, stream=s)
        else:
            density_filter_dev(self.dc, self.dcf, nelx, nely, nelz, self.rmin, stream=s)
            density_filter_dev(self.dV, self.dV0, nelx, nely, nelz, self.rmin, stream=s)
        lmid = oc_update_dev(self.x, self.dcf, self.dV0, self.xnew, self.volfrac, self.move,
                             stream=s)
        self.x, self.xnew = self.xnew, self.x
        return {"c": c, "nit": nit, "relres": relres, "true_relres": true_relres, "lmid": lmid}
