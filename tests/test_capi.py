"""The C ABI library and the MEX gateway, on the host (no GPU needed).

Checks that libgputo.so loads, exports every function include/gputo.h
declares, and that calls fail with a status (never a crash or exit) when no
sm_100 device is present.
"""
import ctypes
import os
import re

import numpy as np
import pytest
from conftest import ROOT


def header_functions():
    src = open(os.path.join(ROOT, "include", "gputo.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(gputo_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_drop_in_entry_points():
    names = header_functions()
    for n in ("gputo_mgcg1", "gputo_compliance_sens", "gputo_density_filter",
              "gputo_status_string", "gputo_solver_create", "gputo_solver_solve_dev"):
        assert n in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol(gputo):
    lib = ctypes.CDLL(gputo.LIB_PATH)
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding knows every one of them
    assert set(header_functions()) <= set(gputo.SIGNATURES)


def test_status_strings_and_version(gputo):
    L = gputo.lib()
    assert L.gputo_status_string(0) == b"ok"
    assert b"memory" in L.gputo_status_string(gputo.GPUTO_ERR_OOM)
    assert L.gputo_status_string(99) == b"unknown status"
    assert b"sm_100a" in L.gputo_version()


def test_default_options_are_the_mex_constants(gputo):
    o = gputo.default_options()
    assert (o.nswp, o.omega, o.prerelax, o.nu) == (3, 0.48, 0.7, 0.3)
    assert o.precision == gputo.PREC_FP64


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_have_gpu(), reason="host-only behaviour")
def test_no_device_returns_status_not_crash(gputo):
    import oracle as O
    p = O.cantilever(4, 2, 2)
    U = np.zeros(p.ndof)
    rr = ctypes.c_double(0)
    nit = ctypes.c_int(0)
    L = gputo.lib()
    st = L.gputo_mgcg1(gputo._p(p.Ke0.reshape(-1).copy()), gputo._p(p.F), gputo._p(U),
                       gputo._p(np.ones(p.nel)), gputo._p(p.fixed), len(p.fixed), 4, 2, 2, 2, 1e-8,
                       10, 0, ctypes.byref(rr), ctypes.byref(nit))
    assert st == gputo.GPUTO_ERR_NO_DEVICE
    assert nit.value == -1
    h = ctypes.c_void_p()
    assert L.gputo_solver_create(ctypes.byref(h), 4, 2, 2, 2, None) == gputo.GPUTO_ERR_NO_DEVICE
    with pytest.raises(gputo.GputoError):
        gputo.density_filter(np.ones(8), 2, 2, 2, 1.5)


def _load_mex(name="libgputo_mex.so"):
    """Load the gateway the way MATLAB would: its mx* symbols resolve from a
    globally loaded libmx -- here the project's stand-in, built on the fly."""
    shim = os.path.join(ROOT, "oracle", "shim")
    so = os.path.join(ROOT, "oracle", "_build_shim", "libmexshim.so")
    os.makedirs(os.path.dirname(so), exist_ok=True)
    if not os.path.exists(so):
        import subprocess
        subprocess.run(["gcc", "-O2", "-fPIC", "-shared", f"-I{shim}", os.path.join(shim, "mex_shim.c"),
                        "-o", so], check=True)
    ctypes.CDLL(so, mode=ctypes.RTLD_GLOBAL)
    return ctypes.CDLL(os.path.join(ROOT, "gpu-to_b200", "lib", name)), ctypes.CDLL(so)


class MxArray(ctypes.Structure):
    _fields_ = [("data", ctypes.POINTER(ctypes.c_double)), ("m", ctypes.c_size_t),
                ("n", ctypes.c_size_t), ("owned", ctypes.c_int), ("scalar", ctypes.c_double)]


def call_mex(mex, args):
    """mexFunction(nlhs, plhs, nrhs, prhs) with numpy arrays / scalars."""
    keep = []
    arr = (MxArray * len(args))()
    for i, a in enumerate(args):
        a = np.ascontiguousarray(np.atleast_1d(np.asarray(a, dtype=np.float64))) if not (
            isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous) else a
        keep.append(a)
        arr[i].data = a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        arr[i].m, arr[i].n, arr[i].owned = a.size, 1, 0
    prhs = (ctypes.POINTER(MxArray) * len(args))(*[ctypes.pointer(arr[i]) for i in range(len(args))])
    plhs = (ctypes.POINTER(MxArray) * 2)()
    mex.mexFunction(2, plhs, len(args), prhs)
    return plhs[0].contents.scalar, plhs[1].contents.scalar


def test_mex_gateway_exports_mexfunction_and_rejects_bad_calls(gputo):
    mex, _ = _load_mex()
    assert hasattr(mex, "mexFunction")
    # too few arguments: cgiters = -1, no crash
    res, it = call_mex(mex, [np.zeros(576)] * 5)
    assert it == -1.0
    # mismatched sizes: rejected before any buffer is touched
    res, it = call_mex(mex, [np.zeros(576), np.zeros(10), np.zeros(10), np.zeros(3), np.ones(1),
                             1, 2, 2, 2, 2, 1e-8, 10])
    assert it == -1.0


def test_mgcg9_gateway_exports_mexfunction_and_rejects_bad_calls(gputo):
    mex, _ = _load_mex("libgputo_mex9.so")
    assert hasattr(mex, "mexFunction")
    res, it = call_mex(mex, [np.zeros(576)] * 12)      # mgcg9 needs 18 arguments
    assert it == -1.0
    res, it = call_mex(mex, [np.zeros(576), np.zeros(10), np.zeros(10), np.zeros(3), np.ones(1),
                             1, 2, 2, 2, 2, 1e-8, 10, 2, 0, 0.3, 1.0, 1.0, 1.0])
    assert it == -1.0


def test_host_output_arrays_are_checked_before_any_device_work(gputo):
    """out= of the host-array calls must be writeable C-contiguous float64
    arrays of the element count; anything else is a ValueError, raised before
    the library is called."""
    x = np.full(64, 0.5)
    for bad in (np.zeros(63), np.zeros(64, dtype=np.float32), np.zeros((64, 2))[:, 0]):
        with pytest.raises(ValueError):
            gputo.density_filter(x, 4, 4, 4, 1.5, out=bad)
        with pytest.raises(ValueError):
            gputo.oc_update(x, -x, x, 0.3, 0.2, out=bad)
        with pytest.raises(ValueError):
            gputo.simp(x, out=(bad, np.zeros(64)))
    ro = np.zeros(64)
    ro.flags.writeable = False
    with pytest.raises(ValueError):
        gputo.density_filter(x, 4, 4, 4, 1.5, out=ro)
