"""The allocation-free compliance entry point, through the C ABI.

gputo_compliance_sens_noalloc_dev serves callers that cannot let a library
call cudaMalloc: a host whose memory manager owns the device's free memory (a
MATLAB gpuArray workspace, a caching allocator), or a real-time loop that must
not hit cudaMalloc's implicit device synchronisation.  Its scratch is a fixed
device array in the library instead of memory it allocates.  This test checks
that it returns what the allocating entry point (gputo_compliance_sens_dev)
returns, on two calls in a row (the second call reuses the scratch the first
one left), and that repeated calls take no device memory.  The file is named
to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the tolerance the other FP64 parity tests use


def _call(lib, fn, Ke0, U, CX, dsK, shape, ce, dc):
    c = ctypes.c_double(0.0)
    Kp = Ke0.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    st = getattr(lib, fn)(Kp, U.data_ptr(), CX.data_ptr(), dsK.data_ptr(), *shape, ce.data_ptr(),
                          dc.data_ptr(), ctypes.byref(c), None)
    assert st == 0, (fn, st, lib.gputo_last_error())
    return c.value


def test_noalloc_compliance_matches_allocating_entry_point(gputo):
    import torch
    assert torch.cuda.is_available(), "GPU test"
    lib = gputo.lib()
    shape = (48, 24, 20)   # 23,040 elements: 12 CTAs of partial sums
    nel = shape[0] * shape[1] * shape[2]
    ndof = 3 * (shape[0] + 1) * (shape[1] + 1) * (shape[2] + 1)
    Ke0 = np.ascontiguousarray(gputo.hex8_stiffness().reshape(-1))
    rng = np.random.default_rng(2024)
    dev = dict(dtype=torch.float64, device="cuda")
    results = []
    for trial in range(2):   # two calls in a row, different inputs
        U = torch.as_tensor(rng.standard_normal(ndof), **dev)
        x = torch.as_tensor(rng.uniform(0.05, 1.0, nel), **dev)
        CX = 1e-9 + x ** 3 * (1 - 1e-9)
        dsK = -3 * (1 - 1e-9) * x ** 2
        ce_ref, dc_ref = torch.empty(nel, **dev), torch.empty(nel, **dev)
        c_ref = _call(lib, "gputo_compliance_sens_dev", Ke0, U, CX, dsK, shape, ce_ref, dc_ref)
        ce, dc = torch.full((nel,), np.nan, **dev), torch.full((nel,), np.nan, **dev)
        torch.cuda.synchronize()
        c = _call(lib, "gputo_compliance_sens_noalloc_dev", Ke0, U, CX, dsK, shape, ce, dc)
        if trial == 1:
            # free device memory moves in pages of about 2 MiB; 100 more calls
            # would take 6.25 MiB if each call allocated its 64 KB and kept it
            free_before = torch.cuda.mem_get_info()[0]
            for _ in range(100):
                c_rep = _call(lib, "gputo_compliance_sens_noalloc_dev", Ke0, U, CX, dsK, shape, ce, dc)
                assert c_rep == c
            free_after = torch.cuda.mem_get_info()[0]
            assert free_before - free_after < (4 << 20), "repeated calls took device memory"
        assert torch.allclose(ce, ce_ref, rtol=RTOL, atol=0)
        assert torch.allclose(dc, dc_ref, rtol=RTOL, atol=0)
        assert abs(c - c_ref) <= RTOL * abs(c_ref)
        results.append(c)
    assert results[0] != results[1]   # the second call did not reuse stale output


def test_noalloc_rejects_grids_above_its_scratch(gputo):
    lib = gputo.lib()
    Ke0 = np.ascontiguousarray(gputo.hex8_stiffness().reshape(-1))
    c = ctypes.c_double(0.0)
    # 512 x 256 x 256 = 33.5M elements > 16,777,216: rejected before any launch
    st = lib.gputo_compliance_sens_noalloc_dev(Ke0.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                               1, 1, 1, 512, 256, 256, 1, 1, ctypes.byref(c), None)
    assert st == gputo.GPUTO_ERR_ARG
    assert b"16,777,216" in lib.gputo_last_error()
