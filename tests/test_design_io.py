"""Design-state files: save / load round trips and error handling (host only,
no GPU).  They stand in for the drivers' MATLAB warm start
(CrossWalk/crosswalk.m:135) and isosurface output."""
import os
import struct

import numpy as np
import pytest

import gputo


def _state(shape, seed=0):
    rng = np.random.default_rng(seed)
    nel = int(np.prod(shape))
    return rng.random(nel), rng.random(nel)


def test_round_trip(tmp_path):
    shape = (6, 3, 4)
    x, xp = _state(shape)
    params = np.array([0.12, 3.0, 3 ** 0.5, 0.2, 3.0, 0.41, 4.0])
    p = tmp_path / "d.gds"
    gputo.design_save(p, shape, 46, params, x, xp)
    assert os.path.getsize(p) == 64 + 8 * (params.size + 2 * x.size)
    shape2, it, params2, x2, xp2 = gputo.design_load(p)
    assert shape2 == shape and it == 46
    np.testing.assert_array_equal(params2, params)
    np.testing.assert_array_equal(x2, x)
    np.testing.assert_array_equal(xp2, xp)


def test_header_layout(tmp_path):
    shape = (2, 1, 1)
    p = tmp_path / "h.gds"
    gputo.design_save(p, shape, 7, [0.5], [0.1, 0.2], [0.3, 0.4])
    raw = open(p, "rb").read()
    assert raw[:8] == b"GPUTODS1"
    version, nx, ny, nz, it, npar, narr = struct.unpack_from("<Iiiiiii", raw, 8)
    assert (version, nx, ny, nz, it, npar, narr) == (1, 2, 1, 1, 7, 1, 2)
    vals = struct.unpack_from("<5d", raw, 64)
    assert vals == (0.5, 0.1, 0.2, 0.3, 0.4)


def test_no_params(tmp_path):
    shape = (2, 2, 2)
    x, xp = _state(shape, 1)
    p = tmp_path / "n.gds"
    gputo.design_save(p, shape, 0, [], x, xp)
    _, _, params, x2, xp2 = gputo.design_load(p)
    assert params.size == 0
    np.testing.assert_array_equal(x2, x)
    np.testing.assert_array_equal(xp2, xp)


@pytest.mark.parametrize("cut", [0, 10, 64, 64 + 8, -8])
def test_truncated_rejected(tmp_path, cut):
    shape = (3, 2, 2)
    x, xp = _state(shape, 2)
    p = tmp_path / "t.gds"
    gputo.design_save(p, shape, 1, [1.0], x, xp)
    raw = open(p, "rb").read()
    open(p, "wb").write(raw[:cut] if cut >= 0 else raw[:len(raw) + cut])
    with pytest.raises(gputo.GputoError):
        gputo.design_load(p)


def test_foreign_and_missing_rejected(tmp_path):
    p = tmp_path / "f.gds"
    open(p, "wb").write(b"NOTADESIGNFILE" + bytes(100))
    with pytest.raises(gputo.GputoError, match="not a design-state file"):
        gputo.design_load(p)
    with pytest.raises(gputo.GputoError, match="cannot open"):
        gputo.design_load(tmp_path / "missing.gds")


def test_params_capacity(tmp_path):
    """A params buffer smaller than the saved count is an error, not an overrun."""
    import ctypes
    p = tmp_path / "c.gds"
    gputo.design_save(p, (1, 1, 1), 0, [1.0, 2.0, 3.0], [0.5], [0.5])
    lib = gputo._lib
    nx, ny, nz, it = (ctypes.c_int() for _ in range(4))
    cap = ctypes.c_int(2)
    buf = (ctypes.c_double * 2)()
    x, xp = ctypes.c_double(), ctypes.c_double()
    r = lib.gputo_design_load(os.fsencode(p), ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(nz),
                              ctypes.byref(it), buf, ctypes.byref(cap), ctypes.byref(x), ctypes.byref(xp))
    assert r != 0 and cap.value == 3


def test_export_volume(tmp_path):
    shape = (4, 3, 2)
    _, xp = _state(shape, 3)
    base = tmp_path / "vol"
    gputo.design_export_volume(base, shape, xp)
    hdr = open(str(base) + ".nhdr").read()
    assert hdr.startswith("NRRD0004\n")
    assert "sizes: 3 2 4\n" in hdr and "type: float\n" in hdr and "data file: vol.raw\n" in hdr
    v = np.fromfile(str(base) + ".raw", dtype="<f4")
    np.testing.assert_array_equal(v, xp.astype(np.float32))
    # element order e = nelz*nely*i + nely*k + j: y fastest, then z, then x
    vol = v.reshape(shape[0], shape[2], shape[1])
    i, k, j = 3, 1, 2
    assert vol[i, k, j] == np.float32(xp[shape[2] * shape[1] * i + shape[1] * k + j])


def test_bad_arguments(tmp_path):
    with pytest.raises(gputo.GputoError):
        gputo.design_save(tmp_path / "b.gds", (0, 1, 1), 0, [], [], [])
