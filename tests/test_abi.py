"""The C-ABI library loads and exports every entry point of
include/fdtd_b200.h; argument validation works without a GPU."""
import ctypes
import os
import re

import pytest

from fdtdsarsim_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, 'include', 'fdtd_b200.h')).read()
    src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
    return sorted(set(re.findall(r'\bint\s+(fdtd_\w+)\s*\(', src)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert 'fdtd_create' in names and 'fdtd_run' in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_native.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert set(declared_functions()) <= set(_native.SIGNATURES)


def test_version_and_error_buffer():
    assert _native.lib.fdtd_version() >= 100
    buf = ctypes.create_string_buffer(8)
    _native.lib.fdtd_last_error(buf, len(buf))


def test_invalid_geometry_rejected_before_device_use():
    g = _native.Geometry(nx=5, ny=5, nz=5, npml=10, tfsf_z=2, nt=10, nt_inc=5, dtype=0,
                         cell_size=1e-3, timestep=1e-12, frequency=5.4e9, db=1.0, dtm0=1.0,
                         dte0dx=1.0)
    with pytest.raises(_native.FdtdError) as ei:
        _native.NativeSim(g, 0)
    assert ei.value.code == _native.FDTD_ERR_INVALID
    assert 'too small' in str(ei.value)
    g.nx = g.ny = g.nz = 30
    g.dtype = 7
    with pytest.raises(_native.FdtdError) as ei:
        _native.NativeSim(g, 0)
    assert ei.value.code == _native.FDTD_ERR_INVALID


def test_null_handle_is_an_error():
    rc = _native.lib.fdtd_run(None, 1)
    assert rc == _native.FDTD_ERR_INVALID
    assert 'null' in _native.last_error()


def test_near2far_rejects_even_planes():
    import numpy as np
    z = np.zeros((4, 4), np.complex64)
    with pytest.raises(_native.FdtdError) as ei:
        _native.near2far(z, z, z, z, 4, 4, 5, 0.01, 2000.0, [0.0], [0.0], 5.4e9)
    assert ei.value.code == _native.FDTD_ERR_INVALID
