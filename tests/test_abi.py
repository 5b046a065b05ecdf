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


def test_binding_constants_match_the_header():
    """Every integer #define of the header that the ctypes binding mirrors
    (FDTD_X as FDTD_X or X) has the header's value; every option is bound."""
    src = open(os.path.join(ROOT, 'include', 'fdtd_b200.h')).read()
    defines = dict((k, int(v)) for k, v in
                   re.findall(r'^#define\s+(FDTD_\w+)\s+(-?\d+)\b', src, flags=re.M))
    checked = 0
    for name, value in defines.items():
        short = name[len('FDTD_'):]
        for attr in (name, short):
            if hasattr(_native, attr):
                assert getattr(_native, attr) == value, (name, attr)
                checked += 1
                break
        else:
            if short.startswith('OPT_'):
                raise AssertionError(f'{name} has no binding constant')
            if short.startswith('POL_'):
                assert _native.POLARIZATIONS[short[4:]] == value, name
                checked += 1
    assert checked >= 20 and defines['FDTD_OPT_BATCH_STREAMS'] == _native.OPT_BATCH_STREAMS


def test_every_entry_point_rejects_null_handles():
    """No entry point dereferences a NULL handle or output pointer: each
    returns FDTD_ERR_INVALID with a message (the destroy calls accept NULL
    and return FDTD_OK), before any device is touched."""
    no_handle = {'fdtd_last_error', 'fdtd_version', 'fdtd_device_count', 'fdtd_fused_plan_boxes',
                 'fdtd_bounds_check_enabled',
                 'fdtd_check_cell_division'}
    for name, argtypes in _native.SIGNATURES.items():
        if name in no_handle:
            continue
        args = [0 if t is _native._I else 0.0 if t is _native._D else None for t in argtypes]
        rc = getattr(_native.lib, name)(*args)
        if name.endswith('_destroy'):
            assert rc == _native.FDTD_OK, name
        else:
            assert rc == _native.FDTD_ERR_INVALID, name
            assert 'null' in _native.last_error(), name


def test_device_name_or_a_clean_error():
    """fdtd_device_name: the autotuner's cache key; without a device an
    FDTD_ERR_CUDA, and the autotuner falls back to a placeholder key."""
    from fdtdsarsim_b200 import tuning
    if _native.device_count() == 0:
        with pytest.raises(_native.FdtdError) as ei:
            _native.device_name(0)
        assert ei.value.code == _native.FDTD_ERR_CUDA
        assert tuning._device_name(0) == 'device0'
    else:
        assert _native.device_name(0) and tuning._device_name(0) == _native.device_name(0)
    with pytest.raises(_native.FdtdError) as ei:
        _native.device_name(-1 if _native.device_count() else 0)
    assert ei.value.code in (_native.FDTD_ERR_INVALID, _native.FDTD_ERR_CUDA)


def test_the_package_imports_without_torch():
    """PyTorch belongs to the autograd wrapper only: importing the package
    and its simulation, sweep, tuning and file modules loads no torch."""
    import subprocess
    import sys
    code = ('import sys; sys.path.insert(0, sys.argv[1]); import fdtdsarsim_b200, '
            'fdtdsarsim_b200.sweep, fdtdsarsim_b200.tuning, fdtdsarsim_b200.gpu.main_sim, '
            'fdtdsarsim_b200.incident, fdtdsarsim_b200.h5lite; '
            'print("torch" in sys.modules)')
    out = subprocess.run([sys.executable, '-c', code, os.path.join(ROOT, 'sar-pixel-simulator_b200')],
                         capture_output=True, text=True, check=True, timeout=300)
    assert out.stdout.strip() == 'False'
