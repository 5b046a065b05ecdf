"""HDF5 interoperability where h5py is installed (the GPU box runs this with
the GPU tests): files written by h5lite, the writer the package uses where
h5py is absent, must open with h5py and hold the same datasets and
attributes. Where h5py is absent the test is skipped and says so."""
import numpy as np
import pytest

from fdtdsarsim_b200 import h5lite, resultsio

pytestmark = pytest.mark.gpu


def test_h5lite_files_open_with_h5py(tmp_path):
    print('resultsio backend:', resultsio.BACKEND)
    h5py = pytest.importorskip('h5py', reason='h5py is not installed on this machine')
    rng = np.random.default_rng(5)
    planes = {f'ex_ph_{s}': (rng.standard_normal((9, 11)) + 1j * rng.standard_normal((9, 11))).astype(np.complex64)
              for s in ('d', 'u')}
    inc = rng.standard_normal((4, 9, 11)).astype(np.float32)
    path = tmp_path / 'result.hdf5'
    with h5lite.File(str(path), 'w') as f:
        g = f.create_group('phasors')
        for k, v in planes.items():
            g.create_dataset(k, data=v)
        f.create_dataset('ex', data=inc)
        p = f.create_group('parameters')
        p.attrs['nx_phasor'] = 11
        p.attrs['frequency'] = 5.4e9
        p.attrs['datatype'] = 'float32'
        p.attrs['use_hh'] = True
    with h5py.File(str(path), 'r') as f:
        for k, v in planes.items():
            got = f['phasors'][k][()]
            assert got.dtype == v.dtype and np.array_equal(got, v), k
        assert np.array_equal(f['ex'][()], inc)
        a = f['parameters'].attrs
        assert int(a['nx_phasor']) == 11 and float(a['frequency']) == 5.4e9
        assert str(a['datatype']) == 'float32' and bool(a['use_hh'])
