"""Stand-ins that let the reference package ``fdtdsarsim`` import and run in a
container without ``h5py`` and ``matplotlib``.

Used only by ``make_golden.py`` (fixture generation). ``h5py`` is replaced by
an in-memory store that keeps every "file" as a dict of numpy arrays plus
attribute dicts; a zero-byte placeholder is written on disk so that the
reference's ``os.path.exists`` checks (``cpu/main_sim.py:66-79``,
``incidentbeam.py:167-172``) behave as they would with real files.
``matplotlib`` is replaced by no-op modules (the reference only plots when a
``disp_*`` flag is set, and every fixture run leaves them off).
"""
import os
import sys
import types

import numpy as np

_STORE = {}


class _Attrs(dict):
    pass


class _Dataset:
    def __init__(self, data):
        self._data = data
        self.attrs = _Attrs()

    @property
    def shape(self):
        return self._data.shape

    @property
    def dtype(self):
        return self._data.dtype

    def __getitem__(self, idx):
        return np.array(self._data[idx], copy=True)

    def __setitem__(self, idx, val):
        self._data[idx] = val

    def __array__(self, dtype=None, copy=None):
        if dtype is None:
            return np.array(self._data, copy=True)
        return np.array(self._data, dtype=dtype, copy=True)

    def __truediv__(self, other):
        return self._data / other


class _Group:
    def __init__(self):
        self._items = {}
        self.attrs = _Attrs()

    def create_group(self, name):
        g = _Group()
        self._items[name] = g
        return g

    def create_dataset(self, name, shape=None, dtype=None, data=None):
        if data is not None:
            arr = np.array(data, dtype=dtype, copy=True)
        else:
            arr = np.zeros(shape, dtype=dtype)
        d = _Dataset(arr)
        self._items[name] = d
        return d

    def __getitem__(self, name):
        node = self
        for part in name.strip('/').split('/'):
            node = node._items[part]
        return node

    def __contains__(self, name):
        return name in self._items

    def keys(self):
        return self._items.keys()

    def items(self):
        return self._items.items()

    def __iter__(self):
        return iter(self._items)


class File(_Group):
    def __init__(self, filename, mode='r'):
        key = os.path.abspath(filename)
        if mode == 'w':
            super().__init__()
            _STORE[key] = self
            with open(key, 'wb'):
                pass
        else:
            if key not in _STORE:
                raise FileNotFoundError(key)
            src = _STORE[key]
            self.__dict__ = src.__dict__

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def close(self):
        pass


def store():
    return _STORE


def install():
    """Register the stand-in modules in ``sys.modules``."""
    h5 = types.ModuleType('h5py')
    h5.File = File
    h5.Dataset = _Dataset
    h5.Group = _Group
    sys.modules['h5py'] = h5

    def _noop(*a, **k):
        return None

    class _Anything:
        def __getattr__(self, name):
            return _noop

        def __call__(self, *a, **k):
            return None

    mpl = types.ModuleType('matplotlib')
    plt = types.ModuleType('matplotlib.pyplot')
    for fn in ('ion', 'pause', 'show', 'figure', 'subplots', 'plot', 'close',
               'colorbar', 'imshow', 'title', 'xlabel', 'ylabel', 'legend'):
        setattr(plt, fn, _noop)
    img = types.ModuleType('matplotlib.image')
    img.AxesImage = _Anything
    anim = types.ModuleType('matplotlib.animation')
    mpl.pyplot = plt
    mpl.image = img
    mpl.animation = anim
    sys.modules['matplotlib'] = mpl
    sys.modules['matplotlib.pyplot'] = plt
    sys.modules['matplotlib.image'] = img
    sys.modules['matplotlib.animation'] = anim
