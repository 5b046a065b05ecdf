"""Result and incident-beam file access with the reference's HDF5 layout.

The reference writes and reads its files through h5py (cpu/main_sim.py:
197-259, cpu/incident_sim.py:94-98,166-224, processresults.py:35-122).
``File(path, mode)`` returns an ``h5py.File`` when h5py is importable, so the
files are the reference's own format. Where h5py is absent, the same
group / dataset / attribute tree is kept in a NumPy ``.npz`` archive next to
the requested path (``name.hdf5`` -> ``name.npz``) behind the subset of the
h5py API the simulator uses: ``create_group``, ``create_dataset``,
``__getitem__`` with '/'-paths, ``__contains__``, ``attrs`` and slicing.
"""
import os

import numpy as np

try:  # pragma: no cover - depends on the machine
    import h5py as _h5py
except ImportError:  # pragma: no cover
    _h5py = None

BACKEND = 'hdf5' if _h5py is not None else 'npz'


def storage_path(path: str) -> str:
    """Path of the file that actually holds ``path``'s content."""
    if BACKEND == 'hdf5':
        return path
    root, ext = os.path.splitext(path)
    return root + '.npz' if ext == '.hdf5' else path + '.npz'


def exists(path: str) -> bool:
    return os.path.isfile(storage_path(path))


class _Attrs(dict):
    pass


class _Dataset:
    def __init__(self, data):
        self._data = data
        self.attrs = _Attrs()

    shape = property(lambda self: self._data.shape)
    dtype = property(lambda self: self._data.dtype)

    def __getitem__(self, idx):
        return self._data[idx]

    def __setitem__(self, idx, val):
        self._data[idx] = val

    def __array__(self, dtype=None, copy=None):
        return np.asarray(self._data, dtype=dtype)

    def __len__(self):
        return len(self._data)


class _Group:
    def __init__(self):
        self._items = {}
        self.attrs = _Attrs()

    def create_group(self, name):
        if name in self._items:
            raise ValueError(f'group {name} already exists')
        g = _Group()
        self._items[name] = g
        return g

    def create_dataset(self, name, shape=None, dtype=None, data=None):
        if name in self._items:
            raise ValueError(f'dataset {name} already exists')
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
        try:
            self[name]
            return True
        except KeyError:
            return False

    def keys(self):
        return self._items.keys()

    def items(self):
        return self._items.items()

    def __iter__(self):
        return iter(self._items)


class NpzFile(_Group):
    """An h5py-like tree stored as one .npz archive."""

    def __init__(self, path, mode='r'):
        super().__init__()
        self._path = storage_path(path)
        self._mode = mode
        if mode in ('r', 'r+', 'a'):
            if not os.path.isfile(self._path):
                if mode == 'a':
                    return
                raise FileNotFoundError(self._path)
            with np.load(self._path, allow_pickle=False) as z:
                for key in z.files:
                    self._insert(key, z[key])
        elif mode not in ('w', 'w-', 'x'):
            raise ValueError(f'unsupported mode {mode}')
        elif mode in ('w-', 'x') and os.path.exists(self._path):
            raise FileExistsError(self._path)

    def _insert(self, key, value):
        path, _, attr = key.partition('@')
        node = self
        parts = [p for p in path.split('/') if p]
        if attr:
            for p in parts:
                if p not in node._items:
                    node._items[p] = _Group()
                node = node._items[p]
            v = value[()] if value.shape == () else value
            if isinstance(v, np.str_):
                v = str(v)
            node.attrs[attr] = v
            return
        for p in parts[:-1]:
            if p not in node._items:
                node._items[p] = _Group()
            node = node._items[p]
        node._items[parts[-1]] = _Dataset(np.array(value))

    def _flatten(self, node, prefix, out):
        for k, v in node.attrs.items():
            out[f'{prefix}@{k}'] = np.asarray(v)
        for name, child in node._items.items():
            p = f'{prefix}/{name}' if prefix else name
            if isinstance(child, _Dataset):
                out[p] = child._data
                for k, v in child.attrs.items():
                    out[f'{p}@{k}'] = np.asarray(v)
            else:
                if not child._items and not child.attrs:
                    out[f'{p}@__group__'] = np.asarray(True)
                self._flatten(child, p, out)

    def close(self):
        if self._mode == 'r':
            return
        out = {}
        self._flatten(self, '', out)
        os.makedirs(os.path.dirname(os.path.abspath(self._path)), exist_ok=True)
        tmp = self._path + '.tmp'
        with open(tmp, 'wb') as fh:
            np.savez(fh, **out)
        os.replace(tmp, self._path)
        self._mode = 'r'

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False


def File(path, mode='r'):
    """Open a result or incident file in the reference's layout."""
    if _h5py is not None:
        return _h5py.File(path, mode)
    return NpzFile(path, mode)
