"""Result and incident-beam file access with the reference's HDF5 layout.

The reference writes and reads its files through h5py (cpu/main_sim.py:
197-259, cpu/incident_sim.py:94-98,166-224, processresults.py:35-122).
``File(path, mode)`` returns an ``h5py.File`` when h5py is importable and
otherwise an ``h5lite.File``, which reads and writes the same HDF5 format
(version-0 superblock, symbol-table groups, contiguous datasets, compact
attributes) without libhdf5. Either way the file on disk is HDF5, at the
path asked for.
"""
import os

try:  # pragma: no cover - depends on the machine
    import h5py as _h5py
except ImportError:  # pragma: no cover
    _h5py = None

from . import h5lite

BACKEND = 'h5py' if _h5py is not None else 'h5lite'


def exists(path: str) -> bool:
    return os.path.isfile(path)


def File(path, mode='r'):
    """Open a result or incident file in the reference's layout."""
    if _h5py is not None:
        return _h5py.File(path, mode)
    return h5lite.File(path, mode)
