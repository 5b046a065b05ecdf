"""HDF5 files without libhdf5 (``resultsio`` uses h5py instead wherever it
is importable).

A reader and writer for the part of the HDF5 format that h5py's default
settings produce for this simulator's files -- the result file
(cpu/main_sim.py:197-259, processresults.py:35-122) and the incident-beam
file (cpu/incident_sim.py:94-98,166-171,195-224): a version-0 superblock,
version-1 object headers, groups indexed by a symbol table (a version-1
B-tree over symbol-table nodes, link names in a local heap), datasets in
contiguous storage, compact attributes, and variable-length UTF-8 strings
in a global heap. Every structure follows the published HDF5 File Format
Specification (The HDF Group): superblock (II.A), B-tree version 1
(III.A.1), symbol-table node (III.B), symbol-table entry (III.C), local
heap (III.D), global heap (III.E), version-1 object header (IV.A.1.a) and
its messages (IV.A.2: dataspace 0x01, link info 0x02, datatype 0x03, fill
value 0x05, link 0x06, layout 0x08, attribute 0x0C, continuation 0x10,
symbol table 0x11, attribute info 0x15).

Types map as h5py maps them: bool is an 8-bit enum {FALSE: 0, TRUE: 1},
complex is a compound {r, i}, str a variable-length UTF-8 string, bytes a
fixed-length null-padded string, Python int / float int64 / float64.

Writing: raw data goes to the end of the file when a dataset is created;
the metadata of the whole tree follows it when the file is closed, and the
superblock is written last. A new file is written as ``<path>.partial`` and
renamed onto its path when it is closed, so that a file at the path is
always complete (a process that dies while writing leaves no result file
for the simulator's skip-if-exists check to mistake for a finished one). A file opened 'r+' or 'a' is read into the
same tree, new raw data is appended, and on close the tree's metadata is
written again at the end (the earlier metadata stays in the file, unused).

Not supported (NotImplementedError when met in a file being read):
version-2/3 superblocks and version-2 object headers (h5py's
libver='latest'), dense link or attribute storage, chunked, filtered or
virtual datasets, shared messages, reference / array / opaque / bitfield
types, variable-length sequences, string datasets.
"""
import os
import struct
import sys

import numpy as np

__all__ = ['File', 'Group', 'Dataset', 'AttributeManager']

SIGNATURE = b'\x89HDF\r\n\x1a\n'
UNDEF = 0xFFFFFFFFFFFFFFFF
HEAP_FREE_NULL = 1        # end of a local heap's free list on disk (no valid offset is odd)
LEAF_K = 4                # a symbol-table node holds 2 * LEAF_K entries
NODE_K = 16               # a group B-tree node holds 2 * NODE_K children
ENTRY_SIZE = 40           # symbol-table entry
SNOD_SIZE = 8 + 2 * LEAF_K * ENTRY_SIZE
BTREE_SIZE = 24 + 2 * NODE_K * 8 + (2 * NODE_K + 1) * 8
GCOL_MIN = 4096           # smallest global heap collection
GCOL_TARGET = 1 << 20     # start a new collection beyond this size
MAX_MESSAGE = 0xFFF8      # largest object header message body (16-bit size, 8-byte aligned)
WRITE_CHUNK = 1 << 28

MSG_NIL, MSG_SPACE, MSG_LINFO, MSG_TYPE, MSG_FILL = 0x00, 0x01, 0x02, 0x03, 0x05
MSG_LINK, MSG_LAYOUT, MSG_FILTER, MSG_ATTR = 0x06, 0x08, 0x0B, 0x0C
MSG_CONT, MSG_STAB, MSG_AINFO = 0x10, 0x11, 0x15


def _pad8(n):
    return (n + 7) & ~7


def _padded(b):
    return bytes(b) + b'\0' * (_pad8(len(b)) - len(b))


def _big_endian(dt):
    return dt.byteorder == '>' or (dt.byteorder == '=' and sys.byteorder == 'big')


# ---------------------------------------------------------------------------
# datatype and dataspace messages
# ---------------------------------------------------------------------------

def _dt_head(cls, bits, size):
    """Class-and-version byte (version 1), 24 class bits, element size."""
    return struct.pack('<BI', 0x10 | cls, bits)[:4] + struct.pack('<I', size)


def _fixed(size, signed, big=False):
    return _dt_head(0, (1 if big else 0) | (0x08 if signed else 0), size) + \
        struct.pack('<HH', 0, 8 * size)


# IEEE layouts: (sign bit, exponent position, exponent size, mantissa size, bias)
_IEEE = {2: (15, 10, 5, 10, 15), 4: (31, 23, 8, 23, 127), 8: (63, 52, 11, 52, 1023)}

# variable-length string (bits: type 1 = string, null-terminated, UTF-8) of
# unsigned 8-bit characters; an element on disk is 16 bytes
# (length, global heap collection address, object index)
VLEN_UTF8 = _dt_head(9, 0x01 | (1 << 8), 16) + _fixed(1, False)


def encode_dtype(dt):
    """Datatype message body (version 1) for a numpy dtype."""
    dt = np.dtype(dt)
    if dt.kind == 'b':
        names = _padded(b'FALSE\0') + _padded(b'TRUE\0')
        return _dt_head(8, 2, 1) + _fixed(1, True) + names + b'\x00\x01'
    big = _big_endian(dt)
    if dt.kind in 'iu':
        return _fixed(dt.itemsize, dt.kind == 'i', big)
    if dt.kind == 'f':
        if dt.itemsize not in _IEEE:
            raise TypeError(f'no HDF5 equivalent for {dt}')
        sign, epos, esize, msize, bias = _IEEE[dt.itemsize]
        bits = (1 if big else 0) | 0x20 | (sign << 8)   # 0x20: implied leading mantissa bit
        return _dt_head(1, bits, dt.itemsize) + struct.pack(
            '<HHBBBBI', 0, 8 * dt.itemsize, epos, esize, 0, msize, bias)
    if dt.kind == 'c':
        half = np.dtype(('>' if big else '<') + f'f{dt.itemsize // 2}')
        return _compound([('r', 0, half), ('i', dt.itemsize // 2, half)], dt.itemsize)
    if dt.kind == 'V' and dt.names:
        return _compound([(n, dt.fields[n][1], dt.fields[n][0]) for n in dt.names], dt.itemsize)
    if dt.kind == 'S':
        return _dt_head(3, 1, max(dt.itemsize, 1))       # null-padded ASCII, as numpy 'S'
    raise TypeError(f'no HDF5 equivalent for {dt}')


def _compound(members, size):
    body = b''
    for name, off, mdt in members:
        body += _padded(name.encode('utf-8') + b'\0')
        body += struct.pack('<IB3xI4x16x', off, 0, 0)     # offset, rank 0, no permutation
        body += encode_dtype(mdt)
    return _dt_head(6, len(members), size) + body


def decode_dtype(buf, pos):
    """(dtype, is_vlen_string, end) of the datatype message at ``pos``."""
    cv, bits, size = buf[pos], int.from_bytes(buf[pos + 1:pos + 4], 'little'), \
        struct.unpack_from('<I', buf, pos + 4)[0]
    cls, ver = cv & 0x0F, cv >> 4
    p = pos + 8
    order = '>' if bits & 1 else '<'
    if cls == 0:
        return np.dtype(f"{order}{'i' if bits & 0x08 else 'u'}{size}"), False, p + 4
    if cls == 1:
        if size not in _IEEE:
            raise NotImplementedError(f'{size}-byte floating point')
        return np.dtype(f'{order}f{size}'), False, p + 12
    if cls == 3:
        return np.dtype(f'S{size}'), False, p
    if cls == 6:
        names, offs, types = [], [], []
        for _ in range(bits & 0xFFFF):
            end = buf.index(b'\0', p)
            names.append(bytes(buf[p:end]).decode('utf-8'))
            if ver < 3:
                p += _pad8(end - p + 1)
                offs.append(struct.unpack_from('<I', buf, p)[0])
                p += 32 if ver == 1 else 4
            else:
                p = end + 1
                nb = 1 if size < 1 << 8 else 2 if size < 1 << 16 else 3 if size < 1 << 24 else 4
                offs.append(int.from_bytes(buf[p:p + nb], 'little'))
                p += nb
            mdt, vstr, p = decode_dtype(buf, p)
            if vstr:
                raise NotImplementedError('compound members of string type')
            types.append(mdt)
        if names == ['r', 'i'] and types[0] == types[1] and types[0].kind == 'f' \
                and offs == [0, types[0].itemsize] and size == 2 * types[0].itemsize:
            return np.dtype(('>' if _big_endian(types[0]) else '<') + f'c{size}'), False, p
        return np.dtype({'names': names, 'formats': types, 'offsets': offs,
                         'itemsize': size}), False, p
    if cls == 8:
        n = bits & 0xFFFF
        base, _, p = decode_dtype(buf, p)
        names = []
        for _ in range(n):
            end = buf.index(b'\0', p)
            names.append(bytes(buf[p:end]))
            p = p + _pad8(end - p + 1) if ver < 3 else end + 1
        vals = np.frombuffer(bytes(buf[p:p + n * base.itemsize]), base, n).tolist()
        p += n * base.itemsize
        if base.itemsize == 1 and sorted(zip(names, vals)) == [(b'FALSE', 0), (b'TRUE', 1)]:
            return np.dtype(bool), False, p
        return base, False, p
    if cls == 9:
        if bits & 0x0F != 1:
            raise NotImplementedError('variable-length sequences')
        _, _, p = decode_dtype(buf, p)
        return np.dtype(object), True, p
    raise NotImplementedError(f'HDF5 datatype class {cls}')


def encode_space(shape):
    """Dataspace message body (version 1; rank 0 is a scalar)."""
    return struct.pack('<BBBB4x', 1, len(shape), 0, 0) + \
        b''.join(struct.pack('<Q', d) for d in shape)


def decode_space(buf, pos):
    """Shape of the dataspace message at ``pos``; None for a null dataspace."""
    ver, rank = buf[pos], buf[pos + 1]
    if ver == 1:
        p = pos + 8
    elif ver == 2:
        if buf[pos + 3] == 2:
            return None
        p = pos + 4
    else:
        raise NotImplementedError(f'dataspace version {ver}')
    return tuple(struct.unpack_from(f'<{rank}Q', buf, p))


# ---------------------------------------------------------------------------
# the tree
# ---------------------------------------------------------------------------

def _attr_value(value):
    """An attribute value in the form it is stored and read back."""
    if isinstance(value, str):
        return value
    if isinstance(value, bytes):
        return np.bytes_(value)
    arr = np.asarray(value)
    if arr.dtype.kind in 'UO':
        flat = [str(x) if arr.dtype.kind == 'U' else x for x in arr.flat]
        if not all(isinstance(x, str) for x in flat):
            raise TypeError(f'Object dtype {arr.dtype} has no native HDF5 equivalent')
        if arr.ndim == 0:
            return flat[0]
        out = np.empty(arr.shape, object)
        out.flat[:] = flat
        return out
    encode_dtype(arr.dtype)                                # raises for unsupported types
    arr = np.array(arr, copy=True)
    return arr[()] if arr.ndim == 0 else arr


class AttributeManager:
    """``node.attrs``: a name -> value mapping kept in the object header."""

    def __init__(self, node):
        self._node = node
        self._items = {}

    def __getitem__(self, name):
        try:
            return self._items[name]
        except KeyError:
            raise KeyError(f"Can't open attribute (can't locate attribute: '{name}')") from None

    def __setitem__(self, name, value):
        self._node.file._check_writable()
        self._items[name] = _attr_value(value)
        self._node.file._dirty = True

    def __delitem__(self, name):
        self._node.file._check_writable()
        del self._items[name]
        self._node.file._dirty = True

    def __contains__(self, name):
        return name in self._items

    def __iter__(self):
        return iter(self.keys())

    def __len__(self):
        return len(self._items)

    def keys(self):
        return sorted(self._items, key=lambda s: s.encode('utf-8'))

    def values(self):
        return [self._items[k] for k in self.keys()]

    def items(self):
        return [(k, self._items[k]) for k in self.keys()]

    def get(self, name, default=None):
        return self._items.get(name, default)


class Dataset:
    """A dataset in contiguous (or, read from another file, compact)
    storage. Reads return copies; writes go straight to the file."""

    def __init__(self, file, name, shape, dtype, addr, compact=None, vlen=False, type_msg=None):
        self.file = file
        self.name = name
        self.shape = tuple(int(d) for d in shape)
        self.dtype = np.dtype(dtype)
        self._addr = addr
        self._compact = compact
        self._vlen = vlen
        self._type_msg = type_msg        # a datatype read from a file is written back unchanged
        self.attrs = AttributeManager(self)

    ndim = property(lambda self: len(self.shape))
    size = property(lambda self: int(np.prod(self.shape, dtype=np.int64)))
    nbytes = property(lambda self: self.size * self.dtype.itemsize)

    def __len__(self):
        if not self.shape:
            raise TypeError('Attempt to take len() of scalar dataset')
        return self.shape[0]

    def __bool__(self):
        return True

    def __repr__(self):
        return f'<HDF5 dataset "{self.name}": shape {self.shape}, type "{self.dtype.str}">'

    def _stored(self):
        return self._addr != UNDEF and self.size > 0

    def _map(self):
        f = self.file
        mm = f._maps.get(id(self))
        if mm is None:
            f._fh.flush()
            end = f._base + self._addr + self.nbytes
            if f.mode == 'r' and os.path.getsize(f._disk) < end:
                raise OSError(f'truncated HDF5 file: dataset {self.name} ends at byte {end}')
            mm = np.memmap(f._disk, self.dtype, 'r' if f.mode == 'r' else 'r+',
                           offset=f._base + self._addr, shape=self.shape or (1,))
            f._maps[id(self)] = mm
        return mm if self.shape else mm.reshape(())

    def _read_all(self):
        f = self.file
        if self._compact is not None:
            return np.frombuffer(self._compact, self.dtype, self.size).reshape(self.shape).copy()
        if not self._stored():
            return np.zeros(self.shape, self.dtype)
        f._fh.flush()
        data = np.fromfile(f._disk, self.dtype, self.size, offset=f._base + self._addr)
        if data.size != self.size:
            raise OSError(f'truncated HDF5 file: dataset {self.name} holds {data.size} of '
                          f'{self.size} elements')
        return data.reshape(self.shape)

    def __getitem__(self, idx):
        self.file._check_open()
        if self._vlen:
            raise NotImplementedError('variable-length string datasets')
        whole = idx is Ellipsis or (isinstance(idx, tuple) and idx == ()) or \
            (isinstance(idx, slice) and idx == slice(None))
        if whole or self._compact is not None or not self._stored():
            return self._read_all()[idx]
        return np.array(self._map()[idx])

    def __setitem__(self, idx, value):
        self.file._check_writable()
        if self._compact is not None or not self._stored():
            raise NotImplementedError('writing to compact or empty datasets')
        self._map()[idx] = value

    def __array__(self, dtype=None, copy=None):
        arr = self[()]
        return np.asarray(arr, dtype=dtype)

    def read_direct(self, dest):
        dest[...] = self[()]


class Group:
    """A group: named links to groups and datasets, and attributes."""

    def __init__(self, file, name):
        self.file = file
        self.name = name
        self._links = {}
        self.attrs = AttributeManager(self)

    def __repr__(self):
        return f'<HDF5 group "{self.name}" ({len(self._links)} members)>'

    def __bool__(self):
        return True

    def _path_of(self, leaf):
        return ('' if self.name == '/' else self.name) + '/' + leaf

    def __getitem__(self, path):
        node = self.file if path.startswith('/') else self
        for part in filter(None, path.split('/')):
            if not isinstance(node, Group) or part not in node._links:
                raise KeyError(f"Unable to open object (object '{part}' doesn't exist)")
            node = node._links[part]
        return node

    def get(self, path, default=None):
        try:
            return self[path]
        except KeyError:
            return default

    def __contains__(self, path):
        return self.get(path) is not None

    def keys(self):
        return sorted(self._links, key=lambda s: s.encode('utf-8'))

    def values(self):
        return [self._links[k] for k in self.keys()]

    def items(self):
        return [(k, self._links[k]) for k in self.keys()]

    def __iter__(self):
        return iter(self.keys())

    def __len__(self):
        return len(self._links)

    def _parent(self, path):
        parts = [p for p in path.split('/') if p]
        if not parts:
            raise ValueError('empty object name')
        node = self.file if path.startswith('/') else self
        for part in parts[:-1]:
            if part not in node._links:
                node._links[part] = Group(self.file, node._path_of(part))
            node = node._links[part]
            if not isinstance(node, Group):
                raise TypeError(f"'{part}' is not a group")
        return node, parts[-1]

    def create_group(self, path):
        self.file._check_writable()
        parent, leaf = self._parent(path)
        if leaf in parent._links:
            raise ValueError('Unable to create group (name already exists)')
        g = Group(self.file, parent._path_of(leaf))
        parent._links[leaf] = g
        self.file._dirty = True
        return g

    def require_group(self, path):
        if path in self:
            node = self[path]
            if not isinstance(node, Group):
                raise TypeError(f"Incompatible object ({type(node).__name__}) already exists")
            return node
        return self.create_group(path)

    def create_dataset(self, path, shape=None, dtype=None, data=None):
        """A contiguous dataset: from ``data`` (written now), or of
        ``shape`` and ``dtype`` (default float32), zero-filled."""
        f = self.file
        f._check_writable()
        if data is not None:
            arr = np.asarray(data, dtype=dtype)
            if shape is not None and tuple(shape) != arr.shape:
                if int(np.prod(shape)) != arr.size:
                    raise ValueError(f'shape {tuple(shape)} does not match the data {arr.shape}')
                arr = arr.reshape(shape)
        else:
            if shape is None:
                raise TypeError('One of data, shape or dtype must be specified')
            arr = None
            shape = (shape,) if isinstance(shape, (int, np.integer)) else tuple(shape)
        dt = np.dtype(dtype if dtype is not None else (arr.dtype if arr is not None else 'f4'))
        if arr is not None:
            dt = arr.dtype
        if dt.kind in 'UOS':
            raise NotImplementedError('string datasets')
        encode_dtype(dt)
        parent, leaf = self._parent(path)
        if leaf in parent._links:
            raise ValueError('Unable to create dataset (name already exists)')
        shp = arr.shape if arr is not None else shape
        nbytes = int(np.prod(shp, dtype=np.int64)) * dt.itemsize
        addr = f._write_raw(arr) if arr is not None else f._reserve(nbytes)
        ds = Dataset(f, parent._path_of(leaf), shp, dt, addr if nbytes else UNDEF)
        parent._links[leaf] = ds
        f._dirty = True
        return ds

    def __delitem__(self, path):
        self.file._check_writable()
        parent, leaf = self._parent(path)
        del parent._links[leaf]
        self.file._dirty = True


# ---------------------------------------------------------------------------
# the file
# ---------------------------------------------------------------------------

class _GlobalHeap:
    """Variable-length strings, gathered while attributes are encoded and
    written as global heap collections before the object headers."""

    def __init__(self):
        self.colls = [[]]
        self.sizes = [0]
        self.addrs = []

    def add(self, data):
        need = 16 + _pad8(len(data))
        if self.colls[-1] and (len(self.colls[-1]) >= 0xFFFE or self.sizes[-1] + need > GCOL_TARGET):
            self.colls.append([])
            self.sizes.append(0)
        self.colls[-1].append(data)
        self.sizes[-1] += need
        return len(self.colls) - 1, len(self.colls[-1])

    def write(self, f):
        for objs, used in zip(self.colls, self.sizes):
            if not objs:
                self.addrs.append(UNDEF)
                continue
            size = max(GCOL_MIN, 16 + used + 16)                  # + the free-space object
            free = size - 16 - used
            blob = bytearray(b'GCOL' + struct.pack('<B3xQ', 1, size))
            for i, d in enumerate(objs):
                blob += struct.pack('<HH4xQ', i + 1, 0, len(d)) + _padded(d)
            blob += struct.pack('<HH4xQ', 0, 0, free) + b'\0' * (free - 16)
            self.addrs.append(f._append(bytes(blob)))


class _AttrPlan:
    def __init__(self, name, value, heap):
        self.name = name.encode('utf-8') + b'\0'
        if isinstance(value, str) or (isinstance(value, np.ndarray) and value.dtype == object):
            strings = [value] if isinstance(value, str) else list(value.flat)
            self.shape = () if isinstance(value, str) else value.shape
            self.dtype = VLEN_UTF8
            self.slots = []
            for s in strings:
                data = s.encode('utf-8')
                self.slots.append((len(data),) + heap.add(data))
            self.raw = None
        else:
            arr = np.asarray(value)
            self.shape, self.dtype, self.raw = arr.shape, encode_dtype(arr.dtype), arr.tobytes()

    def encode(self, heap):
        raw = self.raw
        if raw is None:
            raw = b''.join(struct.pack('<IQI', n, heap.addrs[c], i) for n, c, i in self.slots)
        space = encode_space(self.shape)
        return struct.pack('<BBHHH', 1, 0, len(self.name), len(self.dtype), len(space)) + \
            _padded(self.name) + _padded(self.dtype) + _padded(space) + raw


class File(Group):
    """An HDF5 file with h5py's modes: 'r', 'r+', 'w', 'w-' / 'x', 'a'."""

    def __init__(self, name, mode='r'):
        path = os.fspath(name)
        exists = os.path.exists(path)
        if mode == 'a':
            mode = 'r+' if exists else 'w'
        if mode in ('w-', 'x'):
            if exists:
                raise FileExistsError(f'Unable to create file (file exists: {path})')
            mode = 'w'
        if mode not in ('r', 'r+', 'w'):
            raise ValueError(f'Invalid mode; must be one of r, r+, w, w-, x, a (got {mode})')
        if mode != 'w' and not exists:
            raise FileNotFoundError(f'Unable to open file (no such file: {path})')
        self._fh = None
        super().__init__(self, '/')
        self.filename = path
        self.mode = 'r' if mode == 'r' else 'r+'
        self._maps = {}
        self._gcols = {}
        self._base = 0
        self._dirty = mode == 'w'
        # a new file is written beside its path and renamed onto it when it is
        # complete, so that a file at the path is always a whole HDF5 file
        self._disk = path + '.partial' if mode == 'w' else path
        self._fh = open(self._disk, {'r': 'rb', 'r+': 'r+b', 'w': 'w+b'}[mode])
        try:
            if mode == 'w':
                self._fh.write(b'\0' * 96)          # the superblock, written on close
                self._eof = 96
            else:
                self._load()
        except BaseException:
            self._fh.close()
            self._fh = None
            raise

    # -- plumbing ----------------------------------------------------------
    def _check_open(self):
        if self._fh is None:
            raise ValueError('Not a location (file is closed)')

    def _check_writable(self):
        self._check_open()
        if self.mode == 'r':
            raise ValueError('Unable to modify (no write intent on file)')

    def _read(self, addr, n):
        self._fh.seek(self._base + addr)
        data = self._fh.read(n)
        if len(data) != n:
            raise OSError(f'truncated HDF5 file: {n} bytes at address {addr}')
        return data

    def _append(self, data):
        addr = _pad8(self._eof)
        self._fh.seek(self._base + addr)
        self._fh.write(data)
        self._eof = addr + len(data)
        return addr

    def _place(self, addr, data):
        """Append ``data``, which must land at ``addr`` (precomputed because
        the structure refers to its own address)."""
        got = self._append(data)
        if got != addr:
            raise RuntimeError(f'HDF5 structure placed at {got}, expected {addr}')

    def _reserve(self, nbytes):
        addr = _pad8(self._eof)
        self._eof = addr + nbytes
        self._fh.flush()
        if os.fstat(self._fh.fileno()).st_size < self._base + self._eof:
            self._fh.truncate(self._base + self._eof)
        return addr

    def _write_raw(self, arr):
        arr = np.ascontiguousarray(arr)
        addr = _pad8(self._eof)
        self._fh.seek(self._base + addr)
        flat = arr.reshape(-1).view(np.uint8)
        for i in range(0, flat.size, WRITE_CHUNK):
            self._fh.write(flat[i:i + WRITE_CHUNK])
        self._eof = addr + flat.size
        return addr

    def flush(self):
        self._check_open()
        for mm in self._maps.values():
            mm.flush()
        self._fh.flush()

    def close(self):
        if self._fh is None:
            return
        complete = False
        try:
            for mm in self._maps.values():
                mm.flush()
            self._maps.clear()
            if self.mode != 'r' and self._dirty:
                self._write_metadata()
                self._dirty = False
            complete = True
        finally:
            self._fh.close()
            self._fh = None
        if complete and self._disk != self.filename:
            os.replace(self._disk, self.filename)
            self._disk = self.filename

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False

    def __bool__(self):
        return self._fh is not None

    # -- reading -----------------------------------------------------------
    def _load(self):
        base = None
        for off in (0, 512, 1024, 2048, 4096, 8192):
            self._fh.seek(off)
            if self._fh.read(8) == SIGNATURE:
                base = off
                break
        if base is None:
            raise OSError(f'Unable to open file (file signature not found: {self.filename})')
        self._fh.seek(base)
        sb = self._fh.read(96 + 4)
        ver = sb[8]
        if ver not in (0, 1):
            raise NotImplementedError(f'HDF5 superblock version {ver}')
        if sb[13] != 8 or sb[14] != 8:
            raise NotImplementedError('offset or length sizes other than 8 bytes')
        p = 24 + (4 if ver == 1 else 0)
        base_addr, _, eof, _ = struct.unpack_from('<QQQQ', sb, p)
        self._base = base_addr
        root = sb[p + 32:p + 32 + ENTRY_SIZE]
        _, root_addr = struct.unpack_from('<QQ', root)
        size = os.fstat(self._fh.fileno()).st_size - self._base
        self._eof = max(eof, size)
        self._load_object(root_addr, '/', self, set())

    def _messages(self, addr):
        head = self._read(addr, 16)
        if head[:4] == b'OHDR':
            raise NotImplementedError('version-2 object headers')
        ver, _, _, _, size = struct.unpack_from('<BBHII', head)
        if ver != 1:
            raise ValueError(f'bad object header version {ver} at address {addr}')
        chunks, out = [(addr + 16, size)], []
        while chunks:
            caddr, csize = chunks.pop(0)
            data = self._read(caddr, csize)
            p = 0
            while p + 8 <= csize:
                mtype, msize, mflags = struct.unpack_from('<HHB', data, p)
                body = data[p + 8:p + 8 + msize]
                p += 8 + msize
                if mtype == MSG_CONT:
                    chunks.append(struct.unpack_from('<QQ', body))
                elif mtype != MSG_NIL:
                    if mflags & 0x02:
                        raise NotImplementedError('shared object header messages')
                    out.append((mtype, body))
        return out

    def _load_object(self, addr, name, node, seen):
        msgs = self._messages(addr)
        kinds = {t for t, _ in msgs}
        if node is None:
            if kinds & {MSG_STAB, MSG_LINK, MSG_LINFO}:
                node = Group(self, name)
            elif MSG_LAYOUT in kinds:
                node = self._dataset(name, msgs)
            else:
                raise NotImplementedError(f'object {name} is neither a group nor a dataset')
        for t, body in msgs:
            if t == MSG_ATTR:
                key, value = self._attribute(body)
                node.attrs._items[key] = value
            elif t == MSG_AINFO:
                flags = body[1]
                heap = struct.unpack_from('<Q', body, 2 + (2 if flags & 1 else 0))[0]
                if heap != UNDEF:
                    raise NotImplementedError('dense attribute storage')
        if isinstance(node, Group):
            if addr in seen:
                return node
            seen = seen | {addr}
            for child, caddr in self._read_links(msgs):
                node._links[child] = self._load_object(caddr, node._path_of(child), None, seen)
        return node

    def _read_links(self, msgs):
        out = []
        for t, body in msgs:
            if t == MSG_STAB:
                btree, heap = struct.unpack_from('<QQ', body)
                hdr = self._read(heap, 32)
                if hdr[:4] != b'HEAP':
                    raise ValueError('bad local heap signature')
                dsize, _, daddr = struct.unpack_from('<QQQ', hdr, 8)
                names = self._read(daddr, dsize)
                for noff, oaddr in self._walk(btree):
                    out.append((names[noff:names.index(b'\0', noff)].decode('utf-8'), oaddr))
            elif t == MSG_LINFO:
                flags = body[1]
                heap = struct.unpack_from('<Q', body, 2 + (8 if flags & 1 else 0))[0]
                if heap != UNDEF:
                    raise NotImplementedError('dense link storage')
            elif t == MSG_LINK:
                flags, p = body[1], 2
                ltype = 0
                if flags & 0x08:
                    ltype, p = body[p], p + 1
                p += (8 if flags & 0x04 else 0) + (1 if flags & 0x10 else 0)
                nsz = 1 << (flags & 3)
                nlen = int.from_bytes(body[p:p + nsz], 'little')
                p += nsz
                name = body[p:p + nlen].decode('utf-8')
                if ltype == 0:                           # hard link; soft/external skipped
                    out.append((name, struct.unpack_from('<Q', body, p + nlen)[0]))
        return out

    def _walk(self, addr):
        head = self._read(addr, 24)
        if head[:4] != b'TREE' or head[4] != 0:
            raise ValueError('bad group B-tree node')
        level, n = head[5], struct.unpack_from('<H', head, 6)[0]
        body = self._read(addr + 24, 16 * n + 8)
        out = []
        for i in range(n):
            child = struct.unpack_from('<Q', body, 8 + 16 * i)[0]
            if level > 0:
                out += self._walk(child)
                continue
            snod = self._read(child, 8)
            if snod[:4] != b'SNOD':
                raise ValueError('bad symbol table node')
            k = struct.unpack_from('<H', snod, 6)[0]
            ents = self._read(child + 8, k * ENTRY_SIZE)
            out += [struct.unpack_from('<QQ', ents, ENTRY_SIZE * j) for j in range(k)]
        return out

    def _dataset(self, name, msgs):
        m = dict(msgs)
        if MSG_FILTER in m:
            raise NotImplementedError(f'filtered dataset {name}')
        shape = decode_space(m[MSG_SPACE], 0) or ()
        dtype, vlen, _ = decode_dtype(m[MSG_TYPE], 0)
        lay = m[MSG_LAYOUT]
        ver, addr, compact = lay[0], UNDEF, None
        if ver in (3, 4):
            cls = lay[1]
            if cls == 0:
                n = struct.unpack_from('<H', lay, 2)[0]
                compact = bytes(lay[4:4 + n])
            elif cls == 1:
                addr = struct.unpack_from('<Q', lay, 2)[0]
            else:
                raise NotImplementedError(f'chunked or virtual dataset {name}')
        elif ver in (1, 2):
            rank, cls = lay[1], lay[2]
            if cls == 1:
                addr = struct.unpack_from('<Q', lay, 8)[0]
            elif cls == 0:
                p = 8 + 4 * rank
                n = struct.unpack_from('<I', lay, p)[0]
                compact = bytes(lay[p + 4:p + 4 + n])
            else:
                raise NotImplementedError(f'chunked dataset {name}')
        else:
            raise NotImplementedError(f'layout message version {ver}')
        return Dataset(self, name, shape, dtype, addr, compact, vlen, bytes(m[MSG_TYPE]))

    def _attribute(self, body):
        ver = body[0]
        if ver == 1:
            nlen, tlen, slen = struct.unpack_from('<HHH', body, 2)
            p = 8
            name = body[p:p + nlen].split(b'\0')[0].decode('utf-8')
            p += _pad8(nlen)
            dtype, vlen, _ = decode_dtype(body, p)
            p += _pad8(tlen)
            shape = decode_space(body, p)
            p += _pad8(slen)
        elif ver in (2, 3):
            if body[1] & 0x03:
                raise NotImplementedError('attributes with shared datatypes or dataspaces')
            nlen, tlen, slen = struct.unpack_from('<HHH', body, 2)
            p = 8 + (1 if ver == 3 else 0)
            name = body[p:p + nlen].split(b'\0')[0].decode('utf-8')
            p += nlen
            dtype, vlen, _ = decode_dtype(body, p)
            p += tlen
            shape = decode_space(body, p)
            p += slen
        else:
            raise NotImplementedError(f'attribute message version {ver}')
        if shape is None:
            return name, None
        n = int(np.prod(shape, dtype=np.int64))
        raw = body[p:]
        if vlen:
            items = [self._vlen_string(raw[16 * i:16 * i + 16]) for i in range(n)]
            if shape == ():
                return name, items[0]
            out = np.empty(shape, object)
            out.flat[:] = items
            return name, out
        arr = np.frombuffer(raw, dtype, n).reshape(shape).copy()
        return name, arr[()] if shape == () else arr

    def _vlen_string(self, ref):
        n, addr, idx = struct.unpack('<IQI', ref)
        if n == 0:
            return ''
        objs = self._gcols.get(addr)
        if objs is None:
            head = self._read(addr, 16)
            if head[:4] != b'GCOL':
                raise ValueError('bad global heap collection')
            size = struct.unpack_from('<Q', head, 8)[0]
            data = self._read(addr, size)
            objs, p = {}, 16
            while p + 16 <= size:
                i, _, osize = struct.unpack_from('<HH4xQ', data, p)
                if i == 0:
                    break
                objs[i] = data[p + 16:p + 16 + osize]
                p += 16 + _pad8(osize)
            self._gcols[addr] = objs
        return objs[idx][:n].decode('utf-8')

    # -- writing -----------------------------------------------------------
    def _write_metadata(self):
        heap = _GlobalHeap()
        plans = {}

        def plan(node):
            plans[id(node)] = [_AttrPlan(k, v, heap) for k, v in node.attrs.items()]
            if isinstance(node, Group):
                for child in node._links.values():
                    plan(child)
        plan(self)
        heap.write(self)
        root, btree, lheap = self._write_node(self, plans, heap)
        self._fh.seek(self._base)
        self._fh.write(
            SIGNATURE + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack('<HHI', LEAF_K, NODE_K, 0)
            + struct.pack('<QQQQ', self._base, UNDEF, self._eof, UNDEF)
            + struct.pack('<QQII', 0, root, 1, 0) + struct.pack('<QQ', btree, lheap))
        self._fh.flush()

    def _write_header(self, msgs):
        body = bytearray()
        for t, data in msgs:
            data = _padded(data)
            if len(data) > MAX_MESSAGE:
                raise ValueError(f'object header message of {len(data)} bytes is too large')
            body += struct.pack('<HHB3x', t, len(data), 1 if t == MSG_TYPE else 0) + data
        return self._append(struct.pack('<BBHII4x', 1, 0, len(msgs), 1, len(body)) + body)

    def _write_node(self, node, plans, heap):
        """Object header address, and for a group its B-tree and local heap
        addresses (children first, so that every address is known)."""
        attrs = [(MSG_ATTR, p.encode(heap)) for p in plans[id(node)]]
        if isinstance(node, Dataset):
            data = node._read_all() if node._compact is not None else None
            if data is not None:
                node._addr, node._compact = (self._write_raw(data) if data.size else UNDEF), None
            nbytes = node.nbytes if node._addr != UNDEF else 0
            msgs = [(MSG_FILL, bytes([2, 2, 2, 0])),             # late alloc, fill if set, no fill
                    (MSG_TYPE, node._type_msg or encode_dtype(node.dtype)),
                    (MSG_SPACE, encode_space(node.shape)),
                    (MSG_LAYOUT, struct.pack('<BBQQ', 3, 1, node._addr, nbytes))]
            return self._write_header(msgs + attrs), None, None
        entries = []
        for name in node.keys():
            addr, bt, hp = self._write_node(node._links[name], plans, heap)
            entries.append((name, addr, bt, hp))
        # link names: offset 0 is the empty name that the left-most key refers to
        seg, offs = bytearray(8), []
        for name, *_ in entries:
            offs.append(len(seg))
            seg += _padded(name.encode('utf-8') + b'\0')
        haddr = _pad8(self._eof)
        self._place(haddr, b'HEAP' + struct.pack('<B3xQQQ', 0, len(seg), HEAP_FREE_NULL,
                                                 haddr + 32) + bytes(seg))
        nodes = []                                   # (address, heap offset of the last name)
        for i in range(0, len(entries), 2 * LEAF_K):
            blob = bytearray(b'SNOD' + struct.pack('<BBH', 1, 0, len(entries[i:i + 2 * LEAF_K])))
            for (name, addr, bt, hp), off in zip(entries[i:i + 2 * LEAF_K], offs[i:i + 2 * LEAF_K]):
                if bt is None:
                    blob += struct.pack('<QQII16x', off, addr, 0, 0)
                else:
                    blob += struct.pack('<QQIIQQ', off, addr, 1, 0, bt, hp)
            blob += b'\0' * (SNOD_SIZE - len(blob))
            nodes.append((self._append(bytes(blob)), offs[min(i + 2 * LEAF_K, len(offs)) - 1]))
        level = 0
        while True:
            groups = [nodes[i:i + 2 * NODE_K] for i in range(0, len(nodes), 2 * NODE_K)] or [[]]
            first = _pad8(self._eof)
            addrs = [first + j * BTREE_SIZE for j in range(len(groups))]
            upper, left_key = [], 0
            for j, kids in enumerate(groups):
                blob = bytearray(b'TREE' + struct.pack(
                    '<BBHQQ', 0, level, len(kids), addrs[j - 1] if j else UNDEF,
                    addrs[j + 1] if j + 1 < len(groups) else UNDEF))
                blob += struct.pack('<Q', left_key)
                for caddr, last in kids:
                    blob += struct.pack('<QQ', caddr, last)
                blob += b'\0' * (BTREE_SIZE - len(blob))
                self._place(addrs[j], bytes(blob))
                left_key = kids[-1][1] if kids else 0
                upper.append((addrs[j], left_key))
            if len(upper) == 1:
                break
            nodes, level = upper, level + 1
        return self._write_header([(MSG_STAB, struct.pack('<QQ', upper[0][0], haddr))] + attrs), \
            upper[0][0], haddr
