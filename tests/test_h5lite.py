"""The HDF5 reader/writer used where h5py is absent (fdtdsarsim_b200.h5lite).

There is no libhdf5 in this image, so the format is pinned two ways:
(1) a file written by libhdf5 itself -- scipy's MAT 7.3 test file
(scipy/io/matlab/tests/data/testhdf5_7.4_GLNX86.mat, an HDF5 file behind a
512-byte user block) -- is read, and its datatype, dataspace and attribute
message bytes are compared with this writer's encodings; (2) a structure
walker written here from the HDF5 File Format Specification checks every
invariant libhdf5 enforces when it opens a file (signatures, versions,
message counts and alignment, B-tree key order and node sizes, local-heap
free-list terminator, global-heap collection layout, end-of-file address).
The walker is run on the libhdf5 file first, then on files this writer
produced."""
import os
import struct

import numpy as np
import pytest
import scipy

from fdtdsarsim_b200 import h5lite

LIBHDF5_FILE = os.path.join(os.path.dirname(scipy.__file__), 'io', 'matlab', 'tests', 'data',
                            'testhdf5_7.4_GLNX86.mat')
needs_libhdf5_file = pytest.mark.skipif(not os.path.isfile(LIBHDF5_FILE),
                                        reason="scipy's MAT 7.3 test file is not installed")


# ---------------------------------------------------------------------------
# a structure walker, written from the specification
# ---------------------------------------------------------------------------

class SpecWalker:
    def __init__(self, path):
        self.d = open(path, 'rb').read()
        self.sb = next(o for o in (0, 512, 1024, 2048) if self.d[o:o + 8] == h5lite.SIGNATURE)
        d, o = self.d, self.sb
        assert d[o + 8] == 0, 'superblock version 0'
        assert d[o + 13] == 8 and d[o + 14] == 8, 'offset / length sizes'
        self.leaf_k, self.node_k = struct.unpack_from('<HH', d, o + 16)
        self.base, free_space, self.eof, driver = struct.unpack_from('<QQQQ', d, o + 24)
        assert free_space == h5lite.UNDEF and driver == h5lite.UNDEF
        _, self.root, ctype, _, bt, hp = struct.unpack_from('<QQIIQQ', d, o + 56)
        assert ctype == 1, 'the root entry caches its symbol table'
        self.names = {}
        self.strings = []
        msgs = self.header(self.root)
        stab = [b for t, b in msgs if t == 0x11]
        assert stab and struct.unpack_from('<QQ', stab[0]) == (bt, hp)
        self.group('/', msgs)

    def at(self, addr):
        assert addr != h5lite.UNDEF and addr < self.eof
        return self.base + addr

    def header(self, addr):
        d = self.d
        ver, _, nmsgs, refs, size = struct.unpack_from('<BBHII', d, self.at(addr))
        assert ver == 1 and refs >= 1
        chunks, msgs = [(addr + 16, size)], []
        while chunks:
            caddr, csize = chunks.pop(0)
            p, end = self.at(caddr), self.at(caddr) + csize
            while p < end:
                t, sz = struct.unpack_from('<HH', d, p)
                assert sz % 8 == 0 and p + 8 + sz <= end, 'aligned message inside its chunk'
                body = d[p + 8:p + 8 + sz]
                if t == 0x10:
                    chunks.append(struct.unpack_from('<QQ', body))
                msgs.append((t, body))
                p += 8 + sz
            assert p == end
        assert len(msgs) == nmsgs, 'message count in the prefix'
        for t, body in msgs:
            if t == 0x0C:
                self.attribute(body)
        return msgs

    def attribute(self, body):
        ver, _, nlen, tlen, slen = struct.unpack_from('<BBHHH', body)
        assert ver == 1
        name_end = 8 + h5lite._pad8(nlen)
        assert body[8 + nlen - 1] == 0, 'name size counts the terminating null'
        tpos = name_end
        spos = tpos + h5lite._pad8(tlen)
        dpos = spos + h5lite._pad8(slen)
        dt, vlen, tend = h5lite.decode_dtype(body, tpos)
        assert tend - tpos == tlen, 'datatype size field'
        shape = h5lite.decode_space(body, spos)
        assert 8 + 8 * len(shape) == slen, 'dataspace size field'
        n = int(np.prod(shape))
        nbytes = n * (16 if vlen else dt.itemsize)
        assert len(body) == h5lite._pad8(dpos + nbytes)
        if vlen:
            for i in range(n):
                ln, coll, idx = struct.unpack_from('<IQI', body, dpos + 16 * i)
                self.strings.append(self.gheap_object(coll, idx)[:ln])

    def gheap_object(self, addr, idx):
        d, p0 = self.d, self.at(addr)
        assert d[p0:p0 + 4] == b'GCOL' and d[p0 + 4] == 1
        size = struct.unpack_from('<Q', d, p0 + 8)[0]
        assert size >= 4096
        p, found, seen = p0 + 16, None, []
        while p + 16 <= p0 + size:
            i, _, osize = struct.unpack_from('<HH4xQ', d, p)
            if i == 0:
                assert p + osize == p0 + size, 'free-space object runs to the end'
                break
            seen.append(i)
            if i == idx:
                found = d[p + 16:p + 16 + osize]
            p += 16 + h5lite._pad8(osize)
        assert seen == list(range(1, len(seen) + 1))
        assert found is not None
        return found

    def name(self, seg, off):
        end = seg.index(b'\0', off)
        return seg[off:end]

    def group(self, path, msgs):
        d = self.d
        bt, hp = struct.unpack_from('<QQ', [b for t, b in msgs if t == 0x11][0])
        p = self.at(hp)
        assert d[p:p + 4] == b'HEAP' and d[p + 4] == 0
        dsize, free, daddr = struct.unpack_from('<QQQ', d, p + 8)
        assert free == 1 or free < dsize, 'free list: 1 terminates it (UNDEF is rejected)'
        seg = d[self.at(daddr):self.at(daddr) + dsize]
        assert seg[0] == 0, 'offset 0 holds the empty name'
        entries = []
        self.btree(bt, seg, entries, b'', None)
        names = [self.name(seg, e[0]) for e in entries]
        assert names == sorted(names) and len(set(names)) == len(names)
        self.names[path] = [n.decode() for n in names]
        for (noff, oaddr, ctype, bt_c, hp_c), nm in zip(entries, names):
            msgs = self.header(oaddr)
            child = (path.rstrip('/') + '/' + nm.decode())
            kinds = {t for t, _ in msgs}
            if 0x11 in kinds:
                if ctype == 1:
                    assert struct.unpack_from('<QQ', [b for t, b in msgs if t == 0x11][0]) \
                        == (bt_c, hp_c)
                self.group(child, msgs)
            else:
                assert ctype == 0 and {0x01, 0x03, 0x08} <= kinds
                lay = [b for t, b in msgs if t == 0x08][0]
                if lay[0] == 3 and lay[1] == 1:
                    addr, size = struct.unpack_from('<QQ', lay, 2)
                    if size:
                        assert addr + size <= self.eof

    def btree(self, addr, seg, out, lo, hi):
        d, p = self.d, self.at(addr)
        node_size = 24 + 2 * self.node_k * 8 + (2 * self.node_k + 1) * 8
        assert d[p:p + 4] == b'TREE' and d[p + 4] == 0
        assert self.base + addr + node_size <= len(d), 'the whole node is in the file'
        level, n = d[p + 5], struct.unpack_from('<H', d, p + 6)[0]
        assert n <= 2 * self.node_k
        keys = [self.name(seg, struct.unpack_from('<Q', d, p + 24 + 16 * i)[0])
                for i in range(n + 1)]
        kids = [struct.unpack_from('<Q', d, p + 32 + 16 * i)[0] for i in range(n)]
        assert keys[1:] == sorted(keys[1:])
        for i, c in enumerate(kids):
            if level > 0:
                self.btree(c, seg, out, keys[i], keys[i + 1])
                continue
            q = self.at(c)
            assert d[q:q + 4] == b'SNOD' and d[q + 4] == 1
            k = struct.unpack_from('<H', d, q + 6)[0]
            assert 0 < k <= 2 * self.leaf_k
            for j in range(k):
                e = struct.unpack_from('<QQIIQQ', d, q + 8 + 40 * j)
                nm = self.name(seg, e[0])
                assert (i == 0 or keys[i] < nm) and nm <= keys[i + 1], 'B-tree keys bound the names'
                out.append((e[0], e[1], e[2], e[4], e[5]))


# ---------------------------------------------------------------------------
# the libhdf5 file
# ---------------------------------------------------------------------------

@needs_libhdf5_file
def test_reads_a_libhdf5_file():
    with h5lite.File(LIBHDF5_FILE, 'r') as f:
        assert f.keys() == ['testdouble']
        ds = f['testdouble']
        assert ds.shape == (9, 1) and ds.dtype == np.float64
        np.testing.assert_array_equal(ds[()].ravel(), np.arange(9) * np.pi / 4)
        np.testing.assert_array_equal(ds[2:4, 0], np.arange(2, 4) * np.pi / 4)
        assert ds.attrs['MATLAB_class'] == b'double'
    w = SpecWalker(LIBHDF5_FILE)
    assert w.base == 512 and w.names == {'/': ['testdouble']}


@needs_libhdf5_file
def test_encodings_match_libhdf5_bytes():
    """This writer's float64 datatype, dataspaces and attribute message are
    byte-identical to the ones libhdf5 wrote (the attribute's string type
    differs only in its pad bits: h5py writes numpy bytes NULLPAD, MATLAB
    NULLTERM)."""
    with h5lite.File(LIBHDF5_FILE, 'r') as f:
        (noff, oaddr), = f._walk(struct.unpack_from('<Q', [
            b for t, b in f._messages(SpecWalker(LIBHDF5_FILE).root) if t == 0x11][0])[0])
        msgs = f._messages(oaddr)
    by_type = {}
    for t, b in msgs:
        by_type.setdefault(t, []).append(b)
    assert by_type[0x03][0][:20] == h5lite.encode_dtype('<f8')
    assert by_type[0x01][0] == h5lite.encode_space((9, 1))
    theirs = bytearray(by_type[0x0C][0])
    heap = h5lite._GlobalHeap()
    ours = bytearray(h5lite._padded(
        h5lite._AttrPlan('MATLAB_class', np.bytes_(b'double'), heap).encode(heap)))
    assert len(ours) == len(theirs)
    pad_bits = 8 + 16 + 1                                # the string type's class bits
    assert (ours[pad_bits], theirs[pad_bits]) == (1, 0)
    ours[pad_bits] = theirs[pad_bits]
    assert ours == theirs
    assert h5lite.encode_space(()) == bytes(theirs[8 + 16 + 8:8 + 16 + 16])


# ---------------------------------------------------------------------------
# files this writer produced
# ---------------------------------------------------------------------------

ATTRS = {'int': 5, 'float': 0.021, 'true': True, 'false': np.bool_(False), 'str': 'VV',
         'empty_str': '', 'unicode': 'Ångström', 'ints': [0, 1, 2], 'floats': np.linspace(-80, 80, 161),
         'strs': ['a', 'bé', ''], 'bytes': b'xy', 'complex': 1 + 2j, 'f32': np.float32(1.5),
         'u8': np.uint8(7), 'matrix': np.arange(6, dtype=np.int32).reshape(2, 3)}


def write_sample(path):
    with h5lite.File(path, 'w') as f:
        f.attrs['incident_complete'] = True
        g = f.create_group('phasors')
        for k, v in ATTRS.items():
            g.attrs[k] = v
        rng = np.random.default_rng(3)
        for i in range(28):                                  # the result file's 28 planes
            g.create_dataset(f'p{i:02d}', data=(rng.standard_normal((7, 9))
                                                + 1j * rng.standard_normal((7, 9))).astype(np.complex64))
        g.create_dataset('c128', data=np.arange(4) * (1 - 1j))
        many = f.create_group('nested/deeper/many')
        for i in range(300):                                 # two B-tree levels
            many.create_group(f'g{i:03d}').attrs['i'] = i
        ex = f.create_dataset('ex', shape=(5, 4, 3), dtype='f4')
        for t in range(5):
            ex[t] = t + 0.5
        f.create_dataset('scalar', data=np.float64(2.5))
        f.create_dataset('empty', shape=(0, 3), dtype='f8')
        f.create_dataset('flags', data=np.array([True, False, True]))
        f.create_dataset('be', data=np.arange(3, dtype='>i4'))
        f.create_group('material_metadata')


def test_roundtrip_types_and_structure(tmp_path):
    path = str(tmp_path / 'sample.hdf5')
    write_sample(path)
    w = SpecWalker(path)
    assert w.eof == os.path.getsize(path) and w.base == 0
    assert w.names['/'] == ['be', 'empty', 'ex', 'flags', 'material_metadata', 'nested',
                            'phasors', 'scalar']
    assert len(w.names['/nested/deeper/many']) == 300
    assert set(w.strings) >= {b'VV', b'', 'Ångström'.encode(), b'b\xc3\xa9'}
    with h5lite.File(path, 'r') as f:
        assert bool(f.attrs['incident_complete']) is True
        a = f['phasors'].attrs
        for k, v in ATTRS.items():
            got = a[k]
            if isinstance(v, str):
                assert isinstance(got, str) and got == v
            elif k == 'strs':
                assert list(got) == v
            else:
                np.testing.assert_array_equal(got, np.asarray(v))
                assert np.asarray(got).dtype == np.asarray(v).dtype
        rng = np.random.default_rng(3)
        for i in range(28):
            want = (rng.standard_normal((7, 9)) + 1j * rng.standard_normal((7, 9))).astype(np.complex64)
            got = f[f'phasors/p{i:02d}'][()]
            assert got.dtype == np.complex64
            np.testing.assert_array_equal(got, want)
        np.testing.assert_array_equal(f['phasors']['c128'][:], np.arange(4) * (1 - 1j))
        assert f['nested/deeper/many/g123'].attrs['i'] == 123
        ex = f['ex']
        assert ex.shape == (5, 4, 3) and ex.dtype == np.float32 and len(ex) == 5
        np.testing.assert_array_equal(np.asarray(ex)[:, 0, 0], np.arange(5) + 0.5)
        np.testing.assert_array_equal(ex[3, 1], [3.5] * 3)
        assert f['scalar'][()] == 2.5
        assert f['empty'][()].shape == (0, 3)
        np.testing.assert_array_equal(f['flags'][()], [True, False, True])
        assert f['be'].dtype == np.dtype('>i4')
        np.testing.assert_array_equal(f['be'][()], [0, 1, 2])
        assert len(f['material_metadata']) == 0 and len(f['material_metadata'].attrs) == 0
        assert 'phasors/p05' in f and 'phasors/nope' not in f


def test_read_write_mode_keeps_and_extends(tmp_path):
    path = str(tmp_path / 'r.hdf5')
    write_sample(path)
    with h5lite.File(path, 'r+') as f:
        ff = f.create_group('farfield')
        ff.create_dataset('e_phi', data=np.ones(161, np.complex128))
        ff.attrs['farfields_computed'] = True
        f['phasors'].attrs['int'] = 7
        f['ex'][2, 3, 1] = -1.0
        del f['phasors'].attrs['bytes']
    SpecWalker(path)
    with h5lite.File(path, 'a') as f:
        f['farfield'].attrs['radius'] = 2.0e3
    w = SpecWalker(path)
    assert 'farfield' in w.names['/'] and w.eof == os.path.getsize(path)
    with h5lite.File(path, 'r') as f:
        assert f['phasors'].attrs['int'] == 7 and 'bytes' not in f['phasors'].attrs
        assert f['farfield'].attrs['radius'] == 2.0e3 and f['farfield'].attrs['farfields_computed']
        assert f['ex'][2, 3, 1] == -1.0 and f['ex'][2, 3, 0] == 2.5
        np.testing.assert_array_equal(f['farfield/e_phi'][()], np.ones(161))
        assert f['phasors'].attrs['unicode'] == 'Ångström'


@needs_libhdf5_file
def test_read_write_mode_on_a_libhdf5_file(tmp_path):
    """A file libhdf5 wrote (with a user block) can be extended; its data
    and the user block stay where they were."""
    path = str(tmp_path / 'm.mat')
    with open(LIBHDF5_FILE, 'rb') as src, open(path, 'wb') as dst:
        dst.write(src.read())
    with h5lite.File(path, 'r+') as f:
        f.create_dataset('added', data=np.arange(3.0))
    w = SpecWalker(path)
    assert w.base == 512 and w.names['/'] == ['added', 'testdouble']
    with open(LIBHDF5_FILE, 'rb') as fh:
        assert open(path, 'rb').read(512) == fh.read(512)
    with h5lite.File(path, 'r') as f:
        np.testing.assert_array_equal(f['testdouble'][()].ravel(), np.arange(9) * np.pi / 4)
        assert f['testdouble'].attrs['MATLAB_class'] == b'double'
        np.testing.assert_array_equal(f['added'][()], np.arange(3.0))


def test_errors_follow_h5py(tmp_path):
    path = str(tmp_path / 'e.hdf5')
    with pytest.raises(FileNotFoundError):
        h5lite.File(path, 'r')
    with h5lite.File(path, 'w') as f:
        f.create_group('g')
        with pytest.raises(ValueError):
            f.create_group('g')
        with pytest.raises(TypeError):
            f.attrs['none'] = None
        with pytest.raises(TypeError):
            f.attrs['obj'] = [object()]
        with pytest.raises(KeyError):
            f['missing']
        with pytest.raises(KeyError):
            f.attrs['missing']
    with pytest.raises(FileExistsError):
        h5lite.File(path, 'w-')
    with h5lite.File(path, 'r') as f:
        with pytest.raises(ValueError):
            f.create_group('h')
        with pytest.raises(ValueError):
            f.attrs['x'] = 1
    with pytest.raises(ValueError):
        h5lite.File(path, 'q')
    bad = tmp_path / 'bad.hdf5'
    bad.write_bytes(b'not an hdf5 file' * 10)
    with pytest.raises(OSError):
        h5lite.File(str(bad), 'r')


def test_result_file_layout_through_resultsio(tmp_path):
    """The result file of MainSimGpu.save_results (cpu/main_sim.py:213-257
    layout: /phasors with 24 planes, 4 incident phasors and n*_phasor
    attributes, /parameters with one attribute per dataclass field,
    /material_metadata) is a valid HDF5 file that reads back."""
    import dataclasses
    from fdtdsarsim_b200 import resultsio
    from helpers import make_params
    pc = make_params(25, 23, 27, 14, 10, 6)
    path = str(tmp_path / 'm.hdf5')
    planes = ['ex_ph_d', 'ey_ph_d', 'hx_ph_d', 'hy_ph_d', 'ex_ph_u', 'ey_ph_u', 'hx_ph_u', 'hy_ph_u',
              'ey_ph_l', 'ez_ph_l', 'hy_ph_l', 'hz_ph_l', 'ey_ph_r', 'ez_ph_r', 'hy_ph_r', 'hz_ph_r',
              'ex_ph_f', 'ez_ph_f', 'hx_ph_f', 'hz_ph_f', 'ex_ph_b', 'ez_ph_b', 'hx_ph_b', 'hz_ph_b']
    with resultsio.File(path, 'w') as out:
        pg, parg, mg = (out.create_group(n) for n in ('phasors', 'parameters', 'material_metadata'))
        pg.attrs['nx_phasor'], pg.attrs['ny_phasor'], pg.attrs['nz_phasor'] = 5, 3, 7
        for n in planes + [f'{c}_inc_phasor' for c in ('ex', 'ey', 'hx', 'hy')]:
            pg.create_dataset(n, data=np.full((3, 5), 1 + 1j, np.complex64))
        for grp in dataclasses.fields(pc):
            obj = getattr(pc, grp.name)
            for fld in dataclasses.fields(obj):
                parg.attrs[fld.name] = getattr(obj, fld.name)
        mg.attrs['moisture'] = 0.2
        mg.attrs['epsilon_r'] = np.array([5.0, 8.0])
    w = SpecWalker(path)
    assert len(w.names['/phasors']) == 28
    with resultsio.File(path, 'r') as f:
        assert f['parameters'].attrs['cell_size'] == pc.geom_params.cell_size
        assert f['parameters'].attrs['polarization'] == pc.inc_beam_params.polarization
        assert f['parameters'].attrs['datatype'] == pc.processing_params.datatype
        assert f['phasors'].attrs['nz_phasor'] == 7
        np.testing.assert_array_equal(f['material_metadata'].attrs['epsilon_r'], [5.0, 8.0])
        assert f['phasors/hz_ph_b'].dtype == np.complex64


def test_large_writes_in_pieces_and_dataset_copies(tmp_path, monkeypatch):
    """Raw data longer than one write piece is written in pieces; a dataset
    created from another file's dataset (the reference copies the incident
    phasors that way, cpu/main_sim.py:239-246) copies its values."""
    monkeypatch.setattr(h5lite, 'WRITE_CHUNK', 1000)
    src, dst = str(tmp_path / 'src.hdf5'), str(tmp_path / 'dst.hdf5')
    data = np.random.default_rng(5).standard_normal((17, 33, 7)).astype(np.float32)
    with h5lite.File(src, 'w') as f:
        f.create_group('phasors').create_dataset('ex_inc_phasor', data=data[0] + 1j * data[1])
        f.create_dataset('ex', data=data)
    with h5lite.File(src, 'r') as s, h5lite.File(dst, 'w') as d:
        d.create_group('phasors').create_dataset('ex_inc_phasor', data=s['phasors']['ex_inc_phasor'])
        np.testing.assert_array_equal(s['ex'][()], data)
    with h5lite.File(dst, 'r') as d:
        np.testing.assert_array_equal(d['phasors/ex_inc_phasor'][()], data[0] + 1j * data[1])
    SpecWalker(dst)


def test_writes_survive_optimised_python(tmp_path):
    """Writing does not depend on assert statements (python -O)."""
    import subprocess
    import sys
    path = str(tmp_path / 'o.hdf5')
    code = ('import sys, numpy as np; sys.path.insert(0, sys.argv[2]); '
            'from fdtdsarsim_b200 import h5lite; f = h5lite.File(sys.argv[1], "w"); '
            'g = f.create_group("g"); g.create_dataset("d", data=np.arange(5.0)); f.close()')
    pkg = os.path.dirname(os.path.dirname(h5lite.__file__))
    subprocess.run([sys.executable, '-O', '-c', code, path, pkg], check=True)
    SpecWalker(path)
    with h5lite.File(path, 'r') as f:
        np.testing.assert_array_equal(f['g/d'][()], np.arange(5.0))


def test_reads_object_headers_continued_in_another_chunk(tmp_path):
    """libhdf5 continues a version-1 object header in further chunks when
    its messages outgrow the first one (h5py does this for the reference's
    /parameters group of ~35 attributes). A written header is split here
    into a first chunk that ends with a continuation message (0x10) and a
    second chunk at the end of the file; both readers follow it."""
    path = str(tmp_path / 'cont.hdf5')
    with h5lite.File(path, 'w') as f:
        g = f.create_group('parameters')
        for k in range(12):
            g.attrs[f'a{k:02d}'] = float(k)
        g.attrs['polarization'] = 'VV'
    w = SpecWalker(path)
    raw = bytearray(open(path, 'rb').read())
    # the group's header: the root SNOD's only entry
    with h5lite.File(path, 'r') as f:
        stab = [b for t, b in f._messages(w.root) if t == 0x11][0]
        ((_, addr),) = f._walk(struct.unpack_from('<Q', stab)[0])
    ver, _, nmsgs, refs, size = struct.unpack_from('<BBHII', raw, addr)
    msgs, p = [], addr + 16
    while p < addr + 16 + size:
        t, sz = struct.unpack_from('<HH', raw, p)
        msgs.append(bytes(raw[p:p + 8 + sz]))
        p += 8 + sz
    keep, move = msgs[:5], msgs[5:]
    second = b''.join(move)
    caddr = h5lite._pad8(len(raw))
    cont = struct.pack('<HHB3x', 0x10, 16, 0) + struct.pack('<QQ', caddr, len(second))
    first = b''.join(keep) + cont
    gap = size - len(first)
    assert gap >= 8
    first += struct.pack('<HHB3x', 0, gap - 8, 0) + b'\0' * (gap - 8)    # NIL message
    raw[addr + 16:addr + 16 + size] = first
    struct.pack_into('<H', raw, addr + 2, len(keep) + 1 + 1 + len(move))
    raw += b'\0' * (caddr - len(raw)) + second
    struct.pack_into('<Q', raw, w.sb + 40, len(raw))                    # end-of-file address
    open(path, 'wb').write(bytes(raw))
    SpecWalker(path)
    with h5lite.File(path, 'r') as f:
        a = f['parameters'].attrs
        assert [a[f'a{k:02d}'] for k in range(12)] == [float(k) for k in range(12)]
        assert a['polarization'] == 'VV'


def test_new_file_appears_only_when_complete(tmp_path):
    """A file in 'w' mode is written beside its path and renamed onto it on
    close: while it is being written (or after a writer died) nothing
    partial sits at the path that skip-if-exists checks."""
    path = str(tmp_path / 'm.hdf5')
    f = h5lite.File(path, 'w')
    ds = f.create_dataset('ex', shape=(4, 5), dtype='f4')
    ds[1] = 2.0
    np.testing.assert_array_equal(ds[1], [2.0] * 5)
    assert not os.path.exists(path) and os.path.exists(path + '.partial')
    f.close()
    assert os.path.exists(path) and not os.path.exists(path + '.partial')
    SpecWalker(path)
    with h5lite.File(path, 'r') as g:
        np.testing.assert_array_equal(g['ex'][()][1], [2.0] * 5)
    # an older file at the path stays readable until the new one replaces it
    f = h5lite.File(path, 'w')
    f.create_group('other')
    with h5lite.File(path, 'r') as g:
        assert 'ex' in g
    f.close()
    with h5lite.File(path, 'r') as g:
        assert g.keys() == ['other']
