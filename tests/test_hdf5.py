"""The HDF5 reader and writer behind the output and restart files: a file
written by the HDF5 library itself, round trips, and the structural rules a
library enforces when it opens a file."""
import os
import struct
import zlib

import numpy as np
import pytest

from gospl_b200 import hdf5


def _library_file():
    """An HDF5 file written by the HDF5 library (MATLAB 7.4 v7.3 test data
    shipped with scipy): dataset ``testdouble`` = pi/4 * [0..8]."""
    import scipy.io.matlab as mm
    p = os.path.join(os.path.dirname(mm.__file__), "tests", "data", "testhdf5_7.4_GLNX86.mat")
    return p if os.path.exists(p) else None


def test_reader_reads_a_file_written_by_the_hdf5_library():
    p = _library_file()
    if p is None:
        pytest.skip("no HDF5 library file in this image")
    d = hdf5.read(p)
    assert d["testdouble"].shape == (9, 1) and d["testdouble"].dtype == np.float64
    assert np.array_equal(d["testdouble"][:, 0], np.pi / 4 * np.arange(9))


def lint(path):
    """Check the invariants an HDF5 library enforces when it opens a version 0
    file: end of file, object header message counts and alignment, the local
    heap's free list, sorted symbol-table nodes and their B-tree keys, chunk
    index keys and bounds, and that no two structures overlap.  Returns the
    dataset names."""
    b = open(path, "rb").read()
    assert b[:8] == hdf5.SIGNATURE
    assert b[8:16] == bytes([0, 0, 0, 0, 0, 8, 8, 0])
    leaf_k, group_k, flags = struct.unpack_from("<HHI", b, 16)
    base, free, eof, drv = struct.unpack_from("<QQQQ", b, 24)
    assert (base, free, drv) == (0, hdf5.UNDEF, hdf5.UNDEF) and eof == len(b)
    _, root, ctype = struct.unpack_from("<QQI", b, 56)
    cbt, cheap = struct.unpack_from("<QQ", b, 80)
    assert ctype == 1
    spans = [(0, 96)]

    def ohdr(a):
        ver, _, nmsg, rc, size = struct.unpack_from("<BBHII", b, a)
        assert ver == 1 and rc == 1 and size % 8 == 0
        p, msgs = a + 16, []
        while p < a + 16 + size:
            t, ms, fl = struct.unpack_from("<HHB", b, p)
            assert ms % 8 == 0
            msgs.append((t, b[p + 8:p + 8 + ms]))
            p += 8 + ms
        assert p == a + 16 + size and len(msgs) == nmsg
        spans.append((a, 16 + size))
        return msgs

    stab = [d for t, d in ohdr(root) if t == hdf5.MSG_STAB]
    assert stab and struct.unpack_from("<QQ", stab[0]) == (cbt, cheap)
    sig, ver, dsize, fhead, daddr = struct.unpack_from("<4sB3xQQQ", b, cheap)
    assert sig == b"HEAP" and ver == 0 and dsize % 8 == 0
    spans += [(cheap, 32), (daddr, dsize)]
    assert fhead < dsize
    nxt, fsize = struct.unpack_from("<QQ", b, daddr + fhead)
    assert nxt == hdf5.FREE_NULL and fsize >= 16 and fhead + fsize <= dsize
    heap = b[daddr:daddr + dsize]

    def name(off):
        return heap[off:heap.index(b"\0", off)]

    sig, typ, lev, used = struct.unpack_from("<4sBBH", b, cbt)
    assert sig == b"TREE" and typ == 0 and lev == 0 and 1 <= used <= 2 * group_k
    spans.append((cbt, 24 + 2 * group_k * 8 + (2 * group_k + 1) * 8))
    keys = [struct.unpack_from("<Q", b, cbt + 24 + 16 * i)[0] for i in range(used + 1)]
    kids = [struct.unpack_from("<Q", b, cbt + 32 + 16 * i)[0] for i in range(used)]
    assert keys[0] == 0 and name(0) == b""
    allnames, objs = [], {}
    for i, sn in enumerate(kids):
        sig, ver, _, nsym = struct.unpack_from("<4sBBH", b, sn)
        assert sig == b"SNOD" and ver == 1 and 1 <= nsym <= 2 * leaf_k
        spans.append((sn, 8 + 2 * leaf_k * 40))
        names = []
        for j in range(nsym):
            noff, oh, ct = struct.unpack_from("<QQI", b, sn + 8 + 40 * j)
            assert ct == 0
            names.append(name(noff))
            objs[name(noff).decode()] = oh
        assert names == sorted(names) and name(keys[i + 1]) == names[-1]
        allnames += names
    assert allnames == sorted(allnames) and len(set(allnames)) == len(allnames)
    for nm, oh in objs.items():
        msgs = dict(ohdr(oh))
        assert {hdf5.MSG_SPACE, hdf5.MSG_DTYPE, hdf5.MSG_FILL, hdf5.MSG_LAYOUT} <= set(msgs)
        sp = msgs[hdf5.MSG_SPACE]
        rank = sp[1]
        shape = struct.unpack_from("<%dQ" % rank, sp, 8)
        es = struct.unpack_from("<I", msgs[hdf5.MSG_DTYPE], 4)[0]
        lay = msgs[hdf5.MSG_LAYOUT]
        assert lay[0] == 3
        if lay[1] == 1:
            addr, size = struct.unpack_from("<QQ", lay, 2)
            assert size == es * int(np.prod(shape)) and addr + size <= eof
            spans.append((addr, size))
            continue
        assert lay[1] == 2 and lay[2] == rank + 1 and hdf5.MSG_FILTER in msgs
        bt = struct.unpack_from("<Q", lay, 3)[0]
        chunk = struct.unpack_from("<%dI" % (rank + 1), lay, 11)
        assert chunk[-1] == es and all(c <= s for c, s in zip(chunk, shape))
        ksize = 8 + 8 * (rank + 1)
        nsize = 24 + 64 * 8 + 65 * ksize
        starts = []

        def walk(a):
            sig, typ, lev, used = struct.unpack_from("<4sBBH", b, a)
            assert sig == b"TREE" and typ == 1 and 1 <= used <= 64
            spans.append((a, nsize))
            ks = [struct.unpack_from("<II%dQ" % (rank + 1), b, a + 24 + i * (ksize + 8)) for i in range(used + 1)]
            for i in range(used):
                child = struct.unpack_from("<Q", b, a + 24 + i * (ksize + 8) + ksize)[0]
                assert ks[i][2] < ks[i + 1][2]       # first coordinate ascends
                if lev:
                    walk(child)
                else:
                    nb = ks[i][0]
                    spans.append((child, nb))
                    raw = zlib.decompress(b[child:child + nb])
                    assert len(raw) == es * int(np.prod(chunk[:-1]))
                    starts.append(ks[i][2])

        walk(bt)
        assert starts == list(range(0, shape[0], chunk[0]))
    spans.sort()
    for (a0, n0), (a1, _) in zip(spans, spans[1:]):
        assert a0 + n0 <= a1, "overlapping structures at %d and %d" % (a0, a1)
    assert spans[-1][0] + spans[-1][1] <= eof
    return sorted(objs)


@pytest.mark.parametrize("comp", [None, 0, 4, 9])
def test_writer_round_trip_and_structure(tmp_path, comp):
    rng = np.random.default_rng(3)
    ds = [("elev", rng.standard_normal((1000, 1)).astype(np.float32)),
          ("cells", rng.integers(1, 1000, (1999, 3)).astype(np.int32)),
          ("coords", rng.standard_normal((1000, 3)).astype(np.float32)),
          ("x64", rng.standard_normal(77)), ("u8", rng.integers(0, 255, 13).astype(np.uint8))]
    ds += [("f%02d" % i, rng.standard_normal((50, 1)).astype(np.float32)) for i in range(12)]   # > 8 names
    p = str(tmp_path / "t.h5")
    hdf5.write(p, ds, compression=comp)
    assert lint(p) == sorted(n for n, _ in ds)
    r = hdf5.read(p)
    for n, a in ds:
        assert r[n].dtype == a.dtype and r[n].shape == a.shape and np.array_equal(r[n], a), n
    assert hdf5.contents(p) == sorted(n for n, _ in ds)


def test_writer_two_level_chunk_index(tmp_path, monkeypatch):
    monkeypatch.setattr(hdf5, "CHUNK_BYTES", 64)          # 16 rows a chunk: 313 chunks
    a = np.random.default_rng(4).standard_normal((5000, 1)).astype(np.float32)
    p = str(tmp_path / "big.h5")
    hdf5.write(p, [("a", a)], compression=1)
    lint(p)
    assert np.array_equal(hdf5.read(p)["a"], a)


def test_reader_rejects_missing_datasets(tmp_path):
    p = str(tmp_path / "t.h5")
    hdf5.write(p, [("elev", np.zeros((3, 1), np.float32))])
    with pytest.raises(KeyError):
        hdf5.read(p, ["elev", "erodep"])
    with pytest.raises(ValueError):
        hdf5.write(p, [("a", np.zeros(2)), ("a", np.zeros(2))])
