"""HDF5 files for goSPL's outputs and restarts, without an HDF5 library.

goSPL writes each output step as ``h5/gospl.<step>.p<rank>.h5`` and the mesh
as ``h5/topology.p<rank>.h5`` through h5py (``gospl/tools/outmesh.py:228-486``)
and reads a step back to restart (``outmesh.py:505-620``).  This module writes
and reads the same files with the original ("version 0") HDF5 structures, the
ones h5py produces with its default ``libver="earliest"``:

* superblock version 0 (K = 4 symbol-table leaves, K = 16 group nodes, K = 32
  chunk-index nodes), base address 0;
* one root group held as a symbol table: object header version 1 with a
  symbol-table message, a version 1 B-tree of type 0, symbol-table nodes and
  a local heap of names;
* datasets with object header version 1: dataspace (version 1), datatype
  (IEEE float or two's-complement integer, little-endian), fill value
  (version 2, undefined), data layout version 3 either contiguous or chunked;
  chunked datasets carry a filter pipeline (version 1) with deflate, their
  chunks indexed by a version 1 B-tree of type 1.

``write`` lays out a whole file in one pass: chunks are compressed first, in a
thread pool (``zlib`` releases the interpreter lock while it deflates), then
the metadata and the data are written in address order.  ``read`` walks the
same structures; it also reads files written by the HDF5 library in this
format family (old-style groups, continuation messages, layout versions 1-3,
deflate and shuffle filters) and raises on anything else.
"""
import os
import struct
import zlib
from concurrent.futures import ThreadPoolExecutor

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF
FREE_NULL = 1          # end of a local heap's free list
LEAF_K = 4             # symbol-table node holds 2 * LEAF_K entries
GROUP_K = 16           # group B-tree node holds 2 * GROUP_K children
CHUNK_K = 32           # chunk B-tree node holds 2 * CHUNK_K children
CHUNK_BYTES = 1 << 20  # target uncompressed chunk size

MSG_NIL, MSG_SPACE, MSG_DTYPE, MSG_FILL_OLD, MSG_FILL = 0x0, 0x1, 0x3, 0x4, 0x5
MSG_LAYOUT, MSG_FILTER, MSG_CONT, MSG_STAB = 0x8, 0xB, 0x10, 0x11
FILTER_DEFLATE, FILTER_SHUFFLE = 1, 2


def _pad8(n):
    return (n + 7) & ~7


# ---------------------------------------------------------------- messages
def _dtype_message(dt):
    """Datatype message (class 0 fixed-point or class 1 floating point,
    version 1, little-endian)."""
    dt = np.dtype(dt)
    size = dt.itemsize
    if dt.kind == "f":
        if size == 4:
            sign, eloc, esize, msize, bias = 31, 23, 8, 23, 127
        elif size == 8:
            sign, eloc, esize, msize, bias = 63, 52, 11, 52, 1023
        else:
            raise TypeError("HDF5 output supports float32 and float64, not %s" % dt)
        # bit field: mantissa normalisation 2 (implied msb) in bits 4-5,
        # sign bit location in the second byte
        return (struct.pack("<B3BI", 0x11, 0x20, sign, 0, size)
                + struct.pack("<HHBBBBI", 0, 8 * size, eloc, esize, 0, msize, bias))
    if dt.kind in "iu" and size in (1, 2, 4, 8):
        return struct.pack("<B3BI", 0x10, 0x08 if dt.kind == "i" else 0x00, 0, 0, size) + struct.pack(
            "<HH", 0, 8 * size)
    raise TypeError("HDF5 output supports integer and float arrays, not %s" % dt)


def _space_message(shape):
    return struct.pack("<BBBB4x", 1, len(shape), 0, 0) + b"".join(struct.pack("<Q", d) for d in shape)


def _fill_message(alloc_time):
    # version 2: allocation time, write time "if set", no fill value defined
    return struct.pack("<BBBB", 2, alloc_time, 2, 0)


def _layout_contiguous(addr, size):
    return struct.pack("<BBQQ", 3, 1, addr, size)


def _layout_chunked(btree, chunk, itemsize):
    return struct.pack("<BBBQ", 3, 2, len(chunk) + 1, btree) + b"".join(
        struct.pack("<I", c) for c in tuple(chunk) + (itemsize,))


def _filter_deflate(level):
    # version 1 pipeline, one filter: id 1 (deflate), no name, mandatory,
    # one client value (the level) padded to an even count
    return struct.pack("<BB6x", 1, 1) + struct.pack("<HHHHI4x", FILTER_DEFLATE, 0, 0, 1, level)


def _object_header(messages):
    """Version 1 object header: 16-byte prefix, then messages aligned to 8."""
    body = b""
    for mtype, flags, data in messages:
        size = _pad8(len(data))
        body += struct.pack("<HHB3x", mtype, size, flags) + data + b"\0" * (size - len(data))
    return struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(body)) + body


# ---------------------------------------------------------------- writer
class _Dataset:
    def __init__(self, name, arr, level):
        a = np.asarray(arr)
        if a.dtype.byteorder == ">":
            a = a.astype(a.dtype.newbyteorder("<"))
        self.a = np.ascontiguousarray(a)
        if self.a.ndim == 0:
            self.a = self.a.reshape(1)
        self.name = name
        self.level = level
        self.dtmsg = _dtype_message(self.a.dtype)
        self.chunks = None
        if level is not None and self.a.size > 0:
            rowbytes = max(1, self.a.itemsize * int(np.prod(self.a.shape[1:], dtype=np.int64)))
            rows = int(max(1, min(self.a.shape[0], CHUNK_BYTES // rowbytes)))
            self.chunk = (rows,) + tuple(self.a.shape[1:])
            self.starts = list(range(0, self.a.shape[0], rows))

    def chunk_bytes(self, i):
        r0 = self.starts[i]
        rows = self.chunk[0]
        part = self.a[r0:r0 + rows]
        if part.shape[0] < rows:   # edge chunks are stored at full size
            full = np.zeros(self.chunk, self.a.dtype)
            full[:part.shape[0]] = part
            part = full
        return zlib.compress(memoryview(np.ascontiguousarray(part)).cast("B"), self.level)

    def header(self, data_addr):
        alloc = 1 if self.chunks is None else 3
        msgs = [(MSG_SPACE, 0, _space_message(self.a.shape)), (MSG_DTYPE, 1, self.dtmsg),
                (MSG_FILL, 1, _fill_message(alloc))]
        if self.chunks is None:
            msgs.append((MSG_LAYOUT, 0, _layout_contiguous(data_addr, self.a.nbytes)))
        else:
            msgs.append((MSG_FILTER, 1, _filter_deflate(self.level)))
            msgs.append((MSG_LAYOUT, 0, _layout_chunked(data_addr, self.chunk, self.a.itemsize)))
        return _object_header(msgs)


def _chunk_btree_nodes(ds, chunk_addrs, base):
    """Version 1 B-tree (type 1) over the dataset's chunks, leaves first; returns
    (root address, [(address, bytes)])."""
    rank = ds.a.ndim
    ksize = 8 + 8 * (rank + 1)
    nsize = 24 + 2 * CHUNK_K * 8 + (2 * CHUNK_K + 1) * ksize

    def key(nbytes, start_row):
        return struct.pack("<II", nbytes, 0) + struct.pack("<Q", start_row) + b"\0" * (8 * rank)

    last = ds.starts[-1]
    # right key of the last chunk: one chunk past it in every dimension
    end_key = struct.pack("<II", 0, 0) + b"".join(
        struct.pack("<Q", v) for v in (last + ds.chunk[0],) + tuple(ds.chunk[1:]) + (0,))
    entries = [(key(nb, s), addr) for s, (addr, nb) in zip(ds.starts, chunk_addrs)]
    nodes = []
    level = 0
    addr = base
    while True:
        groups = [entries[i:i + 2 * CHUNK_K] for i in range(0, len(entries), 2 * CHUNK_K)]
        nxt = []
        for g_i, g in enumerate(groups):
            right = groups[g_i + 1][0][0] if g_i + 1 < len(groups) else end_key
            body = struct.pack("<4sBBHQQ", b"TREE", 1, level, len(g), UNDEF, UNDEF)
            for k, child in g:
                body += k + struct.pack("<Q", child)
            body += right
            body += b"\0" * (nsize - len(body))
            nodes.append((addr, body))
            nxt.append((g[0][0], addr))
            addr += nsize
        if len(nxt) == 1:
            return nxt[0][1], nodes
        entries = nxt
        level += 1


def write(path, datasets, compression=4, threads=None):
    """Write ``datasets`` (an iterable of (name, array)) as the root group of
    a new HDF5 file at ``path``.  ``compression`` is a deflate level 0-9
    (chunked datasets, like h5py's ``compression="gzip"``) or None
    (contiguous, uncompressed)."""
    items = [_Dataset(str(name), arr, compression) for name, arr in datasets]
    names = [d.name for d in items]
    if len(set(names)) != len(names):
        raise ValueError("duplicate dataset names")
    for nm in names:
        if not nm or "/" in nm or "\0" in nm:
            raise ValueError("bad dataset name %r" % nm)
    items.sort(key=lambda d: d.name.encode())

    # compress every chunk in parallel
    jobs = [(d, i) for d in items if d.level is not None and d.a.size > 0 for i in range(len(d.starts))]
    if jobs:
        nthreads = threads or min(len(jobs), os.cpu_count() or 1, 32)
        if nthreads > 1:
            with ThreadPoolExecutor(nthreads) as ex:
                blobs = list(ex.map(lambda j: j[0].chunk_bytes(j[1]), jobs))
        else:
            blobs = [d.chunk_bytes(i) for d, i in jobs]
        k = 0
        for d in items:
            if d.level is not None and d.a.size > 0:
                d.chunks = blobs[k:k + len(d.starts)]
                k += len(d.starts)

    # --- root group metadata
    heap = bytearray(8)                  # offset 0: the empty name
    name_off = {}
    for d in items:
        name_off[d.name] = len(heap)
        nb = d.name.encode() + b"\0"
        heap += nb + b"\0" * (_pad8(len(nb)) - len(nb))
    free_off = len(heap)
    heap += struct.pack("<QQ", FREE_NULL, 16)   # one free block, end of the list
    heap_size = len(heap)
    snods = [items[i:i + 2 * LEAF_K] for i in range(0, len(items), 2 * LEAF_K)]
    if len(snods) > 2 * GROUP_K:
        raise ValueError("too many datasets in one file (%d)" % len(items))
    snod_size = 8 + 2 * LEAF_K * 40
    gtree_size = 24 + 2 * GROUP_K * 8 + (2 * GROUP_K + 1) * 8

    root_oh_size = len(_object_header([(MSG_STAB, 0, b"\0" * 16)]))
    a_root = 96
    a_heap = a_root + root_oh_size
    a_heapdata = a_heap + 32
    a_gtree = a_heapdata + heap_size
    a_snod = a_gtree + gtree_size
    addr = a_snod + snod_size * len(snods)
    # per dataset: object header, then its data (or chunk tree and chunks)
    layout = []
    for d in items:
        hsize = len(d.header(0))
        a_hdr = addr
        addr += hsize
        if d.chunks is None:
            a_data = addr
            addr += d.a.nbytes
            layout.append((d, a_hdr, a_data, None))
        else:
            nnodes = 0
            m = len(d.chunks)
            while True:
                m = (m + 2 * CHUNK_K - 1) // (2 * CHUNK_K)
                nnodes += m
                if m == 1:
                    break
            nsize = 24 + 2 * CHUNK_K * 8 + (2 * CHUNK_K + 1) * (8 + 8 * (d.a.ndim + 1))
            a_tree = addr
            addr += nnodes * nsize
            caddrs = []
            for blob in d.chunks:
                caddrs.append((addr, len(blob)))
                addr += len(blob)
            root, nodes = _chunk_btree_nodes(d, caddrs, a_tree)
            layout.append((d, a_hdr, root, nodes))
    eof = addr

    # --- serialise
    with open(path, "wb") as f:
        sb = SIGNATURE + struct.pack("<8B", 0, 0, 0, 0, 0, 8, 8, 0)
        sb += struct.pack("<HHI", LEAF_K, GROUP_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
        sb += struct.pack("<QQII", 0, a_root, 1, 0) + struct.pack("<QQ", a_gtree, a_heap)
        f.write(sb)
        f.write(_object_header([(MSG_STAB, 1, struct.pack("<QQ", a_gtree, a_heap))]))
        f.write(b"HEAP" + struct.pack("<B3xQQQ", 0, heap_size, free_off, a_heapdata))
        f.write(bytes(heap))
        # group B-tree: one leaf level over the symbol-table nodes
        gt = struct.pack("<4sBBHQQ", b"TREE", 0, 0, len(snods), UNDEF, UNDEF)
        gt += struct.pack("<Q", 0)
        for i, s in enumerate(snods):
            gt += struct.pack("<Q", a_snod + i * snod_size)
            gt += struct.pack("<Q", name_off[s[-1].name])
        f.write(gt + b"\0" * (gtree_size - len(gt)))
        hdr_addr = {d.name: a for d, a, _, _ in layout}
        for s in snods:
            sn = struct.pack("<4sBBH", b"SNOD", 1, 0, len(s))
            for d in s:
                sn += struct.pack("<QQII16x", name_off[d.name], hdr_addr[d.name], 0, 0)
            f.write(sn + b"\0" * (snod_size - len(sn)))
        for d, a_hdr, a_data, nodes in layout:
            assert f.tell() == a_hdr
            f.write(d.header(a_data))
            if nodes is None:
                f.write(memoryview(d.a).cast("B"))
            else:
                for _, body in sorted(nodes):
                    f.write(body)
                for blob in d.chunks:
                    f.write(blob)
        assert f.tell() == eof


# ---------------------------------------------------------------- reader
class _File:
    def __init__(self, buf):
        self.b = buf
        off = 0
        while True:
            if buf[off:off + 8] == SIGNATURE:
                break
            off = 512 if off == 0 else off * 2   # user blocks of 512, 1024, ...
            if off + 8 > len(buf):
                raise ValueError("not an HDF5 file")
        ver = buf[off + 8]
        if ver not in (0, 1):
            raise NotImplementedError("HDF5 superblock version %d" % ver)
        if (buf[off + 13], buf[off + 14]) != (8, 8):
            raise NotImplementedError("HDF5 offsets/lengths other than 8 bytes")
        p = off + 24 + (4 if ver == 1 else 0)
        self.base = struct.unpack_from("<Q", buf, p)[0]
        if self.base == 0 and off:
            self.base = off
        self.root = struct.unpack_from("<QQ", buf, p + 32)[1]

    def u(self, fmt, addr):
        return struct.unpack_from(fmt, self.b, self.base + addr)

    def raw(self, addr, n):
        a = self.base + addr
        return self.b[a:a + n]

    # object header (version 1) messages, continuation blocks followed
    def messages(self, addr):
        ver, _, nmsg, _, size = self.u("<BBHII", addr)
        if ver != 1:
            raise NotImplementedError("object header version %d" % ver)
        blocks = [(addr + 16, size)]
        out = []
        while blocks:
            p, size = blocks.pop(0)
            end = p + size
            while p + 8 <= end:
                mtype, msize, flags = self.u("<HHB", p)
                data = self.raw(p + 8, msize)
                if mtype == MSG_CONT:
                    blocks.append(struct.unpack_from("<QQ", data))
                elif mtype != MSG_NIL:
                    out.append((mtype, data))
                p += 8 + msize
        return out

    def heap_name(self, heap_addr, off):
        sig, _, _, _, data = self.u("<4sB3xQQQ", heap_addr)
        if sig != b"HEAP":
            raise ValueError("bad local heap")
        s = self.base + data + off
        return self.b[s:self.b.index(b"\0", s)].decode()

    def group(self, oh):
        """name -> object header address for an old-style (symbol table) group."""
        stab = [d for t, d in self.messages(oh) if t == MSG_STAB]
        if not stab:
            raise NotImplementedError("group without a symbol table (new-style links)")
        btree, heap = struct.unpack_from("<QQ", stab[0])
        out = {}
        self._walk_group(btree, heap, out)
        return out

    def _walk_group(self, node, heap, out):
        sig, ntype, level, nused = self.u("<4sBBH", node)
        if sig != b"TREE" or ntype != 0:
            raise ValueError("bad group B-tree node")
        p = node + 24
        for i in range(nused):
            child = self.u("<Q", p + 8)[0]
            p += 16
            if level > 0:
                self._walk_group(child, heap, out)
                continue
            sig, ver, _, nsym = self.u("<4sBBH", child)
            if sig != b"SNOD":
                raise ValueError("bad symbol-table node")
            for j in range(nsym):
                noff, oh = self.u("<QQ", child + 8 + 40 * j)
                out[self.heap_name(heap, noff)] = oh

    def dataset(self, oh):
        shape = dtype = layout = None
        filters = []
        for t, d in self.messages(oh):
            if t == MSG_SPACE:
                ver, rank = d[0], d[1]
                hdr = 8 if ver == 1 else 4
                shape = tuple(struct.unpack_from("<%dQ" % rank, d, hdr)) if rank else ()
            elif t == MSG_DTYPE:
                dtype = _decode_dtype(d)
            elif t == MSG_LAYOUT:
                layout = d
            elif t == MSG_FILTER:
                filters = _decode_filters(d)
        if shape is None or dtype is None or layout is None:
            raise ValueError("dataset lacks a dataspace, datatype or layout")
        ver = layout[0]
        count = int(np.prod(shape, dtype=np.int64))
        if ver == 3:
            cls = layout[1]
            if cls == 0:          # compact
                size = struct.unpack_from("<H", layout, 2)[0]
                return np.frombuffer(layout[4:4 + size], dtype, count).reshape(shape).copy()
            if cls == 1:
                addr, size = struct.unpack_from("<QQ", layout, 2)
                if addr == UNDEF:
                    return np.zeros(shape, dtype)
                return np.frombuffer(self.raw(addr, count * dtype.itemsize), dtype, count).reshape(shape).copy()
            if cls == 2:
                ndim = layout[2]
                btree = struct.unpack_from("<Q", layout, 3)[0]
                chunk = struct.unpack_from("<%dI" % ndim, layout, 11)[:-1]
                return self._chunked(btree, shape, chunk, dtype, filters)
            raise NotImplementedError("layout class %d" % cls)
        if ver in (1, 2):
            ndim, cls = layout[1], layout[2]
            if cls == 1:
                addr = struct.unpack_from("<Q", layout, 8)[0]
                return np.frombuffer(self.raw(addr, count * dtype.itemsize), dtype, count).reshape(shape).copy()
            if cls == 2:
                btree = struct.unpack_from("<Q", layout, 8)[0]
                chunk = struct.unpack_from("<%dI" % ndim, layout, 16)[:-1]
                return self._chunked(btree, shape, chunk, dtype, filters)
            raise NotImplementedError("layout class %d" % cls)
        raise NotImplementedError("layout message version %d" % ver)

    def _chunked(self, btree, shape, chunk, dtype, filters):
        out = np.zeros(shape, dtype)
        if btree == UNDEF:
            return out
        rank = len(shape)
        for nbytes, mask, offs, addr in self._walk_chunks(btree, rank):
            blob = self.raw(addr, nbytes)
            for k in range(len(filters) - 1, -1, -1):
                fid, cd = filters[k]
                if mask & (1 << k):
                    continue
                if fid == FILTER_DEFLATE:
                    blob = zlib.decompress(blob)
                elif fid == FILTER_SHUFFLE:
                    es = dtype.itemsize
                    blob = np.frombuffer(blob, np.uint8).reshape(es, -1).T.tobytes()
                else:
                    raise NotImplementedError("HDF5 filter %d" % fid)
            c = np.frombuffer(blob, dtype, int(np.prod(chunk, dtype=np.int64))).reshape(chunk)
            dst = tuple(slice(o, min(o + n, s)) for o, n, s in zip(offs, chunk, shape))
            src = tuple(slice(0, x.stop - x.start) for x in dst)
            out[dst] = c[src]
        return out

    def _walk_chunks(self, node, rank):
        sig, ntype, level, nused = self.u("<4sBBH", node)
        if sig != b"TREE" or ntype != 1:
            raise ValueError("bad chunk B-tree node")
        ksize = 8 + 8 * (rank + 1)
        p = node + 24
        for i in range(nused):
            nbytes, mask = self.u("<II", p)
            offs = self.u("<%dQ" % rank, p + 8)
            child = self.u("<Q", p + ksize)[0]
            p += ksize + 8
            if level > 0:
                yield from self._walk_chunks(child, rank)
            else:
                yield nbytes, mask, offs, child


def _decode_dtype(d):
    cls = d[0] & 0x0F
    b0 = d[1]
    size = struct.unpack_from("<I", d, 4)[0]
    order = ">" if b0 & 1 else "<"
    if cls == 0:
        return np.dtype("%s%s%d" % (order, "i" if b0 & 0x08 else "u", size))
    if cls == 1:
        if size not in (2, 4, 8):
            raise NotImplementedError("float of %d bytes" % size)
        return np.dtype("%sf%d" % (order, size))
    raise NotImplementedError("HDF5 datatype class %d" % cls)


def _decode_filters(d):
    ver, nf = d[0], d[1]
    p = 8 if ver == 1 else 2
    out = []
    for _ in range(nf):
        fid = struct.unpack_from("<H", d, p)[0]
        if ver == 1 or fid >= 256:
            nlen, flags, ncd = struct.unpack_from("<HHH", d, p + 2)
            p += 8
            p += _pad8(nlen) if ver == 1 else nlen
        else:
            flags, ncd = struct.unpack_from("<HH", d, p + 2)
            p += 6
        cd = struct.unpack_from("<%dI" % ncd, d, p)
        p += 4 * ncd
        if ver == 1 and ncd % 2:
            p += 4
        out.append((fid, cd))
    return out


def read(path, names=None):
    """Datasets of the root group of the HDF5 file at ``path`` as numpy arrays
    (only ``names`` when given); nested groups are walked with "/" paths."""
    with open(path, "rb") as fh:
        buf = fh.read()
    f = _File(buf)
    out = {}

    def visit(oh, prefix):
        for name, child in sorted(f.group(oh).items()):
            full = prefix + name
            kinds = {t for t, _ in f.messages(child)}
            if MSG_STAB in kinds:
                visit(child, full + "/")
            elif MSG_LAYOUT in kinds and (names is None or full in names):
                out[full] = f.dataset(child)

    visit(f.root, "")
    if names is not None:
        missing = [n for n in names if n not in out]
        if missing:
            raise KeyError("datasets not in %s: %s" % (path, ", ".join(missing)))
    return out


def contents(path):
    """Names of the datasets in the root group of ``path``."""
    with open(path, "rb") as fh:
        buf = fh.read()
    f = _File(buf)
    return sorted(f.group(f.root))
