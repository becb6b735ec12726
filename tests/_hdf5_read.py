"""A reader of the HDF5 subset the library writes, written from the HDF5
file format specification (superblock version 0, version-1 group B-trees
with local heaps and symbol-table nodes, version-1 object headers,
dataspace / datatype / data layout messages, contiguous storage), so the
tests can check the files without an HDF5 library.  It checks every
signature, version and size it meets and returns {path: ndarray} plus the
group listing {group path: [link names in file order]}."""
import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF


class Hdf5Error(ValueError):
    pass


def _need(ok, what):
    if not ok:
        raise Hdf5Error(what)


def read(path):
    buf = open(path, "rb").read()
    _need(buf[:8] == b"\x89HDF\r\n\x1a\n", "signature")
    sb_ver, fs_ver, root_ver, _, sh_ver, so, sl, _ = buf[8:16]
    _need((sb_ver, fs_ver, root_ver, sh_ver) == (0, 0, 0, 0), "superblock versions")
    _need((so, sl) == (8, 8), "offset/length sizes")
    leaf_k, internal_k, flags = struct.unpack_from("<HHI", buf, 16)
    _need(leaf_k > 0 and internal_k > 0 and flags == 0, "superblock K / flags")
    base, freespace, eof, driver = struct.unpack_from("<QQQQ", buf, 24)
    _need(base == 0 and freespace == UNDEF and driver == UNDEF, "superblock addresses")
    _need(eof == len(buf), "end-of-file address %d, file %d bytes" % (eof, len(buf)))
    name_off, root_hdr, cache = struct.unpack_from("<QQI", buf, 56)
    _need(name_off == 0 and cache == 1, "root symbol table entry")
    root_tree, root_heap = struct.unpack_from("<QQ", buf, 56 + 24)

    node_size = 24 + (2 * internal_k + 1) * 8 + 2 * internal_k * 8
    snod_size = 8 + 2 * leaf_k * 40
    out, listing = {}, {}

    def heap_name(heap, off):
        _need(buf[heap:heap + 4] == b"HEAP" and buf[heap + 4] == 0, "local heap")
        size, free, data = struct.unpack_from("<QQQ", buf, heap + 8)
        _need(free == 1 or free < size, "heap free list")
        _need(off < size, "name offset inside the heap")
        end = buf.index(b"\0", data + off)
        _need(end < data + size, "name inside the heap")
        return buf[data + off:end].decode()

    def messages(addr):
        _need(buf[addr] == 1, "object header version")
        n, refs, size = struct.unpack_from("<HII", buf, addr + 2)
        _need(refs >= 1, "reference count")
        p, end, msgs = addr + 16, addr + 16 + size, []
        while p < end:
            typ, msize, mflags = struct.unpack_from("<HHB", buf, p)
            _need(msize % 8 == 0, "message size alignment")
            msgs.append((typ, buf[p + 8:p + 8 + msize]))
            p += 8 + msize
        _need(p == end and len(msgs) == n, "object header message count / size")
        return dict(msgs)

    def dataset(m):
        ds = m[0x0001]
        _need(ds[0] == 1, "dataspace version")
        rank = ds[1]
        dims = struct.unpack_from("<%dQ" % rank, ds, 8)
        dt = m[0x0003]
        cls, ver = dt[0] & 15, dt[0] >> 4
        _need(ver == 1, "datatype version")
        size = struct.unpack_from("<I", dt, 4)[0]
        if cls == 1:
            _need(dt[1] & 0x41 == 0 and (dt[1] >> 4) & 3 == 2 and dt[2] == 63 and size == 8, "f64 bit field")
            off, prec, eloc, esz, mloc, msz, bias = struct.unpack_from("<HHBBBBI", dt, 8)
            _need((off, prec, eloc, esz, mloc, msz, bias) == (0, 64, 52, 11, 0, 52, 1023), "f64 properties")
            dtype = np.dtype("<f8")
        else:
            _need(cls == 0 and dt[1] & 1 == 0 and size == 8, "int64 bit field")
            dtype = np.dtype("<i8") if dt[1] & 8 else np.dtype("<u8")
            _need(struct.unpack_from("<HH", dt, 8) == (0, 64), "int64 properties")
        lay = m[0x0008]
        _need(lay[0] == 3 and lay[1] == 1, "contiguous layout, version 3")
        addr, nbytes = struct.unpack_from("<QQ", lay, 2)
        count = int(np.prod(dims)) if rank else 1
        _need(nbytes == count * size, "storage size")
        if nbytes == 0:
            return np.zeros(dims, dtype)
        _need(addr + nbytes <= len(buf), "data inside the file")
        return np.frombuffer(buf, dtype, count, addr).reshape(dims)

    def group(gpath, tree, heap, hdr):
        m = messages(hdr)
        _need(struct.unpack_from("<QQ", m[0x0011]) == (tree, heap), "cached symbol table matches the header")
        _need(buf[tree:tree + 4] == b"TREE" and buf[tree + 4] == 0 and buf[tree + 5] == 0, "group B-tree leaf")
        used = struct.unpack_from("<H", buf, tree + 6)[0]
        _need(used <= 2 * internal_k and tree + node_size <= len(buf), "B-tree node size")
        keys = [struct.unpack_from("<Q", buf, tree + 24 + 16 * i)[0] for i in range(used + 1)]
        kids = [struct.unpack_from("<Q", buf, tree + 32 + 16 * i)[0] for i in range(used)]
        names = []
        for i, snod in enumerate(kids):
            _need(buf[snod:snod + 4] == b"SNOD" and buf[snod + 4] == 1, "symbol table node")
            n = struct.unpack_from("<H", buf, snod + 6)[0]
            _need(0 < n <= 2 * leaf_k and snod + snod_size <= len(buf), "symbol table node size")
            lo, hi = heap_name(heap, keys[i]), heap_name(heap, keys[i + 1])
            for e in range(n):
                off, ohdr, ctype = struct.unpack_from("<QQI", buf, snod + 8 + 40 * e)
                name = heap_name(heap, off)
                _need(lo < name <= hi, "B-tree keys bound the names")
                names.append(name)
                sub = gpath + name
                m2 = messages(ohdr)
                if 0x0011 in m2:
                    _need(ctype == 1, "a subgroup caches its symbol table")
                    t2, h2 = struct.unpack_from("<QQ", buf, snod + 8 + 40 * e + 24)
                    group(sub + "/", t2, h2, ohdr)
                else:
                    out[sub] = dataset(m2)
        _need(names == sorted(names, key=lambda s: s.encode()), "names in strcmp order")
        listing[gpath] = names

    group("/", root_tree, root_heap, root_hdr)
    return out, listing
