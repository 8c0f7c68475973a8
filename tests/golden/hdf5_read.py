"""Minimal HDF5 reader for the reference's output files (test infrastructure).

Reads the datasets that libmpdata++'s HDF5 writer produces (output/hdf5.hpp:
H5::H5File with the library's default file format, float32 datasets,
contiguous or chunked storage, optional deflate filter): superblock version 0
or 1, version-1 object headers with continuation blocks, a root group held as a
symbol table (version-1 group B-tree, symbol-table nodes, local heap), the
dataspace (versions 1 and 2), datatype (fixed-point and floating-point), data
layout (version 3: contiguous, chunked with a version-1 raw-data B-tree) and
filter pipeline (versions 1 and 2; deflate only) messages, and scalar
attributes (message version 1).

Written from the HDF5 File Format Specification (The HDF Group, version 2.0 of
the format document, sections II.A superblock, III.A.1 version-1 B-trees,
III.B symbol table nodes, III.D local heaps, IV.A.1 version-1 object headers,
IV.A.2 messages 0x0001, 0x0003, 0x0008, 0x000B, 0x000C, 0x0010).  No HDF5 library is
available where this runs; Python's zlib decodes the deflate filter.

Usage:  read_dataset(path, "psi") -> numpy array (C order, as stored)
"""
import zlib

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"


class H5Error(Exception):
    pass


class File:
    def __init__(self, path):
        with open(path, "rb") as f:
            self.b = f.read()
        # the superblock may sit at 0, 512, 1024, ... (user block); the writer uses 0
        off = 0
        while self.b[off:off + 8] != SIGNATURE:
            off = 512 if off == 0 else off * 2
            if off >= len(self.b):
                raise H5Error("not an HDF5 file")
        self.sb = off
        ver = self.b[off + 8]
        if ver not in (0, 1):
            raise H5Error("superblock version %d not supported" % ver)
        self.O = self.b[off + 13]  # size of offsets
        self.L = self.b[off + 14]  # size of lengths
        p = off + 24 + (4 if ver == 1 else 0)
        self.base = self.addr(p)
        p += 4 * self.O  # base, free-space, end-of-file, driver-info addresses
        # root group symbol table entry
        self.root = self.symbol_entry(p)

    # ---- primitive readers ----
    def uint(self, p, n):
        return int.from_bytes(self.b[p:p + n], "little")

    def addr(self, p):
        return self.uint(p, self.O)

    def undefined(self, a):
        return a == (1 << (8 * self.O)) - 1

    def symbol_entry(self, p):
        name_off = self.addr(p)
        header = self.addr(p + self.O)
        cache = self.uint(p + 2 * self.O, 4)
        scratch = p + 2 * self.O + 8
        ent = {"name_off": name_off, "header": header, "cache": cache}
        if cache == 1:
            ent["btree"] = self.addr(scratch)
            ent["heap"] = self.addr(scratch + self.O)
        return ent

    # ---- local heap (names of a group's links) ----
    def heap_data(self, a):
        p = self.base + a
        if self.b[p:p + 4] != b"HEAP":
            raise H5Error("local heap signature missing")
        size = self.uint(p + 8, self.L)
        data = self.addr(p + 8 + 2 * self.L)
        return self.base + data, size

    def heap_string(self, heap, off):
        start, _ = heap
        end = self.b.index(b"\x00", start + off)
        return self.b[start + off:end].decode()

    # ---- version-1 B-trees ----
    def btree_children(self, a, node_type, rank=0):
        """Yield (key, child address) of every leaf entry below the node at a."""
        p = self.base + a
        if self.b[p:p + 4] != b"TREE":
            raise H5Error("B-tree signature missing")
        ntype, level, used = self.b[p + 4], self.b[p + 5], self.uint(p + 6, 2)
        if ntype != node_type:
            raise H5Error("unexpected B-tree node type %d" % ntype)
        p += 8 + 2 * self.O  # siblings
        key_size = self.L if node_type == 0 else 8 + 8 * (rank + 1)
        for _ in range(used):
            key = p
            child = self.addr(p + key_size)
            p += key_size + self.O
            if level > 0:
                yield from self.btree_children(child, node_type, rank)
            else:
                yield key, child

    # ---- groups ----
    def group_links(self, ent):
        if ent.get("cache") != 1:
            hdr = self.object_header(ent["header"])
            st = [m for m in hdr if m[0] == 0x0011]  # symbol table message
            if not st:
                raise H5Error("group without a symbol table (new-style groups not supported)")
            p = st[0][1]
            ent = {"btree": self.addr(p), "heap": self.addr(p + self.O)}
        heap = self.heap_data(ent["heap"])
        links = {}
        for _, snod in self.btree_children(ent["btree"], 0):
            p = self.base + snod
            if self.b[p:p + 4] != b"SNOD":
                raise H5Error("symbol table node signature missing")
            n = self.uint(p + 6, 2)
            q = p + 8
            for _ in range(n):
                e = self.symbol_entry(q)
                links[self.heap_string(heap, e["name_off"])] = e
                q += 2 * self.O + 8 + 16
        return links

    # ---- object headers ----
    def object_header(self, a):
        """List of (type, data offset, size) of the messages of the header at a."""
        p = self.base + a
        if self.b[p] != 1:
            raise H5Error("object header version %d not supported" % self.b[p])
        n_msgs = self.uint(p + 2, 2)
        size = self.uint(p + 8, 4)
        blocks = [(p + 16, size)]
        msgs = []
        while blocks and len(msgs) < n_msgs:
            q, size = blocks.pop(0)
            end = q + size
            while q + 8 <= end and len(msgs) < n_msgs:
                mtype, msize = self.uint(q, 2), self.uint(q + 2, 2)
                data = q + 8
                if mtype == 0x0010:  # continuation
                    blocks.append((self.base + self.addr(data), self.uint(data + self.O, self.L)))
                msgs.append((mtype, data, msize))
                q = data + msize
        return msgs

    # ---- datasets ----
    def dataset(self, name):
        links = self.group_links(self.root)
        if name not in links:
            raise H5Error("no dataset %r (have %s)" % (name, sorted(links)))
        msgs = self.object_header(links[name]["header"])
        by = {}
        for t, d, s in msgs:
            by.setdefault(t, (d, s))
        shape = self._dataspace(*by[0x0001])
        dtype = self._datatype(*by[0x0003])
        filters = self._filters(*by[0x000B]) if 0x000B in by else []
        return self._layout(by[0x0008][0], shape, dtype, filters)

    def _dataspace(self, p, _):
        ver, rank, flags = self.b[p], self.b[p + 1], self.b[p + 2]
        q = p + (8 if ver == 1 else 4)
        return tuple(self.uint(q + i * self.L, self.L) for i in range(rank))

    def _datatype(self, p, _):
        cls = self.b[p] & 0x0F
        bits = self.b[p + 1]
        size = self.uint(p + 4, 4)
        order = ">" if bits & 1 else "<"
        if cls == 1:
            return np.dtype(order + {4: "f4", 8: "f8"}[size])
        if cls == 0:
            signed = bool(bits & 0x08)
            return np.dtype(order + ("i" if signed else "u") + str(size))
        raise H5Error("datatype class %d not supported" % cls)

    def _filters(self, p, _):
        ver, n = self.b[p], self.b[p + 1]
        q = p + (8 if ver == 1 else 2)
        out = []
        for _ in range(n):
            fid = self.uint(q, 2)
            name_len = self.uint(q + 2, 2) if (ver == 1 or fid >= 256) else 0
            n_vals = self.uint(q + 6, 2)
            q += 8
            if name_len:
                q += (name_len + 7) // 8 * 8 if ver == 1 else name_len
            q += 4 * n_vals
            if ver == 1 and n_vals % 2:
                q += 4
            out.append(fid)
        for fid in out:
            if fid != 1:
                raise H5Error("filter %d not supported (deflate only)" % fid)
        return out

    def _layout(self, p, shape, dtype, filters):
        ver, cls = self.b[p], self.b[p + 1]
        if ver != 3:
            raise H5Error("data layout version %d not supported" % ver)
        count = int(np.prod(shape))
        if cls == 1:  # contiguous
            a = self.addr(p + 2)
            if self.undefined(a):
                return np.zeros(shape, dtype)
            start = self.base + a
            return np.frombuffer(self.b, dtype, count, start).reshape(shape).copy()
        if cls != 2:
            raise H5Error("layout class %d not supported" % cls)
        rank1 = self.b[p + 2]
        btree = self.addr(p + 3)
        q = p + 3 + self.O
        cdims = [self.uint(q + 4 * i, 4) for i in range(rank1)]
        chunk = tuple(cdims[:-1])
        if cdims[-1] != dtype.itemsize:
            raise H5Error("chunk element size differs from the datatype")
        out = np.zeros(shape, dtype)
        if self.undefined(btree):
            return out
        rank = len(shape)
        for key, child in self.btree_children(btree, 1, rank):
            nbytes = self.uint(key, 4)
            mask = self.uint(key + 4, 4)
            origin = [self.uint(key + 8 + 8 * i, 8) for i in range(rank)]
            raw = self.b[self.base + child:self.base + child + nbytes]
            if filters and not (mask & 1):
                raw = zlib.decompress(raw)
            block = np.frombuffer(raw, dtype, int(np.prod(chunk))).reshape(chunk)
            sl_out = tuple(slice(o, min(o + c, s)) for o, c, s in zip(origin, chunk, shape))
            sl_in = tuple(slice(0, s.stop - s.start) for s in sl_out)
            out[sl_out] = block[sl_in]
        return out


    # ---- attributes (message 0x000C, version 1) ----
    def attributes(self, name):
        """{attribute: value} of the root member `name` (scalar or 1-element attributes)."""
        links = self.group_links(self.root)
        out = {}
        for t, d, size in self.object_header(links[name]["header"]):
            if t != 0x000C:
                continue
            ver = self.b[d]
            if ver != 1:
                raise H5Error("attribute message version %d not supported" % ver)
            ns, ts, ss = self.uint(d + 2, 2), self.uint(d + 4, 2), self.uint(d + 6, 2)
            p = d + 8
            nm = self.b[p:p + ns].split(b"\0")[0].decode()
            p += (ns + 7) // 8 * 8
            tp = p
            p += (ts + 7) // 8 * 8
            shape = self._dataspace(p, ss)
            p += (ss + 7) // 8 * 8
            count = int(np.prod(shape)) if shape else 1
            if self.b[tp] & 0x0F == 3:  # string
                n = self.uint(tp + 4, 4)
                out[nm] = self.b[p:p + n].split(b"\0")[0].decode()
            else:
                dt = self._datatype(tp, ts)
                v = np.frombuffer(self.b, dt, count, p)
                out[nm] = v[0] if count == 1 else v.copy()
        return out

    def attribute_messages(self, name):
        """{attribute: raw attribute message} of the root member `name`."""
        links = self.group_links(self.root)
        out = {}
        for t, d, size in self.object_header(links[name]["header"]):
            if t == 0x000C:
                ns = self.uint(d + 2, 2)
                out[self.b[d + 8:d + 8 + ns].split(b"\0")[0].decode()] = bytes(self.b[d:d + size])
        return out

    def message_bytes(self, name, mtype):
        """Raw bytes of the first message of type mtype in the header of root member `name`."""
        links = self.group_links(self.root)
        for t, d, size in self.object_header(links[name]["header"]):
            if t == mtype:
                return bytes(self.b[d:d + size])
        return None


def read_dataset(path, name):
    return File(path).dataset(name)


def list_root(path):
    f = File(path)
    return sorted(f.group_links(f.root))
