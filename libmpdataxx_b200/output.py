"""Output on output steps, in the layout of libmpdata++'s output::hdf5_xdmf
(output/hdf5.hpp, output/hdf5_xdmf.hpp, output/detail/xdmf_writer.hpp).

The fields stay on the GPU between output steps; on an output step the
advectees are read back once and written as

  <outdir>/const.h5                  X, Y[, Z] cell-corner coordinates (float32,
                                     shape grid + 1), T (the output times), and a
                                     group "advection" with attributes opts, dt,
                                     di, dj[, dk], var_dt, n_iters
  <outdir>/timestepNNNNNNNNNN.h5     one float32 dataset per output variable
                                     (shape grid)
  <outdir>/timestepNNNNNNNNNN.xmf    the XDMF description of that record
  <outdir>/temp.xmf                  the temporal collection of all records

HDF5 is written by a small writer of this module, from the HDF5 file-format
specification (superblock version 0, version-1 object headers, a root group
held as a symbol table, contiguous datasets): no HDF5 library is needed.  The
message encodings (dataspace with maximum dimensions, IEEE little-endian float
and integer datatypes, fill value version 2, string and scalar attributes) are
the ones the HDF5 library writes for the reference; datasets are contiguous
where the reference's writer chunks and deflates them (output/hdf5.hpp:157-160),
which readers treat alike.  The XDMF files are byte for byte the reference's.
"""
import os

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
LEAF_K, INTERNAL_K = 4, 16   # the library's defaults: 8 links per symbol-table node, 32 per B-tree node
BTREE_NODE = 24 + (2 * INTERNAL_K + 1) * 8 + 2 * INTERNAL_K * 8
SNOD_SIZE = 8 + 2 * LEAF_K * 40


def _pad8(b):
    return b + b"\0" * (-len(b) % 8)


def _u(v, n):
    return int(v).to_bytes(n, "little")


# ---- message encodings ----------------------------------------------------
def _dataspace(shape):
    """Dataspace message version 1 with maximum dimensions equal to the dimensions."""
    b = bytes([1, len(shape), 1, 0]) + _u(0, 4)
    b += b"".join(_u(n, 8) for n in shape) + b"".join(_u(n, 8) for n in shape)
    return b


def _datatype(dt):
    dt = np.dtype(dt)
    if dt == np.float32:
        return bytes([0x11, 0x20, 0x1F, 0x00]) + _u(4, 4) + _u(0, 2) + _u(32, 2) + bytes([23, 8, 0, 23]) + _u(127, 4)
    if dt == np.float64:
        return bytes([0x11, 0x20, 0x3F, 0x00]) + _u(8, 4) + _u(0, 2) + _u(64, 2) + bytes([52, 11, 0, 52]) + _u(1023, 4)
    if dt.kind in "iu" or dt == np.bool_:
        signed = 0x08 if dt.kind == "i" else 0x00
        return bytes([0x10, signed, 0, 0]) + _u(dt.itemsize, 4) + _u(0, 2) + _u(8 * dt.itemsize, 2)
    raise ValueError("unsupported dtype %s" % dt)


def _string_type(n):
    """Fixed-length ASCII string, null-terminated padding (the library's C_S1)."""
    return bytes([0x13, 0, 0, 0]) + _u(n, 4)


FILL_VALUE = bytes([2, 1, 2, 1]) + _u(0, 4)  # version 2, early allocation, fill value defined, no value


def _layout_contiguous(addr, size):
    return bytes([3, 1]) + _u(addr, 8) + _u(size, 8)


def _attribute(name, value):
    """Attribute message version 1 of a scalar (one-element) attribute."""
    nm = name.encode() + b"\0"
    if isinstance(value, str):
        raw = value.encode()
        dtype, data = _string_type(len(raw)), raw
    elif isinstance(value, (bool, np.bool_)):
        dtype, data = _datatype(np.uint8), _u(int(value), 1)
    elif isinstance(value, (int, np.integer)):
        dtype, data = _datatype(np.int32), np.int32(value).tobytes()
    else:
        dtype, data = _datatype(np.float32), np.float32(value).tobytes()
    space = _dataspace((1,))
    head = bytes([1, 0]) + _u(len(nm), 2) + _u(len(dtype), 2) + _u(len(space), 2)
    return head + _pad8(nm) + _pad8(dtype) + _pad8(space) + data


def _message(mtype, data, flags=0):
    data = _pad8(data)
    return _u(mtype, 2) + _u(len(data), 2) + bytes([flags, 0, 0, 0]) + data


def _object_header(messages):
    """Version-1 object header: 16-byte prefix (with alignment padding), then the messages."""
    body = b"".join(messages)
    return bytes([1, 0]) + _u(len(messages), 2) + _u(1, 4) + _u(len(body), 4) + _u(0, 4) + body


# ---- file assembly ---------------------------------------------------------
class _File:
    def __init__(self):
        self.b = bytearray(96)  # superblock, written last

    def alloc(self, n):
        self.b += b"\0" * (-len(self.b) % 8)
        a = len(self.b)
        self.b += b"\0" * n
        return a

    def put(self, a, data):
        self.b[a:a + len(data)] = data

    def group(self, members, attrs=()):
        """Write a group (members: sorted list of (name, object header address,
        scratch or None)); returns (object header address, B-tree, heap)."""
        if len(members) > 2 * LEAF_K:
            raise ValueError("at most %d links per group" % (2 * LEAF_K))
        # local heap of the link names: offset 0 is the empty name
        names = b"\0" * 8
        offs = []
        for name, _, _ in members:
            offs.append(len(names))
            names += _pad8(name.encode() + b"\0")
        heap = self.alloc(32)
        data = self.alloc(len(names))
        self.put(data, names)
        self.put(heap, b"HEAP" + bytes([0, 0, 0, 0]) + _u(len(names), 8) + _u(UNDEF, 8) + _u(data, 8))
        btree = self.alloc(BTREE_NODE)
        node = b"TREE" + bytes([0, 0]) + _u(1 if members else 0, 2) + _u(UNDEF, 8) + _u(UNDEF, 8)
        if members:
            snod = self.alloc(SNOD_SIZE)
            ent = b"SNOD" + bytes([1, 0]) + _u(len(members), 2)
            for (name, hdr, scratch), off in zip(members, offs):
                ent += _u(off, 8) + _u(hdr, 8)
                if scratch is None:
                    ent += _u(0, 4) + _u(0, 4) + b"\0" * 16
                else:
                    ent += _u(1, 4) + _u(0, 4) + _u(scratch[0], 8) + _u(scratch[1], 8)
            self.put(snod, ent)
            node += _u(0, 8) + _u(snod, 8) + _u(offs[-1], 8)
        self.put(btree, node)
        msgs = [_message(0x11, _u(btree, 8) + _u(heap, 8))] + [_message(0x0C, _attribute(k, v)) for k, v in attrs]
        hdr_bytes = _object_header(msgs)
        hdr = self.alloc(len(hdr_bytes))
        self.put(hdr, hdr_bytes)
        return hdr, btree, heap

    def dataset(self, arr):
        arr = np.ascontiguousarray(arr)
        if arr.dtype.byteorder == ">":
            arr = arr.astype(arr.dtype.newbyteorder("<"))
        raw = arr.tobytes()
        data = self.alloc(len(raw))
        self.put(data, raw)
        msgs = [_message(0x01, _dataspace(arr.shape)), _message(0x03, _datatype(arr.dtype)),
                _message(0x05, FILL_VALUE), _message(0x08, _layout_contiguous(data, len(raw)))]
        hdr_bytes = _object_header(msgs)
        hdr = self.alloc(len(hdr_bytes))
        self.put(hdr, hdr_bytes)
        return hdr

    def finish(self, root):
        hdr, btree, heap = root
        sb = b"\x89HDF\r\n\x1a\n" + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + _u(LEAF_K, 2) + _u(INTERNAL_K, 2) + _u(0, 4)
        sb += _u(0, 8) + _u(UNDEF, 8) + _u(len(self.b), 8) + _u(UNDEF, 8)
        sb += _u(0, 8) + _u(hdr, 8) + _u(1, 4) + _u(0, 4) + _u(btree, 8) + _u(heap, 8)
        self.put(0, sb)
        return bytes(self.b)


def write_h5(path, datasets, groups=None):
    """Write an HDF5 file with the given root datasets ({name: array}) and
    groups of scalar attributes ({group: {attribute: value}})."""
    f = _File()
    members = []
    for name in sorted(datasets):
        members.append((name, f.dataset(datasets[name]), None))
    for name in sorted(groups or {}):
        hdr, btree, heap = f.group([], list(groups[name].items()))
        members.append((name, hdr, (btree, heap)))
    members.sort(key=lambda m: m[0].encode())
    data = f.finish(f.group(members))
    with open(path, "wb") as fh:
        fh.write(data)


# ---- XDMF (boost::property_tree's XML writer with one-tab indentation) ------
def _dims(shape):
    return "".join("%d " % n for n in shape)


def xmf_record(hdf_name, time, grid, var_names, const_name="const.h5"):
    nd = len(grid)
    corner = [n + 1 for n in grid]
    axes = ["X", "Y", "Z"][:nd]
    lines = ['<?xml version="1.0" encoding="utf-8"?>', "<Xdmf>", "\t<Domain>",
             '\t\t<Grid Name="Grid" GridType="Uniform" xml:id="gid">',
             '\t\t\t<Time Value="%f"/>' % time,
             '\t\t\t<Topology TopologyType="%s" Dimensions="%s"/>' % ("2DSMesh" if nd == 2 else "3DSMesh", _dims(corner)),
             '\t\t\t<Geometry GeometryType="%s">' % ("X_Y" if nd == 2 else "X_Y_Z")]
    for a in axes:
        lines.append('\t\t\t\t<DataItem Dimensions="%s" NumberType="Float" Format="HDF">%s:/%s</DataItem>'
                     % (_dims(corner), const_name, a))
    lines.append("\t\t\t</Geometry>")
    for v in sorted(var_names):
        lines += ['\t\t\t<Attribute Name="%s" AttributeType="Scalar" Center="Cell">' % v,
                  '\t\t\t\t<DataItem Dimensions="%s" NumberType="Float" Format="HDF">%s:/%s</DataItem>'
                  % (_dims(grid), hdf_name, v),
                  "\t\t\t</Attribute>"]
    lines += ["\t\t</Grid>", "\t</Domain>", "</Xdmf>"]
    return "\n".join(lines) + "\n"


def xmf_temporal(xmf_names):
    lines = ['<?xml version="1.0" encoding="utf-8"?>', '<Xdmf xmlns:xi="http://www.w3.org/2001/XInclude">',
             "\t<Domain>", '\t\t<Grid Name="TimeGrid" GridType="Collection" CollectionType="Temporal">']
    lines += ['\t\t\t<xi:include href="%s" xpointer="gid"/>' % n for n in xmf_names]
    lines += ["\t\t</Grid>", "\t</Domain>", "</Xdmf>"]
    return "\n".join(lines) + "\n"


class hdf5_xdmf:
    """output::hdf5_xdmf for a run of concurr.cuda: start() writes const.h5 and
    record(timestep) reads the output variables back from the GPU (the only
    device-to-host traffic) and writes one record.

    outvars: {equation index: name}, as rt_params_t::outvars."""

    def __init__(self, outdir, grid, dt, dijk, outvars, opts_str="", n_iters=2, n_records=None):
        if len(grid) not in (2, 3):
            raise ValueError("only 2D and 3D output supported")  # hdf5_xdmf.hpp:38
        self.outdir, self.grid, self.dt, self.dijk = outdir, tuple(grid), float(dt), tuple(dijk)
        self.outvars = dict(outvars)
        self.opts_str, self.n_iters, self.n_records = opts_str, int(n_iters), n_records
        self.timesteps, self.times = [], []

    def start(self, times):
        """const.h5: corner coordinates, the output times, run parameters (hdf5.hpp:160-230, 620-660)."""
        os.makedirs(self.outdir, exist_ok=True)
        nd = len(self.grid)
        corner = tuple(n + 1 for n in self.grid)
        idx = np.indices(corner, dtype=np.float64)
        ds = {a: (self.dijk[d] * idx[d]).astype(np.float32) for d, a in enumerate(["X", "Y", "Z"][:nd])}
        ds["T"] = np.asarray(times, dtype=np.float64).astype(np.float32)
        attrs = {"opts": self.opts_str, "dt": self.dt}
        for d, a in enumerate(["di", "dj", "dk"][:nd]):
            attrs[a] = self.dijk[d]
        attrs["var_dt"] = False
        attrs["n_iters"] = self.n_iters
        write_h5(os.path.join(self.outdir, "const.h5"), ds, {"advection": attrs})

    def record(self, timestep, fields):
        """fields: {name: array of shape grid}; writes timestepNNNNNNNNNN.{h5,xmf} and temp.xmf."""
        base = "timestep%010d" % timestep
        write_h5(os.path.join(self.outdir, base + ".h5"),
                 {n: np.asarray(a, dtype=np.float64).astype(np.float32) for n, a in fields.items()})
        with open(os.path.join(self.outdir, base + ".xmf"), "w") as f:
            f.write(xmf_record(base + ".h5", timestep * self.dt, self.grid, list(fields)))
        self.timesteps.append(base + ".xmf")
        with open(os.path.join(self.outdir, "temp.xmf"), "w") as f:
            f.write(xmf_temporal(self.timesteps))

    def run(self, run, nt, outfreq):
        """Advance `run` nt steps, recording at timestep 0 and every outfreq steps
        (solver_common.hpp record_all on outfreq): between records the fields
        never leave the device."""
        steps = list(range(0, nt + 1, outfreq))
        self.start([s * self.dt for s in steps])
        done = 0
        for s in steps:
            if s > done:
                run.advance(s - done)
                done = s
            self.record(s, {name: run.advectee(e) for e, name in self.outvars.items()})
        if nt > done:  # steps after the last output step
            run.advance(nt - done)
