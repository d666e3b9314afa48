"""Reader of OpenVDB files for checking the VDB export (TEST INFRASTRUCTURE ONLY).

Only tests/ use this module, as the checker of the library's VDB writer
(gpu-sims_b200/csrc/vdb.cpp).  It restates the published OpenVDB file layout
(format versions 222-224, uncompressed values) for vec3s and float trees of the
standard 5-4-3 configuration and densifies the grid.  The reference writes
these files through OpenVDB (common/common-cpp/src/vdb_writer.cpp:96-141,
called from volumetric-grid/lattice-boltzmann/src/main.cpp:1767-1790);
OpenVDB is not installed in this image, so parity of the writer against
OpenVDB itself is unpinned: this reader is an independent restatement of
the format, written from its description rather than from the writer.

It reads what the format allows, not only what the writer emits: root
tiles, internal-node tiles (active or not), masked value buffers with their
metadata byte (0-6), and the UniformScale / ScaleTranslate map families.
"""
from __future__ import annotations

import struct

import numpy as np

MAGIC = 0x56444220
LOG2 = {"root": None, 2: 5, 1: 4, 0: 3}   # internal level -> log2 dim
VALUE_TYPES = {"vec3s": (np.float32, 3), "float": (np.float32, 1)}


class _In:
    def __init__(self, data: bytes):
        self.b = data
        self.p = 0

    def take(self, n):
        if self.p + n > len(self.b):
            raise ValueError(f"truncated file at {self.p} (+{n})")
        v = self.b[self.p:self.p + n]
        self.p += n
        return v

    def unpack(self, fmt):
        return struct.unpack("<" + fmt, self.take(struct.calcsize("<" + fmt)))

    def u8(self):
        return self.unpack("B")[0]

    def u32(self):
        return self.unpack("I")[0]

    def i32(self):
        return self.unpack("i")[0]

    def i64(self):
        return self.unpack("q")[0]

    def string(self):
        return self.take(self.u32()).decode()

    def array(self, dtype, count):
        dt = np.dtype(dtype).newbyteorder("<")
        return np.frombuffer(self.take(dt.itemsize * count), dt).copy()


def _mask(r: _In, log2: int) -> np.ndarray:
    """A node mask of 2^(3 log2) bits (64-bit words, bit i of word i >> 6)."""
    words = r.array(np.uint64, (1 << (3 * log2)) // 64)
    bits = np.unpackbits(words.view(np.uint8), bitorder="little")
    return bits.astype(bool)


def _values(r: _In, count: int, value_mask: np.ndarray, vt, comps: int, compression: int,
            background) -> np.ndarray:
    """A value buffer: metadata byte, optional inactive values and selection
    mask, then the values (all, or only the active ones when the grid's
    compression flags ask for active-mask compression)."""
    if compression & 0x1 or compression & 0x4:
        raise ValueError("zip / blosc compressed buffers are not read here")
    meta = r.u8()
    inactive = [np.array(background, vt).reshape(comps)] * 2
    if meta == 1:
        inactive[0] = -np.array(background, vt).reshape(comps)
    if meta in (2, 4, 5):
        inactive[0] = r.array(vt, comps)
    if meta == 5:
        inactive[1] = r.array(vt, comps)
    sel = None
    if meta in (3, 4, 5):
        sel = _mask(r, {512: 3, 4096: 4, 32768: 5}[count])
    mask_compressed = bool(compression & 0x2) and meta != 6
    n = int(value_mask.sum()) if mask_compressed else count
    vals = r.array(vt, n * comps).reshape(n, comps)
    if not mask_compressed:
        return vals
    out = np.empty((count, comps), vt)
    out[value_mask] = vals
    off = ~value_mask
    if sel is None:
        out[off] = inactive[0]
    else:
        out[off & ~sel] = inactive[0]
        out[off & sel] = inactive[1]
    return out


def _node_origin_index(i: int, log2: int, child_span: int):
    """Offset of child i (x slowest, z fastest) in units of voxels."""
    d = 1 << log2
    x, y, z = i >> (2 * log2), (i >> log2) & (d - 1), i & (d - 1)
    return x * child_span, y * child_span, z * child_span


def read(path: str) -> dict:
    """Parses one-grid or multi-grid files; returns a dict with the header
    fields and, per grid, its name, type, metadata, transform, the stream
    positions as stored and as found, its leaves (origin, value mask,
    values), internal and root tiles, active voxel count and bounding box."""
    data = open(path, "rb").read()
    r = _In(data)
    magic = r.i64()
    if magic != MAGIC:
        raise ValueError(f"bad magic {magic:#x}")
    out = {"file_version": r.u32(), "library": (r.u32(), r.u32())}
    if not 222 <= out["file_version"] <= 224:
        raise ValueError(f"file version {out['file_version']} not read here")
    out["has_grid_offsets"] = r.u8()
    out["uuid"] = r.take(36).decode()
    out["file_meta"] = _metadata(r)
    ngrids = r.i32()
    grids = []
    for _ in range(ngrids):
        g = {"name": r.string(), "type": r.string(), "parent": r.string()}
        g["stored_pos"] = r.unpack("qqq")
        grid_pos = r.p
        compression = r.u32()
        g["compression"] = compression
        g["meta"] = _metadata(r)
        g["transform"] = _transform(r)
        if not g["type"].startswith("Tree_") or not g["type"].endswith("_5_4_3"):
            raise ValueError(f"tree type {g['type']} not read here")
        vt_name = g["type"][5:-6]
        if vt_name not in VALUE_TYPES:
            raise ValueError(f"value type {vt_name} not read here")
        vt, comps = VALUE_TYPES[vt_name]
        bufcount = r.i32()
        if bufcount != 1:
            raise ValueError("buffer count must be 1")
        background = r.array(vt, comps)
        ntiles, nchildren = r.u32(), r.u32()
        tiles = []
        for _ in range(ntiles):
            org = r.unpack("iii")
            val = r.array(vt, comps)
            active = r.u8()
            tiles.append((org, val, active))
        topo = []    # (leaf origin, value mask) in file order
        g["tiles"] = []  # (origin, span, value, active) of internal-node tiles

        def internal(origin, level):
            log2 = LOG2[level]
            span = {2: 128, 1: 8}[level]
            cmask = _mask(r, log2)
            vmask = _mask(r, log2)
            vals = _values(r, 1 << (3 * log2), vmask, vt, comps, compression, background)
            for i in np.flatnonzero(~cmask):
                if vmask[i] or not np.array_equal(vals[i], background):
                    o = tuple(int(v) for v in np.add(origin, _node_origin_index(int(i), log2, span)))
                    g["tiles"].append((o, span, vals[i], bool(vmask[i])))
            for i in np.flatnonzero(cmask):
                o = tuple(int(v) for v in np.add(origin, _node_origin_index(int(i), log2, span)))
                if level == 2:
                    internal(o, 1)
                else:
                    topo.append((o, _mask(r, 3)))

        for _ in range(nchildren):
            org = r.unpack("iii")
            internal(org, 2)
        for org, val, active in tiles:
            g["tiles"].append((tuple(org), 4096, val, bool(active)))
        g["block_pos_found"] = r.p
        leaves = []
        for org, topo_mask in topo:
            vmask = _mask(r, 3)
            if not np.array_equal(vmask, topo_mask):
                raise ValueError(f"leaf {org}: buffer mask differs from topology mask")
            vals = _values(r, 512, vmask, vt, comps, compression, background)
            leaves.append((org, vmask, vals))
        g["grid_pos_found"] = grid_pos
        g["end_pos_found"] = r.p
        g["background"] = background
        g["leaves"] = leaves
        g["active_voxels"] = int(sum(int(m.sum()) for _, m, _ in leaves)) + sum(
            s ** 3 for _, s, _, a in g["tiles"] if a)
        if leaves:
            lo, hi = np.full(3, 2 ** 31 - 1), np.full(3, -2 ** 31)
            for org, m, _ in leaves:
                idx = np.flatnonzero(m)
                if idx.size:
                    c = np.stack([idx >> 6, (idx >> 3) & 7, idx & 7], 1) + np.array(org)
                    lo, hi = np.minimum(lo, c.min(0)), np.maximum(hi, c.max(0))
            g["bbox"] = (tuple(int(v) for v in lo), tuple(int(v) for v in hi))
        grids.append(g)
        if out["has_grid_offsets"]:
            r.p = g["stored_pos"][2]
    out["grids"] = grids
    out["trailing_bytes"] = len(data) - r.p
    return out


def dense(grid: dict, shape) -> tuple[np.ndarray, np.ndarray]:
    """The grid on the box [0, shape): values float[N][comps] and the active
    flag bool[N], x-fastest (background and inactive elsewhere)."""
    nx, ny, nz = shape
    comps = grid["background"].size
    out = np.broadcast_to(grid["background"], (nx + 8, ny + 8, nz + 8, comps)).copy()
    act = np.zeros((nx + 8, ny + 8, nz + 8), bool)
    for (x, y, z), span, v, a in grid["tiles"]:
        out[x:x + span, y:y + span, z:z + span] = v
        act[x:x + span, y:y + span, z:z + span] = a
    for (x, y, z), m, vals in grid["leaves"]:
        if x >= nx + 8 or y >= ny + 8 or z >= nz + 8:
            continue
        out[x:x + 8, y:y + 8, z:z + 8] = vals.reshape(8, 8, 8, comps)  # leaf order: z fastest
        act[x:x + 8, y:y + 8, z:z + 8] = m.reshape(8, 8, 8)
    out = out[:nx, :ny, :nz].transpose(2, 1, 0, 3).reshape(-1, comps)
    act = act[:nx, :ny, :nz].transpose(2, 1, 0).reshape(-1)
    return out, act


def _metadata(r: _In) -> dict:
    n = r.u32()
    meta = {}
    for _ in range(n):
        name, typ = r.string(), r.string()
        size = r.u32()
        raw = r.take(size)
        if typ == "string":
            meta[name] = raw.decode()
        elif typ == "bool":
            meta[name] = bool(raw[0])
        elif typ == "int32":
            meta[name] = struct.unpack("<i", raw)[0]
        elif typ == "int64":
            meta[name] = struct.unpack("<q", raw)[0]
        elif typ == "float":
            meta[name] = struct.unpack("<f", raw)[0]
        elif typ == "double":
            meta[name] = struct.unpack("<d", raw)[0]
        elif typ == "vec3i":
            meta[name] = struct.unpack("<iii", raw)
        elif typ == "vec3d":
            meta[name] = struct.unpack("<ddd", raw)
        else:
            meta[name] = (typ, raw)
    return meta


def _transform(r: _In) -> dict:
    kind = r.string()
    if kind in ("UniformScaleMap", "ScaleMap"):
        t = {"map": kind, "translation": (0.0, 0.0, 0.0)}
    elif kind in ("UniformScaleTranslateMap", "ScaleTranslateMap"):
        t = {"map": kind, "translation": r.unpack("ddd")}
    else:
        raise ValueError(f"map {kind} not read here")
    t["scale"], t["voxel_size"], t["scale_inverse"], t["inv_scale_sqr"], t["inv_twice_scale"] = (
        r.unpack("ddd") for _ in range(5))
    return t
