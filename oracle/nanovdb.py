"""NanoVDB-form export, restated in numpy: test infrastructure (the oracle),
not the product.

`export(st, background, grid_name, grid_class)` lays out the bytes libgvdb2's
gvdb2_export_nanovdb writes (records gvdb2_nv_* in include/gvdb2.h), each
field computed as the reference's exporter computes it:
  * ProcessLeaf, gNanoVDB/cuda_export_nanovdb.cu:76-129;
  * ProcessInternalNode and its launch, cuda_export_nanovdb.cu:241-362, with
    getChild, gvdb_library/kernels/cuda_gvdb_nodes.cuh:115-124;
  * ProcessGridExtents, gNanoVDB/gvdb_export_nanovdb.cpp:204-327;
  * the grid and tree fields of ExportToNanoVDB, gvdb_export_nanovdb.cpp:
    379-700, with the transform SetTransform builds (gvdb_volume_gvdb.cpp:
    5770-5798; Matrix4F in gvdb_vec.cpp:218-281 and 487-498).
`parse(buf)` reads such a buffer back into its fields.

One departure, shared with the product: a leaf that an incremental rebuild
left stale has no atlas brick and is written as zeros (the reference reads
the atlas at its old position; its comment at cuda_export_nanovdb.cu:84-86
means such nodes to be ignored).

Parity unpinned against the reference's own exporter: it compiles only with
NanoVDB's headers, which are not present, so no buffer it wrote pins this
restatement; it follows the exporter's source line by line.

`st` is a dict: logdim (levels 0..2 at least), nodes[l] (NODE_DTYPE),
clists[l] ((count, res^3) uint64, l >= 1), leaf_slot (atlas slot per pool
leaf, -1 when stale), tiles (per channel, (slots, t, t, t) as z, y, x),
apron, transform ((pre-translation, angles, scale, translation)).
`state_of` builds it from an oracle volume.
"""
import ctypes
import ctypes.util
import math
import struct

import numpy as np

MAGIC = 0x31564E3242445647  # "GVDB2NV1"
NV_FLOAT, NV_VEC3F = 1, 3
HEADER = 64
FLT_MAX = float(np.finfo(np.float32).max)
FLT_MIN = float(np.finfo(np.float32).tiny)  # numeric_limits<float>::min()
INT_MAX, INT_MIN = 2 ** 31 - 1, -2 ** 31
MASK64 = (1 << 64) - 1
UNDEFL = 0xFFFFFFFF

GRID_FMT = "<QQII3iI3Q4Q4Q256s16f3d6dQII6i3f3f3f12x"
assert struct.calcsize(GRID_FMT) == 608
LEAF_HDR = np.dtype([("bbox_min", "<i4", 3), ("bbox_dif", "u1", 3), ("flags", "u1"), ("vmin", "<f4", 3),
                     ("vmax", "<f4", 3), ("pad", "<u4", 6)])
NODE_HDR = np.dtype([("bbox_min", "<i4", 3), ("bbox_max", "<i4", 3), ("offset", "<u4"), ("flags", "<u4"),
                     ("vmin", "<f4", 3), ("vmax", "<f4", 3), ("pad", "<u4", 2)])
TILE = np.dtype([("key", "<u8"), ("child", "<u4"), ("state", "<u4")])
assert LEAF_HDR.itemsize == NODE_HDR.itemsize == HEADER and TILE.itemsize == 16

_libm = ctypes.CDLL(ctypes.util.find_library("m"))
for _f in ("cosf", "sinf"):
    getattr(_libm, _f).restype = ctypes.c_float
    getattr(_libm, _f).argtypes = [ctypes.c_float]


def _r32(x):
    return (x + 31) & ~31


def leaf_record(ld, nv):
    t3 = 1 << (3 * ld)
    return _r32(HEADER + t3 // 8 + t3 * 4 * nv)


def node_record(ld, nv):
    t3 = 1 << (3 * ld)
    return _r32(HEADER + t3 // 4 + t3 * 4 * nv)


def layout(logdim, counts, nv):
    """Record sizes and section offsets: (rec[3], sec[4] = leaves, level-1,
    level-2, tiles, total)."""
    rec = [leaf_record(logdim[0], nv), node_record(logdim[1], nv), node_record(logdim[2], nv)]
    sec3 = 608
    sec2 = _r32(sec3 + 16 * counts[2])
    sec1 = sec2 + rec[2] * counts[2]
    sec0 = sec1 + rec[1] * counts[1]
    return rec, [sec0, sec1, sec2, sec3], sec0 + rec[0] * counts[0]


def transform_matrix(transform):
    """mXform = T R S PT as SetTransform builds it, column-major, float32."""
    pt, ang, sc, t = [[np.float32(x) for x in part] for part in transform]
    k = np.float32(3.141592) / np.float32(180.0)  # DEGtoRAD, gvdb_types.h:59
    cx, sx = np.float32(_libm.cosf(ang[0] * k)), np.float32(_libm.sinf(ang[0] * k))
    cy, sy = np.float32(_libm.cosf(ang[1] * k)), np.float32(_libm.sinf(ang[1] * k))
    cz, sz = np.float32(_libm.cosf(ang[2] * k)), np.float32(_libm.sinf(ang[2] * k))
    z = np.float32(0)
    d = [cy * cz, cy * sz, -sy, z,
         cz * sx * sy - cx * sz, cx * cz + sx * sy * sz, cy * sx, z,
         cx * cz * sy + sx * sz, -cz * sx + cx * sy * sz, cx * cy, z,
         t[0], t[1], t[2], np.float32(1)]
    for i in range(3):
        d[i + 0] = d[i + 0] * sc[0]
        d[i + 4] = d[i + 4] * sc[1]
        d[i + 8] = d[i + 8] * sc[2]
    for r in range(3):
        d[12 + r] = d[12 + r] + (d[r] * pt[0] + d[4 + r] * pt[1] + d[8 + r] * pt[2])
    return np.array(d, np.float32)


def state_of(o, chans, transform=((0, 0, 0), (0, 0, 0), (1, 1, 1), (0, 0, 0))):
    n0 = o.pool_count(0)
    leaf_slot = np.full(n0, -1, np.int64)
    amap = o.atlas_map()
    for s in range(o.atlas_slots()):
        leaf_slot[int(amap[s]["mLeafID"])] = s
    return dict(logdim=[int(o.res(l)).bit_length() - 1 for l in range(3)], nodes=[o.nodes(l) for l in range(3)],
                clists=[None] + [o.childlists(l) for l in (1, 2)], leaf_slot=leaf_slot,
                tiles=[o.atlas(c).astype(np.float32) for c in chans], apron=int(o.apron()), transform=transform)


def _leaves(st, nv, rec):
    """ProcessLeaf per pool leaf: records (n, rec) uint8."""
    T = 1 << st["logdim"][0]
    t3 = T ** 3
    nodes = st["nodes"][0]
    n = len(nodes)
    out = np.zeros((n, rec), np.uint8)
    a = st["apron"]
    slots = st["leaf_slot"]
    live = np.nonzero(slots >= 0)[0]
    if len(live) == 0:
        return out
    # interior of each live leaf's tile, (leaf, z, y, x) -> (leaf, x, y, z): values[(x*T + y)*T + z]
    vals = np.stack([tl[slots[live]][:, a:a + T, a:a + T, a:a + T].transpose(0, 3, 2, 1).reshape(len(live), t3)
                     for tl in st["tiles"][:nv]], axis=2)  # (leaf, voxel, component)
    hdr = np.zeros(len(live), LEAF_HDR)
    hdr["bbox_min"] = nodes["mPos"][live]
    hdr["bbox_dif"] = T
    hdr["vmin"][:, :nv] = np.fmin.reduce(vals, axis=1, initial=FLT_MAX)
    hdr["vmax"][:, :nv] = np.fmax.reduce(vals, axis=1, initial=-FLT_MAX)
    rows = out[live]
    rows[:, :HEADER] = hdr.view(np.uint8).reshape(len(live), HEADER)
    rows[:, HEADER:HEADER + t3 // 8] = 0xFF  # every voxel active
    v0 = HEADER + t3 // 8
    rows[:, v0:v0 + t3 * 4 * nv] = np.ascontiguousarray(vals, np.float32).view(np.uint8).reshape(len(live), -1)
    out[live] = rows
    return out


def _child_ranges(recs, is_leaf):
    """(box min, box max, vmin, vmax) of child records: a leaf's box is
    corner .. corner + stored extent (LeafNode::bbox), a node's its box."""
    if is_leaf:
        h = recs[:, :HEADER].copy().view(LEAF_HDR).ravel()
        lo = h["bbox_min"].astype(np.int64)
        return lo, lo + h["bbox_dif"].astype(np.int64), h["vmin"], h["vmax"]
    h = recs[:, :HEADER].copy().view(NODE_HDR).ravel()
    return h["bbox_min"].astype(np.int64), h["bbox_max"].astype(np.int64), h["vmin"], h["vmax"]


def _nodes(st, lev, nv, rec, child_recs, background):
    """ProcessInternalNode per pool node of a level: records (n, rec) uint8."""
    T = 1 << st["logdim"][lev]
    t3 = T ** 3
    nodes = st["nodes"][lev]
    n = len(nodes)
    out = np.zeros((n, rec), np.uint8)
    bmin, bmax, cvmin, cvmax = _child_ranges(child_recs, lev == 1) if len(child_recs) else (None,) * 4
    for i in range(n):
        cl = int(nodes["mChildList"][i])
        if cl == UNDEFL:
            continue  # every field 0
        entries = st["clists"][lev][cl >> 16]
        # GVDB order (z*T + y)*T + x -> NanoVDB order (x*T + y)*T + z
        nano = entries.reshape(T, T, T).transpose(2, 1, 0).ravel()
        child = ((nano >> np.uint64(16)) & np.uint64(0xFFFFFFFF)).astype(np.uint32).view(np.int32)  # (int)(e >> 16)
        has = child != -1
        table = np.zeros((t3, nv), np.float32)
        table[~has] = np.asarray(background[:nv], np.float32)
        tv = table.view(np.uint32)
        tv[has, 0] = child[has].view(np.uint32)
        lo = np.full(nv, FLT_MAX, np.float32)
        hi = np.full(nv, -FLT_MAX, np.float32)
        blo = np.full(3, INT_MAX, np.int64)
        bhi = np.full(3, -INT_MAX, np.int64)
        c = child[has]
        if len(c):
            lo = np.fmin.reduce(cvmin[c, :nv], axis=0, initial=FLT_MAX).astype(np.float32)
            hi = np.fmax.reduce(cvmax[c, :nv], axis=0, initial=-FLT_MAX).astype(np.float32)
            blo = np.minimum(blo, bmin[c].min(axis=0))
            bhi = np.maximum(bhi, bmax[c].max(axis=0))
        h = np.zeros(1, NODE_HDR)
        h["bbox_min"], h["bbox_max"] = blo, bhi
        h["offset"] = n - i
        h["vmin"][0, :nv], h["vmax"][0, :nv] = lo, hi
        row = out[i]
        row[:HEADER] = h.view(np.uint8)
        # value mask all off (already 0), then the child mask
        row[HEADER + t3 // 8:HEADER + t3 // 4] = np.packbits(has, bitorder="little")
        row[HEADER + t3 // 4:HEADER + t3 // 4 + t3 * 4 * nv] = table.view(np.uint8).ravel()
    return out


def tile_key(corner, shift):
    """Tile::setChild's key through RootData::CoordToKey, as the exporter
    writes it (gvdb_export_nanovdb.cpp:271-276): each int32 corner component
    shifted right (arithmetic), converted to uint64 (a negative one
    sign-extends over the higher fields), z | y << 21 | x << 42."""
    f = [(int(c) >> shift) & MASK64 for c in corner]
    return f[2] | (f[1] << 21 & MASK64) | (f[0] << 42 & MASK64)


def export(st, background=(0.0, 0.0, 0.0), grid_name="", grid_class=0, nv=NV_FLOAT):
    """The whole buffer, as bytes."""
    ld = st["logdim"][:3]
    counts = [len(st["nodes"][l]) for l in range(3)]
    rec, sec, total = layout(ld, counts, nv)
    bg = list(np.broadcast_to(np.asarray(background, np.float32), (3,)).astype(np.float32))
    leaves = _leaves(st, nv, rec[0])
    n1 = _nodes(st, 1, nv, rec[1], leaves, bg)
    n2 = _nodes(st, 2, nv, rec[2], n1, bg)

    # ProcessGridExtents: one tile per level-2 node, then the root's box and range
    shift = sum(ld)
    h2 = n2[:, :HEADER].copy().view(NODE_HDR).ravel() if counts[2] else np.zeros(0, NODE_HDR)
    tiles = np.zeros(counts[2], TILE)
    bb = [INT_MAX] * 3 + [INT_MIN] * 3
    lo = [FLT_MAX] * 3
    hi = [FLT_MIN if nv == NV_FLOAT else -FLT_MAX, -FLT_MAX, -FLT_MAX]
    for i in range(counts[2]):
        m = [int(x) for x in h2["bbox_min"][i]]
        tiles[i] = (tile_key(m, shift), i, 0)
        for a in range(3):
            bb[a] = min(bb[a], m[a])
            bb[3 + a] = max(bb[3 + a], int(h2["bbox_max"][i][a]))
        for c in range(nv):
            x, y = float(h2["vmin"][i][c]), float(h2["vmax"][i][c])
            lo[c] = lo[c] if lo[c] < x else x  # ExportToNanoVDB_Min: a < b ? a : b
            hi[c] = hi[c] if hi[c] > y else y
    tiles = tiles[np.argsort(tiles["key"], kind="stable")]

    M = transform_matrix(st["transform"])
    Md = [float(x) for x in M]
    vs = [math.sqrt(Md[4 * a] * Md[4 * a] + Md[4 * a + 1] * Md[4 * a + 1] + Md[4 * a + 2] * Md[4 * a + 2])
          for a in range(3)]
    wb = [FLT_MAX] * 3 + [-FLT_MAX] * 3
    for k in range(8):
        p = [float(bb[3 if k & 1 else 0]), float(bb[4 if k & 2 else 1]), float(bb[5 if k & 4 else 2])]
        for a in range(3):
            w = Md[a] * p[0] + Md[4 + a] * p[1] + Md[8 + a] * p[2] + Md[12 + a]
            wb[a] = w if w < wb[a] else wb[a]
            wb[3 + a] = w if w > wb[3 + a] else wb[3 + a]
    pad3 = lambda xs: [float(np.float32(x)) for x in xs[:nv]] + [0.0] * (3 - nv)
    name = grid_name.encode()[:255]
    grid = struct.pack(GRID_FMT, MAGIC, total, nv, grid_class & 0xFFFFFFFF, *ld, 0, *rec, *sec, *counts, 1,
                       name, *[float(x) for x in M], *vs, *wb, counts[0] << (3 * ld[0]), counts[2], 0, *bb,
                       *pad3(bg), *pad3(lo), *pad3(hi))
    out = bytearray(total)
    out[:608] = grid
    out[608:608 + 16 * counts[2]] = tiles.tobytes()
    for s, recs in ((sec[2], n2), (sec[1], n1), (sec[0], leaves)):
        out[s:s + recs.size] = recs.tobytes()
    return bytes(out)


def parse(buf):
    """Fields of a buffer: the grid header as a dict, tiles, and the three
    record arrays (headers as structured arrays, bodies as raw bytes)."""
    buf = bytes(buf)
    f = struct.unpack_from(GRID_FMT, buf, 0)
    keys = (["magic", "total_bytes", "value_type", "grid_class"] + [("log2dim", 3)] + ["pad0", ("record_bytes", 3),
            ("section", 4), ("count", 4), "name", ("index_to_world", 16), ("voxel_size", 3), ("world_bbox", 6),
            "active_voxels", "tile_count", "pad1", ("bbox", 6), ("background", 3), ("vmin", 3), ("vmax", 3)])
    g, i = {}, 0
    for k in keys:
        if isinstance(k, tuple):
            g[k[0]] = tuple(f[i:i + k[1]])
            i += k[1]
        else:
            g[k] = f[i]
            i += 1
    cnt, rec, sec = g["count"], g["record_bytes"], g["section"]
    out = dict(grid=g, tiles=np.frombuffer(buf, TILE, cnt[2], sec[3]))
    for l, dt in ((0, LEAF_HDR), (1, NODE_HDR), (2, NODE_HDR)):
        raw = np.frombuffer(buf, np.uint8, cnt[l] * rec[l], sec[l]).reshape(cnt[l], rec[l])
        out[f"rec{l}"] = raw
        out[f"hdr{l}"] = raw[:, :HEADER].copy().view(dt).ravel()
    return out
