"""VBX files, restated in numpy: test infrastructure (the oracle), not the
product.

`write(path, st)` lays out the bytes that VolumeGVDB::SaveVBX
(gvdb_volume_gvdb.cpp:1626-1768) writes for file version 1.11, and
`read(path)` parses them as LoadVBX (gvdb_volume_gvdb.cpp:507-685) does.
The format is GVDB_FILESPEC.txt, with the two places where the reference's
writer departs from that text followed as the writer has them: a channel
count (int) sits between the brick apron and the atlas size, and each
channel's atlas is preceded by its type and stride (two ints).  The grid
name is written as zeros (the reference writes an uninitialised buffer).

Parity unpinned: the reference ships no VBX file and its host library does
not build here, so no file the reference wrote pins this restatement; it
follows the writer's and reader's source line by line.

`st` is a dict: transform (4 x 3 floats: pre-translation, angles, scale,
translation), logdim[5], range[5], apron, depth, nodes[5] (NODE_DTYPE
arrays), clists[5] (uint64 arrays, (count, res^3); level 0 unused), subdim
(atlas brick counts), tiles (per channel, float32 (slots, T, T, T) as z, y,
x).  `state_of` builds it from an oracle volume.
"""
import struct

import numpy as np

from oracle import NODE_DTYPE

MAJOR, MINOR = 1, 11
T_FLOAT = 3


def state_of(o, nchan, transform=((0, 0, 0), (0, 0, 0), (1, 1, 1), (0, 0, 0))):
    logdim = [int(o.res(l)).bit_length() - 1 for l in range(5)]
    return dict(transform=transform, logdim=logdim, range=[int(o.range(l)) for l in range(5)], apron=int(o.apron()),
                depth=int(o.depth()), nodes=[o.nodes(l) for l in range(5)],
                clists=[np.zeros((0, 0), np.uint64)] + [o.childlists(l) for l in range(1, 5)],
                subdim=tuple(o.atlas_subdim()), tiles=[o.atlas(c).astype(np.float32) for c in range(nchan)])


def atlas_3d(tiles, subdim, t):
    """Slot-major tiles -> the atlas volume (z, y, x); slot s at brick
    (s mod nx, (s / nx) mod ny, s / (nx ny)) (UpdateAtlas, V:2630-2704)."""
    nx, ny, nz = subdim
    a = np.zeros((nz * t, ny * t, nx * t), np.float32)
    for s in range(len(tiles)):
        bx, by, bz = s % nx, (s // nx) % ny, s // (nx * ny)
        a[bz * t:(bz + 1) * t, by * t:(by + 1) * t, bx * t:(bx + 1) * t] = tiles[s]
    return a


def write(path, st):
    res = [1 << d for d in st["logdim"]]
    t = res[0] + 2 * st["apron"]
    nx, ny, nz = st["subdim"]
    ar = (nx * t, ny * t, nz * t)
    out = bytearray()
    out += struct.pack("<BB", MAJOR, MINOR)
    for part in st["transform"]:  # pre-translation, angles, scale, translation
        out += struct.pack("<3f", *part)
    out += struct.pack("<i", 1)  # grids
    table = len(out)
    out += struct.pack("<Q", 0)
    grid = len(out)
    out += bytes(256)  # grid name
    out += struct.pack("<ccc", b"f", b"\x01", b"\x00")  # type, components, compression
    out += struct.pack("<3f", 1, 1, 1)  # voxel size
    out += struct.pack("<i", len(st["nodes"][0]))  # leaf count
    out += struct.pack("<3i", res[0], res[0], res[0])
    out += struct.pack("<i", st["apron"])
    out += struct.pack("<i", len(st["tiles"]))  # channels
    out += struct.pack("<Q", ar[0] * ar[1] * ar[2] * 4)  # one channel's atlas bytes
    out += struct.pack("<cic", b"\x02", 0, b"\x00")  # topology type, reuse, layout
    out += struct.pack("<3i", nx, ny, nz)
    out += struct.pack("<3i", *ar)
    out += struct.pack("<iQ", 5, st["depth"] << 8)  # levels, root Elem(0, depth, 0)
    for l in range(5):
        n = len(st["nodes"][l])
        out += struct.pack("<5i", st["logdim"][l], res[l], st["range"][l], st["range"][l], st["range"][l])
        out += struct.pack("<4i", n, 64, n if l > 0 else 0, 8 * res[l] ** 3 if l > 0 else 0)
    for l in range(5):
        out += np.ascontiguousarray(st["nodes"][l], NODE_DTYPE).tobytes()
    for l in range(1, 5):
        out += np.ascontiguousarray(st["clists"][l], np.uint64).tobytes()
    for tiles in st["tiles"]:
        out += struct.pack("<ii", T_FLOAT, 4)
        out += atlas_3d(tiles, st["subdim"], t).tobytes()
    struct.pack_into("<Q", out, table, grid)
    with open(path, "wb") as f:
        f.write(out)


def read(path):
    with open(path, "rb") as f:
        b = f.read()
    p = [0]

    def take(fmt):
        v = struct.unpack_from("<" + fmt, b, p[0])
        p[0] += struct.calcsize("<" + fmt)
        return v

    major, minor = take("BB")
    transform = tuple(take("3f") for _ in range(4)) if (major == 1 and minor >= 11) or major > 1 else None
    (grids,) = take("i")
    if major >= 2:
        take("B")
    offs = take(f"{grids}Q")
    p[0] = offs[0]
    name = b[p[0]:p[0] + 256]
    p[0] += 256
    dtype, comps, compress = take("ccc")
    voxelsize = take("3f")
    (leafcnt,) = take("i")
    leafdim = take("3i")
    (apron,) = take("i")
    (nchan,) = take("i")
    (atlas_bytes,) = take("Q")
    topo, reuse, layout = take("cic")
    subdim = take("3i")
    ar = take("3i")
    levels, root = take("iQ")
    lv = [take("9i") for _ in range(levels)]
    nodes, clists = [], []
    for l in range(levels):
        n, w = lv[l][5], lv[l][6]
        nodes.append(np.frombuffer(b, NODE_DTYPE, n, p[0]).copy())
        p[0] += n * w
    for l in range(levels):
        n, w = lv[l][7], lv[l][8]
        clists.append(np.frombuffer(b, np.uint64, n * w // 8, p[0]).copy().reshape(n, w // 8) if n else
                      np.zeros((0, 0), np.uint64))
        p[0] += n * w
    atlases = []
    for _ in range(nchan):
        ctype, stride = take("ii")
        cnt = ar[0] * ar[1] * ar[2]
        atlases.append(np.frombuffer(b, np.float32, cnt, p[0]).copy().reshape(ar[2], ar[1], ar[0]))
        p[0] += cnt * stride
    return dict(major=major, minor=minor, transform=transform, grids=grids, offsets=offs, name=name,
                dtype=dtype, components=comps, compression=compress, voxelsize=voxelsize, leafcnt=leafcnt,
                leafdim=leafdim, apron=apron, nchan=nchan, atlas_bytes=atlas_bytes, topology=topo, reuse=reuse,
                layout=layout, subdim=subdim, atlas_res=ar, levels=levels, root=root, level_table=lv, nodes=nodes,
                clists=clists, atlases=atlases, end=p[0], size=len(b))
