// topology.cu -- dynamic topology rebuild and atlas assignment on device.
//
// Reference behaviour restated (paths relative to gvdb-voxels):
//   RebuildTopology state machine     V:1181-1218
//   GetBoundingBox / DetermineDepth   V:5404-5467, V:821-837, V:2915-2931
//   full rebuild (ActivateBricksGPU)  V:1229-1413, P:352-382, V:843-873
//   extra bricks (radius >= 1)        V:931-1016, P:467-512
//   incremental (ActivateIncre...)    V:1020-1156, P:420-465, N:401-467
//   node set-up / links               V:2512-2524, N:470-505
//   UpdateAtlas                       V:2630-2704, A:692-715
//
// The reference sorts N*depth 64-bit keys with Thrust and then allocates
// nodes in a host loop.  Here every point inserts its level-0 brick (and,
// for radius >= 1, the bricks of its activation box) into device hash
// sets; only the unique bricks are sorted, parent levels are derived from
// them, and node pools, child lists and links are written by kernels in
// the reference's exact pool order: per level, sorted base keys, then
// sorted extra keys.  Keys are packed as x<<2b | y<<b | z with b bits per
// axis, which orders them exactly like the reference's (lev,x,y,z) keys.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "dev_common.cuh"

namespace gvdb2 {

namespace {

struct SmallWords { // layout of Volume::dev_small
    int32_t bbox[6];
    int32_t count[8];
    int32_t status;
    int32_t splat_guard[5]; // a splat kernel's failed index check: code, index (hi, lo), bound (hi, lo)
    int32_t pad[12];
};
static_assert(sizeof(SmallWords) == 128, "small word block");

__device__ __forceinline__ int32_t f2ord(float f) {
    int32_t i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
inline float ord2f(int32_t o) {
    int32_t i = o >= 0 ? o : o ^ 0x7FFFFFFF;
    float f;
    std::memcpy(&f, &i, 4);
    return f;
}

// GetBoundingBox (V:5404-5467): min/max of pos + trans over all points.
__global__ void k_bbox(PointsView pos, int64_t n, float3 t, int32_t *bbox) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float3 p = load_f3(pos, i);
        const int3 o = point_origin(pos, i); // batched clouds: the bounds are only sizes, so float is enough
        float w[3] = {p.x + t.x + (float)o.x, p.y + t.y + (float)o.y, p.z + t.z + (float)o.z};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            mn[a] = fminf(mn[a], w[a]);
            mx[a] = fmaxf(mx[a], w[a]);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
    }
    __shared__ float smn[3][32], smx[3][32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0)
        for (int a = 0; a < 3; a++) {
            smn[a][warp] = mn[a];
            smx[a][warp] = mx[a];
        }
    __syncthreads();
    if (warp == 0) {
        for (int a = 0; a < 3; a++) {
            float x = lane < nw ? smn[a][lane] : INFINITY;
            float y = lane < nw ? smx[a][lane] : -INFINITY;
            for (int o = 16; o > 0; o >>= 1) {
                x = fminf(x, __shfl_xor_sync(0xffffffffu, x, o));
                y = fmaxf(y, __shfl_xor_sync(0xffffffffu, y, o));
            }
            if (lane == 0) {
                atomicMin(&bbox[a], f2ord(x));
                atomicMax(&bbox[3 + a], f2ord(y));
            }
        }
    }
}


// Per point: its level-0 brick into the base set; for radius >= 1 every
// level-0 brick of the activation box [int(w)-r, int(w)+k*r] (P:481-482 /
// P:433-434) into the box set.  Box bricks outside the root node are
// skipped (the reference reads past its child list there).
__global__ void k_mark_keys(PointsView pos, int64_t n, float3 orig, float radius, float kmax, int do_box, KeyGeom g,
                            uint64_t *hs_base, uint64_t *hs_box, uint32_t mask, int32_t *counts, int32_t *status) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = i < n;
    float w[3] = {0, 0, 0};
    int oo[3] = {0, 0, 0};
    if (valid) {
        float3 p = load_f3(pos, i);
        w[0] = p.x + orig.x;
        w[1] = p.y + orig.y;
        w[2] = p.z + orig.z;
        if (w[0] < 0 || w[1] < 0 || w[2] < 0) valid = false;
        const int3 o = point_origin(pos, i);
        oo[0] = o.x;
        oo[1] = o.y;
        oo[2] = o.z;
    }
    unsigned act = __ballot_sync(0xffffffffu, valid);
    if (!valid) return;
    int bx = ((int)w[0] + oo[0]) >> g.log2r0, by = ((int)w[1] + oo[1]) >> g.log2r0, bz = ((int)w[2] + oo[2]) >> g.log2r0;
    bool inside = bx >= g.lo[0] && bx < g.lo[0] + g.span && by >= g.lo[1] && by < g.lo[1] + g.span &&
                  bz >= g.lo[2] && bz < g.lo[2] + g.span;
    uint64_t key = inside ? pack_key(bx, by, bz, g.b) : kEmptyKey;
    // warp de-duplication: one insert per distinct key
    unsigned peers = __match_any_sync(act, key);
    if (inside && (int)(threadIdx.x & 31) == __ffs(peers) - 1) {
        int r = hs_insert(hs_base, mask, key);
        if (r > 0) atomicAdd(&counts[0], 1);
        if (r < 0) atomicOr(status, kDevHashFull);
    }
    if (!do_box) return;
    int lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
        int iw = (int)w[a];
        int bmin = (int)((float)iw - radius);
        int bmax = (int)((float)iw + kmax * radius);
        int l = ((bmin < 0 ? 0 : bmin) + oo[a]) >> g.log2r0; // clamped in the cloud's own space
        int h = (bmax + oo[a]) >> g.log2r0;
        l = max(l, g.lo[a]);
        h = min(h, g.lo[a] + g.span - 1);
        lo[a] = l;
        hi[a] = h;
    }
    for (int x = lo[0]; x <= hi[0]; x++)
        for (int y = lo[1]; y <= hi[1]; y++)
            for (int z = lo[2]; z <= hi[2]; z++) {
                uint64_t k = pack_key(x, y, z, g.b);
                int r = hs_insert(hs_box, mask, k);
                if (r > 0) atomicAdd(&counts[1], 1);
                if (r < 0) atomicOr(status, kDevHashFull);
            }
}

__global__ void k_compact_set(const uint64_t *hs, uint32_t cap, uint64_t *out, int32_t *count) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t k = hs[i];
        bool has = k != kEmptyKey;
        unsigned m = __ballot_sync(__activemask(), has);
        if (has) {
            int leader = __ffs(m) - 1;
            int base = 0;
            if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(count, __popc(m));
            base = __shfl_sync(m, base, leader);
            out[base + __popc(m & lanemask_lt())] = k;
        }
    }
}

// keys -> parent keys one level up (shift s bits per axis)
__global__ void k_parentize(const uint64_t *in, int64_t n, int b, int s, uint64_t *out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int x, y, z;
    unpack_key(in[i], b, x, y, z);
    out[i] = pack_key(x >> s, y >> s, z >> s, b);
}

// flags[i] = 1 if keys[i] starts a run (sorted input)
__global__ void k_run_heads(const uint64_t *keys, int64_t n, uint32_t *flags) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__device__ __forceinline__ int64_t bsearch_key(const uint64_t *a, int64_t n, uint64_t k) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (a[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    return (lo < n && a[lo] == k) ? lo : -1;
}

// flags[i] = 1 if keys[i] is not in the sorted set `ref`
__global__ void k_not_in(const uint64_t *keys, int64_t n, const uint64_t *ref, int64_t nref, uint32_t *flags) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = bsearch_key(ref, nref, keys[i]) < 0 ? 1u : 0u;
}

__global__ void k_compact_flagged(const uint64_t *in, int64_t n, const uint32_t *flags, const uint32_t *scan,
                                  uint64_t *out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (flags[i]) out[scan[i]] = in[i];
}

// The root node (V:1290-1300): level `depth`, flags 1, child list Elem(1,depth,0).
__global__ void k_root(Node *root, int depth, int3 rootpos) {
    Node nd;
    memset(&nd, 0, sizeof(nd));
    nd.mLev = (uint8_t)depth;
    nd.mFlags = 1;
    nd.mPos[0] = rootpos.x;
    nd.mPos[1] = rootpos.y;
    nd.mPos[2] = rootpos.z;
    nd.mValue[0] = nd.mValue[1] = nd.mValue[2] = -1;
    nd.mParent = kUndefL;
    nd.mChildList = elem(1, depth, 0);
    *root = nd;
}

struct LevelBuild {
    const uint64_t *base; int64_t nbase;  // sorted base keys at this level
    const uint64_t *extra; int64_t nextra;
    const uint64_t *pbase; int64_t npbase; // parent level
    const uint64_t *pextra; int64_t npextra;
    Node *nodes;
    uint64_t *pclist;      // parent level child lists
    int lev, depth, b;
    int64_t range;         // node extent at this level (voxels)
    int shift;             // log2 res(lev+1)
    int pres;              // res(lev+1)
    int64_t pres3;
    int root_lo[3];        // root corner in units of this level's range (for lev == depth-1)
    uint64_t *leaf_keys; int32_t *leaf_vals; uint32_t leaf_mask; // level 0 only
    int32_t *status;
};

// SetupNode (V:2512-2524) for every node of one level, then the link of
// gvdbLinkBricks (N:470-505): mParent = Elem(0,lev+1,pid) and the parent's
// child slot (z*res+y)*res+x = Elem(0,lev,i).  Parents are found by key in
// the parent level's sorted arrays, which is the node getParent reaches.
__global__ void k_build_link(LevelBuild L) {
    int64_t n = L.nbase + L.nextra;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t key = i < L.nbase ? L.base[i] : L.extra[i - L.nbase];
    int x, y, z;
    unpack_key(key, L.b, x, y, z);
    Node nd;
    memset(&nd, 0, sizeof(nd));
    nd.mLev = (uint8_t)L.lev;
    nd.mFlags = 1;
    nd.mPos[0] = (int32_t)(x * L.range);
    nd.mPos[1] = (int32_t)(y * L.range);
    nd.mPos[2] = (int32_t)(z * L.range);
    nd.mValue[0] = nd.mValue[1] = nd.mValue[2] = -1;
    nd.mParent = kUndefL;
    nd.mChildList = L.lev > 0 ? elem(1, L.lev, (uint64_t)i) : kUndefL;
    int ox, oy, oz; // parent corner in units of this level's range
    int64_t pid;
    if (L.lev == L.depth - 1) {
        pid = 0;
        ox = L.root_lo[0];
        oy = L.root_lo[1];
        oz = L.root_lo[2];
    } else {
        int px = x >> L.shift, py = y >> L.shift, pz = z >> L.shift;
        uint64_t pk = pack_key(px, py, pz, L.b);
        pid = bsearch_key(L.pbase, L.npbase, pk);
        if (pid < 0) {
            pid = bsearch_key(L.pextra, L.npextra, pk);
            if (pid >= 0) pid += L.npbase;
        }
        ox = px << L.shift;
        oy = py << L.shift;
        oz = pz << L.shift;
    }
    int lx = x - ox, ly = y - oy, lz = z - oz;
    if (pid >= 0 && lx >= 0 && lx < L.pres && ly >= 0 && ly < L.pres && lz >= 0 && lz < L.pres) {
        nd.mParent = elem(0, L.lev + 1, (uint64_t)pid);
        int64_t bit = ((int64_t)lz * L.pres + ly) * L.pres + lx;
        L.pclist[pid * L.pres3 + bit] = elem(0, L.lev, (uint64_t)i);
        if (L.lev == 0 && hm_insert(L.leaf_keys, L.leaf_vals, L.leaf_mask, key, (int32_t)i) < 0)
            atomicOr(L.status, kDevHashFull);
    } else {
        atomicOr(L.status, kDevBadIndex);
    }
    L.nodes[i] = nd;
}

// ---- UpdateAtlas --------------------------------------------------------
__global__ void k_leaf_flags(const Node *leaves, int64_t n, uint32_t *flags) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = leaves[i].mFlags ? 1u : 0u;
}

// ComputeBounds (V:1792-1816): min of the flagged leaves' corners and max of
// their far corners (corner + range(0)), both seeded with leaf 0's corner
// whatever its flag, as the reference seeds them.  out[0..3) min, out[3..6)
// max; a block reduces its leaves before one atomic per word.
__global__ void k_leaf_bounds(const Node *leaves, int64_t n, int range0, int32_t *out) {
    __shared__ int32_t red[6];
    if (threadIdx.x < 6) red[threadIdx.x] = threadIdx.x < 3 ? INT32_MAX : INT32_MIN;
    __syncthreads();
    int32_t lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const Node &nd = leaves[i];
        if (i == 0)
            for (int a = 0; a < 3; a++) lo[a] = min(lo[a], nd.mPos[a]), hi[a] = max(hi[a], nd.mPos[a]);
        if (!nd.mFlags) continue;
        for (int a = 0; a < 3; a++) lo[a] = min(lo[a], nd.mPos[a]), hi[a] = max(hi[a], nd.mPos[a] + range0);
    }
    for (int a = 0; a < 3; a++) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    if ((threadIdx.x & 31) == 0)
        for (int a = 0; a < 3; a++) atomicMin(&red[a], lo[a]), atomicMax(&red[3 + a], hi[a]);
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&out[threadIdx.x], red[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&out[threadIdx.x], red[threadIdx.x]);
}

// AtlasAlloc + getAtlasPos (A:692-715) and AssignMapping (V:2681-2689).
__global__ void k_atlas_assign(Node *leaves, int64_t n, const uint32_t *flags, const uint32_t *slot, int sx, int sy,
                               int tile, int apron, AtlasNode *amap, int32_t *slot_leaf, int32_t *leaf_slot) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!flags[i]) {
        leaf_slot[i] = -1; // stale leaf keeps its old mValue, as in the reference
        return;
    }
    int64_t s = slot[i];
    int64_t a2 = (int64_t)sx * sy;
    int bz = (int)(s / a2);
    int64_t r = s - (int64_t)bz * a2;
    int by = (int)(r / sx);
    int bx = (int)(r - (int64_t)by * sx);
    Node &nd = leaves[i];
    nd.mValue[0] = bx * tile + apron;
    nd.mValue[1] = by * tile + apron;
    nd.mValue[2] = bz * tile + apron;
    AtlasNode an;
    an.mPos[0] = nd.mPos[0];
    an.mPos[1] = nd.mPos[1];
    an.mPos[2] = nd.mPos[2];
    an.mLeafID = (int32_t)i;
    amap[s] = an;
    slot_leaf[s] = (int32_t)i;
    leaf_slot[i] = (int32_t)s;
}

// 27-neighbour slot table of every active slot (offset k = (dz+1)*9 + (dy+1)*3 + (dx+1)).
__global__ void k_nbr27(const Node *leaves, const int32_t *slot_leaf, int64_t nslots, const int32_t *leaf_slot,
                        const uint64_t *lk, const int32_t *lv, uint32_t lmask, KeyGeom g, int32_t *nbr) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nslots * 27) return;
    int64_t s = t / 27;
    int k = (int)(t - s * 27);
    int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
    const Node &nd = leaves[slot_leaf[s]];
    int bx = (nd.mPos[0] >> g.log2r0) + dx, by = (nd.mPos[1] >> g.log2r0) + dy, bz = (nd.mPos[2] >> g.log2r0) + dz;
    int32_t out = -1;
    if (bx >= g.lo[0] && bx < g.lo[0] + g.span && by >= g.lo[1] && by < g.lo[1] + g.span && bz >= g.lo[2] &&
        bz < g.lo[2] + g.span) {
        int32_t leaf = hm_lookup(lk, lv, lmask, pack_key(bx, by, bz, g.b));
        if (leaf >= 0) out = leaf_slot[leaf];
    }
    nbr[t] = out;
}

// UpdateNeighbors (V:2527-2556): 6 face neighbours per pool leaf
// (-x,-y,-z,+x,+y,+z), -1 when missing.
__global__ void k_nbr6(const Node *leaves, int64_t n, const uint64_t *lk, const int32_t *lv, uint32_t lmask, KeyGeom g,
                       int32_t *nbr) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * 6) return;
    int64_t i = t / 6;
    int k = (int)(t - i * 6);
    const int dir[6][3] = {{-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    const Node &nd = leaves[i];
    int bx = (nd.mPos[0] >> g.log2r0) + dir[k][0], by = (nd.mPos[1] >> g.log2r0) + dir[k][1],
        bz = (nd.mPos[2] >> g.log2r0) + dir[k][2];
    int32_t out = -1;
    if (bx >= g.lo[0] && bx < g.lo[0] + g.span && by >= g.lo[1] && by < g.lo[1] + g.span && bz >= g.lo[2] &&
        bz < g.lo[2] + g.span)
        out = hm_lookup(lk, lv, lmask, pack_key(bx, by, bz, g.b));
    nbr[t] = out;
}

inline uint32_t next_pow2(uint64_t x) {
    uint64_t p = 1;
    while (p < x) p <<= 1;
    return (uint32_t)std::min<uint64_t>(p, 1ull << 31);
}

SmallWords *host_words(Volume *v) { return reinterpret_cast<SmallWords *>(v->host_small); }
SmallWords *dev_words(Volume *v) { return v->dev_small.as<SmallWords>(); }

// The small device words and their pinned mirror, allocated once and zeroed
// (the flags and counters start clear).
gvdb2_status ensure_small_words(Volume *v) {
    if (!v->dev_small.p) {
        GV_CUDA(v, v->dev_small.ensure(sizeof(SmallWords), v->stream));
        GV_CUDA(v, cudaMemsetAsync(v->dev_small.p, 0, sizeof(SmallWords), v->stream));
    }
    if (!v->host_small) GV_CUDA(v, cudaMallocHost(&v->host_small, sizeof(SmallWords)));
    return GVDB2_OK;
}

// The status a full rebuild left in the small words, once they are back on
// the host (build_from_keys defers its check to the next read-back).
gvdb2_status check_pending_status(Volume *v) {
    gvdb2_status st = GVDB2_OK;
    if (v->status_pending) {
        v->status_pending = false;
        const int32_t w = host_words(v)->status;
        if (w & kDevHashFull) st = fail(v, GVDB2_ERR_CAPACITY, "leaf map overflow in the last full rebuild");
        else if (w & kDevBadIndex) st = fail(v, GVDB2_ERR_STATE, "node without parent in the last full rebuild");
    }
    if (v->splat_guard_pending) {
        v->splat_guard_pending = false;
        const int32_t *g = host_words(v)->splat_guard;
        if (g[0]) {
            const long long idx = ((long long)g[1] << 32) | (uint32_t)g[2], lim = ((long long)g[3] << 32) | (uint32_t)g[4];
            const std::string msg = "a splat kernel met a bin or topology index out of range (check " +
                                    std::to_string(g[0]) + ": " + std::to_string(idx) + " not below " +
                                    std::to_string(lim) + "); the cells concerned were skipped";
            memset(host_words(v)->splat_guard, 0, sizeof(host_words(v)->splat_guard));
            GV_CUDA(v, cudaMemsetAsync(dev_words(v)->splat_guard, 0, sizeof(dev_words(v)->splat_guard), v->stream));
            if (st == GVDB2_OK) st = fail(v, GVDB2_ERR_STATE, msg);
        }
    }
    return st;
}


gvdb2_status read_words(Volume *v) {
    GV_CUDA(v, cudaMemcpyAsync(v->host_small, v->dev_small.p, sizeof(SmallWords), cudaMemcpyDeviceToHost, v->stream));
    GV_CUDA(v, cudaStreamSynchronize(v->stream));
    return check_pending_status(v);
}


// sort + unique of a device key array in place; returns the unique count
gvdb2_status sort_unique(Volume *v, uint64_t *keys, int64_t n, int bits, int64_t *out_n) {
    if (n == 0) {
        *out_n = 0;
        return GVDB2_OK;
    }
    GV_TRY(radix_sort_u64(v, keys, nullptr, n, 0, bits));
    uint32_t *flags = nullptr, *scan = nullptr;
    uint64_t *tmp = nullptr;
    cudaStream_t s = v->stream;
    GV_CUDA(v, cudaMallocAsync((void **)&flags, sizeof(uint32_t) * (size_t)(2 * n + 1), s));
    GV_CUDA(v, cudaMallocAsync((void **)&tmp, sizeof(uint64_t) * (size_t)n, s));
    scan = flags + n;
    k_run_heads<<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(keys, n, flags);
    gvdb2_status st = exclusive_scan_u32(v, flags, scan, n);
    if (st == GVDB2_OK) {
        k_compact_flagged<<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(keys, n, flags, scan, tmp);
        uint32_t un = 0;
        cudaError_t e = cudaMemcpyAsync(&un, scan + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(keys, tmp, sizeof(uint64_t) * un, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) st = cuda_fail(v, e, "sort_unique");
        *out_n = un;
    }
    cudaFreeAsync(flags, s);
    cudaFreeAsync(tmp, s);
    return st;
}

// out = keys \ ref (both sorted); stable
gvdb2_status set_difference(Volume *v, const uint64_t *keys, int64_t n, const uint64_t *ref, int64_t nref,
                            uint64_t *out, int64_t *out_n) {
    if (n == 0) {
        *out_n = 0;
        return GVDB2_OK;
    }
    cudaStream_t s = v->stream;
    uint32_t *flags = nullptr;
    GV_CUDA(v, cudaMallocAsync((void **)&flags, sizeof(uint32_t) * (size_t)(2 * n + 1), s));
    uint32_t *scan = flags + n;
    k_not_in<<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(keys, n, ref, nref, flags);
    gvdb2_status st = exclusive_scan_u32(v, flags, scan, n);
    if (st == GVDB2_OK) {
        k_compact_flagged<<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(keys, n, flags, scan, out);
        uint32_t un = 0;
        cudaError_t e = cudaMemcpyAsync(&un, scan + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(v, e, "set_difference");
        *out_n = un;
    }
    cudaFreeAsync(flags, s);
    return st;
}

gvdb2_status clear_pools(Volume *v) { // Clear (V:2487-2503)
    for (int l = 0; l < kMaxLev; l++) v->pool_cnt[l] = 0;
    v->used_leaves = 0;
    v->all_leaves_flagged = false;
    v->atlas_last = 0;
    v->atlas_valid = false;
    v->rebuild_topo = true;
    return GVDB2_OK;
}

gvdb2_status ensure_pool(Volume *v, int lev, int64_t cnt) {
    GV_CUDA(v, v->pool[lev].ensure(sizeof(Node) * (size_t)std::max<int64_t>(cnt, 1), v->stream));
    if (lev > 0) GV_CUDA(v, v->clist[lev].ensure(sizeof(uint64_t) * (size_t)(std::max<int64_t>(cnt, 1) * v->res3(lev)), v->stream));
    return GVDB2_OK;
}

gvdb2_status build_from_keys(Volume *v, const int64_t nB[], const int64_t nE[], const KeyGeom &g);

// Node key sets of the full rebuild through hash sets and radix sorts (any
// extent): lev_keys[l][0] = sorted base keys (nB[l]), lev_keys[l][1] =
// sorted extra keys (nE[l]).
gvdb2_status key_sets_hash(Volume *v, int n, float radius, const float orig[3], const KeyGeom &g, int64_t nB[],
                           int64_t nE[]) {
    cudaStream_t s = v->stream;
    const int depth = v->depth;
    const int kbits = 3 * g.b;
    const bool do_box = radius >= 1.0f;

    // size the hash sets from the bounding box (and the last rebuild)
    int64_t est = 1;
    for (int a = 0; a < 3; a++) est *= (int64_t)((v->posmax[a] - v->posmin[a]) / (float)v->range(0)) + 3;
    est = std::min<int64_t>(est, (int64_t)n * (do_box ? 8 : 1) + 64);
    est = std::max<int64_t>(est, v->lev_count[0][0] + v->lev_count[0][1]);
    uint32_t cap = next_pow2((uint64_t)std::max<int64_t>(2 * est, 1 << 16));

    int64_t nb = 0, nx = 0;
    for (int attempt = 0; attempt < 4; attempt++) {
        GV_CUDA(v, v->hs_keys[0].ensure(sizeof(uint64_t) * cap, s));
        GV_CUDA(v, v->hs_keys[1].ensure(sizeof(uint64_t) * cap, s));
        GV_CUDA(v, cudaMemsetAsync(v->hs_keys[0].p, 0xFF, sizeof(uint64_t) * cap, s));
        if (do_box) GV_CUDA(v, cudaMemsetAsync(v->hs_keys[1].p, 0xFF, sizeof(uint64_t) * cap, s));
        GV_CUDA(v, cudaMemsetAsync(dev_words(v)->count, 0, sizeof(int32_t) * 8 + sizeof(int32_t), s));
        if (n > 0)
            k_mark_keys<<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(
                v->pos, n, make_float3(orig[0], orig[1], orig[2]), radius, 2.0f, do_box ? 1 : 0, g,
                v->hs_keys[0].as<uint64_t>(), v->hs_keys[1].as<uint64_t>(), cap - 1, dev_words(v)->count,
                &dev_words(v)->status);
        GV_CUDA(v, cudaGetLastError());
        GV_TRY(read_words(v));
        nb = host_words(v)->count[0];
        nx = host_words(v)->count[1];
        bool full = (host_words(v)->status & kDevHashFull) || 2 * std::max(nb, nx) > (int64_t)cap;
        if (!full) break;
        if (attempt == 3) return fail(v, GVDB2_ERR_CAPACITY, "brick hash set overflow");
        cap = next_pow2((uint64_t)cap * 4);
    }
    v->hs_mask = cap - 1;

    // per-level sorted unique key arrays: base B[l] and box X[l]
    for (int l = 0; l < depth; l++) {
        GV_CUDA(v, v->lev_keys[l][0].ensure(sizeof(uint64_t) * (size_t)std::max<int64_t>(nb, 1), s));
        GV_CUDA(v, v->lev_keys[l][1].ensure(sizeof(uint64_t) * (size_t)std::max<int64_t>(do_box ? nx : 1, 1), s));
    }
    GV_CUDA(v, v->tmp_a.ensure(sizeof(uint64_t) * (size_t)std::max<int64_t>(nx, 1), s));
    GV_CUDA(v, cudaMemsetAsync(dev_words(v)->count + 2, 0, sizeof(int32_t) * 2, s));
    k_compact_set<<<grid_for(cap, 256, 4096), 256, 0, s>>>(v->hs_keys[0].as<uint64_t>(), cap,
                                                           v->lev_keys[0][0].as<uint64_t>(), dev_words(v)->count + 2);
    if (do_box)
        k_compact_set<<<grid_for(cap, 256, 4096), 256, 0, s>>>(v->hs_keys[1].as<uint64_t>(), cap,
                                                               v->tmp_a.as<uint64_t>(), dev_words(v)->count + 3);
    GV_CUDA(v, cudaGetLastError());
    int64_t nX[kMaxLev] = {0};
    for (int l = 0; l < kMaxLev; l++) nB[l] = nE[l] = 0;
    GV_TRY(radix_sort_u64(v, v->lev_keys[0][0].as<uint64_t>(), nullptr, nb, 0, kbits));
    nB[0] = nb;
    uint64_t *xkeys[kMaxLev] = {nullptr};
    DevBuf xbuf[kMaxLev];
    if (do_box) {
        GV_TRY(radix_sort_u64(v, v->tmp_a.as<uint64_t>(), nullptr, nx, 0, kbits));
        nX[0] = nx;
        xkeys[0] = v->tmp_a.as<uint64_t>();
    }
    for (int l = 1; l < depth; l++) {
        int sh = v->logdim[l];
        uint64_t *dst = v->lev_keys[l][0].as<uint64_t>();
        if (nB[l - 1] > 0)
            k_parentize<<<grid_for(nB[l - 1], 256, 1ll << 31), 256, 0, s>>>(v->lev_keys[l - 1][0].as<uint64_t>(),
                                                                           nB[l - 1], g.b, sh, dst);
        GV_TRY(sort_unique(v, dst, nB[l - 1], kbits, &nB[l]));
        // parents of the previous level's keys; b stays fixed for all levels
        (void)g;
        if (do_box) {
            cudaError_t e = xbuf[l].ensure(sizeof(uint64_t) * (size_t)std::max<int64_t>(nX[l - 1], 1), s);
            if (e != cudaSuccess) {
                for (int q = 0; q < kMaxLev; q++) xbuf[q].release();
                return cuda_fail(v, e, "box keys");
            }
            xkeys[l] = xbuf[l].as<uint64_t>();
            if (nX[l - 1] > 0)
                k_parentize<<<grid_for(nX[l - 1], 256, 1ll << 31), 256, 0, s>>>(xkeys[l - 1], nX[l - 1], g.b, sh,
                                                                               xkeys[l]);
            gvdb2_status st = sort_unique(v, xkeys[l], nX[l - 1], kbits, &nX[l]);
            if (st) {
                for (int q = 0; q < kMaxLev; q++) xbuf[q].release();
                return st;
            }
        }
    }
    // extra keys E[l] = X[l] \ B[l], sorted (ActivateExtraBricksGPU's
    // "not present after the base link" test)
    for (int l = 0; l < depth; l++) {
        nE[l] = 0;
        if (!do_box) continue;
        cudaError_t e = v->lev_keys[l][1].ensure(sizeof(uint64_t) * (size_t)std::max<int64_t>(nX[l], 1), s);
        if (e != cudaSuccess) return cuda_fail(v, e, "extra keys");
        gvdb2_status st = set_difference(v, xkeys[l], nX[l], v->lev_keys[l][0].as<uint64_t>(), nB[l],
                                         v->lev_keys[l][1].as<uint64_t>(), &nE[l]);
        if (st) {
            for (int q = 0; q < kMaxLev; q++) xbuf[q].release();
            return st;
        }
    }
    for (int q = 0; q < kMaxLev; q++) xbuf[q].release();
    return GVDB2_OK;
}

// Pools, child lists, links and the leaf map from the sorted key sets.
gvdb2_status build_from_keys(Volume *v, const int64_t nB[], const int64_t nE[], const KeyGeom &g) {
    cudaStream_t s = v->stream;
    const int depth = v->depth;
    // pools: level l < depth holds [B[l], E[l]]; the root sits at `depth`
    for (int l = 0; l < kMaxLev; l++) v->pool_cnt[l] = 0;
    for (int l = 0; l < depth; l++) v->pool_cnt[l] = nB[l] + nE[l];
    v->pool_cnt[depth] = 1;
    for (int l = 0; l <= depth; l++) {
        GV_TRY(ensure_pool(v, l, v->pool_cnt[l]));
        v->lev_count[l][0] = nB[l];
        v->lev_count[l][1] = nE[l];
        if (l > 0)
            GV_CUDA(v, cudaMemsetAsync(v->clist[l].p, 0xFF, sizeof(uint64_t) * (size_t)(v->pool_cnt[l] * v->res3(l)), s));
    }
    k_root<<<1, 1, 0, s>>>(v->pool_ptr(depth), depth, make_int3(v->root_pos[0], v->root_pos[1], v->root_pos[2]));

    // leaf map: level-0 key -> pool index
    uint32_t lcap = next_pow2((uint64_t)std::max<int64_t>(2 * v->pool_cnt[0], 1 << 12));
    GV_CUDA(v, v->leafmap_keys.ensure(sizeof(uint64_t) * lcap, s));
    GV_CUDA(v, v->leafmap_vals.ensure(sizeof(int32_t) * lcap, s));
    GV_CUDA(v, cudaMemsetAsync(v->leafmap_keys.p, 0xFF, sizeof(uint64_t) * lcap, s));
    v->leafmap_mask = lcap - 1;
    v->leafmap_is_tree = true;
    GV_CUDA(v, cudaMemsetAsync(&dev_words(v)->status, 0, sizeof(int32_t), s));

    for (int l = 0; l < depth; l++) {
        LevelBuild L;
        L.base = v->lev_keys[l][0].as<uint64_t>();
        L.nbase = nB[l];
        L.extra = v->lev_keys[l][1].as<uint64_t>();
        L.nextra = nE[l];
        L.pbase = l + 1 < depth ? v->lev_keys[l + 1][0].as<uint64_t>() : nullptr;
        L.npbase = l + 1 < depth ? nB[l + 1] : 0;
        L.pextra = l + 1 < depth ? v->lev_keys[l + 1][1].as<uint64_t>() : nullptr;
        L.npextra = l + 1 < depth ? nE[l + 1] : 0;
        L.nodes = v->pool_ptr(l);
        L.pclist = v->clist[l + 1].as<uint64_t>();
        L.lev = l;
        L.depth = depth;
        L.b = g.b;
        L.range = v->range(l);
        L.shift = v->logdim[l + 1];
        L.pres = v->res(l + 1);
        L.pres3 = v->res3(l + 1);
        for (int a = 0; a < 3; a++) L.root_lo[a] = (int)(v->root_pos[a] / v->range(l));
        L.leaf_keys = v->leafmap_keys.as<uint64_t>();
        L.leaf_vals = v->leafmap_vals.as<int32_t>();
        L.leaf_mask = v->leafmap_mask;
        L.status = &dev_words(v)->status;
        int64_t cnt = nB[l] + nE[l];
        if (cnt > 0) k_build_link<<<grid_for(cnt, 256, 1ll << 31), 256, 0, s>>>(L);
        GV_CUDA(v, cudaGetLastError());
    }
    // the status word is checked at the next read-back of the small words
    // (the next rebuild's bounding box, Synchronize or GetInfo), not by a
    // stall here
    v->status_pending = true;
    v->used_leaves = v->pool_cnt[0];
    v->all_leaves_flagged = true;
    return GVDB2_OK;
}

gvdb2_status incremental_activate(Volume *v, int n, float radius, const float orig[3], bool accum);

// ---- full rebuild over brick bitmaps --------------------------------------
//
// For a cloud whose bounding box (in level-0 bricks, widened by the
// activation box) holds at most 2^30 bricks, the node sets of every level are
// bitmaps over that box instead of hash sets.  Bit (x, y, z) sits at
// ((x-ox)*dy + (y-oy))*dz + (z-oz), i.e. in the order of the packed keys, so
// an ordered compaction of the set bits yields the sorted unique keys with
// no sort.  Parent levels are the OR of their children's bits, and the extra
// (box-only) set of a level is box & ~base.  The result is the same node
// sets, in the same order, as the hash path below.
struct BitGrid {
    int o[3];       // first brick per axis (absolute, in this level's units)
    int d[3];       // bricks per axis
    uint32_t *base; // bitmaps, ceil(d0*d1*d2 / 32) words each
    uint32_t *box;
    int64_t words;
};

__device__ __forceinline__ int64_t bg_bit(const BitGrid &G, int x, int y, int z) {
    return ((int64_t)(x - G.o[0]) * G.d[1] + (y - G.o[1])) * G.d[2] + (z - G.o[2]);
}
__device__ __forceinline__ bool bg_in(const BitGrid &G, int x, int y, int z) {
    return x >= G.o[0] && x < G.o[0] + G.d[0] && y >= G.o[1] && y < G.o[1] + G.d[1] && z >= G.o[2] &&
           z < G.o[2] + G.d[2];
}
__device__ __forceinline__ void bg_set(uint32_t *bits, int64_t bit) {
    uint32_t *w = bits + (bit >> 5);
    const uint32_t m = 1u << (bit & 31);
    if (!(__ldcg(w) & m)) atomicOr(w, m);
}

// Level-0 base brick and activation-box bricks of every point, with the
// same rules as k_mark_keys.  A brick outside the grid sets kDevCapacity
// (the host then takes the hash path).  With SMEM the CTA first marks a
// shared copy of both bitmaps (grid-stride over the points) and then ORs
// its non-zero words into the global ones: a small grid would otherwise
// put every point's atomics on the same few L2 lines.
template <bool SMEM>
__global__ void k_mark_bits(PointsView pos, int64_t n, float3 orig, float radius, float kmax, int do_box, KeyGeom g,
                            BitGrid G, int32_t *status) {
    extern __shared__ uint32_t sbits[]; // [2 * words] when SMEM
    uint32_t *base = G.base, *box = G.box;
    if (SMEM) {
        for (int64_t i = threadIdx.x; i < 2 * G.words; i += blockDim.x) sbits[i] = 0;
        __syncthreads();
        base = sbits;
        box = sbits + G.words;
    }
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t iters = (n + stride - 1) / stride; // uniform per warp: whole warps take part in match_any
    for (int64_t it = 0; it < iters; it++) {
        const int64_t i = it * stride + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        bool valid = i < n;
        float w[3] = {0, 0, 0};
        int oo[3] = {0, 0, 0};
        if (valid) {
            float3 p = load_f3(pos, i);
            w[0] = p.x + orig.x;
            w[1] = p.y + orig.y;
            w[2] = p.z + orig.z;
            if (w[0] < 0 || w[1] < 0 || w[2] < 0) valid = false;
            const int3 o = point_origin(pos, i);
            oo[0] = o.x;
            oo[1] = o.y;
            oo[2] = o.z;
        }
        int64_t bit = -1;
        int bx = 0, by = 0, bz = 0;
        if (valid) {
            bx = ((int)w[0] + oo[0]) >> g.log2r0;
            by = ((int)w[1] + oo[1]) >> g.log2r0;
            bz = ((int)w[2] + oo[2]) >> g.log2r0;
            if (brick_in_root(g, bx, by, bz)) {
                if (bg_in(G, bx, by, bz)) bit = bg_bit(G, bx, by, bz);
                else atomicOr(status, kDevCapacity);
            }
        }
        // one atomic per distinct bit per warp
        const unsigned peers = __match_any_sync(0xffffffffu, (unsigned long long)bit);
        if (bit >= 0 && (int)(threadIdx.x & 31) == __ffs(peers) - 1) {
            if (SMEM) atomicOr(base + (bit >> 5), 1u << (bit & 31));
            else bg_set(base, bit);
        }
        if (!valid || !do_box) continue;
        int lo[3], hi[3];
        for (int a = 0; a < 3; a++) {
            const int iw = (int)w[a];
            const int bmin = (int)((float)iw - radius);
            const int bmax = (int)((float)iw + kmax * radius);
            lo[a] = max(((bmin < 0 ? 0 : bmin) + oo[a]) >> g.log2r0, g.lo[a]); // clamped in the cloud's own space
            hi[a] = min((bmax + oo[a]) >> g.log2r0, g.lo[a] + g.span - 1);
        }
        for (int x = lo[0]; x <= hi[0]; x++)
            for (int y = lo[1]; y <= hi[1]; y++)
                for (int z = lo[2]; z <= hi[2]; z++) {
                    if (!bg_in(G, x, y, z)) {
                        atomicOr(status, kDevCapacity);
                        continue;
                    }
                    const int64_t bb = bg_bit(G, x, y, z);
                    if (SMEM) {
                        const uint32_t m = 1u << (bb & 31);
                        if (!(box[bb >> 5] & m)) atomicOr(box + (bb >> 5), m);
                    } else {
                        bg_set(box, bb);
                    }
                }
    }
    if (SMEM) {
        __syncthreads();
        for (int64_t k = threadIdx.x; k < 2 * G.words; k += blockDim.x) {
            const uint32_t m = sbits[k];
            if (m) atomicOr((k < G.words ? G.base + k : G.box + (k - G.words)), m);
        }
    }
}

// Parent bit = OR of its children's bits (shift sh per axis).
__global__ void k_parent_bits(BitGrid C, BitGrid P, int sh) {
    const int64_t nbits = (int64_t)P.d[0] * P.d[1] * P.d[2];
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nbits; t += (int64_t)gridDim.x * blockDim.x) {
        const int Z = (int)(t % P.d[2]) + P.o[2], Y = (int)((t / P.d[2]) % P.d[1]) + P.o[1],
                  X = (int)(t / ((int64_t)P.d[1] * P.d[2])) + P.o[0];
        const int r = 1 << sh;
        int lo[3] = {max(X << sh, C.o[0]), max(Y << sh, C.o[1]), max(Z << sh, C.o[2])};
        int hi[3] = {min((X << sh) + r, C.o[0] + C.d[0]), min((Y << sh) + r, C.o[1] + C.d[1]),
                     min((Z << sh) + r, C.o[2] + C.d[2])};
        bool b0 = false, b1 = false;
        for (int x = lo[0]; x < hi[0] && !(b0 && b1); x++)
            for (int y = lo[1]; y < hi[1] && !(b0 && b1); y++)
                for (int z = lo[2]; z < hi[2]; z++) {
                    const int64_t cb = bg_bit(C, x, y, z);
                    const uint32_t m = 1u << (cb & 31);
                    b0 |= (C.base[cb >> 5] & m) != 0;
                    b1 |= (C.box[cb >> 5] & m) != 0;
                }
        const int64_t pb = bg_bit(P, X, Y, Z);
        if (b0) atomicOr(P.base + (pb >> 5), 1u << (pb & 31));
        if (b1) atomicOr(P.box + (pb >> 5), 1u << (pb & 31));
    }
}

// Ordered compaction of bitmap sets into packed keys: CTA j compacts set j
// (a & ~mask) of `sets`, one thread per 32-bit word in rounds of the block,
// decoding the brick of each set bit incrementally from its word's first
// bit.  count[j] receives the number of keys; out == nullptr only counts.
constexpr int kCompactThreads = 1024;
struct CompactSet {
    const uint32_t *a, *mask;
    BitGrid G;
    uint64_t *out;
    int32_t *count;
};
struct CompactSets {
    CompactSet set[2 * kMaxLev];
    int b;
};
__global__ void __launch_bounds__(kCompactThreads) k_bits_compact(CompactSets S) {
    __shared__ uint32_t warp_sum[32];
    __shared__ uint32_t round_total;
    const CompactSet &C = S.set[blockIdx.x];
    const BitGrid &G = C.G;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nbits = G.d[0] * G.d[1] * G.d[2]; // <= 2^28
    uint32_t running = 0;
    for (int64_t round = 0; round < G.words; round += kCompactThreads) {
        const int64_t wi = round + threadIdx.x;
        uint32_t x = 0;
        if (wi < G.words) {
            x = C.a[wi];
            if (C.mask) x &= ~C.mask[wi];
        }
        const uint32_t local = __popc(x);
        uint32_t inc = local;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) warp_sum[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            const uint32_t ws = warp_sum[lane];
            uint32_t wsum = ws;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, wsum, o);
                if (lane >= o) wsum += y;
            }
            warp_sum[lane] = wsum - ws;
            if (lane == 31) round_total = wsum;
        }
        __syncthreads();
        if (C.out && x) {
            uint32_t pos = running + warp_sum[warp] + inc - local;
            const int b0 = (int)(wi << 5);
            int z = b0 % G.d[2], t = b0 / G.d[2];
            int y = t % G.d[1], xx = t / G.d[1];
            int prev = 0;
            while (x) {
                const int j = __ffs(x) - 1;
                x &= x - 1;
                if (b0 + j >= nbits) break;
                z += j - prev; // advance (x, y, z) from bit b0 + prev to b0 + j
                prev = j;
                while (z >= G.d[2]) {
                    z -= G.d[2];
                    if (++y >= G.d[1]) {
                        y = 0;
                        xx++;
                    }
                }
                C.out[pos++] = pack_key(xx + G.o[0], y + G.o[1], z + G.o[2], S.b);
            }
        }
        running += round_total;
        __syncthreads(); // warp_sum / round_total are rewritten next round
    }
    if (threadIdx.x == 0) *C.count = (int32_t)running;
}

// ---- brick bitmaps of large grids (batched clouds, sparse extents) ---------
//
// Above kLargeGridBits bits at level 0 the per-parent scan of k_parent_bits
// (every child bit read one by one) and the single-CTA compaction of
// k_bits_compact would take milliseconds, so both run over words across
// the whole GPU instead; the sets and their key order are the same.
constexpr int64_t kLargeGridBits = 1ll << 22;
constexpr int kChunkThreads = 256;
constexpr int kChunkWordsPerThread = 16;
constexpr int64_t kChunkWords = (int64_t)kChunkThreads * kChunkWordsPerThread;

// Parent bits from the child level's words: a thread per child word; each
// set bit ORs its parent's bit (read first: siblings mostly set it already).
__global__ void k_parent_bits_words(BitGrid C, BitGrid P, int sh) {
    const int64_t nbits = (int64_t)C.d[0] * C.d[1] * C.d[2];
    for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < C.words;
         w += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int s = 0; s < 2; s++) {
            uint32_t x = s ? C.box[w] : C.base[w];
            uint32_t *pbits = s ? P.box : P.base;
            int64_t last = -1;
            while (x) {
                const int j = __ffs(x) - 1;
                x &= x - 1;
                const int64_t b = (w << 5) + j;
                if (b >= nbits) break;
                const int64_t t = b / C.d[2];
                const int z = (int)(b - t * C.d[2]) + C.o[2];
                const int y = (int)(t % C.d[1]) + C.o[1];
                const int xx = (int)(t / C.d[1]) + C.o[0];
                const int64_t p = bg_bit(P, xx >> sh, y >> sh, z >> sh);
                if (p == last) continue;
                last = p;
                bg_set(pbits, p);
            }
        }
    }
}

// The chunks of every set of a large-grid compaction, numbered across the
// sets: set j owns chunks [first[j], first[j + 1]).
struct ChunkedSets {
    CompactSets S;
    int64_t first[2 * kMaxLev + 1];
    int nsets;
    uint32_t *cnt; // per chunk: set bits, then (after k_chunk_scan) the chunk's first key index
};

__device__ __forceinline__ int chunk_set(const ChunkedSets &K, int64_t c) {
    int j = 0;
    while (j + 1 < K.nsets && K.first[j + 1] <= c) j++;
    return j;
}

__device__ __forceinline__ uint32_t chunk_word(const CompactSet &C, int64_t wi) {
    if (wi >= C.G.words) return 0;
    uint32_t x = C.a[wi];
    if (C.mask) x &= ~C.mask[wi];
    return x;
}

// Exclusive scan of one value per thread over a CTA of kChunkThreads;
// *total receives the CTA's sum.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *warp_sum, uint32_t *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_sum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint32_t ws = lane < kChunkThreads / 32 ? warp_sum[lane] : 0;
        uint32_t wsum = ws;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wsum, o);
            if (lane >= o) wsum += y;
        }
        if (lane < kChunkThreads / 32) warp_sum[lane] = wsum - ws;
        if (lane == 31) *total = wsum;
    }
    __syncthreads();
    return warp_sum[warp] + inc - v;
}

// Pass 1: set bits per chunk.
__global__ void __launch_bounds__(kChunkThreads) k_chunk_count(ChunkedSets K) {
    __shared__ uint32_t warp_sum[32];
    __shared__ uint32_t total;
    const int64_t c = blockIdx.x;
    const int j = chunk_set(K, c);
    const CompactSet &C = K.S.set[j];
    const int64_t w0 = (c - K.first[j]) * kChunkWords + (int64_t)threadIdx.x * kChunkWordsPerThread;
    uint32_t n = 0;
#pragma unroll 4
    for (int k = 0; k < kChunkWordsPerThread; k++) n += __popc(chunk_word(C, w0 + k));
    block_excl_scan(n, warp_sum, &total);
    if (threadIdx.x == 0) K.cnt[c] = total;
}

// Pass 2: a CTA per set turns its chunk counts into first key indices and
// writes the set's key count.
__global__ void __launch_bounds__(kChunkThreads) k_chunk_scan(ChunkedSets K) {
    __shared__ uint32_t warp_sum[32];
    __shared__ uint32_t total;
    const int j = blockIdx.x;
    uint32_t running = 0;
    for (int64_t c0 = K.first[j]; c0 < K.first[j + 1]; c0 += kChunkThreads) {
        const int64_t c = c0 + threadIdx.x;
        const uint32_t v = c < K.first[j + 1] ? K.cnt[c] : 0;
        const uint32_t ex = block_excl_scan(v, warp_sum, &total);
        if (c < K.first[j + 1]) K.cnt[c] = running + ex;
        running += total;
        __syncthreads(); // warp_sum / total are rewritten next round
    }
    if (threadIdx.x == 0) *K.S.set[j].count = (int32_t)running;
}

// Pass 3: each thread writes the keys of its words, in bit order, from its
// chunk's first key index plus its rank in the chunk.
__global__ void __launch_bounds__(kChunkThreads) k_chunk_write(ChunkedSets K) {
    __shared__ uint32_t warp_sum[32];
    __shared__ uint32_t total;
    const int64_t c = blockIdx.x;
    const int j = chunk_set(K, c);
    const CompactSet &C = K.S.set[j];
    const BitGrid &G = C.G;
    const int64_t nbits = (int64_t)G.d[0] * G.d[1] * G.d[2];
    const int64_t w0 = (c - K.first[j]) * kChunkWords + (int64_t)threadIdx.x * kChunkWordsPerThread;
    uint32_t n = 0;
#pragma unroll 4
    for (int k = 0; k < kChunkWordsPerThread; k++) n += __popc(chunk_word(C, w0 + k));
    uint32_t pos = K.cnt[c] + block_excl_scan(n, warp_sum, &total);
    if (!n) return;
    for (int k = 0; k < kChunkWordsPerThread; k++) {
        const int64_t wi = w0 + k;
        uint32_t x = chunk_word(C, wi);
        while (x) {
            const int jb = __ffs(x) - 1;
            x &= x - 1;
            const int64_t b = (wi << 5) + jb;
            if (b >= nbits) break;
            const int64_t t = b / G.d[2];
            const int z = (int)(b - t * G.d[2]);
            const int y = (int)(t % G.d[1]), xx = (int)(t / G.d[1]);
            C.out[pos++] = pack_key(xx + G.o[0], y + G.o[1], z + G.o[2], K.S.b);
        }
    }
}

constexpr int64_t kMaxGridBits = 1ll << 30; // bitmap path up to 2^30 bricks (128 MB per bitmap)

// Node key sets through brick bitmaps; *used = false when the grid would be
// too large or a brick fell outside it (then nothing was changed).
// kmax: the box reaches kmax * radius above a point (2 for the full
// rebuild's extra bricks, 1 for the incremental box); force_box: the box set
// even for radius < 1 (the incremental box).
gvdb2_status key_sets_bitmap(Volume *v, int n, float radius, const float orig[3], const KeyGeom &g, int64_t nB[],
                             int64_t nE[], bool *used, float kmax = 2.0f, bool force_box = false) {
    *used = false;
    cudaStream_t s = v->stream;
    const int depth = v->depth;
    const bool do_box = force_box || radius >= 1.0f;
    const float r = do_box ? radius : 0.0f;
    BitGrid G[kMaxLev];
    int64_t off[kMaxLev + 1];
    off[0] = 0;
    int lo0[3], hi0[3];
    for (int a = 0; a < 3; a++) {
        // the box's reach below and above the points (a forced box of radius
        // < 1 still reaches the voxel below and above)
        const float below = force_box ? std::max(r, 1.0f) : r, above = force_box ? std::max(kmax * r, 1.0f) : 2.0f * r;
        const float lo_v = std::max(0.0f, std::floor(v->posmin[a] - below - 2.0f));
        const float hi_v = v->posmax[a] + above + 2.0f;
        if (!(hi_v < 2.0e9f)) return GVDB2_OK;
        lo0[a] = std::max(g.lo[a], (int)lo_v >> g.log2r0);
        hi0[a] = std::min(g.lo[a] + g.span - 1, (int)hi_v >> g.log2r0);
        if (hi0[a] < lo0[a]) hi0[a] = lo0[a];
    }
    int sh = 0;
    for (int l = 0; l < depth; l++) {
        if (l > 0) sh += v->logdim[l];
        int64_t nbits = 1;
        for (int a = 0; a < 3; a++) {
            G[l].o[a] = lo0[a] >> sh;
            G[l].d[a] = (hi0[a] >> sh) - G[l].o[a] + 1;
            nbits *= G[l].d[a];
        }
        if (nbits > kMaxGridBits) return GVDB2_OK;
        G[l].words = (nbits + 31) / 32;
        off[l + 1] = off[l] + 2 * G[l].words;
    }
    GV_CUDA(v, v->bits.ensure(sizeof(uint32_t) * (size_t)off[depth], s));
    GV_CUDA(v, cudaMemsetAsync(v->bits.p, 0, sizeof(uint32_t) * (size_t)off[depth], s));
    for (int l = 0; l < depth; l++) {
        G[l].base = v->bits.as<uint32_t>() + off[l];
        G[l].box = G[l].base + G[l].words;
    }
    GV_CUDA(v, cudaMemsetAsync(dev_words(v)->count, 0, sizeof(int32_t) * 8 + sizeof(int32_t), s));
    const float3 t3 = make_float3(orig[0], orig[1], orig[2]);
    constexpr int64_t kSmemWords = 24576; // both level-0 bitmaps in 96 KB of shared memory
    if (n > 0 && 2 * G[0].words <= kSmemWords) {
        const size_t smem = sizeof(uint32_t) * 2 * (size_t)G[0].words;
        auto k = k_mark_bits<true>;
        if (smem > 48 * 1024) GV_CUDA(v, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        // as many CTAs as fit on an SM (each keeps its own copy of the bitmaps,
        // flushed once), so that the points' loads overlap
        const int per_sm = (int)std::max<size_t>(1, std::min<size_t>(8, (200u << 10) / std::max<size_t>(smem, 1)));
        k<<<std::min(grid_for(n, 256), per_sm * kSmCount), 256, smem, s>>>(v->pos, n, t3, radius, kmax,
                                                                            do_box ? 1 : 0, g, G[0],
                                                                            &dev_words(v)->status);
    } else if (n > 0) {
        k_mark_bits<false><<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(v->pos, n, t3, radius, kmax, do_box ? 1 : 0, g,
                                                                        G[0], &dev_words(v)->status);
    }
    const int64_t nbits0 = (int64_t)G[0].d[0] * G[0].d[1] * G[0].d[2];
    const bool large = nbits0 > kLargeGridBits; // level 0 is the largest grid
    for (int l = 1; l < depth; l++) {
        const int64_t nbits = (int64_t)G[l].d[0] * G[l].d[1] * G[l].d[2];
        if (large)
            k_parent_bits_words<<<grid_for(G[l - 1].words, 256, 16 * kSmCount), 256, 0, s>>>(G[l - 1], G[l],
                                                                                              v->logdim[l]);
        else
            k_parent_bits<<<grid_for(nbits, 256, 8 * kSmCount), 256, 0, s>>>(G[l - 1], G[l], v->logdim[l]);
    }
    // compaction of every (level, set) in one launch; for small grids the key
    // arrays are sized by the grid and a single pass both counts and writes
    CompactSets C;
    C.b = g.b;
    int nsets = 0;
    int64_t maxbits = 0;
    for (int l = 0; l < depth; l++) {
        maxbits = std::max<int64_t>(maxbits, (int64_t)G[l].d[0] * G[l].d[1] * G[l].d[2]);
        C.set[nsets++] = CompactSet{G[l].base, nullptr, G[l], nullptr, dev_words(v)->count + 2 * l};
        if (do_box) C.set[nsets++] = CompactSet{G[l].box, G[l].base, G[l], nullptr, dev_words(v)->count + 2 * l + 1};
    }
    const bool one_pass = maxbits <= kLargeGridBits;
    ChunkedSets K;
    if (!one_pass) {
        // counts per chunk, then per set, over the whole GPU
        K.nsets = nsets;
        K.first[0] = 0;
        for (int j = 0; j < nsets; j++) K.first[j + 1] = K.first[j] + (C.set[j].G.words + kChunkWords - 1) / kChunkWords;
        GV_CUDA(v, v->bits_chunks.ensure(sizeof(uint32_t) * (size_t)std::max<int64_t>(K.first[nsets], 1), s));
        K.cnt = v->bits_chunks.as<uint32_t>();
    }
    if (one_pass) {
        int k = 0;
        for (int l = 0; l < depth; l++) {
            const int64_t nbits = (int64_t)G[l].d[0] * G[l].d[1] * G[l].d[2];
            GV_CUDA(v, v->lev_keys[l][0].ensure(sizeof(uint64_t) * (size_t)nbits, s));
            C.set[k++].out = v->lev_keys[l][0].as<uint64_t>();
            if (do_box) {
                GV_CUDA(v, v->lev_keys[l][1].ensure(sizeof(uint64_t) * (size_t)nbits, s));
                C.set[k++].out = v->lev_keys[l][1].as<uint64_t>();
            } else {
                GV_CUDA(v, v->lev_keys[l][1].ensure(sizeof(uint64_t), s));
            }
        }
    }
    if (one_pass) {
        k_bits_compact<<<nsets, kCompactThreads, 0, s>>>(C);
    } else {
        K.S = C;
        k_chunk_count<<<(unsigned)K.first[nsets], kChunkThreads, 0, s>>>(K);
        k_chunk_scan<<<nsets, kChunkThreads, 0, s>>>(K);
    }
    GV_CUDA(v, cudaGetLastError());
    GV_TRY(read_words(v));
    if (host_words(v)->status & kDevCapacity) return GVDB2_OK; // a brick outside the grid: hash path
    for (int l = 0; l < kMaxLev; l++) nB[l] = nE[l] = 0;
    for (int l = 0; l < depth; l++) {
        nB[l] = host_words(v)->count[2 * l];
        nE[l] = do_box ? host_words(v)->count[2 * l + 1] : 0;
    }
    if (!one_pass) {
        int k = 0;
        for (int l = 0; l < depth; l++) {
            GV_CUDA(v, v->lev_keys[l][0].ensure(sizeof(uint64_t) * (size_t)std::max<int64_t>(nB[l], 1), s));
            GV_CUDA(v, v->lev_keys[l][1].ensure(sizeof(uint64_t) * (size_t)std::max<int64_t>(nE[l], 1), s));
            C.set[k++].out = v->lev_keys[l][0].as<uint64_t>();
            if (do_box) C.set[k++].out = v->lev_keys[l][1].as<uint64_t>();
        }
        K.S = C;
        k_chunk_write<<<(unsigned)K.first[nsets], kChunkThreads, 0, s>>>(K);
        GV_CUDA(v, cudaGetLastError());
    }
    *used = true;
    return GVDB2_OK;
}

// ActivateBricksGPU (+ ActivateExtraBricksGPU when radius >= 1).
gvdb2_status full_rebuild(Volume *v, int n, float radius, const float orig[3]) {
    KeyGeom g = key_geom(v);
    if (g.span > 65536) return fail(v, GVDB2_ERR_UNSUPPORTED, "root spans more than 65536 bricks per axis");
    int64_t nB[kMaxLev] = {0}, nE[kMaxLev] = {0};
    bool used = false;
    GV_TRY(key_sets_bitmap(v, n, radius, orig, g, nB, nE, &used));
    if (!used) GV_TRY(key_sets_hash(v, n, radius, orig, g, nB, nE));
    return build_from_keys(v, nB, nE, g);
}

// DetermineDepth (V:821-837) with GetCoveringNode (V:2915-2931).
int determine_depth(const Volume *v, int rootpos[3]) {
    for (int lev = 0; lev < kMaxLev; lev++) {
        int a[3], b[3];
        if (lev == kMaxLev - 1) {
            a[0] = a[1] = a[2] = b[0] = b[1] = b[2] = 0;
        } else {
            int64_t range = v->range(std::min(lev, v->nlev - 1));
            for (int k = 0; k < 3; k++) {
                int pa = (int)v->posmin[k], pb = (int)v->posmax[k];
                a[k] = (int)(pa / range * range);
                b[k] = (int)(pb / range * range);
            }
        }
        if (a[0] == b[0] && a[1] == b[1] && a[2] == b[2]) {
            rootpos[0] = a[0];
            rootpos[1] = a[1];
            rootpos[2] = a[2];
            return lev;
        }
    }
    return -1;
}

} // namespace

KeyGeom key_geom(const Volume *v) {
    KeyGeom g;
    g.log2r0 = v->logdim[0];
    int64_t span = v->range(v->depth) / v->range(0);
    g.span = (int)span;
    int64_t hi = span + std::max(v->root_pos[0], std::max(v->root_pos[1], v->root_pos[2])) / v->range(0);
    int b = 1;
    while ((1ll << b) < hi) b++;
    g.b = b;
    for (int a = 0; a < 3; a++) g.lo[a] = (int)(v->root_pos[a] / v->range(0));
    return g;
}

gvdb2_status incremental_rebuild(Volume *v, int n, float radius, const float orig[3], bool accum);

gvdb2_status flush_status(Volume *v) {
    if (!(v->status_pending || v->splat_guard_pending) || !v->dev_small.p) return GVDB2_OK;
    return read_words(v);
}

int32_t *splat_guard_word(Volume *v) { return v->dev_small.p ? dev_words(v)->splat_guard : nullptr; }

gvdb2_status sync_counts(Volume *v) {
    GV_CUDA(v, cudaStreamSynchronize(v->stream));
    return GVDB2_OK;
}

// Grows the device's stream-ordered pool once per point-count high-water
// mark, so that buffers tracking a spreading topology (atlas, splat scratch,
// bins) are later carved from memory already mapped instead of mapping new
// physical memory in the middle of a step.  About 1 KB per point covers the
// rebuild, an atlas of 4 channels and the splat scratch; at most a quarter
// of the free device memory is taken.
void reserve_pool(Volume *v, int64_t n) {
    if (n <= v->pool_reserved_for) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, v->device) != cudaSuccess) return;
    uint64_t reserved = 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return;
    const uint64_t want = std::min<uint64_t>((uint64_t)n * 1024 + (256ull << 20), free_b / 4);
    v->pool_reserved_for = n;
    if (reserved >= want) return;
    void *p = nullptr;
    if (cudaMallocAsync(&p, want - reserved, v->stream) == cudaSuccess) cudaFreeAsync(p, v->stream);
    cudaGetLastError(); // a failed reservation is only a missed optimisation
}

// GetMinMaxVel (V:5469-5521): per axis min and max of the first n
// velocities (the bounding-box reduction with no translation);
// mVelRange = mVelMax - mVelMin.  Read by InsertPointsSubcell_FP16.
gvdb2_status get_min_max_vel(Volume *v, int n) {
    if (!v->vel.base || n <= 0 || n > v->vel.count) return fail(v, GVDB2_ERR_ARG, "GetMinMaxVel needs velocities");
    cudaStream_t s = v->stream;
    GV_TRY(ensure_small_words(v));
    int32_t init[6];
    for (int a = 0; a < 3; a++) {
        init[a] = 0x7F800000;              // ord(+inf)
        init[3 + a] = (int32_t)0x807FFFFF; // ord(-inf)
    }
    GV_CUDA(v, cudaMemcpyAsync(dev_words(v)->bbox, init, sizeof(init), cudaMemcpyHostToDevice, s));
    k_bbox<<<std::min(grid_for(n, 256), 8 * kSmCount), 256, 0, s>>>(v->vel, n, make_float3(0.0f, 0.0f, 0.0f),
                                                                    dev_words(v)->bbox);
    GV_CUDA(v, cudaGetLastError());
    GV_TRY(read_words(v));
    for (int a = 0; a < 3; a++) {
        v->velmin[a] = ord2f(host_words(v)->bbox[a]);
        v->velrange[a] = ord2f(host_words(v)->bbox[3 + a]) - v->velmin[a];
    }
    return GVDB2_OK;
}

gvdb2_status rebuild_topology(Volume *v, int n, float radius, const float orig[3], bool accumulate, int min_depth) {
    if (v->nlev == 0) return fail(v, GVDB2_ERR_STATE, "Configure not called");
    if (n < 0 || (n > 0 && (!v->pos.base || n > v->pos.count)))
        return fail(v, GVDB2_ERR_ARG, "point count exceeds the position view");
    cudaStream_t s = v->stream;
    GV_TRY(ensure_small_words(v));
    reserve_pool(v, n);
    // GetBoundingBox
    int32_t init[6];
    for (int a = 0; a < 3; a++) {
        init[a] = 0x7F800000;            // ord(+inf)
        init[3 + a] = (int32_t)0x807FFFFF; // ord(-inf)
    }
    GV_CUDA(v, cudaMemcpyAsync(dev_words(v)->bbox, init, sizeof(init), cudaMemcpyHostToDevice, s));
    if (n > 0)
        k_bbox<<<std::min(grid_for(n, 256), 8 * kSmCount), 256, 0, s>>>(v->pos, n, make_float3(orig[0], orig[1], orig[2]),
                                                                        dev_words(v)->bbox);
    GV_CUDA(v, cudaGetLastError());
    GV_TRY(read_words(v));
    v->all_leaves_flagged = false;
    for (int a = 0; a < 3; a++) {
        float lo = ord2f(host_words(v)->bbox[a]) - 1.0f, hi = ord2f(host_words(v)->bbox[3 + a]) + 2.0f;
        v->posmin[a] = 0 > lo ? 0 : lo;
        v->posmax[a] = 0 > hi ? 0 : hi;
        if (!std::isfinite(v->posmin[a]) || !std::isfinite(v->posmax[a]) || v->posmax[a] > 2.0e9f)
            return fail(v, GVDB2_ERR_DEPTH, "point extents exceed 5 levels");
    }
    int rootpos[3];
    int depth = determine_depth(v, rootpos);
    if (accumulate && depth < min_depth) depth = min_depth;
    if (depth == 0) return fail(v, GVDB2_ERR_DEPTH, "points extents smaller than 1 brick");
    if (depth > 5 || depth < 0 || depth >= v->nlev) return fail(v, GVDB2_ERR_DEPTH, "point extents exceed 5 levels");

    v->bin_key.valid = false;
    v->nbr6_valid = false;
    v->topo_version++;
    if (accumulate && !v->rebuild_topo) { // AccumulateTopology (V:1158-1178)
        v->depth = depth;
        return incremental_rebuild(v, n, radius, orig, true);
    }
    if (v->rebuild_topo) {
        clear_pools(v);
    } else if (depth != v->cur_depth) {
        clear_pools(v);
        v->rebuild_topo = true;
        v->cur_depth = depth;
    }
    v->depth = depth;
    if (v->rebuild_topo) {
        for (int a = 0; a < 3; a++) v->root_pos[a] = rootpos[a];
        gvdb2_status st = full_rebuild(v, n, radius, orig);
        v->rebuild_topo = false;
        v->atlas_valid = false;
        return st;
    }
    return incremental_rebuild(v, n, radius, orig, false);
}

// ActivateIncreBricksGPU (V:1020-1156); kernels in the incremental section.
gvdb2_status incremental_rebuild(Volume *v, int n, float radius, const float orig[3], bool accum) {
    return incremental_activate(v, n, radius, orig, accum);
}

// Atlas growth along Z with content preserved by slot (AtlasResize, A:622-650).
static gvdb2_status atlas_resize(Volume *v, int64_t bricks) {
    int64_t layer = (int64_t)v->subdim[0] * v->subdim[1];
    int nz = (int)std::ceil((float)bricks / (float)layer);
    if (nz < 1) nz = 1;
    if (nz == v->subdim[2] && v->atlas_cap > 0) return GVDB2_OK;
    int64_t ncap = layer * nz;
    size_t tv = (size_t)v->tile_vox();
    for (int c = 0; c < kMaxChan; c++) {
        if (!v->has_chan[c]) continue;
        size_t old = (size_t)v->atlas_cap * tv * sizeof(float);
        GV_CUDA(v, v->atlas[c].ensure((size_t)ncap * tv * sizeof(float), v->stream, true));
        size_t now = (size_t)ncap * tv * sizeof(float);
        if (now > old) GV_CUDA(v, cudaMemsetAsync(v->atlas[c].as<char>() + old, 0, now - old, v->stream));
    }
    v->subdim[2] = nz;
    v->atlas_cap = ncap;
    return GVDB2_OK;
}

gvdb2_status alloc_channel_storage(Volume *v, int chan) {
    size_t bytes = (size_t)v->atlas_cap * (size_t)v->tile_vox() * sizeof(float);
    GV_CUDA(v, v->atlas[chan].ensure(bytes, v->stream));
    GV_CUDA(v, cudaMemsetAsync(v->atlas[chan].p, 0, bytes, v->stream));
    return GVDB2_OK;
}

gvdb2_status update_atlas(Volume *v) {
    if (!v->any_channel()) return fail(v, GVDB2_ERR_STATE, "no atlas channel");
    cudaStream_t s = v->stream;
    int64_t total = v->pool_cnt[0];
    v->atlas_last = 0;
    uint32_t *flags = nullptr;
    GV_CUDA(v, cudaMallocAsync((void **)&flags, sizeof(uint32_t) * (size_t)(2 * total + 2), s));
    uint32_t *scan = flags + total + 1;
    if (total > 0) k_leaf_flags<<<grid_for(total, 256, 1ll << 31), 256, 0, s>>>(v->pool_ptr(0), total, flags);
    gvdb2_status st = exclusive_scan_u32(v, flags, scan, total);
    uint32_t nflag = 0;
    if (st == GVDB2_OK && v->all_leaves_flagged) {
        nflag = (uint32_t)total; // a full rebuild flags every leaf: no read-back
    } else if (st == GVDB2_OK) {
        cudaError_t e = cudaMemcpyAsync(&nflag, scan + total, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(v, e, "update_atlas count");
    }
    if (st == GVDB2_OK && (v->used_leaves > v->atlas_cap || (int64_t)nflag > v->atlas_cap))
        st = atlas_resize(v, std::max<int64_t>(v->used_leaves, nflag));
    if (st == GVDB2_OK) {
        cudaError_t e = v->amap.ensure(sizeof(AtlasNode) * (size_t)v->atlas_cap, s);
        if (e == cudaSuccess) e = v->slot_leaf.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(v->atlas_cap, 1), s);
        if (e == cudaSuccess) e = v->leaf_slot.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(total, 1), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(v->amap.p, 0xFF, sizeof(AtlasNode) * (size_t)v->atlas_cap, s);
        if (e != cudaSuccess) st = cuda_fail(v, e, "update_atlas alloc");
    }
    if (st == GVDB2_OK && total > 0) {
        k_atlas_assign<<<grid_for(total, 256, 1ll << 31), 256, 0, s>>>(
            v->pool_ptr(0), total, flags, scan, v->subdim[0], v->subdim[1], v->tile_res(), v->apron,
            v->amap.as<AtlasNode>(), v->slot_leaf.as<int32_t>(), v->leaf_slot.as<int32_t>());
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_fail(v, e, "k_atlas_assign");
    }
    cudaFreeAsync(flags, s);
    if (st != GVDB2_OK) return st;
    v->atlas_last = nflag;
    // 27-neighbour slot table for the splat/apron kernels
    GV_CUDA(v, v->nbr27.ensure(sizeof(int32_t) * 27 * (size_t)std::max<int64_t>(nflag, 1), s));
    if (nflag > 0) {
        KeyGeom g = key_geom(v);
        k_nbr27<<<grid_for(27 * (int64_t)nflag, 256, 1ll << 31), 256, 0, s>>>(
            v->pool_ptr(0), v->slot_leaf.as<int32_t>(), nflag, v->leaf_slot.as<int32_t>(), v->leafmap_keys.as<uint64_t>(),
            v->leafmap_vals.as<int32_t>(), v->leafmap_mask, g, v->nbr27.as<int32_t>());
        GV_CUDA(v, cudaGetLastError());
    }
    v->atlas_valid = true;
    v->bin_key.valid = false;
    return GVDB2_OK;
}

gvdb2_status update_neighbors(Volume *v) {
    int64_t n = v->pool_cnt[0];
    if (n == 0) return fail(v, GVDB2_ERR_STATE, "no topology");
    GV_CUDA(v, v->nbr6.ensure(sizeof(int32_t) * 6 * (size_t)n, v->stream));
    KeyGeom g = key_geom(v);
    k_nbr6<<<grid_for(6 * n, 256, 1ll << 31), 256, 0, v->stream>>>(v->pool_ptr(0), n, v->leafmap_keys.as<uint64_t>(),
                                                                    v->leafmap_vals.as<int32_t>(), v->leafmap_mask, g,
                                                                    v->nbr6.as<int32_t>());
    GV_CUDA(v, cudaGetLastError());
    v->nbr6_valid = true;
    return GVDB2_OK;
}

// ComputeBounds (V:1792-1816) for FinishTopology: mVoxMin/mVoxMax (and the
// equal world-space mObjMin/mObjMax), mVoxRes and its running maximum.
gvdb2_status compute_bounds(Volume *v) {
    const int64_t n = v->pool_cnt[0];
    if (n == 0) return GVDB2_OK; // the reference reads leaf 0, which does not exist: bounds unchanged
    cudaStream_t s = v->stream;
    GV_TRY(ensure_small_words(v));
    const int32_t init[6] = {INT32_MAX, INT32_MAX, INT32_MAX, INT32_MIN, INT32_MIN, INT32_MIN};
    GV_CUDA(v, cudaMemcpyAsync(dev_words(v)->bbox, init, sizeof(init), cudaMemcpyHostToDevice, s));
    k_leaf_bounds<<<std::min(grid_for(n, 256), 4 * kSmCount), 256, 0, s>>>(v->pool_ptr(0), n, (int)v->range(0),
                                                                           dev_words(v)->bbox);
    GV_CUDA(v, cudaGetLastError());
    GV_TRY(read_words(v));
    for (int a = 0; a < 3; a++) {
        v->vox_min[a] = (float)host_words(v)->bbox[a];
        v->vox_max[a] = (float)host_words(v)->bbox[3 + a];
        v->vox_res[a] = v->vox_max[a] - v->vox_min[a];
        if (v->vox_res[a] > v->vox_res_max[a]) v->vox_res_max[a] = v->vox_res[a];
    }
    return GVDB2_OK;
}

gvdb2_status clear_channel(Volume *v, int chan) {
    if (chan < 0 || chan >= kMaxChan || !v->has_chan[chan]) return fail(v, GVDB2_ERR_ARG, "bad channel");
    GV_CUDA(v, cudaMemsetAsync(v->atlas[chan].p, 0, (size_t)v->atlas_cap * v->tile_vox() * sizeof(float), v->stream));
    return GVDB2_OK;
}


// ---- incremental rebuild ------------------------------------------------
//
// ActivateIncreBricksGPU (V:1020-1156) keeps the pools and appends:
//   1. every point visits the level-l node corners of its box
//      [int(w)-r, int(w)+r] (gvdbCalcIncreExtraBrickId, P:420-465); a corner
//      the tree cannot reach becomes a new key, a reachable leaf is marked;
//   2. no new key: nothing changes (V:1065);
//   3. leaf flags := marks; new nodes are appended per level in key order;
//   4. link top-down (N:470-505), delink unmarked leaves (N:401-429) and
//      childless interior nodes bottom-up (N:431-467);
//   5. used leaves = flagged leaves (V:1144-1147).
// "Reachable" is the reference's tree walk through the child lists
// (getPosParent / getParent), so a leaf delinked earlier is not found again:
// a point returning there gets a new leaf and the old one stays unflagged in
// the pool, as in the reference.  The leaf map is rebuilt from the flagged
// leaves, which are the ones a tree walk reaches.
namespace {

struct TreeView {
    Node *nodes[kMaxLev];
    uint64_t *clist[kMaxLev];
    int64_t cnt[kMaxLev];
    int res[kMaxLev];
    int64_t range[kMaxLev];
    int top, depth;
};

TreeView tree_view(Volume *v) {
    TreeView T;
    for (int l = 0; l < kMaxLev; l++) {
        T.nodes[l] = v->pool_ptr(l);
        T.clist[l] = v->clist[l].as<uint64_t>();
        T.cnt[l] = v->pool_cnt[l];
        T.res[l] = l < v->nlev ? v->res(l) : 1;
        T.range[l] = l < v->nlev ? v->range(l) : 1;
    }
    T.top = v->top_level();
    T.depth = v->depth;
    return T;
}

// getChild (N:115-124): child index, or -1 for an empty slot
__device__ int64_t tv_child(const TreeView &T, const Node *nd, int64_t bit) {
    uint64_t listid = nd->mChildList;
    if (listid == kUndefL) return -1;
    int clev = (int)((listid >> 8) & 0xFF);
    int64_t cndx = (int64_t)(listid >> 16);
    if (clev <= 0 || clev >= kMaxLev || cndx >= T.cnt[clev]) return -1;
    int64_t r3 = (int64_t)T.res[clev] * T.res[clev] * T.res[clev];
    if (bit < 0 || bit >= r3) return -1;
    uint64_t c = T.clist[clev][cndx * r3 + bit];
    return (int64_t)(int32_t)(uint32_t)(c >> 16);
}

// posInNode (N:313-319) with the bit index; false outside the node
__device__ bool tv_bit(const TreeView &T, int lev, const int32_t np[3], const int pos[3], int64_t *bit) {
    int res = T.res[lev];
    int64_t p[3];
    for (int a = 0; a < 3; a++) {
        int64_t d = (int64_t)pos[a] - np[a];
        p[a] = d * res / T.range[lev];
        if (d < 0 || p[a] >= res) return false;
    }
    *bit = (p[2] * res + p[1]) * res + p[0];
    return true;
}

// getPosParent (N:303-348): node of level stopLev containing pos, or -1
__device__ int64_t tv_pos_parent(const TreeView &T, const int pos[3], int stopLev) {
    if (T.cnt[T.top] < 1) return -1;
    const Node *nd = &T.nodes[T.top][0];
    int l = nd->mLev;
    if (l == 0) return 0;
    while (l > 0) {
        int64_t bit;
        if (!tv_bit(T, l, nd->mPos, pos, &bit)) return -1;
        int64_t c = tv_child(T, nd, bit);
        l--;
        if (c == -1) return -1;
        if (l == stopLev) return c;
        if (c < 0 || c >= T.cnt[l]) return -1;
        nd = &T.nodes[l][c];
    }
    return -1;
}

// getParent (N:350-397): as getPosParent, but 0 when the top node is
// unflagged or already at stopLev
__device__ int64_t tv_parent(const TreeView &T, int stopLev, const int pos[3]) {
    if (T.cnt[T.top] < 1) return -1;
    const Node *nd = &T.nodes[T.top][0];
    if (!nd->mFlags) return 0;
    int l = nd->mLev;
    if (l == stopLev) return 0;
    while (l > stopLev) {
        int64_t bit;
        if (!tv_bit(T, l, nd->mPos, pos, &bit)) return -1;
        l--;
        int64_t c = tv_child(T, nd, bit);
        if (c == -1) return -1;
        if (l == stopLev) return c;
        if (c < 0 || c >= T.cnt[l]) return -1;
        nd = &T.nodes[l][c];
    }
    return -1;
}

// child slot of a node at level lev inside its parent pn (level lev+1)
__device__ bool tv_slot(const TreeView &T, int plev, const Node *pn, const int32_t pos[3], int64_t *bit, bool strict) {
    int res = T.res[plev];
    int p[3];
    for (int a = 0; a < 3; a++) p[a] = (int)((int64_t)(pos[a] - pn->mPos[a]) * res / T.range[plev]);
    if (strict && (p[0] > res || p[0] < 0 || p[1] > res || p[1] < 0 || p[2] > res || p[2] < 0)) return false;
    *bit = ((int64_t)p[2] * res + p[1]) * res + p[0];
    return true;
}

// Step 1: marks and new keys.  A new key is lev<<3b | x<<2b | y<<b | z in
// units of the level's range, which sorts like the reference's keys.
// Warps share their points' nodes: in round t each lane offers its box's
// t-th node, and of the lanes offering the same node the lowest looks it up.
__global__ void k_incre_mark(PointsView pos, int64_t n, float3 orig, float radius, TreeView T, KeyGeom g,
                             uint64_t *hs, uint32_t mask, int32_t *marker, int64_t total, int32_t *count,
                             int32_t *status, const uint64_t *lk, const int32_t *lv, uint32_t lmask, int use_map) {
    // every lane of a warp takes part in the rounds (match_any): a thread
    // without a point offers no nodes
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    bool valid = i < n && T.cnt[T.depth] >= 1;
    float w[3] = {0, 0, 0};
    int o[3] = {0, 0, 0};
    if (valid) {
        const float3 p = load_f3(pos, i);
        w[0] = p.x + orig.x;
        w[1] = p.y + orig.y;
        w[2] = p.z + orig.z;
        if (w[0] < 0 || w[1] < 0 || w[2] < 0) valid = false;
        const int3 o3 = point_origin(pos, i);
        o[0] = o3.x;
        o[1] = o3.y;
        o[2] = o3.z;
    }
    const Node *root = &T.nodes[T.depth][0];
    const int64_t rr_root = T.range[T.depth];
    int bmin[3], bmax[3];
    for (int a = 0; a < 3; a++) {
        const int iw = (int)w[a];
        bmin[a] = (int)((float)iw - radius);
        bmax[a] = (int)((float)iw + radius);
    }
    for (int lev = 0; lev < T.depth; lev++) {
        const int rr = (int)T.range[lev];
        // the box's node corners in absolute coordinates; for a batched cloud
        // whose origin is a multiple of the range they are the cloud's own
        // corners (C truncation included) shifted by the origin
        int clo[3] = {0, 0, 0}, nn[3] = {0, 0, 0};
        int cnt = 0;
        if (valid) {
            for (int a = 0; a < 3; a++) {
                int chi;
                if (o[a] % rr == 0) {
                    clo[a] = bmin[a] / rr * rr + o[a];
                    chi = bmax[a] / rr * rr + o[a];
                } else {
                    clo[a] = (max(bmin[a], 0) + o[a]) / rr * rr;
                    chi = (bmax[a] + o[a]) / rr * rr;
                }
                nn[a] = chi >= clo[a] ? (chi - clo[a]) / rr + 1 : 0;
            }
            cnt = nn[0] * nn[1] * nn[2];
        }
        const int rounds = __reduce_max_sync(0xffffffffu, cnt);
        for (int t = 0; t < rounds; t++) {
            bool has = t < cnt;
            int nd[3] = {0, 0, 0};
            if (has) { // x outer, z inner, as the reference's loops
                nd[0] = clo[0] + (t / (nn[1] * nn[2])) * rr;
                nd[1] = clo[1] + (t / nn[2] % nn[1]) * rr;
                nd[2] = clo[2] + (t % nn[2]) * rr;
                for (int a = 0; a < 3; a++)
                    has = has && !(nd[a] < root->mPos[a] || (int64_t)nd[a] >= root->mPos[a] + rr_root);
            }
            const uint64_t bkey = has ? pack_key(nd[0] / rr, nd[1] / rr, nd[2] / rr, g.b) : 0;
            const uint64_t key = has ? (((uint64_t)lev << (3 * g.b)) | bkey) : ~0ull;
            const unsigned peers = __match_any_sync(0xffffffffu, (unsigned long long)key);
            if (!has || lane != __ffs(peers) - 1) continue;
            // the leaf map holds exactly the leaves linked in the tree, so a
            // level-0 lookup there finds what the walk from the root finds
            const int64_t pid = (lev == 0 && use_map) ? (int64_t)hm_lookup(lk, lv, lmask, bkey) : tv_pos_parent(T, nd, lev);
            if (pid == -1) {
                const int r = hs_insert(hs, mask, key);
                if (r > 0) atomicAdd(count, 1);
                if (r < 0) atomicOr(status, kDevHashFull);
            } else if (lev == 0 && pid >= 0 && pid < total) {
                marker[pid] = 1;
            }
        }
    }
}

// The incremental marking from the activation box's unique nodes (the box
// bitmaps' keys of one level and set): a node the tree has marks its leaf,
// a node it lacks goes into the new-node set.
__global__ void k_incre_keys(const uint64_t *bkeys, int64_t nk, int lev, TreeView T, KeyGeom g, uint64_t *hs,
                             uint32_t mask, int32_t *marker, int64_t total, int32_t *count, int32_t *status,
                             const uint64_t *lk, const int32_t *lv, uint32_t lmask, int use_map) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nk || T.cnt[T.depth] < 1) return;
    const uint64_t bkey = bkeys[i];
    int nd[3];
    unpack_key(bkey, g.b, nd[0], nd[1], nd[2]);
    const int rr = (int)T.range[lev];
    for (int a = 0; a < 3; a++) nd[a] *= rr;
    const int64_t pid = (lev == 0 && use_map) ? (int64_t)hm_lookup(lk, lv, lmask, bkey) : tv_pos_parent(T, nd, lev);
    if (pid == -1) {
        const int r = hs_insert(hs, mask, ((uint64_t)lev << (3 * g.b)) | bkey);
        if (r > 0) atomicAdd(count, 1);
        if (r < 0) atomicOr(status, kDevHashFull);
    } else if (lev == 0 && pid >= 0 && pid < total) {
        marker[pid] = 1;
    }
}

__global__ void k_init_markers(const Node *leaves, int64_t total, int accum, int32_t *marker) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < total) marker[i] = accum ? (int32_t)leaves[i].mFlags : 0;
}

__global__ void k_level_count(const uint64_t *keys, int64_t n, int b, int32_t *lev_cnt) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(&lev_cnt[(int)(keys[i] >> (3 * b))], 1);
}

// V:1078-1081: leaf flags := marks
__global__ void k_apply_markers(Node *leaves, int64_t total, const int32_t *marker) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < total) leaves[i].mFlags = (uint8_t)(marker[i] ? 1 : 0);
}

struct NewNodes {
    const uint64_t *keys;
    int64_t n;
    int b;
    int64_t start[kMaxLev], old_cnt[kMaxLev], range[kMaxLev];
    Node *nodes[kMaxLev];
};

// PoolAlloc + SetupNode for the appended nodes (V:1088-1111); the child
// list of an interior node has the node's own pool index.
__global__ void k_new_nodes(NewNodes A) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    uint64_t key = A.keys[i];
    int lev = (int)(key >> (3 * A.b));
    int x, y, z;
    unpack_key(key, A.b, x, y, z);
    int64_t idx = A.old_cnt[lev] + (i - A.start[lev]);
    Node nd;
    memset(&nd, 0, sizeof(nd));
    nd.mLev = (uint8_t)lev;
    nd.mFlags = 1;
    nd.mPos[0] = (int32_t)(x * A.range[lev]);
    nd.mPos[1] = (int32_t)(y * A.range[lev]);
    nd.mPos[2] = (int32_t)(z * A.range[lev]);
    nd.mValue[0] = nd.mValue[1] = nd.mValue[2] = -1;
    nd.mParent = kUndefL;
    nd.mChildList = lev > 0 ? elem(1, lev, (uint64_t)idx) : kUndefL;
    A.nodes[lev][idx] = nd;
}

// gvdbLinkBricks (N:470-505) for one level
__global__ void k_link_level(TreeView T, int lev) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.cnt[lev]) return;
    Node *nd = &T.nodes[lev][i];
    if (!nd->mFlags) return;
    int pos[3] = {nd->mPos[0], nd->mPos[1], nd->mPos[2]};
    const int pl = lev + 1;
    int64_t pid = tv_parent(T, pl, pos);
    if (pid < 0 || pid >= T.cnt[pl]) return;
    const Node *pn = &T.nodes[pl][pid];
    int64_t bit;
    if (!tv_slot(T, pl, pn, nd->mPos, &bit, true)) return;
    nd->mParent = ((uint64_t)pid << 16) | ((uint64_t)pl << 8);
    int64_t cndx = (int64_t)(pn->mChildList >> 16);
    int64_t r3 = (int64_t)T.res[pl] * T.res[pl] * T.res[pl];
    if (cndx >= T.cnt[pl] || bit >= r3) return;
    T.clist[pl][cndx * r3 + bit] = ((uint64_t)i << 16) | ((uint64_t)lev << 8);
}

// gvdbDelinkLeafBricks (N:401-429)
__global__ void k_delink_leaves(TreeView T) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.cnt[0]) return;
    Node *nd = &T.nodes[0][i];
    if (nd->mFlags || nd->mParent == kUndef64) return;
    int pos[3] = {nd->mPos[0], nd->mPos[1], nd->mPos[2]};
    int64_t pid = tv_parent(T, 1, pos);
    nd->mParent = kUndef64;
    if (pid < 0 || pid >= T.cnt[1]) return;
    const Node *pn = &T.nodes[1][pid];
    int64_t bit;
    tv_slot(T, 1, pn, nd->mPos, &bit, false);
    int64_t r3 = (int64_t)T.res[1] * T.res[1] * T.res[1];
    int64_t cndx = (int64_t)(pn->mChildList >> 16);
    if (bit >= 0 && bit < r3 && cndx < T.cnt[1]) T.clist[1][cndx * r3 + bit] = kUndef64;
}

// gvdbDelinkBricks (N:431-467) for one interior level
__global__ void k_delink_level(TreeView T, int lev) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.cnt[lev]) return;
    Node *nd = &T.nodes[lev][i];
    if (nd->mParent == kUndef64) {
        nd->mFlags = 0;
        return;
    }
    int64_t r3 = (int64_t)T.res[lev] * T.res[lev] * T.res[lev];
    const uint64_t *cl = T.clist[lev] + i * r3;
    for (int64_t c = 0; c < r3; c++)
        if (cl[c] != kUndef64) {
            nd->mFlags = 1;
            return;
        }
    nd->mFlags = 0;
    int pos[3] = {nd->mPos[0], nd->mPos[1], nd->mPos[2]};
    int64_t pid = tv_parent(T, lev + 1, pos);
    nd->mParent = kUndef64;
    if (pid < 0 || pid >= T.cnt[lev + 1]) return;
    const Node *pn = &T.nodes[lev + 1][pid];
    int64_t bit;
    tv_slot(T, lev + 1, pn, nd->mPos, &bit, false);
    int64_t pr3 = (int64_t)T.res[lev + 1] * T.res[lev + 1] * T.res[lev + 1];
    int64_t cndx = (int64_t)(pn->mChildList >> 16);
    if (bit >= 0 && bit < pr3 && cndx < T.cnt[lev + 1]) T.clist[lev + 1][cndx * pr3 + bit] = kUndef64;
}

// leaf map of the flagged leaves; counts them into *used
__global__ void k_leafmap_fill(const Node *leaves, int64_t n, KeyGeom g, uint64_t *lk, int32_t *lv, uint32_t mask,
                               int32_t *used, int32_t *status) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Node &nd = leaves[i];
    if (!nd.mFlags) return;
    atomicAdd(used, 1);
    uint64_t key = pack_key(nd.mPos[0] >> g.log2r0, nd.mPos[1] >> g.log2r0, nd.mPos[2] >> g.log2r0, g.b);
    if (hm_insert(lk, lv, mask, key, (int32_t)i) < 0) atomicOr(status, kDevHashFull);
}

} // namespace

namespace {

gvdb2_status ensure_pool_keep(Volume *v, int lev, int64_t cnt) {
    GV_CUDA(v, v->pool[lev].ensure(sizeof(Node) * (size_t)std::max<int64_t>(cnt, 1), v->stream, true));
    if (lev > 0)
        GV_CUDA(v, v->clist[lev].ensure(sizeof(uint64_t) * (size_t)(std::max<int64_t>(cnt, 1) * v->res3(lev)),
                                        v->stream, true));
    return GVDB2_OK;
}

gvdb2_status incremental_activate(Volume *v, int n, float radius, const float orig[3], bool accum) {
    const int64_t total = v->pool_cnt[0];
    if (total == 0) return GVDB2_OK; // V:1022
    cudaStream_t s = v->stream;
    const int depth = v->depth;
    if (v->pool_cnt[depth] < 1) return fail(v, GVDB2_ERR_STATE, "incremental rebuild without a root at this depth");
    KeyGeom g = key_geom(v);
    if (3 * g.b + 4 > 64) return fail(v, GVDB2_ERR_UNSUPPORTED, "root too large for packed level keys");
    const int b = g.b;
    GV_CUDA(v, v->tmp_c.ensure(sizeof(int32_t) * (size_t)total, s));
    int32_t *marker = v->tmp_c.as<int32_t>();

    // 1. marks and new keys, into a hash set sized from the pool (grown on
    // overflow).  The box's nodes come from brick bitmaps when the cloud's
    // extent allows (each level's nodes once, looked up once), else from
    // every point's box.
    int64_t nB[kMaxLev] = {0}, nE[kMaxLev] = {0};
    bool boxed = false;
    if (n > 0) GV_TRY(key_sets_bitmap(v, n, radius, orig, g, nB, nE, &boxed, 1.0f, true));
    uint32_t cap = next_pow2((uint64_t)std::max<int64_t>(4 * total, 1 << 16));
    int64_t nnew = 0;
    for (int attempt = 0;; attempt++) {
        GV_CUDA(v, v->hs_keys[0].ensure(sizeof(uint64_t) * cap, s));
        GV_CUDA(v, cudaMemsetAsync(v->hs_keys[0].p, 0xFF, sizeof(uint64_t) * cap, s));
        GV_CUDA(v, cudaMemsetAsync(dev_words(v)->count, 0, sizeof(int32_t) * 8 + sizeof(int32_t), s));
        k_init_markers<<<grid_for(total, 256, 1ll << 31), 256, 0, s>>>(v->pool_ptr(0), total, accum ? 1 : 0, marker);
        if (boxed) {
            const TreeView T = tree_view(v);
            for (int l = 0; l < depth; l++)
                for (int set = 0; set < 2; set++) {
                    const int64_t nk = set ? nE[l] : nB[l];
                    if (nk > 0)
                        k_incre_keys<<<grid_for(nk, 256, 1ll << 31), 256, 0, s>>>(
                            v->lev_keys[l][set].as<uint64_t>(), nk, l, T, g, v->hs_keys[0].as<uint64_t>(), cap - 1,
                            marker, total, dev_words(v)->count, &dev_words(v)->status, v->leafmap_keys.as<uint64_t>(),
                            v->leafmap_vals.as<int32_t>(), v->leafmap_mask, v->leafmap_is_tree ? 1 : 0);
                }
        } else if (n > 0)
            k_incre_mark<<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(
                v->pos, n, make_float3(orig[0], orig[1], orig[2]), radius, tree_view(v), g,
                v->hs_keys[0].as<uint64_t>(), cap - 1, marker, total, dev_words(v)->count, &dev_words(v)->status,
                v->leafmap_keys.as<uint64_t>(), v->leafmap_vals.as<int32_t>(), v->leafmap_mask,
                v->leafmap_is_tree ? 1 : 0);
        GV_CUDA(v, cudaGetLastError());
        GV_TRY(read_words(v));
        nnew = host_words(v)->count[0];
        bool full = (host_words(v)->status & kDevHashFull) || 2 * nnew > (int64_t)cap;
        if (!full) break;
        if (attempt == 3) return fail(v, GVDB2_ERR_CAPACITY, "new-node hash set overflow");
        cap = next_pow2((uint64_t)cap * 4);
    }
    // 2. nothing new: pools and flags stay as they are (V:1065)
    if (nnew == 0) return GVDB2_OK;

    // sorted new keys and their count per level
    GV_CUDA(v, v->tmp_a.ensure(sizeof(uint64_t) * (size_t)nnew, s));
    uint64_t *keys = v->tmp_a.as<uint64_t>();
    GV_CUDA(v, cudaMemsetAsync(dev_words(v)->count + 2, 0, sizeof(int32_t), s));
    k_compact_set<<<grid_for(cap, 256, 4096), 256, 0, s>>>(v->hs_keys[0].as<uint64_t>(), cap, keys,
                                                           dev_words(v)->count + 2);
    GV_TRY(radix_sort_u64(v, keys, nullptr, nnew, 0, 3 * b + 3));
    GV_CUDA(v, cudaMemsetAsync(dev_words(v)->count, 0, sizeof(int32_t) * 8, s));
    k_level_count<<<grid_for(nnew, 256, 1ll << 31), 256, 0, s>>>(keys, nnew, b, dev_words(v)->count);
    GV_CUDA(v, cudaGetLastError());
    GV_TRY(read_words(v));
    int64_t add[kMaxLev] = {0};
    for (int l = 0; l < depth && l < 8; l++) add[l] = host_words(v)->count[l];

    // 3. flags := marks, then append the new nodes level by level
    k_apply_markers<<<grid_for(total, 256, 1ll << 31), 256, 0, s>>>(v->pool_ptr(0), total, marker);
    NewNodes A;
    A.keys = keys;
    A.n = nnew;
    A.b = b;
    int64_t start = 0;
    for (int l = 0; l < kMaxLev; l++) {
        A.start[l] = start;
        A.old_cnt[l] = v->pool_cnt[l];
        A.range[l] = l < v->nlev ? v->range(l) : 1;
        start += add[l];
    }
    for (int l = 0; l < depth; l++) {
        if (!add[l]) continue;
        GV_TRY(ensure_pool_keep(v, l, v->pool_cnt[l] + add[l]));
        if (l > 0)
            GV_CUDA(v, cudaMemsetAsync(v->clist[l].as<uint64_t>() + v->pool_cnt[l] * v->res3(l), 0xFF,
                                       sizeof(uint64_t) * (size_t)(add[l] * v->res3(l)), s));
    }
    for (int l = 0; l < kMaxLev; l++) A.nodes[l] = v->pool_ptr(l);
    k_new_nodes<<<grid_for(nnew, 256, 1ll << 31), 256, 0, s>>>(A);
    for (int l = 0; l < depth; l++) v->pool_cnt[l] += add[l];

    // 4. link top-down, delink bottom-up (top level from the new counts,
    // as PrepareVDBPartially sets it)
    TreeView T = tree_view(v);
    for (int l = depth - 1; l >= 0; l--)
        if (T.cnt[l] > 0) k_link_level<<<grid_for(T.cnt[l], 256, 1ll << 31), 256, 0, s>>>(T, l);
    k_delink_leaves<<<grid_for(T.cnt[0], 256, 1ll << 31), 256, 0, s>>>(T);
    for (int l = 1; l < depth; l++)
        if (T.cnt[l] > 0) k_delink_level<<<grid_for(T.cnt[l], 256, 1ll << 31), 256, 0, s>>>(T, l);
    GV_CUDA(v, cudaGetLastError());

    // 5. leaf map of the flagged leaves; used leaves
    uint32_t lcap = next_pow2((uint64_t)std::max<int64_t>(2 * v->pool_cnt[0], 1 << 12));
    GV_CUDA(v, v->leafmap_keys.ensure(sizeof(uint64_t) * lcap, s));
    GV_CUDA(v, v->leafmap_vals.ensure(sizeof(int32_t) * lcap, s));
    GV_CUDA(v, cudaMemsetAsync(v->leafmap_keys.p, 0xFF, sizeof(uint64_t) * lcap, s));
    v->leafmap_mask = lcap - 1;
    v->leafmap_is_tree = true;
    GV_CUDA(v, cudaMemsetAsync(dev_words(v)->count, 0, sizeof(int32_t) * 8 + sizeof(int32_t), s));
    k_leafmap_fill<<<grid_for(v->pool_cnt[0], 256, 1ll << 31), 256, 0, s>>>(
        v->pool_ptr(0), v->pool_cnt[0], g, v->leafmap_keys.as<uint64_t>(), v->leafmap_vals.as<int32_t>(),
        v->leafmap_mask, dev_words(v)->count, &dev_words(v)->status);
    GV_CUDA(v, cudaGetLastError());
    GV_TRY(read_words(v));
    if (host_words(v)->status & kDevHashFull) return fail(v, GVDB2_ERR_CAPACITY, "leaf map overflow");
    v->used_leaves = host_words(v)->count[0];
    v->lev_count[0][0] = v->pool_cnt[0];
    v->lev_count[0][1] = 0;
    v->atlas_valid = false;
    return GVDB2_OK;
}

} // namespace

// LoadVBX: room for `cnt` nodes (and their child lists) at level `lev`.
gvdb2_status pool_reserve(Volume *v, int lev, int64_t cnt) { return ensure_pool(v, lev, cnt); }

// LoadVBX (FinishTopology, V:636): the pools were filled from a file.
// Derive what a rebuild leaves besides them: depth and root position, the
// leaf map of the linked leaves and the used-leaf count.  The next
// RebuildTopology starts over, as after Configure.
gvdb2_status adopt_pools(Volume *v, int depth) {
    cudaStream_t s = v->stream;
    GV_TRY(ensure_small_words(v));
    if (v->status_pending) GV_TRY(read_words(v)); // before the status word is cleared below
    v->all_leaves_flagged = false;
    Node root;
    GV_CUDA(v, cudaMemcpy(&root, v->pool[depth].p, sizeof(Node), cudaMemcpyDeviceToHost));
    v->depth = depth;
    v->cur_depth = depth;
    for (int a = 0; a < 3; a++) {
        v->root_pos[a] = root.mPos[a];
        v->posmin[a] = v->posmax[a] = 0.0f; // no bounding box in the file
    }
    const KeyGeom g = key_geom(v);
    uint32_t lcap = next_pow2((uint64_t)std::max<int64_t>(2 * v->pool_cnt[0], 1 << 12));
    GV_CUDA(v, v->leafmap_keys.ensure(sizeof(uint64_t) * lcap, s));
    GV_CUDA(v, v->leafmap_vals.ensure(sizeof(int32_t) * lcap, s));
    GV_CUDA(v, cudaMemsetAsync(v->leafmap_keys.p, 0xFF, sizeof(uint64_t) * lcap, s));
    v->leafmap_mask = lcap - 1;
    v->leafmap_is_tree = false;
    GV_CUDA(v, cudaMemsetAsync(dev_words(v)->count, 0, sizeof(int32_t) * 8 + sizeof(int32_t), s));
    if (v->pool_cnt[0] > 0)
        k_leafmap_fill<<<grid_for(v->pool_cnt[0], 256, 1ll << 31), 256, 0, s>>>(
            v->pool_ptr(0), v->pool_cnt[0], g, v->leafmap_keys.as<uint64_t>(), v->leafmap_vals.as<int32_t>(),
            v->leafmap_mask, dev_words(v)->count, &dev_words(v)->status);
    GV_CUDA(v, cudaGetLastError());
    GV_TRY(read_words(v));
    if (host_words(v)->status & kDevHashFull) return fail(v, GVDB2_ERR_CAPACITY, "leaf map overflow");
    v->used_leaves = host_words(v)->count[0];
    for (int l = 0; l < kMaxLev; l++) v->lev_count[l][0] = v->lev_count[l][1] = 0;
    v->lev_count[0][0] = v->pool_cnt[0];
    v->rebuild_topo = true;
    v->topo_version++;
    v->bin_key.valid = false;
    v->nbr6_valid = false;
    v->atlas_valid = false;
    v->atlas_last = 0;
    return GVDB2_OK;
}

} // namespace gvdb2
