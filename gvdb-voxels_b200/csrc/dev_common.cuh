// dev_common.cuh -- device helpers shared by the libgvdb2 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gvdb2_internal.h"

namespace gvdb2 {

constexpr int kSmCount = 148;   // B200: 2 dies x 74 SMs
constexpr int kMaxProbe = 4096; // bound on every hash probe sequence

__device__ __forceinline__ float3 load_f3(const PointsView &w, int64_t i) {
    const float *p = reinterpret_cast<const float *>(w.base + i * (int64_t)w.stride + w.offset);
    return make_float3(p[0], p[1], p[2]);
}
// Integer voxel origin of point i's cloud (zero outside a batch).
__device__ __forceinline__ int3 point_origin(const PointsView &w, int64_t i) {
    if (!w.cloud) return make_int3(0, 0, 0);
    const int32_t *o = w.origin + 3 * (int64_t)w.cloud[i];
    return make_int3(o[0], o[1], o[2]);
}
__device__ __forceinline__ float load_f1(const PointsView &w, int64_t i) {
    return *reinterpret_cast<const float *>(w.base + i * (int64_t)w.stride + w.offset);
}

// Brick key of the reference (P:377-380): lev<<48 | x<<32 | y<<16 | z.
__host__ __device__ __forceinline__ uint64_t make_key(int lev, int x, int y, int z) {
    return ((uint64_t)(uint16_t)lev << 48) | ((uint64_t)(uint16_t)x << 32) | ((uint64_t)(uint16_t)y << 16) |
           (uint64_t)(uint16_t)z;
}
__host__ __device__ __forceinline__ int key_x(uint64_t k) { return (int)((k >> 32) & 0xFFFF); }
__host__ __device__ __forceinline__ int key_y(uint64_t k) { return (int)((k >> 16) & 0xFFFF); }
__host__ __device__ __forceinline__ int key_z(uint64_t k) { return (int)(k & 0xFFFF); }
__host__ __device__ __forceinline__ uint64_t elem(int grp, int lev, uint64_t ndx) {
    return (uint64_t)grp | ((uint64_t)lev << 8) | (ndx << 16);
}

// Packed level-0 brick key: x<<2b | y<<b | z, which orders bricks like the
// reference's (x, y, z) key words.  The geometry bounds every lookup to the
// root node so out-of-root coordinates never alias.
struct KeyGeom {
    int log2r0; // log2(range(0))
    int b;      // bits per axis in a packed key
    int lo[3];  // root corner in level-0 bricks
    int span;   // root extent in level-0 bricks
};
KeyGeom key_geom(const Volume *v);

__host__ __device__ __forceinline__ uint64_t pack_key(int x, int y, int z, int b) {
    return ((uint64_t)x << (2 * b)) | ((uint64_t)y << b) | (uint64_t)z;
}
__host__ __device__ __forceinline__ void unpack_key(uint64_t k, int b, int &x, int &y, int &z) {
    uint64_t m = (1ull << b) - 1;
    x = (int)((k >> (2 * b)) & m);
    y = (int)((k >> b) & m);
    z = (int)(k & m);
}
__device__ __forceinline__ bool brick_in_root(const KeyGeom &g, int bx, int by, int bz) {
    return bx >= g.lo[0] && bx < g.lo[0] + g.span && by >= g.lo[1] && by < g.lo[1] + g.span && bz >= g.lo[2] &&
           bz < g.lo[2] + g.span;
}

// Leaf lookup table of the linked leaves (level-0 key -> pool index).
struct LeafLookup {
    const uint64_t *keys;
    const int32_t *vals;
    uint32_t mask;
    KeyGeom g;
};

inline LeafLookup make_lookup(const Volume *v) {
    LeafLookup L;
    L.keys = v->leafmap_keys.as<uint64_t>();
    L.vals = v->leafmap_vals.as<int32_t>();
    L.mask = v->leafmap_mask;
    L.g = key_geom(v);
    return L;
}

__device__ __forceinline__ uint32_t hash_key(uint64_t k) {
    // splitmix64 finaliser
    k ^= k >> 30;
    k *= 0xbf58476d1ce4e5b9ull;
    k ^= k >> 27;
    k *= 0x94d049bb133111ebull;
    k ^= k >> 31;
    return (uint32_t)k;
}

// Insert into a hash set; returns 1 if inserted, 0 if present, -1 if the
// probe bound was hit (table too full).
__device__ __forceinline__ int hs_insert(uint64_t *keys, uint32_t mask, uint64_t key) {
    uint32_t h = hash_key(key) & mask;
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        uint64_t cur = __ldcg(keys + h);
        if (cur == key) return 0;
        if (cur == kEmptyKey) {
            unsigned long long prev =
                atomicCAS(reinterpret_cast<unsigned long long *>(keys + h), (unsigned long long)kEmptyKey,
                          (unsigned long long)key);
            if (prev == kEmptyKey) return 1;
            if (prev == key) return 0;
        }
        h = (h + 1) & mask;
    }
    return -1;
}

// Insert key -> val (keys unique by construction of the caller).
__device__ __forceinline__ int hm_insert(uint64_t *keys, int32_t *vals, uint32_t mask, uint64_t key, int32_t val) {
    uint32_t h = hash_key(key) & mask;
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long *>(keys + h),
                                            (unsigned long long)kEmptyKey, (unsigned long long)key);
        if (prev == kEmptyKey || prev == key) {
            vals[h] = val;
            return 1;
        }
        h = (h + 1) & mask;
    }
    return -1;
}

__device__ __forceinline__ int32_t hm_lookup(const uint64_t *keys, const int32_t *vals, uint32_t mask, uint64_t key) {
    if (mask == 0) return -1;
    uint32_t h = hash_key(key) & mask;
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        uint64_t cur = __ldg(keys + h);
        if (cur == key) return __ldg(vals + h);
        if (cur == kEmptyKey) return -1;
        h = (h + 1) & mask;
    }
    return -1;
}

// Leaf containing world position w (the node getNodeAtPoint reaches,
// N:199-253), or -1.
__device__ __forceinline__ int32_t leaf_at(const LeafLookup &L, float wx, float wy, float wz) {
    if (!(wx >= 0.0f && wy >= 0.0f && wz >= 0.0f)) return -1;
    int bx = (int)wx >> L.g.log2r0, by = (int)wy >> L.g.log2r0, bz = (int)wz >> L.g.log2r0;
    if (!brick_in_root(L.g, bx, by, bz)) return -1;
    return hm_lookup(L.keys, L.vals, L.mask, pack_key(bx, by, bz, L.g.b));
}
__device__ __forceinline__ int32_t leaf_at_brick(const LeafLookup &L, int bx, int by, int bz) {
    if (!brick_in_root(L.g, bx, by, bz)) return -1;
    return hm_lookup(L.keys, L.vals, L.mask, pack_key(bx, by, bz, L.g.b));
}

// leaf_at for a point of a batched cloud: w in the cloud's own space, o its origin.
__device__ __forceinline__ int32_t leaf_at_o(const LeafLookup &L, float wx, float wy, float wz, int3 o) {
    if (!(wx >= 0.0f && wy >= 0.0f && wz >= 0.0f)) return -1;
    return leaf_at_brick(L, ((int)wx + o.x) >> L.g.log2r0, ((int)wy + o.y) >> L.g.log2r0, ((int)wz + o.z) >> L.g.log2r0);
}

// The kernel splats and gathers work on cells: 8^3 blocks of a brick.  A
// brick of res0 = 8m voxels holds m^3 cells; cell id = slot * m^3 +
// (cz * m + cy) * m + cx.  For 8^3 bricks a cell is the brick.
constexpr int kCell = 8;
// Points of a cell are binned by region (see k_bin_count): 3 per axis.
constexpr int kRegions = 27;
__device__ __forceinline__ void cell_coords(int64_t cell, int m, int m3, int64_t &slot, int &cx, int &cy, int &cz) {
    if (m3 == 1) { // 8^3 bricks: the cell is the brick
        slot = cell;
        cx = cy = cz = 0;
        return;
    }
    const int lm = __ffs(m) - 1; // m = res0 / 8 is a power of two: shifts, no division
    slot = cell >> (3 * lm);
    const int ci = (int)(cell & (int64_t)(m3 - 1));
    cx = ci & (m - 1);
    cy = (ci >> lm) & (m - 1);
    cz = ci >> (2 * lm);
}
// The cells that hold points fall in three classes by their point count k:
// huge (k > kHeavyCell), heavy (kLightCell < k <= kHeavyCell) and light
// (0 < k <= kLightCell).  The huge and heavy cells are listed in the order
// of cell_at: huge cells first (list[0 .. cnt[0])), then the heavy ones,
// stored from the back (list[ncell - 1], list[ncell - 2], ..., cnt[1] of
// them).  Light cells are listed apart (light[0 .. cnt[2])).  The gather
// stages a halo tile per huge or heavy cell and reads the taps of light
// cells' points straight from the atlas, one warp per light cell.
constexpr uint32_t kHeavyCell = 1024;
constexpr uint32_t kLightCell = 32;
// Cells of at least kDenseCell points are splatted into partial sums (the
// scatter's dense path), kSlicePts points per CTA.
#ifndef GVDB2_DENSE_CELL
#define GVDB2_DENSE_CELL 512
#endif
constexpr uint32_t kDenseCell = GVDB2_DENSE_CELL;

// Sizes the splat kernels check their data-derived indices against: an
// index out of range (bins inconsistent with the topology) skips the access
// and sets *flag, which the host reports as an error at its next read-back.
struct SplatLimits {
    int32_t *flag;
    int64_t nslot;  // atlas slots
    int64_t npool;  // level-0 pool nodes
    int64_t nentry; // entries of the bin order (the points the bins were made for)
    int64_t ncloud; // batched clouds
};
// The first failing check of a call leaves its code in flag[0] and the
// index and bound in flag[1..4].
__device__ __forceinline__ bool in_range(const SplatLimits &L, int64_t i, int64_t hi, int code) {
    if ((uint64_t)i < (uint64_t)hi) return true;
    if (L.flag && atomicCAS(L.flag, 0, code) == 0) {
        L.flag[1] = (int32_t)(i >> 32), L.flag[2] = (int32_t)i;
        L.flag[3] = (int32_t)(hi >> 32), L.flag[4] = (int32_t)hi;
    }
    return false;
}
constexpr uint32_t kSlicePts = 4096;
// cell_cnt entries: huge, heavy, light cells; dense cells, dense work
// items (slices), dense cells of more than one slice
constexpr int kCntHuge = 0, kCntHeavy = 1, kCntLight = 2, kCntDense = 3, kCntWork = 4, kCntMulti = 5, kCntWords = 8;
// The i-th huge or heavy cell, or -1 past their end.
__device__ __forceinline__ int64_t cell_at(int64_t i, const int32_t *list, const uint32_t *cnt, int64_t ncell) {
    const int64_t h = cnt[0];
    if (i < h) return list[i];
    i -= h;
    return i < (int64_t)cnt[1] ? list[ncell - 1 - i] : -1;
}
// cell of a voxel inside its brick (local voxel coordinates in [0, res0))
__device__ __forceinline__ int cell_of_local(int lx, int ly, int lz, int m) {
    return ((lz >> 3) * m + (ly >> 3)) * m + (lx >> 3);
}
// brick-local coordinate that may lie in a neighbouring brick: the step to
// that brick (-1, 0, 1) and the coordinate inside it
__device__ __forceinline__ int brick_step(int L, int res0, int &local) {
    const int d = L < 0 ? -1 : (L >= res0 ? 1 : 0);
    local = L - d * res0;
    return d;
}

__device__ __forceinline__ bool hs_contains(const uint64_t *keys, uint32_t mask, uint64_t key) {
    uint32_t h = hash_key(key) & mask;
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        uint64_t cur = __ldg(keys + h);
        if (cur == key) return true;
        if (cur == kEmptyKey) return false;
        h = (h + 1) & mask;
    }
    return false;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Warp-aggregated atomicAdd on counters[idx] by 1 for every active lane in
// `active`; returns this lane's rank (the old value + position in group).
__device__ __forceinline__ uint32_t warp_agg_inc(uint32_t *counters, uint32_t idx, uint32_t active) {
    uint32_t peers = __match_any_sync(active, idx);
    int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if ((threadIdx.x & 31) == leader) base = atomicAdd(counters + idx, (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + __popc(peers & lanemask_lt());
}

__device__ __forceinline__ int floor_div(int a, int b) { // b > 0
    int q = a / b;
    return (a % b != 0 && a < 0) ? q - 1 : q;
}

// Per-axis taps of the kernel splats: voxel centres at i + 0.5.
// Tent (radius 1): taps first + {0,1}; cubic B-spline (radius 2): first + {-1..2}.
template <int KERNEL>
struct Taps;

template <>
struct Taps<GVDB2_KERNEL_TENT1> {
    static constexpr int N = 2;
    static constexpr int LO = 0; // first tap = floor(x - 0.5) - LO
    __device__ __forceinline__ static int eval(float x, float w[2]) {
        float u = x - 0.5f;
        float b = floorf(u);
        float t = u - b;
        w[0] = 1.0f - t;
        w[1] = t;
        return (int)b;
    }
    __device__ __forceinline__ static int eval_d(float x, float w[2], float dw[2]) {
        int f = eval(x, w);
        dw[0] = -1.0f;
        dw[1] = 1.0f;
        return f;
    }
};

template <>
struct Taps<GVDB2_KERNEL_CUBIC2> {
    static constexpr int N = 4;
    static constexpr int LO = 1;
    __device__ __forceinline__ static int eval(float x, float w[4]) {
        float u = x - 0.5f;
        float b = floorf(u);
        float t = u - b;
        float s = 1.0f - t;
        const float k6 = 1.0f / 6.0f;
        w[0] = s * s * s * k6;
        w[1] = ((3.0f * t - 6.0f) * t * t + 4.0f) * k6;
        w[2] = (((-3.0f * t + 3.0f) * t + 3.0f) * t + 1.0f) * k6;
        w[3] = t * t * t * k6;
        return (int)b - 1;
    }
    __device__ __forceinline__ static int eval_d(float x, float w[4], float dw[4]) {
        float u = x - 0.5f;
        float b = floorf(u);
        float t = u - b;
        float s = 1.0f - t;
        const float k6 = 1.0f / 6.0f;
        w[0] = s * s * s * k6;
        w[1] = ((3.0f * t - 6.0f) * t * t + 4.0f) * k6;
        w[2] = (((-3.0f * t + 3.0f) * t + 3.0f) * t + 1.0f) * k6;
        w[3] = t * t * t * k6;
        dw[0] = -0.5f * s * s;
        dw[1] = (1.5f * t - 2.0f) * t;
        dw[2] = (-1.5f * t + 1.0f) * t + 0.5f;
        dw[3] = 0.5f * t * t;
        return (int)b - 1;
    }
};

inline int grid_for(int64_t n, int threads, int64_t cap = 1 << 20) {
    int64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

} // namespace gvdb2
