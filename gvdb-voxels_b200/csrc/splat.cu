// splat.cu -- point -> grid scatter, grid -> point gather and their adjoints.
//
// Reference-mode operations:
//   ScatterDensity  (V:5624-5660, P:516-573): distFunc splat at the voxel
//     corner pi = int(p) (+6 face neighbours with expand), channel 0.  The
//     reference's read-modify-write races; here it is an atomic add.
//   GatherDensity / GatherLevelSet (V:5318-5373, P:696-773): per voxel of
//     each subcell, max(r - |p - v|) / min(|p - v| - r) over its list.
// Kernel splats (no reference counterpart): tent (r=1) and cubic B-spline
// (r=2) scatter onto brick interiors and gather back to points.  One CTA
// owns one atlas slot: it accumulates the brick interior in shared memory
// from the brick's own points and the boundary regions of its 26
// neighbours (binning in points.cu), then writes the interior once with
// coalesced stores -- no global atomics, no zero-fill pass.  The gather
// stages the brick plus a 1- or 2-voxel halo from the neighbours'
// interiors in shared memory and serves all of the brick's points from it.
#include <algorithm>

#include "dev_common.cuh"

namespace gvdb2 {

namespace {

// ---------------------------------------------------------------------
// reference mode
// ---------------------------------------------------------------------
__device__ __forceinline__ float dist_func(float ax, float ay, float az, float bx, float by, float bz, float r) {
    bx -= ax;
    by -= ay;
    bz -= az;
    float c = (bx * bx + by * by + bz * bz) / (r * r);
    return 1.0f + c * (-3.0f + c * (3.0f - c));
}

struct AtlasGeom {
    int tile;      // res0 + 2*apron
    int64_t tvox;  // tile^3
    int sx, sy, sz; // atlas brick counts per axis
};

// atlas voxel coordinate -> linear index into a channel, -1 outside
__device__ __forceinline__ int64_t atlas_index(const AtlasGeom &A, int qx, int qy, int qz) {
    if (qx < 0 || qy < 0 || qz < 0) return -1;
    int bx = qx / A.tile, by = qy / A.tile, bz = qz / A.tile;
    if (bx >= A.sx || by >= A.sy || bz >= A.sz) return -1;
    int64_t slot = ((int64_t)bz * A.sy + by) * A.sx + bx;
    int lx = qx - bx * A.tile, ly = qy - by * A.tile, lz = qz - bz * A.tile;
    return slot * A.tvox + ((int64_t)lz * A.tile + ly) * A.tile + lx;
}

__global__ void k_scatter_ref(PointsView pos, int64_t n, float radius, float3 trans, int expand, const int32_t *pnode,
                              int64_t nleaves, const Node *leaves, int res0, AtlasGeom A, float *chan) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t nid = pnode[i];
    if (nid < 0 || nid >= nleaves) return;
    const Node &nd = leaves[nid];
    float3 pp = load_f3(pos, i);
    float p[3] = {pp.x + trans.x - (float)nd.mPos[0], pp.y + trans.y - (float)nd.mPos[1],
                  pp.z + trans.z - (float)nd.mPos[2]};
    float pi[3] = {(float)(int)p[0], (float)(int)p[1], (float)(int)p[2]};
    if (pi[0] < 0 || pi[1] < 0 || pi[2] < 0 || pi[0] >= res0 || pi[1] >= res0 || pi[2] >= res0) return;
    const int nb[7][3] = {{0, 0, 0}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    int cnt = expand ? 7 : 1;
    for (int k = 0; k < cnt; k++) {
        int q[3];
        for (int a = 0; a < 3; a++) q[a] = (int)pi[a] + nb[k][a] + nd.mValue[a];
        int64_t idx = atlas_index(A, q[0], q[1], q[2]);
        if (idx < 0) continue;
        float w = dist_func(p[0], p[1], p[2], pi[0] + nb[k][0], pi[1] + nb[k][1], pi[2] + nb[k][2], radius);
        atomicAdd(chan + idx, w);
    }
}

// gvdbGatherDensity / gvdbGatherLevelSet: one CTA per mapped leaf, one
// thread per voxel of its subcells.
template <bool LEVELSET>
__global__ void k_gather_voxels(int64_t num_sc, int scpb, int sc, float radius, const int32_t *sc_nid,
                                const uint32_t *sc_cnt, const uint32_t *sc_off, const int32_t *sc_pos, const float *pnt,
                                const Node *leaves, int apron, AtlasGeom A, float *chan, int accum) {
    int sc3 = sc * sc * sc;
    int64_t sid = (int64_t)blockIdx.x * scpb + threadIdx.x / sc3;
    if (threadIdx.x >= scpb * sc3 || sid >= num_sc) return;
    int t = threadIdx.x % sc3;
    int tx = t % sc, ty = (t / sc) % sc, tz = t / (sc * sc);
    int wx = sc_pos[3 * sid + 0] + tx, wy = sc_pos[3 * sid + 1] + ty, wz = sc_pos[3 * sid + 2] + tz;
    const Node &nd = leaves[sc_nid[sid]];
    int64_t idx = atlas_index(A, nd.mValue[0] + wx - nd.mPos[0], nd.mValue[1] + wy - nd.mPos[1],
                              nd.mValue[2] + wz - nd.mPos[2]);
    if (idx < 0) return;
    float val = accum ? chan[idx] : (LEVELSET ? 3.0f : 0.0f);
    uint32_t beg = sc_off[sid], cnt = sc_cnt[sid];
    float fx = (float)wx, fy = (float)wy, fz = (float)wz;
    for (uint32_t j = 0; j < cnt; j++) {
        const float *p = pnt + 3 * (int64_t)(beg + j);
        float dx = p[0] - fx, dy = p[1] - fy, dz = p[2] - fz;
        float c = sqrtf(dx * dx + dy * dy + dz * dz);
        if (LEVELSET) val = fminf(val, c - radius);
        else val = fmaxf(val, radius - c);
    }
    chan[idx] = val;
}

// The same gathers for 4^3 subcells, one warp per subcell.  Each lane owns
// two x-adjacent voxels of one (y, z) column, so the y/z part of a squared
// distance is shared.  The subcell's points are staged through shared memory
// in chunks of 64 (one float4 broadcast per point).  The minimum squared
// distance is reduced first and the square root taken once: sqrt and the
// subtraction of the radius are monotonic, so max(r - c) = r - sqrt(min d^2)
// and min(c - r) = sqrt(min d^2) - r, as in P:725-728 / P:764-767.
constexpr int kGvWarps = 8;
template <bool LEVELSET>
__global__ void __launch_bounds__(32 * kGvWarps) k_gather_voxels_sc4(int64_t num_sc, float radius,
                                                                     const int32_t *sc_nid, const uint32_t *sc_cnt,
                                                                     const uint32_t *sc_off, const int32_t *sc_pos,
                                                                     const float *pnt, const Node *leaves, AtlasGeom A,
                                                                     float *chan, int accum) {
    __shared__ float4 buf[kGvWarps][64];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t sid = (int64_t)blockIdx.x * kGvWarps + warp;
    if (sid >= num_sc) return;
    const int col = lane >> 1, tx = (lane & 1) * 2, ty = col & 3, tz = col >> 2;
    const int wx = sc_pos[3 * sid + 0] + tx, wy = sc_pos[3 * sid + 1] + ty, wz = sc_pos[3 * sid + 2] + tz;
    const Node &nd = leaves[sc_nid[sid]];
    const int64_t idx = atlas_index(A, nd.mValue[0] + wx - nd.mPos[0], nd.mValue[1] + wy - nd.mPos[1],
                                    nd.mValue[2] + wz - nd.mPos[2]);
    const float init = LEVELSET ? 3.0f : 0.0f;
    float v0 = init, v1 = init;
    if (accum && idx >= 0) {
        v0 = chan[idx];
        v1 = chan[idx + 1];
    }
    const uint32_t beg = sc_off[sid], cnt = sc_cnt[sid];
    const float fx0 = (float)wx, fx1 = (float)(wx + 1), fy = (float)wy, fz = (float)wz;
    float m0 = INFINITY, m1 = INFINITY;
    float4 *wb = buf[warp];
    for (uint32_t base = 0; base < cnt; base += 64) {
        const uint32_t m = min(64u, cnt - base);
        for (uint32_t k = lane; k < m; k += 32) {
            const float *q = pnt + 3 * (int64_t)(beg + base + k);
            wb[k] = make_float4(q[0], q[1], q[2], 0.0f);
        }
        __syncwarp();
        for (uint32_t j = 0; j < m; j++) {
            const float4 q = wb[j];
            const float dy = q.y - fy, dz = q.z - fz;
            const float syz = fmaf(dy, dy, dz * dz);
            const float dx0 = q.x - fx0, dx1 = q.x - fx1;
            m0 = fminf(m0, fmaf(dx0, dx0, syz));
            m1 = fminf(m1, fmaf(dx1, dx1, syz));
        }
        __syncwarp();
    }
    if (idx < 0) return;
    const float c0 = sqrtf(m0), c1 = sqrtf(m1);
    if (LEVELSET) {
        v0 = fminf(v0, c0 - radius);
        v1 = fminf(v1, c1 - radius);
    } else {
        v0 = fmaxf(v0, radius - c0);
        v1 = fmaxf(v1, radius - c1);
    }
    chan[idx] = v0;
    chan[idx + 1] = v1;
}

// ---------------------------------------------------------------------
// kernel splats
// ---------------------------------------------------------------------
struct SplatArgs {
    PointsView pos;
    float3 trans;
    PointsView weight;
    float wconst;
    int has_weight;
    PointsView attr[kMaxSplatChan];
    uint32_t attr_mask;
    float *chan[kMaxSplatChan];
    int nch;
    const int32_t *slot_leaf;
    const Node *leaves;
    const int32_t *nbr27;
    const uint32_t *bin_off;
    const int32_t *perm;
    int res0, log2r0, apron, tile;
    int64_t tvox;
};

// The bins of neighbour k = (dx,dy,dz) whose points reach this brick:
// along an axis with d = 0 every region, d = -1 the neighbour's high
// region (2), d = +1 its low region (0).  Ranges are listed per (cz, cy)
// row: up to 9 per neighbour, 243 per brick.
constexpr int kRangeSlots = 27 * 9;

__device__ __forceinline__ void neighbour_range(const SplatArgs &S, int64_t slot, int t, uint32_t &beg, uint32_t &end) {
    beg = end = 0;
    int k = t / 9, r = t % 9;
    int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
    int32_t nb = S.nbr27[slot * 27 + k];
    if (nb < 0) return;
    int ylo = dy == 0 ? 0 : (dy < 0 ? 2 : 0), yn = dy == 0 ? 3 : 1;
    int zlo = dz == 0 ? 0 : (dz < 0 ? 2 : 0), zn = dz == 0 ? 3 : 1;
    int xlo = dx == 0 ? 0 : (dx < 0 ? 2 : 0), xhi = dx == 0 ? 2 : xlo;
    if (r >= yn * zn) return;
    int cy = ylo + r % yn, cz = zlo + r / yn;
    int64_t base = (int64_t)nb * 27 + (cz * 3 + cy) * 3;
    beg = S.bin_off[base + xlo];
    end = S.bin_off[base + xhi + 1];
}

// Block-wide exclusive scan of one value per thread (warp_tot: 33 words).
__device__ __forceinline__ uint32_t block_scan_excl(uint32_t x, uint32_t *warp_tot, uint32_t &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? warp_tot[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < nw) warp_tot[lane] = wi - w;
        if (lane == 31) warp_tot[32] = wi;
    }
    __syncthreads();
    uint32_t ex = warp_tot[warp] + inc - x;
    total = warp_tot[32];
    __syncthreads();
    return ex;
}

// Per-channel max |weight * attr| over all points (bounds the fixed-point
// scale of k_scatter_fixed).  out[c] holds the float bits (>= 0 orders as int).
template <int NCH>
__global__ void k_absmax(SplatArgs S, int64_t n, int32_t *out) {
    float m[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) m[c] = 0.0f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float wt = fabsf(S.has_weight ? load_f1(S.weight, i) : S.wconst);
#pragma unroll
        for (int c = 0; c < NCH; c++) m[c] = fmaxf(m[c], ((S.attr_mask >> c) & 1) ? wt * fabsf(load_f1(S.attr[c], i)) : wt);
    }
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        float x = m[c];
        for (int o = 16; o > 0; o >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, o));
        if ((threadIdx.x & 31) == 0) atomicMax(out + c, __float_as_int(x));
    }
}

// Default scatter: one CTA per atlas slot accumulates its 8^3 interior in
// shared memory from its own points and the boundary regions of its 26
// neighbours, then writes the interior once with coalesced stores.  Every
// (point, voxel) pair is added exactly once, by the CTA owning the voxel.
//
// Accumulation is fixed point in two int32 words per voxel: a contribution
// v becomes x = rint(v * 2^s) (64-bit), split into hi = x >> L and
// lo = x & (2^L - 1), each added with a native shared-memory integer atomic
// (B200 runs float shared atomics as compare-and-swap loops, integer ones in
// hardware).  L = 31 - ceil(log2(records + 1)) keeps the lo sums below 2^31;
// s is chosen so that records * max|a| * 2^s < 2^(29 + L), which bounds the
// hi sums below 2^30.  Integer sums do not depend on the order of the
// atomics, so the result is bit-reproducible run to run; each contribution
// is rounded once (to float, as a float splat would) and the sum is exact.
constexpr int kAtomicThreads = 256;
constexpr int kAccPlane = 72; // 8x8 plane padded by 8 words: z-neighbours fall in other banks

template <int KERNEL, int NCH>
__global__ void __launch_bounds__(kAtomicThreads, 6) k_scatter_fixed(SplatArgs S, const int32_t *absmax) {
    using T = Taps<KERNEL>;
    constexpr int N = T::N, RES = 8, ACC = RES * kAccPlane;
    __shared__ int32_t acc_hi[NCH * ACC], acc_lo[NCH * ACC];
    __shared__ uint32_t r_beg[kRangeSlots], r_pre[kRangeSlots + 1];
    __shared__ uint32_t wtot[33];
    const int64_t slot = blockIdx.x;
    for (int i = threadIdx.x; i < NCH * ACC; i += blockDim.x) acc_hi[i] = acc_lo[i] = 0;
    uint32_t b = 0, e = 0;
    if (threadIdx.x < kRangeSlots) neighbour_range(S, slot, threadIdx.x, b, e);
    uint32_t total;
    const uint32_t ex = block_scan_excl(e - b, wtot, total); // ends with a barrier
    if (threadIdx.x < kRangeSlots) {
        r_beg[threadIdx.x] = b;
        r_pre[threadIdx.x] = ex;
    }
    __syncthreads();
    const int L = 31 - (32 - __clz((int)total + 1));
    __shared__ float scale_s[NCH];
    float scale[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        const float bound = (float)total * __int_as_float(absmax[c]);
        int ex2 = 0;
        frexpf(bound, &ex2); // bound < 2^ex2
        scale[c] = bound > 0.0f ? ldexpf(1.0f, 29 + L - ex2) : 0.0f;
        if (threadIdx.x == 0) scale_s[c] = scale[c];
    }
    const Node &nd = S.leaves[S.slot_leaf[slot]];
    const int ox = nd.mPos[0], oy = nd.mPos[1], oz = nd.mPos[2];
    const long long lmask = (1ll << L) - 1;
    for (uint32_t j = threadIdx.x; j < total; j += blockDim.x) {
        int lo = 0, hi = kRangeSlots - 1; // last range with r_pre <= j
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (r_pre[mid] <= j) lo = mid;
            else hi = mid - 1;
        }
        const int32_t p = S.perm[r_beg[lo] + (j - r_pre[lo])];
        const float3 q = load_f3(S.pos, p);
        float wx[N], wy[N], wz[N];
        const int fx = T::eval(q.x + S.trans.x, wx) - ox;
        const int fy = T::eval(q.y + S.trans.y, wy) - oy;
        const int fz = T::eval(q.z + S.trans.z, wz) - oz;
        const float wt = S.has_weight ? load_f1(S.weight, p) : S.wconst;
        float amt[NCH];
#pragma unroll
        for (int c = 0; c < NCH; c++) amt[c] = ((S.attr_mask >> c) & 1) ? wt * load_f1(S.attr[c], p) : wt;
#pragma unroll
        for (int c = 0; c < NCH; c++) amt[c] *= scale[c];
        // z taps in a rolled loop (the weights rotate through registers) keep
        // the unrolled body small enough for the instruction cache
#pragma unroll 1
        for (int tz = 0; tz < N; tz++) {
            const int lz = fz + tz;
            const float wzt = wz[0];
#pragma unroll
            for (int k = 0; k + 1 < N; k++) wz[k] = wz[k + 1];
            if ((unsigned)lz >= (unsigned)RES) continue;
#pragma unroll
            for (int ty = 0; ty < N; ty++) {
                const int ly = fy + ty;
                if ((unsigned)ly >= (unsigned)RES) continue;
                const float wyz = wy[ty] * wzt;
                const int row = lz * kAccPlane + ly * RES;
#pragma unroll
                for (int tx = 0; tx < N; tx++) {
                    const int lx = fx + tx;
                    if ((unsigned)lx >= (unsigned)RES) continue;
                    const float w = wx[tx] * wyz;
#pragma unroll
                    for (int c = 0; c < NCH; c++) {
                        const long long xv = __float2ll_rn(amt[c] * w);
                        atomicAdd(&acc_hi[c * ACC + row + lx], (int)(xv >> L));
                        atomicAdd(&acc_lo[c * ACC + row + lx], (int)(xv & lmask));
                    }
                }
            }
        }
    }
    __syncthreads();
    const int a = S.apron, tl = S.tile;
    for (int i = threadIdx.x; i < NCH * RES * RES * RES; i += blockDim.x) {
        const int c = i >> 9, v = i & 511;
        const int lx = v & 7, ly = (v >> 3) & 7, lz = v >> 6;
        const int k = c * ACC + lz * kAccPlane + ly * RES + lx;
        const long long sum = ((long long)acc_hi[k] << L) + (long long)acc_lo[k];
        const float sc = scale_s[c];
        const float val = sc > 0.0f ? (float)((double)sum / (double)sc) : 0.0f;
        if (c < S.nch) S.chan[c][slot * S.tvox + ((int64_t)(lz + a) * tl + (ly + a)) * tl + (lx + a)] = val;
    }
}

constexpr int kScatterThreads = 512; // one thread per interior voxel of an 8^3 brick
constexpr int kScatterRes = 8;

// Shared-memory bytes of k_scatter_tile for a record capacity `cap`.
__host__ __device__ constexpr size_t scatter_smem_bytes(int ntaps, int nch, int cap) {
    return (size_t)cap * (3 * ntaps + nch + 1) * 4 + (size_t)cap * 6 +
           (size_t)((kScatterRes + ntaps - 1) * (kScatterRes + ntaps - 1) * (kScatterRes + ntaps - 1) + 1) * 4;
}

// Scatter as a gather over shared memory: one CTA per atlas slot, one
// thread per interior voxel.  The CTA stages the records of every point
// whose stencil reaches the brick (its own points and the boundary regions
// of its 26 neighbours): per-axis tap weights, weighted attributes and the
// point index.  Records are counting-sorted by the stencil's first tap
// (a cell of (8+N-1)^3) and each cell's records are ordered by point index.
// A voxel then sums the N^3 cells whose stencils cover it in a fixed order:
// no atomics on the accumulators, and the sum order does not depend on the
// order in which points were binned (bit-reproducible while a brick's
// records fit one chunk; the deterministic option also makes the binning
// stable so multi-chunk bricks reproduce too).
template <int KERNEL, int NCH>
__global__ void __launch_bounds__(kScatterThreads, 3) k_scatter_tile(SplatArgs S, int cap) {
    using T = Taps<KERNEL>;
    constexpr int N = T::N, RES = kScatterRes, CA = RES + N - 1, C3 = CA * CA * CA;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *wgt = reinterpret_cast<float *>(smem_raw); // [3*N][cap]
    float *att = wgt + 3 * N * cap;                    // [NCH][cap]
    int32_t *pid = reinterpret_cast<int32_t *>(att + NCH * cap);
    uint16_t *cellof = reinterpret_cast<uint16_t *>(pid + cap);
    uint16_t *order = cellof + cap;
    uint32_t *coff = reinterpret_cast<uint32_t *>(order + cap); // [C3 + 1]
    uint8_t *tx0 = reinterpret_cast<uint8_t *>(coff + C3 + 1); // first x tap (cell coordinate)
    __shared__ uint32_t r_beg[kRangeSlots], r_pre[kRangeSlots + 1];
    __shared__ uint32_t wtot[33];
    const int64_t slot = blockIdx.x;

    uint32_t b = 0, e = 0;
    if (threadIdx.x < kRangeSlots) neighbour_range(S, slot, threadIdx.x, b, e);
    uint32_t total;
    uint32_t ex = block_scan_excl(e - b, wtot, total);
    if (threadIdx.x < kRangeSlots) {
        r_beg[threadIdx.x] = b;
        r_pre[threadIdx.x] = ex;
    }
    if (threadIdx.x == 0) r_pre[kRangeSlots] = total;
    const Node &nd = S.leaves[S.slot_leaf[slot]];
    const int ox = nd.mPos[0], oy = nd.mPos[1], oz = nd.mPos[2];
    const int vx = threadIdx.x & 7, vy = (threadIdx.x >> 3) & 7, vz = threadIdx.x >> 6;
    float acc[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) acc[c] = 0.0f;

    for (uint32_t base = 0; base < total; base += cap) {
        const int cnt = (int)min((uint32_t)cap, total - base);
        for (int i = threadIdx.x; i <= C3; i += blockDim.x) coff[i] = 0;
        __syncthreads();
        // stage records
        for (int r = threadIdx.x; r < cnt; r += blockDim.x) {
            const uint32_t j = base + r;
            int lo = 0, hi = kRangeSlots - 1; // last range with r_pre <= j
            while (lo < hi) {
                int mid = (lo + hi + 1) >> 1;
                if (r_pre[mid] <= j) lo = mid;
                else hi = mid - 1;
            }
            const int32_t p = S.perm[r_beg[lo] + (j - r_pre[lo])];
            const float3 q = load_f3(S.pos, p);
            float wx[N], wy[N], wz[N];
            const int tx = T::eval(q.x + S.trans.x, wx) - ox + N - 1;
            const int ty = T::eval(q.y + S.trans.y, wy) - oy + N - 1;
            const int tz = T::eval(q.z + S.trans.z, wz) - oz + N - 1;
#pragma unroll
            for (int k = 0; k < N; k++) {
                wgt[(0 * N + k) * cap + r] = wx[k];
                wgt[(1 * N + k) * cap + r] = wy[k];
                wgt[(2 * N + k) * cap + r] = wz[k];
            }
            const float wt = S.has_weight ? load_f1(S.weight, p) : S.wconst;
#pragma unroll
            for (int c = 0; c < NCH; c++) att[c * cap + r] = ((S.attr_mask >> c) & 1) ? wt * load_f1(S.attr[c], p) : wt;
            pid[r] = p;
            const bool ok = tx >= 0 && tx < CA && ty >= 0 && ty < CA && tz >= 0 && tz < CA;
            const int cell = ok ? (tz * CA + ty) * CA + tx : C3;
            cellof[r] = (uint16_t)cell;
            tx0[r] = (uint8_t)tx;
            if (ok) atomicAdd(&coff[cell], 1u);
        }
        __syncthreads();
        // exclusive scan of the cell counts: thread t owns cells [t*K, t*K+K)
        {
            constexpr int K = (C3 + kScatterThreads - 1) / kScatterThreads;
            uint32_t loc[K], sum = 0;
#pragma unroll
            for (int k = 0; k < K; k++) {
                int i = threadIdx.x * K + k;
                loc[k] = i < C3 ? coff[i] : 0u;
                sum += loc[k];
            }
            uint32_t tot;
            uint32_t run = block_scan_excl(sum, wtot, tot);
#pragma unroll
            for (int k = 0; k < K; k++) {
                int i = threadIdx.x * K + k;
                if (i < C3) coff[i] = run;
                run += loc[k];
            }
        }
        __syncthreads();
        // place; afterwards coff[c] is the end of cell c (start = coff[c-1])
        for (int r = threadIdx.x; r < cnt; r += blockDim.x) {
            const int cell = cellof[r];
            if (cell < C3) order[atomicAdd(&coff[cell], 1u)] = (uint16_t)r;
        }
        __syncthreads();
        // order each cell's records by point index
        for (int c = threadIdx.x; c < C3; c += blockDim.x) {
            const int s0 = c ? (int)coff[c - 1] : 0, s1 = (int)coff[c];
            for (int k = s0 + 1; k < s1; k++) {
                const uint16_t rk = order[k];
                const int32_t pk = pid[rk];
                int m = k - 1;
                while (m >= s0 && pid[order[m]] > pk) {
                    order[m + 1] = order[m];
                    m--;
                }
                order[m + 1] = rk;
            }
        }
        __syncthreads();
        // this thread's voxel sums the records whose stencils cover it.  For
        // fixed (dz, dy) the N cells of x offsets 0..N-1 are adjacent in the
        // sorted order, so each row is one contiguous range of records.
#pragma unroll 1
        for (int dz = 0; dz < N; dz++) {
#pragma unroll 1
            for (int dy = 0; dy < N; dy++) {
                const int chi = ((vz - dz + N - 1) * CA + (vy - dy + N - 1)) * CA + (vx + N - 1);
                const int clo = chi - (N - 1);
                const int s0 = clo ? (int)coff[clo - 1] : 0, s1 = (int)coff[chi];
                for (int k = s0; k < s1; k++) {
                    const int r = order[k];
                    const int dx = vx + N - 1 - tx0[r];
                    const float w = wgt[(0 * N + dx) * cap + r] * wgt[(1 * N + dy) * cap + r] * wgt[(2 * N + dz) * cap + r];
#pragma unroll
                    for (int c = 0; c < NCH; c++) acc[c] = fmaf(att[c * cap + r], w, acc[c]);
                }
            }
        }
        __syncthreads();
    }
    const int a = S.apron, tl = S.tile;
    const int64_t at = slot * S.tvox + ((int64_t)(vz + a) * tl + (vy + a)) * tl + (vx + a);
#pragma unroll
    for (int c = 0; c < NCH; c++)
        if (c < S.nch) S.chan[c][at] = acc[c];
}

// ---------------------------------------------------------------------
// tiled gathers: forward, scatter adjoint, gather adjoint
// ---------------------------------------------------------------------
enum GatherMode { kFwd = 0, kScatterBwd = 1, kGatherBwd = 2 };

struct GatherArgs {
    PointsView pos;
    float3 trans;
    const float *chan[kMaxSplatChan];
    int nch;
    float *out;          // kFwd: out[p*out_stride + c]
    int64_t out_stride;
    PointsView weight;   // kScatterBwd
    float wconst;
    int has_weight;
    PointsView attr[kMaxSplatChan];
    uint32_t attr_mask;
    float *grad_pos, *grad_weight, *grad_attr;
    const float *grad_out; // kGatherBwd: [p*nch + c]
    const int32_t *slot_leaf;
    const Node *leaves;
    const int32_t *nbr27;
    const uint32_t *bin_off;
    const int32_t *perm;
    int res0, apron, tile;
    int64_t tvox;
};

template <int KERNEL, int MODE, int NCH>
__global__ void __launch_bounds__(256) k_gather_tile(GatherArgs G) {
    using T = Taps<KERNEL>;
    constexpr int H = T::N / 2;
    constexpr int N = T::N;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *tile = reinterpret_cast<float *>(smem_raw);
    __shared__ int32_t nbs[27];
    const int res = G.res0, ht = res + 2 * H, ht3 = ht * ht * ht;
    const int64_t slot = blockIdx.x;
    const int a = G.apron, tl = G.tile;
    if (threadIdx.x < 27) nbs[threadIdx.x] = G.nbr27[slot * 27 + threadIdx.x];
    __syncthreads();
    // halo tile from the interiors of this brick and its neighbours
    for (int i = threadIdx.x; i < ht3; i += blockDim.x) {
        const int lx = i % ht - H, ly = (i / ht) % ht - H, lz = i / (ht * ht) - H;
        const int dx = lx < 0 ? -1 : (lx >= res ? 1 : 0), dy = ly < 0 ? -1 : (ly >= res ? 1 : 0),
                  dz = lz < 0 ? -1 : (lz >= res ? 1 : 0);
        const int32_t nb = nbs[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)];
        const int64_t off = (int64_t)nb * G.tvox +
                            ((int64_t)(lz - dz * res + a) * tl + (ly - dy * res + a)) * tl + (lx - dx * res + a);
#pragma unroll
        for (int c = 0; c < NCH; c++) tile[c * ht3 + i] = nb >= 0 ? __ldg(G.chan[c] + off) : 0.0f;
    }
    __syncthreads();
    const Node &nd = G.leaves[G.slot_leaf[slot]];
    const int ox = nd.mPos[0] - H, oy = nd.mPos[1] - H, oz = nd.mPos[2] - H;
    const uint32_t beg = G.bin_off[slot * 27], end = G.bin_off[slot * 27 + 27];
    for (uint32_t j = beg + threadIdx.x; j < end; j += blockDim.x) {
        const int32_t pidx = G.perm[j];
        const float3 p = load_f3(G.pos, pidx);
        float wx[N], wy[N], wz[N], dx[N], dy[N], dz[N];
        int fx, fy, fz;
        if (MODE == kFwd) {
            fx = T::eval(p.x + G.trans.x, wx) - ox;
            fy = T::eval(p.y + G.trans.y, wy) - oy;
            fz = T::eval(p.z + G.trans.z, wz) - oz;
        } else {
            fx = T::eval_d(p.x + G.trans.x, wx, dx) - ox;
            fy = T::eval_d(p.y + G.trans.y, wy, dy) - oy;
            fz = T::eval_d(p.z + G.trans.z, wz, dz) - oz;
        }
        float sum[NCH], gx[NCH], gy[NCH], gz[NCH];
#pragma unroll
        for (int c = 0; c < NCH; c++) sum[c] = gx[c] = gy[c] = gz[c] = 0.0f;
#pragma unroll
        for (int tz = 0; tz < N; tz++) {
#pragma unroll
            for (int ty = 0; ty < N; ty++) {
                const int row = ((fz + tz) * ht + (fy + ty)) * ht + fx;
                const float wyz = wy[ty] * wz[tz];
                float dyz = 0.0f, ydz = 0.0f;
                if (MODE != kFwd) {
                    dyz = dy[ty] * wz[tz];
                    ydz = wy[ty] * dz[tz];
                }
#pragma unroll
                for (int tx = 0; tx < N; tx++) {
#pragma unroll
                    for (int c = 0; c < NCH; c++) {
                        const float g = tile[c * ht3 + row + tx];
                        if (MODE != kGatherBwd) sum[c] = fmaf(g, wx[tx] * wyz, sum[c]);
                        if (MODE != kFwd) {
                            gx[c] = fmaf(g, dx[tx] * wyz, gx[c]);
                            gy[c] = fmaf(g, wx[tx] * dyz, gy[c]);
                            gz[c] = fmaf(g, wx[tx] * ydz, gz[c]);
                        }
                    }
                }
            }
        }
        if (MODE == kFwd) {
#pragma unroll
            for (int c = 0; c < NCH; c++) G.out[(int64_t)pidx * G.out_stride + c] = sum[c];
        } else if (MODE == kScatterBwd) {
            const float wt = G.has_weight ? load_f1(G.weight, pidx) : G.wconst;
            float gw = 0.0f, gp0 = 0.0f, gp1 = 0.0f, gp2 = 0.0f;
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                const bool has = (G.attr_mask >> c) & 1;
                const float at = has ? load_f1(G.attr[c], pidx) : 1.0f;
                if (G.grad_attr) G.grad_attr[(int64_t)pidx * NCH + c] = has ? wt * sum[c] : 0.0f;
                gw += at * sum[c];
                gp0 += wt * at * gx[c];
                gp1 += wt * at * gy[c];
                gp2 += wt * at * gz[c];
            }
            if (G.grad_weight) G.grad_weight[pidx] = gw;
            if (G.grad_pos) {
                G.grad_pos[3 * (int64_t)pidx + 0] = gp0;
                G.grad_pos[3 * (int64_t)pidx + 1] = gp1;
                G.grad_pos[3 * (int64_t)pidx + 2] = gp2;
            }
        } else {
            float gp0 = 0.0f, gp1 = 0.0f, gp2 = 0.0f;
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                const float go = G.grad_out[(int64_t)pidx * NCH + c];
                gp0 += go * gx[c];
                gp1 += go * gy[c];
                gp2 += go * gz[c];
            }
            G.grad_pos[3 * (int64_t)pidx + 0] = gp0;
            G.grad_pos[3 * (int64_t)pidx + 1] = gp1;
            G.grad_pos[3 * (int64_t)pidx + 2] = gp2;
        }
    }
}

// Points outside every active brick: gathers and gradients are zero.
__global__ void k_zero_unbinned(const int32_t *pbin, int64_t n, float *out, int64_t stride, int ncols) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !out) return;
    if (pbin[i] >= 0) return;
    for (int c = 0; c < ncols; c++) out[i * stride + c] = 0.0f;
}

AtlasGeom atlas_geom(const Volume *v) {
    AtlasGeom A;
    A.tile = v->tile_res();
    A.tvox = v->tile_vox();
    A.sx = v->subdim[0];
    A.sy = v->subdim[1];
    A.sz = v->subdim[2];
    return A;
}

gvdb2_status check_chans(Volume *v, const int *chans, int nch) {
    if (!chans || nch < 1 || nch > kMaxSplatChan) return fail(v, GVDB2_ERR_ARG, "1 to 8 channels per splat call");
    for (int c = 0; c < nch; c++)
        if (chans[c] < 0 || chans[c] >= kMaxChan || !v->has_chan[chans[c]]) return fail(v, GVDB2_ERR_ARG, "bad channel");
    return GVDB2_OK;
}

template <class Args>
void fill_topology(Volume *v, Args &S) {
    S.slot_leaf = v->slot_leaf.as<int32_t>();
    S.leaves = v->pool_ptr(0);
    S.nbr27 = v->nbr27.as<int32_t>();
    S.bin_off = v->bin_off.as<uint32_t>();
    S.perm = v->perm.as<int32_t>();
    S.res0 = v->res(0);
    S.apron = v->apron;
    S.tile = v->tile_res();
    S.tvox = v->tile_vox();
}

template <class K>
gvdb2_status launch_smem(Volume *v, K kernel, size_t smem, const char *what) {
    if (smem > 48 * 1024) {
        int dev_max = 0;
        GV_CUDA(v, cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, v->device));
        if ((int)smem > dev_max) return fail(v, GVDB2_ERR_UNSUPPORTED, std::string(what) + ": brick tile exceeds shared memory");
        GV_CUDA(v, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    return GVDB2_OK;
}

template <int KERNEL, int NCH>
gvdb2_status launch_scatter(Volume *v, const SplatArgs &S) {
    if (!v->deterministic) {
        int32_t *absmax = nullptr;
        GV_CUDA(v, cudaMallocAsync((void **)&absmax, sizeof(int32_t) * NCH, v->stream));
        GV_CUDA(v, cudaMemsetAsync(absmax, 0, sizeof(int32_t) * NCH, v->stream));
        const int64_t n = v->bin_key.n;
        if (n > 0)
            k_absmax<NCH><<<std::min(grid_for(n, 256), 4 * kSmCount), 256, 0, v->stream>>>(S, n, absmax);
        k_scatter_fixed<KERNEL, NCH><<<(unsigned)v->atlas_last, kAtomicThreads, 0, v->stream>>>(S, absmax);
        cudaError_t e = cudaGetLastError();
        cudaFreeAsync(absmax, v->stream);
        if (e != cudaSuccess) return cuda_fail(v, e, "k_scatter_fixed");
        return GVDB2_OK;
    }
    const int cap = NCH <= 4 ? 768 : 512;
    const size_t smem = scatter_smem_bytes(Taps<KERNEL>::N, NCH, cap);
    auto k = k_scatter_tile<KERNEL, NCH>;
    GV_TRY(launch_smem(v, k, smem, "scatter"));
    k<<<(unsigned)v->atlas_last, kScatterThreads, smem, v->stream>>>(S, cap);
    GV_CUDA(v, cudaGetLastError());
    return GVDB2_OK;
}

template <int KERNEL>
gvdb2_status launch_scatter_n(Volume *v, const SplatArgs &S) {
    switch (S.nch) {
    case 1: return launch_scatter<KERNEL, 1>(v, S);
    case 2: return launch_scatter<KERNEL, 2>(v, S);
    case 3: return launch_scatter<KERNEL, 3>(v, S);
    case 4: return launch_scatter<KERNEL, 4>(v, S);
    default: return launch_scatter<KERNEL, 8>(v, S);
    }
}

gvdb2_status run_scatter(Volume *v, int kernel, const SplatArgs &S) {
    if (v->atlas_last == 0) return GVDB2_OK;
    if (v->res(0) != kScatterRes)
        return fail(v, GVDB2_ERR_UNSUPPORTED, "kernel splats need 8^3 bricks (Configure(...,3))");
    return kernel == GVDB2_KERNEL_TENT1 ? launch_scatter_n<GVDB2_KERNEL_TENT1>(v, S)
                                        : launch_scatter_n<GVDB2_KERNEL_CUBIC2>(v, S);
}

template <int KERNEL, int MODE, int NCH>
gvdb2_status launch_gather(Volume *v, const GatherArgs &G) {
    constexpr int H = Taps<KERNEL>::N / 2;
    const int ht = v->res(0) + 2 * H;
    const size_t smem = sizeof(float) * (size_t)NCH * ht * ht * ht;
    auto k = k_gather_tile<KERNEL, MODE, NCH>;
    GV_TRY(launch_smem(v, k, smem, "gather"));
    k<<<(unsigned)v->atlas_last, 256, smem, v->stream>>>(G);
    GV_CUDA(v, cudaGetLastError());
    return GVDB2_OK;
}

template <int KERNEL, int MODE>
gvdb2_status launch_gather_n(Volume *v, const GatherArgs &G) {
    switch (G.nch) {
    case 1: return launch_gather<KERNEL, MODE, 1>(v, G);
    case 2: return launch_gather<KERNEL, MODE, 2>(v, G);
    case 3: return launch_gather<KERNEL, MODE, 3>(v, G);
    case 4: return launch_gather<KERNEL, MODE, 4>(v, G);
    default: break;
    }
    // 5..8 channels: two passes over channel groups (4 + rest)
    GatherArgs A = G, B = G;
    A.nch = 4;
    B.nch = G.nch - 4;
    for (int c = 0; c < 4; c++) {
        B.chan[c] = G.chan[4 + c];
        B.attr[c] = G.attr[4 + c];
    }
    B.attr_mask = G.attr_mask >> 4;
    if (MODE == kFwd) B.out = G.out + 4;
    if (MODE != kFwd) return fail(v, GVDB2_ERR_UNSUPPORTED, "adjoints take at most 4 channels per call");
    GV_TRY((launch_gather<KERNEL, MODE, 4>(v, A)));
    switch (B.nch) {
    case 1: return launch_gather<KERNEL, MODE, 1>(v, B);
    case 2: return launch_gather<KERNEL, MODE, 2>(v, B);
    case 3: return launch_gather<KERNEL, MODE, 3>(v, B);
    default: return launch_gather<KERNEL, MODE, 4>(v, B);
    }
}

template <int MODE>
gvdb2_status run_gather(Volume *v, int kernel, const GatherArgs &G) {
    if (v->atlas_last == 0) return GVDB2_OK;
    return kernel == GVDB2_KERNEL_TENT1 ? launch_gather_n<GVDB2_KERNEL_TENT1, MODE>(v, G)
                                        : launch_gather_n<GVDB2_KERNEL_CUBIC2, MODE>(v, G);
}

gvdb2_status splat_prologue(Volume *v, int kernel, int n, const float trans[3]) {
    if (kernel != GVDB2_KERNEL_TENT1 && kernel != GVDB2_KERNEL_CUBIC2) return fail(v, GVDB2_ERR_ARG, "unknown kernel");
    if (!v->atlas_valid) return fail(v, GVDB2_ERR_STATE, "UpdateAtlas must follow the topology rebuild");
    int h = kernel == GVDB2_KERNEL_TENT1 ? 1 : 2;
    if (v->res(0) < 2 * h) return fail(v, GVDB2_ERR_UNSUPPORTED, "brick too small for the kernel support");
    return bin_points(v, kernel, n, trans);
}

void set_attrs(uint32_t &mask, PointsView *dst, const gvdb2_points_view *attrs, int nch) {
    mask = 0;
    for (int c = 0; c < kMaxSplatChan; c++) dst[c] = PointsView{};
    for (int c = 0; c < nch; c++)
        if (attrs && attrs[c].base) {
            mask |= 1u << c;
            dst[c] = to_view(attrs[c]);
        }
}

} // namespace

gvdb2_status scatter_density_ref(Volume *v, int n, float radius, float amp, const float trans[3], int expand) {
    (void)amp; // unused by the reference kernel (P:525-573)
    if (!v->has_chan[0]) return fail(v, GVDB2_ERR_STATE, "channel 0 missing");
    if (!v->pnode.p || v->pnode_n < n) return fail(v, GVDB2_ERR_STATE, "InsertPoints must precede ScatterDensity");
    if (n > 0 && (!v->pos.base || n > v->pos.count)) return fail(v, GVDB2_ERR_ARG, "bad point count");
    if (n == 0) return GVDB2_OK;
    k_scatter_ref<<<grid_for(n, 256, 1ll << 31), 256, 0, v->stream>>>(
        v->pos, n, radius, make_float3(trans[0], trans[1], trans[2]), expand, v->pnode.as<int32_t>(), v->pool_cnt[0],
        v->pool_ptr(0), v->res(0), atlas_geom(v), v->atlas[0].as<float>());
    GV_CUDA(v, cudaGetLastError());
    return GVDB2_OK;
}

gvdb2_status gather_voxels(Volume *v, int sc, float radius, int chan, int accum, bool levelset) {
    if (chan < 0 || chan >= kMaxChan || !v->has_chan[chan]) return fail(v, GVDB2_ERR_ARG, "bad channel");
    if (v->num_sc == 0 || sc != v->sc_size) return fail(v, GVDB2_ERR_STATE, "InsertPointsSubcell must precede the gather");
    int sc3 = sc * sc * sc;
    int threads = v->sc_per_brick * sc3;
    if (threads > 1024) return fail(v, GVDB2_ERR_UNSUPPORTED, "brick has more than 1024 voxels");
    int64_t blocks = (v->num_sc + v->sc_per_brick - 1) / v->sc_per_brick;
    if (blocks == 0) return GVDB2_OK;
    const float *pnt = v->sc_len > 0 ? v->sc_pnt.as<float>() : nullptr;
    if (sc == 4) {
        const unsigned g = (unsigned)((v->num_sc + kGvWarps - 1) / kGvWarps);
        if (levelset)
            k_gather_voxels_sc4<true><<<g, 32 * kGvWarps, 0, v->stream>>>(
                v->num_sc, radius, v->sc_nid.as<int32_t>(), v->sc_cnt.as<uint32_t>(), v->sc_off.as<uint32_t>(),
                v->sc_pos.as<int32_t>(), pnt, v->pool_ptr(0), atlas_geom(v), v->atlas[chan].as<float>(), accum);
        else
            k_gather_voxels_sc4<false><<<g, 32 * kGvWarps, 0, v->stream>>>(
                v->num_sc, radius, v->sc_nid.as<int32_t>(), v->sc_cnt.as<uint32_t>(), v->sc_off.as<uint32_t>(),
                v->sc_pos.as<int32_t>(), pnt, v->pool_ptr(0), atlas_geom(v), v->atlas[chan].as<float>(), accum);
        GV_CUDA(v, cudaGetLastError());
        return GVDB2_OK;
    }
    if (levelset)
        k_gather_voxels<true><<<(unsigned)blocks, threads, 0, v->stream>>>(
            v->num_sc, v->sc_per_brick, sc, radius, v->sc_nid.as<int32_t>(), v->sc_cnt.as<uint32_t>(),
            v->sc_off.as<uint32_t>(), v->sc_pos.as<int32_t>(), pnt, v->pool_ptr(0), v->apron, atlas_geom(v),
            v->atlas[chan].as<float>(), accum);
    else
        k_gather_voxels<false><<<(unsigned)blocks, threads, 0, v->stream>>>(
            v->num_sc, v->sc_per_brick, sc, radius, v->sc_nid.as<int32_t>(), v->sc_cnt.as<uint32_t>(),
            v->sc_off.as<uint32_t>(), v->sc_pos.as<int32_t>(), pnt, v->pool_ptr(0), v->apron, atlas_geom(v),
            v->atlas[chan].as<float>(), accum);
    GV_CUDA(v, cudaGetLastError());
    return GVDB2_OK;
}

gvdb2_status scatter_kernel(Volume *v, int kernel, int n, const float trans[3], gvdb2_points_view weight,
                            float weight_const, const gvdb2_points_view *attrs, const int *chans, int nch) {
    GV_TRY(check_chans(v, chans, nch));
    GV_TRY(splat_prologue(v, kernel, n, trans));
    SplatArgs S;
    S.pos = v->pos;
    S.trans = make_float3(trans[0], trans[1], trans[2]);
    S.weight = to_view(weight);
    S.has_weight = weight.base != nullptr;
    S.wconst = weight_const;
    set_attrs(S.attr_mask, S.attr, attrs, nch);
    S.nch = nch;
    for (int c = 0; c < kMaxSplatChan; c++) S.chan[c] = c < nch ? v->atlas[chans[c]].as<float>() : nullptr;
    fill_topology(v, S);
    S.log2r0 = v->logdim[0];
    return run_scatter(v, kernel, S);
}

gvdb2_status gather_kernel(Volume *v, int kernel, int n, const float trans[3], const int *chans, int nch, float *out,
                           int64_t out_stride) {
    GV_TRY(check_chans(v, chans, nch));
    if (!out || out_stride < nch) return fail(v, GVDB2_ERR_ARG, "bad output buffer");
    GV_TRY(splat_prologue(v, kernel, n, trans));
    if (n == 0) return GVDB2_OK;
    k_zero_unbinned<<<grid_for(n, 256, 1ll << 31), 256, 0, v->stream>>>(v->pbin.as<int32_t>(), n, out, out_stride, nch);
    GatherArgs G{};
    G.pos = v->pos;
    G.trans = make_float3(trans[0], trans[1], trans[2]);
    for (int c = 0; c < kMaxSplatChan; c++) G.chan[c] = c < nch ? v->atlas[chans[c]].as<float>() : nullptr;
    G.nch = nch;
    G.out = out;
    G.out_stride = out_stride;
    fill_topology(v, G);
    return run_gather<kFwd>(v, kernel, G);
}

gvdb2_status gather_kernel_prebinned(Volume *v, int kernel, int n, const float trans[3], const int *chans, int nch,
                                     float *out, int64_t out_stride, const uint32_t *bin_off27, const int32_t *perm) {
    GV_TRY(check_chans(v, chans, nch));
    if (!out || out_stride < nch) return fail(v, GVDB2_ERR_ARG, "bad output buffer");
    if (kernel != GVDB2_KERNEL_TENT1 && kernel != GVDB2_KERNEL_CUBIC2) return fail(v, GVDB2_ERR_ARG, "unknown kernel");
    if (!v->atlas_valid) return fail(v, GVDB2_ERR_STATE, "UpdateAtlas must follow the topology rebuild");
    if (n == 0) return GVDB2_OK;
    GatherArgs G{};
    G.pos = v->pos;
    G.trans = make_float3(trans[0], trans[1], trans[2]);
    for (int c = 0; c < kMaxSplatChan; c++) G.chan[c] = c < nch ? v->atlas[chans[c]].as<float>() : nullptr;
    G.nch = nch;
    G.out = out;
    G.out_stride = out_stride;
    fill_topology(v, G);
    G.bin_off = bin_off27;
    G.perm = perm;
    return run_gather<kFwd>(v, kernel, G);
}

gvdb2_status scatter_kernel_backward(Volume *v, int kernel, int n, const float trans[3], gvdb2_points_view weight,
                                     float weight_const, const gvdb2_points_view *attrs, int nch,
                                     const int *grad_chans, float *grad_pos, float *grad_weight, float *grad_attr) {
    GV_TRY(check_chans(v, grad_chans, nch));
    GV_TRY(splat_prologue(v, kernel, n, trans));
    if (n == 0) return GVDB2_OK;
    int g = grid_for(n, 256, 1ll << 31);
    k_zero_unbinned<<<g, 256, 0, v->stream>>>(v->pbin.as<int32_t>(), n, grad_pos, 3, 3);
    k_zero_unbinned<<<g, 256, 0, v->stream>>>(v->pbin.as<int32_t>(), n, grad_weight, 1, 1);
    k_zero_unbinned<<<g, 256, 0, v->stream>>>(v->pbin.as<int32_t>(), n, grad_attr, nch, nch);
    GatherArgs G{};
    G.pos = v->pos;
    G.trans = make_float3(trans[0], trans[1], trans[2]);
    for (int c = 0; c < kMaxSplatChan; c++) G.chan[c] = c < nch ? v->atlas[grad_chans[c]].as<float>() : nullptr;
    G.nch = nch;
    G.weight = to_view(weight);
    G.has_weight = weight.base != nullptr;
    G.wconst = weight_const;
    set_attrs(G.attr_mask, G.attr, attrs, nch);
    G.grad_pos = grad_pos;
    G.grad_weight = grad_weight;
    G.grad_attr = grad_attr;
    fill_topology(v, G);
    return run_gather<kScatterBwd>(v, kernel, G);
}

gvdb2_status gather_kernel_backward(Volume *v, int kernel, int n, const float trans[3], const int *chans, int nch,
                                    const float *grad_out, const int *grad_chans, float *grad_pos) {
    GV_TRY(check_chans(v, chans, nch));
    if (grad_chans) GV_TRY(check_chans(v, grad_chans, nch));
    if (!grad_out) return fail(v, GVDB2_ERR_ARG, "grad_out is required");
    GV_TRY(splat_prologue(v, kernel, n, trans));
    if (grad_chans) { // dL/dG = scatter of dL/dout with unit weight
        SplatArgs S;
        S.pos = v->pos;
        S.trans = make_float3(trans[0], trans[1], trans[2]);
        S.weight = PointsView{};
        S.has_weight = 0;
        S.wconst = 1.0f;
        S.attr_mask = 0;
        for (int c = 0; c < kMaxSplatChan; c++) {
            S.attr[c] = PointsView{};
            if (c < nch) {
                S.attr[c].base = reinterpret_cast<const char *>(grad_out + c);
                S.attr[c].count = n;
                S.attr[c].stride = (int32_t)(sizeof(float) * nch);
                S.attr[c].offset = 0;
                S.attr_mask |= 1u << c;
            }
            S.chan[c] = c < nch ? v->atlas[grad_chans[c]].as<float>() : nullptr;
        }
        S.nch = nch;
        fill_topology(v, S);
        S.log2r0 = v->logdim[0];
        GV_TRY(run_scatter(v, kernel, S));
    }
    if (!grad_pos || n == 0) return GVDB2_OK;
    k_zero_unbinned<<<grid_for(n, 256, 1ll << 31), 256, 0, v->stream>>>(v->pbin.as<int32_t>(), n, grad_pos, 3, 3);
    GatherArgs G{};
    G.pos = v->pos;
    G.trans = make_float3(trans[0], trans[1], trans[2]);
    for (int c = 0; c < kMaxSplatChan; c++) G.chan[c] = c < nch ? v->atlas[chans[c]].as<float>() : nullptr;
    G.nch = nch;
    G.grad_out = grad_out;
    G.grad_pos = grad_pos;
    fill_topology(v, G);
    return run_gather<kGatherBwd>(v, kernel, G);
}

} // namespace gvdb2
