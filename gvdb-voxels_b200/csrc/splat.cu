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

// The entries of the subcell lists: float xyz (InsertPointsSubcell), or
// 16-bit xyz over the rebuild's bounding box (InsertPointsSubcell_FP16),
// read back as q / 65535 * range + min (gvdbGatherLevelSet_fp16, P:792-794).
struct ScList {
    const float *pnt;
    const uint16_t *q;
    float3 qmin, qrange;
};
template <bool FP16>
__device__ __forceinline__ float3 sc_entry(const ScList &L, int64_t e) {
    if (FP16) {
        const uint16_t *q = L.q + 3 * e;
        return make_float3(fmaf(__fdividef((float)q[0], 65535.0f), L.qrange.x, L.qmin.x),
                           fmaf(__fdividef((float)q[1], 65535.0f), L.qrange.y, L.qmin.y),
                           fmaf(__fdividef((float)q[2], 65535.0f), L.qrange.z, L.qmin.z));
    }
    const float *p = L.pnt + 3 * e;
    return make_float3(p[0], p[1], p[2]);
}

// gvdbGatherDensity / gvdbGatherLevelSet (and gvdbGatherLevelSet_fp16): one
// CTA per mapped leaf, one thread per voxel of its subcells.
template <bool LEVELSET, bool FP16>
__global__ void k_gather_voxels(int64_t num_sc, int scpb, int sc, float radius, const int32_t *sc_nid,
                                const uint32_t *sc_cnt, const uint32_t *sc_off, const int32_t *sc_pos, ScList pl,
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
        const float3 p = sc_entry<FP16>(pl, (int64_t)(beg + j));
        float dx = p.x - fx, dy = p.y - fy, dz = p.z - fz;
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
template <bool LEVELSET, bool FP16>
__global__ void __launch_bounds__(32 * kGvWarps) k_gather_voxels_sc4(int64_t num_sc, float radius,
                                                                     const int32_t *sc_nid, const uint32_t *sc_cnt,
                                                                     const uint32_t *sc_off, const int32_t *sc_pos,
                                                                     ScList pl, const Node *leaves, AtlasGeom A,
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
            const float3 q = sc_entry<FP16>(pl, (int64_t)(beg + base + k));
            wb[k] = make_float4(q.x, q.y, q.z, 0.0f);
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
    const uint32_t *reg_off; // per (cell, region) bin its first entry of perm (k_bin_count)
    const int32_t *perm;
    const float4 *bin_pos;   // per entry of perm: translated position, cloud index bits
    float4 *bin_amt;         // per entry of perm: the channel amounts of this call
    int res0, apron, tile;
    int m, m3; // cells per brick edge, per brick
    // huge and heavy cells (order of cell_at), light cells; cell_list ==
    // nullptr: every cell, in cell order
    const int32_t *cell_list, *cell_light, *cell_giant;
    const uint32_t *cell_cnt;
    int64_t ncell;
    int64_t tvox;
};


// ---- owner-computes scatter --------------------------------------------
//
// One warp per cell (an 8^3 block of a brick; the brick itself for 8^3
// bricks) computes the cell's interior voxels from every point whose stencil
// reaches them and writes each voxel once: no atomics, no partial sums in
// memory, no zero-fill pass.  Its sources are the cell's own points and,
// from each of the 26 neighbour cells, the regions of that cell's bin whose
// stencils cross the shared face, edge or corner (k_bin_count bins points by
// cell and region), so every source is a point the cell needs.
//
// The warp turns its sources into records in shared memory, a chunk of at
// most kScCap at a time: per point the x weights on the cell's 8 voxel
// columns and the y weights on its 8 rows (zero where the stencil does not
// reach), the z weights of its N taps and the channel amounts.  A stable
// counting sort orders the chunk by (first z tap, x group); the x group says
// which halves of the cell's x range the stencil reaches (lower only, both,
// upper only).  Lane (y, q, h) owns the voxels x in [4q, 4q+4), row y, z in
// [4h, 4h+4) of every channel in registers.  The 8 lanes of one (q, h) walk
// the same records together -- for each first z tap one contiguous run of
// the sorted chunk, its two x groups that reach half q -- so each record is
// read once per group (a shared-memory broadcast) and the group's loop has
// no divergence; a record adds to the 4 of the group's 8 rows that its
// stencil covers (the other lanes add its zero y weight).  The loop over
// first z taps is unrolled relative to 4h, so every add goes to an
// accumulator plane fixed at compile time: paired register FMAs.
//
// The adds happen in the order of the sources (the bins) and of the stable
// sort, so with deterministic binning the result is bit-reproducible.
#ifndef GVDB2_SC_CAP
#define GVDB2_SC_CAP 128
#endif
#ifndef GVDB2_SC_MIN_BLOCKS
#define GVDB2_SC_MIN_BLOCKS 4
#endif
constexpr int kScWarps = 4;                    // cells per CTA
constexpr int kScCap = GVDB2_SC_CAP;           // records per chunk
constexpr int kScBins = 11 * 3;                // (first z tap + 3, x group)

struct ScChunk {
    // x weights on the cell's voxel columns 0..7: half q (columns 4q..4q+3)
    // of record r sits at xw[r][q ^ (r & 1)], so that the lanes of one
    // quarter-warp reading the same half of different records spread over
    // all eight 16-byte bank groups
    float4 xw[kScCap][2];
    float wy[kScCap][8];  // y weights on the cell's rows 0..7
    float4 wz[kScCap];    // z weights of the taps (zero past N)
    float4 am[kScCap];    // channel amounts (zero past NCH)
    uint16_t key[kScCap];
    uint16_t rank[kScCap];
    uint16_t order[kScCap];
    uint16_t off[kScBins + 1];
    uint2 run[64]; // the cell's sources: runs [x, y) of perm (at most 1 + 2 + 6 + 18 + 4 + 12 + 12 + 8 = 63)
    uint32_t run_first[64]; // sources before run k (the runs read as one sequence)
};

// Sort the chunk's `fill` records by key (stable) into C.order.
__device__ __forceinline__ void sc_sort_chunk(ScChunk &C, int fill, int lane) {
    for (int i = lane; i <= kScBins; i += 32) C.off[i] = 0;
    __syncwarp();
    for (int base = 0; base < fill; base += 32) { // in record order: stable ranks
        const int i = base + lane;
        const bool ok = i < fill;
        const unsigned act = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            const uint32_t k = C.key[i];
            const unsigned peers = __match_any_sync(act, k);
            const uint32_t before = C.off[k];
            C.rank[i] = (uint16_t)(before + __popc(peers & lanemask_lt()));
            __syncwarp(act);
            if (lane == __ffs(peers) - 1) C.off[k] = (uint16_t)(before + __popc(peers));
        }
        __syncwarp();
    }
    // exclusive scan of the counts in place; off[kScBins] becomes fill
    constexpr int per = (kScBins + 1 + 31) / 32;
    uint32_t local[per], sum = 0;
#pragma unroll
    for (int t = 0; t < per; t++) {
        const int i = lane * per + t;
        local[t] = i <= kScBins ? C.off[i] : 0u;
        sum += local[t];
    }
    uint32_t inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    uint32_t run = inc - sum;
    __syncwarp();
#pragma unroll
    for (int t = 0; t < per; t++) {
        const int i = lane * per + t;
        if (i <= kScBins) C.off[i] = (uint16_t)run;
        run += local[t];
    }
    __syncwarp();
    for (int i = lane; i < fill; i += 32) C.order[C.off[C.key[i]] + C.rank[i]] = (uint16_t)i;
    __syncwarp();
}

#ifndef GVDB2_SC_PIPE
#define GVDB2_SC_PIPE 0
#endif
#ifndef GVDB2_SC_PREFETCH
#define GVDB2_SC_PREFETCH 0
#endif
// A record's values that lane (y, q) reads.
struct ScRec {
    float4 xv; // x weights on columns 4q..4q+3
    float wy;  // y weight on row y
    float4 zv; // z weights of the taps
    float4 av; // channel amounts
};
__device__ __forceinline__ ScRec sc_load(const ScChunk &C, int r, int y, int q) {
    return ScRec{C.xw[r][q ^ (r & 1)], C.wy[r][y], C.wz[r], C.am[r]};
}
// Visits the sorted chunk's records i in [lo, hi) in order; with
// GVDB2_SC_PIPE the next record's values are read while the current one is
// added.
template <class Visit>
__device__ __forceinline__ void sc_walk(const ScChunk &C, int lo, int hi, int y, int q, const Visit &visit) {
    if (GVDB2_SC_PIPE) {
        if (lo >= hi) return;
        ScRec cur = sc_load(C, C.order[lo], y, q);
        for (int i = lo; i < hi; i++) {
            ScRec nxt = cur;
            if (i + 1 < hi) nxt = sc_load(C, C.order[i + 1], y, q);
            visit(cur);
            cur = nxt;
        }
    } else {
        for (int i = lo; i < hi; i++) visit(sc_load(C, C.order[i], y, q));
    }
}

// Adds the chunk's records that reach the voxels of lane (y, q, h)'s group:
// for each first z tap, the run of x groups q and q + 1.
template <int KERNEL, int NCH>
__device__ __forceinline__ void sc_accumulate(const ScChunk &C, float2 (&acc)[4][2][NCH], int y, int q, int h) {
    constexpr int N = Taps<KERNEL>::N;
#pragma unroll
    for (int sp = -3; sp <= 3; sp++) { // first z tap relative to 4h
        if (sp + N - 1 < 0) continue;
        const int s = sp + 4 * h; // first z tap relative to the cell, in [-3, 7]
        auto visit = [&](const ScRec &d) {
            const float4 xv = d.xv;
            const float wyv = d.wy;
            const float4 zv = d.zv;
            const float4 av = d.av;
            const float zk[4] = {zv.x, zv.y, zv.z, zv.w};
            const float ak[4] = {av.x, av.y, av.z, av.w};
            const float2 x01 = make_float2(xv.x, xv.y), x23 = make_float2(xv.z, xv.w);
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                const float ay = ak[c] * wyv;
#pragma unroll
                for (int k = 0; k < N; k++) {
                    const int zz = sp + k;
                    if (zz < 0 || zz >= 4) continue;
                    const float t = ay * zk[k];
                    const float2 tt = make_float2(t, t);
                    acc[zz][0][c] = __ffma2_rn(tt, x01, acc[zz][0][c]);
                    acc[zz][1][c] = __ffma2_rn(tt, x23, acc[zz][1][c]);
                }
            }
        };
        const int kb = (s + 3) * 3 + q; // x groups q and q + 1 reach half q
        const int hi = C.off[kb + 2];
        sc_walk(C, C.off[kb], hi, y, q, visit);
    }
}

// The same adds with the accumulators paired along channels ({c, c+1} of
// one voxel in a float2) instead of along x: a record's amounts times its
// y and z weights form the channel pairs directly, and each x weight is used
// as the other factor of every pair (NCH > 1; an odd last channel is paired
// with a zero amount).
template <int KERNEL, int NP>
__device__ __forceinline__ void sc_accumulate_cp(const ScChunk &C, float2 (&acc)[4][4][NP], int y, int q, int h) {
    constexpr int N = Taps<KERNEL>::N;
#pragma unroll
    for (int sp = -3; sp <= 3; sp++) { // first z tap relative to 4h
        if (sp + N - 1 < 0) continue;
        const int s = sp + 4 * h; // first z tap relative to the cell, in [-3, 7]
        auto visit = [&](const ScRec &d) {
            const float4 xv = d.xv;
            const float wyv = d.wy;
            const float4 zv = d.zv;
            const float4 av = d.av;
            const float zk[4] = {zv.x, zv.y, zv.z, zv.w};
            const float2 ap[2] = {make_float2(av.x, av.y), make_float2(av.z, av.w)};
            const float xs[4] = {xv.x, xv.y, xv.z, xv.w};
            float2 ay[NP];
#pragma unroll
            for (int cp = 0; cp < NP; cp++) ay[cp] = __fmul2_rn(ap[cp], make_float2(wyv, wyv));
#pragma unroll
            for (int k = 0; k < N; k++) {
                const int zz = sp + k;
                if (zz < 0 || zz >= 4) continue;
#pragma unroll
                for (int cp = 0; cp < NP; cp++) {
                    const float2 t = __fmul2_rn(ay[cp], make_float2(zk[k], zk[k]));
#pragma unroll
                    for (int x = 0; x < 4; x++) acc[zz][x][cp] = __ffma2_rn(t, make_float2(xs[x], xs[x]), acc[zz][x][cp]);
                }
            }
        };
        const int kb = (s + 3) * 3 + q; // x groups q and q + 1 reach half q
        const int hi = C.off[kb + 2];
        sc_walk(C, C.off[kb], hi, y, q, visit);
    }
}

#ifndef GVDB2_SC_CHPAIR
#define GVDB2_SC_CHPAIR 1
#endif
// Channel pairs for 2 to 4 channels, x pairs for one channel.
template <int NCH> struct ScLayout { static constexpr bool kChPairs = GVDB2_SC_CHPAIR && NCH > 1; };

// Blocks [0, single_blocks) take kScWarps cells each, a warp per cell;
// the rest take one giant cell each (more than kGiantCell points of its
// own), whose sources the CTA's warps share in turn, 32 at a time; their
// accumulators are summed in a fixed order at the end.
template <int KERNEL, int NCH>
__global__ void __launch_bounds__(32 * kScWarps, GVDB2_SC_MIN_BLOCKS) k_scatter_cells(SplatArgs S, int64_t single_blocks) {
    using T = Taps<KERNEL>;
    constexpr int N = T::N;
    static_assert(kScWarps == 4, "a giant cell's warps reduce one accumulator plane each");
    extern __shared__ __align__(16) unsigned char sc_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    ScChunk &C = reinterpret_cast<ScChunk *>(sc_smem)[warp];
    int64_t cell;
    int W; // warps sharing the cell
    if ((int64_t)blockIdx.x < single_blocks) {
        cell = (int64_t)blockIdx.x * kScWarps + warp;
        if (cell >= S.ncell) return;
        if (S.bin_off[cell + 1] - S.bin_off[cell] > kGiantCell) return; // a CTA of its own
        W = 1;
    } else {
        const int64_t gi = (int64_t)blockIdx.x - single_blocks;
        if (gi >= (int64_t)S.cell_cnt[3]) return; // every warp of the CTA
        cell = S.cell_giant[gi];
        W = kScWarps;
    }
    const int wturn = W == 1 ? 0 : warp;
    int64_t slot;
    int cx, cy, cz;
    cell_coords(cell, S.m, S.m3, slot, cx, cy, cz);
    const Node &nd = S.leaves[S.slot_leaf[slot]];
    const int ox = nd.mPos[0] + kCell * cx, oy = nd.mPos[1] + kCell * cy, oz = nd.mPos[2] + kCell * cz;
    // The sources, as runs of perm in a fixed order: lane d < 27 lists those of
    // the neighbour cell in direction d = (dz+1)*9 + (dy+1)*3 + (dx+1): its
    // regions whose stencils reach this cell -- per axis, across the lower
    // face its upper band (2), across the upper face its lower band (0),
    // along the axis all three -- merged into as few runs as the region
    // order allows.
    int nrun = 0;
    uint2 runs[9];
    if (lane < 27) {
        const int dx = lane % 3 - 1, dy = lane / 3 % 3 - 1, dz = lane / 9 - 1;
        const int ncx = cx + dx, ncy = cy + dy, ncz = cz + dz;
        const int bx = ncx < 0 ? -1 : (ncx >= S.m ? 1 : 0), by = ncy < 0 ? -1 : (ncy >= S.m ? 1 : 0),
                  bz = ncz < 0 ? -1 : (ncz >= S.m ? 1 : 0);
        const int32_t ns = (bx | by | bz) == 0 ? (int32_t)slot
                                               : S.nbr27[slot * 27 + (bz + 1) * 9 + (by + 1) * 3 + (bx + 1)];
        if (ns >= 0) {
            const int64_t nc =
                (int64_t)ns * S.m3 + ((ncz - bz * S.m) * S.m + (ncy - by * S.m)) * S.m + (ncx - bx * S.m);
            const uint32_t *ro = S.reg_off + nc * kRegions;
            const int rx0 = dx < 0 ? 2 : 0, ry0 = dy < 0 ? 2 : 0, ry1 = dy > 0 ? 0 : 2;
            const int rz0 = dz < 0 ? 2 : 0, rz1 = dz > 0 ? 0 : 2;
            auto add = [&](int r0, int r1) { // regions [r0, r1)
                const uint2 u = make_uint2(ro[r0], ro[r1]);
                if (u.y > u.x) runs[nrun++] = u;
            };
            if (dx == 0 && dy == 0) {
                if (dz == 0) add(0, kRegions);
                else add(rz0 * 9, rz0 * 9 + 9);
            } else if (dx == 0) {
                for (int rz = rz0; rz <= rz1; rz++) add((rz * 3 + ry0) * 3, (rz * 3 + ry0) * 3 + 3);
            } else {
                for (int rz = rz0; rz <= rz1; rz++)
                    for (int ry = ry0; ry <= ry1; ry++) add((rz * 3 + ry) * 3 + rx0, (rz * 3 + ry) * 3 + rx0 + 1);
            }
        }
    }
    // the lanes' runs one after the other, each with the number of sources
    // before it, so that the warp reads them as one sequence, 32 at a time
    uint32_t len = 0;
#pragma unroll
    for (int k = 0; k < 9; k++)
        if (k < nrun) len += runs[k].y - runs[k].x;
    int first = nrun;
    uint32_t before = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) { // inclusive prefixes over the lanes
        const int t = __shfl_up_sync(0xffffffffu, first, o);
        const uint32_t u = __shfl_up_sync(0xffffffffu, before, o);
        if (lane >= o) first += t, before += u;
    }
    const int total_runs = __shfl_sync(0xffffffffu, first, 31);
    const uint32_t total_src = __shfl_sync(0xffffffffu, before, 31);
    first -= nrun;
    before -= len;
#pragma unroll
    for (int k = 0; k < 9; k++)
        if (k < nrun) {
            C.run[first + k] = runs[k];
            C.run_first[first + k] = before;
            before += runs[k].y - runs[k].x;
        }
    __syncwarp();

    const int y = lane & 7, q = (lane >> 3) & 1, h = lane >> 4;
    constexpr bool kCp = ScLayout<NCH>::kChPairs;
    constexpr int NP = (NCH + 1) / 2;
    float2 acc[4][2][NCH];   // x pairs
    float2 accp[4][4][NP];   // channel pairs
#pragma unroll
    for (int z = 0; z < 4; z++) {
#pragma unroll
        for (int x = 0; x < 2; x++)
#pragma unroll
            for (int c = 0; c < NCH; c++) acc[z][x][c] = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int x = 0; x < 4; x++)
#pragma unroll
            for (int c = 0; c < NP; c++) accp[z][x][c] = make_float2(0.0f, 0.0f);
    }
    auto accumulate = [&]() {
        if constexpr (kCp) sc_accumulate_cp<KERNEL, NP>(C, accp, y, q, h);
        else sc_accumulate<KERNEL, NCH>(C, acc, y, q, h);
    };
    int fill = 0;
    // One lane's source of a step: its point, the cloud origin and the
    // channel amounts (all the global reads of a record).
    struct Src {
        bool ok;
        float3 pt;
        int3 o;
        float a4[4];
    };
    auto fetch = [&](uint32_t vb) {
        Src d;
        d.ok = false;
        d.pt = make_float3(0.f, 0.f, 0.f);
        d.o = make_int3(0, 0, 0);
#pragma unroll
        for (int c = 0; c < 4; c++) d.a4[c] = 0.0f;
        // the run holding sequence index vi (binary search of the run
        // starts) and the perm entry inside it
        const uint32_t vi = vb + lane;
        if (vi < total_src) {
            int lo = 0, hi = total_runs - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (C.run_first[mid] <= vi) lo = mid;
                else hi = mid - 1;
            }
            const uint32_t j = C.run[lo].x + (vi - C.run_first[lo]);
            const float4 q = S.bin_pos[j];
            d.pt = make_float3(q.x, q.y, q.z);
            const int32_t cloud = __float_as_int(q.w);
            if (cloud >= 0) d.o = make_int3(S.pos.origin[3 * cloud], S.pos.origin[3 * cloud + 1], S.pos.origin[3 * cloud + 2]);
            const float4 am = S.bin_amt[j];
            d.a4[0] = am.x, d.a4[1] = am.y, d.a4[2] = am.z, d.a4[3] = am.w;
            d.ok = true;
        }
        return d;
    };
    // The record of each lane's source, appended to the chunk.
    auto build = [&](const Src &d) {
        float wx[N], wyt[N], wzt[N];
        int fx = 0, fy = 0, fz = 0;
        bool ok = d.ok;
        if (ok) {
            fx = T::eval(d.pt.x, wx) + d.o.x - ox; // bin_pos holds the translated position
            fy = T::eval(d.pt.y, wyt) + d.o.y - oy;
            fz = T::eval(d.pt.z, wzt) + d.o.z - oz;
            // the stencil reaches the cell on every axis (true of every
            // source by construction of the regions)
            ok = fx > -N && fx < kCell && fy > -N && fy < kCell && fz > -N && fz < kCell;
        }
        const unsigned mask = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            const int r = fill + __popc(mask & lanemask_lt());
            float *xr = reinterpret_cast<float *>(C.xw[r]);
            float *yr = C.wy[r];
            reinterpret_cast<float4 *>(xr)[0] = reinterpret_cast<float4 *>(xr)[1] = make_float4(0.f, 0.f, 0.f, 0.f);
            reinterpret_cast<float4 *>(yr)[0] = reinterpret_cast<float4 *>(yr)[1] = make_float4(0.f, 0.f, 0.f, 0.f);
            const int sw = (r & 1) * 4; // the halves of odd records are swapped
#pragma unroll
            for (int t = 0; t < N; t++) {
                if ((unsigned)(fx + t) < (unsigned)kCell) xr[(fx + t) ^ sw] = wx[t];
                if ((unsigned)(fy + t) < (unsigned)kCell) yr[fy + t] = wyt[t];
            }
            float zz4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int t = 0; t < N; t++) zz4[t] = wzt[t];
            C.wz[r] = make_float4(zz4[0], zz4[1], zz4[2], zz4[3]);
            C.am[r] = make_float4(d.a4[0], d.a4[1], d.a4[2], d.a4[3]);
            const int xg = fx < 5 - N ? 0 : (fx <= 3 ? 1 : 2); // lower half only, both, upper only
            C.key[r] = (uint16_t)((fz + 3) * 3 + xg);
        }
        fill += __popc(mask);
    };
    auto flush_if_full = [&]() {
        if (fill > kScCap - 32) {
            sc_sort_chunk(C, fill, lane);
            accumulate();
            __syncwarp();
            fill = 0;
        }
    };
    // the steps of 32 sources this warp takes (the warps of a giant cell take turns)
    const uint32_t stride = 32u * W;
    uint32_t vb = 32u * wturn;
    if (GVDB2_SC_PREFETCH) {
        // the next step's reads are in flight while this step's records are
        // built and a full chunk is added
        Src nxt = fetch(vb);
        for (; vb < total_src; vb += stride) {
            const Src cur = nxt;
            if (vb + stride < total_src) nxt = fetch(vb + stride);
            flush_if_full();
            build(cur);
        }
    } else {
        for (; vb < total_src; vb += stride) {
            flush_if_full();
            build(fetch(vb));
        }
    }
    if (fill > 0) {
        sc_sort_chunk(C, fill, lane);
        accumulate();
    }
    if constexpr (kCp) { // to x pairs for the write-out (register renaming)
#pragma unroll
        for (int z = 0; z < 4; z++)
#pragma unroll
            for (int c = 0; c < NCH; c++)
#pragma unroll
                for (int xp = 0; xp < 2; xp++) {
                    const float2 a0 = accp[z][2 * xp][c / 2], a1 = accp[z][2 * xp + 1][c / 2];
                    acc[z][xp][c] = (c & 1) ? make_float2(a0.y, a1.y) : make_float2(a0.x, a1.x);
                }
    }
    // each lane writes its 4 x 4 voxels of every channel once
    const int a = S.apron, tl = S.tile;
    const int64_t base = slot * S.tvox + (int64_t)(kCell * cx + 4 * q + a);
    auto store = [&](int zz, int c, float2 v01, float2 v23) {
        float *dst = S.chan[c] + base + ((int64_t)(kCell * cz + 4 * h + zz + a) * tl + (kCell * cy + y + a)) * tl;
        dst[0] = v01.x;
        dst[1] = v01.y;
        dst[2] = v23.x;
        dst[3] = v23.y;
    };
    if (W == 1) {
#pragma unroll
        for (int zz = 0; zz < 4; zz++)
#pragma unroll
            for (int c = 0; c < NCH; c++) store(zz, c, acc[zz][0][c], acc[zz][1][c]);
        return;
    }
    // giant cell: the warps' accumulators through shared memory, summed in
    // warp order; warp w sums and writes accumulator plane w of every lane
    __syncthreads(); // every warp is done with its chunks
    float2 *red = reinterpret_cast<float2 *>(sc_smem);
    auto at = [&](int w, int zz, int xp, int c) { return (((w * 4 + zz) * 2 + xp) * NCH + c) * 32 + lane; };
#pragma unroll
    for (int zz = 0; zz < 4; zz++)
#pragma unroll
        for (int xp = 0; xp < 2; xp++)
#pragma unroll
            for (int c = 0; c < NCH; c++) red[at(warp, zz, xp, c)] = acc[zz][xp][c];
    __syncthreads();
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        float2 v[2];
#pragma unroll
        for (int xp = 0; xp < 2; xp++) {
            v[xp] = red[at(0, warp, xp, c)];
#pragma unroll
            for (int w = 1; w < kScWarps; w++) {
                const float2 u = red[at(w, warp, xp, c)];
                v[xp].x += u.x;
                v[xp].y += u.y;
            }
        }
        store(warp, c, v[0], v[1]);
    }
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
    int m, m3; // cells per brick edge, per brick
    // huge and heavy cells (order of cell_at), light cells; cell_list ==
    // nullptr: every cell, in cell order
    const int32_t *cell_list, *cell_light;
    const uint32_t *cell_cnt;
    int64_t ncell;
    int64_t tvox;
    const float4 *bin_pos; // per entry of perm: translated position, cloud bits (nullptr: read via perm)
};

// The translated position and cloud origin of point pidx, entry j of the
// bin order: from the bin-ordered copy when there is one (contiguous reads
// for a cell's points), else from the caller's view.
__device__ __forceinline__ void gather_point_at(const GatherArgs &G, int32_t pidx, int64_t j, float3 &w, int3 &o) {
    if (G.bin_pos) {
        const float4 q = G.bin_pos[j];
        w = make_float3(q.x, q.y, q.z);
        const int32_t cloud = __float_as_int(q.w);
        o = cloud >= 0 ? make_int3(G.pos.origin[3 * cloud], G.pos.origin[3 * cloud + 1], G.pos.origin[3 * cloud + 2])
                       : make_int3(0, 0, 0);
    } else {
        const float3 p = load_f3(G.pos, pidx);
        w = make_float3(p.x + G.trans.x, p.y + G.trans.y, p.z + G.trans.z);
        o = point_origin(G.pos, pidx);
    }
}

// One point of a gather, in any mode.  fetch(x, y, z, g) gives g[c], the
// value of channel c at tap (x, y, z) of the cell's extended frame, whose
// origin (ox, oy, oz) is the cell's first voxel minus H.
template <int KERNEL, int MODE, int NCH, class Fetch>
__device__ __forceinline__ void gather_point(const GatherArgs &G, int32_t pidx, int64_t j, int ox, int oy, int oz,
                                             const Fetch &fetch) {
    using T = Taps<KERNEL>;
    constexpr int N = T::N;
    float3 p;
    int3 o;
    gather_point_at(G, pidx, j, p, o);
    float wx[N], wy[N], wz[N], dx[N], dy[N], dz[N];
    int fx, fy, fz;
    if (MODE == kFwd) {
        fx = T::eval(p.x, wx) + o.x - ox;
        fy = T::eval(p.y, wy) + o.y - oy;
        fz = T::eval(p.z, wz) + o.z - oz;
    } else {
        fx = T::eval_d(p.x, wx, dx) + o.x - ox;
        fy = T::eval_d(p.y, wy, dy) + o.y - oy;
        fz = T::eval_d(p.z, wz, dz) + o.z - oz;
    }
    // a binned point's first taps lie in [0, 8]; a point moved since the
    // binning (positions changed in place) gathers 0 and reads nothing outside
    if (!((unsigned)fx <= 8u && (unsigned)fy <= 8u && (unsigned)fz <= 8u)) {
        fx = fy = fz = 0;
#pragma unroll
        for (int k = 0; k < N; k++) wx[k] = wy[k] = wz[k] = dx[k] = dy[k] = dz[k] = 0.0f;
    }
    float sum[NCH], gx[NCH], gy[NCH], gz[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) sum[c] = gx[c] = gy[c] = gz[c] = 0.0f;
#pragma unroll
    for (int tz = 0; tz < N; tz++) {
#pragma unroll
        for (int ty = 0; ty < N; ty++) {
            const float wyz = wy[ty] * wz[tz];
            float dyz = 0.0f, ydz = 0.0f;
            if (MODE != kFwd) {
                dyz = dy[ty] * wz[tz];
                ydz = wy[ty] * dz[tz];
            }
#pragma unroll
            for (int tx = 0; tx < N; tx++) {
                float gv[NCH];
                fetch(fx + tx, fy + ty, fz + tz, gv);
#pragma unroll
                for (int c = 0; c < NCH; c++) {
                    const float g = gv[c];
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

constexpr int kGatherThreads = 256; // threads of a k_gather_tile CTA
constexpr int kGatherChunk = 1024;  // points ordered per pass

// A voxel's channels side by side in the staged tile: one shared-memory
// load per tap serves every channel.
template <int NCH> struct GVec { using T = float4; };
template <> struct GVec<1> { using T = float; };
template <> struct GVec<2> { using T = float2; };
template <int NCH>
__device__ __forceinline__ void gvec_put(typename GVec<NCH>::T &v, const float (&g)[NCH]) {
    if constexpr (NCH == 1) v = g[0];
    else if constexpr (NCH == 2) v = make_float2(g[0], g[1]);
    else if constexpr (NCH == 3) v = make_float4(g[0], g[1], g[2], 0.0f);
    else v = make_float4(g[0], g[1], g[2], g[3]);
}
template <int NCH>
__device__ __forceinline__ void gvec_get(const typename GVec<NCH>::T &v, float *g) {
    if constexpr (NCH == 1) g[0] = v;
    else if constexpr (NCH == 2) g[0] = v.x, g[1] = v.y;
    else {
        g[0] = v.x, g[1] = v.y, g[2] = v.z;
        if constexpr (NCH == 4) g[3] = v.w;
    }
}

template <int KERNEL, int NCH>
constexpr size_t gather_tile_smem() {
    constexpr int ht = kCell + Taps<KERNEL>::N;
    return sizeof(typename GVec<NCH>::T) * ht * ht * ht + sizeof(uint16_t) * 3 * kGatherChunk +
           sizeof(uint32_t) * 1024;
}

// One CTA per huge or heavy cell (every cell when the binning came from the
// caller): stages the cell plus a halo of N/2 voxels (12^3 for the cubic
// B-spline) from the interiors of its brick and the neighbours, the
// channels of a voxel side by side, then serves the cell's points from
// shared memory.  The points are visited in the order of their first tap
// (a counting sort in shared memory, kGatherChunk at a time), so the lanes
// of a warp read neighbouring voxels: few bank conflicts, and lanes on the
// same voxel share one load.
template <int KERNEL, int MODE, int NCH>
__device__ __forceinline__ void gather_tile_cell(const GatherArgs &G, int64_t block) {
    constexpr int N = Taps<KERNEL>::N, H = N / 2;
    constexpr int ht = kCell + 2 * H, ht3 = ht * ht * ht;
    constexpr int nkeys = (kCell + 1) * (kCell + 1) * (kCell + 1); // first taps in [0, 8]^3 of the frame
    using V = typename GVec<NCH>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tile = reinterpret_cast<V *>(smem_raw);
    uint16_t *key = reinterpret_cast<uint16_t *>(tile + ht3);
    uint16_t *rank = key + kGatherChunk;
    uint16_t *order = rank + kGatherChunk;
    uint32_t *hist = reinterpret_cast<uint32_t *>(order + kGatherChunk); // nkeys + 1 (+ scan scratch)
    __shared__ int32_t nbs[27];
    __shared__ uint32_t wsum[kGatherThreads / 32];
    const int res = G.res0;
    const int64_t cell = G.cell_list ? cell_at(block, G.cell_list, G.cell_cnt, G.ncell) : block;
    if (cell < 0) return;
    const uint32_t beg = G.bin_off[cell], end = G.bin_off[cell + 1];
    if (beg == end) return; // no points: nothing to stage
    int64_t slot;
    int cx, cy, cz;
    cell_coords(cell, G.m, G.m3, slot, cx, cy, cz);
    const int a = G.apron, tl = G.tile;
    if (threadIdx.x < 27) nbs[threadIdx.x] = G.nbr27[slot * 27 + threadIdx.x];
    __syncthreads();
    // halo tile from the interiors of this brick and its neighbours; all of a
    // thread's loads are issued before its stores
    constexpr int per = (ht3 + kGatherThreads - 1) / kGatherThreads;
    float val[per][NCH];
#pragma unroll
    for (int k = 0; k < per; k++) {
        const int t = (int)threadIdx.x + k * kGatherThreads;
        const int tx = t % ht, ty = t / ht % ht, tz = t / (ht * ht);
        const int lx = kCell * cx + tx - H, ly = kCell * cy + ty - H, lz = kCell * cz + tz - H;
        const int dx = lx < 0 ? -1 : (lx >= res ? 1 : 0), dy = ly < 0 ? -1 : (ly >= res ? 1 : 0),
                  dz = lz < 0 ? -1 : (lz >= res ? 1 : 0);
        const int32_t nb = t < ht3 ? nbs[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)] : -1;
        const int64_t off = (int64_t)nb * G.tvox +
                            ((int64_t)(lz - dz * res + a) * tl + (ly - dy * res + a)) * tl + (lx - dx * res + a);
#pragma unroll
        for (int c = 0; c < NCH; c++) val[k][c] = nb >= 0 ? __ldg(G.chan[c] + off) : 0.0f;
    }
#pragma unroll
    for (int k = 0; k < per; k++) {
        const int t = (int)threadIdx.x + k * kGatherThreads;
        if (t < ht3) gvec_put<NCH>(tile[t], val[k]);
    }
    const Node &nd = G.leaves[G.slot_leaf[slot]];
    const int ox = nd.mPos[0] + kCell * cx - H, oy = nd.mPos[1] + kCell * cy - H, oz = nd.mPos[2] + kCell * cz - H;
    auto fetch = [&](int x, int y, int z, float g[NCH]) { gvec_get<NCH>(tile[(z * ht + y) * ht + x], g); };
    for (uint32_t cb = beg; cb < end; cb += kGatherChunk) {
        const int cnt = (int)min((uint32_t)kGatherChunk, end - cb);
        for (int i = threadIdx.x; i <= nkeys; i += kGatherThreads) hist[i] = 0;
        __syncthreads(); // (also: the tile is staged)
        // key = the point's first tap in the frame (clamped; a point moved
        // since the binning gathers zero whatever its key)
        for (int j = threadIdx.x; j < cnt; j += kGatherThreads) {
            float3 q;
            int3 o;
            gather_point_at(G, G.bin_pos ? 0 : G.perm[cb + j], (int64_t)cb + j, q, o);
            const int fx = (int)floorf(q.x - 0.5f) - Taps<KERNEL>::LO + o.x - ox;
            const int fy = (int)floorf(q.y - 0.5f) - Taps<KERNEL>::LO + o.y - oy;
            const int fz = (int)floorf(q.z - 0.5f) - Taps<KERNEL>::LO + o.z - oz;
            const int kx = min(max(fx, 0), kCell), ky = min(max(fy, 0), kCell), kz = min(max(fz, 0), kCell);
            const int k = (kz * (kCell + 1) + ky) * (kCell + 1) + kx;
            key[j] = (uint16_t)k;
            rank[j] = (uint16_t)atomicAdd(&hist[k], 1u);
        }
        __syncthreads();
        { // exclusive scan of hist[0 .. nkeys) in place
            constexpr int hp = (nkeys + kGatherThreads - 1) / kGatherThreads;
            uint32_t loc[hp], sum = 0;
#pragma unroll
            for (int t = 0; t < hp; t++) {
                const int i = (int)threadIdx.x * hp + t;
                loc[t] = i < nkeys ? hist[i] : 0u;
                sum += loc[t];
            }
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            uint32_t inc = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            if (lane == 31) wsum[warp] = inc;
            __syncthreads();
            uint32_t run = inc - sum;
            for (int w = 0; w < warp; w++) run += wsum[w];
#pragma unroll
            for (int t = 0; t < hp; t++) {
                const int i = (int)threadIdx.x * hp + t;
                if (i < nkeys) hist[i] = run;
                run += loc[t];
            }
        }
        __syncthreads();
        for (int j = threadIdx.x; j < cnt; j += kGatherThreads) order[hist[key[j]] + rank[j]] = (uint16_t)j;
        __syncthreads();
        for (int j = threadIdx.x; j < cnt; j += kGatherThreads)
            gather_point<KERNEL, MODE, NCH>(G, G.perm[cb + order[j]], (int64_t)cb + order[j], ox, oy, oz, fetch);
        __syncthreads(); // the order arrays are reused by the next chunk
    }
}

// The points of light cells: one warp per cell, one lane per point (a light
// cell holds at most kLightCell = 32), taps read straight from the atlas; a
// staged halo would cost 12^3 floats per channel for a few points.
template <int KERNEL, int MODE, int NCH>
__device__ __forceinline__ void gather_light_cells(const GatherArgs &G, int64_t block) {
    constexpr int H = Taps<KERNEL>::N / 2;
    const int64_t w = (block * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= (int64_t)G.cell_cnt[2]) return;
    const int64_t cell = G.cell_light[w];
    const uint32_t beg = G.bin_off[cell], cnt = G.bin_off[cell + 1] - beg;
    if ((uint32_t)lane >= cnt) return;
    int64_t slot;
    int cx, cy, cz;
    cell_coords(cell, G.m, G.m3, slot, cx, cy, cz);
    const Node &nd = G.leaves[G.slot_leaf[slot]];
    const int fx0 = kCell * cx - H, fy0 = kCell * cy - H, fz0 = kCell * cz - H; // frame origin in the brick
    const int res = G.res0, a = G.apron, tl = G.tile;
    auto fetch = [&](int x, int y, int z, float g[NCH]) {
        const int lx = fx0 + x, ly = fy0 + y, lz = fz0 + z; // brick-local, may step into a neighbour
        const int sx = lx < 0 ? -1 : (lx >= res ? 1 : 0), sy = ly < 0 ? -1 : (ly >= res ? 1 : 0),
                  sz = lz < 0 ? -1 : (lz >= res ? 1 : 0);
        const int d = (sz + 1) * 9 + (sy + 1) * 3 + (sx + 1);
        const int64_t ns = d == 13 ? slot : (int64_t)G.nbr27[slot * 27 + d];
        const int64_t off = ns * G.tvox + ((int64_t)(lz - sz * res + a) * tl + (ly - sy * res + a)) * tl +
                            (lx - sx * res + a);
#pragma unroll
        for (int c = 0; c < NCH; c++) g[c] = ns >= 0 ? __ldg(G.chan[c] + off) : 0.0f;
    };
    gather_point<KERNEL, MODE, NCH>(G, G.perm[beg + lane], (int64_t)beg + lane, nd.mPos[0] + fx0, nd.mPos[1] + fy0, nd.mPos[2] + fz0,
                                    fetch);
}

// Two launches: a halo tile per huge or heavy cell (every cell, in cell
// order, when no cell list is given), then the light cells, a warp each.
// One fused launch measured slower: the light path's registers (66) halved
// the tiles' occupancy.
template <int KERNEL, int MODE, int NCH>
__global__ void __launch_bounds__(kGatherThreads) k_gather_tile(GatherArgs G) {
    gather_tile_cell<KERNEL, MODE, NCH>(G, blockIdx.x);
}
template <int KERNEL, int MODE, int NCH>
__global__ void __launch_bounds__(256) k_gather_light(GatherArgs G) {
    gather_light_cells<KERNEL, MODE, NCH>(G, blockIdx.x);
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

template <class Args>
void fill_topology(Volume *v, Args &S) {
    S.slot_leaf = v->slot_leaf.as<int32_t>();
    S.leaves = v->pool_ptr(0);
    S.nbr27 = v->nbr27.as<int32_t>();
    S.bin_off = v->bin_off.as<uint32_t>();
    S.perm = v->perm.as<int32_t>();
    S.res0 = v->res(0);
    S.m = v->res(0) / kCell;
    S.m3 = S.m * S.m * S.m;
    S.cell_list = v->cell_list.as<int32_t>();
    S.cell_light = v->cell_light.as<int32_t>();
    S.cell_cnt = v->cell_cnt.as<uint32_t>();
    S.ncell = v->atlas_last * S.m3;
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

// The channel amounts of the group in bin order: bin_amt[j] for the point
// perm[j], j below the number of binned points (reg_off[ncell * 27]).
template <int NCH>
__global__ void k_pack_amounts(SplatArgs S) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= (int64_t)S.reg_off[S.ncell * kRegions]) return;
    const int32_t p = S.perm[j];
    const float wt = S.has_weight ? load_f1(S.weight, p) : S.wconst;
    float a4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int c = 0; c < NCH; c++) a4[c] = ((S.attr_mask >> c) & 1) ? wt * load_f1(S.attr[c], p) : wt;
    S.bin_amt[j] = make_float4(a4[0], a4[1], a4[2], a4[3]);
}

// Owner-computes scatter of up to 4 channels (one group): a warp per cell,
// every cell of the active bricks (cells no stencil reaches get zeros).
template <int KERNEL, int NCH>
gvdb2_status scatter_group(Volume *v, const SplatArgs &S0) {
    constexpr size_t smem = sizeof(ScChunk) * kScWarps;
    auto k = k_scatter_cells<KERNEL, NCH>;
    GV_TRY(launch_smem(v, k, smem, "scatter"));
    GV_CUDA(v, v->bin_amt.ensure(sizeof(float4) * (size_t)std::max<int64_t>(v->bin_key.n, 1), v->stream));
    SplatArgs S = S0;
    S.bin_amt = v->bin_amt.as<float4>();
    const int64_t single = (S.ncell + kScWarps - 1) / kScWarps;
    const int64_t blocks = single + v->giant_grid; // giant cells: at most n / kGiantCell of them
    if (v->bin_key.n > 0)
        k_pack_amounts<NCH><<<grid_for(v->bin_key.n, 256, 1ll << 31), 256, 0, v->stream>>>(S);
    if (blocks > 0) k<<<(unsigned)blocks, 32 * kScWarps, smem, v->stream>>>(S, single);
    GV_CUDA(v, cudaGetLastError());
    return GVDB2_OK;
}

// channels [first, first + count) of S as a group of their own
SplatArgs channel_group(const SplatArgs &S, int first, int count) {
    SplatArgs G = S;
    G.attr_mask = (S.attr_mask >> first) & ((1u << count) - 1);
    for (int c = 0; c < kMaxSplatChan; c++) {
        const bool in = c < count;
        G.chan[c] = in ? S.chan[first + c] : nullptr;
        G.attr[c] = in ? S.attr[first + c] : PointsView{};
    }
    G.nch = count;
    return G;
}

template <int KERNEL>
gvdb2_status scatter_groups(Volume *v, const SplatArgs &S) {
    for (int first = 0; first < S.nch; first += 4) {
        const int cnt = std::min(4, S.nch - first);
        const SplatArgs G = channel_group(S, first, cnt);
        switch (cnt) {
        case 1: GV_TRY((scatter_group<KERNEL, 1>(v, G))); break;
        case 2: GV_TRY((scatter_group<KERNEL, 2>(v, G))); break;
        case 3: GV_TRY((scatter_group<KERNEL, 3>(v, G))); break;
        default: GV_TRY((scatter_group<KERNEL, 4>(v, G))); break;
        }
    }
    return GVDB2_OK;
}

gvdb2_status run_scatter(Volume *v, int kernel, const SplatArgs &S) {
    if (v->atlas_last == 0) return GVDB2_OK;
    if (v->res(0) % kCell)
        return fail(v, GVDB2_ERR_UNSUPPORTED, "kernel splats need bricks of a multiple of 8 voxels");
    return kernel == GVDB2_KERNEL_TENT1 ? scatter_groups<GVDB2_KERNEL_TENT1>(v, S)
                                        : scatter_groups<GVDB2_KERNEL_CUBIC2>(v, S);
}

template <int KERNEL, int MODE, int NCH>
gvdb2_status launch_gather(Volume *v, const GatherArgs &G) {
    constexpr size_t smem = gather_tile_smem<KERNEL, NCH>();
    auto k = k_gather_tile<KERNEL, MODE, NCH>;
    GV_TRY(launch_smem(v, k, smem, "gather"));
    // tiles for the huge and heavy cells, then the light cells, a warp each
    // (every cell gets a tile when the caller supplied the binning)
    const int64_t heavy = G.cell_list ? v->heavy_grid : G.ncell;
    if (heavy > 0) k<<<(unsigned)heavy, kGatherThreads, smem, v->stream>>>(G);
    if (G.cell_list && v->light_grid > 0)
        k_gather_light<KERNEL, MODE, NCH><<<(unsigned)((v->light_grid + 7) / 8), 256, 0, v->stream>>>(G);
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

gvdb2_status check_chans(Volume *v, const int *chans, int nch) {
    if (!chans || nch < 1 || nch > kMaxSplatChan) return fail(v, GVDB2_ERR_ARG, "1 to 8 channels per splat call");
    for (int c = 0; c < nch; c++)
        if (chans[c] < 0 || chans[c] >= kMaxChan || !v->has_chan[chans[c]]) return fail(v, GVDB2_ERR_ARG, "bad channel");
    return GVDB2_OK;
}

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

template <bool LEVELSET, bool FP16>
gvdb2_status launch_gather_voxels(Volume *v, int sc, float radius, int chan, int accum) {
    ScList pl;
    pl.pnt = (!FP16 && v->sc_len > 0) ? v->sc_pnt.as<float>() : nullptr;
    pl.q = (FP16 && v->sc_len > 0) ? v->sc_q.as<uint16_t>() : nullptr;
    pl.qmin = make_float3(v->posmin[0], v->posmin[1], v->posmin[2]);
    pl.qrange = make_float3(v->posmax[0] - v->posmin[0], v->posmax[1] - v->posmin[1], v->posmax[2] - v->posmin[2]);
    if (sc == 4) {
        const unsigned g = (unsigned)((v->num_sc + kGvWarps - 1) / kGvWarps);
        k_gather_voxels_sc4<LEVELSET, FP16><<<g, 32 * kGvWarps, 0, v->stream>>>(
            v->num_sc, radius, v->sc_nid.as<int32_t>(), v->sc_cnt.as<uint32_t>(), v->sc_off.as<uint32_t>(),
            v->sc_pos.as<int32_t>(), pl, v->pool_ptr(0), atlas_geom(v), v->atlas[chan].as<float>(), accum);
    } else {
        const int threads = v->sc_per_brick * sc * sc * sc;
        const int64_t blocks = (v->num_sc + v->sc_per_brick - 1) / v->sc_per_brick;
        k_gather_voxels<LEVELSET, FP16><<<(unsigned)blocks, threads, 0, v->stream>>>(
            v->num_sc, v->sc_per_brick, sc, radius, v->sc_nid.as<int32_t>(), v->sc_cnt.as<uint32_t>(),
            v->sc_off.as<uint32_t>(), v->sc_pos.as<int32_t>(), pl, v->pool_ptr(0), v->apron, atlas_geom(v),
            v->atlas[chan].as<float>(), accum);
    }
    GV_CUDA(v, cudaGetLastError());
    return GVDB2_OK;
}

gvdb2_status gather_voxels(Volume *v, int sc, float radius, int chan, int accum, bool levelset, bool fp16) {
    if (chan < 0 || chan >= kMaxChan || !v->has_chan[chan]) return fail(v, GVDB2_ERR_ARG, "bad channel");
    if (v->num_sc == 0 || sc != v->sc_size) return fail(v, GVDB2_ERR_STATE, "InsertPointsSubcell must precede the gather");
    if (fp16 != v->sc_fp16)
        return fail(v, GVDB2_ERR_STATE, fp16 ? "GatherLevelSet_FP16 needs the lists of InsertPointsSubcell_FP16"
                                             : "the subcell lists hold 16-bit entries: use GatherLevelSet_FP16");
    if (fp16 && !levelset) return fail(v, GVDB2_ERR_UNSUPPORTED, "16-bit lists serve the level set only");
    // 4^3 subcells take a warp each; other sizes a CTA per brick
    if (sc != 4 && v->sc_per_brick * sc * sc * sc > 1024)
        return fail(v, GVDB2_ERR_UNSUPPORTED, "subcells other than 4^3 need bricks of at most 1024 voxels");
    if ((v->num_sc + v->sc_per_brick - 1) / v->sc_per_brick == 0) return GVDB2_OK;
    if (fp16) return launch_gather_voxels<true, true>(v, sc, radius, chan, 0);
    return levelset ? launch_gather_voxels<true, false>(v, sc, radius, chan, accum)
                    : launch_gather_voxels<false, false>(v, sc, radius, chan, accum);
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
    S.reg_off = v->reg_off.as<uint32_t>();
    S.cell_giant = v->cell_giant.as<int32_t>();
    S.bin_pos = v->bin_pos.as<float4>();
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
    G.bin_pos = v->bin_pos.as<float4>(); // bins made by bin_points
    return run_gather<kFwd>(v, kernel, G);
}

gvdb2_status gather_kernel_prebinned(Volume *v, int kernel, int n, const float trans[3], const int *chans, int nch,
                                     float *out, int64_t out_stride, const uint32_t *bin_off, const int32_t *perm) {
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
    G.bin_off = bin_off;
    G.perm = perm;
    G.cell_list = nullptr; // bins supplied by the caller: every cell, in cell order
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
    G.bin_pos = v->bin_pos.as<float4>(); // bins made by bin_points
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
        S.reg_off = v->reg_off.as<uint32_t>();
        S.cell_giant = v->cell_giant.as<int32_t>();
        S.bin_pos = v->bin_pos.as<float4>();
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
    G.bin_pos = v->bin_pos.as<float4>(); // bins made by bin_points
    return run_gather<kGatherBwd>(v, kernel, G);
}

} // namespace gvdb2
