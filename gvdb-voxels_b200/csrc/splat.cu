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
    const int32_t *cell_list, *cell_light;
    const uint32_t *cell_cnt;
    int64_t ncell;
    int64_t tvox;
    // dense cells: partial slot per cell (-1: not dense), work items,
    // partial sums, integer accumulators and arrival counters, and the
    // capacities of the slots
    int64_t dense_cap, multi_cap;
    uint32_t slice; // points per dense-cell work item
    SplatLimits lim;
    const int32_t *cell_part;
    const int4 *part_work;
    float *part;
    int32_t *part_acc;
    uint32_t *part_done;
    // cells with a dense cell among their 27 (k_scatter_cells lists them)
    int32_t *merge_list;
    uint32_t *merge_cnt;
};


// ---- dense cells: partial sums ------------------------------------------
//
// A cell of at least the volume's dense threshold (the tuning's `dense`,
// kDenseCell = 512 by default) of points, a dense cell, is splatted on its
// own, each point once with its whole stencil, into an extended tile
// [-H, 8+H)^3 (H = N/2: 12^3 for the cubic B-spline, 10^3 for the tent):
// the cell's partial sums.  The owner-computes scatter below then leaves a
// dense cell's points out of every cell's sources and instead adds, to each
// voxel, the partials of the dense cells among the up to 8 whose extended
// tile covers it.  Where the cells hold many points this splats each point
// once instead of from every cell its stencil reaches (about (1 + 3/8)^3 =
// 2.6 for the cubic B-spline), and its adds all do work.  Whether a cell is
// dense depends on its own point count only, so a cell's result depends on
// its neighbourhood alone (a batched cloud gets what a volume of its own
// gets).
//
// k_scatter_part: one CTA per work item, a slice of up to S.slice points
// (the tuning's `slice`, kSlicePts = 4096 by default)
// of a dense cell, accumulates its points' stencils in shared memory with
// atomics.  A cell of one slice writes its partial directly; the slices of
// a larger cell add their tiles into the cell's global accumulator, and the
// CTA that arrives last (an arrival counter; no CTA waits for another)
// writes the partial and clears the accumulator and counter for the next
// call.  k_scatter_merge then adds the partials to the voxels they cover,
// after the owner-computes pass has written its sums.
//
// The accumulators are fixed-point integers: integer sums do not depend on
// the order of the adds, so the partial is the same whatever the order of
// the points within their bins and whatever the split into slices.  (Float
// shared-memory atomics, half as many, measured 16% slower.)
//
// Fixed point: each contribution x = amount * weight is scaled by 2^s and
// rounded to an integer, split as rint(x) = hi * 2^L + lo with both parts
// found by the float "magic number" rounding (t = x*2^-L + 1.5*2^23 holds
// rint(x*2^-L) in its low mantissa bits; the remainder x - hi*2^L is
// exact), and added with two 32-bit atomics.  With R the cell's points and
// max|a| the largest |amount| among them (weights are at most 1), s and L
// are set per cell and channel so that no sum overflows:
//   L = min(22, 31 - bits(R+1))      -> |sum lo| <= R * 2^(L-1) < 2^31
//   max|a| * 2^s < 2^(21+L)          -> |x * 2^-L| < 2^22 (magic range)
//   R * max|a| * 2^s < 2^(29+L)      -> |sum hi| < 2^29 + R/2
// (One 64-bit atomic per tap and channel instead measured 1.9x slower.)
template <int KERNEL>
struct ExtTile {
    static constexpr int N = Taps<KERNEL>::N;
    static constexpr int H = N / 2;
    static constexpr int E = 8 + N;                 // 12 (cubic) or 10 (tent)
    static constexpr int RS = E;                    // row stride (words)
    static constexpr int PS = N == 4 ? E * E + 8 : E * E; // plane stride: 152 puts a warp's taps in distinct banks
    static constexpr int CS = E * PS;               // channel stride
    static constexpr int E3 = E * E * E;            // floats per channel in the partial
    // Position in a cell's partial of extended-tile voxel (ux, uy, uz) in
    // [0, E)^3.  Per channel the partial holds 27 regions: the cell's 8^3
    // interior first, then the halo beyond each face, edge and corner d in
    // {-1,0,1}^3 (z-major order of d), each z-major with extent 8 along the
    // axes where d is 0 and H where it is not, so that interior rows are
    // whole 32-byte sectors.  Region d starts, in the plain z-major order of
    // the regions, at start_z E^2 + s_z start_y E + s_z s_y start_x, with
    // start and s the region's first extended coordinate and extent along
    // each axis.
    __host__ __device__ static constexpr int part_index(int ux, int uy, int uz) {
        const int dx = ux < H ? -1 : (ux >= 8 + H ? 1 : 0), dy = uy < H ? -1 : (uy >= 8 + H ? 1 : 0),
                  dz = uz < H ? -1 : (uz >= 8 + H ? 1 : 0);
        const int sx0 = dx < 0 ? 0 : (dx == 0 ? H : 8 + H), sy0 = dy < 0 ? 0 : (dy == 0 ? H : 8 + H),
                  sz0 = dz < 0 ? 0 : (dz == 0 ? H : 8 + H);
        const int ex = dx == 0 ? 8 : H, ey = dy == 0 ? 8 : H, ez = dz == 0 ? 8 : H;
        const int local = ((uz - sz0) * ey + (uy - sy0)) * ex + (ux - sx0);
        if ((dx | dy | dz) == 0) return local; // interior
        const int r = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
        const int start = sz0 * E * E + ez * sy0 * E + ez * ey * sx0;
        return 512 + start - (r > 13 ? 512 : 0) + local;
    }
};
// The inverse of part_index: the shared tile address of each partial
// position, so that a partial is written in order (coalesced).
template <int KERNEL>
struct PartAddr {
    uint16_t addr[ExtTile<KERNEL>::E3];
    constexpr PartAddr() : addr() {
        using X = ExtTile<KERNEL>;
        for (int z = 0; z < X::E; z++)
            for (int y = 0; y < X::E; y++)
                for (int x = 0; x < X::E; x++) addr[X::part_index(x, y, z)] = (uint16_t)(z * X::PS + y * X::RS + x);
    }
};
template <int KERNEL>
__device__ constexpr PartAddr<KERNEL> kPartAddr{};

// The partials that cover interior voxel v (x | y << 3 | z << 6) of a cell:
// entry m of row v is the partial position (11 bits) and the neighbour
// direction d (5 bits, z-major in {-1,0,1}^3) of source m, or 0xFFFF when
// source m does not cover v.  Source m steps across the faces named by its
// bits (x, y, z) toward the near face of v when v lies within H of one.
template <int KERNEL>
struct alignas(16) MergeMap {
    uint16_t src[512][8];
    constexpr MergeMap() : src() {
        using X = ExtTile<KERNEL>;
        for (int v = 0; v < 512; v++) {
            const int vx = v & 7, vy = (v >> 3) & 7, vz = v >> 6;
            const int ex = vx < X::H ? -1 : (vx >= 8 - X::H ? 1 : 0);
            const int ey = vy < X::H ? -1 : (vy >= 8 - X::H ? 1 : 0);
            const int ez = vz < X::H ? -1 : (vz >= 8 - X::H ? 1 : 0);
            for (int m = 0; m < 8; m++) {
                const bool used = (!(m & 1) || ex) && (!(m & 2) || ey) && (!(m & 4) || ez);
                const int dx = (m & 1) ? ex : 0, dy = (m & 2) ? ey : 0, dz = (m & 4) ? ez : 0;
                const int d = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
                src[v][m] = used ? (uint16_t)(X::part_index(vx - 8 * dx + X::H, vy - 8 * dy + X::H,
                                                            vz - 8 * dz + X::H) | (d << 11))
                                 : (uint16_t)0xFFFF;
            }
        }
    }
};
template <int KERNEL>
__device__ constexpr MergeMap<KERNEL> kMergeMap{};
static_assert(ExtTile<GVDB2_KERNEL_CUBIC2>::E3 <= 2048 && ExtTile<GVDB2_KERNEL_TENT1>::E3 <= 2048,
              "partial positions fit 11 bits");

constexpr int kPartThreads = 256;
constexpr int kPartChunk = 128; // points staged per pass, one per thread of the first 128
// row stride of the staged x and y weights: a point's taps (one row each)
// fall in different banks
constexpr int kPartRow = kPartChunk + 1;
static_assert(kSlicePts % kPartChunk == 0, "slices are whole chunks"); // tuned slices are multiples of kPartChunk too

template <int KERNEL, int NCH>
constexpr size_t part_smem_bytes() {
    return sizeof(int32_t) * 2 * NCH * ExtTile<KERNEL>::CS +
           sizeof(float4) * 2 * kPartChunk + sizeof(float) * 2 * Taps<KERNEL>::N * kPartRow +
           sizeof(int32_t) * kPartChunk;
}

// The fixed-point scale of R points whose largest |amount| is am, per the
// bounds above: returns 2^s (0 when there is nothing to add), sets `inv` =
// 2^-s and `lvl` = L.
__device__ __forceinline__ float part_scale(uint32_t R, float am, double &inv, int &lvl) {
    int e1 = 0, e2 = 0;
    frexpf(am, &e1);            // am < 2^e1
    frexpf((float)R * am, &e2); // R*am < 2^e2
    const int L = min(22, 31 - (32 - __clz((int)R + 1)));
    lvl = L;
    const int s = min(21 + L - e1, 29 + L - e2);
    const bool on = am > 0.0f && R > 0;
    inv = on ? ldexp(1.0, -s) : 0.0;
    return on ? ldexpf(1.0f, s) : 0.0f;
}

// Adds the fixed-point value of x (already scaled by 2^s) at tile index idx
// of one channel's accumulators: hi at idx, lo at CS + idx.
template <int CS>
__device__ __forceinline__ void part_add(int32_t *acc, int idx, float x, float inv2L, float two2L) {
    const float M = 12582912.0f; // 1.5 * 2^23
    const float t = fmaf(x, inv2L, M);
    const int hi = __float_as_int(t) - 0x4B400000;
    const float r = fmaf(t - M, -two2L, x);
    const int lo = __float_as_int(r + M) - 0x4B400000;
    atomicAdd(acc + idx, hi);
    atomicAdd(acc + CS + idx, lo);
}

// One work item per CTA: slice item.y of item.z of dense cell item.x
// (item.w: the cell's accumulator slot when item.z > 1).  The partial goes
// to part + cell_part[cell] * NCH * E3.
template <int KERNEL, int NCH>
__global__ void __launch_bounds__(kPartThreads) k_scatter_part(SplatArgs S) {
    using T = Taps<KERNEL>;
    using X = ExtTile<KERNEL>;
    constexpr int N = T::N;
    constexpr int AS = 2 * X::CS; // accumulator words per channel (hi, lo)
    extern __shared__ __align__(16) unsigned char part_smem[];
    int32_t *acc = reinterpret_cast<int32_t *>(part_smem);
    // staged points: z weights and scaled amounts as float4 (a lane reads its
    // two z weights in one load, the amounts in one broadcast), x and y
    // weights in padded rows, the first tap's tile address
    float4 *pz = reinterpret_cast<float4 *>(acc + NCH * AS);
    float4 *pa = pz + kPartChunk;
    float(*pw)[kPartRow] = reinterpret_cast<float(*)[kPartRow]>(pa + kPartChunk);
    int32_t *pb = reinterpret_cast<int32_t *>(pw + 2 * N);
    __shared__ double inv_s[NCH];
    __shared__ int32_t amax_bits[NCH]; // largest |amount| of the cell's points, as float bits
    __shared__ int last;
    if (blockIdx.x >= S.cell_cnt[kCntWork]) return;
    const int4 item = S.part_work[blockIdx.x];
    const int64_t cell = item.x;
    const int nslice = item.z;
    // every check below is the same for the whole CTA
    if (!in_range(S.lim, cell, S.ncell, 6)) return;
    const int32_t pslot = S.cell_part[cell];
    if (!in_range(S.lim, pslot, S.dense_cap, 7) || (nslice > 1 && !in_range(S.lim, item.w, S.multi_cap, 8))) return;
    const uint32_t beg = S.bin_off[cell], R = S.bin_off[cell + 1] - beg;
    if (!in_range(S.lim, (int64_t)beg + R - 1, S.lim.nentry, 9)) return;
    const uint32_t s0 = (uint32_t)item.y * S.slice, s1 = min(R, s0 + S.slice);
    int64_t slot;
    int cx, cy, cz;
    cell_coords(cell, S.m, S.m3, slot, cx, cy, cz);
    const int32_t leaf = S.slot_leaf[slot];
    if (!in_range(S.lim, leaf, S.lim.npool, 10)) return;
    static_assert((NCH * AS * sizeof(int32_t)) % 16 == 0, "16-byte zeroing");
    for (int i = threadIdx.x; i < (int)(NCH * AS * sizeof(int32_t) / 16); i += kPartThreads)
        reinterpret_cast<int4 *>(acc)[i] = make_int4(0, 0, 0, 0);
    const Node &nd = S.leaves[leaf];
    const int ox = nd.mPos[0] + kCell * cx - X::H, oy = nd.mPos[1] + kCell * cy - X::H,
              oz = nd.mPos[2] + kCell * cz - X::H;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // the largest |amount| per channel over all the cell's points sets the
    // scale, the same in every slice of the cell
    if (threadIdx.x < NCH) amax_bits[threadIdx.x] = 0;
    float mx[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) mx[c] = 0.0f;
    for (uint32_t j = threadIdx.x; j < R; j += kPartThreads) {
        const float4 a = S.bin_amt[beg + j];
        const float a4[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int c = 0; c < NCH; c++) mx[c] = fmaxf(mx[c], fabsf(a4[c]));
    }
    __syncthreads(); // amax_bits cleared
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        float x = mx[c];
        for (int o = 16; o > 0; o >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, o));
        if (lane == 0 && x > 0.0f) atomicMax(&amax_bits[c], __float_as_int(x));
    }
    __syncthreads();
    float scale[NCH];
    int L = 0;
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        double inv;
        scale[c] = part_scale(R, __int_as_float(amax_bits[c]), inv, L);
        if (threadIdx.x == 0) inv_s[c] = inv;
    }
    const float inv2L = ldexpf(1.0f, -L), two2L = ldexpf(1.0f, L);
    for (uint32_t base = s0; base < s1; base += kPartChunk) {
        const int cnt = (int)min((uint32_t)kPartChunk, s1 - base);
        if (base > s0) __syncthreads(); // previous chunk consumed
        if ((int)threadIdx.x < cnt) { // stage point base + t as record t
            const uint32_t j = beg + base + threadIdx.x;
            const float4 q = S.bin_pos[j]; // translated position, cloud index bits
            const int32_t cloud = __float_as_int(q.w);
            int3 o = make_int3(0, 0, 0);
            if (cloud >= 0 && in_range(S.lim, cloud, S.lim.ncloud, 5))
                o = make_int3(S.pos.origin[3 * cloud], S.pos.origin[3 * cloud + 1], S.pos.origin[3 * cloud + 2]);
            float wx[N], wy[N], wz[N];
            const int fx = T::eval(q.x, wx) + o.x - ox;
            const int fy = T::eval(q.y, wy) + o.y - oy;
            const int fz = T::eval(q.z, wz) + o.z - oz;
            // a point binned to the cell has its first taps in [0, 8] of the
            // extended tile; anything else is dropped, never written outside it
            const bool ok = (unsigned)fx <= 8u && (unsigned)fy <= 8u && (unsigned)fz <= 8u;
            const int r = threadIdx.x;
            pb[r] = ok ? fz * X::PS + fy * X::RS + fx : 0; // tile address of the point's first tap
            float z4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 0; k < N; k++) {
                pw[k][r] = wx[k];
                pw[N + k][r] = wy[k];
                z4[k] = wz[k];
            }
            pz[r] = make_float4(z4[0], z4[1], z4[2], z4[3]);
            const float4 a = S.bin_amt[j];
            const float a4[4] = {a.x, a.y, a.z, a.w};
            float s4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int c = 0; c < NCH; c++) s4[c] = ok ? a4[c] * scale[c] : 0.0f;
            pa[r] = make_float4(s4[0], s4[1], s4[2], s4[3]);
        }
        __syncthreads();
        if constexpr (N == 4) {
            // one point per warp step: lane = (tx, ty, z pair), two taps a lane
            const int tx = lane & 3, ty = (lane >> 2) & 3, tz0 = (lane >> 4) * 2;
            const int loff = tz0 * X::PS + ty * X::RS + tx;
            for (int j = warp; j < cnt; j += kPartThreads / 32) {
                const int a0 = pb[j] + loff;
                const float wxy = pw[tx][j] * pw[N + ty][j];
                const float2 z2 = reinterpret_cast<const float2 *>(pz + j)[tz0 >> 1];
                const float w0 = wxy * z2.x, w1 = wxy * z2.y;
                const float4 a4 = pa[j];
                const float am4[4] = {a4.x, a4.y, a4.z, a4.w};
#pragma unroll
                for (int c = 0; c < NCH; c++) {
                    const float am = am4[c];
                    part_add<X::CS>(acc + c * AS, a0, am * w0, inv2L, two2L);
                    part_add<X::CS>(acc + c * AS, a0 + X::PS, am * w1, inv2L, two2L);
                }
            }
        } else {
            // four points per warp step, one tap a lane
            const int sub = lane >> 3, tx = lane & 1, ty = (lane >> 1) & 1, tz = (lane >> 2) & 1;
            const int loff = tz * X::PS + ty * X::RS + tx;
            for (int j0 = warp * 4; j0 < cnt; j0 += kPartThreads / 8) {
                const int j = j0 + sub;
                if (j >= cnt) continue;
                const int a = pb[j] + loff;
                const float4 z4 = pz[j], a4 = pa[j];
                const float w = pw[tx][j] * pw[N + ty][j] * (tz ? z4.y : z4.x);
                const float am4[4] = {a4.x, a4.y, a4.z, a4.w};
#pragma unroll
                for (int c = 0; c < NCH; c++) part_add<X::CS>(acc + c * AS, a, am4[c] * w, inv2L, two2L);
            }
        }
    }
    __syncthreads();
    // partial position i of channel c: thread t takes i = t, t + 256, ...
    // (coalesced), each looked up in its tile voxel
    float *dst = S.part + (int64_t)pslot * NCH * X::E3;
    static_assert(kPartThreads < X::E3, "one channel step per iteration");
    auto value = [&](int c, int32_t hi, int32_t lo) {
        // |sum| < 2^53: exact in double; the power-of-two scalings are exact
        return (float)((double)(((long long)hi << L) + (long long)lo) * inv_s[c]);
    };
    if (nslice == 1) {
        int c = 0, i0 = threadIdx.x;
        for (int i = threadIdx.x; i < NCH * X::E3; i += kPartThreads) {
            const int k = c * AS + kPartAddr<KERNEL>.addr[i0];
            dst[i] = value(c, acc[k], acc[k + X::CS]);
            if ((i0 += kPartThreads) >= X::E3) i0 -= X::E3, c++;
        }
        return;
    }
    // a cell of several slices: this slice's integer sums into the cell's
    // accumulator (per channel hi[E3], lo[E3], in partial order)
    constexpr int GW = 2 * X::E3; // accumulator words per channel
    int32_t *g = S.part_acc + (int64_t)item.w * NCH * GW;
    {
        int c = 0, i0 = threadIdx.x;
        for (int i = threadIdx.x; i < NCH * X::E3; i += kPartThreads) {
            const int k = c * AS + kPartAddr<KERNEL>.addr[i0];
            int32_t *gc = g + c * GW + i0;
            if (acc[k]) atomicAdd(gc, acc[k]);
            if (acc[k + X::CS]) atomicAdd(gc + X::E3, acc[k + X::CS]);
            if ((i0 += kPartThreads) >= X::E3) i0 -= X::E3, c++;
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(S.part_done + item.w, 1u) == (uint32_t)(nslice - 1);
    __syncthreads();
    if (!last) return;
    // the last slice: every other slice's adds are visible; read the sums
    // and clear the accumulator (atomic exchanges) and the counter
    __threadfence();
    int c = 0, i0 = threadIdx.x;
    for (int i = threadIdx.x; i < NCH * X::E3; i += kPartThreads) {
        int32_t *gc = g + c * GW + i0;
        dst[i] = value(c, atomicExch(gc, 0), atomicExch(gc + X::E3, 0));
        if ((i0 += kPartThreads) >= X::E3) i0 -= X::E3, c++;
    }
    if (threadIdx.x == 0) S.part_done[item.w] = 0;
}

// ---- owner-computes scatter --------------------------------------------
//
// One warp per cell (an 8^3 block of a brick; the brick itself for 8^3
// bricks) computes the cell's interior voxels from every point whose stencil
// reaches them and writes each voxel once: no atomics, no zero-fill pass.
// Its sources are the cell's own points and, from each of the 26 neighbour
// cells, the regions of that cell's bin whose stencils cross the shared
// face, edge or corner (k_bin_count bins points by cell and region), so
// every source is a point the cell needs -- except the points of dense
// cells (this cell's included), whose partial sums k_scatter_merge adds to
// the voxels afterwards.
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
// sort, then k_scatter_merge adds the partials in a fixed order, so with
// deterministic binning the result is bit-reproducible.
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
    uint2 run[64]; // the cell's sources: runs [x, y) of perm (at most 1 + 2 + 10 + 50 = 63)
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

// kScWarps cells per CTA, a warp per cell.
template <int KERNEL, int NCH>
__global__ void __launch_bounds__(32 * kScWarps, GVDB2_SC_MIN_BLOCKS) k_scatter_cells(SplatArgs S) {
    using T = Taps<KERNEL>;
    using X = ExtTile<KERNEL>;
    constexpr int N = T::N;
    extern __shared__ __align__(16) unsigned char sc_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    ScChunk &C = reinterpret_cast<ScChunk *>(sc_smem)[warp];
    const int64_t cell = (int64_t)blockIdx.x * kScWarps + warp;
    if (cell >= S.ncell) return;
    int64_t slot;
    int cx, cy, cz;
    cell_coords(cell, S.m, S.m3, slot, cx, cy, cz);
    const int32_t leaf = S.slot_leaf[slot];
    if (!in_range(S.lim, leaf, S.lim.npool, 1)) return; // the same for the whole warp
    const Node &nd = S.leaves[leaf];
    const int ox = nd.mPos[0] + kCell * cx, oy = nd.mPos[1] + kCell * cy, oz = nd.mPos[2] + kCell * cz;
    // The sources, as runs of perm in a fixed order: lane d < 27 lists those of
    // the neighbour cell in direction d = (dz+1)*9 + (dy+1)*3 + (dx+1): its
    // regions whose stencils reach this cell -- per axis, across the lower
    // face its upper band (2), across the upper face its lower band (0),
    // along the axis all three -- merged into as few runs as the region
    // order allows; a dense neighbour gives its partial slot instead.
    int nrun = 0;
    uint2 runs[9];
    int32_t pslot = -1;
    if (lane < 27) {
        const int dx = lane % 3 - 1, dy = lane / 3 % 3 - 1, dz = lane / 9 - 1;
        const int ncx = cx + dx, ncy = cy + dy, ncz = cz + dz;
        const int bx = ncx < 0 ? -1 : (ncx >= S.m ? 1 : 0), by = ncy < 0 ? -1 : (ncy >= S.m ? 1 : 0),
                  bz = ncz < 0 ? -1 : (ncz >= S.m ? 1 : 0);
        int32_t ns = (bx | by | bz) == 0 ? (int32_t)slot
                                         : S.nbr27[slot * 27 + (bz + 1) * 9 + (by + 1) * 3 + (bx + 1)];
        if (ns >= 0 && !in_range(S.lim, ns, S.lim.nslot, 2)) ns = -1;
        int64_t nc = ns < 0 ? -1
                            : (int64_t)ns * S.m3 + ((ncz - bz * S.m) * S.m + (ncy - by * S.m)) * S.m + (ncx - bx * S.m);
        if (nc >= 0) pslot = S.cell_part[nc];
        if (pslot >= 0 && !in_range(S.lim, pslot, S.dense_cap, 3)) pslot = -1, nc = -1;
        if (nc >= 0 && pslot < 0) {
            const uint32_t *ro = S.reg_off + nc * kRegions;
            const int rx0 = dx < 0 ? 2 : 0, ry0 = dy < 0 ? 2 : 0, ry1 = dy > 0 ? 0 : 2;
            const int rz0 = dz < 0 ? 2 : 0, rz1 = dz > 0 ? 0 : 2;
            auto add = [&](int r0, int r1) { // regions [r0, r1)
                const uint2 u = make_uint2(ro[r0], ro[r1]);
                if (u.y > u.x && in_range(S.lim, (int64_t)u.y - 1, S.lim.nentry, 4)) runs[nrun++] = u;
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
    const bool any_part = __any_sync(0xffffffffu, pslot >= 0);
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
            if (cloud >= 0 && in_range(S.lim, cloud, S.lim.ncloud, 5))
                d.o = make_int3(S.pos.origin[3 * cloud], S.pos.origin[3 * cloud + 1], S.pos.origin[3 * cloud + 2]);
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
    // the sources, 32 a step
    if (GVDB2_SC_PREFETCH) {
        // the next step's reads are in flight while this step's records are
        // built and a full chunk is added
        Src nxt = fetch(0);
        for (uint32_t vb = 0; vb < total_src; vb += 32) {
            const Src cur = nxt;
            if (vb + 32 < total_src) nxt = fetch(vb + 32);
            flush_if_full();
            build(cur);
        }
    } else {
        for (uint32_t vb = 0; vb < total_src; vb += 32) {
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
    // cells with a dense cell around get its partials from k_scatter_merge;
    // one without sources of its own (all zero here) is listed as ~cell and
    // left for the merge to write
    if (any_part) {
        if (lane == 0) S.merge_list[atomicAdd(S.merge_cnt, 1u)] = total_src == 0 ? ~(int32_t)cell : (int32_t)cell;
        if (total_src == 0) return;
    }
    // each lane writes its 4 x 4 voxels of every channel once
    const int a = S.apron, tl = S.tile;
    const int64_t base = slot * S.tvox + (int64_t)(kCell * cx + 4 * q + a);
#pragma unroll
    for (int zz = 0; zz < 4; zz++)
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            float *dst = S.chan[c] + base + ((int64_t)(kCell * cz + 4 * h + zz + a) * tl + (kCell * cy + y + a)) * tl;
            dst[0] = acc[zz][0][c].x;
            dst[1] = acc[zz][0][c].y;
            dst[2] = acc[zz][1][c].x;
            dst[3] = acc[zz][1][c].y;
        }
}

// Adds the dense cells' partials to the cells listed by k_scatter_cells
// (those with a dense cell among their 27): a CTA per listed cell (CTAs
// past the list's end return), a thread per interior voxel, which adds, in
// the order of kMergeMap, the partials that cover the voxel to the sum the
// owner-computes pass wrote -- or writes them, for a cell listed as ~cell
// (no owner sources: its sum is 0, and 0 + x is x).
template <int KERNEL, int NCH>
__global__ void __launch_bounds__(512) k_scatter_merge(SplatArgs S) {
    using X = ExtTile<KERNEL>;
    __shared__ int32_t ne[27]; // partial slot of the dense cell in each direction, or -1
    const uint32_t li = blockIdx.x;
    if (li >= *S.merge_cnt) return;
    {
        const int32_t entry = S.merge_list[li];
        const bool overwrite = entry < 0; // no owner sum to add to
        const int64_t cell = overwrite ? ~entry : entry;
        if (!in_range(S.lim, cell, S.ncell, 23)) return;
        int64_t slot;
        int cx, cy, cz;
        cell_coords(cell, S.m, S.m3, slot, cx, cy, cz);
        if (threadIdx.x < 27) {
            const int d = threadIdx.x;
            const int ncx = cx + d % 3 - 1, ncy = cy + d / 3 % 3 - 1, ncz = cz + d / 9 - 1;
            const int bx = ncx < 0 ? -1 : (ncx >= S.m ? 1 : 0), by = ncy < 0 ? -1 : (ncy >= S.m ? 1 : 0),
                      bz = ncz < 0 ? -1 : (ncz >= S.m ? 1 : 0);
            int32_t ns = (bx | by | bz) == 0 ? (int32_t)slot
                                             : S.nbr27[slot * 27 + (bz + 1) * 9 + (by + 1) * 3 + (bx + 1)];
            int32_t e = -1;
            if (ns >= 0 && in_range(S.lim, ns, S.lim.nslot, 21)) {
                e = S.cell_part[(int64_t)ns * S.m3 + ((ncz - bz * S.m) * S.m + (ncy - by * S.m)) * S.m +
                                (ncx - bx * S.m)];
                if (e >= 0 && !in_range(S.lim, e, S.dense_cap, 22)) e = -1;
            }
            ne[d] = e;
        }
        __syncthreads();
        const int v = threadIdx.x;
        const uint4 row = *reinterpret_cast<const uint4 *>(kMergeMap<KERNEL>.src[v]);
        const uint32_t wr[4] = {row.x, row.y, row.z, row.w};
        float add[NCH];
#pragma unroll
        for (int c = 0; c < NCH; c++) add[c] = 0.0f;
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const uint32_t ent = (wr[m >> 1] >> (16 * (m & 1))) & 0xFFFFu;
            const int32_t e = ent != 0xFFFFu ? ne[ent >> 11] : -1;
            if (e < 0) continue;
            const float *src = S.part + (int64_t)e * NCH * X::E3 + (ent & 2047u);
#pragma unroll
            for (int c = 0; c < NCH; c++) add[c] += __ldcs(src + c * X::E3);
        }
        const int vx = v & 7, vy = (v >> 3) & 7, vz = v >> 6;
        const int a = S.apron, tl = S.tile;
        const int64_t at = slot * S.tvox + ((int64_t)(kCell * cz + vz + a) * tl + (kCell * cy + vy + a)) * tl +
                           (kCell * cx + vx + a);
#pragma unroll
        for (int c = 0; c < NCH; c++) S.chan[c][at] = overwrite ? add[c] : S.chan[c][at] + add[c];
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
    SplatLimits lim;
};

// The translated position and cloud origin of point pidx, entry j of the
// bin order: from the bin-ordered copy when there is one (contiguous reads
// for a cell's points), else from the caller's view.
__device__ __forceinline__ void gather_point_at(const GatherArgs &G, int32_t pidx, int64_t j, float3 &w, int3 &o) {
    if (G.bin_pos) {
        const float4 q = G.bin_pos[j];
        w = make_float3(q.x, q.y, q.z);
        const int32_t cloud = __float_as_int(q.w);
        o = cloud >= 0 && in_range(G.lim, cloud, G.lim.ncloud, 12)
                ? make_int3(G.pos.origin[3 * cloud], G.pos.origin[3 * cloud + 1], G.pos.origin[3 * cloud + 2])
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
    if (!in_range(G.lim, pidx, G.lim.nentry, 13)) return;
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
    // a binned point's first taps lie in [0, 8]; a point read through the
    // caller's view (bins made by the caller) that has moved since its binning
    // gathers 0 and reads nothing outside
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
    const int32_t leaf = G.slot_leaf[slot];
    // the same for the whole CTA
    if (!in_range(G.lim, (int64_t)end - 1, G.lim.nentry, 14) || !in_range(G.lim, leaf, G.lim.npool, 15)) return;
    const int a = G.apron, tl = G.tile;
    if (threadIdx.x < 27) {
        const int32_t nb = G.nbr27[slot * 27 + threadIdx.x];
        nbs[threadIdx.x] = nb >= 0 && in_range(G.lim, nb, G.lim.nslot, 16) ? nb : -1;
    }
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
    const Node &nd = G.leaves[leaf];
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

// The points of light cells: kLightPack light cells per warp (a light cell
// holds at most the tuning's `light` <= kLightCell = 32 points), one lane
// per point, the group's points dealt to the lanes in rounds of 32; taps
// read straight from the atlas (a staged halo would cost 12^3 floats per
// channel for a few points).  Each point is served by one lane with the
// same taps in the same order whichever warp holds it, so the packing
// changes no result.
constexpr int kLightPack = 4;

template <int KERNEL, int MODE, int NCH>
__device__ __forceinline__ void gather_light_point(const GatherArgs &G, int64_t cell, int64_t entry) {
    constexpr int H = Taps<KERNEL>::N / 2;
    int64_t slot;
    int cx, cy, cz;
    cell_coords(cell, G.m, G.m3, slot, cx, cy, cz);
    const int32_t leaf = G.slot_leaf[slot];
    if (!in_range(G.lim, leaf, G.lim.npool, 19)) return;
    const Node &nd = G.leaves[leaf];
    const int fx0 = kCell * cx - H, fy0 = kCell * cy - H, fz0 = kCell * cz - H; // frame origin in the brick
    const int res = G.res0, a = G.apron, tl = G.tile;
    auto fetch = [&](int x, int y, int z, float g[NCH]) {
        const int lx = fx0 + x, ly = fy0 + y, lz = fz0 + z; // brick-local, may step into a neighbour
        const int sx = lx < 0 ? -1 : (lx >= res ? 1 : 0), sy = ly < 0 ? -1 : (ly >= res ? 1 : 0),
                  sz = lz < 0 ? -1 : (lz >= res ? 1 : 0);
        const int d = (sz + 1) * 9 + (sy + 1) * 3 + (sx + 1);
        int64_t ns = d == 13 ? slot : (int64_t)G.nbr27[slot * 27 + d];
        if (ns >= 0 && !in_range(G.lim, ns, G.lim.nslot, 20)) ns = -1;
        const int64_t off = ns * G.tvox + ((int64_t)(lz - sz * res + a) * tl + (ly - sy * res + a)) * tl +
                            (lx - sx * res + a);
#pragma unroll
        for (int c = 0; c < NCH; c++) g[c] = ns >= 0 ? __ldg(G.chan[c] + off) : 0.0f;
    };
    gather_point<KERNEL, MODE, NCH>(G, G.perm[entry], entry, nd.mPos[0] + fx0, nd.mPos[1] + fy0, nd.mPos[2] + fz0,
                                    fetch);
}

template <int KERNEL, int MODE, int NCH>
__device__ __forceinline__ void gather_light_cells(const GatherArgs &G, int64_t block) {
    const int64_t w = (block * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t nlight = (int64_t)G.cell_cnt[2];
    const int64_t i0 = w * kLightPack;
    if (i0 >= nlight) return; // the same for the whole warp
    // lane j < kLightPack reads light cell i0 + j's bin range
    int64_t cell = -1;
    uint32_t beg = 0, cnt = 0;
    if (lane < kLightPack && i0 + lane < nlight) {
        cell = G.cell_light[i0 + lane];
        if (in_range(G.lim, cell, G.ncell, 17)) {
            beg = G.bin_off[cell];
            cnt = G.bin_off[cell + 1] - beg;
        } else {
            cell = -1;
        }
    }
    uint32_t inc = cnt; // inclusive prefix of the group's counts
#pragma unroll
    for (int o = 1; o < kLightPack; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, inc, kLightPack - 1);
    // rounds of 32 points, the same number for the whole warp (the shuffles
    // below take every lane)
    for (uint32_t r = 0; r < total; r += 32) {
        const uint32_t t = r + lane;
        int j = 0; // the group's cell holding index t
#pragma unroll
        for (int k = 0; k < kLightPack - 1; k++) j += t >= __shfl_sync(0xffffffffu, inc, k) ? 1 : 0;
        j = min(j, kLightPack - 1);
        const int64_t c = __shfl_sync(0xffffffffu, cell, j);
        const uint32_t b = __shfl_sync(0xffffffffu, beg, j);
        const uint32_t first = __shfl_sync(0xffffffffu, inc - cnt, j);
        if (t >= total || c < 0) continue;
        const int64_t entry = (int64_t)b + (t - first);
        if (!in_range(G.lim, entry, G.lim.nentry, 18)) continue;
        gather_light_point<KERNEL, MODE, NCH>(G, c, entry);
    }
}

// Two launches: a halo tile per huge or heavy cell (every cell, in cell
// order, when no cell list is given), then the light cells, kLightPack a warp.
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
    S.lim.flag = splat_guard_word(v);
    S.lim.nslot = v->atlas_last;
    S.lim.npool = v->pool_cnt[0];
    S.lim.nentry = v->bin_key.n;
    S.lim.ncloud = v->batch_clouds;
    v->splat_guard_pending = S.lim.flag != nullptr;
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
    if (!in_range(S.lim, p, S.lim.nentry, 11)) {
        S.bin_amt[j] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const float wt = S.has_weight ? load_f1(S.weight, p) : S.wconst;
    float a4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int c = 0; c < NCH; c++) a4[c] = ((S.attr_mask >> c) & 1) ? wt * load_f1(S.attr[c], p) : wt;
    S.bin_amt[j] = make_float4(a4[0], a4[1], a4[2], a4[3]);
}

// A buffer of `bytes` that starts out zero: zeroed whenever it is
// (re)allocated; its users leave it zero again.
gvdb2_status ensure_zeroed(Volume *v, DevBuf &b, size_t bytes) {
    void *old = b.p;
    GV_CUDA(v, b.ensure(bytes, v->stream));
    if (b.p != old) GV_CUDA(v, cudaMemsetAsync(b.p, 0, b.bytes, v->stream));
    return GVDB2_OK;
}

// Scatter of up to 4 channels (one group): the channel amounts in bin order,
// the dense cells' partial sums (a CTA per slice), then the owner-computes
// pass over every cell of the active bricks (cells no stencil reaches get
// zeros).
template <int KERNEL, int NCH>
gvdb2_status scatter_group(Volume *v, const SplatArgs &S0) {
    using X = ExtTile<KERNEL>;
    constexpr size_t smem = sizeof(ScChunk) * kScWarps;
    auto k = k_scatter_cells<KERNEL, NCH>;
    GV_TRY(launch_smem(v, k, smem, "scatter"));
    GV_CUDA(v, v->bin_amt.ensure(sizeof(float4) * (size_t)std::max<int64_t>(v->bin_key.n, 1), v->stream));
    GV_CUDA(v, v->part_buf.ensure(sizeof(float) * (size_t)std::max<int64_t>(v->dense_cap * NCH * X::E3, 1), v->stream));
    GV_TRY(ensure_zeroed(v, v->part_acc, sizeof(int32_t) * (size_t)std::max<int64_t>(v->multi_cap * 2 * NCH * X::E3, 1)));
    GV_TRY(ensure_zeroed(v, v->part_done, sizeof(uint32_t) * (size_t)std::max<int64_t>(v->multi_cap, 1)));
    GV_CUDA(v, v->merge_list.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(S0.ncell, 1) + 16, v->stream));
    SplatArgs S = S0;
    S.bin_amt = v->bin_amt.as<float4>();
    S.part = v->part_buf.as<float>();
    S.part_acc = v->part_acc.as<int32_t>();
    S.part_done = v->part_done.as<uint32_t>();
    S.dense_cap = v->dense_cap;
    S.multi_cap = v->multi_cap;
    S.slice = (uint32_t)v->tune_slice;
    // the list's count sits in its last 16 bytes
    S.merge_cnt = reinterpret_cast<uint32_t *>(v->merge_list.as<char>() + v->merge_list.bytes - 16);
    S.merge_list = v->merge_list.as<int32_t>();
    GV_CUDA(v, cudaMemsetAsync(S.merge_cnt, 0, sizeof(uint32_t), v->stream));
    if (v->bin_key.n > 0)
        k_pack_amounts<NCH><<<grid_for(v->bin_key.n, 256, 1ll << 31), 256, 0, v->stream>>>(S);
    if (v->work_cap > 0) {
        constexpr size_t ps = part_smem_bytes<KERNEL, NCH>();
        auto kp = k_scatter_part<KERNEL, NCH>;
        GV_TRY(launch_smem(v, kp, ps, "scatter"));
        kp<<<(unsigned)v->work_cap, kPartThreads, ps, v->stream>>>(S);
    }
    const int64_t blocks = (S.ncell + kScWarps - 1) / kScWarps;
    if (blocks > 0) k<<<(unsigned)blocks, 32 * kScWarps, smem, v->stream>>>(S);
    // a cell with a dense cell among its 27 neighbours: at most 27 per dense cell
    const int64_t merge_grid = std::min<int64_t>(S.ncell, 27 * v->dense_cap);
    if (merge_grid > 0) k_scatter_merge<KERNEL, NCH><<<(unsigned)merge_grid, 512, 0, v->stream>>>(S);
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
        k_gather_light<KERNEL, MODE, NCH><<<(unsigned)((v->light_grid + 8 * kLightPack - 1) / (8 * kLightPack)), 256, 0,
                                            v->stream>>>(G);
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
    S.cell_part = v->cell_part.as<int32_t>();
    S.part_work = v->part_work.as<int4>();
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
    G.lim.nentry = n;
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
        S.cell_part = v->cell_part.as<int32_t>();
        S.part_work = v->part_work.as<int4>();
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
