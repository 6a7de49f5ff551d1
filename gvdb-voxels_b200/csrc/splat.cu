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
    const int32_t *perm;
    int res0, log2r0, apron, tile;
    int m, m3; // cells per brick edge, per brick
    // huge and heavy cells (order of cell_at), light cells, each cell's index
    // in the splat's own order; cell_list == nullptr: every cell, in cell order
    const int32_t *cell_list, *cell_light, *cell_ext;
    const uint32_t *cell_cnt;
    int64_t ncell;
    const int32_t *cell_nbr;      // per cell, the own-order index of its 27 neighbours (-1: none)
    int64_t tvox;
};


// ---- two-phase scatter ---------------------------------------------------
//
// The kernels work on cells, 8^3 blocks of a brick (the brick itself for
// 8^3 bricks).
// Phase 1 (k_scatter_own): one CTA per cell of more than kLightCell points
// (own_light, in the same launch: one warp per lighter cell) splats only the points
// binned to it, with unclipped stencils, into an extended tile
// that covers every tap of those points: [-H, 8+H)^3 with H = N/2 (12^3 for
// the cubic B-spline, 10^3 for the tent).  The tile is then written out as
// float partial sums.
// Phase 2 (k_scatter_merge): one thread per interior voxel of every cell
// adds, in a fixed neighbour order, the partials whose extended tile covers
// the voxel, and writes the channel once.
//
// Accumulation in phase 1 is exact: each contribution x (in units of 2^-s)
// is rounded to an integer and split as rint(x) = hi * 2^L + lo, both parts
// obtained with the float "magic number" rounding (t = x*2^-L + 1.5*2^23
// holds rint(x*2^-L) in its low mantissa bits; the remainder x - hi*2^L is
// exact), and added with native int32 shared-memory atomics.  The integer
// sums do not depend on the order of the atomics, and the merge sums a fixed
// sequence of floats, so the result is bit-reproducible run to run.
// Bounds (R = points of the brick, max|a| = largest |weighted amount| among
// them, so a brick's result depends on its own points only):
//   L = min(22, 31 - bits(R+1))      -> |sum lo| <= R * 2^(L-1) < 2^31
//   max|a| * 2^s < 2^(21+L)          -> |x * 2^-L| < 2^22 (magic range)
//   R * max|a| * 2^s < 2^(29+L)      -> |sum hi| < 2^29 + R/2
template <int KERNEL>
struct ExtTile {
    static constexpr int N = Taps<KERNEL>::N;
    static constexpr int H = N / 2;
    static constexpr int E = 8 + N;                 // 12 (cubic) or 10 (tent)
    static constexpr int RS = E;                    // row stride (words)
    static constexpr int PS = N == 4 ? E * E + 8 : E * E; // plane stride: 152 puts a warp's 32 taps in 32 banks
    static constexpr int CS = E * PS;               // channel stride
    static constexpr int E3 = E * E * E;            // floats per channel in the global partial
    // Position in the global partial of extended-tile voxel (ux, uy, uz) in
    // [0, E)^3.  Per channel the partial holds 27 regions: the cell's 8^3
    // interior first, then the halo beyond each face, edge and corner d in
    // {-1,0,1}^3 (z-major order of d), each z-major with extent 8 along the
    // axes where d is 0 and H where it is not.  The merge so reads whole
    // 32-byte-aligned rows of the interior (8 floats) and packed rows of
    // the halos, instead of 8 floats straddling two sectors of a 12-float
    // row.  Region d starts, in the plain z-major order of the regions, at
    // start_z E^2 + s_z start_y E + s_z s_y start_x, with start and s the
    // region's first extended coordinate and extent along each axis.
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
// The inverse of part_index: the tile address (plane stride PS, row stride
// RS) of each partial position, so that phase 1 writes its partial in order
// (coalesced) and looks each value up in its tile.
template <int KERNEL, int PS, int RS>
struct PartAddr {
    uint16_t addr[ExtTile<KERNEL>::E3];
    constexpr PartAddr() : addr() {
        constexpr int E = ExtTile<KERNEL>::E;
        for (int z = 0; z < E; z++)
            for (int y = 0; y < E; y++)
                for (int x = 0; x < E; x++)
                    addr[ExtTile<KERNEL>::part_index(x, y, z)] = (uint16_t)(z * PS + y * RS + x);
    }
};
// the CTA tile of a heavy cell (padded plane stride) and a light cell's warp tile
template <int KERNEL>
__device__ constexpr PartAddr<KERNEL, ExtTile<KERNEL>::PS, ExtTile<KERNEL>::RS> kHeavyAddr{};
template <int KERNEL>
__device__ constexpr PartAddr<KERNEL, ExtTile<KERNEL>::E * ExtTile<KERNEL>::E, ExtTile<KERNEL>::E> kLightAddr{};

// The merge's sources per interior voxel v (x | y << 3 | z << 6) of a cell:
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

constexpr int kOwnThreads = 256;
constexpr int kOwnChunk = 128; // points staged per pass

template <int KERNEL, int NCH>
constexpr size_t own_smem_bytes() {
    return sizeof(int32_t) * 2 * NCH * ExtTile<KERNEL>::CS +
           sizeof(float) * (3 * Taps<KERNEL>::N + NCH) * kOwnChunk + sizeof(int32_t) * kOwnChunk;
}

// Split step 2^L of the fixed-point sums of R points.
__device__ __forceinline__ int fixed_level(uint32_t R) {
    const int L = 31 - (32 - __clz((int)R + 1));
    return L > 22 ? 22 : L;
}

// Scale 2^sc applied to the contributions of R points whose largest
// |weighted amount| is am (0 when there is nothing to add); inv = 2^-sc.
__device__ __forceinline__ float fixed_scale(uint32_t R, int L, float am, double &inv) {
    int e1 = 0, e2 = 0;
    frexpf(am, &e1);             // am < 2^e1
    frexpf((float)R * am, &e2);  // R*am < 2^e2
    const int sc = min(21 + L - e1, 29 + L - e2);
    const bool on = am > 0.0f && R > 0;
    inv = on ? ldexp(1.0, -sc) : 0.0;
    return on ? ldexpf(1.0f, sc) : 0.0f;
}

__device__ __forceinline__ void fixed_add(int32_t *hi_acc, int32_t *lo_acc, int idx, float x, float inv2L, float two2L) {
    const float M = 12582912.0f; // 1.5 * 2^23
    const float t = fmaf(x, inv2L, M);
    const int hi = __float_as_int(t) - 0x4B400000;
    const float r = fmaf(t - M, -two2L, x);
    const int lo = __float_as_int(r + M) - 0x4B400000;
    atomicAdd(hi_acc + idx, hi);
    atomicAdd(lo_acc + idx, lo);
}

template <int KERNEL, int NCH>
__device__ __forceinline__ void own_heavy(const SplatArgs &S, float *ext, int64_t block) {
    using T = Taps<KERNEL>;
    using X = ExtTile<KERNEL>;
    constexpr int N = T::N;
    extern __shared__ __align__(16) unsigned char own_smem[];
    int32_t *acc_hi = reinterpret_cast<int32_t *>(own_smem);
    int32_t *acc_lo = acc_hi + NCH * X::CS;
    float(*pw)[kOwnChunk] = reinterpret_cast<float(*)[kOwnChunk]>(acc_lo + NCH * X::CS);
    float(*pa)[kOwnChunk] = pw + 3 * N;
    int32_t *pb = reinterpret_cast<int32_t *>(pa + NCH);
    __shared__ double inv_s[NCH];
    __shared__ int32_t amax_bits[NCH]; // max |weighted amount| of the cell's points, as float bits
    // the block-th huge or heavy cell (light cells: own_light); its partial
    // goes to ext[cell_ext[cell]]
    const int64_t cell = cell_at(block, S.cell_list, S.cell_cnt, S.ncell);
    if (cell < 0) return;
    int64_t slot;
    int cx, cy, cz;
    cell_coords(cell, S.m, S.m3, slot, cx, cy, cz);
    static_assert(X::CS % 4 == 0, "16-byte zeroing");
    for (int i = threadIdx.x; i < NCH * X::CS / 2; i += kOwnThreads) // acc_hi and acc_lo, adjacent
        reinterpret_cast<int4 *>(acc_hi)[i] = make_int4(0, 0, 0, 0);
    if (threadIdx.x < NCH) amax_bits[threadIdx.x] = 0;
    const uint32_t beg = S.bin_off[cell], R = S.bin_off[cell + 1] - beg;
    const Node &nd = S.leaves[S.slot_leaf[slot]];
    const int ox = nd.mPos[0] + kCell * cx - X::H, oy = nd.mPos[1] + kCell * cy - X::H,
              oz = nd.mPos[2] + kCell * cz - X::H;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    // Stage one point as record r of the current chunk (amounts times `scale`).
    auto stage = [&](uint32_t j, int r, const float *scale, float *amt_out) {
        const int32_t p = S.perm[beg + j];
        const float3 q = load_f3(S.pos, p);
        const int3 o = point_origin(S.pos, p);
        float wx[N], wy[N], wz[N];
        const int fx = T::eval(q.x + S.trans.x, wx) + o.x - ox;
        const int fy = T::eval(q.y + S.trans.y, wy) + o.y - oy;
        const int fz = T::eval(q.z + S.trans.z, wz) + o.z - oz;
        // a binned point lies in the brick, so its first taps are in [0, 8];
        // anything else (inconsistent input) is dropped, never written outside the tile
        const bool ok = (unsigned)fx <= 8u && (unsigned)fy <= 8u && (unsigned)fz <= 8u;
        pb[r] = ok ? fz * X::PS + fy * X::RS + fx : 0; // tile address of the point's first tap
#pragma unroll
        for (int k = 0; k < N; k++) {
            pw[k][r] = wx[k];
            pw[N + k][r] = wy[k];
            pw[2 * N + k][r] = wz[k];
        }
        const float wt = S.has_weight ? load_f1(S.weight, p) : S.wconst;
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            const float am = ok ? (((S.attr_mask >> c) & 1) ? wt * load_f1(S.attr[c], p) : wt) : 0.0f;
            amt_out[c] = am;
            pa[c][r] = am * scale[c];
        }
    };

    // Pass over all the brick's points: the first chunk is staged unscaled
    // and every amount enters the brick's max, which sets the scale (so the
    // result depends only on this brick's points).
    float one[NCH], mx[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        one[c] = 1.0f;
        mx[c] = 0.0f;
    }
    __syncthreads(); // amax_bits cleared
    for (uint32_t j = threadIdx.x; j < R; j += kOwnThreads) {
        float am[NCH];
        if (j < (uint32_t)kOwnChunk) {
            stage(j, (int)j, one, am);
        } else {
            const int32_t p = S.perm[beg + j];
            const float wt = S.has_weight ? load_f1(S.weight, p) : S.wconst;
#pragma unroll
            for (int c = 0; c < NCH; c++) am[c] = ((S.attr_mask >> c) & 1) ? wt * load_f1(S.attr[c], p) : wt;
        }
#pragma unroll
        for (int c = 0; c < NCH; c++) mx[c] = fmaxf(mx[c], fabsf(am[c]));
    }
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        float x = mx[c];
        for (int o = 16; o > 0; o >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, o));
        if (lane == 0 && x > 0.0f) atomicMax(&amax_bits[c], __float_as_int(x));
    }
    __syncthreads();
    const int L = fixed_level(R);
    const float inv2L = ldexpf(1.0f, -L), two2L = ldexpf(1.0f, L);
    float scale[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        double inv;
        scale[c] = fixed_scale(R, L, __int_as_float(amax_bits[c]), inv);
        if (threadIdx.x == 0) inv_s[c] = inv;
    }
    { // scale the staged first chunk
        const int cnt0 = (int)min((uint32_t)kOwnChunk, R);
        for (int r = threadIdx.x; r < cnt0; r += kOwnThreads)
#pragma unroll
            for (int c = 0; c < NCH; c++) pa[c][r] *= scale[c];
    }
    for (uint32_t base = 0; base < R; base += kOwnChunk) {
        const int cnt = (int)min((uint32_t)kOwnChunk, R - base);
        if (base > 0) {
            __syncthreads(); // previous chunk consumed
            float am[NCH];
            if ((int)threadIdx.x < cnt) stage(base + threadIdx.x, (int)threadIdx.x, scale, am);
        }
        __syncthreads();
        if constexpr (N == 4) {
            // one point per warp step: lane = (tx, ty, z pair); two taps per lane
            const int tx = lane & 3, ty = (lane >> 2) & 3, tz0 = (lane >> 4) * 2;
            const int loff = tz0 * X::PS + ty * X::RS + tx; // this lane's tap from the first tap
            for (int j = warp; j < cnt; j += kOwnThreads / 32) {
                const int a0 = pb[j] + loff;
                const float wxv = pw[tx][j], wyv = pw[N + ty][j];
                const float w0 = wxv * (wyv * pw[2 * N + tz0][j]);
                const float w1 = wxv * (wyv * pw[2 * N + tz0 + 1][j]);
#pragma unroll
                for (int c = 0; c < NCH; c++) {
                    const float am = pa[c][j];
                    fixed_add(acc_hi + c * X::CS, acc_lo + c * X::CS, a0, am * w0, inv2L, two2L);
                    fixed_add(acc_hi + c * X::CS, acc_lo + c * X::CS, a0 + X::PS, am * w1, inv2L, two2L);
                }
            }
        } else {
            // four points per warp step, one tap per lane
            const int sub = lane >> 3, tx = lane & 1, ty = (lane >> 1) & 1, tz = (lane >> 2) & 1;
            const int loff = tz * X::PS + ty * X::RS + tx;
            for (int j0 = warp * 4; j0 < cnt; j0 += kOwnThreads / 8) {
                const int j = j0 + sub;
                if (j >= cnt) continue;
                const int a = pb[j] + loff;
                const float w = pw[tx][j] * (pw[N + ty][j] * pw[2 * N + tz][j]);
#pragma unroll
                for (int c = 0; c < NCH; c++)
                    fixed_add(acc_hi + c * X::CS, acc_lo + c * X::CS, a, pa[c][j] * w, inv2L, two2L);
            }
        }
    }
    __syncthreads();
    // thread t writes partial positions t, t+256, ... (coalesced) of
    // channel c, looking their tile voxel up in kHeavyAddr
    static_assert(kOwnThreads < X::E3, "one channel step per iteration");
    float *dst = ext + (int64_t)S.cell_ext[cell] * NCH * X::E3;
    int c = 0, j = threadIdx.x;
    for (int i = threadIdx.x; i < NCH * X::E3; i += kOwnThreads) {
        const int k = c * X::CS + kHeavyAddr<KERNEL>.addr[j];
        // |sum| < 2^53: exact in double; the power-of-two scaling is exact
        const long long sum = ((long long)acc_hi[k] << L) + (long long)acc_lo[k];
        dst[i] = (float)((double)sum * inv_s[c]);
        j += kOwnThreads;
        if (j >= X::E3) {
            j -= X::E3;
            c++;
        }
    }
}

// Phase 1 for light cells (at most kLightCell = 32 points): one warp per
// cell, so that a CTA-sized tile and its barriers are not spent on a few
// points.  The warp sorts its points by index, stages their taps in shared
// memory (one lane per point), then per channel accumulates them into a
// warp-private float tile in that order -- each point's taps are distinct
// voxels, handled by distinct lanes, so plain adds suffice and every voxel
// sums its contributions in index order: the partial is bit-reproducible --
// and writes the tile out in the partial layout of phase 1.  A partial of
// at most 32 points is accurate to float rounding.
constexpr int kLightWarps = 8;

template <int KERNEL, int NCH>
constexpr size_t own_light_smem_bytes() {
    return sizeof(float) * kLightWarps * (ExtTile<KERNEL>::E3 + 32 * (1 + 3 * Taps<KERNEL>::N + NCH));
}

template <int KERNEL, int NCH>
__device__ __forceinline__ void own_light(const SplatArgs &S, float *ext, int64_t block) {
    using T = Taps<KERNEL>;
    using X = ExtTile<KERNEL>;
    constexpr int N = T::N, E = X::E, E3 = X::E3;
    extern __shared__ __align__(16) unsigned char light_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float *tile = reinterpret_cast<float *>(light_smem) + warp * E3;
    float *stage = reinterpret_cast<float *>(light_smem) + kLightWarps * E3 + warp * 32 * (1 + 3 * N + NCH);
    int32_t *pbase = reinterpret_cast<int32_t *>(stage); // tile address of each point's first tap
    float *pw = stage + 32;                              // pw[k * 32 + j]: weight k (x taps, y taps, z taps)
    float *pa = pw + 3 * N * 32;                         // pa[c * 32 + j]: amount of channel c
    const int64_t w = block * kLightWarps + warp;
    if (w >= (int64_t)S.cell_cnt[2]) return;
    const int64_t cell = S.cell_light[w];
    const uint32_t beg = S.bin_off[cell], cnt = min(S.bin_off[cell + 1] - beg, 32u); // light: <= 32
    // the cell's points in ascending index order (bitonic sort over the warp)
    int32_t key = (uint32_t)lane < cnt ? S.perm[beg + lane] : INT32_MAX;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const int32_t other = __shfl_xor_sync(0xffffffffu, key, j);
            const bool keep_min = ((lane & j) == 0) == ((lane & k) == 0);
            key = keep_min ? min(key, other) : max(key, other);
        }
    int64_t slot;
    int cx, cy, cz;
    cell_coords(cell, S.m, S.m3, slot, cx, cy, cz);
    const Node &nd = S.leaves[S.slot_leaf[slot]];
    const int ox = nd.mPos[0] + kCell * cx - X::H, oy = nd.mPos[1] + kCell * cy - X::H,
              oz = nd.mPos[2] + kCell * cz - X::H;
    if ((uint32_t)lane < cnt) {
        const int32_t p = key;
        const float3 q = load_f3(S.pos, p);
        const int3 o = point_origin(S.pos, p);
        float wx[N], wy[N], wz[N];
        const int fx = T::eval(q.x + S.trans.x, wx) + o.x - ox;
        const int fy = T::eval(q.y + S.trans.y, wy) + o.y - oy;
        const int fz = T::eval(q.z + S.trans.z, wz) + o.z - oz;
        // a binned point's first taps lie in [0, 8]; anything else is dropped
        const bool ok = (unsigned)fx <= 8u && (unsigned)fy <= 8u && (unsigned)fz <= 8u;
        pbase[lane] = ok ? (fz * E + fy) * E + fx : 0; // tile address of the point's first tap
#pragma unroll
        for (int k = 0; k < N; k++) {
            pw[k * 32 + lane] = wx[k];
            pw[(N + k) * 32 + lane] = wy[k];
            pw[(2 * N + k) * 32 + lane] = wz[k];
        }
        const float wt = S.has_weight ? load_f1(S.weight, p) : S.wconst;
#pragma unroll
        for (int c = 0; c < NCH; c++)
            pa[c * 32 + lane] = ok ? (((S.attr_mask >> c) & 1) ? wt * load_f1(S.attr[c], p) : wt) : 0.0f;
    }
    __syncwarp();
    float *dst = ext + (int64_t)S.cell_ext[cell] * NCH * E3;
    // taps of a point per lane: cubic, lane = (tx, ty, z pair) with two taps;
    // tent, lanes 0-7 = (tx, ty, tz)
    const int tx = N == 4 ? (lane & 3) : (lane & 1), ty = N == 4 ? ((lane >> 2) & 3) : ((lane >> 1) & 1);
    const int tz0 = N == 4 ? (lane >> 4) * 2 : ((lane >> 2) & 1);
    const bool tap_lane = N == 4 || lane < 8;
#pragma unroll 1
    for (int c = 0; c < NCH; c++) {
        float4 *t4 = reinterpret_cast<float4 *>(tile);
        for (int i = lane; i < E3 / 4; i += 32) t4[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        __syncwarp();
        for (uint32_t j = 0; j < cnt; j++) {
            if (tap_lane) {
                const int a0 = pbase[j] + (tz0 * E + ty) * E + tx;
                const float am = pa[c * 32 + j];
                const float wxy = pw[tx * 32 + j], wyv = pw[(N + ty) * 32 + j];
                tile[a0] += am * (wxy * (wyv * pw[(2 * N + tz0) * 32 + j]));
                if (N == 4) tile[a0 + E * E] += am * (wxy * (wyv * pw[(2 * N + tz0 + 1) * 32 + j]));
            }
            __syncwarp();
        }
        float *dc = dst + c * E3;
        for (int i = lane; i < E3; i += 32) dc[i] = tile[kLightAddr<KERNEL>.addr[i]];
        __syncwarp();
    }
}

// Phase 1 in one launch: blocks [0, heavy_blocks) take a huge or heavy cell
// each, the rest kLightWarps light cells each (kOwnThreads = 32 *
// kLightWarps), so the light cells run beside the heavy ones.
static_assert(kOwnThreads == 32 * kLightWarps, "one block size for both kinds of cell");
template <int KERNEL, int NCH>
__global__ void __launch_bounds__(kOwnThreads) k_scatter_own(SplatArgs S, float *ext, int64_t heavy_blocks) {
    if ((int64_t)blockIdx.x < heavy_blocks) own_heavy<KERNEL, NCH>(S, ext, blockIdx.x);
    else own_light<KERNEL, NCH>(S, ext, blockIdx.x - heavy_blocks);
}

// Phase 2 (k_scatter_merge / k_scatter_merge_cta): voxel v of a cell sums,
// in a fixed order, the partials of the cells whose extended tile covers
// it: its own cell and, within H of a face, the neighbours across it (per
// axis d = 0 and e = -1 or +1, never both, H <= 4), looked up in the cell's
// 27-entry neighbour table.  The up to 8 partials are read first
// (predicated), then summed, and the channel is written once.
template <int KERNEL, int NCH>
__device__ __forceinline__ void merge_voxel(const SplatArgs &S, const float *ext, const int32_t *ne, int64_t cell,
                                            int v) {
    using X = ExtTile<KERNEL>;
    const int vx = v & 7, vy = (v >> 3) & 7, vz = v >> 6;
    const uint4 row = *reinterpret_cast<const uint4 *>(kMergeMap<KERNEL>.src[v]);
    const uint32_t w[4] = {row.x, row.y, row.z, row.w};
    float part[8][NCH];
#pragma unroll
    for (int m = 0; m < 8; m++) {
        const uint32_t ent = (w[m >> 1] >> (16 * (m & 1))) & 0xFFFFu;
        const int32_t e = ent != 0xFFFFu ? ne[ent >> 11] : -1;
        const float *src = ext + (int64_t)(e >= 0 ? e : 0) * NCH * X::E3 + (ent & 2047u);
#pragma unroll
        for (int c = 0; c < NCH; c++) part[m][c] = e >= 0 ? __ldcs(src + c * X::E3) : 0.0f;
    }
    float acc[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) acc[c] = 0.0f;
#pragma unroll
    for (int m = 0; m < 8; m++)
#pragma unroll
        for (int c = 0; c < NCH; c++) acc[c] += part[m][c];
    int64_t slot;
    int cx, cy, cz;
    cell_coords(cell, S.m, S.m3, slot, cx, cy, cz);
    const int a = S.apron, tl = S.tile;
    const int Lx = kCell * cx + vx, Ly = kCell * cy + vy, Lz = kCell * cz + vz; // voxel in the brick
    const int64_t at = slot * S.tvox + ((int64_t)(Lz + a) * tl + (Ly + a)) * tl + (Lx + a);
#pragma unroll
    for (int c = 0; c < NCH; c++)
        if (c < S.nch) S.chan[c][at] = acc[c];
}

// Thread per voxel (sparse volumes): no shared memory or barrier, as many
// voxels in flight as the registers allow; the neighbour row is read
// through L1.
template <int KERNEL, int NCH>
__global__ void __launch_bounds__(256) k_scatter_merge(SplatArgs S, const float *ext) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t cell = i >> 9;
    if (cell >= S.ncell) return;
    merge_voxel<KERNEL, NCH>(S, ext, S.cell_nbr + cell * 27, cell, (int)(i & 511));
}

// CTA per cell (dense volumes, where nearly every cell has partials): the
// neighbour row staged once in shared memory.
template <int KERNEL, int NCH>
__global__ void __launch_bounds__(512) k_scatter_merge_cta(SplatArgs S, const float *ext) {
    __shared__ int32_t ne[27];
    const int64_t cell = blockIdx.x;
    if (threadIdx.x < 27) ne[threadIdx.x] = S.cell_nbr[cell * 27 + threadIdx.x];
    __syncthreads();
    merge_voxel<KERNEL, NCH>(S, ext, ne, cell, threadIdx.x);
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
    // huge and heavy cells (order of cell_at), light cells, each cell's index
    // in the splat's own order; cell_list == nullptr: every cell, in cell order
    const int32_t *cell_list, *cell_light, *cell_ext;
    const uint32_t *cell_cnt;
    int64_t ncell;
    const int32_t *cell_nbr; // (not used by the gathers)
    int64_t tvox;
};

// One point of a gather, in any mode.  fetch(x, y, z, g) gives g[c], the
// value of channel c at tap (x, y, z) of the cell's extended frame, whose
// origin (ox, oy, oz) is the cell's first voxel minus H.
template <int KERNEL, int MODE, int NCH, class Fetch>
__device__ __forceinline__ void gather_point(const GatherArgs &G, int32_t pidx, int ox, int oy, int oz,
                                             const Fetch &fetch) {
    using T = Taps<KERNEL>;
    constexpr int N = T::N;
    const float3 p = load_f3(G.pos, pidx);
    const int3 o = point_origin(G.pos, pidx);
    float wx[N], wy[N], wz[N], dx[N], dy[N], dz[N];
    int fx, fy, fz;
    if (MODE == kFwd) {
        fx = T::eval(p.x + G.trans.x, wx) + o.x - ox;
        fy = T::eval(p.y + G.trans.y, wy) + o.y - oy;
        fz = T::eval(p.z + G.trans.z, wz) + o.z - oz;
    } else {
        fx = T::eval_d(p.x + G.trans.x, wx, dx) + o.x - ox;
        fy = T::eval_d(p.y + G.trans.y, wy, dy) + o.y - oy;
        fz = T::eval_d(p.z + G.trans.z, wz, dz) + o.z - oz;
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

template <int KERNEL, int MODE, int NCH>
__device__ __forceinline__ void gather_tile_cell(const GatherArgs &G, int64_t block) {
    constexpr int H = Taps<KERNEL>::N / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *tile = reinterpret_cast<float *>(smem_raw);
    __shared__ int32_t nbs[27];
    // one CTA per 8^3 cell of a brick: the cell plus its halo is staged
    constexpr int ht = kCell + 2 * H, ht3 = ht * ht * ht;
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
    // halo tile from the interiors of this brick and its neighbours: one
    // tile row (fixed y, z) per half-warp, lane l < ht loading x = l; the
    // lane's x neighbour and x offset are fixed for the whole tile
    static_assert(ht <= 16, "a tile row fits a half-warp");
    constexpr int rows_per_pass = kGatherThreads / 16, passes = (ht * ht + rows_per_pass - 1) / rows_per_pass;
    const int hl = threadIdx.x & 15;
    const int lx = hl - H + kCell * cx;
    const int ex = lx < 0 ? -1 : (lx >= res ? 1 : 0);
    const int xo = lx - ex * res + a;
    // row r's brick (-1: outside the volume or no row) and offset of its voxel hl
    auto row_src = [&](int r, int64_t &off) -> int32_t {
        const bool in = hl < ht && r < ht * ht;
        const int ly = r % ht - H + kCell * cy, lz = r / ht - H + kCell * cz;
        const int dy = ly < 0 ? -1 : (ly >= res ? 1 : 0), dz = lz < 0 ? -1 : (lz >= res ? 1 : 0);
        const int32_t nb = in ? nbs[(dz + 1) * 9 + (dy + 1) * 3 + (ex + 1)] : -1;
        off = (int64_t)nb * G.tvox + ((lz - dz * res + a) * tl + (ly - dy * res + a)) * tl + xo;
        return nb;
    };
    if constexpr (MODE == kFwd) {
        // row by row: the forward point phase needs few registers, and
        // holding the whole staging in registers would cut the CTAs per SM
        for (int r = threadIdx.x >> 4; r < ht * ht; r += rows_per_pass) {
            int64_t off;
            const int32_t nb = row_src(r, off);
            if (hl < ht)
#pragma unroll
                for (int c = 0; c < NCH; c++) tile[c * ht3 + r * ht + hl] = nb >= 0 ? __ldg(G.chan[c] + off) : 0.0f;
        }
    } else {
        // the adjoint point phases hold more registers than the staging
        // needs: every load of the thread is issued before the first store
        float val[passes][NCH];
#pragma unroll
        for (int k = 0; k < passes; k++) {
            int64_t off;
            const int32_t nb = row_src((int)(threadIdx.x >> 4) + k * rows_per_pass, off);
#pragma unroll
            for (int c = 0; c < NCH; c++) val[k][c] = nb >= 0 ? __ldg(G.chan[c] + off) : 0.0f;
        }
#pragma unroll
        for (int k = 0; k < passes; k++) {
            const int r = (int)(threadIdx.x >> 4) + k * rows_per_pass;
            if (hl < ht && r < ht * ht)
#pragma unroll
                for (int c = 0; c < NCH; c++) tile[c * ht3 + r * ht + hl] = val[k][c];
        }
    }
    __syncthreads();
    const Node &nd = G.leaves[G.slot_leaf[slot]];
    const int ox = nd.mPos[0] + kCell * cx - H, oy = nd.mPos[1] + kCell * cy - H, oz = nd.mPos[2] + kCell * cz - H;
    auto fetch = [&](int x, int y, int z, float g[NCH]) {
        const int k = (z * ht + y) * ht + x;
#pragma unroll
        for (int c = 0; c < NCH; c++) g[c] = tile[c * ht3 + k];
    };
    for (uint32_t j = beg + threadIdx.x; j < end; j += kGatherThreads)
        gather_point<KERNEL, MODE, NCH>(G, G.perm[j], ox, oy, oz, fetch);
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
    gather_point<KERNEL, MODE, NCH>(G, G.perm[beg + lane], nd.mPos[0] + fx0, nd.mPos[1] + fy0, nd.mPos[2] + fz0,
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
    S.cell_nbr = v->cell_nbr.as<int32_t>();
    S.cell_light = v->cell_light.as<int32_t>();
    S.cell_ext = v->cell_ext.as<int32_t>();
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

// Two-phase scatter of up to 4 channels (one group).
template <int KERNEL, int NCH>
gvdb2_status scatter_group(Volume *v, const SplatArgs &S) {
    using X = ExtTile<KERNEL>;
    cudaStream_t s = v->stream;
    // one partial per cell that holds points (at most cell_grid of them)
    const int64_t nown = v->cell_grid;
    GV_CUDA(v, v->scratch.ensure(sizeof(float) * (size_t)nown * NCH * X::E3 + 256, s));
    float *ext = v->scratch.as<float>();
    constexpr size_t smem = std::max(own_smem_bytes<KERNEL, NCH>(), own_light_smem_bytes<KERNEL, NCH>());
    auto k1 = k_scatter_own<KERNEL, NCH>;
    GV_TRY(launch_smem(v, k1, smem, "scatter"));
    const int64_t own_blocks = v->heavy_grid + (v->light_grid + kLightWarps - 1) / kLightWarps;
    if (own_blocks > 0) k1<<<(unsigned)own_blocks, kOwnThreads, smem, s>>>(S, ext, v->heavy_grid);
    if (4 * nown >= 3 * S.ncell) // dense: most cells hold points
        k_scatter_merge_cta<KERNEL, NCH><<<(unsigned)S.ncell, 512, 0, s>>>(S, ext);
    else
        k_scatter_merge<KERNEL, NCH><<<(unsigned)(S.ncell * 2), 256, 0, s>>>(S, ext);
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
gvdb2_status scatter_two_phase(Volume *v, const SplatArgs &S) {
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
    return kernel == GVDB2_KERNEL_TENT1 ? scatter_two_phase<GVDB2_KERNEL_TENT1>(v, S)
                                        : scatter_two_phase<GVDB2_KERNEL_CUBIC2>(v, S);
}

template <int KERNEL, int MODE, int NCH>
gvdb2_status launch_gather(Volume *v, const GatherArgs &G) {
    constexpr int H = Taps<KERNEL>::N / 2;
    constexpr int ht = kCell + 2 * H;
    const size_t smem = sizeof(float) * (size_t)NCH * ht * ht * ht;
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
