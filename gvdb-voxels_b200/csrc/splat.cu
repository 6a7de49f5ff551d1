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

template <int KERNEL, typename Acc>
__device__ __forceinline__ void acc_add(Acc *a, float v);
template <>
__device__ __forceinline__ void acc_add<GVDB2_KERNEL_TENT1, float>(float *a, float v) { atomicAdd(a, v); }
template <>
__device__ __forceinline__ void acc_add<GVDB2_KERNEL_CUBIC2, float>(float *a, float v) { atomicAdd(a, v); }
template <>
__device__ __forceinline__ void acc_add<GVDB2_KERNEL_TENT1, unsigned long long>(unsigned long long *a, float v) {
    atomicAdd(a, (unsigned long long)__float2ll_rn(v * 4294967296.0f));
}
template <>
__device__ __forceinline__ void acc_add<GVDB2_KERNEL_CUBIC2, unsigned long long>(unsigned long long *a, float v) {
    atomicAdd(a, (unsigned long long)__float2ll_rn(v * 4294967296.0f));
}
__device__ __forceinline__ float acc_value(float a) { return a; }
__device__ __forceinline__ float acc_value(unsigned long long a) {
    return (float)((double)(long long)a * (1.0 / 4294967296.0));
}

// One CTA per atlas slot.  Acc = float (default) or 64-bit fixed point
// (deterministic: integer addition is associative, so the result does not
// depend on the order of the shared-memory atomics).
template <int KERNEL, typename Acc>
__global__ void __launch_bounds__(256) k_scatter_tile(SplatArgs S) {
    using T = Taps<KERNEL>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int res = S.res0, res3 = res * res * res;
    Acc *acc = reinterpret_cast<Acc *>(smem_raw);
    __shared__ uint32_t r_beg[kRangeSlots], r_pre[kRangeSlots + 1];
    __shared__ uint32_t warp_tot[9];
    const int64_t slot = blockIdx.x;

    for (int i = threadIdx.x; i < S.nch * res3; i += blockDim.x) acc[i] = Acc(0);
    // range table + exclusive prefix of range lengths
    uint32_t len = 0;
    if (threadIdx.x < kRangeSlots) {
        uint32_t b, e;
        neighbour_range(S, slot, threadIdx.x, b, e);
        r_beg[threadIdx.x] = b;
        len = e - b;
    }
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        uint32_t x = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[warp] = x;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t run = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
                uint32_t t = warp_tot[w];
                warp_tot[w] = run;
                run += t;
            }
            warp_tot[8] = run;
        }
        __syncthreads();
        if (threadIdx.x < kRangeSlots) r_pre[threadIdx.x] = warp_tot[warp] + x - len;
        if (threadIdx.x == 0) r_pre[kRangeSlots] = warp_tot[8];
        __syncthreads();
    }
    const uint32_t total = r_pre[kRangeSlots];
    const Node &nd = S.leaves[S.slot_leaf[slot]];
    const int ox = nd.mPos[0], oy = nd.mPos[1], oz = nd.mPos[2];

    for (uint32_t j = threadIdx.x; j < total; j += blockDim.x) {
        int lo = 0, hi = kRangeSlots - 1; // last r with r_pre[r] <= j
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (r_pre[mid] <= j) lo = mid;
            else hi = mid - 1;
        }
        int32_t pidx = S.perm[r_beg[lo] + (j - r_pre[lo])];
        float3 p = load_f3(S.pos, pidx);
        float w[3] = {p.x + S.trans.x, p.y + S.trans.y, p.z + S.trans.z};
        float wt = S.has_weight ? load_f1(S.weight, pidx) : S.wconst;
        float amt[kMaxSplatChan];
#pragma unroll
        for (int c = 0; c < kMaxSplatChan; c++)
            if (c < S.nch) amt[c] = ((S.attr_mask >> c) & 1) ? wt * load_f1(S.attr[c], pidx) : wt;
        float wx[T::N], wy[T::N], wz[T::N];
        int fx = T::eval(w[0], wx) - ox, fy = T::eval(w[1], wy) - oy, fz = T::eval(w[2], wz) - oz;
#pragma unroll
        for (int tz = 0; tz < T::N; tz++) {
            int lz = fz + tz;
            if (lz < 0 || lz >= res) continue;
#pragma unroll
            for (int ty = 0; ty < T::N; ty++) {
                int ly = fy + ty;
                if (ly < 0 || ly >= res) continue;
                float wyz = wy[ty] * wz[tz];
                int row = (lz * res + ly) * res;
#pragma unroll
                for (int tx = 0; tx < T::N; tx++) {
                    int lx = fx + tx;
                    if (lx < 0 || lx >= res) continue;
                    float wgt = wx[tx] * wyz;
#pragma unroll
                    for (int c = 0; c < kMaxSplatChan; c++)
                        if (c < S.nch) acc_add<KERNEL, Acc>(&acc[c * res3 + row + lx], amt[c] * wgt);
                }
            }
        }
    }
    __syncthreads();
    const int a = S.apron, tl = S.tile;
    for (int i = threadIdx.x; i < S.nch * res3; i += blockDim.x) {
        int c = i / res3, v = i - c * res3;
        int lx = v % res, ly = (v / res) % res, lz = v / (res * res);
        S.chan[c][slot * S.tvox + ((int64_t)(lz + a) * tl + (ly + a)) * tl + (lx + a)] = acc_value(acc[i]);
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
    int64_t tvox;
};

template <int KERNEL, int MODE>
__global__ void __launch_bounds__(256) k_gather_tile(GatherArgs G) {
    using T = Taps<KERNEL>;
    constexpr int H = T::N / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *tile = reinterpret_cast<float *>(smem_raw);
    const int res = G.res0, ht = res + 2 * H, ht3 = ht * ht * ht;
    const int64_t slot = blockIdx.x;
    const int a = G.apron, tl = G.tile;
    // halo tile from the interiors of this brick and its neighbours
    for (int i = threadIdx.x; i < G.nch * ht3; i += blockDim.x) {
        int c = i / ht3, v = i - c * ht3;
        int lx = v % ht - H, ly = (v / ht) % ht - H, lz = v / (ht * ht) - H;
        int dx = floor_div(lx, res), dy = floor_div(ly, res), dz = floor_div(lz, res);
        int32_t nb = G.nbr27[slot * 27 + (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)];
        float val = 0.0f;
        if (nb >= 0)
            val = G.chan[c][(int64_t)nb * G.tvox +
                            ((int64_t)(lz - dz * res + a) * tl + (ly - dy * res + a)) * tl + (lx - dx * res + a)];
        tile[i] = val;
    }
    __syncthreads();
    const Node &nd = G.leaves[G.slot_leaf[slot]];
    const int ox = nd.mPos[0] - H, oy = nd.mPos[1] - H, oz = nd.mPos[2] - H;
    const uint32_t beg = G.bin_off[slot * 27], end = G.bin_off[slot * 27 + 27];
    for (uint32_t j = beg + threadIdx.x; j < end; j += blockDim.x) {
        int32_t pidx = G.perm[j];
        float3 p = load_f3(G.pos, pidx);
        float w[3] = {p.x + G.trans.x, p.y + G.trans.y, p.z + G.trans.z};
        float wx[T::N], wy[T::N], wz[T::N], dx[T::N], dy[T::N], dz[T::N];
        int fx, fy, fz;
        if (MODE == kFwd) {
            fx = T::eval(w[0], wx) - ox;
            fy = T::eval(w[1], wy) - oy;
            fz = T::eval(w[2], wz) - oz;
        } else {
            fx = T::eval_d(w[0], wx, dx) - ox;
            fy = T::eval_d(w[1], wy, dy) - oy;
            fz = T::eval_d(w[2], wz, dz) - oz;
        }
        float sum[kMaxSplatChan], gx[kMaxSplatChan], gy[kMaxSplatChan], gz[kMaxSplatChan];
#pragma unroll
        for (int c = 0; c < kMaxSplatChan; c++) sum[c] = gx[c] = gy[c] = gz[c] = 0.0f;
#pragma unroll
        for (int tz = 0; tz < T::N; tz++) {
#pragma unroll
            for (int ty = 0; ty < T::N; ty++) {
                int row = ((fz + tz) * ht + (fy + ty)) * ht + fx;
#pragma unroll
                for (int tx = 0; tx < T::N; tx++) {
                    float wyz = wy[ty] * wz[tz];
                    float wgt = wx[tx] * wyz;
#pragma unroll
                    for (int c = 0; c < kMaxSplatChan; c++) {
                        if (c >= G.nch) continue;
                        float g = tile[c * ht3 + row + tx];
                        if (MODE == kFwd || MODE == kScatterBwd) sum[c] += g * wgt;
                        if (MODE != kFwd) {
                            gx[c] += g * (dx[tx] * wyz);
                            gy[c] += g * (wx[tx] * dy[ty] * wz[tz]);
                            gz[c] += g * (wx[tx] * wy[ty] * dz[tz]);
                        }
                    }
                }
            }
        }
        if (MODE == kFwd) {
#pragma unroll
            for (int c = 0; c < kMaxSplatChan; c++)
                if (c < G.nch) G.out[(int64_t)pidx * G.out_stride + c] = sum[c];
        } else if (MODE == kScatterBwd) {
            float wt = G.has_weight ? load_f1(G.weight, pidx) : G.wconst;
            float gw = 0.0f, gp0 = 0.0f, gp1 = 0.0f, gp2 = 0.0f;
#pragma unroll
            for (int c = 0; c < kMaxSplatChan; c++) {
                if (c >= G.nch) continue;
                bool has = (G.attr_mask >> c) & 1;
                float at = has ? load_f1(G.attr[c], pidx) : 1.0f;
                if (G.grad_attr) G.grad_attr[(int64_t)pidx * G.nch + c] = has ? wt * sum[c] : 0.0f;
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
            for (int c = 0; c < kMaxSplatChan; c++) {
                if (c >= G.nch) continue;
                float go = G.grad_out[(int64_t)pidx * G.nch + c];
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

gvdb2_status run_scatter(Volume *v, int kernel, const SplatArgs &S) {
    if (v->atlas_last == 0) return GVDB2_OK;
    const int res3 = v->res(0) * v->res(0) * v->res(0);
    const unsigned g = (unsigned)v->atlas_last;
    cudaStream_t s = v->stream;
    if (v->deterministic) {
        size_t smem = sizeof(unsigned long long) * (size_t)S.nch * res3;
        if (kernel == GVDB2_KERNEL_TENT1) {
            auto k = k_scatter_tile<GVDB2_KERNEL_TENT1, unsigned long long>;
            GV_TRY(launch_smem(v, k, smem, "scatter"));
            k<<<g, 256, smem, s>>>(S);
        } else {
            auto k = k_scatter_tile<GVDB2_KERNEL_CUBIC2, unsigned long long>;
            GV_TRY(launch_smem(v, k, smem, "scatter"));
            k<<<g, 256, smem, s>>>(S);
        }
    } else {
        size_t smem = sizeof(float) * (size_t)S.nch * res3;
        if (kernel == GVDB2_KERNEL_TENT1) {
            auto k = k_scatter_tile<GVDB2_KERNEL_TENT1, float>;
            GV_TRY(launch_smem(v, k, smem, "scatter"));
            k<<<g, 256, smem, s>>>(S);
        } else {
            auto k = k_scatter_tile<GVDB2_KERNEL_CUBIC2, float>;
            GV_TRY(launch_smem(v, k, smem, "scatter"));
            k<<<g, 256, smem, s>>>(S);
        }
    }
    GV_CUDA(v, cudaGetLastError());
    return GVDB2_OK;
}

template <int MODE>
gvdb2_status run_gather(Volume *v, int kernel, const GatherArgs &G) {
    if (v->atlas_last == 0) return GVDB2_OK;
    const int res = v->res(0);
    const int h = kernel == GVDB2_KERNEL_TENT1 ? 1 : 2;
    const int ht = res + 2 * h;
    size_t smem = sizeof(float) * (size_t)G.nch * ht * ht * ht;
    const unsigned g = (unsigned)v->atlas_last;
    if (kernel == GVDB2_KERNEL_TENT1) {
        auto k = k_gather_tile<GVDB2_KERNEL_TENT1, MODE>;
        GV_TRY(launch_smem(v, k, smem, "gather"));
        k<<<g, 256, smem, v->stream>>>(G);
    } else {
        auto k = k_gather_tile<GVDB2_KERNEL_CUBIC2, MODE>;
        GV_TRY(launch_smem(v, k, smem, "gather"));
        k<<<g, 256, smem, v->stream>>>(G);
    }
    GV_CUDA(v, cudaGetLastError());
    return GVDB2_OK;
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
