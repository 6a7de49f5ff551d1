// nanovdb.cu -- NanoVDB-form export of a volume (ExportToNanoVDB,
// gNanoVDB/gvdb_export_nanovdb.cpp:379-700 with the device passes of
// gNanoVDB/cuda_export_nanovdb.cu:76-432).
//
// One device buffer, sections in NanoVDB's order: grid header (grid, tree
// and root fields), root tiles, level-2 nodes, level-1 nodes, leaves.  Record
// layouts are gvdb2_nv_grid / gvdb2_nv_tile / gvdb2_nv_node / gvdb2_nv_leaf
// (include/gvdb2.h).
//
// B200 form: a CTA per leaf stages its atlas tile in shared memory -- whole,
// by bulk copies (cp.async.bulk, mbarrier-completed) when the tiles fit, else
// in slabs of x-planes read in the tile's x-fastest rows -- and writes the
// record's z-fastest values as contiguous runs; min/max reduce in registers,
// then by warp shuffles.  A CTA per interior node walks the child
// table in NanoVDB order, builds the child mask with warp ballots and folds
// the children's ranges.  Every byte of every record is written by the
// kernels (no memset pass over the buffer).  The root is finished on the host
// from the level-2 headers, as the reference finishes it.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "dev_common.cuh"
#include "gvdb2_internal.h"

namespace gvdb2 {
namespace {

constexpr int kNvThreads = 256;
constexpr size_t kNvSlabBytes = 64 * 1024; // shared memory a leaf CTA stages per slab

static_assert(sizeof(gvdb2_nv_grid) == 608, "grid header is 608 bytes");
static_assert(sizeof(gvdb2_nv_node) == GVDB2_NV_HEADER, "node header");
static_assert(sizeof(gvdb2_nv_leaf) == GVDB2_NV_HEADER, "leaf header");
static_assert(sizeof(gvdb2_nv_tile) == 16, "tile");

uint64_t round32(uint64_t x) { return (x + 31) & ~uint64_t(31); }
uint64_t leaf_record(int ld, int nv) {
    const uint64_t t3 = uint64_t(1) << (3 * ld);
    return round32(GVDB2_NV_HEADER + t3 / 8 + t3 * 4 * (uint64_t)nv);
}
uint64_t node_record(int ld, int nv) {
    const uint64_t t3 = uint64_t(1) << (3 * ld);
    return round32(GVDB2_NV_HEADER + t3 / 4 + t3 * 4 * (uint64_t)nv);
}

struct NvLayout {
    int ld[3] = {0, 0, 0};
    int64_t cnt[3] = {0, 0, 0};
    uint64_t rec[3] = {0, 0, 0};
    uint64_t sec[4] = {0, 0, 0, 0}; // leaves, level-1, level-2, tiles
    uint64_t total = 0;
};

gvdb2_status nv_layout(Volume *v, int nv, NvLayout &L) {
    if (nv != GVDB2_NV_FLOAT && nv != GVDB2_NV_VEC3F) return fail(v, GVDB2_ERR_ARG, "value type must be float or vec3f");
    if (v->nlev < 3) return fail(v, GVDB2_ERR_UNSUPPORTED, "NanoVDB export needs at least three levels");
    for (int l = 0; l < 3; l++) {
        // the reference's tables cover log2 dims 2..7 (gvdb_export_nanovdb.cpp:64-71)
        if (v->logdim[l] < 2 || v->logdim[l] > 7) return fail(v, GVDB2_ERR_UNSUPPORTED, "log2 dims of levels 0-2 must lie in [2, 7]");
        L.ld[l] = v->logdim[l];
        L.cnt[l] = v->pool_cnt[l];
        if (L.cnt[l] > INT_MAX) return fail(v, GVDB2_ERR_CAPACITY, "more than INT_MAX nodes on a level");
    }
    L.rec[0] = leaf_record(L.ld[0], nv);
    L.rec[1] = node_record(L.ld[1], nv);
    L.rec[2] = node_record(L.ld[2], nv);
    L.sec[3] = sizeof(gvdb2_nv_grid);
    L.sec[2] = round32(L.sec[3] + sizeof(gvdb2_nv_tile) * (uint64_t)L.cnt[2]);
    L.sec[1] = L.sec[2] + L.rec[2] * (uint64_t)L.cnt[2];
    L.sec[0] = L.sec[1] + L.rec[1] * (uint64_t)L.cnt[1];
    L.total = L.sec[0] + L.rec[0] * (uint64_t)L.cnt[0];
    return GVDB2_OK;
}

struct NvChans {
    const float *c[3];
};

__device__ __forceinline__ void zero_record(uint8_t *rp, uint64_t rec) {
    uint4 *q = reinterpret_cast<uint4 *>(rp);
    for (uint64_t i = threadIdx.x; i < rec / 16; i += blockDim.x) q[i] = make_uint4(0, 0, 0, 0);
}

// Block-wide min/max of NV lanes' values; the result is valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_minmax(float (&lo)[NV], float (&hi)[NV]) {
    __shared__ float red[2 * NV][kNvThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < NV; c++)
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            lo[c] = fminf(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
            hi[c] = fmaxf(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
        }
    if (lane == 0)
#pragma unroll
        for (int c = 0; c < NV; c++) red[c][warp] = lo[c], red[NV + c][warp] = hi[c];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int w = 1; w < kNvThreads / 32; w++)
#pragma unroll
            for (int c = 0; c < NV; c++) lo[c] = fminf(lo[c], red[c][w]), hi[c] = fmaxf(hi[c], red[NV + c][w]);
}

// ProcessLeaf (cuda_export_nanovdb.cu:76-129): one CTA per pool leaf.  The
// brick is read from the leaf's atlas tile (interior at +apron, x fastest)
// and written as values[(x*T + y)*T + z]; min/max start at +-FLT_MAX as the
// reference's do.  Slab s of `slab` x-planes is the record's contiguous run
// [s*slab*T^2, (s+1)*slab*T^2).  Shared memory holds the slab as
// [x][y*T + z] with a row pitch of T^2 + 1 words, so both the staging stores
// (x fastest) and the output reads (z fastest) are free of bank conflicts.
template <int NV>
__global__ void __launch_bounds__(kNvThreads) k_nv_leaves(const Node *leaves, const int32_t *leaf_slot, int64_t nslots,
                                                          NvChans ch, int ld, int apron, int lslab, uint8_t *out,
                                                          uint64_t rec) {
    extern __shared__ float sm[];
    const int64_t leaf = blockIdx.x;
    uint8_t *rp = out + (uint64_t)leaf * rec;
    const int slot = leaf_slot[leaf];
    if (slot < 0 || slot >= nslots) { // stale: no brick in the atlas
        zero_record(rp, rec);
        return;
    }
    const int T = 1 << ld, T2 = T * T, t = T + 2 * apron, slab = 1 << lslab;
    const int pitch = T2 + 1;
    const int64_t t3 = (int64_t)T2 * T;
    const int64_t base = (int64_t)slot * t * t * t;
    uint64_t *mask = reinterpret_cast<uint64_t *>(rp + GVDB2_NV_HEADER);
    float *vals = reinterpret_cast<float *>(rp + GVDB2_NV_HEADER + t3 / 8);
    for (int64_t w = threadIdx.x; w < t3 / 64; w += blockDim.x) mask[w] = ~uint64_t(0); // all voxels active
    float lo[NV], hi[NV];
#pragma unroll
    for (int c = 0; c < NV; c++) lo[c] = FLT_MAX, hi[c] = -FLT_MAX;
    const int n = slab * T2;
    for (int x0 = 0; x0 < T; x0 += slab) {
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const int xl = j & (slab - 1), r = j >> lslab;
            const int y = r & (T - 1), z = r >> ld;
            const int64_t a = base + ((int64_t)(z + apron) * t + (y + apron)) * t + (x0 + xl + apron);
#pragma unroll
            for (int c = 0; c < NV; c++) sm[c * slab * pitch + xl * pitch + y * T + z] = ch.c[c][a];
        }
        __syncthreads();
        float *dst = vals + (int64_t)x0 * T2 * NV;
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const int xl = j >> (2 * ld), r = j & (T2 - 1);
#pragma unroll
            for (int c = 0; c < NV; c++) {
                const float val = sm[c * slab * pitch + xl * pitch + r];
                dst[(int64_t)j * NV + c] = val;
                lo[c] = fminf(lo[c], val);
                hi[c] = fmaxf(hi[c], val);
            }
        }
        __syncthreads();
    }
    // the padding after the values
    const uint64_t used = GVDB2_NV_HEADER + t3 / 8 + t3 * 4 * NV;
    for (uint64_t b = used + threadIdx.x * 4; b < rec; b += blockDim.x * 4) *reinterpret_cast<uint32_t *>(rp + b) = 0;
    block_minmax<NV>(lo, hi);
    if (threadIdx.x == 0) {
        const Node &nd = leaves[leaf];
        gvdb2_nv_leaf h;
        memset(&h, 0, sizeof(h));
        for (int a = 0; a < 3; a++) h.bbox_min[a] = nd.mPos[a], h.bbox_dif[a] = (uint8_t)T;
        for (int c = 0; c < NV; c++) h.vmin[c] = lo[c], h.vmax[c] = hi[c];
        *reinterpret_cast<gvdb2_nv_leaf *>(rp) = h;
    }
}

// Bulk copies: one cp.async.bulk per channel moves a leaf's whole atlas tile
// (a contiguous, 16-byte-aligned run of t^3 floats) into shared memory,
// completing on an mbarrier.  The wait is bounded: past kNvWaitLimit polls
// the CTA sets kDevTimeout in *status, waits once more (bounded) so that no
// copy still lands in its shared memory, and returns without using the data.
constexpr int kNvWaitLimit = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase, int limit) {
    for (int i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(bar), "r"(phase)
                     : "memory");
        if (done) return true;
    }
    return false;
}

// ProcessLeaf with the tile staged by bulk copies (bricks whose NV tiles fit
// kNvSlabBytes): the same record as k_nv_leaves, read from shared memory.
template <int NV>
__global__ void __launch_bounds__(kNvThreads) k_nv_leaves_bulk(const Node *leaves, const int32_t *leaf_slot,
                                                               int64_t nslots, NvChans ch, int ld, int apron,
                                                               uint8_t *out, uint64_t rec, int32_t *status) {
    extern __shared__ __align__(16) float tile[];
    __shared__ __align__(8) uint64_t bar;
    const int64_t leaf = blockIdx.x;
    uint8_t *rp = out + (uint64_t)leaf * rec;
    const int slot = leaf_slot[leaf];
    if (slot < 0 || slot >= nslots) { // stale: no brick in the atlas
        zero_record(rp, rec);
        return;
    }
    const int T = 1 << ld, T2 = T * T, t = T + 2 * apron;
    const int64_t t3 = (int64_t)T2 * T;
    const uint32_t tbytes = (uint32_t)t * t * t * 4u; // a multiple of 32 (t is even)
    const uint32_t b = smem_u32(&bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(tbytes * NV) : "memory");
#pragma unroll
        for (int c = 0; c < NV; c++) {
            const float *src = ch.c[c] + (int64_t)slot * t * t * t;
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             smem_u32(tile + (size_t)c * t * t * t)),
                         "l"(src), "r"(tbytes), "r"(b)
                         : "memory");
        }
    }
    if (!mbar_wait(b, 0, kNvWaitLimit)) {
        if (threadIdx.x == 0) atomicOr(status, kDevTimeout);
        mbar_wait(b, 0, kNvWaitLimit);
        return;
    }
    uint64_t *mask = reinterpret_cast<uint64_t *>(rp + GVDB2_NV_HEADER);
    float *vals = reinterpret_cast<float *>(rp + GVDB2_NV_HEADER + t3 / 8);
    for (int64_t w = threadIdx.x; w < t3 / 64; w += blockDim.x) mask[w] = ~uint64_t(0); // all voxels active
    float lo[NV], hi[NV];
#pragma unroll
    for (int c = 0; c < NV; c++) lo[c] = FLT_MAX, hi[c] = -FLT_MAX;
    // values[(x*T + y)*T + z] from tile voxel (x, y, z) + apron, z-major
    for (int j = threadIdx.x; j < (int)t3; j += blockDim.x) {
        const int x = j >> (2 * ld), y = (j >> ld) & (T - 1), z = j & (T - 1);
        const int s = ((z + apron) * t + (y + apron)) * t + (x + apron);
#pragma unroll
        for (int c = 0; c < NV; c++) {
            const float val = tile[c * t * t * t + s];
            vals[(int64_t)j * NV + c] = val;
            lo[c] = fminf(lo[c], val);
            hi[c] = fmaxf(hi[c], val);
        }
    }
    const uint64_t used = GVDB2_NV_HEADER + t3 / 8 + t3 * 4 * NV;
    for (uint64_t p = used + threadIdx.x * 4; p < rec; p += blockDim.x * 4) *reinterpret_cast<uint32_t *>(rp + p) = 0;
    block_minmax<NV>(lo, hi);
    if (threadIdx.x == 0) {
        const Node &nd = leaves[leaf];
        gvdb2_nv_leaf h;
        memset(&h, 0, sizeof(h));
        for (int a = 0; a < 3; a++) h.bbox_min[a] = nd.mPos[a], h.bbox_dif[a] = (uint8_t)T;
        for (int c = 0; c < NV; c++) h.vmin[c] = lo[c], h.vmax[c] = hi[c];
        *reinterpret_cast<gvdb2_nv_leaf *>(rp) = h;
    }
}

// ProcessInternalNode (cuda_export_nanovdb.cu:241-328): one CTA per pool node
// of a level.  Table slot j = (x*T + y)*T + z holds GVDB child-list entry
// g = (z*T + y)*T + x; an entry's child index is (int)(entry >> 16), -1 for
// an empty slot (getChild, cuda_gvdb_nodes.cuh:115-124).  A child index past
// the child level's pool, or a list past the child-list storage, sets
// `status` and is skipped (never read).
template <int NV>
__global__ void __launch_bounds__(kNvThreads) k_nv_nodes(const Node *nodes, const uint64_t *clist, int ld,
                                                         const uint8_t *child_base, uint64_t child_rec,
                                                         int64_t nchild, int child_is_leaf, float3 bg, int32_t nlevel,
                                                         uint64_t nlists, uint8_t *out, uint64_t rec, int32_t *status) {
    const int64_t idx = blockIdx.x;
    uint8_t *rp = out + (uint64_t)idx * rec;
    const Node &nd = nodes[idx];
    if (nd.mChildList == kUndefL) { // no child list: every field 0 (cuda_export_nanovdb.cu:355-359)
        zero_record(rp, rec);
        return;
    }
    const int T = 1 << ld;
    const int64_t t3 = (int64_t)T * T * T;
    if ((nd.mChildList >> 16) >= nlists) { // a list past the level's child-list storage
        if (threadIdx.x == 0) atomicOr(status, kDevBadIndex);
        zero_record(rp, rec);
        return;
    }
    const uint64_t *list = clist + (nd.mChildList >> 16) * (uint64_t)t3;
    uint64_t *vmask = reinterpret_cast<uint64_t *>(rp + GVDB2_NV_HEADER);
    uint32_t *cmask = reinterpret_cast<uint32_t *>(vmask + t3 / 64);
    float *table = reinterpret_cast<float *>(cmask + t3 / 32);
    const float bgv[3] = {bg.x, bg.y, bg.z};
    float lo[NV], hi[NV];
#pragma unroll
    for (int c = 0; c < NV; c++) lo[c] = FLT_MAX, hi[c] = -FLT_MAX;
    int bl[3] = {INT_MAX, INT_MAX, INT_MAX}, bh[3] = {-INT_MAX, -INT_MAX, -INT_MAX};
    for (int64_t w = threadIdx.x; w < t3 / 64; w += blockDim.x) vmask[w] = 0; // no tile values
    // t3 >= 64 is a multiple of 32, so every warp runs whole iterations
    for (int64_t j = threadIdx.x; j < t3; j += blockDim.x) {
        const int x = (int)(j >> (2 * ld)), y = (int)(j >> ld) & (T - 1), z = (int)j & (T - 1);
        const int64_t g = ((int64_t)z * T + y) * T + x;
        const int c = (int)(list[g] >> 16);
        bool has = c != -1;
        if (has && (c < 0 || c >= nchild)) {
            atomicOr(status, kDevBadIndex);
            has = false;
        }
        const unsigned b = __ballot_sync(0xffffffffu, has);
        if ((threadIdx.x & 31) == 0) cmask[j >> 5] = b;
        float *e = table + j * NV;
        if (has) {
            reinterpret_cast<uint32_t *>(e)[0] = (uint32_t)c;
#pragma unroll
            for (int k = 1; k < NV; k++) e[k] = 0.0f;
            const uint8_t *cp = child_base + (uint64_t)c * child_rec;
            int cl[3], chh[3];
            const float *cv;
            if (child_is_leaf) { // LeafNode::bbox(): corner .. corner + stored extent
                const gvdb2_nv_leaf &lf = *reinterpret_cast<const gvdb2_nv_leaf *>(cp);
                for (int a = 0; a < 3; a++) cl[a] = lf.bbox_min[a], chh[a] = lf.bbox_min[a] + lf.bbox_dif[a];
                cv = lf.vmin;
            } else {
                const gvdb2_nv_node &in = *reinterpret_cast<const gvdb2_nv_node *>(cp);
                for (int a = 0; a < 3; a++) cl[a] = in.bbox_min[a], chh[a] = in.bbox_max[a];
                cv = in.vmin;
            }
#pragma unroll
            for (int k = 0; k < NV; k++) lo[k] = fminf(lo[k], cv[k]), hi[k] = fmaxf(hi[k], cv[3 + k]);
            for (int a = 0; a < 3; a++) bl[a] = min(bl[a], cl[a]), bh[a] = max(bh[a], chh[a]);
        } else {
#pragma unroll
            for (int k = 0; k < NV; k++) e[k] = bgv[k];
        }
    }
    const uint64_t used = GVDB2_NV_HEADER + (uint64_t)t3 / 4 + (uint64_t)t3 * 4 * NV;
    for (uint64_t b = used + threadIdx.x * 4; b < rec; b += blockDim.x * 4) *reinterpret_cast<uint32_t *>(rp + b) = 0;
    // box: reduce by warp shuffles, then across warps in shared memory
    __shared__ int bred[6][kNvThreads / 32];
    for (int a = 0; a < 3; a++)
        for (int o = 16; o; o >>= 1) {
            bl[a] = min(bl[a], __shfl_xor_sync(0xffffffffu, bl[a], o));
            bh[a] = max(bh[a], __shfl_xor_sync(0xffffffffu, bh[a], o));
        }
    if ((threadIdx.x & 31) == 0)
        for (int a = 0; a < 3; a++) bred[a][threadIdx.x >> 5] = bl[a], bred[3 + a][threadIdx.x >> 5] = bh[a];
    block_minmax<NV>(lo, hi); // its __syncthreads also orders bred
    if (threadIdx.x == 0) {
        for (int w = 1; w < kNvThreads / 32; w++)
            for (int a = 0; a < 3; a++) bl[a] = min(bl[a], bred[a][w]), bh[a] = max(bh[a], bred[3 + a][w]);
        gvdb2_nv_node h;
        memset(&h, 0, sizeof(h));
        for (int a = 0; a < 3; a++) h.bbox_min[a] = bl[a], h.bbox_max[a] = bh[a];
        h.offset = (uint32_t)(nlevel - idx); // nodes of the level - index (cuda_export_nanovdb.cu:263-266)
        for (int c = 0; c < NV; c++) h.vmin[c] = lo[c], h.vmax[c] = hi[c];
        *reinterpret_cast<gvdb2_nv_node *>(rp) = h;
    }
}

template <int NV>
gvdb2_status launch_nv(Volume *v, const NvLayout &L, const int32_t *chans, float3 bg, uint8_t *dst, int32_t *status) {
    cudaStream_t s = v->stream;
    const int T = 1 << L.ld[0];
    const int tr = T + 2 * v->apron;
    const size_t tile_all = (size_t)tr * tr * tr * 4 * NV;
    bool aligned = true;
    for (int c = 0; c < NV; c++) aligned &= reinterpret_cast<uintptr_t>(v->atlas[chans[c]].p) % 16 == 0;
    if (L.cnt[0] > 0 && tile_all <= kNvSlabBytes && aligned) {
        // whole tiles by bulk copy (t even: each tile a multiple of 16 bytes)
        NvChans ch{};
        for (int c = 0; c < NV; c++) ch.c[c] = v->atlas[chans[c]].as<float>();
        GV_CUDA(v, cudaFuncSetAttribute(k_nv_leaves_bulk<NV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)tile_all));
        k_nv_leaves_bulk<NV><<<(unsigned)L.cnt[0], kNvThreads, tile_all, s>>>(
            v->pool_ptr(0), v->leaf_slot.as<int32_t>(), v->atlas_last, ch, L.ld[0], v->apron, dst + L.sec[0],
            L.rec[0], status);
        GV_CUDA(v, cudaGetLastError());
    } else if (L.cnt[0] > 0) {
        NvChans ch{};
        for (int c = 0; c < NV; c++) ch.c[c] = v->atlas[chans[c]].as<float>();
        // largest power-of-two slab of x-planes whose staging fits kNvSlabBytes (at least one plane)
        int lslab = L.ld[0];
        while (lslab > 0 && (size_t)(1 << lslab) * (T * T + 1) * 4 * NV > kNvSlabBytes) lslab--;
        const size_t smem = (size_t)(1 << lslab) * (T * T + 1) * 4 * NV;
        GV_CUDA(v, cudaFuncSetAttribute(k_nv_leaves<NV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_nv_leaves<NV><<<(unsigned)L.cnt[0], kNvThreads, smem, s>>>(v->pool_ptr(0), v->leaf_slot.as<int32_t>(),
                                                                      v->atlas_last, ch, L.ld[0], v->apron, lslab,
                                                                      dst + L.sec[0], L.rec[0]);
        GV_CUDA(v, cudaGetLastError());
    }
    for (int lev = 1; lev <= 2; lev++) {
        if (L.cnt[lev] == 0) continue;
        k_nv_nodes<NV><<<(unsigned)L.cnt[lev], kNvThreads, 0, s>>>(
            v->pool_ptr(lev), v->clist[lev].as<uint64_t>(), L.ld[lev], dst + L.sec[lev - 1], L.rec[lev - 1],
            L.cnt[lev - 1], lev == 1, bg, (int32_t)L.cnt[lev],
            v->clist[lev].bytes / (sizeof(uint64_t) << (3 * L.ld[lev])), dst + L.sec[lev], L.rec[lev], status);
        GV_CUDA(v, cudaGetLastError());
    }
    return GVDB2_OK;
}

// The volume's transform as SetTransform builds it (V:5786-5789: T R S PT;
// Matrix4F::RotateZYX / RotateTZYX / RotateTZYXS / PreTranslate,
// gvdb_vec.cpp:218-281, 487-498), column-major, in the reference's float
// arithmetic (DEGtoRAD is 3.141592f / 180.0f, gvdb_types.h:59).
void transform_matrix(const Volume *v, float d[16]) {
    const float kDegToRad = 3.141592f / 180.0f;
    const float *ang = v->xf_angs, *t = v->xf_trans, *sc = v->xf_scale, *pt = v->xf_pretrans;
    const float cx = cosf(ang[0] * kDegToRad), sx = sinf(ang[0] * kDegToRad);
    const float cy = cosf(ang[1] * kDegToRad), sy = sinf(ang[1] * kDegToRad);
    const float cz = cosf(ang[2] * kDegToRad), sz = sinf(ang[2] * kDegToRad);
    d[0] = cy * cz;
    d[1] = cy * sz;
    d[2] = -sy;
    d[3] = 0;
    d[4] = cz * sx * sy - cx * sz;
    d[5] = cx * cz + sx * sy * sz;
    d[6] = cy * sx;
    d[7] = 0;
    d[8] = cx * cz * sy + sx * sz;
    d[9] = -cz * sx + cx * sy * sz;
    d[10] = cx * cy;
    d[11] = 0;
    d[12] = t[0];
    d[13] = t[1];
    d[14] = t[2];
    d[15] = 1;
    for (int i = 0; i < 3; i++) {
        d[i + 0] *= sc[0];
        d[i + 4] *= sc[1];
        d[i + 8] *= sc[2];
    }
    d[12] += d[0] * pt[0] + d[4] * pt[1] + d[8] * pt[2];
    d[13] += d[1] * pt[0] + d[5] * pt[1] + d[9] * pt[2];
    d[14] += d[2] * pt[0] + d[6] * pt[1] + d[10] * pt[2];
}

} // namespace

gvdb2_status nanovdb_size(Volume *v, int value_type, size_t *bytes) {
    if (!bytes) return fail(v, GVDB2_ERR_ARG, "null size");
    NvLayout L;
    GV_TRY(nv_layout(v, value_type, L));
    *bytes = (size_t)L.total;
    return GVDB2_OK;
}

gvdb2_status export_nanovdb(Volume *v, int value_type, const int32_t *chans, const float *background,
                            const char *grid_name, int32_t grid_class, void *dst_device, size_t dst_bytes) {
    NvLayout L;
    GV_TRY(nv_layout(v, value_type, L));
    const int nv = value_type;
    if (!chans || !background || !dst_device) return fail(v, GVDB2_ERR_ARG, "null channels, background or buffer");
    if (reinterpret_cast<uintptr_t>(dst_device) % 32) return fail(v, GVDB2_ERR_ARG, "buffer must be 32-byte aligned");
    for (int c = 0; c < nv; c++)
        if (chans[c] < 0 || chans[c] >= kMaxChan || !v->has_chan[chans[c]])
            return fail(v, GVDB2_ERR_ARG, "channel not allocated");
    if (!v->atlas_valid) return fail(v, GVDB2_ERR_STATE, "UpdateAtlas has not run on the current topology");
    if (dst_bytes < L.total) return fail(v, GVDB2_ERR_CAPACITY, "buffer smaller than gvdb2_nanovdb_size");
    cudaStream_t s = v->stream;
    uint8_t *d = static_cast<uint8_t *>(dst_device);
    // the header region is written last, from the host: its first word
    // carries the kernels' status until then
    int32_t *status = reinterpret_cast<int32_t *>(d);
    GV_CUDA(v, cudaMemsetAsync(status, 0, sizeof(int32_t), s));
    const float3 bg = make_float3(background[0], nv == 3 ? background[1] : 0.0f, nv == 3 ? background[2] : 0.0f);
    GV_TRY(nv == 1 ? launch_nv<1>(v, L, chans, bg, d, status) : launch_nv<3>(v, L, chans, bg, d, status));

    // ProcessGridExtents (gvdb_export_nanovdb.cpp:204-327) from the level-2 headers
    std::vector<gvdb2_nv_node> h2((size_t)L.cnt[2]);
    if (L.cnt[2])
        GV_CUDA(v, cudaMemcpy2DAsync(h2.data(), sizeof(gvdb2_nv_node), d + L.sec[2], L.rec[2], sizeof(gvdb2_nv_node),
                                     (size_t)L.cnt[2], cudaMemcpyDeviceToHost, s));
    int32_t st = 0;
    GV_CUDA(v, cudaMemcpyAsync(&st, status, sizeof(st), cudaMemcpyDeviceToHost, s));
    GV_CUDA(v, cudaStreamSynchronize(s));
    if (st & kDevBadIndex) return fail(v, GVDB2_ERR_STATE, "a child list names a node past its level's pool");
    if (st & kDevTimeout) return fail(v, GVDB2_ERR_STATE, "a leaf's bulk copy did not complete");

    std::vector<uint8_t> hb((size_t)L.sec[2], 0);
    gvdb2_nv_grid &g = *reinterpret_cast<gvdb2_nv_grid *>(hb.data());
    gvdb2_nv_tile *tiles = reinterpret_cast<gvdb2_nv_tile *>(hb.data() + L.sec[3]);
    const int shift = L.ld[0] + L.ld[1] + L.ld[2];
    int32_t bb[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN}; // an empty CoordBBox
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    // ExportToNanoVDB_MinimumValue: numeric_limits<float>::min() (the least
    // positive normal) for a float grid, -FLT_MAX per component for Vec3f
    float hi[3] = {nv == 1 ? FLT_MIN : -FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int64_t i = 0; i < L.cnt[2]; i++) {
        const gvdb2_nv_node &h = h2[(size_t)i];
        // Tile::setChild with RootData::CoordToKey (gvdb_export_nanovdb.cpp:271-276): a
        // negative corner's shifted value sign-extends into the higher fields, as there
        tiles[i].key = (uint64_t)(h.bbox_min[2] >> shift) | ((uint64_t)(h.bbox_min[1] >> shift) << 21) |
                       ((uint64_t)(h.bbox_min[0] >> shift) << 42);
        tiles[i].child = (uint32_t)i;
        tiles[i].state = 0;
        for (int a = 0; a < 3; a++) {
            bb[a] = std::min(bb[a], h.bbox_min[a]);
            bb[3 + a] = std::max(bb[3 + a], h.bbox_max[a]);
        }
        for (int c = 0; c < nv; c++) {
            lo[c] = lo[c] < h.vmin[c] ? lo[c] : h.vmin[c];
            hi[c] = hi[c] > h.vmax[c] ? hi[c] : h.vmax[c];
        }
    }
    // ascending keys for RootNode::findTile; equal keys keep node order
    std::stable_sort(tiles, tiles + L.cnt[2],
                     [](const gvdb2_nv_tile &a, const gvdb2_nv_tile &b) { return a.key < b.key; });

    g.magic = GVDB2_NV_MAGIC;
    g.total_bytes = L.total;
    g.value_type = (uint32_t)nv;
    g.grid_class = (uint32_t)grid_class;
    for (int l = 0; l < 3; l++) g.log2dim[l] = L.ld[l], g.record_bytes[l] = L.rec[l], g.count[l] = (uint64_t)L.cnt[l];
    g.count[3] = 1;
    for (int k = 0; k < 4; k++) g.section[k] = L.sec[k];
    if (grid_name) strncpy(g.name, grid_name, sizeof(g.name) - 1);
    float M[16];
    transform_matrix(v, M);
    memcpy(g.index_to_world, M, sizeof(M));
    for (int a = 0; a < 3; a++) {
        const double x = M[4 * a], y = M[4 * a + 1], z = M[4 * a + 2];
        g.voxel_size[a] = std::sqrt(x * x + y * y + z * z);
    }
    double wb[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int k = 0; k < 8; k++) {
        const double p[3] = {(double)bb[(k & 1) ? 3 : 0], (double)bb[(k & 2) ? 4 : 1], (double)bb[(k & 4) ? 5 : 2]};
        for (int a = 0; a < 3; a++) {
            const double w = (double)M[a] * p[0] + (double)M[4 + a] * p[1] + (double)M[8 + a] * p[2] + (double)M[12 + a];
            wb[a] = w < wb[a] ? w : wb[a];
            wb[3 + a] = w > wb[3 + a] ? w : wb[3 + a];
        }
    }
    memcpy(g.world_bbox, wb, sizeof(wb));
    g.active_voxels = (uint64_t)L.cnt[0] << (3 * L.ld[0]);
    g.tile_count = (uint32_t)L.cnt[2];
    memcpy(g.bbox, bb, sizeof(bb));
    for (int c = 0; c < nv; c++) g.background[c] = background[c], g.vmin[c] = lo[c], g.vmax[c] = hi[c];
    GV_CUDA(v, cudaMemcpyAsync(d, hb.data(), hb.size(), cudaMemcpyHostToDevice, s));
    GV_CUDA(v, cudaStreamSynchronize(s));
    return GVDB2_OK;
}

} // namespace gvdb2
