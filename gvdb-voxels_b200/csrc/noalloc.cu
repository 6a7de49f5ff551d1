// noalloc.cu -- gvdb2_gather_kernel_noalloc: the grid -> point gather without
// any device allocation.
//
// Some callers cannot allocate device memory once they are running: a host
// application that hands the GPU to a fixed memory budget at start-up (a
// game engine or a real-time simulation loop that forbids allocation after
// initialisation), a process whose allocator is owned by another framework,
// or a caller holding a CUDA context in a state where an allocation would
// synchronise the device at a bad time.  gvdb2_gather_kernel allocates its
// per-call binning buffers (point -> bin ids, ranks, the bin-ordered point
// list, per-bin offsets; a bin is an 8^3 cell of an active brick, the whole
// brick for 8^3 bricks); this variant keeps them in one file-scope device
// array instead, sized for at most kNoAllocMaxPoints points and
// kNoAllocMaxBins bins, and computes the same values.
//
// The array exists once per GPU that loads the library and lives until the
// process exits.  Every call shares it, and it keeps the last call's
// contents: the per-brick counters are cleared at the start of each call.
// Two calls whose GPU work overlaps (different streams, or different volumes
// on one device) race on it and must be ordered by the caller.
//
// Host code may not hand the array's name to a kernel: on the host it is only
// a stand-in symbol, not a device address.  The first call on each device
// (with that device current) looks the address up with
// cudaGetSymbolAddress and caches it; that first call should come before any
// stream capture.  The cached address belongs to the device's current
// context: a process that calls cudaDeviceReset must not call this entry
// point on that device afterwards (the module is reloaded at a new address).
#include <mutex>

#include "dev_common.cuh"

namespace gvdb2 {

namespace {

constexpr int64_t kNoAllocMaxPoints = 1 << 20; // 1,048,576 points
constexpr int64_t kNoAllocMaxBins = 1 << 15;   // 32,768 cells: active bricks of 8^3 (1/8 as many of 16^3)
constexpr int64_t kOffWords = kNoAllocMaxBins + 1;
constexpr int64_t kScratchWords = 3 * kNoAllocMaxPoints + kNoAllocMaxBins + kOffWords; // 12.25 MiB

// [0, P) point bins, [P, 2P) ranks, [2P, 3P) bin-ordered point list,
// [3P, 3P+S) per-bin counts, then S+1 per-bin offsets.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
uint32_t *g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array for `device` (current), looked up once.
gvdb2_status scratch_address(Volume *v, uint32_t **out) {
    if (v->device < 0 || v->device >= kMaxDevices) return fail(v, GVDB2_ERR_UNSUPPORTED, "device index too large");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[v->device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(v, e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_scratch_ptr[v->device] = static_cast<uint32_t *>(p);
    }
    *out = g_scratch_ptr[v->device];
    return GVDB2_OK;
}

__global__ void k_na_bin(PointsView pos, int64_t n, float3 trans, LeafLookup L, const int32_t *leaf_slot, int m,
                         int32_t *pslot, uint32_t *prank, uint32_t *counts) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 p = load_f3(pos, i);
    int32_t bin = -1;
    if (p.z != kNoHit) {
        const float wx = p.x + trans.x, wy = p.y + trans.y, wz = p.z + trans.z;
        const int3 o = point_origin(pos, i);
        const int32_t leaf = leaf_at_o(L, wx, wy, wz, o);
        const int32_t slot = leaf >= 0 ? leaf_slot[leaf] : -1;
        if (slot >= 0) {
            const int rm = (1 << L.g.log2r0) - 1; // local voxel = voxel mod res0
            bin = slot * m * m * m + cell_of_local(((int)wx + o.x) & rm, ((int)wy + o.y) & rm, ((int)wz + o.z) & rm, m);
        }
    }
    pslot[i] = bin;
    if (bin >= 0) prank[i] = atomicAdd(&counts[bin], 1u);
}

// One CTA: exclusive scan of the per-brick counts into offsets (S+1 words).
constexpr int kNaScanThreads = 1024;
__global__ void __launch_bounds__(kNaScanThreads) k_na_scan(const uint32_t *counts, int64_t nslots, uint32_t *off) {
    __shared__ uint32_t warp_sum[32];
    const int per = (int)((nslots + kNaScanThreads - 1) / kNaScanThreads);
    const int64_t first = (int64_t)threadIdx.x * per;
    uint32_t local = 0;
    for (int k = 0; k < per; k++)
        if (first + k < nslots) local += counts[first + k];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = local;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_sum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sum[lane], wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        warp_sum[lane] = wi - w;
    }
    __syncthreads();
    uint32_t run = warp_sum[warp] + inc - local;
    for (int k = 0; k < per; k++) {
        if (first + k < nslots) {
            off[first + k] = run;
            run += counts[first + k];
        }
    }
    if (first < nslots && first + per >= nslots) off[nslots] = run; // the thread holding the last brick
}

__global__ void k_na_fill(const int32_t *pslot, const uint32_t *prank, int64_t n, const uint32_t *off, int32_t *perm,
                          float *out, int64_t out_stride, int nch) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t s = pslot[i];
    if (s >= 0) {
        perm[off[s] + prank[i]] = (int32_t)i;
    } else {
        for (int c = 0; c < nch; c++) out[i * out_stride + c] = 0.0f; // outside every active brick
    }
}

} // namespace

} // namespace gvdb2

struct gvdb2_volume {
    gvdb2::Volume v;
};

extern "C" gvdb2_status gvdb2_gather_kernel_noalloc(gvdb2_volume *h, int kernel, int n, const float trans[3],
                                                   const int *chans, int nch, float *out, int64_t out_stride) {
    using namespace gvdb2;
    if (!h) return GVDB2_ERR_ARG;
    Volume *v = &h->v;
    cudaError_t e = cudaSetDevice(v->device);
    if (e != cudaSuccess) return cuda_fail(v, e, "cudaSetDevice");
    if (n < 0 || (n > 0 && (!v->pos.base || n > v->pos.count))) return fail(v, GVDB2_ERR_ARG, "bad point count");
    if (n > kNoAllocMaxPoints)
        return fail(v, GVDB2_ERR_CAPACITY, "gvdb2_gather_kernel_noalloc takes at most 1,048,576 points per call");
    if (!v->atlas_valid) return fail(v, GVDB2_ERR_STATE, "UpdateAtlas must follow the topology rebuild");
    const int m = v->res(0) / kCell; // cells per brick edge
    if (m < 1 || v->res(0) % kCell)
        return fail(v, GVDB2_ERR_UNSUPPORTED, "kernel gathers need bricks of a multiple of 8 voxels");
    if (v->atlas_last * m * m * m > kNoAllocMaxBins)
        return fail(v, GVDB2_ERR_CAPACITY,
                    "gvdb2_gather_kernel_noalloc takes at most 32,768 active 8^3 cells (bricks of 8^3 voxels)");
    if (!out || out_stride < nch) return fail(v, GVDB2_ERR_ARG, "bad output buffer");
    // every argument is checked before the first memset or launch, so a
    // refused call leaves `out` and the scratch array as they were
    if (kernel != GVDB2_KERNEL_TENT1 && kernel != GVDB2_KERNEL_CUBIC2) return fail(v, GVDB2_ERR_ARG, "unknown kernel");
    GV_TRY(check_chans(v, chans, nch));
    const float zero[3] = {0, 0, 0};
    if (!trans) trans = zero;
    uint32_t *base = nullptr;
    GV_TRY(scratch_address(v, &base));
    int32_t *pslot = reinterpret_cast<int32_t *>(base);
    uint32_t *prank = base + kNoAllocMaxPoints;
    int32_t *perm = reinterpret_cast<int32_t *>(base + 2 * kNoAllocMaxPoints);
    uint32_t *counts = base + 3 * kNoAllocMaxPoints;
    uint32_t *off = counts + kNoAllocMaxBins;
    const int64_t nbins = v->atlas_last * m * m * m;
    if (n == 0 || nbins == 0) {
        if (n > 0) // no active brick: every point gathers zero
            GV_CUDA(v, cudaMemset2DAsync(out, sizeof(float) * out_stride, 0, sizeof(float) * nch, n, v->stream));
        return GVDB2_OK;
    }
    GV_CUDA(v, cudaMemsetAsync(counts, 0, sizeof(uint32_t) * (size_t)nbins, v->stream));
    LeafLookup L = make_lookup(v);
    const float3 t = make_float3(trans[0], trans[1], trans[2]);
    const int g = grid_for(n, 256, 1ll << 31);
    k_na_bin<<<g, 256, 0, v->stream>>>(v->pos, n, t, L, v->leaf_slot.as<int32_t>(), m, pslot, prank, counts);
    k_na_scan<<<1, kNaScanThreads, 0, v->stream>>>(counts, nbins, off);
    k_na_fill<<<g, 256, 0, v->stream>>>(pslot, prank, n, off, perm, out, out_stride, nch);
    GV_CUDA(v, cudaGetLastError());
    return gather_kernel_prebinned(v, kernel, n, trans, chans, nch, out, out_stride, off, perm);
}
