// primitives.cu -- in-house device scan and stable LSD radix sort.
//
// These replace the Thrust sort and the three-level Blelloch scan of the
// reference (gvdb_cutils.cu:11-16, P:858-902).  Both are tile-based:
// a reduce pass, a recursive scan of the tile sums, and a down-sweep.
#include "dev_common.cuh"

namespace gvdb2 {

namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t x, uint32_t *smem_warp, uint32_t &excl) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    uint32_t inc = warp_incl_scan(x);
    if (lane == 31) smem_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nwarps ? smem_warp[lane] : 0;
        uint32_t wi = warp_incl_scan(w);
        if (lane < nwarps) smem_warp[lane] = wi - w;
        if (lane == 31) smem_warp[32] = wi;
    }
    __syncthreads();
    excl = smem_warp[warp] + inc - x;
    uint32_t total = smem_warp[32];
    __syncthreads();
    return total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const uint32_t *__restrict__ in, int64_t n,
                                                              uint32_t *__restrict__ sums) {
    __shared__ uint32_t sw[33];
    int64_t base = (int64_t)blockIdx.x * kScanTile;
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        int64_t i = base + (int64_t)j * kScanThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
    uint32_t excl;
    uint32_t tot = block_excl_scan(s, sw, excl);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Scan one tile: coalesced load into shared memory, per-thread serial scan
// of kScanItems consecutive items, block scan of the thread sums.
__global__ void __launch_bounds__(kScanThreads) k_scan_tile(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                                                            int64_t n, const uint32_t *__restrict__ block_off) {
    __shared__ uint32_t tile[kScanTile];
    __shared__ uint32_t sw[33];
    int64_t base = (int64_t)blockIdx.x * kScanTile;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        int64_t i = base + (int64_t)j * kScanThreads + threadIdx.x;
        tile[j * kScanThreads + threadIdx.x] = i < n ? in[i] : 0u;
    }
    __syncthreads();
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        v[j] = tile[threadIdx.x * kScanItems + j];
        s += v[j];
    }
    uint32_t excl;
    uint32_t tot = block_excl_scan(s, sw, excl);
    uint32_t off = block_off ? block_off[blockIdx.x] : 0u;
    uint32_t run = off + excl;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        tile[threadIdx.x * kScanItems + j] = run;
        run += v[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        int64_t i = base + (int64_t)j * kScanThreads + threadIdx.x;
        if (i < n) out[i] = tile[j * kScanThreads + threadIdx.x];
    }
    if (threadIdx.x == 0 && base + kScanTile >= n) out[n] = off + tot; // last tile writes the total
}

// ---------------------------------------------------------------------
// radix sort
// ---------------------------------------------------------------------
constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsItems = 16;                  // per lane
constexpr int kRsTile = kRsThreads * kRsItems; // 4096 keys per block
constexpr int kRsWarpKeys = 32 * kRsItems;    // 512 keys per warp

__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const uint64_t *__restrict__ keys, int64_t n, int shift,
                                                        uint32_t *__restrict__ hist, int nblocks) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * kRsTile;
    for (int j = 0; j < kRsItems; j++) {
        int64_t i = base + (int64_t)j * kRsThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(uint32_t)(keys[i] >> shift) & 0xFF], 1u);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: warp w owns keys [w*512, w*512+512) of the tile and visits
// them in order 32 at a time; ranks inside a group of equal digits come
// from __match_any_sync, so equal keys keep their input order.
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const uint64_t *__restrict__ keys,
                                                           const int32_t *__restrict__ vals, int64_t n, int shift,
                                                           const uint32_t *__restrict__ offs, int nblocks,
                                                           uint64_t *__restrict__ keys_out,
                                                           int32_t *__restrict__ vals_out) {
    __shared__ uint32_t wbase[kRsWarps][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kRsWarps * 256; i += kRsThreads) (&wbase[0][0])[i] = 0;
    __syncthreads();
    int64_t wstart = (int64_t)blockIdx.x * kRsTile + (int64_t)warp * kRsWarpKeys;
    for (int j = 0; j < kRsItems; j++) {
        int64_t i = wstart + j * 32 + lane;
        if (i < n) atomicAdd(&wbase[warp][(uint32_t)(keys[i] >> shift) & 0xFF], 1u);
    }
    __syncthreads();
    {
        int d = threadIdx.x; // 256 threads, one digit each
        uint32_t run = offs[(int64_t)d * nblocks + blockIdx.x];
        for (int w = 0; w < kRsWarps; w++) {
            uint32_t c = wbase[w][d];
            wbase[w][d] = run;
            run += c;
        }
    }
    __syncthreads();
    for (int j = 0; j < kRsItems; j++) {
        int64_t i = wstart + j * 32 + lane;
        bool valid = i < n;
        unsigned active = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            uint64_t k = keys[i];
            uint32_t d = (uint32_t)(k >> shift) & 0xFF;
            unsigned peers = __match_any_sync(active, d);
            uint32_t rank = __popc(peers & lanemask_lt());
            uint32_t pos = wbase[warp][d] + rank;
            keys_out[pos] = k;
            if (vals) vals_out[pos] = vals[i];
            __syncwarp(active);
            if (rank == 0) wbase[warp][d] += __popc(peers);
            __syncwarp(active);
        }
    }
}

} // namespace

gvdb2_status exclusive_scan_u32(Volume *v, const uint32_t *in, uint32_t *out, int64_t n) {
    cudaStream_t s = v->stream;
    if (n <= 0) {
        GV_CUDA(v, cudaMemsetAsync(out, 0, sizeof(uint32_t), s));
        return GVDB2_OK;
    }
    int64_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb == 1) {
        k_scan_tile<<<1, kScanThreads, 0, s>>>(in, out, n, nullptr);
        GV_CUDA(v, cudaGetLastError());
        return GVDB2_OK;
    }
    uint32_t *sums = nullptr;
    GV_CUDA(v, cudaMallocAsync((void **)&sums, sizeof(uint32_t) * (size_t)(2 * nb + 2), s));
    uint32_t *sums_scan = sums + nb + 1;
    k_scan_reduce<<<(unsigned)nb, kScanThreads, 0, s>>>(in, n, sums);
    gvdb2_status st = exclusive_scan_u32(v, sums, sums_scan, nb);
    if (st == GVDB2_OK) {
        k_scan_tile<<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n, sums_scan);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_fail(v, e, "k_scan_tile");
    }
    cudaFreeAsync(sums, s);
    return st;
}

gvdb2_status radix_sort_u64(Volume *v, uint64_t *keys, int32_t *vals, int64_t n, int lo_bit, int hi_bit) {
    cudaStream_t s = v->stream;
    if (n <= 1 || hi_bit <= lo_bit) return GVDB2_OK;
    int64_t nb = (n + kRsTile - 1) / kRsTile;
    if (nb > (1ll << 22)) return fail(v, GVDB2_ERR_UNSUPPORTED, "radix sort input too large");
    uint64_t *kalt = nullptr;
    int32_t *valt = nullptr;
    uint32_t *hist = nullptr;
    GV_CUDA(v, cudaMallocAsync((void **)&kalt, sizeof(uint64_t) * (size_t)n, s));
    if (vals) GV_CUDA(v, cudaMallocAsync((void **)&valt, sizeof(int32_t) * (size_t)n, s));
    GV_CUDA(v, cudaMallocAsync((void **)&hist, sizeof(uint32_t) * (size_t)(2 * 256 * nb + 2), s));
    uint32_t *offs = hist + 256 * nb + 1;
    uint64_t *kin = keys, *kout = kalt;
    int32_t *vin = vals, *vout = valt;
    gvdb2_status st = GVDB2_OK;
    for (int shift = lo_bit; shift < hi_bit && st == GVDB2_OK; shift += 8) {
        k_rs_hist<<<(unsigned)nb, kRsThreads, 0, s>>>(kin, n, shift, hist, (int)nb);
        st = exclusive_scan_u32(v, hist, offs, 256 * nb);
        if (st != GVDB2_OK) break;
        k_rs_scatter<<<(unsigned)nb, kRsThreads, 0, s>>>(kin, vin, n, shift, offs, (int)nb, kout, vout);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_fail(v, e, "k_rs_scatter");
        uint64_t *tk = kin;
        kin = kout;
        kout = tk;
        int32_t *tv = vin;
        vin = vout;
        vout = tv;
    }
    if (st == GVDB2_OK && kin != keys) {
        cudaError_t e = cudaMemcpyAsync(keys, kin, sizeof(uint64_t) * (size_t)n, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess && vals) e = cudaMemcpyAsync(vals, vin, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) st = cuda_fail(v, e, "radix sort copy-back");
    }
    cudaFreeAsync(kalt, s);
    if (valt) cudaFreeAsync(valt, s);
    cudaFreeAsync(hist, s);
    return st;
}

} // namespace gvdb2
