// batch.cu -- many point clouds in one volume (no counterpart in the
// reference, which handles one cloud per VolumeGVDB).
//
// Every cloud lives in its own index space [0, 2^s)^3.  gvdb2_batch_points
// packs the clouds' positions, unchanged, into one array owned by the
// volume, with a cloud index per point.  Cloud c is placed at the integer
// voxel origin of block (c mod K, (c / K) mod K, c / K^2) of a K^3 grid of
// blocks 2^(s+1) voxels apart, K = ceil(cbrt(ncloud)).  The other calls then
// serve all clouds in one pass each: RebuildTopology, UpdateAtlas, the
// kernel splats and gathers, UpdateApron and the adjoints.  Per-point
// outputs come back in the packed order, cloud after cloud.
//
// Why a cloud's results equal, bit for bit, those of a volume of its own:
// - the kernels take floor and fraction of the position in the cloud's own
//   space and add the origin to integer grid coordinates only.  Adding it
//   to the float position instead would round away low mantissa bits: at
//   2048 the float spacing is 4x that below 1024.
// - the gap of 2^s voxels between blocks is wider than any activation box,
//   stencil or apron, so no brick of one cloud is touched by another, and
//   activation boxes are clamped at 0 in the cloud's own space, as in a
//   volume of its own;
// - the origins are multiples of 2^(s+1), hence of the node range of every
//   level up to that size, so the cloud's bricks and the nodes above them up
//   to that level sit on the same grid, shifted;
// - the splat's fixed-point scale depends only on each brick's own points
//   and the merge sums a fixed set of partials in a fixed order.
// The reference-mode point operations (InsertPoints, InsertPointsSubcell and
// what builds on them) take one cloud per volume and refuse a batch.
#include "dev_common.cuh"

namespace gvdb2 {

namespace {

constexpr int kPackClouds = 64; // clouds per packing launch (views travel as kernel parameters)

struct PackArgs {
    PointsView src[kPackClouds];
    int64_t first[kPackClouds + 1]; // packed index of each cloud's first point
    int cloud0;                     // index of src[0]
    int ncloud;
};

__global__ void k_pack_clouds(PackArgs A, float *dst, int32_t *cloud) {
    const int64_t total = A.first[A.ncloud] - A.first[0];
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = A.first[0] + t;
        int lo = 0, hi = A.ncloud - 1; // last cloud with first <= i
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (A.first[mid] <= i) lo = mid;
            else hi = mid - 1;
        }
        const float3 p = load_f3(A.src[lo], i - A.first[lo]);
        dst[3 * i + 0] = p.x;
        dst[3 * i + 1] = p.y;
        dst[3 * i + 2] = p.z;
        cloud[i] = A.cloud0 + lo;
    }
}

} // namespace

int batch_grid(int ncloud) {
    int k = 1;
    while ((int64_t)k * k * k < ncloud) k++;
    return k;
}

void batch_origin(int cloud, int ncloud, int space_log2, int32_t out[3]) {
    const int k = batch_grid(ncloud);
    const int stride = 1 << (space_log2 + 1);
    out[0] = (cloud % k) * stride;
    out[1] = ((cloud / k) % k) * stride;
    out[2] = (cloud / (k * k)) * stride;
}

gvdb2_status batch_points(Volume *v, const gvdb2_points_view *clouds, int ncloud, int space_log2, int64_t *first) {
    if (ncloud < 1 || !clouds) return fail(v, GVDB2_ERR_ARG, "no clouds");
    if (space_log2 < 3 || space_log2 > 20) return fail(v, GVDB2_ERR_ARG, "cloud space must be 2^3 .. 2^20 voxels");
    const int k = batch_grid(ncloud);
    if ((int64_t)k << (space_log2 + 1) > (1ll << 30)) return fail(v, GVDB2_ERR_UNSUPPORTED, "batch extent too large");
    std::vector<int64_t> f(ncloud + 1, 0);
    for (int c = 0; c < ncloud; c++) {
        const gvdb2_points_view &w = clouds[c];
        if (w.count < 0 || (w.count > 0 && (!w.base || w.stride_bytes < 12 || w.offset_bytes < 0)))
            return fail(v, GVDB2_ERR_ARG, "bad cloud view");
        f[c + 1] = f[c] + w.count;
    }
    const int64_t total = f[ncloud];
    if (total > INT32_MAX) return fail(v, GVDB2_ERR_CAPACITY, "batch exceeds 2^31 points");
    cudaStream_t s = v->stream;
    GV_CUDA(v, v->batch_pos.ensure(sizeof(float) * 3 * (size_t)std::max<int64_t>(total, 1), s));
    GV_CUDA(v, v->batch_cloud.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(total, 1), s));
    GV_CUDA(v, v->batch_origin.ensure(sizeof(int32_t) * 3 * (size_t)ncloud, s));
    std::vector<int32_t> org(3 * (size_t)ncloud);
    for (int c = 0; c < ncloud; c++) batch_origin(c, ncloud, space_log2, &org[3 * (size_t)c]);
    GV_CUDA(v, cudaMemcpyAsync(v->batch_origin.p, org.data(), sizeof(int32_t) * org.size(), cudaMemcpyHostToDevice, s));
    for (int c0 = 0; c0 < ncloud; c0 += kPackClouds) {
        PackArgs A;
        A.cloud0 = c0;
        A.ncloud = std::min(kPackClouds, ncloud - c0);
        for (int j = 0; j < A.ncloud; j++) {
            A.src[j] = to_view(clouds[c0 + j]);
            A.first[j] = f[c0 + j];
        }
        A.first[A.ncloud] = f[c0 + A.ncloud];
        const int64_t cnt = A.first[A.ncloud] - A.first[0];
        if (cnt > 0)
            k_pack_clouds<<<grid_for(cnt, 256, 8 * kSmCount), 256, 0, s>>>(A, v->batch_pos.as<float>(),
                                                                          v->batch_cloud.as<int32_t>());
    }
    GV_CUDA(v, cudaGetLastError());
    GV_CUDA(v, cudaStreamSynchronize(s)); // `org` is released on return
    PointsView p;
    p.base = v->batch_pos.as<const char>();
    p.count = total;
    p.stride = 12;
    p.offset = 0;
    p.cloud = v->batch_cloud.as<int32_t>();
    p.origin = v->batch_origin.as<int32_t>();
    v->pos = p;
    v->vel = PointsView{};
    v->clr = PointsView{};
    v->bin_key.valid = false;
    v->batch_clouds = ncloud;
    v->batch_space_log2 = space_log2;
    if (first)
        for (int c = 0; c <= ncloud; c++) first[c] = f[c];
    return GVDB2_OK;
}

} // namespace gvdb2
