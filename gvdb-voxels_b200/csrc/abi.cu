// abi.cu -- the extern "C" boundary of libgvdb2 (declared in include/gvdb2.h).
#include <algorithm>
#include <climits>
#include <cstring>
#include <new>

#include "dev_common.cuh"

struct gvdb2_volume {
    gvdb2::Volume v;
};

namespace gvdb2 {

cudaError_t DevBuf::ensure(size_t need, cudaStream_t s, bool preserve) {
    if (need <= bytes && p) return cudaSuccess;
    // geometric growth: a buffer that tracks a slowly growing topology (the
    // atlas, the splat scratch) is re-allocated O(log) times, not every step
    size_t grow = bytes + bytes / 2;
    size_t nb = std::max(need, grow);
    if (!p && need >= (size_t(1) << 24)) nb = need + need / 4; // large first allocations get headroom
    nb = (nb + 255) & ~size_t(255);
    void *np = nullptr;
    cudaError_t e = cudaMallocAsync(&np, nb, s);
    if (e != cudaSuccess) return e;
    if (preserve && p && bytes) {
        e = cudaMemcpyAsync(np, p, bytes, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) {
            cudaFreeAsync(np, s);
            return e;
        }
    }
    if (p) cudaFreeAsync(p, s);
    p = np;
    bytes = nb;
    stream = s;
    return cudaSuccess;
}

void DevBuf::release() {
    if (p) cudaFreeAsync(p, stream);
    p = nullptr;
    bytes = 0;
}

gvdb2_status fail(Volume *v, gvdb2_status st, const std::string &msg) {
    if (v) v->err = msg;
    return st;
}

gvdb2_status cuda_fail(Volume *v, cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    if (v) v->err = m;
    if (e == cudaErrorMemoryAllocation) return GVDB2_ERR_NOMEM;
    if (e == cudaErrorNoKernelImageForDevice || e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return GVDB2_ERR_NOT_AVAILABLE;
    return GVDB2_ERR_CUDA;
}

static gvdb2_status alloc_channel(Volume *v, int chan) {
    size_t bytes = (size_t)v->atlas_cap * (size_t)v->tile_vox() * sizeof(float);
    GV_CUDA(v, v->atlas[chan].ensure(bytes, v->stream));
    GV_CUDA(v, cudaMemsetAsync(v->atlas[chan].p, 0, bytes, v->stream));
    return GVDB2_OK;
}

} // namespace gvdb2

using gvdb2::Volume;

#define VOL(h) (&(h)->v)
#define CHECK_HANDLE(h)                          \
    do {                                         \
        if (!(h)) return GVDB2_ERR_ARG;          \
        cudaSetDevice((h)->v.device);            \
    } while (0)

extern "C" {

gvdb2_status gvdb2_create(gvdb2_volume **out, int device) {
    if (!out) return GVDB2_ERR_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return GVDB2_ERR_NOT_AVAILABLE;
    if (device < 0) device = 0;
    if (device >= count) return GVDB2_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return GVDB2_ERR_NOT_AVAILABLE;
    // keep freed stream-ordered allocations in the pool for reuse
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    gvdb2_volume *h = new (std::nothrow) gvdb2_volume();
    if (!h) return GVDB2_ERR_NOMEM;
    h->v.device = device;
    if (cudaMallocHost(&h->v.host_small, 128) != cudaSuccess) {
        delete h;
        return GVDB2_ERR_NOMEM;
    }
    // the small device words start clear (their flags and counters are read
    // back before some kernels write them)
    if (h->v.dev_small.ensure(128, nullptr) != cudaSuccess || cudaMemset(h->v.dev_small.p, 0, 128) != cudaSuccess) {
        cudaFreeHost(h->v.host_small);
        delete h;
        return GVDB2_ERR_NOMEM;
    }
    *out = h;
    return GVDB2_OK;
}

gvdb2_status gvdb2_destroy(gvdb2_volume *h) {
    if (!h) return GVDB2_OK;
    cudaSetDevice(h->v.device);
    cudaStreamSynchronize(h->v.stream);
    void *hs = h->v.host_small;
    delete h; // DevBuf destructors free device memory
    cudaDeviceSynchronize();
    if (hs) cudaFreeHost(hs);
    return GVDB2_OK;
}

const char *gvdb2_last_error(const gvdb2_volume *h) { return h ? h->v.err.c_str() : "null volume"; }

gvdb2_status gvdb2_set_stream(gvdb2_volume *h, void *stream) {
    CHECK_HANDLE(h);
    h->v.stream = reinterpret_cast<cudaStream_t>(stream);
    return GVDB2_OK;
}

gvdb2_status gvdb2_synchronize(gvdb2_volume *h) {
    CHECK_HANDLE(h);
    cudaError_t e = cudaStreamSynchronize(h->v.stream);
    if (e != cudaSuccess) return gvdb2::cuda_fail(VOL(h), e, "synchronize");
    return gvdb2::flush_status(VOL(h));
}

gvdb2_status gvdb2_set_option(gvdb2_volume *h, int option, int value) {
    CHECK_HANDLE(h);
    if (option == GVDB2_OPT_DETERMINISTIC) {
        h->v.deterministic = value ? 1 : 0;
        return GVDB2_OK;
    }
    if (option == GVDB2_OPT_AUTOTUNE) {
        h->v.autotune = value != 0;
        return GVDB2_OK;
    }
    return gvdb2::fail(VOL(h), GVDB2_ERR_ARG, "unknown option");
}

gvdb2_status gvdb2_configure(gvdb2_volume *h, int q4, int q3, int q2, int q1, int q0) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    int r[5] = {q0, q1, q2, q3, q4};
    for (int n = 0; n < 5; n++)
        if (r[n] < 0 || r[n] > 6) return gvdb2::fail(v, GVDB2_ERR_ARG, "log2 dims must lie in [0, 6]");
    v->nlev = 5;
    for (int n = 0; n < gvdb2::kMaxLev; n++) v->logdim[n] = 0;
    for (int n = 0; n < 5; n++) v->logdim[n] = r[n] == 0 ? 1 : r[n];
    for (int l = 0; l < gvdb2::kMaxLev; l++) v->pool_cnt[l] = 0;
    v->used_leaves = 0;
    v->all_leaves_flagged = false;
    v->atlas_last = 0;
    v->atlas_valid = false;
    v->rebuild_topo = true;
    v->bin_key.valid = false;
    return GVDB2_OK;
}

gvdb2_status gvdb2_set_transform(gvdb2_volume *h, const float pretrans[3], const float scale[3], const float angs[3],
                                 const float trans[3]) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    if (!pretrans || !scale || !angs || !trans) return gvdb2::fail(v, GVDB2_ERR_ARG, "null transform part");
    for (int a = 0; a < 3; a++) {
        v->xf_pretrans[a] = pretrans[a];
        v->xf_scale[a] = scale[a];
        v->xf_angs[a] = angs[a];
        v->xf_trans[a] = trans[a];
    }
    return GVDB2_OK;
}

gvdb2_status gvdb2_get_transform(gvdb2_volume *h, float pretrans[3], float scale[3], float angs[3], float trans[3]) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    if (!pretrans || !scale || !angs || !trans) return gvdb2::fail(v, GVDB2_ERR_ARG, "null transform part");
    for (int a = 0; a < 3; a++) {
        pretrans[a] = v->xf_pretrans[a];
        scale[a] = v->xf_scale[a];
        angs[a] = v->xf_angs[a];
        trans[a] = v->xf_trans[a];
    }
    return GVDB2_OK;
}

gvdb2_status gvdb2_save_vbx(gvdb2_volume *h, const char *path) {
    CHECK_HANDLE(h);
    return gvdb2::save_vbx(VOL(h), path);
}

gvdb2_status gvdb2_load_vbx(gvdb2_volume *h, const char *path) {
    CHECK_HANDLE(h);
    return gvdb2::load_vbx(VOL(h), path);
}

gvdb2_status gvdb2_nanovdb_size(gvdb2_volume *h, int value_type, size_t *bytes) {
    CHECK_HANDLE(h);
    return gvdb2::nanovdb_size(VOL(h), value_type, bytes);
}

gvdb2_status gvdb2_export_nanovdb(gvdb2_volume *h, int value_type, const int32_t *chans, const float *background,
                                  const char *grid_name, int32_t grid_class, void *dst_device, size_t dst_bytes) {
    CHECK_HANDLE(h);
    return gvdb2::export_nanovdb(VOL(h), value_type, chans, background, grid_name, grid_class, dst_device, dst_bytes);
}

gvdb2_status gvdb2_set_channel_default(gvdb2_volume *h, int cx, int cy, int cz) {
    CHECK_HANDLE(h);
    if (cx < 1 || cy < 1 || cz < 1) return gvdb2::fail(VOL(h), GVDB2_ERR_ARG, "bad axis counts");
    h->v.default_axiscnt[0] = cx;
    h->v.default_axiscnt[1] = cy;
    h->v.default_axiscnt[2] = cz;
    return GVDB2_OK;
}

gvdb2_status gvdb2_add_channel(gvdb2_volume *h, int chan, int dtype, int apron) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    if (v->nlev == 0) return gvdb2::fail(v, GVDB2_ERR_STATE, "Configure not called");
    if (chan < 0 || chan >= gvdb2::kMaxChan || v->has_chan[chan]) return gvdb2::fail(v, GVDB2_ERR_ARG, "bad channel");
    if (dtype != GVDB2_T_FLOAT) return gvdb2::fail(v, GVDB2_ERR_UNSUPPORTED, "only T_FLOAT channels");
    if (apron < 0 || apron > v->res(0)) return gvdb2::fail(v, GVDB2_ERR_ARG, "apron out of range");
    bool any = v->any_channel();
    if (any && apron != v->apron) return gvdb2::fail(v, GVDB2_ERR_UNSUPPORTED, "all channels share one apron");
    if (!any) {
        v->apron = apron;
        for (int a = 0; a < 3; a++) v->subdim[a] = v->default_axiscnt[a];
        v->atlas_cap = (int64_t)v->subdim[0] * v->subdim[1] * v->subdim[2];
    }
    v->has_chan[chan] = true;
    return gvdb2::alloc_channel(v, chan);
}

gvdb2_status gvdb2_set_points(gvdb2_volume *h, gvdb2_points_view pos, gvdb2_points_view vel, gvdb2_points_view clr) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    if (pos.base && (pos.stride_bytes < 12 || pos.offset_bytes < 0 || pos.count < 0))
        return gvdb2::fail(v, GVDB2_ERR_ARG, "position view needs stride >= 12");
    v->pos = gvdb2::to_view(pos);
    v->vel = gvdb2::to_view(vel);
    v->clr = gvdb2::to_view(clr);
    v->bin_key.valid = false;
    v->batch_clouds = 0;
    return GVDB2_OK;
}

gvdb2_status gvdb2_batch_points(gvdb2_volume *h, const gvdb2_points_view *clouds, int ncloud, int space_log2,
                                int64_t *first) {
    CHECK_HANDLE(h);
    return gvdb2::batch_points(VOL(h), clouds, ncloud, space_log2, first);
}

gvdb2_status gvdb2_batch_origin(gvdb2_volume *h, int cloud, int32_t out[3]) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    if (v->batch_clouds == 0) return gvdb2::fail(v, GVDB2_ERR_STATE, "no batch set");
    if (cloud < 0 || cloud >= v->batch_clouds || !out) return gvdb2::fail(v, GVDB2_ERR_ARG, "bad cloud index");
    int o[3];
    gvdb2::batch_origin(cloud, v->batch_clouds, v->batch_space_log2, o);
    for (int a = 0; a < 3; a++) out[a] = o[a];
    return GVDB2_OK;
}

gvdb2_status gvdb2_request_full_rebuild(gvdb2_volume *h, int flag) {
    CHECK_HANDLE(h);
    h->v.rebuild_topo = flag != 0;
    return GVDB2_OK;
}

gvdb2_status gvdb2_rebuild_topology(gvdb2_volume *h, int n, float radius, const float orig[3]) {
    CHECK_HANDLE(h);
    const float zero[3] = {0, 0, 0};
    return gvdb2::rebuild_topology(VOL(h), n, radius, orig ? orig : zero, false, 0);
}

gvdb2_status gvdb2_accumulate_topology(gvdb2_volume *h, int n, float radius, const float orig[3], int min_depth) {
    CHECK_HANDLE(h);
    const float zero[3] = {0, 0, 0};
    return gvdb2::rebuild_topology(VOL(h), n, radius, orig ? orig : zero, true, min_depth);
}

gvdb2_status gvdb2_finish_topology(gvdb2_volume *h, int commit, int bounds) {
    CHECK_HANDLE(h);
    (void)commit; // pools already live on the device; no host mirror to commit
    if (bounds) return gvdb2::compute_bounds(VOL(h));
    return GVDB2_OK;
}

gvdb2_status gvdb2_update_atlas(gvdb2_volume *h) {
    CHECK_HANDLE(h);
    return gvdb2::update_atlas(VOL(h));
}

gvdb2_status gvdb2_activate_space(gvdb2_volume *h, const float *xyz, int64_t n, uint64_t *out) {
    CHECK_HANDLE(h);
    if (n < 0 || (n > 0 && (!xyz || !out))) return gvdb2::fail(VOL(h), GVDB2_ERR_ARG, "ActivateSpace: bad arguments");
    return gvdb2::activate_space(VOL(h), xyz, n, out);
}

gvdb2_status gvdb2_compact_pools(gvdb2_volume *h) {
    CHECK_HANDLE(h);
    return gvdb2::compact_pools(VOL(h));
}

gvdb2_status gvdb2_clear_channel(gvdb2_volume *h, int chan) {
    CHECK_HANDLE(h);
    return gvdb2::clear_channel(VOL(h), chan);
}

gvdb2_status gvdb2_update_neighbors(gvdb2_volume *h) {
    CHECK_HANDLE(h);
    return gvdb2::update_neighbors(VOL(h));
}

gvdb2_status gvdb2_insert_points(gvdb2_volume *h, int n, const float trans[3], int prefix) {
    CHECK_HANDLE(h);
    const float zero[3] = {0, 0, 0};
    return gvdb2::insert_points(VOL(h), n, trans ? trans : zero, prefix);
}

gvdb2_status gvdb2_insert_points_subcell(gvdb2_volume *h, int subcell, int n, float radius, const float trans[3],
                                         int *len) {
    CHECK_HANDLE(h);
    const float zero[3] = {0, 0, 0};
    return gvdb2::insert_points_subcell(VOL(h), subcell, n, radius, trans ? trans : zero, len);
}

gvdb2_status gvdb2_insert_points_subcell_fp16(gvdb2_volume *h, int subcell, int n, float radius, const float trans[3],
                                              int *len) {
    CHECK_HANDLE(h);
    const float zero[3] = {0, 0, 0};
    return gvdb2::insert_points_subcell(VOL(h), subcell, n, radius, trans ? trans : zero, len, true);
}

gvdb2_status gvdb2_get_min_max_vel(gvdb2_volume *h, int n) {
    CHECK_HANDLE(h);
    return gvdb2::get_min_max_vel(VOL(h), n);
}

gvdb2_status gvdb2_scatter_density(gvdb2_volume *h, int n, float radius, float amp, const float trans[3], int expand,
                                   int avg_color) {
    CHECK_HANDLE(h);
    if (avg_color) return gvdb2::fail(VOL(h), GVDB2_ERR_UNSUPPORTED, "colour averaging is not on this path");
    const float zero[3] = {0, 0, 0};
    return gvdb2::scatter_density_ref(VOL(h), n, radius, amp, trans ? trans : zero, expand);
}

static gvdb2_status gather_common(gvdb2_volume *h, int subcell, float radius, int *len, int chan, int chan_clr,
                                  int accum, bool levelset, bool fp16 = false) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    if (chan_clr >= 0 && chan_clr < gvdb2::kMaxChan && v->has_chan[chan_clr] && v->clr.base)
        return gvdb2::fail(v, GVDB2_ERR_UNSUPPORTED, "colour gathers are not on this path");
    if (len && *len == 0 && !levelset) return GVDB2_OK; // GatherDensity returns on an empty list (V:5321)
    return gvdb2::gather_voxels(v, subcell, radius, chan, accum, levelset, fp16);
}

gvdb2_status gvdb2_gather_level_set_fp16(gvdb2_volume *h, int subcell, int n, float radius, const float trans[3],
                                         int *len, int chan_levelset, int chan_clr) {
    (void)n;
    (void)trans;
    CHECK_HANDLE(h);
    if (VOL(h)->used_leaves == 0) return GVDB2_OK; // returns without bricks (V:5378-5379)
    return gather_common(h, subcell, radius, len, chan_levelset, chan_clr, 0, true, true);
}

gvdb2_status gvdb2_gather_density(gvdb2_volume *h, int subcell, int n, float radius, const float trans[3], int *len,
                                  int chan_density, int chan_clr, int accum) {
    (void)n;
    (void)trans;
    return gather_common(h, subcell, radius, len, chan_density, chan_clr, accum, false);
}

gvdb2_status gvdb2_gather_level_set(gvdb2_volume *h, int subcell, int n, float radius, const float trans[3], int *len,
                                    int chan_levelset, int chan_clr, int accum) {
    (void)n;
    (void)trans;
    return gather_common(h, subcell, radius, len, chan_levelset, chan_clr, accum, true);
}

gvdb2_status gvdb2_scatter_reduce_level_set(gvdb2_volume *h, int subcell, int n, float radius, const float trans[3],
                                            int *len, int chan_levelset, int chan_clr, int accum) {
    return gvdb2_gather_level_set(h, subcell, n, radius, trans, len, chan_levelset, chan_clr, accum);
}

gvdb2_status gvdb2_update_apron(gvdb2_volume *h, int chan, float boundval) {
    CHECK_HANDLE(h);
    return gvdb2::update_apron(VOL(h), chan, boundval);
}

gvdb2_status gvdb2_update_apron_faces(gvdb2_volume *h, int chan) {
    CHECK_HANDLE(h);
    return gvdb2::update_apron_faces(VOL(h), chan);
}

gvdb2_status gvdb2_scatter_kernel(gvdb2_volume *h, int kernel, int n, const float trans[3], gvdb2_points_view weight,
                                  float weight_const, const gvdb2_points_view *attrs, const int *chans, int nch) {
    CHECK_HANDLE(h);
    const float zero[3] = {0, 0, 0};
    gvdb2::apply_cached_tuning(VOL(h), "scatter", kernel, nch, n);
    return gvdb2::scatter_kernel(VOL(h), kernel, n, trans ? trans : zero, weight, weight_const, attrs, chans, nch);
}

gvdb2_status gvdb2_gather_kernel(gvdb2_volume *h, int kernel, int n, const float trans[3], const int *chans, int nch,
                                 float *out, int64_t out_stride) {
    CHECK_HANDLE(h);
    const float zero[3] = {0, 0, 0};
    gvdb2::apply_cached_tuning(VOL(h), "gather", kernel, nch, n);
    return gvdb2::gather_kernel(VOL(h), kernel, n, trans ? trans : zero, chans, nch, out, out_stride);
}

gvdb2_status gvdb2_set_tuning(gvdb2_volume *h, const gvdb2_tuning *t) {
    CHECK_HANDLE(h);
    return gvdb2::set_tuning(VOL(h), t);
}

gvdb2_status gvdb2_get_tuning(gvdb2_volume *h, gvdb2_tuning *t) {
    CHECK_HANDLE(h);
    if (!t) return gvdb2::fail(VOL(h), GVDB2_ERR_ARG, "null tuning");
    *t = gvdb2::get_tuning(VOL(h));
    return GVDB2_OK;
}

gvdb2_status gvdb2_set_tune_cache(gvdb2_volume *h, const char *path) {
    CHECK_HANDLE(h);
    h->v.tune_cache = path ? path : "";
    return GVDB2_OK;
}

gvdb2_status gvdb2_autotune_scatter(gvdb2_volume *h, int kernel, int n, const float trans[3], gvdb2_points_view weight,
                                    float weight_const, const gvdb2_points_view *attrs, const int *chans, int nch,
                                    gvdb2_tuning *chosen) {
    CHECK_HANDLE(h);
    gvdb2::Volume *v = VOL(h);
    const float zero[3] = {0, 0, 0};
    const float *t = trans ? trans : zero;
    return gvdb2::autotune(v, "scatter", kernel, nch, n, gvdb2::scatter_candidates(v), [&]() {
        return gvdb2::scatter_kernel(v, kernel, n, t, weight, weight_const, attrs, chans, nch);
    }, chosen);
}

gvdb2_status gvdb2_autotune_gather(gvdb2_volume *h, int kernel, int n, const float trans[3], const int *chans,
                                   int nch, float *out, int64_t out_stride, gvdb2_tuning *chosen) {
    CHECK_HANDLE(h);
    gvdb2::Volume *v = VOL(h);
    const float zero[3] = {0, 0, 0};
    const float *t = trans ? trans : zero;
    return gvdb2::autotune(v, "gather", kernel, nch, n, gvdb2::gather_candidates(v), [&]() {
        return gvdb2::gather_kernel(v, kernel, n, t, chans, nch, out, out_stride);
    }, chosen);
}

gvdb2_status gvdb2_tune_cache_get(const char *path, const char *key, gvdb2_tuning *t, float *ms) {
    return gvdb2::cache_get(path, key, t, ms);
}

gvdb2_status gvdb2_tune_cache_put(const char *path, const char *key, const gvdb2_tuning *t, float ms) {
    return gvdb2::cache_put(path, key, t, ms);
}

gvdb2_status gvdb2_scatter_kernel_backward(gvdb2_volume *h, int kernel, int n, const float trans[3],
                                           gvdb2_points_view weight, float weight_const,
                                           const gvdb2_points_view *attrs, int nch, const int *grad_chans,
                                           float *grad_pos, float *grad_weight, float *grad_attr) {
    CHECK_HANDLE(h);
    const float zero[3] = {0, 0, 0};
    return gvdb2::scatter_kernel_backward(VOL(h), kernel, n, trans ? trans : zero, weight, weight_const, attrs, nch,
                                          grad_chans, grad_pos, grad_weight, grad_attr);
}

gvdb2_status gvdb2_gather_kernel_backward(gvdb2_volume *h, int kernel, int n, const float trans[3], const int *chans,
                                          int nch, const float *grad_out, const int *grad_chans, float *grad_pos) {
    CHECK_HANDLE(h);
    const float zero[3] = {0, 0, 0};
    return gvdb2::gather_kernel_backward(VOL(h), kernel, n, trans ? trans : zero, chans, nch, grad_out, grad_chans,
                                         grad_pos);
}

// ---- inspection ----
gvdb2_status gvdb2_get_info(gvdb2_volume *h, gvdb2_info *out) {
    CHECK_HANDLE(h);
    if (!out) return GVDB2_ERR_ARG;
    Volume *v = VOL(h);
    cudaError_t e = cudaStreamSynchronize(v->stream);
    if (e != cudaSuccess) return gvdb2::cuda_fail(v, e, "get_info");
    GV_TRY(gvdb2::flush_status(v));
    std::memset(out, 0, sizeof(*out));
    out->depth = v->depth;
    out->top_level = v->top_level();
    out->num_levels = v->nlev;
    out->apron = v->apron;
    for (int l = 0; l < 10; l++) {
        out->pool_count[l] = v->pool_cnt[l];
        out->res[l] = v->res(l);
        out->range[l] = v->range(l);
    }
    out->used_leaves = v->used_leaves;
    out->atlas_slots = v->atlas_last;
    out->atlas_capacity = v->atlas_cap;
    for (int a = 0; a < 3; a++) {
        out->atlas_subdim[a] = v->subdim[a];
        out->posmin[a] = v->posmin[a];
        out->posmax[a] = v->posmax[a];
        out->root_pos[a] = v->root_pos[a];
    }
    out->tile_res = v->tile_res();
    for (int a = 0; a < 3; a++) {
        out->vol_min[a] = v->vox_min[a];
        out->vol_max[a] = v->vox_max[a];
        out->vox_res[a] = v->vox_res[a];
        out->vox_res_max[a] = v->vox_res_max[a];
    }
    out->splat_cells = -1;
    if (v->bin_key.valid && v->cell_cnt.p) {
        uint32_t c3[3] = {0, 0, 0};
        e = cudaMemcpy(c3, v->cell_cnt.p, sizeof(c3), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return gvdb2::cuda_fail(v, e, "get_info");
        out->splat_cells = (int64_t)c3[0] + c3[1] + c3[2];
    }
    return GVDB2_OK;
}

static gvdb2_status copy_out(Volume *v, void *host, const void *dev, size_t bytes) {
    if (bytes == 0) return GVDB2_OK;
    if (!host || !dev) return gvdb2::fail(v, GVDB2_ERR_STATE, "nothing to copy");
    cudaError_t e = cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, v->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(v->stream);
    if (e != cudaSuccess) return gvdb2::cuda_fail(v, e, "copy to host");
    return GVDB2_OK;
}

gvdb2_status gvdb2_copy_nodes(gvdb2_volume *h, int lev, void *host, int64_t max_nodes) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    if (lev < 0 || lev >= gvdb2::kMaxLev) return GVDB2_ERR_ARG;
    int64_t n = std::min<int64_t>(v->pool_cnt[lev], max_nodes);
    return copy_out(v, host, v->pool[lev].p, (size_t)n * sizeof(gvdb2::Node));
}

gvdb2_status gvdb2_copy_childlists(gvdb2_volume *h, int lev, uint64_t *host, int64_t max_entries) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    if (lev < 1 || lev >= gvdb2::kMaxLev) return GVDB2_ERR_ARG;
    int64_t n = std::min<int64_t>(v->pool_cnt[lev] * v->res3(lev), max_entries);
    return copy_out(v, host, v->clist[lev].p, (size_t)n * sizeof(uint64_t));
}

gvdb2_status gvdb2_copy_atlas(gvdb2_volume *h, int chan, float *host, int64_t max_floats) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    if (chan < 0 || chan >= gvdb2::kMaxChan || !v->has_chan[chan]) return gvdb2::fail(v, GVDB2_ERR_ARG, "bad channel");
    int64_t n = std::min<int64_t>(v->atlas_last * v->tile_vox(), max_floats);
    return copy_out(v, host, v->atlas[chan].p, (size_t)n * sizeof(float));
}

gvdb2_status gvdb2_copy_atlas_map(gvdb2_volume *h, void *host, int64_t max_entries) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    int64_t n = std::min<int64_t>(v->atlas_valid ? v->atlas_cap : 0, max_entries);
    return copy_out(v, host, v->amap.p, (size_t)n * sizeof(gvdb2::AtlasNode));
}

gvdb2_status gvdb2_copy_neighbors(gvdb2_volume *h, int32_t *host, int64_t max_entries) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    if (!v->nbr6_valid) return gvdb2::fail(v, GVDB2_ERR_STATE, "UpdateNeighbors not called");
    int64_t n = std::min<int64_t>(6 * v->pool_cnt[0], max_entries);
    return copy_out(v, host, v->nbr6.p, (size_t)n * sizeof(int32_t));
}

gvdb2_status gvdb2_copy_point_nodes(gvdb2_volume *h, int32_t *pnode, int32_t *poff, int64_t n, int32_t *gcnt,
                                    int64_t ngcnt) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    n = std::min<int64_t>(n, v->pnode_n);
    if (pnode) GV_TRY(copy_out(v, pnode, v->pnode.p, (size_t)n * sizeof(int32_t)));
    if (poff) GV_TRY(copy_out(v, poff, v->poff.p, (size_t)n * sizeof(int32_t)));
    if (gcnt) GV_TRY(copy_out(v, gcnt, v->gcnt.p, (size_t)std::min<int64_t>(ngcnt, v->pool_cnt[0]) * sizeof(int32_t)));
    return GVDB2_OK;
}

gvdb2_status gvdb2_copy_subcells(gvdb2_volume *h, int32_t *cnt, int32_t *nid, int32_t *pos3, int64_t max_subcells) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    int64_t n = std::min<int64_t>(v->num_sc, max_subcells);
    if (cnt) GV_TRY(copy_out(v, cnt, v->sc_cnt.p, (size_t)n * sizeof(int32_t)));
    if (nid) GV_TRY(copy_out(v, nid, v->sc_nid.p, (size_t)n * sizeof(int32_t)));
    if (pos3) GV_TRY(copy_out(v, pos3, v->sc_pos.p, (size_t)n * 3 * sizeof(int32_t)));
    return GVDB2_OK;
}

gvdb2_status gvdb2_copy_subcell_points_fp16(gvdb2_volume *h, uint16_t *pos3, uint16_t *vel3, int64_t max_entries) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    if (!v->sc_fp16) return gvdb2::fail(v, GVDB2_ERR_STATE, "the subcell lists are not the 16-bit ones");
    int64_t n = std::min<int64_t>(v->sc_len, max_entries);
    if (n <= 0) return GVDB2_OK;
    if (pos3) GV_TRY(copy_out(v, pos3, v->sc_q.p, (size_t)n * 3 * sizeof(uint16_t)));
    if (vel3) {
        if (!v->sc_qvel_valid) return gvdb2::fail(v, GVDB2_ERR_STATE, "no velocity lists (SetPoints without velocities)");
        GV_TRY(copy_out(v, vel3, v->sc_qvel.p, (size_t)n * 3 * sizeof(uint16_t)));
    }
    return GVDB2_OK;
}

gvdb2_status gvdb2_atlas_device_ptr(gvdb2_volume *h, int chan, float **dev_ptr) {
    CHECK_HANDLE(h);
    Volume *v = VOL(h);
    if (!dev_ptr || chan < 0 || chan >= gvdb2::kMaxChan || !v->has_chan[chan]) return GVDB2_ERR_ARG;
    *dev_ptr = v->atlas[chan].as<float>();
    return GVDB2_OK;
}

} // extern "C"
