// gvdb2_volume.hpp -- C++ drop-in facade over the gvdb2 C-ABI.
//
// Mirrors the point-path methods of nvdb::VolumeGVDB
// (source/gvdb_library/src/gvdb_volume_gvdb.h:325-562) with the same
// names, argument order and meaning.  Differences a caller sees:
//  - failures throw gvdb2::Error (the reference prints and exits, A:1006-1034);
//  - point data are passed as device pointers with byte stride/offset
//    (DataPtr::gpu / stride / subdim.x of SetDataGPU, V:4872-4880);
//  - channel data live in linear device memory (atlas_ptr) rather than a
//    CUarray/surface object;
//  - the kernel splats, gathers and adjoints have no reference counterpart.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "gvdb2.h"

namespace gvdb2 {

struct Error : std::runtime_error {
    gvdb2_status status;
    Error(gvdb2_status st, const std::string &what) : std::runtime_error(what), status(st) {}
};

struct Vec3F {
    float x = 0, y = 0, z = 0;
};
struct Vec3I {
    int x = 0, y = 0, z = 0;
};

class VolumeGVDB {
  public:
    explicit VolumeGVDB(int device = 0) { check(gvdb2_create(&v_, device), "SetCudaDevice"); }
    ~VolumeGVDB() { gvdb2_destroy(v_); }
    VolumeGVDB(const VolumeGVDB &) = delete;
    VolumeGVDB &operator=(const VolumeGVDB &) = delete;

    gvdb2_volume *handle() const { return v_; }
    void SetStream(void *cuda_stream) { check(gvdb2_set_stream(v_, cuda_stream), "SetStream"); }
    void Initialize() {}

    void Configure(int q4, int q3, int q2, int q1, int q0) { check(gvdb2_configure(v_, q4, q3, q2, q1, q0), "Configure"); }
    void SetChannelDefault(int cx, int cy, int cz) { check(gvdb2_set_channel_default(v_, cx, cy, cz), "SetChannelDefault"); }
    void AddChannel(unsigned char chan, int dt, int apron) { check(gvdb2_add_channel(v_, chan, dt, apron), "AddChannel"); }

    static gvdb2_points_view View(const void *gpu, long long cnt, int offs, int stride) {
        gvdb2_points_view w;
        w.base = gpu;
        w.count = cnt;
        w.stride_bytes = stride;
        w.offset_bytes = offs;
        return w;
    }
    void SetPoints(gvdb2_points_view pos, gvdb2_points_view vel = gvdb2_points_view{},
                   gvdb2_points_view clr = gvdb2_points_view{}) {
        check(gvdb2_set_points(v_, pos, vel, clr), "SetPoints");
    }

    // Batched clouds (no reference counterpart): packs the clouds, each in
    // its own [0, 2^space_log2)^3 space, into this volume's point set and
    // returns each cloud's first packed index (plus the total at the end).
    std::vector<long long> BatchPoints(const std::vector<gvdb2_points_view> &clouds, int space_log2) {
        std::vector<int64_t> first(clouds.size() + 1, 0);
        check(gvdb2_batch_points(v_, clouds.data(), (int)clouds.size(), space_log2, first.data()), "BatchPoints");
        return std::vector<long long>(first.begin(), first.end());
    }
    Vec3I BatchOrigin(int cloud) {
        int32_t o[3] = {0, 0, 0};
        check(gvdb2_batch_origin(v_, cloud, o), "BatchOrigin");
        return Vec3I{o[0], o[1], o[2]};
    }

    void RequestFullRebuild(bool tf) { check(gvdb2_request_full_rebuild(v_, tf ? 1 : 0), "RequestFullRebuild"); }
    void RebuildTopology(int num_pnts, float radius, Vec3F orig = {}) {
        const float o[3] = {orig.x, orig.y, orig.z};
        check(gvdb2_rebuild_topology(v_, num_pnts, radius, o), "RebuildTopology");
    }
    void AccumulateTopology(int num_pnts, float radius, Vec3F orig = {}, int iDepth = 1) {
        const float o[3] = {orig.x, orig.y, orig.z};
        check(gvdb2_accumulate_topology(v_, num_pnts, radius, o, iDepth), "AccumulateTopology");
    }
    void FinishTopology(bool commit = true, bool bounds = true) {
        check(gvdb2_finish_topology(v_, commit ? 1 : 0, bounds ? 1 : 0), "FinishTopology");
    }
    void UpdateAtlas() { check(gvdb2_update_atlas(v_), "UpdateAtlas"); }
    // drops the nodes incremental rebuilds delinked (no reference counterpart)
    void CompactPools() { check(gvdb2_compact_pools(v_), "CompactPools"); }
    // ActivateSpace(Vector3DF): the leaf's pool reference if it existed, else ID_UNDEFL
    uint64_t ActivateSpace(Vec3F pos) {
        const float p[3] = {pos.x, pos.y, pos.z};
        uint64_t out = GVDB2_ID_UNDEFL;
        check(gvdb2_activate_space(v_, p, 1, &out), "ActivateSpace");
        return out;
    }
    void ClearChannel(unsigned char chan) { check(gvdb2_clear_channel(v_, chan), "ClearChannel"); }
    void UpdateNeighbors() { check(gvdb2_update_neighbors(v_), "UpdateNeighbors"); }

    void InsertPoints(int num_pnts, Vec3F trans = {}, bool prefix = false) {
        const float t[3] = {trans.x, trans.y, trans.z};
        check(gvdb2_insert_points(v_, num_pnts, t, prefix ? 1 : 0), "InsertPoints");
    }
    void InsertPointsSubcell(int subcell_size, int num_pnts, float radius, Vec3F trans, int &pSCPntsLength) {
        const float t[3] = {trans.x, trans.y, trans.z};
        check(gvdb2_insert_points_subcell(v_, subcell_size, num_pnts, radius, t, &pSCPntsLength), "InsertPointsSubcell");
    }
    void InsertPointsSubcell_FP16(int subcell_size, int num_pnts, float radius, Vec3F trans, int &pSCPntsLength) {
        const float t[3] = {trans.x, trans.y, trans.z};
        check(gvdb2_insert_points_subcell_fp16(v_, subcell_size, num_pnts, radius, t, &pSCPntsLength),
              "InsertPointsSubcell_FP16");
    }
    void GetMinMaxVel(int num_pnts) { check(gvdb2_get_min_max_vel(v_, num_pnts), "GetMinMaxVel"); }
    void ScatterDensity(int num_pnts, float radius, float amp, Vec3F trans, bool expand = true, bool avgColor = false) {
        const float t[3] = {trans.x, trans.y, trans.z};
        check(gvdb2_scatter_density(v_, num_pnts, radius, amp, t, expand ? 1 : 0, avgColor ? 1 : 0), "ScatterDensity");
    }
    void GatherDensity(int subcell_size, int num_pnts, float radius, Vec3F trans, int &pSCPntsLength, int chanDensity,
                       int chanClr, bool bAccum = false) {
        const float t[3] = {trans.x, trans.y, trans.z};
        check(gvdb2_gather_density(v_, subcell_size, num_pnts, radius, t, &pSCPntsLength, chanDensity, chanClr,
                                   bAccum ? 1 : 0),
              "GatherDensity");
    }
    void GatherLevelSet(int subcell_size, int num_pnts, float radius, Vec3F trans, int &pSCPntsLength, int chanLevelset,
                        int chanClr, bool bAccum = false) {
        const float t[3] = {trans.x, trans.y, trans.z};
        check(gvdb2_gather_level_set(v_, subcell_size, num_pnts, radius, t, &pSCPntsLength, chanLevelset, chanClr,
                                     bAccum ? 1 : 0),
              "GatherLevelSet");
    }
    void GatherLevelSet_FP16(int subcell_size, int num_pnts, float radius, Vec3F trans, int &pSCPntsLength,
                             int chanLevelSet, int chanClr) {
        const float t[3] = {trans.x, trans.y, trans.z};
        check(gvdb2_gather_level_set_fp16(v_, subcell_size, num_pnts, radius, t, &pSCPntsLength, chanLevelSet, chanClr),
              "GatherLevelSet_FP16");
    }
    void SetTransform(Vec3F pretrans, Vec3F scal, Vec3F angs, Vec3F trans) {
        const float p[3] = {pretrans.x, pretrans.y, pretrans.z}, s[3] = {scal.x, scal.y, scal.z},
                    a[3] = {angs.x, angs.y, angs.z}, t[3] = {trans.x, trans.y, trans.z};
        check(gvdb2_set_transform(v_, p, s, a, t), "SetTransform");
    }
    void SaveVBX(const std::string &fname) { check(gvdb2_save_vbx(v_, fname.c_str()), "SaveVBX"); }
    bool LoadVBX(const std::string &fname) {
        check(gvdb2_load_vbx(v_, fname.c_str()), "LoadVBX");
        return true;
    }
    // ExportToNanoVDB (gNanoVDB/gvdb_export_nanovdb.h:65-66): the export in a
    // device buffer the caller owns (at least NanoVDBSize(nv) bytes, 32-byte
    // aligned); nv = GVDB2_NV_FLOAT with one channel, GVDB2_NV_VEC3F with three.
    size_t NanoVDBSize(int nv) {
        size_t n = 0;
        check(gvdb2_nanovdb_size(v_, nv, &n), "ExportToNanoVDB");
        return n;
    }
    void ExportToNanoVDB(int nv, const int32_t *chans, const float *background, const char *grid_name,
                         int32_t grid_class, void *dst_device, size_t dst_bytes) {
        check(gvdb2_export_nanovdb(v_, nv, chans, background, grid_name, grid_class, dst_device, dst_bytes),
              "ExportToNanoVDB");
    }
    // launch settings of the kernel splats and their autotuner (no reference counterpart)
    void SetTuning(const gvdb2_tuning &t) { check(gvdb2_set_tuning(v_, &t), "SetTuning"); }
    gvdb2_tuning GetTuning() {
        gvdb2_tuning t{};
        check(gvdb2_get_tuning(v_, &t), "GetTuning");
        return t;
    }
    void SetTuneCache(const std::string &path) { check(gvdb2_set_tune_cache(v_, path.c_str()), "SetTuneCache"); }
    void SetAutotune(bool on) { check(gvdb2_set_option(v_, GVDB2_OPT_AUTOTUNE, on ? 1 : 0), "SetAutotune"); }
    void UpdateApron() { check(gvdb2_update_apron(v_, -1, 0.0f), "UpdateApron"); }
    void UpdateApron(unsigned char chan, float boundval = 0.0f) {
        check(gvdb2_update_apron(v_, chan, boundval), "UpdateApron");
    }
    void UpdateApronFaces(unsigned char chan) { check(gvdb2_update_apron_faces(v_, chan), "UpdateApronFaces"); }

    // kernel splats and adjoints (no reference counterpart)
    void ScatterKernel(int kernel, int num_pnts, const int *chans, int nch, gvdb2_points_view weight,
                       float weight_const, const gvdb2_points_view *attrs, Vec3F trans = {}) {
        const float t[3] = {trans.x, trans.y, trans.z};
        check(gvdb2_scatter_kernel(v_, kernel, num_pnts, t, weight, weight_const, attrs, chans, nch), "ScatterKernel");
    }
    void GatherKernel(int kernel, int num_pnts, const int *chans, int nch, float *out, long long out_stride,
                      Vec3F trans = {}) {
        const float t[3] = {trans.x, trans.y, trans.z};
        check(gvdb2_gather_kernel(v_, kernel, num_pnts, t, chans, nch, out, out_stride), "GatherKernel");
    }
    void ScatterDensityBackward(int kernel, int num_pnts, const int *grad_chans, int nch, gvdb2_points_view weight,
                                float weight_const, const gvdb2_points_view *attrs, float *grad_pos, float *grad_weight,
                                float *grad_attr, Vec3F trans = {}) {
        const float t[3] = {trans.x, trans.y, trans.z};
        check(gvdb2_scatter_kernel_backward(v_, kernel, num_pnts, t, weight, weight_const, attrs, nch, grad_chans,
                                            grad_pos, grad_weight, grad_attr),
              "ScatterDensityBackward");
    }
    void GatherDensityBackward(int kernel, int num_pnts, const int *chans, int nch, const float *grad_out,
                               const int *grad_chans, float *grad_pos, Vec3F trans = {}) {
        const float t[3] = {trans.x, trans.y, trans.z};
        check(gvdb2_gather_kernel_backward(v_, kernel, num_pnts, t, chans, nch, grad_out, grad_chans, grad_pos),
              "GatherDensityBackward");
    }

    // inspection
    gvdb2_info Info() {
        gvdb2_info i;
        check(gvdb2_get_info(v_, &i), "Info");
        return i;
    }
    long long getNumTotalNodes(int lev) { return Info().pool_count[lev]; }
    // getVolMin / getVolMax (gvdb_volume_base.h:57-59): the bounds of the
    // last FinishTopology(commit, true), i.e. ComputeBounds (V:1792-1816)
    Vec3F getVolMin() {
        gvdb2_info i = Info();
        return Vec3F{i.vol_min[0], i.vol_min[1], i.vol_min[2]};
    }
    Vec3F getVolMax() {
        gvdb2_info i = Info();
        return Vec3F{i.vol_max[0], i.vol_max[1], i.vol_max[2]};
    }
    long long getNumUsedNodes(int lev) {
        gvdb2_info i = Info();
        return lev == 0 ? i.used_leaves : i.pool_count[lev];
    }
    float *atlas_ptr(int chan) {
        float *p = nullptr;
        check(gvdb2_atlas_device_ptr(v_, chan, &p), "atlas_ptr");
        return p;
    }

  private:
    void check(gvdb2_status st, const char *what) {
        if (st != GVDB2_OK) throw Error(st, std::string(what) + ": " + (v_ ? gvdb2_last_error(v_) : "no volume"));
    }
    gvdb2_volume *v_ = nullptr;
};

} // namespace gvdb2
