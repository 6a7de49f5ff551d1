// gvdb2_internal.h -- host-side state and shared declarations of the
// B200-native point -> sparse-volume pipeline (libgvdb2).
//
// Layout contracts kept from the reference (paths relative to gvdb-voxels):
//   Node        : 64 bytes, source/gvdb_library/src/gvdb_node.h:27-40
//   child lists : 8*res^3 bytes per interior node of pool group 1 (V:2424-2426)
//   pool refs   : grp | lev<<8 | ndx<<16 (gvdb_allocator.h:59-62)
//   brick keys  : lev<<48 | x<<32 | y<<16 | z (P:352-382)
// The atlas departs from the reference's CUarray: per channel a linear run
// of (res+2*apron)^3-float tiles, one per atlas slot, z-major.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <string>
#include <vector>

#include "gvdb2.h"

namespace gvdb2 {

constexpr int kMaxLev = 10;      // MAXLEV, gvdb_volume_gvdb.h:40
constexpr int kMaxChan = 32;     // MAX_CHANNEL, N:22
constexpr int kMaxSplatChan = 8; // channels one kernel splat call may touch
constexpr uint64_t kUndefL = 0xFFFFFFFFull;
constexpr uint64_t kUndef64 = 0xFFFFFFFFFFFFFFFFull;
constexpr uint64_t kEmptyKey = 0xFFFFFFFFFFFFFFFFull;
constexpr float kNoHit = 1.0e10f; // NOHIT, gvdb_types.h:52

struct __align__(16) Node {
    uint8_t mLev, mFlags, mPriority, pad;
    int32_t mPos[3];
    int32_t mValue[3];
    float mVRange[3];
    uint64_t mParent;
    uint64_t mChildList;
    uint64_t mMask;
};
static_assert(sizeof(Node) == 64, "Node must keep the reference's 64-byte layout");

struct AtlasNode {
    int32_t mPos[3];
    int32_t mLeafID;
};
static_assert(sizeof(AtlasNode) == 16, "AtlasNode is 16 bytes");

struct PointsView {
    const char *base = nullptr;
    int64_t count = 0;
    int32_t stride = 0;
    int32_t offset = 0;
    // batched clouds: per-point cloud index and per-cloud integer voxel
    // origin (3 ints).  Positions stay in the cloud's own index space; the
    // origin is added to integer grid coordinates only, after floor and
    // fraction are taken, so no position bit is lost to the offset.
    const int32_t *cloud = nullptr;
    const int32_t *origin = nullptr;
};

// Open-addressed hash set / map of 64-bit brick keys (linear probing).
struct HashTable {
    uint64_t *keys;   // kEmptyKey = free
    int32_t *vals;    // optional payload (map)
    uint32_t mask;    // capacity - 1 (power of two)
    int32_t *count;   // device counter of inserted keys
};

// Device-resident status word set by kernels (never trap).
enum DevStatusBits : int32_t {
    kDevHashFull = 1,
    kDevCapacity = 2,
    kDevBadIndex = 4,
    kDevTimeout = 8, // a bounded wait (bulk copy completion) ran out
};

// Growable device buffer, stream-ordered (cudaMallocAsync / cudaFreeAsync
// on the stream that last grew it).  Non-copyable; frees itself.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    cudaError_t ensure(size_t need, cudaStream_t s, bool preserve = false);
    void release();
    template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

struct Volume {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int deterministic = 0; // stable binning: kernel splats reproduce bit for bit

    // configuration (Configure, V:2364-2434)
    int nlev = 0;
    int logdim[kMaxLev] = {0};
    int default_axiscnt[3] = {16, 16, 1}; // SetChannelDefault(16,16,1), V:2348
    // grid transform (SetTransform, V:5770; default V:77): kept and written
    // to VBX files, not applied by the point path
    float xf_pretrans[3] = {0, 0, 0}, xf_angs[3] = {0, 0, 0}, xf_scale[3] = {1, 1, 1}, xf_trans[3] = {0, 0, 0};

    // channels / atlas
    bool has_chan[kMaxChan] = {false};
    int apron = 0;
    int subdim[3] = {0, 0, 0};
    int64_t atlas_cap = 0;    // bricks the atlas holds
    int64_t atlas_last = 0;   // slots in use (lastEle)
    DevBuf atlas[kMaxChan];   // float tiles
    DevBuf amap;              // AtlasNode per atlas brick
    DevBuf slot_leaf;         // int32 per slot: leaf pool index
    DevBuf leaf_slot;         // int32 per pool leaf: slot or -1
    DevBuf nbr27;             // int32 per slot x 27: neighbour slots
    DevBuf nbr6;              // int32 per pool leaf x 6 (UpdateNeighbors)
    DevBuf apron_list;        // int2 per apron voxel of a tile (UpdateApron)
    int apron_list_n = 0, apron_list_key = -1;
    bool nbr6_valid = false;
    bool atlas_valid = false; // slots assigned for the current topology

    // points (SetPoints, V:4900-4908)
    PointsView pos{}, vel{}, clr{};

    // topology state (host mirrors of device pools)
    bool rebuild_topo = true; // V:2355
    int cur_depth = -1;       // V:2356
    int depth = 0;
    int root_pos[3] = {0, 0, 0};
    float posmin[3] = {0, 0, 0}, posmax[3] = {0, 0, 0};
    // ComputeBounds (V:1792-1816): mVoxMin/mVoxMax (= mObjMin/mObjMax, what
    // getVolMin/getVolMax return), mVoxRes and the largest mVoxRes so far
    float vox_min[3] = {0, 0, 0}, vox_max[3] = {0, 0, 0}, vox_res[3] = {0, 0, 0}, vox_res_max[3] = {0, 0, 0};
    int64_t pool_cnt[kMaxLev] = {0};
    int64_t used_leaves = 0;
    // every pool leaf is flagged (true right after a full rebuild): UpdateAtlas
    // then knows its slot count without reading it back
    bool all_leaves_flagged = false;
    // the device status word of the last full rebuild is checked at the
    // next read-back of the small device words instead of by a read of its own
    bool status_pending = false;
    // a splat kernel ran since the last read-back of the small device words:
    // their splat guard word is checked then
    bool splat_guard_pending = false;
    DevBuf pool[kMaxLev];     // Node arrays
    DevBuf clist[kMaxLev];    // uint64 child lists (lev >= 1)
    uint64_t topo_version = 0;
    int64_t pool_reserved_for = 0; // point count the stream-ordered pool was grown for

    // leaf lookup: level-0 key -> leaf pool index (flagged, i.e. linked, leaves only)
    DevBuf leafmap_keys, leafmap_vals;
    uint32_t leafmap_mask = 0;
    // the leaf map holds exactly the leaves linked in the tree (true after a
    // rebuild; pools adopted from a file or the host tree may hold linked
    // leaves that are not flagged), so the incremental marking may look
    // leaves up there instead of walking from the root
    bool leafmap_is_tree = false;

    // scratch for the rebuild
    DevBuf hs_keys[2];        // hash sets (base, box)
    DevBuf bits;              // brick bitmaps per level (base, box) of the bitmap rebuild
    DevBuf bits_chunks;       // per-chunk set-bit counts of the large-grid compaction
    uint32_t hs_mask = 0;
    DevBuf lev_keys[kMaxLev][2]; // sorted unique keys per level: [0]=base [1]=extra (or new)
    int64_t lev_count[kMaxLev][2] = {{0}};
    DevBuf tmp_a, tmp_b, tmp_c, scratch;
    DevBuf dev_small;         // small device words: counters, status, bbox
    void *host_small = nullptr; // pinned mirror of dev_small

    // batched clouds (gvdb2_batch_points): the packed positions
    DevBuf batch_pos, batch_cloud, batch_origin;
    int batch_clouds = 0, batch_space_log2 = 0;

    // InsertPoints results
    DevBuf pnode, poff, gcnt, goff, psorted;
    int64_t pnode_n = 0;

    // kernel-splat binning: per point its (cell, region) bin and rank, the
    // points in bin order (perm), each (cell, region) bin's first entry
    // (reg_off, 27 per cell) and each cell's (bin_off)
    DevBuf pbin, prank, bin_cnt, bin_off, reg_off, perm;
    // the binned points' data in bin order, so that the splat kernels read
    // a cell's points contiguously: per entry of perm the translated
    // position and the cloud index (float4, w = int bits, -1 outside a
    // batch), made with the bins; and the splat's channel amounts (float4),
    // made by each scatter call
    DevBuf bin_pos, bin_amt;
    // the scatter's dense cells: per cell its partial slot or -1
    // (cell_part); the work items (cell, slice, slices, accumulator slot;
    // part_work); the partial sums, 12^3 or 10^3 floats per dense cell and
    // channel (part_buf); the integer accumulators and arrival counters of
    // cells splatted by several CTAs (part_acc, part_done: zero between
    // calls); their capacities
    DevBuf cell_part, part_work, part_buf, part_acc, part_done;
    // cells whose voxels k_scatter_merge adds partials to (count in the
    // last 16 bytes)
    DevBuf merge_list;
    int64_t dense_cap = 0, work_cap = 0, multi_cap = 0, part_acc_cap = 0;
    // cells that hold points: huge and heavy ones (order of cell_at), light
    // ones and the counts (kCnt*); heavy_grid, light_grid and cell_grid
    // bound the huge+heavy, light and all lists
    DevBuf cell_list, cell_light, cell_cnt;
    int64_t cell_grid = 0, heavy_grid = 0, light_grid = 0;
    struct BinKey {
        bool valid = false;
        int kernel = 0;
        int64_t n = 0;
        PointsView pos{};
        float trans[3] = {0, 0, 0};
        uint64_t topo = 0;
        bool det = false;
        int32_t tune[3] = {0, 0, 0}; // dense, slice, light thresholds the cell lists were made with
    } bin_key;

    // launch settings of the kernel splats (gvdb2_tuning): cells of at least
    // `dense` points take the scatter's partial-sum path (0: none), `slice`
    // points per CTA there; cells of at most `light` points are gathered a
    // warp per cell.  Defaults 512, 4096, 32; the autotuner (tune.cu) picks
    // others per workload class.
    int32_t tune_dense = 512, tune_slice = 4096, tune_light = 32;
    bool autotune = false;   // GVDB2_OPT_AUTOTUNE: apply cached settings per call
    std::string tune_cache;  // on-disk cache path ("" = GVDB2_TUNE_CACHE, else none)

    // subcells (InsertPointsSubcell)
    DevBuf sc_map, sc_flag, sc_cnt, sc_off, sc_nid, sc_pos, sc_pnt;
    // InsertPointsSubcell_FP16: 16-bit entries (3 per list entry) over the
    // bounding box of the last rebuild; velocities over velmin/velrange
    DevBuf sc_q, sc_qvel;
    bool sc_fp16 = false, sc_qvel_valid = false;
    float velmin[3] = {0, 0, 0}, velrange[3] = {0, 0, 0}; // GetMinMaxVel; zero until computed
    int sc_size = 0, sc_dim = 0, sc_per_brick = 0;
    int64_t num_sc = 0, sc_len = 0;

    // ---- helpers ----
    int res(int lev) const { return lev < 0 ? 1 : (1 << logdim[lev]); }
    int64_t res3(int lev) const {
        int64_t r = res(lev);
        return r * r * r;
    }
    int64_t range(int lev) const {
        if (lev < 0) return 1;
        int64_t r = res(0);
        for (int l = 1; l <= lev; l++) r *= res(l);
        return r;
    }
    int tile_res() const { return res(0) + 2 * apron; }
    int64_t tile_vox() const {
        int64_t t = tile_res();
        return t * t * t;
    }
    int top_level() const {
        int tlev = 1; // PrepareVDB, V:3952-3965
        for (int n = nlev - 1; n >= 0; n--)
            if (pool_cnt[n] == 1) tlev = n;
        return tlev;
    }
    bool any_channel() const {
        for (int c = 0; c < kMaxChan; c++)
            if (has_chan[c]) return true;
        return false;
    }
    Node *pool_ptr(int lev) const { return pool[lev].as<Node>(); }
};

// status helpers
gvdb2_status fail(Volume *v, gvdb2_status st, const std::string &msg);
gvdb2_status cuda_fail(Volume *v, cudaError_t e, const char *what);

#define GV_CUDA(v, call)                                         \
    do {                                                         \
        cudaError_t e__ = (call);                                \
        if (e__ != cudaSuccess) return ::gvdb2::cuda_fail((v), e__, #call); \
    } while (0)
#define GV_TRY(expr)                          \
    do {                                      \
        gvdb2_status s__ = (expr);            \
        if (s__ != GVDB2_OK) return s__;      \
    } while (0)

// ---- primitives.cu ----
// exclusive scan of n uint32 -> out[0..n], out[n] = total
gvdb2_status exclusive_scan_u32(Volume *v, const uint32_t *in, uint32_t *out, int64_t n);
// stable LSD radix sort of n uint64 keys (optionally with int32 values) over
// bits [lo_bit, hi_bit); the sorted result is written back to keys/vals.
gvdb2_status radix_sort_u64(Volume *v, uint64_t *keys, int32_t *vals, int64_t n, int lo_bit, int hi_bit);

// ---- topology.cu ----
gvdb2_status rebuild_topology(Volume *v, int n, float radius, const float orig[3], bool accumulate, int min_depth);
gvdb2_status update_atlas(Volume *v);
gvdb2_status alloc_channel_storage(Volume *v, int chan);
gvdb2_status pool_reserve(Volume *v, int lev, int64_t cnt);
gvdb2_status adopt_pools(Volume *v, int depth);
gvdb2_status activate_space(Volume *v, const float *xyz, int64_t n, uint64_t *out);
gvdb2_status compact_pools(Volume *v);
gvdb2_status save_vbx(Volume *v, const char *path);
// ---- tune.cu ----
gvdb2_status set_tuning(Volume *v, const gvdb2_tuning *t);
gvdb2_tuning get_tuning(const Volume *v);
std::string tune_key(Volume *v, const char *op, int kernel, int nch, int64_t n);
void apply_cached_tuning(Volume *v, const char *op, int kernel, int nch, int64_t n);
gvdb2_status cache_get(const char *path, const char *key, gvdb2_tuning *t, float *ms);
gvdb2_status cache_put(const char *path, const char *key, const gvdb2_tuning *t, float ms);
gvdb2_status autotune(Volume *v, const char *op, int kernel, int nch, int64_t n, const std::vector<gvdb2_tuning> &cands,
                      const std::function<gvdb2_status()> &call, gvdb2_tuning *chosen);
std::vector<gvdb2_tuning> scatter_candidates(const Volume *v);
std::vector<gvdb2_tuning> gather_candidates(const Volume *v);
// ---- nanovdb.cu ----
gvdb2_status nanovdb_size(Volume *v, int value_type, size_t *bytes);
gvdb2_status export_nanovdb(Volume *v, int value_type, const int32_t *chans, const float *background,
                            const char *grid_name, int32_t grid_class, void *dst_device, size_t dst_bytes);
gvdb2_status load_vbx(Volume *v, const char *path);
gvdb2_status update_neighbors(Volume *v);
gvdb2_status clear_channel(Volume *v, int chan);
gvdb2_status compute_bounds(Volume *v);
gvdb2_status sync_counts(Volume *v);
// reads back the small device words when a full rebuild's status check is
// pending and reports its error, if any
gvdb2_status flush_status(Volume *v);
// the small device word the splat kernels flag an out-of-range index in
// (nullptr before the first rebuild)
int32_t *splat_guard_word(Volume *v);

// ---- points.cu ----
gvdb2_status insert_points(Volume *v, int n, const float trans[3], int prefix);
gvdb2_status bin_points(Volume *v, int kernel, int n, const float trans[3]);
gvdb2_status insert_points_subcell(Volume *v, int sc, int n, float radius, const float trans[3], int *len,
                                   bool fp16 = false);
gvdb2_status get_min_max_vel(Volume *v, int n);

// ---- splat.cu ----
// 1 to kMaxSplatChan channels, each one that the volume holds
gvdb2_status check_chans(Volume *v, const int *chans, int nch);
gvdb2_status scatter_density_ref(Volume *v, int n, float radius, float amp, const float trans[3], int expand);
gvdb2_status gather_voxels(Volume *v, int sc, float radius, int chan, int accum, bool levelset, bool fp16 = false);
gvdb2_status scatter_kernel(Volume *v, int kernel, int n, const float trans[3], gvdb2_points_view weight,
                            float weight_const, const gvdb2_points_view *attrs, const int *chans, int nch);
gvdb2_status gather_kernel(Volume *v, int kernel, int n, const float trans[3], const int *chans, int nch, float *out,
                           int64_t out_stride);
// gather_kernel with the binning supplied by the caller: bin_off[s] is the
// first entry of slot s in perm and bin_off[s + 1] one past its last
gvdb2_status gather_kernel_prebinned(Volume *v, int kernel, int n, const float trans[3], const int *chans, int nch,
                                     float *out, int64_t out_stride, const uint32_t *bin_off, const int32_t *perm);
gvdb2_status scatter_kernel_backward(Volume *v, int kernel, int n, const float trans[3], gvdb2_points_view weight,
                                     float weight_const, const gvdb2_points_view *attrs, int nch,
                                     const int *grad_chans, float *grad_pos, float *grad_weight, float *grad_attr);
gvdb2_status gather_kernel_backward(Volume *v, int kernel, int n, const float trans[3], const int *chans, int nch,
                                    const float *grad_out, const int *grad_chans, float *grad_pos);

// ---- batch.cu ----
int batch_grid(int ncloud);
void batch_origin(int cloud, int ncloud, int space_log2, int32_t out[3]);
gvdb2_status batch_points(Volume *v, const gvdb2_points_view *clouds, int ncloud, int space_log2, int64_t *first);

// ---- apron.cu ----
gvdb2_status update_apron(Volume *v, int chan, float boundval);
gvdb2_status update_apron_faces(Volume *v, int chan);

inline PointsView to_view(gvdb2_points_view w) {
    PointsView p;
    p.base = reinterpret_cast<const char *>(w.base);
    p.count = w.count;
    p.stride = w.stride_bytes;
    p.offset = w.offset_bytes;
    return p;
}

} // namespace gvdb2
