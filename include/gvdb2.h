/*
 * gvdb2.h -- C-ABI of the B200-native point -> sparse-volume pipeline.
 *
 * Each entry point replaces the nvdb::VolumeGVDB method (or kernel launch
 * sequence) cited beside it; paths are relative to the gvdb-voxels project:
 *   V  = source/gvdb_library/src/gvdb_volume_gvdb.cpp
 *   VH = source/gvdb_library/src/gvdb_volume_gvdb.h
 *
 * Conventions
 *  - Every call returns a gvdb2_status; nothing exits, traps or prints.
 *    gvdb2_last_error() gives a message for the last failure of a volume.
 *  - Point views and gather outputs are DEVICE pointers (the reference's
 *    SetDataGPU contract, V:4872-4880): element i of a view lives at
 *    base + i*stride_bytes + offset_bytes.  Views are non-owning.
 *  - All work is issued on the volume's stream (gvdb2_set_stream); calls
 *    that return a host value (counts, lengths) synchronise that stream.
 *  - The atlas is linear device memory: per channel, one contiguous tile of
 *    (res+2*apron)^3 floats per atlas slot, z-major (x fastest).  Node
 *    pools keep the 64-byte nvdb::Node layout and 8*res^3-byte child lists.
 */
#ifndef GVDB2_H
#define GVDB2_H

#include <stddef.h>
#include <stdint.h>

#if defined(_WIN32)
#define GVDB2_API __declspec(dllexport)
#else
#define GVDB2_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef int gvdb2_status;
#define GVDB2_OK 0
#define GVDB2_ERR_ARG 1          /* invalid argument */
#define GVDB2_ERR_DEPTH 2        /* point extents smaller than one brick or deeper than 5 levels (V:1187-1194) */
#define GVDB2_ERR_STATE 3        /* call order violated (e.g. gather before topology) */
#define GVDB2_ERR_UNSUPPORTED 4  /* configuration outside what this build implements */
#define GVDB2_ERR_NOMEM 5        /* device allocation failed */
#define GVDB2_ERR_CUDA 6         /* a CUDA runtime call failed */
#define GVDB2_ERR_CAPACITY 7     /* a device-side capacity check fired; nothing was written out of bounds */
#define GVDB2_ERR_NOT_AVAILABLE 8 /* CUDA device or kernel image not available */

#define GVDB2_T_FLOAT 3          /* channel type T_FLOAT (gvdb_types.h) */

#define GVDB2_KERNEL_TENT1 1     /* trilinear tent, radius 1 voxel, voxel centres at i+0.5 */
#define GVDB2_KERNEL_CUBIC2 2    /* cubic B-spline, radius 2 voxels */

#define GVDB2_OPT_DETERMINISTIC 1 /* 1: stable binning, so kernel splats and gathers are bit-reproducible */
#define GVDB2_OPT_AUTOTUNE 2      /* 1: kernel splats and gathers take their workload class's cached tuning */

typedef struct gvdb2_volume gvdb2_volume;

typedef struct gvdb2_points_view {
    const void *base;     /* device pointer (NULL = absent) */
    int64_t count;
    int32_t stride_bytes; /* DataPtr::stride */
    int32_t offset_bytes; /* DataPtr::subdim.x */
} gvdb2_points_view;

typedef struct gvdb2_info {
    int32_t depth;            /* root level (DetermineDepth, V:821-837) */
    int32_t top_level;        /* VDBInfo::top_lev (V:3952-3965) */
    int32_t num_levels;       /* configured levels (5) */
    int32_t apron;
    int64_t pool_count[10];   /* getNumTotalNodes per level */
    int64_t used_leaves;      /* getNumUsedNodes(0) */
    int64_t atlas_slots;      /* atlas lastEle (active bricks) */
    int64_t atlas_capacity;   /* bricks the atlas holds */
    int32_t atlas_subdim[3];  /* atlas brick counts per axis */
    int32_t res[10];          /* getRes per level */
    int64_t range[10];        /* getRange per level */
    float posmin[3];          /* mPosMin after GetBoundingBox (V:5450-5460) */
    float posmax[3];
    int32_t root_pos[3];
    int32_t tile_res;         /* res0 + 2*apron */
    int64_t splat_cells;      /* 8^3 brick cells holding points at the last kernel-splat
                                 binning, -1 before one (no counterpart in the reference) */
    /* ComputeBounds (V:1792-1816), set by FinishTopology(bounds): */
    float vol_min[3];         /* getVolMin (gvdb_volume_base.h:57): mObjMin = mVoxMin */
    float vol_max[3];         /* getVolMax (gvdb_volume_base.h:59): mObjMax = mVoxMax */
    float vox_res[3];         /* mVoxRes = mVoxMax - mVoxMin */
    float vox_res_max[3];     /* mVoxResMax, the largest mVoxRes so far */
} gvdb2_info;

/* ---- lifetime (SetCudaDevice VH:325 / V:240-334, Initialize VH:326 / V:2320-2361) ---- */
GVDB2_API gvdb2_status gvdb2_create(gvdb2_volume **out, int device);
GVDB2_API gvdb2_status gvdb2_destroy(gvdb2_volume *v);
GVDB2_API const char *gvdb2_last_error(const gvdb2_volume *v);
GVDB2_API gvdb2_status gvdb2_set_stream(gvdb2_volume *v, void *cuda_stream);
GVDB2_API gvdb2_status gvdb2_synchronize(gvdb2_volume *v);
GVDB2_API gvdb2_status gvdb2_set_option(gvdb2_volume *v, int option, int value);

/* ---- configuration ---- */
GVDB2_API gvdb2_status gvdb2_configure(gvdb2_volume *v, int q4, int q3, int q2, int q1, int q0);   /* Configure, VH:387 / V:2364-2377 */
GVDB2_API gvdb2_status gvdb2_set_channel_default(gvdb2_volume *v, int cx, int cy, int cz);       /* SetChannelDefault, VH:390 */
GVDB2_API gvdb2_status gvdb2_add_channel(gvdb2_volume *v, int chan, int dtype, int apron);       /* AddChannel, VH:392 / V:2437-2453 */
/* Grid transform (SetTransform, V:5770; default pre-translation 0, scale 1,
 * angles 0, translation 0, V:77): kept and stored in VBX files; the point
 * path works in index space and does not apply it. */
GVDB2_API gvdb2_status gvdb2_set_transform(gvdb2_volume *v, const float pretrans[3], const float scale[3],
                                 const float angs[3], const float trans[3]);
GVDB2_API gvdb2_status gvdb2_get_transform(gvdb2_volume *v, float pretrans[3], float scale[3], float angs[3],
                                 float trans[3]);

/* ---- VBX files (GVDB_FILESPEC.txt) ---- */
/* SaveVBX (V:1626-1768): version 1.11, one grid of float channels in atlas
 * layout with the GVDB topology, byte for byte as the reference writes it
 * (the grid name is written as zeros). */
GVDB2_API gvdb2_status gvdb2_save_vbx(gvdb2_volume *v, const char *path);
/* LoadVBX (V:507-685): replaces the configuration, topology and channels
 * with the file's, then assigns the atlas (UpdateAtlas) and fills it.
 * Files with node bitmasks, other data types, compression, brick layout or
 * other than 5 levels return GVDB2_ERR_UNSUPPORTED. */
GVDB2_API gvdb2_status gvdb2_load_vbx(gvdb2_volume *v, const char *path);

/* ---- NanoVDB-form export (gNanoVDB/gvdb_export_nanovdb.h:65-66) ----
 * ExportToNanoVDB (gvdb_export_nanovdb.cpp:379-700, cuda_export_nanovdb.cu:
 * 76-432) written into one device buffer the caller owns, in NanoVDB's
 * section order: grid header (grid, tree and root fields), root tiles,
 * level-2 nodes, level-1 nodes, leaves.  Each GVDB node of levels 0-2 becomes
 * the record of the same pool index; values come from the atlas channel(s):
 * GVDB2_NV_FLOAT reads chans[0], GVDB2_NV_VEC3F reads chans[0..2] as x, y, z
 * (the reference reads one T_FLOAT3 channel; channels here are floats).
 * Records are this library's (below), not NanoVDB's own structs, whose byte
 * layout depends on the NanoVDB version: a consumer with NanoVDB copies the
 * fields across.  Field rules, as the reference sets them:
 *   leaf: value mask all on; values in (x*T + y)*T + z order; min/max over
 *     the brick; bbox_min = mPos, bbox_dif = T (the brick width); a leaf left
 *     stale by an incremental rebuild has no atlas brick and is written as
 *     zeros (the record the reference's exporter means to leave for nodes
 *     no longer in the tree);
 *   level-1/2 node: value mask off; child mask and table in (x*T + y)*T + z
 *     order (GVDB's child lists are (z*T + y)*T + x), a child's pool index or
 *     the background; offset = nodes of the level - index; min/max and box
 *     over the children's;
 *   root: one tile per level-2 node, keyed by its box corner >> (sum of the
 *     three log2 dims), 21 bits per axis, z lowest, sorted by key (ties by
 *     node index); box and min/max over those nodes (a float grid's maximum
 *     starts at FLT_MIN, as the reference's numeric_limits<float>::min());
 *     active voxels = leaves in the pool x T^3.
 * Log2 dims of levels 0-2 must lie in [2, 7] and the volume needs at least
 * three levels.  gvdb2_nanovdb_size gives the buffer size; the export checks
 * it and returns GVDB2_ERR_CAPACITY when dst_bytes is smaller.  The device
 * work runs on the volume's stream; the root is finished on the host from the
 * level-2 nodes' headers (one read-back), as the reference does. */
#define GVDB2_NV_MAGIC 0x31564e3242445647ull /* "GVDB2NV1" */
#define GVDB2_NV_FLOAT 1                     /* GridType Float: one float per voxel */
#define GVDB2_NV_VEC3F 3                     /* GridType Vec3f: three floats per voxel */
#define GVDB2_NV_HEADER 64                   /* bytes of a node's or a leaf's header */

typedef struct gvdb2_nv_grid {
    uint64_t magic;           /* GVDB2_NV_MAGIC */
    uint64_t total_bytes;     /* whole buffer */
    uint32_t value_type;      /* GVDB2_NV_FLOAT or GVDB2_NV_VEC3F (floats per value) */
    uint32_t grid_class;      /* as given (nanovdb::GridClass numbering) */
    int32_t log2dim[3];       /* leaf, level-1, level-2 */
    uint32_t pad0;
    uint64_t record_bytes[3]; /* record size of a leaf, a level-1, a level-2 node */
    uint64_t section[4];      /* byte offsets from the buffer's start: leaves, level-1, level-2, tiles */
    uint64_t count[4];        /* leaves, level-1 nodes, level-2 nodes, 1 (the root) */
    char name[256];           /* grid name, zero padded */
    float index_to_world[16]; /* the volume's transform (SetTransform, V:5770-5798), column-major:
                                 world = M (i, j, k, 1) */
    double voxel_size[3];     /* |M e_a - M 0| per axis */
    double world_bbox[6];     /* the root box's 8 corners through M: min xyz, max xyz */
    uint64_t active_voxels;   /* root */
    uint32_t tile_count;
    uint32_t pad1;
    int32_t bbox[6];          /* root box: min xyz, max xyz */
    float background[3];
    float vmin[3], vmax[3];   /* root min/max (floats past value_type are 0) */
    uint32_t pad2[3];
} gvdb2_nv_grid;

typedef struct gvdb2_nv_tile {
    uint64_t key;   /* (z >> s) | (y >> s) << 21 | (x >> s) << 42 of the node's box corner */
    uint32_t child; /* level-2 node index */
    uint32_t state; /* 0 */
} gvdb2_nv_tile;

/* Header of a level-1/2 node record; then the value mask (T^3/64 uint64,
 * all off), the child mask (T^3/64 uint64), and T^3 table entries of
 * value_type floats (a child's index as a uint32 in the first word, the rest
 * 0, or the background).  Records are padded to 32 bytes. */
typedef struct gvdb2_nv_node {
    int32_t bbox_min[3], bbox_max[3];
    uint32_t offset; /* nodes of this level - this node's index */
    uint32_t flags;  /* 0 */
    float vmin[3], vmax[3];
    uint32_t pad[2];
} gvdb2_nv_node;

/* Header of a leaf record; then the value mask (T^3/64 uint64), then T^3
 * values of value_type floats.  Records are padded to 32 bytes. */
typedef struct gvdb2_nv_leaf {
    int32_t bbox_min[3];
    uint8_t bbox_dif[3];
    uint8_t flags; /* 0 */
    float vmin[3], vmax[3];
    uint32_t pad[6];
} gvdb2_nv_leaf;

GVDB2_API gvdb2_status gvdb2_nanovdb_size(gvdb2_volume *v, int value_type, size_t *bytes);
GVDB2_API gvdb2_status gvdb2_export_nanovdb(gvdb2_volume *v, int value_type, const int32_t *chans,
                                            const float *background, const char *grid_name, int32_t grid_class,
                                            void *dst_device, size_t dst_bytes);

/* ---- points (SetPoints VH:541 / V:4900-4908) ---- */
/* Non-owning views, as the reference's DataPtr.  The kernel splats and
 * gathers bin the points by cell once and reuse the bins while the topology,
 * the point view (base, count, stride, offset) and the translation stay the
 * same.  A caller that changes the positions in place (an advect step on the
 * same buffer) calls gvdb2_set_points again, or rebuilds the topology, before
 * the next splat or gather: either drops the bins.  The bins hold a copy of
 * the positions they were made from, so splats and gathers that reuse bins
 * across positions moved in place see the positions of the binning, as the
 * reference's kernels see its sorted point copy from a stale InsertPoints. */
GVDB2_API gvdb2_status gvdb2_set_points(gvdb2_volume *v, gvdb2_points_view pos, gvdb2_points_view vel, gvdb2_points_view clr);

/* Batched clouds (no counterpart in the reference, which holds one cloud
 * per VolumeGVDB).  Packs `ncloud` clouds, each with positions in its own
 * index space [0, 2^space_log2)^3, into one point set owned by the volume and
 * makes it the volume's points (velocity and colour views are cleared).  The
 * following calls with the total count process every cloud at once;
 * per-point inputs and outputs (attributes, weights, gathered values) are in
 * packed order, cloud after cloud.  first[c] receives the packed index of
 * cloud c's first point (first[ncloud] = total; pass NULL to skip).  Cloud c
 * is placed at the integer voxel origin gvdb2_batch_origin(c); positions
 * keep their own coordinates (the origin is added to grid indices, not to
 * the floats), so a cloud's bricks, voxel values and gathered values equal,
 * bit for bit, those of a volume of its own.  InsertPoints and
 * InsertPointsSubcell take one cloud per volume and return
 * GVDB2_ERR_UNSUPPORTED for a batch. */
GVDB2_API gvdb2_status gvdb2_batch_points(gvdb2_volume *v, const gvdb2_points_view *clouds, int ncloud, int space_log2,
                                          int64_t *first);
/* Voxel offset of cloud `cloud` in the packed set of gvdb2_batch_points. */
GVDB2_API gvdb2_status gvdb2_batch_origin(gvdb2_volume *v, int cloud, int32_t out[3]);

/* ---- topology ---- */
GVDB2_API gvdb2_status gvdb2_request_full_rebuild(gvdb2_volume *v, int flag);                     /* RequestFullRebuild, VH:432 */
GVDB2_API gvdb2_status gvdb2_rebuild_topology(gvdb2_volume *v, int n, float radius, const float orig[3]);  /* RebuildTopology, V:1181-1218 */
GVDB2_API gvdb2_status gvdb2_accumulate_topology(gvdb2_volume *v, int n, float radius, const float orig[3], int min_depth); /* AccumulateTopology, V:1158-1178 */
/* FinishTopology, V:1579-1593: with `bounds`, ComputeBounds (V:1792-1816) over
 * the leaves (read back into gvdb2_info vol_min/vol_max; synchronises the
 * stream); `commit` has nothing to do (the pools live on the device). */
GVDB2_API gvdb2_status gvdb2_finish_topology(gvdb2_volume *v, int commit, int bounds);
GVDB2_API gvdb2_status gvdb2_update_atlas(gvdb2_volume *v);                                       /* UpdateAtlas, V:2630-2704 */
/* ActivateSpace(Vector3DF), V:2766-2856 (with Reparent V:2726-2762): activates
 * the brick holding each of the n HOST positions xyz[3i..3i+2] (truncated to
 * int), in order, creating the root, the path and, for a position outside
 * the tree, a new covering root.  out[i] (host) = the leaf's pool reference
 * when it existed, GVDB2_ID_UNDEFL when the call created it or the position
 * lies outside the top configured level.  Synchronises the stream; the next
 * RebuildTopology starts from a full rebuild.  A refused batch (status other
 * than GVDB2_OK) leaves the pools unchanged and sets every out[i] to
 * GVDB2_ID_UNDEFL. */
#define GVDB2_ID_UNDEFL 0xFFFFFFFFull
GVDB2_API gvdb2_status gvdb2_activate_space(gvdb2_volume *v, const float *xyz, int64_t n, uint64_t *out);
/* Pool compaction (no reference counterpart; the reference keeps the nodes an
 * incremental rebuild delinks, gvdbDelinkLeafBricks / gvdbDelinkBricks,
 * kernels/cuda_gvdb_nodes.cuh:401-467, in its pools for good): drops them and
 * renumbers the rest in order.  Live leaves keep their order, so UpdateAtlas
 * gives them the same slots; call it before the next splat or gather.  The
 * rebuild state is kept: the next RebuildTopology continues incrementally. */
GVDB2_API gvdb2_status gvdb2_compact_pools(gvdb2_volume *v);
GVDB2_API gvdb2_status gvdb2_clear_channel(gvdb2_volume *v, int chan);                            /* ClearChannel, V:1596-1603 */
GVDB2_API gvdb2_status gvdb2_update_neighbors(gvdb2_volume *v);                                   /* UpdateNeighbors, V:2527-2556 */

/* ---- point insertion ---- */
GVDB2_API gvdb2_status gvdb2_insert_points(gvdb2_volume *v, int n, const float trans[3], int prefix);          /* InsertPoints, V:5219-5267 */
GVDB2_API gvdb2_status gvdb2_insert_points_subcell(gvdb2_volume *v, int subcell, int n, float radius,
                                         const float trans[3], int *len);                    /* InsertPointsSubcell, V:4971-5092 */
/* The same lists with 16-bit entries: positions quantized over the bounding
 * box of the last rebuild, (p + trans - mPosMin) / mPosRange * 65535, and,
 * when SetPoints gave velocities, velocities over the range of the last
 * gvdb2_get_min_max_vel (zero before one).  NOHIT and negativity are tested
 * on the translated position, as the reference's 16-bit insert does. */
GVDB2_API gvdb2_status gvdb2_insert_points_subcell_fp16(gvdb2_volume *v, int subcell, int n, float radius,
                                              const float trans[3], int *len);               /* InsertPointsSubcell_FP16, V:5094-5189 */
GVDB2_API gvdb2_status gvdb2_get_min_max_vel(gvdb2_volume *v, int n);                          /* GetMinMaxVel, V:5469-5521 */

/* ---- reference-mode splat / gathers / apron ---- */
GVDB2_API gvdb2_status gvdb2_scatter_density(gvdb2_volume *v, int n, float radius, float amp, const float trans[3],
                                   int expand, int avg_color);                               /* ScatterDensity, V:5624-5660 */
GVDB2_API gvdb2_status gvdb2_gather_density(gvdb2_volume *v, int subcell, int n, float radius, const float trans[3],
                                  int *len, int chan_density, int chan_clr, int accum);       /* GatherDensity, V:5318-5344 */
GVDB2_API gvdb2_status gvdb2_gather_level_set(gvdb2_volume *v, int subcell, int n, float radius, const float trans[3],
                                    int *len, int chan_levelset, int chan_clr, int accum);    /* GatherLevelSet, V:5348-5373 */
/* GatherLevelSet over the 16-bit lists of gvdb2_insert_points_subcell_fp16
 * (never accumulates, as in the reference). */
GVDB2_API gvdb2_status gvdb2_gather_level_set_fp16(gvdb2_volume *v, int subcell, int n, float radius,
                                         const float trans[3], int *len, int chan_levelset,
                                         int chan_clr);                                       /* GatherLevelSet_FP16, V:5375-5402 */
GVDB2_API gvdb2_status gvdb2_scatter_reduce_level_set(gvdb2_volume *v, int subcell, int n, float radius,
                                            const float trans[3], int *len, int chan_levelset,
                                            int chan_clr, int accum); /* same operation as GatherLevelSet, V:5348-5373 */
GVDB2_API gvdb2_status gvdb2_update_apron(gvdb2_volume *v, int chan, float boundval);             /* UpdateApron, V:4411-4457 (chan<0: all) */
GVDB2_API gvdb2_status gvdb2_update_apron_faces(gvdb2_volume *v, int chan);                       /* UpdateApronFaces, V:4461-4496 */

/* ---- kernel splats (no reference counterpart: the reference has no tent /
 * cubic scatter, no grid->point gather and no adjoints) ---- */
/* channel chans[c] := sum_p weight_p * attr_c(p) * W(v + 0.5 - x_p) on the
 * interior voxels of every active brick; weight.base == NULL uses
 * weight_const; attrs[c].base == NULL means attr 1.  Aprons are left for
 * gvdb2_update_apron. */
GVDB2_API gvdb2_status gvdb2_scatter_kernel(gvdb2_volume *v, int kernel, int n, const float trans[3],
                                  gvdb2_points_view weight, float weight_const,
                                  const gvdb2_points_view *attrs, const int *chans, int nch);
/* out[p*out_stride + c] := sum_v G_chans[c][v] * W(v + 0.5 - x_p) (0 for
 * points outside every active brick); out is a device float pointer. */
GVDB2_API gvdb2_status gvdb2_gather_kernel(gvdb2_volume *v, int kernel, int n, const float trans[3], const int *chans,
                                 int nch, float *out, int64_t out_stride);
/* Adjoint of gvdb2_scatter_kernel (ScatterDensityBackward): given dL/dG in
 * channels grad_chans, writes per point grad_pos[3], grad_weight and
 * grad_attr[nch] (device float pointers, row-major; any may be NULL). */
GVDB2_API gvdb2_status gvdb2_scatter_kernel_backward(gvdb2_volume *v, int kernel, int n, const float trans[3],
                                           gvdb2_points_view weight, float weight_const,
                                           const gvdb2_points_view *attrs, int nch, const int *grad_chans,
                                           float *grad_pos, float *grad_weight, float *grad_attr);
/* Adjoint of gvdb2_gather_kernel (GatherDensityBackward): given dL/dout
 * (device, grad_out[p*nch + c]), sets channels grad_chans := dL/dG on the
 * interiors of active bricks (when grad_chans != NULL) and grad_pos[p*3+k]. */
GVDB2_API gvdb2_status gvdb2_gather_kernel_backward(gvdb2_volume *v, int kernel, int n, const float trans[3],
                                          const int *chans, int nch, const float *grad_out,
                                          const int *grad_chans, float *grad_pos);

/* ---- autotuner (no reference counterpart) ----
 * Launch settings of the kernel splats and gathers.  dense: cells of at
 * least this many points take the scatter's partial-sum path (a CTA per
 * slice staging the cell's extended tile in shared memory), the other cells
 * the owner-computes warps; 0 sends every cell to the owner warps (0 or
 * [128, 2^24]).  slice: points per CTA of a dense cell (a multiple of 128 in
 * [128, 65536]).  light: cells of at most this many points are gathered a
 * warp per cell, a lane per point, with taps read from the atlas; the others
 * through a halo tile staged in shared memory (0..32).  Defaults 512, 4096,
 * 32.  Results agree within float rounding under every setting (the summation
 * order changes with the path a cell takes); deterministic mode stays
 * bit-reproducible under any one setting. */
typedef struct gvdb2_tuning {
    int32_t dense, slice, light;
} gvdb2_tuning;
GVDB2_API gvdb2_status gvdb2_set_tuning(gvdb2_volume *v, const gvdb2_tuning *t);
GVDB2_API gvdb2_status gvdb2_get_tuning(gvdb2_volume *v, gvdb2_tuning *t);
/* The on-disk cache: path for this volume (NULL or "": $GVDB2_TUNE_CACHE,
 * else none). */
GVDB2_API gvdb2_status gvdb2_set_tune_cache(gvdb2_volume *v, const char *path);
/* Same arguments and results as gvdb2_scatter_kernel / gvdb2_gather_kernel:
 * times the candidates on this call (CUDA events on the volume's stream,
 * median of three after an untimed run), keeps the fastest on the volume and
 * writes it to the cache under the call's workload class (device and SM
 * count, operation, kernel, channels, brick width, points per active 8^3
 * cell to the nearest power of two); chosen may be NULL.  The scatter tunes
 * dense and slice, the gather light. */
GVDB2_API gvdb2_status gvdb2_autotune_scatter(gvdb2_volume *v, int kernel, int n, const float trans[3],
                                              gvdb2_points_view weight, float weight_const,
                                              const gvdb2_points_view *attrs, const int *chans, int nch,
                                              gvdb2_tuning *chosen);
GVDB2_API gvdb2_status gvdb2_autotune_gather(gvdb2_volume *v, int kernel, int n, const float trans[3],
                                             const int *chans, int nch, float *out, int64_t out_stride,
                                             gvdb2_tuning *chosen);
/* Cache entries by key, for seeding or inspecting a cache file (host only):
 * get returns GVDB2_ERR_STATE when the key is absent; put rewrites the file
 * with the entry added or replaced.  ms may be NULL on get. */
GVDB2_API gvdb2_status gvdb2_tune_cache_get(const char *path, const char *key, gvdb2_tuning *t, float *ms);
GVDB2_API gvdb2_status gvdb2_tune_cache_put(const char *path, const char *key, const gvdb2_tuning *t, float ms);

/* The same gather as gvdb2_gather_kernel, for callers that cannot allocate
 * device memory once running (an application that fixes its GPU memory
 * budget at start-up, a real-time loop that forbids allocation, a process
 * whose allocator belongs to another framework).  No counterpart in the
 * reference.  It performs no device allocation: its binning scratch is one
 * file-scope device array per GPU (12.25 MiB, held until the process exits),
 * which limits a call to 1,048,576 points and 32,768 active bricks of 8^3
 * voxels (4,096 of 16^3, 512 of 32^3: 32,768 8^3 cells); larger
 * calls return GVDB2_ERR_CAPACITY.  The first call on a device looks up the
 * array's address (make it before any stream capture) and keeps it, so the
 * entry point must not be used after a cudaDeviceReset.  All calls share the
 * array, so calls whose GPU work overlaps race and must be ordered by the
 * caller.  Points outside every active brick gather 0. */
GVDB2_API gvdb2_status gvdb2_gather_kernel_noalloc(gvdb2_volume *v, int kernel, int n, const float trans[3],
                                                   const int *chans, int nch, float *out, int64_t out_stride);

/* ---- inspection (host copies; synchronise the stream) ---- */
GVDB2_API gvdb2_status gvdb2_get_info(gvdb2_volume *v, gvdb2_info *out);
GVDB2_API gvdb2_status gvdb2_copy_nodes(gvdb2_volume *v, int lev, void *host, int64_t max_nodes);            /* getNode / pool 0 (64-byte nodes) */
GVDB2_API gvdb2_status gvdb2_copy_childlists(gvdb2_volume *v, int lev, uint64_t *host, int64_t max_entries); /* pool 1 child lists */
GVDB2_API gvdb2_status gvdb2_copy_atlas(gvdb2_volume *v, int chan, float *host, int64_t max_floats);        /* used slots' tiles */
GVDB2_API gvdb2_status gvdb2_copy_atlas_map(gvdb2_volume *v, void *host, int64_t max_entries);              /* 16-byte {int3 pos; int leaf} */
GVDB2_API gvdb2_status gvdb2_copy_neighbors(gvdb2_volume *v, int32_t *host, int64_t max_entries);           /* 6 per pool leaf (-x,-y,-z,+x,+y,+z) */
GVDB2_API gvdb2_status gvdb2_copy_point_nodes(gvdb2_volume *v, int32_t *pnode, int32_t *poff, int64_t n,
                                    int32_t *gcnt, int64_t ngcnt);                                /* InsertPoints results */
GVDB2_API gvdb2_status gvdb2_copy_subcells(gvdb2_volume *v, int32_t *cnt, int32_t *nid, int32_t *pos3, int64_t max_subcells);
/* the 16-bit list entries (3 per entry, grouped by subcell like the counts);
 * vel3 may be NULL */
GVDB2_API gvdb2_status gvdb2_copy_subcell_points_fp16(gvdb2_volume *v, uint16_t *pos3, uint16_t *vel3,
                                                int64_t max_entries);
GVDB2_API gvdb2_status gvdb2_atlas_device_ptr(gvdb2_volume *v, int chan, float **dev_ptr);                 /* device view of a channel */

#ifdef __cplusplus
}
#endif
#endif
