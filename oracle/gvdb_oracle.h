/*
 * gvdb_oracle.h -- CPU restatement of GVDB's point -> sparse-volume path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the correctness oracle for the
 * CUDA implementation in gvdb-voxels_b200/.  Only the test-suite, the smoke
 * check and the CPU-baseline leg of bench.py may load it; the product path
 * never links, calls or falls back to it.
 *
 * Every function restates the algorithm of a reference function; the header
 * comment of each definition in gvdb_oracle.c cites the reference file:line
 * it follows (paths relative to the gvdb-voxels project root):
 *   V  = source/gvdb_library/src/gvdb_volume_gvdb.cpp
 *   A  = source/gvdb_library/src/gvdb_allocator.cpp
 *   P  = source/gvdb_library/kernels/cuda_gvdb_particles.cuh
 *   N  = source/gvdb_library/kernels/cuda_gvdb_nodes.cuh
 *   O  = source/gvdb_library/kernels/cuda_gvdb_operators.cuh
 *
 * Channel data are held in double precision so the FP64 error of a
 * float32 result can be stated.  Reference-mode operations round positions
 * to float exactly as the reference kernels do (which voxel a point lands
 * in is decided in float) and evaluate each contribution in double.
 */
#ifndef GVDB_ORACLE_H
#define GVDB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_OK 0
#define ORC_ERR_ARG 1
#define ORC_ERR_DEPTH 2       /* point extents smaller than one brick or deeper than 5 levels */
#define ORC_ERR_STATE 3       /* call order violated (e.g. no topology) */
#define ORC_ERR_UNSUPPORTED 4
#define ORC_ERR_NOMEM 5

#define ORC_KERNEL_TENT1 1    /* trilinear tent, support radius 1 voxel */
#define ORC_KERNEL_CUBIC2 2   /* cubic B-spline, support radius 2 voxels */

/* 64-byte node record, field for field the layout of nvdb::Node
 * (source/gvdb_library/src/gvdb_node.h:27-40). */
typedef struct orc_node {
    uint8_t mLev, mFlags, mPriority, pad;
    int32_t mPos[3];
    int32_t mValue[3];
    float mVRange[3];
    uint64_t mParent;
    uint64_t mChildList;
    uint64_t mMask;
} orc_node;

/* Atlas map entry, the layout of nvdb AtlasNode / VDBAtlasNode (N:37-40). */
typedef struct orc_atlas_node {
    int32_t mPos[3];
    int32_t mLeafID;
} orc_atlas_node;

/* Array-of-structures view of a point attribute, the meaning of DataPtr as
 * used by SetDataGPU (V:4872-4880): element i is at base + i*stride + offset. */
typedef struct orc_view {
    const void *base;
    int64_t count;
    int32_t stride;
    int32_t offset;
} orc_view;

typedef struct orc_volume orc_volume;

orc_volume *orc_create(void);
void orc_destroy(orc_volume *v);

int orc_configure(orc_volume *v, int q4, int q3, int q2, int q1, int q0);
int orc_set_channel_default(orc_volume *v, int cx, int cy, int cz);
int orc_add_channel(orc_volume *v, int chan, int apron);
void orc_request_full_rebuild(orc_volume *v, int flag);

int orc_rebuild_topology(orc_volume *v, orc_view pos, int n, float radius, const float orig[3]);
int orc_accumulate_topology(orc_volume *v, orc_view pos, int n, float radius, const float orig[3], int min_depth);
int orc_update_atlas(orc_volume *v);
/* ActivateSpace (V:2766-2856): leaf reference if it existed, else ID_UNDEFL */
uint64_t orc_activate_space(orc_volume *v, float x, float y, float z);
int64_t orc_activate_points(orc_volume *v, orc_view pos, int64_t n, float radius, const float orig[3]);
int orc_compute_bounds(const orc_volume *v, float vmin[3], float vmax[3]);
uint64_t orc_root(const orc_volume *v); /* mRoot */
int orc_compact_pools(orc_volume *v); /* drop delinked nodes, renumber the rest */
int orc_clear_channel(orc_volume *v, int chan);

int orc_insert_points(orc_volume *v, orc_view pos, int n, const float trans[3], int32_t *pnode, int32_t *poff, int32_t *gcnt);
int orc_scatter_density(orc_volume *v, orc_view pos, int n, float radius, float amp, const float trans[3], int expand,
                        const int32_t *pnode);
int orc_update_apron(orc_volume *v, int chan, float boundval);
int orc_update_neighbors(orc_volume *v);
int orc_update_apron_faces(orc_volume *v, int chan);

int orc_insert_points_subcell(orc_volume *v, int sc, orc_view pos, int n, float radius, const float trans[3], int *len);
int orc_gather_density(orc_volume *v, int sc, float radius, int chan, int accum);
int orc_gather_level_set(orc_volume *v, int sc, float radius, int chan, int accum);
/* InsertPointsSubcell_FP16 (V:5094-5189), GatherLevelSet_FP16 (V:5375-5402),
 * GetMinMaxVel (V:5469-5521); vel.base == NULL: no velocity lists. */
int orc_insert_points_subcell_fp16(orc_volume *v, int sc, orc_view pos, orc_view vel, int n, float radius,
                                   const float trans[3], int *len);
int orc_gather_level_set_fp16(orc_volume *v, int sc, float radius, int chan);
int orc_get_min_max_vel(orc_volume *v, orc_view vel, int n);

/* Kernel splats (no reference counterpart; specified mathematically).
 * channel chans[c] := sum_p weight_p * attr_c(p) * W(v + 0.5 - x_p) over the
 * interior voxels of every active brick; attrs[c].base == NULL means 1. */
int orc_scatter_kernel(orc_volume *v, int kernel, orc_view pos, int n, const float trans[3], orc_view weight,
                       float weight_const, const orc_view *attrs, const int *chans, int nch);
int orc_gather_kernel(orc_volume *v, int kernel, orc_view pos, int n, const float trans[3], const int *chans, int nch,
                      double *out);
/* Adjoints of the two operations above. */
int orc_scatter_kernel_backward(orc_volume *v, int kernel, orc_view pos, int n, const float trans[3], orc_view weight,
                                float weight_const, const orc_view *attrs, const int *chans, int nch,
                                const int *grad_chans, double *grad_pos, double *grad_weight, double *grad_attr);
int orc_gather_kernel_backward(orc_volume *v, int kernel, orc_view pos, int n, const float trans[3], const int *chans,
                               int nch, const double *grad_out, const int *grad_chans, double *grad_pos);

/* Inspection. */
int orc_depth(const orc_volume *v);
int orc_top_level(const orc_volume *v);
int64_t orc_pool_count(const orc_volume *v, int lev);
int64_t orc_used_leaves(const orc_volume *v);
const orc_node *orc_nodes(const orc_volume *v, int lev);
const uint64_t *orc_childlists(const orc_volume *v, int lev);
int64_t orc_childlist_len(const orc_volume *v, int lev);
int orc_res(const orc_volume *v, int lev);
int orc_range(const orc_volume *v, int lev);
void orc_bbox(const orc_volume *v, float posmin[3], float posmax[3]);
int orc_apron(const orc_volume *v);
int orc_tile_res(const orc_volume *v);
int64_t orc_atlas_slots(const orc_volume *v);
int64_t orc_atlas_capacity(const orc_volume *v);
void orc_atlas_subdim(const orc_volume *v, int out[3]);
double *orc_atlas(orc_volume *v, int chan);
const orc_atlas_node *orc_atlas_map(const orc_volume *v);
const int32_t *orc_neighbors(const orc_volume *v);
int64_t orc_subcell_count(const orc_volume *v);
const int32_t *orc_subcell_cnt(const orc_volume *v);
const int32_t *orc_subcell_nid(const orc_volume *v);
const int32_t *orc_subcell_pos(const orc_volume *v);
const int32_t *orc_subcell_off(const orc_volume *v);
int64_t orc_subcell_len(const orc_volume *v);
const float *orc_subcell_points(const orc_volume *v);
const uint16_t *orc_subcell_points_fp16(const orc_volume *v);
const uint16_t *orc_subcell_vel_fp16(const orc_volume *v);
int64_t orc_leaf_of_point(const orc_volume *v, float x, float y, float z);

#ifdef __cplusplus
}
#endif
#endif
