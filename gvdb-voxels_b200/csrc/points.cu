// points.cu -- point insertion and binning.
//
//   InsertPoints (V:5219-5267, P:19-36, P:59-72): per point the leaf it
//     falls in (pnode), its slot inside that leaf (poff) and per-leaf
//     counts (gcnt); with `prefix`, a counting sort of positions by leaf.
//   Kernel-splat binning (no reference counterpart): a warp-aggregated
//     counting sort of points by (atlas slot, region) where the 27 regions
//     say which neighbouring bricks a point's stencil reaches; the splat
//     kernels read a brick's own points plus the matching regions of its
//     neighbours.
//   InsertPointsSubcell (V:4971-5092, P:109-118, P:218-315, P:677-694).
#include <algorithm>

#include "dev_common.cuh"

namespace gvdb2 {

namespace {

// gvdbInsertPoints (P:19-36): NOHIT positions and points outside every
// leaf get pnode = ID_UNDEFL; others take an atomic slot in their leaf.
__global__ void k_insert_points(PointsView pos, int64_t n, float3 trans, LeafLookup L, int32_t *pnode, int32_t *poff,
                                int32_t *gcnt) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 p = load_f3(pos, i);
    if (p.z == kNoHit) {
        pnode[i] = (int32_t)kUndefL;
        return;
    }
    int32_t leaf = leaf_at(L, p.x + trans.x, p.y + trans.y, p.z + trans.z);
    if (leaf < 0) {
        pnode[i] = (int32_t)kUndefL;
        return;
    }
    pnode[i] = leaf;
    poff[i] = atomicAdd(&gcnt[leaf], 1);
}

// gvdbSortPoints (P:59-72)
__global__ void k_sort_points(PointsView pos, int64_t n, float3 trans, const int32_t *pnode, const int32_t *poff,
                              int64_t nleaves, const uint32_t *goff, float *out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t nid = pnode[i];
    if (nid < 0 || nid >= nleaves) return;
    int64_t k = (int64_t)goff[nid] + poff[i];
    float3 p = load_f3(pos, i);
    out[3 * k + 0] = p.x + trans.x;
    out[3 * k + 1] = p.y + trans.y;
    out[3 * k + 2] = p.z + trans.z;
}

// Bins every point by the 8^3 cell that contains it and by its region in
// that cell: bin = cell * 27 + (rz * 3 + ry) * 3 + rx, cell = slot * m^3 +
// cell in the brick (-1 when no active brick contains it).  Per axis the
// region is 0 when the kernel's stencil reaches into the cell below (first
// tap < 0), 2 when it reaches into the cell above (last tap >= 8), else 1 (a
// stencil is narrower than a cell, so never both).  A cell's points so come
// ordered by region, and the points of a neighbour whose stencils reach a
// cell are a few contiguous runs of that neighbour's bin.  Ranks come from
// warp-aggregated counters.
template <int KERNEL>
__device__ __forceinline__ int region_axis(float w, int cell_lo) {
    // first tap of Taps<KERNEL>::eval, relative to the cell's first voxel
    const int first = (int)floorf(w - 0.5f) - Taps<KERNEL>::LO - cell_lo;
    return first < 0 ? 0 : (first + Taps<KERNEL>::N - 1 >= kCell ? 2 : 1);
}

template <int KERNEL>
__global__ void k_bin_count(PointsView pos, int64_t n, float3 trans, LeafLookup L, const int32_t *leaf_slot, int m,
                            uint32_t *cnt, int32_t *pbin, int32_t *prank) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int32_t bin = -1;
    if (i < n) {
        float3 p = load_f3(pos, i);
        if (p.z != kNoHit) {
            const float w[3] = {p.x + trans.x, p.y + trans.y, p.z + trans.z};
            const int3 o = point_origin(pos, i);
            const int32_t leaf = leaf_at_o(L, w[0], w[1], w[2], o);
            const int32_t slot = leaf >= 0 ? leaf_slot[leaf] : -1;
            if (slot >= 0) {
                const int rm = (1 << L.g.log2r0) - 1; // local voxel = voxel mod res0
                const int vx = (int)w[0] + o.x, vy = (int)w[1] + o.y, vz = (int)w[2] + o.z;
                const int lx = vx & rm, ly = vy & rm, lz = vz & rm;
                // the cell's first voxel along each axis, in the point's grid coordinates
                const int rx = region_axis<KERNEL>(w[0], (vx & ~(kCell - 1)) - o.x);
                const int ry = region_axis<KERNEL>(w[1], (vy & ~(kCell - 1)) - o.y);
                const int rz = region_axis<KERNEL>(w[2], (vz & ~(kCell - 1)) - o.z);
                bin = (slot * m * m * m + cell_of_local(lx, ly, lz, m)) * kRegions + (rz * 3 + ry) * 3 + rx;
            }
        }
    }
    unsigned act = __ballot_sync(0xffffffffu, bin >= 0);
    if (bin >= 0) {
        uint32_t r = warp_agg_inc(cnt, (uint32_t)bin, act);
        pbin[i] = bin;
        prank[i] = (int32_t)r;
    } else if (i < n) {
        pbin[i] = -1;
    }
}

// bin_off[c] = reg_off[c * 27]: each cell's first point (c = ncell: the end)
__global__ void k_cell_off(const uint32_t *reg_off, int64_t ncell, uint32_t *bin_off) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c <= ncell) bin_off[c] = reg_off[c * kRegions];
}

// keys for the stable (deterministic) binning: bin id, unbinned last
__global__ void k_bin_keys(const int32_t *pbin, int64_t n, uint64_t *keys, int32_t *vals) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t b = pbin[i];
    keys[i] = b >= 0 ? (uint64_t)b : 0xFFFFFFFFull;
    vals[i] = (int32_t)i;
}

// Each binned point's entry of the bin order: perm[j] = i and, in the same
// pass, bin_pos[j] = its translated position and cloud index (as
// k_bin_pack_pos writes them; the positions are read in point order).
__global__ void k_bin_fill(const int32_t *pbin, const int32_t *prank, int64_t n, const uint32_t *off, int32_t *perm,
                           PointsView pos, float3 trans, float4 *bin_pos) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t b = pbin[i];
    if (b < 0) return;
    const int64_t j = (int64_t)off[b] + prank[i];
    perm[j] = (int32_t)i;
    const float3 q = load_f3(pos, i);
    const int32_t cloud = pos.cloud ? pos.cloud[i] : -1;
    bin_pos[j] = make_float4(q.x + trans.x, q.y + trans.y, q.z + trans.z, __int_as_float(cloud));
}

// bin_pos[j] = the translated position of the point at bin-order entry j
// (perm[j]) and its cloud index (-1 outside a batch), for the j below the
// number of binned points, reg_off[nreg].
__global__ void k_bin_pack_pos(const int32_t *perm, const uint32_t *reg_off, int64_t nreg, PointsView pos,
                               float3 trans, float4 *bin_pos) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= (int64_t)reg_off[nreg]) return;
    const int32_t p = perm[j];
    const float3 q = load_f3(pos, p);
    const int32_t cloud = pos.cloud ? pos.cloud[p] : -1;
    bin_pos[j] = make_float4(q.x + trans.x, q.y + trans.y, q.z + trans.z, __int_as_float(cloud));
}

// List the cells that hold points by class (huge from the front of `list`,
// heavy from its back, light in `light`; see cell_at).
constexpr int64_t kCellCountReadback = 1 << 16; // cells

// Cells of at least `dense_min` points (dense_min > 0) are the scatter's dense
// cells: each gets a partial slot (part[c], -1 for the other cells),
// ceil(k / slice) work items (cell, slice, slices, accumulator slot) and,
// when that is more than one, an accumulator slot for its integer sums.
// Cells of at most `light` (<= kLightCell) points are light.
__global__ void k_cell_list(const uint32_t *off, int64_t ncell, int32_t *list, int32_t *light, int32_t *part,
                            int4 *work, uint32_t *cnt, uint32_t dense_min, uint32_t slice, uint32_t light_max) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t k = c < ncell ? off[c + 1] - off[c] : 0u;
    const int cls = k == 0 ? -1 : (k > kHeavyCell ? kCntHuge : (k > light_max ? kCntHeavy : kCntLight));
    const unsigned act = __ballot_sync(0xffffffffu, cls >= 0);
    if (cls >= 0) {
        const uint32_t r = warp_agg_inc(cnt, (uint32_t)cls, act);
        if (cls == kCntLight) light[r] = (int32_t)c;
        else list[cls == kCntHuge ? (int64_t)r : ncell - 1 - r] = (int32_t)c;
    }
    const bool dense = dense_min > 0 && k >= dense_min;
    const unsigned dn = __ballot_sync(0xffffffffu, dense);
    int32_t slot = -1;
    if (dense) slot = (int32_t)warp_agg_inc(cnt, (uint32_t)kCntDense, dn);
    if (c < ncell) part[c] = slot;
    if (dense) {
        const uint32_t ns = (k + slice - 1) / slice;
        const uint32_t first = atomicAdd(cnt + kCntWork, ns);
        const int32_t acc = ns > 1 ? (int32_t)atomicAdd(cnt + kCntMulti, 1u) : -1;
        for (uint32_t i = 0; i < ns; i++) work[first + i] = make_int4((int32_t)c, (int32_t)i, (int32_t)ns, acc);
    }
}

// gvdbSetFlagSubcell (P:109-118)
__global__ void k_sc_flag(const Node *leaves, int64_t n, uint32_t *flag) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flag[i] = leaves[i].mParent == kUndef64 ? 0u : 1u;
}

struct ScArgs {
    PointsView pos;
    int64_t n;
    float3 trans;
    float radius;
    int sc, scdim, scpb;
    int64_t num_sc;
    LeafLookup L;
    const Node *leaves;
    int64_t nleaves;
    const uint32_t *mapping;
    // pass 2 (InsertPointsSubcell_FP16): quantization ranges, velocities
    float3 pmin, prange, vmin, vrange;
    PointsView vel;
    uint16_t *q, *qvel;
};

// gvdbInsertSubcell_fp16's 16-bit quantization (P:195-203): (x - lo) /
// range * 65535 with the reference's approximate division, converted as a
// float-to-unsigned-short conversion does: toward zero, clamped, NaN to 0.
__device__ __forceinline__ uint16_t quantize16(float x, float lo, float range) {
    const float t = __fdividef(x - lo, range) * 65535.0f;
    if (!(t > 0.0f)) return 0; // also NaN
    return t >= 65535.0f ? (uint16_t)65535 : (uint16_t)t;
}

// gvdbCountSubcell (P:275-315, pass 0) / gvdbInsertSubcell (P:218-273,
// pass 1) / gvdbInsertSubcell_fp16 (P:154-216, pass 2).  The count pass
// tests the sign after adding trans, the insert pass before, the fp16 insert
// pass tests NOHIT and the sign on the translated position, all as in the
// reference; an insert never writes past the counted capacity of its
// subcell.
template <int PASS>
__global__ void k_sc_visit(ScArgs A, uint32_t *cnt, const uint32_t *cap, const uint32_t *off, float *pnt,
                           int32_t *status) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    float3 p = load_f3(A.pos, i);
    float w[3];
    if (PASS == 2) {
        w[0] = p.x + A.trans.x;
        w[1] = p.y + A.trans.y;
        w[2] = p.z + A.trans.z;
        if (w[2] == kNoHit) return;
        if (w[0] < 0 || w[1] < 0 || w[2] < 0) return;
    } else if (p.z == kNoHit) {
        return;
    } else if (PASS == 0) {
        w[0] = p.x + A.trans.x;
        w[1] = p.y + A.trans.y;
        w[2] = p.z + A.trans.z;
        if (w[0] < 0 || w[1] < 0 || w[2] < 0) return;
    } else {
        if (p.x < 0 || p.y < 0 || p.z < 0) return;
        w[0] = p.x + A.trans.x;
        w[1] = p.y + A.trans.y;
        w[2] = p.z + A.trans.z;
    }
    int mn[3], mx[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        mn[a] = ((int)(w[a] - A.radius) / A.sc) * A.sc;
        mx[a] = ((int)(w[a] + 1 + A.radius) / A.sc) * A.sc;
    }
    for (int sx = mn[0]; sx <= mx[0]; sx += A.sc)
        for (int sy = mn[1]; sy <= mx[1]; sy += A.sc)
            for (int sz = mn[2]; sz <= mx[2]; sz += A.sc) {
                if (sx < 0 || sy < 0 || sz < 0) continue;
                int32_t leaf = leaf_at_brick(A.L, sx >> A.L.g.log2r0, sy >> A.L.g.log2r0, sz >> A.L.g.log2r0);
                if (leaf < 0 || leaf >= A.nleaves) continue;
                const Node &nd = A.leaves[leaf];
                int lx = (sx - nd.mPos[0]) / A.sc, ly = (sy - nd.mPos[1]) / A.sc, lz = (sz - nd.mPos[2]) / A.sc;
                int64_t idx = (int64_t)A.mapping[leaf] * A.scpb + ((int64_t)lz * A.scdim + ly) * A.scdim + lx;
                if (idx < 0 || idx >= A.num_sc) continue;
                if (PASS == 0) {
                    atomicAdd(&cnt[idx], 1u);
                } else {
                    uint32_t o = atomicAdd(&cnt[idx], 1u);
                    if (o >= cap[idx]) {
                        atomicSub(&cnt[idx], 1u); // the list keeps its counted length
                        atomicOr(status, kDevCapacity);
                        continue;
                    }
                    int64_t at = (int64_t)off[idx] + o;
                    if (PASS == 2) {
                        A.q[3 * at + 0] = quantize16(w[0], A.pmin.x, A.prange.x);
                        A.q[3 * at + 1] = quantize16(w[1], A.pmin.y, A.prange.y);
                        A.q[3 * at + 2] = quantize16(w[2], A.pmin.z, A.prange.z);
                        if (A.qvel) {
                            const float3 u = load_f3(A.vel, i);
                            A.qvel[3 * at + 0] = quantize16(u.x, A.vmin.x, A.vrange.x);
                            A.qvel[3 * at + 1] = quantize16(u.y, A.vmin.y, A.vrange.y);
                            A.qvel[3 * at + 2] = quantize16(u.z, A.vmin.z, A.vrange.z);
                        }
                    } else {
                        pnt[3 * at + 0] = w[0];
                        pnt[3 * at + 1] = w[1];
                        pnt[3 * at + 2] = w[2];
                    }
                }
            }
}

// gvdbCalcSubcellPos (P:677-694)
__global__ void k_sc_pos(const Node *leaves, int64_t n, const uint32_t *mapping, int sc, int scdim, int scpb,
                         int64_t num_sc, int32_t *sc_nid, int32_t *sc_pos) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Node &nd = leaves[i];
    if (nd.mParent == kUndef64) return;
    for (int s = 0; s < scpb; s++) {
        int64_t idx = (int64_t)mapping[i] * scpb + s;
        if (idx >= num_sc) continue;
        sc_pos[3 * idx + 0] = nd.mPos[0] + s % scdim * sc;
        sc_pos[3 * idx + 1] = nd.mPos[1] + (s / scdim) % scdim * sc;
        sc_pos[3 * idx + 2] = nd.mPos[2] + (s / scdim / scdim) % scdim * sc;
        sc_nid[idx] = (int32_t)i;
    }
}

} // namespace

gvdb2_status insert_points(Volume *v, int n, const float trans[3], int prefix) {
    if (v->pos.cloud) return fail(v, GVDB2_ERR_UNSUPPORTED, "batched clouds: the reference-mode point operations (InsertPoints, InsertPointsSubcell) take one cloud per volume");
    if (v->pool_cnt[0] == 0) return fail(v, GVDB2_ERR_STATE, "no topology");
    if (n < 0 || (n > 0 && (!v->pos.base || n > v->pos.count))) return fail(v, GVDB2_ERR_ARG, "bad point count");
    cudaStream_t s = v->stream;
    int64_t nl = v->pool_cnt[0];
    GV_CUDA(v, v->pnode.ensure(sizeof(int32_t) * (size_t)std::max(n, 1), s));
    GV_CUDA(v, v->poff.ensure(sizeof(int32_t) * (size_t)std::max(n, 1), s));
    GV_CUDA(v, v->gcnt.ensure(sizeof(int32_t) * (size_t)nl, s));
    GV_CUDA(v, cudaMemsetAsync(v->gcnt.p, 0, sizeof(int32_t) * (size_t)nl, s));
    GV_CUDA(v, cudaMemsetAsync(v->poff.p, 0, sizeof(int32_t) * (size_t)std::max(n, 1), s));
    float3 t = make_float3(trans[0], trans[1], trans[2]);
    LeafLookup L = make_lookup(v);
    if (n > 0)
        k_insert_points<<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(v->pos, n, t, L, v->pnode.as<int32_t>(),
                                                                    v->poff.as<int32_t>(), v->gcnt.as<int32_t>());
    GV_CUDA(v, cudaGetLastError());
    v->pnode_n = n;
    if (prefix) {
        GV_CUDA(v, v->goff.ensure(sizeof(uint32_t) * (size_t)(nl + 1), s));
        GV_TRY(exclusive_scan_u32(v, v->gcnt.as<uint32_t>(), v->goff.as<uint32_t>(), nl));
        GV_CUDA(v, v->psorted.ensure(sizeof(float) * 3 * (size_t)std::max(n, 1), s));
        if (n > 0)
            k_sort_points<<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(v->pos, n, t, v->pnode.as<int32_t>(),
                                                                      v->poff.as<int32_t>(), nl, v->goff.as<uint32_t>(),
                                                                      v->psorted.as<float>());
        GV_CUDA(v, cudaGetLastError());
    }
    return GVDB2_OK;
}

gvdb2_status bin_points(Volume *v, int kernel, int n, const float trans[3]) {
    Volume::BinKey &k = v->bin_key;
    // the regions depend on the kernel's stencil, so the bins do too
    if (k.valid && k.n == n && k.kernel == kernel && k.topo == v->topo_version && k.det == (v->deterministic != 0) &&
        k.pos.base == v->pos.base &&
        k.pos.stride == v->pos.stride && k.pos.offset == v->pos.offset && k.trans[0] == trans[0] &&
        k.trans[1] == trans[1] && k.trans[2] == trans[2] && k.tune[0] == v->tune_dense && k.tune[1] == v->tune_slice &&
        k.tune[2] == v->tune_light)
        return GVDB2_OK;
    if (!v->atlas_valid) return fail(v, GVDB2_ERR_STATE, "UpdateAtlas must follow the topology rebuild");
    if (n < 0 || (n > 0 && (!v->pos.base || n > v->pos.count))) return fail(v, GVDB2_ERR_ARG, "bad point count");
    cudaStream_t s = v->stream;
    const int m = v->res(0) / kCell; // cells per brick edge (bins are 8^3 cells)
    if (m < 1 || v->res(0) % kCell) return fail(v, GVDB2_ERR_UNSUPPORTED, "kernel splats need bricks of a multiple of 8 voxels");
    const int64_t nbins = v->atlas_last * m * m * m; // cells
    const int64_t nreg = nbins * kRegions;          // (cell, region) bins
    if (nreg >= INT32_MAX) return fail(v, GVDB2_ERR_CAPACITY, "more than 2^31 / 27 cells of 8^3 voxels");
    GV_CUDA(v, v->pbin.ensure(sizeof(int32_t) * (size_t)std::max(n, 1), s));
    GV_CUDA(v, v->prank.ensure(sizeof(int32_t) * (size_t)std::max(n, 1), s));
    GV_CUDA(v, v->perm.ensure(sizeof(int32_t) * (size_t)std::max(n, 1), s));
    GV_CUDA(v, v->bin_cnt.ensure(sizeof(uint32_t) * (size_t)(nreg + 1), s));
    GV_CUDA(v, v->reg_off.ensure(sizeof(uint32_t) * (size_t)(nreg + 1), s));
    GV_CUDA(v, v->bin_off.ensure(sizeof(uint32_t) * (size_t)(nbins + 1), s));
    GV_CUDA(v, cudaMemsetAsync(v->bin_cnt.p, 0, sizeof(uint32_t) * (size_t)(nreg + 1), s));
    float3 t = make_float3(trans[0], trans[1], trans[2]);
    LeafLookup L = make_lookup(v);
    if (n > 0) {
        auto kc = kernel == GVDB2_KERNEL_TENT1 ? k_bin_count<GVDB2_KERNEL_TENT1> : k_bin_count<GVDB2_KERNEL_CUBIC2>;
        kc<<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(v->pos, n, t, L, v->leaf_slot.as<int32_t>(), m,
                                                     v->bin_cnt.as<uint32_t>(), v->pbin.as<int32_t>(),
                                                     v->prank.as<int32_t>());
        GV_CUDA(v, cudaGetLastError());
    }
    GV_TRY(exclusive_scan_u32(v, v->bin_cnt.as<uint32_t>(), v->reg_off.as<uint32_t>(), nreg));
    k_cell_off<<<grid_for(nbins + 1, 256, 1ll << 31), 256, 0, s>>>(v->reg_off.as<uint32_t>(), nbins,
                                                                   v->bin_off.as<uint32_t>());
    GV_CUDA(v, cudaGetLastError());
    if (n > 0 && v->deterministic) {
        // stable counting sort: a radix sort of (bin, point index) keeps each
        // bin's points in index order, independent of atomic timing; its key
        // buffer is the volume's scratch (grown like every other buffer)
        GV_CUDA(v, v->tmp_c.ensure(sizeof(uint64_t) * (size_t)n, s));
        uint64_t *keys = v->tmp_c.as<uint64_t>();
        k_bin_keys<<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(v->pbin.as<int32_t>(), n, keys, v->perm.as<int32_t>());
        GV_TRY(radix_sort_u64(v, keys, v->perm.as<int32_t>(), n, 0, 32));
    }
    // the points' positions in bin order: with the bin order itself from
    // the ranks, else from the sorted order
    GV_CUDA(v, v->bin_pos.ensure(sizeof(float4) * (size_t)std::max(n, 1), s));
    if (n > 0 && !v->deterministic) {
        k_bin_fill<<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(v->pbin.as<int32_t>(), v->prank.as<int32_t>(), n,
                                                               v->reg_off.as<uint32_t>(), v->perm.as<int32_t>(), v->pos,
                                                               t, v->bin_pos.as<float4>());
        GV_CUDA(v, cudaGetLastError());
    } else if (n > 0) {
        k_bin_pack_pos<<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(v->perm.as<int32_t>(), v->reg_off.as<uint32_t>(), nreg,
                                                                  v->pos, t, v->bin_pos.as<float4>());
        GV_CUDA(v, cudaGetLastError());
    }
    // the cells that hold points, by class (the gathers' grids), and the
    // scatter's dense cells with their work items
    GV_CUDA(v, v->cell_list.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(nbins, 1), s));
    GV_CUDA(v, v->cell_light.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(nbins, 1), s));
    GV_CUDA(v, v->cell_part.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(nbins, 1), s));
    // bounds from the point count: at most n / dense dense cells, and each
    // slice beyond a cell's first holds `slice` of its points
    const int64_t dmin = v->tune_dense, sl = v->tune_slice;
    v->dense_cap = dmin > 0 ? std::min<int64_t>(nbins, n / dmin) : 0;
    v->work_cap = dmin > 0 ? v->dense_cap + n / sl : 0;
    v->multi_cap = std::min<int64_t>(v->dense_cap, n / (sl + 1));
    GV_CUDA(v, v->part_work.ensure(sizeof(int4) * (size_t)std::max<int64_t>(v->work_cap, 1), s));
    GV_CUDA(v, v->cell_cnt.ensure(sizeof(uint32_t) * kCntWords, s));
    GV_CUDA(v, cudaMemsetAsync(v->cell_cnt.p, 0, sizeof(uint32_t) * kCntWords, s));

    v->cell_grid = v->heavy_grid = v->light_grid = 0;
    if (nbins > 0) {
        const int g = grid_for(nbins, 256, 1ll << 31);
        k_cell_list<<<g, 256, 0, s>>>(v->bin_off.as<uint32_t>(), nbins, v->cell_list.as<int32_t>(),
                                      v->cell_light.as<int32_t>(), v->cell_part.as<int32_t>(),
                                      v->part_work.as<int4>(), v->cell_cnt.as<uint32_t>(), (uint32_t)v->tune_dense,
                                      (uint32_t)v->tune_slice, (uint32_t)v->tune_light);
        GV_CUDA(v, cudaGetLastError());
        v->cell_grid = v->heavy_grid = v->light_grid = nbins;
        if (nbins > kCellCountReadback) {
            // many cells: size the grids by the cells of each class (one
            // 32-byte read) rather than by all cells
            uint32_t cw[kCntWords] = {0};
            GV_CUDA(v, cudaMemcpyAsync(cw, v->cell_cnt.p, sizeof(cw), cudaMemcpyDeviceToHost, s));
            GV_CUDA(v, cudaStreamSynchronize(s));
            v->heavy_grid = (int64_t)cw[kCntHuge] + cw[kCntHeavy];
            v->light_grid = cw[kCntLight];
            v->cell_grid = v->heavy_grid + v->light_grid;
            v->dense_cap = cw[kCntDense];
            v->work_cap = cw[kCntWork];
            v->multi_cap = cw[kCntMulti];
        }
    }
    k.valid = true;
    k.det = v->deterministic != 0;
    k.kernel = kernel;
    k.n = n;
    k.topo = v->topo_version;
    k.pos = v->pos;
    for (int a = 0; a < 3; a++) k.trans[a] = trans[a];
    k.tune[0] = v->tune_dense;
    k.tune[1] = v->tune_slice;
    k.tune[2] = v->tune_light;
    return GVDB2_OK;
}

gvdb2_status insert_points_subcell(Volume *v, int sc, int n, float radius, const float trans[3], int *len,
                                   bool fp16) {
    if (v->pos.cloud) return fail(v, GVDB2_ERR_UNSUPPORTED, "batched clouds: the reference-mode point operations (InsertPoints, InsertPointsSubcell) take one cloud per volume");
    int res0 = v->res(0);
    if (sc <= 0 || res0 % sc) return fail(v, GVDB2_ERR_ARG, "subcell size must divide the brick resolution");
    if (n < 0 || (n > 0 && (!v->pos.base || n > v->pos.count))) return fail(v, GVDB2_ERR_ARG, "bad point count");
    int64_t num_brick = v->used_leaves;
    if (num_brick == 0) return fail(v, GVDB2_ERR_STATE, "InsertPointsSubcell yet no bricks exist");
    cudaStream_t s = v->stream;
    int scdim = res0 / sc, scpb = scdim * scdim * scdim;
    int64_t num_sc = (int64_t)scpb * num_brick, nmap = v->pool_cnt[0];
    v->sc_size = sc;
    v->sc_dim = scdim;
    v->sc_per_brick = scpb;
    v->num_sc = num_sc;
    GV_CUDA(v, v->sc_flag.ensure(sizeof(uint32_t) * (size_t)(nmap + 1), s));
    GV_CUDA(v, v->sc_map.ensure(sizeof(uint32_t) * (size_t)(nmap + 1), s));
    GV_CUDA(v, v->sc_cnt.ensure(sizeof(uint32_t) * (size_t)(2 * num_sc + 2), s));
    GV_CUDA(v, v->sc_off.ensure(sizeof(uint32_t) * (size_t)(num_sc + 1), s));
    GV_CUDA(v, v->sc_nid.ensure(sizeof(int32_t) * (size_t)num_sc, s));
    GV_CUDA(v, v->sc_pos.ensure(sizeof(int32_t) * 3 * (size_t)num_sc, s));
    GV_CUDA(v, cudaMemsetAsync(v->sc_nid.p, 0, sizeof(int32_t) * (size_t)num_sc, s));
    GV_CUDA(v, cudaMemsetAsync(v->sc_pos.p, 0, sizeof(int32_t) * 3 * (size_t)num_sc, s));
    k_sc_flag<<<grid_for(nmap, 256, 1ll << 31), 256, 0, s>>>(v->pool_ptr(0), nmap, v->sc_flag.as<uint32_t>());
    GV_TRY(exclusive_scan_u32(v, v->sc_flag.as<uint32_t>(), v->sc_map.as<uint32_t>(), nmap));
    uint32_t *cnt = v->sc_cnt.as<uint32_t>(), *cap = cnt + num_sc + 1;
    GV_CUDA(v, cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * (size_t)(num_sc + 1), s));
    ScArgs A;
    A.pos = v->pos;
    A.n = n;
    A.trans = make_float3(trans[0], trans[1], trans[2]);
    A.radius = radius;
    A.sc = sc;
    A.scdim = scdim;
    A.scpb = scpb;
    A.num_sc = num_sc;
    A.L = make_lookup(v);
    A.leaves = v->pool_ptr(0);
    A.nleaves = nmap;
    A.mapping = v->sc_map.as<uint32_t>();
    A.pmin = make_float3(v->posmin[0], v->posmin[1], v->posmin[2]); // mPosMin, mPosRange (V:5452-5462)
    A.prange = make_float3(v->posmax[0] - v->posmin[0], v->posmax[1] - v->posmin[1], v->posmax[2] - v->posmin[2]);
    A.vmin = make_float3(v->velmin[0], v->velmin[1], v->velmin[2]);
    A.vrange = make_float3(v->velrange[0], v->velrange[1], v->velrange[2]);
    A.vel = v->vel;
    A.q = A.qvel = nullptr;
    v->sc_fp16 = fp16;
    v->sc_qvel_valid = false;
    int32_t *status = nullptr;
    GV_CUDA(v, cudaMallocAsync((void **)&status, sizeof(int32_t), s));
    GV_CUDA(v, cudaMemsetAsync(status, 0, sizeof(int32_t), s));
    if (n > 0) k_sc_visit<0><<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(A, cnt, nullptr, nullptr, nullptr, status);
    GV_TRY(exclusive_scan_u32(v, cnt, v->sc_off.as<uint32_t>(), num_sc));
    uint32_t total = 0;
    GV_CUDA(v, cudaMemcpyAsync(&total, v->sc_off.as<uint32_t>() + num_sc, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    GV_CUDA(v, cudaStreamSynchronize(s));
    v->sc_len = total;
    if (len) *len = (int)total;
    if (total > 0) {
        GV_CUDA(v, cudaMemcpyAsync(cap, cnt, sizeof(uint32_t) * (size_t)num_sc, cudaMemcpyDeviceToDevice, s));
        GV_CUDA(v, cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * (size_t)num_sc, s));
        if (fp16) {
            GV_CUDA(v, v->sc_q.ensure(sizeof(uint16_t) * 3 * (size_t)total, s));
            A.q = v->sc_q.as<uint16_t>();
            if (v->vel.base) { // velocities too, when SetPoints gave them (P:204-207)
                GV_CUDA(v, v->sc_qvel.ensure(sizeof(uint16_t) * 3 * (size_t)total, s));
                A.qvel = v->sc_qvel.as<uint16_t>();
                v->sc_qvel_valid = true;
            }
            if (n > 0)
                k_sc_visit<2><<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(A, cnt, cap, v->sc_off.as<uint32_t>(),
                                                                         nullptr, status);
        } else {
            GV_CUDA(v, v->sc_pnt.ensure(sizeof(float) * 3 * (size_t)total, s));
            if (n > 0)
                k_sc_visit<1><<<grid_for(n, 256, 1ll << 31), 256, 0, s>>>(A, cnt, cap, v->sc_off.as<uint32_t>(),
                                                                         v->sc_pnt.as<float>(), status);
        }
    }
    k_sc_pos<<<grid_for(nmap, 256, 1ll << 31), 256, 0, s>>>(v->pool_ptr(0), nmap, v->sc_map.as<uint32_t>(), sc, scdim,
                                                            scpb, num_sc, v->sc_nid.as<int32_t>(),
                                                            v->sc_pos.as<int32_t>());
    GV_CUDA(v, cudaGetLastError());
    cudaFreeAsync(status, s);
    return GVDB2_OK;
}

} // namespace gvdb2
