// apron.cu -- apron updates.
//
//   UpdateApron (V:4411-4457, O:72-126): every apron voxel (faces, edges
//     and corners) takes the value of the interior voxel of the leaf that
//     contains its world position (centre = corner + 0.5, N:145-153), or
//     boundval when no leaf does.  The reference resolves each voxel by a
//     root-to-leaf traversal; here the owning brick is one of the 26
//     neighbours recorded per slot when the atlas was assigned, so the
//     kernel is a pure gather: one CTA per brick, one 4-byte read and one
//     4-byte write per apron voxel.
//   UpdateApronFaces (V:4461-4496, O:27-61): faces only, using the 6-entry
//     neighbour table of UpdateNeighbors (V:2527-2556).  A missing
//     neighbour is -1 here; the reference stores 0xFFFF and then fails to
//     recognise it (O:51).
#include <vector>

#include "dev_common.cuh"

namespace gvdb2 {

namespace {

struct ApronChans {
    float *chan[kMaxChan];
    int nch;
};

// One CTA per slot; every channel of the call in one pass.  `list` holds,
// in tile order, every apron voxel of a tile: its tile offset and the
// neighbour k (0..26) that owns it with the offset of the owner's interior
// voxel, so the kernel does no index arithmetic.  A thread takes two list
// entries at a time (488 apron voxels of an 8^3 brick: one round of 256
// threads), and all their loads (up to 4 channels at a time) are issued
// before the stores: the kernel is bound by the latency of these scattered
// reads.
__global__ void __launch_bounds__(256) k_apron(ApronChans C, const int32_t *nbr27, const int2 *list, int nlist,
                                               int64_t tvox, float boundval) {
    const int64_t slot = blockIdx.x;
    __shared__ int32_t nbs[27];
    if (threadIdx.x < 27) nbs[threadIdx.x] = nbr27[slot * 27 + threadIdx.x];
    __syncthreads();
    for (int i = threadIdx.x; i < nlist; i += 2 * blockDim.x) {
        const int i1 = i + blockDim.x;
        const bool two = i1 < nlist;
        const int2 e0 = list[i], e1 = list[two ? i1 : i];
        const int32_t nb0 = nbs[e0.y >> 24], nb1 = nbs[e1.y >> 24];
        const int64_t src0 = (int64_t)nb0 * tvox + (e0.y & 0xFFFFFF), src1 = (int64_t)nb1 * tvox + (e1.y & 0xFFFFFF);
        const int64_t dst0 = slot * tvox + e0.x, dst1 = slot * tvox + e1.x;
        for (int c0 = 0; c0 < C.nch; c0 += 4) {
            float val0[4], val1[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const bool in = c0 + j < C.nch;
                val0[j] = (in && nb0 >= 0) ? __ldcg(C.chan[c0 + j] + src0) : boundval;
                val1[j] = (in && two && nb1 >= 0) ? __ldcg(C.chan[c0 + j] + src1) : boundval;
            }
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (c0 + j < C.nch) {
                    C.chan[c0 + j][dst0] = val0[j];
                    if (two) C.chan[c0 + j][dst1] = val1[j];
                }
        }
    }
}

__global__ void __launch_bounds__(256) k_apron_faces(float *chan, const int32_t *slot_leaf, const int32_t *leaf_slot,
                                                     const int32_t *nbr6, int res, int apron, int tile, int64_t tvox) {
    const int64_t slot = blockIdx.x;
    const int32_t leaf = slot_leaf[slot];
    for (int t = threadIdx.x; t < 3 * res * res; t += blockDim.x) {
        int side = t / (res * res), r = t - side * res * res;
        int su = r % res, sv = r / res;
        int32_t nl = nbr6[(int64_t)leaf * 6 + side];
        if (nl < 0) continue;
        int32_t ns = leaf_slot[nl];
        if (ns < 0) continue;
        int vox[3];
        if (side == 0) { vox[0] = 0; vox[1] = su; vox[2] = sv; }
        else if (side == 1) { vox[0] = su; vox[1] = 0; vox[2] = sv; }
        else { vox[0] = su; vox[1] = sv; vox[2] = 0; }
        int inc[3] = {side == 0, side == 1, side == 2};
        auto idx = [&](int x, int y, int z) { return ((int64_t)(z + apron) * tile + (y + apron)) * tile + (x + apron); };
        int vn[3] = {vox[0] + inc[0] * (res - 1), vox[1] + inc[1] * (res - 1), vox[2] + inc[2] * (res - 1)};
        float v1 = chan[slot * tvox + idx(vox[0], vox[1], vox[2])];
        float v2 = chan[(int64_t)ns * tvox + idx(vn[0], vn[1], vn[2])];
        chan[(int64_t)ns * tvox + idx(vn[0] + inc[0], vn[1] + inc[1], vn[2] + inc[2])] = v1;
        chan[slot * tvox + idx(vox[0] - inc[0], vox[1] - inc[1], vox[2] - inc[2])] = v2;
    }
}

// The apron voxels of a tile in tile order (built once per brick geometry):
// x = tile offset; y = owning neighbour k << 24 | offset of its interior voxel.
gvdb2_status apron_list(Volume *v) {
    const int res = v->res(0), a = v->apron, t = v->tile_res();
    const int key = res * 64 + a;
    if (v->apron_list_key == key && v->apron_list.p) return GVDB2_OK;
    std::vector<int2> h;
    for (int z = 0; z < t; z++)
        for (int y = 0; y < t; y++)
            for (int x = 0; x < t; x++) {
                const int lx = x - a, ly = y - a, lz = z - a;
                const int dx = lx < 0 ? -1 : (lx >= res ? 1 : 0), dy = ly < 0 ? -1 : (ly >= res ? 1 : 0),
                          dz = lz < 0 ? -1 : (lz >= res ? 1 : 0);
                if ((dx | dy | dz) == 0) continue;
                const int k = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
                const int src = ((lz - dz * res + a) * t + (ly - dy * res + a)) * t + (lx - dx * res + a);
                h.push_back(make_int2((z * t + y) * t + x, (k << 24) | src));
            }
    if ((int64_t)t * t * t >= (1 << 24)) return fail(v, GVDB2_ERR_UNSUPPORTED, "brick tile too large for the apron list");
    GV_CUDA(v, v->apron_list.ensure(sizeof(int2) * h.size(), v->stream));
    GV_CUDA(v, cudaMemcpyAsync(v->apron_list.p, h.data(), sizeof(int2) * h.size(), cudaMemcpyHostToDevice, v->stream));
    GV_CUDA(v, cudaStreamSynchronize(v->stream)); // h is released on return
    v->apron_list_n = (int)h.size();
    v->apron_list_key = key;
    return GVDB2_OK;
}

} // namespace

gvdb2_status update_apron(Volume *v, int chan, float boundval) {
    if (v->apron == 0) return GVDB2_OK; // V:4421
    if (!v->atlas_valid) return fail(v, GVDB2_ERR_STATE, "UpdateAtlas must follow the topology rebuild");
    ApronChans C;
    C.nch = 0;
    for (int c = 0; c < kMaxChan; c++) {
        if (chan >= 0 && c != chan) continue;
        if (!v->has_chan[c]) {
            if (chan >= 0) return fail(v, GVDB2_ERR_ARG, "bad channel");
            continue;
        }
        C.chan[C.nch++] = v->atlas[c].as<float>();
    }
    if (v->atlas_last == 0 || C.nch == 0) return GVDB2_OK;
    GV_TRY(apron_list(v));
    k_apron<<<(unsigned)v->atlas_last, 256, 0, v->stream>>>(C, v->nbr27.as<int32_t>(), v->apron_list.as<int2>(),
                                                            v->apron_list_n, v->tile_vox(), boundval);
    GV_CUDA(v, cudaGetLastError());
    return GVDB2_OK;
}

gvdb2_status update_apron_faces(Volume *v, int chan) {
    if (v->apron == 0) return GVDB2_OK;
    if (chan < 0 || chan >= kMaxChan || !v->has_chan[chan]) return fail(v, GVDB2_ERR_ARG, "bad channel");
    if (!v->atlas_valid) return fail(v, GVDB2_ERR_STATE, "UpdateAtlas must follow the topology rebuild");
    if (!v->nbr6_valid) return fail(v, GVDB2_ERR_STATE, "UpdateNeighbors must precede UpdateApronFaces");
    if (v->atlas_last == 0) return GVDB2_OK;
    k_apron_faces<<<(unsigned)v->atlas_last, 256, 0, v->stream>>>(v->atlas[chan].as<float>(), v->slot_leaf.as<int32_t>(),
                                                                  v->leaf_slot.as<int32_t>(), v->nbr6.as<int32_t>(),
                                                                  v->res(0), v->apron, v->tile_res(), v->tile_vox());
    GV_CUDA(v, cudaGetLastError());
    return GVDB2_OK;
}

} // namespace gvdb2
