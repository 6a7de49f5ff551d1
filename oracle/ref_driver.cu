// ref_driver.cu -- replays the reference's own CUDA kernels (TEST INFRASTRUCTURE).
//
// Built by oracle/Makefile (`make ref`) from the gvdb-voxels kernel sources
// where they lie (the include of cuda_gvdb_module.cu below resolves through
// -I to source/gvdb_library/kernels; gvdb_cutils.cu is compiled beside it),
// with the reference's own --use_fast_math, into oracle/_ref/libgvdbref.so.
// It exists to produce golden vectors that pin the oracle to the reference;
// the product never links or calls it.
//
// The reference's host library (gvdb_volume_gvdb.cpp) does not build here
// (it needs OpenGL/X11), so this file restates the host side of VolumeGVDB's
// point path -- pools with host mirrors, the node-allocation loops, link /
// delink launch order, UpdateAtlas, PrepareVDB, PrefixSum -- and launches the
// reference kernels with the reference's launch shapes (citations inline,
// paths relative to the gvdb-voxels project: V = src/gvdb_volume_gvdb.cpp,
// A = src/gvdb_allocator.cpp).  The atlas is a CUDA array with a surface
// object per channel, as AllocateTextureGPU (A:389-455) makes it.
//
// Deliberate departures, each needed to keep a shared GPU from faulting:
//  - key buffers written by the append-style kernels (P:467-512, P:420-465)
//    are sized for the worst case instead of N*depth (the reference has no
//    capacity check there);
//  - UpdateNeighbors stores -1 (0xFFFFFFFF) for a missing neighbour, which
//    the faces kernel recognises (O:51), instead of the reference's 0xFFFF;
//  - InsertPoints sizes its per-brick counters for every leaf (see there);
//  - the apron kernels are refused while leaves without an atlas slot exist.
// P = kernels/cuda_gvdb_particles.cuh, O = kernels/cuda_gvdb_operators.cuh,
// N = kernels/cuda_gvdb_nodes.cuh.  The callers' inputs must keep every box
// the point kernels visit inside the root node (getPosParent, N:303-345, has
// no bounds check); tests/golden/make_golden.py checks that on the CPU.
#include "cuda_gvdb_module.cu"

#include "gvdb_cutils.cuh"

#include <cstdint>
#include <cstring>
#include <vector>

namespace {

typedef unsigned long long u64;
constexpr u64 kUndefL = 0xFFFFFFFFull;
constexpr u64 kUndef64 = 0xFFFFFFFFFFFFFFFFull;

struct HostNode { // nvdb::Node, gvdb_node.h:27-40
    unsigned char mLev, mFlags, mPriority, pad;
    int mPos[3];
    int mValue[3];
    float mVRange[3];
    u64 mParent;
    u64 mChildList;
    u64 mMask;
};
static_assert(sizeof(HostNode) == 64, "Node layout");

struct AtlasNodeH {
    int mPos[3];
    int mLeafID;
};

#define RD_CHECK(x)                          \
    do {                                     \
        cudaError_t e_ = (x);                \
        if (e_ != cudaSuccess) return -(int)e_; \
    } while (0)

struct Pool { // DataPtr of a node pool with its CPU mirror (A:55-91)
    std::vector<char> cpu;
    char *gpu = nullptr;
    size_t width = 0, cap = 0, cnt = 0;
    int alloc(size_t w, size_t initmax) {
        width = w;
        cap = initmax ? initmax : 1;
        cnt = 0;
        cpu.assign(width * cap, 0);
        if (gpu) cudaFree(gpu);
        RD_CHECK(cudaMalloc(&gpu, width * cap));
        RD_CHECK(cudaMemset(gpu, 0, width * cap));
        return 0;
    }
    // PoolAlloc (A:163-192): grow x2 preserving content, append
    long long push() {
        if (cnt >= cap) {
            size_t ncap = cap * 2;
            std::vector<char> nc(width * ncap, 0);
            memcpy(nc.data(), cpu.data(), width * cnt);
            cpu.swap(nc);
            char *ng = nullptr;
            if (cudaMalloc(&ng, width * ncap) != cudaSuccess) return -1;
            cudaMemset(ng, 0, width * ncap);
            cudaMemcpy(ng, gpu, width * cnt, cudaMemcpyDeviceToDevice);
            cudaFree(gpu);
            gpu = ng;
            cap = ncap;
        }
        return (long long)cnt++;
    }
    int commit() { return cnt ? (int)cudaMemcpy(gpu, cpu.data(), width * cnt, cudaMemcpyHostToDevice) : 0; }
    int fetch() { return cnt ? (int)cudaMemcpy(cpu.data(), gpu, width * cnt, cudaMemcpyDeviceToHost) : 0; }
};

struct DevArr { // linear aux buffer (PrepareAux, V:4957-4967)
    char *p = nullptr;
    size_t bytes = 0;
    int ensure(size_t b, bool zero) {
        if (b > bytes) {
            if (p) cudaFree(p);
            p = nullptr;
            bytes = 0;
            RD_CHECK(cudaMalloc(&p, b));
            bytes = b;
        }
        if (zero) RD_CHECK(cudaMemset(p, 0, bytes));
        return 0;
    }
    ~DevArr() {
        if (p) cudaFree(p);
    }
};

struct RefVolume {
    int logdim[MAXLEV] = {0};
    int nlev = 0;
    Pool pool[2][5];
    u64 root = kUndefL;
    bool rebuild = true;
    int cur_depth = -1, depth = 0;
    float posmin[3], posmax[3];
    size_t used_leaves = 0;
    // atlas (channel 0 layout shared by all channels)
    int apron = 0, nchan = 0;
    int default_axis[3] = {16, 16, 1};
    int subdim[3] = {0, 0, 0};
    size_t atlas_last = 0;
    cudaArray_t arr[32] = {nullptr};
    cudaSurfaceObject_t surf[32] = {0};
    std::vector<AtlasNodeH> amap;
    DevArr amap_gpu;
    // VDBInfo
    VDBInfo info;
    VDBInfo *d_info = nullptr;
    // points
    DevArr pos;
    int npts = 0;
    // aux
    DevArr keys, sorted, marker, marker_pre, uniq, unique_cnt, lev_cnt, range_res, extra_cnt, node_marker;
    DevArr scan_a1, scan_s1, scan_a2, scan_s2;
    DevArr pnode, poff, gcnt;
    DevArr sc_flag, sc_map, sc_cnt, sc_pre, sc_pnt, sc_pos, sc_nid, nbr;
    DevArr sc_q; // ushort3 entries of InsertPointsSubcell_FP16
    int num_sc = 0, sc_size = 0, sc_len = 0;
    bool sc_fp16 = false; // the last subcell insert was the FP16 one
    std::vector<int> nbr_host;

    int res(int l) const { return 1 << logdim[l]; }
    int range(int lev) const { // getRange (gvdb_volume_gvdb.h:614-619)
        if (lev == -1) return 1;
        int r = res(0);
        for (int l = 1; l <= lev; l++) r *= res(l);
        return r;
    }
    int tile() const { return res(0) + 2 * apron; }
    HostNode *node(int lev, size_t i) { return reinterpret_cast<HostNode *>(pool[0][lev].cpu.data()) + i; }
    u64 *clist(int lev, size_t i) {
        return reinterpret_cast<u64 *>(pool[1][lev].cpu.data() + i * pool[1][lev].width);
    }
};

// PrepareVDB / PrepareVDBPartially (V:3946-4020)
int prepare_vdb(RefVolume *v) {
    VDBInfo &I = v->info;
    int tlev = 1;
    for (int n = v->nlev - 1; n >= 0; n--) {
        I.dim[n] = v->logdim[n];
        I.res[n] = v->res(n);
        int r = v->range(n);
        I.vdel[n] = make_float3((float)r / v->res(n), (float)r / v->res(n), (float)r / v->res(n));
        I.noderange[n] = make_int3(r, r, r);
        I.nodecnt[n] = (int)v->pool[0][n].cnt;
        I.nodewid[n] = (int)v->pool[0][n].width;
        I.childwid[n] = (int)v->pool[1][n].width;
        I.nodelist[n] = v->pool[0][n].gpu;
        I.childlist[n] = v->pool[1][n].gpu;
        if (I.nodecnt[n] == 1) tlev = n;
    }
    I.atlas_map = reinterpret_cast<VDBAtlasNode *>(v->amap_gpu.p);
    I.atlas_apron = v->apron;
    I.atlas_cnt = make_int3(v->subdim[0], v->subdim[1], v->subdim[2]);
    I.atlas_res = make_int3(v->subdim[0] * v->tile(), v->subdim[1] * v->tile(), v->subdim[2] * v->tile());
    I.brick_res = v->tile();
    for (int n = 0; n < v->apron; n++) {
        I.apron_table[n] = n;
        I.apron_table[(v->apron * 2 - 1) - n] = (v->tile() - 1) - n;
    }
    I.top_lev = tlev;
    I.epsilon = 0.001f;
    I.max_iter = 256;
    I.update = false;
    for (int c = 0; c < v->nchan; c++) I.volOut[c] = v->surf[c];
    RD_CHECK(cudaMemcpy(v->d_info, &I, sizeof(VDBInfo), cudaMemcpyHostToDevice));
    return 0;
}

// PrefixSum (V:4760-4819): three-level scan with the reference kernels
int prefix_sum(RefVolume *v, char *in, char *out, int num) {
    const int naux = SCAN_BLOCKSIZE << 1;
    int blks1 = num / naux + 1, blks2 = blks1 / naux + 1, threads = SCAN_BLOCKSIZE, zon = 1;
    if (blks1 <= 1024) {
        if (v->scan_a1.ensure(sizeof(unsigned) * naux, false) || v->scan_s1.ensure(sizeof(unsigned) * naux, false)) return -1;
    } else {
        if (v->scan_a1.ensure(sizeof(unsigned) * blks2 * naux, false) ||
            v->scan_s1.ensure(sizeof(unsigned) * blks2 * naux, false))
            return -1;
    }
    if (v->scan_a2.ensure(sizeof(unsigned) * naux, false) || v->scan_s2.ensure(sizeof(unsigned) * naux, false)) return -1;
    unsigned *a1 = (unsigned *)v->scan_a1.p, *s1 = (unsigned *)v->scan_s1.p, *a2 = (unsigned *)v->scan_a2.p,
             *s2 = (unsigned *)v->scan_s2.p;
    prefixSum<<<blks1, threads>>>((unsigned *)in, (unsigned *)out, a1, num, zon);
    prefixSum<<<blks2, threads>>>(a1, s1, a2, blks1, zon);
    prefixSum<<<1, threads>>>(a2, s2, nullptr, blks2, zon);
    prefixFixup<<<blks2, threads>>>(s1, s2, blks1);
    prefixFixup<<<blks1, threads>>>((unsigned *)out, s1, num);
    RD_CHECK(cudaGetLastError());
    return 0;
}

// GetBoundingBox (V:5404-5467): gvdbSplitPos + Thrust min/max
int bounding_box(RefVolume *v, int n, float3 trans) {
    DevArr xs, ys, zs, bb;
    if (xs.ensure(sizeof(float) * n, false) || ys.ensure(sizeof(float) * n, false) || zs.ensure(sizeof(float) * n, false) ||
        bb.ensure(sizeof(float) * 6, false))
        return -1;
    gvdbSplitPos<<<n / 256 + 1, 256>>>(n, trans, v->pos.p, 0, 12, (float *)xs.p, (float *)ys.p, (float *)zs.p);
    RD_CHECK(cudaGetLastError());
    CUdeviceptr b = (CUdeviceptr)bb.p;
    gvdbDeviceMinElementF(b + 0, (CUdeviceptr)xs.p, n);
    gvdbDeviceMinElementF(b + 4, (CUdeviceptr)ys.p, n);
    gvdbDeviceMinElementF(b + 8, (CUdeviceptr)zs.p, n);
    gvdbDeviceMaxElementF(b + 12, (CUdeviceptr)xs.p, n);
    gvdbDeviceMaxElementF(b + 16, (CUdeviceptr)ys.p, n);
    gvdbDeviceMaxElementF(b + 20, (CUdeviceptr)zs.p, n);
    float h[6];
    RD_CHECK(cudaMemcpy(h, bb.p, sizeof(h), cudaMemcpyDeviceToHost));
    for (int a = 0; a < 3; a++) {
        float lo = h[a] - 1, hi = h[3 + a] + 2;
        v->posmin[a] = 0 > lo ? 0 : lo;
        v->posmax[a] = 0 > hi ? 0 : hi;
    }
    return 0;
}

// DetermineDepth + GetCoveringNode (V:821-837, V:2915-2931)
int determine_depth(RefVolume *v, int rootpos[3]) {
    for (int lev = 0; lev < MAXLEV; lev++) {
        int a[3], b[3];
        int r = v->range(lev < v->nlev ? lev : v->nlev - 1);
        for (int k = 0; k < 3; k++) {
            if (lev == MAXLEV - 1) {
                a[k] = b[k] = 0;
            } else {
                int pa = (int)v->posmin[k], pb = (int)v->posmax[k];
                a[k] = pa / r * r;
                b[k] = pb / r * r;
            }
        }
        if (a[0] == b[0] && a[1] == b[1] && a[2] == b[2]) {
            rootpos[0] = a[0];
            rootpos[1] = a[1];
            rootpos[2] = a[2];
            return lev;
        }
    }
    return -1;
}

} // namespace

namespace {

inline u64 elem(int grp, int lev, u64 ndx) { return (u64)grp | ((u64)lev << 8) | (ndx << 16); }

// SetupNode (V:2512-2524)
void setup_node(RefVolume *v, int lev, size_t idx, const int pos[3], int marker) {
    HostNode *n = v->node(lev, idx);
    n->mLev = (unsigned char)lev;
    n->mPos[0] = pos[0];
    n->mPos[1] = pos[1];
    n->mPos[2] = pos[2];
    n->mChildList = kUndefL;
    n->mParent = kUndefL;
    n->mValue[0] = n->mValue[1] = n->mValue[2] = -1;
    n->mFlags = (unsigned char)marker;
}

// PoolAlloc + SetupNode + child list memset 0xFF (V:1311-1329)
long long alloc_node(RefVolume *v, int lev, const int pos[3]) {
    long long idx = v->pool[0][lev].push();
    if (idx < 0) return -1;
    setup_node(v, lev, (size_t)idx, pos, 1);
    if (lev > 0) {
        long long c = v->pool[1][lev].push();
        if (c < 0) return -1;
        v->node(lev, idx)->mChildList = elem(1, lev, (u64)c);
        memset(v->clist(lev, (size_t)c), 0xFF, v->pool[1][lev].width);
    }
    return idx;
}

int commit_all(RefVolume *v) {
    for (int g = 0; g < 2; g++)
        for (int l = 0; l < v->nlev; l++)
            if (v->pool[g][l].width && v->pool[g][l].commit()) return -1;
    return 0;
}
int fetch_all(RefVolume *v) {
    for (int g = 0; g < 2; g++)
        for (int l = 0; l < v->nlev; l++)
            if (v->pool[g][l].width && v->pool[g][l].fetch()) return -1;
    return 0;
}

void clear_topology(RefVolume *v) { // Clear (V:2487-2503)
    for (int g = 0; g < 2; g++)
        for (int l = 0; l < 5; l++) v->pool[g][l].cnt = 0;
    v->root = kUndefL;
    v->atlas_last = 0;
    v->used_leaves = 0;
    v->rebuild = true;
}

// keys per point an append kernel may emit: its box spans at most
// (kmax+1)*radius+1 voxels per axis (P:438-439, P:485-486, int truncation
// included), so at most floor(span/range)+2 nodes per axis at each level
size_t box_keys_per_point(RefVolume *v, int depth, float radius, float kmax) {
    size_t total = 0;
    for (int l = 0; l < depth; l++) {
        size_t k = (size_t)(((kmax + 1.0f) * radius + 1.0f) / v->range(l)) + 2;
        total += k * k * k;
    }
    return total + 1;
}

// RadixSortByByte + FindUniqueBrick (V:843-928); returns the unique count
long long sort_unique(RefVolume *v, int num, int depth) {
    if (v->sorted.ensure((size_t)num * 8 + 8, false)) return -1;
    if (num > 0) {
        if (cudaMemcpy(v->sorted.p, v->keys.p, (size_t)num * 8, cudaMemcpyDeviceToDevice)) return -1;
        gvdbDeviceRadixSort((CUdeviceptr)v->sorted.p, (uint32_t)num);
    }
    if (v->marker.ensure((size_t)num * 4 + 4, true) || v->marker_pre.ensure((size_t)num * 4 + 4, true) ||
        v->unique_cnt.ensure(4, true) || v->lev_cnt.ensure(sizeof(int) * MAXLEV, true))
        return -1;
    gvdbFindUnique<<<num / 512 + 1, 512>>>(num, (long long *)v->sorted.p, (int *)v->marker.p, (int *)v->unique_cnt.p,
                                            (int *)v->lev_cnt.p);
    int nu = 0;
    if (cudaMemcpy(&nu, v->unique_cnt.p, 4, cudaMemcpyDeviceToHost)) return -1;
    if (prefix_sum(v, v->marker.p, v->marker_pre.p, num)) return -1;
    if (v->uniq.ensure((size_t)nu * 8 + 8, false)) return -1;
    gvdbCompactUnique<<<num / 512 + 1, 512>>>(num, (long long *)v->sorted.p, (int *)v->marker.p, (int *)v->marker_pre.p,
                                               (long long *)v->uniq.p);
    if (cudaGetLastError()) return -1;
    (void)depth;
    return nu;
}

// host allocation loop over sorted unique keys (V:1308-1331, V:965-988, V:1088-1111)
int alloc_from_unique(RefVolume *v, int nu, int depth) {
    std::vector<int> levcnt(MAXLEV, 0);
    std::vector<unsigned short> keys((size_t)nu * 4 + 4);
    if (cudaMemcpy(levcnt.data(), v->lev_cnt.p, sizeof(int) * depth, cudaMemcpyDeviceToHost)) return -1;
    if (nu && cudaMemcpy(keys.data(), v->uniq.p, (size_t)nu * 8, cudaMemcpyDeviceToHost)) return -1;
    int pre = 0;
    for (int lev = 0; lev < depth; lev++) {
        int r = v->range(lev);
        for (int n = pre; n < pre + levcnt[lev]; n++) {
            int pos[3] = {keys[n * 4 + 2] * r, keys[n * 4 + 1] * r, keys[n * 4 + 0] * r};
            if (alloc_node(v, lev, pos) < 0) return -1;
        }
        pre += levcnt[lev];
    }
    return 0;
}

int link_all(RefVolume *v, int depth, int pblks_override) {
    for (int lev = depth - 1; lev >= 0; lev--) {
        int pblks = pblks_override > 0 ? pblks_override : (int)(v->pool[0][lev].cnt / 512) + 1;
        gvdbLinkBricks<<<pblks, 512>>>(v->d_info, lev);
    }
    RD_CHECK(cudaGetLastError());
    return 0;
}

// ActivateBricksGPU (V:1229-1413) + ActivateExtraBricksGPU (V:931-1016)
int full_rebuild(RefVolume *v, int n, float radius, float3 orig, int depth, const int rootpos[3]) {
    std::vector<int> rr(depth);
    for (int l = 0; l < depth; l++) rr[l] = v->range(l);
    if (v->range_res.ensure(sizeof(int) * MAXLEV, false)) return -1;
    RD_CHECK(cudaMemcpy(v->range_res.p, rr.data(), sizeof(int) * depth, cudaMemcpyHostToDevice));
    if (v->keys.ensure((size_t)n * depth * 8 + 8, false)) return -1;
    gvdbCalcBrickId<<<n / 512 + 1, 512>>>(n, depth, (int *)v->range_res.p, v->pos.p, 0, 12, orig,
                                          (unsigned short *)v->keys.p);
    RD_CHECK(cudaGetLastError());
    long long nu = sort_unique(v, n * depth, depth);
    if (nu < 0) return -1;
    { // root (V:1290-1300)
        long long r = v->pool[0][depth].push();
        long long c = v->pool[1][depth].push();
        if (r < 0 || c < 0) return -1;
        setup_node(v, depth, (size_t)r, rootpos, 1);
        v->node(depth, r)->mFlags = 1;
        v->node(depth, r)->mChildList = elem(1, depth, (u64)c);
        memset(v->clist(depth, (size_t)c), 0xFF, v->pool[1][depth].width);
        v->root = elem(0, depth, (u64)r);
    }
    if (alloc_from_unique(v, (int)nu, depth)) return -1;
    if (commit_all(v) || prepare_vdb(v) || link_all(v, depth, 0) || fetch_all(v)) return -1;
    if (radius >= 1) {
        size_t cap = (size_t)n * box_keys_per_point(v, depth, radius, 2.0f);
        if (v->keys.ensure(cap * 8, true) || v->extra_cnt.ensure(4, true)) return -1;
        gvdbCalcExtraBrickId<<<n / 512 + 1, 512>>>(v->d_info, radius, n, depth, (int *)v->range_res.p, v->pos.p, 0, 12,
                                                   orig, (unsigned short *)v->keys.p, (int *)v->extra_cnt.p);
        int cnt = 0;
        RD_CHECK(cudaMemcpy(&cnt, v->extra_cnt.p, 4, cudaMemcpyDeviceToHost));
        if ((size_t)cnt > cap) return -2; // could not happen within the bound; report rather than read on
        nu = sort_unique(v, cnt, depth);
        if (nu < 0) return -1;
        if (alloc_from_unique(v, (int)nu, depth)) return -1;
        if (commit_all(v) || prepare_vdb(v) || link_all(v, depth, 0) || fetch_all(v)) return -1;
    }
    v->used_leaves = v->pool[0][0].cnt;
    return 0;
}

// ActivateIncreBricksGPU (V:1020-1156)
int incremental_rebuild(RefVolume *v, int n, float radius, float3 orig, int depth, bool accum) {
    size_t total = v->pool[0][0].cnt;
    if (total == 0) return 0;
    std::vector<int> marker(total, 0);
    if (accum)
        for (size_t i = 0; i < total; i++) marker[i] = v->node(0, i)->mFlags;
    if (v->node_marker.ensure(total * 4, false)) return -1;
    RD_CHECK(cudaMemcpy(v->node_marker.p, marker.data(), total * 4, cudaMemcpyHostToDevice));
    size_t cap = (size_t)n * box_keys_per_point(v, depth, radius, 1.0f);
    if (v->keys.ensure(cap * 8, true) || v->extra_cnt.ensure(4, true)) return -1;
    gvdbCalcIncreExtraBrickId<<<n / 512 + 1, 512>>>(v->d_info, radius, n, depth, (int *)v->range_res.p, v->pos.p, 0, 12,
                                                    orig, (unsigned short *)v->keys.p, (int *)v->extra_cnt.p,
                                                    (int *)v->node_marker.p);
    int cnt = 0;
    RD_CHECK(cudaMemcpy(&cnt, v->extra_cnt.p, 4, cudaMemcpyDeviceToHost));
    if ((size_t)cnt > cap) return -2;
    if (cnt == 0) return 0; // V:1065
    long long nu = sort_unique(v, cnt, depth);
    if (nu < 0) return -1;
    RD_CHECK(cudaMemcpy(marker.data(), v->node_marker.p, total * 4, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < total; i++) v->node(0, i)->mFlags = (unsigned char)marker[i];
    if (alloc_from_unique(v, (int)nu, depth)) return -1;
    if (commit_all(v) || prepare_vdb(v)) return -1;
    int pblks = (int)(v->pool[0][0].cnt / 512) + 1;
    if (link_all(v, depth, pblks)) return -1;
    gvdbDelinkLeafBricks<<<pblks, 512>>>(v->d_info);
    for (int lev = 1; lev < depth; lev++) gvdbDelinkBricks<<<pblks, 512>>>(v->d_info, lev);
    RD_CHECK(cudaGetLastError());
    if (fetch_all(v)) return -1;
    size_t used = v->pool[0][0].cnt;
    for (size_t i = 0; i < v->pool[0][0].cnt; i++)
        if (!v->node(0, i)->mFlags) used--;
    v->used_leaves = used;
    return 0;
}

} // namespace

namespace {

// zero a float atlas channel through a 3-D copy from a zeroed linear buffer
// (ClearChannel, V:2407-2423, does the same with cuMemcpy3D)
int clear_array(RefVolume *v, int chan) {
    int t = v->tile();
    size_t w = (size_t)v->subdim[0] * t, h = (size_t)v->subdim[1] * t, d = (size_t)v->subdim[2] * t;
    DevArr zero;
    if (zero.ensure(w * h * d * sizeof(float), true)) return -1;
    cudaMemcpy3DParms p = {};
    p.srcPtr = make_cudaPitchedPtr(zero.p, w * sizeof(float), w, h);
    p.dstArray = v->arr[chan];
    p.extent = make_cudaExtent(w, h, d);
    p.kind = cudaMemcpyDeviceToDevice;
    RD_CHECK(cudaMemcpy3D(&p));
    return 0;
}

// AllocateTextureGPU for a T_FLOAT channel (A:389-455): a 3-D CUDA array with
// surface load/store, reached by the kernels through VDBInfo::volOut.  A
// resize starts from zeros instead of preserving the old bricks; every
// sequence replayed here clears its channels after UpdateAtlas anyway.
int alloc_atlas(RefVolume *v, int chan) {
    if (v->surf[chan]) cudaDestroySurfaceObject(v->surf[chan]);
    if (v->arr[chan]) cudaFreeArray(v->arr[chan]);
    v->surf[chan] = 0;
    v->arr[chan] = nullptr;
    int t = v->tile();
    cudaChannelFormatDesc d = cudaCreateChannelDesc<float>();
    RD_CHECK(cudaMalloc3DArray(&v->arr[chan], &d,
                               make_cudaExtent((size_t)v->subdim[0] * t, (size_t)v->subdim[1] * t, (size_t)v->subdim[2] * t),
                               cudaArraySurfaceLoadStore));
    cudaResourceDesc r = {};
    r.resType = cudaResourceTypeArray;
    r.res.array.array = v->arr[chan];
    RD_CHECK(cudaCreateSurfaceObject(&v->surf[chan], &r));
    return clear_array(v, chan);
}

// Allocator::getAtlasPos (A:704-714): slot -> atlas voxel of the brick's
// first interior voxel
void atlas_pos(const RefVolume *v, size_t id, int out[3]) {
    size_t a2 = (size_t)v->subdim[0] * v->subdim[1];
    int z = (int)(id / a2);
    id -= (size_t)z * a2;
    int y = (int)(id / v->subdim[0]);
    id -= (size_t)y * v->subdim[0];
    int x = (int)id;
    int t = v->tile();
    out[0] = x * t + v->apron;
    out[1] = y * t + v->apron;
    out[2] = z * t + v->apron;
}

// UpdateAtlas (V:2630-2697) with AtlasAlloc / AtlasResize / AllocateAtlasMap /
// ClearMapping / AssignMapping
int update_atlas(RefVolume *v) {
    size_t total = v->pool[0][0].cnt, used = v->used_leaves;
    v->atlas_last = 0;
    size_t amax = (size_t)v->subdim[0] * v->subdim[1] * v->subdim[2];
    if (used > amax) {
        int layer = v->subdim[0] * v->subdim[1];
        v->subdim[2] = (int)ceil(used / (float)layer);
        for (int c = 0; c < v->nchan; c++)
            if (alloc_atlas(v, c)) return -1;
    }
    for (size_t n = 0; n < total; n++) {
        HostNode *nd = v->node(0, n);
        if (!nd->mFlags) continue;
        if (v->atlas_last >= (size_t)v->subdim[0] * v->subdim[1] * v->subdim[2]) { // AtlasAlloc growth (A:692-702)
            v->subdim[2] += 1;
            for (int c = 0; c < v->nchan; c++)
                if (alloc_atlas(v, c)) return -1;
        }
        int p[3];
        atlas_pos(v, v->atlas_last++, p);
        nd->mValue[0] = p[0];
        nd->mValue[1] = p[1];
        nd->mValue[2] = p[2];
    }
    size_t nmap = (size_t)v->subdim[0] * v->subdim[1] * v->subdim[2];
    v->amap.assign(nmap, AtlasNodeH{{0, 0, 0}, (int)kUndefL});
    int t = v->tile();
    for (size_t n = 0; n < total; n++) {
        HostNode *nd = v->node(0, n);
        if (!nd->mFlags) continue;
        int ix = nd->mValue[0] / t, iy = nd->mValue[1] / t, iz = nd->mValue[2] / t;
        AtlasNodeH &a = v->amap[((size_t)iz * v->subdim[1] + iy) * v->subdim[0] + ix];
        a.mPos[0] = nd->mPos[0];
        a.mPos[1] = nd->mPos[1];
        a.mPos[2] = nd->mPos[2];
        a.mLeafID = (int)n;
    }
    if (v->amap_gpu.ensure(nmap * sizeof(AtlasNodeH), false)) return -1;
    RD_CHECK(cudaMemcpy(v->amap_gpu.p, v->amap.data(), nmap * sizeof(AtlasNodeH), cudaMemcpyHostToDevice));
    if (v->pool[0][0].commit()) return -1;
    return prepare_vdb(v);
}

// host getNodeAtPoint (V:4650-4685) over the fetched pools; returns the leaf
// index or -1
long long host_leaf_at(RefVolume *v, float px, float py, float pz) {
    if (v->root == kUndefL) return -1;
    int lev = (int)((v->root >> 8) & 0xFF);
    size_t idx = (size_t)(v->root >> 16);
    for (;;) {
        HostNode *n = v->node(lev, idx);
        float r = (float)v->range(lev);
        float p[3] = {px - n->mPos[0], py - n->mPos[1], pz - n->mPos[2]};
        if (!(p[0] >= 0 && p[1] >= 0 && p[2] >= 0 && p[0] < r && p[1] < r && p[2] < r)) return -1;
        if (lev == 0) return (long long)idx;
        int res = v->res(lev);
        int b[3];
        for (int k = 0; k < 3; k++) b[k] = (int)(p[k] * res / r);
        u64 cl = n->mChildList;
        if (cl == kUndefL) return -1;
        u64 c = v->clist(lev, (size_t)(cl >> 16))[((size_t)b[2] * res + b[1]) * res + b[0]];
        if (c == kUndef64) return -1;
        lev -= 1;
        idx = (size_t)(c >> 16);
    }
}

// RebuildTopology (V:1181-1218) including the mCurrDepth quirk: the full
// branch never records the depth, so the second call rebuilds again
int rebuild_topology(RefVolume *v, int n, float radius, float3 orig) {
    if (bounding_box(v, n, orig)) return -1;
    int rootpos[3];
    int depth = determine_depth(v, rootpos);
    if (depth <= 0 || depth > 5) return -3;
    if (v->rebuild) {
        clear_topology(v);
    } else if (depth != v->cur_depth) {
        clear_topology(v);
        v->rebuild = true;
        v->cur_depth = depth;
    }
    if (v->rebuild) {
        v->depth = depth;
        int rc = full_rebuild(v, n, radius, orig, depth, rootpos);
        if (rc) return rc;
        v->rebuild = false;
    } else {
        int rc = incremental_rebuild(v, n, radius, orig, depth, false);
        if (rc) return rc;
    }
    return 0;
}

} // namespace

namespace {

// InsertPoints without the prefix/sort step (V:5219-5245).  The reference
// sizes the per-brick counters by the atlas slots but indexes them by leaf
// pool index; they are sized here for whichever is larger.
int insert_points(RefVolume *v, int n, float3 trans) {
    int bricks = (int)(v->atlas_last > v->pool[0][0].cnt ? v->atlas_last : v->pool[0][0].cnt);
    if (v->pnode.ensure((size_t)n * 4 + 4, false) || v->poff.ensure((size_t)n * 4 + 4, false) ||
        v->gcnt.ensure((size_t)bricks * 4 + 4, true))
        return -1;
    if (prepare_vdb(v)) return -1;
    gvdbInsertPoints<<<n / 512 + 1, 512>>>(v->d_info, n, v->pos.p, 0, 12, (int *)v->pnode.p, (int *)v->poff.p,
                                           (int *)v->gcnt.p, trans);
    RD_CHECK(cudaGetLastError());
    return 0;
}

// ScatterDensity (V:5624-5655) without colours.  The reference host passes
// the kernel's arguments without the leading VDBInfo pointer; the launch here
// gives the kernel the argument list its signature declares.
int scatter_density(RefVolume *v, int n, float radius, float amp, float3 trans, bool expand) {
    if (prepare_vdb(v)) return -1;
    gvdbScatterPointDensity<<<n / 256 + 1, 256>>>(v->d_info, n, radius, amp, v->pos.p, 0, 12, nullptr, 0, 0,
                                                  (int *)v->pnode.p, trans, expand, nullptr);
    RD_CHECK(cudaGetLastError());
    return 0;
}

// UpdateApron(chan, boundval) (V:4418-4455)
int update_apron(RefVolume *v, int chan, float boundval) {
    if (v->apron == 0) return 0;
    if (prepare_vdb(v)) return -1;
    int bricks = (int)v->pool[0][0].cnt, brickres = v->tile(), brickwid = v->res(0);
    if (bricks == 0) return 0;
    dim3 block(6 * v->apron, 8, 8);
    dim3 grid(bricks, (brickres + 7) / 8, (brickres + 7) / 8);
    gvdbUpdateApronF<<<grid, block>>>(v->d_info, (uchar)chan, bricks, brickres, brickwid, boundval);
    RD_CHECK(cudaGetLastError());
    return 0;
}

// UpdateNeighbors (V:2527-2556)
int update_neighbors(RefVolume *v) {
    size_t brks = v->pool[0][0].cnt;
    v->nbr_host.assign(brks * 6, -1);
    float d = (float)v->res(0);
    for (size_t n = 0; n < brks; n++) {
        HostNode *nd = v->node(0, n);
        float c[3] = {nd->mPos[0] + d / 2, nd->mPos[1] + d / 2, nd->mPos[2] + d / 2};
        int *o = &v->nbr_host[n * 6];
        o[0] = (int)host_leaf_at(v, c[0] - d, c[1], c[2]);
        o[1] = (int)host_leaf_at(v, c[0], c[1] - d, c[2]);
        o[2] = (int)host_leaf_at(v, c[0], c[1], c[2] - d);
        o[3] = (int)host_leaf_at(v, c[0] + d, c[1], c[2]);
        o[4] = (int)host_leaf_at(v, c[0], c[1] + d, c[2]);
        o[5] = (int)host_leaf_at(v, c[0], c[1], c[2] + d);
    }
    if (v->nbr.ensure(brks * 6 * sizeof(int) + 4, false)) return -1;
    if (brks) RD_CHECK(cudaMemcpy(v->nbr.p, v->nbr_host.data(), brks * 6 * sizeof(int), cudaMemcpyHostToDevice));
    return 0;
}

// UpdateApronFaces (V:4461-4492)
int update_apron_faces(RefVolume *v, int chan) {
    if (v->apron == 0) return 0;
    if (prepare_vdb(v)) return -1;
    int bricks = (int)v->pool[0][0].cnt, brickres = v->tile(), brickwid = v->res(0);
    if (bricks == 0) return 0;
    dim3 block(3 * v->apron, 8, 8);
    dim3 grid(bricks, (brickwid + 7) / 8, (brickwid + 7) / 8);
    gvdbUpdateApronFacesF<<<grid, block>>>(v->d_info, (uchar)chan, bricks, brickres, brickwid, (int *)v->nbr.p);
    RD_CHECK(cudaGetLastError());
    return 0;
}

// InsertPointsSubcell (V:4971-5083) and InsertPointsSubcell_FP16
// (V:5094-5189) without velocities and colours
int insert_points_subcell(RefVolume *v, int sc, int n, float radius, float3 trans, int *out_len, bool fp16) {
    *out_len = 0;
    int num_brick = (int)v->used_leaves;
    if (num_brick == 0) return 0;
    if (prepare_vdb(v)) return -1;
    int sc_dim = v->res(0) / sc;
    int per_brick = sc_dim * sc_dim * sc_dim;
    int num_sc = per_brick * num_brick;
    int rr = v->range(0) / sc_dim;
    int3 range = make_int3(rr, rr, rr);
    int nmap = (int)v->pool[0][0].cnt;
    if (v->sc_flag.ensure((size_t)nmap * 4 + 4, true) || v->sc_map.ensure((size_t)nmap * 4 + 4, false)) return -1;
    gvdbSetFlagSubcell<<<nmap / 512 + 1, 512>>>(v->d_info, nmap, (int *)v->sc_flag.p);
    if (prefix_sum(v, v->sc_flag.p, v->sc_map.p, nmap)) return -1;
    if (v->sc_cnt.ensure((size_t)num_sc * 4, true)) return -1;
    gvdbCountSubcell<<<n / 512 + 1, 512>>>(v->d_info, sc, per_brick, n, v->pos.p, 0, 12, (int *)v->sc_cnt.p, range,
                                           trans, sc_dim, radius, num_sc, (int *)v->sc_map.p);
    if (v->sc_pre.ensure((size_t)num_sc * 4, true)) return -1;
    if (prefix_sum(v, v->sc_cnt.p, v->sc_pre.p, num_sc)) return -1;
    int off_last = 0, cnt_last = 0;
    RD_CHECK(cudaMemcpy(&off_last, v->sc_pre.p + (size_t)(num_sc - 1) * 4, 4, cudaMemcpyDeviceToHost));
    RD_CHECK(cudaMemcpy(&cnt_last, v->sc_cnt.p + (size_t)(num_sc - 1) * 4, 4, cudaMemcpyDeviceToHost));
    int len = off_last + cnt_last;
    *out_len = len;
    v->sc_size = sc;
    v->num_sc = num_sc;
    v->sc_len = len;
    v->sc_fp16 = fp16;
    if (len == 0) return 0;
    if (v->sc_cnt.ensure((size_t)num_sc * 4, true)) return -1;
    if (fp16) {
        // mPosMin / mPosRange of the last GetBoundingBox; mVelMin / mVelRange
        // are not used without velocities
        if (v->sc_q.ensure((size_t)len * 6, false)) return -1;
        const float3 pmin = make_float3(v->posmin[0], v->posmin[1], v->posmin[2]);
        const float3 prange = make_float3(v->posmax[0] - v->posmin[0], v->posmax[1] - v->posmin[1],
                                          v->posmax[2] - v->posmin[2]);
        const float3 zero = make_float3(0.0f, 0.0f, 0.0f);
        gvdbInsertSubcell_fp16<<<n / 512 + 1, 512>>>(v->d_info, sc, per_brick, n, (int *)v->sc_cnt.p,
                                                     (int *)v->sc_pre.p, (int *)v->sc_map.p, pmin, prange, zero, zero,
                                                     range, trans, sc_dim, radius, v->pos.p, 0, 12,
                                                     (ushort3 *)v->sc_q.p, nullptr, 0, 0, nullptr, nullptr, 0, 0,
                                                     nullptr);
    } else {
        if (v->sc_pnt.ensure((size_t)len * 12, false)) return -1;
        gvdbInsertSubcell<<<n / 512 + 1, 512>>>(v->d_info, sc, per_brick, n, (int *)v->sc_cnt.p, (int *)v->sc_pre.p,
                                                (int *)v->sc_map.p, range, trans, sc_dim, radius, v->pos.p, 0, 12,
                                                (float3 *)v->sc_pnt.p, nullptr, 0, 0, nullptr, nullptr, 0, 0, nullptr);
    }
    if (v->sc_pos.ensure((size_t)num_sc * 12, false) || v->sc_nid.ensure((size_t)num_sc * 4, false)) return -1;
    gvdbCalcSubcellPos<<<nmap / 512 + 1, 512>>>(v->d_info, (int *)v->sc_nid.p, (int3 *)v->sc_pos.p, nmap, sc_dim,
                                                per_brick, sc, (int *)v->sc_map.p);
    RD_CHECK(cudaGetLastError());
    return 0;
}

// GatherDensity / GatherLevelSet (V:5318-5373) without colours
int gather(RefVolume *v, bool levelset, int n, float radius, int chan, bool accum) {
    if (v->sc_fp16) return -4; // the lists hold ushort3 entries
    if (v->used_leaves == 0 || v->num_sc == 0) return 0;
    if (!levelset && v->sc_len == 0) return 0;
    if (prepare_vdb(v)) return -1;
    dim3 block(v->sc_size, v->sc_size, v->sc_size);
    if (levelset)
        gvdbGatherLevelSet<<<v->num_sc, block>>>(v->d_info, n, v->num_sc, radius, (int *)v->sc_nid.p, (int *)v->sc_cnt.p,
                                                 (int *)v->sc_pre.p, (int3 *)v->sc_pos.p, (float3 *)v->sc_pnt.p, nullptr,
                                                 nullptr, chan, 0, accum);
    else
        gvdbGatherDensity<<<v->num_sc, block>>>(v->d_info, n, v->num_sc, radius, (int *)v->sc_nid.p, (int *)v->sc_cnt.p,
                                                (int *)v->sc_pre.p, (int3 *)v->sc_pos.p, (float3 *)v->sc_pnt.p, nullptr,
                                                nullptr, chan, 0, accum);
    RD_CHECK(cudaGetLastError());
    return 0;
}

// GatherLevelSet_FP16 (V:5375-5402) without colours
int gather_level_set_fp16(RefVolume *v, int n, float radius, int chan) {
    if (!v->sc_fp16 && v->sc_len) return -4; // the lists hold float3 entries
    if (v->used_leaves == 0 || v->num_sc == 0) return 0;
    if (prepare_vdb(v)) return -1;
    const float3 pmin = make_float3(v->posmin[0], v->posmin[1], v->posmin[2]);
    const float3 prange = make_float3(v->posmax[0] - v->posmin[0], v->posmax[1] - v->posmin[1],
                                      v->posmax[2] - v->posmin[2]);
    const float3 zero = make_float3(0.0f, 0.0f, 0.0f);
    dim3 block(v->sc_size, v->sc_size, v->sc_size);
    gvdbGatherLevelSet_fp16<<<v->num_sc, block>>>(v->d_info, n, v->num_sc, radius, pmin, prange, zero, zero,
                                                   (int *)v->sc_nid.p, (int *)v->sc_cnt.p, (int *)v->sc_pre.p,
                                                   (int3 *)v->sc_pos.p, (ushort3 *)v->sc_q.p, nullptr, nullptr, chan, 0);
    RD_CHECK(cudaGetLastError());
    return 0;
}

// read the atlas back as slot-major linear tiles: slot s, voxel (x,y,z) of
// its (res+2*apron)^3 tile at s*T^3 + (z*T + y)*T + x
int copy_atlas_tiles(RefVolume *v, int chan, float *out, size_t max_floats) {
    int t = v->tile();
    size_t w = (size_t)v->subdim[0] * t, h = (size_t)v->subdim[1] * t, d = (size_t)v->subdim[2] * t;
    size_t t3 = (size_t)t * t * t;
    if (v->atlas_last * t3 > max_floats) return -2;
    std::vector<float> all(w * h * d);
    cudaMemcpy3DParms p = {};
    p.srcArray = v->arr[chan];
    p.dstPtr = make_cudaPitchedPtr(all.data(), w * sizeof(float), w, h);
    p.extent = make_cudaExtent(w, h, d);
    p.kind = cudaMemcpyDeviceToHost;
    RD_CHECK(cudaMemcpy3D(&p));
    for (size_t s = 0; s < v->atlas_last; s++) {
        int a[3];
        atlas_pos(v, s, a);
        for (int z = 0; z < t; z++)
            for (int y = 0; y < t; y++)
                for (int x = 0; x < t; x++) {
                    size_t gx = a[0] - v->apron + x, gy = a[1] - v->apron + y, gz = a[2] - v->apron + z;
                    out[s * t3 + ((size_t)z * t + y) * t + x] = all[(gz * h + gy) * w + gx];
                }
    }
    return 0;
}

} // namespace

// ---------------------------------------------------------------------------
// C entry points used by tests/golden/make_golden.py.  Every call returns 0 on
// success, a negative CUDA error or -1/-2/-3/-4 for allocation, capacity,
// depth and state errors.
#define RD_API extern "C" __attribute__((visibility("default")))

RD_API void *rd_create(int device) {
    if (cudaSetDevice(device) != cudaSuccess) return nullptr;
    RefVolume *v = new RefVolume();
    if (cudaMalloc(&v->d_info, sizeof(VDBInfo)) != cudaSuccess) {
        delete v;
        return nullptr;
    }
    memset(&v->info, 0, sizeof(VDBInfo));
    return v;
}

RD_API void rd_destroy(void *h) {
    RefVolume *v = (RefVolume *)h;
    if (!v) return;
    cudaDeviceSynchronize();
    for (int c = 0; c < 32; c++) {
        if (v->surf[c]) cudaDestroySurfaceObject(v->surf[c]);
        if (v->arr[c]) cudaFreeArray(v->arr[c]);
    }
    for (int g = 0; g < 2; g++)
        for (int l = 0; l < 5; l++)
            if (v->pool[g][l].gpu) cudaFree(v->pool[g][l].gpu);
    cudaFree(v->d_info);
    delete v;
}

// Configure(q4..q0) (V:2364-2429): node pools of 64-byte nodes, child-list
// pools of res^3 64-bit references for levels above the leaves
RD_API int rd_configure(void *h, int q4, int q3, int q2, int q1, int q0) {
    RefVolume *v = (RefVolume *)h;
    int r[5] = {q0, q1, q2, q3, q4};
    int maxcnt[5] = {4, 4, 2, 1, 1};
    v->nlev = 5;
    for (int n = 0; n < 5; n++) v->logdim[n] = r[n] == 0 ? 1 : r[n];
    for (int n = 0; n < 5; n++)
        if (v->pool[0][n].alloc(sizeof(HostNode), maxcnt[n])) return -1;
    v->pool[1][0].width = 0;
    for (int n = 1; n < 5; n++) {
        size_t vc = (size_t)v->res(n) * v->res(n) * v->res(n);
        if (v->pool[1][n].alloc(sizeof(u64) * vc, maxcnt[n])) return -1;
    }
    clear_topology(v);
    v->cur_depth = -1;
    return 0;
}

// AddChannel(chan, T_FLOAT, apron) (V:2437-2450): all channels share channel
// 0's atlas layout
RD_API int rd_add_channel(void *h, int chan, int apron) {
    RefVolume *v = (RefVolume *)h;
    if (chan != v->nchan || chan >= 32) return -4;
    v->apron = apron;
    if (chan == 0) {
        v->subdim[0] = v->default_axis[0];
        v->subdim[1] = v->default_axis[1];
        v->subdim[2] = v->default_axis[2];
    }
    v->nchan = chan + 1;
    return alloc_atlas(v, chan);
}

RD_API int rd_set_points(void *h, const float *host_xyz, int n) {
    RefVolume *v = (RefVolume *)h;
    if (v->pos.ensure((size_t)n * 12 + 16, false)) return -1;
    if (n) RD_CHECK(cudaMemcpy(v->pos.p, host_xyz, (size_t)n * 12, cudaMemcpyHostToDevice));
    v->npts = n;
    return 0;
}

RD_API int rd_rebuild_topology(void *h, int n, float radius, const float orig[3]) {
    RefVolume *v = (RefVolume *)h;
    int rc = rebuild_topology(v, n, radius, make_float3(orig[0], orig[1], orig[2]));
    if (rc) return rc;
    RD_CHECK(cudaDeviceSynchronize());
    return 0;
}

// RequestFullRebuild(true) (gvdb_volume_gvdb.h:343)
RD_API int rd_request_full_rebuild(void *h) {
    ((RefVolume *)h)->rebuild = true;
    return 0;
}

RD_API int rd_update_atlas(void *h) { return update_atlas((RefVolume *)h); }

RD_API int rd_clear_channel(void *h, int chan) {
    RefVolume *v = (RefVolume *)h;
    return chan < v->nchan ? clear_array(v, chan) : -4;
}

RD_API int rd_insert_points(void *h, int n, const float trans[3]) {
    RefVolume *v = (RefVolume *)h;
    int rc = insert_points(v, n, make_float3(trans[0], trans[1], trans[2]));
    if (rc) return rc;
    RD_CHECK(cudaDeviceSynchronize());
    return 0;
}

RD_API int rd_copy_point_nodes(void *h, int *pnode, int *poff, int n, int *gcnt, int nbricks) {
    RefVolume *v = (RefVolume *)h;
    if (n > v->npts || (size_t)nbricks > v->atlas_last) return -2;
    RD_CHECK(cudaMemcpy(pnode, v->pnode.p, (size_t)n * 4, cudaMemcpyDeviceToHost));
    RD_CHECK(cudaMemcpy(poff, v->poff.p, (size_t)n * 4, cudaMemcpyDeviceToHost));
    if (nbricks) RD_CHECK(cudaMemcpy(gcnt, v->gcnt.p, (size_t)nbricks * 4, cudaMemcpyDeviceToHost));
    return 0;
}

RD_API int rd_scatter_density(void *h, int n, float radius, float amp, const float trans[3], int expand) {
    RefVolume *v = (RefVolume *)h;
    if (expand && v->apron < 1) return -4; // the expanded stencil writes one voxel into the apron
    int rc = scatter_density(v, n, radius, amp, make_float3(trans[0], trans[1], trans[2]), expand != 0);
    if (rc) return rc;
    RD_CHECK(cudaDeviceSynchronize());
    return 0;
}

// the apron kernels index every leaf's atlas slot: refused while unused
// leaves (with no slot of their own) exist
RD_API int rd_update_apron(void *h, int chan, float boundval) {
    RefVolume *v = (RefVolume *)h;
    if (chan >= v->nchan || v->used_leaves != v->pool[0][0].cnt || v->apron != 1) return -4;
    int rc = update_apron(v, chan, boundval);
    if (rc) return rc;
    RD_CHECK(cudaDeviceSynchronize());
    return 0;
}

RD_API int rd_update_neighbors(void *h) { return update_neighbors((RefVolume *)h); }

RD_API int rd_copy_neighbors(void *h, int *out, long long max_ints) {
    RefVolume *v = (RefVolume *)h;
    if ((long long)v->nbr_host.size() > max_ints) return -2;
    memcpy(out, v->nbr_host.data(), v->nbr_host.size() * sizeof(int));
    return 0;
}

RD_API int rd_update_apron_faces(void *h, int chan) {
    RefVolume *v = (RefVolume *)h;
    if (chan >= v->nchan || v->used_leaves != v->pool[0][0].cnt || v->apron != 1 ||
        v->nbr_host.size() != v->pool[0][0].cnt * 6)
        return -4;
    int rc = update_apron_faces(v, chan);
    if (rc) return rc;
    RD_CHECK(cudaDeviceSynchronize());
    return 0;
}

RD_API int rd_insert_points_subcell(void *h, int sc, int n, float radius, const float trans[3], int *out_len) {
    RefVolume *v = (RefVolume *)h;
    if (sc <= 0 || v->res(0) % sc || sc * sc * sc > 1024) return -4;
    int rc = insert_points_subcell(v, sc, n, radius, make_float3(trans[0], trans[1], trans[2]), out_len, false);
    if (rc) return rc;
    RD_CHECK(cudaDeviceSynchronize());
    return 0;
}

RD_API int rd_insert_points_subcell_fp16(void *h, int sc, int n, float radius, const float trans[3], int *out_len) {
    RefVolume *v = (RefVolume *)h;
    if (sc <= 0 || v->res(0) % sc || sc * sc * sc > 1024) return -4;
    int rc = insert_points_subcell(v, sc, n, radius, make_float3(trans[0], trans[1], trans[2]), out_len, true);
    if (rc) return rc;
    RD_CHECK(cudaDeviceSynchronize());
    return 0;
}

// the ushort3 entries of the FP16 lists, grouped by subcell like rd_copy_subcells
RD_API int rd_copy_subcells_fp16(void *h, unsigned short *q, long long max_pnts) {
    RefVolume *v = (RefVolume *)h;
    if (v->sc_len > max_pnts) return -2;
    if (!v->sc_fp16 || v->sc_q.bytes < (size_t)v->sc_len * 6) return -4;
    if (v->sc_len) RD_CHECK(cudaMemcpy(q, v->sc_q.p, (size_t)v->sc_len * 6, cudaMemcpyDeviceToHost));
    return 0;
}

RD_API int rd_gather_level_set_fp16(void *h, int n, float radius, int chan) {
    RefVolume *v = (RefVolume *)h;
    if (chan >= v->nchan) return -4;
    int rc = gather_level_set_fp16(v, n, radius, chan);
    if (rc) return rc;
    RD_CHECK(cudaDeviceSynchronize());
    return 0;
}

// per-subcell counts (length num_sc) and the subcell point lists grouped by
// subcell; the order inside one subcell follows atomics and is not defined
RD_API int rd_copy_subcells(void *h, int *cnt, int *off, int *nid, float *pnts, long long max_sc, long long max_pnts) {
    RefVolume *v = (RefVolume *)h;
    if (v->num_sc > max_sc || v->sc_len > max_pnts) return -2;
    if (v->num_sc) {
        RD_CHECK(cudaMemcpy(cnt, v->sc_cnt.p, (size_t)v->num_sc * 4, cudaMemcpyDeviceToHost));
        RD_CHECK(cudaMemcpy(off, v->sc_pre.p, (size_t)v->num_sc * 4, cudaMemcpyDeviceToHost));
        RD_CHECK(cudaMemcpy(nid, v->sc_nid.p, (size_t)v->num_sc * 4, cudaMemcpyDeviceToHost));
    }
    // the float3 list only when the last insert wrote one
    if (v->sc_len && !v->sc_fp16 && v->sc_pnt.bytes >= (size_t)v->sc_len * 12)
        RD_CHECK(cudaMemcpy(pnts, v->sc_pnt.p, (size_t)v->sc_len * 12, cudaMemcpyDeviceToHost));
    return 0;
}

RD_API int rd_gather_density(void *h, int n, float radius, int chan, int accum) {
    RefVolume *v = (RefVolume *)h;
    if (chan >= v->nchan) return -4;
    int rc = gather(v, false, n, radius, chan, accum != 0);
    if (rc) return rc;
    RD_CHECK(cudaDeviceSynchronize());
    return 0;
}

RD_API int rd_gather_level_set(void *h, int n, float radius, int chan, int accum) {
    RefVolume *v = (RefVolume *)h;
    if (chan >= v->nchan) return -4;
    int rc = gather(v, true, n, radius, chan, accum != 0);
    if (rc) return rc;
    RD_CHECK(cudaDeviceSynchronize());
    return 0;
}

// counts: pool[0][0..4] then used leaves, atlas slots, depth, top level
RD_API int rd_get_counts(void *h, long long out[9]) {
    RefVolume *v = (RefVolume *)h;
    for (int l = 0; l < 5; l++) out[l] = (long long)v->pool[0][l].cnt;
    out[5] = (long long)v->used_leaves;
    out[6] = (long long)v->atlas_last;
    out[7] = v->depth;
    out[8] = v->info.top_lev;
    return 0;
}

RD_API int rd_copy_nodes(void *h, int lev, void *out, long long max_bytes) {
    RefVolume *v = (RefVolume *)h;
    size_t b = v->pool[0][lev].cnt * sizeof(HostNode);
    if ((long long)b > max_bytes) return -2;
    memcpy(out, v->pool[0][lev].cpu.data(), b);
    return 0;
}

RD_API int rd_copy_childlists(void *h, int lev, void *out, long long max_bytes) {
    RefVolume *v = (RefVolume *)h;
    size_t b = v->pool[1][lev].cnt * v->pool[1][lev].width;
    if ((long long)b > max_bytes) return -2;
    if (b) memcpy(out, v->pool[1][lev].cpu.data(), b);
    return 0;
}

RD_API int rd_copy_atlas_map(void *h, int *out, long long max_ints) {
    RefVolume *v = (RefVolume *)h;
    if ((long long)v->amap.size() * 4 > max_ints) return -2;
    memcpy(out, v->amap.data(), v->amap.size() * sizeof(AtlasNodeH));
    return 0;
}

RD_API int rd_copy_atlas_tiles(void *h, int chan, float *out, long long max_floats) {
    RefVolume *v = (RefVolume *)h;
    if (chan >= v->nchan) return -4;
    return copy_atlas_tiles(v, chan, out, (size_t)max_floats);
}
