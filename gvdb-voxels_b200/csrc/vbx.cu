// vbx.cu -- SaveVBX / LoadVBX: the reference's VBX file (GVDB_FILESPEC.txt),
// written and read as VolumeGVDB::SaveVBX (V:1626-1768) and LoadVBX
// (V:507-685) do for version 1.11, so that files pass both ways.
//
// The layout is the reference's, byte for byte (little-endian, packed):
//   header: major 1, minor 11 (uchar each); pre-translation, Euler angles,
//     scale and translation (3 floats each); grid count 1 (int); the grid
//     offset table (one uint64, filled in last).  No bitmask byte: that
//     belongs to major version 2.
//   grid: a 256-byte name (zeros here; the reference writes an uninitialised
//     buffer), data type 'f', 1 component, compression 0 (uchar each); voxel
//     size (1,1,1); the level-0 pool's node count; brick dims (res0 x3);
//     apron; channel count; the bytes of one channel's atlas (uint64);
//     topology type 2 (uchar); topology reuse 0 (int); atlas layout 0
//     (uchar); atlas brick counts and atlas resolution (3 ints each).
//   topology: level count; the root's pool reference (uint64); per level
//     log2 dim, res, range (3 ints), pool-0 count and width (64, the Node),
//     pool-1 count and width (8 res^3 for levels >= 1, 0 and 0 for level 0);
//     then every level's nodes, then every level's child lists.
//   atlas: per channel its type (T_FLOAT = 3) and stride (4), then the 3D
//     atlas as z-slices of (atlas res x) * (atlas res y) floats, x fastest;
//     slot s sits at brick (s mod nx, (s / nx) mod ny, s / (nx ny)).
// The atlas in device memory is slot-major tiles, so both directions convert
// one layer of bricks at a time.
#include <cstdio>
#include <cstring>
#include <vector>

#include "dev_common.cuh"

namespace gvdb2 {

namespace {

constexpr unsigned char kVbxMajor = 1, kVbxMinor = 11;
constexpr int kNameLen = 256;
constexpr int kTypeFloat = 3; // T_FLOAT (gvdb_types.h)

struct File {
    FILE *f = nullptr;
    bool ok = true;
    ~File() {
        if (f) fclose(f);
    }
    template <class T>
    void put(const T *p, size_t n) {
        if (ok && n && fwrite(p, sizeof(T), n, f) != n) ok = false;
    }
    template <class T>
    void put1(T x) { put(&x, 1); }
    template <class T>
    void get(T *p, size_t n) {
        if (ok && n && fread(p, sizeof(T), n, f) != n) ok = false;
    }
    template <class T>
    T get1() {
        T x{};
        get(&x, 1);
        return x;
    }
};

int channel_count(const Volume *v) {
    // the reference counts its atlases; channels are added as 0, 1, ...
    int n = 0;
    while (n < kMaxChan && v->has_chan[n]) n++;
    return n;
}

} // namespace

gvdb2_status save_vbx(Volume *v, const char *path) {
    if (!path) return fail(v, GVDB2_ERR_ARG, "no file name");
    if (v->nlev == 0) return fail(v, GVDB2_ERR_STATE, "Configure not called");
    const int nchan = channel_count(v);
    if (nchan == 0) return fail(v, GVDB2_ERR_STATE, "no atlas channel");
    if (!v->atlas_valid) return fail(v, GVDB2_ERR_STATE, "UpdateAtlas must follow the topology rebuild");
    cudaStream_t s = v->stream;
    GV_CUDA(v, cudaStreamSynchronize(s));
    File F;
    F.f = fopen(path, "wb");
    if (!F.f) return fail(v, GVDB2_ERR_ARG, std::string("cannot open ") + path);
    const int levels = v->nlev, T = v->tile_res(), res0 = v->res(0);
    const int ax[3] = {v->subdim[0], v->subdim[1], v->subdim[2]};
    const int ar[3] = {ax[0] * T, ax[1] * T, ax[2] * T};
    const uint64_t atlas_bytes = (uint64_t)ar[0] * ar[1] * ar[2] * sizeof(float);

    F.put1(kVbxMajor);
    F.put1(kVbxMinor);
    F.put(v->xf_pretrans, 3);
    F.put(v->xf_angs, 3);
    F.put(v->xf_scale, 3);
    F.put(v->xf_trans, 3);
    F.put1((int32_t)1); // grids
    const long table = ftell(F.f);
    F.put1((uint64_t)0); // grid offset, filled in below
    const uint64_t grid_off = (uint64_t)ftell(F.f);
    char name[kNameLen];
    std::memset(name, 0, sizeof(name));
    F.put(name, kNameLen);
    F.put1('f');
    F.put1((char)1);
    F.put1((char)0);
    const float voxelsize[3] = {1, 1, 1};
    F.put(voxelsize, 3);
    F.put1((int32_t)v->pool_cnt[0]);
    const int32_t leafdim[3] = {res0, res0, res0};
    F.put(leafdim, 3);
    F.put1((int32_t)v->apron);
    F.put1((int32_t)nchan);
    F.put1(atlas_bytes);
    F.put1((char)2);
    F.put1((int32_t)0);
    F.put1((char)0);
    F.put(ax, 3);
    F.put(ar, 3);

    F.put1((int32_t)levels);
    F.put1((uint64_t)elem(0, v->depth, 0)); // Elem(grp, lev, ndx): the root sits alone at level `depth`
    for (int n = 0; n < levels; n++) {
        const int32_t rng = (int32_t)v->range(n);
        const int32_t row[9] = {v->logdim[n], v->res(n), rng, rng, rng, (int32_t)v->pool_cnt[n], (int32_t)sizeof(Node),
                                (int32_t)(n > 0 ? v->pool_cnt[n] : 0),
                                (int32_t)(n > 0 ? sizeof(uint64_t) * v->res3(n) : 0)};
        F.put(row, 9);
    }
    for (int n = 0; n < levels; n++) {
        std::vector<Node> nodes((size_t)v->pool_cnt[n]);
        if (!nodes.empty())
            GV_CUDA(v, cudaMemcpy(nodes.data(), v->pool[n].p, sizeof(Node) * nodes.size(), cudaMemcpyDeviceToHost));
        F.put(nodes.data(), nodes.size());
    }
    for (int n = 1; n < levels; n++) {
        std::vector<uint64_t> cl((size_t)(v->pool_cnt[n] * v->res3(n)));
        if (!cl.empty())
            GV_CUDA(v, cudaMemcpy(cl.data(), v->clist[n].p, sizeof(uint64_t) * cl.size(), cudaMemcpyDeviceToHost));
        F.put(cl.data(), cl.size());
    }

    // atlas: one layer of bricks (T slices) at a time
    const int64_t tv = v->tile_vox(), layer = (int64_t)ax[0] * ax[1];
    std::vector<float> tiles((size_t)(layer * tv));
    std::vector<float> slab((size_t)ar[0] * ar[1] * T);
    for (int c = 0; c < nchan; c++) {
        F.put1((int32_t)kTypeFloat);
        F.put1((int32_t)sizeof(float));
        for (int bz = 0; bz < ax[2]; bz++) {
            const int64_t s0 = bz * layer, ns = std::max<int64_t>(0, std::min<int64_t>(layer, v->atlas_last - s0));
            std::fill(tiles.begin(), tiles.end(), 0.0f); // slots past the last hold zeros
            if (ns > 0)
                GV_CUDA(v, cudaMemcpy(tiles.data(), v->atlas[c].as<float>() + s0 * tv, sizeof(float) * (size_t)(ns * tv),
                                      cudaMemcpyDeviceToHost));
            for (int by = 0; by < ax[1]; by++)
                for (int bx = 0; bx < ax[0]; bx++) {
                    const float *t = tiles.data() + ((int64_t)by * ax[0] + bx) * tv;
                    for (int z = 0; z < T; z++)
                        for (int y = 0; y < T; y++)
                            std::memcpy(&slab[((size_t)z * ar[1] + (size_t)by * T + y) * ar[0] + (size_t)bx * T],
                                        t + ((size_t)z * T + y) * T, sizeof(float) * T);
                }
            F.put(slab.data(), slab.size());
        }
    }
    if (F.ok) {
        fseek(F.f, table, SEEK_SET);
        F.put1(grid_off);
    }
    if (!F.ok) return fail(v, GVDB2_ERR_ARG, std::string("write failed: ") + path);
    return GVDB2_OK;
}

gvdb2_status load_vbx(Volume *v, const char *path) {
    if (!path) return fail(v, GVDB2_ERR_ARG, "no file name");
    File F;
    F.f = fopen(path, "rb");
    if (!F.f) return fail(v, GVDB2_ERR_ARG, std::string("cannot open ") + path);
    auto bad = [&](const char *why) { return fail(v, GVDB2_ERR_UNSUPPORTED, std::string("VBX: ") + why); };
    const unsigned char major = F.get1<unsigned char>(), minor = F.get1<unsigned char>();
    float xf[4][3] = {{0, 0, 0}, {0, 0, 0}, {1, 1, 1}, {0, 0, 0}};
    if ((major == 1 && minor >= 11) || major > 1) F.get(&xf[0][0], 12);
    const int32_t grids = F.get1<int32_t>();
    unsigned char masks = major == 1 && minor == 0 ? 1 : 0;
    if (major >= 2) masks = F.get1<unsigned char>();
    if (!F.ok || grids < 1) return bad("truncated header");
    if (masks) return bad("node bitmasks are not supported");
    std::vector<uint64_t> offs((size_t)grids);
    F.get(offs.data(), offs.size());
    fseek(F.f, (long)offs[0], SEEK_SET); // the first grid
    char name[kNameLen];
    F.get(name, kNameLen);
    const char dtype = F.get1<char>(), comps = F.get1<char>(), compress = F.get1<char>();
    float voxelsize[3];
    F.get(voxelsize, 3);
    F.get1<int32_t>(); // leaf count (the level-0 pool below gives it)
    int32_t leafdim[3];
    F.get(leafdim, 3);
    const int32_t apron = F.get1<int32_t>(), nchan = F.get1<int32_t>();
    F.get1<uint64_t>(); // bytes of one channel's atlas
    const char topo = F.get1<char>();
    F.get1<int32_t>(); // topology reuse
    const char layout = F.get1<char>();
    int32_t ax[3], ar[3];
    F.get(ax, 3);
    F.get(ar, 3);
    const int32_t levels = F.get1<int32_t>();
    const uint64_t root = F.get1<uint64_t>();
    if (!F.ok) return bad("truncated grid header");
    if (dtype != 'f' || comps != 1 || compress != 0) return bad("only uncompressed float grids");
    if (topo != 2 || layout != 0) return bad("only GVDB topology in atlas layout");
    if (levels != 5) return bad("only 5-level trees");
    if (nchan < 1 || nchan > kMaxChan) return bad("channel count");
    int32_t ld[5], cnt0[5], w0[5], cnt1[5], w1[5];
    for (int n = 0; n < levels; n++) {
        int32_t row[9];
        F.get(row, 9);
        ld[n] = row[0];
        cnt0[n] = row[5];
        w0[n] = row[6];
        cnt1[n] = row[7];
        w1[n] = row[8];
        if (ld[n] < 1 || ld[n] > 6 || cnt0[n] < 0 || cnt1[n] < 0) return bad("level table");
        if (w0[n] != (int32_t)sizeof(Node)) return bad("node width differs from the 64-byte Node");
        if (n > 0 && cnt1[n] > 0 && (int64_t)w1[n] != (int64_t)sizeof(uint64_t) << (3 * ld[n])) return bad("child lists");
    }
    if (!F.ok) return bad("truncated level table");
    const int depth = (int)((root >> 8) & 0xFF);
    if ((root & 0xFF) != 0 || (root >> 16) != 0 || depth < 1 || depth >= levels || cnt0[depth] != 1)
        return bad("root is not the single node of its level");
    if (leafdim[0] != (1 << ld[0]) || apron < 0 || apron > leafdim[0]) return bad("brick dims");

    // Configure(levels, ld, cnt0) (V:619) and DestroyChannels (V:640)
    v->nlev = 5;
    for (int n = 0; n < kMaxLev; n++) v->logdim[n] = n < 5 ? ld[n] : 0;
    for (int c = 0; c < kMaxChan; c++) v->has_chan[c] = false;
    for (int a = 0; a < 3; a++) {
        v->xf_pretrans[a] = xf[0][a];
        v->xf_angs[a] = xf[1][a];
        v->xf_scale[a] = xf[2][a];
        v->xf_trans[a] = xf[3][a];
    }
    cudaStream_t s = v->stream;
    for (int l = 0; l < kMaxLev; l++) v->pool_cnt[l] = 0;
    for (int n = 0; n < levels; n++) {
        v->pool_cnt[n] = cnt0[n];
        GV_TRY(pool_reserve(v, n, cnt0[n]));
        std::vector<Node> nodes((size_t)cnt0[n]);
        F.get(nodes.data(), nodes.size());
        if (!nodes.empty())
            GV_CUDA(v, cudaMemcpyAsync(v->pool[n].p, nodes.data(), sizeof(Node) * nodes.size(), cudaMemcpyHostToDevice, s));
        GV_CUDA(v, cudaStreamSynchronize(s)); // `nodes` is released at the end of the iteration
    }
    for (int n = 0; n < levels; n++) {
        if (n == 0 || cnt1[n] == 0) continue;
        if (cnt1[n] != cnt0[n]) return bad("child list count differs from the node count");
        std::vector<uint64_t> cl((size_t)((int64_t)cnt1[n] << (3 * ld[n])));
        F.get(cl.data(), cl.size());
        GV_CUDA(v, cudaMemcpyAsync(v->clist[n].p, cl.data(), sizeof(uint64_t) * cl.size(), cudaMemcpyHostToDevice, s));
        GV_CUDA(v, cudaStreamSynchronize(s));
    }
    if (!F.ok) return bad("truncated pools");
    GV_TRY(adopt_pools(v, depth)); // FinishTopology (V:636)

    // channels, then the slots of UpdateAtlas (V:679), then the atlas data
    v->apron = apron;
    for (int a = 0; a < 3; a++) v->subdim[a] = v->default_axiscnt[a];
    v->atlas_cap = (int64_t)v->subdim[0] * v->subdim[1] * v->subdim[2];
    for (int c = 0; c < nchan; c++) {
        v->has_chan[c] = true;
        GV_TRY(alloc_channel_storage(v, c));
    }
    GV_TRY(update_atlas(v));
    const int T = v->tile_res();
    if (ar[0] != ax[0] * T || ar[1] != ax[1] * T || ar[2] != ax[2] * T) return bad("atlas resolution");
    if ((int64_t)ax[0] * ax[1] * ax[2] < v->atlas_last) return bad("atlas smaller than the active bricks");
    const int64_t tv = v->tile_vox(), layer = (int64_t)ax[0] * ax[1];
    std::vector<float> slab((size_t)ar[0] * ar[1] * T), tiles((size_t)(layer * tv));
    for (int c = 0; c < nchan; c++) {
        const int32_t type = F.get1<int32_t>(), stride = F.get1<int32_t>();
        if (!F.ok || type != kTypeFloat || stride != (int32_t)sizeof(float)) return bad("only T_FLOAT channels");
        for (int bz = 0; bz < ax[2]; bz++) {
            F.get(slab.data(), slab.size());
            if (!F.ok) return bad("truncated atlas");
            const int64_t s0 = bz * layer, ns = std::max<int64_t>(0, std::min<int64_t>(layer, v->atlas_last - s0));
            if (ns == 0) continue;
            for (int64_t k = 0; k < ns; k++) {
                const int bx = (int)(k % ax[0]), by = (int)(k / ax[0]);
                float *t = tiles.data() + k * tv;
                for (int z = 0; z < T; z++)
                    for (int y = 0; y < T; y++)
                        std::memcpy(t + ((size_t)z * T + y) * T,
                                    &slab[((size_t)z * ar[1] + (size_t)by * T + y) * ar[0] + (size_t)bx * T],
                                    sizeof(float) * T);
            }
            GV_CUDA(v, cudaMemcpyAsync(v->atlas[c].as<float>() + s0 * tv, tiles.data(),
                                       sizeof(float) * (size_t)(ns * tv), cudaMemcpyHostToDevice, s));
            GV_CUDA(v, cudaStreamSynchronize(s)); // `tiles` is refilled by the next layer
        }
    }
    return GVDB2_OK;
}

} // namespace gvdb2
