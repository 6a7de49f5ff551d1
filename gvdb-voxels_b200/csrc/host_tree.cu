// Host-side operations on the node pools: ActivateSpace and CompactPools.
//
// ActivateSpace: activate the brick that holds a position, one position at
// a time, by the reference's host tree walk (VolumeGVDB::ActivateSpace,
// source/gvdb_library/src/gvdb_volume_gvdb.cpp:2766-2856, with Reparent
// V:2726-2762, AddChildNode V:2707-2723, InsertChild V:2980-3026 in its
// build without bitmasks, GetCoveringNode V:2915-2931, getPosInNode
// V:2858-2875).
//
// The pools live on the device.  A call mirrors them on the host, walks the
// tree for every position in order (so a batch costs one round trip),
// writes the pools back and re-adopts them (leaf map, root, depth).  The
// walk is inherently serial -- each position may add nodes the next one
// descends through -- and the reference runs it on the host as well.
//
// What the walk does, per position p (truncated to int):
//  * no root yet: a root of level 0 (a leaf) at p's covering brick;
//  * p inside the current node: descend, creating each missing child
//    (a fresh node gets its 0xFF-filled child list with its first child);
//  * p outside the root: a new root at the lowest level whose covering node
//    holds both p and the old root; the old root is linked under it (the
//    path to it is created) and then the path to p.
// The result per position is the leaf's pool reference when the leaf
// existed, ID_UNDEFL when this call created it or nothing could be
// activated (p outside the top configured level).
#include "gvdb2_internal.h"

#include <cmath>
#include <string>
#include <vector>

namespace gvdb2 {

gvdb2_status adopt_pools(Volume *v, int depth);

namespace {

inline uint64_t make_ref(int grp, int lev, uint64_t ndx) { return (uint64_t)grp | ((uint64_t)lev << 8) | (ndx << 16); }
inline int ref_lev(uint64_t r) { return (int)((r >> 8) & 0xFF); }
inline int64_t ref_ndx(uint64_t r) { return (int64_t)(r >> 16); }

// The pools, mirrored on the host.  On the device, level l's child lists
// are res(l)^3 entries per node, indexed by node: a node's list is
// allocated with its first child, so list and node indices agree as long
// as nodes get their lists in node order, which the walk keeps.
struct HostTree {
    Volume *v;
    std::vector<Node> nodes[kMaxLev];
    std::vector<uint64_t> lists[kMaxLev];
    int64_t nlists[kMaxLev] = {0};
    uint64_t root = kUndefL;
    bool broken = false; // a list would land out of node order

    Node &node(uint64_t r) { return nodes[ref_lev(r)][ref_ndx(r)]; }

    // GetCoveringNode: the corner of the level-lev node holding p
    void covering(int lev, const int p[3], int out[3]) const {
        const int64_t rng = v->range(lev);
        for (int a = 0; a < 3; a++) {
            if (lev == kMaxLev - 1) {
                out[a] = 0;
                continue;
            }
            int64_t c = (int64_t)p[a] / rng * rng; // truncating division, then one step down for negatives
            if (p[a] < c) c -= rng;
            out[a] = (int)c;
        }
    }

    // getPosInNode: the child bit of p in node r, false when p is outside
    bool child_bit(uint64_t r, const int p[3], uint32_t &bit) {
        const Node &nd = node(r);
        const int res = v->res(nd.mLev);
        const int64_t rng = v->range(nd.mLev);
        int64_t q[3];
        for (int a = 0; a < 3; a++) {
            q[a] = (int64_t)p[a] - nd.mPos[a];
            if (q[a] < 0 || q[a] >= rng) return false;
            q[a] = q[a] * res / rng;
        }
        bit = (uint32_t)((q[2] * res + q[1]) * res + q[0]);
        return true;
    }

    uint64_t child(uint64_t r, uint32_t bit) {
        const Node &nd = node(r);
        if (nd.mChildList == kUndefL) return kUndef64;
        return lists[nd.mLev][(size_t)(ref_ndx(nd.mChildList) * v->res3(nd.mLev) + bit)];
    }

    // AllocateNode + SetupNode(marker = true): levels beyond the configured
    // ones are refused, as the pool allocator does
    uint64_t new_node(int lev, const int pos[3]) {
        if (lev < 0 || lev >= v->nlev) return kUndefL;
        Node nd{};
        nd.mLev = (uint8_t)lev;
        nd.mFlags = 1;
        for (int a = 0; a < 3; a++) {
            nd.mPos[a] = pos[a];
            nd.mValue[a] = -1;
        }
        nd.mParent = kUndefL;
        nd.mChildList = kUndefL;
        nodes[lev].push_back(nd);
        return make_ref(0, lev, nodes[lev].size() - 1);
    }

    // InsertChild: link c under r at bit, giving r its child list first
    uint64_t link(uint64_t r, uint64_t c, uint32_t bit) {
        node(c).mParent = r;
        const int lev = node(r).mLev;
        const int64_t r3 = v->res3(lev);
        if (node(r).mChildList == kUndefL) {
            const int64_t li = nlists[lev]++;
            if (li != ref_ndx(r)) {
                broken = true;
                return kUndefL;
            }
            lists[lev].resize((size_t)((li + 1) * r3), kUndef64);
            node(r).mChildList = make_ref(1, lev, (uint64_t)li);
        }
        lists[lev][(size_t)(ref_ndx(node(r).mChildList) * r3 + bit)] = c;
        return c;
    }

    // AddChildNode: the level-(lev-1) node at bit's position inside r
    uint64_t add_child(uint64_t r, uint32_t bit) {
        const int lev = node(r).mLev, logr = v->logdim[lev], mask = (1 << logr) - 1;
        const int64_t rng = v->range(lev - 1);
        const int loc[3] = {(int)(bit & mask), (int)((bit >> logr) & mask), (int)((bit >> (2 * logr)) & mask)};
        int pos[3];
        for (int a = 0; a < 3; a++) pos[a] = (int)(loc[a] * rng + node(r).mPos[a]);
        const uint64_t c = new_node(lev - 1, pos);
        return c == kUndefL ? kUndefL : link(r, c, bit);
    }

    // the walk from node r toward p, stopping at level stoplev or, when a
    // stop node is given, linking it where p (its corner) belongs
    uint64_t walk(uint64_t r, const int p[3], bool &fresh, uint64_t stop, int stoplev) {
        if (root == kUndefL && r == root) {
            int c[3];
            covering(stoplev, p, c);
            r = root = new_node(stoplev, c);
            if (r == kUndefL) return kUndefL;
        }
        for (int guard = 0; guard < 4 * kMaxLev; guard++) { // each step moves one level
            uint32_t bit = 0;
            if (!child_bit(r, p, bit)) {
                uint64_t up = node(r).mParent;
                if (up == kUndefL) {
                    up = reroot(node(r).mLev, r, p, fresh);
                    if (up == kUndefL) return kUndefL;
                }
                r = up;
                continue;
            }
            const int lev = node(r).mLev;
            if (stop != kUndefL) {
                const Node &sn = node(stop);
                if (p[0] == sn.mPos[0] && p[1] == sn.mPos[1] && p[2] == sn.mPos[2] && child(r, bit) == kUndef64 &&
                    lev == sn.mLev + 1)
                    return link(r, stop, bit);
            }
            if (lev == stoplev) return r;
            uint64_t c = child(r, bit);
            if (c == kUndef64) {
                c = add_child(r, bit);
                if (c == kUndefL) return kUndefL;
                if (lev == 1) fresh = true;
            }
            if (ref_lev(c) == 0) return c;
            r = c;
        }
        broken = true; // unreachable for a consistent tree
        return kUndefL;
    }

    // Reparent: a root covering both the old root and p
    uint64_t reroot(int lev, uint64_t old, const int p[3], bool &fresh) {
        const int op[3] = {node(old).mPos[0], node(old).mPos[1], node(old).mPos[2]};
        int c1[3] = {0, 0, 0}, c2[3];
        bool cover = false;
        while (!cover && lev < kMaxLev) {
            lev++;
            covering(lev, p, c1);
            covering(lev, op, c2);
            cover = c1[0] == c2[0] && c1[1] == c2[1] && c1[2] == c2[2];
        }
        if (lev >= kMaxLev) return kUndefL;
        const uint64_t nr = new_node(lev, c1);
        if (nr == kUndefL) return kUndefL;
        bool ignored = false;
        walk(nr, op, ignored, old, 0);
        const uint64_t leaf = walk(nr, p, fresh, kUndefL, 0);
        root = nr;
        return leaf == kUndefL ? kUndefL : node(leaf).mParent;
    }
};

} // namespace

namespace {

// The device pools into t (levels 0 .. nlev-1); t.root = the node at the
// volume's depth, when there are nodes.
gvdb2_status read_pools(Volume *v, HostTree &t, const char *what) {
    GV_CUDA(v, cudaStreamSynchronize(v->stream));
    t.v = v;
    int64_t total = 0;
    for (int l = 0; l < v->nlev; l++) {
        const int64_t cnt = v->pool_cnt[l];
        total += cnt;
        t.nodes[l].resize((size_t)cnt);
        if (cnt > 0)
            GV_CUDA(v, cudaMemcpy(t.nodes[l].data(), v->pool[l].p, sizeof(Node) * cnt, cudaMemcpyDeviceToHost));
        if (l > 0) {
            t.lists[l].resize((size_t)(cnt * v->res3(l)));
            if (cnt > 0)
                GV_CUDA(v, cudaMemcpy(t.lists[l].data(), v->clist[l].p, sizeof(uint64_t) * t.lists[l].size(),
                                      cudaMemcpyDeviceToHost));
            t.nlists[l] = cnt;
        }
    }
    if (total > 0) {
        const int d = v->depth;
        if (d < 0 || d >= v->nlev || v->pool_cnt[d] < 1 || t.nodes[d][0].mParent != kUndefL)
            return fail(v, GVDB2_ERR_STATE, std::string(what) + ": no root at the volume's depth");
        t.root = make_ref(0, d, 0);
    }
    return GVDB2_OK;
}

// t's pools back to the device, whole, with their counts.
gvdb2_status write_pools(Volume *v, HostTree &t) {
    cudaStream_t s = v->stream;
    for (int l = 0; l < v->nlev; l++) {
        const int64_t cnt = (int64_t)t.nodes[l].size();
        if (cnt == 0 && v->pool_cnt[l] == 0) continue;
        GV_TRY(pool_reserve(v, l, cnt)); // contents are rewritten whole below
        if (cnt > 0)
            GV_CUDA(v, cudaMemcpyAsync(v->pool[l].p, t.nodes[l].data(), sizeof(Node) * cnt, cudaMemcpyHostToDevice, s));
        if (l > 0 && cnt > 0) {
            t.lists[l].resize((size_t)(cnt * v->res3(l)), kUndef64);
            GV_CUDA(v, cudaMemcpyAsync(v->clist[l].p, t.lists[l].data(), sizeof(uint64_t) * t.lists[l].size(),
                                       cudaMemcpyHostToDevice, s));
        }
        v->pool_cnt[l] = cnt;
    }
    GV_CUDA(v, cudaStreamSynchronize(s)); // the host mirror is released on return
    return GVDB2_OK;
}

} // namespace

namespace {
// A refused batch leaves the device pools as they were; its results are all
// ID_UNDEFL, so no entry refers to a node of the discarded host mirror.
gvdb2_status refuse_batch(Volume *v, gvdb2_status st, const char *msg, uint64_t *out, int64_t n) {
    for (int64_t i = 0; i < n; i++) out[i] = kUndefL;
    return fail(v, st, msg);
}
} // namespace

gvdb2_status activate_space(Volume *v, const float *xyz, int64_t n, uint64_t *out) {
    if (v->nlev <= 0) return fail(v, GVDB2_ERR_STATE, "ActivateSpace before Configure");
    if (n == 0) return GVDB2_OK;
    HostTree t;
    GV_TRY(read_pools(v, t, "ActivateSpace"));
    for (int64_t i = 0; i < n; i++) {
        const float *x = xyz + 3 * i;
        if (!(fabsf(x[0]) < 2.0e9f && fabsf(x[1]) < 2.0e9f && fabsf(x[2]) < 2.0e9f)) {
            out[i] = kUndefL; // beyond int (or NaN): outside every node
            continue;
        }
        const int p[3] = {(int)x[0], (int)x[1], (int)x[2]}; // Vector3DF -> Vector3DI truncates toward zero
        if (t.root == kUndefL && (p[0] < 0 || p[1] < 0 || p[2] < 0))
            return refuse_batch(v, GVDB2_ERR_UNSUPPORTED,
                                "ActivateSpace: a first position with a negative coordinate would root the tree at "
                                "negative brick coordinates", out, n);
        bool fresh = false;
        const uint64_t r = t.walk(t.root, p, fresh, kUndefL, 0);
        if (t.broken)
            return refuse_batch(v, GVDB2_ERR_UNSUPPORTED, "ActivateSpace: child lists out of node order", out, n);
        out[i] = (r == kUndefL || fresh) ? kUndefL : r;
    }
    if (t.root == kUndefL) return GVDB2_OK; // nothing was activated
    if (ref_ndx(t.root) != 0)
        return refuse_batch(v, GVDB2_ERR_UNSUPPORTED, "ActivateSpace: new root is not the first node of its level",
                            out, n);
    GV_TRY(write_pools(v, t));
    return adopt_pools(v, ref_lev(t.root));
}

// Pool compaction (no reference counterpart; the reference keeps delinked
// nodes for good).  An incremental rebuild delinks the nodes it no longer
// needs (mParent = ID_UNDEF64, their parent's slot cleared, gvdbDelinkLeafBricks
// / gvdbDelinkBricks, cuda_gvdb_nodes.cuh:401-467) but leaves them in the
// pools, where every sweep over a level still visits them.  Compaction drops
// them, keeps the order of the rest, and rewrites the references: parents,
// child-list entries and child-list indices (list index = node index).  The
// flagged leaves keep their order, so UpdateAtlas hands out the same slots
// and the channel data stay valid.  The rebuild state (full or incremental,
// depth, bounding box) is kept, so the next RebuildTopology continues as it
// would have.
gvdb2_status compact_pools(Volume *v) {
    if (v->nlev <= 0) return fail(v, GVDB2_ERR_STATE, "CompactPools before Configure");
    HostTree t;
    GV_TRY(read_pools(v, t, "CompactPools"));
    if (t.root == kUndefL) return GVDB2_OK;
    std::vector<int64_t> remap[kMaxLev];
    HostTree c;
    c.v = v;
    for (int l = 0; l < v->nlev; l++) {
        remap[l].assign(t.nodes[l].size(), -1);
        for (size_t i = 0; i < t.nodes[l].size(); i++)
            if (t.nodes[l][i].mParent != kUndef64) remap[l][i] = (int64_t)c.nodes[l].size(), c.nodes[l].push_back(t.nodes[l][i]);
    }
    for (int l = 0; l < v->nlev; l++) {
        const int64_t r3 = l > 0 ? v->res3(l) : 0;
        if (l > 0) c.lists[l].assign((size_t)(c.nodes[l].size() * r3), kUndef64);
        for (size_t i = 0; i < c.nodes[l].size(); i++) {
            Node &nd = c.nodes[l][i];
            if (nd.mParent != kUndefL) { // every kept node below the root has a live parent
                const int pl = ref_lev(nd.mParent);
                const int64_t pi = ref_ndx(nd.mParent);
                if (pl != l + 1 || pi >= (int64_t)remap[pl].size() || remap[pl][pi] < 0)
                    return fail(v, GVDB2_ERR_STATE, "CompactPools: a kept node's parent was delinked");
                nd.mParent = make_ref(0, pl, (uint64_t)remap[pl][pi]);
            }
            if (l == 0 || nd.mChildList == kUndefL) continue;
            const int64_t old = ref_ndx(nd.mChildList);
            nd.mChildList = make_ref(1, l, (uint64_t)i);
            for (int64_t b = 0; b < r3; b++) {
                const uint64_t e = t.lists[l][(size_t)(old * r3 + b)];
                if (e == kUndef64) continue;
                const int64_t ci = ref_ndx(e);
                if (ref_lev(e) != l - 1 || ci >= (int64_t)remap[l - 1].size() || remap[l - 1][ci] < 0)
                    return fail(v, GVDB2_ERR_STATE, "CompactPools: a child list holds a delinked node");
                c.lists[l][(size_t)(i * r3 + b)] = make_ref(0, l - 1, (uint64_t)remap[l - 1][ci]);
            }
        }
    }
    const int rl = ref_lev(t.root);
    if (remap[rl][ref_ndx(t.root)] != 0) return fail(v, GVDB2_ERR_STATE, "CompactPools: the root is not first");
    // the rebuild state survives the re-adoption
    const bool rebuild = v->rebuild_topo;
    const int cur = v->cur_depth;
    float lo[3], hi[3];
    for (int a = 0; a < 3; a++) lo[a] = v->posmin[a], hi[a] = v->posmax[a];
    GV_TRY(write_pools(v, c));
    GV_TRY(adopt_pools(v, rl));
    v->rebuild_topo = rebuild;
    v->cur_depth = cur;
    for (int a = 0; a < 3; a++) v->posmin[a] = lo[a], v->posmax[a] = hi[a];
    return GVDB2_OK;
}

} // namespace gvdb2
