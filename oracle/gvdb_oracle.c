/*
 * gvdb_oracle.c -- CPU restatement of GVDB's point -> sparse-volume path.
 *
 * TEST INFRASTRUCTURE ONLY (see gvdb_oracle.h): the checker for the CUDA
 * implementation, never part of the product path.
 *
 * Reference citations use the aliases of gvdb_oracle.h (V, A, P, N, O) with
 * line numbers of the gvdb-voxels sources.  Where the reference has
 * undefined behaviour (out-of-bounds child-list reads, garbage node ids)
 * the restatement takes the evident intent and says so at the spot.
 */
#include "gvdb_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAXLEV 10            /* MAXLEV, gvdb_volume_gvdb.h:40 */
#define ORC_MAXCHAN 32           /* MAX_CHANNEL, N:22 */
#define ID_UNDEFL 0xFFFFFFFFull  /* gvdb_types.h:55 */
#define ID_UNDEF64 0xFFFFFFFFFFFFFFFFull
#define NOHIT 1.0e10f            /* gvdb_types.h:52 */

struct orc_volume {
    int nlev;
    int logdim[ORC_MAXLEV];
    /* node pools, group 0 (nodes) and group 1 (child lists), A:55-91 */
    orc_node *pool[ORC_MAXLEV];
    int64_t pool_cnt[ORC_MAXLEV], pool_cap[ORC_MAXLEV];
    uint64_t *clist[ORC_MAXLEV];
    int64_t clist_cnt[ORC_MAXLEV], clist_cap[ORC_MAXLEV];
    int64_t used_leaves; /* usedNum of pool (0,0) */
    uint64_t root;
    int rebuild_topo, cur_depth, depth;
    float posmin[3], posmax[3];
    /* atlas (all channels share the brick layout of channel 0) */
    int default_axiscnt[3];
    int subdim[3];
    int apron;
    int has_chan[ORC_MAXCHAN];
    double *atlas[ORC_MAXCHAN];
    int64_t atlas_cap;  /* bricks the atlas holds (subdim product) */
    int64_t atlas_last; /* lastEle: slots handed out */
    orc_atlas_node *amap;
    int64_t amap_cnt;
    int32_t *nbr;
    int64_t nbr_cnt;
    /* subcell lists, V:4971-5092 */
    int sc_size, sc_dim, sc_per_brick;
    int64_t num_sc;
    int32_t *sc_cnt, *sc_off, *sc_nid, *sc_pos;
    float *sc_pnt; /* xyz per list entry (InsertPointsSubcell) */
    int64_t sc_len;
    int sc_fp16;                 /* lists hold quantized entries (InsertPointsSubcell_FP16) */
    uint16_t *sc_q, *sc_qvel;    /* 3 per entry: position, velocity (when set) */
    float velmin[3], velrange[3]; /* GetMinMaxVel (V:5469-5521); zero until computed */
};

/* ------------------------------------------------------------------ */
/* small helpers                                                        */
/* ------------------------------------------------------------------ */

static inline uint64_t elem(int grp, int lev, uint64_t ndx) { /* Elem, gvdb_allocator.h:59 */
    return (uint64_t)grp | ((uint64_t)lev << 8) | (ndx << 16);
}
static inline int res_of(const orc_volume *v, int lev) { /* getRes, gvdb_volume_gvdb.h:592 */
    if (lev < 0) return 1;
    return 1 << v->logdim[lev];
}
static inline int64_t res3_of(const orc_volume *v, int lev) {
    int64_t r = res_of(v, lev);
    return r * r * r;
}
static inline int range_of(const orc_volume *v, int lev) { /* getRange, gvdb_volume_gvdb.h:614-619 */
    if (lev == -1) return 1;
    int r = res_of(v, 0);
    for (int l = 1; l <= lev; l++) r *= res_of(v, l);
    return r;
}
static inline int tile_res(const orc_volume *v) { return res_of(v, 0) + 2 * v->apron; }
static inline int64_t tile_vox(const orc_volume *v) {
    int64_t t = tile_res(v);
    return t * t * t;
}
static const float *view_f3(orc_view w, int64_t i) {
    return (const float *)((const char *)w.base + i * (int64_t)w.stride + w.offset);
}
static float view_f1(orc_view w, int64_t i) { return *(const float *)((const char *)w.base + i * (int64_t)w.stride + w.offset); }

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}

/* ------------------------------------------------------------------ */
/* pools                                                                */
/* ------------------------------------------------------------------ */

/* PoolAlloc (A:163-192): append one element, growing capacity x2. */
static int64_t pool_alloc_node(orc_volume *v, int lev) {
    if (v->pool_cnt[lev] >= v->pool_cap[lev]) {
        int64_t nc = v->pool_cap[lev] ? v->pool_cap[lev] * 2 : 4;
        orc_node *np = (orc_node *)realloc(v->pool[lev], (size_t)nc * sizeof(orc_node));
        if (!np) return -1;
        memset(np + v->pool_cap[lev], 0, (size_t)(nc - v->pool_cap[lev]) * sizeof(orc_node));
        v->pool[lev] = np;
        v->pool_cap[lev] = nc;
    }
    if (lev == 0) v->used_leaves++;
    return v->pool_cnt[lev]++;
}
static int64_t pool_alloc_clist(orc_volume *v, int lev) {
    int64_t r3 = res3_of(v, lev);
    if (v->clist_cnt[lev] >= v->clist_cap[lev]) {
        int64_t nc = v->clist_cap[lev] ? v->clist_cap[lev] * 2 : 4;
        uint64_t *np = (uint64_t *)realloc(v->clist[lev], (size_t)(nc * r3) * sizeof(uint64_t));
        if (!np) return -1;
        v->clist[lev] = np;
        v->clist_cap[lev] = nc;
    }
    return v->clist_cnt[lev]++;
}

/* SetupNode (V:2512-2524). */
static void setup_node(orc_volume *v, int lev, int64_t idx, const int pos[3], int marker) {
    orc_node *nd = &v->pool[lev][idx];
    memset(nd, 0, sizeof(*nd));
    nd->mLev = (uint8_t)lev;
    nd->mPos[0] = pos[0];
    nd->mPos[1] = pos[1];
    nd->mPos[2] = pos[2];
    nd->mChildList = ID_UNDEFL;
    nd->mParent = ID_UNDEFL;
    nd->mValue[0] = nd->mValue[1] = nd->mValue[2] = -1;
    nd->mFlags = (uint8_t)(marker ? 1 : 0);
}

/* Allocate a node plus (for interior levels) its 0xFF-filled child list,
 * as in the host loops of V:1288-1331, V:965-988 and V:1088-1111. */
static int64_t alloc_node_with_list(orc_volume *v, int lev, const int pos[3]) {
    int64_t idx = pool_alloc_node(v, lev);
    if (idx < 0) return -1;
    setup_node(v, lev, idx, pos, 1);
    if (lev > 0) {
        int64_t c = pool_alloc_clist(v, lev);
        if (c < 0) return -1;
        v->pool[lev][idx].mChildList = elem(1, lev, (uint64_t)c);
        memset(v->clist[lev] + c * res3_of(v, lev), 0xFF, (size_t)res3_of(v, lev) * sizeof(uint64_t));
    }
    return idx;
}

/* Clear (V:2487-2503): empty pools and atlas without freeing. */
static void clear_topology(orc_volume *v) {
    for (int l = 0; l < ORC_MAXLEV; l++) {
        v->pool_cnt[l] = 0;
        v->clist_cnt[l] = 0;
    }
    v->used_leaves = 0;
    v->root = ID_UNDEFL;
    v->atlas_last = 0;
    v->rebuild_topo = 1;
}

/* top_lev as set by PrepareVDB / PrepareVDBPartially (V:3952-3965,
 * V:3999-4012): the lowest level whose pool holds exactly one node,
 * default 1. */
static int top_level(const orc_volume *v) {
    int tlev = 1;
    for (int n = v->nlev - 1; n >= 0; n--)
        if (v->pool_cnt[n] == 1) tlev = n;
    return tlev;
}

/* getChild (N:115-124), returning the reference's int result: the child
 * index, or -1 for an empty slot (0xFFFF..FF >> 16 truncated to int). */
static int64_t get_child(const orc_volume *v, const orc_node *nd, int64_t bit) {
    uint64_t listid = nd->mChildList;
    if (listid == ID_UNDEFL) return -1;
    int clev = (int)((listid >> 8) & 0xFF);
    uint64_t cndx = listid >> 16;
    if (clev <= 0 || clev >= ORC_MAXLEV || (int64_t)cndx >= v->clist_cnt[clev]) return -1;
    if (bit < 0 || bit >= res3_of(v, clev)) return -1;
    uint64_t c = v->clist[clev][(int64_t)cndx * res3_of(v, clev) + bit];
    return (int64_t)(int32_t)(uint32_t)(c >> 16);
}

/* posInNode of N:313-319 / N:364-370 / N:445-451: (pos - npos) * res / range
 * with C integer arithmetic.  Returns 0 when the position lies outside the
 * node (the reference then reads outside the child list: undefined). */
static int pos_in_node(const orc_volume *v, int lev, const int32_t npos[3], const int pos[3], int64_t *bit) {
    int res = res_of(v, lev), range = range_of(v, lev);
    int p[3];
    for (int a = 0; a < 3; a++) {
        p[a] = (pos[a] - npos[a]) * res / range;
        if (pos[a] - npos[a] < 0 || p[a] >= res) return 0;
    }
    *bit = ((int64_t)p[2] * res + p[1]) * res + p[0];
    return 1;
}

/* getPosParent (N:303-348): node at level stopLev containing pos, or -1. */
static int64_t get_pos_parent(const orc_volume *v, const int pos[3], int stopLev) {
    int tl = top_level(v);
    if (v->pool_cnt[tl] < 1) return -1;
    const orc_node *nd = &v->pool[tl][0];
    int l = nd->mLev;
    if (l == 0) return 0;
    while (l > 0) {
        int64_t bit;
        if (!pos_in_node(v, l, nd->mPos, pos, &bit)) return -1;
        int64_t c = get_child(v, nd, bit);
        l--;
        if (c == -1) return -1;
        if (l == stopLev) return c;
        nd = &v->pool[l][c];
    }
    return -1;
}

/* getPosLeafParent (N:255-288).  The reference rejects posInNode > res
 * (not >=) and never negative offsets; positions outside the start node
 * therefore read past the child list.  Here those return -1. */
static int64_t get_pos_leaf_parent(const orc_volume *v, const int pos[3]) {
    return get_pos_parent(v, pos, 0);
}

/* getParent (N:350-397): node at stopLev containing pos, starting at the
 * top node; 0 when the top node is unflagged or already at stopLev.  A
 * missing child makes the reference follow a garbage id; here -1. */
static int64_t get_parent(const orc_volume *v, int stopLev, const int pos[3]) {
    int tl = top_level(v);
    if (v->pool_cnt[tl] < 1) return -1;
    const orc_node *nd = &v->pool[tl][0];
    if (!nd->mFlags) return 0;
    int l = nd->mLev;
    if (l == stopLev) return 0;
    while (l > stopLev) {
        int64_t bit;
        if (!pos_in_node(v, l, nd->mPos, pos, &bit)) return -1;
        l--;
        int64_t c = get_child(v, nd, bit);
        if (c == -1) return -1;
        if (l == stopLev) return c;
        nd = &v->pool[l][c];
    }
    return -1;
}

/* getNode traversal of getNodeAtPoint (N:199-226, N:243-253) on a float
 * position: returns the leaf index or -1.  The float compares and
 * int((pos-vmin)/vdel) are exact on integers, so floor(pos) is used. */
static int64_t leaf_at_float(const orc_volume *v, float x, float y, float z) {
    int tl = top_level(v);
    if (v->pool_cnt[tl] < 1 || tl == 0) return -1;
    float fp[3] = {x, y, z};
    int lev = tl;
    const orc_node *nd = &v->pool[lev][0];
    int64_t id = -1;
    while (lev > 0) {
        int range = range_of(v, lev), crange = range_of(v, lev - 1);
        int p[3];
        for (int a = 0; a < 3; a++) {
            float vmin = (float)nd->mPos[a];
            float vmax = vmin + (float)range;
            if (fp[a] < vmin || fp[a] >= vmax) return -1;
            p[a] = (int)((fp[a] - vmin) / (float)crange);
        }
        int dim = v->logdim[lev];
        int64_t b = ((((int64_t)p[2] << dim) + p[1]) << dim) + p[0];
        lev--;
        int64_t c = get_child(v, nd, b);
        if (c == -1) return -1;
        id = c;
        nd = &v->pool[lev][c];
    }
    return id;
}

int64_t orc_leaf_of_point(const orc_volume *v, float x, float y, float z) { return leaf_at_float(v, x, y, z); }

/* Integer-voxel variant used by the kernel splats: leaf containing voxel
 * (x,y,z), -1 if none. */
static int64_t leaf_at_voxel(const orc_volume *v, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0) return -1;
    return leaf_at_float(v, (float)x, (float)y, (float)z);
}

/* ------------------------------------------------------------------ */
/* create / configure                                                   */
/* ------------------------------------------------------------------ */

orc_volume *orc_create(void) {
    orc_volume *v = (orc_volume *)calloc(1, sizeof(orc_volume));
    if (!v) return NULL;
    v->root = ID_UNDEFL;
    v->rebuild_topo = 1;   /* Initialize, V:2355 */
    v->cur_depth = -1;     /* V:2356 */
    v->default_axiscnt[0] = 16;  /* SetChannelDefault(16,16,1), V:2348 */
    v->default_axiscnt[1] = 16;
    v->default_axiscnt[2] = 1;
    return v;
}

static void free_subcells(orc_volume *v) {
    free(v->sc_cnt);
    free(v->sc_off);
    free(v->sc_nid);
    free(v->sc_pos);
    free(v->sc_pnt);
    free(v->sc_q);
    free(v->sc_qvel);
    v->sc_cnt = v->sc_off = v->sc_nid = v->sc_pos = NULL;
    v->sc_pnt = NULL;
    v->sc_q = v->sc_qvel = NULL;
    v->sc_fp16 = 0;
    v->num_sc = v->sc_len = 0;
}

void orc_destroy(orc_volume *v) {
    if (!v) return;
    for (int l = 0; l < ORC_MAXLEV; l++) {
        free(v->pool[l]);
        free(v->clist[l]);
    }
    for (int c = 0; c < ORC_MAXCHAN; c++) free(v->atlas[c]);
    free(v->amap);
    free(v->nbr);
    free_subcells(v);
    free(v);
}

/* Configure(q4..q0) (V:2364-2377) -> Configure(levs, r, n) (V:2380-2434):
 * argument order is top level first, so r[0]=q0 is the brick log-dim. */
int orc_configure(orc_volume *v, int q4, int q3, int q2, int q1, int q0) {
    int r[5] = {q0, q1, q2, q3, q4};
    v->nlev = 5;
    for (int n = 0; n < ORC_MAXLEV; n++) v->logdim[n] = 0;
    for (int n = 0; n < 5; n++) {
        if (r[n] < 0 || r[n] > 10) return ORC_ERR_ARG;
        v->logdim[n] = (r[n] == 0) ? 1 : r[n];
    }
    for (int l = 0; l < ORC_MAXLEV; l++) {
        v->pool_cnt[l] = v->clist_cnt[l] = 0;
    }
    clear_topology(v);
    return ORC_OK;
}

int orc_set_channel_default(orc_volume *v, int cx, int cy, int cz) {
    if (cx < 1 || cy < 1 || cz < 1) return ORC_ERR_ARG;
    v->default_axiscnt[0] = cx;
    v->default_axiscnt[1] = cy;
    v->default_axiscnt[2] = cz;
    return ORC_OK;
}

/* Grow every channel to hold `bricks` slots along Z, preserving content by
 * slot: AtlasResize (A:622-650) keeps X/Y brick counts and copies the old
 * Z layers, and slot -> (x,y,z) brick order (getAtlasPos, A:705-715)
 * depends only on the X/Y counts, so slot contents are preserved. */
static int atlas_resize(orc_volume *v, int64_t bricks) {
    int64_t layer = (int64_t)v->subdim[0] * v->subdim[1];
    int nz = (int)ceil((double)((float)bricks / (float)layer));
    if (nz < 1) nz = 1;
    if (nz == v->subdim[2] && v->atlas_cap > 0) return ORC_OK;
    int64_t ncap = layer * nz;
    int64_t tv = tile_vox(v);
    for (int c = 0; c < ORC_MAXCHAN; c++) {
        if (!v->has_chan[c]) continue;
        double *na = (double *)calloc((size_t)(ncap * tv), sizeof(double));
        if (!na) return ORC_ERR_NOMEM;
        if (v->atlas[c]) {
            int64_t keep = v->atlas_cap < ncap ? v->atlas_cap : ncap;
            memcpy(na, v->atlas[c], (size_t)(keep * tv) * sizeof(double));
            free(v->atlas[c]);
        }
        v->atlas[c] = na;
    }
    v->subdim[2] = nz;
    v->atlas_cap = ncap;
    return ORC_OK;
}

/* AddChannel (V:2437-2453) -> AtlasCreate (A:528-560).  Float channels;
 * every channel shares channel 0's brick layout and apron. */
int orc_add_channel(orc_volume *v, int chan, int apron) {
    if (chan < 0 || chan >= ORC_MAXCHAN || apron < 0 || apron > 4) return ORC_ERR_ARG;
    if (v->has_chan[chan]) return ORC_ERR_ARG;
    int any = 0;
    for (int c = 0; c < ORC_MAXCHAN; c++) any |= v->has_chan[c];
    if (any && apron != v->apron) return ORC_ERR_UNSUPPORTED;
    if (!any) {
        v->apron = apron;
        v->subdim[0] = v->default_axiscnt[0];
        v->subdim[1] = v->default_axiscnt[1];
        v->subdim[2] = v->default_axiscnt[2];
        v->atlas_cap = (int64_t)v->subdim[0] * v->subdim[1] * v->subdim[2];
    }
    v->has_chan[chan] = 1;
    v->atlas[chan] = (double *)calloc((size_t)(v->atlas_cap * tile_vox(v)), sizeof(double));
    return v->atlas[chan] ? ORC_OK : ORC_ERR_NOMEM;
}

void orc_request_full_rebuild(orc_volume *v, int flag) { v->rebuild_topo = flag ? 1 : 0; } /* VH:432 */

/* ------------------------------------------------------------------ */
/* topology                                                             */
/* ------------------------------------------------------------------ */

/* GetBoundingBox (V:5404-5467): min/max of pos+trans over ALL points,
 * then mPosMin = max(0, min-1), mPosMax = max(0, max+2). */
static void bounding_box(orc_volume *v, orc_view pos, int n, const float t[3]) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = 0; i < n; i++) {
        const float *p = view_f3(pos, i);
        for (int a = 0; a < 3; a++) {
            float w = p[a] + t[a];
            if (w < mn[a]) mn[a] = w;
            if (w > mx[a]) mx[a] = w;
        }
    }
    for (int a = 0; a < 3; a++) {
        float lo = mn[a] - 1.0f, hi = mx[a] + 2.0f;
        v->posmin[a] = 0 > lo ? 0 : lo;
        v->posmax[a] = 0 > hi ? 0 : hi;
    }
}

/* GetCoveringNode (V:2915-2931) on the float corner truncated to int. */
static void covering_node(const orc_volume *v, int lev, const float pf[3], int out[3]) {
    int range = range_of(v, lev);
    for (int a = 0; a < 3; a++) {
        int p = (int)pf[a];
        if (lev == ORC_MAXLEV - 1) {
            out[a] = 0;
        } else {
            int np = p / range * range;
            if (p < np) np -= range;
            out[a] = np;
        }
    }
}

/* DetermineDepth (V:821-837). Levels beyond the configured ones have
 * resolution 1, so they repeat the top configured level's range. */
static int determine_depth(const orc_volume *v, int rootpos[3]) {
    for (int lev = 0; lev < ORC_MAXLEV; lev++) {
        int a[3], b[3];
        int l = lev < v->nlev ? lev : (lev == ORC_MAXLEV - 1 ? lev : v->nlev - 1);
        if (lev == ORC_MAXLEV - 1) {
            a[0] = a[1] = a[2] = b[0] = b[1] = b[2] = 0;
        } else {
            covering_node(v, l, v->posmin, a);
            covering_node(v, l, v->posmax, b);
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

/* Brick key layout of gvdbCalcBrickId (P:352-382): four uint16 words
 * {z, y, x, lev} little-endian, i.e. lev<<48 | x<<32 | y<<16 | z. */
static inline uint64_t make_key(int lev, int x, int y, int z) {
    return ((uint64_t)(uint16_t)lev << 48) | ((uint64_t)(uint16_t)x << 32) | ((uint64_t)(uint16_t)y << 16) |
           (uint64_t)(uint16_t)z;
}
static inline int key_lev(uint64_t k) { return (int)((k >> 48) & 0xFF); }

typedef struct {
    uint64_t *k;
    int64_t n, cap;
} keyvec;
static int kv_push(keyvec *kv, uint64_t key) {
    if (kv->n >= kv->cap) {
        int64_t nc = kv->cap ? kv->cap * 2 : 1024;
        uint64_t *nk = (uint64_t *)realloc(kv->k, (size_t)nc * sizeof(uint64_t));
        if (!nk) return -1;
        kv->k = nk;
        kv->cap = nc;
    }
    kv->k[kv->n++] = key;
    return 0;
}

/* RadixSortByByte + FindUniqueBrick (V:843-928, P:336-350, P:934-943):
 * ascending sort, keep first of each run, count per level (lev 255 is
 * kept in the list but not counted). */
static void sort_unique(keyvec *kv, int depth, int64_t levcnt[ORC_MAXLEV]) {
    for (int l = 0; l < ORC_MAXLEV; l++) levcnt[l] = 0;
    if (kv->n == 0) return;
    qsort(kv->k, (size_t)kv->n, sizeof(uint64_t), cmp_u64);
    int64_t u = 0;
    for (int64_t i = 0; i < kv->n; i++) {
        if (i == 0 || kv->k[i] != kv->k[i - 1]) {
            kv->k[u++] = kv->k[i];
            int lev = key_lev(kv->k[i]);
            if (lev != 255 && lev < depth) levcnt[lev]++;
        }
    }
    kv->n = u;
}

/* Host allocation loop over sorted unique keys (V:1308-1331 / V:965-988 /
 * V:1088-1111): per level ascending, per key in sorted order. */
static int alloc_from_keys(orc_volume *v, const keyvec *kv, const int64_t levcnt[], int depth) {
    int64_t pre = 0;
    for (int lev = 0; lev < depth; lev++) {
        int range = range_of(v, lev);
        for (int64_t n = pre; n < pre + levcnt[lev]; n++) {
            uint64_t k = kv->k[n];
            int pos[3] = {(int)((k >> 32) & 0xFFFF) * range, (int)((k >> 16) & 0xFFFF) * range, (int)(k & 0xFFFF) * range};
            if (alloc_node_with_list(v, lev, pos) < 0) return ORC_ERR_NOMEM;
        }
        pre += levcnt[lev];
    }
    return ORC_OK;
}

/* gvdbLinkBricks (N:470-505) for one level. */
static void link_level(orc_volume *v, int lev) {
    int pl = lev + 1;
    for (int64_t i = 0; i < v->pool_cnt[lev]; i++) {
        orc_node *nd = &v->pool[lev][i];
        if (!nd->mFlags) continue;
        int pos[3] = {nd->mPos[0], nd->mPos[1], nd->mPos[2]};
        int64_t pid = get_parent(v, pl, pos);
        if (pid < 0 || pid >= v->pool_cnt[pl]) continue; /* reference: UB (garbage parent id) */
        orc_node *pn = &v->pool[pl][pid];
        int res = res_of(v, pl), range = range_of(v, pl);
        int p[3];
        for (int a = 0; a < 3; a++) p[a] = (nd->mPos[a] - pn->mPos[a]) * res / range;
        int64_t bit = ((int64_t)p[2] * res + p[1]) * res + p[0];
        if (p[0] > res || p[0] < 0 || p[1] > res || p[1] < 0 || p[2] > res || p[2] < 0) continue;
        nd->mParent = ((uint64_t)pid << 16) | ((uint64_t)pl << 8);
        uint64_t cndx = pn->mChildList >> 16;
        if ((int64_t)cndx >= v->pool_cnt[pl]) continue;
        if (bit >= res3_of(v, pl)) continue; /* p == res: reference writes past the list */
        v->clist[pl][(int64_t)cndx * res3_of(v, pl) + bit] = ((uint64_t)i << 16) | ((uint64_t)lev << 8);
    }
}

static void link_all(orc_volume *v, int depth) {
    for (int lev = depth - 1; lev >= 0; lev--) link_level(v, lev);
}

/* Visit the level-`lev` node corners of gvdbCalcExtraBrickId /
 * gvdbCalcIncreExtraBrickId: bmin = int(int(w) - r), bmax = int(int(w) + k*r)
 * with C truncating division (P:433-434, P:481-482, loops P:440-444). */
static void box_bounds(const float w[3], float radius, float kmax, int bmin[3], int bmax[3]) {
    for (int a = 0; a < 3; a++) {
        int iw = (int)w[a];
        bmin[a] = (int)((float)iw - radius);
        bmax[a] = (int)((float)iw + kmax * radius);
    }
}

/* Activation-box corners outside the root node are skipped: the reference's
 * getPosParent (N:303-348) has no bounds check and reads past the root's
 * child list there (undefined); negative corners are outside too. */
static int outside_root(const orc_volume *v, const int nd[3], int depth) {
    if (v->pool_cnt[depth] < 1) return 1;
    const orc_node *r = &v->pool[depth][0];
    int range = range_of(v, depth);
    for (int a = 0; a < 3; a++)
        if (nd[a] < r->mPos[a] || nd[a] >= r->mPos[a] + range) return 1;
    return 0;
}

/* gvdbCalcBrickId (P:352-382) + ActivateBricksGPU host part (V:1229-1413)
 * and, for radius >= 1, ActivateExtraBricksGPU (V:931-1016) with
 * gvdbCalcExtraBrickId (P:467-512). */
static int activate_bricks_full(orc_volume *v, orc_view pos, int n, float radius, const float orig[3], int depth,
                                const int rootpos[3]) {
    keyvec kv = {0};
    for (int64_t i = 0; i < n; i++) {
        const float *p = view_f3(pos, i);
        float w[3] = {p[0] + orig[0], p[1] + orig[1], p[2] + orig[2]};
        if (w[0] < 0 || w[1] < 0 || w[2] < 0) {
            for (int lev = 0; lev < depth; lev++)
                if (kv_push(&kv, make_key(255, 0, 0, 0))) goto nomem;
            continue;
        }
        for (int lev = 0; lev < depth; lev++) {
            int r = range_of(v, lev);
            /* GetCoveringNode device variant (P:88-100): floor(w / r) * r */
            int c[3];
            for (int a = 0; a < 3; a++) c[a] = (int)w[a] / r;
            if (kv_push(&kv, make_key(lev, c[0], c[1], c[2]))) goto nomem;
        }
    }
    int64_t levcnt[ORC_MAXLEV];
    sort_unique(&kv, depth, levcnt);

    /* root first (V:1290-1300) */
    {
        int64_t ridx = alloc_node_with_list(v, depth, rootpos);
        if (ridx < 0) goto nomem;
        v->root = elem(0, depth, (uint64_t)ridx);
    }
    if (alloc_from_keys(v, &kv, levcnt, depth)) goto nomem;
    link_all(v, depth); /* V:1395-1401 */

    if (radius >= 1) {
        kv.n = 0;
        for (int64_t i = 0; i < n; i++) {
            const float *p = view_f3(pos, i);
            float w[3] = {p[0] + orig[0], p[1] + orig[1], p[2] + orig[2]};
            if (w[0] < 0 || w[1] < 0 || w[2] < 0) continue;
            int bmin[3], bmax[3];
            box_bounds(w, radius, 2.0f, bmin, bmax);
            for (int lev = 0; lev < depth; lev++) {
                int rr = range_of(v, lev);
                int nd[3];
                for (nd[0] = bmin[0] / rr * rr; nd[0] <= bmax[0] / rr * rr; nd[0] += rr)
                    for (nd[1] = bmin[1] / rr * rr; nd[1] <= bmax[1] / rr * rr; nd[1] += rr)
                        for (nd[2] = bmin[2] / rr * rr; nd[2] <= bmax[2] / rr * rr; nd[2] += rr) {
                            if (outside_root(v, nd, depth)) continue;
                            if (get_pos_parent(v, nd, lev) == -1)
                                if (kv_push(&kv, make_key(lev, nd[0] / rr, nd[1] / rr, nd[2] / rr))) goto nomem;
                        }
            }
        }
        sort_unique(&kv, depth, levcnt);
        if (alloc_from_keys(v, &kv, levcnt, depth)) goto nomem;
        link_all(v, depth);
    }
    free(kv.k);
    return ORC_OK;
nomem:
    free(kv.k);
    return ORC_ERR_NOMEM;
}

/* gvdbDelinkLeafBricks (N:401-429). */
static void delink_leaves(orc_volume *v) {
    for (int64_t i = 0; i < v->pool_cnt[0]; i++) {
        orc_node *nd = &v->pool[0][i];
        if (nd->mFlags) continue;
        if (nd->mParent == ID_UNDEF64) continue;
        int pos[3] = {nd->mPos[0], nd->mPos[1], nd->mPos[2]};
        int64_t pid = get_parent(v, 1, pos);
        nd->mParent = ID_UNDEF64;
        if (pid < 0 || pid >= v->pool_cnt[1]) continue; /* reference: UB */
        orc_node *pn = &v->pool[1][pid];
        int res = res_of(v, 1), range = range_of(v, 1);
        int p[3];
        for (int a = 0; a < 3; a++) p[a] = (nd->mPos[a] - pn->mPos[a]) * res / range;
        int64_t bit = ((int64_t)p[2] * res + p[1]) * res + p[0];
        uint64_t cndx = pn->mChildList >> 16;
        if (bit >= 0 && bit < res3_of(v, 1)) v->clist[1][(int64_t)cndx * res3_of(v, 1) + bit] = ID_UNDEF64;
    }
}

/* gvdbDelinkBricks (N:431-467) for one interior level. */
static void delink_level(orc_volume *v, int lev) {
    int64_t r3 = res3_of(v, lev);
    for (int64_t i = 0; i < v->pool_cnt[lev]; i++) {
        orc_node *nd = &v->pool[lev][i];
        if (nd->mParent == ID_UNDEF64) {
            nd->mFlags = 0;
            continue;
        }
        const uint64_t *cl = v->clist[lev] + i * r3;
        int any = 0;
        for (int64_t c = 0; c < r3; c++)
            if (cl[c] != ID_UNDEF64) {
                any = 1;
                break;
            }
        if (any) {
            nd->mFlags = 1;
            continue;
        }
        nd->mFlags = 0;
        int pos[3] = {nd->mPos[0], nd->mPos[1], nd->mPos[2]};
        int64_t pid = get_parent(v, lev + 1, pos);
        nd->mParent = ID_UNDEF64;
        if (pid < 0 || pid >= v->pool_cnt[lev + 1]) continue;
        orc_node *pn = &v->pool[lev + 1][pid];
        int res = res_of(v, lev + 1), range = range_of(v, lev + 1);
        int p[3];
        for (int a = 0; a < 3; a++) p[a] = (nd->mPos[a] - pn->mPos[a]) * res / range;
        int64_t bit = ((int64_t)p[2] * res + p[1]) * res + p[0];
        uint64_t cndx = pn->mChildList >> 16;
        if (bit >= 0 && bit < res3_of(v, lev + 1))
            v->clist[lev + 1][(int64_t)cndx * res3_of(v, lev + 1) + bit] = ID_UNDEF64;
    }
}

/* ActivateIncreBricksGPU (V:1020-1156) with gvdbCalcIncreExtraBrickId
 * (P:420-465). */
static int activate_bricks_incremental(orc_volume *v, orc_view pos, int n, float radius, const float orig[3], int depth,
                                       int accum) {
    if (v->pool_cnt[0] == 0) return ORC_OK;
    int64_t total = v->pool_cnt[0];
    int32_t *marker = (int32_t *)calloc((size_t)total, sizeof(int32_t));
    if (!marker) return ORC_ERR_NOMEM;
    if (accum)
        for (int64_t i = 0; i < total; i++) marker[i] = v->pool[0][i].mFlags;
    keyvec kv = {0};
    for (int64_t i = 0; i < n; i++) {
        const float *p = view_f3(pos, i);
        float w[3] = {p[0] + orig[0], p[1] + orig[1], p[2] + orig[2]};
        if (w[0] < 0 || w[1] < 0 || w[2] < 0) continue;
        int bmin[3], bmax[3];
        box_bounds(w, radius, 1.0f, bmin, bmax);
        for (int lev = 0; lev < depth; lev++) {
            int rr = range_of(v, lev);
            int nd[3];
            for (nd[0] = bmin[0] / rr * rr; nd[0] <= bmax[0] / rr * rr; nd[0] += rr)
                for (nd[1] = bmin[1] / rr * rr; nd[1] <= bmax[1] / rr * rr; nd[1] += rr)
                    for (nd[2] = bmin[2] / rr * rr; nd[2] <= bmax[2] / rr * rr; nd[2] += rr) {
                        if (outside_root(v, nd, depth)) continue;
                        int64_t pid = get_pos_parent(v, nd, lev);
                        if (pid == -1) {
                            if (kv_push(&kv, make_key(lev, nd[0] / rr, nd[1] / rr, nd[2] / rr))) goto nomem;
                        } else if (lev == 0 && pid < total) {
                            marker[pid] = 1;
                        }
                    }
        }
    }
    if (kv.n == 0) { /* no new node: return before flags are touched (V:1065) */
        free(kv.k);
        free(marker);
        return ORC_OK;
    }
    int64_t levcnt[ORC_MAXLEV];
    sort_unique(&kv, depth, levcnt);
    for (int64_t i = 0; i < total; i++) v->pool[0][i].mFlags = (uint8_t)(marker[i] ? 1 : 0); /* V:1078-1081 */
    if (alloc_from_keys(v, &kv, levcnt, depth)) goto nomem;
    link_all(v, depth);
    delink_leaves(v);
    for (int lev = 1; lev < depth; lev++) delink_level(v, lev);
    {
        int64_t used = v->pool_cnt[0]; /* V:1144-1147 */
        for (int64_t i = 0; i < v->pool_cnt[0]; i++)
            if (!v->pool[0][i].mFlags) used--;
        v->used_leaves = used;
    }
    free(kv.k);
    free(marker);
    return ORC_OK;
nomem:
    free(kv.k);
    free(marker);
    return ORC_ERR_NOMEM;
}

/* RebuildTopology (V:1181-1218), including the mCurrDepth quirk: the first
 * full rebuild leaves mCurrDepth = -1, so the second call also rebuilds. */
int orc_rebuild_topology(orc_volume *v, orc_view pos, int n, float radius, const float orig[3]) {
    if (v->nlev == 0 || n < 0) return ORC_ERR_ARG;
    bounding_box(v, pos, n, orig);
    int rootpos[3];
    int depth = determine_depth(v, rootpos);
    if (depth == 0 || depth > 5 || depth < 0) return ORC_ERR_DEPTH;
    if (v->rebuild_topo) {
        clear_topology(v);
    } else if (depth != v->cur_depth) {
        clear_topology(v);
        v->rebuild_topo = 1;
        v->cur_depth = depth;
    }
    v->depth = depth;
    int st;
    if (v->rebuild_topo) {
        st = activate_bricks_full(v, pos, n, radius, orig, depth, rootpos);
        v->rebuild_topo = 0;
    } else {
        st = activate_bricks_incremental(v, pos, n, radius, orig, depth, 0);
    }
    return st;
}

/* AccumulateTopology (V:1158-1178). */
int orc_accumulate_topology(orc_volume *v, orc_view pos, int n, float radius, const float orig[3], int min_depth) {
    if (v->nlev == 0 || n < 0) return ORC_ERR_ARG;
    bounding_box(v, pos, n, orig);
    int rootpos[3];
    int depth = determine_depth(v, rootpos);
    if (depth < min_depth) depth = min_depth;
    if (depth == 0 || depth > 5 || depth < 0) return ORC_ERR_DEPTH;
    if (v->rebuild_topo) return orc_rebuild_topology(v, pos, n, radius, orig);
    v->depth = depth;
    return activate_bricks_incremental(v, pos, n, radius, orig, depth, 1);
}

/* ------------------------------------------------------------------ */
/* ActivateSpace: the host tree walk that activates the brick holding   */
/* one position, creating the root, the path and, when the position is  */
/* outside the tree, a new covering root (V:2707-2856, V:2980-3026).    */
/* ------------------------------------------------------------------ */

static orc_node *node_ref(orc_volume *v, uint64_t id) { return &v->pool[(id >> 8) & 0xFF][id >> 16]; }

/* GetCoveringNode (V:2915-2931) of an integer position. */
static void covering_node_i(const orc_volume *v, int lev, const int pos[3], int out[3]) {
    int range = range_of(v, lev);
    for (int a = 0; a < 3; a++) {
        if (lev == ORC_MAXLEV - 1) {
            out[a] = 0;
        } else {
            int np = pos[a] / range * range;
            if (pos[a] < np) np -= range;
            out[a] = np;
        }
    }
}

/* getPosInNode (V:2858-2875), the host form of the device test above:
 * child bit of pos inside node id, 0 if outside. */
static int node_bit(orc_volume *v, uint64_t id, const int pos[3], uint32_t *bit) {
    const orc_node *nd = node_ref(v, id);
    int64_t b = 0;
    const int in = pos_in_node(v, nd->mLev, nd->mPos, pos, &b);
    *bit = in ? (uint32_t)b : 0u;
    return in;
}

/* getChildNode (V:3079-3091, no bitmasks). */
static uint64_t child_at(orc_volume *v, uint64_t id, uint32_t b) {
    const orc_node *nd = node_ref(v, id);
    if (nd->mChildList == ID_UNDEFL) return ID_UNDEF64;
    return v->clist[nd->mLev][(int64_t)(nd->mChildList >> 16) * res3_of(v, nd->mLev) + b];
}

/* InsertChild (V:2980-3026, no bitmasks): the child list is allocated,
 * 0xFF-filled, with the node's first child. */
static uint64_t insert_child(orc_volume *v, uint64_t id, uint64_t child, uint32_t b) {
    node_ref(v, child)->mParent = id;
    const int lev = node_ref(v, id)->mLev;
    if (node_ref(v, id)->mChildList == ID_UNDEFL) {
        int64_t c = pool_alloc_clist(v, lev);
        if (c < 0) return ID_UNDEFL;
        node_ref(v, id)->mChildList = elem(1, lev, (uint64_t)c);
        memset(v->clist[lev] + c * res3_of(v, lev), 0xFF, (size_t)res3_of(v, lev) * sizeof(uint64_t));
    }
    v->clist[lev][(int64_t)(node_ref(v, id)->mChildList >> 16) * res3_of(v, lev) + b] = child;
    return child;
}

/* AddChildNode (V:2707-2723): a node of level plev-1 at the child position
 * of bit b (getPosFromBit, gvdb_volume_gvdb.h:602-609), linked under id. */
static uint64_t add_child_node(orc_volume *v, uint64_t id, const int ppos[3], int plev, uint32_t b) {
    const int lev = plev - 1;
    int64_t idx = pool_alloc_node(v, lev);
    if (idx < 0) return ID_UNDEFL;
    const int logr = v->logdim[plev], mask = (1 << logr) - 1, rng = range_of(v, lev);
    const int p[3] = {(int)(b & mask) * rng + ppos[0], (int)((b >> logr) & mask) * rng + ppos[1],
                      (int)((b >> (2 * logr)) & mask) * rng + ppos[2]};
    setup_node(v, lev, idx, p, 1);
    return insert_child(v, id, elem(0, lev, (uint64_t)idx), b);
}

static uint64_t activate_space(orc_volume *v, uint64_t id, const int pos[3], int *bnew, uint64_t stop, int stoplev);

/* Reparent (V:2726-2762): a root of the lowest level whose covering node
 * holds both the old root and pos; the old root is linked in (stop node)
 * and the path to pos created.  Returns the parent of pos's leaf. */
static uint64_t reparent(orc_volume *v, int lev, uint64_t prev, const int pos[3], int *bnew) {
    const int pp[3] = {node_ref(v, prev)->mPos[0], node_ref(v, prev)->mPos[1], node_ref(v, prev)->mPos[2]};
    int p1[3] = {0, 0, 0}, p2[3];
    int cover = 0;
    while (!cover && lev < ORC_MAXLEV) {
        lev++;
        covering_node_i(v, lev, pos, p1);
        covering_node_i(v, lev, pp, p2);
        cover = p1[0] == p2[0] && p1[1] == p2[1] && p1[2] == p2[2];
    }
    if (lev >= ORC_MAXLEV || lev >= v->nlev) return ID_UNDEFL; /* PoolAlloc refuses unconfigured levels (A:165) */
    int64_t idx = pool_alloc_node(v, lev);
    if (idx < 0) return ID_UNDEFL;
    setup_node(v, lev, idx, p1, 1);
    const uint64_t root = elem(0, lev, (uint64_t)idx);
    int bn = 0;
    activate_space(v, root, pp, &bn, prev, 0);
    const uint64_t leaf = activate_space(v, root, pos, bnew, ID_UNDEFL, 0);
    v->root = root;
    return leaf == ID_UNDEFL ? ID_UNDEFL : node_ref(v, leaf)->mParent;
}

/* ActivateSpace (V:2804-2856) with a stop node and a stop level. */
static uint64_t activate_space(orc_volume *v, uint64_t id, const int pos[3], int *bnew, uint64_t stop, int stoplev) {
    if (v->root == ID_UNDEFL && id == v->root) { /* first node: a root of the stop level */
        int p[3];
        covering_node_i(v, stoplev, pos, p);
        int64_t idx = pool_alloc_node(v, stoplev);
        if (idx < 0) return ID_UNDEFL;
        setup_node(v, stoplev, idx, p, 1);
        v->root = id = elem(0, stoplev, (uint64_t)idx);
    }
    uint32_t b;
    if (node_bit(v, id, pos, &b)) {
        const int lev = node_ref(v, id)->mLev;
        if (stop != ID_UNDEFL) {
            const orc_node *sn = node_ref(v, stop);
            if (pos[0] == sn->mPos[0] && pos[1] == sn->mPos[1] && pos[2] == sn->mPos[2] &&
                child_at(v, id, b) == ID_UNDEF64 && lev == sn->mLev + 1)
                return insert_child(v, id, stop, b);
        }
        if (lev == stoplev) return id;
        uint64_t child = child_at(v, id, b);
        if (child == ID_UNDEF64) {
            const int pp[3] = {node_ref(v, id)->mPos[0], node_ref(v, id)->mPos[1], node_ref(v, id)->mPos[2]};
            child = add_child_node(v, id, pp, lev, b);
            if (child == ID_UNDEFL) return ID_UNDEFL;
            if (lev == 1) *bnew = 1;
        }
        if (((child >> 8) & 0xFF) == 0) return child; /* isLeaf */
        return activate_space(v, child, pos, bnew, stop, stoplev);
    }
    uint64_t parent = node_ref(v, id)->mParent;
    if (parent == ID_UNDEFL) {
        parent = reparent(v, node_ref(v, id)->mLev, id, pos, bnew);
        if (parent == ID_UNDEFL) return ID_UNDEFL;
    }
    return activate_space(v, parent, pos, bnew, stop, stoplev);
}

/* ActivateSpace(Vector3DF) (V:2766-2774): the position truncated to int;
 * returns the leaf's pool reference when it existed already, ID_UNDEFL
 * when it was created or nothing could be activated. */
uint64_t orc_activate_space(orc_volume *v, float x, float y, float z) {
    if (v->nlev == 0) return ID_UNDEFL;
    const int pos[3] = {(int)x, (int)y, (int)z};
    int bnew = 0;
    uint64_t id = activate_space(v, v->root, pos, &bnew, ID_UNDEFL, 0);
    if (id == ID_UNDEFL || bnew) return ID_UNDEFL;
    return id;
}

uint64_t orc_root(const orc_volume *v) { return v->root; }

/* ComputeBounds (V:1792-1816): mVoxMin = mVoxMax = leaf 0's corner (its flag
 * not consulted), then over the flagged leaves the min of the corners and
 * the max of corner + range(0), compared as floats against the int corners
 * as the reference does; mObjMin/mObjMax equal them.  Returns -1 with no
 * leaf (the reference would read a leaf that does not exist). */
int orc_compute_bounds(const orc_volume *v, float vmin[3], float vmax[3]) {
    if (v->nlev == 0 || v->pool_cnt[0] == 0) return -1;
    const int range = range_of(v, 0);
    const orc_node *n0 = &v->pool[0][0];
    for (int a = 0; a < 3; a++) vmin[a] = vmax[a] = (float)n0->mPos[a];
    for (int64_t i = 0; i < v->pool_cnt[0]; i++) {
        const orc_node *nd = &v->pool[0][i];
        if (!nd->mFlags) continue;
        for (int a = 0; a < 3; a++) {
            if ((float)nd->mPos[a] < vmin[a]) vmin[a] = (float)nd->mPos[a];
            if ((float)(nd->mPos[a] + range) > vmax[a]) vmax[a] = (float)(nd->mPos[a] + range);
        }
    }
    return 0;
}

/* The reference's host path of a topology build from points (the CPU-side
 * equivalent of RebuildTopology, V:1181-1218): ActivateSpace (V:2766-2856)
 * at every leaf-brick corner of each point's activation box [int(w) - r,
 * int(w) + 2r] (the box of gvdbCalcExtraBrickId, P:467-512; it holds the
 * point's own brick), one position at a time, in point order, so the leaves
 * cover the same bricks as a full rebuild.  Used as the timed host baseline;
 * returns the number of ActivateSpace calls, or -1 when a walk failed. */
int64_t orc_activate_points(orc_volume *v, orc_view pos, int64_t n, float radius, const float orig[3]) {
    if (v->nlev == 0) return -1;
    const int rr = range_of(v, 0);
    int64_t calls = 0;
    for (int64_t i = 0; i < n; i++) {
        const float *p = view_f3(pos, i);
        const float w[3] = {p[0] + orig[0], p[1] + orig[1], p[2] + orig[2]};
        if (w[0] < 0 || w[1] < 0 || w[2] < 0) continue;
        int bmin[3], bmax[3];
        box_bounds(w, radius, 2.0f, bmin, bmax);
        int nd[3];
        for (nd[0] = bmin[0] / rr * rr; nd[0] <= bmax[0] / rr * rr; nd[0] += rr)
            for (nd[1] = bmin[1] / rr * rr; nd[1] <= bmax[1] / rr * rr; nd[1] += rr)
                for (nd[2] = bmin[2] / rr * rr; nd[2] <= bmax[2] / rr * rr; nd[2] += rr) {
                    if (nd[0] < 0 || nd[1] < 0 || nd[2] < 0) continue;
                    int bnew = 0;
                    if (activate_space(v, v->root, nd, &bnew, ID_UNDEFL, 0) == ID_UNDEFL && !bnew) return -1;
                    calls++;
                }
    }
    return calls;
}

/* CompactPools (no reference counterpart): the nodes an incremental rebuild
 * delinked (mParent = ID_UNDEF64, gvdbDelinkLeafBricks / gvdbDelinkBricks,
 * N:401-467) are dropped; the rest keep their order and their references
 * (parents, child-list entries, child-list index = node index) are
 * renumbered.  Moves run toward lower indices in increasing order, so the
 * compaction is done in place. */
int orc_compact_pools(orc_volume *v) {
    if (v->root == ID_UNDEFL) return ORC_OK;
    int64_t *remap[ORC_MAXLEV] = {0};
    int64_t kept[ORC_MAXLEV] = {0};
    int st = ORC_OK;
    for (int l = 0; l < v->nlev; l++) {
        remap[l] = (int64_t *)malloc(sizeof(int64_t) * (size_t)(v->pool_cnt[l] + 1));
        if (!remap[l]) {
            st = ORC_ERR_STATE;
            goto done;
        }
        for (int64_t i = 0; i < v->pool_cnt[l]; i++) remap[l][i] = v->pool[l][i].mParent == ID_UNDEF64 ? -1 : kept[l]++;
    }
    for (int l = 0; l < v->nlev; l++) {
        const int64_t r3 = l > 0 ? res3_of(v, l) : 0;
        for (int64_t i = 0; i < v->pool_cnt[l]; i++) {
            const int64_t ni = remap[l][i];
            if (ni < 0) continue;
            orc_node nd = v->pool[l][i];
            if (nd.mParent != ID_UNDEFL) {
                const int pl = (int)((nd.mParent >> 8) & 0xFF);
                const int64_t pi = (int64_t)(nd.mParent >> 16);
                if (pl != l + 1 || pi >= v->pool_cnt[pl] || remap[pl][pi] < 0) {
                    st = ORC_ERR_STATE;
                    goto done;
                }
                nd.mParent = elem(0, pl, (uint64_t)remap[pl][pi]);
            }
            if (l > 0 && nd.mChildList != ID_UNDEFL) {
                const uint64_t *src = v->clist[l] + (int64_t)(nd.mChildList >> 16) * r3;
                uint64_t *dst = v->clist[l] + ni * r3;
                for (int64_t b = 0; b < r3; b++) {
                    const uint64_t e = src[b];
                    uint64_t ne = ID_UNDEF64;
                    if (e != ID_UNDEF64) {
                        const int64_t ci = (int64_t)(e >> 16);
                        if ((int)((e >> 8) & 0xFF) != l - 1 || ci >= v->pool_cnt[l - 1] || remap[l - 1][ci] < 0) {
                            st = ORC_ERR_STATE;
                            goto done;
                        }
                        ne = elem(0, l - 1, (uint64_t)remap[l - 1][ci]);
                    }
                    dst[b] = ne; /* dst <= src: an entry is read before it is overwritten */
                }
                nd.mChildList = elem(1, l, (uint64_t)ni);
            }
            v->pool[l][ni] = nd;
        }
    }
    {
        const int rl = (int)((v->root >> 8) & 0xFF);
        v->root = elem(0, rl, (uint64_t)remap[rl][v->root >> 16]);
    }
    for (int l = 0; l < v->nlev; l++) {
        v->pool_cnt[l] = kept[l];
        if (l > 0) v->clist_cnt[l] = kept[l];
    }
done:
    for (int l = 0; l < ORC_MAXLEV; l++) free(remap[l]);
    return st;
}

/* ------------------------------------------------------------------ */
/* atlas                                                                */
/* ------------------------------------------------------------------ */

static void atlas_pos(const orc_volume *v, int64_t id, int out[3]) { /* getAtlasPos, A:705-715 */
    int64_t a2 = (int64_t)v->subdim[0] * v->subdim[1];
    int z = (int)(id / a2);
    id -= (int64_t)z * a2;
    int y = (int)(id / v->subdim[0]);
    id -= (int64_t)y * v->subdim[0];
    int x = (int)id;
    int br = tile_res(v);
    out[0] = x * br + v->apron;
    out[1] = y * br + v->apron;
    out[2] = z * br + v->apron;
}

/* slot of an atlas-voxel coordinate (getAtlasMapNode, A:674-681) */
static int64_t slot_of_atlas_voxel(const orc_volume *v, const int q[3], int local[3]) {
    int br = tile_res(v);
    int b[3];
    for (int a = 0; a < 3; a++) {
        if (q[a] < 0) return -1;
        b[a] = q[a] / br;
        local[a] = q[a] % br;
    }
    if (b[0] >= v->subdim[0] || b[1] >= v->subdim[1] || b[2] >= v->subdim[2]) return -1;
    return ((int64_t)b[2] * v->subdim[1] + b[1]) * v->subdim[0] + b[0];
}
static inline int64_t tile_index(const orc_volume *v, const int local[3]) {
    int br = tile_res(v);
    return ((int64_t)local[2] * br + local[1]) * br + local[0];
}
/* slot of a leaf from its mValue, -1 if unassigned */
static int64_t slot_of_leaf(const orc_volume *v, int64_t leaf) {
    const orc_node *nd = &v->pool[0][leaf];
    int q[3] = {nd->mValue[0], nd->mValue[1], nd->mValue[2]};
    if (q[0] < 0 || q[1] < 0 || q[2] < 0) return -1;
    int local[3];
    int64_t s = slot_of_atlas_voxel(v, q, local);
    if (s < 0 || s >= v->atlas_last) return -1;
    return s;
}

/* UpdateAtlas (V:2630-2704) with AtlasAlloc (A:692-703). */
int orc_update_atlas(orc_volume *v) {
    int any = 0;
    for (int c = 0; c < ORC_MAXCHAN; c++) any |= v->has_chan[c];
    if (!any) return ORC_ERR_STATE;
    int64_t total = v->pool_cnt[0], used = v->used_leaves;
    v->atlas_last = 0; /* AtlasEmptyAll */
    if (used > v->atlas_cap) {
        int st = atlas_resize(v, used);
        if (st) return st;
    }
    for (int64_t n = 0; n < total; n++) {
        orc_node *nd = &v->pool[0][n];
        if (!nd->mFlags) continue;
        if (v->atlas_last >= v->atlas_cap) {
            int st = atlas_resize(v, v->atlas_last + (int64_t)v->subdim[0] * v->subdim[1]);
            if (st) return st;
        }
        int64_t id = v->atlas_last++;
        atlas_pos(v, id, nd->mValue);
    }
    /* AllocateAtlasMap + ClearMapping + AssignMapping (A:471-496, V:2559-2588) */
    free(v->amap);
    v->amap_cnt = v->atlas_cap;
    v->amap = (orc_atlas_node *)malloc((size_t)v->amap_cnt * sizeof(orc_atlas_node));
    if (!v->amap) return ORC_ERR_NOMEM;
    for (int64_t s = 0; s < v->amap_cnt; s++) {
        v->amap[s].mPos[0] = v->amap[s].mPos[1] = v->amap[s].mPos[2] = (int32_t)ID_UNDEFL;
        v->amap[s].mLeafID = (int32_t)ID_UNDEFL;
    }
    for (int64_t n = 0; n < total; n++) {
        orc_node *nd = &v->pool[0][n];
        if (!nd->mFlags) continue;
        int local[3];
        int64_t s = slot_of_atlas_voxel(v, nd->mValue, local);
        if (s < 0) return ORC_ERR_STATE;
        v->amap[s].mPos[0] = nd->mPos[0];
        v->amap[s].mPos[1] = nd->mPos[1];
        v->amap[s].mPos[2] = nd->mPos[2];
        v->amap[s].mLeafID = (int32_t)n;
    }
    return ORC_OK;
}

/* ClearChannel -> AtlasFill -> kernelFillTex (V:1596-1603, A:813-822,
 * cuda_gvdb_copydata.cu:21-27): zero the whole atlas. */
int orc_clear_channel(orc_volume *v, int chan) {
    if (chan < 0 || chan >= ORC_MAXCHAN || !v->has_chan[chan]) return ORC_ERR_ARG;
    memset(v->atlas[chan], 0, (size_t)(v->atlas_cap * tile_vox(v)) * sizeof(double));
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* points                                                               */
/* ------------------------------------------------------------------ */

/* gvdbInsertPoints (P:19-36) as launched by InsertPoints (V:5219-5267).
 * poff follows point order here (the reference's is atomic order). */
int orc_insert_points(orc_volume *v, orc_view pos, int n, const float trans[3], int32_t *pnode, int32_t *poff,
                      int32_t *gcnt) {
    if (v->pool_cnt[0] == 0) return ORC_ERR_STATE;
    if (gcnt) memset(gcnt, 0, (size_t)v->pool_cnt[0] * sizeof(int32_t));
    for (int64_t i = 0; i < n; i++) {
        const float *p = view_f3(pos, i);
        if (p[2] == NOHIT) {
            pnode[i] = (int32_t)ID_UNDEFL;
            continue;
        }
        int64_t leaf = leaf_at_float(v, p[0] + trans[0], p[1] + trans[1], p[2] + trans[2]);
        if (leaf < 0) {
            pnode[i] = (int32_t)ID_UNDEFL;
            continue;
        }
        pnode[i] = (int32_t)leaf;
        int32_t o = gcnt ? gcnt[leaf]++ : 0;
        if (poff) poff[i] = o;
    }
    return ORC_OK;
}

/* distFunc (P:516-523) evaluated in double from the float arguments. */
static double dist_func(const float a[3], float bx, float by, float bz, float r) {
    double x = (double)bx - a[0], y = (double)by - a[1], z = (double)bz - a[2];
    double c = (x * x + y * y + z * z) / ((double)r * r);
    return 1.0 + c * (-3.0 + c * (3.0 - c));
}

/* gvdbScatterPointDensity (P:525-573): reference-mode splat into channel 0
 * at the voxel corner pi = int(p) and, with expand, its 6 face neighbours
 * (possibly apron voxels).  The reference's read-modify-write is racy;
 * here contributions are summed exactly. */
int orc_scatter_density(orc_volume *v, orc_view pos, int n, float radius, float amp, const float trans[3], int expand,
                        const int32_t *pnode) {
    (void)amp; /* unused by the reference kernel */
    if (!v->has_chan[0]) return ORC_ERR_STATE;
    int res = res_of(v, 0);
    static const int nb[7][3] = {{0, 0, 0}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    for (int64_t i = 0; i < n; i++) {
        if ((uint32_t)pnode[i] == ID_UNDEFL) continue;
        if (pnode[i] < 0 || pnode[i] >= v->pool_cnt[0]) continue;
        const orc_node *nd = &v->pool[0][pnode[i]];
        const float *pp = view_f3(pos, i);
        float p[3], pi[3];
        for (int a = 0; a < 3; a++) {
            float w = pp[a] + trans[a];
            p[a] = w - (float)nd->mPos[a];
            pi[a] = (float)(int)p[a];
        }
        if (pi[0] < 0 || pi[1] < 0 || pi[2] < 0 || pi[0] >= res || pi[1] >= res || pi[2] >= res) continue;
        int cnt = expand ? 7 : 1;
        for (int k = 0; k < cnt; k++) {
            int q[3];
            for (int a = 0; a < 3; a++) q[a] = (int)pi[a] + nb[k][a] + nd->mValue[a];
            int local[3];
            int64_t s = slot_of_atlas_voxel(v, q, local);
            if (s < 0) continue;
            double w = dist_func(p, pi[0] + nb[k][0], pi[1] + nb[k][1], pi[2] + nb[k][2], radius);
            v->atlas[0][s * tile_vox(v) + tile_index(v, local)] += w;
        }
    }
    return ORC_OK;
}

/* UpdateApron (V:4418-4457) -> UpdateApron<T> (O:72-126).  Every apron
 * voxel takes the value of the interior voxel of the leaf containing its
 * world position (centre = corner + 0.5, getAtlasToWorld N:145-153), or
 * boundval.  Running over the active slots is equivalent to the reference's
 * run over all pool leaves: a stale leaf's mValue either names a slot whose
 * current owner yields the same writes, or an unmapped slot (no write). */
int orc_update_apron(orc_volume *v, int chan, float boundval) {
    if (chan < 0 || chan >= ORC_MAXCHAN || !v->has_chan[chan]) return ORC_ERR_ARG;
    if (v->apron == 0) return ORC_OK;
    int br = tile_res(v), a = v->apron, res = res_of(v, 0);
    int64_t tv = tile_vox(v);
    double *at = v->atlas[chan];
    for (int64_t s = 0; s < v->atlas_last; s++) {
        const orc_atlas_node *m = &v->amap[s];
        if ((uint32_t)m->mLeafID == ID_UNDEFL) continue;
        for (int z = 0; z < br; z++)
            for (int y = 0; y < br; y++)
                for (int x = 0; x < br; x++) {
                    int inner = x >= a && x < a + res && y >= a && y < a + res && z >= a && z < a + res;
                    if (inner) continue;
                    float wp[3] = {(float)m->mPos[0] + (float)(x - a) + 0.5f, (float)m->mPos[1] + (float)(y - a) + 0.5f,
                                   (float)m->mPos[2] + (float)(z - a) + 0.5f};
                    int64_t leaf = leaf_at_float(v, wp[0], wp[1], wp[2]);
                    double val = boundval;
                    if (leaf >= 0) {
                        int64_t ls = slot_of_leaf(v, leaf);
                        const orc_node *ln = &v->pool[0][leaf];
                        if (ls >= 0) {
                            int lc[3] = {(int)(wp[0] - (float)ln->mPos[0]) + a, (int)(wp[1] - (float)ln->mPos[1]) + a,
                                         (int)(wp[2] - (float)ln->mPos[2]) + a};
                            val = at[ls * tv + tile_index(v, lc)];
                        }
                    }
                    int loc[3] = {x, y, z};
                    at[s * tv + tile_index(v, loc)] = val;
                }
    }
    return ORC_OK;
}

/* UpdateNeighbors (V:2527-2556): 6 face neighbours per pool leaf in the
 * order -x,-y,-z,+x,+y,+z.  A missing neighbour is stored as -1 (the
 * reference stores ElemNdx(ID_UNDEFL) = 0xFFFF, which its kernel then
 * fails to recognise; O:51). */
int orc_update_neighbors(orc_volume *v) {
    int64_t brks = v->pool_cnt[0];
    free(v->nbr);
    v->nbr_cnt = brks;
    v->nbr = (int32_t *)malloc((size_t)(brks * 6 + 1) * sizeof(int32_t));
    if (!v->nbr) return ORC_ERR_NOMEM;
    float d = (float)res_of(v, 0);
    for (int64_t n = 0; n < brks; n++) {
        const orc_node *nd = &v->pool[0][n];
        float ct[3] = {nd->mPos[0] + d / 2, nd->mPos[1] + d / 2, nd->mPos[2] + d / 2};
        static const int dir[6][3] = {{-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        for (int k = 0; k < 6; k++) {
            int64_t leaf = leaf_at_float(v, ct[0] + dir[k][0] * d, ct[1] + dir[k][1] * d, ct[2] + dir[k][2] * d);
            v->nbr[n * 6 + k] = (int32_t)leaf;
        }
    }
    return ORC_OK;
}

/* UpdateApronFaces (V:4461-4496) -> gvdbUpdateApronFacesF (O:27-61): for
 * each leaf and each of its -x,-y,-z neighbours, swap the facing interior
 * layers into each other's apron (faces only).  Only active leaves take
 * part (a stale leaf's mValue names another brick's slot). */
int orc_update_apron_faces(orc_volume *v, int chan) {
    if (chan < 0 || chan >= ORC_MAXCHAN || !v->has_chan[chan]) return ORC_ERR_ARG;
    if (v->apron == 0) return ORC_OK;
    if (!v->nbr || v->nbr_cnt != v->pool_cnt[0]) return ORC_ERR_STATE;
    int res = res_of(v, 0);
    int64_t tv = tile_vox(v);
    double *at = v->atlas[chan];
    for (int64_t b = 0; b < v->pool_cnt[0]; b++) {
        const orc_node *self = &v->pool[0][b];
        if (!self->mFlags) continue;
        int64_t ss = slot_of_leaf(v, b);
        if (ss < 0) continue;
        for (int side = 0; side < 3; side++) {
            int64_t nb = v->nbr[b * 6 + side];
            if (nb < 0) continue;
            int64_t ns = slot_of_leaf(v, nb);
            if (ns < 0) continue;
            for (int su = 0; su < res; su++)
                for (int sv = 0; sv < res; sv++) {
                    int vox[3], inc[3] = {0, 0, 0};
                    if (side == 0) { vox[0] = 0; vox[1] = su; vox[2] = sv; }
                    else if (side == 1) { vox[0] = su; vox[1] = 0; vox[2] = sv; }
                    else { vox[0] = su; vox[1] = sv; vox[2] = 0; }
                    inc[side] = 1;
                    int vn[3], sa[3], na[3], sv1[3], nv1[3];
                    for (int a = 0; a < 3; a++) {
                        vn[a] = vox[a] + inc[a] * (res - 1);
                        sv1[a] = vox[a] + v->apron;            /* self voxel (tile coords) */
                        nv1[a] = vn[a] + v->apron;             /* neighbour voxel */
                        na[a] = vn[a] + inc[a] + v->apron;     /* neighbour apron */
                        sa[a] = vox[a] - inc[a] + v->apron;    /* self apron */
                    }
                    double v1 = at[ss * tv + tile_index(v, sv1)];
                    double v2 = at[ns * tv + tile_index(v, nv1)];
                    at[ns * tv + tile_index(v, na)] = v1;
                    at[ss * tv + tile_index(v, sa)] = v2;
                }
        }
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* subcells + voxel-centric gathers                                     */
/* ------------------------------------------------------------------ */

/* The subcell corners visited for one point by gvdbCountSubcell /
 * gvdbInsertSubcell (P:286-291 / P:236-241). */
static void subcell_box(const float w[3], float radius, int sc, int mn[3], int mx[3]) {
    for (int a = 0; a < 3; a++) {
        mn[a] = ((int)(w[a] - radius) / sc) * sc;
        mx[a] = ((int)(w[a] + 1 + radius) / sc) * sc;
    }
}

/* gvdbInsertSubcell_fp16's 16-bit quantization (P:195-203): (x - lo) /
 * range * 65535, converted as a float-to-unsigned-short conversion on the
 * GPU does: toward zero, clamped to [0, 65535], NaN to 0. */
static uint16_t quantize16(float x, float lo, float range) {
    float t = (x - lo) / range * 65535.0f;
    if (t != t || t <= 0.0f) return 0;
    if (t >= 65535.0f) return 65535;
    return (uint16_t)t;
}

/* InsertPointsSubcell (V:4971-5092): gvdbSetFlagSubcell + PrefixSum ->
 * mapping, gvdbCountSubcell, PrefixSum, gvdbInsertSubcell (list order
 * follows point order here), gvdbCalcSubcellPos (P:677-694).
 * InsertPointsSubcell_FP16 (V:5094-5189) runs the same count, then
 * gvdbInsertSubcell_fp16 (P:154-216): both tests on the translated
 * position (NOHIT on its z), entries quantized over the bounding box of the
 * last rebuild (mPosMin, mPosRange = mPosMax - mPosMin) and, with
 * velocities, over mVelMin/mVelRange. */
static int insert_subcells(orc_volume *v, int sc, orc_view pos, orc_view vel, int n, float radius,
                           const float trans[3], int *len, int fp16) {
    int res = res_of(v, 0);
    if (sc <= 0 || res % sc) return ORC_ERR_ARG;
    int64_t num_brick = v->used_leaves;
    if (num_brick == 0) return ORC_ERR_STATE;
    free_subcells(v);
    int scdim = res / sc;
    int scpb = scdim * scdim * scdim;
    v->sc_size = sc;
    v->sc_dim = scdim;
    v->sc_per_brick = scpb;
    v->num_sc = (int64_t)scpb * num_brick;
    int64_t nmap = v->pool_cnt[0];
    int32_t *mapping = (int32_t *)malloc((size_t)(nmap + 1) * sizeof(int32_t));
    v->sc_cnt = (int32_t *)calloc((size_t)v->num_sc + 1, sizeof(int32_t));
    v->sc_off = (int32_t *)calloc((size_t)v->num_sc + 1, sizeof(int32_t));
    v->sc_nid = (int32_t *)calloc((size_t)v->num_sc + 1, sizeof(int32_t));
    v->sc_pos = (int32_t *)calloc((size_t)(v->num_sc * 3 + 1), sizeof(int32_t));
    if (!mapping || !v->sc_cnt || !v->sc_off || !v->sc_nid || !v->sc_pos) {
        free(mapping);
        return ORC_ERR_NOMEM;
    }
    {
        int32_t acc = 0;
        for (int64_t i = 0; i < nmap; i++) {
            mapping[i] = acc;
            acc += (v->pool[0][i].mParent == ID_UNDEF64) ? 0 : 1; /* P:109-118 */
        }
    }
    int32_t *cap = (int32_t *)calloc((size_t)v->num_sc + 1, sizeof(int32_t));
    if (!cap) {
        free(mapping);
        return ORC_ERR_NOMEM;
    }
    for (int pass = 0; pass < 2; pass++) {
        if (pass == 1) {
            int64_t acc = 0;
            for (int64_t s = 0; s < v->num_sc; s++) {
                v->sc_off[s] = (int32_t)acc;
                acc += v->sc_cnt[s];
            }
            v->sc_len = acc;
            memcpy(cap, v->sc_cnt, (size_t)v->num_sc * sizeof(int32_t));
            memset(v->sc_cnt, 0, (size_t)v->num_sc * sizeof(int32_t));
            int bad = 0;
            if (fp16) {
                v->sc_fp16 = 1;
                v->sc_q = (uint16_t *)malloc((size_t)(acc * 3 + 3) * sizeof(uint16_t));
                bad = !v->sc_q;
                if (vel.base) {
                    v->sc_qvel = (uint16_t *)malloc((size_t)(acc * 3 + 3) * sizeof(uint16_t));
                    bad = bad || !v->sc_qvel;
                }
            } else {
                v->sc_pnt = (float *)malloc((size_t)(acc * 3 + 3) * sizeof(float));
                bad = !v->sc_pnt;
            }
            if (bad) {
                free(mapping);
                free(cap);
                return ORC_ERR_NOMEM;
            }
        }
        for (int64_t i = 0; i < n; i++) {
            const float *p = view_f3(pos, i);
            float w[3];
            if (pass == 0) { /* count: trans added before the sign test (P:283-284) */
                if (p[2] == NOHIT) continue;
                for (int a = 0; a < 3; a++) w[a] = p[a] + trans[a];
                if (w[0] < 0 || w[1] < 0 || w[2] < 0) continue;
            } else if (fp16) { /* fp16 insert: both tests on the translated position (P:169-172) */
                for (int a = 0; a < 3; a++) w[a] = p[a] + trans[a];
                if (w[2] == NOHIT) continue;
                if (w[0] < 0 || w[1] < 0 || w[2] < 0) continue;
            } else { /* insert: sign test before trans (P:231-233) */
                if (p[2] == NOHIT) continue;
                if (p[0] < 0 || p[1] < 0 || p[2] < 0) continue;
                for (int a = 0; a < 3; a++) w[a] = p[a] + trans[a];
            }
            int mn[3], mx[3];
            subcell_box(w, radius, sc, mn, mx);
            int s3[3];
            for (s3[0] = mn[0]; s3[0] <= mx[0]; s3[0] += sc)
                for (s3[1] = mn[1]; s3[1] <= mx[1]; s3[1] += sc)
                    for (s3[2] = mn[2]; s3[2] <= mx[2]; s3[2] += sc) {
                        int64_t leaf = get_pos_leaf_parent(v, s3);
                        if (leaf < 0 || leaf >= nmap) continue;
                        const orc_node *pn = &v->pool[0][leaf];
                        int pin[3];
                        for (int a = 0; a < 3; a++) pin[a] = (s3[a] - pn->mPos[a]) / sc;
                        int64_t local = ((int64_t)pin[2] * scdim + pin[1]) * scdim + pin[0];
                        int64_t idx = (int64_t)mapping[leaf] * scpb + local;
                        if (idx < 0 || idx >= v->num_sc) continue;
                        if (pass == 0) {
                            v->sc_cnt[idx]++;
                        } else {
                            if (v->sc_cnt[idx] >= cap[idx]) continue; /* never past the counted list */
                            int64_t at = v->sc_off[idx] + v->sc_cnt[idx]++;
                            if (fp16) {
                                float range[3];
                                for (int a = 0; a < 3; a++) range[a] = v->posmax[a] - v->posmin[a];
                                for (int a = 0; a < 3; a++) v->sc_q[at * 3 + a] = quantize16(w[a], v->posmin[a], range[a]);
                                if (v->sc_qvel) {
                                    const float *u = view_f3(vel, i);
                                    for (int a = 0; a < 3; a++)
                                        v->sc_qvel[at * 3 + a] = quantize16(u[a], v->velmin[a], v->velrange[a]);
                                }
                            } else {
                                v->sc_pnt[at * 3 + 0] = w[0];
                                v->sc_pnt[at * 3 + 1] = w[1];
                                v->sc_pnt[at * 3 + 2] = w[2];
                            }
                        }
                    }
        }
    }
    for (int64_t i = 0; i < nmap; i++) { /* gvdbCalcSubcellPos */
        const orc_node *pn = &v->pool[0][i];
        if (pn->mParent == ID_UNDEF64) continue;
        for (int s = 0; s < scpb; s++) {
            int64_t idx = (int64_t)mapping[i] * scpb + s;
            if (idx >= v->num_sc) continue;
            v->sc_pos[idx * 3 + 0] = pn->mPos[0] + s % scdim * sc;
            v->sc_pos[idx * 3 + 1] = pn->mPos[1] + (s / scdim) % scdim * sc;
            v->sc_pos[idx * 3 + 2] = pn->mPos[2] + (s / scdim / scdim) % scdim * sc;
            v->sc_nid[idx] = (int32_t)i;
        }
    }
    free(mapping);
    free(cap);
    if (len) *len = (int)v->sc_len;
    return ORC_OK;
}

int orc_insert_points_subcell(orc_volume *v, int sc, orc_view pos, int n, float radius, const float trans[3], int *len) {
    orc_view none = {NULL, 0, 0, 0};
    return insert_subcells(v, sc, pos, none, n, radius, trans, len, 0);
}

int orc_insert_points_subcell_fp16(orc_volume *v, int sc, orc_view pos, orc_view vel, int n, float radius,
                                   const float trans[3], int *len) {
    return insert_subcells(v, sc, pos, vel, n, radius, trans, len, 1);
}

/* GetMinMaxVel (V:5469-5521): per axis min and max of the velocities,
 * mVelRange = mVelMax - mVelMin. */
int orc_get_min_max_vel(orc_volume *v, orc_view vel, int n) {
    if (!vel.base || n <= 0) return ORC_ERR_ARG;
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = 0; i < n; i++) {
        const float *u = view_f3(vel, i);
        for (int a = 0; a < 3; a++) {
            if (u[a] < mn[a]) mn[a] = u[a];
            if (u[a] > mx[a]) mx[a] = u[a];
        }
    }
    for (int a = 0; a < 3; a++) {
        v->velmin[a] = mn[a];
        v->velrange[a] = mx[a] - mn[a];
    }
    return ORC_OK;
}

/* gvdbGatherDensity (P:696-733) / gvdbGatherLevelSet (P:736-773): each
 * voxel of each subcell reduces over that subcell's list with the integer
 * voxel corner as the sample position. */
static int gather_voxels(orc_volume *v, int sc, float radius, int chan, int accum, int levelset) {
    if (chan < 0 || chan >= ORC_MAXCHAN || !v->has_chan[chan]) return ORC_ERR_ARG;
    if (!v->sc_cnt || sc != v->sc_size) return ORC_ERR_STATE;
    float range[3];
    for (int a = 0; a < 3; a++) range[a] = v->posmax[a] - v->posmin[a];
    int64_t tv = tile_vox(v);
    double *at = v->atlas[chan];
    int a = v->apron;
    for (int64_t s = 0; s < v->num_sc; s++) {
        int64_t leaf = v->sc_nid[s];
        if (leaf < 0 || leaf >= v->pool_cnt[0]) continue;
        const orc_node *nd = &v->pool[0][leaf];
        int64_t slot = slot_of_leaf(v, leaf);
        if (slot < 0) continue;
        for (int tz = 0; tz < sc; tz++)
            for (int ty = 0; ty < sc; ty++)
                for (int tx = 0; tx < sc; tx++) {
                    int wp[3] = {v->sc_pos[s * 3 + 0] + tx, v->sc_pos[s * 3 + 1] + ty, v->sc_pos[s * 3 + 2] + tz};
                    int lc[3] = {wp[0] - nd->mPos[0] + a, wp[1] - nd->mPos[1] + a, wp[2] - nd->mPos[2] + a};
                    double *dst = &at[slot * tv + tile_index(v, lc)];
                    double val = accum ? *dst : (levelset ? 3.0 : 0.0);
                    for (int32_t j = 0; j < v->sc_cnt[s]; j++) {
                        const int64_t e = (int64_t)(v->sc_off[s] + j) * 3;
                        float q[3];
                        if (v->sc_fp16) /* gvdbGatherLevelSet_fp16 (P:792-794): q / 65535 * range + min */
                            for (int k = 0; k < 3; k++) q[k] = (float)v->sc_q[e + k] / 65535.0f * range[k] + v->posmin[k];
                        else
                            for (int k = 0; k < 3; k++) q[k] = v->sc_pnt[e + k];
                        const float *p = q;
                        float d[3] = {p[0] - (float)wp[0], p[1] - (float)wp[1], p[2] - (float)wp[2]};
                        double c = sqrt((double)d[0] * d[0] + (double)d[1] * d[1] + (double)d[2] * d[2]);
                        if (levelset) {
                            double t = c - radius;
                            if (t < val) val = t;
                        } else {
                            double t = radius - c;
                            if (t > val) val = t;
                        }
                    }
                    *dst = val;
                }
    }
    return ORC_OK;
}
int orc_gather_density(orc_volume *v, int sc, float radius, int chan, int accum) {
    if (v->sc_fp16) return ORC_ERR_STATE; /* the lists hold quantized entries */
    return gather_voxels(v, sc, radius, chan, accum, 0);
}
int orc_gather_level_set(orc_volume *v, int sc, float radius, int chan, int accum) {
    if (v->sc_fp16) return ORC_ERR_STATE; /* the lists hold quantized entries */
    return gather_voxels(v, sc, radius, chan, accum, 1);
}
/* GatherLevelSet_FP16 (V:5375-5402): the level set over quantized lists,
 * never accumulating (P:775-811). */
int orc_gather_level_set_fp16(orc_volume *v, int sc, float radius, int chan) {
    if (!v->sc_fp16) return ORC_ERR_STATE;
    return gather_voxels(v, sc, radius, chan, 0, 1);
}

/* ------------------------------------------------------------------ */
/* kernel splats (tent r=1, cubic B-spline r=2) and their adjoints       */
/* ------------------------------------------------------------------ */

/* Per-axis taps of a point at world coordinate x: voxel centres sit at
 * i + 0.5 (getAtlasToWorld, N:151).  u = x - 0.5, base = floor(u),
 * t = u - base.  Tent: taps base+{0,1}.  Cubic B-spline: base+{-1..2}. */
static int axis_taps(int kernel, double x, int *first, double w[4], double dw[4]) {
    double u = x - 0.5;
    double b = floor(u);
    double t = u - b;
    if (kernel == ORC_KERNEL_TENT1) {
        *first = (int)b;
        w[0] = 1.0 - t; dw[0] = -1.0;
        w[1] = t;       dw[1] = 1.0;
        return 2;
    }
    *first = (int)b - 1;
    double s = 1.0 - t;
    w[0] = s * s * s / 6.0;                                  dw[0] = -0.5 * s * s;
    w[1] = (3.0 * t * t * t - 6.0 * t * t + 4.0) / 6.0;     dw[1] = 1.5 * t * t - 2.0 * t;
    w[2] = (-3.0 * t * t * t + 3.0 * t * t + 3.0 * t + 1.0) / 6.0; dw[2] = -1.5 * t * t + t + 0.5;
    w[3] = t * t * t / 6.0;                                  dw[3] = 0.5 * t * t;
    return 4;
}

/* Interior voxel (x,y,z) -> pointer into channel `chan`, NULL when its
 * brick is not an active leaf with an atlas slot. */
typedef struct {
    int64_t key[27];
    int64_t slot[27];
    int nused;
} slot_cache;
static int64_t voxel_slot(const orc_volume *v, int x, int y, int z, slot_cache *c, int local[3]) {
    int res = res_of(v, 0);
    if (x < 0 || y < 0 || z < 0) return -1;
    int bx = x / res, by = y / res, bz = z / res;
    local[0] = x - bx * res + v->apron;
    local[1] = y - by * res + v->apron;
    local[2] = z - bz * res + v->apron;
    int64_t key = ((int64_t)bx << 42) | ((int64_t)by << 21) | bz;
    for (int i = 0; i < c->nused; i++)
        if (c->key[i] == key) return c->slot[i];
    int64_t leaf = leaf_at_voxel(v, bx * res, by * res, bz * res);
    int64_t s = -1;
    if (leaf >= 0 && v->pool[0][leaf].mFlags) s = slot_of_leaf(v, leaf);
    if (c->nused < 27) {
        c->key[c->nused] = key;
        c->slot[c->nused] = s;
        c->nused++;
    }
    return s;
}

/* A point takes part when it is not NOHIT and its own voxel lies in an
 * active brick (the rule ScatterDensity applies through InsertPoints'
 * pnode, P:530). */
static int point_active(const orc_volume *v, const float *pp, const float trans[3], float w[3]) {
    if (pp[2] == NOHIT) return 0;
    for (int a = 0; a < 3; a++) w[a] = pp[a] + trans[a];
    if (w[0] < 0 || w[1] < 0 || w[2] < 0) return 0;
    int64_t leaf = leaf_at_float(v, w[0], w[1], w[2]);
    if (leaf < 0 || !v->pool[0][leaf].mFlags) return 0;
    return slot_of_leaf(v, leaf) >= 0;
}

static int check_chans(const orc_volume *v, const int *chans, int nch) {
    if (nch < 1 || nch > ORC_MAXCHAN) return ORC_ERR_ARG;
    for (int c = 0; c < nch; c++)
        if (chans[c] < 0 || chans[c] >= ORC_MAXCHAN || !v->has_chan[chans[c]]) return ORC_ERR_ARG;
    return ORC_OK;
}

static void zero_interiors(orc_volume *v, int chan) {
    int res = res_of(v, 0), a = v->apron;
    int64_t tv = tile_vox(v);
    for (int64_t s = 0; s < v->atlas_last; s++)
        for (int z = 0; z < res; z++)
            for (int y = 0; y < res; y++)
                for (int x = 0; x < res; x++) {
                    int lc[3] = {x + a, y + a, z + a};
                    v->atlas[chan][s * tv + tile_index(v, lc)] = 0.0;
                }
}

int orc_scatter_kernel(orc_volume *v, int kernel, orc_view pos, int n, const float trans[3], orc_view weight,
                       float weight_const, const orc_view *attrs, const int *chans, int nch) {
    if (kernel != ORC_KERNEL_TENT1 && kernel != ORC_KERNEL_CUBIC2) return ORC_ERR_ARG;
    if (check_chans(v, chans, nch)) return ORC_ERR_ARG;
    int64_t tv = tile_vox(v);
    for (int c = 0; c < nch; c++) zero_interiors(v, chans[c]);
    for (int64_t i = 0; i < n; i++) {
        float w[3];
        if (!point_active(v, view_f3(pos, i), trans, w)) continue;
        double wt = weight.base ? view_f1(weight, i) : weight_const;
        double amt[ORC_MAXCHAN];
        for (int c = 0; c < nch; c++) amt[c] = wt * ((attrs && attrs[c].base) ? view_f1(attrs[c], i) : 1.0);
        int f[3], nt = 0;
        double wx[3][4], dw[3][4];
        for (int a = 0; a < 3; a++) nt = axis_taps(kernel, w[a], &f[a], wx[a], dw[a]);
        slot_cache cache = {{0}, {0}, 0};
        for (int k = 0; k < nt; k++)
            for (int j = 0; j < nt; j++)
                for (int ii = 0; ii < nt; ii++) {
                    int local[3];
                    int64_t s = voxel_slot(v, f[0] + ii, f[1] + j, f[2] + k, &cache, local);
                    if (s < 0) continue;
                    double wgt = wx[0][ii] * wx[1][j] * wx[2][k];
                    int64_t off = s * tv + tile_index(v, local);
                    for (int c = 0; c < nch; c++) v->atlas[chans[c]][off] += amt[c] * wgt;
                }
    }
    return ORC_OK;
}

int orc_gather_kernel(orc_volume *v, int kernel, orc_view pos, int n, const float trans[3], const int *chans, int nch,
                      double *out) {
    if (kernel != ORC_KERNEL_TENT1 && kernel != ORC_KERNEL_CUBIC2) return ORC_ERR_ARG;
    if (check_chans(v, chans, nch)) return ORC_ERR_ARG;
    int64_t tv = tile_vox(v);
    for (int64_t i = 0; i < n; i++) {
        for (int c = 0; c < nch; c++) out[i * nch + c] = 0.0;
        float w[3];
        if (!point_active(v, view_f3(pos, i), trans, w)) continue;
        int f[3], nt = 0;
        double wx[3][4], dw[3][4];
        for (int a = 0; a < 3; a++) nt = axis_taps(kernel, w[a], &f[a], wx[a], dw[a]);
        slot_cache cache = {{0}, {0}, 0};
        for (int k = 0; k < nt; k++)
            for (int j = 0; j < nt; j++)
                for (int ii = 0; ii < nt; ii++) {
                    int local[3];
                    int64_t s = voxel_slot(v, f[0] + ii, f[1] + j, f[2] + k, &cache, local);
                    if (s < 0) continue;
                    double wgt = wx[0][ii] * wx[1][j] * wx[2][k];
                    int64_t off = s * tv + tile_index(v, local);
                    for (int c = 0; c < nch; c++) out[i * nch + c] += v->atlas[chans[c]][off] * wgt;
                }
    }
    return ORC_OK;
}

/* Adjoint of orc_scatter_kernel.  With a_pc = weight_p * attr_c(p) and
 * G_c[v] = sum_p a_pc W(v + 0.5 - x_p), given dL/dG_c in grad_chans[c]:
 *   grad_attr[p,c]  = weight_p * sum_v dG_c[v] W
 *   grad_weight[p]  = sum_c attr_c(p) * sum_v dG_c[v] W
 *   grad_pos[p,k]   = sum_c a_pc * sum_v dG_c[v] dW/dx_k            */
int orc_scatter_kernel_backward(orc_volume *v, int kernel, orc_view pos, int n, const float trans[3], orc_view weight,
                                float weight_const, const orc_view *attrs, const int *chans, int nch,
                                const int *grad_chans, double *grad_pos, double *grad_weight, double *grad_attr) {
    (void)chans;
    if (kernel != ORC_KERNEL_TENT1 && kernel != ORC_KERNEL_CUBIC2) return ORC_ERR_ARG;
    if (check_chans(v, grad_chans, nch)) return ORC_ERR_ARG;
    int64_t tv = tile_vox(v);
    for (int64_t i = 0; i < n; i++) {
        double gsum[ORC_MAXCHAN], gdx[ORC_MAXCHAN][3];
        for (int c = 0; c < nch; c++) gsum[c] = gdx[c][0] = gdx[c][1] = gdx[c][2] = 0.0;
        float w[3];
        int act = point_active(v, view_f3(pos, i), trans, w);
        double wt = weight.base ? view_f1(weight, i) : weight_const;
        if (act) {
            int f[3], nt = 0;
            double wx[3][4], dw[3][4];
            for (int a = 0; a < 3; a++) nt = axis_taps(kernel, w[a], &f[a], wx[a], dw[a]);
            slot_cache cache = {{0}, {0}, 0};
            for (int k = 0; k < nt; k++)
                for (int j = 0; j < nt; j++)
                    for (int ii = 0; ii < nt; ii++) {
                        int local[3];
                        int64_t s = voxel_slot(v, f[0] + ii, f[1] + j, f[2] + k, &cache, local);
                        if (s < 0) continue;
                        double wgt = wx[0][ii] * wx[1][j] * wx[2][k];
                        double gx = dw[0][ii] * wx[1][j] * wx[2][k];
                        double gy = wx[0][ii] * dw[1][j] * wx[2][k];
                        double gz = wx[0][ii] * wx[1][j] * dw[2][k];
                        int64_t off = s * tv + tile_index(v, local);
                        for (int c = 0; c < nch; c++) {
                            double g = v->atlas[grad_chans[c]][off];
                            gsum[c] += g * wgt;
                            gdx[c][0] += g * gx;
                            gdx[c][1] += g * gy;
                            gdx[c][2] += g * gz;
                        }
                    }
        }
        double gw = 0.0, gp[3] = {0, 0, 0};
        for (int c = 0; c < nch; c++) {
            double at = (attrs && attrs[c].base) ? view_f1(attrs[c], i) : 1.0;
            if (grad_attr) grad_attr[i * nch + c] = (attrs && attrs[c].base) ? wt * gsum[c] : 0.0;
            gw += at * gsum[c];
            for (int k = 0; k < 3; k++) gp[k] += wt * at * gdx[c][k];
        }
        if (grad_weight) grad_weight[i] = gw;
        if (grad_pos)
            for (int k = 0; k < 3; k++) grad_pos[i * 3 + k] = gp[k];
    }
    return ORC_OK;
}

/* Adjoint of orc_gather_kernel.  out_pc = sum_v G_c[v] W(v + 0.5 - x_p);
 * given dL/dout in grad_out[p*nch + c]:
 *   grad_chans[c][v] = sum_p dout_pc W     (interiors of active bricks)
 *   grad_pos[p,k]    = sum_c dout_pc sum_v G_c[v] dW/dx_k          */
int orc_gather_kernel_backward(orc_volume *v, int kernel, orc_view pos, int n, const float trans[3], const int *chans,
                               int nch, const double *grad_out, const int *grad_chans, double *grad_pos) {
    if (kernel != ORC_KERNEL_TENT1 && kernel != ORC_KERNEL_CUBIC2) return ORC_ERR_ARG;
    if (check_chans(v, chans, nch)) return ORC_ERR_ARG;
    if (grad_chans && check_chans(v, grad_chans, nch)) return ORC_ERR_ARG;
    int64_t tv = tile_vox(v);
    if (grad_chans)
        for (int c = 0; c < nch; c++) zero_interiors(v, grad_chans[c]);
    for (int64_t i = 0; i < n; i++) {
        double gp[3] = {0, 0, 0};
        float w[3];
        if (point_active(v, view_f3(pos, i), trans, w)) {
            int f[3], nt = 0;
            double wx[3][4], dw[3][4];
            for (int a = 0; a < 3; a++) nt = axis_taps(kernel, w[a], &f[a], wx[a], dw[a]);
            slot_cache cache = {{0}, {0}, 0};
            for (int k = 0; k < nt; k++)
                for (int j = 0; j < nt; j++)
                    for (int ii = 0; ii < nt; ii++) {
                        int local[3];
                        int64_t s = voxel_slot(v, f[0] + ii, f[1] + j, f[2] + k, &cache, local);
                        if (s < 0) continue;
                        double wgt = wx[0][ii] * wx[1][j] * wx[2][k];
                        double gx = dw[0][ii] * wx[1][j] * wx[2][k];
                        double gy = wx[0][ii] * dw[1][j] * wx[2][k];
                        double gz = wx[0][ii] * wx[1][j] * dw[2][k];
                        int64_t off = s * tv + tile_index(v, local);
                        for (int c = 0; c < nch; c++) {
                            double go = grad_out[i * nch + c];
                            double g = v->atlas[chans[c]][off];
                            gp[0] += go * g * gx;
                            gp[1] += go * g * gy;
                            gp[2] += go * g * gz;
                            if (grad_chans) v->atlas[grad_chans[c]][off] += go * wgt;
                        }
                    }
        }
        if (grad_pos)
            for (int k = 0; k < 3; k++) grad_pos[i * 3 + k] = gp[k];
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* inspection                                                           */
/* ------------------------------------------------------------------ */

int orc_depth(const orc_volume *v) { return v->depth; }
int orc_top_level(const orc_volume *v) { return top_level(v); }
int64_t orc_pool_count(const orc_volume *v, int lev) { return (lev >= 0 && lev < ORC_MAXLEV) ? v->pool_cnt[lev] : 0; }
int64_t orc_used_leaves(const orc_volume *v) { return v->used_leaves; }
const orc_node *orc_nodes(const orc_volume *v, int lev) { return (lev >= 0 && lev < ORC_MAXLEV) ? v->pool[lev] : NULL; }
const uint64_t *orc_childlists(const orc_volume *v, int lev) {
    return (lev >= 1 && lev < ORC_MAXLEV) ? v->clist[lev] : NULL;
}
int64_t orc_childlist_len(const orc_volume *v, int lev) { return (lev >= 1 && lev < ORC_MAXLEV) ? res3_of(v, lev) : 0; }
int orc_res(const orc_volume *v, int lev) { return res_of(v, lev); }
int orc_range(const orc_volume *v, int lev) { return range_of(v, lev); }
void orc_bbox(const orc_volume *v, float posmin[3], float posmax[3]) {
    for (int a = 0; a < 3; a++) {
        posmin[a] = v->posmin[a];
        posmax[a] = v->posmax[a];
    }
}
int orc_apron(const orc_volume *v) { return v->apron; }
int orc_tile_res(const orc_volume *v) { return tile_res(v); }
int64_t orc_atlas_slots(const orc_volume *v) { return v->atlas_last; }
int64_t orc_atlas_capacity(const orc_volume *v) { return v->atlas_cap; }
void orc_atlas_subdim(const orc_volume *v, int out[3]) {
    out[0] = v->subdim[0];
    out[1] = v->subdim[1];
    out[2] = v->subdim[2];
}
double *orc_atlas(orc_volume *v, int chan) { return (chan >= 0 && chan < ORC_MAXCHAN) ? v->atlas[chan] : NULL; }
const orc_atlas_node *orc_atlas_map(const orc_volume *v) { return v->amap; }
const int32_t *orc_neighbors(const orc_volume *v) { return v->nbr; }
int64_t orc_subcell_count(const orc_volume *v) { return v->num_sc; }
const int32_t *orc_subcell_cnt(const orc_volume *v) { return v->sc_cnt; }
const int32_t *orc_subcell_nid(const orc_volume *v) { return v->sc_nid; }
const int32_t *orc_subcell_pos(const orc_volume *v) { return v->sc_pos; }
const int32_t *orc_subcell_off(const orc_volume *v) { return v->sc_off; }
int64_t orc_subcell_len(const orc_volume *v) { return v->sc_len; }
const float *orc_subcell_points(const orc_volume *v) { return v->sc_pnt; }
const uint16_t *orc_subcell_points_fp16(const orc_volume *v) { return v->sc_q; }
const uint16_t *orc_subcell_vel_fp16(const orc_volume *v) { return v->sc_qvel; }
