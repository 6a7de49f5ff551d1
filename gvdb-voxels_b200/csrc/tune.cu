// tune.cu -- the kernel splats' autotuner and its on-disk cache (no
// reference counterpart: the reference's launches have fixed shapes).
//
// Three launch settings of the splat path are tuned (gvdb2_tuning):
//   dense : cells of at least this many points take the scatter's partial-sum
//           path (a CTA per slice, shared-memory tile), the others the
//           owner-computes warps (0: no cell does) -- the scatter's tile staging;
//   slice : points per CTA of a dense cell -- the work per CTA;
//   light : cells of at most this many points are gathered a warp per cell
//           with taps read from the atlas, the others through a staged halo
//           tile -- the gather's tile staging.
// A candidate is timed with CUDA events on the volume's stream, on the
// caller's own call (median of three after an untimed run that also bins);
// the fastest stays on the volume and goes to the cache under the call's
// workload class: device name and SM count, operation, kernel, channels,
// brick width and the points per active 8^3 cell rounded to a power of two.
// With GVDB2_OPT_AUTOTUNE set, every kernel splat and gather looks its
// class up first and takes a cached setting when there is one.
//
// Cache file: one line per class, "key<TAB>dense slice light ms", rewritten
// whole through a temporary file and a rename, so a reader never sees half
// a file.  Path: gvdb2_set_tune_cache, else $GVDB2_TUNE_CACHE, else no file
// (the choice stays on the volume only).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include <sys/stat.h>
#include <unistd.h>

#include "dev_common.cuh"
#include "gvdb2_internal.h"

namespace gvdb2 {
namespace {

struct Entry {
    gvdb2_tuning t;
    float ms;
};

std::mutex g_cache_mu;

bool parse_line(const std::string &line, std::string &key, Entry &e) {
    const size_t tab = line.find('\t');
    if (tab == std::string::npos || tab == 0) return false;
    key = line.substr(0, tab);
    std::istringstream is(line.substr(tab + 1));
    return (bool)(is >> e.t.dense >> e.t.slice >> e.t.light >> e.ms);
}

std::map<std::string, Entry> read_cache(const std::string &path) {
    std::map<std::string, Entry> m;
    std::ifstream f(path);
    std::string line, key;
    Entry e{};
    while (std::getline(f, line))
        if (parse_line(line, key, e)) m[key] = e;
    return m;
}

bool write_cache(const std::string &path, const std::map<std::string, Entry> &m) {
    const std::string tmp = path + ".tmp." + std::to_string((long long)getpid());
    {
        std::ofstream f(tmp, std::ios::trunc);
        if (!f) return false;
        for (const auto &kv : m)
            f << kv.first << '\t' << kv.second.t.dense << ' ' << kv.second.t.slice << ' ' << kv.second.t.light << ' '
              << kv.second.ms << '\n';
        if (!f) return false;
    }
    return std::rename(tmp.c_str(), path.c_str()) == 0;
}

// The parsed file per path, re-read when its modification time or size
// changes (a lookup per splat call stays off the file system otherwise).
struct Parsed {
    struct timespec mtime {};
    off_t size = -1;
    std::map<std::string, Entry> m;
};
std::map<std::string, Parsed> g_parsed;

const std::map<std::string, Entry> &cached_read(const std::string &path) {
    struct stat sb {};
    Parsed &p = g_parsed[path];
    if (stat(path.c_str(), &sb) != 0) {
        p = Parsed{};
        return p.m;
    }
    if (sb.st_size != p.size || sb.st_mtim.tv_sec != p.mtime.tv_sec || sb.st_mtim.tv_nsec != p.mtime.tv_nsec) {
        p.m = read_cache(path);
        p.size = sb.st_size;
        p.mtime = sb.st_mtim;
    }
    return p.m;
}

std::string cache_path(const Volume *v) {
    if (!v->tune_cache.empty()) return v->tune_cache;
    const char *e = std::getenv("GVDB2_TUNE_CACHE");
    return e ? std::string(e) : std::string();
}

bool valid_tuning(const gvdb2_tuning &t) {
    const bool dense_ok = t.dense == 0 || (t.dense >= 128 && t.dense <= (1 << 24));
    const bool slice_ok = t.slice >= 128 && t.slice <= 65536 && t.slice % 128 == 0;
    return dense_ok && slice_ok && t.light >= 0 && t.light <= (int)kLightCell;
}

} // namespace

gvdb2_status set_tuning(Volume *v, const gvdb2_tuning *t) {
    if (!t || !valid_tuning(*t))
        return fail(v, GVDB2_ERR_ARG, "tuning: dense 0 or in [128, 2^24], slice a multiple of 128 in [128, 65536], light in [0, 32]");
    v->tune_dense = t->dense;
    v->tune_slice = t->slice;
    v->tune_light = t->light;
    return GVDB2_OK;
}

gvdb2_tuning get_tuning(const Volume *v) { return gvdb2_tuning{v->tune_dense, v->tune_slice, v->tune_light}; }

// The workload class of a kernel splat or gather call.
std::string tune_key(Volume *v, const char *op, int kernel, int nch, int64_t n) {
    // the device's name and SM count, looked up once per device
    static std::mutex mu;
    static std::map<int, std::string> names;
    std::string dev;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = names.find(v->device);
        if (it == names.end()) {
            cudaDeviceProp p{};
            if (cudaGetDeviceProperties(&p, v->device) != cudaSuccess) std::strcpy(p.name, "unknown");
            it = names.emplace(v->device, std::string(p.name) + "/" + std::to_string(p.multiProcessorCount)).first;
        }
        dev = it->second;
    }
    const int m = std::max(1, v->res(0) / kCell);
    const double cells = (double)std::max<int64_t>(1, v->atlas_last) * m * m * m;
    const int dens = (int)std::lround(std::log2(std::max(1.0, (double)n / cells)));
    char b[320];
    std::snprintf(b, sizeof(b), "%s|%s|k%d|c%d|r%d|d%d", dev.c_str(), op, kernel, nch, v->res(0), dens);
    for (char *c = b; *c; c++)
        if (*c == '\t' || *c == '\n') *c = ' ';
    return b;
}

// GVDB2_OPT_AUTOTUNE: take the cached setting of this call's class, if any.
void apply_cached_tuning(Volume *v, const char *op, int kernel, int nch, int64_t n) {
    if (!v->autotune) return;
    const std::string path = cache_path(v);
    if (path.empty()) return;
    const std::string key = tune_key(v, op, kernel, nch, n);
    Entry e{};
    bool found = false;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        const auto &m = cached_read(path);
        auto it = m.find(key);
        if (it != m.end()) e = it->second, found = true;
    }
    if (found && valid_tuning(e.t)) {
        v->tune_dense = e.t.dense;
        v->tune_slice = e.t.slice;
        v->tune_light = e.t.light;
    }
}

gvdb2_status cache_get(const char *path, const char *key, gvdb2_tuning *t, float *ms) {
    if (!path || !key || !t) return GVDB2_ERR_ARG;
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto m = read_cache(path);
    auto it = m.find(key);
    if (it == m.end()) return GVDB2_ERR_STATE;
    *t = it->second.t;
    if (ms) *ms = it->second.ms;
    return GVDB2_OK;
}

gvdb2_status cache_put(const char *path, const char *key, const gvdb2_tuning *t, float ms) {
    if (!path || !*path || !key || !*key || !t || !valid_tuning(*t) || std::strpbrk(key, "\t\n")) return GVDB2_ERR_ARG;
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto m = read_cache(path);
    m[key] = Entry{*t, ms};
    return write_cache(path, m) ? GVDB2_OK : GVDB2_ERR_STATE;
}

// Times `call` under each candidate and keeps the fastest; the last run is
// the chosen one's, so the outputs are what one call with it gives.
gvdb2_status autotune(Volume *v, const char *op, int kernel, int nch, int64_t n,
                      const std::vector<gvdb2_tuning> &cands, const std::function<gvdb2_status()> &call,
                      gvdb2_tuning *chosen) {
    const gvdb2_tuning keep = get_tuning(v);
    cudaEvent_t e0, e1;
    GV_CUDA(v, cudaEventCreate(&e0));
    GV_CUDA(v, cudaEventCreate(&e1));
    float best_ms = 1e30f;
    gvdb2_tuning best = keep;
    gvdb2_status st = GVDB2_OK;
    for (const gvdb2_tuning &c : cands) {
        if ((st = set_tuning(v, &c)) != GVDB2_OK) break;
        if ((st = call()) != GVDB2_OK) break; // untimed: bins with this candidate's cell lists
        float t[3];
        for (int r = 0; r < 3 && st == GVDB2_OK; r++) {
            cudaEventRecord(e0, v->stream);
            st = call();
            cudaEventRecord(e1, v->stream);
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&t[r], e0, e1);
        }
        if (st != GVDB2_OK) break;
        std::sort(t, t + 3);
        if (t[1] < best_ms) best_ms = t[1], best = c;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != GVDB2_OK) {
        set_tuning(v, &keep);
        return st;
    }
    GV_TRY(set_tuning(v, &best));
    GV_TRY(call());
    if (chosen) *chosen = best;
    const std::string path = cache_path(v);
    if (!path.empty()) {
        const std::string key = tune_key(v, op, kernel, nch, n);
        if (cache_put(path.c_str(), key.c_str(), &best, best_ms) != GVDB2_OK)
            return fail(v, GVDB2_ERR_STATE, "autotune: cannot write the cache file " + path);
    }
    return GVDB2_OK;
}

std::vector<gvdb2_tuning> scatter_candidates(const Volume *v) {
    std::vector<gvdb2_tuning> c;
    c.push_back(gvdb2_tuning{0, 4096, v->tune_light});
    for (int d : {256, 512, 1024, 2048})
        for (int s : {2048, 4096, 8192}) c.push_back(gvdb2_tuning{d, s, v->tune_light});
    return c;
}

std::vector<gvdb2_tuning> gather_candidates(const Volume *v) {
    std::vector<gvdb2_tuning> c;
    for (int l : {0, 8, 16, 32}) c.push_back(gvdb2_tuning{v->tune_dense, v->tune_slice, l});
    return c;
}

} // namespace gvdb2
