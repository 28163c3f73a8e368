// Project autotuner for the NUDFT tile engine.
//
// For one problem shape and direction it times every launch shape the kernel
// set covers -- "ours" elements per thread (pt), register budget (occupancy
// 4 or 6 blocks per SM) and the number of partitions of the "theirs" range
// (split), and the tensor-core kernel at every split -- with CUDA events on
// the launching stream, and keeps the fastest.
// Results are cached per shape in memory and persisted as text lines
//     v2 <adj> <CG> <G> <use_z> <Mpad> <Npad> <pt> <occ> <split> <tc> <ms>
// and, for batched launches (the split only, timed by the batch itself),
//     b1 <adj> <CG> <G> <use_z> <S> <Npad> <max Mpad> <sum Mpad> <tc> <pt> <occ> <split> <ms>
// in $IMP_TUNE_CACHE (default ~/.cache/impatient_b200/nudft_tune.txt), so a
// shape is tuned once per machine.  IMP_AUTOTUNE=0 turns tuning and the use of
// tuned shapes off (default launch shapes only).
#include "nudft.cuh"

#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <sys/stat.h>
#include <tuple>
#include <vector>

namespace imp {

namespace {

using Key = std::tuple<int, int, int, int, int, int>;

std::mutex g_mu;
std::map<Key, NuLaunch> g_cache;
using BKey = std::tuple<int, int, int, int, int, int, int, long long, int>;
std::map<BKey, NuLaunch> g_bcache;  // batched problems
bool g_loaded = false;

BKey bkey_of(const NuBatchKey &k) {
    return BKey(k.adj, k.CG, k.G, k.use_z, k.S, k.Npad, k.max_mpad, k.mpad_total, k.tc);
}

Key key_of(const NuPlan &p, bool adj) {
    return Key(adj ? 1 : 0, p.CG, p.G, p.use_z ? 1 : 0, p.Mpad, p.Npad);
}

std::string cache_path() {
    if (const char *e = std::getenv("IMP_TUNE_CACHE")) return e;
    const char *h = std::getenv("HOME");
    return std::string(h ? h : "/tmp") + "/.cache/impatient_b200/nudft_tune.txt";
}

void load_locked() {
    if (g_loaded) return;
    g_loaded = true;
    FILE *f = std::fopen(cache_path().c_str(), "r");
    if (!f) return;
    char line[256];
    while (std::fgets(line, sizeof line, f)) {
        int a, cg, g, z, mp, np, pt, occ, split, tc;
        double ms;
        NuBatchKey b;
        if (std::sscanf(line, "b1 %d %d %d %d %d %d %d %lld %d %d %d %d %lf", &b.adj, &b.CG, &b.G,
                        &b.use_z, &b.S, &b.Npad, &b.max_mpad, &b.mpad_total, &b.tc, &pt, &occ,
                        &split, &ms) == 13) {
            NuLaunch l;
            l.tc = b.tc;
            l.pt = pt;
            l.occ = occ;
            l.split = split;
            const bool ok = b.tc ? nu_tc_supported(b.CG)
                                 : (nu_shape_supported(b.CG, pt) && (occ == 4 || occ == 6));
            if (ok && split >= 1 && split <= 64) g_bcache[bkey_of(b)] = l;
            continue;
        }
        if (std::sscanf(line, "v2 %d %d %d %d %d %d %d %d %d %d %lf", &a, &cg, &g, &z, &mp, &np,
                        &pt, &occ, &split, &tc, &ms) != 11)
            continue;  // other versions are re-tuned
        NuLaunch l;
        l.pt = pt;
        l.occ = occ;
        l.split = split;
        l.tc = tc;
        const bool ok = tc ? (nu_tc_supported(cg) && nu_tc_enabled())
                           : (nu_shape_supported(cg, pt) && (occ == 4 || occ == 6));
        if (ok) g_cache[Key(a, cg, g, z, mp, np)] = l;
    }
    std::fclose(f);
}

void persist(const Key &k, const NuLaunch &l, double ms) {
    std::string path = cache_path();
    // create the parent directories
    for (size_t i = 1; i < path.size(); ++i)
        if (path[i] == '/') mkdir(path.substr(0, i).c_str(), 0755);
    FILE *f = std::fopen(path.c_str(), "a");
    if (!f) return;  // the cache is an optimisation; failure to write is not an error
    std::fprintf(f, "v2 %d %d %d %d %d %d %d %d %d %d %.4f\n", std::get<0>(k), std::get<1>(k),
                 std::get<2>(k), std::get<3>(k), std::get<4>(k), std::get<5>(k), l.pt, l.occ,
                 l.split, l.tc, ms);
    std::fclose(f);
}

bool tuning_enabled() {
    const char *e = std::getenv("IMP_AUTOTUNE");
    return !(e && e[0] == '0');
}

void append_line(const char *text) {
    std::string path = cache_path();
    for (size_t i = 1; i < path.size(); ++i)
        if (path[i] == '/') mkdir(path.substr(0, i).c_str(), 0755);
    FILE *f = std::fopen(path.c_str(), "a");
    if (!f) return;  // the cache is an optimisation; failure to write is not an error
    std::fputs(text, f);
    std::fclose(f);
}

std::vector<int> pts_for(int CG) {
    std::vector<int> v;
    for (int pt : {2, 4, 8})
        if (nu_shape_supported(CG, pt)) v.push_back(pt);
    return v;
}

constexpr int kMaxSplit = 64;
constexpr size_t kMaxPartialBytes = size_t(512) << 20;

}  // namespace

bool nu_tuning_enabled() { return tuning_enabled(); }

bool nu_batch_lookup(const NuBatchKey &k, NuLaunch *out) {
    if (!tuning_enabled()) return false;
    std::lock_guard<std::mutex> g(g_mu);
    load_locked();
    auto it = g_bcache.find(bkey_of(k));
    if (it == g_bcache.end()) return false;
    *out = it->second;
    return true;
}

void nu_batch_store(const NuBatchKey &k, const NuLaunch &l, double ms) {
    std::lock_guard<std::mutex> g(g_mu);
    load_locked();
    g_bcache[bkey_of(k)] = l;
    char line[256];
    std::snprintf(line, sizeof line, "b1 %d %d %d %d %d %d %d %lld %d %d %d %d %.4f\n", k.adj,
                  k.CG, k.G, k.use_z, k.S, k.Npad, k.max_mpad, k.mpad_total, k.tc, l.pt, l.occ,
                  l.split, ms);
    append_line(line);
}

size_t nu_tune_partial_bytes(const NuPlan &p, bool adj) {
    const int n_theirs = adj ? p.Mpad : p.Npad;
    size_t best = 0;
    for (int s = 1; s <= kMaxSplit; s *= 2) {
        if (!nu_split_ok(n_theirs, s)) continue;
        NuLaunch l;
        l.split = s;
        const size_t b = adj ? nu_adj_partial_bytes(p, l) : nu_fwd_partial_bytes(p, l);
        if (b <= kMaxPartialBytes && b > best) best = b;
    }
    return best;
}

bool nu_tuned_lookup(const NuPlan &p, bool adj, NuLaunch *out) {
    if (!tuning_enabled()) return false;  // IMP_AUTOTUNE=0: default shapes only
    std::lock_guard<std::mutex> g(g_mu);
    load_locked();
    auto it = g_cache.find(key_of(p, adj));
    if (it == g_cache.end()) return false;
    if (it->second.tc && !nu_tc_enabled()) return false;
    *out = it->second;
    return true;
}

cudaError_t nu_autotune(const NuPlan &p, bool adj, const float2 *tdata, float2 *part,
                        size_t part_bytes, unsigned *dev_err, cudaStream_t st, NuLaunch *out) {
    *out = nu_default_launch(p, adj);
    if (nu_tuned_lookup(p, adj, out)) {
        const size_t need = adj ? nu_adj_partial_bytes(p, *out) : nu_fwd_partial_bytes(p, *out);
        if (need <= part_bytes) return cudaSuccess;
        *out = nu_default_launch(p, adj);
    }
    if (!tuning_enabled()) return cudaSuccess;
    const int n_theirs = adj ? p.Mpad : p.Npad;
    cudaEvent_t e0, e1;
    cudaError_t e;
    if ((e = cudaEventCreate(&e0)) != cudaSuccess) return e;
    if ((e = cudaEventCreate(&e1)) != cudaSuccess) {
        cudaEventDestroy(e0);
        return e;
    }
    float best = 1e30f;
    NuLaunch best_l = *out;
    std::vector<NuLaunch> cands;
    for (int pt : pts_for(p.CG))
        for (int occ : {4, 6})
            for (int s = 1; s <= kMaxSplit; s *= 2) {
                NuLaunch l;
                l.pt = pt;
                l.occ = occ;
                l.split = s;
                cands.push_back(l);
            }
    const int n_ours = adj ? p.Npad : p.Mpad;
    if (nu_tc_enabled() && nu_tc_supported(p.CG) && n_ours % nu_tc_rows(p.CG) == 0)
        for (int s = 1; s <= kMaxSplit; s *= 2) {
            NuLaunch l;
            l.tc = 1;
            l.split = s;
            cands.push_back(l);
        }
    for (const NuLaunch &l : cands) {
        if (!nu_split_ok(n_theirs, l.split)) continue;
        const size_t need = adj ? nu_adj_partial_bytes(p, l) : nu_fwd_partial_bytes(p, l);
        if (need > part_bytes) continue;
        auto run = [&]() {
            return adj ? nu_adjoint_partials(p, l, tdata, part, dev_err, st)
                       : nu_forward_partials(p, l, tdata, part, dev_err, st);
        };
        if ((e = run()) != cudaSuccess) break;  // warm-up
        float ms_min = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {
            cudaEventRecord(e0, st);
            if ((e = run()) != cudaSuccess) break;
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms_min = ms < ms_min ? ms : ms_min;
        }
        if (e != cudaSuccess) break;
        if (ms_min < best) {
            best = ms_min;
            best_l = l;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return e;
    *out = best_l;
    std::lock_guard<std::mutex> g(g_mu);
    load_locked();
    g_cache[key_of(p, adj)] = best_l;
    persist(key_of(p, adj), best_l, best);
    return cudaSuccess;
}

}  // namespace imp
