// Launch-shape autotuner: picks the tile size (k-points per CTA) and the
// k-points per thread for a class of solves by timing every candidate on a
// copy of the problem cut to a few hundred time steps.  Results are cached in
// memory per (variant, precision, RK order, T1 on/off, k-count bucket, SM
// count) and, when SBE_TUNE_CACHE names a file, on disk across processes.
// SBE_AUTOTUNE=0 turns it off (the heuristic of Engine::shape_for is used).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "sbe_engine.h"
#include "sbe_kernels.h"

namespace sbe {

namespace {

std::mutex g_mu;
std::map<std::string, Shape> g_cache;
bool g_loaded = false;

const char *cache_path() { return std::getenv("SBE_TUNE_CACHE"); }

void load_cache()
{
    if (g_loaded) return;
    g_loaded = true;
    const char *path = cache_path();
    if (!path) return;
    std::ifstream f(path);
    std::string k;
    Shape s{};
    while (f >> k >> s.tile_k >> s.kpt) {
        s.threads = s.tile_k / s.kpt;
        g_cache[k] = s;
    }
}

void store(const std::string &k, const Shape &s)
{
    g_cache[k] = s;
    if (const char *path = cache_path()) {
        std::ofstream f(path, std::ios::app);
        f << k << ' ' << s.tile_k << ' ' << s.kpt << '\n';
    }
}

}  // namespace

bool autotune_enabled()
{
    const char *e = std::getenv("SBE_AUTOTUNE");
    return !(e && e[0] == '0');
}

static std::string tune_key(int device, const Problem &p, int precision);

bool autotune_lookup(int device, const Problem &p, int precision, Shape *out)
{
    const std::string key = tune_key(device, p, precision);
    std::lock_guard<std::mutex> lk(g_mu);
    load_cache();
    auto it = g_cache.find(key);
    if (it == g_cache.end()) return false;
    *out = it->second;
    return true;
}

static std::string tune_key(int device, const Problem &p, int precision)
{
    int sms = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device attribute");
    const int bucket = (int)std::floor(2.0 * std::log2((double)std::max(p.ntotal(), 1)));
    std::ostringstream ks;
    ks << (p.gauge == GAUGE_VELOCITY ? "vg" : "lw") << '-' << (precision == PREC_FP64 ? "fp64" : "mixed") << "-rk"
       << p.rk << "-t1" << (p.T1 > 1.0e-16 ? 1 : 0) << "-nk" << bucket << "-sm" << sms;
    return ks.str();
}

Shape autotune_shape(int device, const Problem &p, int precision)
{
    int sms = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device attribute");
    const bool vg = p.gauge == GAUGE_VELOCITY;
    const int nk = p.ntotal();
    const int bucket = (int)std::floor(2.0 * std::log2((double)std::max(nk, 1)));
    std::ostringstream ks;
    ks << (vg ? "vg" : "lw") << '-' << (precision == PREC_FP64 ? "fp64" : "mixed") << "-rk" << p.rk << "-t1"
       << (p.T1 > 1.0e-16 ? 1 : 0) << "-nk" << bucket << "-sm" << sms;
    const std::string key = ks.str();
    std::lock_guard<std::mutex> lk(g_mu);
    load_cache();
    auto it = g_cache.find(key);
    if (it != g_cache.end()) return it->second;

    std::vector<Shape> cand;
    auto addc = [&](int threads, int kpt) {
        if ((long long)threads * kpt > 2LL * nk && threads > 32) return;  // tiles far larger than the grid
        cand.push_back(Shape{threads * kpt, kpt, threads});
    };
    // every CTA size in warps the kernel accepts: the best one balances
    // occupancy against the quantisation of the tile count into waves of
    // resident CTAs
    const int variant = vg ? VAR_HALDANE_VG : VAR_HALDANE_LW;
    for (int t = 32; t <= propagate_max_threads(variant, precision, p.rk, 1); t += 32) addc(t, 1);
    // two k-points per thread: the FP64 velocity gauge and the packed mixed
    // kernels of both gauges
    if (vg || precision != PREC_FP64)
        for (int t = 32; t <= propagate_max_threads(variant, precision, p.rk, 2); t += 32) addc(t, 2);
    Problem q = p;
    const int S = 128;
    q.laser.Nt = std::min(p.laser.Nt, 3 * S);
    cudaStream_t st;
    cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream create");
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    Shape best = cand.front();
    float best_ms = 1e30f;
    for (const Shape &c : cand) {
        float ms = 1e30f;
        try {
            Engine e(device, st, S);
            EngineOptions eo;
            eo.precision = precision;
            eo.tile_k = c.tile_k;
            eo.kpt = c.kpt;
            eo.snapshots = false;
            e.add(q, eo);
            e.step();  // warm-up launch (also builds the lists)
            cuda_check(cudaEventRecord(a, st), "event");
            while (e.max_remaining_ticks() > 0) e.step_frozen();
            cuda_check(cudaEventRecord(b, st), "event");
            cuda_check(cudaEventSynchronize(b), "event sync");
            cudaEventElapsedTime(&ms, a, b);
        } catch (const OomError &) {
            continue;
        }
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    store(key, best);
    return best;
}

}  // namespace sbe
