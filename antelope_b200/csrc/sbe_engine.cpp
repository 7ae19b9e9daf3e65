// Host engine: device buffers of resident solves, launch lists, per-launch
// stepping, output assembly and the reference's file writers.
#include "sbe_engine.h"
#include "sbe_spectrum.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <map>

#include "sbe_kernels.h"
#include "sbe_wannier.h"

namespace sbe {

void cuda_check(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        throw OomError(std::string(what) + ": out of device memory");
    }
    throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {
int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }
}  // namespace

UploadRing::UploadRing(size_t bytes) : cap_(bytes)
{
    cuda_check(cudaMallocHost(&base_, cap_), "cudaMallocHost(upload ring)");
}

UploadRing &UploadRing::shared()
{
    static UploadRing *ring = new UploadRing(32u << 20);  // lives until exit
    return *ring;
}

PinnedPool &PinnedPool::shared()
{
    static PinnedPool *pool = new PinnedPool();  // lives until exit
    return *pool;
}

UploadRing::~UploadRing()
{
    for (auto &sp : inflight_) {
        cudaEventSynchronize(sp.ev);
        cudaEventDestroy(sp.ev);
    }
    for (auto ev : spare_) cudaEventDestroy(ev);
    cudaFreeHost(base_);
}

void UploadRing::upload(void *dst, const void *src, size_t bytes, cudaStream_t st)
{
    if (bytes == 0) return;
    std::unique_lock<std::mutex> lk(mu_, std::defer_lock);
    if (bytes <= cap_) lk.lock();  // the split path below re-enters per piece
    if (bytes > cap_) {  // larger than the ring: stage it in pieces
        const char *s = static_cast<const char *>(src);
        char *d = static_cast<char *>(dst);
        for (size_t off = 0; off < bytes; off += cap_ / 2) upload(d + off, s + off, std::min(cap_ / 2, bytes - off), st);
        return;
    }
    const size_t need = (bytes + 255) & ~size_t(255);
    if (head_ + need > cap_) head_ = 0;
    const size_t lo = head_, hi = head_ + need;
    // wait for copies still reading this region
    for (size_t i = 0; i < inflight_.size();) {
        Span &sp = inflight_[i];
        const bool overlap = sp.lo < hi && lo < sp.hi;
        if (overlap || cudaEventQuery(sp.ev) == cudaSuccess) {
            if (overlap) cuda_check(cudaEventSynchronize(sp.ev), "upload ring wait");
            spare_.push_back(sp.ev);
            inflight_[i] = inflight_.back();
            inflight_.pop_back();
        } else {
            ++i;
        }
    }
    std::memcpy(base_ + lo, src, bytes);
    cuda_check(cudaMemcpyAsync(dst, base_ + lo, bytes, cudaMemcpyHostToDevice, st), "upload");
    cudaEvent_t ev;
    if (spare_.empty()) cuda_check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event create");
    else { ev = spare_.back(); spare_.pop_back(); }
    cuda_check(cudaEventRecord(ev, st), "event record");
    inflight_.push_back(Span{lo, hi, ev});
    head_ = hi;
}

size_t PinnedPool::size_class(size_t b)
{
    size_t c = 4096;
    while (c < b) c <<= 1;
    return c;
}

void *PinnedPool::get(size_t bytes)
{
    std::lock_guard<std::mutex> lk(mu_);
    const size_t c = size_class(bytes);
    auto &v = free_[c];
    if (!v.empty()) {
        void *p = v.back();
        v.pop_back();
        return p;
    }
    void *p = nullptr;
    cuda_check(cudaMallocHost(&p, c), "cudaMallocHost(results)");
    return p;
}

void PinnedPool::put(void *p, size_t bytes)
{
    std::lock_guard<std::mutex> lk(mu_);
    if (p) free_[size_class(bytes)].push_back(p);
}

PinnedPool::~PinnedPool()
{
    for (auto &kv : free_)
        for (void *p : kv.second) cudaFreeHost(p);
}

struct Engine::Solve {
    Problem prob;
    int id = 0, slot = 0, variant = 0, precision = 0, nts = 0;
    Shape shape{};
    int nk = 0, nk_pad = 0, ntiles = 0, Nt = 0, admit_tick = 0, nticks = 0;
    bool g1 = false;
    void *kc = nullptr, *st = nullptr, *tab = nullptr;
    double *partial = nullptr, *jout = nullptr, *constpart = nullptr;
    double *snap_nc = nullptr, *snap_pi = nullptr;  // density snapshots (or null)
    int nshots = 0, k_begin = 0;
    double *h_jout = nullptr, *h_const = nullptr;  // pinned
    cudaEvent_t ev = nullptr;
    bool fetched = false;
    size_t bytes = 0;
};

struct Engine::Group {
    int variant, precision, rk, kpt, threads;
    bool g1;
    std::vector<TileDev> tiles;
    TileDev *d_tiles = nullptr;
    int cap = 0;
};

namespace {
// Device memory of resident solves comes from one pool per device that keeps
// what it has (no release to the driver) and never makes an allocation wait
// for another stream's pending work: a block freed on the compute stream is
// reused by the copy stream only once that free has completed.
cudaMemPool_t engine_pool(int device)
{
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(device);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool;
    cuda_check(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
    uint64_t keep = UINT64_MAX;
    cuda_check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "pool attribute");
    int no = 0;
    cuda_check(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no), "pool attribute");
    pools[device] = pool;
    return pool;
}
}  // namespace

Engine::Engine(int device, cudaStream_t stream, int steps_per_launch)
    : device_(device), stream_(stream), S_(steps_per_launch > 0 ? steps_per_launch : 512)
{
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&up_, cudaStreamNonBlocking), "stream create");
    pool_ = engine_pool(device_);
    capacity_ = 4096;
    cuda_check(cudaMalloc(&d_solves_, sizeof(SolveDev) * capacity_), "cudaMalloc(solves)");
    h_solves_ = new SolveDev[capacity_];
    cuda_check(cudaMalloc(&d_ids_, sizeof(int) * capacity_), "cudaMalloc(ids)");
    h_ids_.assign(capacity_, 0);
    for (int i = capacity_ - 1; i >= 0; --i) free_slots_.push_back(i);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device_) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
}

Engine::~Engine()
{
    cudaStreamSynchronize(up_);
    cudaStreamSynchronize(stream_);
    for (auto &kv : live_) {
        Solve &s = *kv.second;
        cudaFreeAsync(s.kc, stream_);
        cudaFreeAsync(s.st, stream_);
        cudaFreeAsync(s.tab, stream_);
        cudaFreeAsync(s.partial, stream_);
        cudaFreeAsync(s.jout, stream_);
        cudaFreeAsync(s.constpart, stream_);
        if (s.snap_nc) cudaFreeAsync(s.snap_nc, stream_);
        if (s.snap_pi) cudaFreeAsync(s.snap_pi, stream_);
        if (s.ev) {
            cudaEventSynchronize(s.ev);
            cudaEventDestroy(s.ev);
        }
        pinned_.put(s.h_jout, (size_t)s.Nt * NSLOT * 8);
        pinned_.put(s.h_const, (size_t)s.ntiles * NSLOT * 8);
    }
    for (auto &kv : groups_) cudaFreeAsync(kv.second->d_tiles, stream_);
    for (auto &e : prop_ev_) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
    for (auto &e : red_ev_) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
    cudaStreamSynchronize(stream_);
    for (auto ev : pending_) cudaEventDestroy(ev);
    for (auto ev : spare_ev_) cudaEventDestroy(ev);
    cudaStreamDestroy(up_);
    cudaFree(d_solves_);
    delete[] h_solves_;
    cudaFree(d_ids_);
}

void Engine::drain_pending()
{
    for (cudaEvent_t ev : pending_) {
        cuda_check(cudaStreamWaitEvent(stream_, ev, 0), "stream wait");
        spare_ev_.push_back(ev);
    }
    pending_.clear();
}

Shape Engine::shape_for(const Problem &p, const EngineOptions &o) const
{
    const int prec = o.precision >= 0 ? o.precision : p.precision;
    const bool vg = p.gauge == GAUGE_VELOCITY;
    Shape s{};
    // mixed velocity gauge: two k-points per thread in packed f32x2 registers
    // mixed method: two k-points per thread in packed f32x2 registers (both
    // gauges); the FP64 length gauge has one k-point per thread
    s.kpt = o.kpt > 0 ? o.kpt : (prec == PREC_MIXED ? 2 : 1);
    if (!vg && prec == PREC_FP64) s.kpt = 1;
    if (o.tile_k > 0) {
        s.tile_k = o.tile_k;
    } else if (o.kpt <= 0 && autotune_enabled() &&
               (o.allow_tuning || autotune_lookup(device_, p, prec, &s))) {
        return o.allow_tuning ? autotune_shape(device_, p, prec) : s;
    } else if (o.throughput_shape) {
        // solves that share the GPU with many others: full CTAs
        s.tile_k = 256 * s.kpt;
    } else {
        // largest CTA (<= 128 threads) that still gives >= 2 CTAs per SM
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_);
        int threads = 128;
        while (threads > 32 && (long long)p.ntotal() < 2LL * sms * threads * s.kpt) threads /= 2;
        s.tile_k = threads * s.kpt;
    }
    s.threads = s.tile_k / s.kpt;
    const int tmax = propagate_max_threads(vg ? VAR_HALDANE_VG : VAR_HALDANE_LW, prec, p.rk, s.kpt);
    if (s.threads < 32 || s.threads > tmax || s.threads % 32 || s.tile_k % s.kpt)
        throw CfgError(tmax > 256 ? "tile_k / kpt must be a multiple of 32 between 32 and 512"
                                  : "tile_k / kpt must be a multiple of 32 between 32 and 256");
    return s;
}

size_t Engine::bytes_needed(const Problem &p, const EngineOptions &o) const
{
    const Shape sh = shape_for(p, o);
    const int prec = o.precision >= 0 ? o.precision : p.precision;
    const size_t real = prec == PREC_FP64 ? 8 : 4;
    const int ntiles = ceil_div(p.ntotal(), sh.tile_k);
    const size_t nk_pad = (size_t)ntiles * sh.tile_k;
    const int nts = (int)stage_fractions(p.rk).size();
    const bool vg = p.gauge == GAUGE_VELOCITY;
    const size_t nc = vg ? (size_t)VG_NCONST_ALL : (size_t)LW_NCONST, ns = vg ? VG_NSTATE_ALL : LW_NSTATE_ALL;
    const size_t tab = (size_t)p.laser.Nt * nts * (vg ? 2 : LW_NPHASE) * real;
    const size_t nk = o.k_end > 0 ? (size_t)(o.k_end - o.k_begin) : (size_t)p.ntotal();
    const size_t snap = o.snapshots ? (size_t)p.nshots() * nk * 24 : 0;
    return nc * nk_pad * real + ns * nk_pad * 8 + tab + (size_t)S_ * ntiles * NSLOT * 8 + (size_t)p.laser.Nt * NSLOT * 8 +
           (size_t)ntiles * NSLOT * 8 + snap;
}

int Engine::add(const Problem &p, const EngineOptions &o)
{
    if (p.model != MODEL_HALDANE) throw CfgError("only the Haldane model is built on this path");
    if (p.gauge == GAUGE_LENGTH_HAMILTONIAN) throw CfgError("gauge LengthHamiltonian is not implemented");
    if (p.rk != 4 && p.rk != 5) throw CfgError("Haldane solves use RKorder 4 or 5");
    auto s = std::make_unique<Solve>();
    s->prob = p;
    s->id = next_id_++;
    s->precision = o.precision >= 0 ? o.precision : p.precision;
    s->variant = p.gauge == GAUGE_VELOCITY ? VAR_HALDANE_VG : VAR_HALDANE_LW;
    s->shape = shape_for(p, o);
    const int kb = o.k_end > 0 ? o.k_begin : 0, ke = o.k_end > 0 ? o.k_end : p.ntotal();
    if (kb < 0 || ke > p.ntotal() || kb >= ke) throw CfgError("k-slice outside the grid");
    s->nk = ke - kb;
    s->ntiles = ceil_div(s->nk, s->shape.tile_k);
    s->nk_pad = s->ntiles * s->shape.tile_k;
    s->Nt = p.laser.Nt;
    const auto cfr = stage_fractions(p.rk);
    s->nts = (int)cfr.size();
    s->g1 = p.T1 > 1.0e-16;
    if (free_slots_.empty()) throw OomError("too many resident solves (descriptor slots exhausted)");
    const size_t real = s->precision == PREC_FP64 ? 8 : 4;
    const bool vg = s->variant == VAR_HALDANE_VG;
    const size_t nc = vg ? (size_t)VG_NCONST_ALL : (size_t)LW_NCONST;
    const size_t ns = vg ? (size_t)VG_NSTATE_ALL : (size_t)LW_NSTATE_ALL;
    const size_t kc_b = nc * s->nk_pad * real, st_b = ns * s->nk_pad * 8;  // state is FP64 in both methods
    s->k_begin = kb;
    s->nshots = o.snapshots ? p.nshots() : 0;
    const size_t snap_n = (size_t)s->nshots * s->nk;
    const size_t tab_n = (size_t)s->Nt * s->nts * (vg ? 2 : LW_NPHASE);
    const size_t part_b = (size_t)S_ * s->ntiles * NSLOT * 8, jout_b = (size_t)s->Nt * NSLOT * 8;
    const size_t cp_b = (size_t)s->ntiles * NSLOT * 8;

    auto alloc = [&](void **ptr, size_t b, const char *what) {
        cudaError_t e = cudaMallocFromPoolAsync(ptr, b, pool_, up_);
        if (e != cudaSuccess) {
            for (void *q : {s->kc, s->st, s->tab, (void *)s->partial, (void *)s->jout, (void *)s->constpart,
                            (void *)s->snap_nc})
                if (q) cudaFreeAsync(q, up_);
            cuda_check(e, what);
        }
    };
    alloc(&s->kc, kc_b, "alloc constants");
    alloc(&s->st, st_b, "alloc state");
    alloc(&s->tab, tab_n * real, "alloc field table");
    if (reinterpret_cast<uintptr_t>(s->tab) % 16 != 0)   // the kernels read its entries in 16-byte loads
        throw std::runtime_error("field table not 16-byte aligned");
    alloc((void **)&s->partial, part_b, "alloc partials");
    alloc((void **)&s->jout, jout_b, "alloc outputs");
    alloc((void **)&s->constpart, cp_b, "alloc constant parts");
    if (snap_n > 0) {
        alloc((void **)&s->snap_nc, snap_n * 8, "alloc snapshots");
        alloc((void **)&s->snap_pi, snap_n * 16, "alloc snapshots");
    }
    s->bytes = kc_b + st_b + tab_n * real + part_b + jout_b + cp_b + snap_n * 24;
    cuda_check(cudaEventCreateWithFlags(&s->ev, cudaEventDisableTiming), "cudaEventCreate");

    // field table on the device: the laser evaluated at every stage time in
    // FP64 (rounded once to the kernel's Real)
    {
        const LaserDev ld = laser_dev(p.laser);
        cuda_check(launch_field_table(ld, p.laser.atmin, p.laser.dt, s->Nt, s->nts, cfr.data(), vg, p.hal_va,
                                      p.hal_vb, s->tab, s->precision != PREC_FP64, up_),
                   "field table kernel");
    }
    InitArgs ia{};
    ia.nk = s->nk;
    ia.k_offset = kb;
    ia.nk_pad = s->nk_pad;
    ia.tile_k = s->shape.tile_k;
    ia.variant = s->variant;
    ia.nval = p.nval;
    ia.use_fermi = p.use_fermi ? 1 : 0;
    for (int i = 0; i < 3; ++i) ia.N[i] = p.Nk[i];
    for (int i = 0; i < 9; ++i) ia.axes[i] = p.bzaxes[i];
    for (int i = 0; i < 3; ++i) ia.origin[i] = p.bzorigin[i];
    ia.t1 = p.hal_t1;
    ia.t2 = p.hal_t2;
    ia.M0 = p.hal_M0;
    ia.phi0 = p.hal_phi0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 2; ++j) { ia.va[i][j] = p.hal_va[i][j]; ia.vb[i][j] = p.hal_vb[i][j]; }
    ia.Ef = p.Ef;
    ia.dt = p.dt;
    cuda_check(cudaMemsetAsync(s->kc, 0, kc_b, up_), "memset constants");
    cuda_check(cudaMemsetAsync(s->st, 0, st_b, up_), "memset state");
    cuda_check(launch_init_haldane(ia, s->precision, s->kc, s->st, s->constpart, up_), "init kernel");
    cudaEvent_t ready;
    if (spare_ev_.empty()) cuda_check(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming), "event create");
    else { ready = spare_ev_.back(); spare_ev_.pop_back(); }
    cuda_check(cudaEventRecord(ready, up_), "event record");
    pending_.push_back(ready);

    s->slot = free_slots_.back();
    free_slots_.pop_back();
    SolveDev &d = h_solves_[s->slot];
    std::memset(&d, 0, sizeof(d));
    d.nk = s->nk;
    d.ntiles = s->ntiles;
    d.Nt = s->Nt;
    d.admit_tick = tick_;
    d.nk_pad = s->nk_pad;
    d.nts = s->nts;
    d.variant = s->variant;
    d.precision = s->precision;
    d.kc = s->kc;
    d.st = s->st;
    d.tab = s->tab;
    d.partial = s->partial;
    d.jout = s->jout;
    d.shot_every = s->nshots > 0 ? p.shot_every() : 0;
    d.snap_nc = s->snap_nc;
    d.snap_pi = s->snap_pi;
    d.g1 = p.T1 > 1.0e-16 ? p.dt / p.T1 : 0.0;   // SBEs.h:484-493
    d.g2 = p.T2 > 1.0e-16 ? p.dt / p.T2 : 0.0;
    const double t2c = 2.0 * p.hal_t2 * std::cos(p.hal_phi0), t2s = 2.0 * p.hal_t2 * std::sin(p.hal_phi0);
    d.t1dt = p.dt * p.hal_t1;
    d.t2sdt = p.dt * t2s;
    d.Mdt = p.dt * p.hal_M0;
    d.t1 = p.hal_t1;
    d.t2c = t2c;
    d.t2s = t2s;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 2; ++j) { d.va[i][j] = p.hal_va[i][j]; d.vb[i][j] = p.hal_vb[i][j]; }
    ring_.upload(d_solves_ + s->slot, &d, sizeof(SolveDev), stream_);
    s->admit_tick = tick_;
    s->nticks = ceil_div(s->Nt, S_);
    bytes_in_use_ += s->bytes;
    const int id = s->id;
    live_[id] = std::move(s);
    dirty_ = true;
    return id;
}

Engine::Solve &Engine::get(int id)
{
    auto it = live_.find(id);
    if (it == live_.end()) throw CfgError("unknown solve id");
    return *it->second;
}
const Engine::Solve &Engine::get(int id) const
{
    auto it = live_.find(id);
    if (it == live_.end()) throw CfgError("unknown solve id");
    return *it->second;
}

int Engine::remaining_ticks(int id) const
{
    const Solve &s = get(id);
    return std::max(0, s.admit_tick + s.nticks - tick_);
}

int Engine::max_remaining_ticks() const
{
    int m = 0;
    for (const auto &kv : live_) m = std::max(m, kv.second->admit_tick + kv.second->nticks - tick_);
    return m;
}

void Engine::rebuild_lists()
{
    for (auto &kv : groups_) kv.second->tiles.clear();
    nids_ = 0;
    for (auto &kv : live_) {
        Solve &s = *kv.second;
        if (s.admit_tick + s.nticks - tick_ <= 0) continue;
        auto key = std::make_tuple(s.variant, s.precision, s.prob.rk, s.shape.kpt, s.shape.threads, s.g1 ? 1 : 0);
        auto &g = groups_[key];
        if (!g) {
            g = std::make_unique<Group>();
            g->variant = s.variant;
            g->precision = s.precision;
            g->rk = s.prob.rk;
            g->kpt = s.shape.kpt;
            g->threads = s.shape.threads;
            g->g1 = s.g1;
        }
        for (int t = 0; t < s.ntiles; ++t) {
            TileDev td;
            td.solve = s.slot;
            td.k0 = t * s.shape.tile_k;
            td.kcount = std::min(s.shape.tile_k, s.nk - td.k0);
            td.tile = t;
            g->tiles.push_back(td);
        }
        h_ids_[nids_++] = s.slot;
    }
    for (auto &kv : groups_) {
        Group &g = *kv.second;
        if ((int)g.tiles.size() > g.cap) {
            if (g.d_tiles) cudaFreeAsync(g.d_tiles, stream_);
            g.cap = std::max<int>((int)g.tiles.size(), 2 * g.cap);
            cuda_check(cudaMallocAsync((void **)&g.d_tiles, sizeof(TileDev) * g.cap, stream_), "alloc tiles");
        }
        if (!g.tiles.empty()) ring_.upload(g.d_tiles, g.tiles.data(), sizeof(TileDev) * g.tiles.size(), stream_);
    }
    if (nids_ > 0) ring_.upload(d_ids_, h_ids_.data(), sizeof(int) * nids_, stream_);
    dirty_ = false;
}

void Engine::step()
{
    drain_pending();
    // a solve that finished at the previous tick leaves the launch lists
    for (auto &kv : live_)
        if (kv.second->admit_tick + kv.second->nticks == tick_) dirty_ = true;
    if (dirty_) rebuild_lists();
    step_frozen();
}

void Engine::step_frozen()
{
    last_launches_ = 0;
    for (auto &kv : groups_) {
        Group &g = *kv.second;
        if (g.tiles.empty()) continue;
        LaunchArgs la{};
        la.tiles = g.d_tiles;
        la.solves = d_solves_;
        la.ntiles = (int)g.tiles.size();
        la.threads = g.threads;
        la.tick = tick_;
        la.S = S_;
        la.variant = g.variant;
        la.precision = g.precision;
        la.rk = g.rk;
        la.kpt = g.kpt;
        la.has_g1 = g.g1;
        la.stream = stream_;
        std::pair<cudaEvent_t, cudaEvent_t> ev{};
        if (profile_) {
            ev = new_pair();
            cuda_check(cudaEventRecord(ev.first, stream_), "event record");
        }
        cuda_check(launch_propagate(la), "propagate launch");
        if (profile_) {
            cuda_check(cudaEventRecord(ev.second, stream_), "event record");
            prop_ev_.push_back(ev);
        }
        ++last_launches_;
    }
    if (nids_ > 0) {
        std::pair<cudaEvent_t, cudaEvent_t> ev{};
        if (profile_) {
            ev = new_pair();
            cuda_check(cudaEventRecord(ev.first, stream_), "event record");
        }
        cuda_check(launch_reduce(d_solves_, d_ids_, nids_, tick_, S_, stream_), "reduce launch");
        if (profile_) {
            cuda_check(cudaEventRecord(ev.second, stream_), "event record");
            red_ev_.push_back(ev);
        }
    }
    ++tick_;
}

std::pair<cudaEvent_t, cudaEvent_t> Engine::new_pair()
{
    std::pair<cudaEvent_t, cudaEvent_t> p;
    cuda_check(cudaEventCreate(&p.first), "event create");
    cuda_check(cudaEventCreate(&p.second), "event create");
    return p;
}

void Engine::kernel_times(double *prop_ms, int *prop_n, double *red_ms, int *red_n)
{
    auto total = [&](std::vector<std::pair<cudaEvent_t, cudaEvent_t>> &v, double *ms, int *n) {
        double t = 0.0;
        for (auto &e : v) {
            cuda_check(cudaEventSynchronize(e.second), "event sync");
            float x = 0.f;
            cuda_check(cudaEventElapsedTime(&x, e.first, e.second), "event elapsed");
            t += x;
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
        if (ms) *ms = t;
        if (n) *n = (int)v.size();
        v.clear();
    };
    total(prop_ev_, prop_ms, prop_n);
    total(red_ev_, red_ms, red_n);
}

void Engine::fetch_async(int id)
{
    drain_pending();
    Solve &s = get(id);
    // pinned result buffers are taken when a solve finishes, not when it is
    // admitted (a burst of admissions would otherwise wait on page locking)
    if (!s.h_jout) s.h_jout = static_cast<double *>(pinned_.get((size_t)s.Nt * NSLOT * 8));
    if (!s.h_const) s.h_const = static_cast<double *>(pinned_.get((size_t)s.ntiles * NSLOT * 8));
    cuda_check(cudaMemcpyAsync(s.h_jout, s.jout, (size_t)s.Nt * NSLOT * 8, cudaMemcpyDeviceToHost, stream_),
               "copy outputs");
    cuda_check(cudaMemcpyAsync(s.h_const, s.constpart, (size_t)s.ntiles * NSLOT * 8, cudaMemcpyDeviceToHost, stream_),
               "copy constant parts");
    cuda_check(cudaEventRecord(s.ev, stream_), "event record");
    s.fetched = true;
}

bool Engine::ready(int id)
{
    Solve &s = get(id);
    if (!s.fetched) return false;
    cudaError_t e = cudaEventQuery(s.ev);
    if (e == cudaErrorNotReady) return false;
    cuda_check(e, "event query");
    return true;
}

void Engine::raw_outputs(int id, std::vector<double> &jout, double cp[NSLOT])
{
    Solve &s = get(id);
    if (!s.fetched) fetch_async(id);
    cuda_check(cudaEventSynchronize(s.ev), "event sync");
    for (int q = 0; q < NSLOT; ++q) cp[q] = 0.0;
    for (int t = 0; t < s.ntiles; ++t)
        for (int q = 0; q < NSLOT; ++q) cp[q] += s.h_const[(size_t)t * NSLOT + q];
    jout.assign(s.h_jout, s.h_jout + (size_t)s.Nt * NSLOT);
}

int Engine::snapshots(int id, double *occ1d, double *nc, double *pi)
{
    drain_pending();
    Solve &s = get(id);
    if (s.nshots == 0) return 0;
    const Problem &p = s.prob;
    const size_t n = (size_t)s.nshots * s.nk;
    if (occ1d) {
        double *d_occ = nullptr;
        const size_t b = (size_t)s.nshots * p.Nk[0] * 8;
        cuda_check(cudaMallocAsync(reinterpret_cast<void **>(&d_occ), b, stream_), "alloc snapshot bins");
        cudaError_t e = launch_snapshot_bins(s.snap_nc, s.nk, s.k_begin, p.Nk, s.nshots, d_occ, stream_);
        if (e == cudaSuccess) e = cudaMemcpyAsync(occ1d, d_occ, b, cudaMemcpyDeviceToHost, stream_);
        cudaFreeAsync(d_occ, stream_);
        cuda_check(e, "snapshot bins");
    }
    if (nc) cuda_check(cudaMemcpyAsync(nc, s.snap_nc, n * 8, cudaMemcpyDeviceToHost, stream_), "copy snapshots");
    if (pi) cuda_check(cudaMemcpyAsync(pi, s.snap_pi, n * 16, cudaMemcpyDeviceToHost, stream_), "copy snapshots");
    cuda_check(cudaStreamSynchronize(stream_), "snapshot sync");
    return s.nshots;
}

void Engine::harmonics(int id, double w0, int hmax, double *band_power)
{
    drain_pending();
    Solve &s = get(id);
    const Problem &p = s.prob;
    HarmonicsInput in;
    in.jout = s.jout;
    in.stride = NSLOT;
    in.nt = s.Nt;
    in.dt = p.laser.dt;
    in.dV = p.dV;
    double *A = nullptr;
    if (p.gauge == GAUGE_VELOCITY) {  // intra += rho0 parts (per tile) + Nval A(t_n) sum_k w_k
        in.cp = s.constpart;
        in.ntiles = s.ntiles;
        in.cp_stride = NSLOT;
        in.cp_slot = 2;
        // A(t_n) in FP64 on the device (the stage-time table with the single fraction 0)
        const double c0 = 0.0;
        cuda_check(cudaMallocAsync(reinterpret_cast<void **>(&A), 16 * (size_t)s.Nt, stream_), "alloc A table");
        cuda_check(launch_field_table(laser_dev(p.laser), p.laser.atmin, p.laser.dt, s.Nt, 1, &c0, true, nullptr,
                                      nullptr, A, false, stream_),
                   "A table kernel");
        in.A = A;
        in.nvw = p.nval * p.total_weight;
    }
    harmonics_on_device(in, w0, hmax, band_power, stream_);
    if (A) cudaFreeAsync(A, stream_);
}

SolveOutputs Engine::outputs(int id, const std::vector<double> *laser)
{
    std::vector<double> j;
    double cp[NSLOT];
    raw_outputs(id, j, cp);
    SolveOutputs o;
    assemble_outputs(get(id).prob, j, cp, o, laser);
    return o;
}

void Engine::remove(int id)
{
    auto it = live_.find(id);
    if (it == live_.end()) return;
    drain_pending();   // the frees below follow the solve's set-up on the copy stream
    Solve &s = *it->second;
    cudaFreeAsync(s.kc, stream_);
    cudaFreeAsync(s.st, stream_);
    cudaFreeAsync(s.tab, stream_);
    cudaFreeAsync(s.partial, stream_);
    cudaFreeAsync(s.jout, stream_);
    cudaFreeAsync(s.constpart, stream_);
    if (s.snap_nc) cudaFreeAsync(s.snap_nc, stream_);
    if (s.snap_pi) cudaFreeAsync(s.snap_pi, stream_);
    if (s.fetched) cudaEventSynchronize(s.ev);
    pinned_.put(s.h_jout, (size_t)s.Nt * NSLOT * 8);
    pinned_.put(s.h_const, (size_t)s.ntiles * NSLOT * 8);
    cudaEventDestroy(s.ev);
    bytes_in_use_ -= s.bytes;
    free_slots_.push_back(s.slot);
    live_.erase(it);
    dirty_ = true;
}

// ================================================================ outputs
void assemble_outputs(const Problem &p, const std::vector<double> &jout, const double cp[NSLOT], SolveOutputs &o,
                      const std::vector<double> *laser)
{
    const int Nt = p.laser.Nt, N = p.nband;
    o.Nt = Nt;
    o.nband = N;
    o.inter.assign((size_t)Nt * 3, 0.0);
    o.intra.assign((size_t)Nt * 3, 0.0);
    o.occ.assign((size_t)Nt * (N + 1), 0.0);
    o.coh.assign((size_t)Nt * 2, 0.0);
    if (laser && laser->size() == (size_t)Nt * 7) o.laser = *laser;
    else o.laser = laser_rows(p);
    const bool vg = p.gauge == GAUGE_VELOCITY;
    const double W = p.total_weight, dV = p.dV, Ntot = (double)p.ntotal();
    std::vector<double> occ00((size_t)Nt), occ01r((size_t)Nt), occ01i((size_t)Nt);
    for (int n = 0; n < Nt; ++n) {
        const double *j = &jout[(size_t)n * NSLOT];
        const double *A = &o.laser[(size_t)n * 7 + 4];
        double inter[3] = {j[0], j[1], 0.0};
        double intra[3] = {j[2], j[3], 0.0};
        if (vg) {
            intra[0] += cp[2];
            intra[1] += cp[3];
            for (int d = 0; d < 3; ++d) intra[d] += p.nval * A[d] * W;  // SBEs.h:750-757
        }
        for (int d = 0; d < 3; ++d) {
            if (p.inter_intra) {
                o.inter[(size_t)n * 3 + d] = inter[d] * dV;
                o.intra[(size_t)n * 3 + d] = intra[d] * dV;
            } else {  // GenCurrent: the total current goes to the inter column (antelope.cpp:316-324)
                o.inter[(size_t)n * 3 + d] = (inter[d] + intra[d]) * dV;
            }
        }
        const double r00 = j[4] + cp[4], r11 = j[5] + cp[5];
        o.occ[(size_t)n * (N + 1) + 0] = r00 / Ntot;
        o.occ[(size_t)n * (N + 1) + 1] = r11 / Ntot;
        o.occ[(size_t)n * (N + 1) + 2] = (r00 + r11) / Ntot;
        occ00[n] = r00;
        occ01r[n] = j[6] + cp[6];
        occ01i[n] = j[7] + cp[7];
    }
    // coherence__full__evol.dat reads flat element Nval*N + Nval + 1 of the
    // per-step N x N array (antelope.cpp:539-542); for N = 2 that is element 0
    // of the NEXT step, and past the end for the last step (written as 0 here).
    const int e = p.nval * N + p.nval + 1;
    for (int n = 0; n < Nt; ++n) {
        const int row = n + e / (N * N), el = e % (N * N);
        double re = 0.0, im = 0.0;
        if (row < Nt) {
            if (el == 0) re = occ00[row];
            else if (el == 1) { re = occ01r[row]; im = occ01i[row]; }
            else if (el == 2) { re = occ01r[row]; im = -occ01i[row]; }
            else re = o.occ[(size_t)row * (N + 1) + 1] * Ntot;
        }
        o.coh[(size_t)n * 2] = re / Ntot;
        o.coh[(size_t)n * 2 + 1] = im / Ntot;
    }
}

void write_outputs(const Problem &p, const SolveOutputs &o, const std::string &dir)
{
    auto path = [&](const char *f) { return dir.empty() ? std::string(f) : dir + "/" + f; };
    auto open = [&](const char *f) {
        FILE *fp = std::fopen(path(f).c_str(), "w");
        if (!fp) throw CfgError(std::string("cannot open ") + path(f) + " for writing");
        return fp;
    };
    FILE *lf = open("outlaserdata.dat");
    for (int n = 0; n < o.Nt; ++n) {
        const double *L = &o.laser[(size_t)n * 7];
        std::fprintf(lf, "%e    ", L[0]);
        for (int d = 0; d < 3; ++d) std::fprintf(lf, "%e      ", L[1 + d]);
        for (int d = 0; d < 3; ++d) std::fprintf(lf, "%e      ", L[4 + d]);
        std::fprintf(lf, "\n");
    }
    std::fclose(lf);
    std::fclose(open("laserParameters.dat"));  // opened but never written by the reference
    FILE *fi = open("interband_dipole_full_evol.dat");
    FILE *fa = open("intraband_current_full_evol.dat");
    FILE *fo = open("occupation__full__evol.dat");
    FILE *fc = open("coherence__full__evol.dat");
    const int N = o.nband;
    for (int n = 0; n < o.Nt; ++n) {
        for (int d = 0; d < 3; ++d) {
            std::fprintf(fi, "%.16e    ", o.inter[(size_t)n * 3 + d]);
            std::fprintf(fa, "%.16e    ", o.intra[(size_t)n * 3 + d]);
        }
        std::fprintf(fi, "\n");
        std::fprintf(fa, "\n");
        for (int m = 0; m < N; ++m) std::fprintf(fo, "%.16e    ", o.occ[(size_t)n * (N + 1) + m]);
        std::fprintf(fo, "%.16e\n", o.occ[(size_t)n * (N + 1) + N]);
        std::fprintf(fc, "%.16e    ", o.coh[(size_t)n * 2]);
        std::fprintf(fc, "%.16e\n", o.coh[(size_t)n * 2 + 1]);
    }
    std::fclose(fi);
    std::fclose(fa);
    std::fclose(fo);
    std::fclose(fc);
    (void)p;
}

}  // namespace sbe
