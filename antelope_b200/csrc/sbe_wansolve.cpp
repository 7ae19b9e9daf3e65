// Host side of the N-band Wannier solves (length gauge): device buffers,
// model upload, the attempt/controller launch loop, and the assembly of the
// reference's output quantities for N bands (antelope.cpp:514-548).
#include "sbe_wansolve.h"

#include "sbe_kernels.h"
#include "sbe_wannier.h"
#include "sbe_spectrum.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace sbe {

namespace {
template <class T> void dalloc(T **p, size_t bytes, cudaStream_t st, const char *what)
{
    // a continuum model has no tables: its table buffers get a token size
    cuda_check(cudaMallocAsync(reinterpret_cast<void **>(p), std::max<size_t>(bytes, 16), st), what);
}
}  // namespace

WannierSolve::WannierSolve(const Problem &p, int precision, int device, cudaStream_t st, int k_begin, int k_end)
    : prob_(p), precision_(precision), device_(device), stream_(st)
{
    if (p.model != MODEL_SYNTHETIC_WANNIER && p.model != MODEL_TB && p.model != MODEL_MULTIWSM)
        throw CfgError("not a tight-binding problem");
    if (p.gauge != GAUGE_LENGTH_WANNIER && p.gauge != GAUGE_VELOCITY)
        throw CfgError("tight-binding models run in the LengthWannier or Velocity gauge");
    if (p.w_nR > WAN_MAXR) throw CfgError("tight-binding model: at most 64 hopping vectors");
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    const int N = p.nband, NN = N * N;
    std::memset(&w_, 0, sizeof(w_));
    w_.N = N;
    w_.nval = p.nval;
    w_.nR = p.w_nR;
    const int kb = k_end > 0 ? k_begin : 0, ke = k_end > 0 ? k_end : p.ntotal();
    if (kb < 0 || ke > p.ntotal() || kb >= ke) throw CfgError("k-slice outside the grid");
    w_.nk = ke - kb;
    w_.k_offset = kb;
    w_.Nt = p.laser.Nt;
    w_.ntiles = (w_.nk + WAN_WARPS - 1) / WAN_WARPS;
    w_.rk = p.rk;
    w_.inter_intra = p.inter_intra ? 1 : 0;
    w_.use_fermi = p.use_fermi ? 1 : 0;
    w_.has_dip = p.w_d.empty() ? 0 : 1;
    w_.has_jtab = p.w_j.empty() ? 0 : 1;
    w_.vg = p.gauge == GAUGE_VELOCITY ? 1 : 0;
    if (p.model == MODEL_MULTIWSM) {   // formulas in place of tables; its own current operator
        w_.cont = 1;
        w_.has_jtab = 1;
        w_.mw_n = p.mw_n;
        w_.mw_v = p.mw_v;
        w_.mw_alphan = p.mw_alphan;
    }
    w_.Ef = p.Ef;
    w_.dt = p.dt;
    w_.atmin = p.laser.atmin;
    w_.tol = p.rk_tol;
    w_.g1 = p.T1 > 1.0e-16 ? 1.0 / p.T1 : 0.0;  // SBEs.h:484-493
    w_.g2 = p.T2 > 1.0e-16 ? 1.0 / p.T2 : 0.0;
    for (int i = 0; i < 3; ++i) w_.Ngrid[i] = p.Nk[i];
    for (int i = 0; i < 9; ++i) w_.axes[i] = p.bzaxes[i];
    for (int i = 0; i < 3; ++i) w_.origin[i] = p.bzorigin[i];
    w_.laser = laser_dev(p.laser);

    const size_t real = precision_ == 0 ? 8 : 4, cplx = 2 * real;
    const size_t nk = (size_t)w_.nk;
    double *V = nullptr;
    void *h = nullptr, *d = nullptr, *j = nullptr;
    dalloc(&V, sizeof(double) * p.w_vec.size(), st, "alloc hopping vectors");
    dalloc(&h, cplx * p.w_h.size() / 2, st, "alloc h");
    if (w_.has_dip) dalloc(&d, cplx * p.w_d.size() / 2, st, "alloc d");
    if (w_.has_jtab && !w_.cont) dalloc(&j, cplx * p.w_j.size() / 2, st, "alloc current tables");
    for (int b = 0; b < 2; ++b) {
        dalloc(&w_.rho[b], sizeof(double2) * nk * NN, st, "alloc rho");
        dalloc(&w_.U[b], sizeof(double2) * nk * NN, st, "alloc U");
    }
    dalloc(&w_.weight, sizeof(double) * nk, st, "alloc weights");
    if (w_.vg) {
        dalloc(&w_.vg_eps, sizeof(double) * nk * N, st, "alloc band energies");
        dalloc(&w_.vg_f, sizeof(double) * nk * N, st, "alloc occupations");
        dalloc(&w_.vg_P, sizeof(double2) * nk * (w_.cont ? 3 : 2) * NN, st, "alloc momentum matrices");
    }
    dalloc(&w_.tile_err, sizeof(double) * w_.ntiles, st, "alloc tile errors");
    dalloc(&w_.cur_part, sizeof(double) * w_.ntiles * WAN_NSLOT, st, "alloc current partials");
    dalloc(&w_.jout, sizeof(double) * (size_t)w_.Nt * WAN_NSLOT, st, "alloc outputs");
    dalloc(&w_.ctl, sizeof(WanCtl), st, "alloc control");
    dalloc(&w_.stage_AE, sizeof(double) * 36, st, "alloc stage fields");
    dalloc(&w_.stage_cA, cplx * 6 * (size_t)w_.nR, st, "alloc stage phases");
    nshots_ = p.nshots();
    if (nshots_ > 0) {   // density snapshots (antelope.cpp:267-422)
        w_.shot_every = p.shot_every();
        dalloc(&w_.snap_nc, sizeof(double) * nshots_ * nk, st, "alloc snapshots");
        dalloc(&w_.snap_pi, sizeof(double) * 2 * nshots_ * nk, st, "alloc snapshots");
    }
    dalloc(&d_w_, sizeof(WanDev), st, "alloc descriptor");
    w_.V = V;
    w_.h = h;
    w_.d = d;
    w_.jt = j;
    // the tables re-laid for the grouped attempt kernel.  The lattice vectors
    // are taken in pairs (R, -R) (a vector without its negative, R = 0
    // included, stands alone): h_R e^{iKR} + h_-R e^{-iKR} = c sig + s tau
    // with e^{iKR} = c + i s, sig = h_R + h_-R and tau = i (h_R - h_-R), half
    // the multiplications of the two terms.  Entry (p, j, q, 0|1, l) holds sig
    // or tau of quantity q (h, d_x, d_y) of upper element u = l + 8 j, zero
    // past the triangle or without dipoles.
    std::vector<double> gt;
    std::vector<int> gpair, mate(w_.nR, -1);
    if (wan_grouped_applies(w_)) {
        const int nR = w_.nR;
        std::vector<char> used(nR, 0);
        for (int r = 0; r < nR; ++r) {
            if (used[r]) continue;
            used[r] = 1;
            for (int r2 = r + 1; r2 < nR; ++r2)
                if (!used[r2] && p.w_vec[2 * r2] == -p.w_vec[2 * r] && p.w_vec[2 * r2 + 1] == -p.w_vec[2 * r + 1]) {
                    mate[r] = r2;
                    used[r2] = 1;
                    break;
                }
            gpair.push_back(r);
        }
        // more vectors without their negatives than R = 0 (the SyntheticWannier
        // reader already refuses such a model): the grouped kernel's per-k
        // phase arrays are sized for pairs, so wan_attempt would run it
        if ((int)gpair.size() > wan_npair_cap(nR)) gpair.clear();
    }
    if (!gpair.empty()) {
        const int NU = N * (N + 1) / 2, NO = (NU + 7) / 8, row = wan_gtab_row(N);
        const int np = (int)gpair.size();
        gt.assign((size_t)np * row * 2, 0.0);
        std::vector<int> um(NU), un(NU);
        for (int m = 0, u = 0; m < N; ++m)
            for (int n = m; n < N; ++n, ++u) { um[u] = m; un[u] = n; }
        auto entry = [&](int q, int r, int u, double &re, double &im) {
            const size_t src = q == 0 ? ((size_t)(r * N + um[u]) * N + un[u]) * 2
                                      : ((size_t)((r * 2 + q - 1) * N + um[u]) * N + un[u]) * 2;
            const std::vector<double> &tab = q == 0 ? p.w_h : p.w_d;
            re = tab[src];
            im = tab[src + 1];
        };
        for (int pi = 0; pi < np; ++pi)
            for (int jj = 0; jj < NO; ++jj)
                for (int q = 0; q < 3; ++q)
                    for (int l = 0; l < 8; ++l) {
                        const int u = l + 8 * jj;
                        if (u >= NU || (q > 0 && !w_.has_dip)) continue;
                        double a, b, a2 = 0.0, b2 = 0.0;
                        entry(q, gpair[pi], u, a, b);
                        if (mate[gpair[pi]] >= 0) entry(q, mate[gpair[pi]], u, a2, b2);
                        const size_t dst = (((((size_t)pi * NO + jj) * 3 + q) * 2) * 8 + l) * 2;
                        gt[dst] = a + a2;                 // sig
                        gt[dst + 1] = b + b2;
                        gt[dst + 16] = -(b - b2);         // tau = i (h_R - h_-R)
                        gt[dst + 17] = a - a2;
                    }
        void *g = nullptr;
        int *gp = nullptr;
        dalloc(&g, cplx * gt.size() / 2, st, "alloc grouped tables");
        dalloc(&gp, sizeof(int) * np, st, "alloc lattice-vector pairs");
        w_.gtab = g;
        w_.gpair = gp;
        w_.npair = np;
        if (w_.has_dip) {
            void *sg = nullptr;
            dalloc(&sg, cplx * (size_t)6 * np * NO * 2 * 8, st, "alloc stage tables");
            w_.stage_gt = sg;
        }
    }
    UploadRing &ring = UploadRing::shared();
    if (!p.w_vec.empty()) ring.upload(V, p.w_vec.data(), sizeof(double) * p.w_vec.size(), st);
    auto up_real = [&](void *dst, const std::vector<double> &src) {
        if (precision_ == 0) {
            ring.upload(dst, src.data(), src.size() * 8, st);
        } else {
            std::vector<float> f(src.begin(), src.end());
            ring.upload(dst, f.data(), f.size() * 4, st);
        }
    };
    if (!p.w_h.empty()) up_real(h, p.w_h);
    if (w_.has_dip) up_real(d, p.w_d);
    if (w_.has_jtab && !w_.cont) up_real(j, p.w_j);
    if (w_.gtab) up_real(const_cast<void *>(w_.gtab), gt);
    if (w_.gpair) ring.upload(const_cast<int *>(w_.gpair), gpair.data(), sizeof(int) * gpair.size(), st);
    cuda_check(cudaMemsetAsync(w_.jout, 0, sizeof(double) * (size_t)w_.Nt * WAN_NSLOT, st), "clear outputs");
    // initial controller state: t = t_min, h = dt, currents first
    WanCtl c{};
    c.tc = w_.atmin;
    c.h = w_.dt;
    c.n = 0;
    c.buf = 0;
    c.need_current = 1;
    c.shot = -1;
    const double tend = w_.atmin + w_.dt;
    c.hs = c.h;
    c.last = 0;
    if (c.tc + c.hs >= tend - 1e-12 * w_.dt) {
        c.hs = tend - c.tc;
        c.last = 1;
    }
    ring.upload(w_.ctl, &c, sizeof(c), st);
    ring.upload(d_w_, &w_, sizeof(w_), st);
    cuda_check(launch_wan_init(w_, precision_, st), "Wannier init kernel");
    cuda_check(launch_wan_prepare(d_w_, precision_, st), "Wannier stage preparation");
    cuda_check(cudaMallocHost(&h_ctl_, sizeof(WanCtl)), "cudaMallocHost(control)");
}

WannierSolve::~WannierSolve()
{
    cudaStreamSynchronize(stream_);
    cudaFreeAsync((void *)w_.V, stream_);
    cudaFreeAsync((void *)w_.h, stream_);
    if (w_.d) cudaFreeAsync((void *)w_.d, stream_);
    if (w_.jt) cudaFreeAsync((void *)w_.jt, stream_);
    if (w_.gtab) cudaFreeAsync((void *)w_.gtab, stream_);
    if (w_.gpair) cudaFreeAsync((void *)w_.gpair, stream_);
    if (w_.stage_gt) cudaFreeAsync(w_.stage_gt, stream_);
    for (int b = 0; b < 2; ++b) {
        cudaFreeAsync(w_.rho[b], stream_);
        cudaFreeAsync(w_.U[b], stream_);
    }
    cudaFreeAsync(w_.weight, stream_);
    if (w_.vg_eps) cudaFreeAsync(w_.vg_eps, stream_);
    if (w_.vg_f) cudaFreeAsync(w_.vg_f, stream_);
    if (w_.vg_P) cudaFreeAsync(w_.vg_P, stream_);
    cudaFreeAsync(w_.tile_err, stream_);
    cudaFreeAsync(w_.cur_part, stream_);
    cudaFreeAsync(w_.jout, stream_);
    cudaFreeAsync(w_.ctl, stream_);
    cudaFreeAsync(w_.stage_AE, stream_);
    cudaFreeAsync(w_.stage_cA, stream_);
    cudaFreeAsync(d_w_, stream_);
    if (w_.snap_nc) cudaFreeAsync(w_.snap_nc, stream_);
    if (w_.snap_pi) cudaFreeAsync(w_.snap_pi, stream_);
    cudaStreamSynchronize(stream_);
    if (h_ctl_) cudaFreeHost(h_ctl_);
}

void WannierSolve::run(cudaStream_t st)
{
    stream_ = st;
    // attempts are launched in chunks; the controller makes surplus launches
    // after the last step no-ops, and the host checks progress per chunk
    const int chunk = 64;
    const long long max_attempts = 64LL * w_.Nt + 1000;
    long long launched = 0;
    for (;;) {
        for (int c = 0; c < chunk; ++c) {
            cuda_check(launch_wan_attempt(w_, d_w_, precision_, st), "Wannier attempt kernel");
            cuda_check(launch_wan_control(d_w_, precision_, st), "Wannier control kernel");
            cuda_check(launch_wan_snapshot(w_, d_w_, precision_, st), "Wannier snapshot kernel");
        }
        launched += chunk;
        cuda_check(cudaMemcpyAsync(h_ctl_, w_.ctl, sizeof(WanCtl), cudaMemcpyDeviceToHost, st), "copy control");
        cuda_check(cudaStreamSynchronize(st), "sync");
        if (h_ctl_->done) break;
        if (launched > max_attempts) throw CudaError("Wannier solve made no progress (step-size controller)");
    }
    if (h_ctl_->error) throw CudaError("Cash-Karp step size underflow: tolerance unreachable");
    launches_ = (int)((w_.shot_every > 0 ? 3 : 2) * launched);   // attempt, control (, snapshot)
}

void WannierSolve::finish_batched(const WanCtl &c, int launches)
{
    *h_ctl_ = c;
    launches_ = launches;
    if (c.error) throw CudaError("Cash-Karp step size underflow: tolerance unreachable");
}

// ============================================================= batches
WannierBatch::WannierBatch(const std::vector<const Problem *> &probs, int precision, int device, cudaStream_t st)
    : device_(device), stream_(st)
{
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    for (const Problem *p : probs) {
        const int prec = precision >= 0 ? precision : p->precision;
        solves_.push_back(std::make_unique<WannierSolve>(*p, prec, device_, st));
    }
    // launch classes; within a class the solves with the most k-point steps
    // lead the tile list, so their blocks are scheduled first
    for (int i = 0; i < (int)solves_.size(); ++i) {
        const WanDev &w = solves_[i]->dev();
        const int grk = wan_grouped(w) ? w.rk : 0;
        Class *c = nullptr;
        for (Class &x : classes_)
            if (x.N == w.N && x.vg == (w.vg != 0) && x.precision == solves_[i]->precision() && x.grouped_rk == grk)
                c = &x;
        if (!c) {
            classes_.emplace_back();
            c = &classes_.back();
            c->N = w.N;
            c->vg = w.vg != 0;
            c->precision = solves_[i]->precision();
            c->grouped_rk = grk;
        }
        c->members.push_back(i);
        c->nR = std::max(c->nR, w.nR);
        c->shots = c->shots || w.shot_every > 0;
    }
    UploadRing &ring = UploadRing::shared();
    for (Class &c : classes_) {
        std::stable_sort(c.members.begin(), c.members.end(), [&](int a, int b) {
            const WanDev &x = solves_[a]->dev(), &y = solves_[b]->dev();
            return (double)x.nk * x.Nt > (double)y.nk * y.Nt;
        });
        std::vector<const WanDev *> descs;
        std::vector<WanTileRef> tiles;
        for (int j = 0; j < (int)c.members.size(); ++j) {
            const WannierSolve &s = *solves_[c.members[j]];
            descs.push_back(s.dev_ptr());
        }
        // interleave the solves' tiles round-robin (longest first), so that
        // the blocks of one launch spread every solve over the whole GPU
        // (grouped classes: one entry per block of WAN_GROUP_TILES tiles)
        const int unit = c.grouped_rk ? WAN_GROUP_TILES : 1;
        int maxt = 0;
        for (int m : c.members) maxt = std::max(maxt, solves_[m]->dev().ntiles);
        for (int t = 0; t < maxt; t += unit)
            for (int j = 0; j < (int)c.members.size(); ++j)
                if (t < solves_[c.members[j]]->dev().ntiles) tiles.push_back(WanTileRef{j, t});
        c.ntiles = (int)tiles.size();
        dalloc(&c.d_descs, sizeof(WanDev *) * descs.size(), st, "alloc batch descriptors");
        dalloc(&c.d_tiles, sizeof(WanTileRef) * tiles.size(), st, "alloc batch tiles");
        ring.upload(c.d_descs, descs.data(), sizeof(WanDev *) * descs.size(), st);
        ring.upload(c.d_tiles, tiles.data(), sizeof(WanTileRef) * tiles.size(), st);
        per_iter_ += c.shots ? 3 : 2;
    }
    cuda_check(cudaMallocHost(&h_ctls_, sizeof(WanCtl) * std::max<size_t>(1, solves_.size())),
               "cudaMallocHost(batch control)");
}

WannierBatch::~WannierBatch()
{
    cudaStreamSynchronize(stream_);
    for (Class &c : classes_) {
        if (c.d_descs) cudaFreeAsync(c.d_descs, stream_);
        if (c.d_tiles) cudaFreeAsync(c.d_tiles, stream_);
    }
    cudaStreamSynchronize(stream_);
    solves_.clear();
    if (h_ctls_) cudaFreeHost(h_ctls_);
}

void WannierBatch::enqueue_chunk(cudaStream_t st, int iters)
{
    for (int it = 0; it < iters; ++it)
        for (const Class &c : classes_) {
            cuda_check(launch_wan_attempt_batch(c.N, c.nR, c.vg, c.d_descs, c.d_tiles, c.ntiles, c.precision, st,
                                                c.grouped_rk),
                       "Wannier attempt kernel (batch)");
            cuda_check(launch_wan_control_batch(c.d_descs, (int)c.members.size(), c.precision, st),
                       "Wannier control kernel (batch)");
            if (c.shots)
                cuda_check(launch_wan_snapshot_batch(c.N, c.nR, c.d_descs, c.d_tiles, c.ntiles, c.precision, st),
                           "Wannier snapshot kernel (batch)");
        }
}

void WannierBatch::run(cudaStream_t st, bool use_graph)
{
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    stream_ = st;
    for (auto &s : solves_) s->set_stream(st);
    const int chunk = 64;
    long long max_nt = 0;
    for (auto &s : solves_) max_nt = std::max<long long>(max_nt, s->dev().Nt);
    const long long max_iters = 64LL * max_nt + 1000;
    cudaGraphExec_t ge = nullptr;
    if (use_graph) {
        cudaGraph_t g;
        cuda_check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
        enqueue_chunk(st, chunk);
        cuda_check(cudaStreamEndCapture(st, &g), "end capture");
        cuda_check(cudaGraphInstantiate(&ge, g, 0), "graph instantiate");
        cudaGraphDestroy(g);
    }
    long long iters = 0;
    bool all_done = false;
    while (!all_done) {
        if (ge) cuda_check(cudaGraphLaunch(ge, st), "graph launch");
        else enqueue_chunk(st, chunk);
        iters += chunk;
        for (int i = 0; i < (int)solves_.size(); ++i)
            cuda_check(cudaMemcpyAsync(&h_ctls_[i], solves_[i]->dev().ctl, sizeof(WanCtl), cudaMemcpyDeviceToHost, st),
                       "copy control");
        cuda_check(cudaStreamSynchronize(st), "sync");
        all_done = true;
        for (int i = 0; i < (int)solves_.size(); ++i) all_done = all_done && h_ctls_[i].done;
        if (!all_done && iters > max_iters) {
            if (ge) cudaGraphExecDestroy(ge);
            throw CudaError("Wannier batch made no progress (step-size controller)");
        }
    }
    if (ge) cudaGraphExecDestroy(ge);
    launches_ = (int)(per_iter_ * iters);
    for (int i = 0; i < (int)solves_.size(); ++i) solves_[i]->finish_batched(h_ctls_[i], launches_);
}

// ============================================================= server pool
WannierPool::WannierPool(int device, cudaStream_t st) : device_(device), st_(st)
{
    cuda_check(cudaEventCreateWithFlags(&copied_, cudaEventDisableTiming), "event create");
}

WannierPool::~WannierPool()
{
    cudaStreamSynchronize(st_);
    for (Class &c : classes_) {
        if (c.d_descs) cudaFreeAsync(c.d_descs, st_);
        if (c.d_tiles) cudaFreeAsync(c.d_tiles, st_);
    }
    solves_.clear();
    cudaStreamSynchronize(st_);
    if (h_ctls_) cudaFreeHost(h_ctls_);
    if (copied_) cudaEventDestroy(copied_);
}

size_t WannierPool::bytes_needed(const Problem &p, int precision)
{
    const size_t N = (size_t)p.nband, NN = N * N, nk = (size_t)p.ntotal(), nR = (size_t)std::max(p.w_nR, 1);
    const size_t real = precision == 0 ? 8 : 4, cplx = 2 * real;
    const size_t ntiles = (nk + WAN_WARPS - 1) / WAN_WARPS;
    size_t b = 4 * nk * NN * 16 + nk * 8;                              // rho, U (two each), weights
    b += nR * NN * cplx * 5 + nR * 16 + nR * 216 * cplx;               // h, d, current, re-laid and stage tables, vectors
    b += ntiles * 8 * (1 + WAN_NSLOT) + (size_t)p.laser.Nt * WAN_NSLOT * 8;   // tile results, per-step sums
    if (p.gauge == GAUGE_VELOCITY) b += nk * N * 16 + nk * 3 * NN * 16;  // bands, momentum matrices
    return b + 4096;
}

int WannierPool::add(const Problem &p, int precision)
{
    Entry e;
    e.s = std::make_unique<WannierSolve>(p, precision, device_, st_);
    e.bytes = bytes_needed(p, precision);
    bytes_ += e.bytes;
    const int id = next_id_++;
    solves_.emplace(id, std::move(e));
    dirty_ = true;
    return id;
}

void WannierPool::remove(int id)
{
    auto it = solves_.find(id);
    if (it == solves_.end()) return;
    // no launch of a later step touches it once the classes are rebuilt; the
    // solve's destructor waits for the stream before freeing
    bytes_ -= it->second.bytes;
    solves_.erase(it);
    dirty_ = true;
}

int WannierPool::nrunning() const
{
    int n = 0;
    for (const auto &kv : solves_) n += kv.second.done ? 0 : 1;
    return n;
}

bool WannierPool::finished(int id) const
{
    auto it = solves_.find(id);
    return it != solves_.end() && it->second.done;
}

bool WannierPool::failed(int id) const
{
    auto it = solves_.find(id);
    return it != solves_.end() && it->second.failed;
}

std::vector<double> WannierPool::sums(int id)
{
    auto it = solves_.find(id);
    if (it == solves_.end()) throw CudaError("unknown pool solve");
    return it->second.s->sums();
}

void WannierPool::rebuild()
{
    for (Class &c : classes_) {
        if (c.d_descs) cudaFreeAsync(c.d_descs, st_);
        if (c.d_tiles) cudaFreeAsync(c.d_tiles, st_);
    }
    classes_.clear();
    for (auto &kv : solves_) {
        if (kv.second.done) continue;
        const WannierSolve &s = *kv.second.s;
        const WanDev &w = s.dev();
        const int grk = wan_grouped(w) ? w.rk : 0;
        Class *c = nullptr;
        for (Class &x : classes_)
            if (x.N == w.N && x.vg == (w.vg != 0) && x.precision == s.precision() && x.grouped_rk == grk) c = &x;
        if (!c) {
            classes_.emplace_back();
            c = &classes_.back();
            c->N = w.N;
            c->vg = w.vg != 0;
            c->precision = s.precision();
            c->grouped_rk = grk;
        }
        c->ids.push_back(kv.first);
        c->nR = std::max(c->nR, w.nR);
    }
    UploadRing &ring = UploadRing::shared();
    for (Class &c : classes_) {
        std::vector<const WanDev *> descs;
        std::vector<WanTileRef> tiles;
        const int unit = c.grouped_rk ? WAN_GROUP_TILES : 1;
        int maxt = 0;
        for (int id : c.ids) {
            descs.push_back(solves_.at(id).s->dev_ptr());
            maxt = std::max(maxt, solves_.at(id).s->dev().ntiles);
        }
        for (int t = 0; t < maxt; t += unit)
            for (int j = 0; j < (int)c.ids.size(); ++j)
                if (t < solves_.at(c.ids[j]).s->dev().ntiles) tiles.push_back(WanTileRef{j, t});
        c.ntiles = (int)tiles.size();
        dalloc(&c.d_descs, sizeof(WanDev *) * descs.size(), st_, "alloc pool descriptors");
        dalloc(&c.d_tiles, sizeof(WanTileRef) * tiles.size(), st_, "alloc pool tiles");
        ring.upload(c.d_descs, descs.data(), sizeof(WanDev *) * descs.size(), st_);
        ring.upload(c.d_tiles, tiles.data(), sizeof(WanTileRef) * tiles.size(), st_);
    }
    dirty_ = false;
}

void WannierPool::step(int iters)
{
    last_launches_ = 0;
    if (pending_) poll();
    if (dirty_) rebuild();
    if (classes_.empty()) return;
    for (int it = 0; it < iters; ++it)
        for (const Class &c : classes_) {
            cuda_check(launch_wan_attempt_batch(c.N, c.nR, c.vg, c.d_descs, c.d_tiles, c.ntiles, c.precision, st_,
                                                c.grouped_rk),
                       "Wannier attempt kernel (server)");
            cuda_check(launch_wan_control_batch(c.d_descs, (int)c.ids.size(), c.precision, st_),
                       "Wannier control kernel (server)");
            last_launches_ += 2;
        }
    // controllers of the running solves, read by a later poll()
    polled_.clear();
    for (const Class &c : classes_)
        for (int id : c.ids) polled_.push_back(id);
    if ((int)polled_.size() > cap_) {
        if (h_ctls_) {
            cuda_check(cudaStreamSynchronize(st_), "sync");
            cudaFreeHost(h_ctls_);
        }
        cap_ = std::max<int>(64, 2 * (int)polled_.size());
        cuda_check(cudaMallocHost(&h_ctls_, sizeof(WanCtl) * cap_), "cudaMallocHost(pool control)");
    }
    for (int i = 0; i < (int)polled_.size(); ++i)
        cuda_check(cudaMemcpyAsync(&h_ctls_[i], solves_.at(polled_[i]).s->dev().ctl, sizeof(WanCtl),
                                   cudaMemcpyDeviceToHost, st_),
                   "copy control");
    cuda_check(cudaEventRecord(copied_, st_), "event record");
    pending_ = true;
}

void WannierPool::poll()
{
    if (!pending_) return;
    const cudaError_t q = cudaEventQuery(copied_);
    if (q == cudaErrorNotReady) return;
    cuda_check(q, "pool event");
    pending_ = false;
    for (int i = 0; i < (int)polled_.size(); ++i) {
        auto it = solves_.find(polled_[i]);
        if (it == solves_.end() || it->second.done) continue;
        const WanCtl &c = h_ctls_[i];
        if (c.done) {
            it->second.done = true;
            it->second.failed = c.error != 0;
            if (!c.error) it->second.s->finish_batched(c, 0);
            dirty_ = true;
        }
    }
}

void WannierSolve::harmonics(double w0, int hmax, double *band_power)
{
    const Problem &p = prob_;
    HarmonicsInput in;
    in.jout = w_.jout;
    in.stride = WAN_NSLOT;
    in.nt = w_.Nt;
    in.dt = p.laser.dt;
    in.dV = p.dV;
    double *A = nullptr;
    if (w_.vg) {  // intra += Nval A(t_n) sum_k w_k
        // A(t_n) in FP64 on the device (the stage-time table with the single fraction 0)
        const double c0 = 0.0;
        cuda_check(cudaMallocAsync(reinterpret_cast<void **>(&A), 16 * (size_t)w_.Nt, stream_), "alloc A table");
        cuda_check(launch_field_table(laser_dev(p.laser), p.laser.atmin, p.laser.dt, w_.Nt, 1, &c0, true, nullptr,
                                      nullptr, A, false, stream_),
                   "A table kernel");
        in.A = A;
        in.nvw = p.nval * p.total_weight;
    }
    harmonics_on_device(in, w0, hmax, band_power, stream_);
    if (A) cudaFreeAsync(A, stream_);
}

int WannierSolve::snapshots(double *occ1d, double *nc, double *pi)
{
    if (nshots_ == 0) return 0;
    const size_t n = (size_t)nshots_ * w_.nk;
    if (occ1d) {
        double *d_occ = nullptr;
        const size_t b = (size_t)nshots_ * prob_.Nk[0] * 8;
        dalloc(&d_occ, b, stream_, "alloc snapshot bins");
        cudaError_t e = launch_snapshot_bins(w_.snap_nc, w_.nk, w_.k_offset, prob_.Nk, nshots_, d_occ, stream_);
        if (e == cudaSuccess) e = cudaMemcpyAsync(occ1d, d_occ, b, cudaMemcpyDeviceToHost, stream_);
        cudaFreeAsync(d_occ, stream_);
        cuda_check(e, "snapshot bins");
    }
    if (nc) cuda_check(cudaMemcpyAsync(nc, w_.snap_nc, n * 8, cudaMemcpyDeviceToHost, stream_), "copy snapshots");
    if (pi) cuda_check(cudaMemcpyAsync(pi, w_.snap_pi, n * 16, cudaMemcpyDeviceToHost, stream_), "copy snapshots");
    cuda_check(cudaStreamSynchronize(stream_), "snapshot sync");
    return nshots_;
}

std::vector<double> WannierSolve::sums()
{
    std::vector<double> j((size_t)w_.Nt * WAN_NSLOT);
    cuda_check(cudaMemcpyAsync(j.data(), w_.jout, j.size() * 8, cudaMemcpyDeviceToHost, stream_), "copy outputs");
    cuda_check(cudaStreamSynchronize(stream_), "sync");
    return j;
}

SolveOutputs WannierSolve::outputs()
{
    SolveOutputs o;
    assemble_table_outputs(prob_, sums(), o);
    return o;
}

void assemble_table_outputs(const Problem &p, const std::vector<double> &j, SolveOutputs &o)
{
    const int Nt = p.laser.Nt, N = p.nband, NN = N * N;
    const bool vg = p.gauge == GAUGE_VELOCITY;
    o.Nt = Nt;
    o.nband = N;
    o.inter.assign((size_t)Nt * 3, 0.0);
    o.intra.assign((size_t)Nt * 3, 0.0);
    o.occ.assign((size_t)Nt * (N + 1), 0.0);
    o.coh.assign((size_t)Nt * 2, 0.0);
    o.laser.assign((size_t)Nt * 7, 0.0);
    const double dV = p.dV, Ntot = (double)p.ntotal();
    // velocity gauge: intra_a += Nval A_a(t) per k (SBEs.h:750-757), i.e. Nval A_a sum_k w_k
    const double nvw = vg ? p.nval * p.total_weight : 0.0;
    const int e = p.nval * N + p.nval + 1, roff = e / NN;
    for (int n = 0; n < Nt; ++n) {
        const double *r = &j[(size_t)n * WAN_NSLOT];
        const double t = p.laser.atmin + p.laser.dt * n;
        double A[3], E[3];
        p.laser.eval(t, A, E);
        double *L = &o.laser[(size_t)n * 7];
        L[0] = t;
        for (int d = 0; d < 3; ++d) { L[1 + d] = E[d]; L[4 + d] = A[d]; }
        for (int a = 0; a < 3; ++a) {  // z: the continuum model's slots (zero for the in-plane models)
            const double ie = a < 2 ? r[a] : r[WAN_SLOT_INTER_Z];
            const double ia = (a < 2 ? r[2 + a] : r[WAN_SLOT_INTRA_Z]) + nvw * A[a];
            if (p.inter_intra) {
                o.inter[(size_t)n * 3 + a] = ie * dV;
                o.intra[(size_t)n * 3 + a] = ia * dV;
            } else {  // GenCurrent: the total current goes to the inter column (antelope.cpp:316-324)
                o.inter[(size_t)n * 3 + a] = (ie + ia) * dV;
            }
        }
        double tot = 0.0;
        for (int m = 0; m < N; ++m) {
            o.occ[(size_t)n * (N + 1) + m] = r[4 + m] / Ntot;
            tot += r[4 + m];
        }
        o.occ[(size_t)n * (N + 1) + N] = tot / Ntot;
        const int row = n + roff;  // flat element Nval*N+Nval+1 (antelope.cpp:539-542)
        if (row < Nt) {
            o.coh[(size_t)n * 2] = j[(size_t)row * WAN_NSLOT + 4 + N] / Ntot;
            o.coh[(size_t)n * 2 + 1] = j[(size_t)row * WAN_NSLOT + 5 + N] / Ntot;
        }
    }
}

}  // namespace sbe
