// Allocation-free solve: sbe_solve_noalloc (include/sbe.h).
//
// Who needs it: a caller that must not allocate device memory itself -- for
// example code embedded in a host application whose device memory is owned by
// that application's pool allocator (a stray cudaMalloc can fail against the
// pool's reservation or fragment it), or a latency-critical loop in which
// cudaMalloc/cudaFree may implicitly synchronise the whole device.  Such a
// caller still hands over its inputs (a parsed problem) and receives its
// outputs in its own host arrays; everything the regular solver would put in
// freshly allocated device memory (per-k constants, per-k state, field
// table, tile partials, per-step sums, launch descriptors) lives instead in
// one file-scope device array of fixed size, SBE_NOALLOC_SCRATCH_BYTES.
//
// Contract:
//  - The array is part of the library image: every GPU that loads the library
//    holds it (64 MiB) until the process exits.
//  - The first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; make that
//    first call before any stream capture on that device.
//  - All calls on a device share the one array, and it keeps the previous
//    call's contents; every region a kernel reads before writing is cleared
//    or rewritten by each call.  Two calls whose GPU work overlaps would race
//    on it: calls in this process are serialised by a lock and each returns
//    only after its GPU work has finished.
//  - Problems whose arrays do not fit are rejected with SBE_OOM and a message
//    giving the bytes needed; the steps per launch shrink to fit the tile
//    partials into what is left.
//  - No cudaMalloc, cudaFree, cudaMallocHost or other allocating routine is
//    called; host-side staging uses a fixed static buffer.
//  - The caller's current device is restored before returning, and every
//    return -- error paths included -- comes after the GPU work this call
//    queued has finished, so the next call never races on the array.
//  - Default launch shape: the engine's heuristic without the autotuner (two
//    k-points per thread for the mixed method, the largest CTA of at
//    most 128 threads that still gives two CTAs per SM); with the same tile_k
//    and k_per_thread the results equal sbe_solver_*'s bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/sbe.h"
#include "sbe_dev.h"
#include "sbe_handles.h"
#include "sbe_kernels.h"
#include "sbe_problem.h"

using namespace sbe;

#define SBE_NOALLOC_SCRATCH_BYTES (64ull << 20)

static __device__ __align__(256) unsigned char g_noalloc_scratch[SBE_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
constexpr size_t kStageDoubles = 1 << 16;   // 512 KiB host staging buffer
double g_stage[kStageDoubles];
void *g_scratch_ptr[kMaxDevices];
std::mutex g_lock;

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

// Device address of the scratch array on the current device, looked up once.
cudaError_t scratch_address(int device, unsigned char **out)
{
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!g_scratch_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[device] = p;
    }
    *out = static_cast<unsigned char *>(g_scratch_ptr[device]);
    return cudaSuccess;
}

struct Layout {
    size_t kc, st, tab, jout, cp, desc, tiles, ids, partial, end;
    int S;
};

}  // namespace

extern "C" sbe_status sbe_solve_noalloc(const sbe_problem *problem, const sbe_opts *opts, void *stream,
                                        const sbe_outputs *out)
{
    auto sbe_noalloc_fail = [](sbe_status st, const char *m) { return set_error(st, m); };
    if (!problem || !out) return sbe_noalloc_fail(SBE_INVALID_ARGUMENT, "null problem or outputs");
    if (!problem->unsupported.empty()) return sbe_noalloc_fail(SBE_UNSUPPORTED, problem->unsupported.c_str());
    const Problem &p = problem->p;
    if (p.model != MODEL_HALDANE || p.gauge == GAUGE_LENGTH_HAMILTONIAN || (p.rk != 4 && p.rk != 5) ||
        p.shot_number > 0)
        return sbe_noalloc_fail(SBE_UNSUPPORTED, "the allocation-free entry point runs the Haldane solves of "
                                                 "sbe_solver_* (velocity or length gauge, RKorder 4 or 5)");
    const int device = opts ? opts->device : 0;
    const int precision = (opts && opts->precision >= 0) ? opts->precision : p.precision;
    const bool is_vg = p.gauge == GAUGE_VELOCITY;
    // launch shape: the engine's defaults (Engine::shape_for) without the autotuner
    int kpt = (opts && opts->k_per_thread > 0) ? opts->k_per_thread : (precision == PREC_MIXED ? 2 : 1);
    if (!is_vg && precision == PREC_FP64) kpt = 1;
    if (kpt != 1 && kpt != 2) return sbe_noalloc_fail(SBE_INVALID_ARGUMENT, "k_per_thread must be 1 or 2");
    int tile_k = (opts && opts->tile_k > 0) ? opts->tile_k : 0;
    if (tile_k == 0) {
        int sms = 148;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) sms = 148;
        int th = 128;
        while (th > 32 && (long long)p.ntotal() < 2LL * sms * th * kpt) th /= 2;
        tile_k = th * kpt;
    }
    const int threads = tile_k / kpt;
    if (threads < 32 || threads > 256 || threads % 32 || tile_k % kpt)
        return sbe_noalloc_fail(SBE_INVALID_ARGUMENT, "tile_k / k_per_thread must be a multiple of 32 in [32, 256]");
    const bool vg = is_vg;
    const int variant = vg ? VAR_HALDANE_VG : VAR_HALDANE_LW;
    const size_t real = precision == PREC_FP64 ? 8 : 4;
    const int nk = p.ntotal(), Nt = p.laser.Nt;
    const int ntiles = (nk + tile_k - 1) / tile_k;
    const size_t nk_pad = (size_t)ntiles * tile_k;
    static const double c4[3] = {0.0, 0.5, 1.0};                        // SBEs.h:398
    static const double c5[6] = {0.0, 0.25, 3. / 8., 12. / 13., 1.0, 0.5};  // SBEs.h:405
    const double *cfr = p.rk == 4 ? c4 : c5;
    const int nts = p.rk == 4 ? 3 : 6;
    const int ncols = vg ? 2 : LW_NPHASE;
    const size_t nconst = vg ? (size_t)VG_NCONST_ALL : (size_t)LW_NCONST;   // as the init kernel writes

    // carve the scratch array
    Layout L{};
    size_t off = 0;
    L.kc = off;      off += round256(nconst * nk_pad * real);
    const size_t nstate = vg ? (size_t)VG_NSTATE_ALL : (size_t)LW_NSTATE_ALL;
    L.st = off;      off += round256(nstate * nk_pad * 8);
    L.tab = off;     off += round256((size_t)Nt * nts * ncols * real);
    L.jout = off;    off += round256((size_t)Nt * NSLOT * 8);
    L.cp = off;      off += round256((size_t)ntiles * NSLOT * 8);
    L.desc = off;    off += round256(sizeof(SolveDev));
    L.tiles = off;   off += round256((size_t)ntiles * sizeof(TileDev));
    L.ids = off;     off += 256;
    L.partial = off;
    const size_t row = (size_t)ntiles * NSLOT * 8;  // partial bytes per step
    if (off + row > SBE_NOALLOC_SCRATCH_BYTES) {
        std::string m = "problem needs " + std::to_string(off + row) +
                        " bytes of device scratch; the allocation-free entry point has " +
                        std::to_string(SBE_NOALLOC_SCRATCH_BYTES) + " (use sbe_solver_* for larger problems)";
        return sbe_noalloc_fail(SBE_OOM, m.c_str());
    }
    const int Sreq = (opts && opts->steps_per_launch > 0) ? opts->steps_per_launch : 1024;
    L.S = (int)std::min<size_t>((size_t)Sreq, (SBE_NOALLOC_SCRATCH_BYTES - off) / row);
    L.end = off + (size_t)L.S * row;

    std::lock_guard<std::mutex> guard(g_lock);
    auto cu = [&](cudaError_t e, const char *what) -> bool {
        if (e == cudaSuccess) return true;
        std::string m = std::string(what) + ": " + cudaGetErrorString(e);
        sbe_noalloc_fail(SBE_CUDA_ERROR, m.c_str());
        return false;
    };
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // on every return: wait for what this call queued (so an early error
    // cannot leave work running on the shared array after the lock is
    // released), then give the caller back its current device
    struct Leave {
        int prev = -1;
        cudaStream_t st = nullptr;
        ~Leave()
        {
            cudaStreamSynchronize(st);
            if (prev >= 0) cudaSetDevice(prev);
        }
    } leave;
    leave.st = st;
    if (!cu(cudaGetDevice(&leave.prev), "cudaGetDevice")) return SBE_CUDA_ERROR;
    unsigned char *base = nullptr;
    if (!cu(cudaSetDevice(device), "cudaSetDevice")) return SBE_CUDA_ERROR;
    if (!cu(scratch_address(device, &base), "cudaGetSymbolAddress(scratch)")) return SBE_CUDA_ERROR;

    // field table, staged through the static host buffer in row chunks
    {
        const size_t per_row = (size_t)nts * ncols;
        const size_t rows_per_chunk = kStageDoubles / per_row;
        for (size_t r0 = 0; r0 < (size_t)Nt; r0 += rows_per_chunk) {
            const size_t r1 = std::min((size_t)Nt, r0 + rows_per_chunk);
            float *f = reinterpret_cast<float *>(g_stage);
            for (size_t n = r0; n < r1; ++n) {
                const double t = p.laser.atmin + p.laser.dt * (double)n;
                for (int j = 0; j < nts; ++j) {
                    double A[3];
                    p.laser.eval(j == 0 ? t : t + cfr[j] * p.laser.dt, A, nullptr);
                    double v[LW_NPHASE];
                    if (vg) {
                        v[0] = A[0];
                        v[1] = A[1];
                    } else {
                        for (int i = 0; i < 3; ++i) {
                            const double aa = A[0] * p.hal_va[i][0] + A[1] * p.hal_va[i][1];
                            const double ab = A[0] * p.hal_vb[i][0] + A[1] * p.hal_vb[i][1];
                            v[i] = std::cos(aa);
                            v[3 + i] = std::sin(aa);
                            v[6 + i] = std::cos(ab);
                            v[9 + i] = std::sin(ab);
                        }
                    }
                    const size_t o = ((n - r0) * nts + j) * ncols;
                    for (int c = 0; c < ncols; ++c) {
                        if (precision == PREC_FP64) g_stage[o + c] = v[c];
                        else f[o + c] = (float)v[c];
                    }
                }
            }
            if (!cu(cudaMemcpyAsync(base + L.tab + r0 * per_row * real, g_stage, (r1 - r0) * per_row * real,
                                    cudaMemcpyHostToDevice, st), "copy field table") ||
                !cu(cudaStreamSynchronize(st), "sync"))
                return SBE_CUDA_ERROR;
        }
    }
    // launch descriptors
    SolveDev d;
    std::memset(&d, 0, sizeof(d));
    d.nk = nk;
    d.ntiles = ntiles;
    d.Nt = Nt;
    d.admit_tick = 0;
    d.nk_pad = (int)nk_pad;
    d.nts = nts;
    d.variant = variant;
    d.precision = precision;
    d.kc = base + L.kc;
    d.st = base + L.st;
    d.tab = base + L.tab;
    d.partial = reinterpret_cast<double *>(base + L.partial);
    d.jout = reinterpret_cast<double *>(base + L.jout);
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
    const int zero_id = 0;
    if (!cu(cudaMemcpyAsync(base + L.desc, &d, sizeof(d), cudaMemcpyHostToDevice, st), "copy descriptor") ||
        !cu(cudaMemcpyAsync(base + L.ids, &zero_id, sizeof(int), cudaMemcpyHostToDevice, st), "copy id") ||
        !cu(cudaStreamSynchronize(st), "sync"))
        return SBE_CUDA_ERROR;
    {
        TileDev *tb = reinterpret_cast<TileDev *>(g_stage);
        const size_t per_chunk = kStageDoubles * sizeof(double) / sizeof(TileDev);
        for (size_t t0 = 0; t0 < (size_t)ntiles; t0 += per_chunk) {
            const size_t t1 = std::min((size_t)ntiles, t0 + per_chunk);
            for (size_t t = t0; t < t1; ++t) {
                tb[t - t0].solve = 0;
                tb[t - t0].k0 = (int)t * tile_k;
                tb[t - t0].kcount = std::min(tile_k, nk - (int)t * tile_k);
                tb[t - t0].tile = (int)t;
            }
            if (!cu(cudaMemcpyAsync(base + L.tiles + t0 * sizeof(TileDev), tb, (t1 - t0) * sizeof(TileDev),
                                    cudaMemcpyHostToDevice, st), "copy tiles") ||
                !cu(cudaStreamSynchronize(st), "sync"))
                return SBE_CUDA_ERROR;
        }
    }
    // per-k set-up into cleared constants and state
    InitArgs ia{};
    ia.nk = nk;
    ia.nk_pad = (int)nk_pad;
    ia.tile_k = tile_k;
    ia.variant = variant;
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
    if (!cu(cudaMemsetAsync(base + L.kc, 0, nconst * nk_pad * real, st), "clear constants") ||
        !cu(cudaMemsetAsync(base + L.st, 0, nstate * nk_pad * 8, st), "clear state") ||
        !cu(launch_init_haldane(ia, precision, base + L.kc, base + L.st, reinterpret_cast<double *>(base + L.cp), st),
            "init kernel"))
        return SBE_CUDA_ERROR;
    // every time step: propagate the tiles, then sum them
    const int nticks = (Nt + L.S - 1) / L.S;
    LaunchArgs la{};
    la.tiles = reinterpret_cast<const TileDev *>(base + L.tiles);
    la.solves = reinterpret_cast<const SolveDev *>(base + L.desc);
    la.ntiles = ntiles;
    la.threads = threads;
    la.S = L.S;
    la.variant = variant;
    la.precision = precision;
    la.rk = p.rk;
    la.kpt = kpt;
    la.has_g1 = p.T1 > 1.0e-16;
    la.stream = st;
    for (int t = 0; t < nticks; ++t) {
        la.tick = t;
        if (!cu(launch_propagate(la), "propagate launch") ||
            !cu(launch_reduce(la.solves, reinterpret_cast<const int *>(base + L.ids), 1, t, L.S, st), "reduce launch"))
            return SBE_CUDA_ERROR;
    }
    // constant parts, summed in tile order
    double cp[NSLOT] = {0};
    {
        const size_t per_chunk = kStageDoubles / NSLOT;
        for (size_t t0 = 0; t0 < (size_t)ntiles; t0 += per_chunk) {
            const size_t t1 = std::min((size_t)ntiles, t0 + per_chunk);
            if (!cu(cudaMemcpyAsync(g_stage, base + L.cp + t0 * NSLOT * 8, (t1 - t0) * NSLOT * 8,
                                    cudaMemcpyDeviceToHost, st), "copy constant parts") ||
                !cu(cudaStreamSynchronize(st), "sync"))
                return SBE_CUDA_ERROR;
            for (size_t t = 0; t < t1 - t0; ++t)
                for (int q = 0; q < NSLOT; ++q) cp[q] += g_stage[t * NSLOT + q];
        }
    }
    // per-step sums -> the reference's output quantities, one chunk of rows at
    // a time (one extra row for the coherence file's next-row element)
    const int N = p.nband;
    const double W = p.total_weight, dV = p.dV, Ntot = (double)nk;
    const size_t rows_per_chunk = kStageDoubles / NSLOT - 1;
    for (size_t r0 = 0; r0 < (size_t)Nt; r0 += rows_per_chunk) {
        const size_t r1 = std::min((size_t)Nt, r0 + rows_per_chunk);
        const size_t rcopy = std::min((size_t)Nt, r1 + 1) - r0;
        if (!cu(cudaMemcpyAsync(g_stage, base + L.jout + r0 * NSLOT * 8, rcopy * NSLOT * 8, cudaMemcpyDeviceToHost, st),
                "copy per-step sums") ||
            !cu(cudaStreamSynchronize(st), "sync"))
            return SBE_CUDA_ERROR;
        for (size_t n = r0; n < r1; ++n) {
            const double *j = g_stage + (n - r0) * NSLOT;
            const double t = p.laser.atmin + p.laser.dt * (double)n;
            double A[3], E[3];
            p.laser.eval(t, A, E);
            if (out->laser) {
                double *Lr = out->laser + n * 7;
                Lr[0] = t;
                for (int c = 0; c < 3; ++c) { Lr[1 + c] = E[c]; Lr[4 + c] = A[c]; }
            }
            double inter[3] = {j[0], j[1], 0.0}, intra[3] = {j[2], j[3], 0.0};
            if (vg) {
                intra[0] += cp[2];
                intra[1] += cp[3];
                for (int c = 0; c < 3; ++c) intra[c] += p.nval * A[c] * W;  // SBEs.h:750-757
            }
            for (int c = 0; c < 3; ++c) {
                const double vi = p.inter_intra ? inter[c] * dV : (inter[c] + intra[c]) * dV;
                const double va = p.inter_intra ? intra[c] * dV : 0.0;
                if (out->inter) out->inter[n * 3 + c] = vi;
                if (out->intra) out->intra[n * 3 + c] = va;
            }
            const double r00 = j[4] + cp[4], r11 = j[5] + cp[5];
            if (out->occ) {
                out->occ[n * (N + 1) + 0] = r00 / Ntot;
                out->occ[n * (N + 1) + 1] = r11 / Ntot;
                out->occ[n * (N + 1) + 2] = (r00 + r11) / Ntot;
            }
            if (out->coh) {  // flat element Nval*N + Nval + 1 = element 0 of the next row (N = 2)
                out->coh[n * 2] = (n + 1 < (size_t)Nt) ? (g_stage[(n + 1 - r0) * NSLOT + 4] + cp[4]) / Ntot : 0.0;
                out->coh[n * 2 + 1] = 0.0;
            }
        }
    }
    return SBE_OK;
}
