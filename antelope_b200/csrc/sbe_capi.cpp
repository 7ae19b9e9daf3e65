// extern "C" layer (include/sbe.h): problems, single solves, batches, the
// continuous-batching server, and the drop-in run of an inputParam.cfg.
#include "../../include/sbe.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <mutex>
#include <sstream>
#include <thread>
#include <unordered_map>

#include "sbe_engine.h"
#include "sbe_handles.h"
#include "sbe_kernels.h"
#include "sbe_wansolve.h"

using namespace sbe;

namespace {

thread_local std::string g_err;

sbe_status fail(sbe_status st, const std::string &msg)
{
    g_err = msg;
    return st;
}

template <class F>
sbe_status guard(F &&f)
{
    try {
        g_err.clear();
        return f();
    } catch (const OomError &e) {
        return fail(SBE_OOM, e.what());
    } catch (const CudaError &e) {
        return fail(SBE_CUDA_ERROR, e.what());
    } catch (const CfgError &e) {
        return fail(SBE_BAD_CONFIG, e.what());
    } catch (const std::bad_alloc &) {
        return fail(SBE_OOM, "host out of memory");
    } catch (const std::exception &e) {
        return fail(SBE_INVALID_ARGUMENT, e.what());
    }
}

EngineOptions to_engine_opts(const sbe_opts *o)
{
    EngineOptions e;
    if (o) {
        e.precision = o->precision;
        e.tile_k = o->tile_k;
        e.kpt = o->k_per_thread;
        e.steps_per_launch = o->steps_per_launch;
    }
    return e;
}

int default_steps(const sbe_opts *o) { return (o && o->steps_per_launch > 0) ? o->steps_per_launch : 1024; }

sbe_status check_problem(const sbe_problem *p)
{
    if (!p) return fail(SBE_INVALID_ARGUMENT, "null problem");
    if (!p->unsupported.empty()) return fail(SBE_UNSUPPORTED, p->unsupported);
    return SBE_OK;
}

void copy_out(const SolveOutputs &o, const sbe_outputs *out)
{
    if (!out) return;
    if (out->inter) std::memcpy(out->inter, o.inter.data(), o.inter.size() * 8);
    if (out->intra) std::memcpy(out->intra, o.intra.data(), o.intra.size() * 8);
    if (out->occ) std::memcpy(out->occ, o.occ.data(), o.occ.size() * 8);
    if (out->coh) std::memcpy(out->coh, o.coh.data(), o.coh.size() * 8);
    if (out->laser) std::memcpy(out->laser, o.laser.data(), o.laser.size() * 8);
}

// Runs every tick of an engine on `stream`, optionally as one CUDA graph.
void run_engine(Engine &eng, bool use_graph, int *launches)
{
    const int ticks = eng.max_remaining_ticks();
    int n = 0;
    if (use_graph && ticks > 0) {
        eng.step();  // first tick outside the capture: builds the launch lists
        n += eng.last_launches();
        if (ticks > 1) {
            cudaGraph_t g;
            cudaGraphExec_t ge;
            cuda_check(cudaStreamBeginCapture(eng.stream(), cudaStreamCaptureModeThreadLocal), "begin capture");
            for (int t = 1; t < ticks; ++t) {
                eng.step_frozen();
                n += eng.last_launches();
            }
            cuda_check(cudaStreamEndCapture(eng.stream(), &g), "end capture");
            cuda_check(cudaGraphInstantiate(&ge, g, 0), "graph instantiate");
            cuda_check(cudaGraphLaunch(ge, eng.stream()), "graph launch");
            cudaGraphExecDestroy(ge);
            cudaGraphDestroy(g);
        }
    } else {
        for (int t = 0; t < ticks; ++t) {
            eng.step();
            n += eng.last_launches();
        }
    }
    if (launches) *launches = n;
}

}  // namespace

sbe_status sbe::set_error(sbe_status st, const char *msg) { return fail(st, msg); }

// ================================================================= misc
extern "C" int sbe_abi_version(void) { return SBE_ABI_VERSION; }
extern "C" const char *sbe_last_error_message(void) { return g_err.c_str(); }
extern "C" void sbe_opts_default(sbe_opts *o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->precision = -1;
}

// ================================================================= problem
static sbe_status problem_from_text(const std::string &text, sbe_problem **out)
{
    return guard([&]() -> sbe_status {
        if (!out) return fail(SBE_INVALID_ARGUMENT, "null output pointer");
        *out = nullptr;
        std::unique_ptr<CfgValue> root;
        try {
            root = parse_cfg(text);
        } catch (const CfgError &e) {
            return fail(SBE_BAD_CONFIG, std::string("Parse error at ") + e.what());
        }
        auto p = std::make_unique<sbe_problem>();
        p->p = problem_from_cfg(*root, &p->unsupported);
        *out = p.release();
        return SBE_OK;
    });
}

extern "C" sbe_status sbe_problem_from_cfg(const char *path, sbe_problem **out)
{
    if (!path) return fail(SBE_INVALID_ARGUMENT, "null path");
    std::ifstream f(path);
    if (!f) return fail(SBE_BAD_CONFIG, "I/O error while reading file.");  // antelope.cpp:95-99
    std::stringstream ss;
    ss << f.rdbuf();
    return problem_from_text(ss.str(), out);
}

extern "C" sbe_status sbe_problem_from_string(const char *text, sbe_problem **out)
{
    if (!text) return fail(SBE_INVALID_ARGUMENT, "null text");
    return problem_from_text(text, out);
}

extern "C" sbe_status sbe_problem_dims(const sbe_problem *p, sbe_dims *d)
{
    if (!p || !d) return fail(SBE_INVALID_ARGUMENT, "null argument");
    const Problem &q = p->p;
    std::memset(d, 0, sizeof(*d));
    d->Nt = q.laser.Nt;
    d->nband = q.nband;
    d->nval = q.nval;
    d->ntotal = q.ntotal();
    for (int i = 0; i < 3; ++i) d->Nk[i] = q.Nk[i];
    d->gauge = q.gauge;
    d->rk = q.rk;
    d->precision = q.precision;
    d->model = q.model;
    d->inter_intra = q.inter_intra ? 1 : 0;
    d->atmin = q.laser.atmin;
    d->dt = q.dt;
    d->dV = q.dV;
    d->total_weight = q.total_weight;
    return SBE_OK;
}

extern "C" sbe_status sbe_problem_laser(const sbe_problem *p, double *laser)
{
    if (!p || !laser) return fail(SBE_INVALID_ARGUMENT, "null argument");
    const std::vector<double> rows = laser_rows(p->p);
    std::copy(rows.begin(), rows.end(), laser);
    return SBE_OK;
}

extern "C" sbe_status sbe_problem_model(const sbe_problem *p, sbe_model *m)
{
    if (!p || !m) return fail(SBE_INVALID_ARGUMENT, "null argument");
    const Problem &q = p->p;
    if (q.model == MODEL_HALDANE) return fail(SBE_INVALID_ARGUMENT, "the Haldane model has no tables");
    if (q.model == MODEL_MULTIWSM) return fail(SBE_INVALID_ARGUMENT, "MultiWSM is a continuum model with no tables");
    m->nband = q.nband;
    m->nval = q.nval;
    m->nvec = q.w_nR;
    m->has_dipoles = q.w_d.empty() ? 0 : 1;
    m->has_current_tables = q.w_j.empty() ? 0 : 1;
    if (m->vec) std::copy(q.w_vec.begin(), q.w_vec.end(), m->vec);
    if (m->h) std::copy(q.w_h.begin(), q.w_h.end(), m->h);
    if (m->d && !q.w_d.empty()) std::copy(q.w_d.begin(), q.w_d.end(), m->d);
    if (m->j && !q.w_j.empty()) std::copy(q.w_j.begin(), q.w_j.end(), m->j);
    if (m->bz) std::copy(q.bz_model, q.bz_model + 9, m->bz);
    return SBE_OK;
}

extern "C" sbe_status sbe_problem_snapshots(const sbe_problem *p, int *interval, int *nshots, int *n0)
{
    if (!p) return fail(SBE_INVALID_ARGUMENT, "null problem");
    if (interval) *interval = p->p.shot_every();
    if (nshots) *nshots = p->p.nshots();
    if (n0) *n0 = p->p.Nk[0];
    return SBE_OK;
}

extern "C" void sbe_problem_destroy(sbe_problem *p) { delete p; }

// ================================================================= solver
struct sbe_solver {
    Problem prob;
    std::vector<double> laser;          // output laser columns, built while the GPU runs
    std::unique_ptr<Engine> eng;
    std::unique_ptr<WannierSolve> wan;  // N-band Wannier problems
    cudaStream_t own = nullptr;
    cudaEvent_t ready = nullptr;
    int id = -1;
    bool use_graph = false;
    bool ran = false;
    int launches = 0;
    int device = 0;
    long long nt = 0;  // fixed-step solves: steps taken
};

namespace {
sbe_status create_solver(const sbe_problem *p, const sbe_opts *opts, int kb, int ke, sbe_solver **out)
{
    if (sbe_status st = check_problem(p)) return st;
    if (!out) return fail(SBE_INVALID_ARGUMENT, "null output pointer");
    *out = nullptr;
    return guard([&]() -> sbe_status {
        auto s = std::make_unique<sbe_solver>();
        s->prob = p->p;
        s->device = opts ? opts->device : 0;
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        cuda_check(cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking), "stream create");
        cuda_check(cudaEventCreateWithFlags(&s->ready, cudaEventDisableTiming), "event create");
        if (p->p.model != MODEL_HALDANE) {
            const int prec = (opts && opts->precision >= 0) ? opts->precision : p->p.precision;
            s->wan = std::make_unique<WannierSolve>(p->p, prec, s->device, s->own, kb, ke);
        } else {
            s->eng = std::make_unique<Engine>(s->device, s->own, default_steps(opts));
            EngineOptions eo = to_engine_opts(opts);
            eo.k_begin = kb;
            eo.k_end = ke;
            s->id = s->eng->add(p->p, eo);
            s->nt = p->p.laser.Nt;  // antelope.cpp:297-338: one step per output time
            s->use_graph = opts && opts->use_graph && !opts->profile;
            s->eng->set_profile(opts && opts->profile);
        }
        cuda_check(cudaEventRecord(s->ready, s->own), "event record");
        *out = s.release();
        return SBE_OK;
    });
}
}  // namespace

extern "C" sbe_status sbe_solver_create(const sbe_problem *p, const sbe_opts *opts, sbe_solver **out)
{
    return create_solver(p, opts, 0, 0, out);
}

extern "C" sbe_status sbe_solver_create_slice(const sbe_problem *p, const sbe_opts *opts, int k_begin, int k_end,
                                              sbe_solver **out)
{
    if (p && (k_begin < 0 || k_end > p->p.ntotal() || k_begin >= k_end))
        return fail(SBE_INVALID_ARGUMENT, "k-slice outside the grid");
    return create_solver(p, opts, k_begin, k_end, out);
}

extern "C" int sbe_sums_width(const sbe_problem *p)
{
    if (!p) return 0;
    return p->p.model == MODEL_HALDANE ? NSLOT : WAN_NSLOT;
}

extern "C" sbe_status sbe_solver_sums(sbe_solver *s, double *sums)
{
    if (!s || !sums) return fail(SBE_INVALID_ARGUMENT, "null argument");
    if (!s->ran) return fail(SBE_NOT_READY, "sbe_solver_run has not been called");
    return guard([&]() -> sbe_status {
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        if (s->wan) {
            const std::vector<double> j = s->wan->sums();
            std::copy(j.begin(), j.end(), sums);
            const int Nt = (int)(j.size() / WAN_NSLOT);
            std::fill(sums + (size_t)Nt * WAN_NSLOT, sums + (size_t)(Nt + 1) * WAN_NSLOT, 0.0);
        } else {
            std::vector<double> j;
            double cp[NSLOT];
            s->eng->raw_outputs(s->id, j, cp);
            std::copy(j.begin(), j.end(), sums);
            std::copy(cp, cp + NSLOT, sums + j.size());
        }
        return SBE_OK;
    });
}

extern "C" sbe_status sbe_assemble(const sbe_problem *p, const double *sums, const sbe_outputs *out)
{
    if (sbe_status st = check_problem(p)) return st;
    if (!sums || !out) return fail(SBE_INVALID_ARGUMENT, "null argument");
    return guard([&]() -> sbe_status {
        const Problem &q = p->p;
        const int Nt = q.laser.Nt;
        SolveOutputs o;
        if (q.model == MODEL_HALDANE) {
            std::vector<double> j(sums, sums + (size_t)Nt * NSLOT);
            assemble_outputs(q, j, sums + (size_t)Nt * NSLOT, o);
        } else {
            std::vector<double> j(sums, sums + (size_t)Nt * WAN_NSLOT);
            assemble_table_outputs(q, j, o);
        }
        copy_out(o, out);
        return SBE_OK;
    });
}

extern "C" sbe_status sbe_solver_run(sbe_solver *s, void *stream)
{
    if (!s) return fail(SBE_INVALID_ARGUMENT, "null solver");
    if (s->ran) return fail(SBE_INVALID_ARGUMENT, "a solver runs once; create a new one");
    return guard([&]() -> sbe_status {
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->own;
        cuda_check(cudaStreamWaitEvent(st, s->ready, 0), "stream wait");
        if (s->wan) {
            s->wan->run(st);
            s->launches = s->wan->launches();
            s->ran = true;
            return SBE_OK;
        }
        s->eng->set_stream(st);
        run_engine(*s->eng, s->use_graph, &s->launches);
        s->eng->fetch_async(s->id);
        s->ran = true;
        // host work of sbe_solver_get done while the GPU propagates
        s->laser = laser_rows(s->prob);
        return SBE_OK;
    });
}

extern "C" sbe_status sbe_solver_get(sbe_solver *s, const sbe_outputs *out)
{
    if (!s) return fail(SBE_INVALID_ARGUMENT, "null solver");
    if (!s->ran) return fail(SBE_NOT_READY, "sbe_solver_run has not been called");
    return guard([&]() -> sbe_status {
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        SolveOutputs o = s->wan ? s->wan->outputs() : s->eng->outputs(s->id, &s->laser);
        copy_out(o, out);
        return SBE_OK;
    });
}

extern "C" int sbe_solver_launches(const sbe_solver *s) { return s ? s->launches : 0; }

extern "C" sbe_status sbe_solver_steps(const sbe_solver *s, long long *steps, long long *attempts,
                                       long long *rejects)
{
    if (!s) return fail(SBE_INVALID_ARGUMENT, "null solver");
    if (!s->ran) return fail(SBE_NOT_READY, "sbe_solver_run has not been called");
    long long st = 0, at = 0, rj = 0;
    if (s->wan) {
        const WanCtl &c = s->wan->control();
        st = c.steps;
        at = c.attempts;
        rj = c.rejects;
    } else {
        st = at = s->nt;
    }
    if (steps) *steps = st;
    if (attempts) *attempts = at;
    if (rejects) *rejects = rj;
    return SBE_OK;
}

extern "C" sbe_status sbe_solver_kernel_times(sbe_solver *s, double *pms, int *pn, double *rms, int *rn)
{
    if (!s) return fail(SBE_INVALID_ARGUMENT, "null solver");
    return guard([&]() -> sbe_status {
        if (!s->eng) {
            if (pms) *pms = 0;
            if (pn) *pn = 0;
            if (rms) *rms = 0;
            if (rn) *rn = 0;
            return SBE_OK;
        }
        s->eng->kernel_times(pms, pn, rms, rn);
        return SBE_OK;
    });
}

extern "C" sbe_status sbe_solver_snapshots(sbe_solver *s, double *occ1d, double *nc, double *pi)
{
    if (!s) return fail(SBE_INVALID_ARGUMENT, "null solver");
    if (!s->ran) return fail(SBE_NOT_READY, "sbe_solver_run has not been called");
    return guard([&]() -> sbe_status {
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        const int n = s->wan ? s->wan->snapshots(occ1d, nc, pi) : s->eng->snapshots(s->id, occ1d, nc, pi);
        if (n == 0)
            return fail(SBE_INVALID_ARGUMENT, "the problem takes no snapshots (calc.shotNumber <= 0)");
        return SBE_OK;
    });
}

extern "C" sbe_status sbe_solver_harmonics(sbe_solver *s, double w0, int hmax, double *band_power)
{
    if (!s || !band_power) return fail(SBE_INVALID_ARGUMENT, "null argument");
    if (!s->ran) return fail(SBE_NOT_READY, "sbe_solver_run has not been called");
    return guard([&]() -> sbe_status {
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        if (s->wan) s->wan->harmonics(w0, hmax, band_power);
        else s->eng->harmonics(s->id, w0, hmax, band_power);
        return SBE_OK;
    });
}

extern "C" void sbe_solver_destroy(sbe_solver *s)
{
    if (!s) return;
    cudaSetDevice(s->device);
    s->eng.reset();
    s->wan.reset();
    if (s->ready) cudaEventDestroy(s->ready);
    if (s->own) {
        cudaStreamSynchronize(s->own);
        cudaStreamDestroy(s->own);
    }
    delete s;
}

// ================================================================= files
extern "C" sbe_status sbe_write_outputs(const sbe_problem *p, const sbe_outputs *o, const char *dir)
{
    if (!p || !o || !o->inter || !o->intra || !o->occ || !o->coh || !o->laser)
        return fail(SBE_INVALID_ARGUMENT, "all five output arrays are needed to write the files");
    return guard([&]() -> sbe_status {
        const Problem &q = p->p;
        SolveOutputs so;
        so.Nt = q.laser.Nt;
        so.nband = q.nband;
        const size_t Nt = (size_t)so.Nt, N = (size_t)so.nband;
        so.inter.assign(o->inter, o->inter + Nt * 3);
        so.intra.assign(o->intra, o->intra + Nt * 3);
        so.occ.assign(o->occ, o->occ + Nt * (N + 1));
        so.coh.assign(o->coh, o->coh + Nt * 2);
        so.laser.assign(o->laser, o->laser + Nt * 7);
        write_outputs(q, so, dir ? dir : "");
        return SBE_OK;
    });
}

// The snapshot files of antelope.cpp:288-292, 365-368, 416-421:
// occupation_1d_integration.dat rows of "%16e    " values, the binary
// fisrt_conduction.dat (doubles) and fisrt_coherence.dat (complex doubles),
// and snapshot_log.dat, which the reference opens and never writes.
extern "C" sbe_status sbe_write_snapshots(const sbe_problem *p, const double *occ1d, const double *nc,
                                          const double *pi, const char *dir)
{
    if (!p || !occ1d || !nc || !pi) return fail(SBE_INVALID_ARGUMENT, "all three snapshot arrays are needed");
    const Problem &q = p->p;
    const int ns = q.nshots();
    if (ns == 0) return fail(SBE_INVALID_ARGUMENT, "the problem takes no snapshots (calc.shotNumber <= 0)");
    const std::string d = (dir && *dir) ? std::string(dir) + "/" : std::string();
    FILE *f1 = fopen((d + "occupation_1d_integration.dat").c_str(), "w");
    FILE *f2 = fopen((d + "fisrt_conduction.dat").c_str(), "w");
    FILE *f3 = fopen((d + "fisrt_coherence.dat").c_str(), "w");
    FILE *f4 = fopen((d + "snapshot_log.dat").c_str(), "w");
    const bool ok = f1 && f2 && f3 && f4;
    if (ok) {
        const size_t nt = (size_t)q.ntotal();
        for (int k = 0; k < ns; ++k) {
            for (int m = 0; m < q.Nk[0]; ++m) fprintf(f1, "%16e    ", occ1d[(size_t)k * q.Nk[0] + m]);
            fprintf(f1, "\n");
            fwrite(nc + (size_t)k * nt, sizeof(double), nt, f2);
            fwrite(pi + (size_t)k * nt * 2, sizeof(double), nt * 2, f3);
        }
    }
    for (FILE *f : {f1, f2, f3, f4})
        if (f) fclose(f);
    return ok ? SBE_OK : fail(SBE_INVALID_ARGUMENT, "cannot open the snapshot files in " + d);
}

extern "C" sbe_status sbe_run_cfg(const char *cfg_path, const char *out_dir, const sbe_opts *opts)
{
    sbe_problem *p = nullptr;
    if (sbe_status st = sbe_problem_from_cfg(cfg_path, &p)) return st;
    std::unique_ptr<sbe_problem> hold(p);
    sbe_solver *s = nullptr;
    if (sbe_status st = sbe_solver_create(p, opts, &s)) return st;
    std::unique_ptr<sbe_solver, void (*)(sbe_solver *)> sh(s, sbe_solver_destroy);
    if (sbe_status st = sbe_solver_run(s, s->own)) return st;
    const Problem &q = p->p;
    const size_t Nt = q.laser.Nt, N = q.nband;
    std::vector<double> inter(Nt * 3), intra(Nt * 3), occ(Nt * (N + 1)), coh(Nt * 2), laser(Nt * 7);
    sbe_outputs o{inter.data(), intra.data(), occ.data(), coh.data(), laser.data()};
    if (sbe_status st = sbe_solver_get(s, &o)) return st;
    if (sbe_status st = sbe_write_outputs(p, &o, out_dir)) return st;
    if (q.nshots() > 0) {   // density snapshots (antelope.cpp:267-422)
        const size_t ns = q.nshots(), nt = q.ntotal();
        std::vector<double> occ1d(ns * q.Nk[0]), nc(ns * nt), pi(ns * nt * 2);
        if (sbe_status st = sbe_solver_snapshots(s, occ1d.data(), nc.data(), pi.data())) return st;
        return sbe_write_snapshots(p, occ1d.data(), nc.data(), pi.data(), out_dir);
    }
    return SBE_OK;
}

// ================================================================= batch
// Two-band Haldane problems go to the engine (closed-form kernels, one launch
// per launch class per step chunk); table and continuum models to a
// WannierBatch (N-band kernels, one attempt and one control launch per launch
// class per iteration).  A batch may hold both; they run one after the other
// on the batch's stream.
struct sbe_batch {
    std::unique_ptr<Engine> eng;
    std::unique_ptr<WannierBatch> wan;
    cudaStream_t own = nullptr;
    cudaEvent_t ready = nullptr;
    std::vector<int> ids;        // engine solve id, or -1 - (index in the Wannier batch)
    std::vector<long long> nt;   // output steps of each solve
    bool use_graph = false, ran = false;
    int launches = 0, device = 0;
};

extern "C" sbe_status sbe_batch_create(const sbe_problem *const *problems, int n, const sbe_opts *opts,
                                       sbe_batch **out)
{
    if (!problems || n <= 0 || !out) return fail(SBE_INVALID_ARGUMENT, "need at least one problem");
    *out = nullptr;
    for (int i = 0; i < n; ++i)
        if (sbe_status st = check_problem(problems[i])) return st;
    return guard([&]() -> sbe_status {
        auto b = std::make_unique<sbe_batch>();
        b->device = opts ? opts->device : 0;
        cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
        cuda_check(cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking), "stream create");
        cuda_check(cudaEventCreateWithFlags(&b->ready, cudaEventDisableTiming), "event create");
        b->ids.assign(n, -1);
        for (int i = 0; i < n; ++i) b->nt.push_back(problems[i]->p.laser.Nt);
        std::vector<int> order, wan_order;
        for (int i = 0; i < n; ++i) (problems[i]->p.model == MODEL_HALDANE ? order : wan_order).push_back(i);
        if (!order.empty()) {
            b->eng = std::make_unique<Engine>(b->device, b->own, default_steps(opts));
            // longest solves first: their tiles lead every launch's tile list
            std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
                return (double)problems[a]->p.laser.Nt * problems[a]->p.ntotal() >
                       (double)problems[c]->p.laser.Nt * problems[c]->p.ntotal();
            });
            EngineOptions eo = to_engine_opts(opts);
            for (int i : order) b->ids[i] = b->eng->add(problems[i]->p, eo);
            b->eng->set_profile(opts && opts->profile);
        }
        if (!wan_order.empty()) {
            std::vector<const Problem *> probs;
            for (int j = 0; j < (int)wan_order.size(); ++j) {
                probs.push_back(&problems[wan_order[j]]->p);
                b->ids[wan_order[j]] = -1 - j;
            }
            const int prec = opts ? opts->precision : -1;
            b->wan = std::make_unique<WannierBatch>(probs, prec, b->device, b->own);
        }
        cuda_check(cudaEventRecord(b->ready, b->own), "event record");
        b->use_graph = opts && opts->use_graph && !opts->profile;
        *out = b.release();
        return SBE_OK;
    });
}

extern "C" sbe_status sbe_batch_run(sbe_batch *b, void *stream)
{
    if (!b) return fail(SBE_INVALID_ARGUMENT, "null batch");
    if (b->ran) return fail(SBE_INVALID_ARGUMENT, "a batch runs once; create a new one");
    return guard([&]() -> sbe_status {
        cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->own;
        cuda_check(cudaStreamWaitEvent(st, b->ready, 0), "stream wait");
        b->launches = 0;
        if (b->eng) {
            b->eng->set_stream(st);
            run_engine(*b->eng, b->use_graph, &b->launches);
            for (int id : b->ids)
                if (id >= 0) b->eng->fetch_async(id);
        }
        if (b->wan) {
            b->wan->run(st, b->use_graph);
            b->launches += b->wan->launches();
        }
        b->ran = true;
        return SBE_OK;
    });
}

extern "C" sbe_status sbe_batch_get(sbe_batch *b, int index, const sbe_outputs *out)
{
    if (!b || index < 0 || index >= (int)b->ids.size()) return fail(SBE_INVALID_ARGUMENT, "bad batch index");
    if (!b->ran) return fail(SBE_NOT_READY, "sbe_batch_run has not been called");
    return guard([&]() -> sbe_status {
        cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
        const int id = b->ids[index];
        copy_out(id >= 0 ? b->eng->outputs(id) : b->wan->solve(-1 - id).outputs(), out);
        return SBE_OK;
    });
}

extern "C" sbe_status sbe_batch_steps(sbe_batch *b, int index, long long *steps, long long *attempts,
                                      long long *rejects)
{
    if (!b || index < 0 || index >= (int)b->ids.size()) return fail(SBE_INVALID_ARGUMENT, "bad batch index");
    if (!b->ran) return fail(SBE_NOT_READY, "sbe_batch_run has not been called");
    const int id = b->ids[index];
    long long st = 0, at = 0, rj = 0;
    if (id < 0) {
        const WanCtl &c = b->wan->solve(-1 - id).control();
        st = c.steps;
        at = c.attempts;
        rj = c.rejects;
    } else {
        st = at = b->nt[index];   // fixed step: one step per output time
    }
    if (steps) *steps = st;
    if (attempts) *attempts = at;
    if (rejects) *rejects = rj;
    return SBE_OK;
}

extern "C" sbe_status sbe_batch_harmonics(sbe_batch *b, int index, double w0, int hmax, double *band_power)
{
    if (!b || index < 0 || index >= (int)b->ids.size() || !band_power)
        return fail(SBE_INVALID_ARGUMENT, "bad batch index or null output");
    if (!b->ran) return fail(SBE_NOT_READY, "sbe_batch_run has not been called");
    return guard([&]() -> sbe_status {
        cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
        const int id = b->ids[index];
        if (id >= 0) b->eng->harmonics(id, w0, hmax, band_power);
        else b->wan->solve(-1 - id).harmonics(w0, hmax, band_power);
        return SBE_OK;
    });
}

extern "C" sbe_status sbe_batch_snapshots(sbe_batch *b, int index, double *occ1d, double *nc, double *pi)
{
    if (!b || index < 0 || index >= (int)b->ids.size()) return fail(SBE_INVALID_ARGUMENT, "bad batch index");
    if (!b->ran) return fail(SBE_NOT_READY, "sbe_batch_run has not been called");
    return guard([&]() -> sbe_status {
        cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
        const int id = b->ids[index];
        const int n = id >= 0 ? b->eng->snapshots(id, occ1d, nc, pi) : b->wan->solve(-1 - id).snapshots(occ1d, nc, pi);
        if (n == 0)
            return fail(SBE_INVALID_ARGUMENT, "the problem takes no snapshots (calc.shotNumber <= 0)");
        return SBE_OK;
    });
}

extern "C" int sbe_batch_launches(const sbe_batch *b) { return b ? b->launches : 0; }

extern "C" sbe_status sbe_batch_kernel_times(sbe_batch *b, double *pms, int *pn, double *rms, int *rn)
{
    if (!b) return fail(SBE_INVALID_ARGUMENT, "null batch");
    return guard([&]() -> sbe_status {
        if (pms) *pms = 0;
        if (pn) *pn = 0;
        if (rms) *rms = 0;
        if (rn) *rn = 0;
        if (b->eng) b->eng->kernel_times(pms, pn, rms, rn);
        return SBE_OK;
    });
}

extern "C" void sbe_batch_destroy(sbe_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    b->eng.reset();
    b->wan.reset();
    if (b->ready) cudaEventDestroy(b->ready);
    if (b->own) {
        cudaStreamSynchronize(b->own);
        cudaStreamDestroy(b->own);
    }
    delete b;
}

// ================================================================= server
namespace {
using Clock = std::chrono::steady_clock;

struct Request {
    long long id = 0;
    Problem prob;
    std::vector<double> laser;    // laser columns of the outputs, built by the submitting thread
    std::vector<double> jout;     // raw per-step sums, assembled by the waiting thread
    double cp[NSLOT] = {0};
    Clock::time_point t_submit, t_done;
    // ADMITTING: taken off the queue, being set up by the worker outside the lock
    enum State { QUEUED, ADMITTING, RESIDENT, DONE, FAILED, CANCELLED } state = QUEUED;
    int solve = -1;               // engine solve id while the engine holds it
    bool nband = false;           // a table or continuum model: held by the N-band pool
    int wsolve = -1;              // its pool id
    bool fetching = false;
    bool cancel_asked = false;    // cancelled while ADMITTING
    bool delivered = false;       // a wait returned its final state: the worker may erase it
    SolveOutputs out;
    std::string err;
};
}  // namespace

struct sbe_server {
    sbe_server_opts opts{};
    std::unique_ptr<Engine> eng;
    std::unique_ptr<WannierPool> wpool;   // N-band requests
    cudaStream_t stream = nullptr;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    long long next_id = 1;
    std::deque<long long> queue;
    std::unordered_map<long long, std::unique_ptr<Request>> reqs;
    long long n_submitted = 0, n_completed = 0, n_failed = 0, n_launches = 0;
    double budget = 0;
    std::string fatal;
    std::deque<cudaEvent_t> inflight;  // one event per issued tick (bounded run-ahead)

    void loop();
};

void sbe_server::loop()
{
    cudaSetDevice(opts.device);
    EngineOptions eo;
    eo.precision = opts.precision;
    eo.tile_k = opts.tile_k;
    eo.kpt = opts.k_per_thread;
    eo.allow_tuning = false;  // never stall the serving loop on a tuning run
    eo.throughput_shape = true;  // resident solves share the GPU: full CTAs unless a tuned shape is cached
    eo.snapshots = false;     // requests return the file outputs only (sbe_server_wait)
    // admissions set up between two tick issues: a burst of arrivals is
    // admitted in slices while the GPU keeps working on the queued ticks
    constexpr size_t kAdmitPerTurn = 16;
    constexpr int kPoolIters = 32;   // N-band attempted steps per tick
    auto nband_precision = [&](const Problem &p) { return opts.precision >= 0 ? opts.precision : p.precision; };
    wpool = std::make_unique<WannierPool>(opts.device, stream);
    std::vector<cudaEvent_t> pool;
    std::vector<Request *> batch;
    for (;;) {
        batch.clear();
        {
            std::unique_lock<std::mutex> lk(mu);
            // admission: FIFO while memory and slots allow
            size_t planned = 0;
            while (!queue.empty() && batch.size() < kAdmitPerTurn) {
                auto it = reqs.find(queue.front());
                if (it == reqs.end() || it->second->state != Request::QUEUED) {
                    queue.pop_front();
                    continue;
                }
                Request &r = *it->second;
                size_t need = 0;
                try {
                    need = r.nband ? WannierPool::bytes_needed(r.prob, nband_precision(r.prob))
                                   : eng->bytes_needed(r.prob, eo);
                } catch (const std::exception &e) {
                    r.state = Request::FAILED;
                    r.err = e.what();
                    ++n_failed;
                    queue.pop_front();
                    cv_done.notify_all();
                    continue;
                }
                const int resident = eng->nresident() + wpool->nresident() + (int)batch.size();
                const bool slots_ok = opts.max_resident <= 0 || resident < opts.max_resident;
                if (!slots_ok || (double)(eng->bytes_in_use() + wpool->bytes_in_use() + planned + need) > budget) {
                    if (resident == 0) {  // can never fit
                        r.state = Request::FAILED;
                        r.err = "admission refused: request needs more device memory than the budget";
                        ++n_failed;
                        queue.pop_front();
                        cv_done.notify_all();
                        continue;
                    }
                    break;
                }
                r.state = Request::ADMITTING;
                planned += need;
                batch.push_back(&r);
                queue.pop_front();
            }
            if (batch.empty() && eng->nresident() == 0 && wpool->nresident() == 0) {
                if (stop) break;
                cv_work.wait_for(lk, std::chrono::milliseconds(50));
                continue;
            }
        }
        // set the admitted solves up outside the lock, so that submitting
        // and waiting threads are not held up by it
        for (Request *r : batch) {
            try {
                if (r->nband) r->wsolve = wpool->add(r->prob, nband_precision(r->prob));
                else r->solve = eng->add(r->prob, eo);
            } catch (const std::exception &e) {
                r->solve = r->wsolve = -1;
                r->err = e.what();
            }
        }
        if (!batch.empty()) {
            std::lock_guard<std::mutex> g(mu);
            for (Request *r : batch) {
                if ((r->nband ? r->wsolve : r->solve) < 0) {
                    r->state = Request::FAILED;
                    ++n_failed;
                } else {
                    r->state = r->cancel_asked ? Request::CANCELLED : Request::RESIDENT;
                }
            }
            cv_done.notify_all();
        }
        try {
            // bounded run-ahead: at most two ticks queued on the GPU, so new
            // arrivals join after a short wait
            while (inflight.size() >= 2) {
                cuda_check(cudaEventSynchronize(inflight.front()), "tick wait");
                pool.push_back(inflight.front());
                inflight.pop_front();
            }
            const bool eng_work = eng->max_remaining_ticks() > 0, pool_work = wpool->nrunning() > 0;
            if (eng_work) eng->step();
            // the N-band solves advance a few attempted steps per tick
            if (pool_work) wpool->step(kPoolIters);
            if (eng_work || pool_work) {
                cudaEvent_t ev;
                if (pool.empty()) cuda_check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
                else { ev = pool.back(); pool.pop_back(); }
                cuda_check(cudaEventRecord(ev, stream), "event record");
                inflight.push_back(ev);
            }
        } catch (const std::exception &e) {
            std::lock_guard<std::mutex> g(mu);
            fatal = e.what();
            for (auto &kv : reqs)
                if (kv.second->state == Request::RESIDENT || kv.second->state == Request::QUEUED) {
                    kv.second->state = Request::FAILED;
                    kv.second->err = fatal;
                }
            cv_done.notify_all();
            break;
        }
        try {
            wpool->poll();
        } catch (const std::exception &e) {
            std::lock_guard<std::mutex> g(mu);
            fatal = e.what();
            cv_done.notify_all();
            break;
        }
        std::lock_guard<std::mutex> g(mu);
        n_launches += eng->last_launches() + wpool->last_launches();
        // retire finished and cancelled solves; forget requests whose final
        // state a wait has returned
        for (auto it = reqs.begin(); it != reqs.end();) {
            Request &r = *it->second;
            if (r.state == Request::CANCELLED && r.solve >= 0) {
                try {
                    eng->remove(r.solve);
                } catch (...) {
                }
                r.solve = -1;
            }
            if (r.state == Request::CANCELLED && r.wsolve >= 0) {
                try {
                    wpool->remove(r.wsolve);
                } catch (...) {
                }
                r.wsolve = -1;
            }
            const bool final_state = r.state == Request::DONE || r.state == Request::FAILED ||
                                     r.state == Request::CANCELLED;
            if (final_state && r.delivered && r.solve < 0 && r.wsolve < 0) {
                it = reqs.erase(it);
                continue;
            }
            if (r.state == Request::RESIDENT && r.nband && wpool->finished(r.wsolve)) {
                try {
                    if (wpool->failed(r.wsolve)) {
                        r.state = Request::FAILED;
                        r.err = "Cash-Karp step size underflow: tolerance unreachable";
                        ++n_failed;
                    } else {
                        r.jout = wpool->sums(r.wsolve);
                        r.t_done = Clock::now();
                        r.state = Request::DONE;
                        ++n_completed;
                    }
                    wpool->remove(r.wsolve);
                    r.wsolve = -1;
                } catch (const std::exception &e) {
                    r.state = Request::FAILED;
                    r.err = e.what();
                    ++n_failed;
                }
                cv_done.notify_all();
            }
            if (r.state == Request::RESIDENT && !r.nband && eng->finished(r.solve)) {
                try {
                    if (!r.fetching) { eng->fetch_async(r.solve); r.fetching = true; }
                    if (eng->ready(r.solve)) {
                        eng->raw_outputs(r.solve, r.jout, r.cp);
                        eng->remove(r.solve);
                        r.solve = -1;
                        r.t_done = Clock::now();
                        r.state = Request::DONE;
                        ++n_completed;
                        cv_done.notify_all();
                    }
                } catch (const std::exception &e) {
                    r.state = Request::FAILED;
                    r.err = e.what();
                    ++n_failed;
                    cv_done.notify_all();
                }
            }
            ++it;
        }
    }
    for (auto ev : inflight) cudaEventDestroy(ev);
    for (auto ev : pool) cudaEventDestroy(ev);
}

extern "C" sbe_status sbe_server_create(const sbe_server_opts *opts, sbe_server **out)
{
    if (!out) return fail(SBE_INVALID_ARGUMENT, "null output pointer");
    *out = nullptr;
    return guard([&]() -> sbe_status {
        auto s = std::make_unique<sbe_server>();
        if (opts) s->opts = *opts;
        else s->opts.precision = -1;
        cuda_check(cudaSetDevice(s->opts.device), "cudaSetDevice");
        cuda_check(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream create");
        const int S = s->opts.steps_per_launch > 0 ? s->opts.steps_per_launch : 256;
        s->eng = std::make_unique<Engine>(s->opts.device, s->stream, S);
        size_t fr = 0, tot = 0;
        cuda_check(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo");
        s->budget = s->opts.mem_budget_bytes > 0 ? s->opts.mem_budget_bytes
                                                 : std::max(0.0, (double)fr - 4.0 * (1ull << 30));
        sbe_server *raw = s.get();
        s->worker = std::thread([raw]() { raw->loop(); });
        *out = s.release();
        return SBE_OK;
    });
}

extern "C" sbe_status sbe_server_submit(sbe_server *s, const sbe_problem *p, long long *request_id)
{
    if (!s) return fail(SBE_INVALID_ARGUMENT, "null server");
    if (sbe_status st = check_problem(p)) return st;
    auto r = std::make_unique<Request>();
    r->t_submit = Clock::now();
    r->prob = p->p;
    r->nband = p->p.model != MODEL_HALDANE;
    try {
        // the laser output columns, built on the caller's thread
        r->laser = laser_rows(r->prob);
    } catch (const std::exception &e) {
        return fail(SBE_INVALID_ARGUMENT, e.what());
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->fatal.empty()) return fail(SBE_CUDA_ERROR, s->fatal);
    r->id = s->next_id++;
    if (request_id) *request_id = r->id;
    s->queue.push_back(r->id);
    s->reqs[r->id] = std::move(r);
    ++s->n_submitted;
    s->cv_work.notify_all();
    return SBE_OK;
}

extern "C" sbe_status sbe_server_wait(sbe_server *s, long long id, double timeout_s, const sbe_outputs *out,
                                      double *latency_s)
{
    if (!s) return fail(SBE_INVALID_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(SBE_INVALID_ARGUMENT, "unknown request id");
    Request &r = *it->second;
    auto pending = [&]() {
        return r.state == Request::QUEUED || r.state == Request::ADMITTING || r.state == Request::RESIDENT;
    };
    if (timeout_s < 0) s->cv_done.wait(lk, [&]() { return !pending(); });
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&]() { return !pending(); }))
        return fail(SBE_TIMEOUT, "request not finished within the timeout");
    r.delivered = true;   // the worker forgets the request from now on
    if (r.state == Request::CANCELLED) return fail(SBE_CANCELLED, "request was cancelled");
    if (r.state == Request::FAILED) {
        const bool oom = r.err.find("memory") != std::string::npos;
        return fail(oom ? SBE_OOM : SBE_CUDA_ERROR, r.err);
    }
    if (latency_s) *latency_s = std::chrono::duration<double>(r.t_done - r.t_submit).count();
    if (out) {
        // assemble on the waiting thread, outside the lock
        std::vector<double> j = std::move(r.jout), laser = std::move(r.laser);
        double cp[NSLOT];
        for (int q = 0; q < NSLOT; ++q) cp[q] = r.cp[q];
        Problem prob = r.prob;
        const bool nband = r.nband;
        lk.unlock();
        return guard([&]() -> sbe_status {
            SolveOutputs o;
            if (nband) assemble_table_outputs(prob, j, o);
            else assemble_outputs(prob, j, cp, o, &laser);
            copy_out(o, out);
            return SBE_OK;
        });
    }
    return SBE_OK;
}

extern "C" sbe_status sbe_server_cancel(sbe_server *s, long long id)
{
    if (!s) return fail(SBE_INVALID_ARGUMENT, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(SBE_INVALID_ARGUMENT, "unknown request id");
    Request &r = *it->second;
    if (r.state == Request::QUEUED) {
        r.state = Request::CANCELLED;
    } else if (r.state == Request::ADMITTING) {
        r.cancel_asked = true;   // the worker cancels it once its set-up returns
    } else if (r.state == Request::RESIDENT) {
        r.state = Request::CANCELLED;  // the worker, which owns the engine, drops the solve
        s->cv_work.notify_all();
    }
    s->cv_done.notify_all();
    return SBE_OK;
}

extern "C" sbe_status sbe_server_stats(sbe_server *s, long long c[5])
{
    if (!s || !c) return fail(SBE_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    long long resident = 0;
    for (auto &kv : s->reqs) resident += kv.second->state == Request::RESIDENT;
    c[0] = s->n_submitted;
    c[1] = s->n_completed;
    c[2] = s->n_failed;
    c[3] = resident;
    c[4] = s->n_launches;
    return SBE_OK;
}

extern "C" void sbe_server_destroy(sbe_server *s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        for (auto &kv : s->reqs)
            if (kv.second->state == Request::QUEUED) kv.second->state = Request::CANCELLED;
        s->queue.clear();
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->opts.device);
    s->wpool.reset();
    s->eng.reset();
    if (s->stream) {
        cudaStreamSynchronize(s->stream);
        cudaStreamDestroy(s->stream);
    }
    delete s;
}

// ================================================================= peaks
extern "C" sbe_status sbe_measure_fma_peaks(int device, double *fp64, double *fp32, double *fp32x2)
{
    return guard([&]() -> sbe_status {
        cuda_check(cudaSetDevice(device), "cudaSetDevice");
        int sms = 0;
        cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "attr");
        void *buf = nullptr;
        cuda_check(cudaMalloc(&buf, 4096), "cudaMalloc");
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        const int blocks = sms * 8, iters = 1 << 16;
        double res[3] = {0, 0, 0};
        for (int which = 0; which < 3; ++which) {
            cuda_check(launch_fma_peak(which, blocks, 256, buf, 0), "warm-up");
            float best = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {
                cudaEventRecord(a, 0);
                cuda_check(launch_fma_peak(which, blocks, iters, buf, 0), "fma peak");
                cudaEventRecord(b, 0);
                cuda_check(cudaEventSynchronize(b), "sync");
                float ms = 0;
                cudaEventElapsedTime(&ms, a, b);
                best = std::min(best, ms);
            }
            const double flops = (which == 2 ? 4.0 : 2.0) * 8.0 * iters * 256.0 * blocks;
            res[which] = flops / (best * 1e-3) / 1e12;
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        cudaFree(buf);
        if (fp64) *fp64 = res[0];
        if (fp32) *fp32 = res[1];
        if (fp32x2) *fp32x2 = res[2];
        return SBE_OK;
    });
}
