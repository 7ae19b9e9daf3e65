// The tile engine: owns device-resident solves and advances them launch by
// launch.  A single solve, a batched scan and the serving loop are all built
// on it (sbe_capi.cpp).
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "sbe_dev.h"
#include "sbe_problem.h"

namespace sbe {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct OomError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
void cuda_check(cudaError_t e, const char *what);

struct EngineOptions {
    int precision = -1;      // -1: take calc.precision from the problem
    int tile_k = 0;          // k-points per tile (0: tuned default)
    int kpt = 0;             // k-points per thread (0: tuned default)
    int steps_per_launch = 0;  // S (0: default)
    bool allow_tuning = true;  // false: a cached tuned shape or the heuristic, never a tuning run
    bool throughput_shape = false;  // heuristic: full 256-thread CTAs (many solves share the GPU)
    int k_begin = 0, k_end = 0;  // k-slice [k_begin, k_end) of the grid (0, 0: all of it)
    bool snapshots = true;       // take the problem's density snapshots (calc.shotNumber)
};

// Pinned staging for host->device uploads: copies are issued from a pinned
// ring (a pageable source would make cudaMemcpyAsync wait for the stream), and
// a region is reused only after the event recorded behind its copy.
class UploadRing {
public:
    explicit UploadRing(size_t bytes);
    ~UploadRing();
    void upload(void *dst, const void *src, size_t bytes, cudaStream_t st);
    static UploadRing &shared();  // one per process, shared by all engines

private:
    std::mutex mu_;
    struct Span {
        size_t lo, hi;
        cudaEvent_t ev;
    };
    char *base_ = nullptr;
    size_t cap_ = 0, head_ = 0;
    std::vector<Span> inflight_;
    std::vector<cudaEvent_t> spare_;
};

// Reusable pinned host buffers for device->host results (cudaMallocHost and
// cudaFreeHost are expensive and can synchronise the device).
class PinnedPool {
public:
    ~PinnedPool();
    void *get(size_t bytes);
    void put(void *p, size_t bytes);
    static PinnedPool &shared();  // one per process, shared by all engines

private:
    std::mutex mu_;
    static size_t size_class(size_t b);
    std::map<size_t, std::vector<void *>> free_;
};

// One launch shape for a class of solves.
struct Shape {
    int tile_k, kpt, threads;
};

// Outputs of a finished solve in the reference's file quantities.
struct SolveOutputs {
    int Nt = 0, nband = 0;
    std::vector<double> inter, intra;  // [Nt][3], times dV (antelope.cpp:522-527)
    std::vector<double> occ;           // [Nt][N+1], divided by Ntotal, last column the sum (530-536)
    std::vector<double> coh;           // [Nt][2] (539-542)
    std::vector<double> laser;         // [Nt][7]: t, E[3], A[3] (208-235)
};

class Engine {
public:
    Engine(int device, cudaStream_t stream, int steps_per_launch);
    ~Engine();
    Engine(const Engine &) = delete;
    Engine &operator=(const Engine &) = delete;

    // Device bytes a solve of this problem needs (admission control).
    size_t bytes_needed(const Problem &p, const EngineOptions &o) const;
    // Set up a solve (on the engine's copy stream); it starts advancing at the
    // next step().  Its field table is computed on the device.
    int add(const Problem &p, const EngineOptions &o);
    // Advance every resident solve by up to S steps (one propagate launch per
    // launch class, then the tile reduction).
    void step();
    // Same as step() but never rebuilds the launch lists (for CUDA graph
    // capture, where the lists built by the first step() stay valid: tiles of
    // solves that finished return at once).
    void step_frozen();
    void set_stream(cudaStream_t s) { stream_ = s; }
    // Ticks still needed by a solve (0 when finished).
    int remaining_ticks(int id) const;
    bool finished(int id) const { return remaining_ticks(id) == 0; }
    int max_remaining_ticks() const;
    // Queue the D2H copy of a finished solve's per-step sums into pinned
    // memory and record an event; ready() polls it, outputs() assembles.
    void fetch_async(int id);
    bool ready(int id);
    // `laser` may hold the problem's laser_rows() already built by the caller
    SolveOutputs outputs(int id, const std::vector<double> *laser = nullptr);
    // The raw per-step sums [Nt][NSLOT] and the summed constant parts of a
    // fetched solve (waits for the copy); assemble_outputs() turns them into
    // the output arrays.
    void raw_outputs(int id, std::vector<double> &jout, double cp[NSLOT]);
    // Density snapshots of a finished solve (waits for the stream):
    // occ1d[nshots][N0] (the 1-D integrated conduction occupation, summed over
    // this solve's k-points), nc[nshots][nk], pi[nshots][nk][2]; any may be
    // null.  Returns the number of snapshots (0: none were taken).
    int snapshots(int id, double *occ1d, double *nc, double *pi);
    // harmonic band powers h = 1..hmax of a finished solve, from its
    // device-resident sums (sbe_spectrum.h); synchronises the stream
    void harmonics(int id, double w0, int hmax, double *band_power);
    void remove(int id);
    int nresident() const { return (int)live_.size(); }
    int tick() const { return tick_; }
    int steps_per_launch() const { return S_; }
    cudaStream_t stream() const { return stream_; }
    size_t bytes_in_use() const { return bytes_in_use_; }
    // Number of propagate launches issued by the last step() (telemetry).
    int last_launches() const { return last_launches_; }
    // CUDA-event timing of every propagate / reduce launch (telemetry for the
    // roofline; off by default, not usable under graph capture).
    void set_profile(bool on) { profile_ = on; }
    void kernel_times(double *prop_ms, int *prop_n, double *red_ms, int *red_n);
    // Launch shape the engine would use for a solve.
    Shape shape_for(const Problem &p, const EngineOptions &o) const;

private:
    struct Solve;
    struct Group;
    void rebuild_lists();
    Solve &get(int id);
    const Solve &get(int id) const;

    // Admission work (allocations, uploads, per-k set-up) runs on its own
    // copy stream `up_` so it never waits behind queued ticks; the compute
    // stream waits on the events in `pending_` before it next touches solves.
    void drain_pending();
    int device_;
    cudaStream_t stream_;
    cudaStream_t up_ = nullptr;
    cudaMemPool_t pool_ = nullptr;
    std::vector<cudaEvent_t> pending_, spare_ev_;
    int S_;
    int tick_ = 0;
    int next_id_ = 0;
    int capacity_ = 0;
    bool dirty_ = true;
    int last_launches_ = 0;
    bool profile_ = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prop_ev_, red_ev_;
    std::pair<cudaEvent_t, cudaEvent_t> new_pair();
    size_t bytes_in_use_ = 0;
    std::map<int, std::unique_ptr<Solve>> live_;
    std::vector<int> free_slots_;
    SolveDev *d_solves_ = nullptr;
    SolveDev *h_solves_ = nullptr;   // host mirror of the descriptors
    int *d_ids_ = nullptr;
    std::vector<int> h_ids_;
    UploadRing &ring_ = UploadRing::shared();
    PinnedPool &pinned_ = PinnedPool::shared();
    int nids_ = 0;
    int status_dummy_ = 0;
    std::map<std::tuple<int, int, int, int, int, int>, std::unique_ptr<Group>> groups_;
};

// Autotuner (sbe_tune.cpp): the fastest launch shape for this class of solve.
bool autotune_enabled();
Shape autotune_shape(int device, const Problem &p, int precision);
// Cached tuned shape only (no tuning run); false when none is cached.
bool autotune_lookup(int device, const Problem &p, int precision, Shape *out);

// Assemble the reference's output quantities from the per-step slot sums;
// `laser` may hold the problem's laser_rows() already built by the caller.
void assemble_outputs(const Problem &p, const std::vector<double> &jout, const double constpart[NSLOT],
                      SolveOutputs &out, const std::vector<double> *laser = nullptr);

// Write the reference's output files into `dir` (antelope.cpp:176-184,
// 208-235, 514-548), byte-for-byte in its formats.
void write_outputs(const Problem &p, const SolveOutputs &o, const std::string &dir);

}  // namespace sbe
