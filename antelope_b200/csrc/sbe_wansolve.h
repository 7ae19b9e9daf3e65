// One N-band Wannier solve (length gauge) on the GPU; see sbe_wannier.cu.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <vector>

#include "sbe_engine.h"
#include "sbe_wannier.h"

namespace sbe {

class WannierSolve {
public:
    // k_begin/k_end: a k-slice [k_begin, k_end) of the grid (0, 0: all of it)
    WannierSolve(const Problem &p, int precision, int device, cudaStream_t st, int k_begin = 0, int k_end = 0);
    ~WannierSolve();
    WannierSolve(const WannierSolve &) = delete;
    WannierSolve &operator=(const WannierSolve &) = delete;
    // Run every attempted step on `st` (returns when the solve is done).
    void run(cudaStream_t st);
    SolveOutputs outputs();
    // per-step sums [Nt][WAN_NSLOT] of this solve's k-points (host copy)
    std::vector<double> sums();
    // harmonic band powers h = 1..hmax from the device-resident sums
    void harmonics(double w0, int hmax, double *band_power);
    // density snapshots (as Engine::snapshots); returns their number
    int snapshots(double *occ1d, double *nc, double *pi);
    int launches() const { return launches_; }
    const WanCtl &control() const { return *h_ctl_; }

    // used by WannierBatch, which launches this solve's kernels itself
    const WanDev &dev() const { return w_; }
    const WanDev *dev_ptr() const { return d_w_; }
    int precision() const { return precision_; }
    void set_stream(cudaStream_t st) { stream_ = st; }
    // the controller state after a batched run (copied in by the batch)
    void finish_batched(const WanCtl &c, int launches);

private:
    Problem prob_;
    int precision_, device_, nshots_ = 0;
    cudaStream_t stream_;
    WanDev w_{};
    WanDev *d_w_ = nullptr;
    WanCtl *h_ctl_ = nullptr;
    int launches_ = 0;
};

// Many N-band solves advanced together: solves of the same launch class
// (band count, gauge, precision) share one attempt launch over all their
// tiles and one control launch with one block per solve per iteration; each
// solve keeps its own controller (its own Cash-Karp step size, or the fixed
// step), so results equal the solves run alone bit for bit.  Solves that are
// done leave their blocks idle until the longest one finishes.  The host
// launches chunks of iterations and checks the controllers once per chunk;
// with use_graph a chunk is captured once as a CUDA graph and replayed.
class WannierBatch {
public:
    WannierBatch(const std::vector<const Problem *> &probs, int precision, int device, cudaStream_t st);
    ~WannierBatch();
    WannierBatch(const WannierBatch &) = delete;
    WannierBatch &operator=(const WannierBatch &) = delete;
    void run(cudaStream_t st, bool use_graph);
    WannierSolve &solve(int i) { return *solves_[i]; }
    int size() const { return (int)solves_.size(); }
    int launches() const { return launches_; }

private:
    struct Class {
        int N = 0, nR = 0, precision = 0;
        int grouped_rk = 0;   // the grouped attempt kernel (and its RK order), or 0
        bool vg = false, shots = false;
        std::vector<int> members;
        const WanDev **d_descs = nullptr;
        WanTileRef *d_tiles = nullptr;
        int ntiles = 0;
    };
    void enqueue_chunk(cudaStream_t st, int iters);
    std::vector<std::unique_ptr<WannierSolve>> solves_;
    std::vector<Class> classes_;
    int device_ = 0, launches_ = 0, per_iter_ = 0;
    cudaStream_t stream_ = nullptr;
    WanCtl *h_ctls_ = nullptr;
};

// The N-band solves of the continuous-batching server: solves join and leave
// while the others run.  step() advances every unfinished solve by a number
// of iterations -- per launch class one attempt launch over all their tiles
// and one control launch (as WannierBatch) -- and queues a copy of their
// controllers; poll() reads that copy once the GPU has reached it, without
// waiting, so finished solves are noticed one step later at most.  Every solve
// keeps its own controller: its results equal the solve run alone bit for
// bit.  Not thread-safe (the server's worker thread owns it).
class WannierPool {
public:
    WannierPool(int device, cudaStream_t st);
    ~WannierPool();
    WannierPool(const WannierPool &) = delete;
    WannierPool &operator=(const WannierPool &) = delete;
    // device memory a solve of this problem holds
    static size_t bytes_needed(const Problem &p, int precision);
    int add(const Problem &p, int precision);   // returns its id
    void remove(int id);
    size_t bytes_in_use() const { return bytes_; }
    int nresident() const { return (int)solves_.size(); }
    int nrunning() const;
    void step(int iters);
    void poll();
    bool finished(int id) const;
    // a finished solve whose step-size controller gave up (tolerance unreachable)
    bool failed(int id) const;
    std::vector<double> sums(int id);
    int last_launches() const { return last_launches_; }

private:
    struct Entry {
        std::unique_ptr<WannierSolve> s;
        size_t bytes = 0;
        bool done = false, failed = false;
    };
    void rebuild();
    std::map<int, Entry> solves_;
    int device_, next_id_ = 0, last_launches_ = 0;
    size_t bytes_ = 0;
    cudaStream_t st_;
    bool dirty_ = true;
    struct Class {
        int N = 0, nR = 0, precision = 0, grouped_rk = 0;
        bool vg = false;
        std::vector<int> ids;
        const WanDev **d_descs = nullptr;
        WanTileRef *d_tiles = nullptr;
        int ntiles = 0;
    };
    std::vector<Class> classes_;
    std::vector<int> polled_;   // ids whose controllers the last step copied, in slot order
    WanCtl *h_ctls_ = nullptr;
    int cap_ = 0;
    cudaEvent_t copied_ = nullptr;
    bool pending_ = false;
};

// The reference's output arrays of a table model from its per-step sums
// [Nt][WAN_NSLOT] (possibly summed over k-slices; antelope.cpp:514-548).
void assemble_table_outputs(const Problem &p, const std::vector<double> &sums, SolveOutputs &o);

}  // namespace sbe
