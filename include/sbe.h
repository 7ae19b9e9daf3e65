/*
 * sbe.h -- C ABI of the B200 SBE propagator (antelope_b200/libsbe_b200.so).
 *
 * Drop-in for the time propagation of ftachacon/antelope (src/GeneralModel).
 * The reference drives its solver per (time step, k-point) from main():
 *
 *   SBEs(const libconfig::Setting*, GaugeType, int idx_start, int idx_end)  SBEs.h:102,125-430
 *   void RunSBEs(int kindex, double t)                                      SBEs.h:105,596-624
 *   std::tuple<...> GenInterIntraCurrent(int kindex, double t)              SBEs.h:108,694-760
 *   std::array<double,3> GenCurrent(int kindex, double t)                   SBEs.h:107,626-693
 *   time/k loop, k-sum, MPI reduce and file output                          antelope.cpp:297-548
 *
 * A per-(k, t) call cannot cross a device boundary efficiently, so this ABI
 * replaces that whole loop with whole-solve calls: a problem is built from
 * the same inputParam.cfg, a solver runs every time step on the GPU with the
 * k-sum fused into the kernels, and the caller receives the same arrays the
 * reference writes to its .dat files.  Plain C types only; no pointer passed
 * in is retained after a call returns (except the problems of a batch, see
 * below).  Errors never exit the process: every call returns an sbe_status
 * and sets a thread-local message (sbe_last_error_message()).
 */
#ifndef SBE_B200_H
#define SBE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define SBE_ABI_VERSION 1

typedef enum sbe_status {
    SBE_OK = 0,
    SBE_BAD_CONFIG = 1,       /* the reference would exit(EXIT_FAILURE) on this input */
    SBE_UNSUPPORTED = 2,      /* valid input that this library does not build */
    SBE_OOM = 3,              /* device memory exhausted or admission refused */
    SBE_CUDA_ERROR = 4,
    SBE_TIMEOUT = 5,
    SBE_CANCELLED = 6,
    SBE_INVALID_ARGUMENT = 7,
    SBE_NOT_READY = 8
} sbe_status;

typedef struct sbe_problem sbe_problem;
typedef struct sbe_solver sbe_solver;
typedef struct sbe_batch sbe_batch;
typedef struct sbe_server sbe_server;

/* Sizes of a problem: output arrays are Nt rows.  gauge: 0 LengthWannier,
 * 1 LengthHamiltonian, 2 Velocity (constant.h:41-46); rk: 4, 5 or 45. */
typedef struct sbe_dims {
    int Nt, nband, nval, ntotal;
    int Nk[3];
    int gauge, rk, precision, model, inter_intra;
    double atmin, dt, dV, total_weight;
} sbe_dims;

/* Run options.  precision: -1 = calc.precision of the cfg (default fp64),
 * 0 = plain FP64, 1 = mixed FP32 stages / FP64 sums.  tile_k, k_per_thread,
 * steps_per_launch: 0 = tuned defaults; tile_k / k_per_thread (threads per
 * CTA) is a multiple of 32 up to 256, or up to 512 for the two-band velocity
 * gauge with RK4 in FP64 or with one k-point per thread.  use_graph: capture the launches of
 * a run into one CUDA graph.  profile: see sbe_solver_kernel_times. */
typedef struct sbe_opts {
    int device;
    int precision;
    int tile_k;
    int k_per_thread;
    int steps_per_launch;
    int use_graph;
    int profile;   /* 1: time every kernel launch with CUDA events (no graph) */
} sbe_opts;

/* Caller-owned host arrays (any may be NULL):
 *   inter[Nt*3]  columns of interband_dipole_full_evol.dat  (antelope.cpp:522-527)
 *   intra[Nt*3]  columns of intraband_current_full_evol.dat (antelope.cpp:522-527)
 *   occ[Nt*(N+1)] columns of occupation__full__evol.dat      (antelope.cpp:530-536)
 *   coh[Nt*2]    columns of coherence__full__evol.dat       (antelope.cpp:538-542)
 *   laser[Nt*7]  t, E[3], A[3] of outlaserdata.dat           (antelope.cpp:208-235) */
typedef struct sbe_outputs {
    double *inter;
    double *intra;
    double *occ;
    double *coh;
    double *laser;
} sbe_outputs;

int sbe_abi_version(void);
const char *sbe_last_error_message(void);
void sbe_opts_default(sbe_opts *opts);

/* Parse an inputParam.cfg (libconfig text; antelope.cpp:90-129 and the
 * SBEs constructor's reads, SBEs.h:125-241, 432-561).  Same keys, defaults
 * and diagnostics as the reference, plus additive keys: env_name "sin2",
 * calc.precision "fp64"|"mixed", calc.rk "rk4"|"rk5"|"cashkarp45", calc.tol. */
sbe_status sbe_problem_from_cfg(const char *path, sbe_problem **out);
sbe_status sbe_problem_from_string(const char *text, sbe_problem **out);
sbe_status sbe_problem_dims(const sbe_problem *p, sbe_dims *out);
/* Host-only: the columns of outlaserdata.dat (t, E[3], A[3]) into laser[Nt*7]
 * (antelope.cpp:208-235; laser.h:278-322).  Needs no GPU. */
sbe_status sbe_problem_laser(const sbe_problem *p, double *laser);

/* The tight-binding tables a table model runs on: the SyntheticWannier cfg
 * group, or an analytic material of the reference (KaneMele, Haldane2L,
 * WilsonMass, XYHlattice, TMDCs, SquareSBand, Bi2Se3surf) restated as H(k) = sum_v h_v e^{ik.v} and its
 * GenJMatrix as J_a(k) = sum_v j_{a,v} e^{ik.v}.  Call once with the array
 * pointers NULL to read the sizes, then with caller-owned arrays:
 *   vec[nvec*2] Cartesian vectors (bohr), h[nvec*N*N*2], d and j
 *   [nvec*2*N*N*2] (complex interleaved; d / j only when the flags say so),
 *   bz[9] Brillouin-zone axes before ksfactor / BZaxes overrides.
 * The Haldane model (closed-form kernels) and MultiWSM (a continuum model
 * evaluated from its formulas) have no tables:
 * SBE_INVALID_ARGUMENT. */
typedef struct sbe_model {
    int nband, nval, nvec, has_dipoles, has_current_tables;
    double *vec, *h, *d, *j, *bz;
} sbe_model;
sbe_status sbe_problem_model(const sbe_problem *p, sbe_model *m);
/* Density snapshots (calc.shotNumber > 0; antelope.cpp:267-422): every
 * `interval` = int(period0 / shotNumber / dt) steps (period0 of the first pulse,
 * antelope.cpp:274-278), after the step n with n % interval == 0, `nshots` in
 * all; n0 = Npoints[0].  interval = nshots = 0 when snapshots are off.
 * Host-only. */
sbe_status sbe_problem_snapshots(const sbe_problem *p, int *interval, int *nshots, int *n0);
void sbe_problem_destroy(sbe_problem *p);

/* One solve (replaces SBEs + the driver loop of antelope.cpp:297-548). */
sbe_status sbe_solver_create(const sbe_problem *p, const sbe_opts *opts, sbe_solver **out);
/* Enqueue the whole propagation on `stream` (a cudaStream_t; NULL = the
 * solver's own stream).  Returns without waiting for the GPU. */
sbe_status sbe_solver_run(sbe_solver *s, void *stream);
/* Wait for the run and fill the caller's host arrays. */
sbe_status sbe_solver_get(sbe_solver *s, const sbe_outputs *out);
/* Number of propagate kernel launches the last run issued. */
int sbe_solver_launches(const sbe_solver *s);
/* Time-stepping statistics of a finished run: accepted steps, attempted steps
 * and rejected attempts.  Fixed-step methods (RKorder 4 / 5, SBEs.h:596-624)
 * take Nt steps and reject none; the Cash-Karp extension reports its
 * controller's counts (one step size per solve). */
sbe_status sbe_solver_steps(const sbe_solver *s, long long *steps, long long *attempts, long long *rejects);
/* With opts.profile = 1: total device time (ms) and count of the propagate
 * and reduce launches of the run (CUDA events on the launching stream). */
sbe_status sbe_solver_kernel_times(sbe_solver *s, double *propagate_ms, int *propagate_launches,
                                   double *reduce_ms, int *reduce_launches);
void sbe_solver_destroy(sbe_solver *s);

/* Density snapshots of a finished solve (every model, both gauges), the
 * data of the reference's snapshot files (antelope.cpp:340-422); any array
 * may be NULL:
 *   occ1d[nshots*n0]       occupation_1d_integration.dat: Re sum_k w_k rho'_cc
 *                          over the k-points with first grid index i, / Npoints[1];
 *   nc[nshots*ntotal]      fisrt_conduction.dat: rho'_cc of every k-point;
 *   pi[nshots*ntotal*2]    fisrt_coherence.dat: rho'[Nval][Nval-1] (re, im);
 * rho' is rho in the band basis (velocity gauge) or in the eigenbasis of
 * H0(k + A(t_n)) (length gauge, SBEs::WannierToHamiltonian, SBEs.h:927-940).
 * The reference's own loop fills nc / pi through a stale k index
 * (antelope.cpp:384-400); here each k-point gets its own value.  For a k-slice
 * solver, the arrays cover the slice and occ1d holds its part of the sums. */
sbe_status sbe_solver_snapshots(sbe_solver *s, double *occ1d, double *nc, double *pi);
/* Write occupation_1d_integration.dat ("%16e    " per value, one row per
 * snapshot), fisrt_conduction.dat and fisrt_coherence.dat (raw doubles) and
 * the empty snapshot_log.dat into `dir`, as antelope.cpp:288-292, 365-368,
 * 416-421 do; sbe_run_cfg writes them when the cfg asks for snapshots. */
sbe_status sbe_write_snapshots(const sbe_problem *p, const double *occ1d, const double *nc, const double *pi,
                               const char *dir);

/* Harmonic band powers of a finished solve, computed on the GPU from its
 * device-resident results, in the convention of the reference's analysis
 * script (AlsisPythonShort/AnalysisReader_PyDir.py:252-354: Blackman window
 * over the record, FFT times dt, times -i*omega, |.|^2 summed over x and y,
 * with J = interband + intraband current; band h = the bins with
 * h - 1/2 <= omega / w0 < h + 1/2 as IntegrateSpectrumOrder.py:57-70).
 * w0: the fundamental angular frequency (a.u.); band_power[hmax]. */
sbe_status sbe_solver_harmonics(sbe_solver *s, double w0, int hmax, double *band_power);

/* k-sharding of one solve over several GPUs or processes (the reference's
 * ParaRange split of the k-grid over MPI ranks, utility.h:104-115, and the
 * MPI_Reduce of antelope.cpp:482-512):
 *   sbe_solver_create_slice  a solver for flat k-points [k_begin, k_end);
 *   sbe_solver_sums          its per-step k-sums, (Nt + 1) rows of
 *                            sbe_sums_width(p) doubles (the last row holds the
 *                            time-independent parts), additive over slices;
 *   sbe_assemble             the output arrays from sums added over all slices
 *                            (host only, no GPU).
 * The slices' sums are combined by the caller (an NCCL all-reduce, say). */
sbe_status sbe_solver_create_slice(const sbe_problem *p, const sbe_opts *opts, int k_begin, int k_end,
                                   sbe_solver **out);
int sbe_sums_width(const sbe_problem *p);
sbe_status sbe_solver_sums(sbe_solver *s, double *sums);
sbe_status sbe_assemble(const sbe_problem *p, const double *sums, const sbe_outputs *out);

/* Write the reference's six output files into `dir` (antelope.cpp:176-184,
 * 208-235, 514-548) from arrays filled by a get call. */
sbe_status sbe_write_outputs(const sbe_problem *p, const sbe_outputs *o, const char *dir);
/* The whole drop-in: read `cfg_path`, solve on the GPU, write the files in
 * `out_dir` (the reference reads ./inputParam.cfg and writes to ./). */
sbe_status sbe_run_cfg(const char *cfg_path, const char *out_dir, const sbe_opts *opts);

/* Many solves with their own grids, pulses and model parameters advanced
 * together: the reference runs one such parameter point per job
 * (src/_SH/SLURM/loop__run__jobs__mt2.sh).  Two-band Haldane problems share
 * one launch per launch class per step chunk; N-band table and continuum
 * models (the SyntheticWannier group, the analytic materials, MultiWSM) share
 * one attempt launch over all their k-points and one control launch per
 * iteration, each solve keeping its own step-size controller (Cash-Karp or
 * fixed step), so every result equals its solve run alone bit for bit.
 * opts.use_graph captures the launches as CUDA graphs.  The problems must
 * stay alive until sbe_batch_destroy. */
sbe_status sbe_batch_create(const sbe_problem *const *problems, int n, const sbe_opts *opts, sbe_batch **out);
sbe_status sbe_batch_run(sbe_batch *b, void *stream);
sbe_status sbe_batch_get(sbe_batch *b, int index, const sbe_outputs *out);
/* Time-stepping statistics of solve `index` of a finished batch (as
 * sbe_solver_steps). */
sbe_status sbe_batch_steps(sbe_batch *b, int index, long long *steps, long long *attempts, long long *rejects);
int sbe_batch_launches(const sbe_batch *b);
/* Density snapshots of solve `index` of a finished batch (as sbe_solver_snapshots). */
sbe_status sbe_batch_snapshots(sbe_batch *b, int index, double *occ1d, double *nc, double *pi);
sbe_status sbe_batch_harmonics(sbe_batch *b, int i, double w0, int hmax, double *band_power);
sbe_status sbe_batch_kernel_times(sbe_batch *b, double *propagate_ms, int *propagate_launches,
                                  double *reduce_ms, int *reduce_launches);
void sbe_batch_destroy(sbe_batch *b);

/* Continuous-batching server: a worker thread admits submitted solves while
 * device memory allows, advances all resident solves together, and retires
 * them as they finish.  Two-band Haldane requests share the engine's ticks;
 * N-band requests (table and continuum models) advance a few attempted steps
 * per tick in batched launches, each with its own step-size controller.
 * Thread-safe.  Requests return the output arrays of sbe_outputs; density
 * snapshots are taken by sbe_solver_* and sbe_batch_*. */
typedef struct sbe_server_opts {
    int device;
    int precision;
    int steps_per_launch;
    int max_resident;          /* 0 = no limit besides memory */
    double mem_budget_bytes;   /* 0 = free device memory minus 4 GiB */
    int tile_k;
    int k_per_thread;
} sbe_server_opts;

sbe_status sbe_server_create(const sbe_server_opts *opts, sbe_server **out);
sbe_status sbe_server_submit(sbe_server *s, const sbe_problem *p, long long *request_id);
/* Wait up to timeout_s (< 0: forever) for a request; fill its outputs and
 * its latency (submit -> result available, seconds).  A request's final state
 * is returned once: afterwards the server forgets it (unknown request id). */
sbe_status sbe_server_wait(sbe_server *s, long long request_id, double timeout_s, const sbe_outputs *out,
                           double *latency_s);
sbe_status sbe_server_cancel(sbe_server *s, long long request_id);
/* Counters: submitted, completed, failed, resident now, launches issued. */
sbe_status sbe_server_stats(sbe_server *s, long long counters[5]);
void sbe_server_destroy(sbe_server *s);

/* Allocation-free solve, for callers that must not allocate device memory
 * themselves (code inside an application whose device memory belongs to that
 * application's pool allocator, or latency-critical loops where cudaMalloc /
 * cudaFree could synchronise the device).  No counterpart in the reference.
 * Same result as sbe_solver_create + sbe_solver_run + sbe_solver_get (the
 * same kernels), but all device working memory lives in one fixed 64 MiB
 * array inside the library, held on every GPU that loads the library until
 * exit; problems that do not fit are rejected with SBE_OOM.  The first call
 * on a device looks up that array's address (make it before any stream
 * capture on that device).  Calls share the array: they must not overlap on
 * the GPU -- this function serialises its own calls and returns after its
 * GPU work is done.  `stream` may be NULL (the legacy default stream). */
sbe_status sbe_solve_noalloc(const sbe_problem *p, const sbe_opts *opts, void *stream, const sbe_outputs *out);

/* Measured FP64 / FP32 FMA pipe peaks of the device (TFLOP/s), the
 * denominators of the roofline fractions; fp32x2: packed f32x2 FMAs.  No
 * reference counterpart. */
sbe_status sbe_measure_fma_peaks(int device, double *fp64_tflops, double *fp32_tflops, double *fp32x2_tflops);

#ifdef __cplusplus
}
#endif
#endif
