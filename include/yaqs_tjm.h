/*
 * yaqs_tjm.h — C-ABI of the B200 tensor-jump-method (TJM) trajectory engine.
 *
 * This is the drop-in boundary for the analog TJM path of Yaqs.jl
 * (MaxFroehlich1410/yaqs-julia).  A Julia caller passes its own arrays
 * (Array{ComplexF64,3} MPS tensors, Array{ComplexF64,4} MPO tensors) by
 * pointer: ComplexF64 is interleaved (re, im) double pairs and Julia arrays
 * are column-major, so no repacking is needed on the host.  All sites are
 * 0-based here (Julia's are 1-based; the shim subtracts one).
 *
 * Every entry point returns a status code (YAQS_OK == 0).  On failure
 * yaqs_last_error(ctx) returns a message; the caller turns it into error().
 * The library copies inputs to the device and never keeps host pointers
 * after a call returns.  Distinct contexts may be used from distinct host
 * threads; one context must not be used by two threads at once.
 */
#ifndef YAQS_TJM_H
#define YAQS_TJM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (errors of Simulator.jl:136,139, MPS.jl:357-360) ---- */
enum {
  YAQS_OK = 0,
  YAQS_E_ARG = 1,         /* malformed descriptor, size or pointer             */
  YAQS_E_OOM = 2,         /* device memory admission failed                     */
  YAQS_E_NONFINITE = 3,   /* NaN/Inf met where the reference raises an error    */
  YAQS_E_NOCONV = 4,      /* an iterative solver hit its iteration limit        */
  YAQS_E_TIMEOUT = 5,     /* a bounded device wait gave up                      */
  YAQS_E_CUDA = 6,        /* CUDA runtime error                                 */
  YAQS_E_RNG = 7,         /* injected uniform stream exhausted                  */
  YAQS_E_UNSUPPORTED = 8  /* valid for the reference, not served by this engine */
};

typedef struct yaqs_ctx yaqs_ctx;

/*
 * Matrix product state (MPS.jl:33-43).  chi has L+1 entries, chi[0] ==
 * chi[L] == 1.  tensors[i] holds chi[i]*2*chi[i+1] complex values laid out
 * column-major as (left, phys, right) — the Julia layout (MPS.jl:22).
 * Physical dimension is 2 (qubits).
 */
typedef struct {
  int32_t L;
  const int32_t* chi;
  const double* const* tensors;
} yaqs_mps_desc;

/*
 * Matrix product operator (MPO.jl:32-41).  w has L+1 entries, w[0] ==
 * w[L] == 1.  tensors[i] is (w[i], 2, 2, w[i+1]) column-major complex,
 * index order (left, phys_out, phys_in, right) (MPO.jl:19-24).  The
 * operator must be Hermitian: the engine runs Lanczos, which is what the
 * reference's :auto Krylov mode selects for a Hermitian H_eff
 * (Algorithms.jl:120-176).
 */
typedef struct {
  int32_t L;
  const int32_t* w;
  const double* const* tensors;
} yaqs_mpo_desc;

/*
 * One LocalNoiseProcess (Noise.jl:15-20): a 1-site process or a 2-site
 * process on adjacent sites (site[1] == site[0] + 1).  matrix is the jump
 * operator (2x2 or 4x4, column-major, interleaved complex; the 4x4 basis
 * index is p1 + 2*p2, first site fastest, Dissipation.jl:105).  The two
 * classification flags are computed by the caller exactly as the reference
 * does, because the reference uses two different rules:
 *   pauli_name — Dissipation.is_pauli: name in the Pauli/crosstalk list
 *                (Dissipation.jl:14-21) → dissipation is a scalar decay;
 *   pauli_proc — StochasticProcess.is_pauli(op) for 1-site processes
 *                (StochasticProcess.jl:336-341) and is_pauli_proc(proc) for
 *                2-site ones (:343-357) → jump weight uses the local norm.
 *
 * One MPONoiseProcess (Noise.jl:22-33): a 2-site process with
 * site[1] > site[0] + 1 and operator O = a*1 + b*(sig at site[0])(tau at
 * site[1]), the MPO of build_mpo_phys (Noise.jl:71-131).  matrix holds
 * sig (doubles 0..7, column-major 2x2), tau (8..15), a (16..17), b (18..19)
 * and the dissipation rate (20): the state decays by exp(-dt/2 * rate) at
 * site[1] (handle_longrange_scalar!, Dissipation.jl:161-204: a projector
 * pair's first member carries the pair's summed rate and its mate 0).
 * pauli_name must be 1 (the reference errors on other names there);
 * pauli_proc = 1 marks a "pauli_long_range" candidate (is_pauli_proc with
 * stored factors, StochasticProcess.jl:176-185), which the reference selects
 * but never applies; 0 an "mpo_general" one, applied as an MPO followed by
 * MPS.truncate! (StochasticProcess.jl:46-82, MPS.jl:320-440).
 */
typedef struct {
  int32_t nsites;
  int32_t site[2];
  double strength;
  double matrix[32];
  int32_t pauli_name;
  int32_t pauli_proc;
} yaqs_noise_proc;

/* NoiseModel (Noise.jl:35-37).  present == 0 means `nothing`. */
typedef struct {
  int32_t present;
  int32_t n;
  const yaqs_noise_proc* procs;
} yaqs_noise_desc;

/*
 * Observable (SimulationConfigs.jl:23-56).  LOCAL1: 2x2 operator on
 * site[0] (MPS.jl:608-624).  LOCAL2: 4x4 operator on site[0], site[0]+1
 * (MPS.jl:626-651).  ENTROPY: von Neumann entropy -sum s^2 ln s^2 of the
 * Schmidt values across the bond between site[0] and site[0]+1 (an
 * addition; the reference has no entropy observable).
 */
enum { YAQS_OBS_LOCAL1 = 1, YAQS_OBS_LOCAL2 = 2, YAQS_OBS_ENTROPY = 3 };
typedef struct {
  int32_t kind;
  int32_t site[2];
  double matrix[32];
} yaqs_obs_desc;

/*
 * Uniform draws of stochastic_process! (StochasticProcess.jl:221-244).
 * PHILOX:   Philox-4x32-10 keyed by seed, one stream per trajectory (the
 *           stream id is cfg->traj_offset + trajectory index), one draw per
 *           counter value, 53-bit doubles in [0,1).
 * INJECTED: trajectory t consumes uniforms[t*stride + k] for k = 0,1,2,...
 *           in the reference's order (u1 per stochastic step, u2 only when a
 *           jump happens).  Running out returns YAQS_E_RNG.
 */
enum { YAQS_RNG_PHILOX = 0, YAQS_RNG_INJECTED = 1 };
typedef struct {
  int32_t mode;
  uint64_t seed;
  const double* uniforms;
  int64_t stride;
} yaqs_rng_desc;

enum { YAQS_PREC_FP64 = 0, YAQS_PREC_MIXED = 1 };

/*
 * TimeEvolutionConfig (SimulationConfigs.jl:68-92).  n_times is
 * length(0:dt:T).  krylov_dim / krylov_tol are the reference's krylovdim=25
 * and tol=1e-10 (Algorithms.jl:185).  krylov_exit_tol > 0 lets a Lanczos
 * solve stop before krylov_dim once the a-priori bound
 * prod_i(beta_i*|dt|)/k! falls below it (relative to |v|); 0 runs every
 * solve to krylov_dim or breakdown, like the reference.
 */
typedef struct {
  double dt;
  int32_t n_times;
  int32_t num_traj;
  int32_t max_bond_dim;
  double truncation_threshold;
  int32_t order;
  int32_t sample_timesteps;
  int32_t krylov_dim;
  double krylov_tol;
  double krylov_exit_tol;
  int32_t precision;
  int32_t traj_offset;
  int32_t tdvp_mode;      /* YAQS_TDVP_* */
} yaqs_tev_config;

/*
 * TDVP sweep of every time step.
 * 2SITE:   two_site_tdvp! (Algorithms.jl:580-760), the reference's analog path.
 * 1SITE:   single_site_tdvp! (Algorithms.jl:472-533): bond dimensions stay
 *          those of the start state.
 * DYNAMIC: the Python lineage's local_dynamic_tdvp
 *          (mqt-yaqs/src/mqt/yaqs/core/methods/tdvp.py:667-855): per bond a
 *          2-site update while the bond is below max_bond_dim (its split keeps
 *          min(rank, max_bond_dim) values, no threshold), a 1-site update with
 *          bond back-evolution once it has reached it.
 */
enum { YAQS_TDVP_2SITE = 0, YAQS_TDVP_1SITE = 1, YAQS_TDVP_DYNAMIC = 2 };

/* Counters of one run (summed over trajectories). */
typedef struct {
  int64_t matvecs;         /* effective-Hamiltonian products               */
  int64_t krylov_solves;   /* expm_krylov calls                            */
  int64_t svds;            /* two-site splits                              */
  int64_t jumps;           /* applied quantum jumps                        */
  int64_t nonfinite_fixes; /* NaN/Inf replaced before an SVD (Algorithms.jl:414-417) */
  double flops;            /* algorithmic flops of the H_eff products       */
  double device_ms;        /* device time of the run (CUDA events)          */
  int64_t svd_sweeps;      /* Jacobi sweeps summed over the two-site splits */
} yaqs_run_stats;

/* ---- context ---- */
int yaqs_ctx_create(int32_t device, yaqs_ctx** out);
int yaqs_ctx_destroy(yaqs_ctx* ctx);
const char* yaqs_last_error(const yaqs_ctx* ctx);
const char* yaqs_version(void);

/*
 * Relative Frobenius norm ||H - H^dag|| / ||H|| of an MPO, computed on the
 * host (no device work, no context).  Stands in for the reference's
 * _ishermitian_check (src/Algorithms.jl:120-137), which decides between
 * Lanczos and Arnoldi in the :auto Krylov mode; this engine only runs
 * Lanczos, so yaqs_analog_run / _begin refuse a Hamiltonian whose defect
 * exceeds 1e-5 with YAQS_E_UNSUPPORTED.  The estimate is a difference of
 * squared norms: values below about 1e-7 are rounding.
 */
int yaqs_mpo_hermitian_defect(const yaqs_mpo_desc* H, double* defect);

/*
 * Analog TJM run: replaces the trajectory loop of Simulator._run_analog
 * (Simulator.jl:22-69) with every trajectory of the run advancing together
 * on one GPU; each trajectory follows analog_tjm_2 (AnalogTJM.jl:104-137)
 * when cfg->order == 2, else analog_tjm_1 (AnalogTJM.jl:144-176).
 * psi0 is normalised first, as Simulator.run does (Simulator.jl:128).
 * Outputs (any may be NULL):
 *   traj_out   [num_traj][n_obs][n_out]  real(expect) per trajectory
 *   mean_out   [n_obs][n_out]            mean over trajectories
 *              (aggregate_trajectories!, SimulationConfigs.jl:168-181)
 *   maxchi_out [num_traj][n_out]         max bond dimension at each sample
 * with n_out = n_times if sample_timesteps else 1.  The caller applies the
 * reference's num_traj = 1 rule for noiseless runs (Simulator.jl:27-29).
 */
int yaqs_analog_run(yaqs_ctx* ctx, const yaqs_mps_desc* psi0,
                    const yaqs_mpo_desc* H, const yaqs_noise_desc* noise,
                    const yaqs_obs_desc* obs, int32_t n_obs,
                    const yaqs_tev_config* cfg, const yaqs_rng_desc* rng,
                    double* traj_out, double* mean_out, int32_t* maxchi_out,
                    yaqs_run_stats* stats);

/*
 * Digital TJM (DigitalTJM.jl).  A circuit is the flat gate list of a
 * DigitalCircuit (DigitalTJM.jl:35-66): 1-qubit gates (2x2), 2-qubit gates
 * (4x4, basis index p1 + 2*p2 with p1 on the smaller site, exactly as
 * apply_local_gate_exact! reshapes it, DigitalTJM.jl:267-270) and barriers;
 * a barrier with sample != 0 is a "SAMPLE_OBSERVABLES" barrier
 * (DigitalTJM.jl:147-168).  Sites are 0-based, in the order given.
 */
enum { YAQS_GATE_BARRIER = 0, YAQS_GATE_1Q = 1, YAQS_GATE_2Q = 2 };
typedef struct {
  int32_t kind;
  int32_t site[2];
  double matrix[32];
  int32_t sample;
  /*
   * 2-qubit gates applied by TDVP only: the gate is exp(-i coeff g1 (x) g2)
   * with g1 acting on site[0] and g2 on site[1] (2x2 column-major complex),
   * GateLibrary.generator / hamiltonian_coeff (GateLibrary.jl:24-36).
   */
  int32_t has_generator;
  double coeff;
  double gen1[8];
  double gen2[8];
} yaqs_gate_desc;

/* Circuit run settings (the TimeEvolutionConfig fields the digital path
 * reads, plus the TJMOptions of DigitalTJM.jl:70-76). */
/*
 * TEBD: apply_local_gate_exact! (merge, 4x4, SVD) with SWAP chains for
 * long-range gates (DigitalTJM.jl:251-334).  TDVP: the reference's default
 * (TJMOptions(), DigitalTJM.jl:76): the window s1..s2 evolves under the
 * product MPO coeff g1 (x) 1 ... 1 (x) g2 (construct_window_mpo,
 * DigitalTJM.jl:192-236) by one forward circuit 2-site TDVP sweep
 * (_tdvp_sweep_circuit_2site!, Algorithms.jl:606-627, 762-800).
 */
enum { YAQS_METHOD_TEBD = 0, YAQS_METHOD_TDVP = 1 };
typedef struct {
  int32_t num_traj;
  int32_t max_bond_dim;
  double truncation_threshold;
  int32_t local_method;       /* YAQS_METHOD_* for nearest-neighbour gates */
  int32_t long_range_method;  /* YAQS_METHOD_* for gates on sites further apart */
  int32_t precision;
  int32_t traj_offset;
} yaqs_circuit_config;

/*
 * Layering of a circuit as process_circuit (DigitalTJM.jl:86-145) does it:
 * number of layers and number of measurement columns of run_digital_tjm
 * (DigitalTJM.jl:375-379: one per SAMPLE_OBSERVABLES barrier position, or 1).
 */
int yaqs_digital_plan(const yaqs_gate_desc* gates, int32_t n_gates, int32_t* n_layers, int32_t* n_samples);

/*
 * Digital TJM run: replaces the trajectory loop of Simulator._run_digital
 * (Simulator.jl:71-125); each trajectory follows run_digital_tjm
 * (DigitalTJM.jl:363-450) with TEBD gate application and SWAP chains for
 * long-range gates (DigitalTJM.jl:251-330) or TDVP windows, local
 * dissipation and a jump
 * step after every 2-qubit gate (DigitalTJM.jl:405-420), and the
 * observables at the sample barriers.  psi0 is normalised first
 * (Simulator.jl:128).  Outputs as yaqs_analog_run with n_out = n_samples.
 */
int yaqs_digital_run(yaqs_ctx* ctx, const yaqs_mps_desc* psi0, const yaqs_gate_desc* gates, int32_t n_gates,
                     const yaqs_noise_desc* noise, const yaqs_obs_desc* obs, int32_t n_obs,
                     const yaqs_circuit_config* cfg, const yaqs_rng_desc* rng, double* traj_out,
                     double* mean_out, int32_t* maxchi_out, yaqs_run_stats* stats);

/*
 * The same run in steps, for callers that interleave other work or time
 * individual time indices.  yaqs_analog_begin validates the descriptors,
 * copies every input to the device and sizes the workspaces; nothing is
 * evolved yet.  yaqs_analog_advance runs the next n recorded time indices
 * (the first one also performs the t = 0 measurement and the initial
 * half-step, AnalogTJM.jl:114-126) and waits for them; *device_ms receives
 * their device time.  yaqs_analog_remaining tells how many are left.
 * yaqs_analog_finish copies the outputs back (as yaqs_analog_run) and frees
 * the run; it must be called exactly once, also after an error.
 */
typedef struct yaqs_run yaqs_run;
int yaqs_analog_begin(yaqs_ctx* ctx, const yaqs_mps_desc* psi0,
                      const yaqs_mpo_desc* H, const yaqs_noise_desc* noise,
                      const yaqs_obs_desc* obs, int32_t n_obs,
                      const yaqs_tev_config* cfg, const yaqs_rng_desc* rng,
                      yaqs_run** out);
int yaqs_analog_advance(yaqs_run* run, int32_t n, double* device_ms);
int yaqs_analog_remaining(const yaqs_run* run);
/* Counters of the run so far (as returned by yaqs_analog_finish). */
int yaqs_analog_stats(yaqs_run* run, yaqs_run_stats* stats);
int yaqs_analog_finish(yaqs_run* run, double* traj_out, double* mean_out,
                       int32_t* maxchi_out, yaqs_run_stats* stats);

/*
 * Snapshot of one trajectory of a run between begin and finish: its
 * evolving state (the MPS that the next advance continues from; for the
 * analog program the state phi of analog_tjm_2, AnalogTJM.jl:104-137, not
 * the sampled copy) copied to host buffers.  chi_out[L+1] receives the bond
 * dimensions, oc_out the 0-based orthogonality centre, tensors_out the site
 * tensors (chi[i], 2, chi[i+1]) column-major interleaved complex,
 * concatenated site after site: sum_i 4 chi[i] chi[i+1] doubles, returned in
 * *needed.  With tensors_out NULL (or capacity below *needed) only chi_out,
 * oc_out and *needed are filled; the status is YAQS_OK either way unless an
 * argument is invalid.  No counterpart in the reference, whose trajectories
 * return only their observables (Simulator.jl:41-47).
 */
int yaqs_run_state(yaqs_run* run, int32_t traj, int32_t* chi_out, int32_t* oc_out, double* tensors_out,
                   int64_t capacity, int64_t* needed);

/*
 * Checkpoint and restore within a stepped run (no counterpart in the
 * reference).  yaqs_run_position gives the next launch-list position (the
 * number of advance steps taken); yaqs_run_rng the number of uniforms a
 * trajectory has drawn (its Philox counter or its offset in the injected
 * stream).  yaqs_run_restore writes a trajectory's state (as yaqs_run_state
 * returns it; bond dimensions within this run's capacities) and draw count;
 * yaqs_run_seek(run, p) makes the next advance run position p again
 * (1 <= p <= positions), so a run restored from a checkpoint taken at
 * position p repeats the trajectories it recorded from there.
 */
int yaqs_run_position(const yaqs_run* run, int32_t* position);
int yaqs_run_rng(yaqs_run* run, int32_t traj, int64_t* draws);
int yaqs_run_restore(yaqs_run* run, int32_t traj, const int32_t* chi, int32_t oc, const double* tensors,
                     int64_t draws);
int yaqs_run_seek(yaqs_run* run, int32_t position);

/*
 * Device time per engine phase so far (clock cycles summed over CTAs, 16
 * entries: GEMM, MPO apply, Lanczos orthogonalisation, tridiagonal
 * exponential, SVD sweeps, SVD vectors, QR factor, QR form-Q, norm
 * contraction, environment updates, dissipation, jump step, observables,
 * TDVP sweep, whole step, state copy; nested phases overlap).  All zero
 * unless the environment variable YAQS_PROFILE=1 was set at
 * yaqs_analog_begin.  The analogue of the reference's Timing @t keys
 * (src/Yaqs.jl:3-162).
 */
int yaqs_analog_profile(yaqs_run* run, double* cycles);

/*
 * A digital run in steps: as yaqs_digital_run, but returns a run handle
 * that yaqs_analog_advance / _remaining / _stats / _profile / _finish
 * drive.  One advance step is one launch: the first prepares and normalises
 * every trajectory (and takes the start sample), each further one applies
 * one layer of the processed circuit (DigitalTJM.jl:380-430).
 */
int yaqs_digital_begin(yaqs_ctx* ctx, const yaqs_mps_desc* psi0, const yaqs_gate_desc* gates, int32_t n_gates,
                       const yaqs_noise_desc* noise, const yaqs_obs_desc* obs, int32_t n_obs,
                       const yaqs_circuit_config* cfg, const yaqs_rng_desc* rng, yaqs_run** out);

/*
 * Serving.  A request loop that runs many simulations at once on one GPU:
 * analog and digital requests of different L, bond dimension, MPO width and
 * trajectory count (the Simulator.run calls of many users, Simulator.jl:
 * 127-141).  Requests are admitted in arrival order while their trajectory
 * states and outputs fit in hbm_budget; every admitted run advances by
 * `chunk` recorded time indices (analog) or circuit layers (digital) per
 * launch, and all of them share ONE persistent kernel launch whose CTAs pull
 * (run, position, trajectory) work units and share one pool of slot
 * workspaces sized for the largest request the server accepts.  A request
 * that arrives while others run joins at the next launch; a finished run
 * leaves and frees its memory.  Each request's results equal those of the
 * same yaqs_analog_run / yaqs_digital_run call: a trajectory's arithmetic
 * does not depend on which slot or launch runs it.  All functions are safe
 * to call from several host threads.
 */
typedef struct yaqs_server yaqs_server;
typedef struct {
  int32_t max_L;          /* longest chain served */
  int32_t max_bond_dim;   /* largest max_bond_dim served (<= 128) */
  int32_t max_mpo_width;  /* widest MPO bond served (analog, <= 8) */
  int32_t krylov_dim;     /* largest krylov_dim served */
  int32_t mixed;          /* 1: also size the slots for YAQS_PREC_MIXED requests */
  int32_t chunk;          /* positions every run advances per launch (>= 1) */
  int64_t hbm_budget;     /* bytes for admitted runs (0: 90% of the free memory left after the slot pool) */
} yaqs_server_config;

enum { YAQS_REQ_QUEUED = 0, YAQS_REQ_RUNNING = 1, YAQS_REQ_DONE = 2, YAQS_REQ_FAILED = 3 };

typedef struct {
  int64_t submitted, completed, failed, launches;
  int64_t queued_now, running_now;
  int64_t bytes_in_use, hbm_budget;
  int32_t slots;               /* CTAs of every served launch */
  double latency_p50_s;        /* submit -> done over completed requests */
  double latency_p99_s;
  double queue_p50_s;          /* submit -> admitted */
  double queue_p99_s;
  double busy_s;               /* device time of all served launches */
} yaqs_server_stats;

int yaqs_server_create(yaqs_ctx* ctx, const yaqs_server_config* cfg, yaqs_server** out);
/* Copies every descriptor and buffer; the caller may free them on return. */
int yaqs_server_submit_analog(yaqs_server* srv, const yaqs_mps_desc* psi0, const yaqs_mpo_desc* H,
                              const yaqs_noise_desc* noise, const yaqs_obs_desc* obs, int32_t n_obs,
                              const yaqs_tev_config* cfg, const yaqs_rng_desc* rng, int64_t* id);
int yaqs_server_submit_digital(yaqs_server* srv, const yaqs_mps_desc* psi0, const yaqs_gate_desc* gates,
                               int32_t n_gates, const yaqs_noise_desc* noise, const yaqs_obs_desc* obs,
                               int32_t n_obs, const yaqs_circuit_config* cfg, const yaqs_rng_desc* rng,
                               int64_t* id);
/* *state receives YAQS_REQ_*. */
int yaqs_server_poll(yaqs_server* srv, int64_t id, int32_t* state);
/* Waits until the request is done or failed; YAQS_E_TIMEOUT after timeout_s (< 0: no limit). */
int yaqs_server_wait(yaqs_server* srv, int64_t id, double timeout_s);
/*
 * Outputs of a finished request (as yaqs_analog_run / yaqs_digital_run;
 * any pointer may be NULL) and times_s[3] = {queued, running, total}
 * seconds; releases the request.  A failed request returns its status and
 * message (yaqs_server_last_error).
 */
int yaqs_server_take(yaqs_server* srv, int64_t id, double* traj_out, double* mean_out, int32_t* maxchi_out,
                     yaqs_run_stats* stats, double* times_s);
const char* yaqs_server_last_error(yaqs_server* srv);
int yaqs_server_stats_get(yaqs_server* srv, yaqs_server_stats* out);
/* Fails whatever is still queued or running and frees the server. */
int yaqs_server_destroy(yaqs_server* srv);

#ifdef __cplusplus
}
#endif

#endif /* YAQS_TJM_H */
