/*
 * mmp.h — C ABI of the B200 Lawson–Runge–Kutta multimode NLSE solver.
 *
 * Plain C, plain pointers and sizes; no CUDA or C++ types cross this boundary.
 * The C++ drop-in classes (MultimodePropagation_B200.hpp) and the Python
 * bindings (mm_propagation_b200/capi.py) are thin layers over these entry
 * points. Each entry point replaces a piece of alexandreroget/MM_Propagation's
 * C++ solver API; the replaced interface is cited beside it.
 *
 * Conventions
 *  - Every call returns 0 (MMP_OK) or a negative MMP_E* code; mmp_strerror()
 *    turns it into text. The reference checks no return codes at all.
 *  - Complex arrays are interleaved FP64 (re, im) with the mode index
 *    outermost: field[p][t][2], p < n_modes, t < nt. This is the memory order
 *    of ComplexArraysContainer ([mode][sample], include/ComplexArraysContainer.hpp:7-29).
 *  - Callers own every buffer they pass; inputs are copied during the call.
 *  - A solver (or batch) is not thread-safe; use one per host thread. Each
 *    owns one CUDA stream on the device that was current when it was created.
 */
#ifndef MMP_B200_H
#define MMP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------- */
#define MMP_OK 0
#define MMP_EINVAL (-1)     /* malformed parameters (see mmp_validate_params) */
#define MMP_ENOMEM (-2)     /* device or host allocation failed */
#define MMP_ECUDA (-3)      /* a CUDA runtime call failed */
#define MMP_ENONFINITE (-4) /* the field became NaN/Inf during propagation */
#define MMP_ETIMEOUT (-5)   /* a bounded wait expired (server, device-side waits) */
#define MMP_ENOTSUP (-6)    /* valid input outside what this build supports (e.g. NT not 2^k) */
#define MMP_ENODEV (-7)     /* no usable sm_100 device */
#define MMP_ESTATE (-8)     /* call not valid in the object's current state */
#define MMP_EDRIFT (-9)     /* the FP64 energy left the band set by mmp_set_energy_drift_limit */

/* ---- flags (mmp_params.flags) ---------------------------------------------------- */
/* Arithmetic: default is FP32 bulk (FFTs, contraction, Raman) with FP64 dispersion
 * phase, FP64 field accumulation and FP64 monitors. MMP_F_FP64 runs everything in FP64. */
#define MMP_F_FP64 (1u << 0)
/* Pair table: the reference forms V[slot] from slot%M and slot/M instead of from
 * unique_pairs[slot] (src/MultimodePropagation_CPU.cpp:126-133, :195-205). That is
 * the default here, for parity; MMP_F_PHYSICAL_PAIRS uses unique_pairs[slot]. */
#define MMP_F_PHYSICAL_PAIRS (1u << 1)
/* z handling: the reference resets z to 0 at every computeLawsonRK call while the
 * interaction-picture field carries on (src/MultimodePropagation.cpp:158-163).
 * That is the default; MMP_F_CONTINUOUS carries z across calls instead. */
#define MMP_F_CONTINUOUS (1u << 2)
/* Skip the per-step FP64 energy / photon-number monitors. */
#define MMP_F_NO_MONITORS (1u << 3)

/* RK tableau selection (mmp_params.rk_variant) */
#define MMP_RK_BY_ORDER 0      /* method_order 8 -> Butcher11, 6 -> Butcher7(nu=1), else RK4
                                  (src/MultimodePropagation.cpp:15-27) */
#define MMP_RK_BUTCHER7_LAMBDA_MU 1 /* the two-parameter 7-stage tableau
                                       (src/RungeKutta.cpp:75-122), params rk_lambda, rk_mu */

/* One non-zero coupling coefficient Q^(p)_{k,l,m}: struct NonZeroValue plus the
 * output-mode index p (include/Sparse3DArray.hpp:7-11). Entries of the same p
 * keep the order in which they appear in the array: that order is the
 * reference's insertion order and decides the pair table. */
typedef struct mmp_nz {
  uint32_t p, k, l, m;
  double value;
} mmp_nz;

/* struct SimulationParameters (include/MultimodePropagation.hpp:16-33), flattened.
 * Units as in the reference's README (README.md:73-88). */
typedef struct mmp_params {
  uint32_t n_modes;             /* M */
  uint32_t nt;                  /* NT: samples per mode (power of two, 2^6..2^16) */
  uint32_t n_beta;              /* L: dispersion orders per mode (>= 3) */
  const double* dispersion;     /* [M][L] beta_i^(p) in ps^i/m */
  uint32_t n_nonzeros;
  const mmp_nz* coupling;       /* [n_nonzeros], Q in 1/m^2 */
  const double* initial_fields; /* [M][NT][2] in W^(1/2) */
  double time_window;           /* ps */
  double pulse_width;           /* T0, ps */
  double fiber_length;          /* m */
  uint32_t n_steps;
  uint32_t method_order;
  double nonlinearity_const;    /* gamma, 1/(W m) */
  double raman_proportion;      /* f_R (ignored when raman == 0) */
  const double* raman_response; /* [NT] h_R on the time grid, 1/ps; NULL when raman == 0 */
  int32_t raman;                /* 0: MultimodePropagation*_RamanOFF, 1: *_RamanON */
  uint32_t flags;               /* MMP_F_* */
  int32_t rk_variant;           /* MMP_RK_* */
  double rk_lambda, rk_mu;      /* for MMP_RK_BUTCHER7_LAMBDA_MU */
  double center_frequency;      /* omega0 in rad/ps for the photon-number monitor; 0 = off */
} mmp_params;

/* Read-only facts about a solver after creation (the base class's protected
 * members, include/MultimodePropagation.hpp:66-93). */
typedef struct mmp_info {
  uint32_t n_modes, nt, n_stages, n_pairs; /* n_pairs = |unique_pairs| */
  uint32_t n_pair_fields;                  /* distinct (l<=m) pair fields the device forms */
  uint32_t pair_quirk_active;              /* 1 if some unique_pairs[slot] != slot and the
                                              reference slot mapping is in use */
  double t_final, delta_t, z_final, delta_z, z; /* dimensionless, as in the reference */
  double LD, conversion_factor, max_beta2, max_Q;
  uint64_t steps_done;                      /* steps since creation (monotone) */
  uint32_t fp64;                            /* 1 if MMP_F_FP64 */
  uint32_t cluster_ctas;                    /* CTAs that share one FFT row */
  uint32_t raman_recurrence;                /* Raman convolution: 0 by FFT; as a recurrence (h_R
                                               a damped sinusoid h_i = Im(c lambda^i)) 1 in a row
                                               pass, 2 inside the contraction tiles */
  uint32_t graph_branches;                  /* independent solve groups per captured graph */
  uint32_t dense_contraction;               /* 1: the contraction runs as a dense register-blocked
                                               product over (p, k) x pair fields (M <= 16) */
  uint32_t tensor_core_contraction;         /* 1: that dense product runs on the tensor cores
                                               (tcgen05, TF32 operands split hi + lo, FP32 sums) */
  uint32_t contract_pair_chunk;             /* > 0: pair fields held per chunk by the contraction
                                               of tall tiles (Raman recurrence in the tiles) */
  uint32_t contract_sub_block;              /* > 0: the contraction of tall tiles runs the Raman
                                               recurrence serially per pair field, in sub-blocks of
                                               this many samples (merged terms) */
  uint32_t contract_tile;                   /* samples per contraction tile (CTA) */
  uint32_t autotuned;                       /* 1: cluster_ctas, contract_tile and graph_branches
                                               were chosen by timing steps of this batch on
                                               this device (or taken from that choice, cached
                                               for the same shape); batches of one solve keep
                                               the defaults the serving loop uses */
} mmp_info;

typedef struct mmp_solver mmp_solver;

/* Validate parameters without touching the device. Checks the conditions the
 * MATLAB front-end checks (matlab/mm_propagation.cpp:341-527) plus the ones
 * under which the reference silently produces NaN/Inf (max|beta2| == 0,
 * max|Q| == 0, nonlinearity_const == 0, T0 <= 0, fewer than 3 dispersion orders,
 * indices >= M).
 * On failure writes a one-line reason into msg (if msg != NULL). */
int mmp_validate_params(const mmp_params* params, char* msg, size_t msg_len);

/* MultimodePropagationCPU_RamanOFF/ON constructors
 * (src/MultimodePropagation_CPU.cpp:4-21, :163, :225-232; src/MultimodePropagation.cpp:4-12).
 * Uploads everything and leaves the solver at z = 0. */
int mmp_solver_create(const mmp_params* params, mmp_solver** out);

/* virtual void computeLawsonRK(unsigned nz) (include/MultimodePropagation.hpp:41,
 * src/MultimodePropagation_CPU.cpp:24-34): nz Lawson–RK steps of delta_z.
 * Resets z to 0 first unless MMP_F_CONTINUOUS. Returns MMP_ENONFINITE if the
 * field stopped being finite. Blocks until the device is done. */
int mmp_propagate(mmp_solver* s, uint32_t nz);

/* Asynchronous form of mmp_propagate: enqueues the steps on the solver's stream
 * and returns; mmp_synchronize waits and reports the status. */
int mmp_propagate_async(mmp_solver* s, uint32_t nz);
int mmp_synchronize(mmp_solver* s);

/* void computeLawsonRK() (src/MultimodePropagation.cpp:213-216):
 * nz = floor(z_final / delta_z). */
int mmp_propagate_default(mmp_solver* s);

/* virtual ComplexArraysContainer getResult() (src/MultimodePropagation_CPU.cpp:88-104):
 * phi_p = IFFT(exp(L_p z) * FFT(psi_p)) / conversion_factor, into out[M][NT][2]. */
int mmp_get_result(mmp_solver* s, double* out);

/* Replace the field with new initial fields phi0[M][NT][2] (W^(1/2)) and set z = 0,
 * keeping every other parameter: the same as constructing a new solver with
 * other initial_fields, without re-uploading the rest. The fields are checked for
 * NaN/Inf on the device copy before anything of the solve changes (MMP_EINVAL then);
 * the call returns once they are on the device (it waits for the solver's stream). */
int mmp_set_fields(mmp_solver* s, const double* phi0);

/* Per-step FP64 monitors since creation: total energy (pJ, sum over modes of
 * |phi|^2 dt) and photon number (0 when center_frequency == 0), at the end of
 * each step. Copies min(max_steps, steps_done) entries; n_written may be NULL. */
int mmp_get_monitors(mmp_solver* s, double* energy, double* photons, uint64_t max_steps,
                     uint64_t* n_written);

int mmp_get_info(mmp_solver* s, mmp_info* info);

/* No counterpart in the reference, which checks nothing while it propagates. Failure
 * detection from the FP64 energy monitor: after every step the device compares the
 * step's total energy E with E_ref, the energy after the first step since creation or
 * mmp_set_fields, and flags the solve when |E - E_ref| > rel_tol * E_ref; the next
 * mmp_propagate / mmp_synchronize returns MMP_EDRIFT. rel_tol = 0 turns the check off
 * (the default). Energy is a conserved quantity of the Kerr system with a coupling
 * symmetric in (p, k, l, m); with Raman on it is not exactly conserved, so choose the
 * band accordingly. MMP_ESTATE if the solve keeps no monitors (MMP_F_NO_MONITORS). */
int mmp_set_energy_drift_limit(mmp_solver* s, double rel_tol);

/* ~MultimodePropagation (include/MultimodePropagation.hpp:39). NULL is allowed. */
void mmp_solver_destroy(mmp_solver* s);

/* ---- chunked propagation and files (the MEX front end, matlab/mm_propagation.cpp, and
 * the driver, simulations/main.cpp) ---------------------------------------------------- */
/* The MEX front end's n_save loop (matlab/mm_propagation.cpp:61-91): n_save chunks of
 * n_steps / n_save RK steps, the last one plus n_steps % n_save; after chunk i the
 * result is read back into fields[i][M][NT][2] (may be NULL), Z[i] = steps so far *
 * fiber_length / n_steps in metres (may be NULL), elapsed_s[i] = seconds since the call
 * began (may be NULL). z_mode 0 carries z across the chunks, so every snapshot is the
 * field at Z[i]; z_mode 1 restarts z at every chunk as the reference's computeLawsonRK
 * does (src/MultimodePropagation.cpp:158-163), which is what the MEX front end
 * saves. The first chunk starts like mmp_propagate (z = 0 unless MMP_F_CONTINUOUS). */
int mmp_propagate_snapshots(mmp_solver* s, uint32_t n_save, int z_mode, double* fields, double* Z,
                            double* elapsed_s);

/* The MEX front end's dense coupling input (matlab/mm_propagation.cpp:186-209): q[M^4]
 * in MATLAB order (p fastest, then k, l, m) to the non-zero list, in the order the
 * MEX inserts it (which decides the reference's unique_pairs). *n receives the count;
 * at most cap entries are written to out (out may be NULL to count). */
int mmp_coupling_from_dense(uint32_t M, const double* q, mmp_nz* out, uint32_t cap, uint32_t* n);

/* The driver's text dump (simulations/main.cpp:101-103): one line per sample i,
 * |phi0_0[i]| ; ... ; |phi0_{M-1}[i]| ; |phi_0[i]| ; ... ; |phi_{M-1}[i]| in the default
 * iostream number format (%g). phi0 may be NULL (only the output columns). */
int mmp_write_abs_text(const char* path, uint32_t M, uint32_t nt, const double* phi0, const double* phi);

/* The struct the MEX front end saves (matlab/mm_propagation.cpp:280-325), as a MATLAB
 * Level-5 MAT-file (readable by MATLAB's load and scipy.io.loadmat) holding variable
 * `name` (NULL: "output") = struct with Z (1x1 double, m), fields (M x NT complex double)
 * and cpu_time (1x1 double, s). phi is [M][NT][2]. */
int mmp_write_mat(const char* path, const char* name, double Z, uint32_t M, uint32_t nt, const double* phi,
                  double cpu_time);

/* ---- batches: many independent solves advanced by the same launches -------------- */
/* All members must share nt, flags & MMP_F_FP64, raman and the RK tableau; n_modes,
 * coupling, dispersion, fields and lengths may differ. Member i is addressed by index. */
typedef struct mmp_batch mmp_batch;
int mmp_batch_create(const mmp_params* const* params, uint32_t n, mmp_batch** out);
int mmp_batch_propagate(mmp_batch* b, uint32_t nz);
int mmp_batch_propagate_async(mmp_batch* b, uint32_t nz);
int mmp_batch_synchronize(mmp_batch* b);
int mmp_batch_get_result(mmp_batch* b, uint32_t index, double* out);
int mmp_batch_set_fields(mmp_batch* b, uint32_t index, const double* phi0);
int mmp_batch_get_info(mmp_batch* b, uint32_t index, mmp_info* info);
uint32_t mmp_batch_size(const mmp_batch* b);
/* mmp_set_energy_drift_limit for member `index`. */
int mmp_batch_set_energy_drift_limit(mmp_batch* b, uint32_t index, double rel_tol);
void mmp_batch_destroy(mmp_batch* b);

/* ---- serving: a request loop with continuous batching ---------------------------------
 * No counterpart in the reference (one solve per process). A worker thread owns the
 * device. Requests are grouped by kernel shape (nt, precision, Raman, RK tableau, and the
 * contraction form and tile each would get alone) into
 * slot pools; each pool advances all its solves with one captured multi-step CUDA
 * graph per replay on its own stream, so different pools overlap on the device.
 * Between replays the worker retires finished solves (their result is copied to host
 * memory) and admits waiting ones into free slots, first fit, as long as the device
 * memory they need stays within the budget. Each solve stops at its own n_steps on
 * the device. Results equal, bit for bit, those of mmp_solver_create +
 * mmp_propagate(n_steps) + mmp_get_result for the same parameters. */
typedef struct mmp_server mmp_server;
typedef struct mmp_server_config {
  uint64_t memory_budget;   /* device bytes for solve state; 0 = 80% of free memory */
  uint32_t max_slots;       /* solves per pool; 0 = 64 */
  uint32_t steps_per_tick;  /* RK steps per graph replay; 0 = 32 */
  uint32_t flags;           /* MMP_F_* OR-ed into every request's flags */
} mmp_server_config;
typedef struct mmp_request_info {
  int32_t status;           /* MMP_OK, or the error the solve ended with */
  uint32_t n_modes, nt;
  uint64_t steps;           /* RK steps run */
  double submit_s, start_s, done_s; /* seconds since the server was created */
} mmp_request_info;
int mmp_server_create(const mmp_server_config* cfg, mmp_server** out);
/* Copies the parameters (and their arrays); returns at once with a request id. */
int mmp_server_submit(mmp_server* s, const mmp_params* params, uint64_t* id);
/* *done = 1 once the request has finished (successfully or not). */
int mmp_server_poll(mmp_server* s, uint64_t id, int* done);
/* Wait up to timeout_s seconds (< 0: no limit) for the request; then copy its result
 * phi[M][NT][2] into out (if not NULL) and its info, and forget the request.
 * MMP_ETIMEOUT if it did not finish in time (it stays queued). */
int mmp_server_wait(mmp_server* s, uint64_t id, double timeout_s, double* out, mmp_request_info* info);
/* Stops the worker; unfinished requests are dropped. NULL is allowed. */
void mmp_server_destroy(mmp_server* s);

/* ---- measurement (no counterpart in the reference, which has no timing code) --------- */
/* `repeats` calls of mmp_batch_propagate_async(b, nz) bracketed by CUDA events on the
 * batch's own stream; *ms receives the device time between the events. */
int mmp_batch_propagate_timed(mmp_batch* b, uint32_t nz, uint32_t repeats, double* ms);
/* nz steps launched one kernel at a time (no graph) with an event pair around every
 * launch; ms_per_launch[kind] is the mean device time of one launch and launches[kind]
 * the count, kind 0 = pair fields (Raman), 1 = contraction, 2 = per-mode transform
 * kernel. Numerically identical to mmp_batch_propagate. */
int mmp_batch_profile(mmp_batch* b, uint32_t nz, double* ms_per_launch, uint32_t* launches);

/* ---- Runge–Kutta tableaus ---------------------------------------------------------- */
/* Butcher4 / Butcher7(nu=1) / Butcher11 / Butcher7(lambda, mu) (include/RungeKutta.hpp:10-22,
 * src/RungeKutta.cpp:3-175), selected as the solver selects them from method_order and
 * rk_variant. Writes the stage count to *s and a (row-major 11x11, zero-padded), b[11],
 * c[11]; any of a, b, c may be NULL. */
int mmp_tableau(uint32_t method_order, int32_t rk_variant, double rk_lambda, double rk_mu,
                uint32_t* s, double* a, double* b, double* c);

/* ---- the transform on its own ------------------------------------------------------ */
/* Forward_DFT::compute / Inverse_DFT::compute (include/DiscreteFourierTransform.hpp:28-45,
 * src/DiscreteFourierTransform.cpp:24-38), batched over `rows` rows of n samples on the
 * device, through the same FFT code the solver uses. in/out are [rows][n][2] host
 * buffers (may alias). direction -1: unnormalised forward transform; +1: inverse scaled
 * by 1/n, as the reference's Inverse_DFT. fp64 = 0 transforms in FP32, 1 in FP64. */
int mmp_dft(uint32_t n, uint32_t rows, int direction, int fp64, const double* in, double* out);

/* No counterpart in the reference. The same transform as mmp_dft (same arguments,
 * same results) for callers that must not allocate device memory when they call it:
 * a host whose device memory pool belongs to its own caching allocator, a loop that
 * cannot take the device synchronisation a cudaMalloc/cudaFree pair may cause, or a
 * plugin with a memory budget fixed at load time. mmp_dft allocates device copies of
 * in/out on every call; this one stages them in a static device array of about
 * 19 MiB (twiddle tables plus room for 2^20 complex FP64 samples) that every GPU
 * loading the library holds until exit, and calls no cudaMalloc or cudaFree.
 * rows * n above 2^20 returns MMP_EINVAL. The first call on a device (with it
 * current) looks up the array's device address and fills the twiddle tables with a
 * kernel launch: make that first call before any stream capture. All calls on a
 * device share the staging buffer, which keeps the last call's data; calls that
 * overlap on the GPU race, so serialise calls from several host threads. */
int mmp_dft_noalloc(uint32_t n, uint32_t rows, int direction, int fp64, const double* in, double* out);

/* ---- library facts ----------------------------------------------------------------- */
const char* mmp_strerror(int code);
/* Text of the last failure on the calling thread (empty when none). */
const char* mmp_last_error(void);
const char* mmp_version(void);
/* Number of this library's kernels launched so far in this process (all devices). */
uint64_t mmp_kernel_launch_count(void);

/* ---- test hooks (no counterpart in the reference) -------------------------------------
 * Allocation-failure injection: after `after` more successful device allocations by
 * this library, the next one fails as if the device were out of memory (the call that
 * made it returns MMP_ENOMEM); after < 0 turns injection off. One-shot. */
int mmp_debug_fail_alloc(int64_t after);
/* Device allocations this library holds (made and not yet freed), all devices: for
 * checking that a failed call leaks nothing. Includes one twiddle table per device.
 * The environment variable MMP_TILE_WAIT_POLLS, read when a solve is created, sets how
 * many polls the contraction kernels give the first wait for their tile copy (default
 * 2^24, far above any copy time); 0 makes that bounded wait give up at once, so the
 * propagate call reports MMP_ETIMEOUT (the copies still land before a CTA leaves). */
int64_t mmp_debug_live_allocations(void);

#ifdef __cplusplus
}
#endif

#endif /* MMP_B200_H */
