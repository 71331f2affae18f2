/*
 * mmb200 — B200 (sm_100a) implementation of MicroMagnum's effective-field + LLG + Runge-Kutta
 * hot path, behind a C ABI.
 *
 * Conventions shared by every entry point
 *  - Grids are nx*ny*nz cells, linear index i = z*nx*ny + y*nx + x (x fastest), the layout of
 *    the reference's Matrix/VectorMatrix (src/magneto/mmm/exchange/exchange_cpu.cpp:81).
 *  - A vector field is structure-of-arrays: three arrays of N = nx*ny*nz elements back to back
 *    (x components, then y, then z), like the reference's VectorMatrix (matrix/matrix/vector/
 *    VectorMatrix.h:35-79).  Units are the reference's: M and H in A/m, times in seconds.
 *  - All array arguments are DEVICE pointers unless the parameter name ends in `_host`.
 *  - `prec` selects the element type of every array argument of a call: MM_F64 -> double,
 *    MM_F32 -> float.  MM_F64 is the plain mode (the reference's `-G`, CUDA_64), MM_F32 the
 *    single-precision mode (`-g`, CUDA_32).
 *  - `stream` is a cudaStream_t (NULL = legacy default stream).  Calls that return a scalar to
 *    the host synchronise that stream; all others are stream-ordered and return immediately.
 *  - No entry point throws.  Each returns an mm_status; on failure mm_last_error() returns a
 *    message for the calling thread.  The library never falls back to a CPU implementation.
 */
#ifndef MMB200_H
#define MMB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MM_API __attribute__((visibility("default")))
#define MM_ABI_VERSION 1

typedef enum {
	MM_OK = 0,
	MM_ERR_INVALID_ARGUMENT = 1,  /* bad sizes, null pointers, unknown enum value */
	MM_ERR_CUDA = 2,              /* a CUDA runtime call or kernel launch failed */
	MM_ERR_OUT_OF_MEMORY = 3,     /* device allocation failed */
	MM_ERR_UNSUPPORTED = 4,       /* valid request the library does not implement */
	MM_ERR_NOT_FINITE = 5,        /* NaN/Inf detected in a solver state */
	MM_ERR_TIMEOUT = 6            /* a bounded device-side wait gave up */
} mm_status;

typedef enum { MM_F64 = 0, MM_F32 = 1 } mm_precision;

/* Padding strategies of the demag tensor (src/magneto/mmm/demag/tensor_round.h; same values as
 * the reference's PADDING_* enum exported at bindings/mmm/demag.i:27-42). */
typedef enum {
	MM_PADDING_DISABLE = 0,
	MM_PADDING_ROUND_2 = 1,
	MM_PADDING_ROUND_4 = 2,
	MM_PADDING_ROUND_8 = 3,
	MM_PADDING_ROUND_POT = 4,
	MM_PADDING_SMALL_PRIME_FACTORS = 5
} mm_padding;

/* Message describing the last failure on the calling thread ("" if none). */
MM_API const char *mm_last_error(void);
MM_API int mm_abi_version(void);
/* Number of kernels this library has launched in the process (for launch accounting). */
MM_API uint64_t mm_kernel_launch_count(void);

/* Per-kernel timing of the solver and convolution kernels (no counterpart in the reference,
 * whose --prof switch times host sections, Benchmark.cpp:53-109).  When enabled, each launch is
 * bracketed by CUDA events on its stream; mm_profile_get() synchronises and returns, per kernel
 * name, the launch count, the summed device time and the summed algorithmic bytes (each array
 * element crossing HBM once per launch).  Not thread-safe across concurrent solvers. */
MM_API mm_status mm_profile_enable(int on);
MM_API mm_status mm_profile_reset(void);
MM_API int mm_profile_count(void);
MM_API mm_status mm_profile_get(int index, const char **name, int64_t *launches, double *total_ms,
                                double *bytes);

/* ---------------------------------------------------------------------------------------------
 * Field terms: one call per term, same arguments and results as the reference's magneto calls.
 * ------------------------------------------------------------------------------------------- */

/* Exchange field, 6-neighbour stencil, Neumann boundaries, neighbours with Ms == 0 skipped,
 * optional periodic boundaries.  Replaces magneto.exchange (bindings/mmm/exchange.i:24-39 ->
 * mmm/exchange/exchange.cpp:31-58).  If energy_host is non-NULL, *energy_host receives
 * -mu0/2 * dx*dy*dz * sum_i M_i.H_i (the CUDA path's return value, exchange_cuda.cu:456). */
MM_API mm_status mm_exchange(int prec, int nx, int ny, int nz, double dx, double dy, double dz,
                             int pbc_x, int pbc_y, int pbc_z, const void *Ms, const void *A,
                             const void *M, void *H, double *energy_host, void *stream);

/* Uniaxial anisotropy H = 2 k (m.a) a / (mu0 Ms), zero where Ms == 0 or k == 0.  Replaces
 * magneto.uniaxial_anisotropy (bindings/mmm/anisotropy.i:24-31 -> mmm/anisotropy/
 * anisotropy.cpp:33-58).  energy_host (optional) receives sum_i k_i |a_i x m_i|^2, the CPU
 * path's return value (anisotropy_cpu.cpp:64-68). */
MM_API mm_status mm_uniaxial_anisotropy(int prec, size_t n, const void *axis, const void *k,
                                        const void *Ms, const void *M, void *H,
                                        double *energy_host, void *stream);

/* Cubic anisotropy (axis3 = axis1 x axis2).  Replaces magneto.cubic_anisotropy
 * (anisotropy.i:32-39 -> anisotropy.cpp:60-88).  energy_host (optional) receives
 * sum_i k_i (a1^2 a2^2 + a1^2 a3^2 + a2^2 a3^2). */
MM_API mm_status mm_cubic_anisotropy(int prec, size_t n, const void *axis1, const void *axis2,
                                     const void *k, const void *Ms, const void *M, void *H,
                                     double *energy_host, void *stream);

/* LLG right-hand side dM = f1 M x H + f2 M x (M x H).  Replaces magneto.llge
 * (bindings/mmm/llge.i:24-29 -> mmm/llge/llge.cpp:33-59). */
MM_API mm_status mm_llge(int prec, size_t n, const void *f1, const void *f2, const void *M,
                         const void *H, void *dM, void *stream);

/* Zhang-Li spin-transfer torque, finite differences of M (one-sided at the edges, zero along a
 * dimension of size 1).  Replaces magneto.fdm_zhangli (bindings/mmm/zhangli.i:24-32 ->
 * mmm/spintorque/fdm_zhangli.cpp:33-53). */
MM_API mm_status mm_fdm_zhangli(int prec, int nx, int ny, int nz, double dx, double dy,
                                double dz, int do_precess, const void *P, const void *xi,
                                const void *Ms, const void *alpha, const void *j,
                                const void *M, void *dM, void *stream);

/* max_i |M_i| / scale_i over cells with scale_i != 0.  Replaces magneto.scaled_abs_max
 * (bindings/math.i:66 -> math/ScaledAbsMax.cpp:52-68).  Synchronises `stream`. */
MM_API mm_status mm_scaled_abs_max(int prec, size_t n, const void *M, const void *scale,
                                   double *result_host, void *stream);

/* The same result as mm_scaled_abs_max, computed without allocating any memory.  No counterpart
 * in the reference: it exists for callers that must not allocate once their set-up is done, such
 * as a process whose free device memory is already reserved by a pool (a late cudaMalloc would
 * fail there) or a step loop that must not meet the synchronisation a cudaMalloc/cudaMallocHost
 * can imply; mm_scaled_abs_max allocates a device accumulator and a pinned host word on its
 * first call on each device.  Scratch is a fixed 512 KiB array in the library's static device
 * memory: at most 65536 partial maxima of 4096 cells, so n is limited to 268,435,456 cells and
 * larger n returns MM_ERR_INVALID_ARGUMENT.  Nothing in the scratch has to start at zero.  The
 * first call on each device (with that device current) looks up the array's address; make it
 * during set-up, before any stream capture.  That address is kept for the life of the process:
 * a cudaDeviceReset discards the library's device memory and leaves it stale, so a process that
 * resets a device must not call this entry point on it afterwards.  Every call on a device uses
 * the same array, so calls that overlap on the device (other streams, other host threads) race:
 * serialise them.
 * Synchronises `stream`. */
MM_API mm_status mm_scaled_abs_max_noalloc(int prec, size_t n, const void *M, const void *scale,
                                           double *result_host, void *stream);

/* sqrt(mean over the 3n equations of (|y_error_i| / (eps_rel |y_i| + eps_abs))^2), the scaled
 * error norm behind rk_adjust_stepsize (evolver/runge_kutta.cpp:98-130 ->
 * evolver/runge_kutta_cpu.cpp:196-252, Euclidean branch; the reference asserts when CUDA is enabled,
 * this computes it on the device).  Synchronises `stream`. */
MM_API mm_status mm_rk_scaled_error_norm(int prec, size_t n, double eps_abs, double eps_rel, const void *y,
                                         const void *y_error, double *norm_host, void *stream);

/* M_i <- Ms_i M_i / |M_i| (0 where |M_i| == 0).  Replaces VectorMatrix::normalize(Matrix)
 * (matrix/matrix/vector/VectorMatrix.cpp:218-230) as called by the solver after every accepted
 * step (magnum/micromagnetics/micro_magnetics.py:49-50). */
MM_API mm_status mm_normalize(int prec, size_t n, const void *Ms, void *M, void *stream);

/* Runge-Kutta stage state ytmp = y + h * sum_{j<step} b[step][j] k_j and the final combination
 * y += h sum c_j k_j, y_error = h sum ec_j k_j, for any explicit tableau with up to 8 stages.
 * `b` is the row b[step][0..step-1]; k is an array of `nk` device pointers (host array).
 * Replaces magneto.rk_prepare_step / rk_combine_result (bindings/evolver.i:63-92 ->
 * evolver/runge_kutta.cpp:32-96). */
MM_API mm_status mm_rk_prepare_step(int prec, size_t n, int step, double h, const double *b_host,
                                    const void *const *k_host, const void *y, void *ytmp,
                                    void *stream);
MM_API mm_status mm_rk_combine_result(int prec, size_t n, int nk, double h, const double *c_host,
                                      const double *ec_host, const void *const *k_host, void *y,
                                      void *y_error, void *stream);

/* ---------------------------------------------------------------------------------------------
 * Demagnetisation: tensor and zero-padded FFT convolution.
 * ------------------------------------------------------------------------------------------- */

/* Padded FFT length of one dimension: the reference's round_tensor_dimension
 * (mmm/demag/tensor_round.cpp:90-106). */
MM_API int mm_round_tensor_dimension(int dim, int periodic, int padding);

/* Newell demagnetisation tensor, already negated (H = N * M), computed on the GPU in FP64 into
 * N_out (device, 6*ex*ey*ez doubles, component index fastest then x, y, z: the reference's
 * Matrix(Shape(6, ex, ey, ez)) layout, mmm/demag/tensor.cpp:41,167-180).  ex/ey/ez are the
 * padded sizes (mm_round_tensor_dimension).  Replaces magneto.GenerateDemagTensor
 * (bindings/mmm/demag.i:27-42 -> mmm/demag/demag_tensor.cpp:116-186) for non-periodic meshes
 * (padded sizes below 2n - 1 return MM_ERR_UNSUPPORTED; mm_demag_tensor_periodic takes them). */
MM_API mm_status mm_demag_tensor(int nx, int ny, int nz, double dx, double dy, double dz,
                                 int ex, int ey, int ez, double *N_out, void *stream);

/* The demag tensor with periodic boundaries along the axes whose pbc_* is set (e == n there,
 * e >= 2n - 1 elsewhere; round_tensor_dimension), `repeat` periodic images per periodic axis and
 * the sum of the images beyond them (the reference's infinity correction, switched off like the
 * reference's by the environment variable MAGNUM_DEMAG_NO_INFINITY_CORRECTION).  Replaces
 * GenerateDemagTensor / calculateDemagTensor for periodic meshes (mmm/demag/demag_tensor.cpp:116-186,
 * mmm/demag/tensor.cpp:35-191).  Without periodic axes it is mm_demag_tensor.  Stream-ordered. */
MM_API mm_status mm_demag_tensor_periodic(int nx, int ny, int nz, double dx, double dy, double dz, int pbc_x,
                                          int pbc_y, int pbc_z, int repeat, int ex, int ey, int ez, double *N_out,
                                          void *stream);

/* Zero-padded FFT convolution H = N * M with a symmetric tensor field.  Replaces
 * magneto.SymmetricMatrixVectorConvolution_FFT (bindings/math.i:27-33 ->
 * math/conv/SymmetricMatrixVectorConvolution_FFT.cpp:31-65, MatrixVectorConvolution_FFT.cpp:
 * 110-375).  N_device is the tensor in the layout of mm_demag_tensor (FP64); the plan keeps its
 * spectrum in working precision `prec` and owns its scratch.  execute() takes M and writes H in
 * `prec`. */
typedef struct mm_conv mm_conv;
MM_API mm_status mm_conv_create(mm_conv **out, int prec, int nx, int ny, int nz, int ex, int ey,
                                int ez, const double *N_device, void *stream);
MM_API mm_status mm_conv_execute(mm_conv *conv, const void *M, void *H, void *stream);
MM_API mm_status mm_conv_destroy(mm_conv *conv);

/* ---------------------------------------------------------------------------------------------
 * Solver: the fused B200 path.  State, stage vectors, demag spectra and the step controller live
 * on the device; one call advances the state by whole Runge-Kutta steps with the reference's
 * semantics (magnum/evolver/runge_kutta.py:47-137 with MicroMagneticsStepSizeController,
 * magnum/micromagnetics/micro_magnetics_stepsize_controller.py:35-73).
 * ------------------------------------------------------------------------------------------- */

/* Per-region material.  Every cell carries a region index (uint8) into a table of these. */
typedef struct {
	double Ms;             /* saturation magnetisation [A/m]; 0 marks empty cells */
	double A;              /* exchange stiffness [J/m] */
	double alpha;          /* Gilbert damping */
	double k_uniaxial;     /* uniaxial anisotropy constant [J/m^3] */
	double k_cubic;        /* cubic anisotropy constant [J/m^3] */
	double axis1[3];       /* uniaxial axis / first cubic axis */
	double axis2[3];       /* second cubic axis */
	double P;              /* spin polarisation (Zhang-Li) */
	double xi;             /* non-adiabaticity (Zhang-Li) */
	double j[3];           /* current density [A/m^2] (Zhang-Li) */
} mm_material;

typedef enum {
	MM_RK_RKF45 = 0, MM_RK_CC45 = 1, MM_RK_DP54 = 2, MM_RK_RK23 = 3
} mm_tableau;

enum {
	MM_TERM_DEMAG = 1, MM_TERM_EXCHANGE = 2, MM_TERM_UNIAXIAL = 4, MM_TERM_CUBIC = 8,
	MM_TERM_ZHANGLI = 16, MM_TERM_ZEEMAN = 32
};

typedef struct {
	int nx, ny, nz;
	double dx, dy, dz;
	int precision;          /* mm_precision */
	int tableau;            /* mm_tableau */
	int terms;              /* MM_TERM_* bit set */
	int do_precess;         /* LLG precession term (LandauLifshitzGilbert(do_precess)) */
	int zl_do_precess;      /* Zhang-Li precession variant (SpinTorque(do_precess)) */
	int padding;            /* mm_padding for the demag tensor */
	double eps_abs, eps_rel;/* MicroMagneticsStepSizeController tolerances */
	double h0;              /* first step size tried (MicroMagnetics.createState: 1e-13) */
	/* Uniform applied field H(t) = H_ext + H_pulse * min(t / pulse_rise, 1) [A/m];
	 * pulse_rise <= 0 means a static H_ext + H_pulse. */
	double H_ext[3];
	double H_pulse[3];
	double pulse_rise;
	/* 1 (default semantics of the reference): after a rejected step the next attempt reuses the
	 * rejected attempt's last stage as its first (runge_kutta.py:67-70,99-100,131-134).
	 * 0: re-evaluate the first stage after a rejection. */
	int fsal_reuse_after_reject;
	/* Periodic boundaries (the mesh's periodic_bc, RectangularMesh.h:23-26): pbc[a] != 0 makes
	 * axis a periodic for the exchange stencil and the demag tensor (no zero padding along it);
	 * pbc_repeat is the number of periodic images, <= 0 for the reference's defaults 15, 3, 2 for
	 * one, two, three periodic axes (RectangularMesh.h:10-19).  The Zhang-Li gradient stays
	 * one-sided at the box faces, as in the reference (fdm_zhangli_cpu.cpp:100-200). */
	int pbc[3];
	int pbc_repeat;
} mm_solver_config;

typedef struct {
	double t;              /* simulation time [s] */
	double h;              /* last accepted step size */
	double h_next;         /* step size the next attempt will try */
	int64_t steps;         /* accepted steps */
	int64_t attempts;      /* attempts including rejected ones */
	int64_t rejected;      /* rejected attempts */
	double last_error;     /* e_abs of the last attempt (max |m_err|) */
	double last_max_dmdt;  /* max |dm/dt| of the last attempt [rad/s] */
	int not_finite;        /* 1 if a NaN/Inf was seen in the last attempt */
	int stage_kernel;      /* fused stage kernel in use: 0 per-thread loads, 1 staged (run-time
	                        * terms), 2 staged for the term set, 3 staged for the term set and the
	                        * Dormand-Prince stage patterns */
} mm_solver_stats;

typedef struct mm_solver mm_solver;

/* regions_host: N region indices (NULL: every cell region 0); materials_host: num_materials
 * entries (<= 256).  tensor_device: optional FP64 tensor in the mm_demag_tensor layout for the
 * padded sizes of config->padding (NULL: generate it on the GPU). */
MM_API mm_status mm_solver_create(mm_solver **out, const mm_solver_config *config,
                                  int num_materials, const mm_material *materials_host,
                                  const uint8_t *regions_host, const double *tensor_device,
                                  void *stream);
MM_API mm_status mm_solver_destroy(mm_solver *s);

/* Set / read the magnetisation M [A/m] (FP64 device arrays, SoA).  set_M re-normalises to Ms
 * like LandauLifshitzGilbert.update("M") (landau_lifshitz_gilbert.py:84-88), resets t and the
 * step counters, and forgets the first-same-as-last stage. */
MM_API mm_status mm_solver_set_M(mm_solver *s, const double *M_device, void *stream);
MM_API mm_status mm_solver_get_M(mm_solver *s, double *M_device, void *stream);
/* Replace the state by M (normalised to Ms) keeping t, the step size, the counters and the
 * first-same-as-last stage: for callers that keep M in their own buffers between steps. */
MM_API mm_status mm_solver_load_M(mm_solver *s, const double *M_device, void *stream);
MM_API mm_status mm_solver_set_time(mm_solver *s, double t, double h_next, void *stream);

/* One accepted step toward t_max: RungeKutta.evolve(state, t_max) (runge_kutta.py:47-87)
 * followed by finish_step (normalisation).  Synchronises `stream`. */
MM_API mm_status mm_solver_step(mm_solver *s, double t_max, void *stream);

/* Advance until t >= t_end (condition.Time), clamping steps to every multiple of
 * sample_dt (> 0; condition.EveryNthSecond) and writing <M> [A/m] at each such time into
 * samples_host (3 doubles per sample, at most max_samples) with the time into
 * sample_t_host.  *num_samples receives the count.  Pass sample_dt <= 0 for no sampling. */
MM_API mm_status mm_solver_run(mm_solver *s, double t_end, double sample_dt,
                               double *sample_t_host, double *samples_host, int max_samples,
                               int *num_samples, void *stream);

/* One Runge-Kutta attempt with step size h from the current state, with no state update
 * (used for throughput measurement).  Stream-ordered; no host synchronisation. */
MM_API mm_status mm_solver_attempt(mm_solver *s, double h, void *stream);

/* Effective field H_eff [A/m] and dM/dt [A/(m s)] at the current state (FP64 device arrays,
 * either may be NULL), with H_demag alone optionally into H_demag_device. */
MM_API mm_status mm_solver_eval(mm_solver *s, double *H_eff_device, double *dMdt_device,
                                double *H_demag_device, void *stream);

MM_API mm_status mm_solver_stats_get(mm_solver *s, mm_solver_stats *out, void *stream);

/* Relaxation norms of the current state (one RHS evaluation): norms_host3[0] = max |dM/dt|
 * [A/(m s)] (state.dMdt.absMax()), [1] = max |M| [A/m] (state.M.absMax()), [2] = max over cells
 * with Ms != 0 of |m x H_eff| / Ms (dimensionless torque).  Synchronises `stream`. */
MM_API mm_status mm_solver_relax_norms(mm_solver *s, double *norms_host3, void *stream);

/* Energies of the current state in J: energies_host5 = {E_stray, E_exch, E_aniso, E_ext, E_tot}
 * (E_stray = -mu0/2 V sum M.H_stray, stray_field.py:49-52; E_exch = -mu0/2 V sum M.H_exch,
 * exchange_field.py:57-58; E_aniso = V times the anisotropy functions' return values on the CPU
 * path, anisotropy_field.py:84-87 with anisotropy_cpu.cpp:29-119; E_ext = -mu0 V sum M.H_ext,
 * external_field.py:34-35; E_tot their sum, landau_lifshitz_gilbert.py:103-106).  Terms the
 * solver was not created with contribute 0.  One demag evaluation; synchronises `stream`. */
MM_API mm_status mm_solver_energies(mm_solver *s, double *energies_host5, void *stream);

enum { MM_RELAX_DEG_PER_NS = 0, MM_RELAX_TORQUE = 1 };

/* Steps (t_max = 1e100, like Solver.solve with a condition that has no time of interest) until
 * the state is relaxed, checking every check_every_nth_step-th step (state.step % n == 0).
 * MM_RELAX_DEG_PER_NS replaces condition.Relaxed(max_degree_per_ns = threshold,
 * check_every_nth_step) (magnum/solver/condition.py:169-200, deg_per_ns from
 * landau_lifshitz_gilbert.py:127-131): relaxed when deg/ns <= threshold and smaller than at the
 * previous check of this call.  MM_RELAX_TORQUE: relaxed when max |m x H_eff| / Ms < threshold
 * (no reference counterpart; the batched-relaxation criterion).  max_steps < 0: no limit.
 * *relaxed = 1 when the criterion was met; *last_value (optional) = the last deg/ns or torque. */
MM_API mm_status mm_solver_relax(mm_solver *s, int criterion, double threshold, int check_every_nth_step,
                                 long long max_steps, int *relaxed, double *last_value, void *stream);

/* <M> [A/m] averaged over all cells (VectorMatrix::average). Synchronises `stream`. */
MM_API mm_status mm_solver_average_M(mm_solver *s, double *avg_host3, void *stream);

/* ---------------------------------------------------------------------------------------------
 * Batched solves (no reference counterpart: the reference runs one world at a time).
 * Many independent instances of uneven size advance in lock step, one Runge-Kutta attempt per
 * round for every running instance, as grouped launches (one per pass and transform length for
 * the demag convolution, one per stage for the fused stage kernel) replayed from CUDA graphs; step
 * control, the accept step and the stop test run on the device per instance.  Instances occupy
 * slots; they can be added and removed between rounds (the rounds are rebuilt on the next call).
 * Each instance: a box of nx*ny*nz cells with a material mask (1: material with Ms, A, alpha;
 * 0: empty), demag + exchange + LLG (+ Zeeman: H_ext + H_pulse ramped linearly over pulse_rise,
 * the reference's AlternatingField/HomogeneousField ramp), dp54 with the reference's step-size
 * controller, power-of-two padding (a single layer is padded to 2 in z).  Stop test: t_end > 0
 * stops at t = t_end (the step that would pass it is clamped onto it); t_end = 0 stops at the
 * first accepted step whose step count is a multiple of check_every_nth_step and whose state has
 * max |m x H_eff| / Ms < max_torque (H_eff evaluated at the accepted state).
 * ------------------------------------------------------------------------------------------- */
typedef struct {
	int nx, ny, nz;
	double dx, dy, dz;
	double Ms, A, alpha;
	double H_ext[3];      /* A/m */
	double H_pulse[3];    /* A/m, reached after pulse_rise seconds */
	double pulse_rise;
	double t_end;         /* 0: relax (torque test) */
} mm_batch_instance;

typedef struct {
	int precision;            /* MM_F32 (compensated state) or MM_F64 */
	double eps_abs, eps_rel;  /* MicroMagneticsStepSizeController tolerances */
	double h0;                /* first step size */
	double max_torque;        /* stop threshold of max |m x H_eff| / Ms */
	int check_every_nth_step;
} mm_batch_config;

typedef struct {
	int status;               /* -1 free slot, 0 running (or not started), 1 finished, 2 non-finite state */
	int steps, attempts, rejected;
	double t, h;
} mm_batch_result;

typedef struct mm_batch mm_batch;

/* Device bytes one instance keeps resident and the extra transient peak of its set-up. */
MM_API mm_status mm_batch_instance_bytes(const mm_batch_instance *instance, int precision,
                                         size_t *resident, size_t *transient);
/* count instances in slots 0..count-1 (count may be 0); masks_host: their masks back to back
 * (N_i bytes each, 0/1), NULL = all material.  An instance runs once it has a state (set_M). */
MM_API mm_status mm_batch_create(mm_batch **out, const mm_batch_config *config, int count,
                                 const mm_batch_instance *instances_host, const uint8_t *masks_host,
                                 void *stream);
MM_API mm_status mm_batch_destroy(mm_batch *b);
/* A new instance in a free slot (*slot_out); its tensor and spectra are built on `stream`, which
 * may run while rounds of the other instances are on the device. */
MM_API mm_status mm_batch_add(mm_batch *b, const mm_batch_instance *instance, const uint8_t *mask_host,
                              int *slot_out, void *stream);
MM_API mm_status mm_batch_remove(mm_batch *b, int slot);
MM_API int mm_batch_slot_count(mm_batch *b);
/* M of the instance in `slot` (FP64 device array, A/m, normalised to Ms); it (re)starts at t = 0
 * with step size h0 in the next round. */
MM_API mm_status mm_batch_set_M(mm_batch *b, int slot, const double *M_device, void *stream);
MM_API mm_status mm_batch_get_M(mm_batch *b, int slot, double *M_device, void *stream);
MM_API mm_status mm_batch_stop(mm_batch *b, int slot, void *stream);
/* Runs at most max_rounds rounds, checking every check_interval rounds (small device-to-host
 * copies) whether any instance still runs.  *rounds_out: rounds run.  Synchronises `stream`. */
MM_API mm_status mm_batch_relax(mm_batch *b, long long max_rounds, int check_interval,
                                long long *rounds_out, void *stream);
/* One result per slot (mm_batch_slot_count entries). */
MM_API mm_status mm_batch_results(mm_batch *b, mm_batch_result *results_host, void *stream);
/* Kernel launches in one captured round (with and without k_0 evaluations). */
MM_API mm_status mm_batch_launches_per_round(mm_batch *b, int *first, int *later);

/* ---- OMF 1.0 vector-field files (rectangular mesh, one segment) ------------------------------
 * Replace readOMF / writeOMF / OMFHeader (bindings/mmm/io.i; mmm/io/OMFImport.cpp,
 * OMFExport.cpp, OMFHeader.h) for device fields: requests and results of the served solves and
 * the reference's own fixture files.  Text, binary-4 and binary-8 data blocks; binary values are
 * big-endian after the big-endian check value (1234567.0 / 123456789012345.0).  The reference's
 * writer leaves binary-8 values in host byte order (OMFExport.cpp:171-177), which its own reader
 * does not read back on a little-endian host; this writer follows the format. */
typedef enum { MM_OMF_TEXT = 0, MM_OMF_BINARY_4 = 1, MM_OMF_BINARY_8 = 2 } mm_omf_format_t;

typedef struct {
	char title[256];
	char desc[4096];               /* the Desc lines, separated by '\n' */
	char meshunit[64], valueunit[64], meshtype[64];
	double valuemultiplier;
	double xmin, ymin, zmin, xmax, ymax, zmax;
	double ValueRangeMaxMag, ValueRangeMinMag;
	double xbase, ybase, zbase;
	double xstepsize, ystepsize, zstepsize;
	int xnodes, ynodes, znodes;
	int format;                    /* set by the readers: the data block's mm_omf_format_t */
} mm_omf_header;

/* Parses an OMF file held in host memory.  M NULL: the header only.  Otherwise M receives the
 * field (3 * xnodes*ynodes*znodes elements of `prec`, SoA, x fastest) times valuemultiplier, like
 * readOMF (OMFImport.cpp:294-440).  Synchronises `stream`. */
MM_API mm_status mm_omf_parse(const void *bytes_host, size_t length, mm_omf_header *header, int prec, void *M,
                              void *stream);
/* mm_omf_parse of the file at `path`. */
MM_API mm_status mm_omf_read(const char *path, mm_omf_header *header, int prec, void *M, void *stream);
/* Formats the field M (header's xnodes*ynodes*znodes cells) as an OMF file in `format`, with the
 * reference's header lines, scaling (values divided by max |M| when it exceeds 0.001, unless
 * MAGNUM_OMF_NOSCALE is set) and 16 significant digits for text (OMFExport.cpp:55-209).  Sets
 * header->valuemultiplier, ValueRangeMaxMag and ValueRangeMinMag.  *bytes_host is allocated by
 * the library: release it with mm_omf_free.  Synchronises `stream`. */
MM_API mm_status mm_omf_format(mm_omf_header *header, int prec, const void *M, int format, char **bytes_host,
                               size_t *length, void *stream);
MM_API void mm_omf_free(char *bytes_host);
/* mm_omf_format written to the file at `path`. */
MM_API mm_status mm_omf_write(const char *path, mm_omf_header *header, int prec, const void *M, int format,
                              void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MMB200_H */
