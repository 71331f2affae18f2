/*
 * Oracle (TEST INFRASTRUCTURE ONLY): a CPU restatement, in plain C, of the reference
 * (MicroMagnum 0.2rc3) algorithms on the effective-field + LLG + Runge-Kutta path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, as the checker; the product
 * (micromagnum_b200, libmmb200.so) never links or calls it.
 *
 * Parity pinning: every function is checked in tests/ against the reference's own golden
 * fixtures (the OMF files under src/magnum_tests/ref, converted by tests/golden/make_golden.py), its
 * known-answer tests, and against the reference's own CPU C++ compiled in place into
 * oracle/_ref/libmmref.so (oracle/Makefile).
 *
 * Arrays are host double arrays in the reference layout: vector fields SoA (x[N], y[N], z[N]),
 * cell index i = z*nx*ny + y*nx + x; the demag tensor is (component, x, y, z) with the component
 * index fastest, components (xx, xy, xz, yy, yz, zz).
 */
#ifndef MM_ORACLE_H
#define MM_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

void or_set_threads(int n);

double or_exchange(int nx, int ny, int nz, double dx, double dy, double dz, int px, int py, int pz,
                   const double *Ms, const double *A, const double *M, double *H);
double or_uniaxial_anisotropy(size_t n, const double *axis, const double *k, const double *Ms,
                              const double *M, double *H);
double or_cubic_anisotropy(size_t n, const double *axis1, const double *axis2, const double *k,
                           const double *Ms, const double *M, double *H);
void or_llge(size_t n, const double *f1, const double *f2, const double *M, const double *H,
             double *dM);
void or_fdm_zhangli(int nx, int ny, int nz, double dx, double dy, double dz, int do_precess,
                    const double *P, const double *xi, const double *Ms, const double *alpha,
                    const double *j, const double *M, double *dM);
double or_scaled_abs_max(size_t n, const double *M, const double *scale);
void or_normalize(size_t n, const double *Ms, double *M, int float_norm);

int or_round_tensor_dimension(int dim, int periodic, int padding);
/* Newell tensor (negated, H = N * M), non-periodic, evaluated in binary128. */
void or_demag_tensor(int nx, int ny, int nz, double dx, double dy, double dz, int ex, int ey,
                     int ez, double *out);
/* H = N * M by direct summation (long double accumulation). */
void or_conv_direct(const double *N, int nx, int ny, int nz, int ex, int ey, int ez,
                    const double *M, double *H);
/* H = N * M by zero-padded FFTs (double), the reference CPU conv's arithmetic. */
void or_conv_fft(const double *N, int nx, int ny, int nz, int ex, int ey, int ez,
                 const double *M, double *H);

/* ---- Runge-Kutta solver with the reference's semantics -------------------------------------- */
typedef struct or_solver or_solver;

typedef struct {
	int nx, ny, nz;
	double dx, dy, dz;
	int tableau;            /* 0 rkf45, 1 cc45, 2 dp54, 3 rk23 */
	int terms;              /* 1 demag, 2 exchange, 4 uniaxial, 8 cubic, 16 zhangli, 32 zeeman */
	int do_precess, zl_do_precess;
	double eps_abs, eps_rel, h0;
	double H_ext[3], H_pulse[3], pulse_rise;
	int fsal_reuse_after_reject;
	int float_norm;         /* 1: CPU normalize3 (norm from float-cast components) */
	int use_fft;            /* 1: FFT convolution, 0: direct summation */
	int pbc[3];             /* periodic exchange along x, y, z (exchange_cpu.cpp:141-235); the
	                           tensor passed in carries the periodic demag images */
} or_solver_config;

/* Per-cell parameters (arrays of N; vectors SoA).  tensor: (6, ex, ey, ez) as above. */
or_solver *or_solver_create(const or_solver_config *cfg, const double *Ms, const double *A,
                            const double *alpha, const double *k_uni, const double *k_cub,
                            const double *axis1, const double *axis2, const double *P,
                            const double *xi, const double *j, const double *tensor, int ex,
                            int ey, int ez);
void or_solver_destroy(or_solver *s);
void or_solver_set_M(or_solver *s, const double *M);
void or_solver_get_M(or_solver *s, double *M);
/* H_eff and dM/dt at the current state (either may be NULL); H_demag optional. */
void or_solver_eval(or_solver *s, double *H_eff, double *dMdt, double *H_demag);
/* One RungeKutta.evolve(state, t_max) + finish_step. */
void or_solver_step(or_solver *s, double t_max);
/* Solve until t >= t_end, sampling <M> at multiples of sample_dt (<= 0: none); returns count. */
int or_solver_run(or_solver *s, double t_end, double sample_dt, double *sample_t, double *samples,
                  int max_samples);
/* t, h, h_next, steps, attempts, rejected */
void or_solver_stats(or_solver *s, double *out6);
/* One attempt with step h from the current state (timing); state is left unchanged. */
void or_solver_attempt(or_solver *s, double h);

#ifdef __cplusplus
}
#endif
#endif
