// Test infrastructure only (oracle): a C-ABI wrapper, written for this project, around the
// reference's own CPU implementation (MicroMagnum 0.2rc3, src/magneto/...), compiled in place
// from the reference tree by oracle/Makefile into oracle/_ref/libmmref.so.  Nothing here is
// product code; the CUDA library never links or loads it.
//
// Every entry point takes plain host arrays in the reference's SoA layout
// (index i = z*nx*ny + y*nx + x, one array per vector component) and builds the reference's
// Matrix / VectorMatrix containers around copies of them, then calls the reference function
// named in the comment.
//
// The reference's global switches (isCudaEnabled, profiling, log callback) live in
// src/magneto/Magneto.cpp, which needs FFTW and CUDA headers; the tiny stand-ins below keep the
// CPU path selected (CUDA disabled, profiling off) exactly as `magneto_cpu` would run.

#include "config.h"
#include "matrix/matty.h"
#include "mmm/exchange/exchange_cpu.h"
#include "mmm/anisotropy/anisotropy_cpu.h"
#include "mmm/llge/llge_cpu.h"
#include "mmm/spintorque/fdm_zhangli_cpu.h"
#include "mmm/demag/tensor.h"
#include "mmm/demag/tensor_round.h"
#include "math/conv/SymmetricMatrixVectorConvolution_Simple.h"
#include "math/ScaledAbsMax.h"
#include "evolver/runge_kutta.h"

#include <cstring>
#include <vector>
#include <string>

// ---- stand-ins for src/magneto/Magneto.cpp (CPU mode, no profiling, logging dropped) ----
bool isCudaEnabled() { return false; }
bool isCuda64Enabled() { return false; }
bool haveCudaSupport() { return false; }
bool isProfilingEnabled() { return false; }
void callDebugFunction(int, const std::string &) {}

using namespace matty;

namespace {

// The reference's SWIG module calls matty_initialize() at import (matrix/matty.inc.i:385); the
// shim does the same once, on first use.
void ensure_matty()
{
	static bool done = false;
	if (!done) { matty_initialize(); done = true; }
}

Matrix scalar_field(int nx, int ny, int nz, const double *src)
{
	Matrix m(Shape(nx, ny, nz));
	Matrix::wo_accessor acc(m);
	std::memcpy(acc.ptr(), src, sizeof(double) * (size_t)nx * ny * nz);
	return m;
}

VectorMatrix vector_field(int nx, int ny, int nz, const double *src)
{
	const size_t n = (size_t)nx * ny * nz;
	VectorMatrix v(Shape(nx, ny, nz));
	VectorMatrix::accessor acc(v);
	std::memcpy(acc.ptr_x(), src, sizeof(double) * n);
	std::memcpy(acc.ptr_y(), src + n, sizeof(double) * n);
	std::memcpy(acc.ptr_z(), src + 2 * n, sizeof(double) * n);
	return v;
}

void copy_out(const VectorMatrix &v, double *dst)
{
	const size_t n = v.size();
	VectorMatrix::const_accessor acc(v);
	std::memcpy(dst, acc.ptr_x(), sizeof(double) * n);
	std::memcpy(dst + n, acc.ptr_y(), sizeof(double) * n);
	std::memcpy(dst + 2 * n, acc.ptr_z(), sizeof(double) * n);
}

ButcherTableau tableau(int s, const double *a, const double *b, const double *c, const double *ec)
{
	ButcherTableau tab(s);
	for (int i = 0; i < s; ++i) {
		tab.setA(i, a[i]);
		tab.setC(i, c[i]);
		tab.setEC(i, ec[i]);
		for (int j = 0; j < s; ++j) tab.setB(i, j, b[i * s + j]);
	}
	return tab;
}

} // namespace

extern "C" {

// src/magneto/mmm/exchange/exchange_cpu.cpp:43 exchange_cpu
double mmref_exchange(int nx, int ny, int nz, double dx, double dy, double dz,
                      int px, int py, int pz, const double *Ms, const double *A,
                      const double *M, double *H)
{
	ensure_matty();
	Matrix ms = scalar_field(nx, ny, nz, Ms), a = scalar_field(nx, ny, nz, A);
	VectorMatrix m = vector_field(nx, ny, nz, M);
	VectorMatrix h(Shape(nx, ny, nz));
	const double e = exchange_cpu(nx, ny, nz, dx, dy, dz, px != 0, py != 0, pz != 0, ms, a, m, h);
	copy_out(h, H);
	return e;
}

// src/magneto/mmm/anisotropy/anisotropy_cpu.cpp:29 uniaxial_anisotropy_cpu
double mmref_uniaxial_anisotropy(int nx, int ny, int nz, const double *axis, const double *k,
                                 const double *Ms, const double *M, double *H)
{
	ensure_matty();
	VectorMatrix ax = vector_field(nx, ny, nz, axis), m = vector_field(nx, ny, nz, M);
	Matrix kk = scalar_field(nx, ny, nz, k), ms = scalar_field(nx, ny, nz, Ms);
	VectorMatrix h(Shape(nx, ny, nz));
	const double e = uniaxial_anisotropy_cpu(ax, kk, ms, m, h);
	copy_out(h, H);
	return e;
}

// src/magneto/mmm/anisotropy/anisotropy_cpu.cpp:75 cubic_anisotropy_cpu
double mmref_cubic_anisotropy(int nx, int ny, int nz, const double *axis1, const double *axis2,
                              const double *k, const double *Ms, const double *M, double *H)
{
	ensure_matty();
	VectorMatrix a1 = vector_field(nx, ny, nz, axis1), a2 = vector_field(nx, ny, nz, axis2);
	VectorMatrix m = vector_field(nx, ny, nz, M);
	Matrix kk = scalar_field(nx, ny, nz, k), ms = scalar_field(nx, ny, nz, Ms);
	VectorMatrix h(Shape(nx, ny, nz));
	const double e = cubic_anisotropy_cpu(a1, a2, kk, ms, m, h);
	copy_out(h, H);
	return e;
}

// src/magneto/mmm/llge/llge_cpu.cpp:25 llge_cpu
void mmref_llge(int nx, int ny, int nz, const double *f1, const double *f2, const double *M,
                const double *H, double *dM)
{
	ensure_matty();
	Matrix a = scalar_field(nx, ny, nz, f1), b = scalar_field(nx, ny, nz, f2);
	VectorMatrix m = vector_field(nx, ny, nz, M), h = vector_field(nx, ny, nz, H);
	VectorMatrix dm(Shape(nx, ny, nz));
	llge_cpu(a, b, m, h, dm);
	copy_out(dm, dM);
}

// src/magneto/mmm/spintorque/fdm_zhangli_cpu.cpp:57 fdm_zhangli_cpu (per-cell parameter form)
void mmref_fdm_zhangli(int nx, int ny, int nz, double dx, double dy, double dz, int do_precess,
                       const double *P, const double *xi, const double *Ms, const double *alpha,
                       const double *j, const double *M, double *dM)
{
	ensure_matty();
	Matrix p = scalar_field(nx, ny, nz, P), x = scalar_field(nx, ny, nz, xi);
	Matrix ms = scalar_field(nx, ny, nz, Ms), al = scalar_field(nx, ny, nz, alpha);
	VectorMatrix jj = vector_field(nx, ny, nz, j), m = vector_field(nx, ny, nz, M);
	VectorMatrix dm(Shape(nx, ny, nz));
	fdm_zhangli_cpu(nx, ny, nz, dx, dy, dz, do_precess != 0, p, x, ms, al, jj, m, dm);
	copy_out(dm, dM);
}

// src/magneto/mmm/demag/tensor_round.cpp:90 round_tensor_dimension
int mmref_round_tensor_dimension(int dim, int periodic, int padding)
{
	ensure_matty();
	return round_tensor_dimension(dim, periodic != 0, padding);
}

// src/magneto/mmm/demag/demag_tensor.cpp:116-186 GenerateDemagTensor without its file cache:
// calculateDemagTensor (tensor.cpp:35) followed by the negation at demag_tensor.cpp:177.
// out must hold 6*ex*ey*ez doubles, layout (component, x, y, z) with x fastest.
void mmref_demag_tensor(int nx, int ny, int nz, double dx, double dy, double dz,
                        int px, int py, int pz, int repeat, int ex, int ey, int ez, double *out)
{
	ensure_matty();
	const int rx = px ? repeat : 1, ry = py ? repeat : 1, rz = pz ? repeat : 1;
	Matrix N = calculateDemagTensor(dx, dy, dz, nx, ny, nz, ex, ey, ez, rx, ry, rz);
	N.scale(-1);
	Matrix::ro_accessor acc(N);
	std::memcpy(out, acc.ptr(), sizeof(double) * 6 * (size_t)ex * ey * ez);
}

// src/magneto/math/conv/SymmetricMatrixVectorConvolution_Simple.cpp:36 execute (direct sum)
void mmref_conv_simple(const double *N, int nx, int ny, int nz, int ex, int ey, int ez,
                       const double *M, double *H)
{
	ensure_matty();
	Matrix lhs(Shape(6, ex, ey, ez));
	{
		Matrix::wo_accessor acc(lhs);
		std::memcpy(acc.ptr(), N, sizeof(double) * 6 * (size_t)ex * ey * ez);
	}
	SymmetricMatrixVectorConvolution_Simple conv(lhs, nx, ny, nz);
	VectorMatrix m = vector_field(nx, ny, nz, M);
	VectorMatrix h(Shape(nx, ny, nz));
	conv.execute(m, h);
	copy_out(h, H);
}

// src/magneto/math/ScaledAbsMax.cpp:52 scaled_abs_max
double mmref_scaled_abs_max(int nx, int ny, int nz, const double *M, const double *scale)
{
	ensure_matty();
	VectorMatrix m = vector_field(nx, ny, nz, M);
	Matrix s = scalar_field(nx, ny, nz, scale);
	return scaled_abs_max(m, s);
}

// src/magneto/matrix/matrix/vector/VectorMatrix.cpp:218 VectorMatrix::normalize(const Matrix&)
void mmref_normalize(int nx, int ny, int nz, const double *Ms, double *M)
{
	ensure_matty();
	VectorMatrix m = vector_field(nx, ny, nz, M);
	Matrix s = scalar_field(nx, ny, nz, Ms);
	m.normalize(s);
	copy_out(m, M);
}

// src/magneto/evolver/runge_kutta.cpp:32-48 rk_prepare_step (CPU path: runge_kutta_cpu.cpp).
// tab: s stages, b row-major s x s; k: six arrays (unused ones may repeat k[0], as the caller
// magnum/evolver/runge_kutta.py:113 passes them).
void mmref_rk_prepare_step(int nx, int ny, int nz, int step, double h, int s, const double *a, const double *b,
                           const double *c, const double *ec, const double *const *k, const double *y, double *ytmp)
{
	ensure_matty();
	ButcherTableau tab = tableau(s, a, b, c, ec);
	std::vector<VectorMatrix> kv;
	for (int i = 0; i < 6; ++i) kv.push_back(vector_field(nx, ny, nz, k[i]));
	VectorMatrix yv = vector_field(nx, ny, nz, y), yt(Shape(nx, ny, nz));
	rk_prepare_step(step, h, tab, kv[0], kv[1], kv[2], kv[3], kv[4], kv[5], yv, yt);
	copy_out(yt, ytmp);
}

// src/magneto/evolver/runge_kutta.cpp:68-96 rk_combine_result, the six-vector form (the only one
// the SWIG module binds, bindings/evolver.i:79-95).
void mmref_rk_combine_result(int nx, int ny, int nz, double h, int s, const double *a, const double *b,
                             const double *c, const double *ec, const double *const *k, double *y, double *y_error)
{
	ensure_matty();
	ButcherTableau tab = tableau(s, a, b, c, ec);
	std::vector<VectorMatrix> kv;
	for (int i = 0; i < 6; ++i) kv.push_back(vector_field(nx, ny, nz, k[i]));
	VectorMatrix yv = vector_field(nx, ny, nz, y), ye(Shape(nx, ny, nz));
	rk_combine_result(h, tab, kv[0], kv[1], kv[2], kv[3], kv[4], kv[5], yv, ye);
	copy_out(yv, y);
	copy_out(ye, y_error);
}

// src/magneto/evolver/runge_kutta.cpp:98-130 rk_adjust_stepsize (the NR controller's rule).
double mmref_rk_adjust_stepsize(int nx, int ny, int nz, int order, double h, double eps_abs, double eps_rel,
                                const double *y, const double *y_error)
{
	ensure_matty();
	VectorMatrix yv = vector_field(nx, ny, nz, y), ye = vector_field(nx, ny, nz, y_error);
	return rk_adjust_stepsize(order, h, eps_abs, eps_rel, yv, ye);
}

} // extern "C"
