// The fused B200 solver: Runge-Kutta steps of the Landau-Lifshitz-Gilbert equation with the
// reference's step controller, entirely on the device.
//
// Reference path replaced (per RK stage): magnum/evolver/runge_kutta.py:105-118 forms the stage
// state with one axpy per earlier stage, then LandauLifshitzGilbert.calculate_dMdt
// (landau_lifshitz_gilbert.py:92-125) fills H_tot with one kernel per field term (stray field
// convolution, exchange, anisotropy, applied field), adds them with axpys, calls llge and adds
// the Zhang-Li torque; the step ends with rk_combine_result / Python axpys, two scaled_abs_max
// reductions with host synchronisation (micro_magnetics_stepsize_controller.py:35-73) and a
// normalisation (micro_magnetics.py:49-50).
//
// Here each stage is: the demag convolution passes (conv.cu) + ONE fused kernel that evaluates
// exchange, anisotropy, applied field, LLG and Zhang-Li for a cell, writes k_i and the next stage
// state, and (first/last stages) folds the |k_0| and error maxima into device reductions.  A
// one-thread controller kernel applies the reference's accept/reject rule on the device.
//
// State representation: unit magnetisation m = M/Ms (Ms per region), which is the reference's
// ODE scaled cell-wise by the constant 1/Ms: the Runge-Kutta combinations are linear, so the
// trajectory and the controller's scaled errors (|y_err|/Ms) are the same quantities.  Material
// parameters are a per-region table (<= 256 regions, one uint8 index per cell).
//
// Precision modes: MM_F64 is plain double.  MM_F32 computes fields, stages and reductions in
// float and keeps the state as an unevaluated float pair m = hi + lo that is updated with an
// error-free two-sum (a compensated update), so the accumulated state is not limited by float
// rounding of the per-step increment; the controller runs in double.
#include "mm_common.cuh"
#include "conv.cuh"
#include "tma.cuh"

#include <vector>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <utility>

namespace mm {

template <typename T>
struct DevMat {
	T Ms;        // saturation magnetisation
	T cex;       // 2 A / (mu0 Ms)                       exchange prefactor
	T l1, l2;    // LLG on unit m: dm = l1 m x H + l2 m x (m x H)
	T ku;        // 2 k_u / (mu0 Ms)                     uniaxial
	T kc;        // -2 k_c / (mu0 Ms)                    cubic
	T zl1, zl2;  // Zhang-Li on unit m: dm = zl1 m x (m x u') + zl2 m x u', u' = (j.grad)M / Ms
	T a1[3], a2[3], a3[3];
	T j[3];
};

struct DevState {
	double t;         // time at the start of the attempt
	double h;         // step size of the attempt
	double max_err2;  // max |m_err|^2 of the attempt (reduction)
	double max_k02;   // max |k_0|^2 of the attempt (reduction)
	double h_new;     // controller output
	int accept;
	int not_finite;
	int stage_timeout;  // set by a staged stage kernel whose bounded wait gave up
	int pad;
	double max_tq2;   // max (|m x H_eff| / Ms)^2 at the last stage's input (batched relaxations)
};

constexpr int MAXS = 8;

template <typename T>
struct KTab {
	T *k[MAXS];
};

struct Tableau {
	int s, order, fsal;
	double a[MAXS], b[MAXS][MAXS], c[MAXS], ec[MAXS];
};

// magnum/evolver/tableaus.py:54-139
static Tableau make_tableau(int which)
{
	Tableau t{};
	if (which == MM_RK_DP54) {
		t.s = 7; t.order = 5; t.fsal = 1;
		const double a[7] = {0.0, 1.0 / 5.0, 3.0 / 10.0, 4.0 / 5.0, 8.0 / 9.0, 1.0, 1.0};
		const double b[7][6] = {{0},
		                        {1.0 / 5.0},
		                        {3.0 / 40.0, 9.0 / 40.0},
		                        {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0},
		                        {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0},
		                        {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0},
		                        {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
		const double c4[7] = {5179.0 / 57600.0, 0.0, 7571.0 / 16695.0, 393.0 / 640.0, -92097.0 / 339200.0, 187.0 / 2100.0, 1.0 / 40.0};
		const double c5[7] = {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0, 0.0};
		for (int i = 0; i < 7; ++i) {
			t.a[i] = a[i];
			for (int j = 0; j < 6; ++j) t.b[i][j] = b[i][j];
			t.c[i] = c5[i];
			t.ec[i] = c4[i] - c5[i];
		}
	} else if (which == MM_RK_RKF45) {
		t.s = 6; t.order = 4; t.fsal = 0;
		const double a[6] = {0.0, 1.0 / 4.0, 3.0 / 8.0, 12.0 / 13.0, 1.0, 1.0 / 2.0};
		const double b[6][5] = {{0},
		                        {1.0 / 4.0},
		                        {3.0 / 32.0, 9.0 / 32.0},
		                        {1932.0 / 2197.0, -7200.0 / 2197.0, 7296.0 / 2197.0},
		                        {439.0 / 216.0, -8.0, 3680.0 / 513.0, -845.0 / 4104.0},
		                        {-8.0 / 27.0, 2.0, -3544.0 / 2565.0, 1859.0 / 4104.0, -11.0 / 40.0}};
		const double c4[6] = {25.0 / 216.0, 0.0, 1408.0 / 2565.0, 2197.0 / 4104.0, -1.0 / 5.0, 0.0};
		const double c5[6] = {16.0 / 135.0, 0.0, 6656.0 / 12825.0, 28561.0 / 56430.0, -9.0 / 50.0, 2.0 / 55.0};
		for (int i = 0; i < 6; ++i) {
			t.a[i] = a[i];
			for (int j = 0; j < 5; ++j) t.b[i][j] = b[i][j];
			t.c[i] = c4[i];
			t.ec[i] = c4[i] - c5[i];
		}
	} else if (which == MM_RK_CC45) {
		t.s = 6; t.order = 4; t.fsal = 0;
		const double a[6] = {0.0, 1.0 / 5.0, 3.0 / 10.0, 3.0 / 5.0, 1.0, 7.0 / 8.0};
		const double b[6][5] = {{0},
		                        {1.0 / 5.0},
		                        {3.0 / 40.0, 9.0 / 40.0},
		                        {3.0 / 10.0, -9.0 / 10.0, 6.0 / 5.0},
		                        {-11.0 / 54.0, 5.0 / 2.0, -70.0 / 27.0, 35.0 / 27.0},
		                        {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0}};
		const double c4[6] = {2825.0 / 27648.0, 0.0, 18575.0 / 48384.0, 13525.0 / 55296.0, 277.0 / 14336.0, 1.0 / 4.0};
		const double c5[6] = {37.0 / 378.0, 0.0, 250.0 / 621.0, 125.0 / 594.0, 0.0, 512.0 / 1771.0};
		for (int i = 0; i < 6; ++i) {
			t.a[i] = a[i];
			for (int j = 0; j < 5; ++j) t.b[i][j] = b[i][j];
			t.c[i] = c4[i];
			t.ec[i] = c4[i] - c5[i];
		}
	} else {  // rk23
		t.s = 4; t.order = 3; t.fsal = 1;
		const double a[4] = {0.0, 0.5, 3.0 / 4.0, 1.0};
		const double b[4][3] = {{0}, {1.0 / 2.0}, {0.0, 3.0 / 4.0}, {2.0 / 9.0, 1.0 / 3.0, 4.0 / 9.0}};
		const double c2[4] = {7.0 / 24.0, 1.0 / 4.0, 1.0 / 3.0, 1.0 / 8.0};
		const double c3[4] = {2.0 / 9.0, 1.0 / 3.0, 4.0 / 9.0, 0.0};
		for (int i = 0; i < 4; ++i) {
			t.a[i] = a[i];
			for (int j = 0; j < 3; ++j) t.b[i][j] = b[i][j];
			t.c[i] = c3[i];
			t.ec[i] = c2[i] - c3[i];
		}
	}
	return t;
}

// Arguments shared by the per-cell kernels.
template <typename T>
struct CellArgs {
	int nx, ny, nz;
	T wx, wy, wz;                  // 1/dx^2 ...
	T idx2, idy2, idz2;            // 1/(2 dx) ... (Zhang-Li central differences)
	T idx1, idy1, idz1;            // 1/dx ...     (one-sided differences)
	int terms;
	int pbc;                       // periodic axes: bit 0 x, bit 1 y, bit 2 z (exchange stencil)
	const uint8_t *reg;            // nullptr: every cell is region 0
	const DevMat<T> *mat;
	int nmat;
	double Hext[3], Hpulse[3], rise;
};

template <typename T>
__device__ __forceinline__ const DevMat<T> &mat_of(const CellArgs<T> &a, size_t i)
{
	return a.mat[a.reg ? a.reg[i] : 0];
}

// Applied field at time t (constant part plus the linearly rising pulse).
template <typename T>
__device__ __forceinline__ V3<T> zeeman_field(const CellArgs<T> &a, double t)
{
	double f = 1.0;
	if ((a.terms & MM_TERM_ZEEMAN) && a.rise > 0) f = t / a.rise < 1.0 ? t / a.rise : 1.0;
	return (a.terms & MM_TERM_ZEEMAN) ? v3<T>((T)(a.Hext[0] + a.Hpulse[0] * f), (T)(a.Hext[1] + a.Hpulse[1] * f),
	                                          (T)(a.Hext[2] + a.Hpulse[2] * f))
	                                  : v3<T>(0, 0, 0);
}

// Field terms and dm/dt of one non-empty cell (material M, unit state m) from its gathered
// neighbourhood: nb[q] / nms[q] are the unit state and Ms of the neighbours x-1, x+1, y-1, y+1,
// z-1, z+1 (zero where the neighbour is outside the box).  Hd: demag field, Hz: applied field.
// Whether term t is on: a compile-time answer when the kernel was specialised for the term set TM
// (TM >= 0), else the run-time bit set.
template <int TM, typename T>
__device__ __forceinline__ bool term_on(const CellArgs<T> &a, int t)
{
	if constexpr (TM >= 0) return (TM & t) != 0;
	else return (a.terms & t) != 0;
}

// Term sets the staged stage kernel is compiled for (besides the run-time one): the granular
// slab's and the thin film's.
constexpr int TM_RUNTIME = -1;
constexpr int TM_SLAB = MM_TERM_DEMAG | MM_TERM_EXCHANGE | MM_TERM_UNIAXIAL | MM_TERM_ZHANGLI;
constexpr int TM_FILM = MM_TERM_DEMAG | MM_TERM_EXCHANGE;

template <typename T, int TM = TM_RUNTIME>
__device__ __forceinline__ void cell_core(const CellArgs<T> &a, const DevMat<T> &M, const V3<T> &m,
                                          const V3<T> (&nb)[6], const T (&nms)[6], int x, int yy, int z,
                                          V3<T> Hd, V3<T> Hz, V3<T> &Heff, V3<T> &dm)
{
	const T ms = M.Ms;
	V3<T> H = term_on<TM>(a, MM_TERM_DEMAG) ? Hd : v3<T>(0, 0, 0);
	if (term_on<TM>(a, MM_TERM_EXCHANGE)) {
		// exchange_cpu.cpp:60-139: H = 2A/(mu0 Ms) sum_nb w (m_nb - m), empty neighbours skipped
		const T w[6] = {a.wx, a.wx, a.wy, a.wy, a.wz, a.wz};
		V3<T> sum = v3<T>(0, 0, 0);
#pragma unroll
		for (int q = 0; q < 6; ++q)
			if (nms[q] != T(0)) sum = sum + w[q] * (nb[q] - m);
		H = H + M.cex * sum;
	}
	if (term_on<TM>(a, MM_TERM_UNIAXIAL)) {
		// anisotropy_cpu.cpp:29-73 (k == 0 gives ku == 0)
		const V3<T> ax = v3<T>(M.a1[0], M.a1[1], M.a1[2]);
		H = H + (M.ku * dot(m, ax)) * ax;
	}
	if (term_on<TM>(a, MM_TERM_CUBIC)) {
		// anisotropy_cpu.cpp:75-119 on m/|m|
		const T len = sqrt(dot(m, m));
		const V3<T> u = len > T(0) ? (T(1) / len) * m : v3<T>(0, 0, 0);
		const V3<T> u1 = v3<T>(M.a1[0], M.a1[1], M.a1[2]), u2 = v3<T>(M.a2[0], M.a2[1], M.a2[2]),
		            u3 = v3<T>(M.a3[0], M.a3[1], M.a3[2]);
		const T p1 = dot(u1, u), p2 = dot(u2, u), p3 = dot(u3, u);
		const T s1 = p1 * p1, s2 = p2 * p2, s3 = p3 * p3;
		H = H + M.kc * (((s2 + s3) * p1) * u1 + ((s1 + s3) * p2) * u2 + ((s1 + s2) * p3) * u3);
	}
	H = H + Hz;
	Heff = H;
	// llge_cpu.cpp:25-45 on unit m
	const V3<T> mxh = cross(m, H);
	dm = M.l1 * mxh + M.l2 * cross(m, mxh);
	if (term_on<TM>(a, MM_TERM_ZHANGLI)) {
		// fdm_zhangli_cpu.cpp:100-200: u = (j.grad)M from raw M = Ms m (no Ms masking),
		// one-sided at the borders, zero along a dimension of size 1
		const V3<T> Mc = scale_rn(ms, m);
		// one-sided at either face (both faces at once along a dimension of size 1: zero), central
		// inside, with the operands selected rather than branched on
		auto grad = [&](int c, int dim, int lo, T inv1, T inv2) -> V3<T> {
			const V3<T> Ml = scale_rn(nms[lo], nb[lo]), Mr = scale_rn(nms[lo + 1], nb[lo + 1]);
			const bool at_lo = c == 0, at_hi = c == dim - 1;
			const V3<T> A = at_lo ? Mc : Ml, B = at_hi ? Mc : Mr;
			return (at_lo || at_hi ? inv1 : inv2) * (B - A);
		};
		V3<T> u = v3<T>(0, 0, 0);
		if (M.j[0] != T(0)) u = u + M.j[0] * grad(x, a.nx, 0, a.idx1, a.idx2);
		if (M.j[1] != T(0)) u = u + M.j[1] * grad(yy, a.ny, 2, a.idy1, a.idy2);
		if (M.j[2] != T(0)) u = u + M.j[2] * grad(z, a.nz, 4, a.idz1, a.idz2);
		u = (T(1) / ms) * u;
		const V3<T> mxu = cross(m, u);
		dm = dm + M.zl1 * cross(m, mxu) + M.zl2 * mxu;
	}
}

// The six neighbours x-1, x+1, y-1, y+1, z-1, z+1 of cell i = (x, yy, z): whether each exists and
// its index.  Along a periodic axis the face cells wrap around (exchange_cpu.cpp:141-235).
template <typename T>
__device__ __forceinline__ void neighbours(const CellArgs<T> &a, int x, int yy, int z, size_t i, bool (&has)[6],
                                           size_t (&off)[6])
{
	const size_t nx = a.nx, nxy = (size_t)a.nx * a.ny, wy = (size_t)(a.ny - 1) * nx, wz = (size_t)(a.nz - 1) * nxy;
	const bool px = a.pbc & 1, py = a.pbc & 2, pz = a.pbc & 4;
	has[0] = x > 0 || px;
	off[0] = x > 0 ? i - 1 : i + (nx - 1);
	has[1] = x < a.nx - 1 || px;
	off[1] = x < a.nx - 1 ? i + 1 : i - (nx - 1);
	has[2] = yy > 0 || py;
	off[2] = yy > 0 ? i - nx : i + wy;
	has[3] = yy < a.ny - 1 || py;
	off[3] = yy < a.ny - 1 ? i + nx : i - wy;
	has[4] = z > 0 || pz;
	off[4] = z > 0 ? i - nxy : i + wz;
	has[5] = z < a.nz - 1 || pz;
	off[5] = z < a.nz - 1 ? i + nxy : i - wz;
}

// Effective field (without the demag term) and dm/dt of one cell of the unit-m field y.
// Hd: demag field of the cell (added when the term is on); msr: Ms per region (shared memory).
// The six neighbours are loaded once and serve both the exchange stencil and the Zhang-Li
// gradient.  Returns false for empty cells.
template <typename T>
__device__ __forceinline__ bool cell_rhs(const CellArgs<T> &a, const T *__restrict__ msr,
                                         const T *__restrict__ y, size_t n, int x, int yy, int z, size_t i,
                                         V3<T> Hd, double t, V3<T> &Heff, V3<T> &dm)
{
	const DevMat<T> &M = mat_of(a, i);
	const V3<T> Hz = zeeman_field(a, t);
	const T ms = M.Ms;
	if (ms == T(0)) {
		// empty cell: no magnetisation and no torque, but the stray and applied fields exist
		// there (H_tot is the sum of the terms, each zero except these two)
		Heff = ((a.terms & MM_TERM_DEMAG) ? Hd : v3<T>(0, 0, 0)) + Hz;
		dm = v3<T>(0, 0, 0);
		return false;
	}
	const V3<T> m = load3(y, i, n);
	bool has[6];
	size_t off[6];
	neighbours(a, x, yy, z, i, has, off);
	V3<T> nb[6];
	T nms[6];
#pragma unroll
	for (int q = 0; q < 6; ++q) {
		if (has[q]) {
			nb[q] = load3(y, off[q], n);
			nms[q] = a.reg ? msr[a.reg[off[q]]] : ms;
		} else {
			nb[q] = v3<T>(0, 0, 0);
			nms[q] = T(0);
		}
	}
	cell_core<T>(a, M, m, nb, nms, x, yy, z, Hd, Hz, Heff, dm);
	return true;
}

// Ms per region into shared memory (all threads of the block call this).
template <typename T>
__device__ __forceinline__ void load_ms_table(const CellArgs<T> &a, T *msr)
{
	const int tid = threadIdx.x + blockDim.x * threadIdx.y;
	for (int r = tid; r < a.nmat; r += blockDim.x * blockDim.y) msr[r] = a.mat[r].Ms;
	__syncthreads();
}

// Per-stage coefficients (by value).
struct StageCoef {
	int stage;        // i
	int last;         // i == s-1
	int write_next;   // not last: write y_{i+1}
	int write_new;    // last: write y_{n+1} (always in MM_F32, non-FSAL in MM_F64)
	int reduce_k0;    // fold max |k_0|^2
	double a_i;       // time node of this stage
	double bn[MAXS];  // b[i+1][0..i] (not last)  or  c[0..s-1] (last)
	double ec[MAXS];  // error weights (last)
};

// Whether the combination of stage S reads k_l (uniform over a launch).
__host__ __device__ inline bool stage_needs_k(const StageCoef &sc, int S, int l)
{
	return l < S && (sc.last ? (sc.ec[l] != 0.0 || (sc.write_new && sc.bn[l] != 0.0))
	                         : ((sc.write_next && sc.bn[l] != 0.0) || (sc.reduce_k0 && l == 0)));
}

// Operand list of a staged stage launch, in order: the demag field (term on), y_n and its
// compensation (when the stage writes a state), the k_l the combination reads.  Sets the operand
// index of each (-1: not read) and returns the count.
__host__ __device__ inline int stage_ops(const StageCoef &sc, int S, bool comp, bool demag, int *kop, int &op_hd,
                                         int &op_hi, int &op_lo)
{
	int n = 0;
	const bool out = sc.last ? sc.write_new : sc.write_next;
	op_hd = demag ? n++ : -1;
	op_hi = out ? n++ : -1;
	op_lo = out && comp ? n++ : -1;
#pragma unroll
	for (int l = 0; l < MAXS; ++l) kop[l] = stage_needs_k(sc, S, l) ? n++ : -1;
	return n;
}

// Structure of one stage as a bit pattern: which k_l the combination reads (bits 0-6), last (7),
// write_next (8), write_new (9), reduce_k0 (10), which b/c weights are nonzero (11-17), which
// error weights are nonzero (18-24), and bit 25 set.  A staged stage kernel compiled for a
// pattern folds its operand indices and weight tests at compile time; PAT_RUNTIME reads them
// from the coefficients.
constexpr int PAT_RUNTIME = -1;
constexpr int PAT_KBITS = 7;  // stage vectors a pattern describes (k_0 .. k_6)
__host__ __device__ constexpr int pat_make(int needk, bool last, bool wnext, bool wnew, bool rk0, int bnm, int ecm)
{
	return needk | (last ? 1 << 7 : 0) | (wnext ? 1 << 8 : 0) | (wnew ? 1 << 9 : 0) | (rk0 ? 1 << 10 : 0) |
	       (bnm << 11) | (ecm << 18) | (1 << 25);
}
__host__ __device__ constexpr bool pat_bit(int pat, int bit) { return ((pat >> bit) & 1) != 0; }
__host__ __device__ constexpr int pat_nops(int pat, bool comp, bool demag)
{
	const bool out = pat_bit(pat, 7) ? pat_bit(pat, 9) : pat_bit(pat, 8);
	int n = (demag ? 1 : 0) + (out ? 1 : 0) + (out && comp ? 1 : 0);
	for (int q = 0; q < PAT_KBITS; ++q) n += pat_bit(pat, q) ? 1 : 0;
	return n;
}
// operand index of k_l under a pattern (operands: demag field, y_n, its compensation, the k_l read)
__host__ __device__ constexpr int pat_kop(int pat, bool comp, bool demag, int l)
{
	const bool out = pat_bit(pat, 7) ? pat_bit(pat, 9) : pat_bit(pat, 8);
	int n = (demag ? 1 : 0) + (out ? 1 : 0) + (out && comp ? 1 : 0);
	for (int q = 0; q < l; ++q) n += pat_bit(pat, q) ? 1 : 0;
	return pat_bit(pat, l) ? n : -1;
}
__host__ inline int pattern_of(const StageCoef &sc, int S)
{
	int needk = 0, bnm = 0, ecm = 0;
	for (int l = 0; l < MAXS; ++l) {
		const bool k = stage_needs_k(sc, S, l), b = sc.bn[l] != 0.0, e = sc.ec[l] != 0.0;
		if (l >= PAT_KBITS && (k || b || e)) return PAT_RUNTIME;  // beyond what a pattern holds
		needk |= k ? 1 << l : 0;
		bnm |= b ? 1 << l : 0;
		ecm |= e ? 1 << l : 0;
	}
	return pat_make(needk, sc.last, sc.write_next, sc.write_new, sc.reduce_k0, bnm, ecm);
}
// The Dormand-Prince 5(4) stages (magnum/evolver/tableaus.py): nonzero masks of b[i][0..i-1]
// (b[6][1] = 0), of c = b[6] and of the error weights c4 - c5 (zero at l = 1 only).
constexpr int dp54_bmask(int i) { return i == 6 ? 0x3D : (1 << i) - 1; }
constexpr int DP54_CMASK = 0x3D, DP54_ECMASK = 0x7D;
constexpr int dp54_pattern(int S, bool comp)
{
	if (S == 0) return pat_make(0, false, true, false, false, dp54_bmask(1), 0);
	const bool last = S == 6, rk0 = S == 1, wnew = last && comp;
	const int bnm = last ? DP54_CMASK : dp54_bmask(S + 1);
	const int ecm = last ? DP54_ECMASK : 0;
	int needk = 0;
	for (int l = 0; l < S; ++l) {
		const bool need = last ? (pat_bit(ecm, l) || (wnew && pat_bit(bnm, l)))
		                       : (pat_bit(bnm, l) || (rk0 && l == 0));
		needk |= need ? 1 << l : 0;
	}
	return pat_make(needk, last, !last, wnew, rk0, bnm, ecm);
}

// One fused stage: k_i = f(y_in) (demag field from Hd), then the next stage state
// y_{i+1} = y_n + h sum_{l<=i} b_{i+1,l} k_l, or on the last stage the error maximum and y_{n+1}.
// COMP: compensated float state (y_n = yhi + ylo).  S = i is a template argument, so the sums
// over earlier stages unroll and their loads issue together.  The grid is persistent: each block
// loads the Ms table once and walks tiles of 32*STAGE_CPT x 8 cells; each thread handles CPT
// cells 32 apart in x (every warp access stays a contiguous 128-byte run) and issues all their
// loads before any store, so twice the bytes are in flight per thread.
constexpr int STAGE_CPT = 2;
template <typename T>
constexpr int stage_min_blocks() { return sizeof(T) == 4 ? 3 : 2; }  // FP64 needs ~126 registers

// One tile (32*STAGE_CPT x 8 cells of plane z) of the fused stage; the maxima of the error, of
// |k_0| and (TORQUE) of |m x H_eff| / Ms accumulate in e2, k02, tq2.
// Asynchronous element copy global -> shared (LDGSTS), finished by cp_async_wait_all().
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src)
{
	const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
	if constexpr (sizeof(T) == 4)
		asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
	else
		asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Prefetch slots per cell of a stage tile: y_n (3), its compensation (3), k_0..k_{MAXS-2} (3 each).
constexpr int STAGE_PRE = 6 + 3 * (MAXS - 1);
template <typename T>
constexpr size_t stage_smem() { return (size_t)STAGE_PRE * STAGE_CPT * 256 * sizeof(T); }

// Deviation form of the FP32 batched stages.  The state is y = hi + D with hi the instance's base
// state (fixed between rebases) and D its deviation (small); the base field hb = H_demag(hi) +
// H_exch(hi) is computed once per rebase.  A stage input y_l = hi + D_l is carried as D_l alone, its
// demag field is the convolution of D_l, and the right-hand side is split into a base part built
// from hi and hb + H_zeeman only (bit-identical in every stage of a step while the applied field is
// constant) and a part built from D_l and the fields of D_l:
//   H = Hb + dH,  Hb = hb + H_z(t),  dH = H_demag(D) + H_exch(D)
//   y x H = hi x Hb + [hi x dH + D x (Hb + dH)] = Tb + dT
//   y x (y x H) = hi x Tb + [hi x dT + D x (Tb + dT)] = Ub + dU
//   dm/dt = (l1 Tb + l2 Ub) + (l1 dT + l2 dU)
// Rounding in a stage then differs from the other stages of the step only in proportion to the
// deviation terms, so the embedded error estimate keeps no floor of order float epsilon times the
// field: a direct FP32 evaluation of y_l has one (~1e-4 relative to h max |dm/dt| near equilibrium
// for 4 nm cells), at which the controller's relative test stalls the step size.  Terms: demag,
// exchange and the applied field (the batched instances' physics).
template <typename T>
__device__ __forceinline__ bool cell_rhs_delta(const CellArgs<T> &a, const T *__restrict__ msr,
                                               const T *__restrict__ D, size_t n, int x, int yy, int z, size_t i,
                                               V3<T> hi, V3<T> hb, V3<T> hdD, double t, V3<T> &Tt, V3<T> &dm)
{
	const DevMat<T> &M = mat_of(a, i);
	const V3<T> Hz = zeeman_field(a, t);
	if (M.Ms == T(0)) {
		Tt = v3<T>(0, 0, 0);
		dm = v3<T>(0, 0, 0);
		return false;
	}
	const V3<T> d = load3(D, i, n);
	V3<T> dH = (a.terms & MM_TERM_DEMAG) ? hdD : v3<T>(0, 0, 0);
	if (a.terms & MM_TERM_EXCHANGE) {
		bool has[6];
		size_t off[6];
		neighbours(a, x, yy, z, i, has, off);
		const T w[6] = {a.wx, a.wx, a.wy, a.wy, a.wz, a.wz};
		V3<T> sum = v3<T>(0, 0, 0);
#pragma unroll
		for (int q = 0; q < 6; ++q) {
			if (!has[q]) continue;
			const T ms_q = a.reg ? msr[a.reg[off[q]]] : M.Ms;
			if (ms_q != T(0)) sum = sum + w[q] * (load3(D, off[q], n) - d);
		}
		dH = dH + M.cex * sum;
	}
	const V3<T> Hb = hb + Hz;
	const V3<T> Tb = cross(hi, Hb);
	const V3<T> dT = cross(hi, dH) + cross(d, Hb + dH);
	Tt = Tb + dT;
	const V3<T> Ub = cross(hi, Tb);
	const V3<T> dU = cross(hi, dT) + cross(d, Tt);
	dm = (M.l1 * Tb + M.l2 * Ub) + (M.l1 * dT + M.l2 * dU);
	return true;
}

// One tile (32*STAGE_CPT x 8 cells of plane z) of the fused stage; the maxima of the error, of
// |k_0| and (TORQUE) of |m x H_eff| / Ms accumulate in e2, k02, tq2.  The operands of the stage
// combination (y_n, its compensation, the earlier stage vectors with nonzero weight) are copied
// into shared memory asynchronously while the field and k_i are computed; `pre` is the block's
// STAGE_PRE * STAGE_CPT * 256 slots.
// DELTA (the FP32 batched form, with COMP): y_in, the combination and y_out are deviations from
// the base state yhi (ylo: the step's own deviation D_n), hb the base field (cell_rhs_delta), and
// the last stage writes the deviation of y_{n+1} into y_out alone (y_out_lo is not written).
// PAT: the stage's structure at compile time (as in k_stage_tma), PAT_RUNTIME: from sc.
template <typename T, bool COMP, int S, bool TORQUE, bool DELTA = false, int PAT = PAT_RUNTIME>
__device__ __forceinline__ void stage_tile(const CellArgs<T> &a, const T *__restrict__ msr, const StageCoef &sc,
                                           const T *__restrict__ y_in, const T *__restrict__ Hd,
                                           const T *__restrict__ yhi, const T *__restrict__ ylo, T *const *K,
                                           T *__restrict__ y_out, T *__restrict__ y_out_lo,
                                           const DevState *__restrict__ st, int tile, int tiles_x, int tiles_y,
                                           T &e2, T &k02, T &tq2, T *pre, const T *__restrict__ hb = nullptr)
{
	static_assert(!DELTA || COMP, "the deviation form is the compensated FP32 form's");
	constexpr bool CT = PAT != PAT_RUNTIME;
	const bool s_last = CT ? pat_bit(PAT, 7) : sc.last != 0;
	const bool s_wnext = CT ? pat_bit(PAT, 8) : sc.write_next != 0;
	const bool s_wnew = CT ? pat_bit(PAT, 9) : sc.write_new != 0;
	const bool s_rk0 = CT ? pat_bit(PAT, 10) : sc.reduce_k0 != 0;
	const size_t n = (size_t)a.nx * a.ny * a.nz;
	const double h = st->h;
	const int tx = tile % tiles_x, rest = tile / tiles_x;
	const int yy = (rest % tiles_y) * blockDim.y + threadIdx.y;
	const int z = rest / tiles_y;
	const double t = st->t + sc.a_i * h;
	const int tid = threadIdx.x + blockDim.x * threadIdx.y;
	auto slot = [&](int u, int k) -> T & { return pre[(u * STAGE_PRE + k) * 256 + tid]; };
	auto pre3 = [&](int u, int k) { return v3<T>(slot(u, k), slot(u, k + 1), slot(u, k + 2)); };
	V3<T> ki[STAGE_CPT];
	size_t idx[STAGE_CPT];
	bool in[STAGE_CPT];
	// which operands the combination needs (uniform over the block)
	const bool out = s_last ? s_wnew : s_wnext;
	bool needk[MAXS];
#pragma unroll
	for (int l = 0; l < MAXS; ++l) needk[l] = CT ? (l < PAT_KBITS && pat_bit(PAT, l)) : stage_needs_k(sc, S, l);
#pragma unroll
	for (int u = 0; u < STAGE_CPT; ++u) {
		const int x = tx * (blockDim.x * STAGE_CPT) + threadIdx.x + u * blockDim.x;
		in[u] = x < a.nx && yy < a.ny;
		idx[u] = ((size_t)z * a.ny + (in[u] ? yy : 0)) * a.nx + (in[u] ? x : 0);
		if (in[u]) {
			for (int c = 0; c < 3; ++c) {
				const size_t e = idx[u] + c * n;
				if (out && !DELTA) cp_async_elem(&slot(u, c), yhi + e);
				if (out && COMP) cp_async_elem(&slot(u, 3 + c), ylo + e);
#pragma unroll
				for (int l = 0; l < S; ++l)
					if (needk[l]) cp_async_elem(&slot(u, 6 + 3 * l + c), K[l] + e);
			}
		}
	}
#pragma unroll
	for (int u = 0; u < STAGE_CPT; ++u) {
		const int x = tx * (blockDim.x * STAGE_CPT) + threadIdx.x + u * blockDim.x;
		if (in[u] && DELTA) {
			const V3<T> hd = (a.terms & MM_TERM_DEMAG) ? load3(Hd, idx[u], n) : v3<T>(0, 0, 0);
			V3<T> Tt;
			const bool mat = cell_rhs_delta<T>(a, msr, y_in, n, x, yy, z, idx[u], load3(yhi, idx[u], n),
			                                   load3(hb, idx[u], n), hd, t, Tt, ki[u]);
			if (TORQUE && mat) {
				const T ms = mat_of(a, idx[u]).Ms;
				tq2 = nan_max(tq2, dot(Tt, Tt) / (ms * ms));
			}
		} else if (in[u]) {
			V3<T> Heff;
			const V3<T> hd = (a.terms & MM_TERM_DEMAG) ? load3(Hd, idx[u], n) : v3<T>(0, 0, 0);
			cell_rhs<T>(a, msr, y_in, n, x, yy, z, idx[u], hd, t, Heff, ki[u]);
			if (TORQUE) {
				const T ms = mat_of(a, idx[u]).Ms;
				if (ms != T(0)) {
					const V3<T> c = cross(load3(y_in, idx[u], n), Heff);
					tq2 = nan_max(tq2, dot(c, c) / (ms * ms));
				}
			}
		}
	}
	cp_async_wait_all();
#pragma unroll
	for (int u = 0; u < STAGE_CPT; ++u) {
		if (!in[u]) continue;
		const size_t i = idx[u];
		if (!s_last) {
			if (s_wnext) {
				V3<T> acc = COMP ? pre3(u, 3) : pre3(u, 0);
#pragma unroll
				for (int l = 0; l < S; ++l) {
					const T f = (T)(h * sc.bn[l]);
					if (CT ? pat_bit(PAT, 11 + l) : f != T(0)) acc = acc + f * pre3(u, 6 + 3 * l);
				}
				acc = acc + (T)(h * sc.bn[S]) * ki[u];
				if (COMP && !DELTA) acc = pre3(u, 0) + acc;
				store3(y_out, i, n, acc);
			}
			if (s_rk0) {
				const V3<T> k0 = S == 0 ? ki[u] : pre3(u, 6);
				k02 = max(k02, dot(k0, k0));
			}
		} else {
			V3<T> err = v3<T>(0, 0, 0);
			V3<T> acc = v3<T>(0, 0, 0);
#pragma unroll
			for (int l = 0; l <= S; ++l) {
				const T fe = (T)(h * sc.ec[l]);
				const T fc = (T)(h * sc.bn[l]);
				if (CT ? (!pat_bit(PAT, 18 + l) && (!s_wnew || !pat_bit(PAT, 11 + l)))
				       : (fe == T(0) && (!s_wnew || fc == T(0))))
					continue;
				const V3<T> kl = l == S ? ki[u] : pre3(u, 6 + 3 * l);
				err = err + fe * kl;
				if (s_wnew) acc = acc + fc * kl;
			}
			e2 = nan_max(e2, dot(err, err));
			if (s_wnew) {
				if (DELTA) {
					store3(y_out, i, n, pre3(u, 3) + acc);  // deviation of y_{n+1} from the base state
				} else if (COMP) {
					// y_{n+1} = hi + (lo + delta) with an error-free sum: new hi + new lo
					const V3<T> hi = pre3(u, 0);
					const V3<T> d = pre3(u, 3) + acc;
					const V3<T> s = hi + d;
					const V3<T> bb = s - hi;
					const V3<T> lo = (hi - (s - bb)) + (d - bb);
					store3(y_out, i, n, s);
					store3(y_out_lo, i, n, lo);
				} else {
					store3(y_out, i, n, pre3(u, 0) + acc);
				}
			}
		}
		store3(K[S], i, n, ki[u]);
	}
}

template <typename T, bool COMP, int S>
__global__ void __launch_bounds__(256, stage_min_blocks<T>())
    k_stage(CellArgs<T> a, StageCoef sc, const T *__restrict__ y_in, const T *__restrict__ Hd,
            const T *__restrict__ yhi, const T *__restrict__ ylo, const KTab<T> *__restrict__ ktab,
            T *__restrict__ y_out, T *__restrict__ y_out_lo, const DevState *__restrict__ st, double *red_err,
            double *red_k0, int tiles_x, int tiles_y, int ntiles)
{
	__shared__ T msr[256];
	extern __shared__ __align__(16) unsigned char stage_pre[];
	load_ms_table(a, msr);
	T *const *K = ktab->k;
	T e2 = T(0), k02 = T(0), tq2 = T(0);
	for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
		stage_tile<T, COMP, S, false>(a, msr, sc, y_in, Hd, yhi, ylo, K, y_out, y_out_lo, st, tile, tiles_x, tiles_y,
		                              e2, k02, tq2, reinterpret_cast<T *>(stage_pre));
	if (sc.last) block_max_to(red_err, e2);
	if (sc.reduce_k0) block_max_to(red_k0, k02);
}

// ---- Staged fused stage (single instance) -------------------------------------------------------
// Column tiles of ST_X x ST_Y cells march through z.  A step (one tile plane) needs the stage input
// y_in of planes z-1, z, z+1 with a one-cell halo in x and y, their region ids, and the per-cell
// operands of plane z (stage_ops).  Everything arrives in shared memory by tensor-map copies
// (cp.async.bulk.tensor) issued ST_AHEAD steps ahead by one thread: a halo plane is one box of
// (ST_X + 8) x (ST_Y + 2) x 3 components starting at x0 - 4 (16-byte aligned; the box edges past
// the grid read as zero and are never used, the stencil treats those neighbours as absent), its
// region ids one box starting at x0 - 16, each operand one box of ST_X x ST_Y x 3.  Halo planes go
// to a ring (each plane of a tile is loaded once), operands to ST_NOB buffers.  Each CTA
// takes an equal contiguous range of the (tile, z) steps, so the work is balanced to one step.
constexpr int ST_X = 64, ST_Y = 4;
constexpr int ST_CPT = 1;                        // cells per consumer thread and step
constexpr int ST_CONS = ST_X * ST_Y / ST_CPT;    // consumer threads (plus one producer warp)
constexpr int ST_XH = ST_X + 8;   // y_in row: x0 - 4 .. x0 + ST_X + 4
constexpr int ST_XR = ST_X + 32;  // region row: x0 - 16 .. x0 + ST_X + 16
constexpr int ST_YH = ST_Y + 2;
constexpr int ST_AHEAD = 1;             // steps whose copies are in flight while one is computed
constexpr int ST_RING = ST_AHEAD + 3;   // halo planes: the three being read plus the ones arriving
constexpr int ST_NOB = ST_AHEAD + 1;    // operand buffers

// Tensor maps of one stage launch: the stage input, region ids, demag field, y_n and its
// compensation, and every physical stage-vector buffer (the launch finds the buffer behind each
// k_l of the device-side table, which first-same-as-last tableaus permute).
struct StageMaps {
	CUtensorMap yin, reg, hd, hi, lo;
	CUtensorMap k[MAXS];
	const void *kptr[MAXS];
};

template <typename T>
struct StTmaGeom {
	static constexpr size_t YSLOT = ((size_t)3 * ST_YH * ST_XH * sizeof(T) + 127) / 128 * 128;  // bytes
	static constexpr size_t YBOX = (size_t)3 * ST_YH * ST_XH * sizeof(T);
	static constexpr size_t RSLOT = ((size_t)ST_YH * ST_XR + 127) / 128 * 128;
	static constexpr size_t RBOX = (size_t)ST_YH * ST_XR;
	static constexpr size_t YB = ST_RING * YSLOT;
	static constexpr size_t RB = ST_RING * RSLOT;
	static constexpr size_t OPB = (size_t)3 * ST_Y * ST_X * sizeof(T);  // one operand, one plane
	static constexpr size_t smem(int nops)
	{
		return YB + RB + ST_NOB * (size_t)nops * OPB + 8 * (ST_RING + 2 * ST_NOB);
	}
	static constexpr int MINB = sizeof(T) == 4 ? 3 : 1;
};

// Whether a box takes the staged stage kernel: rows of y_in (and of the region ids) start on
// 16-byte boundaries, and every element index of a 3N vector fits 32 bits (the consumers address
// their stores with 32-bit offsets).
inline bool stage_tma_fits(int nx, size_t esize, bool regions, size_t ncells)
{
	return (nx * esize) % 16 == 0 && (!regions || nx % 16 == 0) && 3 * ncells < (size_t)1 << 31;
}

template <typename T, bool COMP, int S, int TM, int PAT = PAT_RUNTIME>
__global__ void __launch_bounds__(ST_CONS + 32, StTmaGeom<T>::MINB)
    k_stage_tma(const __grid_constant__ StageMaps maps, CellArgs<T> a, StageCoef sc, const KTab<T> *__restrict__ ktab,
                T *__restrict__ y_out, T *__restrict__ y_out_lo, DevState *__restrict__ st, int tiles_x,
                int tiles_y)
{
	using G = StTmaGeom<T>;
	__shared__ T msr[256];
	__shared__ const CUtensorMap *opmap[MAXS + 3];
	__shared__ T fb[MAXS], fe[MAXS];  // h b_l and h e_l at working precision
	__shared__ int abort_flag;
	extern __shared__ __align__(128) unsigned char smem_st[];
	unsigned char *ys = smem_st;
	uint8_t *rs = smem_st + G::YB;
	T *os = reinterpret_cast<T *>(smem_st + G::YB + G::RB);
	const bool demag = term_on<TM>(a, MM_TERM_DEMAG);
	int kop[MAXS], op_hd, op_hi, op_lo;
	const int nops = stage_ops(sc, S, COMP, demag, kop, op_hd, op_hi, op_lo);
	// the consumers' view of the stage structure: compile-time constants under a pattern (the host
	// launches a pattern only where it equals the coefficients' own, and only with the demag term)
	constexpr bool CT = PAT != PAT_RUNTIME;
	static_assert(!CT || (TM >= 0 && (TM & MM_TERM_DEMAG)), "stage patterns assume a fixed term set with demag");
	const bool s_last = CT ? pat_bit(PAT, 7) : sc.last != 0;
	const bool s_wnext = CT ? pat_bit(PAT, 8) : sc.write_next != 0;
	const bool s_wnew = CT ? pat_bit(PAT, 9) : sc.write_new != 0;
	const bool s_rk0 = CT ? pat_bit(PAT, 10) : sc.reduce_k0 != 0;
	constexpr bool CT_OUT = CT && (pat_bit(PAT, 7) ? pat_bit(PAT, 9) : pat_bit(PAT, 8));
	const int c_hd = CT ? 0 : op_hd, c_hi = CT ? (CT_OUT ? 1 : -1) : op_hi,
	          c_lo = CT ? (CT_OUT && COMP ? 2 : -1) : op_lo;
	auto c_kop = [&](int l) -> int { return CT ? pat_kop(PAT, COMP, true, l) : kop[l]; };
	const int c_nops = CT ? pat_nops(PAT, COMP, true) : nops;
	// barriers: halo planes arrived [ST_RING], operands arrived [ST_NOB], step done [ST_NOB]
	uint64_t *bar = reinterpret_cast<uint64_t *>(smem_st + G::YB + G::RB + ST_NOB * (size_t)nops * G::OPB);
	uint64_t *bar_o = bar + ST_RING, *bar_done = bar + ST_RING + ST_NOB;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	constexpr int CONSUMERS = ST_CONS / 32;
	const int nx = a.nx, ny = a.ny, nz = a.nz;
	const size_t n = (size_t)nx * ny * nz;
	if (tid == 0) {
		for (int b = 0; b < ST_RING + ST_NOB; ++b) mbar_init(&bar[b], 1);
		for (int b = 0; b < ST_NOB; ++b) mbar_init(&bar_done[b], CONSUMERS);
		fence_proxy_async();
		abort_flag = 0;
		if (op_hd >= 0) opmap[op_hd] = &maps.hd;
		if (op_hi >= 0) opmap[op_hi] = &maps.hi;
		if (op_lo >= 0) opmap[op_lo] = &maps.lo;
		for (int l = 0; l < MAXS; ++l) {
			fb[l] = (T)(st->h * sc.bn[l]);
			fe[l] = (T)(st->h * sc.ec[l]);
		}
		for (int l = 0; l < MAXS; ++l) {
			if (kop[l] < 0) continue;
			const void *p = ktab->k[l];
			opmap[kop[l]] = &maps.k[0];
			for (int q = 0; q < MAXS; ++q)
				if (maps.kptr[q] == p) opmap[kop[l]] = &maps.k[q];
		}
	}
	load_ms_table(a, msr);  // ends with __syncthreads
	const long long nsteps = (long long)tiles_x * tiles_y * nz;
	const int L0 = (int)(nsteps * blockIdx.x / gridDim.x), L1 = (int)(nsteps * (blockIdx.x + 1) / gridDim.x);
	// a step's position: plane z of the column tile at (x0, y0); advanced without divisions
	struct Pos {
		int x0, y0, z;
	};
	auto advance = [&](Pos &q) {
		if (++q.z < nz) return;
		q.z = 0;
		q.x0 += ST_X;
		if (q.x0 < nx) return;
		q.x0 = 0;
		q.y0 += ST_Y;
	};
	Pos start;
	{
		const int tile = L0 / nz;
		start.z = L0 - tile * nz;
		start.x0 = (tile % tiles_x) * ST_X;
		start.y0 = (tile / tiles_x) * ST_Y;
	}
	// halo planes get consecutive ring indices g (plane g in slot g % ST_RING, its k-th use of the
	// slot completing phase k); a step that starts a tile (or the CTA's range) loads planes z-1,
	// z, z+1, a later one plane z+1.  Returns the ring index of plane z; g_next counts the planes.
	auto plan = [&](const Pos &q, bool first, int &g_next) -> int {
		int gz;
		if (first) {
			if (q.z > 0) ++g_next;
			gz = g_next++;
		} else {
			gz = g_next - 1;
		}
		if (q.z + 1 < nz) ++g_next;
		return gz;
	};
	T e2 = T(0), k02 = T(0);
	int prod_j = 0, prod_g = 0;  // steps and halo planes whose copies the producer issued

	if (warp == CONSUMERS) {
		// producer: issues step j's copies once step j - ST_NOB (the last reader of the buffers
		// they overwrite) is done
		if (lane == 0) {
			Pos q = start;
			int g_next = 0;
			for (int j = 0; L0 + j < L1; ++j, advance(q)) {
				if (j >= ST_NOB) {
					const int d = j - ST_NOB;
					bool ok = false;
					if (!*(volatile int *)&abort_flag) ok = mbar_wait(&bar_done[d % ST_NOB], (d / ST_NOB) & 1);
					if (!ok) {
						*(volatile int *)&abort_flag = 1;
						break;
					}
				}
				fence_proxy_async();
				const int g0 = g_next;
				plan(q, j == 0 || q.z == 0, g_next);
				for (int g = g0; g < g_next; ++g) {
					const int p = q.z + 1 - (g_next - 1 - g) - (q.z + 1 < nz ? 0 : 1);
					uint64_t *b = &bar[g % ST_RING];
					mbar_expect_tx(b, (uint32_t)(G::YBOX + (a.reg ? G::RBOX : 0)));
					tma_load_4d(ys + (g % ST_RING) * G::YSLOT, &maps.yin, q.x0 - 4, q.y0 - 1, p, 0, b);
					if (a.reg) tma_load_3d(rs + (g % ST_RING) * G::RSLOT, &maps.reg, q.x0 - 16, q.y0 - 1, p, b);
				}
				const int ob = j % ST_NOB;
				uint64_t *b = &bar_o[ob];
				mbar_expect_tx(b, (uint32_t)(nops * G::OPB));
				for (int k = 0; k < nops; ++k)
					tma_load_4d(os + (size_t)(ob * nops + k) * 3 * ST_Y * ST_X, opmap[k], q.x0, q.y0, q.z, 0, b);
				prod_j = j + 1;
				prod_g = g_next;
			}
		}
	} else {
		// consumers: ST_CPT cells per thread and step
		T *const kS = ktab->k[S];
		const double t = st->t + sc.a_i * st->h;
		const V3<T> Hz = zeeman_field(a, t);
		const int lx = tid % ST_X, ly0 = tid / ST_X;  // cells (lx, ly0 + u ST_Y / ST_CPT)
		const int hc = lx + 4;
		Pos cur = start;
		int g_next = 0, g_waited = 0;
		for (int j = 0; L0 + j < L1; ++j, advance(cur)) {
			const int z = cur.z, x0 = cur.x0, y0 = cur.y0;
			const int gz = plan(cur, j == 0 || z == 0, g_next);
			const int ob = j % ST_NOB;
			// every lane waits (a completed phase returns at once), so each lane's reads follow
			// its own observation of the copies
			bool late = *(volatile int *)&abort_flag != 0;
			const int g_need = gz + (z + 1 < nz ? 1 : 0);
			for (; !late && g_waited <= g_need; ++g_waited)
				late = !mbar_wait(&bar[g_waited % ST_RING], (g_waited / ST_RING) & 1);
			if (!late) late = !mbar_wait(&bar_o[ob], (j / ST_NOB) & 1);
			if (__any_sync(0xffffffffu, late)) {
				if (lane == 0) *(volatile int *)&abort_flag = 1;
				break;
			}
#pragma unroll
			for (int u = 0; u < ST_CPT; ++u) {
				const int ly = ly0 + u * (ST_Y / ST_CPT), hr = ly + 1;
				const int x = x0 + lx, yy = y0 + ly;
				if (x < nx && yy < ny) {
					const uint32_t i = ((uint32_t)z * ny + yy) * nx + x, n32 = (uint32_t)n;
					// this cell in the ring slots of planes z-1, z, z+1 (component stride YC) and in
					// the operand buffer (operand stride OS, component stride OC); 32-bit offsets
					constexpr int YC = ST_YH * ST_XH, OC = ST_Y * ST_X, OS = 3 * OC;
					const int cell_off = hr * ST_XH + hc;
					const T *yz = reinterpret_cast<const T *>(ys + (gz % ST_RING) * G::YSLOT) + cell_off;
					const T *ym = reinterpret_cast<const T *>(ys + ((gz + ST_RING - 1) % ST_RING) * G::YSLOT) + cell_off;
					const T *yp = reinterpret_cast<const T *>(ys + ((gz + 1) % ST_RING) * G::YSLOT) + cell_off;
					const int rcell = hr * ST_XR + hc + 12;
					const uint8_t *rz = rs + (gz % ST_RING) * G::RSLOT + rcell;
					const uint8_t *rm = rs + ((gz + ST_RING - 1) % ST_RING) * G::RSLOT + rcell;
					const uint8_t *rp = rs + ((gz + 1) % ST_RING) * G::RSLOT + rcell;
					const T *oc = os + ob * c_nops * OS + ly * ST_X + lx;
					auto O3 = [&](int k) -> V3<T> {
						const T *o = oc + k * OS;
						return v3<T>(o[0], o[OC], o[2 * OC]);
					};
					auto Y3 = [&](const T *p, int off) -> V3<T> { return v3<T>(p[off], p[off + YC], p[off + 2 * YC]); };
					const int rg = a.reg ? *rz : 0;
					const DevMat<T> &M = a.mat[rg < a.nmat ? rg : 0];
					const V3<T> hd = demag ? O3(c_hd) : v3<T>(0, 0, 0);
					V3<T> Heff, ki;
					if (M.Ms == T(0)) {
						ki = v3<T>(0, 0, 0);
					} else {
						const V3<T> m = Y3(yz, 0);
						const bool has[6] = {x > 0, x < nx - 1, yy > 0, yy < ny - 1, z > 0, z < nz - 1};
						const T *yq[6] = {yz, yz, yz, yz, ym, yp};
						const uint8_t *rq[6] = {rz, rz, rz, rz, rm, rp};
						const int dq[6] = {-1, 1, -ST_XH, ST_XH, 0, 0};
						const int drq[6] = {-1, 1, -ST_XR, ST_XR, 0, 0};
						V3<T> nb[6];
						T nms[6];
						// every neighbour read stays inside the staged planes (the halo past the grid
						// reads as zero, a missing plane z -+ 1 is a stale ring slot), so the reads
						// are unconditional and the neighbours outside the box are masked afterwards:
						// their Ms always (the halo's region ids read as region 0), their m only
						// along z (an x or y neighbour past the grid is the zero fill already)
#pragma unroll
						for (int q = 0; q < 6; ++q) {
							const V3<T> v = Y3(yq[q], dq[q]);
							const T ms_q = a.reg ? msr[rq[q][drq[q]]] : M.Ms;
							nb[q] = (q < 4 || has[q]) ? v : v3<T>(0, 0, 0);
							nms[q] = has[q] ? ms_q : T(0);
						}
						cell_core<T, TM>(a, M, m, nb, nms, x, yy, z, hd, Hz, Heff, ki);
					}
					T *const pk = kS + i, *const py = y_out + i;
					auto put3 = [&](T *p, V3<T> v) {
						p[0] = v.x;
						p[n32] = v.y;
						p[2 * n32] = v.z;
					};
					if (!s_last) {
						if (s_wnext) {
							V3<T> acc = COMP ? O3(c_lo) : O3(c_hi);
#pragma unroll
							for (int l = 0; l < S; ++l) {
								const T f = fb[l];
								if (CT ? pat_bit(PAT, 11 + l) : f != T(0)) acc = acc + f * O3(c_kop(l));
							}
							acc = acc + fb[S] * ki;
							if (COMP) acc = O3(c_hi) + acc;
							put3(py, acc);
						}
						if (s_rk0) {
							const V3<T> k0 = S == 0 ? ki : O3(c_kop(0));
							k02 = max(k02, dot(k0, k0));
						}
					} else {
						V3<T> err = v3<T>(0, 0, 0);
						V3<T> acc = v3<T>(0, 0, 0);
#pragma unroll
						for (int l = 0; l <= S; ++l) {
							const T fel = fe[l];
							const T fc = fb[l];
							if (CT ? (!pat_bit(PAT, 18 + l) && (!s_wnew || !pat_bit(PAT, 11 + l)))
							       : (fel == T(0) && (!s_wnew || fc == T(0))))
								continue;
							const V3<T> kl = l == S ? ki : O3(c_kop(l));
							err = err + fel * kl;
							if (s_wnew) acc = acc + fc * kl;
						}
						e2 = nan_max(e2, dot(err, err));
						if (s_wnew) {
							if (COMP) {
								// y_{n+1} = hi + (lo + delta) with an error-free sum: new hi + new lo
								const V3<T> hi = O3(c_hi);
								const V3<T> d = O3(c_lo) + acc;
								const V3<T> s = hi + d;
								const V3<T> bb = s - hi;
								const V3<T> lo = (hi - (s - bb)) + (d - bb);
								put3(py, s);
								put3(y_out_lo + i, lo);
							} else {
								put3(py, O3(c_hi) + acc);
							}
						}
					}
					put3(pk, ki);
				}
			}
			__syncwarp();
			if (lane == 0) mbar_arrive(&bar_done[ob]);
		}
	}
	__syncthreads();  // producer and consumers joined
	if (warp == CONSUMERS && lane == 0) {
		// let every copy issued land before the CTA can retire (immediate unless a wait gave up):
		// wait for the last phase armed on each barrier
		for (int b = 0; b < ST_NOB && b < prod_j; ++b)
			mbar_wait(&bar_o[b], ((b + ((prod_j - 1 - b) / ST_NOB) * ST_NOB) / ST_NOB) & 1);
		for (int sl = 0; sl < ST_RING && sl < prod_g; ++sl)
			mbar_wait(&bar[sl], ((sl + ((prod_g - 1 - sl) / ST_RING) * ST_RING) / ST_RING) & 1);
	}
	if (abort_flag) {
		if (tid == 0) atomicExch(&st->stage_timeout, 1);
		return;
	}
	if (sc.last) block_max_to(&st->max_err2, e2);
	if (sc.reduce_k0) block_max_to(&st->max_k02, k02);
}

// Accepted step: m <- y_{n+1} / |y_{n+1}| (VectorMatrix::normalize to Ms, in unit form).
template <typename T, bool COMP>
__device__ __forceinline__ void accept_cell(size_t n, const T *__restrict__ ynew, const T *__restrict__ ynew_lo,
                                            T *__restrict__ m, T *__restrict__ m_lo, size_t i)
{
	{
		if (COMP) {
			const double x = (double)ynew[i] + (double)ynew_lo[i];
			const double y = (double)ynew[i + n] + (double)ynew_lo[i + n];
			const double z = (double)ynew[i + 2 * n] + (double)ynew_lo[i + 2 * n];
			const double len = sqrt(x * x + y * y + z * z);
			const double s = len > 0 ? 1.0 / len : 0.0;
			const double v[3] = {x * s, y * s, z * s};
			for (int c = 0; c < 3; ++c) {
				const float hi = (float)v[c];
				m[i + c * n] = hi;
				m_lo[i + c * n] = (float)(v[c] - (double)hi);
			}
		} else {
			const V3<T> v = load3(ynew, i, n);
			const T len = sqrt(dot(v, v));
			store3(m, i, n, len > T(0) ? (T(1) / len) * v : v3<T>(0, 0, 0));
		}
	}
}

template <typename T, bool COMP>
__global__ void __launch_bounds__(256) k_accept(size_t n, const T *__restrict__ ynew,
                                                const T *__restrict__ ynew_lo, T *__restrict__ m,
                                                T *__restrict__ m_lo)
{
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
		accept_cell<T, COMP>(n, ynew, ynew_lo, m, m_lo, i);
}

// MicroMagneticsStepSizeController.adjust_stepsize (micro_magnetics_stepsize_controller.py:
// 35-73), in double, on one thread; also swaps k_0 / k_last for first-same-as-last tableaus.
template <typename T>
__device__ __forceinline__ void control_attempt(DevState *st, KTab<T> *ktab, double eps_abs, double eps_rel,
                                                int order, int fsal, int s, DevState *host_copy,
                                                const int *conv_timeout)
{
	const double h = st->h;
	const double e_abs = sqrt(st->max_err2);
	const double max_dydt = sqrt(st->max_k02);
	int accept;
	double h_new;
	const int finite = isfinite(e_abs) && isfinite(max_dydt);
	if (h * max_dydt == 0.0) {
		accept = 1;
		h_new = 5e-14;
	} else {
		const double e_rel = e_abs / (h * max_dydt);
		accept = (e_abs <= eps_abs) && (e_rel <= eps_rel);
		// e_abs == 0 (ZeroDivisionError in the reference) grows the step by the maximum factor
		const double sa = e_abs > 0 ? 0.85 * pow(eps_abs / e_abs, 1.0 / (order + 1.0)) : 5.0;
		const double sr = e_rel > 0 ? 0.85 * pow(eps_rel / e_rel, 1.0 / order) : 5.0;
		double sc = fmin(sa, sr);
		sc = fmin(fmax(sc, 0.2), 5.0);
		h_new = fmin(fmax(h * sc, 1e-15), 1e-10);
		if (h_new == 1e-15) accept = 1;
	}
	const int timed_out = (conv_timeout ? *conv_timeout : 0) | st->stage_timeout;
	if (!finite || timed_out) accept = 0;
	st->accept = accept;
	st->h_new = h_new;
	st->not_finite = timed_out ? 2 : !finite;
	if (host_copy) *host_copy = *st;
	st->max_err2 = 0.0;
	st->max_k02 = 0.0;
	if (fsal) {
		T *t = ktab->k[0];
		ktab->k[0] = ktab->k[s - 1];
		ktab->k[s - 1] = t;
	}
}

template <typename T>
__global__ void k_controller(DevState *st, KTab<T> *ktab, double eps_abs, double eps_rel, int order,
                             int fsal, int s, DevState *host_copy, const int *conv_timeout)
{
	control_attempt<T>(st, ktab, eps_abs, eps_rel, order, fsal, s, host_copy, conv_timeout);
}

// Effective field and dM/dt in A/m (FP64 outputs) at the state m.
template <typename T>
__global__ void __launch_bounds__(256) k_eval(CellArgs<T> a, const T *__restrict__ m,
                                              const T *__restrict__ Hd, double t,
                                              double *__restrict__ Heff_out,
                                              double *__restrict__ dMdt_out,
                                              double *__restrict__ Hd_out)
{
	__shared__ T msr[256];
	load_ms_table(a, msr);
	const int x = blockIdx.x * blockDim.x + threadIdx.x;
	const int yy = blockIdx.y * blockDim.y + threadIdx.y;
	const int z = blockIdx.z;
	if (x >= a.nx || yy >= a.ny) return;
	const size_t n = (size_t)a.nx * a.ny * a.nz;
	const size_t i = ((size_t)z * a.ny + yy) * a.nx + x;
	V3<T> Heff, dm;
	const V3<T> hd = (a.terms & MM_TERM_DEMAG) ? load3(Hd, i, n) : v3<T>(0, 0, 0);
	cell_rhs<T>(a, msr, m, n, x, yy, z, i, hd, t, Heff, dm);
	const double ms = (double)mat_of(a, i).Ms;
	if (Heff_out) { Heff_out[i] = Heff.x; Heff_out[i + n] = Heff.y; Heff_out[i + 2 * n] = Heff.z; }
	if (dMdt_out) { dMdt_out[i] = ms * dm.x; dMdt_out[i + n] = ms * dm.y; dMdt_out[i + 2 * n] = ms * dm.z; }
	if (Hd_out) { Hd_out[i] = hd.x; Hd_out[i + n] = hd.y; Hd_out[i + 2 * n] = hd.z; }
}

// Relaxation norms of the current state, reduced into red[0..2]: max |dM/dt|^2 [(A/(m s))^2],
// max |M|^2 [(A/m)^2] (VectorMatrix::absMax, squared) and max (|m x H_eff| / Ms)^2 over cells
// with Ms != 0 (the torque criterion of batched relaxations).
template <typename T>
__global__ void __launch_bounds__(256) k_relax_norms(CellArgs<T> a, const T *__restrict__ m,
                                                     const T *__restrict__ Hd, double t, double *red)
{
	__shared__ T msr[256];
	load_ms_table(a, msr);
	const int x = blockIdx.x * blockDim.x + threadIdx.x;
	const int yy = blockIdx.y * blockDim.y + threadIdx.y;
	const int z = blockIdx.z;
	double dm2 = 0.0, M2 = 0.0, tq2 = 0.0;
	if (x < a.nx && yy < a.ny) {
		const size_t n = (size_t)a.nx * a.ny * a.nz;
		const size_t i = ((size_t)z * a.ny + yy) * a.nx + x;
		V3<T> Heff, dm;
		const V3<T> hd = (a.terms & MM_TERM_DEMAG) ? load3(Hd, i, n) : v3<T>(0, 0, 0);
		cell_rhs<T>(a, msr, m, n, x, yy, z, i, hd, t, Heff, dm);
		const double ms = (double)mat_of(a, i).Ms;
		if (ms != 0.0) {
			const V3<T> mi = load3(m, i, n);
			const double mx = mi.x, my = mi.y, mz = mi.z;
			const double hx = Heff.x, hy = Heff.y, hz = Heff.z;
			const double cx = my * hz - mz * hy, cy = mz * hx - mx * hz, cz = mx * hy - my * hx;
			dm2 = ms * ms * ((double)dm.x * dm.x + (double)dm.y * dm.y + (double)dm.z * dm.z);
			M2 = ms * ms * (mx * mx + my * my + mz * mz);
			tq2 = (cx * cx + cy * cy + cz * cz) / (ms * ms);
		}
	}
	block_max_to(red, dm2);
	block_max_to(red + 1, M2);
	block_max_to(red + 2, tq2);
}

// Energy sums of the current state, accumulated into acc[0..4]: sum M.H_demag, sum M.H_exch,
// sum k_u |a x m|^2, sum k_c (s1 s2 + s1 s3 + s2 s3), sum M.H_ext (the reference's E_stray,
// E_exch, E_aniso and E_ext before their prefactors: stray_field.py:49-52, exchange_field.py:57-58,
// anisotropy_cpu.cpp:29-119 (the CPU path's energy forms), external_field.py:34-35).  k_u and
// k_c are recovered from the material record (ku = 2 k_u / (mu0 Ms), kc = -2 k_c / (mu0 Ms)).
template <typename T>
__global__ void __launch_bounds__(256) k_energies(CellArgs<T> a, const T *__restrict__ m,
                                                  const T *__restrict__ Hd, double t, double *acc)
{
	__shared__ T msr[256];
	load_ms_table(a, msr);
	const int x = blockIdx.x * blockDim.x + threadIdx.x;
	const int yy = blockIdx.y * blockDim.y + threadIdx.y;
	const int z = blockIdx.z;
	double es = 0.0, ex = 0.0, eu = 0.0, ec = 0.0, ez = 0.0;
	if (x < a.nx && yy < a.ny) {
		const size_t n = (size_t)a.nx * a.ny * a.nz;
		const size_t i = ((size_t)z * a.ny + yy) * a.nx + x;
		const DevMat<T> &M = mat_of(a, i);
		const double ms = (double)M.Ms;
		if (ms != 0.0) {
			const V3<T> mi = load3(m, i, n);
			const double mx = ms * (double)mi.x, my = ms * (double)mi.y, mz = ms * (double)mi.z;
			if (a.terms & MM_TERM_DEMAG) {
				const V3<T> h = load3(Hd, i, n);
				es = mx * h.x + my * h.y + mz * h.z;
			}
			if (a.terms & MM_TERM_EXCHANGE) {
				bool has[6];
				size_t off[6];
				neighbours(a, x, yy, z, i, has, off);
				const T w[6] = {a.wx, a.wx, a.wy, a.wy, a.wz, a.wz};
				V3<T> sum = v3<T>(0, 0, 0);
#pragma unroll
				for (int q = 0; q < 6; ++q) {
					if (!has[q]) continue;
					const T nms = a.reg ? msr[a.reg[off[q]]] : M.Ms;
					if (nms != T(0)) sum = sum + w[q] * (load3(m, off[q], n) - mi);
				}
				const V3<T> h = M.cex * sum;
				ex = mx * h.x + my * h.y + mz * h.z;
			}
			if ((a.terms & MM_TERM_UNIAXIAL) && M.ku != T(0)) {
				const double k = (double)M.ku * MU0 * ms / 2.0;
				const double ax = M.a1[0], ay = M.a1[1], az = M.a1[2];
				const double ux = mi.x, uy = mi.y, uz = mi.z;
				const double cx = ay * uz - az * uy, cy = az * ux - ax * uz, cz = ax * uy - ay * ux;
				eu = k * (cx * cx + cy * cy + cz * cz);
			}
			if ((a.terms & MM_TERM_CUBIC) && M.kc != T(0)) {
				const double k = -(double)M.kc * MU0 * ms / 2.0;
				const double ux = mi.x, uy = mi.y, uz = mi.z;
				const double len = sqrt(ux * ux + uy * uy + uz * uz);
				const double s = len > 0 ? 1.0 / len : 0.0;
				const double p1 = s * (M.a1[0] * ux + M.a1[1] * uy + M.a1[2] * uz);
				const double p2 = s * (M.a2[0] * ux + M.a2[1] * uy + M.a2[2] * uz);
				const double p3 = s * (M.a3[0] * ux + M.a3[1] * uy + M.a3[2] * uz);
				const double s1 = p1 * p1, s2 = p2 * p2, s3 = p3 * p3;
				ec = k * (s1 * s2 + s1 * s3 + s2 * s3);
			}
			if (a.terms & MM_TERM_ZEEMAN) {
				const V3<T> h = zeeman_field(a, t);
				ez = mx * h.x + my * h.y + mz * h.z;
			}
		}
	}
	block_sum_to(acc, es);
	block_sum_to(acc + 1, ex);
	block_sum_to(acc + 2, eu);
	block_sum_to(acc + 3, ec);
	block_sum_to(acc + 4, ez);
}

// M (A/m, FP64) -> unit state, normalised (LandauLifshitzGilbert.update("M")).
template <typename T, bool COMP>
__global__ void k_set_M(size_t n, const double *__restrict__ M, const uint8_t *__restrict__ reg,
                        const DevMat<T> *__restrict__ mat, T *__restrict__ m, T *__restrict__ m_lo)
{
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
		const double ms = (double)mat[reg ? reg[i] : 0].Ms;
		const double x = M[i], y = M[i + n], z = M[i + 2 * n];
		const double len = sqrt(x * x + y * y + z * z);
		const double s = (ms != 0.0 && len > 0) ? 1.0 / len : 0.0;
		const double v[3] = {x * s, y * s, z * s};
		for (int c = 0; c < 3; ++c) {
			const T hi = (T)v[c];
			m[i + c * n] = hi;
			if (COMP) m_lo[i + c * n] = (T)(v[c] - (double)hi);
		}
	}
}

template <typename T, bool COMP>
__global__ void k_get_M(size_t n, const T *__restrict__ m, const T *__restrict__ m_lo,
                        const uint8_t *__restrict__ reg, const DevMat<T> *__restrict__ mat,
                        double *__restrict__ M)
{
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
		const double ms = (double)mat[reg ? reg[i] : 0].Ms;
		for (int c = 0; c < 3; ++c) {
			double v = (double)m[i + c * n];
			if (COMP) v += (double)m_lo[i + c * n];
			M[i + c * n] = ms * v;
		}
	}
}

template <typename T, bool COMP>
__global__ void __launch_bounds__(256) k_average_M(size_t n, const T *__restrict__ m, const T *__restrict__ m_lo,
                                                   const uint8_t *__restrict__ reg,
                                                   const DevMat<T> *__restrict__ mat, double *out3)
{
	double s[3] = {0, 0, 0};
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
		const double ms = (double)mat[reg ? reg[i] : 0].Ms;
		for (int c = 0; c < 3; ++c) {
			double v = (double)m[i + c * n];
			if (COMP) v += (double)m_lo[i + c * n];
			s[c] += ms * v;
		}
	}
	for (int c = 0; c < 3; ++c) block_sum_to(out3 + c, s[c]);
}

} // namespace mm

using namespace mm;

struct mm_solver {
	mm_solver_config cfg{};
	size_t n = 0;
	int px = 0, py = 0, pz = 0;
	Tableau tab{};
	ConvPlan *conv = nullptr;
	void *mat = nullptr;           // DevMat<T>[nmat]
	void *ms_tab = nullptr;        // T[256] (Ms per region, zero past nmat; the demag input scale)
	uint8_t *reg = nullptr;
	void *m = nullptr, *m_lo = nullptr;        // state (unit), low part (F32)
	void *ys[2] = {nullptr, nullptr};          // stage state ping-pong
	void *ynew_lo = nullptr;                   // F32: low part of y_{n+1}
	void *k[MAXS] = {};
	void *hd = nullptr;                        // demag field
	void *ktab = nullptr;                      // KTab<T> on device
	DevState *dst = nullptr;                   // device state
	DevState *hst = nullptr;                   // pinned host copy of the controller output
	double *avg = nullptr;                     // device scratch for <M>
	double *avg_h = nullptr;                   // pinned
	int last_stage_buf = 0;                    // ys[] index holding y_{n+1}
	int nmat = 1;
	// host-side solver state (RungeKutta.evolve semantics, runge_kutta.py:47-87)
	double t = 0, h = 0, h_next = 0;
	bool have_next = false;
	bool k0_valid = false;
	int64_t steps = 0, attempts = 0, rejected = 0;
	double last_err = 0, last_dmdt = 0;
	int not_finite = 0;
	// host-side copy of the k pointer order (device table is swapped by the controller)
	void *kh[MAXS] = {};
	CellArgs<double> args64{};
	CellArgs<float> args32{};
	// captured attempts (index: first stage evaluated or reused) and their kernel counts
	cudaGraphExec_t gexec[2] = {nullptr, nullptr};
	uint64_t gkernels[2] = {0, 0};
	int glast[2] = {0, 0};
	// graphs are captured and replayed on a private stream (capture is not allowed on the legacy
	// default stream), ordered after / before the caller's stream with events
	cudaStream_t gs = nullptr;
	cudaEvent_t ev_in = nullptr, ev_out = nullptr;
	// staged stage kernel: used when the rows are 16-byte aligned; grid and shared memory per stage
	bool st_tma = false;
	int st_tm = -1;                  // term set the staged kernel is specialised for (-1: run time)
	bool st_pat = false;             // staged kernels compiled for the Dormand-Prince stage patterns
	int st_resident = 0;             // resident blocks of k_stage on this solver's device
	int st_grid[MAXS] = {};
	size_t st_smem[MAXS] = {};
	StageMaps st_maps{};             // yin set per launch from st_yin
	CUtensorMap st_yin[3];           // halo-box maps over m, ys[0], ys[1]
};

namespace mm {
namespace {

inline int grid1(size_t n)
{
	const size_t want = (n + 255) / 256;
	const size_t cap = (size_t)num_sms() * 8;
	return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

template <typename T>
void fill_args(mm_solver *s, CellArgs<T> &a)
{
	const mm_solver_config &c = s->cfg;
	a.nx = c.nx; a.ny = c.ny; a.nz = c.nz;
	a.wx = (T)(1.0 / (c.dx * c.dx)); a.wy = (T)(1.0 / (c.dy * c.dy)); a.wz = (T)(1.0 / (c.dz * c.dz));
	a.idx1 = (T)(1.0 / c.dx); a.idy1 = (T)(1.0 / c.dy); a.idz1 = (T)(1.0 / c.dz);
	a.idx2 = (T)(1.0 / (2 * c.dx)); a.idy2 = (T)(1.0 / (2 * c.dy)); a.idz2 = (T)(1.0 / (2 * c.dz));
	a.terms = c.terms;
	a.pbc = (c.pbc[0] ? 1 : 0) | (c.pbc[1] ? 2 : 0) | (c.pbc[2] ? 4 : 0);
	a.reg = s->reg;
	a.mat = (const DevMat<T> *)s->mat;
	a.nmat = s->nmat;
	for (int q = 0; q < 3; ++q) { a.Hext[q] = c.H_ext[q]; a.Hpulse[q] = c.H_pulse[q]; }
	a.rise = c.pulse_rise;
}

template <typename T>
mm_status build_materials(mm_solver *s, int nmat, const mm_material *mats)
{
	std::vector<DevMat<T>> h(nmat);
	std::vector<T> ms(nmat);
	const mm_solver_config &c = s->cfg;
	for (int r = 0; r < nmat; ++r) {
		const mm_material &m = mats[r];
		DevMat<T> d{};
		const double Ms = m.Ms;
		d.Ms = (T)Ms;
		ms[r] = (T)Ms;
		if (Ms != 0.0) {
			d.cex = (T)((2.0 / MU0) * m.A / Ms);
			// landau_lifshitz_gilbert.py:133-158 factors, scaled to unit m
			const double gp = GYROMAGNETIC_RATIO / (1.0 + m.alpha * m.alpha);
			d.l1 = (T)(c.do_precess ? -gp : 0.0);
			d.l2 = (T)(-m.alpha * gp);
			d.ku = (T)(2.0 * m.k_uniaxial / Ms / MU0);
			d.kc = (T)((-2.0 / MU0) * m.k_cubic / Ms);
			// fdm_zhangli_cpu.cpp:85-101 factors, scaled to unit m and u' = u/Ms
			const double bj = m.P * MU_BOHR / (ELECTRON_CHARGE * Ms * (1.0 + m.xi * m.xi));
			const double bjp = bj / (1.0 + m.alpha * m.alpha);
			const double c1 = c.zl_do_precess ? (1.0 + m.alpha * m.xi) : (m.alpha * m.xi);
			const double c2 = c.zl_do_precess ? (m.xi - m.alpha) : (-m.alpha);
			d.zl1 = (T)(-bjp * c1);
			d.zl2 = (T)(-bjp * c2);
		}
		for (int q = 0; q < 3; ++q) {
			d.a1[q] = (T)m.axis1[q];
			d.a2[q] = (T)m.axis2[q];
			d.j[q] = (T)m.j[q];
		}
		d.a3[0] = (T)(m.axis1[1] * m.axis2[2] - m.axis1[2] * m.axis2[1]);
		d.a3[1] = (T)(m.axis1[2] * m.axis2[0] - m.axis1[0] * m.axis2[2]);
		d.a3[2] = (T)(m.axis1[0] * m.axis2[1] - m.axis1[1] * m.axis2[0]);
		h[r] = d;
	}
	MM_CUDA(cudaMalloc(&s->mat, sizeof(DevMat<T>) * nmat));
	MM_CUDA(cudaMemcpy(s->mat, h.data(), sizeof(DevMat<T>) * nmat, cudaMemcpyHostToDevice));
	MM_CUDA(cudaMalloc(&s->ms_tab, sizeof(T) * 256));  // full 8-bit region range, zero past nmat
	MM_CUDA(cudaMemset(s->ms_tab, 0, sizeof(T) * 256));
	MM_CUDA(cudaMemcpy(s->ms_tab, ms.data(), sizeof(T) * nmat, cudaMemcpyHostToDevice));
	return MM_OK;
}

template <typename T>
mm_status alloc_state(mm_solver *s)
{
	const size_t b3 = sizeof(T) * 3 * s->n;
	const bool comp = s->cfg.precision == MM_F32;
	MM_CUDA(cudaMalloc(&s->m, b3));
	MM_CUDA(cudaMemset(s->m, 0, b3));
	if (comp) {
		MM_CUDA(cudaMalloc(&s->m_lo, b3));
		MM_CUDA(cudaMemset(s->m_lo, 0, b3));
		MM_CUDA(cudaMalloc(&s->ynew_lo, b3));
	}
	for (int q = 0; q < 2; ++q) MM_CUDA(cudaMalloc(&s->ys[q], b3));
	for (int q = 0; q < s->tab.s; ++q) {
		MM_CUDA(cudaMalloc(&s->k[q], b3));
		MM_CUDA(cudaMemset(s->k[q], 0, b3));
		s->kh[q] = s->k[q];
	}
	MM_CUDA(cudaMalloc(&s->hd, b3));
	MM_CUDA(cudaMemset(s->hd, 0, b3));
	KTab<T> kt{};
	for (int q = 0; q < s->tab.s; ++q) kt.k[q] = (T *)s->k[q];
	MM_CUDA(cudaMalloc(&s->ktab, sizeof(KTab<T>)));
	MM_CUDA(cudaMemcpy(s->ktab, &kt, sizeof(kt), cudaMemcpyHostToDevice));
	MM_CUDA(cudaMalloc(&s->dst, sizeof(DevState)));
	MM_CUDA(cudaMemset(s->dst, 0, sizeof(DevState)));
	MM_CUDA(cudaMallocHost(&s->hst, sizeof(DevState)));
	std::memset(s->hst, 0, sizeof(DevState));
	MM_CUDA(cudaMalloc(&s->avg, 8 * sizeof(double)));
	MM_CUDA(cudaMallocHost(&s->avg_h, 8 * sizeof(double)));
	return MM_OK;
}

template <typename T>
const CellArgs<T> &args_of(mm_solver *s);
template <>
const CellArgs<double> &args_of<double>(mm_solver *s) { return s->args64; }
template <>
const CellArgs<float> &args_of<float>(mm_solver *s) { return s->args32; }

dim3 cell_grid(const mm_solver_config &c) { return dim3((c.nx + 31) / 32, (c.ny + 7) / 8, c.nz); }
dim3 stage_grid(const mm_solver_config &c)
{
	return dim3((c.nx + 32 * STAGE_CPT - 1) / (32 * STAGE_CPT), (c.ny + 7) / 8, c.nz);
}

// Device word a staged convolution pass sets when a bounded wait gave up (NULL without one).
const int *conv_timeout_flag(const mm_solver *s) { return s->conv ? s->conv->err : nullptr; }

// Demag field of the state y (unit, T) into s->hd.
template <typename T>
mm_status demag(mm_solver *s, const void *y, cudaStream_t st)
{
	if (!(s->cfg.terms & MM_TERM_DEMAG)) return MM_OK;
	return conv_execute(s->conv, y, s->reg, s->ms_tab, s->hd, st);
}


// Algorithmic bytes of one fused stage launch: stencil input, demag field, region ids, the step
// base, the earlier stages with nonzero weights, and the outputs.
template <typename T>
double stage_bytes(const mm_solver *s, const StageCoef &sc)
{
	const bool comp = sizeof(T) == 4;
	const double v = 3.0 * (double)s->n * sizeof(T);
	double b = v;                                               // y_in
	if (s->cfg.terms & MM_TERM_DEMAG) b += v;                    // H_demag
	if (s->reg) b += (double)s->n;                               // region ids
	b += v;                                                      // k_i written
	const bool out = sc.last ? sc.write_new : sc.write_next;
	if (out) {
		b += v * (comp ? 2 : 1);                                 // y_n (hi, lo)
		b += v * (comp && sc.last ? 2 : 1);                      // y_out (+ lo)
	}
	for (int l = 0; l < sc.stage; ++l)
		if (sc.bn[l] != 0.0 || (sc.last && sc.ec[l] != 0.0)) b += v;
	if (sc.reduce_k0 && sc.stage > 0 && sc.bn[0] == 0.0) b += v;
	return b;
}

// The per-thread-load stage kernel needs more than the default 48 KB of dynamic shared memory.
// The attribute belongs to the current device, so every solver creation sets it on its own device.
template <typename T, bool COMP, int... S>
mm_status stage_smem_attrs(std::integer_sequence<int, S...>)
{
	const int bytes = (int)stage_smem<T>();
	cudaError_t e = cudaSuccess;
	((e = e == cudaSuccess ? cudaFuncSetAttribute(k_stage<T, COMP, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                              bytes)
	                       : e),
	 ...);
	MM_CUDA(e);
	return MM_OK;
}

// Resident blocks of the fused stage kernel on the current device (occupancy of the S = 6
// instance).  Solver creation stores the count in the solver, so that no later call queries
// occupancy during stream capture.
template <typename T, bool COMP>
mm_status stage_resident(int *resident)
{
	MM_TRY((stage_smem_attrs<T, COMP>(std::make_integer_sequence<int, MAXS>())));
	int per_sm = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stage<T, COMP, 6>, 256, stage_smem<T>()) !=
	        cudaSuccess ||
	    per_sm < 1) {
		cudaGetLastError();
		per_sm = stage_min_blocks<T>();
	}
	*resident = per_sm * num_sms();
	return MM_OK;
}

// Launches the fused stage kernel for stage S on a persistent grid of at most the resident blocks.
template <typename T, bool COMP, int S>
void stage_launch(const mm_solver *s, const CellArgs<T> &a, const StageCoef &sc, const T *yin, const T *yhi,
                  const T *ylo, const KTab<T> *kt, T *yout, DevState *ds, cudaStream_t st)
{
	const int resident = s->st_resident;
	const dim3 tg = stage_grid(s->cfg);
	const int ntiles = (int)(tg.x * tg.y * tg.z);
	const int grid = ntiles < resident ? ntiles : resident;
	k_stage<T, COMP, S><<<grid, dim3(32, 8, 1), stage_smem<T>(), st>>>(a, sc, yin, (const T *)s->hd, yhi, ylo, kt, yout,
	                                                     (T *)s->ynew_lo, ds, &ds->max_err2, &ds->max_k02,
	                                                     (int)tg.x, (int)tg.y, ntiles);
}

// Coefficients of stage i of an attempt (i = 0: the k_0 evaluation when it is not reused).
StageCoef stage_coef(const Tableau &tb, int i, bool comp)
{
	StageCoef sc{};
	sc.stage = i;
	sc.a_i = tb.a[i];
	if (i == 0) {
		sc.write_next = 1;
		sc.bn[0] = tb.b[1][0];
		return sc;
	}
	sc.last = (i == tb.s - 1);
	sc.reduce_k0 = (i == 1);
	if (!sc.last) {
		sc.write_next = 1;
		for (int l = 0; l <= i; ++l) sc.bn[l] = tb.b[i + 1][l];
	} else {
		sc.write_new = comp || !tb.fsal;
		for (int l = 0; l <= i; ++l) {
			sc.bn[l] = tb.c[l];
			sc.ec[l] = tb.ec[l];
		}
	}
	return sc;
}

template <typename T, bool COMP, int S>
mm_status stage_tma_prepare(mm_solver *s)
{
	using G = StTmaGeom<T>;
	int kop[MAXS], hd, hi, lo;
	const StageCoef sc = stage_coef(s->tab, S, COMP);
	const int nops = stage_ops(sc, S, COMP, (s->cfg.terms & MM_TERM_DEMAG) != 0, kop, hd, hi, lo);
	const size_t smem = G::smem(nops);
	int dev = 0, optin = 0;
	MM_CUDA(cudaGetDevice(&dev));
	MM_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
	if (smem + 2 * 256 * sizeof(T) > (size_t)optin) return fail(MM_ERR_UNSUPPORTED, "staged stage: shared memory");
	const void *fn = s->st_tm == TM_SLAB   ? (const void *)k_stage_tma<T, COMP, S, TM_SLAB>
	                 : s->st_tm == TM_FILM ? (const void *)k_stage_tma<T, COMP, S, TM_FILM>
	                                       : (const void *)k_stage_tma<T, COMP, S, TM_RUNTIME>;
	if constexpr (S <= 6) {
		if (s->st_pat)
			fn = s->st_tm == TM_SLAB ? (const void *)k_stage_tma<T, COMP, S, TM_SLAB, dp54_pattern(S, COMP)>
			                         : (const void *)k_stage_tma<T, COMP, S, TM_FILM, dp54_pattern(S, COMP)>;
	}
	MM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 2 * 256 * (int)sizeof(T)));
	int per_sm = 0;
	MM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, ST_CONS + 32, smem));
	if (per_sm < 1) return fail(MM_ERR_UNSUPPORTED, "staged stage kernel does not fit on an SM");
	const mm_solver_config &c = s->cfg;
	const long long nsteps = (long long)((c.nx + ST_X - 1) / ST_X) * ((c.ny + ST_Y - 1) / ST_Y) * c.nz;
	long long grid = std::min<long long>((long long)per_sm * num_sms(), nsteps);
	// MMB200_STAGE_GRID caps the grid (more steps per CTA; used by the tests)
	if (const char *cap = std::getenv("MMB200_STAGE_GRID"))
		if (std::atoi(cap) > 0) grid = std::min<long long>(grid, std::atoi(cap));
	s->st_grid[S] = (int)grid;
	s->st_smem[S] = smem;
	return MM_OK;
}

// Tensor maps of the staged stage kernel over the solver's buffers.
template <typename T>
mm_status stage_tma_maps(mm_solver *s)
{
	const mm_solver_config &c = s->cfg;
	const uint64_t e = sizeof(T);
	const uint64_t dims[4] = {(uint64_t)c.nx, (uint64_t)c.ny, (uint64_t)c.nz, 3};
	const uint64_t strides[3] = {c.nx * e, (uint64_t)c.nx * c.ny * e, (uint64_t)s->n * e};
	const uint32_t hbox[4] = {ST_XH, ST_YH, 1, 3}, obox[4] = {ST_X, ST_Y, 1, 3};
	StageMaps &m = s->st_maps;
	const void *yin[3] = {s->m, s->ys[0], s->ys[1]};
	for (int q = 0; q < 3; ++q) MM_TRY(tma_encode_as(&s->st_yin[q], yin[q], 4, dims, strides, hbox, (int)e));
	MM_TRY(tma_encode_as(&m.hd, s->hd, 4, dims, strides, obox, (int)e));
	MM_TRY(tma_encode_as(&m.hi, s->m, 4, dims, strides, obox, (int)e));
	if (s->m_lo) MM_TRY(tma_encode_as(&m.lo, s->m_lo, 4, dims, strides, obox, (int)e));
	for (int q = 0; q < MAXS; ++q) {
		m.kptr[q] = s->k[q];
		if (s->k[q]) MM_TRY(tma_encode_as(&m.k[q], s->k[q], 4, dims, strides, obox, (int)e));
	}
	if (s->reg) {
		const uint64_t rd[3] = {(uint64_t)c.nx, (uint64_t)c.ny, (uint64_t)c.nz};
		const uint64_t rs[2] = {(uint64_t)c.nx, (uint64_t)c.nx * c.ny};
		const uint32_t rb[3] = {ST_XR, ST_YH, 1};
		MM_TRY(tma_encode_as(&m.reg, s->reg, 3, rd, rs, rb, 1));
	}
	return MM_OK;
}

// Grid and shared memory of the staged stage kernel for every stage of the tableau (at solver
// creation, so that no later call queries occupancy during stream capture).
template <typename T, int... S>
mm_status stage_tma_setup(mm_solver *s, std::integer_sequence<int, S...>)
{
	constexpr bool COMP = sizeof(T) == 4;
	const char *env = std::getenv("MMB200_STAGE_TMA");
	// the staged kernel's halo boxes do not wrap around: periodic meshes take the per-thread kernel
	const bool periodic = s->cfg.pbc[0] || s->cfg.pbc[1] || s->cfg.pbc[2];
	s->st_tma = stage_tma_fits(s->cfg.nx, sizeof(T), s->reg != nullptr, s->n) && !(env && env[0] == '0') && !periodic;
	if (!s->st_tma) return MM_OK;
	s->st_tm = s->cfg.terms == TM_SLAB ? TM_SLAB : s->cfg.terms == TM_FILM ? TM_FILM : TM_RUNTIME;
	if (const char *gen = std::getenv("MMB200_STAGE_GENERIC"))  // the run-time term set (comparison tests)
		if (gen[0] == '1') s->st_tm = TM_RUNTIME;
	// the Dormand-Prince stage patterns (the fixed term sets include demag), unless
	// MMB200_STAGE_PATTERN=0; every stage's pattern must equal its coefficients' own
	s->st_pat = (s->st_tm == TM_SLAB || s->st_tm == TM_FILM) && s->cfg.tableau == MM_RK_DP54 && s->tab.s == 7;
	if (const char *pe = std::getenv("MMB200_STAGE_PATTERN"))
		if (pe[0] == '0') s->st_pat = false;
	for (int i = 0; i < s->tab.s && s->st_pat; ++i) {
		// the pattern, and the operand layout the consumers derive from it, must equal the
		// coefficients' own (the producer and the shared-memory size follow the coefficients)
		const StageCoef sc = stage_coef(s->tab, i, COMP);
		const int pat = dp54_pattern(i, COMP);
		int kop[MAXS], hd, hi, lo;
		const int nops = stage_ops(sc, i, COMP, true, kop, hd, hi, lo);
		const bool out = pat_bit(pat, 7) ? pat_bit(pat, 9) : pat_bit(pat, 8);
		bool same = pattern_of(sc, i) == pat && pat_nops(pat, COMP, true) == nops && hd == 0 &&
		            hi == (out ? 1 : -1) && lo == (out && COMP ? 2 : -1);
		for (int l = 0; l < MAXS; ++l) same = same && (l < PAT_KBITS ? pat_kop(pat, COMP, true, l) == kop[l] : kop[l] < 0);
		if (!same) s->st_pat = false;
	}
	mm_status r = stage_tma_maps<T>(s);
	((r = (r == MM_OK && S < s->tab.s) ? stage_tma_prepare<T, COMP, S>(s) : r), ...);
	if (r != MM_OK) {
		// a box the tensor-map encoder or the SM does not take: the per-thread-load stage kernel
		s->st_tma = false;
		cudaGetLastError();
	}
	return MM_OK;
}

template <typename T, bool COMP, int S>
void stage_tma_launch(const mm_solver *s, const CellArgs<T> &a, const StageCoef &sc, const T *yin, const T *yhi,
                      const T *ylo, const KTab<T> *kt, T *yout, DevState *ds, cudaStream_t st)
{
	const mm_solver_config &c = s->cfg;
	StageMaps maps = s->st_maps;
	maps.yin = s->st_yin[yin == (const T *)s->ys[0] ? 1 : (yin == (const T *)s->ys[1] ? 2 : 0)];
	(void)yhi;
	(void)ylo;
	const int tx = (c.nx + ST_X - 1) / ST_X, ty = (c.ny + ST_Y - 1) / ST_Y;
	if constexpr (S <= 6) {
		if (s->st_pat && s->st_tm == TM_SLAB) {
			k_stage_tma<T, COMP, S, TM_SLAB, dp54_pattern(S, COMP)><<<s->st_grid[S], ST_CONS + 32, s->st_smem[S], st>>>(
			    maps, a, sc, kt, yout, (T *)s->ynew_lo, ds, tx, ty);
			return;
		}
		if (s->st_pat && s->st_tm == TM_FILM) {
			k_stage_tma<T, COMP, S, TM_FILM, dp54_pattern(S, COMP)><<<s->st_grid[S], ST_CONS + 32, s->st_smem[S], st>>>(
			    maps, a, sc, kt, yout, (T *)s->ynew_lo, ds, tx, ty);
			return;
		}
	}
	if (s->st_tm == TM_SLAB)
		k_stage_tma<T, COMP, S, TM_SLAB><<<s->st_grid[S], ST_CONS + 32, s->st_smem[S], st>>>(
		    maps, a, sc, kt, yout, (T *)s->ynew_lo, ds, tx, ty);
	else if (s->st_tm == TM_FILM)
		k_stage_tma<T, COMP, S, TM_FILM><<<s->st_grid[S], ST_CONS + 32, s->st_smem[S], st>>>(
		    maps, a, sc, kt, yout, (T *)s->ynew_lo, ds, tx, ty);
	else
		k_stage_tma<T, COMP, S, TM_RUNTIME><<<s->st_grid[S], ST_CONS + 32, s->st_smem[S], st>>>(
		    maps, a, sc, kt, yout, (T *)s->ynew_lo, ds, tx, ty);
}

template <typename T, bool COMP>
mm_status launch_stage(const mm_solver *s, const CellArgs<T> &a, const StageCoef &sc, const T *yin, const T *yhi,
                       const T *ylo, const KTab<T> *kt, T *yout, DevState *ds, cudaStream_t st)
{
	if (s->st_tma) {
		switch (sc.stage) {
		case 0: stage_tma_launch<T, COMP, 0>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
		case 1: stage_tma_launch<T, COMP, 1>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
		case 2: stage_tma_launch<T, COMP, 2>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
		case 3: stage_tma_launch<T, COMP, 3>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
		case 4: stage_tma_launch<T, COMP, 4>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
		case 5: stage_tma_launch<T, COMP, 5>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
		case 6: stage_tma_launch<T, COMP, 6>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
		case 7: stage_tma_launch<T, COMP, 7>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
		default: return fail(MM_ERR_INVALID_ARGUMENT, "stage index beyond the supported tableau size");
		}
		return after_launch("k_stage_tma");
	}
	switch (sc.stage) {
	case 0: stage_launch<T, COMP, 0>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
	case 1: stage_launch<T, COMP, 1>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
	case 2: stage_launch<T, COMP, 2>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
	case 3: stage_launch<T, COMP, 3>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
	case 4: stage_launch<T, COMP, 4>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
	case 5: stage_launch<T, COMP, 5>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
	case 6: stage_launch<T, COMP, 6>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
	case 7: stage_launch<T, COMP, 7>(s, a, sc, yin, yhi, ylo, kt, yout, ds, st); break;
	default: return fail(MM_ERR_INVALID_ARGUMENT, "stage index beyond the supported tableau size");
	}
	return after_launch("k_stage");
}

// y_1 = y_n + h b_10 k_0 when k_0 is the previous attempt's last stage (first same as last).
template <typename T, bool COMP>
__global__ void __launch_bounds__(256) k_prepare1(size_t n3, double b10, const T *__restrict__ yhi,
                                                  const T *__restrict__ ylo,
                                                  const KTab<T> *__restrict__ ktab,
                                                  const DevState *__restrict__ st, T *__restrict__ y1)
{
	const T f = (T)(st->h * b10);
	const T *k0 = ktab->k[0];
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x) {
		if (COMP) y1[i] = yhi[i] + (ylo[i] + f * k0[i]);
		else y1[i] = yhi[i] + f * k0[i];
	}
}

// One Runge-Kutta attempt from the current state with the step size and start time already in
// the device state.  Stage i >= 1 reads y_i from ys[(i-1)&1] and writes y_{i+1} to ys[i&1];
// the last stage writes y_{n+1} to ys[(s-1)&1] or, for first-same-as-last tableaus in FP64,
// leaves it as its own input ys[(s-2)&1].
template <typename T>
mm_status attempt(mm_solver *s, bool eval_k0, cudaStream_t st)
{
	constexpr bool COMP = sizeof(T) == 4;
	const Tableau &tb = s->tab;
	const CellArgs<T> &a = args_of<T>(s);
	DevState *ds = s->dst;
	const T *yhi = (const T *)s->m, *ylo = (const T *)s->m_lo;
	const KTab<T> *kt = (const KTab<T> *)s->ktab;
	T *ys[2] = {(T *)s->ys[0], (T *)s->ys[1]};
	if (eval_k0) {
		const StageCoef sc = stage_coef(tb, 0, COMP);
		MM_TRY(demag<T>(s, s->m, st));
		ProfToken tk = prof_begin(st);
		MM_TRY((launch_stage<T, COMP>(s, a, sc, yhi, yhi, ylo, kt, ys[0], ds, st)));
		prof_end(tk, s->st_tma ? "k_stage_tma" : "k_stage", stage_bytes<T>(s, sc), st);
	} else {
		const size_t n3 = 3 * s->n;
		ProfToken tk = prof_begin(st);
		k_prepare1<T, COMP><<<grid1(n3), 256, 0, st>>>(n3, tb.b[1][0], yhi, ylo, kt, ds, ys[0]);
		MM_TRY(after_launch("k_prepare1"));
		prof_end(tk, "k_prepare1", (double)n3 * sizeof(T) * (COMP ? 4 : 3), st);
	}
	for (int i = 1; i < tb.s; ++i) {
		const StageCoef sc = stage_coef(tb, i, COMP);
		const T *yin = ys[(i - 1) & 1];
		MM_TRY(demag<T>(s, yin, st));
		ProfToken tk = prof_begin(st);
		MM_TRY((launch_stage<T, COMP>(s, a, sc, yin, yhi, ylo, kt, ys[i & 1], ds, st)));
		prof_end(tk, s->st_tma ? "k_stage_tma" : "k_stage", stage_bytes<T>(s, sc), st);
		if (sc.last) s->last_stage_buf = sc.write_new ? (i & 1) : ((i - 1) & 1);
	}
	return MM_OK;
}

template <typename T>
mm_status controller(mm_solver *s, cudaStream_t st)
{
	k_controller<T><<<1, 1, 0, st>>>(s->dst, (KTab<T> *)s->ktab, s->cfg.eps_abs, s->cfg.eps_rel, s->tab.order,
	                                 s->tab.fsal, s->tab.s, s->hst, conv_timeout_flag(s));
	MM_TRY(after_launch("k_controller"));
	MM_CUDA(cudaStreamSynchronize(st));
	return MM_OK;
}

template <typename T>
mm_status accept_state(mm_solver *s, cudaStream_t st)
{
	constexpr bool COMP = sizeof(T) == 4;
	ProfToken tk = prof_begin(st);
	k_accept<T, COMP><<<grid1(s->n), 256, 0, st>>>(s->n, (const T *)s->ys[s->last_stage_buf],
	                                                (const T *)s->ynew_lo, (T *)s->m, (T *)s->m_lo);
	MM_TRY(after_launch("k_accept"));
	prof_end(tk, "k_accept", 3.0 * s->n * sizeof(T) * (COMP ? 4 : 2), st);
	return MM_OK;
}

mm_status put_time(mm_solver *s, double t, double h, cudaStream_t st)
{
	// the two leading fields of the device state; pinned staging keeps the copy stream-ordered
	s->hst->t = t;
	s->hst->h = h;
	MM_CUDA(cudaMemcpyAsync(s->dst, s->hst, 2 * sizeof(double), cudaMemcpyHostToDevice, st));
	return MM_OK;
}

// One attempt + controller as a CUDA graph: the H2D copy of (t, h) from the pinned host state,
// the demag passes and fused stages, and the controller, replayed with a single launch.  Kernel
// parameters never change between attempts (step size and time are read from device memory, the
// first-same-as-last exchange is a device-side pointer swap), so one graph per variant serves the
// whole run.
template <typename T>
mm_status attempt_graph(mm_solver *s, bool eval_k0, cudaStream_t st)
{
	const int v = eval_k0 ? 1 : 0;
	if (!s->gs) {
		MM_CUDA(cudaStreamCreateWithFlags(&s->gs, cudaStreamNonBlocking));
		MM_CUDA(cudaEventCreateWithFlags(&s->ev_in, cudaEventDisableTiming));
		MM_CUDA(cudaEventCreateWithFlags(&s->ev_out, cudaEventDisableTiming));
	}
	cudaStream_t user = st;
	st = s->gs;
	MM_CUDA(cudaEventRecord(s->ev_in, user));
	MM_CUDA(cudaStreamWaitEvent(st, s->ev_in, 0));
	if (!s->gexec[v]) {
		const uint64_t before = launch_counter().load();
		MM_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
		mm_status r = cuda_status(cudaMemcpyAsync(s->dst, s->hst, 2 * sizeof(double), cudaMemcpyHostToDevice, st),
		                          "cudaMemcpyAsync");
		if (r == MM_OK) r = attempt<T>(s, eval_k0, st);
		if (r == MM_OK) {
			k_controller<T><<<1, 1, 0, st>>>(s->dst, (KTab<T> *)s->ktab, s->cfg.eps_abs, s->cfg.eps_rel,
			                                 s->tab.order, s->tab.fsal, s->tab.s, s->hst, conv_timeout_flag(s));
			r = after_launch("k_controller");
		}
		cudaGraph_t g = nullptr;
		const cudaError_t e = cudaStreamEndCapture(st, &g);
		if (r != MM_OK) {
			if (g) cudaGraphDestroy(g);
			return r;
		}
		MM_CUDA(e);
		const cudaError_t ei = cudaGraphInstantiate(&s->gexec[v], g, 0);
		cudaGraphDestroy(g);
		MM_CUDA(ei);
		s->gkernels[v] = launch_counter().load() - before;
		launch_counter().fetch_sub(s->gkernels[v]);  // counted when the graph runs
		s->glast[v] = s->last_stage_buf;
	}
	MM_CUDA(cudaGraphLaunch(s->gexec[v], st));
	launch_counter().fetch_add(s->gkernels[v]);
	s->last_stage_buf = s->glast[v];
	MM_CUDA(cudaEventRecord(s->ev_out, st));
	MM_CUDA(cudaStreamWaitEvent(user, s->ev_out, 0));
	return MM_OK;
}

// One attempt + controller; returns the decision in s->hst.
template <typename T>
mm_status attempt_and_control(mm_solver *s, double h, cudaStream_t st)
{
	const bool eval_k0 = !(s->tab.fsal && s->k0_valid);
	if (profiling_on()) {
		// per-kernel event timing needs direct launches
		MM_TRY(put_time(s, s->t, h, st));
		MM_TRY(attempt<T>(s, eval_k0, st));
		MM_TRY(controller<T>(s, st));
	} else {
		s->hst->t = s->t;
		s->hst->h = h;
		MM_TRY(attempt_graph<T>(s, eval_k0, st));
		MM_CUDA(cudaStreamSynchronize(st));
	}
	s->attempts++;
	if (s->tab.fsal) s->k0_valid = true;
	return MM_OK;
}

// RungeKutta.evolve(state, t_max) (runge_kutta.py:47-87) + finish_step.
template <typename T>
mm_status evolve(mm_solver *s, double t_max, cudaStream_t st)
{
	double h_try = s->have_next ? s->h_next : s->h;
	double h_new = h_try;
	for (;;) {
		MM_TRY(attempt_and_control<T>(s, h_try, st));
		const DevState &d = *s->hst;
		if (d.not_finite == 2)
			return fail(MM_ERR_TIMEOUT, "solver: a TMA-staged FFT pass gave up waiting for its loads");
		if (d.not_finite) {
			s->not_finite = 1;
			return fail(MM_ERR_NOT_FINITE, "solver: non-finite value in the state or its derivative");
		}
		h_new = d.h_new;
		if (!d.accept) {
			s->rejected++;
			if (!s->cfg.fsal_reuse_after_reject) s->k0_valid = false;
			h_try = h_new;
			continue;
		}
		break;
	}
	if (s->t + h_try > t_max) {
		// runge_kutta.py:75-78: redo the step with the clamped size, accepted without a check
		h_try = t_max - s->t;
		// the controller's decision is ignored; it keeps the reductions reset and the
		// first-same-as-last swap in step
		MM_TRY(attempt_and_control<T>(s, h_try, st));
	}
	MM_TRY(accept_state<T>(s, st));
	s->t += h_try;
	s->h = h_try;
	s->h_next = h_new;
	s->have_next = true;
	s->steps++;
	return MM_OK;
}

template <typename T>
mm_status average(mm_solver *s, double *out3, cudaStream_t st)
{
	constexpr bool COMP = sizeof(T) == 4;
	MM_CUDA(cudaMemsetAsync(s->avg, 0, 3 * sizeof(double), st));
	k_average_M<T, COMP><<<grid1(s->n), 256, 0, st>>>(s->n, (const T *)s->m, (const T *)s->m_lo, s->reg,
	                                                   (const DevMat<T> *)s->mat, s->avg);
	MM_TRY(after_launch("k_average_M"));
	MM_CUDA(cudaMemcpyAsync(s->avg_h, s->avg, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
	MM_CUDA(cudaStreamSynchronize(st));
	for (int c = 0; c < 3; ++c) out3[c] = s->avg_h[c] / (double)s->n;
	return MM_OK;
}

// Relaxation norms (square roots of k_relax_norms' maxima) of the current state; synchronises.
template <typename T>
mm_status relax_norms(mm_solver *s, double out3[3], cudaStream_t st)
{
	MM_TRY(demag<T>(s, s->m, st));
	MM_CUDA(cudaMemsetAsync(s->avg, 0, 3 * sizeof(double), st));
	k_relax_norms<T><<<cell_grid(s->cfg), dim3(32, 8, 1), 0, st>>>(args_of<T>(s), (const T *)s->m,
	                                                               (const T *)s->hd, s->t, s->avg);
	MM_TRY(after_launch("k_relax_norms"));
	MM_CUDA(cudaMemcpyAsync(s->avg_h, s->avg, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
	MM_CUDA(cudaStreamSynchronize(st));
	for (int c = 0; c < 3; ++c) out3[c] = sqrt(s->avg_h[c]);
	return MM_OK;
}

// Energies of the current state [J]: E_stray, E_exch, E_aniso, E_ext and their sum E_tot (the
// terms the solver was created with; an absent term contributes 0).  Synchronises.
template <typename T>
mm_status energies(mm_solver *s, double out5[5], cudaStream_t st)
{
	if (s->cfg.terms & MM_TERM_DEMAG) MM_TRY(demag<T>(s, s->m, st));
	MM_CUDA(cudaMemsetAsync(s->avg, 0, 5 * sizeof(double), st));
	k_energies<T><<<cell_grid(s->cfg), dim3(32, 8, 1), 0, st>>>(args_of<T>(s), (const T *)s->m, (const T *)s->hd,
	                                                            s->t, s->avg);
	MM_TRY(after_launch("k_energies"));
	MM_CUDA(cudaMemcpyAsync(s->avg_h, s->avg, 5 * sizeof(double), cudaMemcpyDeviceToHost, st));
	MM_CUDA(cudaStreamSynchronize(st));
	const double V = s->cfg.dx * s->cfg.dy * s->cfg.dz;
	out5[0] = -MU0 / 2.0 * V * s->avg_h[0];
	out5[1] = -MU0 / 2.0 * V * s->avg_h[1];
	out5[2] = V * (s->avg_h[2] + s->avg_h[3]);
	out5[3] = -MU0 * V * s->avg_h[4];
	out5[4] = out5[0] + out5[1] + out5[2] + out5[3];
	return MM_OK;
}

void free_solver(mm_solver *s)
{
	if (!s) return;
	for (int v = 0; v < 2; ++v)
		if (s->gexec[v]) cudaGraphExecDestroy(s->gexec[v]);
	if (s->gs) cudaStreamDestroy(s->gs);
	if (s->ev_in) cudaEventDestroy(s->ev_in);
	if (s->ev_out) cudaEventDestroy(s->ev_out);
	delete s->conv;
	cudaFree(s->mat);
	cudaFree(s->ms_tab);
	cudaFree(s->reg);
	cudaFree(s->m);
	cudaFree(s->m_lo);
	cudaFree(s->ys[0]);
	cudaFree(s->ys[1]);
	cudaFree(s->ynew_lo);
	for (int q = 0; q < MAXS; ++q) cudaFree(s->k[q]);
	cudaFree(s->hd);
	cudaFree(s->ktab);
	cudaFree(s->dst);
	cudaFreeHost(s->hst);
	cudaFree(s->avg);
	cudaFreeHost(s->avg_h);
	delete s;
}

template <typename T>
mm_status create_impl(mm_solver *s, int nmat, const mm_material *mats, const uint8_t *regions,
                      const double *tensor, cudaStream_t st)
{
	s->nmat = nmat;
	MM_TRY(build_materials<T>(s, nmat, mats));
	if (regions) {
		for (size_t i = 0; i < s->n; ++i)
			if (regions[i] >= nmat) return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_create: region index out of range");
		MM_CUDA(cudaMalloc(&s->reg, s->n));
		MM_CUDA(cudaMemcpy(s->reg, regions, s->n, cudaMemcpyHostToDevice));
	}
	MM_TRY(alloc_state<T>(s));
	fill_args<double>(s, s->args64);
	fill_args<float>(s, s->args32);
	if (s->cfg.terms & MM_TERM_DEMAG) {
		const mm_solver_config &c = s->cfg;
		double *N = nullptr;
		const size_t tb = sizeof(double) * 6 * (size_t)s->px * s->py * s->pz;
		if (!tensor) {
			MM_CUDA(cudaMalloc(&N, tb));
			const int naxes = (c.pbc[0] != 0) + (c.pbc[1] != 0) + (c.pbc[2] != 0);
			const int repeat = c.pbc_repeat > 0 ? c.pbc_repeat : (naxes == 1 ? 15 : naxes == 2 ? 3 : 2);
			const mm_status r = mm_demag_tensor_periodic(c.nx, c.ny, c.nz, c.dx, c.dy, c.dz, c.pbc[0] != 0,
			                                             c.pbc[1] != 0, c.pbc[2] != 0, repeat, s->px, s->py,
			                                             s->pz, N, st);
			if (r != MM_OK) { cudaFree(N); return r; }
		}
		const mm_status r = conv_plan_create(&s->conv, c.precision, c.nx, c.ny, c.nz, s->px, s->py, s->pz,
		                                     tensor ? tensor : N, st);
		if (N) cudaFree(N);
		MM_TRY(r);
	}
	MM_TRY((stage_resident<T, sizeof(T) == 4>(&s->st_resident)));
	MM_TRY(stage_tma_setup<T>(s, std::make_integer_sequence<int, MAXS>()));
	MM_CUDA(cudaStreamSynchronize(st));
	return MM_OK;
}

} // namespace
} // namespace mm

namespace mm {
namespace {
mm_status solver_create(mm_solver **out, const mm_solver_config *config, int num_materials,
                        const mm_material *materials_host, const uint8_t *regions_host,
                        const double *tensor_device, void *stream, int min_pz);
} // namespace
} // namespace mm

extern "C" {

MM_API mm_status mm_solver_create(mm_solver **out, const mm_solver_config *config, int num_materials,
                                  const mm_material *materials_host, const uint8_t *regions_host,
                                  const double *tensor_device, void *stream)
{
	return solver_create(out, config, num_materials, materials_host, regions_host, tensor_device, stream, 1);
}

} // extern "C"

namespace mm {
namespace {

// mm_solver_create with a lower bound on the padded z length (the batch pads a single layer to
// 2 so that every instance takes the 3-D power-of-two passes).
mm_status solver_create(mm_solver **out, const mm_solver_config *config, int num_materials,
                        const mm_material *materials_host, const uint8_t *regions_host,
                        const double *tensor_device, void *stream, int min_pz)
{
	if (!out || !config || !materials_host || num_materials <= 0 || num_materials > 256)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_create: invalid argument");
	const mm_solver_config &c = *config;
	if (c.nx <= 0 || c.ny <= 0 || c.nz <= 0 || !(c.dx > 0) || !(c.dy > 0) || !(c.dz > 0))
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_create: invalid mesh");
	if (c.precision != MM_F64 && c.precision != MM_F32)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_create: invalid precision");
	if (c.tableau < MM_RK_RKF45 || c.tableau > MM_RK_RK23)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_create: invalid tableau");
	if (!(c.eps_abs > 0) || !(c.eps_rel > 0) || !(c.h0 > 0))
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_create: tolerances and h0 must be positive");
	if ((size_t)c.nx * c.ny * c.nz > (size_t)1 << 31)
		return fail(MM_ERR_UNSUPPORTED, "mm_solver_create: more than 2^31 cells");
	mm_solver *s = new mm_solver();
	s->cfg = c;
	s->n = (size_t)c.nx * c.ny * c.nz;
	s->tab = make_tableau(c.tableau);
	s->px = mm_round_tensor_dimension(c.nx, c.pbc[0] != 0, c.padding);
	s->py = mm_round_tensor_dimension(c.ny, c.pbc[1] != 0, c.padding);
	s->pz = mm_round_tensor_dimension(c.nz, c.pbc[2] != 0, c.padding);
	if (s->pz > 0 && s->pz < min_pz) s->pz = min_pz;
	if (s->px <= 0 || s->py <= 0 || s->pz <= 0) {
		delete s;
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_create: invalid padding");
	}
	s->h = c.h0;
	cudaStream_t st = as_stream(stream);
	const mm_status r = c.precision == MM_F64
	                        ? create_impl<double>(s, num_materials, materials_host, regions_host, tensor_device, st)
	                        : create_impl<float>(s, num_materials, materials_host, regions_host, tensor_device, st);
	if (r != MM_OK) {
		free_solver(s);
		return r;
	}
	*out = s;
	return MM_OK;
}

} // namespace
} // namespace mm

extern "C" {

MM_API mm_status mm_solver_destroy(mm_solver *s)
{
	free_solver(s);
	return MM_OK;
}

MM_API mm_status mm_solver_set_M(mm_solver *s, const double *M, void *stream)
{
	if (!s || !M) return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_set_M: null argument");
	cudaStream_t st = as_stream(stream);
	if (s->cfg.precision == MM_F64)
		k_set_M<double, false><<<grid1(s->n), 256, 0, st>>>(s->n, M, s->reg, (const DevMat<double> *)s->mat,
		                                                     (double *)s->m, nullptr);
	else
		k_set_M<float, true><<<grid1(s->n), 256, 0, st>>>(s->n, M, s->reg, (const DevMat<float> *)s->mat,
		                                                   (float *)s->m, (float *)s->m_lo);
	MM_TRY(after_launch("k_set_M"));
	s->t = 0;
	s->h = s->cfg.h0;
	s->have_next = false;
	s->k0_valid = false;
	s->steps = s->attempts = s->rejected = 0;
	s->not_finite = 0;
	return MM_OK;
}

MM_API mm_status mm_solver_load_M(mm_solver *s, const double *M, void *stream)
{
	if (!s || !M) return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_load_M: null argument");
	cudaStream_t st = as_stream(stream);
	if (s->cfg.precision == MM_F64)
		k_set_M<double, false><<<grid1(s->n), 256, 0, st>>>(s->n, M, s->reg, (const DevMat<double> *)s->mat,
		                                                     (double *)s->m, nullptr);
	else
		k_set_M<float, true><<<grid1(s->n), 256, 0, st>>>(s->n, M, s->reg, (const DevMat<float> *)s->mat,
		                                                   (float *)s->m, (float *)s->m_lo);
	return after_launch("k_set_M");
}

MM_API mm_status mm_solver_get_M(mm_solver *s, double *M, void *stream)
{
	if (!s || !M) return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_get_M: null argument");
	cudaStream_t st = as_stream(stream);
	if (s->cfg.precision == MM_F64)
		k_get_M<double, false><<<grid1(s->n), 256, 0, st>>>(s->n, (const double *)s->m, nullptr, s->reg,
		                                                     (const DevMat<double> *)s->mat, M);
	else
		k_get_M<float, true><<<grid1(s->n), 256, 0, st>>>(s->n, (const float *)s->m, (const float *)s->m_lo,
		                                                   s->reg, (const DevMat<float> *)s->mat, M);
	return after_launch("k_get_M");
}

MM_API mm_status mm_solver_set_time(mm_solver *s, double t, double h_next, void *stream)
{
	(void)stream;
	if (!s || !(h_next > 0)) return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_set_time: invalid argument");
	s->t = t;
	s->h_next = h_next;
	s->have_next = true;
	return MM_OK;
}

MM_API mm_status mm_solver_step(mm_solver *s, double t_max, void *stream)
{
	if (!s) return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_step: null solver");
	cudaStream_t st = as_stream(stream);
	MM_TRY(s->cfg.precision == MM_F64 ? evolve<double>(s, t_max, st) : evolve<float>(s, t_max, st));
	MM_CUDA(cudaStreamSynchronize(st));
	return MM_OK;
}

MM_API mm_status mm_solver_run(mm_solver *s, double t_end, double sample_dt, double *sample_t_host,
                               double *samples_host, int max_samples, int *num_samples, void *stream)
{
	if (!s) return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_run: null solver");
	cudaStream_t st = as_stream(stream);
	const bool sampling = sample_dt > 0 && samples_host && sample_t_host;
	int count = 0;
	auto handle = [&]() -> mm_status {
		// condition.EveryNthSecond.check (condition.py:121-133)
		if (!sampling) return MM_OK;
		const double r = fmod(s->t, sample_dt);
		if ((fabs(r) < 1e-16 || fabs(r - sample_dt) < 1e-16) && count < max_samples) {
			sample_t_host[count] = s->t;
			MM_TRY(s->cfg.precision == MM_F64 ? average<double>(s, samples_host + 3 * count, st)
			                                  : average<float>(s, samples_host + 3 * count, st));
			++count;
		}
		return MM_OK;
	};
	MM_TRY(handle());
	while (!(s->t >= t_end)) {
		// Solver.step_with_t_max (solver.py:76-85): the next time of interest of the handlers
		double t1 = 1e100;
		if (sampling) {
			const double toi = ((double)(long long)(s->t / sample_dt) + 1) * sample_dt;
			if (toi > s->t && toi < t1) t1 = toi;
		}
		MM_TRY(s->cfg.precision == MM_F64 ? evolve<double>(s, t1, st) : evolve<float>(s, t1, st));
		MM_TRY(handle());
	}
	if (num_samples) *num_samples = count;
	MM_CUDA(cudaStreamSynchronize(st));
	return MM_OK;
}

MM_API mm_status mm_solver_attempt(mm_solver *s, double h, void *stream)
{
	if (!s || !(h > 0)) return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_attempt: invalid argument");
	cudaStream_t st = as_stream(stream);
	MM_TRY(put_time(s, s->t, h, st));
	const bool eval_k0 = !(s->tab.fsal && s->k0_valid);
	if (s->cfg.precision == MM_F64) {
		MM_TRY(attempt<double>(s, eval_k0, st));
		k_controller<double><<<1, 1, 0, st>>>(s->dst, (KTab<double> *)s->ktab, s->cfg.eps_abs, s->cfg.eps_rel,
		                                      s->tab.order, s->tab.fsal, s->tab.s, s->hst, conv_timeout_flag(s));
	} else {
		MM_TRY(attempt<float>(s, eval_k0, st));
		k_controller<float><<<1, 1, 0, st>>>(s->dst, (KTab<float> *)s->ktab, s->cfg.eps_abs, s->cfg.eps_rel,
		                                     s->tab.order, s->tab.fsal, s->tab.s, s->hst, conv_timeout_flag(s));
	}
	MM_TRY(after_launch("k_controller"));
	if (s->tab.fsal) s->k0_valid = true;
	s->attempts++;
	return MM_OK;
}

MM_API mm_status mm_solver_eval(mm_solver *s, double *H_eff, double *dMdt, double *H_demag, void *stream)
{
	if (!s) return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_eval: null solver");
	cudaStream_t st = as_stream(stream);
	const dim3 grid = cell_grid(s->cfg), block(32, 8, 1);
	if (s->cfg.precision == MM_F64) {
		MM_TRY(demag<double>(s, s->m, st));
		k_eval<double><<<grid, block, 0, st>>>(s->args64, (const double *)s->m, (const double *)s->hd, s->t, H_eff,
		                                       dMdt, H_demag);
	} else {
		MM_TRY(demag<float>(s, s->m, st));
		k_eval<float><<<grid, block, 0, st>>>(s->args32, (const float *)s->m, (const float *)s->hd, s->t, H_eff,
		                                      dMdt, H_demag);
	}
	return after_launch("k_eval");
}

MM_API mm_status mm_solver_energies(mm_solver *s, double *energies_host5, void *stream)
{
	if (!s || !energies_host5) return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_energies: null argument");
	cudaStream_t st = as_stream(stream);
	return s->cfg.precision == MM_F64 ? energies<double>(s, energies_host5, st) : energies<float>(s, energies_host5, st);
}

MM_API mm_status mm_solver_relax_norms(mm_solver *s, double *norms_host3, void *stream)
{
	if (!s || !norms_host3) return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_relax_norms: null argument");
	cudaStream_t st = as_stream(stream);
	return s->cfg.precision == MM_F64 ? relax_norms<double>(s, norms_host3, st) : relax_norms<float>(s, norms_host3, st);
}

MM_API mm_status mm_solver_relax(mm_solver *s, int criterion, double threshold, int check_every_nth_step,
                                 long long max_steps, int *relaxed, double *last_value, void *stream)
{
	if (!s || !relaxed || check_every_nth_step < 1 || !(threshold > 0) ||
	    (criterion != MM_RELAX_DEG_PER_NS && criterion != MM_RELAX_TORQUE))
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_relax: invalid argument");
	cudaStream_t st = as_stream(stream);
	const bool f64 = s->cfg.precision == MM_F64;
	*relaxed = 0;
	bool have_last = false;
	double last = 0.0;
	for (long long taken = 0;; ++taken) {
		// condition.Relaxed.check (condition.py:178-199): only every nth step
		if (s->steps % check_every_nth_step == 0) {
			double nrm[3];
			MM_TRY(f64 ? relax_norms<double>(s, nrm, st) : relax_norms<float>(s, nrm, st));
			if (criterion == MM_RELAX_DEG_PER_NS) {
				// LandauLifshitzGilbert.calculate_deg_per_ns (landau_lifshitz_gilbert.py:127-131)
				const double deg_per_step = (180.0 / M_PI) * atan2(nrm[0] * s->h, nrm[1]);
				const double deg_per_ns = 1e-9 * deg_per_step / s->h;
				const bool done = have_last && deg_per_ns < last && deg_per_ns <= threshold;
				last = deg_per_ns;
				have_last = true;
				if (done) { *relaxed = 1; break; }
			} else {
				last = nrm[2];
				if (nrm[2] < threshold) { *relaxed = 1; break; }
			}
		}
		if (max_steps >= 0 && taken >= max_steps) break;
		MM_TRY(f64 ? evolve<double>(s, 1e100, st) : evolve<float>(s, 1e100, st));
	}
	if (last_value) *last_value = last;
	MM_CUDA(cudaStreamSynchronize(st));
	return MM_OK;
}

MM_API mm_status mm_solver_stats_get(mm_solver *s, mm_solver_stats *out, void *stream)
{
	(void)stream;
	if (!s || !out) return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_stats_get: null argument");
	out->t = s->t;
	out->h = s->h;
	out->h_next = s->have_next ? s->h_next : s->h;
	out->steps = s->steps;
	out->attempts = s->attempts;
	out->rejected = s->rejected;
	out->last_error = sqrt(s->hst->max_err2);
	out->last_max_dmdt = sqrt(s->hst->max_k02);
	out->not_finite = s->not_finite;
	out->stage_kernel = !s->st_tma ? 0 : s->st_tm == TM_RUNTIME ? 1 : s->st_pat ? 3 : 2;
	return MM_OK;
}

MM_API mm_status mm_solver_average_M(mm_solver *s, double *avg3, void *stream)
{
	if (!s || !avg3) return fail(MM_ERR_INVALID_ARGUMENT, "mm_solver_average_M: null argument");
	cudaStream_t st = as_stream(stream);
	return s->cfg.precision == MM_F64 ? average<double>(s, avg3, st) : average<float>(s, avg3, st);
}

} // extern "C"

// ================================================================================================
// Batched solves: many independent instances of uneven size advance in lock step, one
// Runge-Kutta attempt per round for every running instance.  Each instance is a full solver (own
// state, stages, tensor and spectra); a round runs as grouped launches (one per pass and transform
// length for the convolution, one per stage for the fused stage kernel) over work lists of
// (instance, tile), and the step controller, the accept step and the stop test run on the device
// per instance, so a captured round needs no host decision.  Instances join and leave between
// rounds (slots); the work lists and the captured rounds are rebuilt when the membership changes.
// ================================================================================================
namespace mm {
namespace {

// Device bookkeeping of one instance.
struct BState {
	int steps, attempts, rejected, status;  // status: 0 running, 1 finished, 2 non-finite state
	double t, h;
};
struct BSlot {
	BState bs;
	int active;  // takes part in rounds
	int need_k0; // the next round evaluates k_0 at the state (after set-up or a new state)
	int rebase;  // FP32: the next round first moves the deviation into the base state and
	             // recomputes the base field (after set-up, then every BATCH_REBASE attempts)
};

template <typename T>
struct BDesc {
	CellArgs<T> a;
	T *m, *m_lo, *ys[2], *hd, *ynew_lo;
	T *hb;  // FP32 deviation form: the base field H_demag(m) + H_exch(m) (the ynew_lo buffer)
	KTab<T> *kt;
	DevState *ds;
	BSlot *slot;
	double t_end;  // > 0: stop at this time (clamping the last step); 0: stop on the torque test
	int n, tiles_x, tiles_y, ntiles;
};

constexpr int BATCH_TILES = 4;     // stage tiles per block of the grouped stage kernel (1 for small batches)
constexpr int BATCH_CHUNK = 4096;  // elements per block of the grouped element-wise kernels
// FP32 batches (deviation form, cell_rhs_delta): attempts between rebases of an instance.  The
// stage inputs' rounding grows with the deviation accumulated since the last rebase.
constexpr int BATCH_REBASE = 32;
static_assert(BATCH_REBASE <= 32, "the due rounds are kept as a 32-bit mask of residues");

// Grouped fused stage: block = (instance, first tile); in = 0: the state m, 1/2: ys[0]/ys[1].
// K0: the k_0 evaluation of instances that need it (others skip it).
template <typename T, bool COMP, int S, bool TORQUE, int PAT>
__global__ void __launch_bounds__(256, TORQUE ? 2 : stage_min_blocks<T>())
    k_stage_grp(const BDesc<T> *__restrict__ d, StageCoef sc, int in, int out, const int2 *__restrict__ items, int tpi)
{
	const int2 it = items[blockIdx.x];
	const BDesc<T> &g = d[it.x];
	if (!g.slot->active || (S == 0 && !g.slot->need_k0)) return;
	__shared__ CellArgs<T> a;
	__shared__ T msr[256];
	extern __shared__ __align__(16) unsigned char stage_pre[];
	if (threadIdx.x == 0 && threadIdx.y == 0) a = g.a;
	__syncthreads();
	load_ms_table(a, msr);
	// (FP32: the deviation form, whose k_0 input is the deviation D_n itself)
	const T *y_in = in == 0 ? (COMP ? g.m_lo : g.m) : g.ys[in - 1];
	T *const *K = g.kt->k;  // read per use (cached), not held in registers
	T e2 = T(0), k02 = T(0), tq2 = T(0);
	for (int k = 0; k < tpi && it.y + k < g.ntiles; ++k)
		stage_tile<T, COMP, S, TORQUE, COMP, PAT>(a, msr, sc, y_in, g.hd, g.m, g.m_lo, K, g.ys[out], g.ynew_lo, g.ds,
		                                     it.y + k, g.tiles_x, g.tiles_y, e2, k02, tq2,
		                                     reinterpret_cast<T *>(stage_pre), g.hb);
	if (pat_bit(PAT, 7)) block_max_to(&g.ds->max_err2, e2);
	if (pat_bit(PAT, 10)) block_max_to(&g.ds->max_k02, k02);
	if (TORQUE) block_max_to(&g.ds->max_tq2, tq2);
}

// Grouped first-same-as-last first stage, y_1 = y_n + h b_10 k_0, into ys[0] (instances whose
// k_0 is the previous attempt's last stage).
template <typename T, bool COMP>
__global__ void __launch_bounds__(256) k_prepare1_grp(const BDesc<T> *__restrict__ d, double b10,
                                                      const int2 *__restrict__ items)
{
	const int2 it = items[blockIdx.x];
	const BDesc<T> &g = d[it.x];
	if (!g.slot->active || g.slot->need_k0) return;
	const size_t n3 = 3 * (size_t)g.n;
	const T f = (T)(g.ds->h * b10);
	const T *k0 = g.kt->k[0];
	const size_t end = min(n3, (size_t)(it.y + 1) * BATCH_CHUNK);
	for (size_t i = (size_t)it.y * BATCH_CHUNK + threadIdx.x; i < end; i += blockDim.x) {
		if (COMP) g.ys[0][i] = g.m_lo[i] + f * k0[i];  // deviation of y_1
		else g.ys[0][i] = g.m[i] + f * k0[i];
	}
}

// FP32 rebase (instances flagged for it): the base state takes the deviation, hi + D = s + e
// with s = fl(hi + D) and the rounding error e exact (two-sum), so the state is unchanged.
__global__ void __launch_bounds__(256) k_rebase_grp(const BDesc<float> *__restrict__ d, const int2 *__restrict__ items)
{
	const int2 it = items[blockIdx.x];
	const BDesc<float> &g = d[it.x];
	if (!g.slot->active || !g.slot->rebase) return;
	const size_t n3 = 3 * (size_t)g.n;
	const size_t end = min(n3, (size_t)(it.y + 1) * BATCH_CHUNK);
	for (size_t i = (size_t)it.y * BATCH_CHUNK + threadIdx.x; i < end; i += blockDim.x) {
		const float a = g.m[i], b = g.m_lo[i];
		const float s = a + b;
		const float bb = s - a;
		g.m[i] = s;
		g.m_lo[i] = (a - (s - bb)) + (b - bb);
	}
}

// FP32 base field after a rebase: hb holds H_demag(hi) (the grouped convolution's second output);
// the material cells add H_exch(hi), with the stencil of cell_core (exchange_cpu.cpp:60-139).
__global__ void __launch_bounds__(256) k_base_grp(const BDesc<float> *__restrict__ d, const int2 *__restrict__ items)
{
	const int2 it = items[blockIdx.x];
	const BDesc<float> &g = d[it.x];
	if (!g.slot->active || !g.slot->rebase || !(g.a.terms & MM_TERM_EXCHANGE)) return;
	const CellArgs<float> &a = g.a;
	const size_t n = (size_t)g.n;
	const size_t end = min(n, (size_t)(it.y + 1) * BATCH_CHUNK);
	for (size_t i = (size_t)it.y * BATCH_CHUNK + threadIdx.x; i < end; i += blockDim.x) {
		const DevMat<float> &M = mat_of(a, i);
		if (M.Ms == 0.f) continue;
		const int x = (int)(i % a.nx), yy = (int)(i / a.nx % a.ny), z = (int)(i / ((size_t)a.nx * a.ny));
		bool has[6];
		size_t off[6];
		neighbours(a, x, yy, z, i, has, off);
		const float w[6] = {a.wx, a.wx, a.wy, a.wy, a.wz, a.wz};
		const V3<float> m = load3(g.m, i, n);
		V3<float> sum = v3<float>(0, 0, 0);
#pragma unroll
		for (int q = 0; q < 6; ++q)
			if (has[q] && mat_of(a, off[q]).Ms != 0.f) sum = sum + w[q] * (load3(g.m, off[q], n) - m);
		store3(g.hb, i, n, load3(g.hb, i, n) + M.cex * sum);
	}
}

// Grouped accept: m <- y_{n+1}/|y_{n+1}| for the instances whose attempt the controller accepted.
template <typename T, bool COMP>
__global__ void __launch_bounds__(256) k_accept_grp(const BDesc<T> *__restrict__ d, int last_buf,
                                                    const int2 *__restrict__ items)
{
	const int2 it = items[blockIdx.x];
	const BDesc<T> &g = d[it.x];
	if (!g.ds->accept) return;
	const size_t n = (size_t)g.n;
	const T *ynew = g.ys[last_buf];
	const size_t end = min(n, (size_t)(it.y + 1) * BATCH_CHUNK);
	for (size_t i = (size_t)it.y * BATCH_CHUNK + threadIdx.x; i < end; i += blockDim.x) {
		if (COMP) {
			// deviation form: y_{n+1} = hi + D (in double), normalised; hi stays, D takes the rest
			double v[3], l2 = 0.0;
			for (int c = 0; c < 3; ++c) {
				v[c] = (double)g.m[i + c * n] + (double)ynew[i + c * n];
				l2 += v[c] * v[c];
			}
			const double sc = l2 > 0 ? 1.0 / sqrt(l2) : 0.0;
			for (int c = 0; c < 3; ++c) g.m_lo[i + c * n] = (T)(v[c] * sc - (double)g.m[i + c * n]);
		} else {
			accept_cell<T, COMP>(n, ynew, g.ynew_lo, g.m, g.m_lo, i);
		}
	}
}

// Grouped step controller (one thread per instance): the single-instance controller's decision,
// then time and step-size update, counters, and the stop test on the accepted state: t >= t_end
// for a timed solve (the step before t_end is clamped onto it), else max |m x H_eff| / Ms below
// the threshold at a multiple of check_every accepted steps (its torque was reduced by the last
// stage, whose input is y_{n+1} for a first-same-as-last tableau).  A finished instance leaves
// the rounds; the accept kernel still applies its last step.
template <typename T>
__global__ void k_controller_grp(const BDesc<T> *__restrict__ d, int count, double eps_abs, double eps_rel,
                                 int order, int fsal, int s, double tq_thr2, int check_every)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= count) return;
	DevState *st = d[i].ds;
	BSlot *sl = d[i].slot;
	if (!sl->active) {
		st->accept = 0;
		return;
	}
	const double h = st->h;
	const double tq2 = st->max_tq2;
	st->max_tq2 = 0.0;
	control_attempt<T>(st, d[i].kt, eps_abs, eps_rel, order, fsal, s, nullptr, nullptr);
	BState &b = sl->bs;
	b.attempts++;
	sl->need_k0 = 0;
	sl->rebase = b.attempts % BATCH_REBASE == 0;
	const double t_end = d[i].t_end;
	if (st->not_finite) {
		b.status = 2;
		sl->active = 0;
		st->accept = 0;
	} else if (st->accept) {
		st->t += h;
		st->h = st->h_new;
		b.steps++;
		if (t_end > 0.0) {
			if (st->t >= t_end) {
				b.status = 1;
				sl->active = 0;
			} else if (st->t + st->h > t_end) {
				st->h = t_end - st->t;
			}
		} else if (check_every > 0 && b.steps % check_every == 0 && tq2 < tq_thr2) {
			b.status = 1;
			sl->active = 0;
		}
	} else {
		st->h = st->h_new;
		b.rejected++;
		if (t_end > 0.0 && st->t + st->h > t_end) st->h = t_end - st->t;
	}
	b.t = st->t;
	b.h = st->h;
}

// (Re)starts one instance: t = 0, step size h0 (clamped to t_end), counters and reductions
// cleared, k_0 to be evaluated by the next round.
__global__ void k_slot_start(DevState *st, BSlot *sl, double h0, double t_end)
{
	const double h = (t_end > 0.0 && h0 > t_end) ? t_end : h0;
	st->t = 0.0;
	st->h = h;
	st->max_err2 = st->max_k02 = st->max_tq2 = 0.0;
	st->accept = 0;
	st->not_finite = 0;
	sl->bs = BState{0, 0, 0, 0, 0.0, h};
	sl->active = 1;
	sl->need_k0 = 1;
	sl->rebase = 1;
}

// Stops an instance (its slot keeps its results).
__global__ void k_slot_stop(BSlot *sl) { sl->active = 0; }

} // namespace
} // namespace mm

struct mm_batch {
	int prec = MM_F32;
	mm_batch_config cfg{};
	struct Slot {
		mm_solver *s = nullptr;  // nullptr: free slot
		mm::BSlot *dev = nullptr;
		double t_end = 0.0;
		bool stopped = false;    // seen stopped by a run-flag check: left out of rebuilt rounds
		long long start_round = 0;  // the batch round in which the instance's first attempt runs
	};
	std::vector<Slot> slots;
	std::vector<int> members;                     // slot index of each member of the built rounds
	bool dirty = true;                            // membership changed since the rounds were built
	bool any_need_k0 = false;                     // some member starts with the next round
	mm::ConvGroup *conv = nullptr;
	void *desc = nullptr;                         // BDesc<T>[members]
	int2 *stage_items = nullptr, *cell3_items = nullptr, *cell_items = nullptr;
	int tiles_per_item = 4;                       // stage tiles per item of the grouped stage kernel
	int n_stage = 0, n_cell3 = 0, n_cell = 0;
	mm::BSlot *slots_h = nullptr;                 // pinned copies for result queries
	size_t slots_h_cap = 0;
	cudaStream_t gs = nullptr;
	cudaEvent_t ev_in = nullptr, ev_out = nullptr;
	// [0] round with k_0 evaluations, [1] without, [2] FP32 rebase phase
	cudaGraphExec_t gexec[3] = {nullptr, nullptr, nullptr};
	int launches_per_round[3] = {0, 0, 0};
	long long rounds_total = 0;  // rounds run since creation (an instance's attempt count is the
	                             // number of rounds since its start_round)
	unsigned rebase_mask = 0;    // FP32: start rounds of the members, mod BATCH_REBASE
};

namespace mm {
namespace {

void drop_rounds(mm_batch *b)
{
	for (auto &g : b->gexec)
		if (g) cudaGraphExecDestroy(g);
	b->gexec[0] = b->gexec[1] = b->gexec[2] = nullptr;
	conv_group_destroy(b->conv);
	b->conv = nullptr;
	cudaFree(b->desc);
	cudaFree(b->stage_items);
	cudaFree(b->cell3_items);
	cudaFree(b->cell_items);
	b->desc = nullptr;
	b->stage_items = b->cell3_items = b->cell_items = nullptr;
	b->n_stage = b->n_cell3 = b->n_cell = 0;
	b->members.clear();
}

void free_batch(mm_batch *b)
{
	if (!b) return;
	if (b->gs) cudaStreamSynchronize(b->gs);
	drop_rounds(b);
	if (b->gs) cudaStreamDestroy(b->gs);
	if (b->ev_in) cudaEventDestroy(b->ev_in);
	if (b->ev_out) cudaEventDestroy(b->ev_out);
	cudaFreeHost(b->slots_h);
	for (auto &sl : b->slots) {
		free_solver(sl.s);
		cudaFree(sl.dev);
	}
	delete b;
}

// The batch always runs the Dormand-Prince tableau: its stage kernels are compiled for the dp54
// stage patterns (checked against the coefficients at capture).
template <typename T, bool COMP, int S>
void launch_stage_grp(const mm_batch *b, const StageCoef &sc, int in, int out, cudaStream_t st)
{
	const BDesc<T> *d = (const BDesc<T> *)b->desc;
	constexpr int PAT = dp54_pattern(S, COMP);
	if (sc.last)
		k_stage_grp<T, COMP, S, true, PAT><<<b->n_stage, dim3(32, 8, 1), stage_smem<T>(), st>>>(d, sc, in, out,
		                                                                                    b->stage_items,
		                                                                                    b->tiles_per_item);
	else
		k_stage_grp<T, COMP, S, false, PAT><<<b->n_stage, dim3(32, 8, 1), stage_smem<T>(), st>>>(d, sc, in, out,
		                                                                                     b->stage_items,
		                                                                                     b->tiles_per_item);
}

template <typename T, bool COMP>
mm_status stage_grp(const mm_batch *b, const StageCoef &sc, int in, int out, cudaStream_t st)
{
	if (sc.stage < 0 || sc.stage > 6 || pattern_of(sc, sc.stage) != dp54_pattern(sc.stage, COMP))
		return fail(MM_ERR_INVALID_ARGUMENT, "batch: stage coefficients differ from the Dormand-Prince stage patterns");
	switch (sc.stage) {
	case 0: launch_stage_grp<T, COMP, 0>(b, sc, in, out, st); break;
	case 1: launch_stage_grp<T, COMP, 1>(b, sc, in, out, st); break;
	case 2: launch_stage_grp<T, COMP, 2>(b, sc, in, out, st); break;
	case 3: launch_stage_grp<T, COMP, 3>(b, sc, in, out, st); break;
	case 4: launch_stage_grp<T, COMP, 4>(b, sc, in, out, st); break;
	case 5: launch_stage_grp<T, COMP, 5>(b, sc, in, out, st); break;
	case 6: launch_stage_grp<T, COMP, 6>(b, sc, in, out, st); break;
	default: return fail(MM_ERR_UNSUPPORTED, "batch: stage index beyond the dp54 tableau");
	}
	return after_launch("k_stage_grp");
}

// One lock-step round over the members: an attempt each, the controller decision and the accept
// step.  with_k0: instances flagged need_k0 evaluate k_0 at their state first; the others take
// it from the previous attempt's last stage (first same as last, also after a rejection, like
// the reference).
template <typename T>
mm_status batch_round(mm_batch *b, bool with_k0, cudaStream_t st)
{
	constexpr bool COMP = sizeof(T) == 4;
	const Tableau tb = make_tableau(MM_RK_DP54);
	const BDesc<T> *d = (const BDesc<T> *)b->desc;
	if (with_k0) {
		StageCoef sc{};
		sc.stage = 0;
		sc.a_i = tb.a[0];
		sc.write_next = 1;
		sc.bn[0] = tb.b[1][0];
		MM_TRY(conv_group_execute(b->conv, COMP ? 3 : 0, 1, st));
		MM_TRY((stage_grp<T, COMP>(b, sc, 0, 0, st)));
	}
	k_prepare1_grp<T, COMP><<<b->n_cell3, 256, 0, st>>>(d, tb.b[1][0], b->cell3_items);
	MM_TRY(after_launch("k_prepare1_grp"));
	int last_buf = 0;
	for (int i = 1; i < tb.s; ++i) {
		StageCoef sc{};
		sc.stage = i;
		sc.last = (i == tb.s - 1);
		sc.a_i = tb.a[i];
		sc.reduce_k0 = (i == 1);
		if (!sc.last) {
			sc.write_next = 1;
			for (int l = 0; l <= i; ++l) sc.bn[l] = tb.b[i + 1][l];
		} else {
			sc.write_new = COMP || !tb.fsal;
			for (int l = 0; l <= i; ++l) {
				sc.bn[l] = tb.c[l];
				sc.ec[l] = tb.ec[l];
			}
		}
		const int in = 1 + ((i - 1) & 1);
		MM_TRY(conv_group_execute(b->conv, in, 0, st));
		MM_TRY((stage_grp<T, COMP>(b, sc, in, i & 1, st)));
		if (sc.last) last_buf = sc.write_new ? (i & 1) : ((i - 1) & 1);
	}
	const double thr = b->cfg.max_torque;
	const int count = (int)b->members.size();
	k_controller_grp<T><<<(count + 127) / 128, 128, 0, st>>>(d, count, b->cfg.eps_abs, b->cfg.eps_rel, tb.order, tb.fsal,
	                                                        tb.s, thr * thr, b->cfg.check_every_nth_step);
	MM_TRY(after_launch("k_controller_grp"));
	k_accept_grp<T, COMP><<<b->n_cell, 256, 0, st>>>(d, last_buf, b->cell_items);
	MM_TRY(after_launch("k_accept_grp"));
	return MM_OK;
}

// FP32 rebase phase, replayed before the rounds in which some member is due (the flag of each
// instance decides whether it takes part): base state, then its field (convolution output 1,
// gated by the rebase flag), then its exchange part.
mm_status batch_rebase(mm_batch *b, cudaStream_t st)
{
	const BDesc<float> *df = (const BDesc<float> *)b->desc;
	k_rebase_grp<<<b->n_cell3, 256, 0, st>>>(df, b->cell3_items);
	MM_TRY(after_launch("k_rebase_grp"));
	MM_TRY(conv_group_execute(b->conv, 0, 2, st, 1));
	k_base_grp<<<b->n_cell, 256, 0, st>>>(df, b->cell_items);
	return after_launch("k_base_grp");
}

template <typename T, bool COMP, int... S>
mm_status stage_grp_attrs(std::integer_sequence<int, S...>)
{
	const int bytes = (int)stage_smem<T>();
	cudaError_t e = cudaSuccess;
	((e = e == cudaSuccess ? cudaFuncSetAttribute(k_stage_grp<T, COMP, S, false, dp54_pattern(S, COMP)>,
	                                              cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)
	                       : e),
	 ...);
	((e = e == cudaSuccess ? cudaFuncSetAttribute(k_stage_grp<T, COMP, S, true, dp54_pattern(S, COMP)>,
	                                              cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)
	                       : e),
	 ...);
	MM_CUDA(e);
	return MM_OK;
}

// Captures one round into a graph on the batch's private stream.
template <typename T>
mm_status batch_graph(mm_batch *b, int v)
{
	cudaGraph_t g = nullptr;
	const uint64_t l0 = launch_counter().load();
	MM_CUDA(cudaStreamBeginCapture(b->gs, cudaStreamCaptureModeThreadLocal));
	const mm_status r = v == 2 ? batch_rebase(b, b->gs) : batch_round<T>(b, v == 0, b->gs);
	const cudaError_t e = cudaStreamEndCapture(b->gs, &g);
	if (r != MM_OK) {
		if (g) cudaGraphDestroy(g);
		return r;
	}
	MM_CUDA(e);
	const cudaError_t ei = cudaGraphInstantiate(&b->gexec[v], g, 0);
	cudaGraphDestroy(g);
	MM_CUDA(ei);
	b->launches_per_round[v] = (int)(launch_counter().load() - l0);
	launch_counter().fetch_sub(b->launches_per_round[v]);  // counted again at each replay
	return MM_OK;
}

// Work lists, descriptors, grouped convolution and captured rounds of the current members.
template <typename T>
mm_status build_rounds(mm_batch *b, cudaStream_t st)
{
	drop_rounds(b);
	std::vector<BDesc<T>> h;
	std::vector<ConvGroupMember> mem;
	std::vector<int2> si, c3, c1;
	// stage tiles per work item: four while the tiles fill the device twice over, else one (a
	// small batch, such as the tail of a relaxation, then spreads over more SMs; per-cell
	// arithmetic and the maxima do not depend on the grouping)
	{
		long long tiles = 0;
		for (const mm_batch::Slot &sl : b->slots)
			if (sl.s && !sl.stopped) {
				const dim3 tg = stage_grid(sl.s->cfg);
				tiles += (long long)tg.x * tg.y * tg.z;
			}
		b->tiles_per_item = tiles >= 2LL * BATCH_TILES * 3 * num_sms() ? BATCH_TILES : 1;
	}
	for (int k = 0; k < (int)b->slots.size(); ++k) {
		const mm_batch::Slot &sl = b->slots[k];
		if (!sl.s || sl.stopped) continue;
		mm_solver *s = sl.s;
		const int i = (int)b->members.size();
		b->members.push_back(k);
		BDesc<T> d{};
		d.a = args_of<T>(s);
		d.m = (T *)s->m;
		d.m_lo = (T *)s->m_lo;
		d.ys[0] = (T *)s->ys[0];
		d.ys[1] = (T *)s->ys[1];
		d.hd = (T *)s->hd;
		d.ynew_lo = (T *)s->ynew_lo;
		d.hb = sizeof(T) == 4 ? (T *)s->ynew_lo : nullptr;
		d.kt = (KTab<T> *)s->ktab;
		d.ds = s->dst;
		d.slot = sl.dev;
		d.t_end = sl.t_end;
		d.n = (int)s->n;
		const dim3 tg = stage_grid(s->cfg);
		d.tiles_x = (int)tg.x;
		d.tiles_y = (int)tg.y;
		d.ntiles = (int)(tg.x * tg.y * tg.z);
		h.push_back(d);
		for (int t = 0; t < d.ntiles; t += b->tiles_per_item) si.push_back(make_int2(i, t));
		for (int c = 0; (size_t)c * BATCH_CHUNK < 3 * s->n; ++c) c3.push_back(make_int2(i, c));
		for (int c = 0; (size_t)c * BATCH_CHUNK < s->n; ++c) c1.push_back(make_int2(i, c));
		mem.push_back(ConvGroupMember{s->conv, {s->m, s->ys[0], s->ys[1], s->m_lo},
		                              {s->hd, sizeof(T) == 4 ? s->ynew_lo : nullptr}, s->reg, s->ms_tab,
		                              &sl.dev->active});
	}
	b->dirty = false;
	if (b->members.empty()) return MM_OK;
	MM_TRY(conv_group_create(&b->conv, mem.data(), (int)mem.size(), st));
	auto up = [&](void **dst, const void *src, size_t bytes) -> mm_status {
		MM_CUDA(cudaMalloc(dst, bytes));
		MM_CUDA(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, st));
		return MM_OK;
	};
	MM_TRY(up(&b->desc, h.data(), sizeof(BDesc<T>) * h.size()));
	MM_TRY(up((void **)&b->stage_items, si.data(), sizeof(int2) * si.size()));
	MM_TRY(up((void **)&b->cell3_items, c3.data(), sizeof(int2) * c3.size()));
	MM_TRY(up((void **)&b->cell_items, c1.data(), sizeof(int2) * c1.size()));
	b->n_stage = (int)si.size();
	b->n_cell3 = (int)c3.size();
	b->n_cell = (int)c1.size();
	MM_CUDA(cudaStreamSynchronize(st));
	MM_TRY((stage_grp_attrs<T, sizeof(T) == 4>(std::make_integer_sequence<int, 7>())));
	MM_TRY(batch_graph<T>(b, 0));
	MM_TRY(batch_graph<T>(b, 1));
	if (sizeof(T) == 4) MM_TRY(batch_graph<T>(b, 2));
	// residues (mod BATCH_REBASE) of the members' start rounds: the rounds that need the rebase phase
	b->rebase_mask = 0;
	for (int k : b->members) b->rebase_mask |= 1u << (b->slots[k].start_round % BATCH_REBASE);
	return MM_OK;
}

// Device bytes of one instance: resident (state, stage vectors, spectra, tensor spectrum) and the
// extra transient peak of its set-up (the FP64 tensor and its FFT workspace).
void instance_bytes(const mm_batch_instance &q, int prec, size_t *resident, size_t *transient)
{
	const size_t s = prec == MM_F32 ? 4 : 8, n = (size_t)q.nx * q.ny * q.nz;
	const int px = mm_round_tensor_dimension(q.nx, 0, MM_PADDING_ROUND_POT);
	const int py = mm_round_tensor_dimension(q.ny, 0, MM_PADDING_ROUND_POT);
	int pz = mm_round_tensor_dimension(q.nz, 0, MM_PADDING_ROUND_POT);
	if (pz < 2) pz = 2;
	const size_t hx = px / 2 + 1, qy = py / 2 + 1, qz = pz / 2 + 1;
	const size_t E = prec == MM_F32 ? 1 : 2;
	size_t w = hx * E;
	const size_t nb = (w + 255) / 256;
	w = (w + 2 * nb - 1) / (2 * nb) * (2 * nb);
	const size_t lx = w / E;
	const size_t vecs = (prec == MM_F32 ? 3 : 1) + 2 + 7 + 1;  // m (+lo, ynew_lo), ys[2], k[7], H_demag
	const size_t tensor = 6 * qz * qy * hx * s;
	*resident = vecs * 3 * n * s + n + 3 * (size_t)q.nz * py * lx * 2 * s + tensor + (1 << 16);
	if (conv_group_fused(prec, py, pz, q.nz)) *resident += tensor;  // the fused pass's kx-major copy
	*transient = 6 * (size_t)px * py * pz * 8 + (size_t)px * py * pz * 16;
}

template <typename T>
mm_status add_instance(mm_batch *b, const mm_batch_instance &q, const uint8_t *mask, int *slot_out,
                       cudaStream_t st)
{
	mm_solver_config c{};
	c.nx = q.nx; c.ny = q.ny; c.nz = q.nz;
	c.dx = q.dx; c.dy = q.dy; c.dz = q.dz;
	c.precision = b->prec;
	c.tableau = MM_RK_DP54;
	c.terms = MM_TERM_DEMAG | MM_TERM_EXCHANGE;
	bool zeeman = false;
	for (int k = 0; k < 3; ++k) {
		c.H_ext[k] = q.H_ext[k];
		c.H_pulse[k] = q.H_pulse[k];
		zeeman = zeeman || q.H_ext[k] != 0.0 || q.H_pulse[k] != 0.0;
	}
	if (zeeman) c.terms |= MM_TERM_ZEEMAN;
	c.pulse_rise = q.pulse_rise;
	c.do_precess = 1;
	c.zl_do_precess = 1;
	c.padding = MM_PADDING_ROUND_POT;
	c.eps_abs = b->cfg.eps_abs;
	c.eps_rel = b->cfg.eps_rel;
	c.h0 = b->cfg.h0;
	c.fsal_reuse_after_reject = 1;
	mm_material mats[2] = {};
	mats[1].Ms = q.Ms;
	mats[1].A = q.A;
	mats[1].alpha = q.alpha;
	mats[0].alpha = q.alpha;
	const size_t n = (size_t)q.nx * q.ny * q.nz;
	std::vector<uint8_t> ones;
	if (!mask) {
		ones.assign(n, 1);
		mask = ones.data();
	}
	mm_solver *s = nullptr;
	MM_TRY(solver_create(&s, &c, 2, mats, mask, nullptr, st, 2));
	BSlot *dev = nullptr;
	const cudaError_t e = cudaMalloc(&dev, sizeof(BSlot));
	if (e != cudaSuccess) {
		free_solver(s);
		return cuda_status(e, "cudaMalloc");
	}
	cudaMemsetAsync(dev, 0, sizeof(BSlot), st);  // not running until it gets a state
	int k = 0;
	while (k < (int)b->slots.size() && b->slots[k].s) ++k;
	if (k == (int)b->slots.size()) b->slots.emplace_back();
	b->slots[k].s = s;
	b->slots[k].dev = dev;
	b->slots[k].t_end = q.t_end;
	b->dirty = true;
	*slot_out = k;
	MM_CUDA(cudaStreamSynchronize(st));
	return MM_OK;
}

mm_batch::Slot *slot_of(mm_batch *b, int k)
{
	return (b && k >= 0 && k < (int)b->slots.size() && b->slots[k].s) ? &b->slots[k] : nullptr;
}

} // namespace
} // namespace mm

extern "C" {

MM_API mm_status mm_batch_instance_bytes(const mm_batch_instance *instance, int precision, size_t *resident,
                                         size_t *transient)
{
	if (!instance || !resident || !transient || (precision != MM_F64 && precision != MM_F32))
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_batch_instance_bytes: invalid argument");
	instance_bytes(*instance, precision, resident, transient);
	return MM_OK;
}

MM_API mm_status mm_batch_create(mm_batch **out, const mm_batch_config *cfg, int count,
                                 const mm_batch_instance *inst_host, const uint8_t *masks_host, void *stream)
{
	if (!out || !cfg || count < 0 || (count > 0 && !inst_host))
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_batch_create: invalid argument");
	if (cfg->precision != MM_F64 && cfg->precision != MM_F32)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_batch_create: invalid precision");
	if (!(cfg->eps_abs > 0) || !(cfg->eps_rel > 0) || !(cfg->h0 > 0) || !(cfg->max_torque >= 0) ||
	    cfg->check_every_nth_step < 1)
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_batch_create: invalid tolerances, h0, torque or check interval");
	cudaStream_t st = as_stream(stream);
	mm_batch *b = new mm_batch();
	b->prec = cfg->precision;
	b->cfg = *cfg;
	mm_status r = cuda_status(cudaStreamCreateWithFlags(&b->gs, cudaStreamNonBlocking), "cudaStreamCreate");
	if (r == MM_OK) r = cuda_status(cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming), "cudaEventCreate");
	if (r == MM_OK) r = cuda_status(cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming), "cudaEventCreate");
	size_t off = 0;
	for (int i = 0; i < count && r == MM_OK; ++i) {
		int slot = 0;
		r = b->prec == MM_F64 ? add_instance<double>(b, inst_host[i], masks_host ? masks_host + off : nullptr, &slot, st)
		                      : add_instance<float>(b, inst_host[i], masks_host ? masks_host + off : nullptr, &slot, st);
		off += (size_t)inst_host[i].nx * inst_host[i].ny * inst_host[i].nz;
	}
	if (r != MM_OK) {
		free_batch(b);
		return r;
	}
	*out = b;
	return MM_OK;
}

MM_API mm_status mm_batch_destroy(mm_batch *b)
{
	std::lock_guard<std::mutex> lock(capture_mutex());
	free_batch(b);
	return MM_OK;
}

MM_API mm_status mm_batch_add(mm_batch *b, const mm_batch_instance *instance, const uint8_t *mask_host,
                              int *slot_out, void *stream)
{
	if (!b || !instance || !slot_out) return fail(MM_ERR_INVALID_ARGUMENT, "mm_batch_add: invalid argument");
	cudaStream_t st = as_stream(stream);
	std::lock_guard<std::mutex> lock(capture_mutex());
	return b->prec == MM_F64 ? add_instance<double>(b, *instance, mask_host, slot_out, st)
	                         : add_instance<float>(b, *instance, mask_host, slot_out, st);
}

MM_API mm_status mm_batch_remove(mm_batch *b, int slot)
{
	mm_batch::Slot *sl = slot_of(b, slot);
	if (!sl) return fail(MM_ERR_INVALID_ARGUMENT, "mm_batch_remove: no such slot");
	MM_CUDA(cudaStreamSynchronize(b->gs));
	std::lock_guard<std::mutex> lock(capture_mutex());
	free_solver(sl->s);
	cudaFree(sl->dev);
	*sl = mm_batch::Slot{};
	b->dirty = true;
	return MM_OK;
}

MM_API int mm_batch_slot_count(mm_batch *b) { return b ? (int)b->slots.size() : 0; }

MM_API mm_status mm_batch_set_M(mm_batch *b, int slot, const double *M_device, void *stream)
{
	mm_batch::Slot *sl = slot_of(b, slot);
	if (!sl || !M_device) return fail(MM_ERR_INVALID_ARGUMENT, "mm_batch_set_M: invalid argument");
	cudaStream_t st = as_stream(stream);
	MM_CUDA(cudaStreamSynchronize(b->gs));
	MM_TRY(mm_solver_set_M(sl->s, M_device, stream));
	if (sl->stopped) {  // left out of the rounds since it stopped: back in
		sl->stopped = false;
		b->dirty = true;
	}
	sl->start_round = b->rounds_total;  // its first attempt runs in the next round
	b->rebase_mask |= 1u << (sl->start_round % BATCH_REBASE);
	k_slot_start<<<1, 1, 0, st>>>(sl->s->dst, sl->dev, b->cfg.h0, sl->t_end);
	MM_TRY(after_launch("k_slot_start"));
	MM_CUDA(cudaStreamSynchronize(st));
	b->any_need_k0 = true;
	return MM_OK;
}

MM_API mm_status mm_batch_get_M(mm_batch *b, int slot, double *M_device, void *stream)
{
	mm_batch::Slot *sl = slot_of(b, slot);
	if (!sl || !M_device) return fail(MM_ERR_INVALID_ARGUMENT, "mm_batch_get_M: invalid argument");
	MM_CUDA(cudaStreamSynchronize(b->gs));
	return mm_solver_get_M(sl->s, M_device, stream);
}

MM_API mm_status mm_batch_stop(mm_batch *b, int slot, void *stream)
{
	mm_batch::Slot *sl = slot_of(b, slot);
	if (!sl) return fail(MM_ERR_INVALID_ARGUMENT, "mm_batch_stop: no such slot");
	MM_CUDA(cudaStreamSynchronize(b->gs));
	k_slot_stop<<<1, 1, 0, as_stream(stream)>>>(sl->dev);
	return after_launch("k_slot_stop");
}

MM_API mm_status mm_batch_relax(mm_batch *b, long long max_rounds, int check_interval, long long *rounds_out,
                                void *stream)
{
	if (!b || max_rounds < 0 || check_interval < 1) return fail(MM_ERR_INVALID_ARGUMENT, "mm_batch_relax: invalid argument");
	cudaStream_t st = as_stream(stream);
	long long done = 0;
	// Rounds replay the graphs of the current members.  When a run-flag check finds a quarter of
	// them stopped, the rounds are rebuilt over the running ones (fewer work items and launches per
	// round; an instance's arithmetic does not depend on the members around it).
	for (bool compact = true; compact && done < max_rounds;) {
		compact = false;
		if (b->dirty) {
			std::lock_guard<std::mutex> lock(capture_mutex());
			MM_TRY(b->prec == MM_F64 ? build_rounds<double>(b, st) : build_rounds<float>(b, st));
		}
		if (b->members.empty()) break;
		const size_t cnt = b->members.size();
		if (b->slots_h_cap < cnt) {
			cudaFreeHost(b->slots_h);
			b->slots_h = nullptr;
			MM_CUDA(cudaMallocHost(&b->slots_h, sizeof(BSlot) * cnt));
			b->slots_h_cap = cnt;
		}
		MM_CUDA(cudaEventRecord(b->ev_in, st));
		MM_CUDA(cudaStreamWaitEvent(b->gs, b->ev_in, 0));
		while (done < max_rounds) {
			if (b->gexec[2] && (b->rebase_mask >> (b->rounds_total % BATCH_REBASE) & 1u)) {
				MM_CUDA(cudaGraphLaunch(b->gexec[2], b->gs));
				launch_counter().fetch_add(b->launches_per_round[2]);
			}
			const int v = b->any_need_k0 ? 0 : 1;
			MM_CUDA(cudaGraphLaunch(b->gexec[v], b->gs));
			launch_counter().fetch_add(b->launches_per_round[v]);
			b->any_need_k0 = false;
			++done;
			++b->rounds_total;
			if (done % check_interval == 0 || done == max_rounds) {
				for (size_t i = 0; i < cnt; ++i)
					MM_CUDA(cudaMemcpyAsync(&b->slots_h[i], b->slots[b->members[i]].dev, sizeof(BSlot),
					                        cudaMemcpyDeviceToHost, b->gs));
				MM_CUDA(cudaStreamSynchronize(b->gs));
				size_t left = 0;
				for (size_t i = 0; i < cnt; ++i) {
					left += b->slots_h[i].active ? 1 : 0;
					if (!b->slots_h[i].active) b->slots[b->members[i]].stopped = true;
				}
				if (!left) break;
				if (4 * left <= 3 * cnt && cnt > 1) {
					b->dirty = true;
					compact = true;
					break;
				}
			}
		}
		MM_CUDA(cudaEventRecord(b->ev_out, b->gs));
		MM_CUDA(cudaStreamWaitEvent(st, b->ev_out, 0));
	}
	MM_CUDA(cudaStreamSynchronize(st));
	if (rounds_out) *rounds_out = done;
	return MM_OK;
}

// Results of every slot (status -1 for a free slot).
MM_API mm_status mm_batch_results(mm_batch *b, mm_batch_result *out_host, void *stream)
{
	if (!b || !out_host) return fail(MM_ERR_INVALID_ARGUMENT, "mm_batch_results: invalid argument");
	cudaStream_t st = as_stream(stream);
	MM_CUDA(cudaStreamSynchronize(b->gs));
	for (size_t k = 0; k < b->slots.size(); ++k) {
		const mm_batch::Slot &sl = b->slots[k];
		if (!sl.s) {
			out_host[k] = mm_batch_result{-1, 0, 0, 0, 0.0, 0.0};
			continue;
		}
		BSlot h{};
		MM_CUDA(cudaMemcpyAsync(&h, sl.dev, sizeof(BSlot), cudaMemcpyDeviceToHost, st));
		MM_CUDA(cudaStreamSynchronize(st));
		out_host[k] = mm_batch_result{h.bs.status, h.bs.steps, h.bs.attempts, h.bs.rejected, h.bs.t, h.bs.h};
	}
	return MM_OK;
}

MM_API mm_status mm_batch_launches_per_round(mm_batch *b, int *first, int *later)
{
	if (!b) return fail(MM_ERR_INVALID_ARGUMENT, "mm_batch_launches_per_round: null batch");
	if (first) *first = b->launches_per_round[0];
	if (later) *later = b->launches_per_round[1];
	return MM_OK;
}

} // extern "C"
