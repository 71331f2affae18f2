// Zero-padded FFT convolution H = N * M with the symmetric demag tensor (internal API).
#pragma once

#include <cuda.h>

#include "mm_common.cuh"
#include "fft.cuh"

namespace mm {

struct ConvPlan {
	int prec = MM_F64;
	int nx = 0, ny = 0, nz = 0;     // grid
	int px = 0, py = 0, pz = 0;     // padded (FFT) lengths
	int hx = 0;                     // px/2 + 1 stored x frequencies
	int lx = 0;                     // spectrum row stride (>= hx complex, rows 16-byte aligned)
	int xbox_n = 1, xbox_w = 0;     // a spectrum row as xbox_n TMA boxes of xbox_w 8-byte elements
	int qy = 0, qz = 0;             // py/2 + 1, pz/2 + 1 stored tensor frequencies
	bool is2d = false;              // nz == 1 && pz == 1
	bool fast_x = false, fast_y = false, fast_z = false;  // power-of-two register-FFT passes
	bool reg_z = false;             // z pass with whole columns in registers (nz <= pz/2, pz small)
	bool tma_y = false;             // y passes fed by TMA-staged tiles (persistent CTAs)
	CUtensorMap tm_yf{}, tm_yi{};   // spectrum views of the forward (ny rows) and inverse (py rows) y pass
	int grid_yf = 0, grid_yi = 0;   // persistent grid sizes of those passes
	int *err = nullptr;             // device word set when a bounded wait of a staged pass gave up
	bool tma_xf = false, tma_xi = false;  // x passes fed by TMA-staged tiles
	bool tma_xf_scale = false;            // ... also with the Ms[region] input scale
	int grid_xf = 0, grid_xi = 0;
	int xf_box_n = 1, xf_box_w = 0;       // a real input row as boxes of 8-byte elements
	CUtensorMap tm_xi{};                  // spectrum rows y < ny of each plane, for the inverse x pass
	static constexpr int XF_CACHE = 4;    // forward-pass maps, one per input buffer seen
	const void *xf_ptr[XF_CACHE] = {};
	CUtensorMap xf_map[XF_CACHE] = {};
	int xf_next = 0;
	const void *xr_ptr = nullptr;         // region map the region tensor map was encoded for
	CUtensorMap xr_map{};                 // region bytes of the forward pass's rows
	FftRadices rx{}, ry{}, rz{};
	void *tw_x = nullptr, *tw_y = nullptr, *tw_z = nullptr;  // cplx<T> twiddle tables
	void *tensor = nullptr;         // reduced real tensor spectrum, T[6][qz][qy][hx]
	void *tensor_kx = nullptr;      // the same, kx-major T[hx][qz][qy][6] (made by the first grouped
	                                // convolution whose fused y+z pass takes this plan)
	void *spec = nullptr;           // cplx<T>[3][nz][py][lx]
	// launch geometry
	int lp_x = 1;                   // complex lines (= 2 real rows) per CTA in the x passes
	int tb_y = 1, tb_z = 1;         // columns per CTA in the y and z passes
	size_t smem_x = 0, smem_y = 0, smem_z = 0;
	double max_imag_rel = 0.0;      // largest |Im N^| / max |Re N^| seen at set-up

	size_t spec_bytes() const;
	~ConvPlan();
};

// Builds the plan and the tensor spectrum from an FP64 tensor in the reference layout
// (component fastest, then x, y, z) of padded size px*py*pz.
mm_status conv_plan_create(ConvPlan **out, int prec, int nx, int ny, int nz, int px, int py,
                           int pz, const double *N_device, cudaStream_t st);

// H = N * (Ms[region] * M) when regions/ms_table are given (ms_table: 256 entries), else H = N * M.
// M and H are SoA arrays of T (T = double for MM_F64, float for MM_F32).
mm_status conv_execute(ConvPlan *p, const void *M, const uint8_t *regions, const void *ms_table,
                       void *H, cudaStream_t st);

// Number of kernel launches one conv_execute issues.
int conv_launches(const ConvPlan *p);

// Grouped convolution over many plans of the same precision, each with power-of-two 3-D padding
// and a register z pass: one launch per pass and transform length covers every member.  M[k]
// are up to four candidate inputs per member and H[k] up to two outputs (each selected per call;
// H[1] may be NULL, then only output 0 is allowed); flags (device, optional) are the member's run
// flags: flags[0] == 0 skips it, and with gate != 0 so does flags[gate] == 0.
struct ConvGroup;
struct ConvGroupMember {
	ConvPlan *plan;
	const void *M[4];
	void *H[2];
	const uint8_t *reg;
	const void *ms_tab;  // 256 entries
	const int *flags;    // device run flags, NULL: always run
};
mm_status conv_group_create(ConvGroup **out, const ConvGroupMember *members, int count, cudaStream_t st);
mm_status conv_group_execute(ConvGroup *g, int input, int gate, cudaStream_t st, int output = 0);
int conv_group_launches(const ConvGroup *g);
void conv_group_destroy(ConvGroup *g);
// Whether a member with these padded lengths takes the grouped fused y+z pass (which keeps a
// second, kx-major copy of its reduced tensor).
int conv_group_fused(int prec, int py, int pz, int nz);

FftRadices fft_factor(int n);

} // namespace mm
