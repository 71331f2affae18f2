// OOMMF OMF 1.0 vector-field files (rectangular mesh, one segment): the reference's readOMF /
// writeOMF (src/magneto/mmm/io/OMFImport.cpp, OMFExport.cpp, OMFHeader.h), for device fields.
//
// Reading: the header lines are parsed on the host with the reference's grammar (line ends LF,
// CR, CRLF or LFCR; "# key: value" comment lines; the keys of OMFHeader; "Begin: Data Text |
// Binary 4 | Binary 8").  Binary payloads (big-endian values after a big-endian check value) go
// to the device as they are and one kernel swaps the bytes, scales by valuemultiplier and
// scatters the interleaved (x, y, z) triples into the SoA field.  Text payloads are parsed by
// host threads (one line per cell, three numbers) into interleaved doubles, then the same kernel
// finishes them.
//
// Writing: one device reduction gives min/max |v| (OMFExport.cpp:196-209), the field is scaled by
// 1/max when max > 0.001 unless MAGNUM_OMF_NOSCALE is set (OMFExport.cpp:61-79), and a kernel
// writes the interleaved, byte-swapped payload; text values are formatted on the host with 16
// significant digits, like the reference's ostream precision(16).  Binary 8 values are written
// big-endian as the OMF 1.0 format (and the reference's reader) expect; the reference's writer
// leaves them in host order (OMFExport.cpp:171-177), so its binary-8 files do not read back
// through its own reader on a little-endian host.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "mm_common.cuh"

namespace mm {
namespace {

constexpr int OMF_TPB = 256;

// ---- device: interleaved payload <-> SoA field ------------------------------------------------
template <typename S>
__device__ __forceinline__ S from_be(S v);

template <>
__device__ __forceinline__ float from_be<float>(float v)
{
	return __int_as_float((int)__byte_perm((unsigned)__float_as_int(v), 0, 0x0123));
}

template <>
__device__ __forceinline__ double from_be<double>(double v)
{
	const unsigned long long u = (unsigned long long)__double_as_longlong(v);
	const unsigned lo = (unsigned)(u & 0xffffffffull), hi = (unsigned)(u >> 32);
	const unsigned long long r = ((unsigned long long)__byte_perm(lo, 0, 0x0123) << 32) | __byte_perm(hi, 0, 0x0123);
	return __longlong_as_double((long long)r);
}

// src: 3n values (x, y, z per cell), big-endian when BE; dst: SoA of T.
template <typename S, bool BE, typename T>
__global__ void __launch_bounds__(OMF_TPB) k_omf_unpack(size_t n, const S *__restrict__ src, double mult,
                                                        T *__restrict__ dst)
{
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
		for (int c = 0; c < 3; ++c) {
			S v = src[3 * i + c];
			if (BE) v = from_be<S>(v);
			dst[c * n + i] = (T)((double)v * mult);
		}
	}
}

// min / max of |v| over the cells (as ordered bit patterns of non-negative doubles).
template <typename T>
__global__ void __launch_bounds__(OMF_TPB) k_omf_range(size_t n, const T *__restrict__ M,
                                                       unsigned long long *minmax)
{
	double lo = INFINITY, hi = 0.0;
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
		const double x = M[i], y = M[i + n], z = M[i + 2 * n];
		const double len = sqrt(x * x + y * y + z * z);
		lo = fmin(lo, len);
		hi = fmax(hi, len);
	}
	for (int o = 16; o > 0; o >>= 1) {
		lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
		hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
	}
	if ((threadIdx.x & 31) == 0) {
		atomicMin(&minmax[0], (unsigned long long)__double_as_longlong(lo));
		atomicMax(&minmax[1], (unsigned long long)__double_as_longlong(hi));
	}
}

// SoA field -> interleaved (x, y, z) values times `scale`, big-endian when BE.
template <typename S, bool BE, typename T>
__global__ void __launch_bounds__(OMF_TPB) k_omf_pack(size_t n, const T *__restrict__ M, double scale,
                                                      S *__restrict__ out)
{
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
		for (int c = 0; c < 3; ++c) {
			S v = (S)((double)M[c * n + i] * scale);
			if (BE) v = from_be<S>(v);  // the swap is its own inverse
			out[3 * i + c] = v;
		}
	}
}

int omf_grid(size_t n)
{
	const size_t want = (n + OMF_TPB - 1) / OMF_TPB, cap = (size_t)num_sms() * 8;
	return (int)std::max<size_t>(1, std::min(want, cap));
}

// ---- host: the reference's line and header grammar ----------------------------------------------
struct Reader {
	const char *p, *end;
	std::string line;
	bool eof = false;

	// OMFImport::acceptLine: a line ends at LF, CR, CRLF or LFCR.
	void next()
	{
		line.clear();
		if (p >= end) {
			eof = true;
			line = "<end-of-file>";
			return;
		}
		while (p < end) {
			const char c = *p++;
			if (c == '\n' || c == '\r') {
				const char other = c == '\n' ? '\r' : '\n';
				if (p < end && *p == other) ++p;
				return;
			}
			line += c;
		}
	}
};

std::string trim(const std::string &s)
{
	size_t a = 0, b = s.size();
	while (a < b && std::isspace((unsigned char)s[a])) ++a;
	while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
	return s.substr(a, b - a);
}

// OMFImport.cpp parseCommentLine: "# key: value" (key non-empty).
bool comment(const std::string &line, std::string &key, std::string &value)
{
	if (line.size() < 2 || line[0] != '#') return false;
	const size_t colon = line.find(':', 1);
	if (colon == std::string::npos) return false;
	key = trim(line.substr(1, colon - 1));
	value = trim(line.substr(colon + 1));
	return !key.empty();
}

void put(char *dst, size_t cap, const std::string &v)
{
	const size_t n = std::min(cap - 1, v.size());
	std::memcpy(dst, v.data(), n);
	dst[n] = 0;
}

bool header_key(mm_omf_header *h, const std::string &k, const std::string &v)
{
	const double d = std::strtod(v.c_str(), nullptr);
	if (k == "Title") put(h->title, sizeof h->title, v);
	else if (k == "Desc") {
		std::string all(h->desc);
		if (!all.empty()) all += '\n';
		all += v;
		put(h->desc, sizeof h->desc, all);
	} else if (k == "meshunit") put(h->meshunit, sizeof h->meshunit, v);
	else if (k == "valueunit") put(h->valueunit, sizeof h->valueunit, v);
	else if (k == "meshtype") put(h->meshtype, sizeof h->meshtype, v);
	else if (k == "valuemultiplier") h->valuemultiplier = d;
	else if (k == "xmin") h->xmin = d;
	else if (k == "ymin") h->ymin = d;
	else if (k == "zmin") h->zmin = d;
	else if (k == "xmax") h->xmax = d;
	else if (k == "ymax") h->ymax = d;
	else if (k == "zmax") h->zmax = d;
	else if (k == "ValueRangeMinMag") h->ValueRangeMinMag = d;
	else if (k == "ValueRangeMaxMag") h->ValueRangeMaxMag = d;
	else if (k == "xbase") h->xbase = d;
	else if (k == "ybase") h->ybase = d;
	else if (k == "zbase") h->zbase = d;
	else if (k == "xstepsize") h->xstepsize = d;
	else if (k == "ystepsize") h->ystepsize = d;
	else if (k == "zstepsize") h->zstepsize = d;
	else if (k == "xnodes") h->xnodes = std::atoi(v.c_str());
	else if (k == "ynodes") h->ynodes = std::atoi(v.c_str());
	else if (k == "znodes") h->znodes = std::atoi(v.c_str());
	else return false;  // unknown keys are skipped, as the reference does
	return true;
}

mm_status expect(Reader &r, const char *key, const char *value, const char *what)
{
	std::string k, v;
	if (!comment(r.line, k, v) || k != key || (value && v != value))
		return fail(MM_ERR_INVALID_ARGUMENT, std::string("OMF: expected '") + what + "', found '" + r.line + "'");
	return MM_OK;
}

// Text payload: one line per cell, three numbers; `lines` points at the first data line.
mm_status parse_text(Reader &r, size_t n, std::vector<double> &vals)
{
	// line starts of the n data lines (the reference's acceptLine rules)
	std::vector<const char *> starts(n + 1);
	const char *q = r.p;
	for (size_t i = 0; i < n; ++i) {
		if (q >= r.end) return fail(MM_ERR_INVALID_ARGUMENT, "OMF: the text data ends after " + std::to_string(i) +
		                                                         " of " + std::to_string(n) + " lines");
		starts[i] = q;
		while (q < r.end && *q != '\n' && *q != '\r') ++q;
		if (q < r.end) {
			const char c = *q++;
			const char other = c == '\n' ? '\r' : '\n';
			if (q < r.end && *q == other) ++q;
		}
	}
	starts[n] = q;
	vals.resize(3 * n);
	const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
	const size_t nt = std::min<size_t>(hw, std::max<size_t>(1, n / 4096));
	std::vector<size_t> bad(nt, (size_t)-1);
	auto work = [&](size_t t) {
		const size_t a = n * t / nt, b = n * (t + 1) / nt;
		std::string buf;
		for (size_t i = a; i < b; ++i) {
			buf.assign(starts[i], starts[i + 1]);
			const char *s = buf.c_str();
			char *e = nullptr;
			for (int c = 0; c < 3; ++c) {
				errno = 0;
				const double v = std::strtod(s, &e);
				if (e == s) {
					bad[t] = i;
					return;
				}
				vals[3 * i + c] = v;
				s = e;
			}
		}
	};
	std::vector<std::thread> th;
	for (size_t t = 1; t < nt; ++t) th.emplace_back(work, t);
	work(0);
	for (auto &x : th) x.join();
	for (size_t t = 0; t < nt; ++t)
		if (bad[t] != (size_t)-1) {
			const size_t i = bad[t];
			return fail(MM_ERR_INVALID_ARGUMENT, "OMF: failed to parse the data line '" +
			                                         trim(std::string(starts[i], starts[i + 1])) + "'");
		}
	r.p = q;
	r.next();
	return MM_OK;
}

template <typename T>
mm_status unpack(const void *host, size_t n, int esize, bool be, double mult, T *M, cudaStream_t st)
{
	void *d = nullptr;
	const size_t bytes = 3 * n * (size_t)esize;
	MM_CUDA(cudaMallocAsync(&d, bytes, st));
	cudaError_t e = cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, st);
	if (e == cudaSuccess) {
		if (esize == 4)
			k_omf_unpack<float, true, T><<<omf_grid(n), OMF_TPB, 0, st>>>(n, (const float *)d, mult, M);
		else if (be)
			k_omf_unpack<double, true, T><<<omf_grid(n), OMF_TPB, 0, st>>>(n, (const double *)d, mult, M);
		else
			k_omf_unpack<double, false, T><<<omf_grid(n), OMF_TPB, 0, st>>>(n, (const double *)d, mult, M);
	}
	const mm_status r = e == cudaSuccess ? after_launch("k_omf_unpack") : cuda_status(e, "OMF upload");
	cudaFreeAsync(d, st);
	MM_TRY(r);
	// the host buffer may be released by the caller as soon as this returns
	MM_CUDA(cudaStreamSynchronize(st));
	return MM_OK;
}

float be_float(const unsigned char *b)
{
	const uint32_t u = (uint32_t)b[0] << 24 | (uint32_t)b[1] << 16 | (uint32_t)b[2] << 8 | b[3];
	float f;
	std::memcpy(&f, &u, 4);
	return f;
}

double be_double(const unsigned char *b)
{
	uint64_t u = 0;
	for (int i = 0; i < 8; ++i) u = u << 8 | b[i];
	double d;
	std::memcpy(&d, &u, 8);
	return d;
}

mm_status parse(const char *bytes, size_t len, mm_omf_header *h, int prec, void *M, cudaStream_t st)
{
	std::memset(h, 0, sizeof *h);
	Reader r{bytes, bytes + len};
	r.next();
	std::string k, v;
	if (!comment(r.line, k, v) || k != "OOMMF") return fail(MM_ERR_INVALID_ARGUMENT, "OMF: expected 'OOMMF' at line 1");
	r.next();
	if (!comment(r.line, k, v) || k != "Segment count")
		return fail(MM_ERR_INVALID_ARGUMENT, "OMF: expected 'Segment count' at line 2");
	r.next();
	MM_TRY(expect(r, "Begin", "Segment", "Begin: Segment"));
	r.next();
	MM_TRY(expect(r, "Begin", "Header", "Begin: Header"));
	r.next();
	while (true) {
		if (r.eof) return fail(MM_ERR_INVALID_ARGUMENT, "OMF: the file ends inside the header");
		if (comment(r.line, k, v)) {
			if (k == "End" && v == "Header") break;
			header_key(h, k, v);
		}
		r.next();
	}
	r.next();
	if (!comment(r.line, k, v) || k != "Begin")
		return fail(MM_ERR_INVALID_ARGUMENT, "OMF: expected 'Begin: Data <type>', found '" + r.line + "'");
	int esize = 0;
	if (v == "Data Text") h->format = MM_OMF_TEXT;
	else if (v == "Data Binary 4") h->format = MM_OMF_BINARY_4, esize = 4;
	else if (v == "Data Binary 8") h->format = MM_OMF_BINARY_8, esize = 8;
	else return fail(MM_ERR_INVALID_ARGUMENT, "OMF: expected a 'Data Text', 'Data Binary 4' or 'Data Binary 8' block");
	const std::string tag = v;
	if (h->xnodes <= 0 || h->ynodes <= 0 || h->znodes <= 0)
		return fail(MM_ERR_INVALID_ARGUMENT, "OMF: xnodes, ynodes and znodes must be positive");
	if (!M) return MM_OK;  // header only
	if (prec != MM_F64 && prec != MM_F32) return fail(MM_ERR_INVALID_ARGUMENT, "OMF: invalid precision");
	const size_t n = (size_t)h->xnodes * h->ynodes * h->znodes;
	const double mult = h->valuemultiplier;
	if (esize == 0) {
		std::vector<double> vals;
		MM_TRY(parse_text(r, n, vals));
		MM_TRY(prec == MM_F64 ? unpack<double>(vals.data(), n, 8, false, mult, (double *)M, st)
		                      : unpack<float>(vals.data(), n, 8, false, mult, (float *)M, st));
	} else {
		const unsigned char *b = (const unsigned char *)r.p;
		const size_t need = (size_t)esize * (1 + 3 * n);
		if ((size_t)(r.end - r.p) < need) return fail(MM_ERR_INVALID_ARGUMENT, "OMF: the binary data is truncated");
		if (esize == 4 ? be_float(b) != 1234567.0f : be_double(b) != 123456789012345.0)
			return fail(MM_ERR_INVALID_ARGUMENT, std::string("OMF: wrong check value (binary ") +
			                                         (esize == 4 ? "4" : "8") + " format)");
		MM_TRY(prec == MM_F64 ? unpack<double>(b + esize, n, esize, true, mult, (double *)M, st)
		                      : unpack<float>(b + esize, n, esize, true, mult, (float *)M, st));
		r.p += need;
		r.next();                       // the rest of the payload's line (a newline)
		if (r.line.empty()) r.next();
	}
	if (!comment(r.line, k, v) || k != "End" || v != tag)
		return fail(MM_ERR_INVALID_ARGUMENT, "OMF: expected 'End: " + tag + "', found '" + r.line + "'");
	r.next();
	MM_TRY(expect(r, "End", "Segment", "End: Segment"));
	return MM_OK;
}

// ---- writer -------------------------------------------------------------------------------------
std::string g16(double v)
{
	char b[64];
	std::snprintf(b, sizeof b, "%.16g", v);
	return b;
}

template <typename T>
mm_status payload(const T *M, size_t n, int format, double scale, std::string &out, cudaStream_t st)
{
	const int esize = format == MM_OMF_BINARY_4 ? 4 : 8;
	const size_t bytes = 3 * n * (size_t)esize;
	void *d = nullptr;
	MM_CUDA(cudaMallocAsync(&d, bytes, st));
	if (format == MM_OMF_BINARY_4)
		k_omf_pack<float, true, T><<<omf_grid(n), OMF_TPB, 0, st>>>(n, M, scale, (float *)d);
	else if (format == MM_OMF_BINARY_8)
		k_omf_pack<double, true, T><<<omf_grid(n), OMF_TPB, 0, st>>>(n, M, scale, (double *)d);
	else
		k_omf_pack<double, false, T><<<omf_grid(n), OMF_TPB, 0, st>>>(n, M, scale, (double *)d);
	mm_status r = after_launch("k_omf_pack");
	std::vector<char> host(r == MM_OK ? bytes : 0);
	if (r == MM_OK) r = cuda_status(cudaMemcpyAsync(host.data(), d, bytes, cudaMemcpyDeviceToHost, st), "OMF download");
	cudaFreeAsync(d, st);
	if (r == MM_OK) r = cuda_status(cudaStreamSynchronize(st), "OMF download");
	MM_TRY(r);
	if (format != MM_OMF_TEXT) {
		out.append(host.data(), bytes);
		out += '\n';
		return MM_OK;
	}
	const double *v = (const double *)host.data();
	const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
	const size_t nt = std::min<size_t>(hw, std::max<size_t>(1, n / 4096));
	std::vector<std::string> parts(nt);
	auto work = [&](size_t t) {
		const size_t a = n * t / nt, b = n * (t + 1) / nt;
		std::string &s = parts[t];
		s.reserve((b - a) * 64);
		for (size_t i = a; i < b; ++i) {
			s += g16(v[3 * i]);
			s += ' ';
			s += g16(v[3 * i + 1]);
			s += ' ';
			s += g16(v[3 * i + 2]);
			s += '\n';
		}
	};
	std::vector<std::thread> th;
	for (size_t t = 1; t < nt; ++t) th.emplace_back(work, t);
	work(0);
	for (auto &x : th) x.join();
	for (auto &p : parts) out += p;
	return MM_OK;
}

template <typename T>
mm_status format_omf(mm_omf_header *h, const T *M, int format, std::string &out, cudaStream_t st)
{
	if (h->xnodes <= 0 || h->ynodes <= 0 || h->znodes <= 0)
		return fail(MM_ERR_INVALID_ARGUMENT, "OMF: xnodes, ynodes and znodes must be positive");
	const size_t n = (size_t)h->xnodes * h->ynodes * h->znodes;
	ScalarScratch *sc = nullptr;
	MM_TRY(scalar_scratch(&sc));
	const unsigned long long init[2] = {0x7ff0000000000000ull, 0ull};  // +inf, +0
	MM_CUDA(cudaMemcpyAsync(sc->dev, init, sizeof init, cudaMemcpyHostToDevice, st));
	k_omf_range<T><<<omf_grid(n), OMF_TPB, 0, st>>>(n, M, (unsigned long long *)sc->dev);
	MM_TRY(after_launch("k_omf_range"));
	unsigned long long mm[2];
	MM_CUDA(cudaMemcpyAsync(mm, sc->dev, sizeof mm, cudaMemcpyDeviceToHost, st));
	MM_CUDA(cudaStreamSynchronize(st));
	double lo, hi;
	std::memcpy(&lo, &mm[0], 8);
	std::memcpy(&hi, &mm[1], 8);
	double scale = 1.0;
	if (!std::getenv("MAGNUM_OMF_NOSCALE") && hi > 0.001) {
		scale /= hi;
		hi *= scale;
		lo *= scale;
	}
	h->valuemultiplier = 1.0 / scale;
	h->ValueRangeMaxMag = hi;
	h->ValueRangeMinMag = lo;
	auto line = [&](const char *k, const std::string &v) {
		out += "# ";
		out += k;
		out += ": ";
		out += v;
		out += '\n';
	};
	line("OOMMF", "rectangular mesh v1.0");
	line("Segment count", "1");
	line("Begin", "Segment");
	line("Begin", "Header");
	line("Title", h->title);
	{
		std::string d(h->desc), part;
		std::stringstream ss(d);
		while (!d.empty() && std::getline(ss, part)) line("Desc", part);
	}
	line("meshunit", h->meshunit);
	line("valueunit", h->valueunit);
	line("valuemultiplier", g16(h->valuemultiplier));
	line("xmin", g16(h->xmin));
	line("ymin", g16(h->ymin));
	line("zmin", g16(h->zmin));
	line("xmax", g16(h->xmax));
	line("ymax", g16(h->ymax));
	line("zmax", g16(h->zmax));
	line("ValueRangeMaxMag", g16(hi));
	line("ValueRangeMinMag", g16(lo));
	line("meshtype", h->meshtype);
	line("xbase", g16(h->xbase));
	line("ybase", g16(h->ybase));
	line("zbase", g16(h->zbase));
	line("xstepsize", g16(h->xstepsize));
	line("ystepsize", g16(h->ystepsize));
	line("zstepsize", g16(h->zstepsize));
	line("xnodes", std::to_string(h->xnodes));
	line("ynodes", std::to_string(h->ynodes));
	line("znodes", std::to_string(h->znodes));
	line("End", "Header");
	const char *tag = format == MM_OMF_TEXT ? "Data Text" : format == MM_OMF_BINARY_4 ? "Data Binary 4" : "Data Binary 8";
	line("Begin", tag);
	if (format == MM_OMF_BINARY_4) {
		const unsigned char magic[4] = {0x49, 0x96, 0xb4, 0x38};  // 1234567.0f, big-endian
		out.append((const char *)magic, 4);
	} else if (format == MM_OMF_BINARY_8) {
		const unsigned char magic[8] = {0x42, 0xdc, 0x12, 0x21, 0x83, 0x77, 0xde, 0x40};  // 123456789012345.0
		out.append((const char *)magic, 8);
	}
	MM_TRY(payload<T>(M, n, format, scale, out, st));
	line("End", tag);
	line("End", "Segment");
	return MM_OK;
}

mm_status read_file(const char *path, std::string &data)
{
	std::ifstream in(path, std::ios::binary);
	if (!in.good()) return fail(MM_ERR_INVALID_ARGUMENT, std::string("OMF: could not open file: ") + path);
	std::stringstream ss;
	ss << in.rdbuf();
	data = ss.str();
	return MM_OK;
}

bool bad_format(int f) { return f != MM_OMF_TEXT && f != MM_OMF_BINARY_4 && f != MM_OMF_BINARY_8; }

} // namespace
} // namespace mm

using namespace mm;

extern "C" {

MM_API mm_status mm_omf_parse(const void *bytes_host, size_t length, mm_omf_header *header, int prec, void *M,
                              void *stream)
{
	if (!bytes_host || !header) return fail(MM_ERR_INVALID_ARGUMENT, "mm_omf_parse: null argument");
	return parse((const char *)bytes_host, length, header, prec, M, as_stream(stream));
}

MM_API mm_status mm_omf_read(const char *path, mm_omf_header *header, int prec, void *M, void *stream)
{
	if (!path || !header) return fail(MM_ERR_INVALID_ARGUMENT, "mm_omf_read: null argument");
	std::string data;
	MM_TRY(read_file(path, data));
	return parse(data.data(), data.size(), header, prec, M, as_stream(stream));
}

MM_API mm_status mm_omf_format(mm_omf_header *header, int prec, const void *M, int format, char **bytes_host,
                               size_t *length, void *stream)
{
	if (!header || !M || !bytes_host || !length || bad_format(format) || (prec != MM_F64 && prec != MM_F32))
		return fail(MM_ERR_INVALID_ARGUMENT, "mm_omf_format: invalid argument");
	std::string out;
	MM_TRY(prec == MM_F64 ? format_omf<double>(header, (const double *)M, format, out, as_stream(stream))
	                      : format_omf<float>(header, (const float *)M, format, out, as_stream(stream)));
	char *buf = (char *)std::malloc(out.size() ? out.size() : 1);
	if (!buf) return fail(MM_ERR_OUT_OF_MEMORY, "mm_omf_format: host allocation failed");
	std::memcpy(buf, out.data(), out.size());
	*bytes_host = buf;
	*length = out.size();
	return MM_OK;
}

MM_API void mm_omf_free(char *bytes_host) { std::free(bytes_host); }

MM_API mm_status mm_omf_write(const char *path, mm_omf_header *header, int prec, const void *M, int format,
                              void *stream)
{
	if (!path) return fail(MM_ERR_INVALID_ARGUMENT, "mm_omf_write: null path");
	char *buf = nullptr;
	size_t len = 0;
	MM_TRY(mm_omf_format(header, prec, M, format, &buf, &len, stream));
	std::ofstream out(path, std::ios::binary);
	if (!out.good()) {
		std::free(buf);
		return fail(MM_ERR_INVALID_ARGUMENT, std::string("mm_omf_write: could not open ") + path + " for writing");
	}
	out.write(buf, (std::streamsize)len);
	std::free(buf);
	if (!out.good()) return fail(MM_ERR_CUDA, std::string("mm_omf_write: write to ") + path + " failed");
	return MM_OK;
}

} // extern "C"
