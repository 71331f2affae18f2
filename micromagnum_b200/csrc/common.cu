// Library-wide state: per-thread error message, launch counter, SM count, scalar scratch.
#include "mm_common.cuh"

#include <mutex>
#include <vector>

namespace mm {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }

std::atomic<uint64_t> &launch_counter()
{
	static std::atomic<uint64_t> c{0};
	return c;
}

int num_sms()
{
	int dev = 0, n = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) return 148;
	if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
	return n > 0 ? n : 148;
}

// One scratch slot per device, created on first use and kept until process exit.  It holds the
// accumulators of reductions whose result is returned to the host (energies, maxima).
std::mutex &capture_mutex()
{
	static std::mutex mu;
	return mu;
}

mm_status scalar_scratch(ScalarScratch **out)
{
	static std::mutex mu;
	static std::vector<ScalarScratch> slots;
	int dev = 0;
	MM_CUDA(cudaGetDevice(&dev));
	std::lock_guard<std::mutex> lock(mu);
	if ((int)slots.size() <= dev) slots.resize(dev + 1);
	ScalarScratch &s = slots[dev];
	if (!s.dev) {
		MM_CUDA(cudaMalloc(&s.dev, 8 * sizeof(double)));
		MM_CUDA(cudaMallocHost(&s.host, 8 * sizeof(double)));
	}
	*out = &s;
	return MM_OK;
}

// ---- profiler ------------------------------------------------------------------------------------
namespace {
struct ProfRecord {
	std::string name;
	double bytes;
	cudaEvent_t start, stop;
};
struct ProfTotals {
	std::string name;
	int64_t launches = 0;
	double total_ms = 0.0;
	double bytes = 0.0;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRecord> g_prof_pending;
std::vector<ProfTotals> g_prof_totals;
std::vector<cudaEvent_t> g_event_pool;

cudaEvent_t take_event()
{
	if (!g_event_pool.empty()) {
		cudaEvent_t e = g_event_pool.back();
		g_event_pool.pop_back();
		return e;
	}
	cudaEvent_t e = nullptr;
	cudaEventCreate(&e);
	return e;
}

void drain_pending()
{
	for (ProfRecord &r : g_prof_pending) {
		float ms = 0.f;
		cudaEventSynchronize(r.stop);
		cudaEventElapsedTime(&ms, r.start, r.stop);
		ProfTotals *t = nullptr;
		for (ProfTotals &x : g_prof_totals)
			if (x.name == r.name) t = &x;
		if (!t) {
			g_prof_totals.push_back(ProfTotals{r.name});
			t = &g_prof_totals.back();
		}
		t->launches++;
		t->total_ms += ms;
		t->bytes += r.bytes;
		g_event_pool.push_back(r.start);
		g_event_pool.push_back(r.stop);
	}
	g_prof_pending.clear();
}
} // namespace

bool profiling_on() { return g_prof_on; }

ProfToken prof_begin(cudaStream_t st)
{
	ProfToken t;
	if (!g_prof_on) return t;
	std::lock_guard<std::mutex> lock(g_prof_mu);
	t.start = take_event();
	cudaEventRecord(t.start, st);
	return t;
}

void prof_end(ProfToken tok, const char *name, double bytes, cudaStream_t st)
{
	if (!g_prof_on || !tok.start) return;
	std::lock_guard<std::mutex> lock(g_prof_mu);
	cudaEvent_t stop = take_event();
	cudaEventRecord(stop, st);
	g_prof_pending.push_back(ProfRecord{name, bytes, tok.start, stop});
	if (g_prof_pending.size() > 4096) drain_pending();
}

} // namespace mm

extern "C" {

MM_API mm_status mm_profile_enable(int on)
{
	std::lock_guard<std::mutex> lock(mm::g_prof_mu);
	mm::g_prof_on = on != 0;
	return MM_OK;
}

MM_API mm_status mm_profile_reset(void)
{
	std::lock_guard<std::mutex> lock(mm::g_prof_mu);
	mm::drain_pending();
	mm::g_prof_totals.clear();
	return MM_OK;
}

MM_API int mm_profile_count(void)
{
	std::lock_guard<std::mutex> lock(mm::g_prof_mu);
	mm::drain_pending();
	return (int)mm::g_prof_totals.size();
}

MM_API mm_status mm_profile_get(int index, const char **name, int64_t *launches, double *total_ms,
                                double *bytes)
{
	std::lock_guard<std::mutex> lock(mm::g_prof_mu);
	mm::drain_pending();
	if (index < 0 || index >= (int)mm::g_prof_totals.size())
		return mm::fail(MM_ERR_INVALID_ARGUMENT, "mm_profile_get: index out of range");
	const auto &t = mm::g_prof_totals[index];
	if (name) *name = t.name.c_str();
	if (launches) *launches = t.launches;
	if (total_ms) *total_ms = t.total_ms;
	if (bytes) *bytes = t.bytes;
	return MM_OK;
}

MM_API const char *mm_last_error(void) { return mm::g_last_error.c_str(); }
MM_API int mm_abi_version(void) { return MM_ABI_VERSION; }
MM_API uint64_t mm_kernel_launch_count(void) { return mm::launch_counter().load(); }

} // extern "C"
