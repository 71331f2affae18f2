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

} // namespace mm

extern "C" {

MM_API const char *mm_last_error(void) { return mm::g_last_error.c_str(); }
MM_API int mm_abi_version(void) { return MM_ABI_VERSION; }
MM_API uint64_t mm_kernel_launch_count(void) { return mm::launch_counter().load(); }

} // extern "C"
