// gdn_cuda_error_l2_noalloc: the FP64 L2 error norm of an RK3 state for
// callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: hosts whose device
// memory is owned by another allocator or by a fixed budget set at start-up,
// and long-running services that must not allocate after initialisation.
// They already hold their inputs and outputs; what they cannot provide is the
// library's own scratch.  This entry point keeps that scratch in a
// fixed-size array that lives in the library's device image: every GPU that
// loads the library holds it (about 192 KB) until the process exits.
//
// Limits and rules:
//   - at most kMaxBlocks x kBlockElems = 8,388,608 elements per call; larger
//     meshes are rejected with GDN_CUDA_ERR_INVALID;
//   - every call shares the one array per device and it keeps the last
//     call's contents (each call overwrites every slot it reads, so nothing
//     needs clearing): calls that overlap on the GPU (two streams, two host
//     threads) race and must be serialised by the caller;
//   - the call synchronises its stream before it returns, so the result is
//     in the caller's host variable on return;
//   - the first call on a device (that device current, in its primary
//     context) looks up the array's device address there and keeps it: make
//     that first call before any stream capture begins; the kept address does
//     not survive cudaDeviceReset.
#include <atomic>
#include <cstdio>

#include "common.cuh"

namespace gdn {

constexpr int kNoAllocBlockElems = 2048; // elements per partial sum
constexpr int kNoAllocMaxBlocks = 4096; // => 8,388,608 elements at most
constexpr int kNoAllocThreads = 256;

struct WpgParam {
	double v[10]; // nodal quadrature weights, passed by value
};

// [kNoAllocMaxBlocks][6] per-block partial sums, then [8] results
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxBlocks * 6 + 8];

// Block b sums elements [b * kNoAllocBlockElems, ...) in a fixed order, so
// the result does not depend on how many blocks run.
__global__ void __launch_bounds__(kNoAllocThreads)
	noalloc_error_partial(const double *__restrict__ w, const double *__restrict__ xyz,
						  const double *__restrict__ det, long long ne, Data d, double t, WpgParam wpg,
						  double *__restrict__ scratch)
{
	__shared__ double red[6][kNoAllocThreads];
	double acc[6] = {0, 0, 0, 0, 0, 0};
	const long long e_begin = (long long)blockIdx.x * kNoAllocBlockElems;
	const long long e_end = min(ne, e_begin + kNoAllocBlockElems);
	for (long long u = e_begin * 10 + threadIdx.x; u < e_end * 10; u += kNoAllocThreads) {
		const long long e = u / 10;
		const int i = (int)(u % 10);
		const double x[3] = {xyz[3 * u], xyz[3 * u + 1], xyz[3 * u + 2]};
		double we[6];
		exact_w(d, x, t, we);
		const double de = det[e];
		for (int c = 0; c < 6; c++) {
			const double diff = w[u * 6 + c] - we[c];
			acc[c] += diff * diff * wpg.v[i] * de;
		}
	}
	for (int c = 0; c < 6; c++)
		red[c][threadIdx.x] = acc[c];
	__syncthreads();
	for (int s = kNoAllocThreads / 2; s > 0; s >>= 1) {
		if ((int)threadIdx.x < s)
			for (int c = 0; c < 6; c++)
				red[c][threadIdx.x] += red[c][threadIdx.x + s];
		__syncthreads();
	}
	if (threadIdx.x == 0)
		for (int c = 0; c < 6; c++)
			scratch[blockIdx.x * 6 + c] = red[c][0];
}

__global__ void __launch_bounds__(kNoAllocThreads) noalloc_error_final(int nblk, double *__restrict__ scratch)
{
	__shared__ double red[6][kNoAllocThreads];
	double acc[6] = {0, 0, 0, 0, 0, 0};
	for (int b = threadIdx.x; b < nblk; b += kNoAllocThreads)
		for (int c = 0; c < 6; c++)
			acc[c] += scratch[b * 6 + c];
	for (int c = 0; c < 6; c++)
		red[c][threadIdx.x] = acc[c];
	__syncthreads();
	for (int s = kNoAllocThreads / 2; s > 0; s >>= 1) {
		if ((int)threadIdx.x < s)
			for (int c = 0; c < 6; c++)
				red[c][threadIdx.x] += red[c][threadIdx.x + s];
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		double* out = scratch + kNoAllocMaxBlocks * 6;
		double e = 0.0;
		for (int c = 0; c < 6; c++) {
			out[1 + c] = red[c][0];
			e += sqrt(fabs(red[c][0])) / 6.0;
		}
		out[0] = e;
	}
}

// device address of g_noalloc_scratch, looked up once per device (atomic:
// first calls from several host threads may race to fill a slot, and each
// stores the same address)
static std::atomic<void *> g_noalloc_ptr[256];

} // namespace gdn

using namespace gdn;

extern "C" int gdn_cuda_error_l2_noalloc(const double *w, const double *xyz, const double *det, long long nbelems,
										 const double *wpg, const gdn_cuda_data *data, double t, void *stream,
										 double *err)
{
	if (!w || !xyz || !det || !wpg || !data || !err || nbelems <= 0)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "error_l2_noalloc: bad arguments");
	if (nbelems > (long long)kNoAllocMaxBlocks * kNoAllocBlockElems) {
		char buf[200];
		std::snprintf(buf, sizeof(buf),
					  "error_l2_noalloc: %lld elements exceed the fixed scratch limit of %lld elements",
					  nbelems, (long long)kNoAllocMaxBlocks * kNoAllocBlockElems);
		return gdn_set_error(GDN_CUDA_ERR_INVALID, buf);
	}
	if (data->kind != GDN_CUDA_DATA_PLANE && data->kind != GDN_CUDA_DATA_CAVITY &&
		data->kind != GDN_CUDA_DATA_STATIONARY)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "error_l2_noalloc: unknown analytic data kind");
	int dev = 0;
	GDN_CUDA_TRY(cudaGetDevice(&dev));
	if (dev < 0 || dev >= 256)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "error_l2_noalloc: device ordinal out of range");
	void *cached = g_noalloc_ptr[dev].load(std::memory_order_acquire);
	if (!cached) {
		void *ptr = nullptr;
		cudaError_t rc = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
		if (rc != cudaSuccess || !ptr)
			return gdn_cuda_fail(rc, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
		g_noalloc_ptr[dev].store(ptr, std::memory_order_release);
		cached = ptr;
	}
	double *scratch = static_cast<double *>(cached);
	Data d;
	d.kind = data->kind;
	for (int c = 0; c < 3; c++) {
		d.khat[c] = data->khat[c];
		d.pol[c] = data->pol[c];
	}
	d.kmag = data->kmag;
	d.amp = data->amp;
	d.phase = data->phase;
	WpgParam wp;
	for (int i = 0; i < 10; i++)
		wp.v[i] = wpg[i];
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	const int nblk = (int)((nbelems + kNoAllocBlockElems - 1) / kNoAllocBlockElems);
	noalloc_error_partial<<<nblk, kNoAllocThreads, 0, s>>>(w, xyz, det, nbelems, d, t, wp, scratch);
	GDN_CUDA_TRY(cudaGetLastError());
	noalloc_error_final<<<1, kNoAllocThreads, 0, s>>>(nblk, scratch);
	GDN_CUDA_TRY(cudaGetLastError());
	GDN_CUDA_TRY(cudaMemcpyAsync(err, scratch + kNoAllocMaxBlocks * 6, sizeof(double), cudaMemcpyDeviceToHost, s));
	GDN_CUDA_TRY(cudaStreamSynchronize(s));
	return GDN_CUDA_OK;
}
