// PageRank on the GPU: fm::alg::PageRank (matrix/libmatrix-algs/
// PageRank.cpp:63-133) with the same float arithmetic, so that every vertex
// whose in-degree row is summed in the reference's order (at most
// FMX_EXACT_ROW_MAX entries) follows it bit for bit.
//
//   deg  = max(A 1, 1)                                (:49-59, :75)
//   pr   = 1.0 / n  (double, stored as float)         (:31-47, :80)
//   loop while converged < n and iters < max_iters    (:96-130):
//     in  = pr / deg;  pr1 = in * deg                 (:100-104)
//     out = A^T in                                    (:108, the transpose, :92)
//     pr2 = out * d + (1 - d) / n                     (:116-117, two roundings)
//     converged = #{ |pr1 - pr2| < 0.001 / n }        (:94, :118-123)
//     pr  = pr2
//
// One iteration is one pass: the SpMV on the transpose (k = 1) applies the
// damping, counts the converged vertices and writes the next input where it
// closes each row (rows summed in chunks get the same update in the fixup
// kernel), and a one-thread kernel runs the loop test on the device.  The
// input is double-buffered (other rows still gather this iteration's input
// while the next one is written).  Iterations are queued in batches with one
// host read of the loop state per batch; an iteration queued after the loop
// ended returns at once, so the result and the count match a loop that
// tests on the host after every iteration.
#include "fmx_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

namespace fmx {
namespace pagerank {

constexpr int kThreads = 256;
constexpr uint64_t kBatch = 8;          // iterations queued per host read of the loop state

#define PCUDA_TRY(call)                                                         \
	do {                                                                        \
		cudaError_t err__ = (call);                                             \
		if (err__ != cudaSuccess)                                               \
			return set_error(FMX_ERR_CUDA, "%s failed: %s (%s:%d)", #call,      \
					cudaGetErrorString(err__), __FILE__, __LINE__);             \
	} while (0)
#define P_TRY(call)                                                             \
	do {                                                                        \
		int rc__ = (call);                                                      \
		if (rc__ != FMX_OK) return rc__;                                        \
	} while (0)

__global__ void fill_kernel(float *p, int64_t n, float v)
{
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) p[i] = v;
}

// deg = max(deg, 1); pr = p0; in = pr / deg; pr1 = in * deg
__global__ void init_kernel(float *__restrict__ deg, float *__restrict__ pr, float *__restrict__ in,
		float *__restrict__ pr1, int64_t n, float p0)
{
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
		const float d = fmaxf(deg[i], 1.0f);
		deg[i] = d;
		pr[i] = p0;
		const float x = __fdiv_rn(p0, d);
		in[i] = x;
		pr1[i] = __fmul_rn(x, d);
	}
}

unsigned grid_for(int64_t n)
{
	int dev = 0, sms = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	return unsigned(std::max<int64_t>(1, std::min<int64_t>((n + kThreads - 1) / kThreads, int64_t(std::max(sms, 1)) * 8)));
}

} // namespace pagerank
} // namespace fmx

using namespace fmx;
using namespace fmx::pagerank;

extern "C" {

int fmx_pagerank(const fmx_matrix *m, uint64_t max_iters, float damping, float *pr, uint64_t *iters, void *stream)
{
	if (!m || !pr) return set_error(FMX_ERR_INVAL, "null argument");
	device_guard on_device(matrix_device(m));    // before the buffers: freed on the matrix's device
	if (!on_device.ok()) return set_error(FMX_ERR_CUDA, "cannot make the matrix's device %d current", matrix_device(m));
	uint64_t nr = 0, nc = 0, nz = 0;
	int prim = 0;
	P_TRY(fmx_matrix_info(m, &nr, &nc, &nz, &prim, nullptr));
	if (nr != nc) return set_error(FMX_ERR_DIM, "PageRank needs a square matrix");
	if (prim != FMX_P_BOOL && prim != FMX_P_FLOAT) return set_error(FMX_ERR_TYPE, "binary or float-weighted matrices");
	fmx_matrix *mt = nullptr;
	P_TRY(fmx_matrix_transpose(m, &mt));
	struct guard {
		fmx_matrix *t;
		cudaStream_t st;
		std::vector<void *> bufs;
		~guard()
		{
			for (void *p : bufs) cudaFreeAsync(p, st);
			fmx_matrix_free(t);
		}
	} g{mt, static_cast<cudaStream_t>(stream), {}};
	cudaStream_t st = g.st;
	const int64_t n = int64_t(nr);
	float *deg, *in0, *in1, *pr1;
	uint32_t *mask;
	unsigned long long *state;
	auto alloc = [&](void **q, size_t bytes) -> int {
		cudaError_t e = work_alloc(q, std::max<size_t>(bytes, 16), st);
		if (e != cudaSuccess) return set_error(FMX_ERR_OOM, "PageRank vectors: %s", cudaGetErrorString(e));
		g.bufs.push_back(*q);
		return FMX_OK;
	};
	const size_t mask_words = size_t((n + 31) / 32);
	for (float **b : {&deg, &in0, &in1, &pr1}) P_TRY(alloc(reinterpret_cast<void **>(b), size_t(n) * sizeof(float)));
	P_TRY(alloc(reinterpret_cast<void **>(&mask), mask_words * sizeof(uint32_t)));
	P_TRY(alloc(reinterpret_cast<void **>(&state), 3 * sizeof(unsigned long long)));
	// the loop state comes back through three pinned words per host thread
	static thread_local unsigned long long *hstate = nullptr;
	if (!hstate) PCUDA_TRY(cudaMallocHost(&hstate, 3 * sizeof(unsigned long long)));
	const unsigned gb = grid_for(n);
	fill_kernel<<<gb, kThreads, 0, st>>>(in1, n, 1.0f);
	PCUDA_TRY(cudaGetLastError());
	P_TRY(fmx_spmm(m, FMX_F32, in1, 1, FMX_F32, deg, 1, 1, nullptr, nullptr, st));
	const float p0 = float(1.0 / double(n));
	pr_epi e{};
	e.deg = deg;
	e.heavy_mask = mask;
	e.pr = pr;
	e.pr1 = pr1;
	e.state = state;
	e.damping = damping;
	e.teleport = float((1.0 - double(damping)) / double(n));
	e.eps = float(0.001 / double(n));
	e.n = uint64_t(n);
	e.max_iters = max_iters;
	init_kernel<<<gb, kThreads, 0, st>>>(deg, pr, in0, pr1, n, p0);
	PCUDA_TRY(cudaGetLastError());
	PCUDA_TRY(cudaMemsetAsync(mask, 0, mask_words * sizeof(uint32_t), st));
	PCUDA_TRY(cudaMemsetAsync(state, 0, 3 * sizeof(unsigned long long), st));
	P_TRY(pagerank_heavy_mask(mt, mask, st));
	uint64_t it = 0, queued = 0;
	while (n > 0 && queued < max_iters) {
		const uint64_t batch = std::min<uint64_t>(kBatch, max_iters - queued);
		for (uint64_t b = 0; b < batch; b++, queued++) {
			const float *in = (queued & 1) ? in1 : in0;
			e.in_next = (queued & 1) ? in0 : in1;
			P_TRY(pagerank_iteration(mt, in, e, st));
		}
		PCUDA_TRY(cudaMemcpyAsync(hstate, state, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
		PCUDA_TRY(cudaStreamSynchronize(st));
		it = hstate[2];
		if (hstate[1]) break;
	}
	if (iters) *iters = it;
	return FMX_OK;
}

} // extern "C"
