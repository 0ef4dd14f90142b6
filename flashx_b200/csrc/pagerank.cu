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
// One iteration is the SpMV (fmx_spmm on the transpose, k = 1) and one fused
// kernel that applies the damping, counts the converged vertices and writes
// the next iteration's input (pr / deg and its in * deg reconstruction).
#include "fmx_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

namespace fmx {
namespace pagerank {

constexpr int kThreads = 256;

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

// pr2 = out * d + t; count |pr1 - pr2| < eps; pr = pr2; in = pr2 / deg;
// pr1 = in * deg (the next iteration's reconstruction)
__global__ void __launch_bounds__(kThreads) update_kernel(const float *__restrict__ out, const float *__restrict__ deg,
		float *__restrict__ pr, float *__restrict__ in, float *__restrict__ pr1, int64_t n, float damping,
		float teleport, float eps, unsigned long long *__restrict__ converged)
{
	__shared__ unsigned int red[kThreads / 32];
	unsigned int cnt = 0;
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
		const float p2 = __fadd_rn(__fmul_rn(out[i], damping), teleport);
		const float diff = fabsf(__fsub_rn(pr1[i], p2));
		cnt += diff < eps;
		pr[i] = p2;
		const float d = deg[i];
		const float x = __fdiv_rn(p2, d);
		in[i] = x;
		pr1[i] = __fmul_rn(x, d);
	}
	for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cnt;
	__syncthreads();
	if (threadIdx.x == 0) {
		unsigned long long s = 0;
		for (int w = 0; w < kThreads / 32; w++) s += red[w];
		atomicAdd(converged, s);
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
	float *deg, *in, *pr1, *out, *ones;
	unsigned long long *conv;
	for (float **b : {&deg, &in, &pr1, &out, &ones}) {
		void *q = nullptr;
		cudaError_t e = cudaMallocAsync(&q, size_t(std::max<int64_t>(n, 1)) * sizeof(float), st);
		if (e != cudaSuccess) return set_error(FMX_ERR_OOM, "PageRank vectors: %s", cudaGetErrorString(e));
		g.bufs.push_back(q);
		*b = static_cast<float *>(q);
	}
	{
		void *q = nullptr;
		PCUDA_TRY(cudaMallocAsync(&q, sizeof(unsigned long long), st));
		g.bufs.push_back(q);
		conv = static_cast<unsigned long long *>(q);
	}
	// the convergence count comes back through one pinned word per host thread
	static thread_local unsigned long long *hconv = nullptr;
	if (!hconv) PCUDA_TRY(cudaMallocHost(&hconv, sizeof(unsigned long long)));
	const unsigned gb = grid_for(n);
	fill_kernel<<<gb, kThreads, 0, st>>>(ones, n, 1.0f);
	PCUDA_TRY(cudaGetLastError());
	P_TRY(fmx_spmm(m, FMX_F32, ones, 1, FMX_F32, deg, 1, 1, nullptr, nullptr, st));
	const float p0 = float(1.0 / double(n));
	const float eps = float(0.001 / double(n));
	const float teleport = float((1.0 - double(damping)) / double(n));
	init_kernel<<<gb, kThreads, 0, st>>>(deg, pr, in, pr1, n, p0);
	PCUDA_TRY(cudaGetLastError());
	uint64_t it = 0, converged = 0;
	while (converged < uint64_t(n) && it < max_iters) {
		PCUDA_TRY(cudaMemsetAsync(conv, 0, sizeof(unsigned long long), st));
		P_TRY(fmx_spmm(mt, FMX_F32, in, 1, FMX_F32, out, 1, 1, nullptr, nullptr, st));
		update_kernel<<<gb, kThreads, 0, st>>>(out, deg, pr, in, pr1, n, damping, teleport, eps, conv);
		PCUDA_TRY(cudaGetLastError());
		PCUDA_TRY(cudaMemcpyAsync(hconv, conv, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
		PCUDA_TRY(cudaStreamSynchronize(st));
		converged = *hconv;
		it++;
	}
	if (iters) *iters = it;
	return FMX_OK;
}

} // extern "C"
