// Learned warm start for the block eigensolver: a 2-layer graph network that
// maps vertex features to a 16-column start block.  It has no counterpart in
// the reference; it feeds fmx_eigen_solve's X0.
//
//   F  (n x 16)   standardised log(1 + degree) (the degree read back from the
//                 D^-1/2 scale), then 15 N(0,1) channels
//   Z  (n x 64)   [F, A_s F, A_s^2 F, A_s^3 F]      (A_s = D^-1/2 A D^-1/2)
//   H  (n x 64)   relu(Z W1 + b1)                   layer 1, hidden 64
//   Y  (n x 16)   A_s (H W2)                        layer 2
//   loss          1 - ||U^T Q||_F^2 / nev,  Q an orthonormal basis of span(Y),
//                 U the solver's nev eigenvectors (orthonormal columns)
//
// Every propagation is the library's SpMM (fmx_spmm with the D^-1/2 row
// scales fused); the products with W1, W2 and the weight gradients run on
// the tcgen05 tensor-core kernels (fmx_dense_gemm / fmx_dense_gram) with BF16
// operands and FP32 accumulation (3xTF32 for gradient checks).  The weights
// are kept in FP32 for the optimiser (Adam) and enter every product as BF16.
//
// Gradient of the loss (G = Y^T Y, M = U^T Y, f = tr(M G^-1 M^T)):
//   dL/dY = -(2 / nev) (I - Y G^-1 Y^T) U M G^-1 = U P1 + Y P2,
//   P1 = -(2 / nev) M G^-1,   P2 = (2 / nev) G^-1 M^T M G^-1.
// Backward: dZ2 = A_s dY (A_s symmetric), dW2 = H^T dZ2, dH = dZ2 W2^T masked
// by H > 0, db1 = column sums of dH, dW1 = Z^T dH.
#include "fmx_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

namespace fmx {
namespace gnn {

constexpr int kF = 16;                    // input channels
constexpr int kHops = 3;                  // propagations of the input
constexpr int kZ = kF * (kHops + 1);      // layer-1 inputs (64)
constexpr int kH = 64;                    // hidden width
constexpr int kOut = FMX_GNN_OUT;         // output columns (16)
constexpr int kMaxNev = 64;
constexpr int kThreads = 256;
// flat parameter layout: W1 (kZ x kH, row-major), b1 (kH), W2 (kH x kOut)
constexpr int kOffW1 = 0, kOffB1 = kZ * kH, kOffW2 = kZ * kH + kH;
constexpr int kParams = kZ * kH + kH + kH * kOut;
static_assert(kParams == FMX_GNN_PARAMS, "parameter count");
static_assert(kZ == FMX_GNN_FEATURES, "feature width");

#define GCUDA_TRY(call)                                                         \
	do {                                                                        \
		cudaError_t err__ = (call);                                             \
		if (err__ != cudaSuccess)                                               \
			return set_error(FMX_ERR_CUDA, "%s failed: %s (%s:%d)", #call,      \
					cudaGetErrorString(err__), __FILE__, __LINE__);             \
	} while (0)
#define G_TRY(call)                                                             \
	do {                                                                        \
		int rc__ = (call);                                                      \
		if (rc__ != FMX_OK) return rc__;                                        \
	} while (0)

// splitmix64 finaliser (Steele, Lea, Flood 2014)
__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
	z += 0x9E3779B97F4A7C15ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}


// log(1 + degree) of a row from its D^-1/2 scale s (0 for an empty row):
// degree = 1 / s^2, within a few ulps of the row sum the scale came from
__device__ __forceinline__ float log_degree(float s) { return s > 0.f ? log1pf(1.f / (s * s)) : 0.f; }

// per-CTA sum and sum of squares of log(1 + degree) over the rows (FP64)
__global__ void __launch_bounds__(kThreads) logdeg_stats_kernel(const float *__restrict__ scale, int64_t n,
		double *__restrict__ part)
{
	__shared__ double s1[kThreads], s2[kThreads];
	double a = 0, c = 0;
	for (int64_t i = blockIdx.x * int64_t(kThreads) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kThreads) {
		const double v = log_degree(scale[i]);
		a += v;
		c += v * v;
	}
	s1[threadIdx.x] = a;
	s2[threadIdx.x] = c;
	__syncthreads();
	for (int w = kThreads / 2; w > 0; w >>= 1) {
		if (threadIdx.x < w) {
			s1[threadIdx.x] += s1[threadIdx.x + w];
			s2[threadIdx.x] += s2[threadIdx.x + w];
		}
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		part[2 * blockIdx.x] = s1[0];
		part[2 * blockIdx.x + 1] = s2[0];
	}
}

// F = Z[:, 0:16], a thread per row: channel 0 the standardised log-degree,
// channels 1..15 N(0, 1), pairs of them by the Box-Muller transform of two
// counter-based uniforms (cos and sin of the same pair)
__global__ void features_kernel(const float *__restrict__ scale, int64_t n, const double *__restrict__ part,
		int nparts, uint64_t seed, float *__restrict__ Z)
{
	__shared__ float mean, inv_std;
	if (threadIdx.x == 0) {
		double a = 0, c = 0;
		for (int p = 0; p < nparts; p++) {
			a += part[2 * p];
			c += part[2 * p + 1];
		}
		const double m = a / double(n > 0 ? n : 1);
		const double var = c / double(n > 0 ? n : 1) - m * m;
		mean = float(m);
		inv_std = float(var > 1e-20 ? 1.0 / sqrt(var) : 1.0);
	}
	__syncthreads();
	for (int64_t row = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; row < n; row += int64_t(gridDim.x) * blockDim.x) {
		float f[kF];
		f[0] = (log_degree(scale[row]) - mean) * inv_std;
#pragma unroll
		for (int q = 0; q < kF / 2; q++) {
			const uint64_t key = seed * 0x9E3779B97F4A7C15ull ^ (uint64_t(row) * kF + uint64_t(q));
			const uint64_t z = mix64(key);
			const float u1 = (float(uint32_t(z) >> 8) + 1.f) * (1.f / 16777216.f);     // (0, 1]
			const float u2 = float(uint32_t(z >> 32) >> 8) * (1.f / 16777216.f);       // [0, 1)
			const float r = sqrtf(-2.f * logf(u1));
			float sn, cs;
			sincospif(2.f * u2, &sn, &cs);
			if (2 * q + 1 < kF) f[2 * q + 1] = r * cs;
			if (2 * q + 2 < kF) f[2 * q + 2] = r * sn;
		}
		float4 *o = reinterpret_cast<float4 *>(Z + row * kZ);
#pragma unroll
		for (int v = 0; v < kF / 4; v++) o[v] = make_float4(f[4 * v], f[4 * v + 1], f[4 * v + 2], f[4 * v + 3]);
	}
}

// H = relu(H + b1) in place (n x kH, 16-byte vectors)
__global__ void bias_relu_kernel(float4 *__restrict__ H, const float4 *__restrict__ b1, int64_t n)
{
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n * (kH / 4); i += int64_t(gridDim.x) * blockDim.x) {
		const float4 b = b1[uint32_t(i) % uint32_t(kH / 4)];
		float4 h = H[i];
		h.x = fmaxf(h.x + b.x, 0.f); h.y = fmaxf(h.y + b.y, 0.f);
		h.z = fmaxf(h.z + b.z, 0.f); h.w = fmaxf(h.w + b.w, 0.f);
		H[i] = h;
	}
}

// dH *= (H > 0) in place; part[cta][j] = the CTA's column sums of the masked
// dH (db1), added in a fixed order per thread and over the CTA
__global__ void __launch_bounds__(kThreads) relu_grad_kernel(float *__restrict__ dH, const float *__restrict__ H,
		int64_t n, float *__restrict__ part)
{
	__shared__ float red[kThreads];
	const int col = threadIdx.x % kH, lane_row = threadIdx.x / kH;        // kThreads / kH = 4 rows per step
	float acc = 0.f;
	for (int64_t row = int64_t(blockIdx.x) * (kThreads / kH) + lane_row; row < n;
			row += int64_t(gridDim.x) * (kThreads / kH)) {
		const int64_t i = row * kH + col;
		const float g = H[i] > 0.f ? dH[i] : 0.f;
		dH[i] = g;
		acc += g;
	}
	red[threadIdx.x] = acc;
	__syncthreads();
	if (threadIdx.x < kH) {
		float s = 0.f;
		for (int r = 0; r < kThreads / kH; r++) s += red[r * kH + threadIdx.x];
		part[size_t(blockIdx.x) * kH + threadIdx.x] = s;
	}
}

__global__ void sum_parts_kernel(const float *__restrict__ part, int nparts, int len, float *__restrict__ out)
{
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x) {
		float s = 0.f;
		for (int p = 0; p < nparts; p++) s += part[size_t(p) * len + i];
		out[i] = s;
	}
}

// out (cols x rows) = in^T (rows x cols), small
__global__ void transpose_kernel(const float *__restrict__ in, int rows, int cols, float *__restrict__ out)
{
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows * cols; i += gridDim.x * blockDim.x) {
		const int r = i / cols, c = i % cols;
		out[c * rows + r] = in[i];
	}
}

__global__ void f32_to_f64_kernel(const float *a, double *o, int count)
{
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) o[i] = double(a[i]);
}

// Loss and the two small gradient factors, one CTA, FP64:
//   Gi = (G + shift)^-1 (Cholesky), K = M Gi (nev x 16), f = tr(K M^T),
//   P1 = -(2 / nev) K, P2 = (2 / nev) K^T K, loss = 1 - f / nev.
__global__ void __launch_bounds__(kThreads) loss_kernel(const double *__restrict__ G, const double *__restrict__ M,
		int nev, float *__restrict__ P1, float *__restrict__ P2, double *__restrict__ loss)
{
	__shared__ double R[kOut][kOut], Ri[kOut][kOut], Gi[kOut][kOut], K[kMaxNev][kOut];
	__shared__ double fred[kThreads];
	const int t = threadIdx.x;
	if (t == 0) {
		double tr = 0;
		for (int i = 0; i < kOut; i++) tr += G[i * kOut + i];
		const double shift = 1e-12 * (tr > 0 ? tr : 1.0);
		// upper Cholesky G = R^T R
		for (int k = 0; k < kOut; k++) {
			double dkk = G[k * kOut + k] + shift;
			for (int p = 0; p < k; p++) dkk -= R[p][k] * R[p][k];
			R[k][k] = sqrt(dkk > shift ? dkk : shift);
			for (int j = k + 1; j < kOut; j++) {
				double s = G[k * kOut + j];
				for (int p = 0; p < k; p++) s -= R[p][k] * R[p][j];
				R[k][j] = s / R[k][k];
			}
			for (int j = 0; j < k; j++) R[k][j] = 0;
		}
		// Ri = R^-1 (upper triangular), column by column
		for (int j = 0; j < kOut; j++)
			for (int i = kOut - 1; i >= 0; i--) {
				if (i > j) { Ri[i][j] = 0; continue; }
				double s = (i == j) ? 1.0 : 0.0;
				for (int p = i + 1; p <= j; p++) s -= R[i][p] * Ri[p][j];
				Ri[i][j] = s / R[i][i];
			}
	}
	__syncthreads();
	// Gi = Ri Ri^T
	for (int e = t; e < kOut * kOut; e += kThreads) {
		const int i = e / kOut, j = e % kOut;
		double s = 0;
		for (int p = 0; p < kOut; p++) s += Ri[i][p] * Ri[j][p];
		Gi[i][j] = s;
	}
	__syncthreads();
	// K = M Gi
	for (int e = t; e < nev * kOut; e += kThreads) {
		const int i = e / kOut, j = e % kOut;
		double s = 0;
		for (int p = 0; p < kOut; p++) s += M[i * kOut + p] * Gi[p][j];
		K[i][j] = s;
	}
	__syncthreads();
	double f = 0;
	for (int e = t; e < nev * kOut; e += kThreads) f += K[e / kOut][e % kOut] * M[e];
	fred[t] = f;
	const double sc = 2.0 / double(nev);
	for (int e = t; e < nev * kOut; e += kThreads) P1[e] = float(-sc * K[e / kOut][e % kOut]);
	for (int e = t; e < kOut * kOut; e += kThreads) {
		const int i = e / kOut, j = e % kOut;
		double s = 0;
		for (int p = 0; p < nev; p++) s += K[p][i] * K[p][j];
		P2[e] = float(sc * s);
	}
	__syncthreads();
	if (t == 0) {
		double s = 0;
		for (int i = 0; i < kThreads; i++) s += fred[i];
		*loss = 1.0 - s / double(nev);
	}
}

// dY = U P1 + Y P2 (FP32): a thread per (row, output column)
__global__ void __launch_bounds__(kThreads) dy_kernel(const float *__restrict__ U, int64_t ldu, int nev,
		const float *__restrict__ Y, const float *__restrict__ P1, const float *__restrict__ P2, int64_t n,
		float *__restrict__ dY)
{
	__shared__ float s1[kMaxNev * kOut], s2[kOut * kOut];
	for (int i = threadIdx.x; i < nev * kOut; i += kThreads) s1[i] = P1[i];
	for (int i = threadIdx.x; i < kOut * kOut; i += kThreads) s2[i] = P2[i];
	__syncthreads();
	const int j = threadIdx.x % kOut;
	for (int64_t row = int64_t(blockIdx.x) * (kThreads / kOut) + threadIdx.x / kOut; row < n;
			row += int64_t(gridDim.x) * (kThreads / kOut)) {
		float s = 0.f;
		for (int k = 0; k < nev; k++) s = fmaf(U[row * ldu + k], s1[k * kOut + j], s);
		for (int k = 0; k < kOut; k++) s = fmaf(Y[row * kOut + k], s2[k * kOut + j], s);
		dY[row * kOut + j] = s;
	}
}

// Adam (Kingma and Ba, 2015) on the flat parameter vector
__global__ void adam_kernel(float *__restrict__ p, float *__restrict__ m, float *__restrict__ v,
		const float *__restrict__ g, int count, float lr, float b1, float b2, float eps, float c1, float c2)
{
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
		const float gi = g[i];
		const float mi = b1 * m[i] + (1.f - b1) * gi;
		const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
		m[i] = mi;
		v[i] = vi;
		p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
	}
}

int sm_count()
{
	int dev = 0, s = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev);
	return s > 0 ? s : 1;
}

unsigned grid_for(int64_t count)
{
	return unsigned(std::max<int64_t>(1, std::min<int64_t>((count + kThreads - 1) / kThreads, int64_t(sm_count()) * 8)));
}

// stream-ordered device scratch of one call
struct scratch {
	cudaStream_t st = nullptr;
	std::vector<void *> bufs;
	~scratch()
	{
		for (void *p : bufs) cudaFreeAsync(p, st);
	}
	template <class T>
	int get(T **p, size_t count)
	{
		void *q = nullptr;
		cudaError_t e = work_alloc(&q, std::max<size_t>(count, 1) * sizeof(T), st);
		if (e != cudaSuccess) return set_error(FMX_ERR_OOM, "GNN scratch of %zu bytes: %s", count * sizeof(T),
				cudaGetErrorString(e));
		bufs.push_back(q);
		*p = static_cast<T *>(q);
		return FMX_OK;
	}
};

} // namespace gnn
} // namespace fmx

struct fmx_gnn {
	int device = 0;
	float *p = nullptr, *m = nullptr, *v = nullptr, *g = nullptr, *w2t = nullptr;
	int *err = nullptr;
	int64_t t = 0;
};

using namespace fmx;
using namespace fmx::gnn;

namespace {

int check_matrix(const fmx_matrix *m, int64_t *n)
{
	uint64_t nr = 0, nc = 0, nz = 0;
	int prim = 0;
	G_TRY(fmx_matrix_info(m, &nr, &nc, &nz, &prim, nullptr));
	if (nr != nc) return set_error(FMX_ERR_DIM, "the graph network needs a square matrix");
	if (prim != FMX_P_BOOL && prim != FMX_P_FLOAT) return set_error(FMX_ERR_TYPE, "binary or float-weighted matrices");
	*n = int64_t(nr);
	return FMX_OK;
}

int check_precision(int precision)
{
	if (precision != FMX_DENSE_BF16 && precision != FMX_DENSE_TF32X3)
		return set_error(FMX_ERR_INVAL, "precision: FMX_DENSE_BF16 or FMX_DENSE_TF32X3");
	return FMX_OK;
}

// H = relu(Z W1 + b1) (n x 64), Z2 = H W2 (n x 16), Y = A_s Z2 (n x 16)
int forward(const fmx_gnn *g, const fmx_matrix *m, const float *scale, const float *Z, int64_t n, int precision,
		float *H, float *Z2, float *Y, cudaStream_t st)
{
	G_TRY(fmx_dense_gemm(precision, Z, kZ, n, kZ, g->p + kOffW1, kH, kH, H, kH, g->err, st));
	bias_relu_kernel<<<grid_for(n * kH / 4), kThreads, 0, st>>>(reinterpret_cast<float4 *>(H),
			reinterpret_cast<const float4 *>(g->p + kOffB1), n);
	GCUDA_TRY(cudaGetLastError());
	G_TRY(fmx_dense_gemm(precision, H, kH, n, kH, g->p + kOffW2, kOut, kOut, Z2, kOut, g->err, st));
	G_TRY(fmx_spmm(m, FMX_F32, Z2, kOut, FMX_F32, Y, kOut, kOut, scale, scale, st));
	return FMX_OK;
}

int read_err(const fmx_gnn *g, cudaStream_t st)
{
	int e = 0;
	GCUDA_TRY(cudaMemcpyAsync(&e, g->err, sizeof(int), cudaMemcpyDeviceToHost, st));
	GCUDA_TRY(cudaStreamSynchronize(st));
	if (e) return set_error(FMX_ERR_CUDA, "a tensor-core wait ran out of time");
	return FMX_OK;
}

} // namespace

extern "C" {

int fmx_gnn_create(int device, uint64_t seed, fmx_gnn **out)
{
	if (!out) return set_error(FMX_ERR_INVAL, "null output");
	*out = nullptr;
	int cur = 0;
	cudaGetDevice(&cur);
	GCUDA_TRY(cudaSetDevice(device));
	fmx_gnn *g = new fmx_gnn;
	g->device = device;
	cudaError_t e = cudaMalloc((void **)&g->p, sizeof(float) * (4 * size_t(kParams) + kH * kOut) + 256);
	if (e != cudaSuccess) {
		delete g;
		cudaSetDevice(cur);
		return set_error(FMX_ERR_OOM, "GNN parameters: %s", cudaGetErrorString(e));
	}
	g->m = g->p + kParams;
	g->v = g->m + kParams;
	g->g = g->v + kParams;
	g->w2t = g->g + kParams;
	g->err = reinterpret_cast<int *>(g->w2t + kH * kOut);
	// Glorot-uniform weights (counter-based, seeded), zero bias
	std::vector<float> h(kParams, 0.f);
	auto uni = [&](uint64_t i) {
		uint64_t z = seed * 0x9E3779B97F4A7C15ull + i * 0xBF58476D1CE4E5B9ull;
		z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
		z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
		z ^= z >> 31;
		return double(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
	};
	const double a1 = std::sqrt(6.0 / (kZ + kH)), a2 = std::sqrt(6.0 / (kH + kOut));
	for (int i = 0; i < kZ * kH; i++) h[kOffW1 + i] = float(a1 * uni(uint64_t(i)));
	for (int i = 0; i < kH * kOut; i++) h[kOffW2 + i] = float(a2 * uni(uint64_t(kZ * kH + i)));
	e = cudaMemcpy(g->p, h.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice);
	if (e == cudaSuccess) e = cudaMemset(g->m, 0, sizeof(float) * 3 * size_t(kParams));
	if (e == cudaSuccess) e = cudaMemset(g->err, 0, sizeof(int));
	cudaSetDevice(cur);
	if (e != cudaSuccess) {
		cudaFree(g->p);
		delete g;
		return set_error(FMX_ERR_CUDA, "GNN initialisation: %s", cudaGetErrorString(e));
	}
	*out = g;
	return FMX_OK;
}

int fmx_gnn_free(fmx_gnn *g)
{
	if (!g) return FMX_OK;
	int cur = 0;
	cudaGetDevice(&cur);
	cudaSetDevice(g->device);
	cudaFree(g->p);
	cudaSetDevice(cur);
	delete g;
	return FMX_OK;
}

int fmx_gnn_set_params(fmx_gnn *g, const float *host)
{
	if (!g || !host) return set_error(FMX_ERR_INVAL, "null argument");
	GCUDA_TRY(cudaMemcpy(g->p, host, sizeof(float) * kParams, cudaMemcpyHostToDevice));
	GCUDA_TRY(cudaMemset(g->m, 0, sizeof(float) * 3 * size_t(kParams)));
	g->t = 0;
	return FMX_OK;
}

int fmx_gnn_get_params(const fmx_gnn *g, float *host)
{
	if (!g || !host) return set_error(FMX_ERR_INVAL, "null argument");
	GCUDA_TRY(cudaMemcpy(host, g->p, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
	return FMX_OK;
}

int fmx_gnn_features(const fmx_matrix *m, const float *scale, uint64_t seed, float *Z, void *stream)
{
	if (!m || !Z || !scale) return set_error(FMX_ERR_INVAL, "null argument");
	if (reinterpret_cast<uintptr_t>(Z) % 16) return set_error(FMX_ERR_INVAL, "Z must be 16-byte aligned");
	int64_t n = 0;
	G_TRY(check_matrix(m, &n));
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	scratch s;
	s.st = st;
	double *part = nullptr;
	const int parts = int(grid_for(n));
	G_TRY(s.get(&part, size_t(2 * parts)));
	logdeg_stats_kernel<<<parts, kThreads, 0, st>>>(scale, n, part);
	GCUDA_TRY(cudaGetLastError());
	features_kernel<<<grid_for(n), kThreads, 0, st>>>(scale, n, part, parts, seed, Z);
	GCUDA_TRY(cudaGetLastError());
	for (int h = 1; h <= kHops; h++)
		G_TRY(fmx_spmm(m, FMX_F32, Z + (h - 1) * kF, kZ, FMX_F32, Z + h * kF, kZ, kF, scale, scale, st));
	return FMX_OK;
}

int fmx_gnn_forward(const fmx_gnn *g, const fmx_matrix *m, const float *scale, const float *Z, int precision,
		float *Y, void *stream)
{
	if (!g || !m || !Z || !Y) return set_error(FMX_ERR_INVAL, "null argument");
	G_TRY(check_precision(precision));
	int64_t n = 0;
	G_TRY(check_matrix(m, &n));
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	scratch s;
	s.st = st;
	float *H = nullptr, *Z2 = nullptr;
	G_TRY(s.get(&H, size_t(n) * kH));
	G_TRY(s.get(&Z2, size_t(n) * kOut));
	G_TRY(forward(g, m, scale, Z, n, precision, H, Z2, Y, st));
	return read_err(g, st);
}

int fmx_gnn_loss_grad(fmx_gnn *g, const fmx_matrix *m, const float *scale, const float *Z, const float *U,
		int64_t ldu, int nev, int precision, double *loss, float *grad_host, void *stream)
{
	if (!g || !m || !Z || !U) return set_error(FMX_ERR_INVAL, "null argument");
	if (nev < 1 || nev > kMaxNev || ldu < nev) return set_error(FMX_ERR_INVAL, "nev in 1..%d with ldu >= nev", kMaxNev);
	G_TRY(check_precision(precision));
	int64_t n = 0;
	G_TRY(check_matrix(m, &n));
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	scratch s;
	s.st = st;
	float *H, *Z2, *Y, *dY, *dZ2, *dH, *P1, *P2, *bpart, *gpart;
	double *G, *M, *dpart, *dloss;
	const int rparts = int(grid_for(n * kH));
	const int gparts = std::max({fmx_dense_gram_parts(FMX_DENSE_F64, n), fmx_dense_gram_parts(precision, n)});
	G_TRY(s.get(&H, size_t(n) * kH));
	G_TRY(s.get(&Z2, size_t(n) * kOut));
	G_TRY(s.get(&Y, size_t(n) * kOut));
	G_TRY(s.get(&dY, size_t(n) * kOut));
	G_TRY(s.get(&dZ2, size_t(n) * kOut));
	G_TRY(s.get(&dH, size_t(n) * kH));
	G_TRY(s.get(&P1, size_t(kMaxNev) * kOut));
	G_TRY(s.get(&P2, size_t(kOut) * kOut));
	G_TRY(s.get(&bpart, size_t(rparts) * kH));
	G_TRY(s.get(&gpart, size_t(gparts) * kZ * kH));
	G_TRY(s.get(&dpart, size_t(gparts) * kMaxNev * kOut));
	G_TRY(s.get(&G, size_t(kOut) * kOut));
	G_TRY(s.get(&M, size_t(kMaxNev) * kOut));
	G_TRY(s.get(&dloss, 1));
	G_TRY(forward(g, m, scale, Z, n, precision, H, Z2, Y, st));
	// loss and dL/dY
	G_TRY(fmx_dense_gram(FMX_DENSE_F64, Y, kOut, kOut, Y, kOut, kOut, n, dpart, G, nullptr, st));
	G_TRY(fmx_dense_gram(FMX_DENSE_F64, U, ldu, nev, Y, kOut, kOut, n, dpart, M, nullptr, st));
	loss_kernel<<<1, kThreads, 0, st>>>(G, M, nev, P1, P2, dloss);
	GCUDA_TRY(cudaGetLastError());
	dy_kernel<<<grid_for(n * kOut), kThreads, 0, st>>>(U, ldu, nev, Y, P1, P2, n, dY);
	GCUDA_TRY(cudaGetLastError());
	// layer 2: Y = A_s Z2, Z2 = H W2
	G_TRY(fmx_spmm(m, FMX_F32, dY, kOut, FMX_F32, dZ2, kOut, kOut, scale, scale, st));
	G_TRY(fmx_dense_gram(precision, H, kH, kH, dZ2, kOut, kOut, n, gpart, g->g + kOffW2, g->err, st));
	transpose_kernel<<<4, kThreads, 0, st>>>(g->p + kOffW2, kH, kOut, g->w2t);
	GCUDA_TRY(cudaGetLastError());
	G_TRY(fmx_dense_gemm(precision, dZ2, kOut, n, kOut, g->w2t, kH, kH, dH, kH, g->err, st));
	// layer 1: H = relu(Z W1 + b1)
	relu_grad_kernel<<<rparts, kThreads, 0, st>>>(dH, H, n, bpart);
	GCUDA_TRY(cudaGetLastError());
	sum_parts_kernel<<<1, kH, 0, st>>>(bpart, rparts, kH, g->g + kOffB1);
	GCUDA_TRY(cudaGetLastError());
	G_TRY(fmx_dense_gram(precision, Z, kZ, kZ, dH, kH, kH, n, gpart, g->g + kOffW1, g->err, st));
	if (loss) GCUDA_TRY(cudaMemcpyAsync(loss, dloss, sizeof(double), cudaMemcpyDeviceToHost, st));
	if (grad_host) GCUDA_TRY(cudaMemcpyAsync(grad_host, g->g, sizeof(float) * kParams, cudaMemcpyDeviceToHost, st));
	return read_err(g, st);
}

int fmx_gnn_adam_step(fmx_gnn *g, float lr, void *stream)
{
	if (!g) return set_error(FMX_ERR_INVAL, "null model");
	const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
	g->t++;
	const float c1 = float(1.0 - std::pow(double(b1), double(g->t)));
	const float c2 = float(1.0 - std::pow(double(b2), double(g->t)));
	adam_kernel<<<grid_for(kParams), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(g->p, g->m, g->v, g->g,
			kParams, lr, b1, b2, eps, c1, c2);
	GCUDA_TRY(cudaGetLastError());
	return FMX_OK;
}

} // extern "C"
