// Block eigensolver on B200: the largest eigenpairs of a symmetric sparse
// operator  A_s = diag(s) A diag(s)  (s = D^-1/2 gives the normalised
// adjacency of NA_eigen_Operator, matrix/test/test-eigen.cpp:88-136).
//
// Replaces fm::eigen::compute_eigen (matrix/eigensolver/eigensolver.cpp:
// 118-308), whose Krylov-Schur / Davidson / LOBPCG iterations live in the
// external Trilinos Anasazi.  The method here is Chebyshev-filtered subspace
// iteration (Zhou and Saad, "Self-consistent-field calculations using
// Chebyshev-filtered subspace iteration", J. Comput. Phys. 219, 2006) on a
// block of b <= 64 vectors:
//
//   filter   Y = p_m(A_s) X, p_m the degree-m Chebyshev polynomial that is
//            bounded by 1 on the unwanted interval [lo, cut] and scaled to 1
//            at the top of the spectrum (three-term recurrence; the first
//            product A_s X is the one the last Rayleigh-Ritz step computed)
//   CholQR2  G = Y^T Y (FP64), R = chol(G + shift), Y <- Y R^-1, twice
//   RR       W = A_s Q, H = Q^T W, H = V diag(theta) V^T (FP64 Jacobi),
//            X = Q V, A_s X = W V, residuals ||A_s x - theta x|| (FP64)
//
// so one pass costs m SpMMs of b columns.  The cut is the b-th Ritz value,
// capped so that the filter still amplifies the top of the spectrum by a
// fixed factor (an eigenvalue of multiplicity >= b, like the eigenvalue 1 of
// a graph with many components, would otherwise pull the cut up to it and
// stall the iteration).
//
// Precision modes:
//   FMX_EIGEN_PLAIN  FP32 SpMM operands; every dense product on CUDA cores
//                    with FP64 accumulation.
//   FMX_EIGEN_MIXED  the filter runs in correction form, Y = X p(Theta) + E,
//                    with every filter SpMM on BF16 operands (FP32
//                    accumulation): their rounding error is relative to the
//                    correction E, which shrinks with the residual, so BF16
//                    does not floor the accuracy.  The Rayleigh-Ritz SpMM
//                    stays FP32.  While the largest wanted residual exceeds
//                    `tensor_until`, the CholQR basis update runs on tensor
//                    cores (3xTF32, tcgen05), after it in FP64 (3xTF32 is
//                    accurate to about 1e-5 relative).  The Gram products,
//                    the Cholesky factor, the projected eigenproblem and the
//                    residual norms are FP64 throughout.
#include "fmx_internal.h"

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

namespace fmx {
namespace eig {

constexpr int kMaxB = 64;
constexpr int kThreads = 256;
#ifndef FMX_MIXED_MAX_DEGREE
#define FMX_MIXED_MAX_DEGREE 10
#endif
constexpr int kMixedMaxDegree = FMX_MIXED_MAX_DEGREE;

#define ECUDA_TRY(call)                                                         \
	do {                                                                        \
		cudaError_t err__ = (call);                                             \
		if (err__ != cudaSuccess)                                               \
			return set_error(FMX_ERR_CUDA, "%s failed: %s (%s:%d)", #call,      \
					cudaGetErrorString(err__), __FILE__, __LINE__);             \
	} while (0)
#define E_TRY(call)                                                             \
	do {                                                                        \
		int rc__ = (call);                                                      \
		if (rc__ != FMX_OK) return rc__;                                        \
	} while (0)

__device__ __forceinline__ float ldf(const float *p) { return *p; }
__device__ __forceinline__ float ldf(const __nv_bfloat16 *p) { return __bfloat162float(*p); }
__device__ __forceinline__ void stf(float *p, float v) { *p = v; }
__device__ __forceinline__ void stf(__nv_bfloat16 *p, float v) { *p = __float2bfloat16_rn(v); }

// splitmix64 finaliser (Steele, Lea, Flood 2014): counter-based uniform bits
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z)
{
	z += 0x9E3779B97F4A7C15ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

// X = uniform(-1, 1), the reference's MvRandom (FM_MultiVector.h:661-676)
__global__ void random_block_kernel(float *X, int64_t count, uint64_t seed)
{
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count; i += int64_t(gridDim.x) * blockDim.x) {
		const uint64_t u = mix64(seed * 0x100000001B3ull ^ uint64_t(i));
		X[i] = float(double(u >> 11) * (2.0 / 9007199254740992.0) - 1.0);
	}
}

// out[r][j] = in[r][j] for the first c columns of n rows (pitches in floats):
// the eigenvectors leave the solver's n x b block this way (a pitched copy of
// 4.2M rows of 32 bytes took about 0.4 ms)
__global__ void copy_cols_kernel(const float *in, int64_t ldi, float *out, int64_t ldo, int64_t n, int c)
{
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n * c; i += int64_t(gridDim.x) * blockDim.x) {
		const int64_t r = i / c;
		const int j = int(i - r * c);
		out[r * ldo + j] = in[r * ldi + j];
	}
}

// One Chebyshev step on flat n x b blocks:  O = alpha (W - c0 Y) - beta P
template <class YT, class PT, class OT>
__global__ void cheb_kernel(const float *__restrict__ W, const YT *__restrict__ Y, const PT *__restrict__ P,
		OT *__restrict__ O, int64_t count, float alpha, float c0, float beta)
{
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count; i += int64_t(gridDim.x) * blockDim.x) {
		float v = alpha * (W[i] - c0 * ldf(Y + i));
		if (P) v -= beta * ldf(P + i);
		stf(O + i, v);
	}
}

// One step of the filter in correction form, on flat n x b blocks:
//   O = alpha W - ac0 E - beta P + cr[col] R + cx[col] X
// (each of W, E, P, R, X may be absent); R FP32 or BF16.  With Rb, the step
// also writes R rounded to BF16 there (the first step of a pass, so that the
// later BF16 steps read half the bytes of R).
struct col_coefs {
	float r[kMaxB];
	float x[kMaxB];
};

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float4 ld4(const __nv_bfloat16 *p)
{
	const uint2 u = *reinterpret_cast<const uint2 *>(p);        // element 0 in the low half
	return make_float4(__uint_as_float(u.x << 16), __uint_as_float(u.x & 0xffff0000u),
			__uint_as_float(u.y << 16), __uint_as_float(u.y & 0xffff0000u));
}
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ void st4(__nv_bfloat16 *p, float4 v)
{
	__nv_bfloat162 a = __floats2bfloat162_rn(v.x, v.y), c = __floats2bfloat162_rn(v.z, v.w);
	uint2 u;
	u.x = *reinterpret_cast<uint32_t *>(&a);
	u.y = *reinterpret_cast<uint32_t *>(&c);
	*reinterpret_cast<uint2 *>(p) = u;
}

__device__ __forceinline__ void ld8(const float *p, float (&t)[8])
{
	const float4 a = ld4(p), c = ld4(p + 4);
	t[0] = a.x; t[1] = a.y; t[2] = a.z; t[3] = a.w; t[4] = c.x; t[5] = c.y; t[6] = c.z; t[7] = c.w;
}
__device__ __forceinline__ void ld8(const __nv_bfloat16 *p, float (&t)[8])
{
	const uint4 u = *reinterpret_cast<const uint4 *>(p);        // element 0 in the low half
	const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
	for (int q = 0; q < 4; q++) {
		t[2 * q] = __uint_as_float(w[q] << 16);
		t[2 * q + 1] = __uint_as_float(w[q] & 0xffff0000u);
	}
}
__device__ __forceinline__ void st8(float *p, const float (&v)[8])
{
	st4(p, make_float4(v[0], v[1], v[2], v[3]));
	st4(p + 4, make_float4(v[4], v[5], v[6], v[7]));
}
__device__ __forceinline__ void st8(__nv_bfloat16 *p, const float (&v)[8])
{
	uint32_t w[4];
#pragma unroll
	for (int q = 0; q < 4; q++) {
		__nv_bfloat162 h = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
		memcpy(&w[q], &h, 4);
	}
	*reinterpret_cast<uint4 *>(p) = make_uint4(w[0], w[1], w[2], w[3]);
}

template <class WT, class ET, class PT, class RT, class OT>
__global__ void corr_kernel(const WT *__restrict__ W, const ET *__restrict__ E, const PT *__restrict__ P,
		const RT *__restrict__ R, const float *__restrict__ X, OT *__restrict__ O, int64_t count, int b,
		float alpha, float ac0, float beta, col_coefs cf, __nv_bfloat16 *__restrict__ Rb)
{
	const bool pow2 = (b & (b - 1)) == 0;
	const int64_t tstride = int64_t(gridDim.x) * blockDim.x;
	if ((b & 7) == 0) {
		// eight consecutive elements of one row per thread (16-byte loads of
		// BF16 blocks); each element's arithmetic is the four-wide path's
		for (int64_t i8 = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i8 < count / 8; i8 += tstride) {
			const int64_t i = 8 * i8;
			const int col = pow2 ? int(i & (b - 1)) : int(i % b);
			float v[8], t[8];
#pragma unroll
			for (int q = 0; q < 8; q++) v[q] = 0.f;
			if (W) {
				ld8(W + i, t);
#pragma unroll
				for (int q = 0; q < 8; q++) v[q] = alpha * t[q];
			}
			if (E) {
				ld8(E + i, t);
#pragma unroll
				for (int q = 0; q < 8; q++) v[q] -= ac0 * t[q];
			}
			if (P) {
				ld8(P + i, t);
#pragma unroll
				for (int q = 0; q < 8; q++) v[q] -= beta * t[q];
			}
			if (R) {
				ld8(R + i, t);
				if (Rb) st8(Rb + i, t);
#pragma unroll
				for (int q = 0; q < 8; q++) v[q] += cf.r[col + q] * t[q];
			}
			if (X) {
				ld8(X + i, t);
#pragma unroll
				for (int q = 0; q < 8; q++) v[q] += cf.x[col + q] * t[q];
			}
			st8(O + i, v);
		}
		return;
	}
	if ((b & 3) == 0) {
		// four consecutive elements of one row per thread
		for (int64_t i4 = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i4 < count / 4; i4 += tstride) {
			const int64_t i = 4 * i4;
			const int col = pow2 ? int(i & (b - 1)) : int(i % b);
			float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
			if (W) {
				const float4 t = ld4(W + i);
				v = make_float4(alpha * t.x, alpha * t.y, alpha * t.z, alpha * t.w);
			}
			if (E) {
				const float4 t = ld4(E + i);
				v.x -= ac0 * t.x; v.y -= ac0 * t.y; v.z -= ac0 * t.z; v.w -= ac0 * t.w;
			}
			if (P) {
				const float4 t = ld4(P + i);
				v.x -= beta * t.x; v.y -= beta * t.y; v.z -= beta * t.z; v.w -= beta * t.w;
			}
			if (R) {
				const float4 t = ld4(R + i);
				if (Rb) st4(Rb + i, t);
				v.x += cf.r[col] * t.x; v.y += cf.r[col + 1] * t.y; v.z += cf.r[col + 2] * t.z; v.w += cf.r[col + 3] * t.w;
			}
			if (X) {
				const float4 t = ld4(X + i);
				v.x += cf.x[col] * t.x; v.y += cf.x[col + 1] * t.y; v.z += cf.x[col + 2] * t.z; v.w += cf.x[col + 3] * t.w;
			}
			st4(O + i, v);
		}
		return;
	}
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count; i += tstride) {
		const int col = pow2 ? int(i & (b - 1)) : int(i % b);
		float v = 0.f;
		if (W) v = alpha * ldf(W + i);
		if (E) v -= ac0 * ldf(E + i);
		if (P) v -= beta * ldf(P + i);
		if (R) {
			const float r = ldf(R + i);
			if (Rb) stf(Rb + i, r);
			v += cf.r[col] * r;
		}
		if (X) v += cf.x[col] * X[i];
		stf(O + i, v);
	}
}

// Basis update with FP64 accumulation:
//   X[r][j] = sum_k Q[r][k] V[k][perm j]       (written when WRITE)
//   NX[r][j] = sum_k W[r][k] V[k][perm j]      (HAS_W; written when WRITE; with
//                                               resid_out, NX - theta X instead)
//   part[cta][j] += (NX[r][j] - theta[j] X[r][j])^2, part[cta][b + j] += X[r][j]^2   (RES)
// A thread owns one row and a group of up to 16 output columns (G = 1, 2 or
// 4 threads per row for b <= 16, 32, 64); V sits in shared memory, read as a
// broadcast.  Residual sums are reduced per warp with shuffles, then over the
// warps in a fixed order (deterministic for a fixed grid).
constexpr int kRitzCols = 16;

__host__ __device__ inline int ritz_threads_per_row(int b) { return b <= 16 ? 1 : (b <= 32 ? 2 : 4); }

template <bool HAS_W, bool RES, bool WRITE>
__global__ void __launch_bounds__(kThreads)
ritz_kernel(const float *__restrict__ Q, const float *__restrict__ W, int b, const double *__restrict__ V,
		const int *__restrict__ perm, const double *__restrict__ theta, float *__restrict__ X,
		float *__restrict__ NX, int64_t n, double *__restrict__ part, int resid_out)
{
	__shared__ double sV[kMaxB * kMaxB];
	__shared__ double red[kThreads / 32][2 * kMaxB];
	const int tid = threadIdx.x;
	for (int i = tid; i < kMaxB * kMaxB; i += kThreads) {
		const int k = i / kMaxB, j = i % kMaxB;
		sV[i] = (k < b && j < b) ? V[k * b + (perm ? perm[j] : j)] : 0.0;
	}
	__syncthreads();
	const int G = ritz_threads_per_row(b);
	const int g = tid % G;
	const int j0 = g * kRitzCols;
	double th[kRitzCols];
#pragma unroll
	for (int jj = 0; jj < kRitzCols; jj++) th[jj] = (RES && j0 + jj < b) ? theta[j0 + jj] : 0.0;
	double racc[kRitzCols], xacc[kRitzCols];
#pragma unroll
	for (int jj = 0; jj < kRitzCols; jj++) racc[jj] = xacc[jj] = 0;
	const int64_t rows_per_pass = int64_t(gridDim.x) * (kThreads / G);
	const bool vec = (b % 4) == 0;
	for (int64_t row = int64_t(blockIdx.x) * (kThreads / G) + tid / G; row < n; row += rows_per_pass) {
		const float *q = Q + row * b;
		const float *w = HAS_W ? W + row * b : nullptr;
		double x[kRitzCols], y[kRitzCols];
#pragma unroll
		for (int jj = 0; jj < kRitzCols; jj++) x[jj] = y[jj] = 0;
		if (vec) {
			// chunks of 16 input columns: all loads first (8 x 16 bytes in
			// flight), then the FMAs
			for (int k0 = 0; k0 < b; k0 += 16) {
				const int kn = min(16, b - k0);             // a multiple of 4
				float qs[16], ws[16];
#pragma unroll
				for (int u = 0; u < 4; u++) {
					float4 qv = make_float4(0.f, 0.f, 0.f, 0.f), wv = qv;
					if (4 * u < kn) {
						qv = *reinterpret_cast<const float4 *>(q + k0 + 4 * u);
						if (HAS_W) wv = *reinterpret_cast<const float4 *>(w + k0 + 4 * u);
					}
					qs[4 * u] = qv.x; qs[4 * u + 1] = qv.y; qs[4 * u + 2] = qv.z; qs[4 * u + 3] = qv.w;
					ws[4 * u] = wv.x; ws[4 * u + 1] = wv.y; ws[4 * u + 2] = wv.z; ws[4 * u + 3] = wv.w;
				}
#pragma unroll
				for (int u = 0; u < 16; u++) {
					const double *vr = sV + (k0 + u) * kMaxB + j0;   // rows >= b of sV are zero
#pragma unroll
					for (int jj = 0; jj < kRitzCols; jj++) {
						x[jj] = fma(double(qs[u]), vr[jj], x[jj]);
						if (HAS_W) y[jj] = fma(double(ws[u]), vr[jj], y[jj]);
					}
				}
			}
		} else {
			for (int k = 0; k < b; k++) {
				const double qk = q[k];
				const double wk = HAS_W ? double(w[k]) : 0.0;
				const double *vr = sV + k * kMaxB + j0;
#pragma unroll
				for (int jj = 0; jj < kRitzCols; jj++) {
					x[jj] = fma(qk, vr[jj], x[jj]);
					if (HAS_W) y[jj] = fma(wk, vr[jj], y[jj]);
				}
			}
		}
		if (WRITE) {
			float *xo = X + row * b + j0;
			float *yo = HAS_W ? NX + row * b + j0 : nullptr;
#pragma unroll
			for (int jj = 0; jj < kRitzCols; jj++)
				if (j0 + jj < b) {
					xo[jj] = float(x[jj]);
					if (HAS_W) yo[jj] = float(resid_out ? y[jj] - th[jj] * x[jj] : y[jj]);
				}
		}
		if (RES) {
#pragma unroll
			for (int jj = 0; jj < kRitzCols; jj++) {
				const double d = y[jj] - th[jj] * x[jj];
				racc[jj] = fma(d, d, racc[jj]);
				xacc[jj] = fma(x[jj], x[jj], xacc[jj]);
			}
		}
	}
	if (RES) {
		const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
		for (int jj = 0; jj < kRitzCols; jj++) {
			for (int off = 16; off >= G; off >>= 1) {
				racc[jj] += __shfl_down_sync(0xffffffffu, racc[jj], off);
				xacc[jj] += __shfl_down_sync(0xffffffffu, xacc[jj], off);
			}
		}
		if (lane < G) {
#pragma unroll
			for (int jj = 0; jj < kRitzCols; jj++)
				if (j0 + jj < b) {
					red[warp][j0 + jj] = racc[jj];
					red[warp][b + j0 + jj] = xacc[jj];
				}
		}
		__syncthreads();
		for (int i = tid; i < 2 * b; i += kThreads) {
			double sum = 0;
			for (int w2 = 0; w2 < kThreads / 32; w2++) sum += red[w2][i];
			part[size_t(blockIdx.x) * 2 * b + i] = sum;
		}
	}
}

// D = A B + C on the FP64 tensor path, one 8 x 8 x 4 tile per warp
// (mma.sync m8n8k4 .f64): lane (g = lane / 4, t = lane % 4) holds A[g][t],
// B[t][g] and D[g][2t], D[g][2t + 1].
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b)
{
	asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
			: "+d"(d[0]), "+d"(d[1]) : "d"(a), "d"(b));
}

// The basis update of ritz_kernel for b <= 8 NT (NT = 2 or 4 column tiles of
// 8) on the FP64 tensor path: a warp takes 8 rows per step (the MMA's M).
// The input columns are the MMA's K in 2 NT steps, relabelled so that lane
// t's A element at step s is column 16 (s / 4) + 4 t + s % 4 (one 16-byte
// load per row, operand and 16 columns); V' = V[:, perm] (zero beyond b)
// sits in 2 NT x NT B-fragment registers per lane for the whole kernel.
// NT 8-column tiles give X (and NX from W); lane (g, t) ends with columns
// 8 ni + 2t, 8 ni + 2t + 1 of row 8 * tile + g.  Products of FP32 inputs
// are exact in FP64; residual sums are reduced over lanes, then warps, in a
// fixed order.  Same outputs and partial layout as ritz_kernel.
template <int NT, bool HAS_W, bool RES, bool WRITE>
__global__ void __launch_bounds__(kThreads)
ritz_dmma_kernel(const float *__restrict__ Q, const float *__restrict__ W, int b, const double *__restrict__ V,
		const int *__restrict__ perm, const double *__restrict__ theta, float *__restrict__ X,
		float *__restrict__ NX, int64_t n, double *__restrict__ part, int resid_out, bool vec)
{
	constexpr int KS = 2 * NT;                // k-steps of 4 columns
	constexpr int H = NT / 2;                 // 16-column halves
	__shared__ double red[kThreads / 32][64];
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int g = lane >> 2, t = lane & 3;
	double vb[KS][NT];
#pragma unroll
	for (int st = 0; st < KS; st++)
#pragma unroll
		for (int ni = 0; ni < NT; ni++) {
			const int k = 16 * (st / 4) + 4 * t + st % 4, j = 8 * ni + g;
			vb[st][ni] = (k < b && j < b) ? V[k * b + (perm ? perm[j] : j)] : 0.0;
		}
	double th[NT][2], racc[NT][2], xacc[NT][2];
#pragma unroll
	for (int ni = 0; ni < NT; ni++)
#pragma unroll
		for (int i = 0; i < 2; i++) {
			const int j = 8 * ni + 2 * t + i;
			th[ni][i] = (RES && j < b) ? theta[j] : 0.0;
			racc[ni][i] = xacc[ni][i] = 0.0;
		}
	const int64_t tiles = (n + 7) / 8;
	const int64_t tstride = int64_t(gridDim.x) * (kThreads / 32);
	// a tile's rows: this lane's 4-column groups of row tile * 8 + g
	auto load = [&](int64_t tile, float (&qa)[KS], float (&wa)[KS]) {
		const int64_t row = tile * 8 + g;
#pragma unroll
		for (int st = 0; st < KS; st++) qa[st] = wa[st] = 0.f;
		if (tile < tiles && row < n) {
#pragma unroll
			for (int h = 0; h < H; h++) {
				const int c0 = 16 * h + 4 * t;
				if (vec && c0 + 3 < b) {
					const float4 qv = *reinterpret_cast<const float4 *>(Q + row * b + c0);
					qa[4 * h] = qv.x; qa[4 * h + 1] = qv.y; qa[4 * h + 2] = qv.z; qa[4 * h + 3] = qv.w;
					if (HAS_W) {
						const float4 wv = *reinterpret_cast<const float4 *>(W + row * b + c0);
						wa[4 * h] = wv.x; wa[4 * h + 1] = wv.y; wa[4 * h + 2] = wv.z; wa[4 * h + 3] = wv.w;
					}
				} else {
#pragma unroll
					for (int e = 0; e < 4; e++)
						if (c0 + e < b) {
							qa[4 * h + e] = Q[row * b + c0 + e];
							if (HAS_W) wa[4 * h + e] = W[row * b + c0 + e];
						}
				}
			}
		}
	};
	// the next tile's rows load while this one's products run (one tile in
	// flight per warp left the update at 0.43 of the HBM bound)
	float qa[KS], wa[KS], qn[KS], wn[KS];
	int64_t tile = int64_t(blockIdx.x) * (kThreads / 32) + warp;
	load(tile, qa, wa);
	for (; tile < tiles; tile += tstride) {
		const int64_t row = tile * 8 + g;
		const bool rv = row < n;
		load(tile + tstride, qn, wn);
		double cx[NT][2], cy[NT][2];
#pragma unroll
		for (int ni = 0; ni < NT; ni++) cx[ni][0] = cx[ni][1] = cy[ni][0] = cy[ni][1] = 0.0;
#pragma unroll
		for (int st = 0; st < KS; st++) {
			const double aq = qa[st], aw = wa[st];
#pragma unroll
			for (int ni = 0; ni < NT; ni++) {
				dmma_8x8x4(cx[ni], aq, vb[st][ni]);
				if (HAS_W) dmma_8x8x4(cy[ni], aw, vb[st][ni]);
			}
		}
		if (WRITE && rv) {
#pragma unroll
			for (int ni = 0; ni < NT; ni++) {
				const int j = 8 * ni + 2 * t;
				float2 xo, yo;
				xo.x = float(cx[ni][0]); xo.y = float(cx[ni][1]);
				if (HAS_W) {
					yo.x = float(resid_out ? cy[ni][0] - th[ni][0] * cx[ni][0] : cy[ni][0]);
					yo.y = float(resid_out ? cy[ni][1] - th[ni][1] * cx[ni][1] : cy[ni][1]);
				}
				if (vec && j + 1 < b) {
					*reinterpret_cast<float2 *>(X + row * b + j) = xo;
					if (HAS_W) *reinterpret_cast<float2 *>(NX + row * b + j) = yo;
				} else {
					if (j < b) {
						X[row * b + j] = xo.x;
						if (HAS_W) NX[row * b + j] = yo.x;
					}
					if (j + 1 < b) {
						X[row * b + j + 1] = xo.y;
						if (HAS_W) NX[row * b + j + 1] = yo.y;
					}
				}
			}
		}
		if (RES) {
			// rows beyond n had zero inputs: they add nothing
#pragma unroll
			for (int ni = 0; ni < NT; ni++)
#pragma unroll
				for (int i = 0; i < 2; i++) {
					const double d = cy[ni][i] - th[ni][i] * cx[ni][i];
					racc[ni][i] = fma(d, d, racc[ni][i]);
					xacc[ni][i] = fma(cx[ni][i], cx[ni][i], xacc[ni][i]);
				}
		}
#pragma unroll
		for (int st = 0; st < KS; st++) {
			qa[st] = qn[st];
			wa[st] = wn[st];
		}
	}
	if (RES) {
		// lanes of one t hold the same columns: add over g (lane bits 2-4)
#pragma unroll
		for (int ni = 0; ni < NT; ni++)
#pragma unroll
			for (int i = 0; i < 2; i++)
				for (int o = 4; o < 32; o <<= 1) {
					racc[ni][i] += __shfl_xor_sync(0xffffffffu, racc[ni][i], o);
					xacc[ni][i] += __shfl_xor_sync(0xffffffffu, xacc[ni][i], o);
				}
		if (lane < 4)
#pragma unroll
			for (int ni = 0; ni < NT; ni++)
#pragma unroll
				for (int i = 0; i < 2; i++) {
					red[warp][8 * ni + 2 * t + i] = racc[ni][i];
					red[warp][32 + 8 * ni + 2 * t + i] = xacc[ni][i];
				}
		__syncthreads();
		for (int i = tid; i < 2 * b; i += kThreads) {
			const int slot = i < b ? i : 32 + (i - b);
			double sum = 0;
			for (int w2 = 0; w2 < kThreads / 32; w2++) sum += red[w2][slot];
			part[size_t(blockIdx.x) * 2 * b + i] = sum;
		}
	}
}

// ritz_kernel or, for b <= 32, ritz_dmma_kernel
template <bool HAS_W, bool RES, bool WRITE>
static void launch_ritz(int grid, cudaStream_t st, const float *Q, const float *W, int b, const double *V,
		const int *perm, const double *theta, float *X, float *NX, int64_t n, double *part, int resid_out)
{
	auto al = [](const void *p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; };
	// 16-byte row loads and 8-byte column-pair stores when every row starts
	// on a 16-byte boundary (b % 4 == 0) and the bases are aligned
	const bool vec = b % 4 == 0 && al(Q, 16) && al(W, 16) && al(X, 8) && al(NX, 8);
	if (b <= 16)
		ritz_dmma_kernel<2, HAS_W, RES, WRITE><<<grid, kThreads, 0, st>>>(Q, W, b, V, perm, theta, X, NX, n, part,
				resid_out, vec);
	else if (b <= 32)
		ritz_dmma_kernel<4, HAS_W, RES, WRITE><<<grid, kThreads, 0, st>>>(Q, W, b, V, perm, theta, X, NX, n, part,
				resid_out, vec);
	else
		ritz_kernel<HAS_W, RES, WRITE><<<grid, kThreads, 0, st>>>(Q, W, b, V, perm, theta, X, NX, n, part, resid_out);
}

// out[i] = sum over the partials: one warp per element, a fixed xor tree
__global__ void reduce_parts_kernel(const double *__restrict__ part, int nparts, int len, double *__restrict__ out)
{
	const int lane = threadIdx.x & 31;
	const int warps = int((gridDim.x * blockDim.x) >> 5);
	for (int i = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < len; i += warps) {
		double s = 0;
		for (int p = lane; p < nparts; p += 32) s += part[size_t(p) * len + i];
		for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
		if (lane == 0) out[i] = s;
	}
}

// G += rel * max(diag G) * I  (the shift of shifted CholQR: keeps the
// Cholesky factor defined for numerically rank-deficient blocks)
__global__ void shift_diag_kernel(double *G, int b, double rel)
{
	if (threadIdx.x == 0 && blockIdx.x == 0) {
		double m = 0;
		for (int i = 0; i < b; i++) m = fmax(m, G[i * b + i]);
		for (int i = 0; i < b; i++) G[i * b + i] += rel * m;
	}
}

__global__ void f64_to_f32_kernel(const double *a, float *o, int count)
{
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) o[i] = float(a[i]);
}

// Ritz value order: descending value (largest algebraic) or descending
// magnitude (largest magnitude); writes the permutation and the sorted values.
__global__ void order_kernel(const double *w, int b, int by_magnitude, int *perm, double *theta)
{
	if (threadIdx.x != 0 || blockIdx.x != 0) return;
	int p[kMaxB];
	for (int i = 0; i < b; i++) p[i] = i;
	for (int i = 1; i < b; i++) {                 // stable insertion sort
		const int x = p[i];
		const double kx = by_magnitude ? fabs(w[x]) : w[x];
		int j = i - 1;
		while (j >= 0 && (by_magnitude ? fabs(w[p[j]]) : w[p[j]]) < kx) {
			p[j + 1] = p[j];
			j--;
		}
		p[j + 1] = x;
	}
	for (int i = 0; i < b; i++) {
		perm[i] = p[i];
		theta[i] = w[p[i]];
	}
}

// s = D^-1/2 from the row sums d (0 where d = 0)
__global__ void inv_sqrt_kernel(const float *d, float *s, int64_t n)
{
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
		s[i] = d[i] > 0.f ? float(1.0 / sqrt(double(d[i]))) : 0.f;
}

__global__ void fill_kernel(float *p, int64_t n, float v)
{
	for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) p[i] = v;
}

int sm_count()
{
	int dev = 0, s = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev);
	return s > 0 ? s : 1;
}

unsigned flat_grid(int64_t count)
{
	const int64_t want = (count + kThreads - 1) / kThreads;
	return unsigned(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(sm_count()) * 8)));
}

// Device buffers of one solve, released in the destructor (stream-ordered).
struct workspace {
	cudaStream_t st = nullptr;
	std::vector<void *> bufs;
	~workspace()
	{
		for (void *p : bufs) cudaFreeAsync(p, st);
	}
	template <class T>
	int get(T **p, size_t count)
	{
		void *q = nullptr;
		cudaError_t e = work_alloc(&q, std::max<size_t>(count, 1) * sizeof(T), st);
		if (e != cudaSuccess)
			return set_error(FMX_ERR_OOM, "eigensolver workspace of %zu bytes: %s", count * sizeof(T),
					cudaGetErrorString(e));
		bufs.push_back(q);
		*p = static_cast<T *>(q);
		return FMX_OK;
	}
};

// Small per-pass results copied to the host in one transfer.
struct small_out {
	double theta[kMaxB];
	double res2[2 * kMaxB];          // residual^2 then ||x||^2 per column
	int chol_info[4];
	int tc_err;
	int pad;
};

struct solver {
	const fmx_matrix *m;
	fmx_matrix *mt = nullptr;        // the transpose (FMX_EIGEN_OP_GRAM)
	int64_t nrows = 0;               // rows of A (the Gram operator's intermediate)
	void *tmp = nullptr;             // A x for the Gram operator: nrows x b
	const float *s;                  // row scale or null
	fmx_eigen_options o;
	int64_t n;
	int b;
	cudaStream_t st;
	workspace ws;
	float *X = nullptr, *NX = nullptr, *W = nullptr, *B[3] = {nullptr, nullptr, nullptr};
	__nv_bfloat16 *Rb = nullptr;     // mixed precision: R in BF16 for the correction steps
	double *G = nullptr, *T = nullptr, *H = nullptr, *wv = nullptr, *V = nullptr, *eye = nullptr;
	double *part = nullptr, *dsmall_theta = nullptr;
	float *Tf = nullptr, *gpart = nullptr;
	int *perm = nullptr, *tc_err = nullptr, *info = nullptr;
	small_out *dsmall = nullptr, *hsmall = nullptr;
	int ritz_grid = 1;
	int64_t spmm_calls = 0, num_ops = 0;

	// One application of the operator to k columns: diag(s) A diag(s) X, or
	// A^T (A X) for the Gram operator (the intermediate in the output's type
	// when the input is BF16, as the SpMM's type pairs require).
	int spmm(int xt, const void *Xin, int k, void *Out, int yt = FMX_F32)
	{
		if (o.op == FMX_EIGEN_OP_GRAM) {
			const int tt = xt == FMX_BF16 ? yt : FMX_F32;
			E_TRY(fmx_spmm(m, xt, Xin, b, tt, tmp, b, k, nullptr, nullptr, st));
			E_TRY(fmx_spmm(mt, tt, tmp, b, yt, Out, b, k, nullptr, nullptr, st));
			spmm_calls += 2;
			num_ops += 2 * k;
			return FMX_OK;
		}
		E_TRY(fmx_spmm(m, xt, Xin, b, yt, Out, b, k, s, s, st));
		spmm_calls++;
		num_ops += k;
		return FMX_OK;
	}

	int setup()
	{
		ws.st = st;
		const size_t nb = size_t(n) * b;
		if (o.op == FMX_EIGEN_OP_GRAM) {
			float *t = nullptr;
			E_TRY(ws.get(&t, size_t(nrows) * b));
			tmp = t;
		}
		E_TRY(ws.get(&X, nb));
		E_TRY(ws.get(&NX, nb));
		E_TRY(ws.get(&W, nb));
		for (auto &p : B) E_TRY(ws.get(&p, nb));
		if (o.precision == FMX_EIGEN_MIXED) E_TRY(ws.get(&Rb, nb));
		E_TRY(ws.get(&G, b * b));
		E_TRY(ws.get(&T, b * b));
		E_TRY(ws.get(&H, b * b));
		E_TRY(ws.get(&wv, b));
		E_TRY(ws.get(&V, b * b));
		E_TRY(ws.get(&eye, b * b));
		E_TRY(ws.get(&Tf, b * b));
		E_TRY(ws.get(&perm, b));
		E_TRY(ws.get(&tc_err, 1));
		E_TRY(ws.get(&info, 4));
		E_TRY(ws.get(&dsmall, 1));
		// rows per CTA and pass: 8 per warp on the FP64 tensor path (b <= 32),
		// else one row per 1, 2 or 4 threads
		const int R = b <= 32 ? 8 * (kThreads / 32) : kThreads / ritz_threads_per_row(b);
		ritz_grid = int(std::max<int64_t>(1, std::min<int64_t>((n + R - 1) / R, int64_t(sm_count()) * (b <= 32 ? 4 : 2))));
		E_TRY(ws.get(&part, size_t(ritz_grid) * 2 * b));
		const int gparts = std::max({fmx_dense_gram_parts(FMX_DENSE_F64, n), fmx_dense_gram_parts(FMX_DENSE_TF32X3, n)});
		E_TRY(ws.get(&gpart, size_t(gparts) * b * b * 2));      // room for double partials
		std::vector<double> I(size_t(b) * b, 0.0);
		for (int i = 0; i < b; i++) I[size_t(i) * b + i] = 1.0;
		ECUDA_TRY(cudaMemcpyAsync(eye, I.data(), I.size() * sizeof(double), cudaMemcpyHostToDevice, st));
		ECUDA_TRY(cudaMemsetAsync(tc_err, 0, sizeof(int), st));
		ECUDA_TRY(cudaMemsetAsync(info, 0, 4 * sizeof(int), st));
		// pinned, once per host thread (a page-locked allocation per solve can
		// stall for a long time in a process that holds much pinned memory)
		static thread_local small_out *pinned = nullptr;
		if (!pinned) ECUDA_TRY(cudaMallocHost(&pinned, sizeof(small_out)));
		hsmall = pinned;
		return FMX_OK;
	}

	~solver()
	{
		cudaStreamSynchronize(st);
		if (mt) fmx_matrix_free(mt);
	}

	// tensor-core dense products: mixed precision, low-precision phase only
	// (3xTF32 is accurate to about 1e-5 relative, which would floor the
	// residuals there)
	bool lowp = false;
	bool tensor_cores() const { return lowp; }
	// mixed precision: the filter runs in correction form on BF16 operands and
	// the Rayleigh-Ritz step leaves R = A_s X - X Theta in NX
	bool corr = false;

	// Y (n x b) -> orthonormal Q (n x b) by two passes of CholQR; the first
	// is shifted.  `pass` selects the chol info slot pair (0 or 2).
	int cholqr2(const float *Y, float *tmp, float *Q)
	{
		const float *in = Y;
		float *outs[2] = {tmp, Q};
		for (int p = 0; p < 2; p++) {
			E_TRY(fmx_dense_gram(FMX_DENSE_F64, in, b, b, in, b, b, n, gpart, G, nullptr, st));
			if (p == 0) {
				shift_diag_kernel<<<1, 1, 0, st>>>(G, b, 1e-13);
				ECUDA_TRY(cudaGetLastError());
			}
			E_TRY(fmx_dense_chol_inv(G, b, T, info + p, st));
			// The Gram stays FP64 in both modes: the filtered block can be
			// ill-conditioned and the Cholesky needs its accuracy.  The update
			// runs on the tensor cores in the low-precision phase (139 us at
			// n = 4.2M, b = 16; the FP64 row stream takes 114 us, and using it
			// here too measured 0.2 ms faster per mixed solve at R-MAT scale 22).
			if (tensor_cores()) {
				f64_to_f32_kernel<<<1, 256, 0, st>>>(T, Tf, b * b);
				ECUDA_TRY(cudaGetLastError());
				E_TRY(fmx_dense_gemm(FMX_DENSE_TF32X3, in, b, n, b, Tf, b, b, outs[p], b, tc_err, st));
			} else {
				launch_ritz<false, false, true>(ritz_grid, st, in, nullptr, b, T, nullptr, nullptr, outs[p], nullptr, n,
						nullptr, 0);
				ECUDA_TRY(cudaGetLastError());
			}
			in = outs[p];
		}
		return FMX_OK;
	}

	// Rayleigh-Ritz on the orthonormal Q: X, NX, sorted Ritz values and
	// residual partials; copies the small results to the host (synchronises).
	int rayleigh_ritz(const float *Q)
	{
		E_TRY(spmm(FMX_F32, Q, b, W));
		// The Rayleigh quotient Q^T W stays an FP64 Gram in both modes.  The
		// 3xTF32 tensor-core Gram is faster at b = 16 (165 against 263 us at
		// n = 4.2M), but its 7e-5 relative error reaches Theta and through it
		// the correction form's R = A X - X Theta: at R-MAT scale 22 the mixed
		// solve then took a fifth filter pass (51 SpMMs, 66 ms, against 42 and
		// 55 ms).
		E_TRY(fmx_dense_gram(FMX_DENSE_F64, Q, b, b, W, b, b, n, gpart, H, nullptr, st));
		E_TRY(fmx_dense_sym_eig(H, b, wv, V, st));
		order_kernel<<<1, 1, 0, st>>>(wv, b, o.which == FMX_EIGEN_LM, perm, dsmall->theta);
		ECUDA_TRY(cudaGetLastError());
		launch_ritz<true, true, true>(ritz_grid, st, Q, W, b, V, perm, dsmall->theta, X, NX, n, part, int(corr));
		ECUDA_TRY(cudaGetLastError());
		return finish_small();
	}

	int finish_small()
	{
		reduce_parts_kernel<<<(2 * b + 7) / 8, 256, 0, st>>>(part, ritz_grid, 2 * b, dsmall->res2);
		ECUDA_TRY(cudaGetLastError());
		ECUDA_TRY(cudaMemcpyAsync(dsmall->chol_info, info, 4 * sizeof(int), cudaMemcpyDeviceToDevice, st));
		ECUDA_TRY(cudaMemcpyAsync(&dsmall->tc_err, tc_err, sizeof(int), cudaMemcpyDeviceToDevice, st));
		ECUDA_TRY(cudaMemcpyAsync(hsmall, dsmall, sizeof(small_out), cudaMemcpyDeviceToHost, st));
		ECUDA_TRY(cudaStreamSynchronize(st));
		if (hsmall->tc_err) return set_error(FMX_ERR_CUDA, "a tensor-core wait ran out of time");
		if (hsmall->chol_info[0] || hsmall->chol_info[1])
			return set_error(FMX_ERR_UNSUPPORTED, "CholQR broke down: the filtered block lost rank "
					"(pivot %d / %d); lower the Chebyshev degree", hsmall->chol_info[0], hsmall->chol_info[1]);
		return FMX_OK;
	}

	double residual(int j) const
	{
		const double norm_a = std::max(std::fabs(o.lower), std::fabs(o.upper));
		const double x2 = hsmall->res2[b + j];
		return std::sqrt(hsmall->res2[j] / (x2 > 0 ? x2 : 1.0)) / (norm_a > 0 ? norm_a : 1.0);
	}
	double max_residual(int cnt) const
	{
		double r = 0;
		for (int j = 0; j < cnt; j++) r = std::max(r, residual(j));
		return r;
	}

	// Explicit check of the current X: W = A_s X, residuals against theta.
	int explicit_check()
	{
		E_TRY(spmm(FMX_F32, X, b, W));
		launch_ritz<true, true, false>(ritz_grid, st, X, W, b, eye, nullptr, dsmall->theta, nullptr, nullptr, n, part, 0);
		ECUDA_TRY(cudaGetLastError());
		return finish_small();
	}

	template <class YT, class PT, class OT>
	int cheb(const float *Wm, const YT *Y, const PT *P, OT *Out, float alpha, float c0, float beta)
	{
		const int64_t cnt = n * b;
		cheb_kernel<YT, PT, OT><<<flat_grid(cnt), kThreads, 0, st>>>(Wm, Y, P, Out, cnt, alpha, c0, beta);
		ECUDA_TRY(cudaGetLastError());
		return FMX_OK;
	}

	// Y_m = p_m(A_s) X into B[k] (FP32); returns k.  Y_1 comes from NX = A_s X.
	int filter(double cut, int mdeg, int *out_k)
	{
		double lo = o.lower, up = o.upper;
		if (o.which == FMX_EIGEN_LM) lo = -cut;
		const double e = std::max((cut - lo) / 2, 1e-12 * (up - lo));
		const double c0 = (cut + lo) / 2;
		const double s1 = e / (up - c0);
		double sj = s1;
		E_TRY(cheb(NX, X, (const float *)nullptr, B[0], float(s1 / e), float(c0), 0.f));
		int cur = 0, prev = -1;                           // prev -1 = X
		for (int j = 2; j <= mdeg; j++) {
			const double sn = 1.0 / (2.0 / s1 - sj);
			E_TRY(spmm(FMX_F32, B[cur], b, W));
			const int nxt = (cur + 1) % 3 == prev ? (cur + 2) % 3 : (cur + 1) % 3;
			const float *P = prev < 0 ? X : B[prev];
			E_TRY(cheb(W, (const float *)B[cur], P, B[nxt], float(2 * sn / e), float(c0), float(sj * sn)));
			prev = cur;
			cur = nxt;
			sj = sn;
		}
		*out_k = cur;
		return FMX_OK;
	}

	template <class WT, class ET, class PT, class RT, class OT>
	int corr_step(const WT *Wm, const ET *E, const PT *P, const RT *R, const float *Xs, OT *Out, float alpha,
			float ac0, float beta, const col_coefs &cf, __nv_bfloat16 *Rb = nullptr)
	{
		const int64_t cnt = n * b;
		corr_kernel<WT, ET, PT, RT, OT><<<flat_grid(cnt), kThreads, 0, st>>>(Wm, E, P, R, Xs, Out, cnt, b, alpha, ac0,
				beta, cf, Rb);
		ECUDA_TRY(cudaGetLastError());
		return FMX_OK;
	}

	// The same filter in correction form: Y_j = X D_j + E_j with D_j =
	// p_j(Theta) (diagonal, carried on the host) and
	//   E_1 = a_1 R,   E_j = a_j (A_s E_{j-1} - c0 E_{j-1} + R D_{j-1}) - b_j E_{j-2},
	// where R = A_s X - X Theta comes from the last Rayleigh-Ritz step.  The
	// SpMMs act on E_j in BF16: their rounding error is relative to the
	// correction, which shrinks with the residual, so BF16 operands do not
	// floor the attainable accuracy.  Y_m = X D_m + E_m is written in FP32.
	int filter_corr(double cut, int mdeg, int *out_k)
	{
		double lo = o.lower, up = o.upper;
		if (o.which == FMX_EIGEN_LM) lo = -cut;
		const double e = std::max((cut - lo) / 2, 1e-12 * (up - lo));
		const double c0 = (cut + lo) / 2;
		const double s1 = e / (up - c0);
		typedef __nv_bfloat16 bf;
		const float *R = NX;
		std::vector<double> Dp(b, 1.0), Dc(b), Dn(b);     // D_{j-2}, D_{j-1}, D_j
		for (int j = 0; j < b; j++) Dc[j] = (s1 / e) * (hsmall->theta[j] - c0);
		col_coefs cf{};
		// E_1 (or Y_1 when m = 1)
		for (int j = 0; j < b; j++) {
			cf.r[j] = float(s1 / e);
			cf.x[j] = float(Dc[j]);
		}
		if (mdeg == 1) {
			E_TRY(corr_step((const float *)nullptr, (const float *)nullptr, (const float *)nullptr, R, X, B[0], 0.f,
					0.f, 0.f, cf));
			*out_k = 0;
			return FMX_OK;
		}
		// E_1, and R in BF16 for the middle steps (their BF16 operands carry
		// the same relative rounding)
		E_TRY(corr_step((const float *)nullptr, (const float *)nullptr, (const float *)nullptr, R,
				(const float *)nullptr, (bf *)B[0], 0.f, 0.f, 0.f, cf, Rb));
		int cur = 0, prev = -1;
		double sj = s1;
		for (int jdeg = 2; jdeg <= mdeg; jdeg++) {
			const double sn = 1.0 / (2.0 / s1 - sj);
			const double alpha = 2 * sn / e, beta = sj * sn;
			const bool last = jdeg == mdeg;
			// W = A_s E in BF16 too: its rounding is relative to the correction
			E_TRY(spmm(FMX_BF16, B[cur], b, W, FMX_BF16));
			for (int j = 0; j < b; j++) {
				Dn[j] = alpha * (hsmall->theta[j] - c0) * Dc[j] - beta * Dp[j];
				cf.r[j] = float(alpha * Dc[j]);
				cf.x[j] = float(Dn[j]);
			}
			const int nxt = (cur + 1) % 3 == prev ? (cur + 2) % 3 : (cur + 1) % 3;
			const bf *E = (const bf *)B[cur];
			const bf *P = prev < 0 ? nullptr : (const bf *)B[prev];
			const float a = float(alpha), ac = float(alpha * c0), bt = float(beta);
			const bf *Wb = (const bf *)W;
			if (last) E_TRY(corr_step(Wb, E, P, R, X, B[nxt], a, ac, bt, cf));
			else E_TRY(corr_step(Wb, E, P, (const bf *)Rb, (const float *)nullptr, (bf *)B[nxt], a, ac, bt, cf));
			prev = cur;
			cur = nxt;
			sj = sn;
			Dp.swap(Dc);
			Dc.swap(Dn);
		}
		*out_k = cur;
		return FMX_OK;
	}

	// Filter degree for the next pass (the per-vector degree rule of ChASE,
	// Winkelmann et al., ACM TOMS 45(2), 2019, applied to the slowest wanted
	// vector): a Ritz pair at theta_j, with the damped interval [lo, cut]
	// mapped to [-1, 1], has its residual divided by about T_m(t_j), t_j =
	// (theta_j - c0) / e, after m steps.  So m = acosh(r_j / tol) / acosh(t_j),
	// rounded up, at least 2 and at most o.degree; o.degree when a wanted
	// Ritz value lies inside the damped interval.
	int degree_for(double cut) const
	{
		double lo = o.lower;
		if (o.which == FMX_EIGEN_LM) lo = -cut;
		const double e = std::max((cut - lo) / 2, 1e-12 * (o.upper - o.lower));
		const double c0 = (cut + lo) / 2;
		const double target = 0.5 * o.tol;
		double m = 2;
		for (int j = 0; j < o.nev; j++) {
			const double r = residual(j);
			if (r <= target) continue;
			const double th = o.which == FMX_EIGEN_LM ? std::fabs(hsmall->theta[j]) : hsmall->theta[j];
			const double t = (th - c0) / e;
			if (!(t > 1.0 + 1e-9)) return max_degree();
			m = std::max(m, std::ceil(std::acosh(r / target) / std::acosh(t)));
		}
		return int(std::min<double>(m, max_degree()));
	}

	// In correction form the BF16 error of the recurrence grows with its
	// length, so the mixed mode filters with at most 10 steps.  Measured on
	// R-MAT scale 22 (top 8): cap 8 57.1 ms, 10 55.2 ms, 12 58.1 ms, 16 61.8 ms;
	// on 40 held-out SBM graphs cap 10 took 4 % less total time than cap 8.
	int max_degree() const { return corr ? std::min(o.degree, kMixedMaxDegree) : o.degree; }

	int run(double *evals, float *evecs, int64_t ldv, double *residuals, fmx_eigen_status *status)
	{
		const auto t0 = std::chrono::steady_clock::now();
		E_TRY(setup());
		lowp = o.precision == FMX_EIGEN_MIXED;
		corr = o.precision == FMX_EIGEN_MIXED;
		// start block
		if (o.X0 && o.ldx0 == b) {
			// one linear copy: a pitched copy of n 64-byte rows took 0.45 ms
			// at n = 4.2M against 0.08 ms
			ECUDA_TRY(cudaMemcpyAsync(B[0], o.X0, size_t(n) * b * sizeof(float), cudaMemcpyDeviceToDevice, st));
		} else if (o.X0) {
			ECUDA_TRY(cudaMemcpy2DAsync(B[0], size_t(b) * sizeof(float), o.X0, size_t(o.ldx0) * sizeof(float),
					size_t(b) * sizeof(float), size_t(n), cudaMemcpyDeviceToDevice, st));
		} else {
			random_block_kernel<<<flat_grid(n * b), kThreads, 0, st>>>(B[0], n * b, o.seed);
			ECUDA_TRY(cudaGetLastError());
		}
		E_TRY(cholqr2(B[0], B[1], B[2]));
		E_TRY(rayleigh_ritz(B[2]));
		int iters = 0, converged = 0;
		double maxres = max_residual(o.nev);
		const double tau = 1.1;                      // least amplification of the top end
		bool checked = false;
		while (true) {
			if (maxres <= o.tol) {
				// confirm with an explicit product of the returned vectors
				E_TRY(explicit_check());
				maxres = max_residual(o.nev);
				checked = true;
				if (maxres <= o.tol) break;
			}
			if (iters >= o.max_iters) break;
			iters++;
			double cut = o.which == FMX_EIGEN_LM ? std::fabs(hsmall->theta[b - 1]) : hsmall->theta[b - 1];
			double cap;
			if (o.which == FMX_EIGEN_LM) cap = o.upper / tau;
			else cap = (2 * o.upper - o.lower * (1 - tau)) / (1 + tau);
			cut = std::min(cut, cap);
			if (o.which == FMX_EIGEN_LA) cut = std::max(cut, o.lower + 1e-6 * (o.upper - o.lower));
			else cut = std::max(cut, 1e-6 * o.upper);
			lowp = o.precision == FMX_EIGEN_MIXED && maxres > o.tensor_until;
			int k = 0;
			const int mdeg = degree_for(cut);
			if (corr) E_TRY(filter_corr(cut, mdeg, &k));
			else E_TRY(filter(cut, mdeg, &k));
			E_TRY(cholqr2(B[k], B[(k + 1) % 3], B[(k + 2) % 3]));
			E_TRY(rayleigh_ritz(B[(k + 2) % 3]));
			maxres = max_residual(o.nev);
			checked = false;
			lowp = false;
		}
		if (!checked) {
			E_TRY(explicit_check());
			maxres = max_residual(o.nev);
		}
		for (int j = 0; j < o.nev; j++)
			if (residual(j) <= o.tol) converged++;
		if (evals)
			for (int j = 0; j < o.nev; j++) evals[j] = hsmall->theta[j];
		if (residuals)
			for (int j = 0; j < o.nev; j++) residuals[j] = residual(j);
		if (evecs && n > 0) {
			copy_cols_kernel<<<flat_grid(n * o.nev), kThreads, 0, st>>>(X, b, evecs, ldv, n, o.nev);
			ECUDA_TRY(cudaGetLastError());
		}
		ECUDA_TRY(cudaStreamSynchronize(st));
		if (status) {
			status->iters = iters;
			status->converged = converged;
			status->num_ops = num_ops;
			status->spmm_calls = spmm_calls;
			status->max_residual = maxres;
			status->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
		}
		return FMX_OK;
	}
};

} // namespace eig
} // namespace fmx

using namespace fmx;
using namespace fmx::eig;

extern "C" {

void fmx_eigen_default_options(fmx_eigen_options *o, int nev)
{
	if (!o) return;
	std::memset(o, 0, sizeof(*o));
	o->nev = nev;
	o->block_size = std::min(kMaxB, std::max(2 * nev, 16));
	o->degree = 16;
	o->max_iters = 500;
	o->which = FMX_EIGEN_LA;
	o->precision = FMX_EIGEN_PLAIN;
	o->tol = 1e-8;
	o->lower = -1.0;
	o->upper = 1.0;
	o->tensor_until = 1e-3;
	o->seed = 1;
	o->X0 = nullptr;
	o->ldx0 = 0;
	o->op = FMX_EIGEN_OP_SCALED;
}

int fmx_eigen_solve(const fmx_matrix *m, const float *row_scale, const fmx_eigen_options *opt, double *evals,
		float *evecs, int64_t ldv, double *residuals, fmx_eigen_status *status, void *stream)
{
	if (!m || !opt) return set_error(FMX_ERR_INVAL, "null matrix or options");
	device_guard on_device(matrix_device(m));
	if (!on_device.ok()) return set_error(FMX_ERR_CUDA, "cannot make the matrix's device %d current", matrix_device(m));
	uint64_t nrows = 0, ncols = 0, nnz = 0;
	int prim = 0;
	E_TRY(fmx_matrix_info(m, &nrows, &ncols, &nnz, &prim, nullptr));
	const fmx_eigen_options &o = *opt;
	if (o.op != FMX_EIGEN_OP_SCALED && o.op != FMX_EIGEN_OP_GRAM)
		return set_error(FMX_ERR_INVAL, "op: FMX_EIGEN_OP_SCALED or FMX_EIGEN_OP_GRAM");
	if (o.op == FMX_EIGEN_OP_SCALED && nrows != ncols)
		return set_error(FMX_ERR_DIM, "the eigensolver needs a square matrix (%llu x %llu)",
				(unsigned long long)nrows, (unsigned long long)ncols);
	if (o.op == FMX_EIGEN_OP_GRAM && row_scale)
		return set_error(FMX_ERR_INVAL, "the Gram operator A^T A takes no row scale");
	if (o.block_size < 1 || o.block_size > kMaxB) return set_error(FMX_ERR_UNSUPPORTED, "block_size in 1..%d", kMaxB);
	if (o.nev < 1 || o.nev > o.block_size) return set_error(FMX_ERR_INVAL, "nev in 1..block_size (got %d, %d)", o.nev,
			o.block_size);
	if (uint64_t(o.block_size) > ncols) return set_error(FMX_ERR_DIM, "block_size exceeds the matrix size");
	if (o.degree < 1 || o.degree > 100) return set_error(FMX_ERR_INVAL, "degree in 1..100");
	if (o.which != FMX_EIGEN_LA && o.which != FMX_EIGEN_LM) return set_error(FMX_ERR_INVAL, "which: LA or LM");
	if (o.precision != FMX_EIGEN_PLAIN && o.precision != FMX_EIGEN_MIXED)
		return set_error(FMX_ERR_INVAL, "precision: plain or mixed");
	if (!(o.upper > o.lower)) return set_error(FMX_ERR_INVAL, "spectrum bounds need lower < upper");
	if (o.X0 && o.ldx0 < o.block_size) return set_error(FMX_ERR_DIM, "ldx0 < block_size");
	if (evecs && ldv < o.nev) return set_error(FMX_ERR_DIM, "ldv < nev");
	if (prim != FMX_P_BOOL && prim != FMX_P_FLOAT)
		return set_error(FMX_ERR_TYPE, "the eigensolver takes binary or float-weighted matrices");
	solver sv;
	sv.m = m;
	if (o.op == FMX_EIGEN_OP_GRAM) E_TRY(fmx_matrix_transpose(m, &sv.mt));
	sv.nrows = int64_t(nrows);
	sv.s = o.op == FMX_EIGEN_OP_GRAM ? nullptr : row_scale;
	sv.o = o;
	sv.n = int64_t(ncols);
	sv.b = o.block_size;
	sv.st = static_cast<cudaStream_t>(stream);
	return sv.run(evals, evecs, ldv, residuals, status);
}

int fmx_na_scale(const fmx_matrix *m, float *s, void *stream)
{
	if (!m || !s) return set_error(FMX_ERR_INVAL, "null argument");
	device_guard on_device(matrix_device(m));
	if (!on_device.ok()) return set_error(FMX_ERR_CUDA, "cannot make the matrix's device %d current", matrix_device(m));
	uint64_t nrows = 0, ncols = 0, nnz = 0;
	int prim = 0;
	E_TRY(fmx_matrix_info(m, &nrows, &ncols, &nnz, &prim, nullptr));
	if (nrows != ncols) return set_error(FMX_ERR_DIM, "D^-1/2 A D^-1/2 needs a square matrix");
	if (prim != FMX_P_BOOL && prim != FMX_P_FLOAT) return set_error(FMX_ERR_TYPE, "binary or float-weighted matrices");
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	workspace ws;
	ws.st = st;
	float *ones = nullptr, *deg = nullptr;
	const int64_t n = int64_t(nrows);
	E_TRY(ws.get(&ones, size_t(n)));
	E_TRY(ws.get(&deg, size_t(n)));
	fill_kernel<<<flat_grid(n), kThreads, 0, st>>>(ones, n, 1.f);
	ECUDA_TRY(cudaGetLastError());
	E_TRY(fmx_spmm(m, FMX_F32, ones, 1, FMX_F32, deg, 1, 1, nullptr, nullptr, stream));
	inv_sqrt_kernel<<<flat_grid(n), kThreads, 0, st>>>(deg, s, n);
	ECUDA_TRY(cudaGetLastError());
	return FMX_OK;
}

} // extern "C"
