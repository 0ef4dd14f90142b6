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
//   FMX_EIGEN_MIXED  while the largest wanted residual exceeds `bf16_until`
//                    (the low-precision phase): BF16 SpMM operands (FP32
//                    accumulation), and the CholQR basis update and the
//                    Rayleigh quotient Q^T W on tensor cores (3xTF32,
//                    tcgen05); the CholQR Gram, the Cholesky factor, the
//                    projected eigenproblem and the residual norms stay FP64.
//                    After it, the passes are those of the plain mode (3xTF32
//                    is accurate to about 1e-5 relative, too coarse for the
//                    last digits of a 1e-6 residual).
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

// Basis update with FP64 accumulation, on row tiles of the n x b blocks:
//   X[r][j] = sum_k Q[r][k] V[k][perm j]       (written when WRITE)
//   NX[r][j] = sum_k W[r][k] V[k][perm j]      (HAS_W; written when WRITE)
//   part[cta][j] += (NX[r][j] - theta[j] X[r][j])^2, part[cta][b + j] += X[r][j]^2   (RES)
// Partials are summed in a fixed order (deterministic).
template <bool HAS_W, bool RES, bool WRITE>
__global__ void __launch_bounds__(kThreads)
ritz_kernel(const float *__restrict__ Q, const float *__restrict__ W, int b, const double *__restrict__ V,
		const int *__restrict__ perm, const double *__restrict__ theta, float *__restrict__ X,
		float *__restrict__ NX, int64_t n, double *__restrict__ part)
{
	__shared__ double sV[kMaxB * kMaxB];
	__shared__ float sQ[kThreads], sW[kThreads];
	__shared__ double red[2 * kThreads];
	const int tid = threadIdx.x;
	const int R = kThreads / b;                  // rows per tile
	for (int i = tid; i < b * b; i += kThreads) {
		const int k = i / b, j = i % b;
		sV[k * kMaxB + j] = V[k * b + (perm ? perm[j] : j)];
	}
	const int r = tid / b, j = tid % b;
	const bool active = r < R;
	const double th = (RES && active) ? theta[j] : 0.0;
	double acc_r = 0, acc_x = 0;
	for (int64_t r0 = int64_t(blockIdx.x) * R; r0 < n; r0 += int64_t(gridDim.x) * R) {
		__syncthreads();
		const int64_t base = r0 * b;
		const int64_t lim = min(int64_t(R), n - r0) * b;
		if (tid < lim) {
			sQ[tid] = Q[base + tid];
			if (HAS_W) sW[tid] = W[base + tid];
		}
		__syncthreads();
		if (active && r0 + r < n) {
			double x = 0, y = 0;
			for (int k = 0; k < b; k++) {
				const double v = sV[k * kMaxB + j];
				x += double(sQ[r * b + k]) * v;
				if (HAS_W) y += double(sW[r * b + k]) * v;
			}
			if (WRITE) {
				X[base + tid] = float(x);
				if (HAS_W) NX[base + tid] = float(y);
			}
			if (RES) {
				const double d = y - th * x;
				acc_r += d * d;
				acc_x += x * x;
			}
		}
	}
	if (RES) {
		__syncthreads();
		red[tid] = acc_r;
		red[kThreads + tid] = acc_x;
		__syncthreads();
		if (tid < b) {
			double sr = 0, sx = 0;
			for (int q = 0; q < R; q++) {
				sr += red[q * b + tid];
				sx += red[kThreads + q * b + tid];
			}
			part[size_t(blockIdx.x) * 2 * b + tid] = sr;
			part[size_t(blockIdx.x) * 2 * b + b + tid] = sx;
		}
	}
}

__global__ void reduce_parts_kernel(const double *__restrict__ part, int nparts, int len, double *__restrict__ out)
{
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x) {
		double s = 0;
		for (int p = 0; p < nparts; p++) s += part[size_t(p) * len + i];
		out[i] = s;
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
__global__ void f32_to_f64_kernel(const float *a, double *o, int count)
{
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) o[i] = double(a[i]);
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
		cudaError_t e = cudaMallocAsync(&q, std::max<size_t>(count, 1) * sizeof(T), st);
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
	const float *s;                  // row scale or null
	fmx_eigen_options o;
	int64_t n;
	int b;
	cudaStream_t st;
	workspace ws;
	float *X = nullptr, *NX = nullptr, *W = nullptr, *B[3] = {nullptr, nullptr, nullptr};
	double *G = nullptr, *T = nullptr, *H = nullptr, *wv = nullptr, *V = nullptr, *eye = nullptr;
	double *part = nullptr, *dsmall_theta = nullptr;
	float *Tf = nullptr, *Hf = nullptr, *gpart = nullptr;
	int *perm = nullptr, *tc_err = nullptr, *info = nullptr;
	small_out *dsmall = nullptr, *hsmall = nullptr;
	int ritz_grid = 1;
	int64_t spmm_calls = 0, num_ops = 0;

	int spmm(int xt, const void *Xin, int k, float *Out)
	{
		E_TRY(fmx_spmm(m, xt, Xin, b, FMX_F32, Out, b, k, s, s, st));
		spmm_calls++;
		num_ops += k;
		return FMX_OK;
	}

	int setup()
	{
		ws.st = st;
		const size_t nb = size_t(n) * b;
		E_TRY(ws.get(&X, nb));
		E_TRY(ws.get(&NX, nb));
		E_TRY(ws.get(&W, nb));
		for (auto &p : B) E_TRY(ws.get(&p, nb));
		E_TRY(ws.get(&G, b * b));
		E_TRY(ws.get(&T, b * b));
		E_TRY(ws.get(&H, b * b));
		E_TRY(ws.get(&wv, b));
		E_TRY(ws.get(&V, b * b));
		E_TRY(ws.get(&eye, b * b));
		E_TRY(ws.get(&Tf, b * b));
		E_TRY(ws.get(&Hf, b * b));
		E_TRY(ws.get(&perm, b));
		E_TRY(ws.get(&tc_err, 1));
		E_TRY(ws.get(&info, 4));
		E_TRY(ws.get(&dsmall, 1));
		const int R = kThreads / b;
		ritz_grid = int(std::max<int64_t>(1, std::min<int64_t>((n + R - 1) / R, int64_t(sm_count()) * 4)));
		E_TRY(ws.get(&part, size_t(ritz_grid) * 2 * b));
		const int gparts = std::max({fmx_dense_gram_parts(FMX_DENSE_F64, n), fmx_dense_gram_parts(FMX_DENSE_TF32X3, n)});
		E_TRY(ws.get(&gpart, size_t(gparts) * b * b * 2));      // room for double partials
		std::vector<double> I(size_t(b) * b, 0.0);
		for (int i = 0; i < b; i++) I[size_t(i) * b + i] = 1.0;
		ECUDA_TRY(cudaMemcpyAsync(eye, I.data(), I.size() * sizeof(double), cudaMemcpyHostToDevice, st));
		ECUDA_TRY(cudaMemsetAsync(tc_err, 0, sizeof(int), st));
		ECUDA_TRY(cudaMemsetAsync(info, 0, 4 * sizeof(int), st));
		ECUDA_TRY(cudaMallocHost(&hsmall, sizeof(small_out)));
		return FMX_OK;
	}

	~solver()
	{
		if (hsmall) {
			cudaStreamSynchronize(st);
			cudaFreeHost(hsmall);
		}
	}

	// tensor-core dense products: mixed precision, low-precision phase only
	// (3xTF32 is accurate to about 1e-5 relative, which would floor the
	// residuals there)
	bool lowp = false;
	bool tensor_cores() const { return lowp; }

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
			if (tensor_cores()) {
				f64_to_f32_kernel<<<1, 256, 0, st>>>(T, Tf, b * b);
				ECUDA_TRY(cudaGetLastError());
				E_TRY(fmx_dense_gemm(FMX_DENSE_TF32X3, in, b, n, b, Tf, b, b, outs[p], b, tc_err, st));
			} else {
				ritz_kernel<false, false, true><<<ritz_grid, kThreads, 0, st>>>(in, nullptr, b, T, nullptr, nullptr,
						outs[p], nullptr, n, nullptr);
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
		if (tensor_cores()) {
			E_TRY(fmx_dense_gram(FMX_DENSE_TF32X3, Q, b, b, W, b, b, n, gpart, Hf, tc_err, st));
			f32_to_f64_kernel<<<1, 256, 0, st>>>(Hf, H, b * b);
			ECUDA_TRY(cudaGetLastError());
		} else {
			E_TRY(fmx_dense_gram(FMX_DENSE_F64, Q, b, b, W, b, b, n, gpart, H, nullptr, st));
		}
		E_TRY(fmx_dense_sym_eig(H, b, wv, V, st));
		order_kernel<<<1, 1, 0, st>>>(wv, b, o.which == FMX_EIGEN_LM, perm, dsmall->theta);
		ECUDA_TRY(cudaGetLastError());
		ritz_kernel<true, true, true><<<ritz_grid, kThreads, 0, st>>>(Q, W, b, V, perm, dsmall->theta, X, NX, n, part);
		ECUDA_TRY(cudaGetLastError());
		return finish_small();
	}

	int finish_small()
	{
		reduce_parts_kernel<<<1, 128, 0, st>>>(part, ritz_grid, 2 * b, dsmall->res2);
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
		ritz_kernel<true, true, false><<<ritz_grid, kThreads, 0, st>>>(X, W, b, eye, nullptr, dsmall->theta, nullptr,
				nullptr, n, part);
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

	// Y_m = p_m(A_s) X into B[k]; returns k.  Y_1 comes from NX = A_s X.
	int filter(double cut, bool lowp, int *out_k)
	{
		const int mdeg = o.degree;
		double lo = o.lower, up = o.upper;
		if (o.which == FMX_EIGEN_LM) lo = -cut;
		const double e = std::max((cut - lo) / 2, 1e-12 * (up - lo));
		const double c0 = (cut + lo) / 2;
		const double s1 = e / (up - c0);
		double sj = s1;
		typedef __nv_bfloat16 bf;
		// Y1 (index 0 in B)
		int cur = 0;
		const bool last1 = mdeg == 1;
		if (lowp && !last1) E_TRY(cheb(NX, X, (const float *)nullptr, (bf *)B[0], float(s1 / e), float(c0), 0.f));
		else E_TRY(cheb(NX, X, (const float *)nullptr, B[0], float(s1 / e), float(c0), 0.f));
		int prev = -1;                                    // -1 = X
		for (int j = 2; j <= mdeg; j++) {
			const double sn = 1.0 / (2.0 / s1 - sj);
			const float alpha = float(2 * sn / e), beta = float(sj * sn);
			const bool cur_bf = lowp;                     // Y_{j-1} is BF16 when lowp (j - 1 < m)
			const bool prev_bf = lowp && prev >= 0;
			const bool out_bf = lowp && j < mdeg;
			E_TRY(spmm(cur_bf ? FMX_BF16 : FMX_F32, B[cur], b, W));
			const int nxt = (cur + 1) % 3 == prev ? (cur + 2) % 3 : (cur + 1) % 3;
			const void *P = prev < 0 ? static_cast<const void *>(X) : static_cast<const void *>(B[prev]);
			int rc;
			if (cur_bf) {
				const bf *Y = (const bf *)B[cur];
				if (prev_bf) rc = out_bf ? cheb(W, Y, (const bf *)P, (bf *)B[nxt], alpha, float(c0), beta)
				                         : cheb(W, Y, (const bf *)P, B[nxt], alpha, float(c0), beta);
				else rc = out_bf ? cheb(W, Y, (const float *)P, (bf *)B[nxt], alpha, float(c0), beta)
				                 : cheb(W, Y, (const float *)P, B[nxt], alpha, float(c0), beta);
			} else {
				rc = cheb(W, (const float *)B[cur], (const float *)P, B[nxt], alpha, float(c0), beta);
			}
			E_TRY(rc);
			prev = cur;
			cur = nxt;
			sj = sn;
		}
		*out_k = cur;
		return FMX_OK;
	}

	int run(double *evals, float *evecs, int64_t ldv, double *residuals, fmx_eigen_status *status)
	{
		const auto t0 = std::chrono::steady_clock::now();
		E_TRY(setup());
		lowp = o.precision == FMX_EIGEN_MIXED;
		// start block
		if (o.X0) {
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
			lowp = o.precision == FMX_EIGEN_MIXED && maxres > o.bf16_until;
			int k = 0;
			E_TRY(filter(cut, lowp, &k));
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
		if (evecs) {
			ECUDA_TRY(cudaMemcpy2DAsync(evecs, size_t(ldv) * sizeof(float), X, size_t(b) * sizeof(float),
					size_t(o.nev) * sizeof(float), size_t(n), cudaMemcpyDeviceToDevice, st));
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
	o->degree = 10;
	o->max_iters = 500;
	o->which = FMX_EIGEN_LA;
	o->precision = FMX_EIGEN_PLAIN;
	o->tol = 1e-8;
	o->lower = -1.0;
	o->upper = 1.0;
	o->bf16_until = 1e-2;
	o->seed = 1;
	o->X0 = nullptr;
	o->ldx0 = 0;
}

int fmx_eigen_solve(const fmx_matrix *m, const float *row_scale, const fmx_eigen_options *opt, double *evals,
		float *evecs, int64_t ldv, double *residuals, fmx_eigen_status *status, void *stream)
{
	if (!m || !opt) return set_error(FMX_ERR_INVAL, "null matrix or options");
	uint64_t nrows = 0, ncols = 0, nnz = 0;
	int prim = 0;
	E_TRY(fmx_matrix_info(m, &nrows, &ncols, &nnz, &prim, nullptr));
	if (nrows != ncols) return set_error(FMX_ERR_DIM, "the eigensolver needs a square matrix (%llu x %llu)",
			(unsigned long long)nrows, (unsigned long long)ncols);
	const fmx_eigen_options &o = *opt;
	if (o.block_size < 1 || o.block_size > kMaxB) return set_error(FMX_ERR_UNSUPPORTED, "block_size in 1..%d", kMaxB);
	if (o.nev < 1 || o.nev > o.block_size) return set_error(FMX_ERR_INVAL, "nev in 1..block_size (got %d, %d)", o.nev,
			o.block_size);
	if (uint64_t(o.block_size) > nrows) return set_error(FMX_ERR_DIM, "block_size exceeds the matrix size");
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
	sv.s = row_scale;
	sv.o = o;
	sv.n = int64_t(nrows);
	sv.b = o.block_size;
	sv.st = static_cast<cudaStream_t>(stream);
	return sv.run(evals, evecs, ldv, residuals, status);
}

int fmx_na_scale(const fmx_matrix *m, float *s, void *stream)
{
	if (!m || !s) return set_error(FMX_ERR_INVAL, "null argument");
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
