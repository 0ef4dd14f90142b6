// SpMM on B200 (sm_100a): Y = diag(s_out) * A * diag(s_in) * X.
//
// Replaces FlashMatrix's CPU SpMM tasks (row_part_func / coo_func /
// block_spmm_task_impl::run_on_block, matrix/sparse_matrix.h:219-375, driven
// by block_compute_task::run, matrix/sparse_matrix.cpp:251-314).
//
// Layout in HBM (built once per matrix, kept resident):
//   row_ptr  uint32[nrows+1]   rows of the decoded 2D image, ascending
//   col      int32 [nnz]       global column ids, per row in the order the
//                              reference visits them (ascending block column,
//                              then ascending column)
//   val      entry[nnz]        only for weighted images
//   light    int32 [n_light]   rows of degree <= kLightMax, degree-sorted
//                              (descending) inside bands of kBand rows
//   tasks    split_task[]      rows longer than kLightMax: one warp per row
//                              (medium) or per kChunk-entry chunk (heavy)
//   heavy    heavy_row[]       heavy rows: their chunks' partial sums are added
//                              in chunk order by spmm_fixup_kernel
//   partial  AccT[n_partials][kPartialStride] scratch for heavy chunks
//
// Work units: a warp is split into R = floor(32/G) lane groups of G lanes;
// a group owns one output row of a light warp and sums its entries
// sequentially in ascending column order (the reference's order), loading
// each X row as G 16-byte vectors.  No atomics: every output row is written
// by exactly one group (light), one warp (medium) or the fixup warp (heavy).
#include "fmx_internal.h"

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <thread>

namespace fmx {

// ---------------------------------------------------------------------------
// Schedule parameters
// ---------------------------------------------------------------------------
constexpr uint32_t kLightMax = 512;     // rows summed by one lane group
constexpr uint32_t kHeavyMin = 16384;   // rows split into chunks above this
constexpr uint32_t kChunk = 4096;       // entries per heavy chunk
constexpr uint32_t kBand = 65536;       // degree sort stays inside row bands
constexpr int kPartialStride = 256;     // AccT slots per partial (one panel)
constexpr int kThreads = 256;           // threads per SpMM block

struct split_task {
	int32_t row;
	uint32_t start, end;
	int32_t slot;        // -1: write Y[row]; else partial slot
};
struct heavy_row {
	int32_t row;
	uint32_t first, count;
};

#define CUDA_TRY(call)                                                          \
	do {                                                                        \
		cudaError_t err__ = (call);                                             \
		if (err__ != cudaSuccess)                                               \
			return set_error(FMX_ERR_CUDA, "%s failed: %s (%s:%d)", #call,      \
					cudaGetErrorString(err__), __FILE__, __LINE__);             \
	} while (0)

// Device-resident part of one orientation of a matrix.
struct gpu_part {
	int device = 0;
	uint64_t nrows = 0, ncols = 0, nnz = 0;
	int prim = 0;
	size_t esize = 0;
	uint32_t *row_ptr = nullptr;
	int32_t *col = nullptr;
	void *val = nullptr;
	int32_t *light = nullptr;
	uint32_t n_light = 0;
	split_task *tasks = nullptr;
	uint32_t n_tasks = 0;
	heavy_row *heavy = nullptr;
	uint32_t n_heavy = 0;
	uint32_t n_partials = 0;
	void *partial = nullptr;
	uint64_t bytes = 0;
	// staging buffers of fmx_spmm_host (grow-only, guarded by stage_mu)
	std::mutex stage_mu;
	void *stage_x = nullptr, *stage_y = nullptr;
	size_t stage_xb = 0, stage_yb = 0;
	~gpu_part() {
		int cur = 0;
		cudaGetDevice(&cur);
		cudaSetDevice(device);
		void *ps[] = {row_ptr, col, val, light, tasks, heavy, partial, stage_x, stage_y};
		for (void *p : ps)
			if (p) cudaFree(p);
		cudaSetDevice(cur);
	}
};

} // namespace fmx

struct fmx_matrix {
	std::shared_ptr<fmx::gpu_part> a;    // this orientation
	std::shared_ptr<fmx::gpu_part> at;   // the transpose (null when symmetric)
	bool symmetric = true;
};

namespace fmx {

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------

// Arithmetic without contraction: dest = dest + src * w, rounded per step,
// like the reference's dest_row[j] += src_row[j] * data (no FMA).
__device__ __forceinline__ float acc_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float acc_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double acc_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double acc_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ int32_t acc_add(int32_t a, int32_t b) { return int32_t(uint32_t(a) + uint32_t(b)); }
__device__ __forceinline__ int32_t acc_mul(int32_t a, int32_t b) { return int32_t(uint32_t(a) * uint32_t(b)); }
__device__ __forceinline__ int64_t acc_add(int64_t a, int64_t b) { return int64_t(uint64_t(a) + uint64_t(b)); }
__device__ __forceinline__ int64_t acc_mul(int64_t a, int64_t b) { return int64_t(uint64_t(a) * uint64_t(b)); }

template <class A> __device__ __forceinline__ A to_acc(float v) { return A(v); }
template <class A> __device__ __forceinline__ A to_acc(double v) { return A(v); }
template <class A> __device__ __forceinline__ A to_acc(int32_t v) { return A(v); }
template <class A> __device__ __forceinline__ A to_acc(int64_t v) { return A(v); }
template <class A> __device__ __forceinline__ A to_acc(__nv_bfloat16 v) { return A(__bfloat162float(v)); }

template <class Y, class A> __device__ __forceinline__ Y from_acc(A v) { return Y(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_acc<__nv_bfloat16, float>(float v) { return __float2bfloat16_rn(v); }

// Streaming loads/stores for the index stream and the output (touched once,
// evict-first in L1 and L2) so that the gathered X rows keep the L2.
__device__ __forceinline__ int32_t ld_stream(const int32_t *p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float *p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double *p) { return __ldcs(p); }
__device__ __forceinline__ int64_t ld_stream(const int64_t *p) { return (int64_t)__ldcs((const long long *)p); }

// A 16-byte vector of VEC elements of T (VEC * sizeof(T) == 16), or a scalar.
template <class T, int VEC>
struct xvec {
	T v[VEC];
};

template <class T, int VEC>
__device__ __forceinline__ xvec<T, VEC> ld_x(const T *p)
{
	xvec<T, VEC> r;
	if constexpr (VEC * sizeof(T) == 16) {
		uint4 u = __ldg(reinterpret_cast<const uint4 *>(p));
		memcpy(&r, &u, 16);
	} else {
		static_assert(VEC == 1, "scalar path");
		r.v[0] = __ldg(p);
	}
	return r;
}
template <>
__device__ __forceinline__ xvec<__nv_bfloat16, 1> ld_x<__nv_bfloat16, 1>(const __nv_bfloat16 *p)
{
	xvec<__nv_bfloat16, 1> r;
	unsigned short u = __ldg(reinterpret_cast<const unsigned short *>(p));
	memcpy(&r.v[0], &u, 2);
	return r;
}

template <class T, int VEC>
__device__ __forceinline__ void st_y(T *p, const T (&v)[VEC])
{
	if constexpr (VEC * sizeof(T) == 16) {
		uint4 u;
		memcpy(&u, v, 16);
		__stcs(reinterpret_cast<uint4 *>(p), u);
	} else if constexpr (VEC * sizeof(T) == 32) {
		uint4 u[2];
		memcpy(u, v, 32);
		__stcs(reinterpret_cast<uint4 *>(p), u[0]);
		__stcs(reinterpret_cast<uint4 *>(p) + 1, u[1]);
	} else if constexpr (VEC * sizeof(T) == 8) {
		uint2 u;
		memcpy(&u, v, 8);
		__stcs(reinterpret_cast<uint2 *>(p), u);
	} else {
#pragma unroll
		for (int i = 0; i < VEC; i++) p[i] = v[i];
	}
}

struct spmm_args {
	const uint32_t *row_ptr;
	const int32_t *col;
	const void *val;
	const int32_t *light;
	const split_task *tasks;
	const void *X;
	void *Y;
	const void *s_in;
	const void *s_out;
	void *partial;
	int64_t ldx, ldy;
	int k;           // columns in this panel
	int G;           // lanes per row group
	int R;           // row groups per warp
	int nv;          // vectors per lane (generic path)
	uint32_t n_light;
	uint32_t n_tasks;
	uint64_t n_light_warps;
};

// WT = void for a binary matrix (every entry is 1).
template <class WT, class A>
__device__ __forceinline__ A ld_w(const void *val, uint32_t e)
{
	if constexpr (std::is_void<WT>::value) {
		return A(1);
	} else {
		return A(ld_stream(static_cast<const WT *>(val) + e));
	}
}

// Sum entries [e0, e1) of one row into acc (NV vectors of VEC per lane).
// Lane columns: c0 + v * G * VEC + [0, VEC).
template <class XT, class A, class WT, int VEC, int NV, bool SCALE_IN>
__device__ __forceinline__ void row_sum(const spmm_args &a, uint32_t e0, uint32_t e1,
		int colbase, int nv, A (&acc)[NV][VEC])
{
	const XT *X = static_cast<const XT *>(a.X);
	const A *sin = static_cast<const A *>(a.s_in);
	const int stride = a.G * VEC;
	constexpr int U = (NV == 1) ? 8 : 2;
	uint32_t e = e0;
	for (; e + U <= e1; e += U) {
		int32_t c[U];
#pragma unroll
		for (int u = 0; u < U; u++) c[u] = ld_stream(a.col + e + u);
		A w[U], sc[U];
#pragma unroll
		for (int u = 0; u < U; u++) w[u] = ld_w<WT, A>(a.val, e + u);
		if constexpr (SCALE_IN) {
#pragma unroll
			for (int u = 0; u < U; u++) sc[u] = sin[c[u]];
		}
		xvec<XT, VEC> x[U][NV];
#pragma unroll
		for (int u = 0; u < U; u++)
#pragma unroll
			for (int v = 0; v < NV; v++)
				if (v < nv && colbase + v * stride < a.k)
					x[u][v] = ld_x<XT, VEC>(X + int64_t(c[u]) * a.ldx + colbase + v * stride);
#pragma unroll
		for (int u = 0; u < U; u++)
#pragma unroll
			for (int v = 0; v < NV; v++)
				if (v < nv && colbase + v * stride < a.k)
#pragma unroll
					for (int i = 0; i < VEC; i++) {
						// (x * s_in) * w, rounded per step like scale_rows then SpMM
						A xv = to_acc<A>(x[u][v].v[i]);
						if constexpr (SCALE_IN) xv = acc_mul(xv, sc[u]);
						if constexpr (!std::is_void<WT>::value) xv = acc_mul(xv, w[u]);
						acc[v][i] = acc_add(acc[v][i], xv);
					}
	}
	for (; e < e1; e++) {
		int32_t c = ld_stream(a.col + e);
		A w = ld_w<WT, A>(a.val, e);
		A sc = A(1);
		if constexpr (SCALE_IN) sc = sin[c];
#pragma unroll
		for (int v = 0; v < NV; v++)
			if (v < nv && colbase + v * stride < a.k) {
				xvec<XT, VEC> x = ld_x<XT, VEC>(X + int64_t(c) * a.ldx + colbase + v * stride);
#pragma unroll
				for (int i = 0; i < VEC; i++) {
					A xv = to_acc<A>(x.v[i]);
					if constexpr (SCALE_IN) xv = acc_mul(xv, sc);
					if constexpr (!std::is_void<WT>::value) xv = acc_mul(xv, w);
					acc[v][i] = acc_add(acc[v][i], xv);
				}
			}
	}
}

template <class YT, class A, int VEC, int NV, bool SCALE_OUT>
__device__ __forceinline__ void store_row(const spmm_args &a, int32_t row, int colbase, int nv,
		const A (&acc)[NV][VEC])
{
	YT *Y = static_cast<YT *>(a.Y);
	A so = A(1);
	if constexpr (SCALE_OUT) so = static_cast<const A *>(a.s_out)[row];
	const int stride = a.G * VEC;
#pragma unroll
	for (int v = 0; v < NV; v++)
		if (v < nv && colbase + v * stride < a.k) {
			YT out[VEC];
#pragma unroll
			for (int i = 0; i < VEC; i++) {
				A t = acc[v][i];
				if constexpr (SCALE_OUT) t = acc_mul(t, so);
				out[i] = from_acc<YT, A>(t);
			}
			st_y<YT, VEC>(Y + int64_t(row) * a.ldy + colbase + v * stride, out);
		}
}

template <class XT, class YT, class A, class WT, int VEC, int NV, bool SCALE_IN, bool SCALE_OUT>
__global__ void __launch_bounds__(kThreads)
spmm_kernel(const spmm_args a)
{
	__shared__ A red[kThreads / 32][32][NV * VEC];
	const int lane = threadIdx.x & 31;
	const int wib = threadIdx.x >> 5;
	const uint64_t gw = (uint64_t(blockIdx.x) * kThreads + threadIdx.x) >> 5;
	const int G = a.G, R = a.R;
	const int grp = lane / G;
	const int sub = lane - grp * G;
	const int colbase = sub * VEC;
	A acc[NV][VEC];
#pragma unroll
	for (int v = 0; v < NV; v++)
#pragma unroll
		for (int i = 0; i < VEC; i++) acc[v][i] = A(0);

	if (gw < a.n_tasks) {
		// One long row (or one chunk of a heavy row) over all R groups: group g
		// sums a contiguous 1/R of the entries; the group sums are then added
		// in group order.
		const split_task t = a.tasks[gw];
		const uint32_t len = t.end - t.start;
		if (grp < R) {
			uint32_t b = t.start + uint32_t((uint64_t(len) * grp) / R);
			uint32_t e = t.start + uint32_t((uint64_t(len) * (grp + 1)) / R);
			row_sum<XT, A, WT, VEC, NV, SCALE_IN>(a, b, e, colbase, a.nv, acc);
		}
#pragma unroll
		for (int v = 0; v < NV; v++)
#pragma unroll
			for (int i = 0; i < VEC; i++) red[wib][lane][v * VEC + i] = acc[v][i];
		__syncwarp();
		if (grp == 0) {
			for (int g = 1; g < R; g++)
#pragma unroll
				for (int v = 0; v < NV; v++)
#pragma unroll
					for (int i = 0; i < VEC; i++)
						acc[v][i] = acc_add(acc[v][i], red[wib][g * G + sub][v * VEC + i]);
			if (t.slot < 0) {
				store_row<YT, A, VEC, NV, SCALE_OUT>(a, t.row, colbase, a.nv, acc);
			} else {
				A *p = static_cast<A *>(a.partial) + int64_t(t.slot) * kPartialStride;
				const int stride = G * VEC;
#pragma unroll
				for (int v = 0; v < NV; v++)
					if (v < a.nv && colbase + v * stride < a.k)
#pragma unroll
						for (int i = 0; i < VEC; i++) p[colbase + v * stride + i] = acc[v][i];
			}
		}
		return;
	}
	const uint64_t lw = gw - a.n_tasks;
	if (lw >= a.n_light_warps || grp >= R) return;
	const uint64_t li = lw * R + grp;
	if (li >= a.n_light) return;
	const int32_t row = a.light[li];
	const uint32_t e0 = a.row_ptr[row], e1 = a.row_ptr[row + 1];
	row_sum<XT, A, WT, VEC, NV, SCALE_IN>(a, e0, e1, colbase, a.nv, acc);
	store_row<YT, A, VEC, NV, SCALE_OUT>(a, row, colbase, a.nv, acc);
}

// Heavy rows: add the chunk partials in chunk order, scale, convert, store.
template <class YT, class A, bool SCALE_OUT>
__global__ void spmm_fixup_kernel(const heavy_row *heavy, uint32_t n_heavy, const A *partial,
		YT *Y, int64_t ldy, int k, const A *s_out)
{
	const uint64_t w = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (w >= n_heavy) return;
	const heavy_row h = heavy[w];
	for (int j = lane; j < k; j += 32) {
		A s = partial[int64_t(h.first) * kPartialStride + j];
		for (uint32_t c = 1; c < h.count; c++)
			s = acc_add(s, partial[int64_t(h.first + c) * kPartialStride + j]);
		if constexpr (SCALE_OUT) s = acc_mul(s, s_out[h.row]);
		Y[int64_t(h.row) * ldy + j] = from_acc<YT, A>(s);
	}
}

// ---------------------------------------------------------------------------
// Host: building the resident layout
// ---------------------------------------------------------------------------

template <class T>
static int upload(T **dst, const T *src, size_t n, uint64_t &bytes)
{
	*dst = nullptr;
	if (!n) return FMX_OK;
	cudaError_t e = cudaMalloc(reinterpret_cast<void **>(dst), n * sizeof(T));
	if (e != cudaSuccess)
		return set_error(e == cudaErrorMemoryAllocation ? FMX_ERR_OOM : FMX_ERR_CUDA,
				"cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
	bytes += n * sizeof(T);
	CUDA_TRY(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
	return FMX_OK;
}

static int make_part(const host_csr &csr, int device, std::shared_ptr<gpu_part> &out)
{
	auto p = std::make_shared<gpu_part>();
	p->device = device;
	p->nrows = csr.nrows; p->ncols = csr.ncols; p->nnz = csr.nnz;
	p->prim = csr.prim; p->esize = csr.esize;

	// schedule
	const uint64_t n = csr.nrows;
	std::vector<int32_t> light;
	std::vector<split_task> heavy_tasks, medium_tasks;
	std::vector<heavy_row> heavy;
	light.reserve(n);
	uint32_t slots = 0;
	std::vector<uint32_t> bucket_count(kLightMax + 2);
	std::vector<int32_t> band_rows;
	for (uint64_t b0 = 0; b0 < n; b0 += kBand) {
		uint64_t b1 = std::min<uint64_t>(n, b0 + kBand);
		std::fill(bucket_count.begin(), bucket_count.end(), 0);
		for (uint64_t r = b0; r < b1; r++) {
			uint32_t d = csr.row_ptr[r + 1] - csr.row_ptr[r];
			if (d <= kLightMax) bucket_count[kLightMax - d + 1]++;
		}
		// counting sort by degree, descending, stable by row
		for (uint32_t i = 1; i < bucket_count.size(); i++) bucket_count[i] += bucket_count[i - 1];
		band_rows.assign(bucket_count.back(), 0);
		for (uint64_t r = b0; r < b1; r++) {
			uint32_t d = csr.row_ptr[r + 1] - csr.row_ptr[r];
			if (d <= kLightMax) band_rows[bucket_count[kLightMax - d]++] = int32_t(r);
			else if (d <= kHeavyMin) medium_tasks.push_back({int32_t(r), csr.row_ptr[r], csr.row_ptr[r + 1], -1});
			else {
				uint32_t cnt = (d + kChunk - 1) / kChunk;
				heavy.push_back({int32_t(r), slots, cnt});
				for (uint32_t c = 0; c < cnt; c++) {
					uint32_t s = csr.row_ptr[r] + c * kChunk;
					uint32_t e = std::min(csr.row_ptr[r + 1], s + kChunk);
					heavy_tasks.push_back({int32_t(r), s, e, int32_t(slots + c)});
				}
				slots += cnt;
			}
		}
		light.insert(light.end(), band_rows.begin(), band_rows.end());
	}
	std::stable_sort(medium_tasks.begin(), medium_tasks.end(), [](const split_task &x, const split_task &y) {
		return (x.end - x.start) > (y.end - y.start);
	});
	std::vector<split_task> tasks;
	tasks.reserve(heavy_tasks.size() + medium_tasks.size());
	tasks.insert(tasks.end(), heavy_tasks.begin(), heavy_tasks.end());
	tasks.insert(tasks.end(), medium_tasks.begin(), medium_tasks.end());

	int cur = 0;
	cudaGetDevice(&cur);
	CUDA_TRY(cudaSetDevice(device));
	int rc = FMX_OK;
	uint64_t &bytes = p->bytes;
	rc = upload(&p->row_ptr, csr.row_ptr.data(), csr.row_ptr.size(), bytes);
	if (!rc) rc = upload(&p->col, csr.col.data(), csr.col.size(), bytes);
	if (!rc && csr.esize) {
		char *v = nullptr;
		rc = upload(&v, csr.val.data(), csr.val.size(), bytes);
		p->val = v;
	}
	if (!rc) rc = upload(&p->light, light.data(), light.size(), bytes);
	if (!rc) rc = upload(&p->tasks, tasks.data(), tasks.size(), bytes);
	if (!rc) rc = upload(&p->heavy, heavy.data(), heavy.size(), bytes);
	p->n_light = uint32_t(light.size());
	p->n_tasks = uint32_t(tasks.size());
	p->n_heavy = uint32_t(heavy.size());
	p->n_partials = slots;
	if (!rc && slots) {
		size_t sz = size_t(slots) * kPartialStride * 8;
		cudaError_t e = cudaMalloc(&p->partial, sz);
		if (e != cudaSuccess)
			rc = set_error(FMX_ERR_OOM, "cudaMalloc of %zu partial bytes failed: %s", sz, cudaGetErrorString(e));
		else bytes += sz;
	}
	cudaSetDevice(cur);
	if (rc) return rc;
	out = p;
	return FMX_OK;
}

// ---------------------------------------------------------------------------
// Host: launching
// ---------------------------------------------------------------------------

template <class XT, class YT, class A, class WT, int VEC, int NV>
static int launch_t(const gpu_part &p, spmm_args a, bool sin, bool sout, cudaStream_t st)
{
	uint64_t warps = a.n_tasks + a.n_light_warps;
	uint64_t blocks = (warps * 32 + kThreads - 1) / kThreads;
	if (blocks) {
		if (blocks > 0x7FFFFFFFULL) return set_error(FMX_ERR_UNSUPPORTED, "grid too large");
		const dim3 grid{static_cast<unsigned>(blocks)};
		if (sin && sout) spmm_kernel<XT, YT, A, WT, VEC, NV, true, true><<<grid, kThreads, 0, st>>>(a);
		else if (sin) spmm_kernel<XT, YT, A, WT, VEC, NV, true, false><<<grid, kThreads, 0, st>>>(a);
		else if (sout) spmm_kernel<XT, YT, A, WT, VEC, NV, false, true><<<grid, kThreads, 0, st>>>(a);
		else spmm_kernel<XT, YT, A, WT, VEC, NV, false, false><<<grid, kThreads, 0, st>>>(a);
		CUDA_TRY(cudaGetLastError());
	}
	if (p.n_heavy) {
		unsigned fb = unsigned((uint64_t(p.n_heavy) * 32 + 255) / 256);
		if (sout) spmm_fixup_kernel<YT, A, true><<<fb, 256, 0, st>>>(p.heavy, p.n_heavy, static_cast<const A *>(a.partial),
				static_cast<YT *>(a.Y), a.ldy, a.k, static_cast<const A *>(a.s_out));
		else spmm_fixup_kernel<YT, A, false><<<fb, 256, 0, st>>>(p.heavy, p.n_heavy, static_cast<const A *>(a.partial),
				static_cast<YT *>(a.Y), a.ldy, a.k, static_cast<const A *>(a.s_out));
		CUDA_TRY(cudaGetLastError());
	}
	return FMX_OK;
}

static bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// Run one orientation over all column panels.
template <class XT, class YT, class A, class WT>
static int run_typed(const gpu_part &p, const void *X, int64_t ldx, void *Y, int64_t ldy, int64_t k,
		const void *sin, const void *sout, cudaStream_t st)
{
	constexpr int VEC = int(16 / sizeof(XT));
	// 16-byte vectors along k when every X and Y row starts 16-byte aligned
	// and k is a multiple of VEC; otherwise scalar lanes.
	const bool vec_ok = (k % VEC == 0) && (ldx % VEC == 0) && (ldy % VEC == 0) &&
			aligned16(X) && aligned16(Y) && (VEC * sizeof(YT)) % 8 == 0;
	const int64_t panel = vec_ok ? int64_t(32) * VEC : 128;
	for (int64_t c0 = 0; c0 < k; c0 += panel) {
		const int kp = int(std::min<int64_t>(panel, k - c0));
		spmm_args a{};
		a.row_ptr = p.row_ptr; a.col = p.col; a.val = p.val; a.light = p.light; a.tasks = p.tasks;
		a.X = static_cast<const XT *>(X) + c0;
		a.Y = static_cast<YT *>(Y) + c0;
		a.s_in = sin; a.s_out = sout; a.partial = p.partial;
		a.ldx = ldx; a.ldy = ldy; a.k = kp;
		a.n_light = p.n_light; a.n_tasks = p.n_tasks;
		int rc;
		if (vec_ok) {
			a.G = kp / VEC;           // <= 32
			a.R = 32 / a.G;
			a.nv = 1;
			a.n_light_warps = (uint64_t(p.n_light) + a.R - 1) / a.R;
			rc = launch_t<XT, YT, A, WT, VEC, 1>(p, a, sin, sout, st);
		} else {
			int g = 1;
			while (g < 32 && g * 4 < kp) g *= 2;
			a.G = g;
			a.R = 32 / g;
			a.nv = (kp + g - 1) / g;   // <= 4
			a.n_light_warps = (uint64_t(p.n_light) + a.R - 1) / a.R;
			rc = launch_t<XT, YT, A, WT, 1, 4>(p, a, sin, sout, st);
		}
		if (rc) return rc;
	}
	return FMX_OK;
}

template <class XT, class YT, class A>
static int run_w(const gpu_part &p, const void *X, int64_t ldx, void *Y, int64_t ldy, int64_t k,
		const void *sin, const void *sout, cudaStream_t st)
{
	switch (p.prim) {
	case FMX_P_BOOL: return run_typed<XT, YT, A, void>(p, X, ldx, Y, ldy, k, sin, sout, st);
	case FMX_P_FLOAT:
		if constexpr (std::is_floating_point<A>::value) return run_typed<XT, YT, A, float>(p, X, ldx, Y, ldy, k, sin, sout, st);
		break;
	case FMX_P_DOUBLE:
		if constexpr (std::is_same<A, double>::value) return run_typed<XT, YT, A, double>(p, X, ldx, Y, ldy, k, sin, sout, st);
		break;
	case FMX_P_INTEGER:
		if constexpr (std::is_integral<A>::value) return run_typed<XT, YT, A, int32_t>(p, X, ldx, Y, ldy, k, sin, sout, st);
		break;
	case FMX_P_LONG:
		if constexpr (std::is_same<A, int64_t>::value) return run_typed<XT, YT, A, int64_t>(p, X, ldx, Y, ldy, k, sin, sout, st);
		break;
	}
	return set_error(FMX_ERR_TYPE, "matrix entry type %d does not match the dense type "
			"(sparse_matrix.cpp:759-766 allows a binary matrix or equal types; float entries "
			"with FP64 operands as spmm_creator<double,float>)", p.prim);
}

int spmm_part(const gpu_part &p, int xt, const void *X, int64_t ldx, int yt, void *Y, int64_t ldy,
		int64_t k, const void *sin, const void *sout, cudaStream_t st)
{
	if (k <= 0) return set_error(FMX_ERR_DIM, "k must be positive (got %lld)", (long long)k);
	if (!X || !Y) return set_error(FMX_ERR_INVAL, "null X or Y");
	if (ldx < k || ldy < k) return set_error(FMX_ERR_DIM, "leading dimensions (%lld, %lld) smaller than k=%lld",
			(long long)ldx, (long long)ldy, (long long)k);
	int cur = 0;
	cudaGetDevice(&cur);
	if (cur != p.device) CUDA_TRY(cudaSetDevice(p.device));
	int rc;
	if (xt == FMX_F32 && yt == FMX_F32) rc = run_w<float, float, float>(p, X, ldx, Y, ldy, k, sin, sout, st);
	else if (xt == FMX_F64 && yt == FMX_F64) rc = run_w<double, double, double>(p, X, ldx, Y, ldy, k, sin, sout, st);
	else if (xt == FMX_BF16 && yt == FMX_F32) rc = run_w<__nv_bfloat16, float, float>(p, X, ldx, Y, ldy, k, sin, sout, st);
	else if (xt == FMX_BF16 && yt == FMX_BF16) rc = run_w<__nv_bfloat16, __nv_bfloat16, float>(p, X, ldx, Y, ldy, k, sin, sout, st);
	else if (xt == FMX_I32 && yt == FMX_I32) {
		rc = (sin || sout) ? set_error(FMX_ERR_UNSUPPORTED, "row scales need a floating-point type")
				: run_w<int32_t, int32_t, int32_t>(p, X, ldx, Y, ldy, k, nullptr, nullptr, st);
	} else if (xt == FMX_I64 && yt == FMX_I64) {
		rc = (sin || sout) ? set_error(FMX_ERR_UNSUPPORTED, "row scales need a floating-point type")
				: run_w<int64_t, int64_t, int64_t>(p, X, ldx, Y, ldy, k, nullptr, nullptr, st);
	} else rc = set_error(FMX_ERR_TYPE, "unsupported type pair x=%d y=%d "
			"(input and output matrices need the same type, sparse_matrix.cpp:754-758)", xt, yt);
	if (cur != p.device) cudaSetDevice(cur);
	return rc;
}

// ---------------------------------------------------------------------------
// R-MAT (counter-based; identical streams on host and device)
// ---------------------------------------------------------------------------

struct rmat_params {
	uint64_t seed_key;
	uint32_t t_a, t_ab, t_abc;      // cumulative quadrant thresholds * 2^32
	int scale;
	int permute;
	uint64_t pm[4];                 // odd multipliers of the relabelling
	uint64_t pa[4];                 // addends
};

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z)
{
	// splitmix64 finaliser (Steele, Lea, Flood 2014)
	z += 0x9E3779B97F4A7C15ULL;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
	return z ^ (z >> 31);
}

// A seeded bijection on [0, 2^scale): odd multiplies, adds and xor-shifts,
// each invertible modulo 2^scale.
__host__ __device__ __forceinline__ uint32_t relabel(const rmat_params &p, uint32_t v)
{
	const uint64_t mask = (p.scale >= 64) ? ~0ULL : ((1ULL << p.scale) - 1);
	uint64_t x = v;
	const int sh = p.scale / 2 + 1;
	for (int r = 0; r < 4; r++) {
		x = (x * p.pm[r] + p.pa[r]) & mask;
		x ^= x >> sh;
	}
	return uint32_t(x);
}

__host__ __device__ __forceinline__ void rmat_edge(const rmat_params &p, uint64_t e, uint32_t &src, uint32_t &dst)
{
	uint64_t h0 = mix64(p.seed_key ^ (e * 0xD6E8FEB86659FD93ULL));
	uint32_t r = 0, c = 0;
	uint64_t h = 0;
	for (int l = 0; l < p.scale; l++) {
		if ((l & 1) == 0) h = mix64(h0 + uint64_t(l) * 0x9E3779B97F4A7C15ULL);
		uint32_t u = (l & 1) ? uint32_t(h >> 32) : uint32_t(h);
		uint32_t rb = u >= p.t_ab;                 // quadrants c, d: row bit set
		uint32_t cb = (u >= p.t_a && u < p.t_ab) || u >= p.t_abc;  // b, d: col bit set
		r = (r << 1) | rb;
		c = (c << 1) | cb;
	}
	if (p.permute) { r = relabel(p, r); c = relabel(p, c); }
	src = r; dst = c;
}

static int rmat_setup(int scale, double a, double b, double c, uint64_t seed, int permute, rmat_params &p)
{
	if (scale < 1 || scale > 31) return set_error(FMX_ERR_INVAL, "R-MAT scale %d outside 1..31", scale);
	if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0))
		return set_error(FMX_ERR_INVAL, "R-MAT probabilities a=%g b=%g c=%g invalid", a, b, c);
	auto th = [](double x) -> uint32_t {
		double v = x * 4294967296.0;
		return v >= 4294967295.0 ? 0xFFFFFFFFu : uint32_t(v);
	};
	p.seed_key = mix64(seed ^ 0x5851F42D4C957F2DULL);
	p.t_a = th(a); p.t_ab = th(a + b); p.t_abc = th(a + b + c);
	p.scale = scale;
	p.permute = permute;
	uint64_t s = mix64(seed + 0x1234567ULL);
	for (int r = 0; r < 4; r++) {
		s = mix64(s);
		p.pm[r] = s | 1ULL;
		s = mix64(s);
		p.pa[r] = s;
	}
	return FMX_OK;
}

__global__ void rmat_kernel(rmat_params p, uint64_t n, uint32_t *src, uint32_t *dst)
{
	for (uint64_t e = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n; e += uint64_t(gridDim.x) * blockDim.x) {
		uint32_t s, d;
		rmat_edge(p, e, s, d);
		src[e] = s;
		dst[e] = d;
	}
}

} // namespace fmx

using namespace fmx;

extern "C" {

int fmx_matrix_create(const fmx_image *img, const fmx_image *t_img, int device, fmx_matrix **out)
{
	if (!img || !out) return set_error(FMX_ERR_INVAL, "null argument");
	*out = nullptr;
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
		return set_error(FMX_ERR_CUDA, "no CUDA device is available");
	if (device < 0 || device >= ndev) return set_error(FMX_ERR_INVAL, "device %d out of range (%d devices)", device, ndev);
	if (t_img && (t_img->im.h.nrows != img->im.h.ncols || t_img->im.h.ncols != img->im.h.nrows))
		return set_error(FMX_ERR_DIM, "transpose image is %llux%llu, expected %llux%llu",
				(unsigned long long)t_img->im.h.nrows, (unsigned long long)t_img->im.h.ncols,
				(unsigned long long)img->im.h.ncols, (unsigned long long)img->im.h.nrows);
	std::unique_ptr<fmx_matrix> m(new (std::nothrow) fmx_matrix);
	if (!m) return set_error(FMX_ERR_OOM, "out of host memory");
	const fmx_image *parts[2] = {img, t_img};
	for (int i = 0; i < 2; i++) {
		if (!parts[i]) continue;
		host_csr csr;
		int rc;
		try {
			rc = decode_to_csr(parts[i]->im, csr, default_threads());
		} catch (const std::bad_alloc &) {
			rc = set_error(FMX_ERR_OOM, "host allocation failed while decoding the image");
		}
		if (rc) return rc;
		rc = make_part(csr, device, i == 0 ? m->a : m->at);
		if (rc) return rc;
	}
	m->symmetric = (t_img == nullptr);
	*out = m.release();
	return FMX_OK;
}

int fmx_matrix_load(const char *mat_idx_path, const char *mat_path, const char *t_mat_idx_path,
		const char *t_mat_path, int device, fmx_matrix **out)
{
	fmx_image *a = nullptr, *t = nullptr;
	int rc = fmx_image_load(mat_idx_path, mat_path, &a);
	if (!rc && t_mat_idx_path && t_mat_path) rc = fmx_image_load(t_mat_idx_path, t_mat_path, &t);
	if (!rc) rc = fmx_matrix_create(a, t, device, out);
	fmx_image_free(a);
	fmx_image_free(t);
	return rc;
}

int fmx_matrix_info(const fmx_matrix *m, uint64_t *nrows, uint64_t *ncols, uint64_t *nnz, int *prim_type, int *symmetric)
{
	if (!m || !m->a) return set_error(FMX_ERR_INVAL, "null matrix");
	if (nrows) *nrows = m->a->nrows;
	if (ncols) *ncols = m->a->ncols;
	if (nnz) *nnz = m->a->nnz;
	if (prim_type) *prim_type = m->a->prim;
	if (symmetric) *symmetric = m->symmetric ? 1 : 0;
	return FMX_OK;
}

int fmx_matrix_device_bytes(const fmx_matrix *m, uint64_t *bytes)
{
	if (!m || !m->a || !bytes) return set_error(FMX_ERR_INVAL, "null argument");
	*bytes = m->a->bytes + (m->at ? m->at->bytes : 0);
	return FMX_OK;
}

int fmx_matrix_transpose(const fmx_matrix *m, fmx_matrix **out)
{
	if (!m || !out) return set_error(FMX_ERR_INVAL, "null argument");
	std::unique_ptr<fmx_matrix> t(new (std::nothrow) fmx_matrix);
	if (!t) return set_error(FMX_ERR_OOM, "out of host memory");
	t->symmetric = m->symmetric;
	if (m->symmetric) t->a = m->a;
	else { t->a = m->at; t->at = m->a; }
	*out = t.release();
	return FMX_OK;
}

int fmx_matrix_free(fmx_matrix *m)
{
	delete m;
	return FMX_OK;
}

int fmx_spmm(const fmx_matrix *m, int x_type, const void *X, int64_t ldx, int y_type, void *Y,
		int64_t ldy, int64_t k, const void *row_scale_in, const void *row_scale_out, void *stream)
{
	if (!m || !m->a) return set_error(FMX_ERR_INVAL, "null matrix");
	return spmm_part(*m->a, x_type, X, ldx, y_type, Y, ldy, k, row_scale_in, row_scale_out,
			static_cast<cudaStream_t>(stream));
}

static size_t dtype_size(int t)
{
	switch (t) {
	case FMX_F32: case FMX_I32: return 4;
	case FMX_F64: case FMX_I64: return 8;
	case FMX_BF16: return 2;
	}
	return 0;
}

int fmx_spmm_host(const fmx_matrix *m, int x_type, const void *X_host, int64_t ldx, int y_type,
		void *Y_host, int64_t ldy, int64_t k)
{
	if (!m || !m->a || !X_host || !Y_host) return set_error(FMX_ERR_INVAL, "null argument");
	size_t xs = dtype_size(x_type), ys = dtype_size(y_type);
	if (!xs || !ys) return set_error(FMX_ERR_TYPE, "unknown dtype");
	if (k <= 0 || ldx < k || ldy < k) return set_error(FMX_ERR_DIM, "bad k / leading dimensions");
	gpu_part &p = *m->a;
	std::lock_guard<std::mutex> guard(p.stage_mu);
	int cur = 0;
	cudaGetDevice(&cur);
	CUDA_TRY(cudaSetDevice(p.device));
	size_t xb = size_t(p.ncols) * k * xs, yb = size_t(p.nrows) * k * ys;
	int rc = FMX_OK;
	auto grow = [&](void *&buf, size_t &have, size_t need) -> int {
		if (have >= need) return FMX_OK;
		if (buf) cudaFree(buf);
		buf = nullptr; have = 0;
		if (cudaMalloc(&buf, need) != cudaSuccess) return set_error(FMX_ERR_OOM, "cudaMalloc of %zu staging bytes failed", need);
		have = need;
		return FMX_OK;
	};
	rc = grow(p.stage_x, p.stage_xb, xb);
	if (!rc) rc = grow(p.stage_y, p.stage_yb, yb);
	cudaStream_t st = nullptr;
	if (!rc && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) rc = set_error(FMX_ERR_CUDA, "stream creation failed");
	if (!rc && cudaMemcpy2DAsync(p.stage_x, k * xs, X_host, ldx * xs, k * xs, p.ncols, cudaMemcpyHostToDevice, st) != cudaSuccess)
		rc = set_error(FMX_ERR_CUDA, "copy of X to the device failed");
	if (!rc) rc = spmm_part(p, x_type, p.stage_x, k, y_type, p.stage_y, k, k, nullptr, nullptr, st);
	if (!rc && cudaMemcpy2DAsync(Y_host, ldy * ys, p.stage_y, k * ys, k * ys, p.nrows, cudaMemcpyDeviceToHost, st) != cudaSuccess)
		rc = set_error(FMX_ERR_CUDA, "copy of Y to the host failed");
	if (st) {
		cudaError_t e = cudaStreamSynchronize(st);
		if (!rc && e != cudaSuccess) rc = set_error(FMX_ERR_CUDA, "SpMM failed: %s", cudaGetErrorString(e));
		cudaStreamDestroy(st);
	}
	cudaSetDevice(cur);
	return rc;
}

int fmx_matrix_schedule(const fmx_matrix *m, uint64_t *n_light_rows, uint64_t *n_split_tasks,
		uint64_t *n_heavy_rows, uint64_t *kernels_per_spmm)
{
	if (!m || !m->a) return set_error(FMX_ERR_INVAL, "null matrix");
	const gpu_part &p = *m->a;
	if (n_light_rows) *n_light_rows = p.n_light;
	if (n_split_tasks) *n_split_tasks = p.n_tasks;
	if (n_heavy_rows) *n_heavy_rows = p.n_heavy;
	if (kernels_per_spmm) *kernels_per_spmm = 1 + (p.n_heavy ? 1 : 0);
	return FMX_OK;
}

int fmx_rmat_edges_host(int scale, uint64_t nedges, double a, double b, double c, uint64_t seed,
		int permute, uint32_t *src, uint32_t *dst, int nthreads)
{
	rmat_params p;
	int rc = rmat_setup(scale, a, b, c, seed, permute, p);
	if (rc) return rc;
	if (nedges && (!src || !dst)) return set_error(FMX_ERR_INVAL, "null output arrays");
	if (nthreads <= 0) nthreads = default_threads();
	std::vector<std::thread> th;
	uint64_t per = (nedges + nthreads - 1) / nthreads;
	for (int t = 0; t < nthreads; t++)
		th.emplace_back([&, t]() {
			uint64_t b0 = uint64_t(t) * per, b1 = std::min(nedges, b0 + per);
			for (uint64_t e = b0; e < b1; e++) rmat_edge(p, e, src[e], dst[e]);
		});
	for (auto &x : th) x.join();
	return FMX_OK;
}

int fmx_rmat_edges_device(int scale, uint64_t nedges, double a, double b, double c, uint64_t seed,
		int permute, uint32_t *src_dev, uint32_t *dst_dev, void *stream)
{
	rmat_params p;
	int rc = rmat_setup(scale, a, b, c, seed, permute, p);
	if (rc) return rc;
	if (!nedges) return FMX_OK;
	if (!src_dev || !dst_dev) return set_error(FMX_ERR_INVAL, "null output arrays");
	unsigned blocks = unsigned(std::min<uint64_t>((nedges + 255) / 256, 148ULL * 64));
	rmat_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(p, nedges, src_dev, dst_dev);
	CUDA_TRY(cudaGetLastError());
	return FMX_OK;
}

} // extern "C"
