// SpMM on B200 (sm_100a): Y = diag(s_out) * A * diag(s_in) * X.
//
// Replaces FlashMatrix's CPU SpMM tasks (row_part_func / coo_func /
// block_spmm_task_impl::run_on_block, matrix/sparse_matrix.h:219-375, driven
// by block_compute_task::run, matrix/sparse_matrix.cpp:251-314).
//
// Layout in HBM (built once per matrix from the decoded 2D image, resident):
//   col      uint32[]           one entry stream.  Bit 31 is set on the last
//                               entry of a row; with bit 30 set, bits 0-29 hold
//                               a hot slot, else the column id.  First every
//                               row in ascending order: a row of 1..kExactMax
//                               entries as its entries in the order the
//                               reference visits them (ascending block column,
//                               then column); an empty or longer row as one
//                               entry naming the pack's zero row.  Then the
//                               entries of the longer rows (> kExactMax).
//   val      entry[]            only for weighted images, same order
//   hot_col  int32[H]           the H <= kHotMax columns of highest in-degree;
//                               entry slot s + 1 names hot_col[s], slot 0 the
//                               pack's zero row
//   ranges   range_t[]          work units, sorted by entry count (largest
//                               first): a run of consecutive rows of up to ~kRange
//                               entries, or one of the equal chunks (<= kChunk
//                               entries) of a longer row.  Each starts at a
//                               multiple of 8 entries and is padded to one
//                               with zero-row entries (after the last row end
//                               of a run they are never stored; in a chunk
//                               they add zeros), so steps need no bounds.
//   heavy    heavy_row[]        longer rows: spmm_fixup_kernel overwrites their
//                               Y rows with their chunk partials added in
//                               chunk order
// Scratch (allocated with the matrix):
//   xhot     (H+1) x 128 bytes  per call, the hot columns' X rows of the
//                               current panel, packed back to back (times s_in
//                               when given) after row 0, which stays zero
//   partial  AccT[chunks][kPartialStride]  chunk sums of longer rows
//
// Why the hot pack: the X gathers of an R-MAT graph are random 64-byte reads
// that mostly miss the L2, and a hot row shares its 128-byte line with a cold
// one.  Packing the highest in-degree rows (about 87% of the gathers at scale
// 24) two to a line keeps them in a range the L2 can hold.
//
// Execution: persistent grids whose lane groups take ranges round-robin and
// walk them as a stream of entries in aligned steps; when an entry closes a
// row, the group stores that row (the range's first row plus the rows closed
// before it).  Every row of up to kExactMax entries is summed by one group in
// the reference's order (bit-identical results).  No atomics: every output
// row is written exactly once.  Three row kernels share that scheme:
//   spmm_wide_kernel  FP32 panels of 32, 64 or 128 bytes, and unweighted BF16
//                     into BF16: a lane owns 32 bytes of each gathered row;
//                     8 column ids per 32-byte load
//   spmm_kernel       16-byte lanes (BF16 into FP32, weighted BF16, FP64,
//                     integer and odd widths), with L2 evict_last hints on
//                     hot-pack gathers and evict_first on cold rows
//   spmv_kernel       k = 1: a warp per range, gathers staged in shared memory
// Each call first packs the hot rows: pack_hot_vec_kernel in 16-byte units,
// pack_hot_kernel one element per thread (k = 1 and rows of odd widths).
#include "fmx_internal.h"

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <thread>

#include "part.h"

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

// Packed FP32 pairs (sm_100 add.rn.f32x2): two IEEE round-to-nearest adds
// per instruction, the same results as two scalar adds.
__device__ __forceinline__ uint64_t pack2(float a, float b)
{
	uint64_t r;
	asm("mov.b64 %0, {%1,%2};" : "=l"(r) : "f"(a), "f"(b));
	return r;
}
__device__ __forceinline__ void unpack2(uint64_t v, float &a, float &b)
{
	asm("mov.b64 {%0,%1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b)
{
	uint64_t r;
	asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
	return r;
}

// Streaming (read-once) loads and stores: evict-first in L1 and L2 so that
// the gathered X rows keep the caches.
__device__ __forceinline__ float ld_stream(const float *p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double *p) { return __ldcs(p); }
__device__ __forceinline__ int32_t ld_stream(const int32_t *p) { return __ldcs(p); }
__device__ __forceinline__ int64_t ld_stream(const int64_t *p) { return (int64_t)__ldcs((const long long *)p); }

// VEC elements of T: one 16-byte vector, or a scalar (VEC == 1).
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
	} else if constexpr (sizeof(T) == 2) {
		unsigned short u = __ldg(reinterpret_cast<const unsigned short *>(p));
		memcpy(&r, &u, 2);
	} else {
		static_assert(VEC == 1, "scalar path");
		r.v[0] = __ldg(p);
	}
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

// L2 eviction priorities for the gathers (createpolicy, PTX ISA 7.4+).
__device__ __forceinline__ uint64_t policy_evict_last()
{
	uint64_t p;
	asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
	return p;
}
__device__ __forceinline__ uint64_t policy_evict_first()
{
	uint64_t p;
	asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
	return p;
}

// Read-only gather of VEC elements of T (16 bytes, or one scalar) with an L2
// eviction-priority hint.
template <class T, int VEC>
__device__ __forceinline__ xvec<T, VEC> ld_x_hint(const T *p, uint64_t pol)
{
	xvec<T, VEC> r;
	if constexpr (VEC * sizeof(T) == 16) {
		uint32_t a, b, c, d;
		asm volatile("ld.global.nc.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
				: "=r"(a), "=r"(b), "=r"(c), "=r"(d) : "l"(p), "l"(pol));
		uint4 u = make_uint4(a, b, c, d);
		memcpy(&r, &u, 16);
	} else if constexpr (sizeof(T) == 8) {
		static_assert(VEC == 1, "scalar path");
		uint64_t a;
		asm volatile("ld.global.nc.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(a) : "l"(p), "l"(pol));
		memcpy(&r, &a, 8);
	} else if constexpr (sizeof(T) == 4) {
		static_assert(VEC == 1, "scalar path");
		uint32_t a;
		asm volatile("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(a) : "l"(p), "l"(pol));
		memcpy(&r, &a, 4);
	} else {
		static_assert(VEC == 1 && sizeof(T) == 2, "scalar path");
		unsigned short a;
		asm volatile("ld.global.nc.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(a) : "l"(p), "l"(pol));
		memcpy(&r, &a, 2);
	}
	return r;
}

// Store one 16-byte vector when `pred` holds, without a branch (a predicated
// streaming store); other widths fall back to a guarded plain store.
template <class T, int VEC>
__device__ __forceinline__ void st_y_if(T *p, const T (&v)[VEC], bool pred)
{
	if constexpr (VEC * sizeof(T) == 16) {
		uint32_t u[4];
		memcpy(u, v, 16);
		asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %5, 0;\n\t"
				"@q st.global.cs.v4.u32 [%0], {%1,%2,%3,%4};\n\t}"
				:: "l"(p), "r"(u[0]), "r"(u[1]), "r"(u[2]), "r"(u[3]), "r"(uint32_t(pred)) : "memory");
	} else {
		if (pred) st_y<T, VEC>(p, v);
	}
}

struct spmm_args {
	const uint32_t *col;
	const void *val;
	const range_t *ranges;
	const void *X;
	const void *xhot;    // packed hot rows of this panel, row stride hot_ld
	void *Y;
	const void *s_in;
	const void *s_out;
	void *partial;
	int64_t ldx, ldy;
	int hot_ld;      // elements per packed hot row
	int k;           // columns in this panel
	int G;           // lanes per row group
	int R;           // row groups per warp
	int nv;          // vectors per lane (scalar path)
	uint32_t n_ranges;
};

// The running sums of one lane: NV vectors of VEC elements.  FP32 with
// VEC == 4 or 8 is kept as packed pairs.
template <class A, int VEC, int NV>
struct accum {
	static constexpr bool kPacked = std::is_same<A, float>::value && (VEC % 2 == 0) && NV == 1;
	A s[NV][VEC];
	uint64_t p[VEC / 2 > 0 ? VEC / 2 : 1];

	__device__ __forceinline__ void zero()
	{
		if constexpr (kPacked) {
#pragma unroll
			for (int i = 0; i < VEC / 2; i++) p[i] = 0;
		} else {
#pragma unroll
			for (int v = 0; v < NV; v++)
#pragma unroll
				for (int i = 0; i < VEC; i++) s[v][i] = A(0);
		}
	}
	__device__ __forceinline__ void zero_if(bool z)
	{
		if constexpr (kPacked) {
#pragma unroll
			for (int i = 0; i < VEC / 2; i++) p[i] = z ? 0ull : p[i];
		} else {
#pragma unroll
			for (int v = 0; v < NV; v++)
#pragma unroll
				for (int i = 0; i < VEC; i++) s[v][i] = z ? A(0) : s[v][i];
		}
	}
	// s[v] += x (* m1) (* m2), each operation rounded (no contraction)
	template <class XT, int NMUL>
	__device__ __forceinline__ void add(int v, const xvec<XT, VEC> &x, A m1, A m2)
	{
		if constexpr (kPacked) {
			// products stay scalar __fmul_rn (never fused into the add);
			// only the adds are packed
#pragma unroll
			for (int i = 0; i < VEC / 2; i++) {
				float t0 = to_acc<float>(x.v[2 * i]), t1 = to_acc<float>(x.v[2 * i + 1]);
				if constexpr (NMUL >= 1) { t0 = __fmul_rn(t0, m1); t1 = __fmul_rn(t1, m1); }
				if constexpr (NMUL >= 2) { t0 = __fmul_rn(t0, m2); t1 = __fmul_rn(t1, m2); }
				p[i] = add2(p[i], pack2(t0, t1));
			}
		} else {
#pragma unroll
			for (int i = 0; i < VEC; i++) {
				A t = to_acc<A>(x.v[i]);
				if constexpr (NMUL >= 1) t = acc_mul(t, m1);
				if constexpr (NMUL >= 2) t = acc_mul(t, m2);
				s[v][i] = acc_add(s[v][i], t);
			}
		}
	}
	__device__ __forceinline__ A get(int v, int i) const
	{
		if constexpr (kPacked) {
			float a, b;
			unpack2(p[i / 2], a, b);
			return (i & 1) ? b : a;
		} else {
			return s[v][i];
		}
	}
};

template <class YT, class A, int VEC, int NV, bool SCALE_OUT>
__device__ __forceinline__ void store_row(const spmm_args &a, int32_t row, int colbase,
		const accum<A, VEC, NV> &acc)
{
	YT *Y = static_cast<YT *>(a.Y);
	A so = A(1);
	if constexpr (SCALE_OUT) so = static_cast<const A *>(a.s_out)[row];
	const int stride = a.G * VEC;
#pragma unroll
	for (int v = 0; v < NV; v++)
		if (v < a.nv && colbase + v * stride < a.k) {
			YT out[VEC];
#pragma unroll
			for (int i = 0; i < VEC; i++) {
				A t = acc.get(v, i);
				if constexpr (SCALE_OUT) t = acc_mul(t, so);
				out[i] = from_acc<YT, A>(t);
			}
			st_y<YT, VEC>(Y + int64_t(row) * a.ldy + colbase + v * stride, out);
		}
}

template <int U>
__device__ __forceinline__ void ld_idx(const uint32_t *col, uint32_t step, uint32_t (&r)[U])
{
	const uint4 *p = reinterpret_cast<const uint4 *>(col) + (U / 4) * step;
#pragma unroll
	for (int q = 0; q < U / 4; q++) {
		// cached: a group reads each 128-byte line of its stream over several steps
		uint4 a = __ldg(p + q);
		r[4 * q] = a.x; r[4 * q + 1] = a.y; r[4 * q + 2] = a.z; r[4 * q + 3] = a.w;
	}
}

template <class WT, class A, int U>
__device__ __forceinline__ void ld_w(const void *val, uint32_t step, A (&w)[U])
{
	if constexpr (std::is_void<WT>::value) {
#pragma unroll
		for (int u = 0; u < U; u++) w[u] = A(1);
	} else {
		{
			// cached like the column ids: the streaming form, which skips
			// L1, fetched each weight line from L2 again at every step (in
			// the 32-byte-lane kernel, cached 32-byte weight loads took a
			// weighted call at R-MAT scale 24, k = 16 from 3.43 to 2.58 ms)
			const uint4 *p = reinterpret_cast<const uint4 *>(static_cast<const WT *>(val) + size_t(step) * U);
			constexpr int per = int(16 / sizeof(WT));
			static_assert(U % per == 0, "whole 16-byte weight loads");
#pragma unroll
			for (int q = 0; q < U / per; q++) {
				uint4 a = __ldg(p + q);
				WT t[per];
				memcpy(t, &a, 16);
#pragma unroll
				for (int i = 0; i < per; i++) w[q * per + i] = A(t[i]);
			}
		}
	}
}

// One range in steps of U entries.  Row runs (slot == kNoSlot) store each
// row when its end flag passes; chunks of longer rows leave their sum in
// partial[slot].  Hot entries read the packed rows (which already carry
// s_in); the others read X and, with SCALE_IN, s_in.
// The PageRank update at a row close (EPI): rows of the fixup's heavy list
// are left to the fixup.
__device__ __forceinline__ void pr_update(const pr_epi &e, int64_t row, float out, unsigned &cnt)
{
	const float p2 = __fadd_rn(__fmul_rn(out, e.damping), e.teleport);
	const float diff = fabsf(__fsub_rn(e.pr1[row], p2));
	cnt += diff < e.eps;
	e.pr[row] = p2;
	const float d = e.deg[row];
	const float x = __fdiv_rn(p2, d);
	e.in_next[row] = x;
	e.pr1[row] = __fmul_rn(x, d);
}

template <class XT, class YT, class A, class WT, int VEC, int NV, int U, bool SCALE_IN, bool SCALE_OUT,
		bool EPI = false>
__device__ __forceinline__ void run_range(const spmm_args &a, const range_t rg, int colbase,
		uint64_t pol_hot, uint64_t pol_cold, const pr_epi &e, unsigned &cnt)
{
	const XT *X = static_cast<const XT *>(a.X);
	const XT *H = static_cast<const XT *>(a.xhot);
	const int stride = a.G * VEC;
	constexpr bool kBinary = std::is_void<WT>::value;
	const bool runs = rg.slot == kNoSlot;
	accum<A, VEC, NV> acc;
	acc.zero();
	uint32_t row = rg.row0;
	uint32_t s = rg.e0 / U;
	const uint32_t s_end = s + rg.len / U;
	uint32_t raw[U];
	ld_idx<U>(a.col, s, raw);
	for (; s < s_end; s++) {
		A w[U];
		if constexpr (!kBinary) ld_w<WT, A, U>(a.val, s, w);
		// issue this step's gathers
		xvec<XT, VEC> x[U][NV];
		A sc[U];
		uint32_t ends = 0;
#pragma unroll
		for (int u = 0; u < U; u++) {
			const uint32_t c = raw[u] & kIdxMask;
			const bool hot = raw[u] & kHot;
			const XT *xr = (hot ? H : X) + int64_t(c) * (hot ? int64_t(a.hot_ld) : a.ldx) + colbase;
			const uint64_t pol = hot ? pol_hot : pol_cold;
			if constexpr (NV == 1) {
				// 16-byte lanes: every lane of a group owns a valid vector
				x[u][0] = ld_x_hint<XT, VEC>(xr, pol);
			} else {
#pragma unroll
				for (int v = 0; v < NV; v++)
					if (v < a.nv && colbase + v * stride < a.k)
						x[u][v] = ld_x_hint<XT, VEC>(xr + v * stride, pol);
			}
			if constexpr (SCALE_IN) sc[u] = hot ? A(1) : static_cast<const A *>(a.s_in)[c];
			ends |= (raw[u] >> 31) << u;
		}
		// the next step's column ids load while the gathers are in flight
		if (s + 1 < s_end) ld_idx<U>(a.col, s + 1, raw);
		// add up in entry order; a set end flag closes the row
#pragma unroll
		for (int u = 0; u < U; u++) {
#pragma unroll
			for (int v = 0; v < NV; v++)
				if (NV == 1 || (v < a.nv && colbase + v * stride < a.k)) {
					// (x * s_in) * w, rounded per step like scale_rows then SpMM;
					// for hot entries x * s_in was rounded by the pack
					if constexpr (SCALE_IN && !kBinary) acc.template add<XT, 2>(v, x[u][v], sc[u], w[u]);
					else if constexpr (SCALE_IN) acc.template add<XT, 1>(v, x[u][v], sc[u], A(1));
					else if constexpr (!kBinary) acc.template add<XT, 1>(v, x[u][v], w[u], A(1));
					else acc.template add<XT, 0>(v, x[u][v], A(1), A(1));
				}
			const bool end = runs && ((ends >> u) & 1u);
			if constexpr (EPI) {
				static_assert(NV == 1 && VEC == 1 && std::is_same<A, float>::value, "PageRank: k = 1, FP32");
				if (end && !((__ldg(e.heavy_mask + (row >> 5)) >> (row & 31)) & 1u))
					pr_update(e, int64_t(row), acc.get(0, 0), cnt);
			} else if constexpr (NV == 1) {
				// branch-free row close: predicated store, select-reset
				YT *Yp = static_cast<YT *>(a.Y) + int64_t(row) * a.ldy + colbase;
				A so = A(1);
				if constexpr (SCALE_OUT) so = end ? static_cast<const A *>(a.s_out)[row] : A(1);
				YT out[VEC];
#pragma unroll
				for (int i = 0; i < VEC; i++) {
					A t = acc.get(0, i);
					if constexpr (SCALE_OUT) t = acc_mul(t, so);
					out[i] = from_acc<YT, A>(t);
				}
				st_y_if<YT, VEC>(Yp, out, end);
			} else {
				if (end) store_row<YT, A, VEC, NV, SCALE_OUT>(a, int32_t(row), colbase, acc);
			}
			acc.zero_if(end);
			row += end;
		}
	}
	if (!runs) {
		A *p = static_cast<A *>(a.partial) + int64_t(rg.slot) * kPartialStride;
#pragma unroll
		for (int v = 0; v < NV; v++)
			if (v < a.nv && colbase + v * stride < a.k)
#pragma unroll
				for (int i = 0; i < VEC; i++) p[colbase + v * stride + i] = acc.get(v, i);
	}
}

template <class XT, class YT, class A, class WT, int VEC, int NV, int U, bool SCALE_IN, bool SCALE_OUT,
		bool EPI = false>
__global__ void __launch_bounds__(kThreads, sizeof(XT) == 2 ? FMX_SPMM_MIN_BLOCKS_2B : FMX_SPMM_MIN_BLOCKS)
spmm_kernel(const spmm_args a, const pr_epi e)
{
	if constexpr (EPI) {
		if (e.state[1]) return;           // converged in an earlier iteration
	}
	const int lane = threadIdx.x & 31;
	const uint32_t gw = (blockIdx.x * kThreads + threadIdx.x) >> 5;
	const uint32_t nw = (gridDim.x * kThreads) >> 5;
	const int G = a.G, R = a.R;
	const int grp = lane / G;
	if (grp >= R) return;
	const int colbase = (lane - grp * G) * VEC;
	const uint32_t gg = gw * uint32_t(R) + uint32_t(grp);
	const uint32_t ng = nw * uint32_t(R);
	const uint64_t pol_hot = policy_evict_last(), pol_cold = policy_evict_first();
	unsigned cnt = 0;
	for (uint32_t r = gg; r < a.n_ranges; r += ng)
		run_range<XT, YT, A, WT, VEC, NV, U, SCALE_IN, SCALE_OUT, EPI>(a, a.ranges[r], colbase, pol_hot, pol_cold,
				e, cnt);
	if constexpr (EPI) {
		// G = 1: every lane of the warp is a row group and reaches this point
		cnt = __reduce_add_sync(0xffffffffu, cnt);
		if (lane == 0 && cnt) atomicAdd(e.state, (unsigned long long)cnt);
	}
}

// ---------------------------------------------------------------------------
// 32-byte lanes (the main path for row panels of 32, 64 or 128 bytes).
//
// A lane owns 32 bytes of every X row it gathers (8 FP32 or 16 BF16
// elements), so a row panel of P bytes takes G = P / 32 lanes (1, 2 or 4) and
// a warp runs 32 / G lane groups.  Each entry costs one 256-bit load per lane
// and one decode per lane (the 16-byte-lane kernel spends a decode on every
// 16 bytes); a warp-wide load still touches one 128-byte line per row.
// Loads use no L2 policy: the measured gain of the hot/cold hints did not pay
// for selecting them per entry.  The arithmetic is the 16-byte-lane kernel's
// (products rounded, adds in entry order as packed FP32 pairs), so results
// are bit-identical.
// ---------------------------------------------------------------------------
#ifndef FMX_WIDE_MIN_BLOCKS
#define FMX_WIDE_MIN_BLOCKS 4
#endif

__device__ __forceinline__ void ld32_nc(const void *p, uint32_t (&r)[8])
{
	asm volatile("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
			: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
			: "l"(p));
}
// 32-byte streaming store when `pred` holds (predicated, no branch).
__device__ __forceinline__ void st32_if(void *p, const uint32_t (&v)[8], bool pred)
{
	asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %9, 0;\n\t"
			"@q st.global.cs.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};\n\t}"
			:: "l"(p), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]),
			   "r"(uint32_t(pred)) : "memory");
}

// The VEC elements of one 32-byte load as FP32 (BF16 widened exactly).
template <class XT, int VEC>
__device__ __forceinline__ void widen(const uint32_t (&r)[8], float (&f)[VEC])
{
	if constexpr (sizeof(XT) == 4) {
#pragma unroll
		for (int i = 0; i < 8; i++) f[i] = __uint_as_float(r[i]);
	} else {
#pragma unroll
		for (int i = 0; i < 8; i++) {
			f[2 * i] = __uint_as_float(r[i] << 16);
			f[2 * i + 1] = __uint_as_float(r[i] & 0xFFFF0000u);
		}
	}
}

template <class XT, class YT, class WT, int U, bool SCALE_IN, bool SCALE_OUT>
__device__ __forceinline__ void run_range_wide(const spmm_args &a, const range_t rg, int colbase)
{
	constexpr int VEC = int(32 / sizeof(XT));
	constexpr bool kBinary = std::is_void<WT>::value;
	const char *Xb = static_cast<const char *>(a.X) + size_t(colbase) * sizeof(XT);
	const char *Hb = static_cast<const char *>(a.xhot) + size_t(colbase) * sizeof(XT);
	const uint32_t xs = uint32_t(a.ldx) * uint32_t(sizeof(XT)), hs = uint32_t(a.hot_ld) * uint32_t(sizeof(XT));
	char *Yb = static_cast<char *>(a.Y) + size_t(colbase) * sizeof(YT);
	const uint64_t ys = uint64_t(a.ldy) * sizeof(YT);
	const bool runs = rg.slot == kNoSlot;
	uint64_t p[VEC / 2];
#pragma unroll
	for (int i = 0; i < VEC / 2; i++) p[i] = 0;
	uint32_t row = rg.row0;
	// pairs of 4-entry steps (a range is a whole number of kStep = 8
	// entries): one 32-byte load of 8 column ids, and of 8 weights, per lane
	// per pair, issued with the first step's gathers; the next pair's column
	// ids load with the second step's gathers
	static_assert(U == 4 && kStep == 2 * U, "pairs of 4-entry steps");
	uint32_t s = rg.e0 / kStep;
	const uint32_t s_end = s + rg.len / kStep;
	uint32_t raw8[2 * U];
	ld32_nc(a.col + size_t(s) * kStep, raw8);
	for (; s < s_end; s++) {
		uint32_t w8[2 * U];
		if constexpr (!kBinary) ld32_nc(static_cast<const WT *>(a.val) + size_t(s) * kStep, w8);
#pragma unroll
		for (int half = 0; half < 2; half++) {
		float w[U];
		if constexpr (!kBinary) {
#pragma unroll
			for (int u = 0; u < U; u++) w[u] = __uint_as_float(w8[half * U + u]);
		}
		uint32_t xv[U][8];
		float sc[U];
		uint32_t ends = 0;
#pragma unroll
		for (int u = 0; u < U; u++) {
			const uint32_t rw = raw8[half * U + u];
			const uint32_t c = rw & kIdxMask;
			const bool hot = rw & kHot;
			ld32_nc((hot ? Hb : Xb) + uint64_t(c) * (hot ? hs : xs), xv[u]);
			if constexpr (SCALE_IN) sc[u] = hot ? 1.f : static_cast<const float *>(a.s_in)[c];
			ends |= (rw >> 31) << u;
		}
		if (half == 1 && s + 1 < s_end) ld32_nc(a.col + size_t(s + 1) * kStep, raw8);
#pragma unroll
		for (int u = 0; u < U; u++) {
			float f[VEC];
			widen<XT, VEC>(xv[u], f);
#pragma unroll
			for (int i = 0; i < VEC / 2; i++) {
				float t0 = f[2 * i], t1 = f[2 * i + 1];
				// (x * s_in) * w, each product rounded, like scale_rows then SpMM
				if constexpr (SCALE_IN) { t0 = __fmul_rn(t0, sc[u]); t1 = __fmul_rn(t1, sc[u]); }
				if constexpr (!kBinary) { t0 = __fmul_rn(t0, w[u]); t1 = __fmul_rn(t1, w[u]); }
				p[i] = add2(p[i], pack2(t0, t1));
			}
			const bool end = runs && ((ends >> u) & 1u);
			float so = 1.f;
			if constexpr (SCALE_OUT) so = end ? static_cast<const float *>(a.s_out)[row] : 1.f;
			float o[VEC];
#pragma unroll
			for (int i = 0; i < VEC / 2; i++) {
				unpack2(p[i], o[2 * i], o[2 * i + 1]);
				if constexpr (SCALE_OUT) { o[2 * i] = __fmul_rn(o[2 * i], so); o[2 * i + 1] = __fmul_rn(o[2 * i + 1], so); }
			}
			char *yp = Yb + uint64_t(row) * ys;
			if constexpr (sizeof(YT) == 4) {
#pragma unroll
				for (int h = 0; h < VEC / 8; h++) {
					uint32_t v[8];
#pragma unroll
					for (int i = 0; i < 8; i++) v[i] = __float_as_uint(o[8 * h + i]);
					st32_if(yp + 32 * h, v, end);
				}
			} else {
				uint32_t v[8];
#pragma unroll
				for (int i = 0; i < 8; i++) {
					__nv_bfloat162 b2 = __floats2bfloat162_rn(o[2 * i], o[2 * i + 1]);
					memcpy(&v[i], &b2, 4);
				}
				st32_if(yp, v, end);
			}
#pragma unroll
			for (int i = 0; i < VEC / 2; i++) p[i] = end ? 0ull : p[i];
			row += end;
		}
		}
	}
	if (!runs) {
		float *q = static_cast<float *>(a.partial) + int64_t(rg.slot) * kPartialStride + colbase;
#pragma unroll
		for (int i = 0; i < VEC / 2; i++) unpack2(p[i], q[2 * i], q[2 * i + 1]);
	}
}

template <class XT, class YT, class WT, int U, bool SCALE_IN, bool SCALE_OUT>
__global__ void __launch_bounds__(kThreads, FMX_WIDE_MIN_BLOCKS) spmm_wide_kernel(const spmm_args a)
{
	constexpr int VEC = int(32 / sizeof(XT));
	const int lane = threadIdx.x & 31;
	const uint32_t gw = (blockIdx.x * kThreads + threadIdx.x) >> 5;
	const uint32_t nw = (gridDim.x * kThreads) >> 5;
	const int G = a.G, R = a.R;
	const int grp = lane / G;
	if (grp >= R) return;
	const int colbase = (lane - grp * G) * VEC;
	const uint32_t gg = gw * uint32_t(R) + uint32_t(grp);
	const uint32_t ng = nw * uint32_t(R);
	for (uint32_t r = gg; r < a.n_ranges; r += ng)
		run_range_wide<XT, YT, WT, U, SCALE_IN, SCALE_OUT>(a, a.ranges[r], colbase);
}

// k = 1 (SpMV): a warp per range.  The 32 lanes load the range's column ids
// (coalesced) and gather its X values into shared memory, one entry each;
// then each lane sums whole rows of the range from shared memory in entry
// order, with one running sum per row and every add rounded, which is the
// lane-group kernel's arithmetic: rows of up to 256 entries come out
// identical.  A chunk of a longer row is added up by the whole warp (each
// lane its own entries, then a fixed xor tree) into its partial slot.  (The lane-group
// kernel at k = 1 gives each lane a whole range and waits on one step of 4
// gathers at a time.)
constexpr int kSpmvMax = 512;            // most entries of one range
static_assert(((kRange - 1 + kExactMax + kStep - 1) / kStep) * kStep <= uint32_t(kSpmvMax) &&
		kChunk <= uint32_t(kSpmvMax), "a range fits the SpMV kernel's staging");

template <class T, class WT, bool EPI>
__global__ void __launch_bounds__(kThreads) spmv_kernel(const spmm_args a, const pr_epi e)
{
	if constexpr (EPI) {
		if (e.state[1]) return;           // converged in an earlier iteration
	}
	constexpr int kWarps = kThreads / 32;
	constexpr int J = kSpmvMax / 32;
	constexpr bool kBinary = std::is_void<WT>::value;
	__shared__ T sval[kWarps][kSpmvMax];
	__shared__ uint16_t send[kWarps][kSpmvMax];
	const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
	const uint32_t gw = (blockIdx.x * kThreads + threadIdx.x) >> 5;
	const uint32_t nw = (gridDim.x * kThreads) >> 5;
	const T *X = static_cast<const T *>(a.X);
	const T *H = static_cast<const T *>(a.xhot);
	const uint64_t pol_hot = policy_evict_last(), pol_cold = policy_evict_first();
	unsigned cnt = 0;
	for (uint32_t r = gw; r < a.n_ranges; r += nw) {
		const range_t rg = a.ranges[r];
		const bool runs = rg.slot == kNoSlot;
		uint32_t raw[J];
#pragma unroll
		for (int j = 0; j < J; j++) {
			const uint32_t i = uint32_t(j * 32 + lane);
			raw[j] = i < rg.len ? __ldcs(a.col + rg.e0 + i) : 0u;
		}
		T t[J];
#pragma unroll
		for (int j = 0; j < J; j++) {
			const uint32_t i = uint32_t(j * 32 + lane);
			t[j] = T(0);
			if (i < rg.len) {
				const uint32_t c = raw[j] & kIdxMask;
				const bool hot = raw[j] & kHot;
				t[j] = ld_x_hint<T, 1>((hot ? H : X) + int64_t(c) * (hot ? int64_t(1) : a.ldx),
						hot ? pol_hot : pol_cold).v[0];
			}
		}
		if constexpr (!kBinary) {
#pragma unroll
			for (int j = 0; j < J; j++) {
				const uint32_t i = uint32_t(j * 32 + lane);
				if (i < rg.len) t[j] = acc_mul(t[j], T(__ldcs(static_cast<const WT *>(a.val) + rg.e0 + i)));
			}
		}
		// stage the products and the row ends (entry index of each row's last entry)
		int nrow = 0;
#pragma unroll
		for (int j = 0; j < J; j++) {
			const uint32_t i = uint32_t(j * 32 + lane);
			const bool is_end = runs && i < rg.len && (raw[j] >> 31);
			const uint32_t b = __ballot_sync(0xffffffffu, is_end);
			if (is_end) send[wib][nrow + __popc(b & ((1u << lane) - 1u))] = uint16_t(i);
			nrow += __popc(b);
			sval[wib][i] = t[j];
		}
		__syncwarp();
		if (runs) {
			for (int q = lane; q < nrow; q += 32) {
				const int b0 = q ? int(send[wib][q - 1]) + 1 : 0, b1 = send[wib][q];
				T acc = T(0);
				for (int i = b0; i <= b1; i++) acc = acc_add(acc, sval[wib][i]);
				const uint32_t row = rg.row0 + uint32_t(q);
				if constexpr (EPI) {
					if (!((__ldg(e.heavy_mask + (row >> 5)) >> (row & 31)) & 1u)) pr_update(e, int64_t(row), acc, cnt);
				} else {
					static_cast<T *>(a.Y)[int64_t(row) * a.ldy] = acc;
				}
			}
		} else {
			// a chunk: each lane adds its entries (j order), then a fixed xor tree
			T acc = T(0);
#pragma unroll
			for (int j = 0; j < J; j++) acc = acc_add(acc, t[j]);
#pragma unroll
			for (int o = 16; o > 0; o >>= 1) acc = acc_add(acc, __shfl_xor_sync(0xffffffffu, acc, o));
			if (lane == 0) static_cast<T *>(a.partial)[int64_t(rg.slot) * kPartialStride] = acc;
		}
		__syncwarp();
	}
	if constexpr (EPI) {
		cnt = __reduce_add_sync(0xffffffffu, cnt);
		if (lane == 0 && cnt) atomicAdd(e.state, (unsigned long long)cnt);
	}
}

// Pack the hot columns' X rows of this panel behind a zero row:
// xhot[0][j] = 0 and xhot[s+1][j] = X[hot_col[s]][c0 + j] (times
// s_in[hot_col[s]], rounded, when SCALE_IN), j < kp.  The zero row is
// rewritten every call because a narrower earlier panel packs over it.
template <class XT, class A, bool SCALE_IN>
__global__ void pack_hot_kernel(const int32_t *hot_col, uint32_t n_hot, const XT *X, int64_t ldx, int kp,
		XT *xhot, int hot_ld, const A *s_in)
{
	const uint64_t total = uint64_t(n_hot + 1) * kp;
	for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += uint64_t(gridDim.x) * blockDim.x) {
		const uint32_t s = uint32_t(t / kp);
		const int j = int(t - uint64_t(s) * kp);
		XT v = XT(0);
		if (s > 0) {
			const int32_t c = __ldg(hot_col + s - 1);
			v = X[int64_t(c) * ldx + j];
			if constexpr (SCALE_IN) v = from_acc<XT, A>(acc_mul(to_acc<A>(v), s_in[c]));
		}
		xhot[int64_t(s) * hot_ld + j] = v;
	}
}

// The same in 16-byte units (rows of whole units, 16-byte aligned), with 4
// units in flight per thread: the copy is a gather of random rows of X, and
// one 4-byte element per thread left it at a third of the bandwidth its
// bytes allow.
template <class XT, class A, bool SCALE_IN>
__global__ void pack_hot_vec_kernel(const int32_t *hot_col, uint32_t n_hot, const XT *X, int64_t ldx, int units,
		XT *xhot, int hot_ld, const A *s_in)
{
	constexpr int E = int(16 / sizeof(XT));
	constexpr int D = 4;
	const uint64_t total = uint64_t(n_hot + 1) * units;
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for (uint64_t t0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t0 < total; t0 += D * stride) {
		uint4 v[D];
		int32_t c[D];
#pragma unroll
		for (int q = 0; q < D; q++) {
			const uint64_t t = t0 + q * stride;
			v[q] = make_uint4(0, 0, 0, 0);
			c[q] = -1;
			if (t < total) {
				const uint32_t sl = uint32_t(t / units);
				const int u = int(t - uint64_t(sl) * units);
				if (sl > 0) {
					c[q] = __ldg(hot_col + sl - 1);
					v[q] = __ldg(reinterpret_cast<const uint4 *>(X + int64_t(c[q]) * ldx) + u);
				}
			}
		}
#pragma unroll
		for (int q = 0; q < D; q++) {
			const uint64_t t = t0 + q * stride;
			if (t >= total) continue;
			const uint32_t sl = uint32_t(t / units);
			const int u = int(t - uint64_t(sl) * units);
			if constexpr (SCALE_IN) {
				if (c[q] >= 0) {
					XT e[E];
					memcpy(e, &v[q], 16);
					const A sc = s_in[c[q]];
#pragma unroll
					for (int i = 0; i < E; i++) e[i] = from_acc<XT, A>(acc_mul(to_acc<A>(e[i]), sc));
					memcpy(&v[q], e, 16);
				}
			}
			*reinterpret_cast<uint4 *>(xhot + int64_t(sl) * hot_ld + int64_t(u) * E) = v[q];
		}
	}
}

// The hot pack of one panel: 16-byte units when the rows allow it.
template <class XT, class A>
static int launch_pack(const gpu_part &p, const XT *X, int64_t ldx, int kp, XT *xhot, int hot_ld, const A *s_in,
		cudaStream_t st)
{
	const bool vec = (kp * sizeof(XT)) % 16 == 0 && (ldx * sizeof(XT)) % 16 == 0 && (hot_ld * sizeof(XT)) % 16 == 0 &&
			(reinterpret_cast<uintptr_t>(X) & 15) == 0 && (reinterpret_cast<uintptr_t>(xhot) & 15) == 0;
	if (vec) {
		const int units = int(kp * sizeof(XT) / 16);
		const uint64_t total = uint64_t(p.n_hot + 1) * units;
		const unsigned pb = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((total + 1023) / 1024, 148ull * 8)));
		if (s_in) pack_hot_vec_kernel<XT, A, true><<<pb, 256, 0, st>>>(p.hot_col, p.n_hot, X, ldx, units, xhot, hot_ld, s_in);
		else pack_hot_vec_kernel<XT, A, false><<<pb, 256, 0, st>>>(p.hot_col, p.n_hot, X, ldx, units, xhot, hot_ld, nullptr);
	} else {
		const uint64_t total = uint64_t(p.n_hot + 1) * kp;
		const unsigned pb = unsigned(std::min<uint64_t>((total + 255) / 256, 148ull * 16));
		if (s_in) pack_hot_kernel<XT, A, true><<<pb, 256, 0, st>>>(p.hot_col, p.n_hot, X, ldx, kp, xhot, hot_ld, s_in);
		else pack_hot_kernel<XT, A, false><<<pb, 256, 0, st>>>(p.hot_col, p.n_hot, X, ldx, kp, xhot, hot_ld, nullptr);
	}
	CUDA_TRY(cudaGetLastError());
	return FMX_OK;
}

// Part `part` of P adds chunks part, part + P, ... of one column unit (a
// float4 when vec, else one element) into two running sums (even and odd
// steps).
template <class A>
__device__ __forceinline__ void chunk_sums(const A *pc, uint32_t part, uint32_t P, uint32_t count, bool vec,
		A (&s0)[4], A (&s1)[4])
{
	constexpr bool kVec4 = std::is_same<A, float>::value;
	uint32_t c = part;
	for (; c + P < count; c += 2u * P) {
		if constexpr (kVec4) {
			if (vec) {
				const float4 a = *reinterpret_cast<const float4 *>(pc + int64_t(c) * kPartialStride);
				const float4 b = *reinterpret_cast<const float4 *>(pc + int64_t(c + P) * kPartialStride);
				s0[0] = acc_add(s0[0], a.x); s0[1] = acc_add(s0[1], a.y);
				s0[2] = acc_add(s0[2], a.z); s0[3] = acc_add(s0[3], a.w);
				s1[0] = acc_add(s1[0], b.x); s1[1] = acc_add(s1[1], b.y);
				s1[2] = acc_add(s1[2], b.z); s1[3] = acc_add(s1[3], b.w);
				continue;
			}
		}
		s0[0] = acc_add(s0[0], pc[int64_t(c) * kPartialStride]);
		s1[0] = acc_add(s1[0], pc[int64_t(c + P) * kPartialStride]);
	}
	if (c < count) {
		if constexpr (kVec4) {
			if (vec) {
				const float4 a = *reinterpret_cast<const float4 *>(pc + int64_t(c) * kPartialStride);
				s0[0] = acc_add(s0[0], a.x); s0[1] = acc_add(s0[1], a.y);
				s0[2] = acc_add(s0[2], a.z); s0[3] = acc_add(s0[3], a.w);
				return;
			}
		}
		s0[0] = acc_add(s0[0], pc[int64_t(c) * kPartialStride]);
	}
}

// The longest heavy rows (more than kBlockChunks chunks, the first n_block of
// the list): a block of 8 warps per row, 8 * 32 / L parts, each warp's parts
// combined by the xor tree and the 8 warp sums added in warp order.  The
// chain of one part is then at most count / (8 * 32 / L) chunks long instead
// of count / (32 / L), which bounded the whole fixup by its longest row.
template <class YT, class A, bool SCALE_OUT, bool EPI = false>
__global__ void __launch_bounds__(256) spmm_fixup_block_kernel(const heavy_row *heavy, const A *partial, YT *Y,
		int64_t ldy, int k, const A *s_out, int L, const pr_epi e)
{
	if constexpr (EPI) {
		if (e.state[1]) return;
	}
	__shared__ A red[8][32][4];
	constexpr bool kVec4 = std::is_same<A, float>::value;
	const bool vec = kVec4 && (k % 4) == 0;
	const int units = vec ? k / 4 : k;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int per_warp = 32 / L;
	const int P = 8 * per_warp;
	const int cl = lane % L, part = warp * per_warp + lane / L;
	const heavy_row h = heavy[blockIdx.x];
	for (int u0 = 0; u0 < units; u0 += L) {           // the same trip count on every thread
		const int u = u0 + cl;
		const bool mine = u < units;
		A s0[4] = {A(0), A(0), A(0), A(0)}, s1[4] = {A(0), A(0), A(0), A(0)};
		if (mine) chunk_sums<A>(partial + int64_t(h.first) * kPartialStride + (vec ? 4 * u : u), uint32_t(part),
				uint32_t(P), h.count, vec, s0, s1);
		A t[4];
#pragma unroll
		for (int i = 0; i < 4; i++) t[i] = acc_add(s0[i], s1[i]);
		for (int o = L; o < 32; o <<= 1)
#pragma unroll
			for (int i = 0; i < 4; i++) t[i] = acc_add(t[i], __shfl_xor_sync(0xffffffffu, t[i], o));
		if (lane < L)
#pragma unroll
			for (int i = 0; i < 4; i++) red[warp][lane][i] = t[i];
		__syncthreads();
		if (warp == 0 && lane < L && mine) {
			A v[4];
#pragma unroll
			for (int i = 0; i < 4; i++) {
				v[i] = red[0][lane][i];
				for (int w = 1; w < 8; w++) v[i] = acc_add(v[i], red[w][lane][i]);
			}
			if constexpr (EPI) {
				unsigned c = 0;
				pr_update(e, h.row, v[0], c);
				if (c) atomicAdd(e.state, 1ull);
			} else {
				A so = A(1);
				if constexpr (SCALE_OUT) so = s_out[h.row];
				YT *y = Y + int64_t(h.row) * ldy + (vec ? 4 * u : u);
				for (int i = 0; i < (vec ? 4 : 1); i++) {
					A x = v[i];
					if constexpr (SCALE_OUT) x = acc_mul(x, so);
					y[i] = from_acc<YT, A>(x);
				}
			}
		}
		__syncthreads();
	}
}

// Heavy rows: add the chunk partials, scale, convert, store.  A row's
// columns are covered by L lanes (L = k / 4 float4 lanes for FP32 panels of
// k % 4 == 0, else one lane per column, rounded up to a power of two, at most
// 32) and its chunks by P parts: part q adds chunks q, q + P, ... into two
// running sums, and the parts are combined by a fixed xor tree.  The heavy
// rows come longest first: each of the first n_long rows (more than
// kLongChunks chunks) gets a warp with P = 32 / L; the rest go 32 / (2 L)
// rows to a warp with P = 2 (one row and P = 1 when L = 32).  Deterministic,
// with many loads in flight.
template <class YT, class A, bool SCALE_OUT, bool EPI = false>
__global__ void spmm_fixup_kernel(const heavy_row *heavy, uint32_t n_heavy, uint32_t n_long, const A *partial,
		YT *Y, int64_t ldy, int k, const A *s_out, int L, const pr_epi e)
{
	if constexpr (EPI) {
		if (e.state[1]) return;
	}
	constexpr bool kVec4 = std::is_same<A, float>::value;
	const bool vec = kVec4 && (k % 4) == 0;
	const int units = vec ? k / 4 : k;
	const uint64_t w = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	const bool long_rows = w < n_long;
	const int P = long_rows ? 32 / L : (L < 32 ? 2 : 1);
	const int lanes = L * P;                          // per row
	const uint64_t r = long_rows ? w : uint64_t(n_long) + (w - n_long) * uint64_t(32 / lanes) + uint64_t(lane / lanes);
	const int sub = lane % lanes, part = sub / L, cl = sub % L;
	const bool live = r < n_heavy;
	heavy_row h{0, 0, 0};
	if (live) h = heavy[r];
	for (int u0 = 0; u0 < units; u0 += L) {           // the same trip count on every lane
		const int u = u0 + cl;
		const bool mine = live && u < units;
		A s0[4] = {A(0), A(0), A(0), A(0)}, s1[4] = {A(0), A(0), A(0), A(0)};
		if (mine) chunk_sums<A>(partial + int64_t(h.first) * kPartialStride + (vec ? 4 * u : u), uint32_t(part),
				uint32_t(P), h.count, vec, s0, s1);
		const int nv = vec ? 4 : 1;
		A t[4];
#pragma unroll
		for (int i = 0; i < 4; i++) t[i] = acc_add(s0[i], s1[i]);
		for (int o = L; o < lanes; o <<= 1)
#pragma unroll
			for (int i = 0; i < 4; i++) t[i] = acc_add(t[i], __shfl_xor_sync(0xffffffffu, t[i], o));
		if constexpr (EPI) {
			if (mine && part == 0) {
				unsigned c = 0;
				pr_update(e, h.row, t[0], c);
				if (c) atomicAdd(e.state, 1ull);
			}
			continue;
		}
		if (mine && part == 0) {
			A so = A(1);
			if constexpr (SCALE_OUT) so = s_out[h.row];
			YT *y = Y + int64_t(h.row) * ldy + (vec ? 4 * u : u);
			for (int i = 0; i < nv; i++) {
				A v = t[i];
				if constexpr (SCALE_OUT) v = acc_mul(v, so);
				y[i] = from_acc<YT, A>(v);
			}
		}
	}
}

template <class YT, class A, bool SCALE_OUT, bool EPI = false>
static int launch_fixup(const gpu_part &p, const A *partial, YT *Y, int64_t ldy, int k, const A *s_out,
		cudaStream_t st, const pr_epi &e = pr_epi{})
{
	if (!p.n_heavy) return FMX_OK;
	const bool vec = std::is_same<A, float>::value && (k % 4) == 0;
	const int units = vec ? k / 4 : k;
	int L = 1;
	while (L < units && L < 32) L <<= 1;
	const uint32_t nb = p.n_block_heavy;
	if (nb) {
		spmm_fixup_block_kernel<YT, A, SCALE_OUT, EPI><<<nb, 256, 0, st>>>(p.heavy, partial, Y, ldy, k, s_out, L, e);
		CUDA_TRY(cudaGetLastError());
	}
	if (p.n_heavy == nb) return FMX_OK;
	const uint64_t n_long = p.n_long_heavy - nb;
	const uint64_t n_short = p.n_heavy - p.n_long_heavy;
	const uint64_t per_warp = uint64_t(32 / (L * (L < 32 ? 2 : 1)));    // short rows per warp
	const uint64_t warps = n_long + (n_short + per_warp - 1) / per_warp;
	const unsigned fb = unsigned((warps * 32 + 255) / 256);
	spmm_fixup_kernel<YT, A, SCALE_OUT, EPI><<<fb, 256, 0, st>>>(p.heavy + nb, p.n_heavy - nb, uint32_t(n_long),
			partial, Y, ldy, k, s_out, L, e);
	CUDA_TRY(cudaGetLastError());
	return FMX_OK;
}

// ---------------------------------------------------------------------------
// Host: building the resident layout
// ---------------------------------------------------------------------------

template <class T>
static int upload(T **dst, const T *src, size_t n, uint64_t &bytes, size_t alloc_n = 0)
{
	*dst = nullptr;
	alloc_n = std::max(alloc_n, n);
	if (!alloc_n) return FMX_OK;
	cudaError_t e = cudaMalloc(reinterpret_cast<void **>(dst), alloc_n * sizeof(T));
	if (e != cudaSuccess)
		return set_error(e == cudaErrorMemoryAllocation ? FMX_ERR_OOM : FMX_ERR_CUDA,
				"cudaMalloc of %zu bytes failed: %s", alloc_n * sizeof(T), cudaGetErrorString(e));
	bytes += alloc_n * sizeof(T);
	if (n) CUDA_TRY(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
	if (alloc_n > n) CUDA_TRY(cudaMemset(reinterpret_cast<char *>(*dst) + n * sizeof(T), 0, (alloc_n - n) * sizeof(T)));
	return FMX_OK;
}

template <class F>
static void par_for(uint64_t n, F fn)
{
	int nt = std::max(1, std::min<int>(default_threads(), int((n + 65535) / 65536)));
	std::vector<std::thread> th;
	uint64_t per = (n + nt - 1) / nt;
	for (int t = 0; t < nt; t++)
		th.emplace_back([&, t]() {
			uint64_t b = uint64_t(t) * per, e = std::min(n, b + per);
			if (b < e) fn(b, e);
		});
	for (auto &x : th) x.join();
}

// A streamed part's pinned host copy of the entry stream, its two device
// slots (the largest slice plus kStep entries, zeroed) and its copy stream
// and events.  Called with the part's device current.
static int stream_buffers(gpu_part &p, const std::vector<uint32_t> &col, const std::vector<char> &val, size_t es)
{
	uint64_t cap = 0;
	for (const auto &sl : p.slices) cap = std::max<uint64_t>(cap, sl.e1 - sl.e0);
	cap += kStep;
	auto host = [&](void **h, const void *src, size_t n) -> int {
		cudaError_t e = cudaHostAlloc(h, std::max<size_t>(n, 16), cudaHostAllocDefault);
		if (e != cudaSuccess) return set_error(FMX_ERR_OOM, "pinned host stream of %zu bytes: %s", n, cudaGetErrorString(e));
		if (n) memcpy(*h, src, n);
		p.host_bytes += n;
		return FMX_OK;
	};
	if (int rc = host(reinterpret_cast<void **>(&p.h_col), col.data(), col.size() * sizeof(uint32_t))) return rc;
	if (es)
		if (int rc = host(&p.h_val, val.data(), val.size())) return rc;
	for (int b = 0; b < 2; b++) {
		CUDA_TRY(cudaMalloc(&p.slot_col[b], cap * sizeof(uint32_t)));
		CUDA_TRY(cudaMemset(p.slot_col[b], 0, cap * sizeof(uint32_t)));
		p.bytes += cap * sizeof(uint32_t);
		if (es) {
			CUDA_TRY(cudaMalloc(&p.slot_val[b], cap * es));
			CUDA_TRY(cudaMemset(p.slot_val[b], 0, cap * es));
			p.bytes += cap * es;
		}
		CUDA_TRY(cudaEventCreateWithFlags(&p.ev_copied[b], cudaEventDisableTiming));
		CUDA_TRY(cudaEventCreateWithFlags(&p.ev_free[b], cudaEventDisableTiming));
	}
	CUDA_TRY(cudaEventCreateWithFlags(&p.ev_start, cudaEventDisableTiming));
	CUDA_TRY(cudaStreamCreateWithFlags(&p.copy_st, cudaStreamNonBlocking));
	return FMX_OK;
}

// slice_entries > 0: a streamed part whose slices hold about that many entries.
static int make_part(const host_csr &csr, int device, std::shared_ptr<gpu_part> &out, uint64_t slice_entries = 0)
{
	if (csr.ncols > (1ull << 30))
		return set_error(FMX_ERR_UNSUPPORTED, "%llu columns: the entry stream holds 30-bit column ids",
				(unsigned long long)csr.ncols);
	auto p = std::make_shared<gpu_part>();
	p->device = device;
	p->nrows = csr.nrows; p->ncols = csr.ncols; p->nnz = csr.nnz;
	p->prim = csr.prim; p->esize = csr.esize;
	const uint64_t n = csr.nrows;
	const size_t es = csr.esize;

	// hot columns: the highest in-degrees (at least 2), up to kHotMax
	std::vector<std::atomic<uint32_t>> indeg(csr.ncols);
	par_for(csr.ncols, [&](uint64_t b, uint64_t e) { for (uint64_t i = b; i < e; i++) indeg[i].store(0, std::memory_order_relaxed); });
	par_for(csr.nnz, [&](uint64_t b, uint64_t e) {
		for (uint64_t i = b; i < e; i++) indeg[csr.col[i]].fetch_add(1, std::memory_order_relaxed);
	});
	std::vector<int32_t> hot_col;
	std::vector<int32_t> slot_of(csr.ncols, -1);
	{
		// counting sort of the columns by in-degree, descending, capped
		const uint32_t cap = 1u << 16;
		std::vector<uint64_t> cnt(cap + 2, 0);
		for (uint64_t c = 0; c < csr.ncols; c++) {
			uint32_t d = std::min(indeg[c].load(std::memory_order_relaxed), cap);
			if (d >= 2) cnt[cap - d + 1]++;
		}
		for (size_t i = 1; i < cnt.size(); i++) cnt[i] += cnt[i - 1];
		const uint64_t nhot = std::min<uint64_t>(kHotMax, cnt.back());
		std::vector<int32_t> order(cnt.back());
		for (uint64_t c = 0; c < csr.ncols; c++) {
			uint32_t d = std::min(indeg[c].load(std::memory_order_relaxed), cap);
			if (d >= 2) order[cnt[cap - d]++] = int32_t(c);
		}
		hot_col.assign(order.begin(), order.begin() + nhot);
		// slot 0 is the zero row; hot columns take slots 1..nhot
		for (uint64_t s = 0; s < nhot; s++) slot_of[hot_col[s]] = int32_t(s + 1);
	}

	// Work segments: runs of consecutive rows (every row in order; an exact
	// row with its entries, an empty or longer row as one zero-row entry),
	// then the equal chunks of the longer rows (the rule of seg_row_len in
	// part.h, which make_part_device follows too).  Each segment starts at a
	// multiple of kStep in the stream and is padded to one.
	const uint32_t zero_entry = 0u | kHot;          // slot 0: the zero row
	struct seg_t { uint64_t row0, row1; uint32_t b, e; uint32_t slot; uint64_t at; uint32_t len; };
	std::vector<seg_t> segs;
	std::vector<heavy_row> heavy;
	uint32_t n_exact = 0;
	{
		uint64_t total = 0;
		for (uint64_t r = 0; r < n; r++) total += seg_row_len(csr.row_ptr[r + 1] - csr.row_ptr[r]);
		const uint32_t run = range_entries(total);
		uint64_t L = 0, bucket = ~0ull;           // lens of the rows before r
		for (uint64_t r = 0; r < n; r++) {
			const uint32_t d = csr.row_ptr[r + 1] - csr.row_ptr[r];
			const uint32_t len = seg_row_len(d);
			n_exact += (d >= 1 && d <= kExactMax);
			if (L / run != bucket) {
				segs.push_back({r, r + 1, 0, 0, kNoSlot, 0, 0});
				bucket = L / run;
			} else {
				segs.back().row1 = r + 1;
			}
			L += len;
			segs.back().len += len;
		}
	}
	uint32_t slots = 0;
	for (uint64_t r = 0; r < n; r++) {
		const uint32_t d = csr.row_ptr[r + 1] - csr.row_ptr[r];
		if (d <= kExactMax) continue;
		const uint32_t cnt = (d + kChunk - 1) / kChunk;   // equal chunks of <= kChunk entries
		heavy.push_back({int32_t(r), slots, cnt});
		for (uint32_t c = 0; c < cnt; c++) {
			const uint32_t b = uint32_t(uint64_t(d) * c / cnt), e = uint32_t(uint64_t(d) * (c + 1) / cnt);
			segs.push_back({r, r + 1, b, e, slots + c, 0, e - b});
		}
		slots += cnt;
	}
	uint64_t total = 0;
	for (auto &g : segs) {
		g.at = total;
		g.len = (g.len + kStep - 1) / kStep * kStep;
		total += g.len;
	}
	if (total >= (1ull << 32) - 64)
		return set_error(FMX_ERR_UNSUPPORTED, "%llu stream entries: offsets are 32-bit", (unsigned long long)total);
	std::vector<range_t> ranges(segs.size());
	for (size_t i = 0; i < segs.size(); i++)
		ranges[i] = {uint32_t(segs[i].at), segs[i].len, uint32_t(segs[i].row0), segs[i].slot};
	// largest ranges first, so that round-robin assignment balances the groups
	// (within each slice of a streamed part: a slice is whole segments in
	// stream order, at least slice_entries entries but the last)
	auto by_len = [](const range_t &x, const range_t &y) { return x.len > y.len; };
	if (slice_entries) {
		p->streamed = true;
		uint64_t e0 = 0;
		size_t i0 = 0;
		for (size_t i = 0; i < segs.size(); i++) {
			const uint64_t e1 = segs[i].at + segs[i].len;
			if (e1 - e0 >= slice_entries || i + 1 == segs.size()) {
				p->slices.push_back({e0, e1, uint32_t(i0), uint32_t(i + 1 - i0)});
				std::stable_sort(ranges.begin() + i0, ranges.begin() + i + 1, by_len);
				e0 = e1;
				i0 = i + 1;
			}
		}
	} else {
		std::stable_sort(ranges.begin(), ranges.end(), by_len);
	}

	// the entry stream (plus kStep entries so that index prefetches stay in bounds)
	const size_t padded = total + kStep;
	std::vector<uint32_t> col(total, zero_entry);
	std::vector<char> val(total * es, 0);
	std::atomic<uint64_t> hot_entries{0};
	auto put = [&](uint64_t r, uint32_t b, uint32_t e, uint64_t at) {
		const uint32_t rb = csr.row_ptr[r];
		uint64_t h = 0;
		for (uint32_t i = b; i < e; i++) {
			const uint32_t c = uint32_t(csr.col[rb + i]);
			const int32_t sl = slot_of[c];
			col[at + (i - b)] = sl >= 0 ? (uint32_t(sl) | kHot) : c;
			h += sl >= 0;
		}
		if (es) memcpy(&val[at * es], &csr.val[size_t(rb + b) * es], size_t(e - b) * es);
		return h;
	};
	par_for(segs.size(), [&](uint64_t sb, uint64_t se) {
		uint64_t h = 0;
		for (uint64_t i = sb; i < se; i++) {
			const seg_t &g = segs[i];
			if (g.slot != kNoSlot) { h += put(g.row0, g.b, g.e, g.at); continue; }
			uint64_t at = g.at;
			for (uint64_t r = g.row0; r < g.row1; r++) {
				const uint32_t d = csr.row_ptr[r + 1] - csr.row_ptr[r];
				if (d >= 1 && d <= kExactMax) {
					h += put(r, 0, d, at);
					at += d;
				} else {
					at += 1;                 // the zero-row entry already there
				}
				col[at - 1] |= kEnd;
			}
		}
		hot_entries += h;
	});
	p->hot_entries = hot_entries.load();

	int cur = 0;
	cudaGetDevice(&cur);
	CUDA_TRY(cudaSetDevice(device));
	int rc = FMX_OK;
	uint64_t &bytes = p->bytes;
	if (p->streamed) {
		rc = stream_buffers(*p, col, val, es);
	} else {
		rc = upload(&p->col, col.data(), col.size(), bytes, padded);
		if (!rc && es) {
			char *v = nullptr;
			rc = upload(&v, val.data(), val.size(), bytes, padded * es);
			p->val = v;
		}
	}
	if (!rc) rc = upload(&p->hot_col, hot_col.data(), hot_col.size(), bytes);
	if (!rc) rc = upload(&p->ranges, ranges.data(), ranges.size(), bytes);
	// longest first (the fixup gives each long row a warp and packs the short
	// ones several to a warp); ties keep row order
	std::stable_sort(heavy.begin(), heavy.end(), [](const heavy_row &x, const heavy_row &y) { return x.count > y.count; });
	p->n_long_heavy = uint32_t(std::count_if(heavy.begin(), heavy.end(),
			[](const heavy_row &h) { return h.count > kLongChunks; }));
	p->n_block_heavy = uint32_t(std::count_if(heavy.begin(), heavy.end(),
			[](const heavy_row &h) { return h.count > kBlockChunks; }));
	if (!rc) rc = upload(&p->heavy, heavy.data(), heavy.size(), bytes);
	p->n_hot = uint32_t(hot_col.size());
	p->n_exact = n_exact;
	p->n_ranges = uint32_t(ranges.size());
	p->n_heavy = uint32_t(heavy.size());
	p->n_partials = slots;
	auto scratch = [&](void **ptr, size_t sz, const char *what) {
		if (rc || !sz) return;
		cudaError_t e = cudaMalloc(ptr, sz);
		if (e != cudaSuccess)
			rc = set_error(FMX_ERR_OOM, "cudaMalloc of %zu %s bytes failed: %s", sz, what, cudaGetErrorString(e));
		else bytes += sz;
	};
	scratch(&p->partial, size_t(slots) * kPartialStride * 8, "partial-sum");
	scratch(&p->xhot, size_t(p->n_hot + 1) * kPanelBytes, "hot-pack");
	if (!rc && cudaMemset(p->xhot, 0, size_t(p->n_hot + 1) * kPanelBytes) != cudaSuccess)
		rc = set_error(FMX_ERR_CUDA, "clearing the hot pack failed");
	cudaSetDevice(cur);
	if (rc) return rc;
	out = p;
	return FMX_OK;
}

// ---------------------------------------------------------------------------
// Host: launching
// ---------------------------------------------------------------------------

template <class K>
static unsigned persistent_blocks(K kernel, int device)
{
	int sms = 0, per = 0;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kThreads, 0);
	return unsigned(std::max(1, sms) * std::max(1, per));
}

// The persistent grid of `kernel` on `device`, kept in `slot` (one array of
// slots per kernel instantiation, indexed by device; racing first calls
// compute the same value).
template <class K>
static unsigned cached_blocks(std::atomic<unsigned> &slot, K kernel, int device)
{
	unsigned b = slot.load(std::memory_order_relaxed);
	if (!b) {
		b = persistent_blocks(kernel, device);
		slot.store(b, std::memory_order_relaxed);
	}
	return b;
}

#ifndef FMX_SPMM_STEP
#define FMX_SPMM_STEP 4                  // entries gathered per stream step (4 or 8)
#endif

// Run launch(args) over the part's ranges: once for a resident entry stream;
// slice by slice for a streamed part.  Each slice is copied from pinned host
// memory into one of two device slots on the part's copy stream; the kernel
// of slice i (on st) waits for its copy, and the copy of slice i + 2 waits
// for that kernel, so copies overlap the kernels.  The slot pointer is
// rebased by the slice's first entry, so the ranges keep their absolute
// entry offsets.  The slots are the part's scratch: calls on one part must
// not overlap on the GPU (as for the hot pack and the partial sums).
template <class F>
static int over_slices(const gpu_part &p, spmm_args a, cudaStream_t st, F &&launch)
{
	if (!p.streamed) return launch(a);
	gpu_part &q = const_cast<gpu_part &>(p);
	CUDA_TRY(cudaEventRecord(q.ev_start, st));
	CUDA_TRY(cudaStreamWaitEvent(q.copy_st, q.ev_start, 0));
	for (size_t i = 0; i < p.slices.size(); i++) {
		const gpu_part::slice_t &sl = p.slices[i];
		const int b = int(i & 1);
		if (i >= 2) CUDA_TRY(cudaStreamWaitEvent(q.copy_st, q.ev_free[b], 0));
		const uint64_t ne = sl.e1 - sl.e0;
		CUDA_TRY(cudaMemcpyAsync(q.slot_col[b], p.h_col + sl.e0, ne * sizeof(uint32_t), cudaMemcpyHostToDevice,
				q.copy_st));
		if (p.esize)
			CUDA_TRY(cudaMemcpyAsync(q.slot_val[b], static_cast<const char *>(p.h_val) + sl.e0 * p.esize,
					ne * p.esize, cudaMemcpyHostToDevice, q.copy_st));
		CUDA_TRY(cudaEventRecord(q.ev_copied[b], q.copy_st));
		CUDA_TRY(cudaStreamWaitEvent(st, q.ev_copied[b], 0));
		a.col = q.slot_col[b] - sl.e0;
		a.val = p.esize ? static_cast<const void *>(static_cast<const char *>(q.slot_val[b]) - sl.e0 * p.esize)
				: nullptr;
		a.ranges = p.ranges + sl.r0;
		a.n_ranges = sl.nr;
		if (int rc = launch(a)) return rc;
		CUDA_TRY(cudaEventRecord(q.ev_free[b], st));
	}
	return FMX_OK;
}

template <class XT, class YT, class A, class WT, int VEC, int NV, bool SI, bool SO>
static int launch_one(const gpu_part &p, const spmm_args &a, cudaStream_t st)
{
	auto kern = spmm_kernel<XT, YT, A, WT, VEC, NV, FMX_SPMM_STEP, SI, SO>;
	static std::atomic<unsigned> blocks[64];
	const unsigned b = cached_blocks(blocks[p.device & 63], kern, p.device);
	kern<<<b, kThreads, 0, st>>>(a, pr_epi{});
	CUDA_TRY(cudaGetLastError());
	return FMX_OK;
}

template <class XT, class YT, class WT, bool SI, bool SO>
static int launch_wide(const gpu_part &p, const spmm_args &a, cudaStream_t st)
{
	auto kern = spmm_wide_kernel<XT, YT, WT, 4, SI, SO>;
	static std::atomic<unsigned> blocks[64];
	const unsigned b = cached_blocks(blocks[p.device & 63], kern, p.device);
	kern<<<b, kThreads, 0, st>>>(a);
	CUDA_TRY(cudaGetLastError());
	return FMX_OK;
}

template <class XT, class YT, class A, class WT, int VEC, int NV>
static int launch_t(const gpu_part &p, spmm_args a, bool sin, bool sout, cudaStream_t st, bool wide = false)
{
	if (int rc = launch_pack<XT, A>(p, static_cast<const XT *>(a.X), a.ldx, a.k, static_cast<XT *>(p.xhot), a.hot_ld,
			sin ? static_cast<const A *>(a.s_in) : nullptr, st))
		return rc;
	int rc = over_slices(p, a, st, [&](const spmm_args &sa) -> int {
		if constexpr (std::is_same<A, float>::value &&
				(sizeof(XT) == 4 || (sizeof(YT) == 2 && std::is_void<WT>::value)) &&
				(std::is_same<WT, void>::value || std::is_same<WT, float>::value)) {
			if (wide) {
				if (sin && sout) return launch_wide<XT, YT, WT, true, true>(p, sa, st);
				if (sin) return launch_wide<XT, YT, WT, true, false>(p, sa, st);
				if (sout) return launch_wide<XT, YT, WT, false, true>(p, sa, st);
				return launch_wide<XT, YT, WT, false, false>(p, sa, st);
			}
		}
		if (sin && sout) return launch_one<XT, YT, A, WT, VEC, NV, true, true>(p, sa, st);
		if (sin) return launch_one<XT, YT, A, WT, VEC, NV, true, false>(p, sa, st);
		if (sout) return launch_one<XT, YT, A, WT, VEC, NV, false, true>(p, sa, st);
		return launch_one<XT, YT, A, WT, VEC, NV, false, false>(p, sa, st);
	});
	if (rc) return rc;
	if (sout) rc = launch_fixup<YT, A, true>(p, static_cast<const A *>(a.partial), static_cast<YT *>(a.Y), a.ldy, a.k,
			static_cast<const A *>(a.s_out), st);
	else rc = launch_fixup<YT, A, false>(p, static_cast<const A *>(a.partial), static_cast<YT *>(a.Y), a.ldy, a.k,
			nullptr, st);
	if (rc) return rc;
	return FMX_OK;
}

static bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }
static bool aligned32(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 31) == 0; }

// Run one orientation over all column panels (kPanelBytes of X row each).
// k = 1 without row scales: pack, the warp-per-range SpMV, fixup.
// `xhot` and `partial` default to the part's own scratch.
template <class T, class WT, bool EPI>
static int run_spmv(const gpu_part &p, const T *X, int64_t ldx, T *Y, int64_t ldy, cudaStream_t st,
		const pr_epi &e = pr_epi{}, void *xhot = nullptr, void *partial = nullptr)
{
	if (!xhot) xhot = p.xhot;
	if (!partial) partial = p.partial;
	spmm_args a{};
	a.col = p.col; a.val = p.val; a.ranges = p.ranges;
	a.X = X; a.xhot = xhot; a.hot_ld = 1;
	a.Y = Y;
	a.partial = partial;
	a.ldx = ldx; a.ldy = ldy; a.k = 1;
	a.G = 1; a.R = 32; a.nv = 1;
	a.n_ranges = p.n_ranges;
	const unsigned pb = unsigned(std::min<uint64_t>((uint64_t(p.n_hot) + 256) / 256, 148ull * 16));
	pack_hot_kernel<T, T, false><<<pb, 256, 0, st>>>(p.hot_col, p.n_hot, X, ldx, 1, static_cast<T *>(xhot), 1,
			nullptr);
	CUDA_TRY(cudaGetLastError());
	auto kern = spmv_kernel<T, WT, EPI>;
	static std::atomic<unsigned> blocks[64];
	const unsigned b = cached_blocks(blocks[p.device & 63], kern, p.device);
	if (int rc = over_slices(p, a, st, [&](const spmm_args &sa) -> int {
			kern<<<b, kThreads, 0, st>>>(sa, e);
			CUDA_TRY(cudaGetLastError());
			return FMX_OK;
		}))
		return rc;
	return launch_fixup<T, T, false, EPI>(p, static_cast<const T *>(partial), Y, ldy, 1, nullptr, st, e);
}

template <class XT, class YT, class A, class WT>
static int run_typed(const gpu_part &p, const void *X, int64_t ldx, void *Y, int64_t ldy, int64_t k,
		const void *sin, const void *sout, cudaStream_t st)
{
	if constexpr (std::is_same<XT, A>::value && std::is_same<YT, A>::value && std::is_floating_point<A>::value) {
		if (k == 1 && !sin && !sout)
			return run_spmv<A, WT, false>(p, static_cast<const A *>(X), ldx, static_cast<A *>(Y), ldy, st);
	}
	constexpr int VEC = int(16 / sizeof(XT));
	constexpr int kPanel = kPanelBytes / int(sizeof(XT));
	// 16-byte vectors along k when every X and Y row starts 16-byte aligned
	// and k is a multiple of VEC; otherwise scalar lanes.
	const bool vec_ok = (k % VEC == 0) && (ldx % VEC == 0) && (ldy % VEC == 0) &&
			aligned16(X) && aligned16(Y) && (VEC * sizeof(YT)) % 8 == 0;
	for (int64_t c0 = 0; c0 < k; c0 += kPanel) {
		const int kp = int(std::min<int64_t>(kPanel, k - c0));
		spmm_args a{};
		a.col = p.col; a.val = p.val; a.ranges = p.ranges;
		a.X = static_cast<const XT *>(X) + c0;
		a.xhot = p.xhot;
		a.hot_ld = kp;                // packed rows back to back (two 64-byte rows per line)
		a.Y = static_cast<YT *>(Y) + c0;
		a.s_in = sin; a.s_out = sout; a.partial = p.partial;
		a.ldx = ldx; a.ldy = ldy; a.k = kp;
		a.n_ranges = p.n_ranges;
		int rc;
		// 32-byte lanes: FP32 accumulation, a panel of whole 32-byte lanes,
		// X, Y and the packed rows 32-byte aligned
		// (BF16 rows of 16 elements take the 16-byte lanes: measured at R-MAT
		// scale 24, k = 16, one 32-byte lane per row loads an index group per
		// lane and ran 2.2 ms against 1.8 ms)
		// FP32, and unweighted BF16 with BF16 output (the eigensolver's
		// correction SpMMs: 0.82 against 0.89 ms per call at scale 22,
		// k = 16); BF16 into FP32 and weighted BF16 keep the 16-byte lanes,
		// where the wider accumulators spill
		constexpr bool kWideBf16 = sizeof(YT) == 2 && std::is_void<WT>::value;
		const bool wide = std::is_same<A, float>::value && (sizeof(XT) == 4 || kWideBf16) && vec_ok &&
				(kp * sizeof(XT)) % 32 == 0 &&
				(ldx * sizeof(XT)) % 32 == 0 && (ldy * sizeof(YT)) % 32 == 0 && aligned32(a.X) && aligned32(a.Y);
		if (wide) {
			a.G = int(kp * sizeof(XT) / 32);     // 1, 2 or 4
			a.R = 32 / a.G;
			a.nv = 1;
			rc = launch_t<XT, YT, A, WT, VEC, 1>(p, a, sin, sout, st, true);
		} else if (vec_ok) {
			a.G = kp / VEC;           // <= 8
			a.R = 32 / a.G;
			a.nv = 1;
			rc = launch_t<XT, YT, A, WT, VEC, 1>(p, a, sin, sout, st);
		} else {
			int g = 1;
			while (g < 32 && g * 4 < kp) g *= 2;
			a.G = g;
			a.R = 32 / g;
			a.nv = (kp + g - 1) / g;   // <= 4
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
// Fused PageRank iteration (SpMV on A^T with the update at each row close)
// ---------------------------------------------------------------------------

// The iteration's convergence test (PageRank.cpp:96,124-129): one thread.
__global__ void pr_finish_kernel(unsigned long long *state, unsigned long long n, unsigned long long max_iters)
{
	if (threadIdx.x == 0 && !state[1]) {
		const unsigned long long it = ++state[2];
		if (state[0] >= n || it >= max_iters) state[1] = 1;
		state[0] = 0;
	}
}

__global__ void heavy_mask_kernel(const heavy_row *heavy, uint32_t n_heavy, uint32_t *mask)
{
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_heavy; i += gridDim.x * blockDim.x) {
		const uint32_t r = uint32_t(heavy[i].row);
		atomicOr(mask + (r >> 5), 1u << (r & 31));
	}
}

int pagerank_heavy_mask(const fmx_matrix *mt, uint32_t *mask, cudaStream_t st)
{
	const gpu_part &p = *mt->a;
	if (!p.n_heavy) return FMX_OK;
	heavy_mask_kernel<<<unsigned(std::min<uint32_t>((p.n_heavy + 255) / 256, 1024)), 256, 0, st>>>(p.heavy,
			p.n_heavy, mask);
	CUDA_TRY(cudaGetLastError());
	return FMX_OK;
}

template <class WT>
static int pr_iteration_typed(const gpu_part &p, const float *in, const pr_epi &e, cudaStream_t st)
{
	// the update writes pr, pr1 and the next input instead of Y
	if (int rc = run_spmv<float, WT, true>(p, in, 1, nullptr, 1, st, e)) return rc;
	pr_finish_kernel<<<1, 32, 0, st>>>(e.state, e.n, e.max_iters);
	CUDA_TRY(cudaGetLastError());
	return FMX_OK;
}

int pagerank_iteration(const fmx_matrix *mt, const float *in, const pr_epi &e, cudaStream_t st)
{
	const gpu_part &p = *mt->a;
	if (p.prim == FMX_P_BOOL) return pr_iteration_typed<void>(p, in, e, st);
	if (p.prim == FMX_P_FLOAT) return pr_iteration_typed<float>(p, in, e, st);
	return set_error(FMX_ERR_TYPE, "PageRank: binary or float-weighted matrices");
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

int matrix_device(const fmx_matrix *m) { return m && m->a ? m->a->device : 0; }

int matrix_from_csr(const host_csr &a, const host_csr *at, int device, fmx_matrix **out)
{
	*out = nullptr;
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
		return set_error(FMX_ERR_CUDA, "no CUDA device is available");
	if (device < 0 || device >= ndev) return set_error(FMX_ERR_INVAL, "device %d out of range (%d devices)", device, ndev);
	std::unique_ptr<fmx_matrix> m(new (std::nothrow) fmx_matrix);
	if (!m) return set_error(FMX_ERR_OOM, "out of host memory");
	if (int rc = make_part(a, device, m->a)) return rc;
	if (at)
		if (int rc = make_part(*at, device, m->at)) return rc;
	m->symmetric = at == nullptr;
	*out = m.release();
	return FMX_OK;
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

int fmx_matrix_create_streamed(const fmx_image *img, const fmx_image *t_img, int device, uint64_t slice_entries,
		fmx_matrix **out)
{
	if (!img || !out) return set_error(FMX_ERR_INVAL, "null argument");
	*out = nullptr;
	if (!slice_entries) slice_entries = uint64_t(1) << 26;
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
			if (!rc) rc = make_part(csr, device, i == 0 ? m->a : m->at, slice_entries);
		} catch (const std::bad_alloc &) {
			rc = set_error(FMX_ERR_OOM, "host allocation failed while decoding the image");
		}
		if (rc) return rc;
	}
	m->symmetric = (t_img == nullptr);
	*out = m.release();
	return FMX_OK;
}

int fmx_matrix_stream_info(const fmx_matrix *m, uint64_t *slices, uint64_t *host_bytes)
{
	if (!m || !m->a) return set_error(FMX_ERR_INVAL, "null matrix");
	if (slices) *slices = m->a->streamed ? m->a->slices.size() : 0;
	if (host_bytes) *host_bytes = m->a->host_bytes;
	return FMX_OK;
}

int fmx_matrix_build_device(const uint32_t *src, const uint32_t *dst, const void *vals, int val_type,
		uint64_t nedges, uint64_t nrows, uint64_t ncols, int flags, int device, void *stream, fmx_matrix **out)
{
	if (!out || (nedges && (!src || !dst)) || (val_type != FMX_P_BOOL && nedges && !vals))
		return set_error(FMX_ERR_INVAL, "null argument");
	*out = nullptr;
	if (flags & ~(FMX_BUILD_DEDUP | FMX_BUILD_KEEP_SELF_LOOPS | FMX_BUILD_TRANSPOSE))
		return set_error(FMX_ERR_INVAL, "flags 0x%x: the device builder takes DEDUP, KEEP_SELF_LOOPS and TRANSPOSE",
				flags);
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(FMX_ERR_CUDA, "no CUDA device is available");
	if (device < 0 || device >= ndev) return set_error(FMX_ERR_INVAL, "device %d out of range (%d devices)", device, ndev);
	int cur = 0;
	cudaGetDevice(&cur);
	CUDA_TRY(cudaSetDevice(device));
	std::unique_ptr<fmx_matrix> m(new (std::nothrow) fmx_matrix);
	int rc = m ? FMX_OK : set_error(FMX_ERR_OOM, "out of host memory");
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	try {
		uint64_t nr = nrows, nc = ncols;
		{
			dev_csr csr;
			if (!rc) rc = edges_to_dev_csr(src, dst, vals, val_type, nedges, nrows, ncols, flags, st, csr);
			if (!rc) rc = make_part_device(csr, device, st, m->a);
			nr = csr.nrows;
			nc = csr.ncols;
		}
		if (!rc && (flags & FMX_BUILD_TRANSPOSE)) {
			dev_csr t;
			rc = edges_to_dev_csr(dst, src, vals, val_type, nedges, nc, nr, flags, st, t);
			if (!rc) rc = make_part_device(t, device, st, m->at);
		}
		if (!rc && cudaStreamSynchronize(st) != cudaSuccess) rc = set_error(FMX_ERR_CUDA, "device builder failed");
	} catch (const std::bad_alloc &) {
		rc = set_error(FMX_ERR_OOM, "host allocation failed in the device builder");
	}
	cudaSetDevice(cur);
	if (rc) return rc;
	m->symmetric = !(flags & FMX_BUILD_TRANSPOSE);
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
	// one linear copy each way when the rows are contiguous (a pitched copy
	// of 64-byte rows moves far below the link rate)
	auto copy = [&](void *dst, size_t dpitch, const void *src, size_t spitch, size_t width, size_t rows,
			cudaMemcpyKind kind) {
		if (dpitch == width && spitch == width) return cudaMemcpyAsync(dst, src, width * rows, kind, st);
		return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, kind, st);
	};
	if (!rc && copy(p.stage_x, k * xs, X_host, ldx * xs, k * xs, p.ncols, cudaMemcpyHostToDevice) != cudaSuccess)
		rc = set_error(FMX_ERR_CUDA, "copy of X to the device failed");
	if (!rc) rc = spmm_part(p, x_type, p.stage_x, k, y_type, p.stage_y, k, k, nullptr, nullptr, st);
	if (!rc && copy(Y_host, ldy * ys, p.stage_y, k * ys, k * ys, p.nrows, cudaMemcpyDeviceToHost) != cudaSuccess)
		rc = set_error(FMX_ERR_CUDA, "copy of Y to the host failed");
	if (st) {
		cudaError_t e = cudaStreamSynchronize(st);
		if (!rc && e != cudaSuccess) rc = set_error(FMX_ERR_CUDA, "SpMM failed: %s", cudaGetErrorString(e));
		cudaStreamDestroy(st);
	}
	cudaSetDevice(cur);
	return rc;
}

int fmx_spmm_host_async(const fmx_matrix *m, int x_type, const void *X_host, int64_t ldx, int y_type,
		void *Y_host, int64_t ldy, int64_t k, void *stream)
{
	if (!m || !m->a || !X_host || !Y_host) return set_error(FMX_ERR_INVAL, "null argument");
	size_t xs = dtype_size(x_type), ys = dtype_size(y_type);
	if (!xs || !ys) return set_error(FMX_ERR_TYPE, "unknown dtype");
	if (k <= 0 || ldx < k || ldy < k) return set_error(FMX_ERR_DIM, "bad k / leading dimensions");
	gpu_part &p = *m->a;
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	std::lock_guard<std::mutex> guard(p.stage_mu);
	int cur = 0;
	cudaGetDevice(&cur);
	CUDA_TRY(cudaSetDevice(p.device));
	const size_t xb = size_t(p.ncols) * k * xs, yb = size_t(p.nrows) * k * ys;
	int rc = FMX_OK;
	auto ev = [&](cudaEvent_t &e) {
		if (!rc && !e && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
			rc = set_error(FMX_ERR_CUDA, "event creation failed");
	};
	auto stm = [&](cudaStream_t &s) {
		if (!rc && !s && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
			rc = set_error(FMX_ERR_CUDA, "stream creation failed");
	};
	stm(p.h2d_st);
	stm(p.d2h_st);
	ev(p.ev_scratch);
	gpu_part::async_slot &sl = p.aslot[p.anext & 1];
	ev(sl.x_ready);
	ev(sl.spmm_done);
	ev(sl.y_out);
	if (!rc && (sl.xb < xb || sl.yb < yb)) {
		// growing: the slot's earlier call must be through first
		cudaEventSynchronize(sl.spmm_done);
		cudaEventSynchronize(sl.y_out);
		auto grow = [&](void *&buf, size_t &have, size_t need) -> int {
			if (have >= need) return FMX_OK;
			if (buf) cudaFree(buf);
			buf = nullptr; have = 0;
			if (cudaMalloc(&buf, need) != cudaSuccess)
				return set_error(FMX_ERR_OOM, "cudaMalloc of %zu staging bytes failed", need);
			have = need;
			return FMX_OK;
		};
		rc = grow(sl.x, sl.xb, xb);
		if (!rc) rc = grow(sl.y, sl.yb, yb);
	}
	auto copy = [&](void *dst, size_t dpitch, const void *src, size_t spitch, size_t width, size_t rows,
			cudaMemcpyKind kind, cudaStream_t s) {
		if (dpitch == width && spitch == width) return cudaMemcpyAsync(dst, src, width * rows, kind, s);
		return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, kind, s);
	};
	auto wait = [&](cudaStream_t s, cudaEvent_t e) {
		if (!rc && cudaStreamWaitEvent(s, e, 0) != cudaSuccess) rc = set_error(FMX_ERR_CUDA, "stream wait failed");
	};
	auto record = [&](cudaEvent_t e, cudaStream_t s) {
		if (!rc && cudaEventRecord(e, s) != cudaSuccess) rc = set_error(FMX_ERR_CUDA, "event record failed");
	};
	// X in, on the copy-in stream, once the slot's last SpMM has read its X
	wait(p.h2d_st, sl.spmm_done);
	if (!rc && copy(sl.x, k * xs, X_host, ldx * xs, k * xs, p.ncols, cudaMemcpyHostToDevice, p.h2d_st) != cudaSuccess)
		rc = set_error(FMX_ERR_CUDA, "copy of X to the device failed");
	record(sl.x_ready, p.h2d_st);
	// the SpMM on the caller's stream: X arrived, the slot's last Y copied
	// out, and the SpMM issued before this one done (shared scratch)
	wait(st, sl.x_ready);
	wait(st, sl.y_out);
	wait(st, p.ev_scratch);
	if (!rc) rc = spmm_part(p, x_type, sl.x, k, y_type, sl.y, k, k, nullptr, nullptr, st);
	record(sl.spmm_done, st);
	record(p.ev_scratch, st);
	// Y out, on the copy-out stream; the call ends on the caller's stream
	// when Y has arrived
	wait(p.d2h_st, sl.spmm_done);
	if (!rc && copy(Y_host, ldy * ys, sl.y, k * ys, k * ys, p.nrows, cudaMemcpyDeviceToHost, p.d2h_st) != cudaSuccess)
		rc = set_error(FMX_ERR_CUDA, "copy of Y to the host failed");
	record(sl.y_out, p.d2h_st);
	wait(st, sl.y_out);
	p.anext++;
	cudaSetDevice(cur);
	return rc;
}

int fmx_matrix_hot(const fmx_matrix *m, uint64_t *n_hot_cols, uint64_t *hot_entries, uint64_t *scratch_bytes)
{
	if (!m || !m->a) return set_error(FMX_ERR_INVAL, "null matrix");
	const gpu_part &p = *m->a;
	if (n_hot_cols) *n_hot_cols = p.n_hot;
	if (hot_entries) *hot_entries = p.hot_entries;
	if (scratch_bytes) *scratch_bytes = uint64_t(p.n_hot + 1) * kPanelBytes + uint64_t(p.n_partials) * kPartialStride * 8;
	return FMX_OK;
}

int fmx_matrix_layout_digest(const fmx_matrix *m, int transpose, uint64_t *digest)
{
	if (!m || !m->a || !digest) return set_error(FMX_ERR_INVAL, "null argument");
	const gpu_part *pp = transpose && !m->symmetric ? m->at.get() : m->a.get();
	if (!pp) return set_error(FMX_ERR_INVAL, "the matrix has no transpose part");
	const gpu_part &p = *pp;
	if (p.streamed) return set_error(FMX_ERR_UNSUPPORTED, "a streamed matrix keeps its entry stream in host memory");
	device_guard on_device(p.device);
	if (!on_device.ok()) return set_error(FMX_ERR_CUDA, "cannot make device %d current", p.device);
	uint64_t h = 0xcbf29ce484222325ull;          // FNV-1a, 64 bits
	auto mix_host = [&](const void *q, size_t bytes) {
		const unsigned char *c = static_cast<const unsigned char *>(q);
		for (size_t i = 0; i < bytes; i++) { h ^= c[i]; h *= 0x100000001b3ull; }
	};
	std::vector<unsigned char> buf;
	auto mix = [&](const void *dev, size_t bytes) -> int {
		mix_host(&bytes, sizeof(bytes));
		buf.resize(bytes);
		if (bytes) CUDA_TRY(cudaMemcpy(buf.data(), dev, bytes, cudaMemcpyDeviceToHost));
		mix_host(buf.data(), bytes);
		return FMX_OK;
	};
	std::vector<range_t> rg(p.n_ranges);
	if (p.n_ranges) CUDA_TRY(cudaMemcpy(rg.data(), p.ranges, rg.size() * sizeof(range_t), cudaMemcpyDeviceToHost));
	uint64_t total = 0;
	for (const range_t &r : rg) total = std::max<uint64_t>(total, uint64_t(r.e0) + r.len);
	const size_t padded = size_t(total) + kStep;
	const uint64_t counts[] = {p.nrows, p.ncols, p.nnz, p.n_hot, p.n_exact, p.n_ranges, p.n_heavy, p.n_long_heavy,
			p.n_block_heavy, p.n_partials, p.hot_entries};
	mix_host(counts, sizeof(counts));
	for (int rc : {mix(p.ranges, rg.size() * sizeof(range_t)), mix(p.col, padded * sizeof(uint32_t)),
			mix(p.val, p.esize ? padded * p.esize : 0), mix(p.heavy, size_t(p.n_heavy) * sizeof(heavy_row)),
			mix(p.hot_col, size_t(p.n_hot) * sizeof(int32_t))})
		if (rc) return rc;
	*digest = h;
	return FMX_OK;
}

int fmx_matrix_schedule(const fmx_matrix *m, uint64_t *n_light_rows, uint64_t *n_split_tasks,
		uint64_t *n_heavy_rows, uint64_t *kernels_per_spmm)
{
	if (!m || !m->a) return set_error(FMX_ERR_INVAL, "null matrix");
	const gpu_part &p = *m->a;
	if (n_light_rows) *n_light_rows = p.n_exact;
	if (n_split_tasks) *n_split_tasks = p.n_ranges;
	if (n_heavy_rows) *n_heavy_rows = p.n_heavy;
	if (kernels_per_spmm)
		*kernels_per_spmm = 2 + (p.n_block_heavy ? 1 : 0) + (p.n_heavy > p.n_block_heavy ? 1 : 0);
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

// ---------------------------------------------------------------------------
// SpMM that allocates nothing
//
// For callers that cannot allocate device memory while they run: code inside
// a memory pool or arena that owns all of the device's memory, code running
// where the allocator is off limits (a custom allocator's own callbacks, a
// signal-driven or real-time path), or hosts that forbid device allocation
// after start-up.  fmx_spmm itself allocates nothing per call either, but its
// scratch is allocated with the matrix; this entry point instead uses a fixed
// scratch array compiled into the library, so its scratch exists on every
// GPU that loads libfmx from load until process exit.
// ---------------------------------------------------------------------------
namespace fmx {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;     // 32 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[64];

// The device address of the scratch array on `device` (the current device).
// Host code cannot use g_noalloc_scratch directly: there it is only a host
// stand-in for the symbol, not a device address.
static int noalloc_scratch(int device, void **ptr)
{
	if (device < 0 || device >= 64) return set_error(FMX_ERR_UNSUPPORTED, "device %d out of range for the fixed scratch", device);
	std::lock_guard<std::mutex> g(g_noalloc_mu);
	if (!g_noalloc_ptr[device]) {
		void *p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess || !p)
			return set_error(FMX_ERR_CUDA, "cudaGetSymbolAddress of the fixed scratch failed: %s", cudaGetErrorString(e));
		g_noalloc_ptr[device] = p;
	}
	*ptr = g_noalloc_ptr[device];
	return FMX_OK;
}

template <class WT>
static int run_noalloc(const gpu_part &p, const float *X, int64_t ldx, float *Y, int64_t ldy, int64_t k,
		void *xhot, void *partial, cudaStream_t st)
{
	// the kernels fmx_spmm runs for the same call, on the fixed scratch
	if (k == 1) return run_spmv<float, WT, false>(p, X, ldx, Y, ldy, st, pr_epi{}, xhot, partial);
	constexpr int VEC = 4;
	constexpr int kPanel = kPanelBytes / int(sizeof(float));
	const bool vec_ok = (k % VEC == 0) && (ldx % VEC == 0) && (ldy % VEC == 0) && aligned16(X) && aligned16(Y);
	for (int64_t c0 = 0; c0 < k; c0 += kPanel) {
		const int kp = int(std::min<int64_t>(kPanel, k - c0));
		spmm_args a{};
		a.col = p.col; a.val = p.val; a.ranges = p.ranges;
		a.X = X + c0;
		a.xhot = xhot;
		a.hot_ld = kp;
		a.Y = Y + c0;
		a.partial = partial;
		a.ldx = ldx; a.ldy = ldy; a.k = kp;
		a.n_ranges = p.n_ranges;
		int rc = launch_pack<float, float>(p, X + c0, ldx, kp, static_cast<float *>(xhot), kp, nullptr, st);
		if (rc) return rc;
		if (vec_ok) {
			a.G = kp / VEC;
			a.R = 32 / a.G;
			a.nv = 1;
			rc = launch_one<float, float, float, WT, VEC, 1, false, false>(p, a, st);
		} else {
			int g = 1;
			while (g < 32 && g * 4 < kp) g *= 2;
			a.G = g;
			a.R = 32 / g;
			a.nv = (kp + g - 1) / g;
			rc = launch_one<float, float, float, WT, 1, 4, false, false>(p, a, st);
		}
		if (rc) return rc;
		const int frc = launch_fixup<float, float, false>(p, static_cast<const float *>(partial), Y + c0, ldy, kp,
				nullptr, st);
		if (frc) return frc;
	}
	return FMX_OK;
}

} // namespace fmx

extern "C" int fmx_spmm_noalloc(const fmx_matrix *m, const float *X, int64_t ldx, float *Y, int64_t ldy,
		int64_t k, void *stream)
{
	using namespace fmx;
	if (!m || !m->a || !X || !Y) return set_error(FMX_ERR_INVAL, "null argument");
	const gpu_part &p = *m->a;
	if (k <= 0 || ldx < k || ldy < k) return set_error(FMX_ERR_DIM, "bad k (%lld) or leading dimensions", (long long)k);
	if (p.prim != FMX_P_BOOL && p.prim != FMX_P_FLOAT)
		return set_error(FMX_ERR_TYPE, "fmx_spmm_noalloc takes binary or float-weighted matrices");
	if (p.streamed) return set_error(FMX_ERR_UNSUPPORTED, "fmx_spmm_noalloc takes matrices resident in HBM");
	// scratch layout: the hot pack (widest panel), then the long-row partial sums
	const size_t hot_bytes = (size_t(p.n_hot + 1) * kPanelBytes + 255) / 256 * 256;
	const size_t need = hot_bytes + size_t(p.n_partials) * kPartialStride * sizeof(float);
	if (need > kNoAllocScratchBytes)
		return set_error(FMX_ERR_UNSUPPORTED, "this matrix needs %zu bytes of SpMM scratch; the fixed scratch of "
				"fmx_spmm_noalloc holds %zu bytes (use fmx_spmm)", need, kNoAllocScratchBytes);
	int cur = 0;
	cudaGetDevice(&cur);
	if (cur != p.device && cudaSetDevice(p.device) != cudaSuccess)
		return set_error(FMX_ERR_CUDA, "cannot select device %d", p.device);
	void *base = nullptr;
	int rc = noalloc_scratch(p.device, &base);
	if (!rc) {
		void *xhot = base;
		void *partial = static_cast<char *>(base) + hot_bytes;
		cudaStream_t st = static_cast<cudaStream_t>(stream);
		rc = (p.prim == FMX_P_BOOL) ? run_noalloc<void>(p, X, ldx, Y, ldy, k, xhot, partial, st)
		                            : run_noalloc<float>(p, X, ldx, Y, ldy, k, xhot, partial, st);
	}
	if (cur != p.device) cudaSetDevice(cur);
	return rc;
}
