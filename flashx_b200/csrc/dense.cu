// Dense kernels of the block eigensolver (the FlashMatrix eigensolver's
// dense products: block_multi_vector::MvTransMv / gemm / MvNorm,
// matrix/eigensolver/block_dense_matrix.cpp:997-1530, FM_MultiVector.h:389-676).
//
// Tall-skinny operands: X is n x K (n in the millions, K <= 64), row-major.
//
//  tc_gemm   Y = X B           (basis update; B is K x N, small)
//  tc_gram   G = X^T W         (projection; W is n x N; MN-major operands for
//                               BF16, K-major (staged transposed) for TF32)
//     on the 5th-generation tensor cores: tcgen05.mma with the operands staged
//     in shared memory by the CTA's threads and the 128 x N FP32 accumulator
//     in tensor memory (TMEM), read back with tcgen05.ld.  Two precisions:
//       BF16   one MMA per K step, FP32 accumulate (early, loose iterations)
//       TF32x3 x = hi + lo split (hi = tf32(x), lo = tf32(x - hi)); the
//              products hi*hi + hi*lo + lo*hi reach FP32 accuracy
//     For 16-column blocks stored back to back the 3xTF32 forms copy X rows
//     into place as the hi parts (tc_gemm_x3s, tc_gram_x3s), since the MMA
//     reads FP32 as TF32 by dropping the low mantissa bits.
//  gram_f64  G = X^T W in FP64 on the CUDA cores (Cholesky-QR, residuals)
//  small FP64 kernels on one CTA: Cholesky factor inverse, Jacobi
//  eigendecomposition (the projected Rayleigh-Ritz problem).
//
// Every mbarrier wait is bounded; a wait that runs out sets *err and the
// kernel finishes without touching the result, so a hang cannot happen.
#include "fmx_internal.h"

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

namespace fmx {
int set_error(int code, const char *fmt, ...);
}

namespace fmx {
namespace dense {

#define DCUDA_TRY(call)                                                         \
	do {                                                                        \
		cudaError_t err__ = (call);                                             \
		if (err__ != cudaSuccess)                                               \
			return set_error(FMX_ERR_CUDA, "%s failed: %s (%s:%d)", #call,      \
					cudaGetErrorString(err__), __FILE__, __LINE__);             \
	} while (0)

constexpr int kTile = 128;          // rows per tensor-core tile (MMA M)
constexpr uint32_t kWaitPolls = 1u << 20;

// ---------------------------------------------------------------------------
// tcgen05 / mbarrier primitives (PTX ISA 8.6, sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t phase)
{
	uint32_t ok;
	asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
			"selp.u32 %0, 1, 0, p;\n\t}" : "=r"(ok) : "r"(smem_u32(bar)), "r"(phase) : "memory");
	return ok != 0;
}
// Bounded wait: false when the phase did not complete in kWaitPolls polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t phase)
{
	for (uint32_t i = 0; i < kWaitPolls; i++)
		if (mbar_try_wait(bar, phase)) return true;
	return false;
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols)
{
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
			:: "r"(smem_u32(dst_smem)), "r"(ncols) : "memory");
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}

// D(tmem) (+)= A(smem) * B(smem), one instruction, issued by one thread.
template <bool TF32>
__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
	const uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
	if constexpr (TF32)
		asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
				"tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
				:: "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate),
				   "r"(m0), "r"(m1), "r"(m2), "r"(m3) : "memory");
	else
		asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
				"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
				:: "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate),
				   "r"(m0), "r"(m1), "r"(m2), "r"(m3) : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
			:: "r"(smem_u32(bar)) : "memory");
}
// 32 lanes x 16 consecutive 32-bit columns: thread t of the warp gets lane t.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
	uint32_t r[16];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
			: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
			  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
			: "r"(taddr) : "memory");
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
	for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor, no swizzle (canonical "interleave"
// layout of 8-row x 16-byte core matrices): start, leading and stride byte
// offsets in 16-byte units, version 1 (sm100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes,
		uint32_t layout = 0)
{
	uint64_t d = 0;
	d |= uint64_t((addr >> 4) & 0x3FFF);
	d |= uint64_t((lbo_bytes >> 4) & 0x3FFF) << 16;
	d |= uint64_t((sbo_bytes >> 4) & 0x3FFF) << 32;
	d |= uint64_t(1) << 46;                  // version
	d |= uint64_t(layout & 7) << 61;         // 0: no swizzle; 1: 128-byte swizzle of 32-byte atoms
	return d;                                // base offset 0
}
// The 128-byte swizzle of 32-byte atoms (layout type 1), the one MN-major
// form TF32 operands take (unswizzled MN-major TF32 products came out zero):
// an operand is blocks of 32 elements along M (N), each holding a tile's K
// rows as 128-byte rows, 4 rows to a 512-byte atom, the 32-byte chunk index
// XORed with the row's index in its atom.  Byte offset of element e (along M
// or N) of K row r:
__host__ __device__ constexpr uint32_t sw32_offset(int e, int r)
{
	return uint32_t(e / 32) * 16384u + uint32_t(r / 4) * 512u + uint32_t(r % 4) * 128u +
			uint32_t(((e % 32) / 8) ^ (r % 4)) * 32u + uint32_t(e % 8) * 4u;
}
constexpr uint32_t kSw32Block = 16384;   // bytes of one 32-element block of a 128-row tile
constexpr uint32_t kSw32Atom = 512;      // bytes of 4 K rows
// Instruction descriptor: FP32 accumulate, A/B format (1 = BF16, 2 = TF32),
// majors (0 = K-major, 1 = MN-major), N, M = 128.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t fmt, uint32_t a_mn, uint32_t b_mn, uint32_t n)
{
	return (1u << 4) | (fmt << 7) | (fmt << 10) | (a_mn << 15) | (b_mn << 16) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ float tf32_round(float x)
{
	uint32_t r;
	asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
	return __uint_as_float(r);
}

// ---------------------------------------------------------------------------
// Y (n x N) = X (n x K) B (K x N).  A = X tile (128 x Kp), K-major: 16-byte
// K units, each unit holding all 128 rows back to back (LBO = 128 rows x 16 B,
// SBO = 8 rows x 16 B).  B^T (N x Kp) in the same layout.  Kp = K padded to
// the MMA K step (16 BF16 / 8 TF32 elements = 32 bytes).
// ---------------------------------------------------------------------------
template <bool TF32>
struct gemm_cfg {
	static constexpr int E = TF32 ? 4 : 8;        // elements per 16-byte unit
	static constexpr int KSTEP = TF32 ? 8 : 16;   // elements per MMA
	static constexpr int PARTS = TF32 ? 2 : 1;    // hi (+ lo)
};

template <bool TF32>
__device__ __forceinline__ void put_units(char *base, int unit_stride, int row, const float *v, int K, int Kp, int part)
{
	// write row `row` of a K-major operand: units of E elements at base + u*unit_stride + row*16
	constexpr int E = gemm_cfg<TF32>::E;
	for (int u = 0; u < Kp / E; u++) {
		uint32_t w[4];
		if constexpr (TF32) {
#pragma unroll
			for (int i = 0; i < 4; i++) {
				const int k = u * 4 + i;
				const float x = k < K ? v[k] : 0.f;
				const float hi = tf32_round(x);
				w[i] = __float_as_uint(part == 0 ? hi : tf32_round(x - hi));
			}
		} else {
#pragma unroll
			for (int i = 0; i < 4; i++) {
				const int k = u * 8 + 2 * i;
				const float a = k < K ? v[k] : 0.f, b = k + 1 < K ? v[k + 1] : 0.f;
				__nv_bfloat162 h = __floats2bfloat162_rn(a, b);
				memcpy(&w[i], &h, 4);
			}
		}
		*reinterpret_cast<uint4 *>(base + size_t(u) * unit_stride + size_t(row) * 16) = make_uint4(w[0], w[1], w[2], w[3]);
	}
}

template <bool TF32>
__global__ void __launch_bounds__(128)
tc_gemm_kernel(const float *__restrict__ X, int64_t ldx, int K, const float *__restrict__ B, int ldb, int N,
		float *__restrict__ Y, int64_t ldy, int64_t n, int *err)
{
	using C = gemm_cfg<TF32>;
	const int Kp = (K + C::KSTEP - 1) / C::KSTEP * C::KSTEP;
	const int Np = (N + 15) / 16 * 16;                 // MMA N (multiple of 16 for M = 128)
	extern __shared__ __align__(1024) char smem[];
	const size_t a_bytes = size_t(Kp / C::E) * kTile * 16;
	const size_t b_bytes = size_t(Kp / C::E) * Np * 16;
	char *sa = smem;                                   // PARTS x a_bytes
	char *sb = smem + C::PARTS * a_bytes;              // PARTS x b_bytes
	__shared__ uint64_t bar;
	__shared__ uint32_t tmem_base;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const uint32_t ncols = Np <= 32 ? 32 : (Np <= 64 ? 64 : 128);

	// B^T once: row j of B^T = column j of B
	for (int j = tid; j < Np; j += blockDim.x) {
		float col[64];
		for (int k = 0; k < Kp; k++) col[k] = (j < N && k < K) ? B[size_t(k) * ldb + j] : 0.f;
		for (int part = 0; part < C::PARTS; part++)
			put_units<TF32>(sb + part * b_bytes, Np * 16, j, col, Kp, Kp, part);
	}
	if (warp == 0) tmem_alloc(&tmem_base, ncols);
	if (tid == 0) { mbar_init(&bar, 1); asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
	fence_async_smem();
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = tmem_base;
	const uint32_t idesc = instr_desc(TF32 ? 2 : 1, 0, 0, uint32_t(Np));
	uint32_t phase = 0;
	bool ok = true;
	const int64_t ntiles = (n + kTile - 1) / kTile;
	// fast path: whole 16-byte units of aligned rows, no padding along K
	const bool vx = Kp == K && (ldx % 4) == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0;
	const bool vy = (N % 4) == 0 && (ldy % 4) == 0 && (reinterpret_cast<uintptr_t>(Y) & 15) == 0;
	for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
		const int64_t row = t * kTile + tid;
		if (vx) {
			const float4 *xr = reinterpret_cast<const float4 *>(X + row * ldx);
			for (int u = 0; u < Kp / C::E; u++) {
				uint32_t w0[4], w1[4];
				if constexpr (TF32) {
					const float4 x = row < n ? xr[u] : make_float4(0.f, 0.f, 0.f, 0.f);
					const float xs[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
					for (int i = 0; i < 4; i++) {
						const float hi = tf32_round(xs[i]);
						w0[i] = __float_as_uint(hi);
						w1[i] = __float_as_uint(tf32_round(xs[i] - hi));
					}
				} else {
					const float4 a = row < n ? xr[2 * u] : make_float4(0.f, 0.f, 0.f, 0.f);
					const float4 c = row < n ? xr[2 * u + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
					const float xs[8] = {a.x, a.y, a.z, a.w, c.x, c.y, c.z, c.w};
#pragma unroll
					for (int i = 0; i < 4; i++) {
						__nv_bfloat162 h = __floats2bfloat162_rn(xs[2 * i], xs[2 * i + 1]);
						memcpy(&w0[i], &h, 4);
					}
				}
				*reinterpret_cast<uint4 *>(sa + size_t(u) * kTile * 16 + size_t(tid) * 16) =
						make_uint4(w0[0], w0[1], w0[2], w0[3]);
				if constexpr (TF32)
					*reinterpret_cast<uint4 *>(sa + a_bytes + size_t(u) * kTile * 16 + size_t(tid) * 16) =
							make_uint4(w1[0], w1[1], w1[2], w1[3]);
			}
		} else {
			float v[64];
			for (int k = 0; k < Kp; k++) v[k] = (row < n && k < K) ? X[row * ldx + k] : 0.f;
			for (int part = 0; part < C::PARTS; part++)
				put_units<TF32>(sa + part * a_bytes, kTile * 16, tid, v, Kp, Kp, part);
		}
		fence_async_smem();
		__syncthreads();
		if (tid == 0) {
			tc_fence_after();
			uint32_t acc = 0;
			// passes: (hi, hi), then for TF32 (hi, lo) and (lo, hi)
			const int npass = TF32 ? 3 : 1;
			for (int pass = 0; pass < npass; pass++) {
				const int pa = (pass == 2) ? 1 : 0, pb = (pass == 1) ? 1 : 0;
				for (int s = 0; s < Kp / C::KSTEP; s++) {
					const uint32_t a_addr = smem_u32(sa + pa * a_bytes) + uint32_t(s) * 2 * kTile * 16;
					const uint32_t b_addr = smem_u32(sb + pb * b_bytes) + uint32_t(s) * 2 * Np * 16;
					umma<TF32>(tmem, smem_desc(a_addr, kTile * 16, 128), smem_desc(b_addr, Np * 16, 128), idesc, acc);
					acc = 1;
				}
			}
			umma_commit(&bar);
		}
		__syncwarp();
		ok = __syncthreads_and(mbar_wait(&bar, phase));
		phase ^= 1;
		tc_fence_after();
		if (ok) {
			// warp w reads TMEM lanes 32w..32w+31 = tile rows 32w..32w+31
			const int64_t r = t * kTile + warp * 32 + lane;
			for (int c0 = 0; c0 < Np; c0 += 16) {
				float o[16];
				tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0), o);
				if (r < n) {
					if (vy && c0 + 16 <= N) {
						float4 *yr = reinterpret_cast<float4 *>(Y + r * ldy + c0);
#pragma unroll
						for (int q = 0; q < 4; q++) yr[q] = make_float4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
					} else {
						for (int i = 0; i < 16 && c0 + i < N; i++) Y[r * ldy + c0 + i] = o[i];
					}
				}
			}
		}
		tc_fence_before();
		__syncthreads();
	}
	if (!ok && tid == 0) atomicExch(err, 1);
	__syncthreads();
	if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------------------
// Pipelined tensor-core kernels: Y = X B (GEMM) and part[cta] = X^T W (Gram).
//
// Rows of X (and W) stream through shared memory in tiles of 128 rows: each
// converter thread copies its own row of a tile with 16-byte cp.async copies
// (through L2, no L1 allocation), kRawStages tiles ahead, into a ring of raw
// stages, and waits only for its own copies (cp.async.wait_group).  (A
// single producer thread issuing one cp.async.bulk copy per tile measured
// about 1,900 cycles per 8 KB tile per SM: the bulk-copy path, not memory,
// bounded the kernel.)
// Warp roles (320 threads, one CTA per SM):
//   warp 0     idle
//   warp 1     MMA issuer (one lane) and TMEM owner
//   warps 2-5  converters (thread r owns row r of a tile): raw rows -> MMA
//              operands in a ring of OS operand stages; 3xTF32 splits
//              x = hi + lo (hi = x with the low 13 mantissa bits cleared,
//              exact in TF32; lo = x - hi); BF16 rounds to nearest
//   warps 6-9  GEMM epilogue: TMEM lane quarter (warp % 4) -> Y rows, from a
//              ring of AS accumulators, so the MMAs of later tiles overlap
// Barriers (every wait bounded; one that runs out sets *err, and before the
// CTA exits every converter waits for its copies and the MMA lane for its
// MMAs):
//   opr[i]     operands written           opf[i]    the MMAs read them
//   accf[i]    accumulator complete       acce[i]   epilogue drained it
// Operand layouts, no swizzle, 16-byte units:
//   GEMM, K-major: tile row r, K unit u at u * 2048 + r * 16 (LBO 2048 B
//     between K units, SBO 128 B between 8-row groups); B^T likewise.
//   Gram, K = the tile's rows, M = 64 (D row m in TMEM lane (m % 16) +
//     32 (m / 16)); A rows at or above M feed D rows that are never read.
//     BF16: MN-major as the rows arrive, unit along M/N at unit * 2048 +
//     row * 16 (SBO 2048, LBO 128); A's 8 units run past the real ones
//     into memory the allocation covers.  3xTF32: K-major, element (m, k)
//     at (k / 4) * LB + m * 16 + (k % 4) * 4 (LBO LB, SBO 128) with LB = 16
//     bytes more than the real rows (128 * ceil(M / 8) for A, 16 Np for B),
//     so the threads' 4-byte stores hit 32 banks; A's 64 rows per K unit
//     overlap the next unit's rows, which only feeds unread D rows.
// ---------------------------------------------------------------------------
// Raw tiles in flight per converter thread and converter groups (when they
// fit), measured at n = 4.2M, 16 columns.  GEMM: 3 and 4 (BF16 144 us; 1 and
// 6: 156 us).  Gram: 1 and 6 (BF16 162 us; 3 and 4: 203 us, 2 and 4: 175 us):
// the Gram's raw rows are twice as wide, and more groups in flight beat a
// deeper ring per group.
#ifndef FMX_PIPE_GEMM_RS
#define FMX_PIPE_GEMM_RS 3
#endif
#ifndef FMX_PIPE_GEMM_NG
#define FMX_PIPE_GEMM_NG 4
#endif
#ifndef FMX_PIPE_GRAM_RS
#define FMX_PIPE_GRAM_RS 1
#endif
#ifndef FMX_PIPE_GRAM_NG
#define FMX_PIPE_GRAM_NG 6
#endif
constexpr int kGemmRS = FMX_PIPE_GEMM_RS, kGemmNG = FMX_PIPE_GEMM_NG;
constexpr int kGramRS = FMX_PIPE_GRAM_RS, kGramNG = FMX_PIPE_GRAM_NG;
constexpr size_t kPipeSmemBudget = size_t(200) << 10;   // the rings' target size
constexpr size_t kPipeSmemMax = size_t(220) << 10;      // at most (227 KB per CTA, less the static part)

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned)
// from global to shared memory, completing on `bar` (no multicast).
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
			:: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
// 16-byte asynchronous copy global -> shared through L2 (no L1 allocation);
// a thread waits for its own copies with cp.async.wait_group.
__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory"); }

constexpr uint32_t instr_desc_m64(uint32_t fmt, uint32_t a_mn, uint32_t b_mn, uint32_t n)
{
	return (1u << 4) | (fmt << 7) | (fmt << 10) | (a_mn << 15) | (b_mn << 16) | ((n >> 3) << 17) | ((64u >> 4) << 24);
}

// Shared-memory plan of the pipelined kernels (host and device agree).
struct pipe_plan {
	bool gram, tf32;
	int K, N, Kp, Np;                 // GEMM: X is n x K; Gram: X n x K (= M), W n x N
	int64_t ldx, ldw;
	size_t raw, op, acc_cols;         // bytes of a raw stage and an operand stage
	size_t bpart;                     // GEMM: bytes of one part of B^T
	size_t tail;                      // bytes the last operand stage's MMA reads past its end
	int lba, lbb;                     // Gram 3xTF32: K-unit strides of A and B
	int mh = 0;                       // Gram 3xTF32: first A row of the lo parts
	size_t a_op, b_op;                // Gram: bytes of A and B operands (one part)
	int ru;                           // 16-byte units per raw row
	int NG, RS, OS, AS;               // converter groups, raw stages per group, operand and accumulator stages
	size_t smem;
	__host__ __device__ pipe_plan(bool gram_, bool tf32_, int K_, int N_, int64_t ldx_, int64_t ldw_, int rs_, int ng_)
		: gram(gram_), tf32(tf32_), K(K_), N(N_), ldx(ldx_), ldw(ldw_)
	{
		const int KSTEP = tf32 ? 8 : 16;
		Kp = (K + KSTEP - 1) / KSTEP * KSTEP;
		Np = (N + 15) / 16 * 16;
		ru = (K + 3) / 4 + (gram ? (N + 3) / 4 : 0);      // 16-byte units of a raw row
		raw = size_t(kTile) * 16 * size_t(ru);
		bpart = 0; tail = 0; lba = lbb = 0; a_op = b_op = 0;
		if (!gram) {
			const size_t part = tf32 ? size_t(Kp / 4) * kTile * 16 : size_t(Kp / 8) * kTile * 16;
			op = (tf32 ? 2 : 1) * part;
			bpart = tf32 ? size_t(Kp / 4) * Np * 16 : size_t(Kp / 8) * Np * 16;
		} else if (tf32) {
			// A rows: X hi at 0.., X lo at mh..; B rows: W hi at 0.., W lo at Np..
			mh = K <= 16 ? 16 : 32;
			lba = 2 * mh * 16 + 16;
			lbb = 2 * Np * 16 + 16;
			a_op = size_t(kTile / 4) * lba;
			b_op = size_t(kTile / 4) * lbb;
			op = a_op + b_op;
			// A's last K unit is read for 64 rows
			tail = size_t(64 * 16) > size_t(lba) ? size_t(64 * 16 - lba) : 0;
		} else {
			a_op = size_t((K + 7) / 8) * kTile * 16;
			b_op = size_t(Np / 8) * kTile * 16;
			op = a_op + b_op;
			tail = size_t(8) * kTile * 16 > a_op ? size_t(8) * kTile * 16 - a_op : 0;
		}
		AS = gram ? 1 : (Np <= 32 ? 8 : (Np <= 64 ? 4 : 2));
		acc_cols = gram ? size_t((tf32 ? 2 : 1) * Np) : size_t(AS) * Np;
		if (acc_cols < 32) acc_cols = 32;
		// raw stages: RS tiles in flight per converter thread, NG groups;
		// operand stages: two per group when they fit, else one
		const size_t fixed = 2 * bpart + tail;
		NG = ng_;
		RS = rs_;
		OS = fixed + size_t(2 * NG) * op + size_t(NG * RS) * raw <= kPipeSmemBudget ? 2 * NG : NG;
		smem = size_t(NG * RS) * raw + size_t(OS) * op + 2 * bpart + tail;
	}
	__host__ __device__ bool fits() const { return smem <= kPipeSmemMax; }
};

// threads of a CTA with NG converter groups: warp 0 (idle), warp 1 (MMA), NG
// groups of 4 converter warps, 4 epilogue warps
constexpr int pipe_threads(int ng) { return 32 * (6 + 4 * ng); }

template <bool TF32, bool GRAM, int kRawStages, int NGROUPS>
__global__ void __launch_bounds__(pipe_threads(NGROUPS), 1)
tc_pipe_kernel(const float *__restrict__ X, int64_t ldx, int K, const float *__restrict__ Wm, int64_t ldw, int N,
		const float *__restrict__ B, int ldb, float *__restrict__ Y, int64_t ldy, float *__restrict__ part, int64_t n,
		int *err)
{
	const pipe_plan P(GRAM, TF32, K, N, ldx, ldw, kRawStages, NGROUPS);
	constexpr int KSTEP = TF32 ? 8 : 16;
	const int Kp = P.Kp, Np = P.Np, RS = P.RS, OS = P.OS, AS = P.AS;
	extern __shared__ __align__(1024) char smem[];
	// layout: raw ring, operand ring (plus the tail the last one reads), B^T
	char *raw0 = smem;
	char *op0 = smem + size_t(NGROUPS * RS) * P.raw;
	char *sb = op0 + size_t(OS) * P.op + P.tail;
	__shared__ uint64_t opr[2 * NGROUPS], opf[2 * NGROUPS], accf[8], acce[8];
	constexpr int kEpi0 = 2 + 4 * NGROUPS;             // first epilogue warp
	__shared__ uint32_t tmem_base;
	__shared__ int bad;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const uint32_t ncols = P.acc_cols <= 32 ? 32 : (P.acc_cols <= 64 ? 64 : (P.acc_cols <= 128 ? 128 : 256));

	for (size_t i = tid; i < P.smem / 16; i += blockDim.x) reinterpret_cast<uint4 *>(smem)[i] = make_uint4(0, 0, 0, 0);
	__syncthreads();
	if constexpr (!GRAM) {
		for (int j = tid; j < Np; j += blockDim.x) {
			float col[64];
			for (int k = 0; k < Kp; k++) col[k] = (j < N && k < K) ? B[size_t(k) * ldb + j] : 0.f;
			for (int pt = 0; pt < (TF32 ? 2 : 1); pt++) put_units<TF32>(sb + pt * P.bpart, Np * 16, j, col, Kp, Kp, pt);
		}
	}
	if (warp == 1) tmem_alloc(&tmem_base, ncols);
	if (tid == 0) {
		for (int i = 0; i < OS; i++) { mbar_init(&opr[i], 4); mbar_init(&opf[i], 1); }
		for (int i = 0; i < AS; i++) { mbar_init(&accf[i], 1); mbar_init(&acce[i], 4); }
		bad = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	fence_async_smem();
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = tmem_base;
	const int64_t ntiles = (n + kTile - 1) / kTile;
	const int64_t my_tiles = int64_t(blockIdx.x) < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
	bool ok = true;
	auto tile_row = [&](int64_t i) { return (int64_t(blockIdx.x) + i * int64_t(gridDim.x)) * kTile; };
	// operand stage o: GEMM: part 1 (hi / BF16), part 2 (lo); Gram: A then B
	auto OPA1 = [&](int o) { return op0 + size_t(o) * P.op; };
	auto OPA2 = [&](int o) { return OPA1(o) + P.op / 2; };    // GEMM 3xTF32: the lo part
	auto OPB1 = [&](int o) { return OPA1(o) + P.a_op; };

	if (warp == 0) {
		// idle
	} else if (warp == 1) {
		// ---- MMA issuer ----
		if (lane == 0) {
			uint32_t idesc;
			// the 3xTF32 Gram stacks hi and lo: D = [X hi; X lo]^T-rows x [W hi, W lo]
			if constexpr (GRAM) idesc = TF32 ? instr_desc_m64(2, 0, 0, uint32_t(2 * Np)) : instr_desc_m64(1, 1, 1, uint32_t(Np));
			else idesc = instr_desc(TF32 ? 2 : 1, 0, 0, uint32_t(Np));
			// descriptors once: the start address is the low field (16-byte
			// units), so an operand at byte offset `off` from the base is the
			// base descriptor plus off / 16 (shared addresses stay < 256 KB)
			uint64_t dA, dB;
			uint32_t a_step, b_step, a_pass2 = 0, b_pass1 = 0;
			if constexpr (!GRAM) {
				dA = smem_desc(smem_u32(op0), kTile * 16, 128);
				dB = smem_desc(smem_u32(sb), Np * 16, 128);
				a_step = 2 * kTile * 16 / 16;
				b_step = 2 * Np * 16 / 16;
				a_pass2 = uint32_t(P.op / 2 / 16);
				b_pass1 = uint32_t(P.bpart / 16);
			} else if constexpr (TF32) {
				dA = smem_desc(smem_u32(op0), P.lba, 128);
				dB = smem_desc(smem_u32(op0) + uint32_t(P.a_op), P.lbb, 128);
				a_step = 2 * P.lba / 16;
				b_step = 2 * P.lbb / 16;
			} else {
				dA = smem_desc(smem_u32(op0), 128, kTile * 16);
				dB = smem_desc(smem_u32(op0) + uint32_t(P.a_op), 128, kTile * 16);
				a_step = b_step = 2 * 128 / 16;
			}
			const int nks = GRAM ? kTile / KSTEP : Kp / KSTEP;
			int64_t issued = 0;
			uint32_t acc = 0;
			for (int64_t i = 0; i < my_tiles && ok; i++) {
				const int o = int(i % OS), b = int(i % AS);
				if (!GRAM && i >= AS && !mbar_wait(&acce[b], uint32_t((i / AS - 1) & 1))) { ok = false; break; }
				if (!mbar_wait(&opr[o], uint32_t((i / OS) & 1))) { ok = false; break; }
				tc_fence_after();
				const uint64_t stage_off = uint64_t(o) * (P.op / 16);
				const uint32_t d = GRAM ? tmem : tmem + uint32_t(b * Np);
				if constexpr (!GRAM) acc = 0;
				for (int pass = 0; pass < ((TF32 && !GRAM) ? 3 : 1); pass++) {
					// GEMM: (hi, hi), (hi, lo), (lo, hi); Gram: all in one
					uint64_t a = dA + stage_off + (pass == 2 ? a_pass2 : 0);
					uint64_t bd = dB + (GRAM ? stage_off : 0) + (pass == 1 ? b_pass1 : 0);
					for (int ks = 0; ks < nks; ks++) {
						umma<TF32>(d, a, bd, idesc, acc);
						acc = 1;
						a += a_step;
						bd += b_step;
					}
				}
				umma_commit(&opf[o]);
				if constexpr (!GRAM) umma_commit(&accf[b]);
				issued = i + 1;
			}
			if constexpr (GRAM) {
				umma_commit(&accf[0]);
			} else {
				// the MMAs issued must be complete before TMEM is released
				if (issued && !mbar_wait(&accf[(issued - 1) % AS], uint32_t(((issued - 1) / AS) & 1))) ok = false;
			}
		}
	} else if (warp < kEpi0) {
		// ---- converters: group g takes tiles g, g + NG, ...; its thread r
		// copies and converts row r of each ----
		const int g = (warp - 2) / 4;
		const int r = tid - 64 - 128 * g;
		const int xu = (K + 3) / 4, wu = GRAM ? (N + 3) / 4 : 0;
		auto row_of = [&](int st) {
			return raw0 + size_t(g * RS + st) * P.raw + size_t(r) * size_t(P.ru) * 16;
		};
		// local tile j of the group is tile g + j NG of the CTA
		auto issue = [&](int64_t j) {
			const int64_t i = g + j * NGROUPS;
			if (i < my_tiles) {
				const int64_t row = tile_row(i) + r;
				if (row < n) {
					char *d = row_of(int(j % RS));
					const float *sx = X + row * ldx;
					for (int u = 0; u < xu; u++) cp_async16(d + 16 * u, sx + 4 * u);
					if (GRAM) {
						const float *sw = Wm + row * ldw;
						for (int u = 0; u < wu; u++) cp_async16(d + 16 * (xu + u), sw + 4 * u);
					}
				}
			}
			cp_async_commit();                        // one group per tile (empty past the end)
		};
		for (int j = 0; j < kRawStages - 1; j++) issue(j);
		for (int64_t j = 0, i = g; i < my_tiles && ok; j++, i += NGROUPS) {
			const int s = int(j % RS), o = int(i % OS);
			issue(j + kRawStages - 1);                    // into the stage read in the last iteration
			cp_async_wait<kRawStages - 1>();              // this thread's copies of tile i have landed
			if (i >= OS && !mbar_wait(&opf[o], uint32_t((i / OS - 1) & 1))) { ok = false; break; }
			const bool live = tile_row(i) + r < n;
			for (int side = 0; side < (GRAM ? 2 : 1); side++) {
				const int L = side ? N : K;
				const float *xr = reinterpret_cast<const float *>(row_of(s) + (side ? size_t(xu) * 16 : 0));
				if (TF32 && GRAM) {
					// K-major transpose (4-byte stores, 32 banks per warp)
					char *o1 = side ? OPB1(o) : OPA1(o);
					const int lb = side ? P.lbb : P.lba;
					char *b1 = o1 + size_t(r / 4) * lb + (r % 4) * 4;
					char *b2 = b1 + size_t(side ? Np : P.mh) * 16;      // the lo rows
					const int units = (L + 3) / 4;
					int u = r % units;                   // rotated start: the reads of a wavefront spread over banks
					for (int u0 = 0; u0 < units; u0++, u = (u + 1 == units) ? 0 : u + 1) {
						float xs[4];
#pragma unroll
						for (int q = 0; q < 4; q++) xs[q] = 0.f;
						if (live) {
							if (4 * u + 3 < L) {
								const float4 x = reinterpret_cast<const float4 *>(xr)[u];
								xs[0] = x.x; xs[1] = x.y; xs[2] = x.z; xs[3] = x.w;
							} else {
								for (int q = 0; 4 * u + q < L; q++) xs[q] = xr[4 * u + q];
							}
						}
#pragma unroll
						for (int q = 0; q < 4; q++) {
							const int m = 4 * u + q;
							if (m < L) {
								const uint32_t hb = __float_as_uint(xs[q]) & 0xFFFFE000u;
								*reinterpret_cast<uint32_t *>(b1 + size_t(m) * 16) = hb;
								*reinterpret_cast<float *>(b2 + size_t(m) * 16) = __fsub_rn(xs[q], __uint_as_float(hb));
							}
						}
					}
				} else if (TF32) {
					// GEMM, K-major units of 4: hi and lo
					char *o1 = OPA1(o), *o2 = OPA2(o);
					const int units = K / 4;
					int u = r % units;                   // rotated start: a wavefront's reads spread over banks
					for (int u0 = 0; u0 < units; u0++, u = (u + 1 == units) ? 0 : u + 1) {
						const float4 x = live ? reinterpret_cast<const float4 *>(xr)[u] : make_float4(0.f, 0.f, 0.f, 0.f);
						const uint32_t xs[4] = {__float_as_uint(x.x), __float_as_uint(x.y), __float_as_uint(x.z),
								__float_as_uint(x.w)};
						uint32_t hi[4], lo[4];
#pragma unroll
						for (int q = 0; q < 4; q++) {
							hi[q] = xs[q] & 0xFFFFE000u;
							lo[q] = __float_as_uint(__fsub_rn(__uint_as_float(xs[q]), __uint_as_float(hi[q])));
						}
						*reinterpret_cast<uint4 *>(o1 + size_t(u) * kTile * 16 + size_t(r) * 16) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
						*reinterpret_cast<uint4 *>(o2 + size_t(u) * kTile * 16 + size_t(r) * 16) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
					}
				} else {
					// BF16 units of 8 (GEMM K-major, Gram MN-major: the same writes)
					char *o1 = GRAM ? (side ? OPB1(o) : OPA1(o)) : OPA1(o);
					const int units = (L + 7) / 8;
					int u = r % units;
					for (int u0 = 0; u0 < units; u0++, u = (u + 1 == units) ? 0 : u + 1) {
						float xs[8];
						if (live && 8 * u + 8 <= L) {
							const float4 a4 = reinterpret_cast<const float4 *>(xr)[2 * u];
							const float4 c4 = reinterpret_cast<const float4 *>(xr)[2 * u + 1];
							xs[0] = a4.x; xs[1] = a4.y; xs[2] = a4.z; xs[3] = a4.w;
							xs[4] = c4.x; xs[5] = c4.y; xs[6] = c4.z; xs[7] = c4.w;
						} else {
#pragma unroll
							for (int q = 0; q < 8; q++) xs[q] = (live && 8 * u + q < L) ? xr[8 * u + q] : 0.f;
						}
						uint32_t w[4];
#pragma unroll
						for (int q = 0; q < 4; q++) {
							__nv_bfloat162 h = __floats2bfloat162_rn(xs[2 * q], xs[2 * q + 1]);
							memcpy(&w[q], &h, 4);
						}
						*reinterpret_cast<uint4 *>(o1 + size_t(u) * kTile * 16 + size_t(r) * 16) = make_uint4(w[0], w[1], w[2], w[3]);
					}
				}
			}
			fence_async_smem();
			__syncwarp();
			if (lane == 0) mbar_arrive(&opr[o]);
		}
		cp_async_wait<0>();                               // no copy in flight when the CTA exits
		if (GRAM && g == 0) {
			// read out D: warp quarter q holds rows 16 q .. 16 q + 15 in lanes 32 q .. 32 q + 15
			const bool done = ok && mbar_wait(&accf[0], 0);
			const bool all = __all_sync(0xffffffffu, done);
			ok = ok && done;
			if (all) {
				tc_fence_after();
				const int q = warp & 3;
				const int dm = 16 * q + lane;                  // the D row of this lane (lane < 16)
				if constexpr (TF32) {
					// two partials per CTA: rows < mh give hi W hi + hi W lo, rows
					// >= mh give lo W hi
					const bool hi_row = dm < P.mh;
					const int m = hi_row ? dm : dm - P.mh;
					float *pp = part + (size_t(2 * blockIdx.x) + (hi_row ? 0 : 1)) * K * N;
					for (int c0 = 0; c0 < Np; c0 += 16) {
						float o[16], o2[16];
						tmem_ld16(tmem + (uint32_t(q * 32) << 16) + uint32_t(c0), o);
						tmem_ld16(tmem + (uint32_t(q * 32) << 16) + uint32_t(Np + c0), o2);
						if (lane < 16 && m < K)
							for (int c = 0; c < 16 && c0 + c < N; c++)
								pp[size_t(m) * N + c0 + c] = my_tiles ? (hi_row ? __fadd_rn(o[c], o2[c]) : o[c]) : 0.f;
					}
				} else {
					for (int c0 = 0; c0 < Np; c0 += 16) {
						float o[16];
						tmem_ld16(tmem + (uint32_t(q * 32) << 16) + uint32_t(c0), o);
						if (lane < 16 && dm < K)
							for (int c = 0; c < 16 && c0 + c < N; c++)
								part[(size_t(blockIdx.x) * K + dm) * N + c0 + c] = my_tiles ? o[c] : 0.f;
					}
				}
			}
		}
	} else if constexpr (!GRAM) {
		// ---- GEMM epilogue: TMEM lanes 32q..32q+31 = tile rows ----
		const int q = warp & 3;
		const bool vy = (N % 4) == 0 && (ldy % 4) == 0 && (reinterpret_cast<uintptr_t>(Y) & 15) == 0;
		for (int64_t i = 0; i < my_tiles && ok; i++) {
			const int b = int(i % AS);
			if (!mbar_wait(&accf[b], uint32_t((i / AS) & 1))) { ok = false; break; }
			tc_fence_after();
			const int64_t row = tile_row(i) + q * 32 + lane;
			for (int c0 = 0; c0 < Np; c0 += 16) {
				float o[16];
				tmem_ld16(tmem + (uint32_t(q * 32) << 16) + uint32_t(b * Np + c0), o);
				if (row < n) {
					if (vy && c0 + 16 <= N) {
						float4 *yr = reinterpret_cast<float4 *>(Y + row * ldy + c0);
#pragma unroll
						for (int v = 0; v < 4; v++) yr[v] = make_float4(o[4 * v], o[4 * v + 1], o[4 * v + 2], o[4 * v + 3]);
					} else {
						for (int c = 0; c < 16 && c0 + c < N; c++) Y[row * ldy + c0 + c] = o[c];
					}
				}
			}
			tc_fence_before();
			__syncwarp();
			if (lane == 0) mbar_arrive(&acce[b]);
		}
	}
	if (!ok) atomicExch(&bad, 1);
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	if (tid == 0 && bad) atomicExch(err, 1);
	if (warp == 1) tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------------------
// G (M x N) = X^T W over row chunks of 128: A = X^T chunk and B = W chunk are
// MN-major (rows of X and W are contiguous along M and N).  Core matrix =
// 8 chunk rows x 16 bytes; LBO = 128 B between 8-row groups, SBO = 16 groups
// x 128 B between 16-byte units along M (or N).  M is padded to 128 with zero
// units.  Each CTA leaves its partial in part[blockIdx.x]; gram_reduce adds
// the partials in CTA order.
// ---------------------------------------------------------------------------
template <bool TF32>
__device__ __forceinline__ void put_mn_row(char *base, int krow, const float *v, int M, int Mp, int part)
{
	constexpr int E = TF32 ? 4 : 8;
	for (int u = 0; u < Mp / E; u++) {
		uint32_t w[4];
		if constexpr (TF32) {
#pragma unroll
			for (int i = 0; i < 4; i++) {
				const int m = u * 4 + i;
				const float x = m < M ? v[m] : 0.f;
				const float hi = tf32_round(x);
				w[i] = __float_as_uint(part == 0 ? hi : tf32_round(x - hi));
			}
		} else {
#pragma unroll
			for (int i = 0; i < 4; i++) {
				const int m = u * 8 + 2 * i;
				__nv_bfloat162 h = __floats2bfloat162_rn(m < M ? v[m] : 0.f, m + 1 < M ? v[m + 1] : 0.f);
				memcpy(&w[i], &h, 4);
			}
		}
		*reinterpret_cast<uint4 *>(base + size_t(u) * 2048 + size_t(krow >> 3) * 128 + size_t(krow & 7) * 16) =
				make_uint4(w[0], w[1], w[2], w[3]);
	}
}

// K-major operand of the Gram for TF32: column m of the chunk (K = the
// chunk's rows) as 16-byte units of 4 rows; unit (k / 4) of row m lives at
// base + (k / 4) * ustride + m * 16 + (k % 4) * 4.  Rows m >= M stay zero.
__device__ __forceinline__ void put_k_col(char *base, int ustride, int krow, const float *v, int M, int part)
{
	for (int m = 0; m < M; m++) {
		const float x = v[m];
		const float hi = tf32_round(x);
		*reinterpret_cast<float *>(base + size_t(krow >> 2) * ustride + size_t(m) * 16 + size_t(krow & 3) * 4) =
				part == 0 ? hi : tf32_round(x - hi);
	}
}

template <bool TF32>
__global__ void __launch_bounds__(128)
tc_gram_kernel(const float *__restrict__ X, int64_t ldx, int M, const float *__restrict__ W, int64_t ldw, int N,
		int64_t n, float *__restrict__ part, int *err)
{
	// BF16: MN-major operands (rows of X and W copied as they are).
	// TF32: K-major operands (X^T and W^T, written transposed).
	constexpr int E = TF32 ? 4 : 8;
	constexpr int KSTEP = TF32 ? 8 : 16;             // chunk rows per MMA
	constexpr int PARTS = TF32 ? 2 : 1;
	const int Np = (N + 15) / 16 * 16;
	extern __shared__ __align__(1024) char smem[];
	const size_t a_bytes = TF32 ? size_t(kTile / 4) * kTile * 16 : size_t(kTile / E) * 2048;  // M padded to 128
	const size_t b_bytes = TF32 ? size_t(kTile / 4) * Np * 16 : size_t(Np / E) * 2048;
	char *sa = smem, *sb = smem + PARTS * a_bytes;
	__shared__ uint64_t bar;
	__shared__ uint32_t tmem_base;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const uint32_t ncols = Np <= 32 ? 32 : (Np <= 64 ? 64 : 128);
	// zero the operands once: the padding (M rows or units beyond M, N) is
	// never rewritten
	for (size_t i = tid; i < (PARTS * (a_bytes + b_bytes)) / 16; i += blockDim.x)
		reinterpret_cast<uint4 *>(sa)[i] = make_uint4(0, 0, 0, 0);
	if (warp == 0) tmem_alloc(&tmem_base, ncols);
	if (tid == 0) { mbar_init(&bar, 1); asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = tmem_base;
	const uint32_t idesc = TF32 ? instr_desc(2, 0, 0, uint32_t(Np)) : instr_desc(1, 1, 1, uint32_t(Np));
	const int Mp = (M + E - 1) / E * E;
	uint32_t phase = 0;
	uint32_t acc = 0;
	bool ok = true;
	const int64_t nchunks = (n + kTile - 1) / kTile;
	for (int64_t c = blockIdx.x; c < nchunks && ok; c += gridDim.x) {
		const int64_t row = c * kTile + tid;
		float v[64];
		for (int m = 0; m < Mp; m++) v[m] = (row < n && m < M) ? X[row * ldx + m] : 0.f;
		if constexpr (TF32) {
			for (int p = 0; p < PARTS; p++) put_k_col(sa + p * a_bytes, kTile * 16, tid, v, M, p);
		} else {
			put_mn_row<false>(sa, tid, v, M, Mp, 0);
		}
		for (int j = 0; j < Np; j++) v[j] = (row < n && j < N) ? W[row * ldw + j] : 0.f;
		if constexpr (TF32) {
			for (int p = 0; p < PARTS; p++) put_k_col(sb + p * b_bytes, Np * 16, tid, v, N, p);
		} else {
			put_mn_row<false>(sb, tid, v, N, Np, 0);
		}
		fence_async_smem();
		__syncthreads();
		if (tid == 0) {
			tc_fence_after();
			const int npass = TF32 ? 3 : 1;
			for (int pass = 0; pass < npass; pass++) {
				const int pa = (pass == 2) ? 1 : 0, pb = (pass == 1) ? 1 : 0;
				for (int s = 0; s < kTile / KSTEP; s++) {
					if constexpr (TF32) {
						// K-major: 8 chunk rows = 2 units; LBO = unit stride, SBO = 8 rows x 16 B
						const uint32_t a_addr = smem_u32(sa + pa * a_bytes) + uint32_t(s) * 2 * kTile * 16;
						const uint32_t b_addr = smem_u32(sb + pb * b_bytes) + uint32_t(s) * 2 * Np * 16;
						umma<true>(tmem, smem_desc(a_addr, kTile * 16, 128), smem_desc(b_addr, Np * 16, 128), idesc, acc);
					} else {
						// MN-major: 16 chunk rows = 2 groups of 128 bytes; LBO = group
						// stride, SBO = 16-byte unit stride along M (N)
						const uint32_t off = uint32_t(s) * 2 * 128;
						umma<false>(tmem, smem_desc(smem_u32(sa) + off, 128, 2048), smem_desc(smem_u32(sb) + off, 128, 2048),
								idesc, acc);
					}
					acc = 1;
				}
			}
			umma_commit(&bar);
		}
		__syncwarp();
		ok = __syncthreads_and(mbar_wait(&bar, phase));
		phase ^= 1;
		tc_fence_after();
		tc_fence_before();
		__syncthreads();                           // operands free for the next chunk
	}
	// rows 0..M-1 of D: warp w holds rows 32w..32w+31.  The condition must be
	// the same for every thread: tcgen05.ld is a warp-collective instruction.
	const bool had_chunks = int64_t(blockIdx.x) < nchunks;
	if (ok && had_chunks) {
		const int r = warp * 32 + lane;
		for (int c0 = 0; c0 < Np; c0 += 16) {
			float o[16];
			tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0), o);
			if (r < M)
				for (int i = 0; i < 16 && c0 + i < N; i++) part[(size_t(blockIdx.x) * M + r) * N + c0 + i] = o[i];
		}
	} else if (ok) {
		for (int i = tid; i < M * N; i += blockDim.x) part[size_t(blockIdx.x) * M * N + i] = 0.f;
	}
	if (!ok && tid == 0) atomicExch(err, 1);
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	if (warp == 0) tmem_dealloc(tmem, ncols);
}

// G[i] = sum over the partials of part[p][i]: one warp per element, lane l
// adding partials l, l + 32, ... and the lanes combined by a fixed xor tree
// (deterministic for a given number of partials)
template <class T>
__global__ void gram_reduce_kernel(const T *part, int nparts, int MN, T *G)
{
	const int lane = threadIdx.x & 31;
	const int warps = int((gridDim.x * blockDim.x) >> 5);
	for (int i = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < MN; i += warps) {
		T s = 0;
		for (int p = lane; p < nparts; p += 32) s += part[size_t(p) * MN + i];
		for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
		if (lane == 0) G[i] = s;
	}
}

// ---------------------------------------------------------------------------
// FP64 Gram on CUDA cores: part[cta] = sum over the CTA's rows of x^T w (FP64)
// Each thread owns a 4 x 4 block of G and every `groups`-th row: per row it
// loads its 4 columns of x and of w straight from global memory (16-byte
// loads when the leading dimensions allow, L1-shared by the threads of the
// same row) and does 16 FP64 FMAs; four rows are in flight per thread.  The
// row groups' blocks are added in a fixed order at the end (deterministic).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float4 ld4_guard(const float *p, int c, int lim, bool vec)
{
	if (vec && c + 3 < lim) return *reinterpret_cast<const float4 *>(p + c);
	float4 v;
	v.x = c < lim ? p[c] : 0.f;
	v.y = c + 1 < lim ? p[c + 1] : 0.f;
	v.z = c + 2 < lim ? p[c + 2] : 0.f;
	v.w = c + 3 < lim ? p[c + 3] : 0.f;
	return v;
}

__global__ void __launch_bounds__(256)
gram_f64_kernel(const float *__restrict__ X, int64_t ldx, int M, const float *__restrict__ W, int64_t ldw, int N,
		int64_t n, double *__restrict__ part)
{
	__shared__ double red[256 * 16];
	const int tid = threadIdx.x;
	const int nbi = (M + 3) / 4, nbj = (N + 3) / 4, nblk = nbi * nbj;    // <= 256
	const int groups = 256 / nblk;
	const int blk = tid % nblk, grp = tid / nblk;
	const int bi = blk / nbj, bj = blk % nbj;
	const bool active = grp < groups;
	const bool vx = (ldx % 4) == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0;
	const bool vw = (ldw % 4) == 0 && (reinterpret_cast<uintptr_t>(W) & 15) == 0;
	double acc[4][4];
#pragma unroll
	for (int a = 0; a < 4; a++)
#pragma unroll
		for (int c = 0; c < 4; c++) acc[a][c] = 0;
	if (active) {
		const int64_t stride = int64_t(gridDim.x) * groups;
		int64_t row = int64_t(blockIdx.x) * groups + grp;
		for (; row + 3 * stride < n; row += 4 * stride) {
			float4 a[4], c[4];
#pragma unroll
			for (int u = 0; u < 4; u++) {
				a[u] = ld4_guard(X + (row + u * stride) * ldx, 4 * bi, M, vx);
				c[u] = ld4_guard(W + (row + u * stride) * ldw, 4 * bj, N, vw);
			}
#pragma unroll
			for (int u = 0; u < 4; u++) {
				const double av[4] = {a[u].x, a[u].y, a[u].z, a[u].w}, cv[4] = {c[u].x, c[u].y, c[u].z, c[u].w};
#pragma unroll
				for (int p = 0; p < 4; p++)
#pragma unroll
					for (int q = 0; q < 4; q++) acc[p][q] = fma(av[p], cv[q], acc[p][q]);
			}
		}
		for (; row < n; row += stride) {
			const float4 a = ld4_guard(X + row * ldx, 4 * bi, M, vx);
			const float4 c = ld4_guard(W + row * ldw, 4 * bj, N, vw);
			const double av[4] = {a.x, a.y, a.z, a.w}, cv[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
			for (int p = 0; p < 4; p++)
#pragma unroll
				for (int q = 0; q < 4; q++) acc[p][q] = fma(av[p], cv[q], acc[p][q]);
		}
#pragma unroll
		for (int p = 0; p < 4; p++)
#pragma unroll
			for (int q = 0; q < 4; q++) red[(size_t(grp) * nblk + blk) * 16 + p * 4 + q] = acc[p][q];
	}
	__syncthreads();
	for (int pr = tid; pr < M * N; pr += 256) {
		const int i = pr / N, j = pr % N;
		const int b2 = (i / 4) * nbj + j / 4, e = (i % 4) * 4 + j % 4;
		double sum = 0;
		for (int g = 0; g < groups; g++) sum += red[(size_t(g) * nblk + b2) * 16 + e];
		part[size_t(blockIdx.x) * M * N + pr] = sum;
	}
}

// FP64 Gram for M, N <= 16 on the FP64 tensor path (mma.sync m8n8k4 .f64):
// a warp takes 4 rows per step (the MMA's K).  Lane (g = lane / 4,
// t = lane % 4) holds x[r][g] and x[r][8 + g] for r = row + t (A fragments
// of the two 8-row halves of x^T) and the same of w (B fragments), so every
// input element is loaded and converted once; 4 MMAs update the 2 x 2 tiles
// of G.  Products of FP32 inputs are exact in FP64.  The 8 warps' tiles are
// added in warp order (deterministic for a fixed grid).
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b)
{
	asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
			: "+d"(d[0]), "+d"(d[1]) : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(256)
gram_dmma_kernel(const float *__restrict__ X, int64_t ldx, int M, const float *__restrict__ W, int64_t ldw, int N,
		int64_t n, double *__restrict__ part)
{
	__shared__ double red[8][16 * 16];
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int g = lane >> 2, t = lane & 3;
	double c[2][2][2];
#pragma unroll
	for (int mi = 0; mi < 2; mi++)
#pragma unroll
		for (int ni = 0; ni < 2; ni++) c[mi][ni][0] = c[mi][ni][1] = 0.0;
	const int64_t steps = (n + 3) / 4;
	const int64_t nw = int64_t(gridDim.x) * 8;
	int64_t q = int64_t(blockIdx.x) * 8 + warp;
	// two steps per trip: all loads first
	for (; q + nw < steps; q += 2 * nw) {
		double a[2][2], bb[2][2];
#pragma unroll
		for (int u = 0; u < 2; u++) {
			const int64_t r = 4 * (q + u * nw) + t;
			const bool rv = r < n;
			a[u][0] = (rv && g < M) ? double(X[r * ldx + g]) : 0.0;
			a[u][1] = (rv && 8 + g < M) ? double(X[r * ldx + 8 + g]) : 0.0;
			bb[u][0] = (rv && g < N) ? double(W[r * ldw + g]) : 0.0;
			bb[u][1] = (rv && 8 + g < N) ? double(W[r * ldw + 8 + g]) : 0.0;
		}
#pragma unroll
		for (int u = 0; u < 2; u++)
#pragma unroll
			for (int mi = 0; mi < 2; mi++)
#pragma unroll
				for (int ni = 0; ni < 2; ni++) dmma_8x8x4(c[mi][ni], a[u][mi], bb[u][ni]);
	}
	for (; q < steps; q += nw) {
		const int64_t r = 4 * q + t;
		const bool rv = r < n;
		const double a0 = (rv && g < M) ? double(X[r * ldx + g]) : 0.0;
		const double a1 = (rv && 8 + g < M) ? double(X[r * ldx + 8 + g]) : 0.0;
		const double b0 = (rv && g < N) ? double(W[r * ldw + g]) : 0.0;
		const double b1 = (rv && 8 + g < N) ? double(W[r * ldw + 8 + g]) : 0.0;
		dmma_8x8x4(c[0][0], a0, b0);
		dmma_8x8x4(c[0][1], a0, b1);
		dmma_8x8x4(c[1][0], a1, b0);
		dmma_8x8x4(c[1][1], a1, b1);
	}
	// D fragment: G[8 mi + g][8 ni + 2 t + i]
#pragma unroll
	for (int mi = 0; mi < 2; mi++)
#pragma unroll
		for (int ni = 0; ni < 2; ni++)
#pragma unroll
			for (int i = 0; i < 2; i++) red[warp][(8 * mi + g) * 16 + 8 * ni + 2 * t + i] = c[mi][ni][i];
	__syncthreads();
	for (int pr = tid; pr < M * N; pr += 256) {
		const int i = pr / N, j = pr % N;
		double sum = red[0][i * 16 + j];
		for (int w = 1; w < 8; w++) sum += red[w][i * 16 + j];
		part[size_t(blockIdx.x) * M * N + pr] = sum;
	}
}

// ---------------------------------------------------------------------------
// Small FP64 problems on one CTA (b <= 64)
// ---------------------------------------------------------------------------

// T = R^{-1} with G = R^T R (upper Cholesky).  info = 0, or the 1-based
// column whose pivot was not positive.  One CTA of 64 threads.
__global__ void chol_inv_kernel(const double *__restrict__ G, int b, double *__restrict__ T, int *info)
{
	extern __shared__ double dyn[];                  // two 64 x 65 FP64 matrices
	double (*R)[65] = reinterpret_cast<double (*)[65]>(dyn);
	double (*Ti)[65] = reinterpret_cast<double (*)[65]>(dyn + 64 * 65);
	const int t = threadIdx.x;
	for (int i = t; i < b * b; i += blockDim.x) R[i / b][i % b] = G[i];
	__syncthreads();
	__shared__ int bad;
	if (t == 0) bad = 0;
	__syncthreads();
	for (int k = 0; k < b; k++) {
		if (t == 0) {
			double d = R[k][k];
			for (int p = 0; p < k; p++) d -= R[p][k] * R[p][k];
			if (!(d > 0) && !bad) bad = k + 1;
			R[k][k] = d > 0 ? sqrt(d) : 1.0;
		}
		__syncthreads();
		for (int j = k + 1 + t; j < b; j += blockDim.x) {
			double s = R[k][j];
			for (int p = 0; p < k; p++) s -= R[p][k] * R[p][j];
			R[k][j] = s / R[k][k];
		}
		__syncthreads();
	}
	// inverse of the upper-triangular R, column by column
	for (int j = t; j < b; j += blockDim.x) {
		for (int i = b - 1; i >= 0; i--) {
			if (i > j) { Ti[i][j] = 0; continue; }
			double s = (i == j) ? 1.0 : 0.0;
			for (int p = i + 1; p <= j; p++) s -= R[i][p] * Ti[p][j];
			Ti[i][j] = s / R[i][i];
		}
	}
	__syncthreads();
	for (int i = t; i < b * b; i += blockDim.x) T[i] = Ti[i / b][i % b];
	if (t == 0) *info = bad;
}

// Symmetric eigendecomposition H = V diag(w) V^T by cyclic Jacobi rotations
// (round-robin pairs: m/2 disjoint rotations per step).  Eigenvalues in
// descending order, V columns matching.  One CTA of kJacobiThreads threads:
// a step's row and column updates are (pair, index) items spread over the
// threads (disjoint pairs touch disjoint rows and columns), the off-diagonal
// norm is a CTA reduction, and the final order is a parallel rank count.
constexpr int kJacobiThreads = 256;
constexpr double kJacobiOff2 = 1e-24;    // stop when sum of squared off-diagonals / diagonal's is below

__global__ void __launch_bounds__(kJacobiThreads) jacobi_eig_kernel(const double *__restrict__ H, int b,
		double *__restrict__ w, double *__restrict__ V, int max_sweeps)
{
	extern __shared__ double dyn[];                  // two 64 x 65 FP64 matrices
	double (*A)[65] = reinterpret_cast<double (*)[65]>(dyn);
	double (*Q)[65] = reinterpret_cast<double (*)[65]>(dyn + 64 * 65);
	__shared__ int pr[32], pc[32];
	__shared__ double cs[32], sn[32];
	__shared__ int cand[64], order[64];
	__shared__ int ncand;
	__shared__ double red_o[kJacobiThreads / 32], red_d[kJacobiThreads / 32];
	__shared__ double off;
	const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
	const int m = (b + 1) & ~1;                       // even size (pad with a zero row/column)
	const int half = m / 2;
	for (int i = t; i < m * m; i += blockDim.x) {
		const int r = i / m, c = i % m;
		A[r][c] = (r < b && c < b) ? 0.5 * (H[r * b + c] + H[c * b + r]) : 0.0;
		Q[r][c] = (r == c) ? 1.0 : 0.0;
	}
	__syncthreads();
	for (int sweep = 0; sweep < max_sweeps; sweep++) {
		double so = 0, sd = 0;
		for (int i = t; i < m * m; i += blockDim.x) {
			const int r = i / m, c = i % m;
			const double v = A[r][c] * A[r][c];
			if (r == c) sd += v; else so += v;
		}
		for (int o = 16; o > 0; o >>= 1) {
			so += __shfl_xor_sync(0xffffffffu, so, o);
			sd += __shfl_xor_sync(0xffffffffu, sd, o);
		}
		if (lane == 0) { red_o[wid] = so; red_d[wid] = sd; }
		__syncthreads();
		if (t == 0) {
			double a = 0, d = 0;
			for (int i = 0; i < int(blockDim.x) / 32; i++) { a += red_o[i]; d += red_d[i]; }
			off = a / (d > 0 ? d : 1.0);
		}
		__syncthreads();
		if (off < kJacobiOff2) break;
		for (int step = 0; step < m - 1; step++) {
			// round-robin tournament pairing of 0..m-1
			if (t < half) {
				int a = t == 0 ? 0 : 1 + (t - 1 + step) % (m - 1);
				int bb = 1 + (m - 2 - t + step) % (m - 1);
				if (a > bb) { int x = a; a = bb; bb = x; }
				pr[t] = a; pc[t] = bb;
				const double app = A[a][a], aqq = A[bb][bb], apq = A[a][bb];
				double c = 1, s2 = 0;
				if (fabs(apq) > 1e-300) {
					const double tau = (aqq - app) / (2 * apq);
					const double tt = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1 + tau * tau));
					c = 1 / sqrt(1 + tt * tt);
					s2 = tt * c;
				}
				cs[t] = c; sn[t] = s2;
			}
			__syncthreads();
			// rows: A <- J^T A
			for (int i = t; i < half * m; i += blockDim.x) {
				const int q = i / m, k = i % m;
				const int p0 = pr[q], p1 = pc[q];
				const double x = A[p0][k], y = A[p1][k];
				A[p0][k] = cs[q] * x - sn[q] * y;
				A[p1][k] = sn[q] * x + cs[q] * y;
			}
			__syncthreads();
			// columns: A <- A J, Q <- Q J
			for (int i = t; i < half * m; i += blockDim.x) {
				const int q = i / m, k = i % m;
				const int p0 = pr[q], p1 = pc[q];
				double x = A[k][p0], y = A[k][p1];
				A[k][p0] = cs[q] * x - sn[q] * y;
				A[k][p1] = sn[q] * x + cs[q] * y;
				x = Q[k][p0]; y = Q[k][p1];
				Q[k][p0] = cs[q] * x - sn[q] * y;
				Q[k][p1] = sn[q] * x + cs[q] * y;
			}
			__syncthreads();
		}
	}
	// descending order of the b real eigenvalues (the padding one, if any, is dropped)
	if (t == 0) {
		int cnt = 0;
		for (int i = 0; i < m; i++) {
			const bool pad = (m != b) && (fabs(Q[b][i]) > 0.5);   // eigenvector of the zero padding
			if (!pad && cnt < b) cand[cnt++] = i;
		}
		ncand = cnt;
	}
	__syncthreads();
	if (t < ncand) {
		const double mine = A[cand[t]][cand[t]];
		int rank = 0;
		for (int j = 0; j < ncand; j++) {
			const double o = A[cand[j]][cand[j]];
			rank += (o > mine) || (o == mine && j < t);
		}
		order[rank] = cand[t];
	}
	__syncthreads();
	for (int i = t; i < b; i += blockDim.x) w[i] = A[order[i]][order[i]];
	for (int i = t; i < b * b; i += blockDim.x) V[i] = Q[i / b][order[i % b]];
}

// ---------------------------------------------------------------------------
// The same problem for b <= 32, with each thread owning a 2 x 2 block and one
// barrier per Jacobi step.  In a step the m indices form m/2 pairs, and
// thread (P, R) owns the entries of A with row in pair P and column in pair R
// (and Q's entries of those rows and columns), so the step's two-sided
// rotation J^T A J changes its block with only its two rotations:
// about 3 shared-memory accesses per entry, against 14 when each thread owns
// one entry and reads the rows and columns it mixes.  A 32-thread rotation
// warp computes step s + 1's rotations meanwhile, from the same A and step
// s's rotations: for each next pair it evaluates a_pp, a_qq and a_pq after
// step s by the block formula itself (so they equal what the owners store).
// Pairings (round robin) and the index tables are built once.  The angle:
// t = sign(d) e / (|d| + sqrt(d^2 + e^2)), d = a_qq - a_pp, e = 2 a_pq,
// evaluated in FP32 (hardware reciprocal square root and reciprocal) on d
// and e scaled by a power of two.  An angle off by 1e-6 leaves a_pq at 1e-6
// of its size instead of zero, which later steps remove.  c and s are then
// normalised in FP64 by two Newton steps for c^2 + s^2 = 1 (multiply by
// 3/2 - n/2, n = c^2 + s^2), so each rotation is orthogonal to FP64 rounding
// and the eigenvalues keep FP64 accuracy.
// ---------------------------------------------------------------------------
constexpr int kJF = 32;
constexpr int kJFHalf = kJF / 2;
constexpr int kJFBlockThreads = kJFHalf * kJFHalf;   // 256 block owners at most
constexpr int kJFThreads = kJFBlockThreads + 32;     // + the rotation warp

// c, s of the rotation that (nearly) zeroes a_pq (c = 1, s = 0 when a_pq = 0
// or negligible against a_qq - a_pp).  New vectors: a' = c a - s q,
// q' = s a + c q.
__device__ __forceinline__ void jf_rotation(double app, double aqq, double apq, double &c, double &s)
{
	c = 1.0;
	s = 0.0;
	if (apq == 0.0) return;
	const double d = aqq - app, e = 2.0 * apq;
	const double M = fmax(fabs(d), fabs(e));
	float df, ef;
	if (M > 1e-30 && M < 1e30) {
		df = float(d);                                 // t depends on e / d only
		ef = float(e);
	} else {
		// 2^-k that brings M into [0.5, 1) (exponent field arithmetic, exact)
		int ex = int((__double_as_longlong(M) >> 52) & 0x7ff) - 1022;
		ex = max(-1021, min(1022, ex));
		const double sc = __longlong_as_double((long long)(1023 - ex) << 52);
		df = float(d * sc);
		ef = float(e * sc);
	}
	if (ef == 0.f) return;
	const float x = __fmaf_rn(df, df, ef * ef);        // > 0
	const float r = x * rsqrtf(x);                     // sqrt(d^2 + e^2)
	float t = __fdividef(ef, fabsf(df) + r);
	if (df < 0.f) t = -t;
	const float c32 = rsqrtf(__fmaf_rn(t, t, 1.f));
	double cc = double(c32), ss = double(t) * double(c32);   // exact products of floats
#pragma unroll
	for (int it = 0; it < 2; it++) {
		const double nrm = __fma_rn(cc, cc, ss * ss);
		const double f = __fma_rn(-0.5, nrm, 1.5);
		cc *= f;
		ss *= f;
	}
	c = cc;
	s = ss;
}

// The 2 x 2 block (rows aP, qP; columns aR, qR) of J^T A J: columns mixed by
// pair R's rotation, then rows by pair P's.
__device__ __forceinline__ void jf_block(double x00, double x01, double x10, double x11, double cP, double sP,
		double cR, double sR, double &z00, double &z01, double &z10, double &z11)
{
	const double y00 = __fma_rn(-sR, x01, __dmul_rn(cR, x00));
	const double y01 = __fma_rn(cR, x01, __dmul_rn(sR, x00));
	const double y10 = __fma_rn(-sR, x11, __dmul_rn(cR, x10));
	const double y11 = __fma_rn(cR, x11, __dmul_rn(sR, x10));
	z00 = __fma_rn(-sP, y10, __dmul_rn(cP, y00));
	z01 = __fma_rn(-sP, y11, __dmul_rn(cP, y01));
	z10 = __fma_rn(cP, y10, __dmul_rn(sP, y00));
	z11 = __fma_rn(cP, y11, __dmul_rn(sP, y01));
}

// Entry (role rp of pair P, role rr of pair R) of J^T A J (role 0: the
// pair's lower index).
__device__ __forceinline__ double jf_pick(const double (*A)[kJF + 1], int aP, int qP, int aR, int qR, double cP,
		double sP, double cR, double sR, int rp, int rr)
{
	double z00, z01, z10, z11;
	jf_block(A[aP][aR], A[aP][qR], A[qP][aR], A[qP][qR], cP, sP, cR, sR, z00, z01, z10, z11);
	return rp ? (rr ? z11 : z10) : (rr ? z01 : z00);
}

__global__ void __launch_bounds__(kJFThreads) jacobi_fast_kernel(const double *__restrict__ H, int b,
		double *__restrict__ w, double *__restrict__ V, int max_sweeps)
{
	constexpr int NW = kJFBlockThreads / 32;
	__shared__ double Ab[2][kJF][kJF + 1], Qb[2][kJF][kJF + 1];
	__shared__ double rc[2][kJFHalf], rs[2][kJFHalf];   // rotation of each pair slot: this step, the next
	__shared__ uint8_t pa[kJF - 1][kJFHalf], pq[kJF - 1][kJFHalf];
	__shared__ uint8_t sr[kJF - 1][kJF];                 // slot | role << 5 of each index, per step
	__shared__ uint32_t nx[kJF - 1][kJFHalf];            // rotation warp: see below
	__shared__ uint32_t nxi[kJF - 1][kJFHalf];
	__shared__ int order[kJF];
	__shared__ double red[2][NW];
	const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
	const int m = (b + 1) & ~1;                         // even size (pad with a zero row/column)
	const int half = m / 2, mm = m * m, steps = m - 1;
	const bool owner = t < half * half;
	const int P = owner ? t / half : 0, R = owner ? t % half : 0;
	const bool rot = wid == NW && lane < half;          // the rotation warp's active lanes
	for (int e = t; e < mm; e += kJFThreads) {
		const int r = e / m, c = e % m;
		Ab[0][r][c] = (r < b && c < b) ? 0.5 * (H[r * b + c] + H[c * b + r]) : 0.0;
		Qb[0][r][c] = (r == c) ? 1.0 : 0.0;
	}
	// round-robin tournament pairing of 0..m-1: step st, slot k
	for (int e = t; e < steps * half; e += kJFThreads) {
		const int st = e / half, k = e % half;
		int a = k == 0 ? 0 : 1 + (k - 1 + st) % (m - 1);
		int q = 1 + (m - 2 - k + st) % (m - 1);
		if (a > q) { const int x = a; a = q; q = x; }
		pa[st][k] = uint8_t(a);
		pq[st][k] = uint8_t(q);
		sr[st][a] = uint8_t(k);
		sr[st][q] = uint8_t(k | 32);
	}
	if (t < kJF) order[t] = t;                          // complete even if the padding is not recognised
	__syncthreads();
	// rotation warp, slot k of step s: the pair (a, q) of step s + 1 (step 0
	// after the last), packed a | q << 8 | (slot | role << 5 of a in step s)
	// << 16 | (the same of q) << 24; and the two step-s pairs holding a and q,
	// packed a1 | q1 << 8 | a2 << 16 | q2 << 24
	for (int e = t; e < steps * half; e += kJFThreads) {
		const int st = e / half, k = e % half;
		const int ns = st + 1 < steps ? st + 1 : 0;
		const int a = pa[ns][k], q = pq[ns][k];
		const int ka = sr[st][a] & 31, kq = sr[st][q] & 31;
		nx[st][k] = uint32_t(a) | (uint32_t(q) << 8) | (uint32_t(sr[st][a]) << 16) | (uint32_t(sr[st][q]) << 24);
		nxi[st][k] = uint32_t(pa[st][ka]) | (uint32_t(pq[st][ka]) << 8) | (uint32_t(pa[st][kq]) << 16) |
				(uint32_t(pq[st][kq]) << 24);
	}
	// step 0's rotations, from A itself
	if (t < half) {
		const int a = pa[0][t], q = pq[0][t];
		double c, sn;
		jf_rotation(Ab[0][a][a], Ab[0][q][q], Ab[0][a][q], c, sn);
		rc[0][t] = c;
		rs[0][t] = sn;
	}
	__syncthreads();
	int cur = 0, par = 0;
	for (int sweep = 0; sweep < max_sweeps; sweep++) {
		double so = 0, sd = 0;
		if (owner) {
			const int aP = pa[0][P], qP = pq[0][P], aR = pa[0][R], qR = pq[0][R];
			const double x00 = Ab[cur][aP][aR], x01 = Ab[cur][aP][qR], x10 = Ab[cur][qP][aR], x11 = Ab[cur][qP][qR];
			if (P == R) { sd = x00 * x00 + x11 * x11; so = x01 * x01 + x10 * x10; }
			else so = x00 * x00 + x01 * x01 + x10 * x10 + x11 * x11;
		}
		for (int o = 16; o > 0; o >>= 1) {
			so += __shfl_xor_sync(0xffffffffu, so, o);
			sd += __shfl_xor_sync(0xffffffffu, sd, o);
		}
		if (wid < NW && lane == 0) { red[0][wid] = so; red[1][wid] = sd; }
		__syncthreads();
		so = 0; sd = 0;
		for (int i = 0; i < NW; i++) { so += red[0][i]; sd += red[1][i]; }
		// the same decision in every thread (see kJacobiOff2)
		if (so / (sd > 0 ? sd : 1.0) < kJacobiOff2) break;
		for (int step = 0; step < steps; step++) {
			const double (*A)[kJF + 1] = Ab[cur];
			const double *cs = rc[par], *ss = rs[par];
			if (owner) {
				const double (*Q)[kJF + 1] = Qb[cur];
				double (*An)[kJF + 1] = Ab[cur ^ 1];
				double (*Qn)[kJF + 1] = Qb[cur ^ 1];
				const int aP = pa[step][P], qP = pq[step][P], aR = pa[step][R], qR = pq[step][R];
				const double cP = cs[P], sP = ss[P], cR = cs[R], sR = ss[R];
				double z00, z01, z10, z11;
				jf_block(A[aP][aR], A[aP][qR], A[qP][aR], A[qP][qR], cP, sP, cR, sR, z00, z01, z10, z11);
				An[aP][aR] = z00; An[aP][qR] = z01; An[qP][aR] = z10; An[qP][qR] = z11;
				// Q J: rows aP and qP, columns of pair R
				const double u0 = Q[aP][aR], v0 = Q[aP][qR], u1 = Q[qP][aR], v1 = Q[qP][qR];
				Qn[aP][aR] = __fma_rn(-sR, v0, __dmul_rn(cR, u0));
				Qn[aP][qR] = __fma_rn(cR, v0, __dmul_rn(sR, u0));
				Qn[qP][aR] = __fma_rn(-sR, v1, __dmul_rn(cR, u1));
				Qn[qP][qR] = __fma_rn(cR, v1, __dmul_rn(sR, u1));
			} else if (rot) {
				const uint32_t pk = nx[step][lane], pi = nxi[step][lane];
				const int ka = (pk >> 16) & 31, ra = (pk >> 21) & 1, kq = (pk >> 24) & 31, rq = (pk >> 29) & 1;
				const int a1 = pi & 0xff, q1 = (pi >> 8) & 0xff, a2 = (pi >> 16) & 0xff, q2 = pi >> 24;
				const double c1 = cs[ka], s1 = ss[ka], c2 = cs[kq], s2 = ss[kq];
				const double app = jf_pick(A, a1, q1, a1, q1, c1, s1, c1, s1, ra, ra);
				const double aqq = jf_pick(A, a2, q2, a2, q2, c2, s2, c2, s2, rq, rq);
				const double apq = jf_pick(A, a1, q1, a2, q2, c1, s1, c2, s2, ra, rq);
				double c, sn;
				jf_rotation(app, aqq, apq, c, sn);
				rc[par ^ 1][lane] = c;
				rs[par ^ 1][lane] = sn;
			}
			cur ^= 1;
			par ^= 1;
			__syncthreads();
		}
	}
	const double (*A)[kJF + 1] = Ab[cur];
	const double (*Q)[kJF + 1] = Qb[cur];
	// descending order of the b real eigenvalues (the padding one, if any, is dropped)
	if (t < 32) {
		const bool real = lane < m && !((m != b) && (fabs(Q[b][lane]) > 0.5));
		const unsigned rmask = __ballot_sync(0xffffffffu, real);
		const double mine = lane < m ? A[lane][lane] : 0.0;
		if (real) {
			int rank = 0;
			for (int j = 0; j < m; j++) {
				if (!((rmask >> j) & 1u)) continue;
				const double o = A[j][j];
				rank += (o > mine) || (o == mine && j < lane);
			}
			if (rank < b) order[rank] = lane;
		}
	}
	__syncthreads();
	for (int i = t; i < b; i += kJFThreads) w[i] = A[order[i]][order[i]];
	for (int i = t; i < b * b; i += kJFThreads) V[i] = Q[i / b][order[i % b]];
}

// ---------------------------------------------------------------------------
// G = X^T W in 3xTF32 for 16-column blocks stored back to back (the
// eigensolver's b = 16), on MN-major operands in the swizzled 32-byte-atom
// layout (sw32_offset).  A 128-row tile is two 16 KB blocks, one per side;
// block row r holds
//   elements 0-15   the row's 16 FP32 values, copied from global memory by
//                   cp.async straight into place: the MMA reads them as
//                   TF32, so they are the hi parts (x with its low 13
//                   mantissa bits dropped)
//   elements 16-31  the lo parts x - hi, written by the converters
// so the converters write 4 bytes per element instead of 8, and no
// transpose.  One MMA per 8 rows: A = the X block (M = 64; rows 32-63 read
// the W block that follows and are never read out), B = the W block (N =
// 32), so D holds [hi*hi | hi*lo] over [lo*hi | lo*lo].  Converter groups of
// 4 warps (a thread per tile row) own rings of kX3Stages stages; group g
// takes the CTA's tiles g, g + kX3Groups, ...; one thread of warp 0 issues
// the MMAs; every wait is bounded.  Two partials per CTA (rows of hi parts:
// hi*hi + hi*lo; rows of lo parts: lo*hi), reduced by gram_reduce_kernel.
// ---------------------------------------------------------------------------
// 6 groups of 1 stage: measured at n = 4.2M, 165 us; 4 x 1 183, 3 x 2 181,
// 2 x 3 224 us (more tiles in flight per CTA, no deeper ring per group)
#ifndef FMX_X3_GROUPS
#define FMX_X3_GROUPS 6
#endif
#ifndef FMX_X3_STAGES
#define FMX_X3_STAGES 1
#endif
constexpr int kX3Groups = FMX_X3_GROUPS, kX3Stages = FMX_X3_STAGES;
constexpr uint32_t kX3Stage = 2 * kSw32Block;   // X block + W block
constexpr int kX3Threads = 32 * (1 + 4 * kX3Groups);
constexpr size_t kX3Smem = size_t(kX3Groups) * kX3Stages * kX3Stage;

__global__ void __launch_bounds__(kX3Threads, 1)
tc_gram_x3s_kernel(const float *__restrict__ X, const float *__restrict__ W, int64_t n, float *__restrict__ part,
		int *err)
{
	extern __shared__ __align__(1024) char smem[];
	__shared__ uint64_t full[kX3Groups * kX3Stages], empty[kX3Groups * kX3Stages], accf;
	__shared__ uint32_t tmem_base;
	__shared__ int bad;
	constexpr uint32_t ncols = 32;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	if (warp == 0) tmem_alloc(&tmem_base, ncols);
	if (tid == 0) {
		for (int i = 0; i < kX3Groups * kX3Stages; i++) { mbar_init(&full[i], 4); mbar_init(&empty[i], 1); }
		mbar_init(&accf, 1);
		bad = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = tmem_base;
	const int64_t ntiles = (n + kTile - 1) / kTile;
	const int64_t my_tiles = int64_t(blockIdx.x) < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
	auto tile_row = [&](int64_t i) { return (int64_t(blockIdx.x) + i * int64_t(gridDim.x)) * kTile; };
	// tile i: group i % G, its (i / G)-th tile, stage (i / G) % S of that group
	auto stage_of = [&](int64_t i) { return int((i % kX3Groups) * kX3Stages + (i / kX3Groups) % kX3Stages); };
	auto use_of = [&](int64_t i) { return uint32_t((i / kX3Groups) / kX3Stages); };
	bool ok = true;
	if (warp == 0) {
		if (lane == 0) {
			const uint32_t idesc = instr_desc_m64(2, 1, 1, 32);
			for (int64_t i = 0; i < my_tiles && ok; i++) {
				const int s = stage_of(i);
				if (!mbar_wait(&full[s], use_of(i) & 1)) { ok = false; break; }
				tc_fence_after();
				const uint32_t base = smem_u32(smem + size_t(s) * kX3Stage);
				uint64_t a = smem_desc(base, kSw32Block, kSw32Atom, 1);
				uint64_t b = smem_desc(base + kSw32Block, kSw32Block, kSw32Atom, 1);
				for (int ks = 0; ks < kTile / 8; ks++) {        // 8 K rows = 2 atoms per MMA
					umma<true>(tmem, a, b, idesc, (i > 0 || ks > 0) ? 1u : 0u);
					a += 2 * kSw32Atom / 16;
					b += 2 * kSw32Atom / 16;
				}
				umma_commit(&empty[s]);
			}
			umma_commit(&accf);
		}
	} else {
		const int g = (warp - 1) / 4;
		const int r = tid - 32 - 128 * g;                  // the thread's tile row
		const int h = (r >> 2) & 1;                        // 16-byte half taken first: a warp's 16-byte
		                                                   // accesses then cover all 32 banks
		// local tile j of the group: the CTA's tile g + j G
		auto issue = [&](int64_t j) {
			const int64_t i = g + j * kX3Groups;
			if (i < my_tiles && ok) {
				const int s = stage_of(i);
				// the stage's previous tile must be through the MMA
				if (i >= int64_t(kX3Groups) * kX3Stages && !mbar_wait(&empty[s], (use_of(i) - 1) & 1)) ok = false;
				const int64_t row = tile_row(i) + r;
				if (ok && row < n) {
					char *xb = smem + size_t(s) * kX3Stage;
					const float *sx = X + row * 16, *sw = W + row * 16;
#pragma unroll
					for (int q = 0; q < 4; q++) {
						const int u = q ^ h;
						cp_async16(xb + sw32_offset(4 * u, r), sx + 4 * u);
						cp_async16(xb + kSw32Block + sw32_offset(4 * u, r), sw + 4 * u);
					}
				}
			}
			cp_async_commit();                            // one group per tile (empty past the end)
		};
		for (int j = 0; j < kX3Stages - 1; j++) issue(j);
		for (int64_t j = 0, i = g; i < my_tiles && ok; j++, i += kX3Groups) {
			issue(j + kX3Stages - 1);
			cp_async_wait<kX3Stages - 1>();                // this thread's copies of tile i have landed
			ok = __all_sync(0xffffffffu, ok);              // warp-uniform exit (the __syncwarp below)
			if (!ok) break;
			const int s = stage_of(i);
			const bool live = tile_row(i) + r < n;
			for (int side = 0; side < 2; side++) {
				char *blk = smem + size_t(s) * kX3Stage + side * kSw32Block;
#pragma unroll
				for (int q = 0; q < 4; q++) {
					const int u = q ^ h;
					uint4 v = live ? *reinterpret_cast<const uint4 *>(blk + sw32_offset(4 * u, r)) : make_uint4(0, 0, 0, 0);
					if (!live) *reinterpret_cast<uint4 *>(blk + sw32_offset(4 * u, r)) = v;   // a row past n adds zeros
					const uint32_t x[4] = {v.x, v.y, v.z, v.w};
					uint32_t lo[4];
#pragma unroll
					for (int e = 0; e < 4; e++)
						lo[e] = __float_as_uint(__fsub_rn(__uint_as_float(x[e]), __uint_as_float(x[e] & 0xFFFFE000u)));
					*reinterpret_cast<uint4 *>(blk + sw32_offset(16 + 4 * u, r)) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
				}
			}
			fence_async_smem();                            // cp.async data and lo parts -> the MMA
			__syncwarp();
			if (lane == 0) mbar_arrive(&full[s]);
		}
		cp_async_wait<0>();                                // no copy in flight when the CTA exits
		if (g == 0) {
			// warp quarter q holds D rows 16 q .. 16 q + 15 in lanes 32 q .. 32 q + 15
			const bool done = ok && mbar_wait(&accf, 0);
			const bool all = __all_sync(0xffffffffu, done);
			ok = ok && done;
			if (all) {
				tc_fence_after();
				const int q = warp & 3;
				const int dm = 16 * q + lane;
				const bool hi_row = dm < 16;
				const int m = hi_row ? dm : dm - 16;
				float o[16], o2[16];
				tmem_ld16(tmem + (uint32_t(q * 32) << 16), o);
				tmem_ld16(tmem + (uint32_t(q * 32) << 16) + 16u, o2);
				if (lane < 16 && m < 16) {
					float *pp = part + (size_t(2 * blockIdx.x) + (hi_row ? 0 : 1)) * 256 + size_t(m) * 16;
					for (int c = 0; c < 16; c++) pp[c] = my_tiles ? (hi_row ? __fadd_rn(o[c], o2[c]) : o[c]) : 0.f;
				}
			}
		}
	}
	if (!ok) atomicExch(&bad, 1);
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	if (tid == 0 && bad) atomicExch(err, 1);
	if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------------------
// Y = X B in 3xTF32 for 16 x 16 B and 16-column X and Y stored back to back
// (the eigensolver's basis updates at b = 16).  A = the X tile, K-major in
// the no-swizzle layout (16-byte unit u of row r at u 2048 + r 16): each
// row's 4 units are copied by cp.async straight into place, where the MMA
// reads them as TF32, their hi parts; the converters write only the lo parts
// x - hi into a second such tile.  B^T hi and lo (B split by rounding) sit
// in shared memory for the whole kernel.  Per tile, three MMA passes of two
// K steps (hi B_hi, hi B_lo, lo B_hi) into one of kGx3Acc TMEM accumulators,
// which 4 epilogue warps drain into Y while the next tiles run.  Converter
// groups of 4 warps own rings of kGx3Stages stages; every wait is bounded.
// ---------------------------------------------------------------------------
// 4 groups of 2 stages: measured at n = 4.2M, 139 us; 3 x 2 140, 3 x 3 144,
// 2 x 4 171, 2 x 6 182 us (more stages in flight per group are slower)
#ifndef FMX_GX3_GROUPS
#define FMX_GX3_GROUPS 4
#endif
#ifndef FMX_GX3_STAGES
#define FMX_GX3_STAGES 2
#endif
constexpr int kGx3Groups = FMX_GX3_GROUPS, kGx3Stages = FMX_GX3_STAGES, kGx3Acc = 8;
constexpr uint32_t kGx3Part = 4u * kTile * 16;   // one 128 x 16 FP32 tile (4 units)
constexpr uint32_t kGx3Stage = 2 * kGx3Part;      // hi (copied) + lo
constexpr uint32_t kGx3BPart = 4u * 16 * 16;      // B^T (16 x 16) in 4 units
constexpr int kGx3Threads = 32 * (1 + 4 * kGx3Groups + 4);
constexpr size_t kGx3Smem = size_t(kGx3Groups) * kGx3Stages * kGx3Stage + 2 * kGx3BPart;

__global__ void __launch_bounds__(kGx3Threads, 1)
tc_gemm_x3s_kernel(const float *__restrict__ X, const float *__restrict__ B, int ldb, float *__restrict__ Y,
		int64_t n, int *err)
{
	extern __shared__ __align__(1024) char smem[];
	__shared__ uint64_t full[kGx3Groups * kGx3Stages], empty[kGx3Groups * kGx3Stages], accf[kGx3Acc], acce[kGx3Acc];
	__shared__ uint32_t tmem_base;
	__shared__ int bad;
	constexpr uint32_t ncols = 16 * kGx3Acc;
	constexpr int kEpi0 = 1 + 4 * kGx3Groups;          // first epilogue warp
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	char *sb = smem + size_t(kGx3Groups) * kGx3Stages * kGx3Stage;   // B^T hi, then lo
	for (int j = tid; j < 16; j += blockDim.x) {
		float col[16];
		for (int k = 0; k < 16; k++) col[k] = B[size_t(k) * ldb + j];
		for (int pt = 0; pt < 2; pt++) put_units<true>(sb + pt * kGx3BPart, 16 * 16, j, col, 16, 16, pt);
	}
	if (warp == 0) tmem_alloc(&tmem_base, ncols);
	if (tid == 0) {
		for (int i = 0; i < kGx3Groups * kGx3Stages; i++) { mbar_init(&full[i], 4); mbar_init(&empty[i], 1); }
		for (int i = 0; i < kGx3Acc; i++) { mbar_init(&accf[i], 1); mbar_init(&acce[i], 4); }
		bad = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	fence_async_smem();                                 // B^T -> the MMA
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = tmem_base;
	const int64_t ntiles = (n + kTile - 1) / kTile;
	const int64_t my_tiles = int64_t(blockIdx.x) < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
	auto tile_row = [&](int64_t i) { return (int64_t(blockIdx.x) + i * int64_t(gridDim.x)) * kTile; };
	auto stage_of = [&](int64_t i) { return int((i % kGx3Groups) * kGx3Stages + (i / kGx3Groups) % kGx3Stages); };
	auto use_of = [&](int64_t i) { return uint32_t((i / kGx3Groups) / kGx3Stages); };
	bool ok = true;
	if (warp == 0) {
		if (lane == 0) {
			const uint32_t idesc = instr_desc(2, 0, 0, 16);
			const uint64_t dB = smem_desc(smem_u32(sb), 16 * 16, 128);
			int64_t issued = 0;
			for (int64_t i = 0; i < my_tiles && ok; i++) {
				const int s = stage_of(i), b = int(i % kGx3Acc);
				if (i >= kGx3Acc && !mbar_wait(&acce[b], uint32_t((i / kGx3Acc - 1) & 1))) { ok = false; break; }
				if (!mbar_wait(&full[s], use_of(i) & 1)) { ok = false; break; }
				tc_fence_after();
				const uint64_t dHi = smem_desc(smem_u32(smem + size_t(s) * kGx3Stage), kTile * 16, 128);
				const uint32_t d = tmem + uint32_t(b * 16);
				uint32_t acc = 0;
				for (int pass = 0; pass < 3; pass++) {
					// (hi, B hi), (hi, B lo), (lo, B hi)
					uint64_t a = dHi + (pass == 2 ? kGx3Part / 16 : 0);
					uint64_t bd = dB + (pass == 1 ? kGx3BPart / 16 : 0);
					for (int ks = 0; ks < 2; ks++) {            // 16 K = two MMAs of 8
						umma<true>(d, a, bd, idesc, acc);
						acc = 1;
						a += 2 * kTile * 16 / 16;
						bd += 2 * 16 * 16 / 16;
					}
				}
				umma_commit(&empty[s]);
				umma_commit(&accf[b]);
				issued = i + 1;
			}
			// the MMAs issued must be complete before TMEM is released
			if (issued && !mbar_wait(&accf[(issued - 1) % kGx3Acc], uint32_t(((issued - 1) / kGx3Acc) & 1))) ok = false;
		}
	} else if (warp < kEpi0) {
		const int g = (warp - 1) / 4;
		const int r = tid - 32 - 128 * g;                  // the thread's tile row
		auto issue = [&](int64_t j) {
			const int64_t i = g + j * kGx3Groups;
			if (i < my_tiles && ok) {
				const int s = stage_of(i);
				if (i >= int64_t(kGx3Groups) * kGx3Stages && !mbar_wait(&empty[s], (use_of(i) - 1) & 1)) ok = false;
				const int64_t row = tile_row(i) + r;
				if (ok && row < n) {
					char *hb = smem + size_t(s) * kGx3Stage;
					const float *sx = X + row * 16;
#pragma unroll
					for (int u = 0; u < 4; u++) cp_async16(hb + size_t(u) * kTile * 16 + size_t(r) * 16, sx + 4 * u);
				}
			}
			cp_async_commit();                            // one group per tile (empty past the end)
		};
		for (int j = 0; j < kGx3Stages - 1; j++) issue(j);
		for (int64_t j = 0, i = g; i < my_tiles && ok; j++, i += kGx3Groups) {
			issue(j + kGx3Stages - 1);
			cp_async_wait<kGx3Stages - 1>();               // this thread's copies of tile i have landed
			ok = __all_sync(0xffffffffu, ok);              // warp-uniform exit (the __syncwarp below)
			if (!ok) break;
			const int s = stage_of(i);
			char *hb = smem + size_t(s) * kGx3Stage;
			const bool live = tile_row(i) + r < n;
#pragma unroll
			for (int u = 0; u < 4; u++) {
				char *ph = hb + size_t(u) * kTile * 16 + size_t(r) * 16;
				uint4 v = live ? *reinterpret_cast<const uint4 *>(ph) : make_uint4(0, 0, 0, 0);
				if (!live) *reinterpret_cast<uint4 *>(ph) = v;   // a row past n adds zeros
				const uint32_t x[4] = {v.x, v.y, v.z, v.w};
				uint32_t lo[4];
#pragma unroll
				for (int e = 0; e < 4; e++)
					lo[e] = __float_as_uint(__fsub_rn(__uint_as_float(x[e]), __uint_as_float(x[e] & 0xFFFFE000u)));
				*reinterpret_cast<uint4 *>(ph + kGx3Part) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
			}
			fence_async_smem();                            // cp.async data and lo parts -> the MMA
			__syncwarp();
			if (lane == 0) mbar_arrive(&full[s]);
		}
		cp_async_wait<0>();                                // no copy in flight when the CTA exits
	} else {
		// epilogue: TMEM lanes 32 q .. 32 q + 31 are tile rows
		const int q = warp & 3;
		for (int64_t i = 0; i < my_tiles && ok; i++) {
			const int b = int(i % kGx3Acc);
			const bool got = mbar_wait(&accf[b], uint32_t((i / kGx3Acc) & 1));
			ok = __all_sync(0xffffffffu, got);
			if (!ok) break;
			tc_fence_after();
			const int64_t row = tile_row(i) + q * 32 + lane;
			float o[16];
			tmem_ld16(tmem + (uint32_t(q * 32) << 16) + uint32_t(b * 16), o);
			if (row < n) {
				float4 *yr = reinterpret_cast<float4 *>(Y + row * 16);
#pragma unroll
				for (int v = 0; v < 4; v++) yr[v] = make_float4(o[4 * v], o[4 * v + 1], o[4 * v + 2], o[4 * v + 3]);
			}
			tc_fence_before();
			__syncwarp();
			if (lane == 0) mbar_arrive(&acce[b]);
		}
	}
	if (!ok) atomicExch(&bad, 1);
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	if (tid == 0 && bad) atomicExch(err, 1);
	if (warp == 0) tmem_dealloc(tmem, ncols);
}

int sms(int device)
{
	int s = 0;
	cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, device);
	return s > 0 ? s : 1;
}

} // namespace dense
} // namespace fmx

using namespace fmx;
using namespace fmx::dense;

extern "C" {

int fmx_dense_gemm(int precision, const float *X, int64_t ldx, int64_t n, int K, const float *B, int ldb, int N,
		float *Y, int64_t ldy, int *err, void *stream)
{
	if (!X || !B || !Y || !err) return set_error(FMX_ERR_INVAL, "null argument");
	if (K < 1 || K > 64 || N < 1 || N > 64) return set_error(FMX_ERR_UNSUPPORTED, "tensor-core GEMM takes K, N in 1..64");
	if (precision != FMX_DENSE_BF16 && precision != FMX_DENSE_TF32X3)
		return set_error(FMX_ERR_INVAL, "unknown precision %d", precision);
	const bool tf32 = precision == FMX_DENSE_TF32X3;
	const int E = tf32 ? 4 : 8, KSTEP = tf32 ? 8 : 16, parts = tf32 ? 2 : 1;
	const int Kp = (K + KSTEP - 1) / KSTEP * KSTEP, Np = (N + 15) / 16 * 16;
	int dev = 0;
	cudaGetDevice(&dev);
	const int64_t tiles = (n + kTile - 1) / kTile;
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	if (tf32 && K == 16 && N == 16 && ldx == 16 && ldy == 16 && (reinterpret_cast<uintptr_t>(X) & 15) == 0 &&
			(reinterpret_cast<uintptr_t>(Y) & 15) == 0 && n > 0) {
		// 16-column blocks back to back: hi parts copied into place
		DCUDA_TRY(cudaFuncSetAttribute(tc_gemm_x3s_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kGx3Smem)));
		const unsigned g = unsigned(std::max<int64_t>(1, std::min<int64_t>(tiles, sms(dev))));
		tc_gemm_x3s_kernel<<<g, kGx3Threads, kGx3Smem, st>>>(X, B, ldb, Y, n, err);
		DCUDA_TRY(cudaGetLastError());
		return FMX_OK;
	}
	// the pipelined kernel when the rows of X can be bulk-copied (16-byte
	// aligned rows of whole 16-byte units)
	if (K % 4 == 0 && ldx % 4 == 0 && ldx <= 64 && (reinterpret_cast<uintptr_t>(X) & 15) == 0 && n > 0) {
		// kGemmNG converter groups when they fit, else two, else one
		const pipe_plan P4(false, tf32, K, N, ldx, 0, kGemmRS, kGemmNG), P2(false, tf32, K, N, ldx, 0, kGemmRS, 2),
				P1(false, tf32, K, N, ldx, 0, kGemmRS, 1);
		if (P4.fits() || P2.fits() || P1.fits()) {
			const pipe_plan &P = P4.fits() ? P4 : (P2.fits() ? P2 : P1);
			auto kern = P4.fits() ? (tf32 ? tc_pipe_kernel<true, false, kGemmRS, kGemmNG> : tc_pipe_kernel<false, false, kGemmRS, kGemmNG>)
			          : P2.fits() ? (tf32 ? tc_pipe_kernel<true, false, kGemmRS, 2> : tc_pipe_kernel<false, false, kGemmRS, 2>)
			                      : (tf32 ? tc_pipe_kernel<true, false, kGemmRS, 1> : tc_pipe_kernel<false, false, kGemmRS, 1>);
			DCUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(P.smem)));
			const unsigned grid = unsigned(std::max<int64_t>(1, std::min<int64_t>(tiles, int64_t(sms(dev)))));
			kern<<<grid, pipe_threads(P.NG), P.smem, st>>>(X, ldx, K, nullptr, 0, N, B, ldb, Y, ldy, nullptr, n, err);
			DCUDA_TRY(cudaGetLastError());
			return FMX_OK;
		}
	}
	const size_t smem = size_t(parts) * (size_t(Kp / E) * kTile * 16 + size_t(Kp / E) * Np * 16);
	// as many CTAs per SM as registers and shared memory allow, but no more
	// than the SM's 512 TMEM columns hold (each CTA allocates tmem_cols)
	const int tmem_cols = Np <= 32 ? 32 : (Np <= 64 ? 64 : 128);
	auto kern = tf32 ? tc_gemm_kernel<true> : tc_gemm_kernel<false>;
	DCUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
	int per_sm = 0;
	DCUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem));
	per_sm = std::max(1, std::min(per_sm, 512 / tmem_cols));
	const unsigned grid = unsigned(std::max<int64_t>(1, std::min<int64_t>(tiles, int64_t(sms(dev)) * per_sm)));
	kern<<<grid, 128, smem, st>>>(X, ldx, K, B, ldb, N, Y, ldy, n, err);
	DCUDA_TRY(cudaGetLastError());
	return FMX_OK;
}

int fmx_dense_gram_parts(int precision, int64_t n)
{
	int dev = 0;
	cudaGetDevice(&dev);
	const int64_t chunks = (n + kTile - 1) / kTile;
	if (precision == FMX_DENSE_F64) return int(std::max<int64_t>(1, std::min<int64_t>((n + 63) / 64, int64_t(sms(dev)) * 4)));
	// tensor cores: one CTA per SM; the pipelined 3xTF32 kernel leaves two
	// partials per CTA (the older kernels launch one CTA per partial)
	const int ctas = int(std::max<int64_t>(1, std::min<int64_t>(chunks, int64_t(sms(dev)))));
	return precision == FMX_DENSE_TF32X3 ? 2 * ctas : ctas;
}

int fmx_dense_gram(int precision, const float *X, int64_t ldx, int M, const float *W, int64_t ldw, int N, int64_t n,
		void *part, void *G, int *err, void *stream)
{
	if (!X || !W || !part || !G) return set_error(FMX_ERR_INVAL, "null argument");
	if (M < 1 || M > 64 || N < 1 || N > 64) return set_error(FMX_ERR_UNSUPPORTED, "Gram takes M, N in 1..64");
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	const int parts = fmx_dense_gram_parts(precision, n);
	if (precision == FMX_DENSE_F64) {
		if (M <= 16 && N <= 16)
			gram_dmma_kernel<<<parts, 256, 0, st>>>(X, ldx, M, W, ldw, N, n, static_cast<double *>(part));
		else
			gram_f64_kernel<<<parts, 256, 0, st>>>(X, ldx, M, W, ldw, N, n, static_cast<double *>(part));
		DCUDA_TRY(cudaGetLastError());
		gram_reduce_kernel<double><<<(M * N + 7) / 8, 256, 0, st>>>(static_cast<const double *>(part), parts, M * N,
				static_cast<double *>(G));
		DCUDA_TRY(cudaGetLastError());
		return FMX_OK;
	}
	if (!err) return set_error(FMX_ERR_INVAL, "null error flag");
	const bool tf32 = precision == FMX_DENSE_TF32X3;
	if (!tf32 && precision != FMX_DENSE_BF16) return set_error(FMX_ERR_INVAL, "unknown precision %d", precision);
	if (tf32 && M == 16 && N == 16 && ldx == 16 && ldw == 16 && (reinterpret_cast<uintptr_t>(X) & 15) == 0 &&
			(reinterpret_cast<uintptr_t>(W) & 15) == 0 && n > 0) {
		// 16-column blocks back to back: hi parts copied into place, one pass
		DCUDA_TRY(cudaFuncSetAttribute(tc_gram_x3s_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kX3Smem)));
		tc_gram_x3s_kernel<<<parts / 2, kX3Threads, kX3Smem, st>>>(X, W, n, static_cast<float *>(part), err);
		DCUDA_TRY(cudaGetLastError());
		gram_reduce_kernel<float><<<(M * N + 7) / 8, 256, 0, st>>>(static_cast<const float *>(part), parts, M * N,
				static_cast<float *>(G));
		DCUDA_TRY(cudaGetLastError());
		return FMX_OK;
	}
	if (ldx % 4 == 0 && ldw % 4 == 0 && ldx <= 64 && ldw <= 64 && (reinterpret_cast<uintptr_t>(X) & 15) == 0 &&
			(reinterpret_cast<uintptr_t>(W) & 15) == 0 && n > 0 && (!tf32 || M <= 32)) {
		const pipe_plan P4(true, tf32, M, N, ldx, ldw, kGramRS, kGramNG), P2(true, tf32, M, N, ldx, ldw, kGramRS, 2),
				P1(true, tf32, M, N, ldx, ldw, kGramRS, 1);
		if (P4.fits() || P2.fits() || P1.fits()) {
			// the pipelined kernel: one CTA per SM, partials reduced in CTA order
			const pipe_plan &P = P4.fits() ? P4 : (P2.fits() ? P2 : P1);
			auto kern = P4.fits() ? (tf32 ? tc_pipe_kernel<true, true, kGramRS, kGramNG> : tc_pipe_kernel<false, true, kGramRS, kGramNG>)
			          : P2.fits() ? (tf32 ? tc_pipe_kernel<true, true, kGramRS, 2> : tc_pipe_kernel<false, true, kGramRS, 2>)
			                      : (tf32 ? tc_pipe_kernel<true, true, kGramRS, 1> : tc_pipe_kernel<false, true, kGramRS, 1>);
			DCUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(P.smem)));
			// the 3xTF32 kernel leaves two partials per CTA
			kern<<<tf32 ? parts / 2 : parts, pipe_threads(P.NG), P.smem, st>>>(X, ldx, M, W, ldw, N, nullptr, 0, nullptr, 0,
					static_cast<float *>(part), n, err);
			DCUDA_TRY(cudaGetLastError());
			gram_reduce_kernel<float><<<(M * N + 7) / 8, 256, 0, st>>>(static_cast<const float *>(part), parts, M * N,
					static_cast<float *>(G));
			DCUDA_TRY(cudaGetLastError());
			return FMX_OK;
		}
	}
	const int Np = (N + 15) / 16 * 16;
	const size_t smem = tf32 ? size_t(2) * (size_t(kTile / 4) * kTile * 16 + size_t(kTile / 4) * Np * 16)
	                         : size_t(kTile / 8) * 2048 + size_t(Np / 8) * 2048;
	if (tf32) {
		DCUDA_TRY(cudaFuncSetAttribute(tc_gram_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
		tc_gram_kernel<true><<<parts, 128, smem, st>>>(X, ldx, M, W, ldw, N, n, static_cast<float *>(part), err);
	} else {
		DCUDA_TRY(cudaFuncSetAttribute(tc_gram_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
		tc_gram_kernel<false><<<parts, 128, smem, st>>>(X, ldx, M, W, ldw, N, n, static_cast<float *>(part), err);
	}
	DCUDA_TRY(cudaGetLastError());
	gram_reduce_kernel<float><<<(M * N + 7) / 8, 256, 0, st>>>(static_cast<const float *>(part), parts, M * N,
			static_cast<float *>(G));
	DCUDA_TRY(cudaGetLastError());
	return FMX_OK;
}

int fmx_dense_chol_inv(const double *G, int b, double *T, int *info, void *stream)
{
	if (!G || !T || !info) return set_error(FMX_ERR_INVAL, "null argument");
	if (b < 1 || b > 64) return set_error(FMX_ERR_UNSUPPORTED, "b in 1..64");
	const int smem = 2 * 64 * 65 * int(sizeof(double));
	DCUDA_TRY(cudaFuncSetAttribute(chol_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
	chol_inv_kernel<<<1, 64, smem, static_cast<cudaStream_t>(stream)>>>(G, b, T, info);
	DCUDA_TRY(cudaGetLastError());
	return FMX_OK;
}

int fmx_dense_sym_eig(const double *H, int b, double *w, double *V, void *stream)
{
	if (!H || !w || !V) return set_error(FMX_ERR_INVAL, "null argument");
	if (b < 1 || b > 64) return set_error(FMX_ERR_UNSUPPORTED, "b in 1..64");
	if (b <= kJF) {
		jacobi_fast_kernel<<<1, kJFThreads, 0, static_cast<cudaStream_t>(stream)>>>(H, b, w, V, 30);
		DCUDA_TRY(cudaGetLastError());
		return FMX_OK;
	}
	const int smem = 2 * 64 * 65 * int(sizeof(double));
	DCUDA_TRY(cudaFuncSetAttribute(jacobi_eig_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
	jacobi_eig_kernel<<<1, kJacobiThreads, smem, static_cast<cudaStream_t>(stream)>>>(H, b, w, V, 30);
	DCUDA_TRY(cudaGetLastError());
	return FMX_OK;
}

} // extern "C"
