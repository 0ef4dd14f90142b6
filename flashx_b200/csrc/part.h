// The resident form of one orientation of a matrix (gpu_part) and the
// schedule constants shared by the SpMM kernels (spmm.cu) and the two
// schedulers that build it: make_part on the host (spmm.cu) and
// make_part_device on the GPU (schedule_gpu.cu).
#ifndef FMX_PART_H
#define FMX_PART_H

#include "fmx_internal.h"

#include <cuda_runtime.h>

#include <memory>
#include <mutex>
#include <vector>

namespace fmx {

// ---------------------------------------------------------------------------
// Schedule parameters
// ---------------------------------------------------------------------------
constexpr uint32_t kExactMax = FMX_EXACT_ROW_MAX;  // rows summed by one lane group
constexpr uint32_t kChunk = 256;        // most entries per chunk of a longer row
#ifndef FMX_RANGE_ENTRIES
#define FMX_RANGE_ENTRIES 256           // 128 measured within 1 % at R-MAT scale 24, k = 16, but 15 %
                                        // slower for k = 1 (a warp per range) and 5 % at scale 26
#endif
constexpr uint32_t kRange = FMX_RANGE_ENTRIES;  // most target entries per multi-row range
#ifndef FMX_RANGE_MIN
#define FMX_RANGE_MIN 128               // 32 or 64 took SBM eigensolves (n 10k-200k) 5-15 % further,
                                        // but slowed PageRank at R-MAT scale 16 (k = 1) by 9-23 %
#endif
#ifndef FMX_RANGE_FILL_PER_GROUP
#define FMX_RANGE_FILL_PER_GROUP 1
#endif
constexpr uint32_t kRangeMin = FMX_RANGE_MIN;   // fewest: small matrices get shorter runs, so that they
                                                // still fill the grid
// lane groups of a full grid at k = 16 (148 SMs x 32 warps x 16 groups)
// times the runs each should get before runs shrink below kRange
constexpr uint64_t kRangeFill = uint64_t(FMX_RANGE_FILL_PER_GROUP) * 148 * 32 * 16;
constexpr uint32_t kLongChunks = 8;     // heavy rows with more chunks get a warp each in the fixup
constexpr uint32_t kBlockChunks = 64;   // heavy rows with more chunks get a block of 8 warps each
#ifndef FMX_HOT_MAX
#define FMX_HOT_MAX (1u << 20)
#endif
constexpr uint32_t kHotMax = FMX_HOT_MAX;  // most packed hot columns
constexpr int kPanelBytes = 128;        // X row bytes per panel (hot pack row)
constexpr int kPartialStride = 256;     // AccT slots per partial (one panel)
constexpr int kThreads = 256;           // threads per SpMM block
#ifndef FMX_SPMM_MIN_BLOCKS
#define FMX_SPMM_MIN_BLOCKS 5           // resident blocks per SM the register budget targets
#endif
#ifndef FMX_SPMM_MIN_BLOCKS_2B
#define FMX_SPMM_MIN_BLOCKS_2B 4        // the same for 2-byte (BF16) operands: measured at R-MAT
                                        // scale 22, k = 16, 4 blocks of more registers beat 5
                                        // (0.837 against 0.894 ms), while FP32 at scale 24
                                        // prefers 5 (2.56 against 2.73 ms)
#endif
constexpr int kStep = 8;                // entries per index load group (alignment unit)
constexpr uint32_t kEnd = 0x80000000u;  // last entry of a row
constexpr uint32_t kHot = 0x40000000u;  // entry refers to a hot slot
constexpr uint32_t kIdxMask = 0x3FFFFFFFu;
constexpr uint32_t kNoSlot = 0xFFFFFFFFu;

struct range_t {
	uint32_t e0;         // first entry (a multiple of kStep)
	uint32_t len;        // entries, padded to a multiple of kStep
	uint32_t row0;       // first row (row runs)
	uint32_t slot;       // kNoSlot for row runs; else the chunk's partial slot
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
	uint32_t *col = nullptr;
	void *val = nullptr;
	int32_t *hot_col = nullptr;
	uint32_t n_hot = 0;
	void *xhot = nullptr;                // (n_hot + 1) * kPanelBytes
	uint32_t n_exact = 0;                // rows summed in the reference's order
	range_t *ranges = nullptr;
	uint32_t n_ranges = 0;
	heavy_row *heavy = nullptr;
	uint32_t n_heavy = 0;
	uint32_t n_long_heavy = 0;           // the first heavy rows, of more than kLongChunks chunks
	uint32_t n_block_heavy = 0;          // the first of those, of more than kBlockChunks chunks
	uint32_t n_partials = 0;
	void *partial = nullptr;
	uint64_t hot_entries = 0;            // entries that read the hot pack
	uint64_t bytes = 0;
	// streamed part: the entry stream stays in pinned host memory and each
	// SpMM copies it slice by slice into two device slots (copy_st), the
	// kernel of one slice overlapping the copy of the next
	struct slice_t { uint64_t e0, e1; uint32_t r0, nr; };   // entries [e0, e1), ranges [r0, r0 + nr)
	bool streamed = false;
	uint32_t *h_col = nullptr;
	void *h_val = nullptr;
	std::vector<slice_t> slices;
	uint32_t *slot_col[2] = {nullptr, nullptr};
	void *slot_val[2] = {nullptr, nullptr};
	cudaStream_t copy_st = nullptr;
	cudaEvent_t ev_start = nullptr, ev_copied[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
	uint64_t host_bytes = 0;
	// staging buffers of fmx_spmm_host (grow-only, guarded by stage_mu)
	std::mutex stage_mu;
	void *stage_x = nullptr, *stage_y = nullptr;
	size_t stage_xb = 0, stage_yb = 0;
	// fmx_spmm_host_async (guarded by stage_mu): a ring of two staging slots
	// (grow-only), one stream for the copies of X in and one for the copies
	// of Y out, so each direction runs back to back; per slot, events for X
	// arrived, the SpMM done (X consumed, Y ready) and Y copied out; and the
	// event that orders the calls' SpMMs, which share the scratch above
	struct async_slot { void *x = nullptr, *y = nullptr; size_t xb = 0, yb = 0;
		cudaEvent_t x_ready = nullptr, spmm_done = nullptr, y_out = nullptr; };
	async_slot aslot[2];
	unsigned anext = 0;
	cudaStream_t h2d_st = nullptr, d2h_st = nullptr;
	cudaEvent_t ev_scratch = nullptr;
	~gpu_part() {
		int cur = 0;
		cudaGetDevice(&cur);
		cudaSetDevice(device);
		void *ps[] = {col, val, hot_col, xhot, ranges, heavy, partial, stage_x, stage_y, slot_col[0], slot_col[1],
				slot_val[0], slot_val[1]};
		for (void *p : ps)
			if (p) cudaFree(p);
		if (h_col) cudaFreeHost(h_col);
		if (h_val) cudaFreeHost(h_val);
		for (cudaEvent_t e : {ev_start, ev_copied[0], ev_copied[1], ev_free[0], ev_free[1], ev_scratch})
			if (e) cudaEventDestroy(e);
		for (async_slot &a : aslot) {
			if (a.x) cudaFree(a.x);
			if (a.y) cudaFree(a.y);
			for (cudaEvent_t e : {a.x_ready, a.spmm_done, a.y_out})
				if (e) cudaEventDestroy(e);
		}
		for (cudaStream_t s : {h2d_st, d2h_st})
			if (s) cudaStreamDestroy(s);
		if (copy_st) cudaStreamDestroy(copy_st);
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

// The work segments' rule, shared by both schedulers: rows are taken in
// order with `len` = their entry count (1..kExactMax) or 1 (an empty or
// longer row: one zero-row entry); row r opens a new run when the running
// total of the lens before it, L[r], enters a new multiple of the run size
// R = range_entries(L[n]) (L[r] / R differs from L[r-1] / R).  A run
// therefore holds at most kRange - 1 + kExactMax entries.  A row longer than
// kExactMax also gets ceil(d / kChunk) equal chunks, chunk c holding entries
// [d c / cnt, d (c + 1) / cnt).
__host__ __device__ inline uint32_t seg_row_len(uint32_t d) { return (d >= 1 && d <= kExactMax) ? d : 1; }

// Run size for rows whose lens add up to `total`: kRange, or less (down to
// kRangeMin, a multiple of kStep) when that would leave fewer than
// kRangeFill runs, so that small matrices still spread over the grid.
// Measured on 40 held-out SBM graphs (n 10k-200k, about 2M entries, runs of
// 128 instead of 256): plain eigensolves 4.8 -> 3.6 ms median.
__host__ __device__ inline uint32_t range_entries(uint64_t total)
{
	uint64_t r = total / kRangeFill;
	r = r < kRangeMin ? kRangeMin : (r > kRange ? kRange : r);
	return uint32_t(r / kStep * kStep);
}

// Device-resident CSR (rows ascending, columns in entry order); the
// pointers are owned by `own` and released on `st` when it is destroyed.
struct dev_csr {
	uint64_t nrows = 0, ncols = 0, nnz = 0;
	int prim = 0;
	size_t esize = 0;
	const uint32_t *row_ptr = nullptr;   // nrows + 1
	const int32_t *col = nullptr;        // nnz
	const char *val = nullptr;           // nnz * esize bytes (null when binary)
	cudaStream_t st = nullptr;
	std::vector<void *> own;
	dev_csr() = default;
	dev_csr(const dev_csr &) = delete;
	dev_csr &operator=(const dev_csr &) = delete;
	~dev_csr();
};

// Edge list on the current device -> dev_csr: the CSR that decode_to_csr
// gives for the host builder's image of the same edges (sorted, first
// occurrence kept under FMX_BUILD_DEDUP, self-loops dropped unless
// FMX_BUILD_KEEP_SELF_LOOPS; flags as fmx_image_build's).
int edges_to_dev_csr(const uint32_t *src, const uint32_t *dst, const void *vals, int val_type, uint64_t nedges,
		uint64_t nrows, uint64_t ncols, int flags, cudaStream_t st, dev_csr &out);

// make_part on the GPU: the same gpu_part (entry stream, values, ranges,
// heavy rows, hot columns, scratch) as the host scheduler builds from the
// same CSR, without the CSR leaving the device.
int make_part_device(const dev_csr &csr, int device, cudaStream_t st, std::shared_ptr<gpu_part> &out);

} // namespace fmx

#endif
