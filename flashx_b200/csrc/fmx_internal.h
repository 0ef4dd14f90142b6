// Internal declarations shared by the host (C++) and device (CUDA) halves of
// libfmx.  Not installed; the public surface is include/fmx.h.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <memory>
#include <atomic>

#include <cuda_runtime_api.h>

#include "../../include/fmx.h"

namespace fmx {

// ---- error reporting ------------------------------------------------------
// Sets the thread-local message returned by fmx_last_error() and returns code.
int set_error(int code, const char *fmt, ...);

// ---- the reference's on-disk 2D format -------------------------------------
// matrix_header::info (matrix/matrix_header.h:102-121), x86-64 layout,
// padded to one 4096-byte page.
constexpr size_t kPage = 4096;
constexpr int64_t kMagic = 0x123456789FFFFFFLL;
constexpr int kVersion = 2;
constexpr int kSparse = 2;    // matrix_type::SPARSE
constexpr int kRow2D = 2;     // matrix_layout_t::L_ROW_2D
constexpr uint32_t kMaxBlock = 32768;  // block_max_num_rows/cols (matrix_header.h:42-43)

struct header_info {
	int64_t magic_number;
	int32_t version_number;
	int32_t type;
	uint64_t entry_size;
	uint64_t nrows;
	uint64_t ncols;
	int32_t layout;
	int32_t data_type;
	uint64_t block_2d_height;
	uint64_t block_2d_width;
};
static_assert(sizeof(header_info) == 64, "matrix_header field layout");

// sparse_block_2d header (matrix/sparse_matrix_format.h:215-224).
struct tile_header {
	uint32_t brow, bcol, nnz;
	uint16_t nrow, ncoo;
};
static_assert(sizeof(tile_header) == 16, "sparse_block_2d is 16 bytes");

inline size_t tile_bytes(const tile_header &t, size_t esize) {
	return sizeof(tile_header) + size_t(t.nrow) * 2 + size_t(t.nnz) * 2 + 2 + esize * t.nnz;
}
inline size_t tile_rheader(const tile_header &t) {
	return size_t(t.nrow - t.ncoo) * 2 + size_t(t.nnz - t.ncoo) * 2 + 2;
}

size_t prim_size(int prim);   // 0 for bool, -1 (SIZE_MAX) for unknown
bool is_pow2(uint64_t v);

// A host image: owns the .mat_idx and .mat bytes.
struct image {
	std::vector<char> idx;
	std::vector<char> mat;
	header_info h{};
	uint64_t nbrows = 0;
	uint64_t nnz = 0;          // filled by validate()
	const int64_t *offs() const { return reinterpret_cast<const int64_t *>(idx.data() + kPage); }
};

// Check the header pair, the index and every tile's bounds; counts nnz.
int validate(image &img, bool deep);

// Host CSR decoded from an image: rows ascending, columns in the order the
// reference visits them (ascending block column, then ascending column).
struct host_csr {
	uint64_t nrows = 0, ncols = 0, nnz = 0;
	int prim = 0;              // entry prim type (FMX_P_*)
	size_t esize = 0;          // entry bytes (0 = binary)
	std::vector<uint32_t> row_ptr;   // nrows + 1 (nnz < 2^32 enforced)
	std::vector<int32_t> col;
	std::vector<char> val;     // nnz * esize bytes
};
int decode_to_csr(const image &img, host_csr &out, int nthreads);

int default_threads();

// Stream-ordered workspace from the current device's library pool (freed
// memory stays reserved for the next call; fmx_release_cached returns it).
cudaError_t work_alloc(void **p, size_t bytes, cudaStream_t st);

// The device a matrix lives on.
int matrix_device(const fmx_matrix *m);
// Makes `device` current for its lifetime and then restores the caller's;
// ok() is false when `device` could not be made current.
struct device_guard {
	int prev = -1;
	bool ok_ = true;
	explicit device_guard(int device)
	{
		int cur = 0;
		if (cudaGetDevice(&cur) != cudaSuccess) {
			ok_ = false;
		} else if (cur != device) {
			if (cudaSetDevice(device) == cudaSuccess) prev = cur;
			else ok_ = false;
		}
	}
	bool ok() const { return ok_; }
	~device_guard()
	{
		if (prev >= 0) cudaSetDevice(prev);
	}
	device_guard(const device_guard &) = delete;
	device_guard &operator=(const device_guard &) = delete;
};

// A matrix from host CSR (and its transpose, or null for a symmetric one).
int matrix_from_csr(const host_csr &a, const host_csr *at, int device, fmx_matrix **out);

// ---- fused PageRank iteration ----------------------------------------------
// The update of fm::alg::PageRank (PageRank.cpp:110-123) applied where the
// SpMV on A^T closes a row: p2 = out * d + teleport; converged += |pr1 - p2|
// < eps; pr = p2; in_next = p2 / deg; pr1 = in_next * deg.  state[0] counts
// this iteration's converged vertices, state[1] is the done flag (set once
// every vertex converged or the iteration cap is reached; the kernels of
// later iterations then return at once), state[2] the iterations run.
struct pr_epi {
	const float *deg;
	const uint32_t *heavy_mask;    // bit per row summed by the fixup (chunked rows)
	float *pr, *pr1, *in_next;
	unsigned long long *state;
	float damping, teleport, eps;
	unsigned long long n, max_iters;
};
// One iteration on the transpose part of `mt`: SpMV of `in` with the update
// fused, then the iteration's convergence test on the device.
int pagerank_iteration(const fmx_matrix *mt, const float *in, const pr_epi &e, cudaStream_t st);
// Set heavy_mask (ceil(nrows / 32) words, zeroed by the caller) from mt's
// chunked rows.
int pagerank_heavy_mask(const fmx_matrix *mt, uint32_t *mask, cudaStream_t st);

} // namespace fmx

struct fmx_image {
	fmx::image im;
};
