// Edge list -> sorted, deduplicated CSR on the GPU: the sort and scatter half
// of fm::create_2d_matrix (matrix/fm_utils.cpp:267-433) for a device-resident
// edge list.  The rows come out in ascending column order, each (row, col)
// kept once with the value of its first occurrence in the input (the order
// the host builder keeps, FMX_BUILD_DEDUP), self-loops dropped unless
// FMX_BUILD_KEEP_SELF_LOOPS.  The CSR then goes through the same scheduler as
// an image decoded on the host, so both paths give the same resident layout.
//
//   1. keys (row << cbits | col) of the kept edges, payload = input position
//   2. stable LSD radix sort of the keys (CUB, over the key's bits only)
//   3. first-of-run flags (all ones without dedup), exclusive scan, scatter
//   4. row pointers from the row boundaries of the sorted keys
//   5. values gathered by the sorted input positions
#include "part.h"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

namespace fmx {
namespace gbuild {

constexpr int kBuildThreads = 256;

#define BCUDA_TRY(call)                                                         \
	do {                                                                        \
		cudaError_t err__ = (call);                                             \
		if (err__ != cudaSuccess)                                               \
			return set_error(FMX_ERR_CUDA, "%s failed: %s (%s:%d)", #call,      \
					cudaGetErrorString(err__), __FILE__, __LINE__);             \
	} while (0)

unsigned grid_for(uint64_t n)
{
	int dev = 0, sms = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	return unsigned(std::max<uint64_t>(1, std::min<uint64_t>((n + kBuildThreads - 1) / kBuildThreads, uint64_t(std::max(sms, 1)) * 16)));
}

// largest vertex id over both endpoints (for nrows / ncols = 0: the
// reference sizes both dimensions by it, fm_utils.cpp:730-739,788)
__global__ void max_ids_kernel(const uint32_t *src, const uint32_t *dst, uint64_t n, unsigned int *mx)
{
	uint32_t a = 0;
	for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
		a = max(a, max(src[i], dst[i]));
	for (int o = 16; o > 0; o >>= 1) a = max(a, __shfl_xor_sync(0xffffffffu, a, o));
	if ((threadIdx.x & 31) == 0) atomicMax(mx, a);
}

// key = row << cbits | col for kept edges, all-ones (sorted last) otherwise;
// out-of-range ids are counted as errors
__global__ void keys_kernel(const uint32_t *src, const uint32_t *dst, uint64_t n, int keep_self, int cbits,
		uint64_t nrows, uint64_t ncols, uint64_t *keys, uint32_t *pos, unsigned long long *bad)
{
	for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
		const uint32_t r = src[i], c = dst[i];
		uint64_t k = ~0ull;
		if (r >= nrows || c >= ncols) atomicAdd(bad, 1ull);
		else if (keep_self || r != c) k = (uint64_t(r) << cbits) | c;
		keys[i] = k;
		pos[i] = uint32_t(i);
	}
}

// flag[i] = 1 for a kept key that starts its run (or every kept key)
__global__ void flags_kernel(const uint64_t *keys, uint64_t n, int dedup, uint32_t *flag)
{
	for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
		const uint64_t k = keys[i];
		flag[i] = (k != ~0ull) && (!dedup || i == 0 || keys[i - 1] != k);
	}
}

// scatter the kept entries: col, input position
__global__ void scatter_kernel(const uint64_t *keys, const uint32_t *pos, const uint32_t *flag, const uint32_t *at,
		uint64_t n, uint64_t cmask, int32_t *col, uint32_t *opos, uint32_t *row)
{
	for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
		if (!flag[i]) continue;
		const uint32_t j = at[i];
		col[j] = int32_t(keys[i] & cmask);
		opos[j] = pos[i];
		row[j] = uint32_t(keys[i] >> __popcll(cmask));
	}
}

// row_ptr[r] = first entry of a row >= r (rows are sorted), row_ptr[nrows] =
// nnz: entry i (i = nnz standing for the end) sets the rows after the
// previous entry's row up to its own, so every row pointer is written once
__global__ void rowptr_kernel(const uint32_t *row, uint64_t nnz, uint64_t nrows, uint32_t *row_ptr)
{
	for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i <= nnz; i += uint64_t(gridDim.x) * blockDim.x) {
		const int64_t prev = i == 0 ? -1 : int64_t(row[i - 1]);
		const int64_t cur = i == nnz ? int64_t(nrows) : int64_t(row[i]);
		for (int64_t r = prev + 1; r <= cur; r++) row_ptr[r] = uint32_t(i);
	}
}

__global__ void gather_kernel(const char *vals, size_t esize, const uint32_t *opos, uint64_t nnz, char *out)
{
	for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < nnz; i += uint64_t(gridDim.x) * blockDim.x)
		for (size_t b = 0; b < esize; b++) out[i * esize + b] = vals[size_t(opos[i]) * esize + b];
}

struct dbuf {
	cudaStream_t st;
	std::vector<void *> p;
	~dbuf()
	{
		for (void *q : p) cudaFreeAsync(q, st);
	}
	template <class T>
	int get(T **out, size_t count)
	{
		void *q = nullptr;
		cudaError_t e = work_alloc(&q, std::max<size_t>(count, 1) * sizeof(T), st);
		if (e != cudaSuccess) return set_error(FMX_ERR_OOM, "device builder: %zu bytes: %s", count * sizeof(T),
				cudaGetErrorString(e));
		p.push_back(q);
		*out = static_cast<T *>(q);
		return FMX_OK;
	}
};

} // namespace gbuild

dev_csr::~dev_csr()
{
	for (void *q : own) cudaFreeAsync(q, st);
}

int edges_to_dev_csr(const uint32_t *src, const uint32_t *dst, const void *vals, int val_type, uint64_t nedges,
		uint64_t nrows, uint64_t ncols, int flags, cudaStream_t st, dev_csr &out)
{
	using namespace gbuild;
	if (nedges >= (1ull << 31)) return set_error(FMX_ERR_UNSUPPORTED, "the device builder takes < 2^31 edges");
	const size_t esize = val_type == FMX_P_BOOL ? 0 : prim_size(val_type);
	if (esize == size_t(-1)) return set_error(FMX_ERR_TYPE, "unknown value type %d", val_type);
	dbuf b{st, {}};
	if (nrows == 0 || ncols == 0) {
		unsigned int *mx = nullptr;
		unsigned int h = 0;
		if (int rc = b.get(&mx, 1)) return rc;
		BCUDA_TRY(cudaMemsetAsync(mx, 0, sizeof(unsigned int), st));
		if (nedges) max_ids_kernel<<<grid_for(nedges), kBuildThreads, 0, st>>>(src, dst, nedges, mx);
		BCUDA_TRY(cudaGetLastError());
		BCUDA_TRY(cudaMemcpyAsync(&h, mx, sizeof(h), cudaMemcpyDeviceToHost, st));
		BCUDA_TRY(cudaStreamSynchronize(st));
		if (nrows == 0) nrows = uint64_t(h) + 1;
		if (ncols == 0) ncols = uint64_t(h) + 1;
	}
	if (nrows > (1ull << 31) || ncols > (1ull << 31))
		return set_error(FMX_ERR_UNSUPPORTED, "matrix %llux%llu exceeds int32 indices", (unsigned long long)nrows,
				(unsigned long long)ncols);
	int cbits = 1;
	while ((1ull << cbits) < ncols) cbits++;
	int rbits = 1;
	while ((1ull << rbits) < nrows) rbits++;
	const int n = int(nedges);
	uint64_t *k0, *k1;
	uint32_t *p0, *p1, *flag, *at, *row;
	unsigned long long *bad;
	uint32_t *opos;
	for (int rc : {b.get(&k0, nedges), b.get(&k1, nedges), b.get(&p0, nedges), b.get(&p1, nedges),
			b.get(&flag, nedges + 1), b.get(&at, nedges + 1), b.get(&bad, 1)})
		if (rc) return rc;
	BCUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(unsigned long long), st));
	if (nedges) keys_kernel<<<grid_for(nedges), kBuildThreads, 0, st>>>(src, dst, nedges, (flags & FMX_BUILD_KEEP_SELF_LOOPS) ? 1 : 0,
			cbits, nrows, ncols, k0, p0, bad);
	BCUDA_TRY(cudaGetLastError());
	// stable sort over the key bits in use plus one: kept keys are below
	// 2^(rbits + cbits), dropped ones (all ones) have that bit set and sort last
	const int end_bit = std::min(64, rbits + cbits + 1);
	cub::DoubleBuffer<uint64_t> dk(k0, k1);
	cub::DoubleBuffer<uint32_t> dp(p0, p1);
	size_t tbytes = 0;
	BCUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tbytes, dk, dp, n, 0, end_bit, st));
	void *tmp = nullptr;
	if (int rc = b.get(reinterpret_cast<char **>(&tmp), tbytes)) return rc;
	BCUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tbytes, dk, dp, n, 0, end_bit, st));
	const uint64_t *keys = dk.Current();
	const uint32_t *pos = dp.Current();
	if (nedges) flags_kernel<<<grid_for(nedges), kBuildThreads, 0, st>>>(keys, nedges, (flags & FMX_BUILD_DEDUP) ? 1 : 0, flag);
	BCUDA_TRY(cudaGetLastError());
	BCUDA_TRY(cudaMemsetAsync(flag + nedges, 0, sizeof(uint32_t), st));
	size_t sbytes = 0;
	BCUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, sbytes, flag, at, n + 1, st));
	void *stmp = nullptr;
	if (int rc = b.get(reinterpret_cast<char **>(&stmp), sbytes)) return rc;
	BCUDA_TRY(cub::DeviceScan::ExclusiveSum(stmp, sbytes, flag, at, n + 1, st));
	uint32_t nnz = 0;
	unsigned long long hbad = 0;
	BCUDA_TRY(cudaMemcpyAsync(&nnz, at + nedges, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
	BCUDA_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost, st));
	BCUDA_TRY(cudaStreamSynchronize(st));
	if (hbad) return set_error(FMX_ERR_INVAL, "%llu edges have ids outside %llu x %llu", hbad,
			(unsigned long long)nrows, (unsigned long long)ncols);
	// the CSR arrays outlive this call: they belong to `out`
	out.st = st;
	auto keep = [&](void **q, size_t bytes) -> int {
		cudaError_t e = work_alloc(q, std::max<size_t>(bytes, 16), st);
		if (e != cudaSuccess) return set_error(FMX_ERR_OOM, "device builder: %zu bytes: %s", bytes, cudaGetErrorString(e));
		out.own.push_back(*q);
		return FMX_OK;
	};
	int32_t *col = nullptr;
	uint32_t *row_ptr = nullptr;
	char *gv = nullptr;
	for (int rc : {keep(reinterpret_cast<void **>(&col), size_t(nnz) * sizeof(int32_t)),
			keep(reinterpret_cast<void **>(&row_ptr), (nrows + 1) * sizeof(uint32_t)), b.get(&opos, nnz),
			b.get(&row, nnz)})
		if (rc) return rc;
	if (nedges) scatter_kernel<<<grid_for(nedges), kBuildThreads, 0, st>>>(keys, pos, flag, at, nedges, (1ull << cbits) - 1,
			col, opos, row);
	BCUDA_TRY(cudaGetLastError());
	rowptr_kernel<<<grid_for(uint64_t(nnz) + 1), kBuildThreads, 0, st>>>(row, nnz, nrows, row_ptr);
	BCUDA_TRY(cudaGetLastError());
	if (esize) {
		if (int rc = keep(reinterpret_cast<void **>(&gv), size_t(nnz) * esize)) return rc;
		if (nnz) gather_kernel<<<grid_for(nnz), kBuildThreads, 0, st>>>(static_cast<const char *>(vals), esize, opos, nnz, gv);
		BCUDA_TRY(cudaGetLastError());
	}
	out.nrows = nrows;
	out.ncols = ncols;
	out.nnz = nnz;
	out.prim = val_type;
	out.esize = esize;
	out.row_ptr = row_ptr;
	out.col = col;
	out.val = gv;
	return FMX_OK;
}

} // namespace fmx
