// make_part on the GPU: the resident layout of one orientation (entry
// stream, values, ranges, heavy rows, hot columns, scratch) from a CSR that
// is already on the device, so the device builder's CSR never crosses PCIe.
// It is the host scheduler (make_part in spmm.cu) restated as data-parallel
// passes and gives the same bytes:
//
//   1. in-degrees (atomic counts), hot columns = the stable radix sort of
//      the columns of in-degree >= 2 by min(indeg, 2^16) descending, ties in
//      column order; slot_of[c] = 1 + its rank below kHotMax, else -1
//   2. per row: len = seg_row_len(d), chunk count, heavy flag; exclusive
//      scans give the lens before each row (L), the first chunk of each
//      heavy row and its heavy index
//   3. run segments: row r opens one when L[r] / R differs from L[r - 1] / R,
//      R = range_entries(L[n]) (the rule in part.h); chunk segments follow in
//      heavy-row order; padded lengths, scanned into stream offsets
//   4. ranges: the stable radix sort of the segments by padded length,
//      longest first
//   5. the stream: a warp per row writes its entries (hot slots or column
//      ids, the row-end bit) and values; chunks of heavy rows likewise
//   6. heavy rows: the stable sort by chunk count, most first
#include "part.h"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

namespace fmx {
namespace gsched {

constexpr int kT = 256;
constexpr uint32_t kDegCap = 1u << 16;     // in-degrees are ranked up to this cap
constexpr uint32_t kNoHotKey = 0x1FFFFu;   // columns of in-degree < 2 sort after every hot candidate
constexpr int kDegBits = 17;
constexpr uint32_t kLenKeyTop = 1024;      // range sort key = kLenKeyTop - padded length
constexpr int kLenBits = 11;

static_assert(kRange - 1 + kExactMax + kStep <= kLenKeyTop, "padded range lengths fit the sort key");

#define SCUDA_TRY(call)                                                         \
	do {                                                                        \
		cudaError_t err__ = (call);                                             \
		if (err__ != cudaSuccess)                                               \
			return set_error(FMX_ERR_CUDA, "%s failed: %s (%s:%d)", #call,      \
					cudaGetErrorString(err__), __FILE__, __LINE__);             \
	} while (0)

static unsigned grid(uint64_t n)
{
	int dev = 0, sms = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	return unsigned(std::max<uint64_t>(1, std::min<uint64_t>((n + kT - 1) / kT, uint64_t(std::max(sms, 1)) * 16)));
}

#define GRID_STRIDE(i, n) \
	for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < (n); i += uint64_t(gridDim.x) * blockDim.x)

__global__ void indeg_kernel(const int32_t *col, uint64_t nnz, uint32_t *indeg)
{
	GRID_STRIDE(i, nnz) atomicAdd(&indeg[col[i]], 1u);
}

__global__ void hot_keys_kernel(const uint32_t *indeg, uint64_t ncols, uint32_t *key, uint32_t *val,
		unsigned long long *ncand)
{
	unsigned long long c_local = 0;
	GRID_STRIDE(c, ncols) {
		const uint32_t d = indeg[c];
		key[c] = d >= 2 ? kDegCap - min(d, kDegCap) : kNoHotKey;
		val[c] = uint32_t(c);
		c_local += d >= 2;
	}
	for (int o = 16; o > 0; o >>= 1) c_local += __shfl_xor_sync(0xffffffffu, c_local, o);
	if ((threadIdx.x & 31) == 0 && c_local) atomicAdd(ncand, c_local);
}

__global__ void slot_kernel(const uint32_t *hot, uint32_t nhot, int32_t *slot_of)
{
	GRID_STRIDE(s, nhot) slot_of[hot[s]] = int32_t(s + 1);
}

// rows [0, n): len, chunk count, heavy flag; index n holds zeros (the scans
// then end with the totals)
__global__ void row_info_kernel(const uint32_t *row_ptr, uint64_t n, uint64_t *lens, uint32_t *chunks,
		uint32_t *hflag, unsigned long long *n_exact)
{
	unsigned long long ex = 0;
	GRID_STRIDE(r, n + 1) {
		if (r == n) { lens[r] = 0; chunks[r] = 0; hflag[r] = 0; continue; }
		const uint32_t d = row_ptr[r + 1] - row_ptr[r];
		lens[r] = seg_row_len(d);
		const bool heavy = d > kExactMax;
		chunks[r] = heavy ? (d + kChunk - 1) / kChunk : 0;
		hflag[r] = heavy;
		ex += (d >= 1 && d <= kExactMax);
	}
	for (int o = 16; o > 0; o >>= 1) ex += __shfl_xor_sync(0xffffffffu, ex, o);
	if ((threadIdx.x & 31) == 0 && ex) atomicAdd(n_exact, ex);
}

// start[r] = 1 when row r opens a run of `run` entries (index n holds 0)
__global__ void start_kernel(const uint64_t *L, uint64_t n, uint32_t run, uint32_t *start)
{
	GRID_STRIDE(r, n + 1) start[r] = r < n && (r == 0 || L[r] / run != L[r - 1] / run);
}

// run segment s = sidx[r] of a row r that opens one: first row, lens before it
__global__ void run_seg_kernel(const uint32_t *start, const uint32_t *sidx, const uint64_t *L, uint64_t n,
		uint32_t *seg_row0, uint64_t *seg_L0, uint32_t *seg_slot)
{
	GRID_STRIDE(r, n) {
		if (!start[r]) continue;
		const uint32_t s = sidx[r];
		seg_row0[s] = uint32_t(r);
		seg_L0[s] = L[r];
		seg_slot[s] = kNoSlot;
	}
}

// run lengths from consecutive starts (the last run ends at L[n])
__global__ void run_len_kernel(const uint64_t *seg_L0, uint32_t s_run, const uint64_t *L, uint64_t n,
		uint32_t *seg_plen)
{
	GRID_STRIDE(s, s_run) {
		const uint64_t e = s + 1 < s_run ? seg_L0[s + 1] : L[n];
		const uint32_t len = uint32_t(e - seg_L0[s]);
		seg_plen[s] = (len + kStep - 1) / kStep * kStep;
	}
}

// heavy rows: their list entry (row order) and chunk segments
__global__ void heavy_kernel(const uint32_t *row_ptr, const uint32_t *hflag, const uint32_t *hidx,
		const uint32_t *chunks, const uint32_t *cfirst, uint64_t n, uint32_t s_run, heavy_row *hlist,
		uint32_t *hkey, uint32_t *hval, uint32_t *seg_row0, uint32_t *seg_plen, uint32_t *seg_slot,
		unsigned long long *n_long, unsigned long long *n_block)
{
	GRID_STRIDE(r, n) {
		if (!hflag[r]) continue;
		const uint32_t d = row_ptr[r + 1] - row_ptr[r];
		const uint32_t cnt = chunks[r], first = cfirst[r], h = hidx[r];
		hlist[h] = heavy_row{int32_t(r), first, cnt};
		hkey[h] = 0xFFFFFFFFu - cnt;
		hval[h] = h;
		if (cnt > kLongChunks) atomicAdd(n_long, 1ull);
		if (cnt > kBlockChunks) atomicAdd(n_block, 1ull);
		for (uint32_t c = 0; c < cnt; c++) {
			const uint32_t b = uint32_t(uint64_t(d) * c / cnt), e = uint32_t(uint64_t(d) * (c + 1) / cnt);
			const uint32_t s = s_run + first + c;
			seg_row0[s] = uint32_t(r);
			seg_plen[s] = (e - b + kStep - 1) / kStep * kStep;
			seg_slot[s] = first + c;
		}
	}
}

__global__ void len_keys_kernel(const uint32_t *seg_plen, uint32_t nseg, uint32_t *key, uint32_t *val)
{
	GRID_STRIDE(s, nseg) {
		key[s] = kLenKeyTop - seg_plen[s];
		val[s] = uint32_t(s);
	}
}

__global__ void ranges_kernel(const uint32_t *perm, uint32_t nseg, const uint64_t *at, const uint32_t *seg_plen,
		const uint32_t *seg_row0, const uint32_t *seg_slot, range_t *ranges)
{
	GRID_STRIDE(i, nseg) {
		const uint32_t s = perm[i];
		ranges[i] = range_t{uint32_t(at[s]), seg_plen[s], seg_row0[s], seg_slot[s]};
	}
}

__global__ void fill_stream_kernel(uint32_t *col, uint64_t total, uint64_t padded)
{
	GRID_STRIDE(i, padded) col[i] = i < total ? (0u | kHot) : 0u;
}

__global__ void gather_heavy_kernel(const uint32_t *perm, const heavy_row *hlist, uint32_t nh, heavy_row *out)
{
	GRID_STRIDE(i, nh) out[i] = hlist[perm[i]];
}

__device__ __forceinline__ void copy_val(char *dst, const char *src, size_t es)
{
	if (es == 4) *reinterpret_cast<uint32_t *>(dst) = *reinterpret_cast<const uint32_t *>(src);
	else if (es == 8) *reinterpret_cast<uint64_t *>(dst) = *reinterpret_cast<const uint64_t *>(src);
	else for (size_t b = 0; b < es; b++) dst[b] = src[b];
}

// entries [b, e) of row r at stream offset `at`: hot slot or column id, the
// row-end bit on the row's last entry when `close`; returns the hot count
__device__ __forceinline__ uint32_t put_entries(const int32_t *col, const char *val, size_t es, uint32_t rb,
		uint32_t b, uint32_t e, uint64_t at, bool close, const int32_t *slot_of, uint32_t *out, char *oval,
		int lane)
{
	uint32_t h = 0;
	for (uint32_t i = b + lane; i < e; i += 32) {
		const uint32_t c = uint32_t(col[rb + i]);
		const int32_t sl = slot_of[c];
		uint32_t v = sl >= 0 ? (uint32_t(sl) | kHot) : c;
		if (close && i + 1 == e) v |= kEnd;
		out[at + (i - b)] = v;
		if (es) copy_val(oval + (at + (i - b)) * es, val + size_t(rb + i) * es, es);
		h += sl >= 0;
	}
	return h;
}

// a warp per row: the row's place in its run, then its chunks
__global__ void scatter_kernel(const uint32_t *row_ptr, const int32_t *col, const char *val, size_t es, uint64_t n,
		const uint64_t *L, const uint32_t *start, const uint32_t *sidx, const uint64_t *seg_L0, const uint64_t *at,
		const uint32_t *chunks, const uint32_t *cfirst, uint32_t s_run, const int32_t *slot_of, uint32_t *out,
		char *oval, unsigned long long *hot_entries)
{
	const int lane = threadIdx.x & 31;
	const uint64_t w0 = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5;
	const uint64_t nw = (uint64_t(gridDim.x) * blockDim.x) >> 5;
	unsigned long long h = 0;
	for (uint64_t r = w0; r < n; r += nw) {
		const uint32_t rb = row_ptr[r], d = row_ptr[r + 1] - rb;
		const uint32_t seg = sidx[r] + start[r] - 1;
		const uint64_t base = at[seg] + (L[r] - seg_L0[seg]);
		if (d >= 1 && d <= kExactMax) {
			h += put_entries(col, val, es, rb, 0, d, base, true, slot_of, out, oval, lane);
		} else if (lane == 0) {
			out[base] = (0u | kHot) | kEnd;          // the zero-row entry of an empty or longer row
		}
		const uint32_t cnt = chunks[r];
		for (uint32_t c = 0; c < cnt; c++) {
			const uint32_t b = uint32_t(uint64_t(d) * c / cnt), e = uint32_t(uint64_t(d) * (c + 1) / cnt);
			h += put_entries(col, val, es, rb, b, e, at[s_run + cfirst[r] + c], false, slot_of, out, oval, lane);
		}
	}
	for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
	if (lane == 0 && h) atomicAdd(hot_entries, h);
}

struct tmp {
	cudaStream_t st;
	std::vector<void *> p;
	~tmp()
	{
		for (void *q : p) cudaFreeAsync(q, st);
	}
	template <class T>
	int get(T **out, size_t count)
	{
		void *q = nullptr;
		cudaError_t e = work_alloc(&q, std::max<size_t>(count, 1) * sizeof(T), st);
		if (e != cudaSuccess)
			return set_error(FMX_ERR_OOM, "device scheduler: %zu bytes: %s", count * sizeof(T), cudaGetErrorString(e));
		p.push_back(q);
		*out = static_cast<T *>(q);
		return FMX_OK;
	}
};

template <class K, class V>
static int sort_pairs(tmp &t, K *k0, K *k1, V *v0, V *v1, uint64_t n, int bits, const K **ko, const V **vo)
{
	cub::DoubleBuffer<K> dk(k0, k1);
	cub::DoubleBuffer<V> dv(v0, v1);
	size_t bytes = 0;
	SCUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, bytes, dk, dv, int(n), 0, bits, t.st));
	char *w = nullptr;
	if (int rc = t.get(&w, bytes)) return rc;
	SCUDA_TRY(cub::DeviceRadixSort::SortPairs(w, bytes, dk, dv, int(n), 0, bits, t.st));
	*ko = dk.Current();
	*vo = dv.Current();
	return FMX_OK;
}

template <class TI, class TO>
static int excl_scan(tmp &t, const TI *in, TO *out, uint64_t n)
{
	size_t bytes = 0;
	SCUDA_TRY(cub::DeviceScan::ExclusiveScan(nullptr, bytes, in, out, cub::Sum(), TO(0), int(n), t.st));
	char *w = nullptr;
	if (int rc = t.get(&w, bytes)) return rc;
	SCUDA_TRY(cub::DeviceScan::ExclusiveScan(w, bytes, in, out, cub::Sum(), TO(0), int(n), t.st));
	return FMX_OK;
}

template <class T>
static int fetch(const T *dev, T &host, cudaStream_t st)
{
	SCUDA_TRY(cudaMemcpyAsync(&host, dev, sizeof(T), cudaMemcpyDeviceToHost, st));
	SCUDA_TRY(cudaStreamSynchronize(st));
	return FMX_OK;
}

template <class T>
static int dalloc(T **p, size_t count, uint64_t &bytes)
{
	*p = nullptr;
	if (!count) return FMX_OK;
	cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), count * sizeof(T));
	if (e != cudaSuccess)
		return set_error(e == cudaErrorMemoryAllocation ? FMX_ERR_OOM : FMX_ERR_CUDA, "cudaMalloc of %zu bytes failed: %s",
				count * sizeof(T), cudaGetErrorString(e));
	bytes += count * sizeof(T);
	return FMX_OK;
}

#define TRY(x) do { if (int rc__ = (x)) return rc__; } while (0)

} // namespace gsched

int make_part_device(const dev_csr &csr, int device, cudaStream_t st, std::shared_ptr<gpu_part> &out)
{
	using namespace gsched;
	if (csr.ncols > (1ull << 30))
		return set_error(FMX_ERR_UNSUPPORTED, "%llu columns: the entry stream holds 30-bit column ids",
				(unsigned long long)csr.ncols);
	device_guard on_device(device);
	if (!on_device.ok()) return set_error(FMX_ERR_CUDA, "cannot make device %d current", device);
	auto p = std::make_shared<gpu_part>();
	p->device = device;
	p->nrows = csr.nrows; p->ncols = csr.ncols; p->nnz = csr.nnz;
	p->prim = csr.prim; p->esize = csr.esize;
	const uint64_t n = csr.nrows, nc = csr.ncols, nnz = csr.nnz;
	const size_t es = csr.esize;
	tmp t{st, {}};
	unsigned long long *cnt;                     // ncand, n_exact, hot_entries, n_long, n_block
	TRY(t.get(&cnt, 5));
	SCUDA_TRY(cudaMemsetAsync(cnt, 0, 5 * sizeof(unsigned long long), st));

	// 1. hot columns
	uint32_t *indeg, *hk0, *hk1, *hv0, *hv1;
	int32_t *slot_of;
	TRY(t.get(&indeg, nc)); TRY(t.get(&hk0, nc)); TRY(t.get(&hk1, nc)); TRY(t.get(&hv0, nc)); TRY(t.get(&hv1, nc));
	TRY(t.get(&slot_of, nc));
	SCUDA_TRY(cudaMemsetAsync(indeg, 0, std::max<uint64_t>(nc, 1) * sizeof(uint32_t), st));
	SCUDA_TRY(cudaMemsetAsync(slot_of, 0xFF, std::max<uint64_t>(nc, 1) * sizeof(int32_t), st));
	if (nnz) indeg_kernel<<<grid(nnz), kT, 0, st>>>(csr.col, nnz, indeg);
	if (nc) hot_keys_kernel<<<grid(nc), kT, 0, st>>>(indeg, nc, hk0, hv0, cnt + 0);
	SCUDA_TRY(cudaGetLastError());
	const uint32_t *hkey = hk0, *hot_sorted = hv0;
	if (nc) TRY(sort_pairs(t, hk0, hk1, hv0, hv1, nc, kDegBits, &hkey, &hot_sorted));
	unsigned long long ncand = 0;
	TRY(fetch(cnt + 0, ncand, st));
	const uint32_t nhot = uint32_t(std::min<unsigned long long>(kHotMax, ncand));
	if (nhot) slot_kernel<<<grid(nhot), kT, 0, st>>>(hot_sorted, nhot, slot_of);
	SCUDA_TRY(cudaGetLastError());

	// 2. rows
	uint64_t *lens, *L;
	uint32_t *chunks, *hflag, *cfirst, *hidx, *start, *sidx;
	TRY(t.get(&lens, n + 1)); TRY(t.get(&L, n + 1)); TRY(t.get(&chunks, n + 1)); TRY(t.get(&hflag, n + 1));
	TRY(t.get(&cfirst, n + 1)); TRY(t.get(&hidx, n + 1)); TRY(t.get(&start, n + 1)); TRY(t.get(&sidx, n + 1));
	row_info_kernel<<<grid(n + 1), kT, 0, st>>>(csr.row_ptr, n, lens, chunks, hflag, cnt + 1);
	SCUDA_TRY(cudaGetLastError());
	TRY(excl_scan(t, lens, L, n + 1));
	TRY(excl_scan(t, chunks, cfirst, n + 1));
	TRY(excl_scan(t, hflag, hidx, n + 1));
	uint64_t total_len = 0;
	TRY(fetch(L + n, total_len, st));
	start_kernel<<<grid(n + 1), kT, 0, st>>>(L, n, range_entries(total_len), start);
	SCUDA_TRY(cudaGetLastError());
	TRY(excl_scan(t, start, sidx, n + 1));
	uint32_t s_run = 0, n_chunks = 0, n_heavy = 0;
	SCUDA_TRY(cudaMemcpyAsync(&s_run, sidx + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
	SCUDA_TRY(cudaMemcpyAsync(&n_chunks, cfirst + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
	TRY(fetch(hidx + n, n_heavy, st));
	const uint64_t nseg = uint64_t(s_run) + n_chunks;

	// 3. segments
	uint32_t *seg_row0, *seg_plen, *seg_slot;
	uint64_t *seg_L0, *at;
	heavy_row *hlist;
	uint32_t *hk2, *hk3, *hv2, *hv3;
	TRY(t.get(&seg_row0, nseg)); TRY(t.get(&seg_plen, nseg + 1)); TRY(t.get(&seg_slot, nseg));
	TRY(t.get(&seg_L0, s_run)); TRY(t.get(&at, nseg + 1)); TRY(t.get(&hlist, n_heavy));
	TRY(t.get(&hk2, n_heavy)); TRY(t.get(&hk3, n_heavy)); TRY(t.get(&hv2, n_heavy)); TRY(t.get(&hv3, n_heavy));
	if (n) run_seg_kernel<<<grid(n), kT, 0, st>>>(start, sidx, L, n, seg_row0, seg_L0, seg_slot);
	if (s_run) run_len_kernel<<<grid(s_run), kT, 0, st>>>(seg_L0, s_run, L, n, seg_plen);
	if (n_heavy)
		heavy_kernel<<<grid(n), kT, 0, st>>>(csr.row_ptr, hflag, hidx, chunks, cfirst, n, s_run, hlist, hk2, hv2,
				seg_row0, seg_plen, seg_slot, cnt + 3, cnt + 4);
	SCUDA_TRY(cudaMemsetAsync(seg_plen + nseg, 0, sizeof(uint32_t), st));
	SCUDA_TRY(cudaGetLastError());
	TRY(excl_scan(t, seg_plen, at, nseg + 1));
	uint64_t total = 0;
	TRY(fetch(at + nseg, total, st));
	if (total >= (1ull << 32) - 64)
		return set_error(FMX_ERR_UNSUPPORTED, "%llu stream entries: offsets are 32-bit", (unsigned long long)total);

	// 4. ranges, longest first
	uint32_t *lk0, *lk1, *lv0, *lv1;
	TRY(t.get(&lk0, nseg)); TRY(t.get(&lk1, nseg)); TRY(t.get(&lv0, nseg)); TRY(t.get(&lv1, nseg));
	uint64_t &bytes = p->bytes;
	TRY(dalloc(&p->ranges, nseg, bytes));
	if (nseg) {
		len_keys_kernel<<<grid(nseg), kT, 0, st>>>(seg_plen, uint32_t(nseg), lk0, lv0);
		SCUDA_TRY(cudaGetLastError());
		const uint32_t *lk = lk0, *perm = lv0;
		TRY(sort_pairs(t, lk0, lk1, lv0, lv1, nseg, kLenBits, &lk, &perm));
		ranges_kernel<<<grid(nseg), kT, 0, st>>>(perm, uint32_t(nseg), at, seg_plen, seg_row0, seg_slot, p->ranges);
		SCUDA_TRY(cudaGetLastError());
	}

	// 5. the stream (plus kStep entries so that index prefetches stay in bounds)
	const uint64_t padded = total + kStep;
	TRY(dalloc(&p->col, padded, bytes));
	fill_stream_kernel<<<grid(padded), kT, 0, st>>>(p->col, total, padded);
	SCUDA_TRY(cudaGetLastError());
	char *val = nullptr;
	if (es) {
		TRY(dalloc(&val, padded * es, bytes));
		SCUDA_TRY(cudaMemsetAsync(val, 0, padded * es, st));
		p->val = val;
	}
	if (n)
		scatter_kernel<<<grid(n * 32), kT, 0, st>>>(csr.row_ptr, csr.col, csr.val, es, n, L, start, sidx, seg_L0, at,
				chunks, cfirst, s_run, slot_of, p->col, val, cnt + 2);
	SCUDA_TRY(cudaGetLastError());

	// 6. heavy rows, most chunks first
	TRY(dalloc(&p->heavy, n_heavy, bytes));
	if (n_heavy) {
		const uint32_t *hk = hk2, *hperm = hv2;
		TRY(sort_pairs(t, hk2, hk3, hv2, hv3, n_heavy, 32, &hk, &hperm));
		gather_heavy_kernel<<<grid(n_heavy), kT, 0, st>>>(hperm, hlist, n_heavy, p->heavy);
		SCUDA_TRY(cudaGetLastError());
	}
	TRY(dalloc(&p->hot_col, nhot, bytes));
	if (nhot) SCUDA_TRY(cudaMemcpyAsync(p->hot_col, hot_sorted, nhot * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));

	unsigned long long hc[5] = {};
	SCUDA_TRY(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, st));
	SCUDA_TRY(cudaStreamSynchronize(st));
	p->n_hot = nhot;
	p->n_exact = uint32_t(hc[1]);
	p->hot_entries = hc[2];
	p->n_long_heavy = uint32_t(hc[3]);
	p->n_block_heavy = uint32_t(hc[4]);
	p->n_ranges = uint32_t(nseg);
	p->n_heavy = n_heavy;
	p->n_partials = n_chunks;
	TRY(dalloc(reinterpret_cast<char **>(&p->partial), size_t(n_chunks) * kPartialStride * 8, bytes));
	TRY(dalloc(reinterpret_cast<char **>(&p->xhot), size_t(nhot + 1) * kPanelBytes, bytes));
	SCUDA_TRY(cudaMemsetAsync(p->xhot, 0, size_t(nhot + 1) * kPanelBytes, st));
	SCUDA_TRY(cudaStreamSynchronize(st));
	out = p;
	return FMX_OK;
}

} // namespace fmx
