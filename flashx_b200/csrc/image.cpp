// Host side of libfmx: the reference's 2D image (.mat_idx / .mat), its
// validation, a parallel edge-list -> image builder, and the decoder that
// turns an image into the row-major CSR the GPU layout is built from.
//
// Format: matrix/sparse_matrix_format.h:35-436 and matrix/matrix_header.h
// of FlashX.  The builder follows the semantics of fm::create_2d_matrix
// (matrix/fm_utils.cpp:617-715,726-841); the code is this library's own:
// a parallel count/scatter by row, per-row sorts, and per-block-row tile
// serialisation in parallel.
#include "fmx_internal.h"

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <thread>
#include <mutex>
#include <numeric>

namespace fmx {

static thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...)
{
	char buf[1024];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof(buf), fmt, ap);
	va_end(ap);
	g_last_error = buf;
	return code;
}

const char *last_error_str() { return g_last_error.c_str(); }

size_t prim_size(int prim)
{
	switch (prim) {
	case FMX_P_BOOL: return 0;
	case FMX_P_INTEGER: case FMX_P_FLOAT: return 4;
	case FMX_P_LONG: case FMX_P_DOUBLE: return 8;
	}
	return SIZE_MAX;
}

bool is_pow2(uint64_t v) { return v && !(v & (v - 1)); }

static int ilog2(uint64_t v) { int l = 0; while ((uint64_t(1) << l) < v) l++; return l; }

int default_threads()
{
	const char *e = getenv("FMX_HOST_THREADS");
	if (e && atoi(e) > 0) return atoi(e);
	unsigned n = std::thread::hardware_concurrency();
	return n ? int(n) : 1;
}

// Run fn(i) for i in [0, n) on `nthreads` threads, dynamically chunked.
template <class F>
static void parallel_for(uint64_t n, int nthreads, uint64_t chunk, F fn)
{
	if (nthreads <= 1 || n <= chunk) {
		for (uint64_t i = 0; i < n; i++) fn(i);
		return;
	}
	std::atomic<uint64_t> next{0};
	auto work = [&]() {
		for (;;) {
			uint64_t b = next.fetch_add(chunk);
			if (b >= n) break;
			uint64_t e = std::min(n, b + chunk);
			for (uint64_t i = b; i < e; i++) fn(i);
		}
	};
	std::vector<std::thread> th;
	int t = int(std::min<uint64_t>(nthreads, (n + chunk - 1) / chunk));
	for (int i = 1; i < t; i++) th.emplace_back(work);
	work();
	for (auto &x : th) x.join();
}

// ---------------------------------------------------------------------------
// Validation
// ---------------------------------------------------------------------------

static inline uint16_t rd16(const char *p) { uint16_t v; memcpy(&v, p, 2); return v; }

static int check_header(const header_info &h, const char *what)
{
	if (h.magic_number != kMagic)
		return set_error(FMX_ERR_IMAGE, "%s: wrong magic number %llx", what, (unsigned long long)h.magic_number);
	if (h.version_number != kVersion)
		return set_error(FMX_ERR_IMAGE, "%s: wrong version number %d", what, h.version_number);
	if (h.type != kSparse || h.layout != kRow2D)
		return set_error(FMX_ERR_IMAGE, "%s: not a 2D-partitioned sparse matrix (type %d, layout %d)", what, h.type, h.layout);
	if (!is_pow2(h.block_2d_height) || !is_pow2(h.block_2d_width) ||
			h.block_2d_height > kMaxBlock || h.block_2d_width > kMaxBlock)
		return set_error(FMX_ERR_IMAGE, "%s: block size %llux%llu is not a power of two <= 32768", what,
				(unsigned long long)h.block_2d_height, (unsigned long long)h.block_2d_width);
	size_t es = prim_size(h.data_type);
	if (es == SIZE_MAX)
		return set_error(FMX_ERR_TYPE, "%s: unsupported entry type %d", what, h.data_type);
	if (h.entry_size != es)
		return set_error(FMX_ERR_IMAGE, "%s: entry size %llu does not match type %d", what,
				(unsigned long long)h.entry_size, h.data_type);
	if (h.nrows == 0 || h.ncols == 0 || h.nrows > (1ULL << 31) || h.ncols > (1ULL << 31))
		return set_error(FMX_ERR_UNSUPPORTED, "%s: %llux%llu matrix outside 1..2^31 rows/cols (int32 indices)", what,
				(unsigned long long)h.nrows, (unsigned long long)h.ncols);
	return FMX_OK;
}

// Walk one block row; returns its nnz or a negative status.  With `deep`,
// every row part and COO entry is checked against the block and matrix bounds
// (sparse_block_2d::verify, sparse_matrix_format.cpp:36-60).
static int64_t walk_block_row(const image &img, uint64_t b, bool deep)
{
	const header_info &h = img.h;
	const uint64_t bh = h.block_2d_height, bw = h.block_2d_width;
	const size_t es = h.entry_size;
	const uint64_t nbcols = (h.ncols + bw - 1) / bw;
	const char *p = img.mat.data() + img.offs()[b];
	const char *end = img.mat.data() + img.offs()[b + 1];
	int64_t nnz = 0;
	int64_t prev_col = -1;
	while (p < end) {
		if (end - p < (ptrdiff_t)sizeof(tile_header))
			return set_error(FMX_ERR_IMAGE, "block row %llu: truncated tile header", (unsigned long long)b);
		tile_header t;
		memcpy(&t, p, sizeof(t));
		if (t.brow != b)
			return set_error(FMX_ERR_IMAGE, "block row %llu: tile claims block row %u", (unsigned long long)b, t.brow);
		if (t.nnz == 0) {
			// An empty tile (the 16-byte placeholder of an empty block row,
			// fm_utils.cpp:341-351) ends the walk.
			break;
		}
		size_t sz = tile_bytes(t, es);
		if ((size_t)(end - p) < sz)
			return set_error(FMX_ERR_IMAGE, "block row %llu: tile (%u,%u) overruns the block row", (unsigned long long)b, t.brow, t.bcol);
		if ((int64_t)t.bcol <= prev_col || t.bcol >= nbcols)
			return set_error(FMX_ERR_IMAGE, "block row %llu: tile column %u out of order or range", (unsigned long long)b, t.bcol);
		prev_col = t.bcol;
		if (t.ncoo > t.nrow || t.ncoo > t.nnz || t.nrow > bh || (t.nrow - t.ncoo) > (t.nnz - t.ncoo))
			return set_error(FMX_ERR_IMAGE, "tile (%u,%u): inconsistent counts nnz=%u nrow=%u ncoo=%u", t.brow, t.bcol, t.nnz, t.nrow, t.ncoo);
		if (deep) {
			const uint64_t rlim = std::min<uint64_t>(bh, h.nrows - uint64_t(b) * bh);
			const uint64_t clim = std::min<uint64_t>(bw, h.ncols - uint64_t(t.bcol) * bw);
			const char *rp = p + sizeof(tile_header);
			const char *rend = rp + tile_rheader(t) - 2;
			uint64_t rows = 0, ents = 0;
			int64_t prev_row = -1;
			while (rp < rend) {
				uint16_t w = rd16(rp);
				if (!(w & 0x8000))
					return set_error(FMX_ERR_IMAGE, "tile (%u,%u): row part without a row header", t.brow, t.bcol);
				int64_t row = w & 0x7FFF;
				if ((uint64_t)row >= rlim || row <= prev_row)
					return set_error(FMX_ERR_IMAGE, "tile (%u,%u): row %lld out of range or order", t.brow, t.bcol, (long long)row);
				prev_row = row;
				rp += 2;
				uint64_t cnt = 0;
				while (rp < rend && !(rd16(rp) & 0x8000)) {
					if (rd16(rp) >= clim)
						return set_error(FMX_ERR_IMAGE, "tile (%u,%u): column %u out of range", t.brow, t.bcol, rd16(rp));
					rp += 2; cnt++;
				}
				if (cnt < 1)
					return set_error(FMX_ERR_IMAGE, "tile (%u,%u): empty row part", t.brow, t.bcol);
				rows++; ents += cnt;
			}
			if (rd16(rend) != 0xFFFF)
				return set_error(FMX_ERR_IMAGE, "tile (%u,%u): missing end-of-row-parts marker", t.brow, t.bcol);
			if (rows != uint64_t(t.nrow - t.ncoo) || ents != uint64_t(t.nnz - t.ncoo))
				return set_error(FMX_ERR_IMAGE, "tile (%u,%u): row parts hold %llu rows / %llu entries, header says %u / %u",
						t.brow, t.bcol, (unsigned long long)rows, (unsigned long long)ents, t.nrow - t.ncoo, t.nnz - t.ncoo);
			const char *coo = p + sizeof(tile_header) + tile_rheader(t);
			for (uint32_t i = 0; i < t.ncoo; i++) {
				uint16_t r = rd16(coo + 4 * i), c = rd16(coo + 4 * i + 2);
				if (!(r & 0x8000) || (r & 0x7FFF) >= rlim || c >= clim)
					return set_error(FMX_ERR_IMAGE, "tile (%u,%u): COO entry %u out of range", t.brow, t.bcol, i);
			}
		}
		nnz += t.nnz;
		p += sz;
	}
	return nnz;
}

int validate(image &img, bool deep)
{
	if (img.idx.size() < kPage + 16 || img.mat.size() < kPage)
		return set_error(FMX_ERR_IMAGE, "image too small (idx %zu bytes, mat %zu bytes)", img.idx.size(), img.mat.size());
	memcpy(&img.h, img.idx.data(), sizeof(header_info));
	int rc = check_header(img.h, ".mat_idx header");
	if (rc) return rc;
	header_info mh;
	memcpy(&mh, img.mat.data(), sizeof(header_info));
	rc = check_header(mh, ".mat header");
	if (rc) return rc;
	if (memcmp(&mh, &img.h, sizeof(header_info)) != 0)
		return set_error(FMX_ERR_IMAGE, ".mat and .mat_idx headers differ");
	img.nbrows = (img.h.nrows + img.h.block_2d_height - 1) / img.h.block_2d_height;
	if (img.idx.size() < kPage + 8 * (img.nbrows + 1))
		return set_error(FMX_ERR_IMAGE, ".mat_idx holds fewer than %llu offsets", (unsigned long long)(img.nbrows + 1));
	// The index is 8-byte aligned inside the vector (page offset).
	const int64_t *o = img.offs();
	if (o[0] != (int64_t)kPage)
		return set_error(FMX_ERR_IMAGE, "first block row offset %lld != 4096", (long long)o[0]);
	for (uint64_t b = 0; b < img.nbrows; b++)
		if (o[b + 1] <= o[b])
			return set_error(FMX_ERR_IMAGE, "block row offsets not increasing at %llu", (unsigned long long)b);
	if ((uint64_t)o[img.nbrows] > img.mat.size())
		return set_error(FMX_ERR_IMAGE, "index points past the end of .mat (%lld > %zu)", (long long)o[img.nbrows], img.mat.size());
	std::vector<int64_t> per(img.nbrows);
	std::atomic<int> bad{0};
	std::mutex mu;
	std::string first_err;
	int first_rc = 0;
	parallel_for(img.nbrows, default_threads(), 4, [&](uint64_t b) {
		if (bad.load(std::memory_order_relaxed)) return;
		int64_t r = walk_block_row(img, b, deep);
		if (r < 0) {
			std::lock_guard<std::mutex> g(mu);
			if (!bad.exchange(1)) { first_rc = int(r); first_err = g_last_error; }
		} else per[b] = r;
	});
	if (bad) { g_last_error = first_err; return first_rc; }
	img.nnz = 0;
	for (auto v : per) img.nnz += uint64_t(v);
	return FMX_OK;
}

// ---------------------------------------------------------------------------
// Decoder: image -> host CSR
// ---------------------------------------------------------------------------

int decode_to_csr(const image &img, host_csr &out, int nthreads)
{
	const header_info &h = img.h;
	const uint64_t bh = h.block_2d_height, bw = h.block_2d_width;
	const size_t es = h.entry_size;
	if (img.nnz >= (1ULL << 32))
		return set_error(FMX_ERR_UNSUPPORTED, "%llu non-zeros: row offsets are 32-bit (< 2^32 entries)", (unsigned long long)img.nnz);
	out.nrows = h.nrows; out.ncols = h.ncols; out.nnz = img.nnz;
	out.prim = h.data_type; out.esize = es;
	try {
		out.row_ptr.assign(h.nrows + 1, 0);
		out.col.resize(img.nnz);
		out.val.resize(img.nnz * es);
	} catch (...) {
		return set_error(FMX_ERR_OOM, "host allocation of the decoded CSR failed");
	}
	uint32_t *cnt = out.row_ptr.data() + 1;
	auto for_tiles = [&](uint64_t b, auto fn) {
		const char *p = img.mat.data() + img.offs()[b];
		const char *end = img.mat.data() + img.offs()[b + 1];
		while (p < end) {
			tile_header t;
			memcpy(&t, p, sizeof(t));
			if (t.nnz == 0) break;
			fn(t, p);
			p += tile_bytes(t, es);
		}
	};
	// pass 1: entries per row
	parallel_for(img.nbrows, nthreads, 8, [&](uint64_t b) {
		for_tiles(b, [&](const tile_header &t, const char *p) {
			uint64_t r0 = uint64_t(t.brow) * bh;
			const char *rp = p + sizeof(tile_header);
			const char *rend = rp + tile_rheader(t) - 2;
			while (rp < rend) {
				uint16_t row = rd16(rp) & 0x7FFF;
				rp += 2;
				uint32_t c = 0;
				while (!(rd16(rp) & 0x8000)) { rp += 2; c++; }
				cnt[r0 + row] += c;
			}
			const char *coo = p + sizeof(tile_header) + tile_rheader(t);
			for (uint32_t i = 0; i < t.ncoo; i++) cnt[r0 + (rd16(coo + 4 * i) & 0x7FFF)] += 1;
		});
	});
	for (uint64_t r = 0; r < h.nrows; r++) out.row_ptr[r + 1] += out.row_ptr[r];
	// pass 2: fill, per row in the reference's visiting order
	parallel_for(img.nbrows, nthreads, 8, [&](uint64_t b) {
		uint64_t r0 = b * bh;
		uint64_t r1 = std::min<uint64_t>(h.nrows, r0 + bh);
		std::vector<uint32_t> cur(out.row_ptr.begin() + r0, out.row_ptr.begin() + r1);
		for_tiles(b, [&](const tile_header &t, const char *p) {
			int64_t c0 = int64_t(t.bcol) * bw;
			const char *vals = p + sizeof(tile_header) + size_t(t.nrow) * 2 + size_t(t.nnz) * 2 + 2;
			const char *rp = p + sizeof(tile_header);
			const char *rend = rp + tile_rheader(t) - 2;
			size_t vi = 0;
			while (rp < rend) {
				uint16_t row = rd16(rp) & 0x7FFF;
				rp += 2;
				while (!(rd16(rp) & 0x8000)) {
					uint32_t pos = cur[row]++;
					out.col[pos] = int32_t(c0 + rd16(rp));
					if (es) memcpy(&out.val[size_t(pos) * es], vals + vi * es, es);
					rp += 2; vi++;
				}
			}
			const char *coo = p + sizeof(tile_header) + tile_rheader(t);
			const char *coov = vals + size_t(t.nnz - t.ncoo) * es;
			for (uint32_t i = 0; i < t.ncoo; i++) {
				uint16_t row = rd16(coo + 4 * i) & 0x7FFF;
				uint32_t pos = cur[row]++;
				out.col[pos] = int32_t(c0 + rd16(coo + 4 * i + 2));
				if (es) memcpy(&out.val[size_t(pos) * es], coov + size_t(i) * es, es);
			}
		});
	});
	return FMX_OK;
}

// ---------------------------------------------------------------------------
// Builder: edge list -> image
// ---------------------------------------------------------------------------

namespace {

struct tile_count { uint32_t nnz, nrow, ncoo; };

} // namespace

static int build_image(const uint32_t *src, const uint32_t *dst, const void *vals, int prim,
		uint64_t nedges, uint64_t nrows, uint64_t ncols, uint32_t bh, uint32_t bw, int flags,
		int nthreads, image &img)
{
	const size_t es = prim_size(prim);
	if (es == SIZE_MAX) return set_error(FMX_ERR_TYPE, "unsupported value type %d", prim);
	if (es && !vals) return set_error(FMX_ERR_INVAL, "value type %d given without values", prim);
	if (!is_pow2(bh) || !is_pow2(bw) || bh > kMaxBlock || bw > kMaxBlock)
		return set_error(FMX_ERR_INVAL, "block size %ux%u must be powers of two <= 32768", bh, bw);
	if (nedges && (!src || !dst)) return set_error(FMX_ERR_INVAL, "null edge arrays");
	if (nthreads <= 0) nthreads = default_threads();
	const bool dedup = flags & FMX_BUILD_DEDUP;
	const bool keep_self = flags & FMX_BUILD_KEEP_SELF_LOOPS;
	const bool ref_vals = flags & FMX_BUILD_REF_VALUE_LAYOUT;

	if (nrows == 0 || ncols == 0) {
		// max vertex id + 1 (fm_utils.cpp:730-739,788)
		std::vector<uint32_t> mx(nthreads, 0);
		std::atomic<int> tid{0};
		uint64_t per = (nedges + nthreads - 1) / std::max(1, nthreads);
		std::vector<std::thread> th;
		for (int t = 0; t < nthreads; t++)
			th.emplace_back([&, t]() {
				uint64_t b = uint64_t(t) * per, e = std::min(nedges, b + per);
				uint32_t m = 0;
				for (uint64_t i = b; i < e; i++) m = std::max(m, std::max(src[i], dst[i]));
				mx[t] = m;
			});
		for (auto &x : th) x.join();
		uint64_t m = *std::max_element(mx.begin(), mx.end());
		if (nrows == 0) nrows = m + 1;
		if (ncols == 0) ncols = m + 1;
	}
	if (nrows > (1ULL << 31) || ncols > (1ULL << 31))
		return set_error(FMX_ERR_UNSUPPORTED, "matrix %llux%llu exceeds int32 indices", (unsigned long long)nrows, (unsigned long long)ncols);

	// 1. count kept edges per row
	std::vector<std::atomic<uint32_t>> rc(nrows + 1);
	for (auto &a : rc) a.store(0, std::memory_order_relaxed);
	std::atomic<int> range_err{0};
	parallel_for((nedges + 65535) / 65536, nthreads, 1, [&](uint64_t c) {
		uint64_t b = c * 65536, e = std::min(nedges, b + 65536);
		for (uint64_t i = b; i < e; i++) {
			if (src[i] >= nrows || dst[i] >= ncols) { range_err = 1; continue; }
			if (!keep_self && src[i] == dst[i]) continue;
			rc[src[i] + 1].fetch_add(1, std::memory_order_relaxed);
		}
	});
	if (range_err) return set_error(FMX_ERR_INVAL, "edge endpoint outside the %llux%llu matrix", (unsigned long long)nrows, (unsigned long long)ncols);
	std::vector<uint64_t> rp(nrows + 1, 0);
	for (uint64_t r = 0; r < nrows; r++) rp[r + 1] = rp[r] + rc[r + 1].load(std::memory_order_relaxed);
	const uint64_t m = rp[nrows];
	// 2. scatter (column, input position) pairs by row; order is fixed by the
	//    per-row sort on (column, input position) that follows.
	std::vector<uint32_t> cols(m);
	std::vector<uint64_t> pos(es ? m : 0);
	{
		std::vector<std::atomic<uint64_t>> cur(nrows);
		for (uint64_t r = 0; r < nrows; r++) cur[r].store(rp[r], std::memory_order_relaxed);
		parallel_for((nedges + 65535) / 65536, nthreads, 1, [&](uint64_t c) {
			uint64_t b = c * 65536, e = std::min(nedges, b + 65536);
			for (uint64_t i = b; i < e; i++) {
				if (!keep_self && src[i] == dst[i]) continue;
				uint64_t p = cur[src[i]].fetch_add(1, std::memory_order_relaxed);
				cols[p] = dst[i];
				if (es) pos[p] = i;
			}
		});
	}
	// 3. sort each row (ascending column; ties by input position so that
	//    std::unique-style dedup keeps the first occurrence) and dedup.
	std::vector<uint64_t> newlen(nrows);
	parallel_for(nrows, nthreads, 4096, [&](uint64_t r) {
		uint64_t b = rp[r], e = rp[r + 1];
		if (!es) {
			std::sort(cols.begin() + b, cols.begin() + e);
			uint64_t n = e - b;
			if (dedup && n) n = std::unique(cols.begin() + b, cols.begin() + e) - (cols.begin() + b);
			newlen[r] = n;
		} else {
			std::vector<std::pair<uint32_t, uint64_t>> tmp(e - b);
			for (uint64_t i = b; i < e; i++) tmp[i - b] = {cols[i], pos[i]};
			std::sort(tmp.begin(), tmp.end());
			uint64_t n = 0;
			for (uint64_t i = 0; i < tmp.size(); i++) {
				if (dedup && n && tmp[i].first == cols[b + n - 1]) continue;
				cols[b + n] = tmp[i].first; pos[b + n] = tmp[i].second; n++;
			}
			newlen[r] = n;
		}
	});
	// compact rows in place (rows only move left)
	std::vector<uint64_t> crp(nrows + 1, 0);
	for (uint64_t r = 0; r < nrows; r++) crp[r + 1] = crp[r] + newlen[r];
	if (crp[nrows] != m) {
		for (uint64_t r = 0; r < nrows; r++) {
			if (crp[r] == rp[r]) continue;
			std::copy(cols.begin() + rp[r], cols.begin() + rp[r] + newlen[r], cols.begin() + crp[r]);
			if (es) std::copy(pos.begin() + rp[r], pos.begin() + rp[r] + newlen[r], pos.begin() + crp[r]);
		}
	}
	rp.swap(crp);
	const uint64_t nnz = rp[nrows];

	// 4. per block row: tile counts, sizes, then serialisation
	const int wlog = ilog2(bw);
	const uint64_t nbrows = (nrows + bh - 1) / bh;
	const uint64_t nbcols = (ncols + bw - 1) / bw;
	std::vector<uint64_t> brow_bytes(nbrows);
	auto count_tiles = [&](uint64_t b, std::vector<tile_count> &tc) {
		std::fill(tc.begin(), tc.end(), tile_count{0, 0, 0});
		uint64_t r0 = b * bh, r1 = std::min<uint64_t>(nrows, r0 + bh);
		for (uint64_t r = r0; r < r1; r++) {
			uint64_t j = rp[r];
			while (j < rp[r + 1]) {
				uint32_t bc = cols[j] >> wlog;
				uint64_t j1 = j + 1;
				while (j1 < rp[r + 1] && (cols[j1] >> wlog) == bc) j1++;
				tc[bc].nrow++;
				tc[bc].nnz += uint32_t(j1 - j);
				if (j1 - j == 1) tc[bc].ncoo++;
				j = j1;
			}
		}
	};
	{
		std::atomic<uint64_t> next{0};
		auto work = [&]() {
			std::vector<tile_count> tc(nbcols);
			for (;;) {
				uint64_t b = next.fetch_add(1);
				if (b >= nbrows) break;
				count_tiles(b, tc);
				uint64_t bytes = 0;
				for (uint64_t c = 0; c < nbcols; c++) {
					if (!tc[c].nnz) continue;
					tile_header t{uint32_t(b), uint32_t(c), tc[c].nnz, uint16_t(tc[c].nrow), uint16_t(tc[c].ncoo)};
					bytes += tile_bytes(t, es);
				}
				brow_bytes[b] = bytes ? bytes : sizeof(tile_header);
			}
		};
		std::vector<std::thread> th;
		for (int t = 1; t < nthreads; t++) th.emplace_back(work);
		work();
		for (auto &x : th) x.join();
	}
	std::vector<int64_t> offs(nbrows + 1);
	offs[0] = kPage;
	for (uint64_t b = 0; b < nbrows; b++) offs[b + 1] = offs[b] + int64_t(brow_bytes[b]);
	header_info h{};
	h.magic_number = kMagic; h.version_number = kVersion; h.type = kSparse;
	h.entry_size = es; h.nrows = nrows; h.ncols = ncols; h.layout = kRow2D;
	h.data_type = prim; h.block_2d_height = bh; h.block_2d_width = bw;
	try {
		img.mat.assign((size_t(offs[nbrows]) + kPage - 1) / kPage * kPage, 0);
		img.idx.assign(kPage + 8 * (nbrows + 1), 0);
	} catch (...) {
		return set_error(FMX_ERR_OOM, "host allocation of the image failed");
	}
	memcpy(img.mat.data(), &h, sizeof(h));
	memcpy(img.idx.data(), &h, sizeof(h));
	memcpy(img.idx.data() + kPage, offs.data(), 8 * (nbrows + 1));
	const char *vbytes = static_cast<const char *>(vals);
	{
		std::atomic<uint64_t> next{0};
		auto work = [&]() {
			std::vector<tile_count> tc(nbcols);
			struct cursor { char *rpart, *coo, *nzv, *coov; };
			std::vector<cursor> cur(nbcols);
			std::vector<char *> bases(nbcols);
			for (;;) {
				uint64_t b = next.fetch_add(1);
				if (b >= nbrows) break;
				char *out = img.mat.data() + offs[b];
				count_tiles(b, tc);
				size_t at = 0;
				bool any = false;
				for (uint64_t c = 0; c < nbcols; c++) {
					bases[c] = nullptr;
					if (!tc[c].nnz) continue;
					any = true;
					tile_header t{uint32_t(b), uint32_t(c), tc[c].nnz, uint16_t(tc[c].nrow), uint16_t(tc[c].ncoo)};
					char *base = out + at;
					memcpy(base, &t, sizeof(t));
					bases[c] = base;
					cur[c].rpart = base + sizeof(t);
					cur[c].coo = base + sizeof(t) + tile_rheader(t);
					cur[c].nzv = base + sizeof(t) + size_t(t.nrow) * 2 + size_t(t.nnz) * 2 + 2;
					cur[c].coov = cur[c].nzv + size_t(t.nnz - t.ncoo) * es;
					at += tile_bytes(t, es);
				}
				if (!any) {
					tile_header t{uint32_t(b), 0, 0, 0, 0};
					memcpy(out, &t, sizeof(t));
					continue;
				}
				uint64_t r0 = b * bh, r1 = std::min<uint64_t>(nrows, r0 + bh);
				for (uint64_t r = r0; r < r1; r++) {
					uint16_t rowhdr = uint16_t((r & (bh - 1)) | 0x8000);
					uint64_t j = rp[r];
					while (j < rp[r + 1]) {
						uint32_t bc = cols[j] >> wlog;
						uint64_t j1 = j + 1;
						while (j1 < rp[r + 1] && (cols[j1] >> wlog) == bc) j1++;
						// the reference's builder copies a tile's values from
						// the start of the row (fm_utils.cpp:240-241,259-260)
						uint64_t vfrom = ref_vals ? rp[r] : j;
						cursor &cu = cur[bc];
						if (j1 - j == 1) {
							uint16_t cc = uint16_t(cols[j] & (bw - 1));
							memcpy(cu.coo, &rowhdr, 2);
							memcpy(cu.coo + 2, &cc, 2);
							cu.coo += 4;
							if (es) { memcpy(cu.coov, vbytes + pos[vfrom] * es, es); cu.coov += es; }
						} else {
							memcpy(cu.rpart, &rowhdr, 2);
							cu.rpart += 2;
							for (uint64_t q = j; q < j1; q++) {
								uint16_t cc = uint16_t(cols[q] & (bw - 1));
								memcpy(cu.rpart, &cc, 2);
								cu.rpart += 2;
							}
							if (es)
								for (uint64_t q = 0; q < j1 - j; q++) {
									memcpy(cu.nzv, vbytes + pos[vfrom + q] * es, es);
									cu.nzv += es;
								}
						}
						j = j1;
					}
				}
				const uint16_t endm = 0xFFFF;
				for (uint64_t c = 0; c < nbcols; c++)
					if (bases[c]) memcpy(cur[c].rpart, &endm, 2);
			}
		};
		std::vector<std::thread> th;
		for (int t = 1; t < nthreads; t++) th.emplace_back(work);
		work();
		for (auto &x : th) x.join();
	}
	img.h = h;
	img.nbrows = nbrows;
	img.nnz = nnz;
	return FMX_OK;
}

} // namespace fmx

using namespace fmx;

extern "C" {

int fmx_image_build(const uint32_t *src, const uint32_t *dst, const void *vals, int val_type,
		uint64_t nedges, uint64_t nrows, uint64_t ncols, uint32_t block_h, uint32_t block_w,
		int flags, int nthreads, fmx_image **out)
{
	if (!out) return set_error(FMX_ERR_INVAL, "null output handle");
	*out = nullptr;
	if (flags & ~(FMX_BUILD_DEDUP | FMX_BUILD_KEEP_SELF_LOOPS | FMX_BUILD_REF_VALUE_LAYOUT))
		return set_error(FMX_ERR_INVAL, "unknown build flags 0x%x", flags);
	std::unique_ptr<fmx_image> h(new (std::nothrow) fmx_image);
	if (!h) return set_error(FMX_ERR_OOM, "out of host memory");
	int rc;
	try {
		rc = build_image(src, dst, vals, val_type, nedges, nrows, ncols, block_h, block_w, flags, nthreads, h->im);
	} catch (const std::bad_alloc &) {
		return set_error(FMX_ERR_OOM, "host allocation failed while building the image");
	}
	if (rc) return rc;
	*out = h.release();
	return FMX_OK;
}

int fmx_image_from_bytes(const void *idx, size_t idx_len, const void *mat, size_t mat_len, fmx_image **out)
{
	if (!out || !idx || !mat) return set_error(FMX_ERR_INVAL, "null argument");
	*out = nullptr;
	std::unique_ptr<fmx_image> h(new (std::nothrow) fmx_image);
	if (!h) return set_error(FMX_ERR_OOM, "out of host memory");
	try {
		h->im.idx.assign((const char *)idx, (const char *)idx + idx_len);
		h->im.mat.assign((const char *)mat, (const char *)mat + mat_len);
	} catch (...) {
		return set_error(FMX_ERR_OOM, "host allocation failed");
	}
	int rc = validate(h->im, true);
	if (rc) return rc;
	*out = h.release();
	return FMX_OK;
}

static int read_file(const char *path, std::vector<char> &buf)
{
	FILE *f = fopen(path, "rb");
	if (!f) return set_error(FMX_ERR_IO, "can't open %s", path);
	fseek(f, 0, SEEK_END);
	long sz = ftell(f);
	fseek(f, 0, SEEK_SET);
	try { buf.resize(size_t(sz)); } catch (...) { fclose(f); return set_error(FMX_ERR_OOM, "out of host memory reading %s", path); }
	size_t got = sz ? fread(buf.data(), 1, size_t(sz), f) : 0;
	fclose(f);
	if (got != size_t(sz)) return set_error(FMX_ERR_IO, "can't read %s", path);
	return FMX_OK;
}

int fmx_image_load(const char *mat_idx_path, const char *mat_path, fmx_image **out)
{
	if (!out || !mat_idx_path || !mat_path) return set_error(FMX_ERR_INVAL, "null argument");
	*out = nullptr;
	std::unique_ptr<fmx_image> h(new (std::nothrow) fmx_image);
	if (!h) return set_error(FMX_ERR_OOM, "out of host memory");
	int rc = read_file(mat_idx_path, h->im.idx);
	if (!rc) rc = read_file(mat_path, h->im.mat);
	if (!rc) rc = validate(h->im, true);
	if (rc) return rc;
	*out = h.release();
	return FMX_OK;
}

int fmx_image_dump(const fmx_image *img, const char *mat_idx_path, const char *mat_path)
{
	if (!img || !mat_idx_path || !mat_path) return set_error(FMX_ERR_INVAL, "null argument");
	const std::vector<char> *parts[2] = {&img->im.idx, &img->im.mat};
	const char *paths[2] = {mat_idx_path, mat_path};
	for (int i = 0; i < 2; i++) {
		FILE *f = fopen(paths[i], "wb");
		if (!f) return set_error(FMX_ERR_IO, "can't open %s for writing", paths[i]);
		size_t n = parts[i]->size();
		size_t w = n ? fwrite(parts[i]->data(), 1, n, f) : 0;
		fclose(f);
		if (w != n) return set_error(FMX_ERR_IO, "can't write %s", paths[i]);
	}
	return FMX_OK;
}

int fmx_image_bytes(const fmx_image *img, const void **idx, size_t *idx_len, const void **mat, size_t *mat_len)
{
	if (!img) return set_error(FMX_ERR_INVAL, "null image");
	if (idx) *idx = img->im.idx.data();
	if (idx_len) *idx_len = img->im.idx.size();
	if (mat) *mat = img->im.mat.data();
	if (mat_len) *mat_len = img->im.mat.size();
	return FMX_OK;
}

int fmx_image_info(const fmx_image *img, uint64_t *nrows, uint64_t *ncols, uint64_t *nnz,
		uint32_t *entry_size, int *prim_type, uint32_t *block_h, uint32_t *block_w)
{
	if (!img) return set_error(FMX_ERR_INVAL, "null image");
	if (nrows) *nrows = img->im.h.nrows;
	if (ncols) *ncols = img->im.h.ncols;
	if (nnz) *nnz = img->im.nnz;
	if (entry_size) *entry_size = uint32_t(img->im.h.entry_size);
	if (prim_type) *prim_type = img->im.h.data_type;
	if (block_h) *block_h = uint32_t(img->im.h.block_2d_height);
	if (block_w) *block_w = uint32_t(img->im.h.block_2d_width);
	return FMX_OK;
}

int fmx_image_verify(const fmx_image *img)
{
	if (!img) return set_error(FMX_ERR_INVAL, "null image");
	// validate() rewrites only fields derived from the bytes
	fmx_image *mut = const_cast<fmx_image *>(img);
	return validate(mut->im, true);
}

int fmx_image_free(fmx_image *img)
{
	delete img;
	return FMX_OK;
}

} // extern "C"
