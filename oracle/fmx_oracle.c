/*
 * fmx_oracle.c -- CPU ORACLE for the FlashMatrix 2D-tiled SpMM.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load this library, and only
 * as the checker or the timed CPU baseline.  The product (libfmx.so) never
 * links, loads or falls back to it.
 *
 * A plain-C restatement of the reference's algorithms for this path, each
 * function citing the FlashX file:line it follows:
 *   - the 2D image format  matrix/sparse_matrix_format.h:35-436,
 *                          matrix/matrix_header.h:42-184
 *   - the format builder   matrix/fm_utils.cpp:228-433,435-535,617-715,726-841
 *   - the SpMM traversal   matrix/sparse_matrix.cpp:251-314 (super blocks),
 *                          :120-186 (Hilbert order), :329-393 (out_part),
 *                          matrix/sparse_matrix.h:219-375 (row_part_func,
 *                          coo_func, run_on_block), :450-463 (super block size)
 *   - work distribution    matrix/matrix_io.cpp:163-236 (b2d_io_generator),
 *                          libsafs/in_mem_io.cpp:488-512 (per-task memcpy)
 *   - PageRank             matrix/libmatrix-algs/PageRank.cpp:31-133
 *   - the FlashGraph 1D format and its row SpMM
 *                          flash-graph/graph_file_header.h:27-37,
 *                          flash-graph/vertex.h:444-562 (vertex records),
 *                          flash-graph/utils.cpp:399-420 (file layout),
 *                          flash-graph/fg_sparse_matrix.cpp:83-106 (run_on_row)
 *   - Hilbert curve        matrix/hilbert_curve.cpp:6-34
 * It is pinned against the reference's own header code compiled in place
 * (oracle/ref_walk.cpp -> oracle/_ref/) and against the golden fixtures in
 * tests/golden/.
 *
 * Arithmetic: every output row is accumulated as dest += src * value in the
 * dense type, in ascending column order, starting from zero, without fused
 * multiply-add (the reference is built with -mavx and no FMA,
 * Makefile.common:60).  Build with -ffp-contract=off.
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <time.h>
#include <unistd.h>

#define ORC_PAGE 4096
#define ORC_MAGIC 0x123456789FFFFFFLL
#define ORC_VERSION 2

/* prim_type codes, matrix/generic_type.h:57-70 */
enum { P_BOOL = 0, P_INTEGER = 4, P_LONG = 6, P_FLOAT = 8, P_DOUBLE = 9 };
/* dense type codes of this library */
enum { D_F32 = 0, D_F64 = 1, D_I32 = 3, D_I64 = 4 };

/* matrix_header::info, matrix/matrix_header.h:102-121 (x86-64 layout). */
typedef struct {
	int64_t magic_number;
	int32_t version_number;
	int32_t type;          /* matrix_type: SPARSE = 2 */
	uint64_t entry_size;
	uint64_t nrows;
	uint64_t ncols;
	int32_t layout;        /* matrix_layout_t: L_ROW_2D = 2 */
	int32_t data_type;     /* prim_type */
	uint64_t block_2d_height;
	uint64_t block_2d_width;
} orc_header;

/* sparse_block_2d header, matrix/sparse_matrix_format.h:215-224 (16 bytes). */
typedef struct {
	uint32_t brow, bcol, nnz;
	uint16_t nrow, ncoo;
} orc_tile;

static inline uint16_t rd16(const char *p) { uint16_t v; memcpy(&v, p, 2); return v; }
static inline void wr16(char *p, uint16_t v) { memcpy(p, &v, 2); }

/* sparse_block_2d::get_size, sparse_matrix_format.h:233-241,294-299 */
static inline size_t tile_size(const orc_tile *t, size_t esize)
{
	size_t rindex = (size_t)t->nrow * 2 + (size_t)t->nnz * 2 + 2;
	return sizeof(orc_tile) + rindex + esize * t->nnz;
}
/* get_rheader_size, sparse_matrix_format.h:246-253 */
static inline size_t tile_rheader(const orc_tile *t)
{
	return (size_t)(t->nrow - t->ncoo) * 2 + (size_t)(t->nnz - t->ncoo) * 2 + 2;
}

static int ilog2u(uint64_t v) { int l = 0; while ((1ULL << l) < v) l++; return l; }

/* ===================================================================== */
/* Builder: fm_utils.cpp create_2d_matrix                                 */
/* ===================================================================== */

typedef struct { uint32_t r, c; uint64_t i; } orc_edge;

/*
 * The edges in (row, column) order, equal keys in input order: std::sort by
 * (row, column) (fm_utils.cpp:469,521) with duplicates resolved the way
 * std::unique keeps them, as the first occurrence in the input.  A stable
 * LSD radix sort over the key bits gives exactly that order; it runs its
 * passes on `nth` threads (per-thread digit counts, thread-ordered scatter,
 * so each pass stays stable).
 */
#define ORC_RADIX_BITS 11
typedef struct {
	orc_edge *from, *to;
	uint64_t n, b0, b1;
	int shift, cbits, nth, t;
	uint64_t *cnt;      /* [nth][1 << ORC_RADIX_BITS] */
	pthread_barrier_t *bar;
} orc_rs_arg;

static inline uint32_t orc_digit(const orc_edge *e, int shift, int cbits)
{
	const uint64_t key = ((uint64_t)e->r << cbits) | e->c;
	return (uint32_t)(key >> shift) & ((1u << ORC_RADIX_BITS) - 1);
}

static void *orc_rs_worker(void *p)
{
	orc_rs_arg *a = p;
	const uint32_t nb = 1u << ORC_RADIX_BITS;
	uint64_t *mine = a->cnt + (uint64_t)a->t * nb;
	memset(mine, 0, sizeof(uint64_t) * nb);
	for (uint64_t i = a->b0; i < a->b1; i++) mine[orc_digit(&a->from[i], a->shift, a->cbits)]++;
	pthread_barrier_wait(a->bar);
	if (a->t == 0) {
		/* exclusive offsets in (digit, thread) order */
		uint64_t s = 0;
		for (uint32_t d = 0; d < nb; d++)
			for (int t = 0; t < a->nth; t++) {
				uint64_t c = a->cnt[(uint64_t)t * nb + d];
				a->cnt[(uint64_t)t * nb + d] = s;
				s += c;
			}
	}
	pthread_barrier_wait(a->bar);
	for (uint64_t i = a->b0; i < a->b1; i++) a->to[mine[orc_digit(&a->from[i], a->shift, a->cbits)]++] = a->from[i];
	return NULL;
}

static int orc_sort_edges(orc_edge *e, uint64_t m, uint64_t nrows, uint64_t ncols)
{
	if (m < 2) return 0;
	const int rbits = ilog2u(nrows), cbits = ilog2u(ncols);
	const int bits = rbits + cbits;
	orc_edge *tmp = malloc(sizeof(orc_edge) * m);
	if (!tmp) return -1;
	long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
	int nth = (int)(m / (1u << 20));
	if (nth > ncpu) nth = (int)ncpu;
	if (nth > 64) nth = 64;
	if (nth < 1) nth = 1;
	uint64_t *cnt = malloc(sizeof(uint64_t) * (uint64_t)nth << ORC_RADIX_BITS);
	pthread_t th[64];
	orc_rs_arg args[64];
	pthread_barrier_t bar;
	pthread_barrier_init(&bar, NULL, (unsigned)nth);
	orc_edge *from = e, *to = tmp;
	for (int shift = 0; shift < bits; shift += ORC_RADIX_BITS) {
		for (int t = 0; t < nth; t++) {
			args[t] = (orc_rs_arg){from, to, m, m * (uint64_t)t / (uint64_t)nth, m * (uint64_t)(t + 1) / (uint64_t)nth,
					shift, cbits, nth, t, cnt, &bar};
			if (t) pthread_create(&th[t], NULL, orc_rs_worker, &args[t]);
		}
		orc_rs_worker(&args[0]);
		for (int t = 1; t < nth; t++) pthread_join(th[t], NULL);
		orc_edge *x = from; from = to; to = x;
	}
	pthread_barrier_destroy(&bar);
	if (from != e) memcpy(e, from, sizeof(orc_edge) * m);
	free(cnt);
	free(tmp);
	return 0;
}

/*
 * orc_build_image: edge list -> (.mat_idx bytes, .mat bytes).
 * Semantics of fm_utils.cpp:
 *   - nrows/ncols = max vid + 1 when 0 is passed (:730-739,788);
 *   - every row exists (a sentinel edge per vertex, :763-782), so every block
 *     row is present; an empty block row is one empty 16-byte tile (:341-351);
 *   - self-loops dropped unless keep_self (:459-462,510-513);
 *   - columns sorted per row (:469,521); duplicates dropped only with dedup
 *     (:470-474,522-526), std::unique keeping the first of equal columns;
 *   - per tile a row with 1 entry goes to COO, >= 2 to a row part (:228-265);
 *     tiles in ascending block column, rows ascending inside a tile;
 *   - values: with ref_value_layout, each tile copies its values from the
 *     start of the row (:240-241,259-260, `v.get_data(0)`); otherwise each
 *     entry keeps its own value.
 *   - index: offs[0] = 4096 (header page), offs[i+1] = offs[i] + size of
 *     block row i (:701-712); the image is header + block rows, rounded up to
 *     a page (sparse_matrix_format.cpp:323-333).
 * vals: NULL or nedges entries of esize bytes.  Returns 0 or -1.
 */
int orc_build_image(const uint32_t *src, const uint32_t *dst, const void *vals,
		int prim, uint64_t nedges, uint64_t nrows, uint64_t ncols,
		uint32_t bh, uint32_t bw, int dedup, int keep_self, int ref_value_layout,
		char **idx_out, size_t *idx_len, char **mat_out, size_t *mat_len)
{
	size_t esize = prim == P_BOOL ? 0 : (prim == P_FLOAT || prim == P_INTEGER) ? 4 : 8;
	if (nrows == 0 || ncols == 0) {
		uint64_t mx = 0;
		for (uint64_t i = 0; i < nedges; i++) {
			if (src[i] > mx) mx = src[i];
			if (dst[i] > mx) mx = dst[i];
		}
		if (nrows == 0) nrows = mx + 1;
		if (ncols == 0) ncols = mx + 1;
	}
	int hlog = ilog2u(bh), wlog = ilog2u(bw);
	uint64_t nbrows = (nrows + bh - 1) / bh;
	uint64_t nbcols = (ncols + bw - 1) / bw;

	orc_edge *e = malloc(sizeof(orc_edge) * (nedges ? nedges : 1));
	uint64_t m = 0;
	for (uint64_t i = 0; i < nedges; i++) {
		if (src[i] >= nrows || dst[i] >= ncols) { free(e); return -1; }
		if (!keep_self && src[i] == dst[i]) continue;
		e[m].r = src[i]; e[m].c = dst[i]; e[m].i = i; m++;
	}
	if (orc_sort_edges(e, m, nrows, ncols)) { free(e); return -1; }
	if (dedup && m) {
		uint64_t w = 1;
		for (uint64_t i = 1; i < m; i++)
			if (e[i].r != e[w - 1].r || e[i].c != e[w - 1].c) e[w++] = e[i];
		m = w;
	}
	/* row pointers */
	uint64_t *rp = calloc(nrows + 1, sizeof(uint64_t));
	for (uint64_t i = 0; i < m; i++) rp[e[i].r + 1]++;
	for (uint64_t r = 0; r < nrows; r++) rp[r + 1] += rp[r];

	/* pass 1: sizes per block row (collect_block_info, :267-327) */
	typedef struct { uint32_t nnz; uint32_t nrow; uint32_t ncoo; } binfo;
	binfo *bi = malloc(sizeof(binfo) * nbcols);
	uint64_t *offs = malloc(sizeof(uint64_t) * (nbrows + 1));
	size_t total = ORC_PAGE;
	offs[0] = ORC_PAGE;
	for (uint64_t b = 0; b < nbrows; b++) {
		memset(bi, 0, sizeof(binfo) * nbcols);
		uint64_t r0 = b * bh, r1 = r0 + bh < nrows ? r0 + bh : nrows;
		for (uint64_t r = r0; r < r1; r++) {
			uint64_t j = rp[r];
			while (j < rp[r + 1]) {
				uint64_t bc = e[j].c >> wlog, j1 = j;
				while (j1 < rp[r + 1] && (e[j1].c >> wlog) == bc) j1++;
				bi[bc].nrow++; bi[bc].nnz += (uint32_t)(j1 - j);
				if (j1 - j == 1) bi[bc].ncoo++;
				j = j1;
			}
		}
		size_t bytes = 0;
		for (uint64_t c = 0; c < nbcols; c++) {
			if (!bi[c].nnz) continue;
			orc_tile t = { (uint32_t)b, (uint32_t)c, bi[c].nnz, (uint16_t)bi[c].nrow, (uint16_t)bi[c].ncoo };
			bytes += tile_size(&t, esize);
		}
		if (!bytes) bytes = sizeof(orc_tile);
		total += bytes;
		offs[b + 1] = total;
	}
	size_t mlen = (total + ORC_PAGE - 1) / ORC_PAGE * ORC_PAGE;
	char *mat = calloc(mlen, 1);
	orc_header h;
	memset(&h, 0, sizeof(h));
	h.magic_number = ORC_MAGIC; h.version_number = ORC_VERSION; h.type = 2;
	h.entry_size = esize; h.nrows = nrows; h.ncols = ncols; h.layout = 2;
	h.data_type = prim; h.block_2d_height = bh; h.block_2d_width = bw;
	memcpy(mat, &h, sizeof(h));

	/* pass 2: serialise (run_blocks, :329-433; add_nz, :228-265) */
	typedef struct { char *base; char *rpart; char *coo; char *nzv; char *coov; uint32_t nnz_done, nrow_done; } bptr;
	bptr *bp = malloc(sizeof(bptr) * nbcols);
	for (uint64_t b = 0; b < nbrows; b++) {
		char *out = mat + offs[b];
		memset(bi, 0, sizeof(binfo) * nbcols);
		uint64_t r0 = b * bh, r1 = r0 + bh < nrows ? r0 + bh : nrows;
		for (uint64_t r = r0; r < r1; r++) {
			uint64_t j = rp[r];
			while (j < rp[r + 1]) {
				uint64_t bc = e[j].c >> wlog, j1 = j;
				while (j1 < rp[r + 1] && (e[j1].c >> wlog) == bc) j1++;
				bi[bc].nrow++; bi[bc].nnz += (uint32_t)(j1 - j);
				if (j1 - j == 1) bi[bc].ncoo++;
				j = j1;
			}
		}
		size_t cur = 0; int any = 0;
		for (uint64_t c = 0; c < nbcols; c++) {
			bp[c].base = NULL;
			if (!bi[c].nnz) continue;
			any = 1;
			orc_tile t = { (uint32_t)b, (uint32_t)c, bi[c].nnz, (uint16_t)bi[c].nrow, (uint16_t)bi[c].ncoo };
			char *base = out + cur;
			memcpy(base, &t, sizeof(t));
			bp[c].base = base;
			bp[c].rpart = base + sizeof(orc_tile);
			bp[c].coo = base + sizeof(orc_tile) + tile_rheader(&t);
			bp[c].nzv = base + sizeof(orc_tile) + (size_t)t.nrow * 2 + (size_t)t.nnz * 2 + 2;
			bp[c].coov = bp[c].nzv + (size_t)(t.nnz - t.ncoo) * esize;
			cur += tile_size(&t, esize);
		}
		if (!any) {
			orc_tile t = { (uint32_t)b, 0, 0, 0, 0 };
			memcpy(out, &t, sizeof(t));
			continue;
		}
		for (uint64_t r = r0; r < r1; r++) {
			uint64_t j = rp[r];
			while (j < rp[r + 1]) {
				uint64_t bc = e[j].c >> wlog, j1 = j;
				while (j1 < rp[r + 1] && (e[j1].c >> wlog) == bc) j1++;
				uint64_t vsrc = ref_value_layout ? rp[r] : j;  /* v.get_data(0) */
				if (j1 - j == 1) {
					wr16(bp[bc].coo, (uint16_t)((r & (bh - 1)) | 0x8000));
					wr16(bp[bc].coo + 2, (uint16_t)(e[j].c & (bw - 1)));
					bp[bc].coo += 4;
					if (esize) {
						memcpy(bp[bc].coov, (const char *)vals + e[vsrc].i * esize, esize);
						bp[bc].coov += esize;
					}
				} else {
					wr16(bp[bc].rpart, (uint16_t)((r & (bh - 1)) | 0x8000));
					bp[bc].rpart += 2;
					for (uint64_t q = j; q < j1; q++) {
						wr16(bp[bc].rpart, (uint16_t)(e[q].c & (bw - 1)));
						bp[bc].rpart += 2;
					}
					if (esize)
						for (uint64_t q = 0; q < j1 - j; q++) {
							memcpy(bp[bc].nzv, (const char *)vals + e[vsrc + q].i * esize, esize);
							bp[bc].nzv += esize;
						}
				}
				j = j1;
			}
		}
		/* finalize: the end-of-row-parts marker (sparse_matrix_format.cpp:119-126) */
		for (uint64_t c = 0; c < nbcols; c++)
			if (bp[c].base) wr16(bp[c].rpart, 0xFFFF);
	}
	size_t ilen = ORC_PAGE + sizeof(int64_t) * (nbrows + 1);
	char *idx = calloc(ilen, 1);
	memcpy(idx, &h, sizeof(h));
	for (uint64_t b = 0; b <= nbrows; b++) {
		int64_t o = (int64_t)offs[b];
		memcpy(idx + ORC_PAGE + 8 * b, &o, 8);
	}
	free(bp); free(bi); free(offs); free(rp); free(e);
	*idx_out = idx; *idx_len = ilen; *mat_out = mat; *mat_len = mlen;
	return 0;
}

void orc_free(void *p) { free(p); }

/* ===================================================================== */
/* Image access                                                           */
/* ===================================================================== */

typedef struct {
	orc_header h;
	const int64_t *offs;   /* nbrows + 1 (unaligned-safe copy) */
	int64_t *offs_copy;
	uint64_t nbrows;
	size_t esize;
	const char *mat;
	size_t mat_len;
} orc_img;

static int orc_open(const char *idx, size_t idx_len, const char *mat, size_t mat_len, orc_img *im)
{
	if (idx_len < ORC_PAGE || mat_len < ORC_PAGE) return -1;
	memcpy(&im->h, idx, sizeof(orc_header));
	if (im->h.magic_number != ORC_MAGIC || im->h.version_number != ORC_VERSION) return -1;
	uint64_t bh = im->h.block_2d_height;
	if (!bh) return -1;
	im->nbrows = (im->h.nrows + bh - 1) / bh;
	if (idx_len < ORC_PAGE + 8 * (im->nbrows + 1)) return -1;
	im->offs_copy = malloc(8 * (im->nbrows + 1));
	memcpy(im->offs_copy, idx + ORC_PAGE, 8 * (im->nbrows + 1));
	im->offs = im->offs_copy;
	im->esize = im->h.entry_size;
	im->mat = mat; im->mat_len = mat_len;
	if ((size_t)im->offs[im->nbrows] > mat_len) { free(im->offs_copy); return -1; }
	return 0;
}
static void orc_close(orc_img *im) { free(im->offs_copy); }

/* get_non_zeros (sparse_matrix_format.cpp:62-88) over the whole image:
 * writes (row, col) pairs in image order; returns the count, or -1 on a
 * malformed image.  rows/cols may be NULL to only count. */
int64_t orc_nonzeros(const char *idx, size_t idx_len, const char *mat, size_t mat_len,
		uint64_t *rows, uint64_t *cols, uint64_t cap)
{
	orc_img im;
	if (orc_open(idx, idx_len, mat, mat_len, &im)) return -1;
	uint64_t bh = im.h.block_2d_height, bw = im.h.block_2d_width, n = 0;
	for (uint64_t b = 0; b < im.nbrows; b++) {
		const char *p = im.mat + im.offs[b], *end = im.mat + im.offs[b + 1];
		while (p < end) {
			orc_tile t; memcpy(&t, p, sizeof(t));
			uint64_t r0 = (uint64_t)t.brow * bh, c0 = (uint64_t)t.bcol * bw;
			if (t.nnz) {
				const char *rpp = p + sizeof(orc_tile);
				const char *rend = rpp + tile_rheader(&t) - 2;
				while (rpp < rend) {
					uint16_t row = rd16(rpp) & 0x7FFF; rpp += 2;
					while (rd16(rpp) <= 0x7FFF) {
						if (rows && n < cap) { rows[n] = r0 + row; cols[n] = c0 + rd16(rpp); }
						n++; rpp += 2;
					}
				}
				const char *coo = p + sizeof(orc_tile) + tile_rheader(&t);
				for (uint32_t i = 0; i < t.ncoo; i++) {
					if (rows && n < cap) {
						rows[n] = r0 + (rd16(coo + 4 * i) & 0x7FFF);
						cols[n] = c0 + rd16(coo + 4 * i + 2);
					}
					n++;
				}
			}
			p += tile_size(&t, im.esize);
		}
	}
	orc_close(&im);
	return (int64_t)n;
}

/* ===================================================================== */
/* SpMM (block_spmm_task_impl::run_on_block and friends)                  */
/* ===================================================================== */

/* hilbert_rot / hilbert_xy2d, matrix/hilbert_curve.cpp:6-34 */
static void orc_hilbert_rot(int n, int *x, int *y, int rx, int ry)
{
	if (ry == 0) {
		if (rx == 1) { *x = n - 1 - *x; *y = n - 1 - *y; }
		int t = *x; *x = *y; *y = t;
	}
}
int orc_hilbert_xy2d(int n, int x, int y)
{
	int rx, ry, s, d = 0;
	for (s = n / 2; s > 0; s /= 2) {
		rx = (x & s) > 0; ry = (y & s) > 0;
		d += s * s * ((3 * rx) ^ ry);
		orc_hilbert_rot(s, &x, &y, rx, ry);
	}
	return d;
}

typedef struct {
	orc_img *im;
	int dtype;             /* D_F32 / D_F64 / D_I32 / D_I64 */
	const void *X; void *Y;
	uint64_t k;
	uint64_t sb;           /* super block size in block rows */
	int hilbert;
	int *horder;           /* sb*sb hilbert visit order (flat tile index) */
	uint64_t brow_begin, brow_end;   /* block rows to process */
	int copy_task;         /* memcpy each task's block rows (in_mem_io.cpp:500-501) */
	/* b2d_io_generator state (matrix_io.cpp:163-236) */
	pthread_mutex_t lock;
	uint64_t next_brow, balance_point;
} orc_job;

static double entry_as_double(const char *v, int prim)
{
	switch (prim) {
	case P_FLOAT: { float f; memcpy(&f, v, 4); return f; }
	case P_DOUBLE: { double d; memcpy(&d, v, 8); return d; }
	case P_INTEGER: { int32_t i; memcpy(&i, v, 4); return i; }
	case P_LONG: { int64_t l; memcpy(&l, v, 8); return (double)l; }
	}
	return 1.0;
}
static int64_t entry_as_i64(const char *v, int prim)
{
	switch (prim) {
	case P_INTEGER: { int32_t i; memcpy(&i, v, 4); return i; }
	case P_LONG: { int64_t l; memcpy(&l, v, 8); return l; }
	case P_FLOAT: { float f; memcpy(&f, v, 4); return (int64_t)f; }
	case P_DOUBLE: { double d; memcpy(&d, v, 8); return (int64_t)d; }
	}
	return 1;
}

/* dest_row[j] += src_row[j] * data, sparse_matrix.h:242-243,300-301 */
static inline void axpy_row(int dtype, char *dst, const char *src, uint64_t k,
		const char *val, int prim, size_t esize)
{
	if (dtype == D_F32) {
		float *d = (float *)dst; const float *s = (const float *)src;
		if (!esize) { for (uint64_t j = 0; j < k; j++) d[j] += s[j] * 1.0f; }
		else {
			float v = (float)entry_as_double(val, prim);
			for (uint64_t j = 0; j < k; j++) { float p = s[j] * v; d[j] = d[j] + p; }
		}
	} else if (dtype == D_F64) {
		double *d = (double *)dst; const double *s = (const double *)src;
		double v = esize ? entry_as_double(val, prim) : 1.0;
		for (uint64_t j = 0; j < k; j++) { double p = s[j] * v; d[j] = d[j] + p; }
	} else if (dtype == D_I32) {
		uint32_t *d = (uint32_t *)dst; const uint32_t *s = (const uint32_t *)src;
		uint32_t v = esize ? (uint32_t)entry_as_i64(val, prim) : 1u;
		for (uint64_t j = 0; j < k; j++) d[j] += s[j] * v;
	} else {
		uint64_t *d = (uint64_t *)dst; const uint64_t *s = (const uint64_t *)src;
		uint64_t v = esize ? (uint64_t)entry_as_i64(val, prim) : 1u;
		for (uint64_t j = 0; j < k; j++) d[j] += s[j] * v;
	}
}

static size_t dsize(int dtype) { return (dtype == D_F32 || dtype == D_I32) ? 4 : 8; }

/* run_on_block, sparse_matrix.h:344-375 */
static void orc_run_on_block(orc_job *jb, const char *tile, char *out_rows, uint64_t out_row0)
{
	orc_tile t; memcpy(&t, tile, sizeof(t));
	if (!t.nnz) return;
	orc_img *im = jb->im;
	uint64_t bh = im->h.block_2d_height, bw = im->h.block_2d_width;
	size_t es = dsize(jb->dtype), esize = im->esize;
	int prim = im->h.data_type;
	const char *in_rows = (const char *)jb->X + (uint64_t)t.bcol * bw * jb->k * es;
	char *out = out_rows + ((uint64_t)t.brow * bh - out_row0) * jb->k * es;
	const char *vals = tile + sizeof(orc_tile) + (size_t)t.nrow * 2 + (size_t)t.nnz * 2 + 2;
	/* row parts (row_part_func, :229-246) */
	const char *rpp = tile + sizeof(orc_tile);
	const char *rend = rpp + tile_rheader(&t) - 2;
	uint64_t vi = 0;
	while (rpp < rend) {
		uint16_t row = rd16(rpp) & 0x7FFF; rpp += 2;
		char *dest = out + (uint64_t)row * jb->k * es;
		while (rd16(rpp) <= 0x7FFF) {
			uint16_t col = rd16(rpp); rpp += 2;
			axpy_row(jb->dtype, dest, in_rows + (uint64_t)col * jb->k * es, jb->k,
					vals + vi * esize, prim, esize);
			vi++;
		}
	}
	/* COO singletons (coo_func, :288-303) */
	const char *coo = tile + sizeof(orc_tile) + tile_rheader(&t);
	const char *coov = vals + (size_t)(t.nnz - t.ncoo) * esize;
	for (uint32_t i = 0; i < t.ncoo; i++) {
		uint16_t row = rd16(coo + 4 * i) & 0x7FFF, col = rd16(coo + 4 * i + 2);
		axpy_row(jb->dtype, out + (uint64_t)row * jb->k * es,
				in_rows + (uint64_t)col * jb->k * es, jb->k, coov + i * esize, prim, esize);
	}
}

/* block_compute_task::run (sparse_matrix.cpp:251-314) over block rows
 * [b0, b1), followed by notify_complete (:354-393): out_part zeroed, filled,
 * then copied into Y. */
static void orc_task(orc_job *jb, uint64_t b0, uint64_t b1, char **bufp, size_t *bufcap,
		char **outp, size_t *outcap)
{
	orc_img *im = jb->im;
	uint64_t bh = im->h.block_2d_height, bw = im->h.block_2d_width;
	size_t es = dsize(jb->dtype);
	const char *base = im->mat + im->offs[b0];
	size_t len = (size_t)(im->offs[b1] - im->offs[b0]);
	if (jb->copy_task) {
		if (*bufcap < len) { free(*bufp); *bufp = malloc(len); *bufcap = len; }
		memcpy(*bufp, base, len);
		base = *bufp;
	}
	uint64_t row0 = b0 * bh;
	uint64_t nr = b1 * bh < im->h.nrows ? (b1 - b0) * bh : im->h.nrows - row0;
	size_t olen = nr * jb->k * es;
	if (*outcap < olen) { free(*outp); *outp = malloc(olen ? olen : 1); *outcap = olen; }
	memset(*outp, 0, olen);
	uint64_t nb = b1 - b0;
	const char **it = malloc(sizeof(char *) * (nb + 1));
	for (uint64_t i = 0; i <= nb; i++) it[i] = base + (im->offs[b0 + i] - im->offs[b0]);
	const char **cur = malloc(sizeof(char *) * nb);
	for (uint64_t i = 0; i < nb; i++) cur[i] = it[i];
	const char **blocks = malloc(sizeof(char *) * nb * nb);
	int use_h = jb->hilbert && nb == jb->sb;
	uint64_t sbc = 0;
	int has;
	do {
		has = 0;
		for (uint64_t i = 0; i < nb; i++) {
			for (uint64_t j = 0; j < nb; j++) {
				blocks[i * nb + j] = NULL;
				if (cur[i] >= it[i + 1]) continue;
				orc_tile t; memcpy(&t, cur[i], sizeof(t));
				if (t.bcol == sbc + j) {
					blocks[i * nb + j] = cur[i];
					cur[i] += tile_size(&t, im->esize);
				}
			}
			has |= cur[i] < it[i + 1];
		}
		sbc += nb;
		if (use_h) {
			for (uint64_t q = 0; q < nb * nb; q++)
				if (blocks[jb->horder[q]]) orc_run_on_block(jb, blocks[jb->horder[q]], *outp, row0);
		} else {
			for (uint64_t q = 0; q < nb * nb; q++)
				if (blocks[q]) orc_run_on_block(jb, blocks[q], *outp, row0);
		}
	} while (has);
	memcpy((char *)jb->Y + row0 * jb->k * es, *outp, olen);
	(void)bw;
	free(blocks); free(cur); free(it);
}

/* b2d_io_generator::get_next_io (matrix_io.cpp:212-236) */
static int orc_next(orc_job *jb, uint64_t *b0, uint64_t *b1)
{
	int ok = 0;
	pthread_mutex_lock(&jb->lock);
	if (jb->next_brow < jb->brow_end) {
		uint64_t n = jb->next_brow >= jb->balance_point ? 1 : jb->sb;
		uint64_t left = jb->brow_end - jb->next_brow;
		if (n > left) n = left;
		*b0 = jb->next_brow; *b1 = jb->next_brow + n;
		jb->next_brow += n;
		ok = 1;
	}
	pthread_mutex_unlock(&jb->lock);
	return ok;
}

static void *orc_worker(void *arg)
{
	orc_job *jb = arg;
	char *buf = NULL, *out = NULL; size_t bc = 0, oc = 0;
	uint64_t b0, b1;
	while (orc_next(jb, &b0, &b1)) orc_task(jb, b0, b1, &buf, &bc, &out, &oc);
	free(buf); free(out);
	return NULL;
}

/* cal_super_block_size (sparse_matrix.h:450-463) with k rounded down to a
 * power of two (spmm_creator ctor, :668-671). */
static uint64_t orc_sb_size(uint64_t bh, uint64_t k, size_t es, uint64_t cache_size)
{
	uint64_t k2 = 1; while (k2 * 2 <= k) k2 *= 2;
	uint64_t size = cache_size / (es * k2) / bh / 2;
	if (size < 1) size = 1;
	uint64_t mx = 16 * 1024 / bh; if (mx < 1) mx = 1;
	return size < mx ? size : mx;
}

/*
 * orc_spmm: Y = A * X over block rows [brow_begin, brow_end) (all when
 * brow_end == 0) of the image, with `nthreads` workers pulling block-row
 * ranges (sparse_matrix::compute, sparse_matrix.cpp:431-473).
 * cpu_cache_size 0 -> 1 MiB (matrix_config.h:87).  Returns 0 or -1.
 */
int orc_spmm(const char *idx, size_t idx_len, const char *mat, size_t mat_len,
		int dtype, const void *X, void *Y, uint64_t k, int nthreads, int hilbert,
		uint64_t cpu_cache_size, int copy_task, uint64_t brow_begin, uint64_t brow_end)
{
	orc_img im;
	if (orc_open(idx, idx_len, mat, mat_len, &im)) return -1;
	if (dtype != D_F32 && dtype != D_F64 && dtype != D_I32 && dtype != D_I64) { orc_close(&im); return -1; }
	orc_job jb;
	memset(&jb, 0, sizeof(jb));
	jb.im = &im; jb.dtype = dtype; jb.X = X; jb.Y = Y; jb.k = k;
	jb.sb = orc_sb_size(im.h.block_2d_height, k, dsize(dtype), cpu_cache_size ? cpu_cache_size : (1 << 20));
	jb.hilbert = hilbert;
	if (hilbert) {
		/* hilbert_exec_order ctor (sparse_matrix.cpp:144-159): sort (i,j) by d */
		uint64_t n = jb.sb;
		jb.horder = malloc(sizeof(int) * n * n);
		int *d = malloc(sizeof(int) * n * n);
		for (uint64_t i = 0; i < n * n; i++) { jb.horder[i] = (int)i; d[i] = orc_hilbert_xy2d((int)n, (int)(i / n), (int)(i % n)); }
		for (uint64_t a = 1; a < n * n; a++) {   /* insertion sort, n is small */
			int v = jb.horder[a]; uint64_t b = a;
			while (b > 0 && d[jb.horder[b - 1]] > d[v]) { jb.horder[b] = jb.horder[b - 1]; b--; }
			jb.horder[b] = v;
		}
		free(d);
	}
	jb.copy_task = copy_task;
	jb.brow_begin = brow_begin;
	jb.brow_end = brow_end ? brow_end : im.nbrows;
	if (jb.brow_end > im.nbrows || jb.brow_begin > jb.brow_end) { free(jb.horder); orc_close(&im); return -1; }
	jb.next_brow = jb.brow_begin;
	if (nthreads < 1) nthreads = 1;
	/* balance point (matrix_io.cpp:195-205); min_num_brows = 1 */
	uint64_t nbr = jb.brow_end - jb.brow_begin;
	if (jb.sb > 1)
		jb.balance_point = nbr > jb.sb * (uint64_t)nthreads ? jb.brow_end - (uint64_t)nthreads : jb.brow_begin;
	else
		jb.balance_point = jb.brow_end;
	pthread_mutex_init(&jb.lock, NULL);
	if (nthreads == 1) orc_worker(&jb);
	else {
		pthread_t *th = malloc(sizeof(pthread_t) * nthreads);
		for (int i = 0; i < nthreads; i++) pthread_create(&th[i], NULL, orc_worker, &jb);
		for (int i = 0; i < nthreads; i++) pthread_join(th[i], NULL);
		free(th);
	}
	pthread_mutex_destroy(&jb.lock);
	free(jb.horder);
	orc_close(&im);
	return 0;
}

/* Number of block rows of an image (for sampled timing). */
int64_t orc_num_block_rows(const char *idx, size_t idx_len)
{
	orc_header h;
	if (idx_len < ORC_PAGE) return -1;
	memcpy(&h, idx, sizeof(h));
	if (h.magic_number != ORC_MAGIC || !h.block_2d_height) return -1;
	return (int64_t)((h.nrows + h.block_2d_height - 1) / h.block_2d_height);
}

/* Non-zeros stored in block rows [b0, b1) (the sample size of a timed run). */
int64_t orc_block_rows_nnz(const char *idx, size_t idx_len, const char *mat, size_t mat_len,
		uint64_t b0, uint64_t b1)
{
	orc_img im;
	if (orc_open(idx, idx_len, mat, mat_len, &im)) return -1;
	int64_t n = 0;
	for (uint64_t b = b0; b < b1 && b < im.nbrows; b++) {
		const char *p = im.mat + im.offs[b], *end = im.mat + im.offs[b + 1];
		while (p < end) {
			orc_tile t; memcpy(&t, p, sizeof(t));
			n += t.nnz;
			p += tile_size(&t, im.esize);
		}
	}
	orc_close(&im);
	return n;
}

/* ===================================================================== */
/* Tile verification (sparse_block_2d::verify, sparse_matrix_format.cpp:36-60;
 * SpM_2d_storage::verify, :371-415).  Returns 0 when valid, else a negative
 * code naming the first failed check.                                    */
/* ===================================================================== */
int orc_verify(const char *idx, size_t idx_len, const char *mat, size_t mat_len)
{
	orc_img im;
	if (orc_open(idx, idx_len, mat, mat_len, &im)) return -1;
	uint64_t bh = im.h.block_2d_height, bw = im.h.block_2d_width;
	for (uint64_t b = 0; b < im.nbrows; b++) {
		if (im.offs[b] >= im.offs[b + 1]) { orc_close(&im); return -2; }
		const char *p = im.mat + im.offs[b], *end = im.mat + im.offs[b + 1];
		size_t tot = 0;
		long prev_col = -1;
		while (p < end) {
			orc_tile t; memcpy(&t, p, sizeof(t));
			size_t sz = tile_size(&t, im.esize);
			if (t.brow != b) { orc_close(&im); return -3; }
			if (t.nnz) {
				if ((long)t.bcol <= prev_col) { orc_close(&im); return -4; }
				prev_col = t.bcol;
				if (p + sz > end) { orc_close(&im); return -5; }
				uint64_t rows = 0; long prev_row = -1;
				const char *rpp = p + sizeof(orc_tile);
				const char *rend = rpp + tile_rheader(&t) - 2;
				while (rpp < rend) {
					uint16_t hw = rd16(rpp);
					if (!(hw & 0x8000)) { orc_close(&im); return -6; }
					long row = hw & 0x7FFF; rpp += 2;
					uint64_t nz = 0;
					while (rpp < rend && rd16(rpp) <= 0x7FFF) { nz++; rpp += 2; }
					if (nz > bw) { orc_close(&im); return -7; }
					if (row > 0 && prev_row >= row) { orc_close(&im); return -8; }
					prev_row = row; rows++;
				}
				if (rd16(rend) != 0xFFFF) { orc_close(&im); return -9; }
				rows += t.ncoo;
				if (rows > bh || rows != t.nrow) { orc_close(&im); return -10; }
			}
			if (!t.nnz && p + sz > end) sz = (size_t)(end - p); /* 16-byte empty block row */
			tot += sz;
			p += sz;
		}
		if (tot != (size_t)(im.offs[b + 1] - im.offs[b])) { orc_close(&im); return -11; }
	}
	orc_close(&im);
	return 0;
}

/* ===================================================================== */
/* PageRank (matrix/libmatrix-algs/PageRank.cpp:31-133) on an image of A  */
/* (out-edges; rows = sources).  `t_idx`/`t_mat` is the image of A^T,     */
/* which the reference multiplies (mat->transpose(), :92).                */
/* ===================================================================== */
int orc_pagerank(const char *idx, size_t idx_len, const char *mat, size_t mat_len,
		const char *t_idx, size_t t_idx_len, const char *t_mat, size_t t_mat_len,
		uint64_t max_iters, float damping, int nthreads, float *pr_out, uint64_t *iters_out)
{
	orc_img im;
	if (orc_open(idx, idx_len, mat, mat_len, &im)) return -1;
	uint64_t n = im.h.nrows;
	orc_close(&im);
	/* out-degree = A * 1 (get_out_degree, :49-59), clamped to >= 1 (:75) */
	float *one = malloc(sizeof(float) * n), *deg = malloc(sizeof(float) * n);
	float *pr = malloc(sizeof(float) * n), *in = malloc(sizeof(float) * n), *out = malloc(sizeof(float) * n);
	for (uint64_t i = 0; i < n; i++) one[i] = 1.0f;
	if (orc_spmm(idx, idx_len, mat, mat_len, D_F32, one, deg, 1, nthreads, 0, 0, 0, 0, 0)) return -1;
	/* pr = 1.0 / num_vertices in double, stored as float (mat_init_operate, :31-47) */
	const float p0 = (float)(1.0 / (double)n);
	for (uint64_t i = 0; i < n; i++) { if (deg[i] < 1.0f) deg[i] = 1.0f; pr[i] = p0; }
	const float eps = (float)(0.001 / (double)n);          /* :94 */
	const float teleport = (float)((1.0 - (double)damping) / (double)n); /* :117 */
	uint64_t converge = 0, it = 0;
	while (converge < n && it < max_iters) {
		for (uint64_t i = 0; i < n; i++) in[i] = pr[i] / deg[i];
		for (uint64_t i = 0; i < n; i++) pr[i] = in[i] * deg[i];  /* pr1 = in * deg (:104) */
		if (orc_spmm(t_idx, t_idx_len, t_mat, t_mat_len, D_F32, in, out, 1, nthreads, 0, 0, 0, 0, 0)) return -1;
		converge = 0;
		for (uint64_t i = 0; i < n; i++) {
			float p2 = out[i] * damping + teleport;
			float d = pr[i] - p2; if (d < 0) d = -d;
			if (d < eps) converge++;
			pr[i] = p2;
		}
		it++;
	}
	memcpy(pr_out, pr, sizeof(float) * n);
	*iters_out = it;
	free(one); free(deg); free(pr); free(in); free(out);
	return 0;
}

double orc_now(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return ts.tv_sec + ts.tv_nsec * 1e-9;
}

/* ------------------------------------------------------------------------
 * The synthetic R-MAT workload (test infrastructure)
 *
 * The benchmark graphs are R-MAT graphs with FlashX's quadrant probabilities
 * (flash-graph/tools/rmat-gen.cpp:43-44).  The reference draws them with
 * Boost.Graph's rmat_iterator, which is not in the tree; both arms of the
 * benchmark instead use one counter-based stream: edge e depends only on
 * (seed, e).  This is a second implementation of that stream, so that the
 * CPU arm never loads the GPU library; tests/test_oracle_pin.py checks that
 * it yields the same edges as the library's generator.
 *   per edge: h0 = mix(key ^ e * 0xD6E8FEB86659FD93); for each of the
 *   `scale` levels one 32-bit draw u (two per mix of h0 + l * golden), row
 *   bit = u >= a + b, column bit = a <= u < a + b or u >= a + b + c (both
 *   as fractions of 2^32), most significant bit first; then, with permute,
 *   both ids go through a seeded bijection of [0, 2^scale): four rounds of
 *   x = (x * odd + add) mod 2^scale, x ^= x >> (scale / 2 + 1).
 * ------------------------------------------------------------------------ */
static uint64_t orc_mix64(uint64_t z)
{
	/* splitmix64's finaliser (Steele, Lea and Flood, 2014) */
	z += 0x9E3779B97F4A7C15ULL;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
	return z ^ (z >> 31);
}

typedef struct {
	uint64_t key;
	uint32_t ta, tab, tabc;
	int scale, permute;
	uint64_t mul[4], add[4];
	uint32_t *src, *dst;
	uint64_t e0, e1;
} orc_rmat_job;

static uint32_t orc_rmat_relabel(const orc_rmat_job *p, uint32_t v)
{
	const uint64_t mask = (1ULL << p->scale) - 1;
	const int sh = p->scale / 2 + 1;
	uint64_t x = v;
	for (int r = 0; r < 4; r++) {
		x = (x * p->mul[r] + p->add[r]) & mask;
		x ^= x >> sh;
	}
	return (uint32_t)x;
}

static void *orc_rmat_worker(void *arg)
{
	orc_rmat_job *p = arg;
	for (uint64_t e = p->e0; e < p->e1; e++) {
		const uint64_t h0 = orc_mix64(p->key ^ (e * 0xD6E8FEB86659FD93ULL));
		uint32_t r = 0, c = 0;
		uint64_t h = 0;
		for (int l = 0; l < p->scale; l++) {
			if ((l & 1) == 0) h = orc_mix64(h0 + (uint64_t)l * 0x9E3779B97F4A7C15ULL);
			const uint32_t u = (l & 1) ? (uint32_t)(h >> 32) : (uint32_t)h;
			r = (r << 1) | (uint32_t)(u >= p->tab);
			c = (c << 1) | (uint32_t)((u >= p->ta && u < p->tab) || u >= p->tabc);
		}
		if (p->permute) { r = orc_rmat_relabel(p, r); c = orc_rmat_relabel(p, c); }
		p->src[e] = r;
		p->dst[e] = c;
	}
	return NULL;
}

/* nedges R-MAT edges of 2^scale vertices into src/dst.  Returns 0 or -1. */
int orc_rmat_edges(int scale, uint64_t nedges, double a, double b, double c, uint64_t seed, int permute,
		uint32_t *src, uint32_t *dst, int nthreads)
{
	if (scale < 1 || scale > 31 || !(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0)) return -1;
	orc_rmat_job p;
	memset(&p, 0, sizeof(p));
	#define ORC_TH(x) ((x) * 4294967296.0 >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)((x) * 4294967296.0))
	p.key = orc_mix64(seed ^ 0x5851F42D4C957F2DULL);
	p.ta = ORC_TH(a); p.tab = ORC_TH(a + b); p.tabc = ORC_TH(a + b + c);
	#undef ORC_TH
	p.scale = scale; p.permute = permute;
	uint64_t s = orc_mix64(seed + 0x1234567ULL);
	for (int r = 0; r < 4; r++) {
		s = orc_mix64(s); p.mul[r] = s | 1ULL;
		s = orc_mix64(s); p.add[r] = s;
	}
	p.src = src; p.dst = dst;
	if (nthreads < 1) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
	if (nthreads > 256) nthreads = 256;
	if (nthreads < 1) nthreads = 1;
	orc_rmat_job jobs[256];
	pthread_t th[256];
	for (int t = 0; t < nthreads; t++) {
		jobs[t] = p;
		jobs[t].e0 = nedges * (uint64_t)t / (uint64_t)nthreads;
		jobs[t].e1 = nedges * (uint64_t)(t + 1) / (uint64_t)nthreads;
		if (t) pthread_create(&th[t], NULL, orc_rmat_worker, &jobs[t]);
	}
	orc_rmat_worker(&jobs[0]);
	for (int t = 1; t < nthreads; t++) pthread_join(th[t], NULL);
	return 0;
}

/* ------------------------------------------------------------------------
 * The FlashGraph 1D format (test infrastructure: writer and row SpMM)
 *
 * File: graph_header, one 4096-byte page (graph_file_header.h:27-37,43:
 * int64 magic 0x123456789ABCDEF, int version 4, int type (DIRECTED 0,
 * UNDIRECTED 1, TS_DIRECTED 2, TS_UNDIRECTED 3), size_t num_vertices,
 * size_t num_edges, int edge_data_size, int max_num_timestamps).  Then one
 * record per vertex, ids 0..n-1 in order (ext_mem_undirected_vertex,
 * vertex.h:444-562): u32 id, u32 edge_data_size, u32 num_edges, u32
 * neighbors[num_edges]; with edge data, the data array starts at
 * ROUNDUP(12 + 4 num_edges, edge_data_size) and the record ends at
 * ROUNDUP(that + num_edges * edge_data_size, 4), ROUNDUP(off, base) =
 * (off + base - 1) & ~(base - 1) (libsafs/common_c.h:36).  A directed graph
 * stores every vertex's in-edge record, then every out-edge record
 * (mem_directed_graph::dump_graph, utils.cpp:399-420); an undirected graph
 * one record per vertex.  Row i of the matrix is vertex i's out-edge record
 * (the in-edge record for the transpose), fg_sparse_matrix.cpp:473-575.
 * ------------------------------------------------------------------------ */
#define ORC_FG_MAGIC 0x123456789ABCDEFLL
#define ORC_FG_VERSION 4

typedef struct {
	int64_t magic;
	int32_t version, type;
	uint64_t num_vertices, num_edges;
	int32_t edge_data_size, max_num_timestamps;
} orc_fg_header;

static uint64_t orc_roundup(uint64_t off, uint64_t base) { return (off + base - 1) & ~(base - 1); }

/* Byte offset of the edge data and total size of a record (vertex.h:458-528). */
uint64_t orc_fg_data_off(uint32_t ne, uint32_t eds) { return eds ? orc_roundup(12 + 4ull * ne, eds) : 12 + 4ull * ne; }
uint64_t orc_fg_vsize(uint32_t ne, uint32_t eds)
{
	return eds ? orc_roundup(orc_fg_data_off(ne, eds) + (uint64_t)ne * eds, 4) : 12 + 4ull * ne;
}

typedef struct { uint32_t v, nbr; uint64_t pos; } orc_fg_edge;
static int cmp_fg_edge(const void *a, const void *b)
{
	const orc_fg_edge *x = a, *y = b;
	if (x->v != y->v) return x->v < y->v ? -1 : 1;
	if (x->nbr != y->nbr) return x->nbr < y->nbr ? -1 : 1;
	return x->pos < y->pos ? -1 : (x->pos > y->pos);
}

static uint64_t orc_fg_put_part(char *out, const orc_fg_edge *e, uint64_t ne, uint64_t nv, const char *vals,
		uint32_t eds)
{
	uint64_t at = 0, i = 0;
	for (uint64_t v = 0; v < nv; v++) {
		uint64_t j = i;
		while (j < ne && e[j].v == v) j++;
		const uint32_t cnt = (uint32_t)(j - i);
		char *r = out ? out + at : NULL;
		if (r) {
			uint32_t h[3] = {(uint32_t)v, eds, cnt};
			memcpy(r, h, 12);
			for (uint64_t q = i; q < j; q++) memcpy(r + 12 + 4 * (q - i), &e[q].nbr, 4);
			if (eds)
				for (uint64_t q = i; q < j; q++)
					memcpy(r + orc_fg_data_off(cnt, eds) + (q - i) * eds, vals + e[q].pos * eds, eds);
		}
		at += orc_fg_vsize(cnt, eds);
		i = j;
	}
	return at;
}

/*
 * An FlashGraph adjacency image of the edge list: every neighbor list sorted
 * by id (input order among equal ids), duplicates and self-loops kept, edge
 * data of `eds` bytes per edge (vals) or none.  *out is malloc'ed (free with
 * orc_free).  Returns 0 or -1.
 */
int orc_fg_build(const uint32_t *src, const uint32_t *dst, const void *vals, uint32_t eds, uint64_t nedges,
		uint64_t nv, int directed, char **out, uint64_t *out_len)
{
	if (eds && !vals) return -1;
	for (uint64_t i = 0; i < nedges; i++)
		if (src[i] >= nv || dst[i] >= nv) return -1;
	/* undirected: the caller lists both directions (as fg's edge lists do) */
	orc_fg_edge *eo = malloc(sizeof(orc_fg_edge) * (nedges ? nedges : 1));
	orc_fg_edge *ei = directed ? malloc(sizeof(orc_fg_edge) * (nedges ? nedges : 1)) : NULL;
	for (uint64_t i = 0; i < nedges; i++) {
		eo[i].v = src[i]; eo[i].nbr = dst[i]; eo[i].pos = i;
		if (ei) { ei[i].v = dst[i]; ei[i].nbr = src[i]; ei[i].pos = i; }
	}
	qsort(eo, nedges, sizeof(orc_fg_edge), cmp_fg_edge);
	if (ei) qsort(ei, nedges, sizeof(orc_fg_edge), cmp_fg_edge);
	uint64_t len = ORC_PAGE + orc_fg_put_part(NULL, eo, nedges, nv, vals, eds);
	if (ei) len += orc_fg_put_part(NULL, ei, nedges, nv, vals, eds);
	char *b = calloc(1, len);
	orc_fg_header h;
	memset(&h, 0, sizeof(h));
	h.magic = ORC_FG_MAGIC; h.version = ORC_FG_VERSION; h.type = directed ? 0 : 1;
	h.num_vertices = nv; h.num_edges = directed ? nedges : nedges / 2; h.edge_data_size = (int32_t)eds;
	memcpy(b, &h, sizeof(h));
	uint64_t at = ORC_PAGE;
	if (ei) at += orc_fg_put_part(b + at, ei, nedges, nv, vals, eds);
	orc_fg_put_part(b + at, eo, nedges, nv, vals, eds);
	free(eo); free(ei);
	*out = b; *out_len = len;
	return 0;
}

/*
 * Y = A X (or A^T X with transpose) over an FlashGraph adjacency image,
 * fg_row_spmm_task::run_on_row (fg_sparse_matrix.cpp:83-106): per vertex
 * record, res = 0, then res[j] += X[neighbor][j] * data in record order
 * (data = 1 without edge data), then Y[id] = res.  `prim` names the edge
 * data's type (P_BOOL without data).  Returns 0 or -1.
 */
int orc_fg_spmm(const char *adj, uint64_t len, int transpose, int prim, int dtype, const void *X, void *Y,
		uint64_t k)
{
	orc_fg_header h;
	if (len < ORC_PAGE) return -1;
	memcpy(&h, adj, sizeof(h));
	if (h.magic != ORC_FG_MAGIC || h.version != ORC_FG_VERSION || (h.type != 0 && h.type != 1)) return -1;
	const uint64_t nv = h.num_vertices;
	const uint32_t eds = (uint32_t)h.edge_data_size;
	const size_t ds = dsize(dtype);
	uint64_t at = ORC_PAGE;
	/* a directed graph's in-edge records come first */
	const int want_in = h.type == 0 && transpose;
	for (int part = 0; part < (h.type == 0 ? 2 : 1); part++) {
		const int use = h.type == 0 ? (part == 0) == want_in : 1;
		for (uint64_t v = 0; v < nv; v++) {
			uint32_t r[3];
			if (at + 12 > len) return -1;
			memcpy(r, adj + at, 12);
			if (r[0] != v || r[1] != eds) return -1;
			const uint64_t sz = orc_fg_vsize(r[2], eds);
			if (at + sz > len) return -1;
			if (use) {
				char *y = (char *)Y + v * k * ds;
				memset(y, 0, k * ds);
				for (uint32_t i = 0; i < r[2]; i++) {
					uint32_t c;
					memcpy(&c, adj + at + 12 + 4ull * i, 4);
					if (c >= nv) return -1;
					axpy_row(dtype, y, (const char *)X + (uint64_t)c * k * ds, k,
							eds ? adj + at + orc_fg_data_off(r[2], eds) + (uint64_t)i * eds : NULL, prim, eds);
				}
			}
			at += sz;
		}
	}
	return 0;
}
