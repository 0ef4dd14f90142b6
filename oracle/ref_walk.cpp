/*
 * ref_walk.cpp -- walks a 2D matrix image with FlashX's OWN tile classes.
 *
 * TEST INFRASTRUCTURE ONLY (the checker of the checker).  Built by
 * oracle/Makefile against the reference headers where they lie
 * (FlashX matrix/sparse_matrix_format.h, matrix/matrix_header.h,
 * matrix/generic_type.h) plus matrix/hilbert_curve.cpp, into oracle/_ref/.
 * Nothing from the reference is copied into this repository; the three SAFS
 * headers that sparse_matrix_format.h includes are replaced by the stubs in
 * oracle/ref_stubs/.
 *
 * The tile iteration below uses the reference's inline methods
 * (sparse_block_2d::get_first_edge_iterator / get_next_edge_iterator /
 * is_rparts_end / get_coo_start / get_coo_val_start, rp_edge_iterator,
 * block_row_iterator).  The per-entry arithmetic restates row_part_func and
 * coo_func (matrix/sparse_matrix.h:229-246,288-303), which live in a header
 * that cannot be compiled here.
 */
#include <stdint.h>
#include <string.h>
#include <vector>
#include "sparse_matrix_format.h"
#include "hilbert_curve.h"

using namespace fm;

namespace {

template<class T, class S>
void walk_block(const sparse_block_2d &block, const block_2d_size &bs, size_t esize,
		const T *X, T *out, size_t k)
{
	if (block.is_empty())
		return;
	const T *in_rows = X + block.get_block_col_idx() * bs.get_num_cols() * k;
	if (block.has_rparts()) {
		rp_edge_iterator it = block.get_first_edge_iterator(esize);
		while (!block.is_rparts_end(it)) {
			T *dest = out + k * it.get_rel_row_idx();
			while (it.has_next()) {
				S data = 1;
				if (esize)
					data = it.get_curr_data<S>();
				size_t col = it.next();
				const T *src = in_rows + k * col;
				for (size_t j = 0; j < k; j++)
					dest[j] += src[j] * data;
			}
			it = block.get_next_edge_iterator(it, esize);
		}
	}
	const local_coo_t *coos = block.get_coo_start();
	const S *vals = esize ? (const S *) block.get_coo_val_start(esize) : NULL;
	for (size_t i = 0; i < block.get_num_coo_vals(); i++) {
		S data = 1;
		if (vals)
			data = vals[i];
		const T *src = in_rows + k * coos[i].get_col_idx();
		T *dest = out + k * coos[i].get_row_idx();
		for (size_t j = 0; j < k; j++)
			dest[j] += src[j] * data;
	}
}

template<class T, class S>
int walk_all(const char *idx, const char *mat, const T *X, T *Y, size_t k)
{
	const matrix_header &h = *(const matrix_header *) idx;
	block_2d_size bs = h.get_2d_block_size();
	size_t esize = h.get_entry_size();
	size_t nbrows = bs.cal_num_block_rows(h.get_num_rows());
	const char *offp = idx + sizeof(matrix_header);
	for (size_t b = 0; b < nbrows; b++) {
		int64_t o0, o1;
		memcpy(&o0, offp + 8 * b, 8);
		memcpy(&o1, offp + 8 * (b + 1), 8);
		size_t r0 = b * bs.get_num_rows();
		size_t nr = std::min(bs.get_num_rows(), h.get_num_rows() - r0);
		std::vector<T> out(nr * k, 0);
		/* Copy the block row, as in_mem_io does, so tiles are read from a
		 * buffer of their own (libsafs/in_mem_io.cpp:500-501). */
		std::vector<char> buf(mat + o0, mat + o1);
		block_row_iterator it((const sparse_block_2d *) buf.data(),
				(const sparse_block_2d *) (buf.data() + buf.size()));
		while (it.has_next()) {
			const sparse_block_2d &blk = it.next(esize);
			walk_block<T, S>(blk, bs, esize, X, out.data() - 0, k);
		}
		memcpy(Y + r0 * k, out.data(), nr * k * sizeof(T));
	}
	return 0;
}

}

extern "C" {

int ref_sizeof_tile(void) { return (int) sizeof(sparse_block_2d); }
int ref_sizeof_header(void) { return (int) sizeof(matrix_header); }
int ref_sizeof_coo(void) { return (int) sizeof(local_coo_t); }
int ref_hilbert_xy2d(int n, int x, int y) { return hilbert_xy2d(n, x, y); }

/* Header fields through the reference's own accessors. */
int ref_header(const char *idx, uint64_t *nrows, uint64_t *ncols, uint64_t *entry_size,
		uint64_t *bh, uint64_t *bw, int *is_sparse, int *magic_ok, int *version_ok)
{
	const matrix_header &h = *(const matrix_header *) idx;
	*nrows = h.get_num_rows();
	*ncols = h.get_num_cols();
	*entry_size = h.get_entry_size();
	block_2d_size bs = h.get_2d_block_size();
	*bh = bs.get_num_rows();
	*bw = bs.get_num_cols();
	*is_sparse = h.is_sparse();
	*magic_ok = h.is_matrix_file();
	*version_ok = h.is_right_version();
	return 0;
}

/* dtype: 0 float, 1 double, 3 int32, 4 int64 (dense = sparse type, or a
 * binary matrix); 5 = double dense with float entries (spmm_creator<double,
 * float>, test-eigen.cpp:47). */
int ref_spmm(const char *idx, const char *mat, int dtype, const void *X, void *Y, uint64_t k)
{
	switch (dtype) {
	case 0: return walk_all<float, float>(idx, mat, (const float *) X, (float *) Y, k);
	case 1: return walk_all<double, double>(idx, mat, (const double *) X, (double *) Y, k);
	case 3: return walk_all<int, int>(idx, mat, (const int *) X, (int *) Y, k);
	case 4: return walk_all<long, long>(idx, mat, (const long *) X, (long *) Y, k);
	case 5: return walk_all<double, float>(idx, mat, (const double *) X, (double *) Y, k);
	}
	return -1;
}

/* sparse_block_2d::get_non_zeros order (sparse_matrix_format.cpp:62-88)
 * through the reference's iterators; returns the number of entries. */
int64_t ref_nonzeros(const char *idx, const char *mat, uint64_t *rows, uint64_t *cols,
		uint64_t cap)
{
	const matrix_header &h = *(const matrix_header *) idx;
	block_2d_size bs = h.get_2d_block_size();
	size_t esize = h.get_entry_size();
	size_t nbrows = bs.cal_num_block_rows(h.get_num_rows());
	const char *offp = idx + sizeof(matrix_header);
	uint64_t n = 0;
	for (size_t b = 0; b < nbrows; b++) {
		int64_t o0, o1;
		memcpy(&o0, offp + 8 * b, 8);
		memcpy(&o1, offp + 8 * (b + 1), 8);
		std::vector<char> buf(mat + o0, mat + o1);
		block_row_iterator it((const sparse_block_2d *) buf.data(),
				(const sparse_block_2d *) (buf.data() + buf.size()));
		while (it.has_next()) {
			const sparse_block_2d &blk = it.next(esize);
			if (blk.is_empty())
				continue;
			size_t r0 = blk.get_block_row_idx() * bs.get_num_rows();
			size_t c0 = blk.get_block_col_idx() * bs.get_num_cols();
			if (blk.has_rparts()) {
				rp_edge_iterator e = blk.get_first_edge_iterator();
				while (!blk.is_rparts_end(e)) {
					while (e.has_next()) {
						size_t row = e.get_rel_row_idx();
						size_t col = e.next();
						if (rows && n < cap) { rows[n] = r0 + row; cols[n] = c0 + col; }
						n++;
					}
					e = blk.get_next_edge_iterator(e);
				}
			}
			const local_coo_t *coo = blk.get_coo_start();
			for (size_t i = 0; i < blk.get_num_coo_vals(); i++) {
				if (rows && n < cap) {
					rows[n] = r0 + coo[i].get_row_idx();
					cols[n] = c0 + coo[i].get_col_idx();
				}
				n++;
			}
		}
	}
	return (int64_t) n;
}

}
