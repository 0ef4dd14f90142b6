/*
 * Drives include/fmx_flashmatrix.hpp (the FlashMatrix-side binding) against
 * the stand-in stores of flashmatrix_standin.h.
 *
 *   shim_check <mat_idx> <mat> <k> <x.f32> <y.f32>
 *
 * Loads the image through fm::gpu_sparse_matrix::load; on failure exits 2
 * (the binding has logged the reason).  Otherwise checks that multiply
 * refuses mismatched types, dimensions and a column-major input (false plus
 * a log line, as sparse_matrix::multiply does), then multiplies the
 * row-major FP32 X of x.f32 (ncols x k) into Y, writes y.f32 and exits 0.
 */
#include "flashmatrix_standin.h"
#include "fmx_flashmatrix.hpp"

#include <cstdio>

using fm::detail::mem_matrix_store;
using fm::matrix_layout_t;

int main(int argc, char **argv)
{
	if (argc != 6) {
		std::fprintf(stderr, "usage: shim_check mat_idx mat k x.f32 y.f32\n");
		return 1;
	}
	const size_t k = std::strtoul(argv[3], nullptr, 10);
	fm::gpu_sparse_matrix::ptr m = fm::gpu_sparse_matrix::load(argv[1], argv[2]);
	if (!m) return 2;
	const size_t nr = m->get_num_rows(), nc = m->get_num_cols();
	auto f32 = [&](size_t r, size_t c, matrix_layout_t l) {
		return std::make_shared<mem_matrix_store>(r, c, fm::get_scalar_type<float>(), 4, l);
	};
	auto x = f32(nc, k, matrix_layout_t::L_ROW);
	FILE *fx = std::fopen(argv[4], "rb");
	if (!fx || std::fread(x->get_raw_arr(), 4, nc * k, fx) != nc * k) return 1;
	std::fclose(fx);
	int bad = 0;
	auto yd = std::make_shared<mem_matrix_store>(nr, k, fm::get_scalar_type<double>(), 8, matrix_layout_t::L_ROW);
	bad += m->multiply(x, yd);                                  // types differ
	bad += m->multiply(x, f32(nr + 1, k, matrix_layout_t::L_ROW)); // rows
	bad += m->multiply(f32(nc, k, matrix_layout_t::L_COL), f32(nr, k, matrix_layout_t::L_ROW));
	if (bad) {
		std::fprintf(stderr, "multiply accepted an invalid call\n");
		return 3;
	}
	auto y = f32(nr, k, matrix_layout_t::L_ROW);
	if (!m->multiply(x, y)) return 4;
	auto t = m->transpose();
	if (!t || t->get_num_rows() != nc) return 5;
	FILE *fy = std::fopen(argv[5], "wb");
	if (!fy || std::fwrite(y->get_raw_arr(), 4, nr * k, fy) != nr * k) return 1;
	std::fclose(fy);
	std::printf("ok %zu x %zu nnz %zu\n", nr, nc, m->get_nnz());
	return 0;
}
