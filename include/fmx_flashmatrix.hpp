/*
 * fmx_flashmatrix.hpp -- the binding a FlashMatrix maintainer adds to route
 * fm::sparse_matrix::multiply to the B200 library (header-only C++ over the
 * C ABI of fmx.h).
 *
 * Include it inside FlashMatrix after its own headers: it uses
 * fm::detail::matrix_store / mem_matrix_store (matrix/matrix_store.h,
 * matrix/mem_matrix_store.h), fm::get_scalar_type (matrix/generic_type.h),
 * fm::matrix_layout_t and BOOST_LOG_TRIVIAL, exactly as
 * matrix/sparse_matrix.cpp does.
 *
 * fm::gpu_sparse_matrix mirrors the part of fm::sparse_matrix
 * (matrix/sparse_matrix.h:475-651) that the SpMM path uses:
 *   load(idx, mat[, t_idx, t_mat])  the same .mat_idx / .mat files that
 *                                   SpM_2d_index::load, SpM_2d_storage::load
 *                                   and sparse_matrix::create read
 *                                   (sparse_matrix.cpp:679-707)
 *   get_num_rows / get_num_cols / get_nnz / is_symmetric / transpose
 *   multiply(in, out) -> bool       sparse_matrix::multiply
 *                                   (sparse_matrix.cpp:709-771): the same
 *                                   type and dimension checks, false plus a
 *                                   log line on failure, out overwritten.
 * The dense stores stay in host memory (mem_matrix_store::get_raw_arr,
 * matrix/mem_matrix_store.h:116-119); multiply stages them through the GPU
 * with fmx_spmm_host.  Inputs must be in-memory and row-major (the reference
 * converts other inputs with dense_matrix::conv2(L_ROW) first,
 * sparse_matrix.cpp:721-724; this binding asks the caller to do so).
 */
#ifndef FMX_FLASHMATRIX_HPP
#define FMX_FLASHMATRIX_HPP

#include <memory>
#include <string>

#include "fmx.h"

namespace fm
{

class gpu_sparse_matrix
{
	fmx_matrix *m = nullptr;
	size_t nrows = 0, ncols = 0, nnz = 0;
	int prim = FMX_P_BOOL;
	bool symmetric = true;

	static bool failed(int rc)
	{
		if (rc == FMX_OK) return false;
		BOOST_LOG_TRIVIAL(error) << fmx_last_error();
		return true;
	}
	void read_info()
	{
		uint64_t r = 0, c = 0, z = 0;
		int sym = 1;
		fmx_matrix_info(m, &r, &c, &z, &prim, &sym);
		nrows = r; ncols = c; nnz = z;
		symmetric = sym != 0;
	}
	static int dense_code(const scalar_type &t)
	{
		if (t == get_scalar_type<float>()) return FMX_F32;
		if (t == get_scalar_type<double>()) return FMX_F64;
		if (t == get_scalar_type<int>()) return FMX_I32;
		if (t == get_scalar_type<long>()) return FMX_I64;
		return -1;
	}
	static int prim_code(const scalar_type &t)
	{
		if (t == get_scalar_type<float>()) return FMX_P_FLOAT;
		if (t == get_scalar_type<double>()) return FMX_P_DOUBLE;
		if (t == get_scalar_type<int>()) return FMX_P_INTEGER;
		if (t == get_scalar_type<long>()) return FMX_P_LONG;
		return -1;
	}

public:
	typedef std::shared_ptr<gpu_sparse_matrix> ptr;

	gpu_sparse_matrix() = default;
	gpu_sparse_matrix(const gpu_sparse_matrix &) = delete;
	gpu_sparse_matrix &operator=(const gpu_sparse_matrix &) = delete;
	~gpu_sparse_matrix() { fmx_matrix_free(m); }

	/* sparse_matrix::create(SpM_2d_index::load(idx), SpM_2d_storage::load(mat)
	 * [, t_index, t_storage]) with the matrix resident on `device`; null plus
	 * a log line on failure. */
	static ptr load(const std::string &idx_file, const std::string &mat_file, int device = 0)
	{
		return load(idx_file, mat_file, std::string(), std::string(), device);
	}
	static ptr load(const std::string &idx_file, const std::string &mat_file, const std::string &t_idx_file,
			const std::string &t_mat_file, int device = 0)
	{
		ptr g(new gpu_sparse_matrix());
		const bool t = !t_idx_file.empty() && !t_mat_file.empty();
		if (failed(fmx_matrix_load(idx_file.c_str(), mat_file.c_str(), t ? t_idx_file.c_str() : nullptr,
				t ? t_mat_file.c_str() : nullptr, device, &g->m)))
			return ptr();
		g->read_info();
		return g;
	}

	size_t get_num_rows() const { return nrows; }
	size_t get_num_cols() const { return ncols; }
	size_t get_nnz() const { return nnz; }
	bool is_symmetric() const { return symmetric; }

	/* sparse_matrix::transpose: a view of the same resident matrix. */
	ptr transpose() const
	{
		ptr g(new gpu_sparse_matrix());
		if (failed(fmx_matrix_transpose(m, &g->m))) return ptr();
		g->read_info();
		return g;
	}

	/* sparse_matrix::multiply(in, out): out = this * in. */
	bool multiply(detail::matrix_store::const_ptr in, detail::matrix_store::ptr out) const
	{
		if (in->get_type() != out->get_type()) {
			BOOST_LOG_TRIVIAL(error) << "input and output matrices need to have the same type";
			return false;
		}
		const int dt = dense_code(in->get_type());
		if (dt < 0) {
			BOOST_LOG_TRIVIAL(error) << "the dense type is not float, double, int or long";
			return false;
		}
		/* entries binary or of the dense type; float entries also with
		 * double operands (spmm_creator<double, float>) */
		if (prim != FMX_P_BOOL && prim != prim_code(in->get_type()) &&
				!(prim == FMX_P_FLOAT && dt == FMX_F64)) {
			BOOST_LOG_TRIVIAL(error) << "matrix element type doesn't match";
			return false;
		}
		if (in->get_num_rows() != ncols || in->get_num_cols() != out->get_num_cols() ||
				out->get_num_rows() != nrows) {
			BOOST_LOG_TRIVIAL(error) << "the input and output matrix have incompatible dimensions";
			return false;
		}
		if (!in->is_in_mem() || !out->is_in_mem() || in->store_layout() != matrix_layout_t::L_ROW ||
				out->store_layout() != matrix_layout_t::L_ROW) {
			BOOST_LOG_TRIVIAL(error) << "gpu_sparse_matrix::multiply needs in-memory row-major stores "
					"(convert with conv2(matrix_layout_t::L_ROW) first)";
			return false;
		}
		auto min = detail::mem_matrix_store::cast(in);
		auto mout = detail::mem_matrix_store::cast(out);
		const int64_t k = int64_t(in->get_num_cols());
		return !failed(fmx_spmm_host(m, dt, min->get_raw_arr(), k, dt, mout->get_raw_arr(), k, k));
	}

	/* The handle, for the other entry points of fmx.h (fmx_spmm on device
	 * buffers, fmx_eigen_solve, fmx_pagerank). */
	const fmx_matrix *handle() const { return m; }
};

}

#endif
