/*
 * Minimal stand-ins for the FlashMatrix declarations that
 * include/fmx_flashmatrix.hpp uses, with the reference's names and
 * signatures (matrix/generic_type.h:233-300 scalar_type and get_scalar_type,
 * matrix/matrix_store.h:141-208 matrix_store, matrix/mem_matrix_store.h:43-119
 * mem_matrix_store and its cast, matrix/matrix_header.h matrix_layout_t, and
 * Boost.Log's BOOST_LOG_TRIVIAL).  Test infrastructure: they let the binding
 * compile and run without the reference library, which cannot be built here.
 */
#ifndef FLASHMATRIX_STANDIN_H
#define FLASHMATRIX_STANDIN_H

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <memory>
#include <sstream>
#include <vector>

namespace fm
{

/* One log record per statement, written with its end of line when the
 * statement ends, as a Boost.Log trivial-logger record is. */
struct standin_log
{
	std::ostringstream s;
	explicit standin_log(const char *level) { s << "[" << level << "] "; }
	~standin_log() { std::cerr << s.str() << std::endl; }
	template<class T> standin_log &operator<<(const T &v) { s << v; return *this; }
};
#define BOOST_LOG_TRIVIAL(lvl) ::fm::standin_log(#lvl)

enum class matrix_layout_t { L_COL, L_ROW };

class scalar_type
{
	int code;
public:
	explicit scalar_type(int c): code(c) {}
	virtual ~scalar_type() = default;
	virtual bool operator==(const scalar_type &t) const { return code == t.code; }
	virtual bool operator!=(const scalar_type &t) const { return code != t.code; }
	int get_code() const { return code; }
};

template<class T> struct type_code;
template<> struct type_code<bool> { static const int v = 0; };
template<> struct type_code<int> { static const int v = 4; };
template<> struct type_code<long> { static const int v = 6; };
template<> struct type_code<float> { static const int v = 8; };
template<> struct type_code<double> { static const int v = 9; };

template<class T>
const scalar_type &get_scalar_type()
{
	static const scalar_type t(type_code<T>::v);
	return t;
}

namespace detail
{

class matrix_store
{
	size_t nrow, ncol;
	const scalar_type &type;
	bool in_mem;
public:
	typedef std::shared_ptr<matrix_store> ptr;
	typedef std::shared_ptr<const matrix_store> const_ptr;
	matrix_store(size_t r, size_t c, bool mem, const scalar_type &t): nrow(r), ncol(c), type(t), in_mem(mem) {}
	virtual ~matrix_store() = default;
	size_t get_num_rows() const { return nrow; }
	size_t get_num_cols() const { return ncol; }
	const scalar_type &get_type() const { return type; }
	bool is_in_mem() const { return in_mem; }
	virtual matrix_layout_t store_layout() const = 0;
};

class mem_matrix_store: public matrix_store
{
	std::vector<char> data;
	matrix_layout_t layout;
public:
	typedef std::shared_ptr<mem_matrix_store> ptr;
	typedef std::shared_ptr<const mem_matrix_store> const_ptr;
	mem_matrix_store(size_t r, size_t c, const scalar_type &t, size_t esize, matrix_layout_t l):
		matrix_store(r, c, true, t), data(r * c * esize), layout(l) {}
	matrix_layout_t store_layout() const override { return layout; }
	const char *get_raw_arr() const { return data.data(); }
	char *get_raw_arr() { return data.data(); }
	static ptr cast(matrix_store::ptr s) { return std::dynamic_pointer_cast<mem_matrix_store>(s); }
	static const_ptr cast(matrix_store::const_ptr s) { return std::dynamic_pointer_cast<const mem_matrix_store>(s); }
};

}

}

#endif
