/* Stub for building FlashGraph's flash-graph/vertex.h without SAFS (oracle
 * test code).  Declares the page_byte_array members that vertex.h's inline
 * code names; nothing here is defined or called.  ROUNDUP and the other
 * helpers come from the reference's own libsafs/common_c.h. */
#ifndef FMX_ORACLE_STUB_CACHE_H
#define FMX_ORACLE_STUB_CACHE_H
#include <iostream>
#include <string.h>
#include <stddef.h>
#include <sys/types.h>
#include "common_c.h"
#define BOOST_VERIFY(x) ((void)(x))
#define BOOST_LOG_TRIVIAL(level) std::cerr
namespace safs {
class page_byte_array {
public:
	template<class T> class const_iterator {
	public:
		const_iterator &operator+=(size_t);
		const_iterator &operator++();
		T operator*() const;
		bool operator==(const const_iterator &) const;
		bool operator!=(const const_iterator &) const;
		long operator-(const const_iterator &) const;
	};
	template<class T> class seq_const_iterator {
	public:
		bool has_next() const;
		T next();
		T curr() const;
	};
	size_t get_size() const;
	void memcpy(off_t rel_off, char *buf, size_t size) const;
	template<class T> T get(off_t off) const;
	template<class T> const_iterator<T> begin(off_t off = 0) const;
	template<class T> const_iterator<T> end() const;
	template<class T> seq_const_iterator<T> get_seq_iterator(off_t start, off_t end) const;
};
}
#endif
