/* Stub for building FlashX's matrix/sparse_matrix_format.h without SAFS.
 * Declares only the names that header mentions (oracle test code). */
#ifndef FMX_ORACLE_STUB_IN_MEM_IO_H
#define FMX_ORACLE_STUB_IN_MEM_IO_H
#include <memory>
#include <limits>
#include <vector>
#include <string>
#include <sys/types.h>
namespace safs {
class NUMA_buffer { public: typedef std::shared_ptr<NUMA_buffer> ptr; };
class file_io_factory { public: typedef std::shared_ptr<file_io_factory> shared_ptr; };
}
#endif
