/* Stub: flash-graph/graph_file_header.h includes libsafs/common.h, which
 * needs Boost.Log; the header only needs the C helpers of common_c.h
 * (oracle test code). */
#ifndef FMX_ORACLE_STUB_COMMON_H
#define FMX_ORACLE_STUB_COMMON_H
#include <assert.h>
#include "common_c.h"
#endif
