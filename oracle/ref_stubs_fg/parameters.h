/* Stub: flash-graph/graph_file_header.h includes libsafs/parameters.h and
 * uses none of its names (oracle test code). */
#ifndef FMX_ORACLE_STUB_PARAMETERS_H
#define FMX_ORACLE_STUB_PARAMETERS_H
#endif
