/* Stub: flash-graph/vertex.h includes libsafs/container.h, which needs
 * Boost; vertex.h uses none of its names (oracle test code). */
#ifndef FMX_ORACLE_STUB_CONTAINER_H
#define FMX_ORACLE_STUB_CONTAINER_H
#include <vector>
#endif
