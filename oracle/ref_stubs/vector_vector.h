/* Stub: FlashX matrix/vector_vector.h; the tile header only forward-declares it. */
#ifndef FMX_ORACLE_STUB_VECTOR_VECTOR_H
#define FMX_ORACLE_STUB_VECTOR_VECTOR_H
namespace fm { class vector_vector; }
#endif
