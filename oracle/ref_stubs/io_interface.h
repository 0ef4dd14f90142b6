/* Stub: FlashX libsafs/io_interface.h is not needed by the tile structs. */
#ifndef FMX_ORACLE_STUB_IO_INTERFACE_H
#define FMX_ORACLE_STUB_IO_INTERFACE_H
#endif
