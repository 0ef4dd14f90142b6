// Status strings and library identity for the C ABI (include/fmx.h).
#include "fmx_internal.h"

namespace fmx {
const char *last_error_str();
}

extern "C" {

const char *fmx_strerror(int status)
{
	switch (status) {
	case FMX_OK: return "ok";
	case FMX_ERR_INVAL: return "invalid argument";
	case FMX_ERR_DIM: return "incompatible dimensions";
	case FMX_ERR_TYPE: return "unsupported or mismatched type";
	case FMX_ERR_IMAGE: return "malformed matrix image";
	case FMX_ERR_OOM: return "out of memory";
	case FMX_ERR_CUDA: return "CUDA error";
	case FMX_ERR_IO: return "I/O error";
	case FMX_ERR_UNSUPPORTED: return "unsupported";
	}
	return "unknown status";
}

const char *fmx_last_error(void) { return fmx::last_error_str(); }

const char *fmx_version(void) { return "fmx 0.1 sm_100a"; }

}
