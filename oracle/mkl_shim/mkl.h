/* Oracle infrastructure (test-only): umbrella header of the MKL stand-in. */
#ifndef LFTS_ORACLE_MKL_SHIM_H_
#define LFTS_ORACLE_MKL_SHIM_H_
#include "mkl_service.h"
#include "mkl_dfti.h"
#endif
