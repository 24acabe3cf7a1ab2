/* eigen_e2drtm_double MEX (core/e2drtm_eigend.m:122) on libswd.so. */
#define SWD_T double
#define SWD_CLASS mxDOUBLE_CLASS
#define SWD_IN swd_in_double
#define SWD_IV swd_iv_double
#define SWD_RTM swd_e2drtm_double
#define SWD_NAME "eigen_e2drtm_double"
#include "e2drtm_shim.h"
