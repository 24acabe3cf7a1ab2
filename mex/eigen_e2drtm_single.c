/* eigen_e2drtm_single MEX (core/e2drtm_eigen.m:122) on libswd.so. */
#define SWD_T float
#define SWD_CLASS mxSINGLE_CLASS
#define SWD_IN swd_in_single
#define SWD_IV swd_iv_single
#define SWD_RTM swd_e2drtm_single
#define SWD_NAME "eigen_e2drtm_single"
#include "e2drtm_shim.h"
