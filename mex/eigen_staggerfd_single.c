/* eigen_staggerfd_single MEX (core/staggerfd_eigen.m:139) on libswd.so. */
#define SWD_T float
#define SWD_CLASS mxSINGLE_CLASS
#define SWD_IN swd_in_single
#define SWD_IV swd_iv_single
#define SWD_FD swd_staggerfd_single
#define SWD_NAME "eigen_staggerfd_single"
#include "staggerfd_shim.h"
