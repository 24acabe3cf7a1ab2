/* eigen_staggerfd_double MEX (core/staggerfd_eigend.m:139) on libswd.so. */
#define SWD_T double
#define SWD_CLASS mxDOUBLE_CLASS
#define SWD_IN swd_in_double
#define SWD_IV swd_iv_double
#define SWD_FD swd_staggerfd_double
#define SWD_NAME "eigen_staggerfd_double"
#include "staggerfd_shim.h"
