/* ADWDgrad_norm (core/ADWDgrad_norm.m:1-102) on libswd.so. */
#define SWD_ADWD_NORM 1
#define SWD_NAME "ADWDgrad_norm"
#include "adwdgrad_shim.h"
