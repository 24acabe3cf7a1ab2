/* ADWDgrad_1 (core/ADWDgrad_1.m:1-81) on libswd.so. */
#define SWD_ADWD_NORM 0
#define SWD_NAME "ADWDgrad_1"
#include "adwdgrad_shim.h"
