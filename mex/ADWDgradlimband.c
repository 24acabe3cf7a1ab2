/* ADWDgradlimband (core/ADWDgradlimband.m:1-102) on libswd.so. */
#define SWD_ADWD_NORM 0
#define SWD_ADWD_LIMBAND 1
#define SWD_NAME "ADWDgradlimband"
#include "adwdgrad_shim.h"
