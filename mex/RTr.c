/* RTr (core/RTr.m) on libswd.so. */
#include <string.h>
#define SWD_SIDE 0
#define SWD_AD 0
#define SWD_NAME "RTr"
#include "radon_shim.h"
