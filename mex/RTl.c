/* RTl (core/RTl.m) on libswd.so. */
#include <string.h>
#define SWD_SIDE 1
#define SWD_AD 0
#define SWD_NAME "RTl"
#include "radon_shim.h"
