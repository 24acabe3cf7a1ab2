/* RTlAD (core/RTlAD.m) on libswd.so. */
#include <string.h>
#define SWD_SIDE 1
#define SWD_AD 1
#define SWD_NAME "RTlAD"
#include "radon_shim.h"
