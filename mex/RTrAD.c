/* RTrAD (core/RTrAD.m) on libswd.so. */
#include <string.h>
#define SWD_SIDE 0
#define SWD_AD 1
#define SWD_NAME "RTrAD"
#include "radon_shim.h"
