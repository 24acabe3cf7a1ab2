/* ADWDgrad_1 of the field-data drivers (fieldexamples/outcrop/core/ADWDgrad_1.m:1-81 and the
 * same file under fieldexamples/QadimahFault/core) on libswd.so: the core ADWDgrad_1 with the
 * adjoint source divided by its largest magnitude (:79).  Build it into the field driver's core
 * directory in place of the reference's MEX-less .m. */
#define SWD_ADWD_NORM 0
#define SWD_ADWD_MAXNORM 1
#define SWD_NAME "ADWDgrad_1"
#include "adwdgrad_shim.h"
