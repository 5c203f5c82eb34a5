/* Build shim (test infrastructure only).  The SDK's AEEStdErr.h is not
 * available; the reference pins only AEE_SUCCESS == 0.  The nonzero values
 * below are this project's choice and match include/calculator.h. */
#ifndef ROVER_SHIM_AEESTDERR_H
#define ROVER_SHIM_AEESTDERR_H
#define AEE_SUCCESS 0
#define AEE_EFAILED 1
#define AEE_ENOMEMORY 2
#define AEE_EBADPARM 14
#define AEE_EUNSUPPORTED 20
#endif
