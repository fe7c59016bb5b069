/* Host stand-in for <curand.h> (reference-pinning harness): the reference
 * includes it but uses only the device API of <curand_kernel.h>. */
#ifndef GEGS_REF_SHIM_CURAND_H
#define GEGS_REF_SHIM_CURAND_H
#include "curand_kernel.h"
#endif
