/* Type-only stand-in for <optix.h>: the reference's include/macro_helper.h names OptixResult
 * and OPTIX_SUCCESS. Nothing of OptiX is used by the CPU build of the reference. */
#pragma once
typedef int OptixResult;
#define OPTIX_SUCCESS 0
