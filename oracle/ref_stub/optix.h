/* ORACLE build shim: the reference's device/params.h includes <optix.h> only
 * for the traversable-handle type; the CPU harness needs nothing else. */
#pragma once
typedef unsigned long long OptixTraversableHandle;
