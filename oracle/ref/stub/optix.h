/* Host stand-in for the OptiX types the reference headers name (include/scene.h:32-34,
 * include/mesh/mesh_type.h:46-47). No OptiX code is compiled into the host build. */
#pragma once
typedef unsigned long long OptixTraversableHandle;
typedef struct OptixPipeline_stub* OptixPipeline;
typedef struct OptixShaderBindingTable { int unused; } OptixShaderBindingTable;
typedef unsigned long long CUdeviceptr;
