// The CUDA part of libgdon3d_cuda.so as one translation unit: the reference
// tables live in __constant__ memory that every kernel reads, and a single
// translation unit shares them without relocatable device code.
#include "aux.cu"
#include "rk3.cu"
#include "kinetic.cu"
#include "api.cu"
#include "noalloc.cu"
#include "mesh_gpu.cu"
