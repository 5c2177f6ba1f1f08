/* Host-only stand-in for the CUDA runtime header, used ONLY to compile the
 * reference's own sources (Mesh.cu, Geometry.cu, ICHDevice.cu) as plain C++
 * for the test oracle.  __host__/__device__ become nothing; the few runtime
 * calls the reference's host code names (cudaMalloc/cudaMemcpy/cudaFree in
 * Mesh::copyToGPU / clearGPU, cudaGetErrorString in book.cuh) map onto libc.
 * This is test infrastructure, never part of the product library. */
#pragma once
#include <cstdlib>
#include <cstring>
#define __host__
#define __device__
#define __global__
typedef int cudaError_t;
enum { cudaSuccess = 0 };
enum cudaMemcpyKind { cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2 };
struct uchar4 { unsigned char x, y, z, w; };
static inline const char* cudaGetErrorString(cudaError_t) { return "host-shim"; }
static inline cudaError_t cudaMalloc(void** p, size_t n) { *p = std::malloc(n); return *p ? 0 : 2; }
static inline cudaError_t cudaFree(void* p) { std::free(p); return 0; }
static inline cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) { std::memcpy(d, s, n); return 0; }
