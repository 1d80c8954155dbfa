/*
 * Host-only stand-in for <cuda_runtime.h>, used ONLY to compile the
 * reference's CPU gate path (operation.cc, gate_operations.cc,
 * gate_operations_impl_cpu.cc) into oracle/_ref/ as a test oracle.
 *
 * The reference GateOperation constructor allocates a device copy of every
 * gate matrix (operation.cc:106-109) and frees it in the destructor
 * (operation.cc:112-114); the CPU path never touches that copy.  Without a
 * driver those calls would fail and CUDA_CHECK would exit the process, so
 * here they map onto host malloc/free/memcpy.  Nothing in the product links
 * this file.
 */
#ifndef SQ_ORACLE_SHIM_CUDA_RUNTIME_H
#define SQ_ORACLE_SHIM_CUDA_RUNTIME_H

#include <cstdlib>
#include <cstring>

typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 };
enum cudaMemcpyKind {
  cudaMemcpyHostToHost = 0,
  cudaMemcpyHostToDevice = 1,
  cudaMemcpyDeviceToHost = 2,
  cudaMemcpyDeviceToDevice = 3,
  cudaMemcpyDefault = 4
};

static inline cudaError_t cudaMalloc(void **p, size_t n) {
  *p = std::malloc(n ? n : 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
static inline cudaError_t cudaFree(void *p) {
  std::free(p);
  return cudaSuccess;
}
static inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n,
                                     cudaMemcpyKind) {
  std::memcpy(d, s, n);
  return cudaSuccess;
}
static inline const char *cudaGetErrorName(cudaError_t) { return "shim"; }
static inline const char *cudaGetErrorString(cudaError_t) { return "shim"; }

#endif
