// One fused-sweep kernel instantiation per object file.  snuqs_b200/build.py
// compiles this file once per (precision, tile bits, CTAs per SM) with
// -DSQ_REAL=... -DSQ_M=... -DSQ_MINB=..., in parallel, and the engine picks
// the kernel through sweep_registry.h.
#include "sweep_kernels.cuh"
#include "sweep_registry.h"

#if !defined(SQ_REAL) || !defined(SQ_M) || !defined(SQ_MINB)
#error "compile with -DSQ_REAL=<double|float> -DSQ_M=<tile bits> -DSQ_MINB=<CTAs per SM>"
#endif

const void *SQ_SWEEP_PTR_NAME(SQ_REAL, SQ_M)() {
  return reinterpret_cast<const void *>(&sq::sweep_kernel<SQ_REAL, SQ_M, SQ_MINB>);
}
