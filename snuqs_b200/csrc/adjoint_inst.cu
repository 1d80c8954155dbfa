// One two-state adjoint sweep kernel instantiation per object file (see
// sweep_inst.cu); snuqs_b200/build.py compiles it with -DSQ_REAL=... -DSQ_M=...
#include "adjoint_kernels.cuh"
#include "sweep_registry.h"

#if !defined(SQ_REAL) || !defined(SQ_M)
#error "compile with -DSQ_REAL=<double|float> -DSQ_M=<tile bits>"
#endif

const void *SQ_ADJOINT_PTR_NAME(SQ_REAL, SQ_M)() {
  return reinterpret_cast<const void *>(&sq::adjoint_sweep_kernel<SQ_REAL, SQ_M>);
}
