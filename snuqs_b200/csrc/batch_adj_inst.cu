// One batched-adjoint-gradient kernel instantiation per object file (see
// sweep_inst.cu); snuqs_b200/build.py compiles it with -DSQ_REAL=... -DSQ_M=...
#include "batch_kernels.cuh"
#include "sweep_registry.h"

#if !defined(SQ_REAL) || !defined(SQ_M)
#error "compile with -DSQ_REAL=<double|float> -DSQ_M=<tile bits>"
#endif

const void *SQ_BATCH_ADJ_PTR_NAME(SQ_REAL, SQ_M)() {
  return reinterpret_cast<const void *>(&sq::batch_adjoint_kernel<SQ_REAL, SQ_M>);
}
