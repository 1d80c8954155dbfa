// Host-side lookup of the compiled fused-sweep kernels (one object file per
// instantiation, see sweep_inst.cu).
#pragma once

#define SQ_SWEEP_CAT(a, b, c) a##_##b##_##c
#define SQ_SWEEP_PTR_NAME(real, m) SQ_SWEEP_CAT(sq_sweep_kernel_ptr, real, m)

#define SQ_DECLARE_SWEEP(real, m) const void *SQ_SWEEP_PTR_NAME(real, m)();
SQ_DECLARE_SWEEP(double, 4)
SQ_DECLARE_SWEEP(double, 7)
SQ_DECLARE_SWEEP(double, 10)
SQ_DECLARE_SWEEP(double, 11)
SQ_DECLARE_SWEEP(double, 12)
SQ_DECLARE_SWEEP(float, 4)
SQ_DECLARE_SWEEP(float, 7)
SQ_DECLARE_SWEEP(float, 10)
SQ_DECLARE_SWEEP(float, 12)
#undef SQ_DECLARE_SWEEP

#define SQ_ADJOINT_PTR_NAME(real, m) SQ_SWEEP_CAT(sq_adjoint_kernel_ptr, real, m)
#define SQ_DECLARE_ADJOINT(real, m) const void *SQ_ADJOINT_PTR_NAME(real, m)();
SQ_DECLARE_ADJOINT(double, 4)
SQ_DECLARE_ADJOINT(double, 7)
SQ_DECLARE_ADJOINT(double, 10)
SQ_DECLARE_ADJOINT(float, 4)
SQ_DECLARE_ADJOINT(float, 7)
SQ_DECLARE_ADJOINT(float, 11)
#undef SQ_DECLARE_ADJOINT

#define SQ_BATCH_PTR_NAME(real, m) SQ_SWEEP_CAT(sq_batch_kernel_ptr, real, m)
const void *SQ_BATCH_PTR_NAME(double, 10)();
const void *SQ_BATCH_PTR_NAME(double, 11)();
const void *SQ_BATCH_PTR_NAME(double, 12)();
const void *SQ_BATCH_PTR_NAME(float, 10)();
const void *SQ_BATCH_PTR_NAME(float, 11)();
const void *SQ_BATCH_PTR_NAME(float, 12)();
#define SQ_BATCH_ADJ_PTR_NAME(real, m) SQ_SWEEP_CAT(sq_batch_adjoint_kernel_ptr, real, m)
const void *SQ_BATCH_ADJ_PTR_NAME(double, 10)();
const void *SQ_BATCH_ADJ_PTR_NAME(double, 11)();
const void *SQ_BATCH_ADJ_PTR_NAME(float, 11)();
const void *SQ_BATCH_ADJ_PTR_NAME(float, 12)();
