// JIT-specialised sweep kernels (see jit.cu).
#pragma once
#include <string>
#include <vector>

#include "host_ops.h"

namespace sq {

bool jit_available();
// Counts a sweep launch that ran a JIT kernel (true) or fell back (false).
void jit_note_launch(bool jit);
// CUDA source of the kernel specialised for `ps` (`minb` CTAs per SM);
// multi: its multi-state form (jit_msweep_kernel).
// from_zero (multi-state only): the first phase starts from |0...0> in every
// state instead of reading it (empty source when the sweep's first phase does
// not load from HBM).
std::string jit_source(const PlannedSweep &ps, bool c64, int minb, bool multi = false, bool from_zero = false);
// The part of that source that depends on `ps` (the cache key).
std::string jit_body(const PlannedSweep &ps, bool c64, int minb, bool multi = false, bool from_zero = false);
// Dynamic shared memory the JIT kernel of `ps` needs.
size_t jit_smem(const PlannedSweep &ps, bool c64);
// CTAs per SM the kernels of (precision, tile bits) are built for.
int jit_minb(bool c64, uint32_t m);
// Launchable kernel (a cudaKernel_t as const void*) for `ps`, compiling and
// caching it on first use; nullptr with `err` set when it cannot be built.
const void *jit_sweep_kernel(const PlannedSweep &ps, bool c64, std::string &err);
// Two-state (adjoint reverse) sweeps: the JIT kernel (cudaKernel_t as const
// void*, or nullptr with `err`), its dynamic shared memory, its source, and
// a parallel pre-compile of several sweeps.
const void *jit_adjoint_kernel(const PlannedSweep &ps, bool c64, std::string &err);
size_t jit_adjoint_smem(const PlannedSweep &ps, bool c64);
std::string jit_adjoint_body(const PlannedSweep &ps, bool c64, int minb);
int jit_adjoint_minb(bool c64);
void jit_prepare_adjoint(const std::vector<const PlannedSweep *> &sweeps, bool c64);
// Batched gradients of circuits that share one packed plan structure
// (`plan`: one circuit's packed records, nfwd forward then nrev reverse
// sweeps, every sweep of m == M): the kernel (or nullptr with `err`), its
// generated body, and the full source of a body.
const void *jit_batch_adjoint_kernel(const unsigned char *plan, uint32_t nfwd, uint32_t nrev, uint32_t n,
                                     uint32_t M, bool c64, std::string &err);
std::string jit_batch_adjoint_body(const unsigned char *plan, uint32_t nfwd, uint32_t nrev, uint32_t n,
                                   uint32_t M, bool c64);
std::string jit_batch_source(const std::string &body);
// Multi-state sweeps (sq_jit_msweep: one launch applies the sweep to K states
// that share its structure, sq::MultiParams): the kernel (or nullptr with
// `err`), its dynamic shared memory, and a parallel pre-compile.
const void *jit_msweep_kernel(const PlannedSweep &ps, bool c64, std::string &err, bool from_zero = false);
size_t jit_msweep_smem(const PlannedSweep &ps, bool c64);
void jit_prepare_multi(const std::vector<const PlannedSweep *> &sweeps, bool c64,
                       const std::vector<const PlannedSweep *> &from_zero = {});
// Compiles the kernels of several sweeps in parallel (fills the cache).
void jit_prepare(const std::vector<const PlannedSweep *> &sweeps, bool c64);

}  // namespace sq
