// sq_expect_pauli_noalloc: the Pauli-string expectation without any device
// allocation.
//
// sq_expect_pauli keeps its per-block partial sums in a small buffer that each
// state handle cudaMalloc's on first use.  Some callers cannot allocate: code
// that records work into a CUDA graph, where a cudaMalloc would break the
// capture; applications whose memory pool owns every byte of the device and
// forbids allocations behind its back; and callers that hold only a raw
// device pointer to a state vector (no sq_state handle to hang a buffer on).
// This entry point serves them: the partial sums live in a fixed array in
// this file, `static __device__`, which every device that loads the library
// holds until the process exits; nothing is allocated per call.  The caller
// passes the state and the output location.  The first call on a device
// looks up the array's device address (make that first call before any
// stream capture).  The address is saved per device together with the CUDA
// context that was current at the look-up; when the context changes (after
// cudaDeviceReset, or a primary context torn down and rebuilt) the next call
// looks the address up again instead of using a stale one.  All calls on a
// device share the array, so calls that overlap on the GPU race: order them
// on one stream or with events.
//
// The array's limits: at most kNoAllocMaxBlocks (2048) reduction blocks
// (16 KiB of FP64 partials), at most 1024 Pauli terms and 256 distinct
// (X/Y mask, Y parity) groups per call.  Larger requests are rejected.
// Each call stages the grouped terms on the calling thread's stack (about
// 45 KiB: the kernel's parameter block and four term arrays).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/snuqs_b200.h"
#include "reduce_kernels.cuh"

int sq_detail_fail(int code, const char *msg);  // engine.cu: sets sq_last_error()

namespace {

constexpr uint32_t kNoAllocMaxBlocks = 2048;
constexpr int kMaxDevices = 64;

// Shared by every call on a device; each call overwrites the slots it uses.
static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxBlocks];

std::mutex g_mu;
double *g_partials_ptr[kMaxDevices] = {};
void *g_partials_ctx[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};

int fail(int code, const char *msg) { return sq_detail_fail(code, msg); }

// The current CUDA context (driver cuCtxGetCurrent, reached through the
// runtime's entry-point query so that the library needs no libcuda link).
int current_context(void **ctx) {
  using GetCurrent = int (*)(void **);
  static GetCurrent fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<GetCurrent>(f);
  }();
  if (!fn) return fail(SQ_ERR_CUDA, "sq_expect_pauli_noalloc: cuCtxGetCurrent unavailable");
  *ctx = nullptr;
  if (fn(ctx) != 0 || !*ctx) return fail(SQ_ERR_CUDA, "sq_expect_pauli_noalloc: no current context");
  return SQ_OK;
}

// Device set-up, with that device current, once per device and context: the
// host-side name of a __device__ array is not a device address, so look the
// address up (and again whenever the device's context has changed).
int setup_device(int dev, double **partials, int *sms) {
  void *ctx = nullptr;
  const int cs = current_context(&ctx);
  if (cs != SQ_OK) return cs;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_partials_ptr[dev] || g_partials_ctx[dev] != ctx) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess) return fail(SQ_ERR_CUDA, cudaGetErrorString(e));
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail(SQ_ERR_CUDA, cudaGetErrorString(e));
    g_partials_ptr[dev] = static_cast<double *>(p);
    g_partials_ctx[dev] = ctx;
    g_sms[dev] = n;
  }
  *partials = g_partials_ptr[dev];
  *sms = g_sms[dev];
  return SQ_OK;
}

}  // namespace

extern "C" int sq_expect_pauli_noalloc(const void *state, uint32_t num_qubits, int dtype,
                                       const char *paulis, const double *weights,
                                       uint32_t n_terms, double *out_device, void *stream) {
  if (!state || !out_device || (n_terms && (!paulis || !weights)))
    return fail(SQ_ERR_INVALID, "sq_expect_pauli_noalloc: null pointer");
  if (dtype != SQ_C128 && dtype != SQ_C64)
    return fail(SQ_ERR_INVALID, "sq_expect_pauli_noalloc: bad dtype");
  if (num_qubits < 1 || num_qubits > 40)
    return fail(SQ_ERR_INVALID, "sq_expect_pauli_noalloc: num_qubits must be in [1, 40]");
  if (n_terms > uint32_t(sq::kMaxTerms))
    return fail(SQ_ERR_UNSUPPORTED,
                "sq_expect_pauli_noalloc: more than 1024 Pauli terms (use sq_expect_pauli)");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(SQ_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(SQ_ERR_UNSUPPORTED, "device ordinal >= 64");
  double *partials = nullptr;
  int sms = 0;
  const int st = setup_device(dev, &partials, &sms);
  if (st != SQ_OK) return st;

  // Terms -> (flip mask, Z-or-Y mask, Y count); sort by (flip mask, Y parity)
  // into contiguous groups.  Fixed-size arrays: nothing here allocates.
  const uint32_t n = num_qubits;
  uint64_t xm[sq::kMaxTerms], zym[sq::kMaxTerms];
  int ny[sq::kMaxTerms];
  uint16_t idx[sq::kMaxTerms];
  for (uint32_t t = 0; t < n_terms; ++t) {
    xm[t] = zym[t] = 0;
    ny[t] = 0;
    idx[t] = uint16_t(t);
    for (uint32_t q = 0; q < n; ++q) {
      const uint64_t bit = uint64_t(1) << (n - 1 - q);
      switch (paulis[size_t(t) * n + q]) {
        case 'I': case 'i': break;
        case 'X': case 'x': xm[t] |= bit; break;
        case 'Y': case 'y': xm[t] |= bit; zym[t] |= bit; ny[t]++; break;
        case 'Z': case 'z': zym[t] |= bit; break;
        default: return fail(SQ_ERR_INVALID, "sq_expect_pauli_noalloc: bad Pauli character");
      }
    }
  }
  std::stable_sort(idx, idx + n_terms, [&](uint16_t a, uint16_t b) {
    if (xm[a] != xm[b]) return xm[a] < xm[b];
    return (ny[a] & 1) < (ny[b] & 1);
  });
  sq::PauliParams P;  // 22 KiB on the stack
  std::memset(&P, 0, sizeof(P));
  P.n = n;
  uint32_t nt = 0;
  for (uint32_t pos = 0; pos < n_terms;) {
    const uint32_t i0 = idx[pos];
    uint32_t end = pos;
    while (end < n_terms && xm[idx[end]] == xm[i0] && (ny[idx[end]] & 1) == (ny[i0] & 1)) ++end;
    if (P.ngroups >= uint32_t(sq::kMaxGroups))
      return fail(SQ_ERR_UNSUPPORTED,
                  "sq_expect_pauli_noalloc: more than 256 distinct Pauli groups");
    sq::PauliGroup &g = P.g[P.ngroups++];
    g.x = xm[i0];
    g.odd = ny[i0] & 1;
    g.t0 = nt;
    for (uint32_t k = pos; k < end; ++k) {
      const uint32_t t = idx[k];
      // (-i)^ny folded into a real factor (see reduce_kernels.cuh).
      P.zy[nt] = zym[t];
      P.f[nt] = weights[t] * (((ny[t] / 2) & 1) ? -1.0 : 1.0);
      ++nt;
    }
    g.t1 = nt;
    pos = end;
  }

  const uint64_t pairs = uint64_t(1) << (n - 1);
  const uint32_t blocks = uint32_t(std::max<uint64_t>(
      1, std::min<uint64_t>({(pairs + sq::kReduceThreads - 1) / sq::kReduceThreads,
                             uint64_t(sms) * 4, uint64_t(kNoAllocMaxBlocks)})));
  auto s = static_cast<cudaStream_t>(stream);
  // accumulate = 0: every used partial slot is overwritten, so the previous
  // call's contents need no clearing.
  if (dtype == SQ_C64)
    sq::pauli_expect_kernel<float><<<blocks, sq::kReduceThreads, 0, s>>>(
        static_cast<const float2 *>(state), P, partials, 0);
  else
    sq::pauli_expect_kernel<double><<<blocks, sq::kReduceThreads, 0, s>>>(
        static_cast<const double2 *>(state), P, partials, 0);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(SQ_ERR_CUDA, cudaGetErrorString(e));
  // Fixed-order sum of the partials into the caller's output (deterministic).
  sq::finalize_sum_kernel<<<1, sq::kReduceThreads, 0, s>>>(partials, blocks, out_device);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(SQ_ERR_CUDA, cudaGetErrorString(e));
  return SQ_OK;
}
