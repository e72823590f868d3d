// One running-DFT sample of one monitor without any device allocation.
//
// Some callers cannot allocate device memory: a host runtime that hands the library only the buffers it owns
// (its fields and accumulators) and forbids cudaMalloc on its own threads, or a process whose allocations must
// all come from one external pool. For them, this file keeps the scratch that the sample's energy reduction
// needs (one double per block of points) in a file-scope device array instead of in caller-provided scratch.
//
// The array is a fixed, modest size (kNoAllocPartials doubles, 64 KiB) and every GPU that loads the library
// holds it until the process exits. All calls share it and it keeps whatever the last call left in it; a call
// writes every partial it reads before reading it, so nothing needs clearing between calls. Two calls whose
// work overlaps on the GPU (for example on two streams) race on the array and must not be issued.
//
// The sample itself is the engine's own kernel pair (k_monitor, k_energy in monitors.cuh) with the partials
// pointed at the static array, so it is the engine's sample to the last bit.
#include <cuda.h>  // types of the driver entry points looked up below (nothing links against libcuda)

#include <mutex>
#include <string>

#include "lsfdtd.h"

#include "common.cuh"
#include "monitors.cuh"

namespace lsfdtd {
int report_error(int code, const std::string& msg);
}

using namespace lsfdtd;

namespace {

constexpr long long kNoAllocPartials = 8192;  // blocks of 256 points: up to 2,097,152 sampled points per call

static __device__ __align__(256) double g_noalloc_partials[kNoAllocPartials];

// errors are reported through lsfdtd_last_error (defined in lsfdtd.cu)
int noalloc_fail(int code, const std::string& msg) { return lsfdtd::report_error(code, msg); }

// The array's device address belongs to a CUDA context (the module's globals are loaded per context), not to
// a device index: after cudaDeviceReset the device's primary context is a new one, and a caller may run on a
// context of its own. So the address is looked up once per context, keyed by the driver's id of the current
// context (cuCtxGetId: unique for the life of the process, never reused), with that context current. Host code
// must not pass the array's name itself to a kernel: on the host it only stands for the array.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

struct CtxAddr {
  unsigned long long id;
  double* addr;
};
constexpr int kMaxContexts = 64;
std::mutex g_addr_mutex;
CtxAddr g_cache[kMaxContexts] = {};
int g_cache_n = 0, g_cache_next = 0;
CtxGetCurrentFn g_get_current = nullptr;
CtxGetIdFn g_get_id = nullptr;
bool g_entry_looked_up = false;

// the current context's id, or 0 when the driver cannot say (then the address is looked up on every call)
unsigned long long current_context_id() {
  if (!g_entry_looked_up) {
    g_entry_looked_up = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();  // a failed lookup leaves no error behind
  }
  if (!g_get_current || !g_get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (g_get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (g_get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

int partials_address(double** out) {
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  unsigned long long id = current_context_id();
  if (id)
    for (int i = 0; i < g_cache_n; ++i)
      if (g_cache[i].id == id) {
        *out = g_cache[i].addr;
        return LSFDTD_OK;
      }
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);  // makes the device's context current if needed
  if (e != cudaSuccess || !p)
    return noalloc_fail(LSFDTD_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  *out = static_cast<double*>(p);
  if (!id) id = current_context_id();  // the first runtime call of the process has just created the context
  if (id) {
    const int slot = g_cache_n < kMaxContexts ? g_cache_n++ : (g_cache_next++ % kMaxContexts);
    g_cache[slot] = {id, *out};
  }
  return LSFDTD_OK;
}

template <typename S>
int sample(const lsfdtd_monitor_desc* m, const int64_t* step, double dt, double* energy, cudaStream_t s) {
  // block counts in 64-bit arithmetic, checked against the array before any narrowing
  const long long blocks_e = ((long long)m->n_e + kMonBlock - 1) / kMonBlock;
  const long long blocks_h = m->n_h > 0 ? ((long long)m->n_h + kMonBlock - 1) / kMonBlock : 0;
  const long long blocks = blocks_e + blocks_h;
  if (blocks > kNoAllocPartials)
    return noalloc_fail(LSFDTD_EINVAL, "lsfdtd_dft_sample_noalloc: " + std::to_string(blocks) +
                                           " blocks of 256 points exceed the static scratch of " +
                                           std::to_string(kNoAllocPartials) + " (split the monitor)");
  double* partials = nullptr;
  int r = partials_address(&partials);
  if (r != LSFDTD_OK) return r;
  MonArgs<S> a{};
  a.nf = m->n_freq;
  a.omega = m->omega;
  a.ne = m->n_e;
  a.nh = m->n_h;
  a.e_idx = reinterpret_cast<const long long*>(m->e_idx);
  a.h1 = reinterpret_cast<const long long*>(m->h_idx1);
  a.h2 = reinterpret_cast<const long long*>(m->h_idx2);
  a.acc_e = static_cast<cplx<double>*>(m->acc_e);
  a.acc_h = static_cast<cplx<double>*>(m->acc_h);
  a.Esrc = static_cast<const S*>(m->E_src);
  a.Hsrc = static_cast<const S*>(m->H_src);
  a.dt = dt;
  a.nstep = reinterpret_cast<const long long*>(step);
  a.want_energy = (m->energy && m->n_h > 0 && energy) ? 1 : 0;
  a.blocks_e = blocks_e;
  a.partial = partials;
  k_monitor<S><<<(unsigned)blocks, kMonBlock, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(LSFDTD_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  if (a.want_energy) {
    k_energy<<<1, 32, 0, s>>>(partials, 0, blocks, 0, 0, energy);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(LSFDTD_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  }
  return LSFDTD_OK;
}

}  // namespace

extern "C" {

int32_t lsfdtd_dft_sample_noalloc(const lsfdtd_monitor_desc* m, int32_t precision, int32_t is_complex,
                                  const int64_t* step, double dt, double* energy, void* stream) {
  if (!m || !step || !m->omega || !m->e_idx || !m->acc_e || !m->E_src)
    return noalloc_fail(LSFDTD_EINVAL, "lsfdtd_dft_sample_noalloc: null argument");
  if (m->n_e <= 0 || m->n_freq <= 0) return noalloc_fail(LSFDTD_EINVAL, "lsfdtd_dft_sample_noalloc: empty monitor");
  if (m->n_h > 0 && (!m->h_idx1 || !m->h_idx2 || !m->acc_h || !m->H_src))
    return noalloc_fail(LSFDTD_EINVAL, "lsfdtd_dft_sample_noalloc: H arrays missing");
  if (precision != LSFDTD_F32 && precision != LSFDTD_F64)
    return noalloc_fail(LSFDTD_EINVAL, "lsfdtd_dft_sample_noalloc: unknown precision");
  auto s = static_cast<cudaStream_t>(stream);
  const bool real_src = m->space == 1 || !is_complex;
  if (precision == LSFDTD_F32)
    return real_src ? sample<float>(m, step, dt, energy, s) : sample<cplx<float>>(m, step, dt, energy, s);
  return real_src ? sample<double>(m, step, dt, energy, s) : sample<cplx<double>>(m, step, dt, energy, s);
}

}  // extern "C"
