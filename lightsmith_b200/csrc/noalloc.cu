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

constexpr int kNoAllocPartials = 8192;  // blocks of 256 points: up to 2,097,152 sampled points per call

static __device__ __align__(256) double g_noalloc_partials[kNoAllocPartials];

// errors are reported through lsfdtd_last_error (defined in lsfdtd.cu)
int noalloc_fail(int code, const std::string& msg) { return lsfdtd::report_error(code, msg); }

// the device address of the array on the current device, looked up once per device (host code must not
// pass the array's name itself to a kernel: on the host it only stands for the array)
constexpr int kMaxDevices = 64;
std::mutex g_addr_mutex;
double* g_addr[kMaxDevices] = {};

int partials_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(LSFDTD_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(LSFDTD_EUNSUPPORTED, "device index out of range");
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || !p)
      return noalloc_fail(LSFDTD_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_addr[dev] = static_cast<double*>(p);
  }
  *out = g_addr[dev];
  return LSFDTD_OK;
}

// the sample of k_monitor (monitors.cuh), with its partials in the static array
template <typename S>
__global__ void __launch_bounds__(kMonBlock) k_monitor_noalloc(MonArgs<S> a) {
  __shared__ double ph_re[kMonFreqTile], ph_im[kMonFreqTile];
  __shared__ double red[kMonBlock / 32];
  const bool is_h = blockIdx.x >= a.blocks_e;
  const long long p = (long long)(is_h ? blockIdx.x - a.blocks_e : blockIdx.x) * kMonBlock + threadIdx.x;
  const long long np = is_h ? a.nh : a.ne;
  const bool live = p < np;
  cplx<double> s = {0.0, 0.0};
  double e2 = 0.0;
  if (live) {
    if (!is_h) {
      const S v = a.Esrc[a.e_idx[p]];
      s = to_c64(v);
      e2 = norm2(v);
    } else {
      const S v = (a.Hsrc[a.h1[p]] + a.Hsrc[a.h2[p]]) * (typename real_of<S>::type)0.5;
      s = to_c64(v);
      e2 = norm2(v);
    }
  }
  const double t = (double)(*a.nstep) * a.dt - (is_h ? 0.5 * a.dt : 0.0);
  cplx<double>* acc = is_h ? a.acc_h : a.acc_e;
  for (int f0 = 0; f0 < a.nf; f0 += kMonFreqTile) {
    const int nt = min(kMonFreqTile, a.nf - f0);
    __syncthreads();
    for (int f = threadIdx.x; f < nt; f += kMonBlock) {
      double sn, cs;
      sincos(a.omega[f0 + f] * t, &sn, &cs);
      ph_re[f] = cs;
      ph_im[f] = sn;
    }
    __syncthreads();
    if (live) {
      for (int f = 0; f < nt; ++f) {
        cplx<double>* q = acc + (long long)(f0 + f) * np + p;
        const cplx<double> ph = {ph_re[f], ph_im[f]};
        *q = *q + ph * s;
      }
    }
  }
  if (a.want_energy) {
    double v = warp_sum(e2);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
      double w = threadIdx.x < kMonBlock / 32 ? red[threadIdx.x] : 0.0;
      w = warp_sum(w);
      if (threadIdx.x == 0) a.partial[blockIdx.x] = w;
    }
  }
}

// energy = the sum of the first `count` partials (a fixed-order warp sum)
__global__ void k_energy_noalloc(const double* partial, long long count, double* energy) {
  const int lane = threadIdx.x;
  double v = 0.0;
  for (long long i = lane; i < count; i += 32) v += partial[i];
  v = warp_sum(v);
  if (lane == 0) *energy = v;
}

template <typename S>
int sample(const lsfdtd_monitor_desc* m, const int64_t* step, double dt, double* energy, cudaStream_t s) {
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
  a.blocks_e = cdiv(m->n_e, kMonBlock);
  const long long blocks = (long long)a.blocks_e + (m->n_h > 0 ? cdiv(m->n_h, kMonBlock) : 0);
  if (blocks > kNoAllocPartials)
    return noalloc_fail(LSFDTD_EINVAL, "lsfdtd_dft_sample_noalloc: " + std::to_string(blocks) +
                                           " blocks of 256 points exceed the static scratch of " +
                                           std::to_string(kNoAllocPartials) + " (split the monitor)");
  double* partials = nullptr;
  int r = partials_address(&partials);
  if (r != LSFDTD_OK) return r;
  a.partial = partials;
  k_monitor_noalloc<S><<<(unsigned)blocks, kMonBlock, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(LSFDTD_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  if (a.want_energy) {
    k_energy_noalloc<<<1, 32, 0, s>>>(partials, blocks, energy);
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
