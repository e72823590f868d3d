// Running-DFT monitors with float64 accumulators and the decay-energy proxy.
//
// At a sample (every dft_stride steps, n steps completed): acc_e[f, p] += e^{i w_f t_e} E[e_idx[p]] with
// t_e = n dt, and acc_h[f, p] += e^{i w_f t_h} (H[h1[p]] + H[h2[p]]) / 2 with t_h = t_e - dt/2
// (backends/_fdtd/engine.py:564-592). Each block forms its frequencies' phases once in shared memory; each
// thread owns one point, so the accumulator rows are read and written coalesced. The energy
// sum |E|^2 + |H_avg|^2 of a flagged monitor is reduced per block with warp shuffles into a scratch
// partial, then a single-warp pass sums the partials of each energy group in a fixed order (deterministic).
#pragma once

#include "common.cuh"

namespace lsfdtd {

constexpr int kMonBlock = 256;
constexpr int kMonFreqTile = 128;

template <typename S>
struct MonArgs {
  int nf;
  const double* omega;
  long long ne, nh;
  const long long* e_idx;
  const long long* h1;
  const long long* h2;
  cplx<double>* acc_e;
  cplx<double>* acc_h;
  const S* Esrc;
  const S* Hsrc;
  double dt;
  const long long* nstep;
  int want_energy;
  double* partial;  // one double per block
  long long blocks_e;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <typename S>
__global__ void __launch_bounds__(kMonBlock) k_monitor(MonArgs<S> a) {
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
      // the mean of the two H samples is formed in the field precision, as the reference does
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

// energy[g] = sum of the partials [first, first + count) of each group present (a fixed-order warp sum)
static __global__ void k_energy(const double* partial, long long first0, long long count0, long long first1,
                         long long count1, double* energy) {
  const int lane = threadIdx.x;
  for (int g = 0; g < 2; ++g) {
    const long long first = g ? first1 : first0, count = g ? count1 : count0;
    if (count <= 0) continue;
    double v = 0.0;
    for (long long i = lane; i < count; i += 32) v += partial[first + i];
    v = warp_sum(v);
    if (lane == 0) energy[g] = v;
  }
}

}  // namespace lsfdtd
