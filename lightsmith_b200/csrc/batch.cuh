// Many independent Bloch-periodic oblique runs advanced by one persistent kernel.
//
// A periodic cell at fixed in-plane wavevector is solved once per (angle, wavelength, polarisation)
// (backends/_fdtd/periodic.py:426-459): complex fields, periodic x and y with Bloch ghost phases, CPML along
// z, a TF/SF plane fed by a 3 x 3 x nz column (tfsf.py:214-296) and running DFTs on two planes and on the
// column. lightsmith runs these one after the other, each a few dozen small kernels per step. Here a cluster
// of kBatchCluster CTAs takes whole runs from a list (longest first, spread over the clusters by the host) and
// advances each through its steps inside one launch, its CTAs sharing the nodes of every phase:
//
//   H phase: H curl and z CPML of every node (update_h_node's arithmetic), the plane correction of H at
//            k_src - 1 (correct_H) applied by the thread that updated the node, the node's low ghost copies
//            (x, then y, then the corner, as the ghost refresh orders them) written through; and the column's
//            H at (1, 1, z) with its own ghosts;
//   E phase: the same for E, with correct_E at k_src and the high ghosts; the column's E with the current
//            sheet at k_launch added before the column's ghost copies. lightsmith refreshes E's ghosts at the
//            start of the next H update instead, so after a launch's last step they are left as they were
//            and refreshed when the run enters its next launch: between launches an engine's arrays are,
//            ghosts included, what its own steps would have left;
//   gather:  the conformal off-diagonal terms of E (k_offdiag's rows, one thread per target), the targets'
//            high ghosts written through;
//   sample:  every dft_stride steps, the running DFT of each monitor point (k_monitor's arithmetic).
//
// A run whose E turns non-finite in a step (a diverging run, as lightsmith's run loop would report it,
// setup.py:749-756) sets its engine's status word and retires after that step: its step counter records the
// steps it ran and later launches skip it, so it no longer holds its cluster.
//
// The cluster's hardware barrier (barrier.cluster, release / acquire) separates the phases; nothing else is
// shared between threads. Every CTA of a cluster walks the same run list and step counts, so each reaches
// every barrier. The run's step counter is the engine's own, so an engine that took part in a batch is in the
// state its own steps would have left.
//
// GROUP: the CTAs of a run are a group of any size (a cooperative launch keeps every CTA resident) that meet
// at a barrier in global memory (group_barrier) instead of the cluster's. Few runs then advance at once, each
// on many SMs, and the runs in flight stay in L2 from one step to the next. A barrier wait is bounded: a CTA
// that gives up sets the run's status word to 1 and returns, and the group's other CTAs give up at their next
// barrier.
#pragma once

#include "common.cuh"
#include "monitors.cuh"
#include "yee.cuh"

namespace lsfdtd {

constexpr int kBatchMaxMon = 4;
constexpr int kBatchNonFinite = 2;  // status word value of a run whose fields turned non-finite (it retires)
constexpr int kBatchThreads = 512;
constexpr int kBatchCluster = 8;  // CTAs per run by default (the portable cluster size); 2 to 16 at launch

// every thread of every CTA of the cluster arrives; global writes before it are visible after it
__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// polls of a group barrier's counter before a CTA gives up (each after a 256 ns sleep: a few seconds, where a
// barrier of the batched sweep takes microseconds)
constexpr long long kGroupSpinLimit = 8LL << 20;

// every thread of the ncta CTAs counting on `count` arrives (one 64-bit counter per group, zero at the launch's
// start, bumped once per CTA and barrier: the barrier's generation is ticket / ncta); global writes before it
// are visible after it. False when this CTA gave up waiting (then on every thread of the CTA).
__device__ __forceinline__ bool group_barrier(unsigned long long* count, unsigned ncta) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();  // release: the CTA's writes (ordered before thread 0's by the CTA barrier) at GPU scope
    const unsigned long long ticket = atomicAdd(count, 1ull);
    const unsigned long long target = (ticket / ncta + 1) * ncta;
    bool good = false;
    for (long long spin = 0; spin < kGroupSpinLimit; ++spin) {
      unsigned long long v;
      asm volatile("ld.acquire.gpu.global.u64 %0, [%1];\n" : "=l"(v) : "l"(count) : "memory");
      if (v >= target) {
        good = true;
        break;
      }
      __nanosleep(256);
    }
    __threadfence();
    ok = good ? 1 : 0;
  }
  __syncthreads();
  return ok != 0;
}

// unsigned division by a run constant with one multiply-high (Granlund and Montgomery, "Division by
// Invariant Integers using Multiplication", PLDI 1994, fig. 4.1): exact for every 32-bit numerator
struct UDiv {
  unsigned m, s1, s2;
};
inline UDiv udiv_make(unsigned d) {
  unsigned l = 0;
  while ((1ull << l) < d) ++l;
  UDiv u;
  u.m = (unsigned)(((1ull << 32) * ((1ull << l) - d)) / d + 1);
  u.s1 = l < 1 ? l : 1;
  u.s2 = l > 1 ? l - 1 : 0;
  return u;
}
__device__ __forceinline__ unsigned udiv(unsigned n, UDiv u) {
  const unsigned t = __umulhi(u.m, n);
  return (t + ((n - t) >> u.s1)) >> u.s2;
}

template <typename F>
struct BlochRun {
  using R = typename real_of<F>::type;
  YeeArgs<F> g;    // the cell: periodic x and y, CPML along z only
  YeeArgs<F> col;  // the source's 3 x 3 x nz column
  F gph[2][2];     // the cell's ghost phases [axis x, y][low, high]
  F cph[2][2];     // the column's
  const F* phase;  // (nx, ny) phases of the TF/SF plane
  F amp0, amp1;    // sheet amplitudes (E_x, E_y)
  const R* wave;   // sheet waveform per step
  R cE, cH;        // plane-correction coefficients
  int k_src, k_launch;
  int stride;
  long long last;  // the run's final step count
  long long* nstep;  // the engine's step counter (steps completed)
  int* status;       // the engine's status word: set to kBatchNonFinite when the run's E turns non-finite
  // conformal off-diagonal 1/eps terms (k_offdiag's tables): row q adds sum_k od_w[q, k] H_flat[od_h[q, k]] to
  // E_flat[od_e[q]] after the E update
  const long long* od_e;
  const long long* od_h;
  const F* od_w;
  long long od_n;
  int od_width;
  int n_mon;
  MonArgs<F> mon[kBatchMaxMon];
  UDiv div_n2, div_ny;  // by the nodes along z and the real cells along y
};

// the z slab holding node z for field FLD (-1: none) and the node's psi index in it
template <int FLD, typename F>
__device__ __forceinline__ int slab_z(const YeeArgs<F>& g, int c, int x, int y, int z, long long* q) {
  const PmlAxis<F>& p = g.pml[2];
  if (!p.on) return -1;
#pragma unroll
  for (int sd = 0; sd < 2; ++sd) {
    const int st = p.start[FLD][c][sd], ln = p.len[FLD][c][sd];
    if (z >= st && z < st + ln) {
      *q = ((long long)x * g.n[1] + y) * ln + (z - st);
      return sd;
    }
  }
  return -1;
}

// one monitor point's DFT update (k_monitor's arithmetic): i < ne an E point, else H point i - ne
template <typename F>
__device__ __forceinline__ void batch_sample_point(const MonArgs<F>& m, long long i, long long n) {
  const bool is_h = i >= m.ne;
  const long long p = is_h ? i - m.ne : i;
  cplx<double> s;
  if (!is_h) {
    s = to_c64(m.Esrc[m.e_idx[p]]);
  } else {
    const F v = (m.Hsrc[m.h1[p]] + m.Hsrc[m.h2[p]]) * (typename real_of<F>::type)0.5;
    s = to_c64(v);
  }
  const double t = (double)n * m.dt - (is_h ? 0.5 * m.dt : 0.0);
  const long long np = is_h ? m.nh : m.ne;
  cplx<double>* acc = is_h ? m.acc_h : m.acc_e;
  for (int f = 0; f < m.nf; ++f) {
    double sn, cs;
    sincos(m.omega[f] * t, &sn, &cs);
    cplx<double>* q = acc + (long long)f * np + p;
    const cplx<double> ph = {cs, sn};
    *q = *q + ph * s;
  }
}

// complex64: two CTAs per SM (64 registers per thread), for twice the nodes in flight
// launched with a cluster dimension (CTAs per run) set at launch: the CTA's rank in its cluster, the
// cluster's index in the grid and its size come from the special registers
// (GROUP: CTAs blockIdx.x / gsize share a run list; gbar holds each group's barrier counter)
template <typename F, bool GROUP>
__global__ void __launch_bounds__(kBatchThreads, sizeof(F) == 8 ? 2 : 1)
    k_bloch_batch(const BlochRun<F>* runs, const int* order, const int* first, int steps, int gsize,
                  unsigned long long* gbar) {
  using R = typename real_of<F>::type;
  __shared__ BlochRun<F> r;
  unsigned cl, rank, ncta;
  if constexpr (GROUP) {
    cl = blockIdx.x / (unsigned)gsize;
    rank = blockIdx.x % (unsigned)gsize;
    ncta = (unsigned)gsize;
  } else {
    asm("mov.u32 %0, %%clusterid.x;" : "=r"(cl));
    asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    asm("mov.u32 %0, %%cluster_nctarank;" : "=r"(ncta));
  }
  // the barrier between phases; false: this CTA gave up waiting (a group barrier), the run's status word is
  // set and the CTA returns
  auto sync = [&]() -> bool {
    if constexpr (GROUP) {
      if (group_barrier(gbar + 16 * cl, ncta)) return true;
      if (threadIdx.x == 0) atomicExch(r.status, 1);
      return false;
    } else {
      cluster_barrier();
      return true;
    }
  };
  const unsigned t0 = rank * blockDim.x + threadIdx.x, tstride = ncta * blockDim.x;
  for (int q = first[cl]; q < first[cl + 1]; ++q) {
    // the run's descriptor into each CTA's shared memory (read by every thread at every node)
    {
      const int* src = reinterpret_cast<const int*>(runs + order[q]);
      int* dst = reinterpret_cast<int*>(&r);
      for (int w = threadIdx.x; w < (int)(sizeof(BlochRun<F>) / sizeof(int)); w += blockDim.x) dst[w] = src[w];
    }
    __syncthreads();
    const YeeArgs<F>& g = r.g;
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const unsigned nx = n0 - 2, ny = n1 - 2, un2 = n2;
    const long long s1 = n2, s0 = (long long)n1 * n2;
    const unsigned us1 = n2, us0 = (unsigned)n1 * n2;  // 32-bit node offsets within a component
    const unsigned n_main = nx * ny * un2;  // fewer than 2^32 nodes (checked on the host)
    const unsigned n_work = n_main + un2;   // the cell's interior nodes, then the column's (1, 1, z)
    // a thread's nodes advance by tstride: (z, y, x) carried forward with two carries, not divided anew
    const unsigned dq = udiv(tstride, r.div_n2), dz = tstride - dq * un2;
    const unsigned dxm = udiv(dq, r.div_ny), dym = dq - dxm * ny;
    const unsigned q0 = udiv(t0, r.div_n2), z00 = t0 - q0 * un2;
    const unsigned xm00 = udiv(q0, r.div_ny), ym00 = q0 - xm00 * ny;
    const long long cs1 = n2, cs0 = 3LL * n2;
    const long long ccol = 4LL * n2;  // flat index of the column node (1, 1, 0)
    long long n = *r.nstep;
    // a run that turned non-finite in an earlier launch is skipped (the word was written before this launch)
    long long n_end = *reinterpret_cast<volatile int*>(r.status) == kBatchNonFinite ? n : min(n + (long long)steps, r.last);
    // this thread's E values of the run times zero, summed: zero while every value is finite, NaN after one
    // is not (cheaper than testing each value)
    R nonfinite = R(0);
    if (!sync()) return;  // every thread has read the counter
    if (n < n_end) {
      // E's high ghosts as lightsmith refreshes them before each H update (x = n0 - 1 from x = 1, then
      // y = n1 - 1 from y = 1, and the corner), for the cell and the column: the E phase of a launch's last
      // step leaves them for this refresh, so that between launches they hold what the engine's own steps
      // would have left
      const unsigned n_gx = ny * un2, n_gy = nx * un2;
      for (unsigned w = t0; w < n_gx + n_gy + 2 * un2; w += tstride) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (w < n_gx) {
            const long long yz = (long long)(1 + w / un2) * s1 + w % un2;
            g.E[c][(long long)(n0 - 1) * s0 + yz] = g.E[c][s0 + yz] * r.gph[0][1];
          } else if (w < n_gx + n_gy) {
            const unsigned q2 = w - n_gx;
            const long long xz = (long long)(1 + q2 / un2) * s0 + q2 % un2;
            g.E[c][xz + (long long)(n1 - 1) * s1] = g.E[c][xz + s1] * r.gph[1][1];
          } else if (w < n_gx + n_gy + un2) {
            const long long z = w - n_gx - n_gy;
            g.E[c][(long long)(n0 - 1) * s0 + (long long)(n1 - 1) * s1 + z] =
                (g.E[c][s0 + s1 + z] * r.gph[0][1]) * r.gph[1][1];
          } else {
            const long long z = w - n_gx - n_gy - un2;
            const F e = r.col.E[c][ccol + z];
            const F gx = e * r.cph[0][1];
            r.col.E[c][2 * cs0 + cs1 + z] = gx;
            r.col.E[c][2 * cs0 + 2 * cs1 + z] = gx * r.cph[1][1];
            r.col.E[c][cs0 + 2 * cs1 + z] = e * r.cph[1][1];
          }
        }
      }
      if (!sync()) return;
    }
#pragma unroll 1
    for (; n < n_end; ++n) {
      const bool through = n + 1 < n_end;  // E ghosts written through, except after the launch's last step
      // ---- H phase ----
      unsigned zc = z00, ymc = ym00, xmc = xm00;
      for (unsigned w = t0; w < n_work; w += tstride, zc += dz, ymc += dym + (zc >= un2 ? 1u : 0u),
                    zc -= zc >= un2 ? un2 : 0u, xmc += dxm + (ymc >= ny ? 1u : 0u), ymc -= ymc >= ny ? ny : 0u) {
        if (w < n_main) {
          // periodic x and y: every component is stepped at every interior (x, y); along z, H_x and H_y
          // stop one node short of the last plane (in_h_region), and only z carries CPML
          const int z = (int)zc;
          const int x = 1 + (int)xmc, y = 1 + (int)ymc;
          const unsigned p = (unsigned)x * us0 + (unsigned)y * us1 + (unsigned)z;
          const bool zin = z <= n2 - 2;
          const F e0 = g.E[0][p], e1 = g.E[1][p], e2 = g.E[2][p];
          const F e2y = g.E[2][p + us1], e2x = g.E[2][p + us0], e1x = g.E[1][p + us0], e0y = g.E[0][p + us1];
          const F e1z = zin ? g.E[1][p + 1] : e1, e0z = zin ? g.E[0][p + 1] : e0;
          // (a, b) per component: H_c -= cH (dE_{d2}/dd1 - dE_{d1}/dd2)
          const F av[3] = {e2y - e2, e0z - e0, e1x - e1};
          const F bv[3] = {e1z - e1, e2x - e2, e0y - e0};
          long long q = 0;
          const int side = zin ? slab_z<1>(g, 0, x, y, z, &q) : -1;
          // every load of the node before its first store (the stores could alias them for the compiler)
          F h0v[3] = {g.H[0][p], g.H[1][p], g.H[2][p]};
          const PmlAxis<F>& pz = g.pml[2];
          F psi0[2] = {zero<F>(), zero<F>()};
          R pb = R(0), pc = R(0), pk = R(0);
          if (side >= 0) {
            psi0[0] = pz.psi[1][0][side][q];
            psi0[1] = pz.psi[1][1][side][q];
            pb = pz.b[1][z];
            pc = pz.c[1][z];
            pk = pz.k[1] ? pz.k[1][z] : R(0);
          }
          F inc[2] = {zero<F>(), zero<F>()};
          const bool plane = z == r.k_src - 1;
          if (plane) {
            const F ph = r.phase[(x - 1) * (int)ny + (y - 1)];
            inc[0] = ph * r.col.E[1][ccol + r.k_src];
            inc[1] = ph * r.col.E[0][ccol + r.k_src];
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            if (c < 2 && !zin) continue;
            const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
            const F curl = g.uniform ? (av[c] - bv[c]) : (av[c] * g.inv_d[d1] - bv[c] * g.inv_d[d2]);
            F h = h0v[c];
            h = h - curl * g.cH;
            if (c < 2 && side >= 0) {  // apply_cpml's arithmetic for the z slab
              const F der = c == 1 ? av[c] : bv[c];
              R sgn = (2 == d1) ? R(1) : R(-1);
              sgn = -sgn;
              R sc = g.uniform ? g.cH : g.cH / pz.div;
              sc = sgn * sc;
              F psi = psi0[c] * pb;
              if (pz.k[1]) h += (sc * pk) * der;
              psi += der * (sc * pc);
              pz.psi[1][c][side][q] = psi;
              h += psi;
            }
            if (plane && c < 2) h = c == 0 ? h - r.cH * inc[0] : h + r.cH * inc[1];  // correct_H
            g.H[c][p] = h;
            // low ghosts (x = 0 from x = n0 - 2, then y = 0 from y = n1 - 2, and the corner)
            if (x == n0 - 2) {
              const F gx = h * r.gph[0][0];
              g.H[c][y * s1 + z] = gx;
              if (y == n1 - 2) g.H[c][z] = gx * r.gph[1][0];
            }
            if (y == n1 - 2) g.H[c][x * s0 + z] = h * r.gph[1][0];
          }
        } else {  // the column's node (1, 1, z)
          const int z = (int)(w - n_main);
          const YeeArgs<F>& cg = r.col;
          update_h_node(cg, 1, 1, z);
          const long long p = ccol + z;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const F h = cg.H[c][p];
            const F gx = h * r.cph[0][0];
            cg.H[c][cs1 + z] = gx;
            cg.H[c][z] = gx * r.cph[1][0];
            cg.H[c][cs0 + z] = h * r.cph[1][0];
          }
        }
      }
      if (!sync()) return;
      // ---- E phase ----
      const R w_src = r.wave[n];
      zc = z00, ymc = ym00, xmc = xm00;
      for (unsigned w = t0; w < n_work; w += tstride, zc += dz, ymc += dym + (zc >= un2 ? 1u : 0u),
                    zc -= zc >= un2 ? un2 : 0u, xmc += dxm + (ymc >= ny ? 1u : 0u), ymc -= ymc >= ny ? ny : 0u) {
        if (w < n_main) {
          // along z, E_x and E_y are stepped on [1, n2 - 2], E_z on [0, n2 - 2] (in_e_region)
          const int z = (int)zc;
          const int x = 1 + (int)xmc, y = 1 + (int)ymc;
          const unsigned p = (unsigned)x * us0 + (unsigned)y * us1 + (unsigned)z;
          if (z > n2 - 2) continue;
          const bool zlo = z >= 1;
          const F h0 = g.H[0][p], h1 = g.H[1][p], h2 = g.H[2][p];
          const F h2y = g.H[2][p - us1], h2x = g.H[2][p - us0], h1x = g.H[1][p - us0], h0y = g.H[0][p - us1];
          const F h1z = zlo ? g.H[1][p - 1] : h1, h0z = zlo ? g.H[0][p - 1] : h0;
          // (a, b) per component: E_c += cbE_c (dH_{d2}/dd1 - dH_{d1}/dd2)
          const F av[3] = {h2 - h2y, h0 - h0z, h1 - h1x};
          const F bv[3] = {h1 - h1z, h2 - h2x, h0 - h0y};
          long long q = 0;
          const int side = zlo ? slab_z<0>(g, 0, x, y, z, &q) : -1;
          // every load of the node before its first store
          const F e0v[3] = {g.E[0][p], g.E[1][p], g.E[2][p]};
          const R cbv[3] = {g.cbE[0][p], g.cbE[1][p], g.cbE[2][p]};
          const PmlAxis<F>& pz = g.pml[2];
          F psi0[2] = {zero<F>(), zero<F>()};
          R pb = R(0), pc = R(0), pk = R(0);
          if (side >= 0) {
            psi0[0] = pz.psi[0][0][side][q];
            psi0[1] = pz.psi[0][1][side][q];
            pb = pz.b[0][z];
            pc = pz.c[0][z];
            pk = pz.k[0] ? pz.k[0][z] : R(0);
          }
          F inc[2] = {zero<F>(), zero<F>()};
          const bool plane = z == r.k_src;
          if (plane) {
            const F ph = r.phase[(x - 1) * (int)ny + (y - 1)];
            inc[0] = ph * r.col.H[1][ccol + r.k_src - 1];
            inc[1] = ph * r.col.H[0][ccol + r.k_src - 1];
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            if (c < 2 && !zlo) continue;
            const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
            const F curl = g.uniform ? (av[c] - bv[c]) : (av[c] * g.inv_d[d1] - bv[c] * g.inv_d[d2]);
            const R cb = cbv[c];
            F e = e0v[c];
            e = e + curl * cb;
            if (c < 2 && side >= 0) {  // apply_cpml's arithmetic for the z slab
              const F der = c == 1 ? av[c] : bv[c];
              const R sgn = (2 == d1) ? R(1) : R(-1);
              R sc = g.uniform ? cb : cb / pz.div;
              sc = sgn * sc;
              F psi = psi0[c] * pb;
              if (pz.k[0]) e += (sc * pk) * der;
              psi += der * (sc * pc);
              pz.psi[0][c][side][q] = psi;
              e += psi;
            }
            if (plane && c < 2) e = c == 0 ? e + r.cE * inc[0] : e - r.cE * inc[1];  // correct_E
            nonfinite += e.re * R(0) + e.im * R(0);
            g.E[c][p] = e;
            // high ghosts (x = n0 - 1 from x = 1, then y = n1 - 1 from y = 1, and the corner)
            if (!through) continue;
            if (x == 1) {
              const F gx = e * r.gph[0][1];
              g.E[c][(long long)(n0 - 1) * s0 + y * s1 + z] = gx;
              if (y == 1) g.E[c][(long long)(n0 - 1) * s0 + (long long)(n1 - 1) * s1 + z] = gx * r.gph[1][1];
            }
            if (y == 1) g.E[c][x * s0 + (long long)(n1 - 1) * s1 + z] = e * r.gph[1][1];
          }
        } else {  // the column's node (1, 1, z), then the sheet, then its ghosts
          const int z = (int)(w - n_main);
          const YeeArgs<F>& cg = r.col;
          update_e_node(cg, 1, 1, z);
          const long long p = ccol + z;
          if (z == r.k_launch) {
            cg.E[0][p] = cg.E[0][p] + r.amp0 * w_src;
            cg.E[1][p] = cg.E[1][p] + r.amp1 * w_src;
          }
#pragma unroll
          for (int c = 0; c < 3 && through; ++c) {
            const F e = cg.E[c][p];
            const F gx = e * r.cph[0][1];
            cg.E[c][2 * cs0 + cs1 + z] = gx;
            cg.E[c][2 * cs0 + 2 * cs1 + z] = gx * r.cph[1][1];
            cg.E[c][cs0 + 2 * cs1 + z] = e * r.cph[1][1];
          }
        }
      }
      if (__any_sync(0xffffffffu, nonfinite != R(0)) && (threadIdx.x & 31) == 0) atomicExch(r.status, kBatchNonFinite);
      if (!sync()) return;
      if (*reinterpret_cast<volatile int*>(r.status) == kBatchNonFinite) {  // every CTA reads it after the barrier
        n_end = n + 1;
        break;
      }
      // ---- the conformal off-diagonal gather (after the whole E update, as lightsmith adds it) ----
      if (r.od_n > 0) {
        const long long cells = (long long)n0 * s0;
        for (long long q = t0; q < r.od_n; q += tstride) {
          const long long tt = r.od_e[q];
          F acc = zero<F>();
          for (int kk = 0; kk < r.od_width; ++kk)
            acc = acc + r.od_w[q * r.od_width + kk] * g.H[0][r.od_h[q * r.od_width + kk]];
          const F e = g.E[0][tt] + acc;
          g.E[0][tt] = e;
          if (!through) continue;
          const int c = (int)(tt / cells);
          const long long rem = tt - c * cells;
          const int x = (int)(rem / s0), y = (int)((rem / s1) % n1);
          const long long z = rem % s1;
          if (x == 1) {
            const F gx = e * r.gph[0][1];
            g.E[c][(long long)(n0 - 1) * s0 + y * s1 + z] = gx;
            if (y == 1) g.E[c][(long long)(n0 - 1) * s0 + (long long)(n1 - 1) * s1 + z] = gx * r.gph[1][1];
          }
          if (y == 1) g.E[c][x * s0 + (long long)(n1 - 1) * s1 + z] = e * r.gph[1][1];
        }
        if (!sync()) return;
      }
      // ---- DFT sample after every dft_stride steps ----
      if ((n + 1) % r.stride == 0) {
        for (int m = 0; m < r.n_mon; ++m) {
          const MonArgs<F>& mon = r.mon[m];
          for (long long i = t0; i < mon.ne + mon.nh; i += tstride) batch_sample_point(mon, i, n + 1);
        }
        if (!sync()) return;
      }
    }
    if (rank == 0 && threadIdx.x == 0) *r.nstep = n_end;
    if (!sync()) return;  // the counter is written and every CTA is done with the descriptor
  }
}

}  // namespace lsfdtd
