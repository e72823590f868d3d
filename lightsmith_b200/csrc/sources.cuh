// Source kernels: table-fed TF/SF box, point dipole, 1D-fed TF/SF line, Bloch column plane, port mode source.
//
// Every kernel reads the completed-step counter n from device memory, so a captured CUDA graph replays the
// right time. Corrections that reach one node from several box faces are summed by the one thread that owns
// the node (a CSR list per target node, in the reference's face order): no atomics, deterministic results.
#pragma once

#include "common.cuh"

namespace lsfdtd {

// quintic Lagrange interpolation on the stencil -2..3: denominators prod_{k != j} (x_j - x_k)
// (backends/_fdtd/layered.py:164-187)
template <typename R>
__device__ __forceinline__ R table_read(const R* T, long long n, long long i0, R u0, long long base, int m,
                                        long long cmax) {
  const long long q = n + i0;
  const long long r = q % m;
  long long c = (q - r) / m;
  if (c > cmax) c = cmax;
  const R u = (R(r) + u0) / R(m);
  R d[6];
#pragma unroll
  for (int s = 0; s < 6; ++s) d[s] = u - R(s - 2);
  const R den[6] = {R(-120), R(24), R(-12), R(12), R(-24), R(120)};
  const R* t = T + base + c;
  R out = R(0);
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    R w = R(1);
    bool first = true;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (k == j) continue;
      w = first ? d[k] : w * d[k];
      first = false;
    }
    const R term = (w / den[j]) * t[j];
    out = j == 0 ? term : out + term;
  }
  return out;
}

template <typename R>
struct TableArgs {
  const R* T;
  int m;
  long long cmax;
  long long n_nodes;
  const long long* nodes;
  const long long* offsets;  // CSR: entries of node t are offsets[t] .. offsets[t+1]
  const long long* base;
  const long long* i0;
  const R* u0;
  const R* coef;
  R* target;                 // flat E or H
  const long long* nstep;
};

template <typename R>
__global__ void k_table_correct(TableArgs<R> a) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_nodes) return;
  const long long n = *a.nstep;
  const long long node = a.nodes[t];
  R v = a.target[node];
  for (long long e = a.offsets[t]; e < a.offsets[t + 1]; ++e)
    v = v + a.coef[e] * table_read(a.T, n, a.i0[e], a.u0[e], a.base[e], a.m, a.cmax);
  a.target[node] = v;
}

// the step's correction values of one kind in the source's slab order, for the fused pass to add as it steps
// (k_table_correct adds them node by node instead): vals[e] = coef * T(n) of the entry at CSR position perm[e]
template <typename R>
__global__ void k_table_values(TableArgs<R> a, const long long* perm, long long n_entries, R* vals) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_entries) return;
  const long long q = perm[e];
  vals[e] = a.coef[q] * table_read(a.T, *a.nstep, a.i0[q], a.u0[q], a.base[q], a.m, a.cmax);
}

// the incident-reference view: E_inc (3 components) at the end of the step
template <typename R>
__global__ void k_table_view(const R* Tinc, int m, long long cmax, const long long* base, const long long* i0,
                             const R* u0, R* view, const long long* nstep) {
  const int c = threadIdx.x;
  if (c >= 3) return;
  view[c] = table_read(Tinc, *nstep, i0[c], u0[c], base[c], m, cmax);
}

// point dipole: E[idx] -= coef * wave[n]  (backends/_fdtd/emission.py:139-140)
template <typename R>
__global__ void k_dipole(R* E, const long long* idx, const R* coef, int n_idx, const R* wave,
                         const long long* nstep) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_idx) return;
  const R w = wave[*nstep];
  E[idx[t]] = E[idx[t]] - coef[t] * w;
}

// 1D-fed TF/SF corrections: target += coef * (src[i0] + w (src[i0 + 1] - src[i0]))  (tfsf.py:184-193)
template <typename R>
struct LineArgs {
  long long n_nodes;
  const long long* nodes;
  const long long* offsets;
  const long long* i0;
  const R* w;
  const R* coef;
  const R* src;
  R* target;
};

template <typename R>
__global__ void k_line_correct(LineArgs<R> a) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_nodes) return;
  const long long node = a.nodes[t];
  R v = a.target[node];
  for (long long e = a.offsets[t]; e < a.offsets[t + 1]; ++e) {
    const R s0 = a.src[a.i0[e]];
    const R s = s0 + a.w[e] * (a.src[a.i0[e] + 1] - s0);
    v = v + a.coef[e] * s;
  }
  a.target[node] = v;
}

// 1D line, H half step: H[i] = H[i] da[i] - db[i] (E[i+1] - E[i]), i < M - 1  (tfsf.py:201-204)
template <typename R>
__global__ void k_line_h(R* E, R* H, const R* da, const R* db, int M) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M - 1) return;
  R h = H[i] * da[i];
  H[i] = h - db[i] * (E[i + 1] - E[i]);
}

// 1D line, E half step and the soft source at m_src  (tfsf.py:206-211)
template <typename R>
__global__ void k_line_e(R* E, R* H, const R* ca, const R* cb, int M, int m_src, const R* wave,
                         const long long* nstep) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 1 || i >= M - 1) return;
  R e = E[i] * ca[i];
  e = e - cb[i] * (H[i] - H[i - 1]);
  if (i == m_src) e = e + wave[*nstep];
  E[i] = e;
}

// Bloch column plane corrections (tfsf.py:274-286). kind 0: H on plane k_src - 1 from the column's E at
// k_src; kind 1: E on plane k_src from the column's H at k_src - 1. The column is 3 x 3 x nz, its real cell
// at (1, 1).
template <typename F>
__global__ void k_column_plane(F* t0, F* t1, const F* c0, const F* c1, const F* phase, int nx, int ny, int n1, int n2,
                               int k_src, int ncz, typename real_of<F>::type coef, int kind) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nx * ny) return;
  const int x = t / ny, y = t % ny;
  const F ph = phase[t];
  const long long col = (1LL * 3 + 1) * ncz;  // node (1, 1, 0) of the column
  if (kind == 0) {
    const long long p = ((long long)(x + 1) * n1 + (y + 1)) * n2 + (k_src - 1);
    const F inc1 = ph * c1[col + k_src];  // E_y
    const F inc0 = ph * c0[col + k_src];  // E_x
    t0[p] = t0[p] - coef * inc1;
    t1[p] = t1[p] + coef * inc0;
  } else {
    const long long p = ((long long)(x + 1) * n1 + (y + 1)) * n2 + k_src;
    const F inc1 = ph * c1[col + k_src - 1];  // H_y
    const F inc0 = ph * c0[col + k_src - 1];  // H_x
    t0[p] = t0[p] + coef * inc1;
    t1[p] = t1[p] - coef * inc0;
  }
}

// the column's current sheet: E_x, E_y at (1, 1, k_launch) += amp * wave[n]  (tfsf.py:291-296)
template <typename F>
__global__ void k_column_sheet(F* e0, F* e1, int ncz, int k_launch, F amp0, F amp1,
                               const typename real_of<F>::type* wave, const long long* nstep) {
  if (threadIdx.x != 0) return;
  const typename real_of<F>::type w = wave[*nstep];
  const long long p = (1LL * 3 + 1) * ncz + k_launch;
  e0[p] = e0[p] + amp0 * w;
  e1[p] = e1[p] + amp1 * w;
}

// port mode source: F[idx[t]] += sum_r m[t, r] tab[n, r]  (ports.py:368-372)
template <typename R>
__global__ void k_mode(R* F, const long long* idx, const R* m, const R* tab, int n_rows, int r, const long long* nstep) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_rows) return;
  const R* row = tab + (*nstep) * r;
  R s = R(0);
  for (int k = 0; k < r; ++k) s = k == 0 ? m[(long long)t * r] * row[0] : s + m[(long long)t * r + k] * row[k];
  F[idx[t]] = F[idx[t]] + s;
}

__global__ void k_bump(long long* nstep) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *nstep += 1;
}

}  // namespace lsfdtd
