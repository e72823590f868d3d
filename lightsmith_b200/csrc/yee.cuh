// Yee E/H curl updates with the CPML psi terms fused in, and the periodic (Bloch) ghost-plane refresh.
//
// Step semantics follow lightsmith's engine (backends/_fdtd/engine.py): H_c -= cH (dE_{d2}/dd1 - dE_{d1}/dd2)
// with forward differences over H_c's stepped region (engine.py:630-635), E_c += cbE_c (dH_{d2}/dd1 -
// dH_{d1}/dd2) with backward differences over E_c's region (engine.py:645-652), then the CPML terms of each
// axis d != c: psi = b psi + c' der; F += k' der (kappa > 1 only); F += psi (engine.py:636-643, 656-663).
// The derivative of a CPML term along d1 is the curl's own difference a, along d2 its b, so the psi update
// reads no field value the curl did not already load.
#pragma once

#include "common.cuh"

namespace lsfdtd {

// One CPML axis: graded 1D profiles over the axis' node (E) and half-integer (H) positions, and the psi slabs.
template <typename F>
struct PmlAxis {
  using R = typename real_of<F>::type;
  int on;
  const R* b[2];   // [E, H] profiles, length n_d
  const R* c[2];
  const R* k[2];   // (1/kappa - 1), null where kappa == 1 everywhere
  R div;           // non-cubic cells: c' and k' carry 1/dx_d (1 for cubic cells)
  // psi slab per [field E/H][component][side lo/hi]: start index along d, length, storage
  int start[2][3][2];
  int len[2][3][2];
  F* psi[2][3][2];
};

template <typename F>
struct YeeArgs {
  using R = typename real_of<F>::type;
  int n[3];
  int periodic[3];
  int mirror[3];   // per axis: 0, or +1 / -1 for a symmetric / antisymmetric mirror plane at node 1
  int uniform;     // cubic cells: coefficients carry dt/dx and differences are not rescaled
  R inv_d[3];
  R cH;
  F* E[3];
  F* H[3];
  const R* cbE[3];  // per component, full grid (the three may alias one array)
  PmlAxis<F> pml[3];
  // nodes [in_lo, in_hi) per axis stepped for every component of both fields and outside every CPML slab
  // (empty when unset): there the in-place kernels need no region test and no CPML term
  int in_lo[3], in_hi[3];
};

// mir: the mirror planes (null: none); along a mirror axis E_c starts at node 2 when it is tangential to an
// antisymmetric plane, else at 1 (engine.py:41-60)
__device__ __forceinline__ bool in_e_region(int c, const int* x, const int* n, const int* per,
                                            const int* mir = nullptr) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int lo = (per[a] || a != c) ? 1 : 0;
    if (mir && mir[a]) lo = (mir[a] < 0 && a != c) ? 2 : 1;
    if (x[a] < lo || x[a] >= n[a] - 1) return false;
  }
  return true;
}

// H_c along a mirror axis starts at node 2 when it is normal to an antisymmetric plane, else at 1
__device__ __forceinline__ bool in_h_region(int c, const int* x, const int* n, const int* per,
                                            const int* mir = nullptr) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int lo = per[a] ? 1 : 0;
    int hi = per[a] ? n[a] - 1 : (a == c ? n[a] : n[a] - 1);
    if (mir && mir[a]) lo = (mir[a] < 0 && a == c) ? 2 : 1;
    if (x[a] < lo || x[a] >= hi) return false;
  }
  return true;
}

// index of a psi slab entry: the cell's coordinates with axis d replaced by the offset into the slab
__device__ __forceinline__ long long psi_index(const int* x, const int* n, int d, int off, int len) {
  int i0 = d == 0 ? off : x[0];
  int i1 = d == 1 ? off : x[1];
  int i2 = d == 2 ? off : x[2];
  int n1 = d == 1 ? len : n[1];
  int n2 = d == 2 ? len : n[2];
  return ((long long)i0 * n1 + i1) * n2 + i2;
}

// F += CPML terms of component c along every axis d != c. der1 / der2 are the raw differences along
// d1 / d2; scale is the curl coefficient of this node (cH, or cbE of the node), FLD 0 = E, 1 = H.
// UNI: 1 cubic cells, 0 not, -1 as the grid's uniform flag says (known when the caller is compiled or not)
template <int FLD, int UNI = -1, typename F>
__device__ __forceinline__ void apply_cpml(F& v, const YeeArgs<F>& g, int c, const int* x, F der1, F der2,
                                           typename real_of<F>::type scale) {
  using R = typename real_of<F>::type;
  const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d == c) continue;
    const PmlAxis<F>& p = g.pml[d];
    if (!p.on) continue;
    const F der = d == d1 ? der1 : der2;
    // curl sign of the term: E_c gets +dH_{d2}/dd1 - dH_{d1}/dd2, H_c the opposite
    R sgn = (d == d1) ? R(1) : R(-1);
    if (FLD == 1) sgn = -sgn;
    const int u = x[d];
    const bool uni = UNI < 0 ? (bool)g.uniform : UNI == 1;
    R s = uni ? scale : scale / p.div;
    s = sgn * s;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const int st = p.start[FLD][c][side], ln = p.len[FLD][c][side];
      if (u < st || u >= st + ln) continue;
      F* ps = p.psi[FLD][c][side] + psi_index(x, g.n, d, u - st, ln);
      F psi = *ps * p.b[FLD][u];
      if (p.k[FLD]) v += (s * p.k[FLD][u]) * der;
      psi += der * (s * p.c[FLD][u]);
      *ps = psi;
      v += psi;
    }
  }
}

// H update of node (i, j, k), all three components (in place); UNI as apply_cpml's
template <typename F, int UNI = -1>
__device__ __forceinline__ void update_h_node(const YeeArgs<F>& g, int i, int j, int k) {
  const bool uni = UNI < 0 ? (bool)g.uniform : UNI == 1;
  const int x[3] = {i, j, k};
  const long long s1 = g.n[2], s0 = (long long)g.n[1] * g.n[2];
  const long long p = i * s0 + j * s1 + k;
  const long long step[3] = {s0, s1, 1};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!in_h_region(c, x, g.n, g.periodic, g.mirror)) continue;
    const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    const F a = g.E[d2][p + step[d1]] - g.E[d2][p];
    const F b = g.E[d1][p + step[d2]] - g.E[d1][p];
    F curl = uni ? (a - b) : (a * g.inv_d[d1] - b * g.inv_d[d2]);
    F h = g.H[c][p];
    h = h - curl * g.cH;
    apply_cpml<1, UNI>(h, g, c, x, a, b, g.cH);
    g.H[c][p] = h;
  }
}

// E update of node (i, j, k), all three components (in place); UNI as apply_cpml's
template <typename F, int UNI = -1>
__device__ __forceinline__ void update_e_node(const YeeArgs<F>& g, int i, int j, int k) {
  using R = typename real_of<F>::type;
  const bool uni = UNI < 0 ? (bool)g.uniform : UNI == 1;
  const int x[3] = {i, j, k};
  const long long s1 = g.n[2], s0 = (long long)g.n[1] * g.n[2];
  const long long p = i * s0 + j * s1 + k;
  const long long step[3] = {s0, s1, 1};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!in_e_region(c, x, g.n, g.periodic, g.mirror)) continue;
    const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    const F a = g.H[d2][p] - g.H[d2][p - step[d1]];
    const F b = g.H[d1][p] - g.H[d1][p - step[d2]];
    F curl = uni ? (a - b) : (a * g.inv_d[d1] - b * g.inv_d[d2]);
    const R cb = g.cbE[c][p];
    F e = g.E[c][p];
    e = e + curl * cb;
    apply_cpml<0, UNI>(e, g, c, x, a, b, cb);
    g.E[c][p] = e;
  }
}

template <typename F>
__device__ __forceinline__ bool in_inner(const YeeArgs<F>& g, int i, int j, int k) {
  return i >= g.in_lo[0] && i < g.in_hi[0] && j >= g.in_lo[1] && j < g.in_hi[1] && k >= g.in_lo[2] &&
         k < g.in_hi[2];
}

// H update: one thread per node (i, j, k), all three components; one instantiation per cell shape (UNI 1:
// cubic cells). A warp whose nodes are all inner takes the stencil without region tests or CPML terms (the
// same arithmetic in the same order as update_h_node's for such nodes)
template <typename F, int UNI>
__global__ void __launch_bounds__(256) k_update_h(const __grid_constant__ YeeArgs<F> g) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (k >= g.n[2] || j >= g.n[1]) return;
  const int i = blockIdx.z;
  if (__all_sync(__activemask(), in_inner(g, i, j, k))) {
    const bool uni = UNI < 0 ? (bool)g.uniform : UNI == 1;
    const long long s1 = g.n[2], s0 = (long long)g.n[1] * g.n[2];
    const long long p = i * s0 + j * s1 + k;
    const long long step[3] = {s0, s1, 1};
    F e0[3], e1[3][3];  // E at the node and at its +1 neighbours, every load before the first store
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      e0[c] = g.E[c][p];
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (d != c) e1[c][d] = g.E[c][p + step[d]];
    }
    F h[3] = {g.H[0][p], g.H[1][p], g.H[2][p]};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
      const F a = e1[d2][d1] - e0[d2];
      const F b = e1[d1][d2] - e0[d1];
      const F curl = uni ? (a - b) : (a * g.inv_d[d1] - b * g.inv_d[d2]);
      g.H[c][p] = h[c] - curl * g.cH;
    }
    return;
  }
  update_h_node<F, UNI>(g, i, j, k);
}

// E update: one thread per node, all three components; inner warps as in k_update_h
template <typename F, int UNI>
__global__ void __launch_bounds__(256) k_update_e(const __grid_constant__ YeeArgs<F> g) {
  using R = typename real_of<F>::type;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (k >= g.n[2] || j >= g.n[1]) return;
  const int i = blockIdx.z;
  if (__all_sync(__activemask(), in_inner(g, i, j, k))) {
    const bool uni = UNI < 0 ? (bool)g.uniform : UNI == 1;
    const long long s1 = g.n[2], s0 = (long long)g.n[1] * g.n[2];
    const long long p = i * s0 + j * s1 + k;
    const long long step[3] = {s0, s1, 1};
    F h0[3], h1[3][3];  // H at the node and at its -1 neighbours
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      h0[c] = g.H[c][p];
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (d != c) h1[c][d] = g.H[c][p - step[d]];
    }
    F e[3] = {g.E[0][p], g.E[1][p], g.E[2][p]};
    R cb[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) cb[c] = g.cbE[c][p];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
      const F a = h0[d2] - h1[d2][d1];
      const F b = h0[d1] - h1[d1][d2];
      const F curl = uni ? (a - b) : (a * g.inv_d[d1] - b * g.inv_d[d2]);
      g.E[c][p] = e[c] + curl * cb[c];
    }
    return;
  }
  update_e_node<F, UNI>(g, i, j, k);
}

// Periodic ghost planes of one axis: dst plane <- src plane times a Bloch phase (engine.py:595-611).
template <typename F>
__global__ void k_ghost(F* f0, F* f1, F* f2, int n0, int n1, int n2, int axis, int dst, int src, double ph_re,
                        double ph_im) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  // the plane normal to `axis`: enumerate its two other coordinates
  int na = axis == 0 ? n1 : n0, nb = axis == 2 ? n1 : n2;
  if (t >= 3 * na * nb) return;
  const int comp = t / (na * nb);
  const int r = t % (na * nb);
  const int u = r / nb, v = r % nb;
  int xd[3], xs[3];
  if (axis == 0) { xd[0] = dst; xs[0] = src; xd[1] = xs[1] = u; xd[2] = xs[2] = v; }
  else if (axis == 1) { xd[1] = dst; xs[1] = src; xd[0] = xs[0] = u; xd[2] = xs[2] = v; }
  else { xd[2] = dst; xs[2] = src; xd[0] = xs[0] = u; xd[1] = xs[1] = v; }
  F* f = comp == 0 ? f0 : (comp == 1 ? f1 : f2);
  const long long pd = ((long long)xd[0] * n1 + xd[1]) * n2 + xd[2];
  const long long ps = ((long long)xs[0] * n1 + xs[1]) * n2 + xs[2];
  f[pd] = apply_phase<F>(f[ps], ph_re, ph_im);
}

// Conformal off-diagonal 1/eps terms (engine.py:653-655): row t adds sum_k w[t][k] H[h[t][k]] to E[e[t]]; the
// targets are distinct, so one thread per row needs no atomics. E and H are the flat component-stacked fields.
template <typename F>
__global__ void k_offdiag(const long long* e, const long long* h, const F* w, long long n, int width, F* E,
                          const F* H) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const long long* hr = h + t * width;
  const F* wr = w + t * width;
  F acc = zero<F>();
  for (int k = 0; k < width; ++k) acc = acc + wr[k] * H[hr[k]];
  E[e[t]] = E[e[t]] + acc;
}

// Symmetric (PMC) mirror plane along `axis`: the two tangential H components' ghost plane 0 set to minus
// plane 1, before an E update (engine.py:290-298, 649-650). One thread per node of the plane and component.
template <typename F>
__global__ void k_mirror_ghost(F* h0, F* h1, F* h2, int n0, int n1, int n2, int axis) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int na = axis == 0 ? n1 : n0, nb = axis == 2 ? n1 : n2;  // the plane's two other axes, in order
  const long long per = (long long)na * nb;
  if (t >= 2 * per) return;
  const int comp = (axis + 1 + (int)(t / per)) % 3;  // a tangential component
  const long long r = t % per;
  const int u = (int)(r / nb), v = (int)(r % nb);
  long long pg, ps;  // the node on plane 0 along axis, and its image on plane 1
  if (axis == 0) {
    pg = (long long)u * n2 + v;
    ps = (long long)n1 * n2 + pg;
  } else if (axis == 1) {
    pg = (long long)u * n1 * n2 + v;
    ps = pg + n2;
  } else {
    pg = ((long long)u * n1 + v) * n2;
    ps = pg + 1;
  }
  F* f = comp == 0 ? h0 : (comp == 1 ? h1 : h2);
  f[pg] = zero<F>() - f[ps];
}

}  // namespace lsfdtd
