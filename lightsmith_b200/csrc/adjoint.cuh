// The discrete adjoint of the FDTD step (real fields), for gradients of a DFT objective.
//
// A forward step is linear in the state (E, H and the CPML psi): H^{n+1/2} from H^{n-1/2} and E^n
// (update_h_node), then E^{n+1} from E^n and H^{n+1/2} (update_e_node); sources add terms that do not depend
// on the fields. The reverse step applies the transposes in the opposite order to the adjoint state
// (Ebar, Hbar, psibar): first the E update's, which adds to Hbar, then the H update's, which adds to Ebar.
//
// Per E node p and component c in its stepped region, the update reads the differences a = H_{d2}(p) -
// H_{d2}(p - e_{d1}) and b = H_{d1}(p) - H_{d1}(p - e_{d2}); its transpose gives the adjoints abar(c, p) and
// bbar(c, p) of those differences (the curl coefficient times Ebar_c(p), plus the CPML terms of the axis the
// difference runs along: psibar_total = psibar + Ebar, dbar = psibar_total s c + Ebar s k, and the psi's own
// adjoint psibar <- b psibar_total). A difference's adjoint lands on the two H nodes it reads, so the kernel
// gathers, for H node q: Hbar_j(q) += abar(j+1, q) - abar(j+1, q + e_{j+2}) + bbar(j+2, q) - bbar(j+2,
// q + e_{j+1}) (indices mod 3). The H update's transpose is the same with forward differences. psibar is
// double buffered (each kernel reads the step's old values, also at neighbours, and writes the new ones).
// A warp whose nodes and neighbours are all interior (stepped, in no slab) takes the plain stencil; any
// other warp takes the stencil with the stepped-region tests as masks plus the slab terms per axis.
// A periodic axis steps nodes 1 .. n-2 of both fields between two ghost planes, which the forward step fills
// by copies (E's high ghost n-1 from plane 1 before the H update, H's low ghost 0 from plane n-2 before the
// E update); their transposes (k_adj_ghost) move a ghost plane's adjoint onto its source plane and clear it,
// after the transposed E update for H and after the transposed H update for E. A mirror plane at node 1
// narrows the stepped regions (the masks follow in_e_region and in_h_region); a symmetric one also fills
// tangential H's plane 0 with minus plane 1 before the E update, transposed by k_adj_mirror. The conformal
// off-diagonal terms, added to E after its update from the same H, are transposed (k_adj_offdiag) before it.
//
// The objective's adjoint source (the DFT samples' weights times e^{i omega t}) is added to Ebar and Hbar at
// the steps the monitor sampled, before that step's reverse. The gradient with respect to the E curl
// coefficient, dJ/dcbE_c(p) = sum_n Ebar_c^{n+1}(p) curl_c(H^{n+1/2})(p), is accumulated (in double) over a
// box of nodes away from the CPML slabs, from H^{n+1/2} of the box (with its low halo) recomputed forward.
#pragma once

#include "ade.cuh"
#include "common.cuh"
#include "tensor.cuh"
#include "yee.cuh"

namespace lsfdtd {

template <typename R>
struct AdjArgs {
  YeeArgs<R> y;             // the forward engine's coefficients, CPML profiles and slab extents
  R* Eb[3];                 // adjoint fields
  R* Hb[3];
  R* pe_old[3][3][2];       // psibar of E [axis][component][side]: read (this step) / written (the step before)
  R* pe_new[3][3][2];
  R* ph_old[3][3][2];       // psibar of H
  R* ph_new[3][3][2];
  int box_lo[3], box_hi[3];  // gradient box (nodes)
  int ein_lo[3], ein_hi[3];  // nodes stepped for every E component and outside every E slab, per axis
  int hin_lo[3], hin_hi[3];  // the same for H
  const R* hist;            // H^{n+1/2} over [box_lo - 1, box_hi) per component
  double* grad;             // dJ/dcbE per component over the box
};

// slab of axis d holding coordinate u (sides share the extent of both components c != d), or -1
template <int FLD, typename R>
__device__ __forceinline__ int adj_side(const PmlAxis<R>& pm, int c, int u) {
  if (pm.len[FLD][c][0] > 0 && u >= pm.start[FLD][c][0] && u < pm.start[FLD][c][0] + pm.len[FLD][c][0]) return 0;
  if (pm.len[FLD][c][1] > 0 && u >= pm.start[FLD][c][1] && u < pm.start[FLD][c][1] + pm.len[FLD][c][1]) return 1;
  return -1;
}

// Transposed E update at H node x for a warp with any node outside the interior: the curl stencil with the
// stepped-region tests as masks, then, per axis d whose slab holds x or x + e_d, the CPML terms of the two
// components c != d (warp-uniform branches for d = 0, 1), and x's own E psibar.
template <bool UNI, typename R>
__device__ __forceinline__ void adj_e_lean(const AdjArgs<R>& A, const int* x, long long p, const long long* st,
                                           R* acc) {
  const YeeArgs<R>& g = A.y;
  // E_c's stepped range along each axis (in_e_region): [1, n - 1), or [0, n - 1) along c itself on a
  // non-periodic axis; along a mirror axis from node 1, or from 2 for the tangential components of an
  // antisymmetric plane. okc: x in range along the component's own axis, oko: along another, nb: x + e_a
  bool okc[3], oko[3], nb[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int lo_oth = g.mirror[a] < 0 ? 2 : 1, lo_own = (g.periodic[a] || g.mirror[a]) ? 1 : 0;
    oko[a] = x[a] >= lo_oth && x[a] < g.n[a] - 1;
    okc[a] = x[a] >= lo_own && x[a] < g.n[a] - 1;
    nb[a] = x[a] + 1 >= lo_oth && x[a] + 1 < g.n[a] - 1;
  }
  R eb0[3], cb0[3], eb1[3][3], cb1[3][3];
  bool m0[3], m1[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    m0[c] = okc[c] && oko[d1] && oko[d2];
    eb0[c] = m0[c] ? A.Eb[c][p] : R(0);
    cb0[c] = m0[c] ? g.cbE[c][p] : R(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (d == c) continue;
      m1[c][d] = nb[d] && okc[c] && oko[3 - c - d];
      eb1[c][d] = m1[c][d] ? A.Eb[c][p + st[d]] : R(0);
      cb1[c][d] = m1[c][d] ? g.cbE[c][p + st[d]] : R(0);
    }
  }
  acc[0] = acc[1] = acc[2] = R(0);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (c == d) continue;
      const int jh = 3 - c - d;
      R v = eb0[c] * cb0[c] - eb1[c][d] * cb1[c][d];
      if (!UNI) v = v * g.inv_d[d];
      acc[jh] += d == (c + 1) % 3 ? v : -v;
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const PmlAxis<R>& pm = g.pml[d];
    if (!pm.on) continue;
    const int cr = (d + 1) % 3;
    const int s0 = adj_side<0>(pm, cr, x[d]), s1 = adj_side<0>(pm, cr, x[d] + 1);
    if (s0 < 0 && s1 < 0) continue;
    const int u = x[d];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (c == d) continue;
      const int jh = 3 - c - d;
      R t = R(0);
      if (s0 >= 0 && m0[c]) {
        const long long q = psi_index(x, g.n, d, u - pm.start[0][c][s0], pm.len[0][c][s0]);
        const R tot = A.pe_old[d][c][s0][q] + eb0[c];
        A.pe_new[d][c][s0][q] = tot * pm.b[0][u];
        R w = tot * pm.c[0][u];
        if (pm.k[0]) w += eb0[c] * pm.k[0][u];
        t += UNI ? cb0[c] * w : (cb0[c] / pm.div) * w;
      }
      if (s1 >= 0 && m1[c][d]) {
        int y[3] = {x[0], x[1], x[2]};
        y[d] += 1;
        const long long q = psi_index(y, g.n, d, u + 1 - pm.start[0][c][s1], pm.len[0][c][s1]);
        R w = (A.pe_old[d][c][s1][q] + eb1[c][d]) * pm.c[0][u + 1];
        if (pm.k[0]) w += eb1[c][d] * pm.k[0][u + 1];
        t -= UNI ? cb1[c][d] * w : (cb1[c][d] / pm.div) * w;
      }
      acc[jh] += d == (c + 1) % 3 ? t : -t;
    }
  }
}

// transpose of the E update: Hbar += (dE^{n+1}/dH^{n+1/2})^T Ebar; psibar_E to the step before; gradient.
// UNI: cubic cells (one instantiation per cell shape). Latency-bound: five CTAs per SM (at most 51 registers)
template <typename R, bool UNI>
__global__ void __launch_bounds__(256, 5) k_adj_e(const __grid_constant__ AdjArgs<R> A) {
  const YeeArgs<R>& g = A.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, i = blockIdx.z;
  if (k >= g.n[2] || j >= g.n[1]) return;
  const int x[3] = {i, j, k};
  const long long p = ((long long)i * g.n[1] + j) * g.n[2] + k;
  const long long st[3] = {(long long)g.n[1] * g.n[2], g.n[2], 1};
  // the node and its +1 neighbours along every axis are E-inner: every difference adjoint is test-free
  bool fast = true;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) fast = fast && x[ax] >= A.ein_lo[ax] && x[ax] + 1 < A.ein_hi[ax];
  R acc[3];
  if (__all_sync(__activemask(), fast)) {
    // Ebar_c cbE_c at the node and at its +1 neighbours, every load before the first store
    R u0[3], u1[3][3];  // u0[c]: at the node; u1[c][d]: at the node + e_d
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      u0[c] = A.Eb[c][p] * g.cbE[c][p];
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (d != c) u1[c][d] = A.Eb[c][p + st[d]] * g.cbE[c][p + st[d]];
    }
#pragma unroll
    for (int jj = 0; jj < 3; ++jj) {
      const int ca = (jj + 1) % 3, da = (jj + 2) % 3;
      const int cb = (jj + 2) % 3, db = (jj + 1) % 3;
      R va0 = u0[ca], va1 = u1[ca][da], vb0 = -u0[cb], vb1 = -u1[cb][db];
      if (!UNI) {
        va0 = va0 * g.inv_d[da];
        va1 = va1 * g.inv_d[da];
        vb0 = vb0 * g.inv_d[db];
        vb1 = vb1 * g.inv_d[db];
      }
      acc[jj] = (va0 - va1) + (vb0 - vb1);
    }
  } else {
    adj_e_lean<UNI>(A, x, p, st, acc);  // also this node's E psibar
  }
  const R hb0 = A.Hb[0][p], hb1 = A.Hb[1][p], hb2 = A.Hb[2][p];
  A.Hb[0][p] = hb0 + acc[0];
  A.Hb[1][p] = hb1 + acc[1];
  A.Hb[2][p] = hb2 + acc[2];
  // the gradient over the box (inside every component's stepped region, outside every E slab)
  if (i >= A.box_lo[0] && i < A.box_hi[0] && j >= A.box_lo[1] && j < A.box_hi[1] && k >= A.box_lo[2] &&
      k < A.box_hi[2]) {
    const int h0 = A.box_hi[0] - A.box_lo[0] + 1, h1 = A.box_hi[1] - A.box_lo[1] + 1,
              h2 = A.box_hi[2] - A.box_lo[2] + 1;
    const long long hs = (long long)h0 * h1 * h2;
    auto H = [&](int comp, int dx, int dy, int dz) {
      const long long o = ((long long)(i - A.box_lo[0] + 1 + dx) * h1 + (j - A.box_lo[1] + 1 + dy)) * h2 +
                          (k - A.box_lo[2] + 1 + dz);
      return A.hist[comp * hs + o];
    };
    const int b0 = A.box_hi[0] - A.box_lo[0], b1 = A.box_hi[1] - A.box_lo[1], b2 = A.box_hi[2] - A.box_lo[2];
    const long long o = ((long long)(i - A.box_lo[0]) * b1 + (j - A.box_lo[1])) * b2 + (k - A.box_lo[2]);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
      const int s1[3] = {d1 == 0, d1 == 1, d1 == 2}, s2[3] = {d2 == 0, d2 == 1, d2 == 2};
      const R a = H(d2, 0, 0, 0) - H(d2, -s1[0], -s1[1], -s1[2]);
      const R b = H(d1, 0, 0, 0) - H(d1, -s2[0], -s2[1], -s2[2]);
      const R curl = UNI ? (a - b) : (a * g.inv_d[d1] - b * g.inv_d[d2]);
      A.grad[(long long)c * b0 * b1 * b2 + o] += (double)A.Eb[c][p] * (double)curl;
    }
  }
}

// Transposed H update at E node x for a warp with any node outside the interior (backward neighbours, H's
// stepped region and CPML signs), with x's own H psibar.
template <bool UNI, typename R>
__device__ __forceinline__ void adj_h_lean(const AdjArgs<R>& A, const int* x, long long p, const long long* st,
                                           R* acc) {
  const YeeArgs<R>& g = A.y;
  // H_c's stepped range (in_h_region): [0, n - 1), or [0, n) along c itself; [1, n - 1) along a periodic
  // axis; along a mirror axis from node 1, or from 2 for the normal component of an antisymmetric plane.
  // own[a]: x in range along axis a != c, alc[a]: along a == c, back[a]: x - e_a in range along a != c
  bool own[3], back[3], alc[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int lo_oth = (g.periodic[a] || g.mirror[a]) ? 1 : 0;
    const int lo_own = g.mirror[a] < 0 ? 2 : lo_oth, hi_own = g.periodic[a] ? g.n[a] - 1 : g.n[a];
    own[a] = x[a] >= lo_oth && x[a] < g.n[a] - 1;
    alc[a] = x[a] >= lo_own && x[a] < hi_own;
    back[a] = x[a] - 1 >= lo_oth;
  }
  R hb0[3], hb1[3][3];
  bool m0[3], m1[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    m0[c] = own[(c + 1) % 3] && own[(c + 2) % 3] && alc[c];
    hb0[c] = m0[c] ? A.Hb[c][p] : R(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (d == c) continue;
      m1[c][d] = back[d] && own[3 - c - d] && alc[c];
      hb1[c][d] = m1[c][d] ? A.Hb[c][p - st[d]] : R(0);
    }
  }
  acc[0] = acc[1] = acc[2] = R(0);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (c == d) continue;
      const int jh = 3 - c - d;
      R v = hb1[c][d] * g.cH - hb0[c] * g.cH;
      if (!UNI) v = v * g.inv_d[d];
      acc[jh] += d == (c + 1) % 3 ? -v : v;
    }
  }
  const R sH = g.cH;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const PmlAxis<R>& pm = g.pml[d];
    if (!pm.on) continue;
    const int cr = (d + 1) % 3;
    const int s0 = adj_side<1>(pm, cr, x[d]), s1 = adj_side<1>(pm, cr, x[d] - 1);
    if (s0 < 0 && s1 < 0) continue;
    const int u = x[d];
    const R sc = UNI ? sH : sH / pm.div;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (c == d) continue;
      const int jh = 3 - c - d;
      R t = R(0);
      if (s1 >= 0 && m1[c][d]) {
        int y[3] = {x[0], x[1], x[2]};
        y[d] -= 1;
        const long long q = psi_index(y, g.n, d, u - 1 - pm.start[1][c][s1], pm.len[1][c][s1]);
        R w = (A.ph_old[d][c][s1][q] + hb1[c][d]) * pm.c[1][u - 1];
        if (pm.k[1]) w += hb1[c][d] * pm.k[1][u - 1];
        t += sc * w;
      }
      if (s0 >= 0 && m0[c]) {
        const long long q = psi_index(x, g.n, d, u - pm.start[1][c][s0], pm.len[1][c][s0]);
        const R tot = A.ph_old[d][c][s0][q] + hb0[c];
        A.ph_new[d][c][s0][q] = tot * pm.b[1][u];
        R w = tot * pm.c[1][u];
        if (pm.k[1]) w += hb0[c] * pm.k[1][u];
        t -= sc * w;
      }
      acc[jh] += d == (c + 1) % 3 ? -t : t;
    }
  }
}

// transpose of the H update: Ebar += (dH^{n+1/2}/dE^n)^T Hbar; psibar_H to the step before
template <typename R, bool UNI>
__global__ void __launch_bounds__(256, 5) k_adj_h(const __grid_constant__ AdjArgs<R> A) {
  const YeeArgs<R>& g = A.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, i = blockIdx.z;
  if (k >= g.n[2] || j >= g.n[1]) return;
  const int x[3] = {i, j, k};
  const long long p = ((long long)i * g.n[1] + j) * g.n[2] + k;
  const long long st[3] = {(long long)g.n[1] * g.n[2], g.n[2], 1};
  // the node and its -1 neighbours along every axis are H-inner
  bool fast = true;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) fast = fast && x[ax] - 1 >= A.hin_lo[ax] && x[ax] < A.hin_hi[ax];
  R acc[3];
  if (__all_sync(__activemask(), fast)) {
    // Hbar_c at the node and at its -1 neighbours, every load before the first store
    R h0[3], hm[3][3];  // h0[c]: at the node; hm[c][d]: at the node - e_d
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      h0[c] = A.Hb[c][p];
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (d != c) hm[c][d] = A.Hb[c][p - st[d]];
    }
#pragma unroll
    for (int jj = 0; jj < 3; ++jj) {
      const int ca = (jj + 1) % 3, da = (jj + 2) % 3;
      const int cb = (jj + 2) % 3, db = (jj + 1) % 3;
      // a of H_ca: -Hbar cH (along da); b of H_cb: +Hbar cH (along db)
      R va1 = -(hm[ca][da] * g.cH), va0 = -(h0[ca] * g.cH), vb1 = hm[cb][db] * g.cH, vb0 = h0[cb] * g.cH;
      if (!UNI) {
        va1 = va1 * g.inv_d[da];
        va0 = va0 * g.inv_d[da];
        vb1 = vb1 * g.inv_d[db];
        vb0 = vb0 * g.inv_d[db];
      }
      acc[jj] = (va1 - va0) + (vb1 - vb0);
    }
  } else {
    adj_h_lean<UNI>(A, x, p, st, acc);  // also this node's H psibar
  }
  const R eb0 = A.Eb[0][p], eb1 = A.Eb[1][p], eb2 = A.Eb[2][p];
  A.Eb[0][p] = eb0 + acc[0];
  A.Eb[1][p] = eb1 + acc[1];
  A.Eb[2][p] = eb2 + acc[2];
}

// Transpose of one periodic ghost plane's copy (dst <- src, real fields): the adjoint of dst is added to src
// and dst's cleared, for the three components over the plane normal to `axis` (k_ghost's enumeration).
template <typename R>
__global__ void k_adj_ghost(R* f0, R* f1, R* f2, int n0, int n1, int n2, int axis, int dst, int src) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int na = axis == 0 ? n1 : n0, nb = axis == 2 ? n1 : n2;
  if (t >= 3 * na * nb) return;
  const int comp = t / (na * nb);
  const int r = t % (na * nb);
  const int u = r / nb, v = r % nb;
  int xd[3], xs[3];
  if (axis == 0) { xd[0] = dst; xs[0] = src; xd[1] = xs[1] = u; xd[2] = xs[2] = v; }
  else if (axis == 1) { xd[1] = dst; xs[1] = src; xd[0] = xs[0] = u; xd[2] = xs[2] = v; }
  else { xd[2] = dst; xs[2] = src; xd[0] = xs[0] = u; xd[1] = xs[1] = v; }
  R* f = comp == 0 ? f0 : (comp == 1 ? f1 : f2);
  const long long pd = ((long long)xd[0] * n1 + xd[1]) * n2 + xd[2];
  const long long ps = ((long long)xs[0] * n1 + xs[1]) * n2 + xs[2];
  f[ps] += f[pd];
  f[pd] = R(0);
}

// Transpose of a symmetric mirror plane's ghost fill (k_mirror_ghost: the tangential H components' plane 0
// set to minus plane 1): plane 1's adjoint loses plane 0's, and plane 0's is cleared.
template <typename R>
__global__ void k_adj_mirror(R* h0, R* h1, R* h2, int n0, int n1, int n2, int axis) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int na = axis == 0 ? n1 : n0, nb = axis == 2 ? n1 : n2;
  const long long per = (long long)na * nb;
  if (t >= 2 * per) return;
  const int comp = (axis + 1 + (int)(t / per)) % 3;
  const long long r = t % per;
  const int u = (int)(r / nb), v = (int)(r % nb);
  long long pg, ps;
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
  R* f = comp == 0 ? h0 : (comp == 1 ? h1 : h2);
  f[ps] -= f[pg];
  f[pg] = R(0);
}

// Transpose of the conformal off-diagonal terms (k_offdiag: E[e[t]] += sum_k w[t][k] H[h[t][k]] after the E
// update). The caller gives the rows transposed, one per H node that any term reads: row r adds
// sum_{j in [ptr[r], ptr[r + 1])} w[j] Ebar[e[j]] to Hbar[h[r]]. The rows' H nodes are distinct, so one thread
// per row needs no atomics, and each sum runs in the caller's order (the result does not depend on the launch).
template <typename R>
__global__ void k_adj_offdiag(const long long* h, const long long* ptr, const long long* e, const R* w,
                              long long rows, const R* Eb, R* Hb) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  R acc = R(0);
  for (long long j = ptr[r]; j < ptr[r + 1]; ++j) acc += w[j] * Eb[e[j]];
  Hb[h[r]] += acc;
}

// ---- the vertex-tensor ADE, transposed ----
// Forward, after the groups (tensor.cuh): D' = D + E[idx] - E_prev per node; per vertex the means D~_d of its
// d-nodes and s = n . D~; per tensor slot sigma = s + n_c (D_p - D~_c) into its harmonic (a) and arithmetic (b)
// operators, out = (b + n_c a) / 2; per plain slot out = m[D] / 2; then E[idx] = E_prev = out[i] + out[nN + i].
// Every map is linear with fixed coefficients, so the reverse step needs no forward values: it applies the
// transposes in the opposite order to an adjoint state laid out as the forward's (the bars of D, E_prev and of
// the path and pole states; `out`'s place holds each output's adjoint). Fan-ins are gathers over maps the caller
// builds (the slots of each vertex, the contributions to each node), so every sum runs in a fixed order. The
// work array: contrib, per (vertex, axis, side) [6 nV], tensor slot [nT] and plain slot [nP] the adjoint that
// entry sends to one node's D'; then sig [nT], each tensor slot's sigma adjoint.

// the poles of medium s at slot t of n, transposed: from the adjoint tbar of their sum (added to each new P_k's
// adjoint), the adjoints of the old P_k and P'_k (in place) and the returned adjoint of the drive
template <typename R>
__device__ __forceinline__ R adj_tm_poles(const TensorArgs<R>& b, int s, R* P, long long t, long long n, R tbar) {
  R drive = R(0);
  for (int k = 0; k < b.n_poles[s]; ++k) {
    R* pk = P + (2 * k) * n;
    R* pp = P + (2 * k + 1) * n;
    const R hat = pk[t] + tbar;
    pk[t] = b.c1[s][k] * hat + pp[t];
    pp[t] = b.c2[s][k] * hat;
    drive += b.c3[s][k] * hat;
  }
  return drive;
}

// E[idx] = E_prev = out[i] + out[nN + i]: both slots' adjoint is that of the node's new E and E_prev; E's own
// adjoint there restarts (the curl update's value was overwritten) and D's path adds to it (k_adj_tm_nodes_d)
template <typename R>
__global__ void k_adj_tm_out(TensorArgs<R> b, R* Eb) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.nN) return;
  const long long q = b.idx[i];
  const R e = Eb[q] + b.Ep[i];
  Eb[q] = R(0);
  b.Ep[i] = R(0);
  b.out[i] = e;
  b.out[b.nN + i] = e;
}

template <typename R>
__global__ void k_adj_tm_plain(TensorArgs<R> b, R* work) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= b.nP) return;
  const int m = (int)b.p_medium[p];
  R ybar = R(0.5) * b.out[b.p_pos[p]];
  R ubar;
  if (!b.n_poles[m]) {
    ubar = ybar * (R(1) / b.eps_inf[m]);
  } else {  // y = (u - sum of the poles) / eps_inf, kept as the next step's drive
    ybar += b.pl_E[m][p];
    ubar = ybar * b.inv_inf[m];
    b.pl_E[m][p] = adj_tm_poles(b, m, b.pl_P[m], p, b.nP, -ubar);
  }
  work[6 * b.nV + b.nT + p] = ubar;
}

template <typename R>
__global__ void k_adj_tm_slots(TensorArgs<R> b, R* work) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.nT) return;
  const R nc = b.t_nc[t];
  const R cbar = b.out[b.t_pos[t]];
  // b[u_b] = (u_b - sum_s f_s poles_s(y_prev)) / <eps>, kept as y
  R den = R(0);
  for (int s = 0; s < b.n_media; ++s) den += b.frac[s * b.nT + t] * b.eps_inf[s];
  const R accbar = (R(0.5) * cbar + b.ar_y[t]) * (R(1) / den);
  R drive = R(0);
  for (int s = 0; s < b.n_media; ++s)
    if (b.n_poles[s]) drive += adj_tm_poles(b, s, b.ar_P[s], t, b.nT, -(b.frac[s * b.nT + t] * accbar));
  b.ar_y[t] = drive;
  // a[u_a] = u_a h0 + sum_s f_s E_s, E_s = (u_a - poles_s(E_s prev)) / eps_inf_s
  const R yabar = R(0.5) * nc * cbar;
  R h0 = R(0);
  for (int s = 0; s < b.n_media; ++s)
    if (!b.n_poles[s]) h0 += b.frac[s * b.nT + t] / b.eps_inf[s];
  R uabar = yabar * h0;
  for (int s = 0; s < b.n_media; ++s) {
    if (!b.n_poles[s]) continue;
    const R g = (b.frac[s * b.nT + t] * yabar + b.ha_E[s][t]) * b.inv_inf[s];
    uabar += g;
    b.ha_E[s][t] = adj_tm_poles(b, s, b.ha_P[s], t, b.nT, -g);
  }
  // u_a = sigma, u_b = D_p - n_c sigma, sigma = s_v + n_c (D_p - D~_c)
  const R sg = uabar - nc * accbar;
  const R dpbar = accbar + nc * sg;
  work[6 * b.nV + b.nT + b.nP + t] = sg;
  work[6 * b.nV + t] = (b.scale ? b.scale[b.t_g[t]] : R(1)) * dpbar;
}

// per vertex: s's adjoint (its slots' sigma adjoints) and D~_d's (n_d times it, less n_c sigma adjoint of the
// slots on component d), each mean's half to its two d-nodes with their parity
template <typename R>
__global__ void k_adj_tm_vertices(TensorArgs<R> b, R* work, const long long* vs_ptr, const long long* vs_idx) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= b.nV) return;
  const R* sig = work + 6 * b.nV + b.nT + b.nP;
  R sv = R(0), ex[3] = {R(0), R(0), R(0)};
  for (long long j = vs_ptr[v]; j < vs_ptr[v + 1]; ++j) {
    const long long t = vs_idx[j];
    const R sgt = sig[t];
    sv += sgt;
    const int c = (int)(b.t_vc[t] - 3 * v);
    ex[c] -= b.t_nc[t] * sgt;
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const R h = R(0.5) * (b.normal[v * 3 + d] * sv + ex[d]);
    const long long e = v * 6 + 2 * d;
    work[e] = (b.scale ? b.scale[e] : R(1)) * h;
    work[e + 1] = (b.scale ? b.scale[e + 1] : R(1)) * h;
  }
}

// D' = D + E[idx] - E_prev: D' gathers its adjoint (the step after's, plus every entry that read it); it is
// D's, E's at the node, and minus E_prev's
template <typename R>
__global__ void k_adj_tm_nodes_d(TensorArgs<R> b, R* Eb, const R* work, const long long* nd_ptr,
                                 const long long* nd_src) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.nN) return;
  R dd = b.D[i];
  for (long long j = nd_ptr[i]; j < nd_ptr[i + 1]; ++j) dd += work[nd_src[j]];
  b.D[i] = dd;
  b.Ep[i] = -dd;
  Eb[b.idx[i]] += dd;
}

constexpr int kAdjMaxFreq = 128;

// the objective's frequencies, passed by value
struct AdjFreqs {
  double omega[kAdjMaxFreq];
  int nf;
};

// each point's adjoint source value at one sample (after n steps), in double: E point p sum_f Re(G_e[f][p]
// e^{i w_f t_e}) at v[p], H point q half of sum_f Re(G_h[f][q] e^{i w_f t_h}) at v[ne + q]
__global__ void k_adj_inject_values(const double* ge, long long ne, const double* gh, long long nh,
                                    const __grid_constant__ AdjFreqs fr, double dt, long long n, double* v) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ne + nh) return;
  const bool is_h = t >= ne;
  const long long p = is_h ? t - ne : t;
  const double tt = (double)n * dt - (is_h ? 0.5 * dt : 0.0);
  const double* g = is_h ? gh : ge;
  const long long np = is_h ? nh : ne;
  double s = 0.0;
  for (int f = 0; f < fr.nf; ++f) {
    double sn, cs;
    sincos(fr.omega[f] * tt, &sn, &cs);
    const double* gp = g + 2 * ((long long)f * np + p);
    s += gp[0] * cs - gp[1] * sn;
  }
  v[t] = is_h ? 0.5 * s : s;
}

// the values gathered per distinct target node, in the maps' order, and added once: E targets first, then H
template <typename R>
__global__ void k_adj_inject_gather(R* Eb, R* Hb, const double* v, long long ne, const long long* e_tgt,
                                    const long long* e_ptr, const long long* e_src, long long n_e,
                                    const long long* h_tgt, const long long* h_ptr, const long long* h_src,
                                    long long n_h) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n_e) {
    double s = 0.0;
    for (long long j = e_ptr[r]; j < e_ptr[r + 1]; ++j) s += v[e_src[j]];
    Eb[e_tgt[r]] += (R)s;
  } else if (r < n_e + n_h) {
    const long long q = r - n_e;
    double s = 0.0;
    for (long long j = h_ptr[q]; j < h_ptr[q + 1]; ++j) s += v[ne + h_src[j]];
    Hb[h_tgt[q]] += (R)s;
  }
}

// the objective's adjoint source at one sample (after n steps): Ebar[e_idx[p]] += sum_f Re(G_e[f][p]
// e^{i w_f t_e}); Hbar[h1[q]], Hbar[h2[q]] += sum_f Re(G_h[f][q] e^{i w_f t_h}) / 2 each (the monitor's H
// sample is the mean of the two)
template <typename R>
__global__ void k_adj_inject(R* Eb, R* Hb, const long long* e_idx, const double* ge, long long ne,
                             const long long* h1, const long long* h2, const double* gh, long long nh,
                             const __grid_constant__ AdjFreqs fr, double dt, long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const double te = (double)n * dt, th = te - 0.5 * dt;
  if (t < ne) {
    double v = 0.0;
    for (int f = 0; f < fr.nf; ++f) {
      double sn, cs;
      sincos(fr.omega[f] * te, &sn, &cs);
      const double* gp = ge + 2 * ((long long)f * ne + t);
      v += gp[0] * cs - gp[1] * sn;
    }
    atomicAdd(Eb + e_idx[t], (R)v);
  } else if (t < ne + nh) {
    const long long q = t - ne;
    double v = 0.0;
    for (int f = 0; f < fr.nf; ++f) {
      double sn, cs;
      sincos(fr.omega[f] * th, &sn, &cs);
      const double* gp = gh + 2 * ((long long)f * nh + q);
      v += gp[0] * cs - gp[1] * sn;
    }
    const R h = (R)(0.5 * v);
    atomicAdd(Hb + h1[q], h);
    atomicAdd(Hb + h2[q], h);
  }
}

// the transpose of a pure dispersive group's step (k_ade) at each of its nodes. Forward, with e the node's E
// after the curl update: D' = D + (e - E_prev); P_k' = c1 P_k + c2 Pp_k + c3 E_prev; Pp_k' = P_k;
// e' = (D' - sum_k P_k') / eps_inf; E' = E_prev' = e'. Backward, from the adjoints of the outputs (Ebar at the
// node, and the adjoint state Dbar, Epbar, Pbar_k, Ppbar_k of the step after): g = Ebar + Epbar; Dbar +=
// g / eps_inf; Phat_k = Pbar_k - g / eps_inf; Epbar = -Dbar + sum_k c3 Phat_k; Pbar_k = c1 Phat_k + Ppbar_k;
// Ppbar_k = c2 Phat_k; and the adjoint of e (the new Ebar at the node) is Dbar. The state's layout is k_ade's.
//
// A mixed group's step (k_ade's mixed branch, lightsmith's engine.py:776-791) is linear too. With g = Ebar +
// Epbar the adjoint of e': the harmonic path's hbar = w g, each medium's e_s adjoint esbar_s = f_s hbar +
// Ehbar_s, Dbar += h0 hbar + sum_s esbar_s / eps_inf_s, and per pole Phat = Phbar - esbar_s / eps_inf_s, the
// drive's adjoint (the new Ehbar_s) sum_k c3 Phat; the arithmetic path's abar = ((1 - w) g + Eabar) inv_a,
// Dbar += abar, per pole Phat = Pabar - f_s abar, the new Eabar = sum_{s,k} c3 Phat; then as for a pure node
// Pbar = c1 Phat + Ppbar, Ppbar = c2 Phat, and the adjoints of e and of the old D and E_prev are Dbar, Dbar,
// -Dbar. A path the group does not run leaves its state, and so its adjoint, as it was.
template <typename R>
__device__ void adj_ade_mixed(const AdeArgs<R>& g, R* Eb, R* bar, long long t) {
  const long long n = g.n;
  const int S = g.n_media;
  R* Db = bar;
  R* Epb = bar + n;
  R* Eab = bar + 2 * n;
  R* Ehb = bar + 3 * n;  // [S][n]
  int n_tot = 0;
  for (int s = 0; s < S; ++s) n_tot += g.n_poles[s];
  R* Phb = bar + (3 + S) * n;      // [sum poles][2][n]
  R* Pab = Phb + 2 * n_tot * n;    // same layout
  const long long node = g.idx[t];
  const R w = g.w[t];
  const R gs = Eb[node] + Epb[t];
  R dbar = Db[t];
  if (g.has_h) {
    const R hbar = w * gs;
    dbar += g.h0[t] * hbar;
    int off = 0;
    for (int s = 0; s < S; ++s) {
      const R esb = g.frac[s * n + t] * hbar + Ehb[s * n + t];
      dbar += g.inv_inf[s] * esb;
      R drive = R(0);
      for (int k = 0; k < g.n_poles[s]; ++k) {
        R* pk = Phb + (2 * (off + k)) * n;
        R* pp = Phb + (2 * (off + k) + 1) * n;
        const R ph = pk[t] - g.inv_inf[s] * esb;
        drive += g.c3[s][k] * ph;
        const R npk = g.c1[s][k] * ph + pp[t];
        pp[t] = g.c2[s][k] * ph;
        pk[t] = npk;
      }
      Ehb[s * n + t] = drive;
      off += g.n_poles[s];
    }
  }
  if (g.has_a) {
    const R abar = ((R(1) - w) * gs + Eab[t]) * g.inv_a[t];
    dbar += abar;
    R drive = R(0);
    int off = 0;
    for (int s = 0; s < S; ++s) {
      const R fb = g.frac[s * n + t] * abar;
      for (int k = 0; k < g.n_poles[s]; ++k) {
        R* pk = Pab + (2 * (off + k)) * n;
        R* pp = Pab + (2 * (off + k) + 1) * n;
        const R ph = pk[t] - fb;
        drive += g.c3[s][k] * ph;
        const R npk = g.c1[s][k] * ph + pp[t];
        pp[t] = g.c2[s][k] * ph;
        pk[t] = npk;
      }
      off += g.n_poles[s];
    }
    Eab[t] = drive;
  }
  Db[t] = dbar;
  Epb[t] = -dbar;
  Eb[node] = dbar;
}

template <typename R>
__global__ void k_adj_ade(const AdeArgs<R> g, R* Eb, R* bar) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.n) return;
  if (g.mixed) {
    adj_ade_mixed(g, Eb, bar, t);
    return;
  }
  const long long n = g.n;
  R* Db = bar;
  R* Epb = bar + n;
  R* Pb = bar + 2 * n;
  const long long node = g.idx[t];
  const R inv = g.inv_inf[0];
  const R gs = Eb[node] + Epb[t];
  const R dbar = Db[t] + inv * gs;
  R epb = -dbar;
  for (int k = 0; k < g.n_poles[0]; ++k) {
    R* pk = Pb + (2 * k) * n;
    R* pp = Pb + (2 * k + 1) * n;
    const R ph = pk[t] - inv * gs;
    epb += g.c3[0][k] * ph;
    const R npk = g.c1[0][k] * ph + pp[t];
    pp[t] = g.c2[0][k] * ph;
    pk[t] = npk;
  }
  Db[t] = dbar;
  Epb[t] = epb;
  Eb[node] = dbar;
}

// H over the gradient box and its low halo: dst[c][x - lo + 1][y - lo + 1][z - lo + 1]
template <typename R>
__global__ void k_adj_hist(const R* H0, const R* H1, const R* H2, R* dst, int n1, int n2, int lo0, int lo1, int lo2,
                           int h0, int h1, int h2) {
  const long long hs = (long long)h0 * h1 * h2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * hs) return;
  const int c = (int)(t / hs);
  const long long r = t % hs;
  const int a = (int)(r / ((long long)h1 * h2)), b = (int)((r / h2) % h1), z = (int)(r % h2);
  const R* H = c == 0 ? H0 : (c == 1 ? H1 : H2);
  dst[t] = H[((long long)(lo0 - 1 + a) * n1 + (lo1 - 1 + b)) * n2 + (lo2 - 1 + z)];
}

}  // namespace lsfdtd
