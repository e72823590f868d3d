// The discrete adjoint of the FDTD step (real fields, no periodic axis), for gradients of a DFT objective.
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
//
// The objective's adjoint source (the DFT samples' weights times e^{i omega t}) is added to Ebar and Hbar at
// the steps the monitor sampled, before that step's reverse. The gradient with respect to the E curl
// coefficient, dJ/dcbE_c(p) = sum_n Ebar_c^{n+1}(p) curl_c(H^{n+1/2})(p), is accumulated (in double) over a
// box of nodes away from the CPML slabs, from H^{n+1/2} of the box (with its low halo) recomputed forward.
#pragma once

#include "common.cuh"
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

// psi index of node x in the slab of axis d (field FLD, component c), or -1 when x is not in it
template <int FLD, typename R>
__device__ __forceinline__ long long adj_slab(const PmlAxis<R>& p, int d, int c, const int* x, const int* n,
                                              int* side) {
  if (!p.on) return -1;
  const int u = x[d];
#pragma unroll
  for (int sd = 0; sd < 2; ++sd) {
    const int st = p.start[FLD][c][sd], ln = p.len[FLD][c][sd];
    if (ln > 0 && u >= st && u < st + ln) {
      *side = sd;
      return psi_index(x, n, d, u - st, ln);
    }
  }
  return -1;
}

__device__ __forceinline__ bool adj_in_grid(const int* x, const int* n) {
  return x[0] >= 0 && x[0] < n[0] && x[1] >= 0 && x[1] < n[1] && x[2] >= 0 && x[2] < n[2];
}

// adjoint of difference `which` (0: a, along d1; 1: b, along d2) of component c's E update at node x
// FAST: x is known to be stepped for every component and outside every slab (no tests, no CPML term)
template <bool FAST, typename R>
__device__ __forceinline__ R adj_e_diff(const AdjArgs<R>& A, int c, int which, const int* x) {
  const YeeArgs<R>& g = A.y;
  if (!FAST && (!adj_in_grid(x, g.n) || !in_e_region(c, x, g.n, g.periodic))) return R(0);
  const long long p = ((long long)x[0] * g.n[1] + x[1]) * g.n[2] + x[2];
  const int d1 = (c + 1) % 3, d2 = (c + 2) % 3, d = which ? d2 : d1;
  const R eb = A.Eb[c][p];
  const R cb = g.cbE[c][p];
  R v = which ? -(eb * cb) : eb * cb;
  if (!g.uniform) v = v * g.inv_d[d];
  if (FAST) return v;
  int side;
  const long long q = adj_slab<0>(g.pml[d], d, c, x, g.n, &side);
  if (q >= 0) {
    const PmlAxis<R>& pm = g.pml[d];
    const R sgn = which ? R(-1) : R(1);
    R s = g.uniform ? cb : cb / pm.div;
    s = sgn * s;
    const R tot = A.pe_old[d][c][side][q] + eb;
    v += tot * (s * pm.c[0][x[d]]);
    if (pm.k[0]) v += eb * (s * pm.k[0][x[d]]);
  }
  return v;
}

// the same for the H update (forward differences, coefficient -cH, H's CPML signs)
template <bool FAST, typename R>
__device__ __forceinline__ R adj_h_diff(const AdjArgs<R>& A, int c, int which, const int* x) {
  const YeeArgs<R>& g = A.y;
  if (!FAST && (!adj_in_grid(x, g.n) || !in_h_region(c, x, g.n, g.periodic))) return R(0);
  const long long p = ((long long)x[0] * g.n[1] + x[1]) * g.n[2] + x[2];
  const int d1 = (c + 1) % 3, d2 = (c + 2) % 3, d = which ? d2 : d1;
  const R hb = A.Hb[c][p];
  R v = which ? hb * g.cH : -(hb * g.cH);
  if (!g.uniform) v = v * g.inv_d[d];
  if (FAST) return v;
  int side;
  const long long q = adj_slab<1>(g.pml[d], d, c, x, g.n, &side);
  if (q >= 0) {
    const PmlAxis<R>& pm = g.pml[d];
    const R sgn = which ? R(1) : R(-1);
    R s = g.uniform ? g.cH : g.cH / pm.div;
    s = sgn * s;
    const R tot = A.ph_old[d][c][side][q] + hb;
    v += tot * (s * pm.c[1][x[d]]);
    if (pm.k[1]) v += hb * (s * pm.k[1][x[d]]);
  }
  return v;
}

// transpose of the E update: Hbar += (dE^{n+1}/dH^{n+1/2})^T Ebar; psibar_E to the step before; gradient
template <typename R>
__global__ void __launch_bounds__(256) k_adj_e(const __grid_constant__ AdjArgs<R> A) {
  const YeeArgs<R>& g = A.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, i = blockIdx.z;
  if (k >= g.n[2] || j >= g.n[1]) return;
  const int x[3] = {i, j, k};
  const long long p = ((long long)i * g.n[1] + j) * g.n[2] + k;
  // the node and its +1 neighbours along every axis are E-inner: every difference adjoint is test-free
  bool fast = true;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) fast = fast && x[ax] >= A.ein_lo[ax] && x[ax] + 1 < A.ein_hi[ax];
  R acc[3];
  if (fast) {
    // Ebar_c cbE_c at the node and at its +1 neighbours, every load before the first store
    const long long st[3] = {(long long)g.n[1] * g.n[2], g.n[2], 1};
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
      if (!g.uniform) {
        va0 = va0 * g.inv_d[da];
        va1 = va1 * g.inv_d[da];
        vb0 = vb0 * g.inv_d[db];
        vb1 = vb1 * g.inv_d[db];
      }
      acc[jj] = (va0 - va1) + (vb0 - vb1);
    }
  } else {
#pragma unroll
    for (int jj = 0; jj < 3; ++jj) {
      const int ca = (jj + 1) % 3, da = (jj + 2) % 3;  // the component whose difference a reads H_jj along da
      const int cb = (jj + 2) % 3, db = (jj + 1) % 3;  // and whose difference b reads it along db
      int xa[3] = {i, j, k}, xb[3] = {i, j, k};
      xa[da] += 1;
      xb[db] += 1;
      acc[jj] = (adj_e_diff<false>(A, ca, 0, x) - adj_e_diff<false>(A, ca, 0, xa)) +
                (adj_e_diff<false>(A, cb, 1, x) - adj_e_diff<false>(A, cb, 1, xb));
    }
  }
  const R hb0 = A.Hb[0][p], hb1 = A.Hb[1][p], hb2 = A.Hb[2][p];
  A.Hb[0][p] = hb0 + acc[0];
  A.Hb[1][p] = hb1 + acc[1];
  A.Hb[2][p] = hb2 + acc[2];
  // this node's E psibar, and the gradient
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!in_e_region(c, x, g.n, g.periodic)) continue;
    const R eb = A.Eb[c][p];
#pragma unroll
    for (int d = 0; d < 3 && !fast; ++d) {  // an inner node lies in no slab
      if (d == c) continue;
      int side;
      const long long q = adj_slab<0>(g.pml[d], d, c, x, g.n, &side);
      if (q >= 0) A.pe_new[d][c][side][q] = (A.pe_old[d][c][side][q] + eb) * g.pml[d].b[0][x[d]];
    }
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
      const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
      const int s1[3] = {d1 == 0, d1 == 1, d1 == 2}, s2[3] = {d2 == 0, d2 == 1, d2 == 2};
      const R a = H(d2, 0, 0, 0) - H(d2, -s1[0], -s1[1], -s1[2]);
      const R b = H(d1, 0, 0, 0) - H(d1, -s2[0], -s2[1], -s2[2]);
      const R curl = g.uniform ? (a - b) : (a * g.inv_d[d1] - b * g.inv_d[d2]);
      const int b0 = A.box_hi[0] - A.box_lo[0], b1 = A.box_hi[1] - A.box_lo[1], b2 = A.box_hi[2] - A.box_lo[2];
      const long long o = ((long long)(i - A.box_lo[0]) * b1 + (j - A.box_lo[1])) * b2 + (k - A.box_lo[2]);
      A.grad[(long long)c * b0 * b1 * b2 + o] += (double)eb * (double)curl;
    }
  }
}

// transpose of the H update: Ebar += (dH^{n+1/2}/dE^n)^T Hbar; psibar_H to the step before
template <typename R>
__global__ void __launch_bounds__(256) k_adj_h(const __grid_constant__ AdjArgs<R> A) {
  const YeeArgs<R>& g = A.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, i = blockIdx.z;
  if (k >= g.n[2] || j >= g.n[1]) return;
  const int x[3] = {i, j, k};
  const long long p = ((long long)i * g.n[1] + j) * g.n[2] + k;
  // the node and its -1 neighbours along every axis are H-inner
  bool fast = true;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) fast = fast && x[ax] - 1 >= A.hin_lo[ax] && x[ax] < A.hin_hi[ax];
  R acc[3];
  if (fast) {
    // Hbar_c at the node and at its -1 neighbours, every load before the first store
    const long long st[3] = {(long long)g.n[1] * g.n[2], g.n[2], 1};
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
      if (!g.uniform) {
        va1 = va1 * g.inv_d[da];
        va0 = va0 * g.inv_d[da];
        vb1 = vb1 * g.inv_d[db];
        vb0 = vb0 * g.inv_d[db];
      }
      acc[jj] = (va1 - va0) + (vb1 - vb0);
    }
  } else {
#pragma unroll
    for (int jj = 0; jj < 3; ++jj) {
      const int ca = (jj + 1) % 3, da = (jj + 2) % 3;
      const int cb = (jj + 2) % 3, db = (jj + 1) % 3;
      int xa[3] = {i, j, k}, xb[3] = {i, j, k};
      xa[da] -= 1;
      xb[db] -= 1;
      acc[jj] = (adj_h_diff<false>(A, ca, 0, xa) - adj_h_diff<false>(A, ca, 0, x)) +
                (adj_h_diff<false>(A, cb, 1, xb) - adj_h_diff<false>(A, cb, 1, x));
    }
  }
  const R eb0 = A.Eb[0][p], eb1 = A.Eb[1][p], eb2 = A.Eb[2][p];
  A.Eb[0][p] = eb0 + acc[0];
  A.Eb[1][p] = eb1 + acc[1];
  A.Eb[2][p] = eb2 + acc[2];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!in_h_region(c, x, g.n, g.periodic)) continue;
    const R hb = A.Hb[c][p];
#pragma unroll
    for (int d = 0; d < 3 && !fast; ++d) {  // an inner node lies in no slab
      if (d == c) continue;
      int side;
      const long long q = adj_slab<1>(g.pml[d], d, c, x, g.n, &side);
      if (q >= 0) A.ph_new[d][c][side][q] = (A.ph_old[d][c][side][q] + hb) * g.pml[d].b[1][x[d]];
    }
  }
}

// the objective's adjoint source at one sample (after n steps): Ebar[e_idx] += Re(ge e^{i w t_e}),
// Hbar[h1], Hbar[h2] += Re(gh e^{i w t_h}) / 2 each (the monitor's H sample is the mean of the two)
template <typename R>
__global__ void k_adj_inject(R* Eb, R* Hb, const long long* e_idx, const double* ge, long long ne,
                             const long long* h1, const long long* h2, const double* gh, long long nh, double omega,
                             double dt, long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const double te = (double)n * dt, th = te - 0.5 * dt;
  if (t < ne) {
    double sn, cs;
    sincos(omega * te, &sn, &cs);
    atomicAdd(Eb + e_idx[t], (R)(ge[2 * t] * cs - ge[2 * t + 1] * sn));
  } else if (t < ne + nh) {
    const long long q = t - ne;
    double sn, cs;
    sincos(omega * th, &sn, &cs);
    const R v = (R)(0.5 * (gh[2 * q] * cs - gh[2 * q + 1] * sn));
    atomicAdd(Hb + h1[q], v);
    atomicAdd(Hb + h2[q], v);
  }
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
