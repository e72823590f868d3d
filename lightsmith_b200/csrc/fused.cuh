// One FDTD step (H half step then E half step, CPML included) in a single pass over the grid.
//
// Each CTA owns a tile of TZ = 32 nodes along z (contiguous) by TY nodes along y and marches through a
// segment of x planes. For plane i it holds E^n(i) and E^n(i+1) (tile plus a one-node halo) in shared
// memory, computes H^{n+1/2}(i) on the tile and on the low-side halo row and column it needs, then
// E^{n+1}(i) on the tile, reading H^{n+1/2}(i-1) of its own nodes from registers. The next plane is
// fetched into registers while the current one is computed.
//
// The halo H of a tile is recomputed by the tile itself, so E, H and the H-side CPML psi are double
// buffered: a step reads the "in" buffers and writes the "out" buffers, and no CTA can observe a value
// another CTA has already advanced. Per cell and step that is E, H and one coefficient read once and E, H
// written once (52 B in FP32), plus the psi of CPML cells. Nodes outside a component's stepped region are
// copied, so the two buffers always agree there.
//
// The arithmetic per value is that of k_update_h / k_update_e (and of lightsmith's engine.py:613-663).
#pragma once

#include "common.cuh"
#include "yee.cuh"

namespace lsfdtd {

template <typename F>
struct FusedArgs {
  YeeArgs<F> y;        // in buffers (E, H, psi) and coefficients
  F* Eo[3];            // out buffers
  F* Ho[3];
  F* psiHo[3][3][2];   // out H psi per [axis d][component][side]
  int seg;             // x planes per CTA
};

// CPML terms with separate psi in / out (out may be null: a halo node, computed but not stored)
template <int FLD, typename F>
__device__ __forceinline__ void cpml_io(F& v, const YeeArgs<F>& g, F* const (*psi_out)[3][2], int c, const int* x,
                                        F der1, F der2, typename real_of<F>::type scale, bool store) {
  using R = typename real_of<F>::type;
  const int d1 = (c + 1) % 3;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d == c) continue;
    const PmlAxis<F>& p = g.pml[d];
    if (!p.on) continue;
    const F der = d == d1 ? der1 : der2;
    R sgn = (d == d1) ? R(1) : R(-1);
    if (FLD == 1) sgn = -sgn;
    const int u = x[d];
    R s = g.uniform ? scale : scale / p.div;
    s = sgn * s;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const int st = p.start[FLD][c][side], ln = p.len[FLD][c][side];
      if (u < st || u >= st + ln) continue;
      const long long q = psi_index(x, g.n, d, u - st, ln);
      F psi = p.psi[FLD][c][side][q] * p.b[FLD][u];
      if (p.k[FLD]) v += (s * p.k[FLD][u]) * der;
      psi += der * (s * p.c[FLD][u]);
      if (store) {
        F* dst = FLD == 1 ? psi_out[d][c][side] : p.psi[FLD][c][side];
        dst[q] = psi;
      }
      v += psi;
    }
  }
}

template <typename F, int TY>
__global__ void __launch_bounds__(32 * TY) k_fused_step(FusedArgs<F> a) {
  using R = typename real_of<F>::type;
  constexpr int TZ = 32, SY = TY + 2, SZ = TZ + 2, NT = TZ * TY;
  constexpr int NE = 3 * SY * SZ;            // E values of one plane with its halo
  constexpr int NQ = (NE + NT - 1) / NT;     // per thread
  __shared__ F sE[2][3][SY][SZ];
  __shared__ F sH[3][TY + 1][TZ + 1];
  const YeeArgs<F>& g = a.y;
  const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TZ + tx;
  const int z0 = blockIdx.x * TZ, y0 = blockIdx.y * TY;
  const int k = z0 + tx, j = y0 + ty;
  const int xs = blockIdx.z * a.seg;
  const int xe = min(n0, xs + a.seg);
  if (xs >= n0) return;
  const bool own = k < n2 && j < n1;
  const long long s1 = n2, s0 = (long long)n1 * n2;

  F pre[NQ];
  auto issue = [&](int i) {
#pragma unroll
    for (int u = 0; u < NQ; ++u) {
      const int q = tid + u * NT;
      F v = zero<F>();
      if (q < NE && i < n0) {
        const int c = q / (SY * SZ), r = q % (SY * SZ);
        const int y = y0 - 1 + r / SZ, z = z0 - 1 + r % SZ;
        if (y >= 0 && y < n1 && z >= 0 && z < n2) v = g.E[c][i * s0 + y * s1 + z];
      }
      pre[u] = v;
    }
  };
  auto commit = [&](int buf) {
#pragma unroll
    for (int u = 0; u < NQ; ++u) {
      const int q = tid + u * NT;
      if (q < NE) {
        const int c = q / (SY * SZ), r = q % (SY * SZ);
        sE[buf][c][r / SZ][r % SZ] = pre[u];
      }
    }
  };
  // H^{n+1/2}_c at plane i, local shared-memory position (yy, zz) of node (i, y0-1+yy, z0-1+zz)
  auto h_at = [&](int c, int cur, int i, int yy, int zz, bool store) -> F {
    const int x[3] = {i, y0 - 1 + yy, z0 - 1 + zz};
    const long long p = i * s0 + (long long)x[1] * s1 + x[2];
    const F h0 = g.H[c][p];
    if (!in_h_region(c, x, g.n, g.periodic)) {
      if (store) a.Ho[c][p] = h0;
      return h0;
    }
    const int nx = cur ^ 1;
    F av, bv;
    if (c == 0) {
      av = sE[cur][2][yy + 1][zz] - sE[cur][2][yy][zz];
      bv = sE[cur][1][yy][zz + 1] - sE[cur][1][yy][zz];
    } else if (c == 1) {
      av = sE[cur][0][yy][zz + 1] - sE[cur][0][yy][zz];
      bv = sE[nx][2][yy][zz] - sE[cur][2][yy][zz];
    } else {
      av = sE[nx][1][yy][zz] - sE[cur][1][yy][zz];
      bv = sE[cur][0][yy + 1][zz] - sE[cur][0][yy][zz];
    }
    const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    const F curl = g.uniform ? (av - bv) : (av * g.inv_d[d1] - bv * g.inv_d[d2]);
    F h = h0 - curl * g.cH;
    cpml_io<1>(h, g, a.psiHo, c, x, av, bv, g.cH, store);
    if (store) a.Ho[c][p] = h;
    return h;
  };

  int cur = 0;
  F prev_hy = zero<F>(), prev_hz = zero<F>();
  if (xs > 0) {
    // H_y, H_z of plane xs - 1 on the tile, for the x differences of E(xs); stored by the CTA that owns it
    issue(xs - 1);
    commit(0);
    issue(xs);
    commit(1);
    __syncthreads();
    if (own) {
      prev_hy = h_at(1, 0, xs - 1, ty + 1, tx + 1, false);
      prev_hz = h_at(2, 0, xs - 1, ty + 1, tx + 1, false);
    }
    __syncthreads();
    issue(xs + 1);
    commit(0);
    cur = 1;
    __syncthreads();
  } else {
    issue(0);
    commit(0);
    issue(1);
    commit(1);
    __syncthreads();
  }

  for (int i = xs; i < xe; ++i) {
    issue(i + 2);
    F h_own[3];
    if (own) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        h_own[c] = h_at(c, cur, i, ty + 1, tx + 1, true);
        sH[c][ty + 1][tx + 1] = h_own[c];
      }
    }
    // the low halo: H_x, H_z on row y0 - 1 and H_x, H_y on column z0 - 1
    if (ty == 0 && y0 > 0 && k < n2) {
      sH[0][0][tx + 1] = h_at(0, cur, i, 0, tx + 1, false);
      sH[2][0][tx + 1] = h_at(2, cur, i, 0, tx + 1, false);
    }
    if (tx == 0 && z0 > 0 && j < n1) {
      sH[0][ty + 1][0] = h_at(0, cur, i, ty + 1, 0, false);
      sH[1][ty + 1][0] = h_at(1, cur, i, ty + 1, 0, false);
    }
    __syncthreads();
    if (own) {
      const int x[3] = {i, j, k};
      const long long p = i * s0 + (long long)j * s1 + k;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const F e0 = sE[cur][c][ty + 1][tx + 1];
        if (!in_e_region(c, x, g.n, g.periodic)) {
          a.Eo[c][p] = e0;
          continue;
        }
        F av, bv;
        if (c == 0) {
          av = sH[2][ty + 1][tx + 1] - sH[2][ty][tx + 1];
          bv = sH[1][ty + 1][tx + 1] - sH[1][ty + 1][tx];
        } else if (c == 1) {
          av = sH[0][ty + 1][tx + 1] - sH[0][ty + 1][tx];
          bv = h_own[2] - prev_hz;
        } else {
          av = h_own[1] - prev_hy;
          bv = sH[0][ty + 1][tx + 1] - sH[0][ty][tx + 1];
        }
        const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
        const F curl = g.uniform ? (av - bv) : (av * g.inv_d[d1] - bv * g.inv_d[d2]);
        const R cb = g.cbE[c][p];
        F e = e0 + curl * cb;
        cpml_io<0>(e, g, a.psiHo, c, x, av, bv, cb, true);
        a.Eo[c][p] = e;
      }
      prev_hy = h_own[1];
      prev_hz = h_own[2];
    }
    __syncthreads();
    commit(cur);  // E^n(i+2) replaces E^n(i)
    cur ^= 1;
    __syncthreads();
  }
}

}  // namespace lsfdtd
