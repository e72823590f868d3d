// One FDTD step (H half step then E half step, CPML included) in a single pass over the grid.
//
// Each CTA owns a tile of TZ = 32 nodes along z (contiguous) by TY nodes along y and marches through a
// segment of x planes. A ring of S shared-memory stages holds, per x plane, E^n (tile plus a one-node halo),
// H^n (tile plus the low-side halo) and the E coefficient (tile); the stages are filled with cp.async several
// planes ahead of the computation, so the copies of the next planes are in flight while plane i is computed.
// For plane i the CTA computes H^{n+1/2}(i) on the tile and on the low halo row and column it needs, then
// E^{n+1}(i) on the tile, reading H^{n+1/2}(i-1) of its own nodes from registers.
//
// The halo H of a tile is recomputed by the tile itself, so E, H and the H-side CPML psi are double
// buffered: a step reads the "in" buffers and writes the "out" buffers, and no CTA can observe a value
// another CTA has already advanced. Per cell and step that is E, H and one coefficient read once and E, H
// written once (52 B in FP32), plus the psi of CPML cells. Nodes outside a component's stepped region are
// copied, so the two buffers always agree there. Tiles and planes away from the CPML slabs and the PEC
// walls take a path without any region or CPML test.
//
// The arithmetic per value is that of k_update_h / k_update_e (and of lightsmith's engine.py:613-663).
#pragma once

#include "common.cuh"
#include "yee.cuh"

namespace lsfdtd {

// TF/SF corrections of H applied inside the fused pass (a table-fed source's correct_H, layered.py:231-242):
// box b adds vals[off + ((x - lo0) (hi1 - lo1) + (y - lo1)) (hi2 - lo2) + (z - lo2)] to H_c at the nodes
// [lo, hi) of the box, boxes in the source's slab order; vals holds the step's values, one per entry
constexpr int kMaxHBoxes = 24;
struct HCorrBox {
  int c;
  int lo[3], hi[3];
  int off;
};
struct HCorr {
  int n;  // boxes (0: none)
  HCorrBox box[kMaxHBoxes];
  const void* vals;
};

template <typename F>
struct FusedArgs {
  YeeArgs<F> y;        // in buffers (E, H, psi) and coefficients
  F* Eo[3];            // out buffers
  F* Ho[3];
  F* psiHo[3][3][2];   // out H psi per [axis d][component][side]
  int seg;             // x planes per CTA
  int inner_lo[3];     // nodes [inner_lo, inner_hi) along each axis are stepped for every component and lie
  int inner_hi[3];     // outside every CPML slab
  int pml_lo[3];       // CPML cells per axis and side (0: none)
  int pml_hi[3];
  int box_lo[3];       // the interior box of the split step: nodes [box_lo, box_hi) per axis, each of them and
  int box_hi[3];       // its low-side neighbours inside [inner_lo, inner_hi); box_lo[2] a multiple of four
  HCorr hc;            // TF/SF corrections of H (the lean pass only)
};

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, bool valid) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 4 : 0));
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

template <typename T>
__device__ __forceinline__ void cp_async(T* smem, const T* gmem, bool valid) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte field values");
  if constexpr (sizeof(T) == 4)
    cp_async4(smem, gmem, valid);
  else
    cp_async8(smem, gmem, valid);
}

// CPML terms with separate psi in / out for H (out may be skipped: a halo node, computed but not stored)
template <int FLD, typename F>
__device__ __forceinline__ void cpml_io(F& v, const FusedArgs<F>& a, int c, const int* x, F der1, F der2,
                                        typename real_of<F>::type scale, bool store) {
  using R = typename real_of<F>::type;
  const YeeArgs<F>& g = a.y;
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
        F* dst = FLD == 1 ? a.psiHo[d][c][side] : p.psi[FLD][c][side];
        dst[q] = psi;
      }
      v += psi;
    }
  }
}

template <typename F, int TY>
struct FusedStage {
  static constexpr int TZ = 32, SY = TY + 2, SZ = TZ + 2;
  F E[3][SY][SZ];           // E^n at (y0 - 1 + yy, z0 - 1 + zz)
  F H[3][TY + 1][TZ + 1];   // H^n at (y0 - 1 + yy, z0 - 1 + zz)
  typename real_of<F>::type cb[TY][TZ];
};

template <typename F, int TY, int S>
__global__ void __launch_bounds__(32 * TY) k_fused_step(const __grid_constant__ FusedArgs<F> a) {
  using R = typename real_of<F>::type;
  using Stage = FusedStage<F, TY>;
  constexpr int TZ = 32, SY = TY + 2, SZ = TZ + 2, NT = TZ * TY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Stage* st = reinterpret_cast<Stage*>(smem_raw);
  F(*sH)[3][TY + 1][TZ + 1] = reinterpret_cast<F(*)[3][TY + 1][TZ + 1]>(smem_raw + S * sizeof(Stage));

  const YeeArgs<F>& g = a.y;
  const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TZ + tx;
  const int z0 = blockIdx.x * TZ, y0 = blockIdx.y * TY;
  const int k = z0 + tx, j = y0 + ty;
  const int xs = blockIdx.z * a.seg;
  if (xs >= n0) return;
  const int xe = min(n0, xs + a.seg);
  const int xb = xs > 0 ? xs - 1 : 0;  // first plane held: xs - 1 supplies H(xs - 1) for the x differences
  const bool own = k < n2 && j < n1;
  const long long s1 = n2, s0 = (long long)n1 * n2;
  // the tile and its halo rows/columns are all interior along y and z
  const bool tile_inner = y0 - 1 >= a.inner_lo[1] && y0 + TY <= a.inner_hi[1] && z0 - 1 >= a.inner_lo[2] &&
                          z0 + TZ <= a.inner_hi[2];

  // copies of plane p into stage p % S (out-of-grid values are zero-filled)
  auto fetch = [&](int p) {
    Stage& sg = st[((p % S) + S) % S];
    const bool pin = p < n0;
    const long long pb = (long long)(pin ? p : 0) * s0;
    for (int q = tid; q < 3 * SY * SZ; q += NT) {
      const int c = q / (SY * SZ), r = q % (SY * SZ);
      const int y = y0 - 1 + r / SZ, z = z0 - 1 + r % SZ;
      const bool v = pin && y >= 0 && y < n1 && z >= 0 && z < n2;
      cp_async(&sg.E[c][r / SZ][r % SZ], g.E[c] + (v ? pb + y * s1 + z : 0), v);
    }
    for (int q = tid; q < 3 * (TY + 1) * (TZ + 1); q += NT) {
      const int c = q / ((TY + 1) * (TZ + 1)), r = q % ((TY + 1) * (TZ + 1));
      const int y = y0 - 1 + r / (TZ + 1), z = z0 - 1 + r % (TZ + 1);
      const bool v = pin && y >= 0 && y < n1 && z >= 0 && z < n2;
      cp_async(&sg.H[c][r / (TZ + 1)][r % (TZ + 1)], g.H[c] + (v ? pb + y * s1 + z : 0), v);
    }
    {
      const bool v = pin && own;
      cp_async(&sg.cb[ty][tx], g.cbE[0] + (v ? pb + j * s1 + k : 0), v);
    }
    cp_async_commit();
  };

  // H^{n+1/2}_c of node (i, y0 - 1 + yy, z0 - 1 + zz); ci / cn: stages of planes i and i + 1
  auto h_at = [&](int c, const Stage& ci, const Stage& cn, int i, int yy, int zz, bool fast, bool store) -> F {
    const int x[3] = {i, y0 - 1 + yy, z0 - 1 + zz};
    const F h0 = ci.H[c][yy][zz];
    const long long p = i * s0 + (long long)x[1] * s1 + x[2];
    if (!fast && !in_h_region(c, x, g.n, g.periodic)) {
      if (store) a.Ho[c][p] = h0;
      return h0;
    }
    F av, bv;
    if (c == 0) {
      av = ci.E[2][yy + 1][zz] - ci.E[2][yy][zz];
      bv = ci.E[1][yy][zz + 1] - ci.E[1][yy][zz];
    } else if (c == 1) {
      av = ci.E[0][yy][zz + 1] - ci.E[0][yy][zz];
      bv = cn.E[2][yy][zz] - ci.E[2][yy][zz];
    } else {
      av = cn.E[1][yy][zz] - ci.E[1][yy][zz];
      bv = ci.E[0][yy + 1][zz] - ci.E[0][yy][zz];
    }
    const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    const F curl = g.uniform ? (av - bv) : (av * g.inv_d[d1] - bv * g.inv_d[d2]);
    F h = h0 - curl * g.cH;
    if (!fast) cpml_io<1>(h, a, c, x, av, bv, g.cH, store);
    if (store) a.Ho[c][p] = h;
    return h;
  };

  // prime the ring: planes xb .. xb + S - 2
#pragma unroll 1
  for (int p = xb; p < xb + S - 1; ++p) fetch(p);

  F prev_hy = zero<F>(), prev_hz = zero<F>();
#pragma unroll 1
  for (int i = xb; i < xe; ++i) {
    cp_async_wait<S - 3>();  // planes i and i + 1 have landed
    __syncthreads();
    fetch(i + S - 1);        // into the stage of plane i - 1, which every thread has finished with
    const Stage& ci = st[i % S];
    const Stage& cn = st[(i + 1) % S];
    const bool fast = tile_inner && i >= a.inner_lo[0] && i < a.inner_hi[0];
    if (i < xs) {  // the plane before the segment: H_y, H_z of the tile only, stored by the CTA owning it
      if (own) {
        prev_hy = h_at(1, ci, cn, i, ty + 1, tx + 1, fast, false);
        prev_hz = h_at(2, ci, cn, i, ty + 1, tx + 1, fast, false);
      }
      continue;
    }
    F(&hs)[3][TY + 1][TZ + 1] = sH[i & 1];
    F h_own[3];
    if (own) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        h_own[c] = h_at(c, ci, cn, i, ty + 1, tx + 1, fast, true);
        hs[c][ty + 1][tx + 1] = h_own[c];
      }
    }
    // the low halo: H_x, H_z on row y0 - 1 and H_x, H_y on column z0 - 1
    if (ty == 0 && y0 > 0 && k < n2) {
      hs[0][0][tx + 1] = h_at(0, ci, cn, i, 0, tx + 1, fast, false);
      hs[2][0][tx + 1] = h_at(2, ci, cn, i, 0, tx + 1, fast, false);
    }
    if (tx == 0 && z0 > 0 && j < n1) {
      hs[0][ty + 1][0] = h_at(0, ci, cn, i, ty + 1, 0, fast, false);
      hs[1][ty + 1][0] = h_at(1, ci, cn, i, ty + 1, 0, fast, false);
    }
    __syncthreads();
    if (own) {
      const int x[3] = {i, j, k};
      const long long p = i * s0 + (long long)j * s1 + k;
      const R cb = ci.cb[ty][tx];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const F e0 = ci.E[c][ty + 1][tx + 1];
        if (!fast && !in_e_region(c, x, g.n, g.periodic)) {
          a.Eo[c][p] = e0;
          continue;
        }
        F av, bv;
        if (c == 0) {
          av = hs[2][ty + 1][tx + 1] - hs[2][ty][tx + 1];
          bv = hs[1][ty + 1][tx + 1] - hs[1][ty + 1][tx];
        } else if (c == 1) {
          av = hs[0][ty + 1][tx + 1] - hs[0][ty + 1][tx];
          bv = h_own[2] - prev_hz;
        } else {
          av = h_own[1] - prev_hy;
          bv = hs[0][ty + 1][tx + 1] - hs[0][ty][tx + 1];
        }
        const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
        const F curl = g.uniform ? (av - bv) : (av * g.inv_d[d1] - bv * g.inv_d[d2]);
        const R cbc = (c == 0 || g.cbE[c] == g.cbE[0]) ? cb : g.cbE[c][p];
        F e = e0 + curl * cbc;
        if (!fast) cpml_io<0>(e, a, c, x, av, bv, cbc, true);
        a.Eo[c][p] = e;
      }
      prev_hy = h_own[1];
      prev_hz = h_own[2];
    }
  }
  cp_async_wait<0>();
}

template <typename F, int TY, int S>
constexpr size_t fused_smem_bytes() {
  return S * sizeof(FusedStage<F, TY>) + 2 * 3 * (TY + 1) * (32 + 1) * sizeof(F);
}

}  // namespace lsfdtd
