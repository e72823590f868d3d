// The fused single-pass FDTD step with its x-plane ring filled by the Tensor Memory Accelerator.
//
// Same step and tiling as k_fused_step (fused.cuh): a CTA owns a 32 (z) x TY (y) tile, marches through a
// segment of x planes and computes H^{n+1/2} then E^{n+1} per plane from a ring of S shared-memory stages.
// Here one thread fills a stage with seven bulk tensor copies (cp.async.bulk.tensor, no multicast): the
// three E^n components over y0-1 .. y0+TY and z0-4 .. z0+35, the three H^n components over y0-1 .. y0+TY-1
// and the same z range, and the coefficient tile. Each stage has an mbarrier that the copies complete;
// the other threads do no copy work at all, which is what limited the cp.async ring.
//
// With BOX, the kernel steps only the interior box of the split step (FusedArgs::box_lo/box_hi): every node
// it updates or recomputes lies inside every component's stepped region and outside every CPML slab, so the
// region and CPML code is compiled out; the nodes outside the box are stepped by k_shell_h and k_shell_e
// (shell.cuh).
//
// Every box starts at z0 - 4 (a multiple of four nodes, so 16-byte aligned in both precisions) and may
// start before the grid or run past it; the tensor maps fill such nodes with zeros. Waits on an mbarrier are
// bounded by a clock budget: a CTA that exceeds it (copies that never complete) records status 1, waits a
// bounded time for its copies still in flight and returns.
#pragma once

#include <cuda.h>

#include "common.cuh"
#include "fused.cuh"

namespace lsfdtd {

// CTAs of the lean pass over boxes of tiles and x planes: box b holds CTAs first .. first + count - 1, z tiles
// [t0[0], t1[0]) (of 32 nodes), y tiles [t0[1], t1[1]) (of the launch's tile rows) and x planes [x0, x1) in
// segments of seg planes, z tile fastest, then y tile, then segment
struct CtaBox {
  int t0[2], t1[2];
  int x0, x1, seg;
  int first;
};
constexpr int kMaxCtaBoxes = 12;
struct CtaMap {
  int n;
  CtaBox box[kMaxCtaBoxes];
};

template <typename F>
struct TmaArgs {
  FusedArgs<F> f;
  CtaMap map;          // the CTAs of this launch (k_fused_pml)
  CUtensorMap mE[3];   // E^n components, box 40 x (TY + 2) x 1
  CUtensorMap mH[3];   // H^n components, box 40 x (TY + 1) x 1
  CUtensorMap mC;      // cbE (component 0), box 32 x TY x 1
  int* status;         // set to 1 when a copy wait exceeded its budget
  // clock cycles a CTA waits for one plane's copies before it gives up; negative: a timeout test, in which
  // every wait is on a barrier that nothing completes and gives up after -wait_budget cycles (the copies the
  // pass issued still complete, and it drains them before it returns)
  long long wait_budget;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
          "r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ float shfl_up(unsigned m, float v) { return __shfl_up_sync(m, v, 1); }
__device__ __forceinline__ double shfl_up(unsigned m, double v) { return __shfl_up_sync(m, v, 1); }

__device__ __forceinline__ bool mbar_test_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// budgets below this many cycles are polled with the non-blocking test (try_wait may suspend the thread for
// longer than such a budget, until the phase completes)
constexpr long long kPollBelow = 1LL << 20;

// bounded wait: false when the budget ran out
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, long long budget) {
  if (budget < kPollBelow) {
    const long long t0 = clock64();
    while (!mbar_test_wait(bar, parity))
      if (clock64() - t0 > budget) return false;
    return true;
  }
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > budget) return false;
  }
  return true;
}

// the default wait budget: about 2 s, where copies of a few KB take microseconds
constexpr long long kWaitBudget = 4000000000LL;
constexpr long long kDrainBudget = 200000000LL;

template <typename F, int TY>
struct TmaStage {
  static constexpr int BZ = 40;                      // z0 - 4 .. z0 + 35
  static constexpr size_t align128(size_t b) { return (b + 127) / 128 * 128; }
  static constexpr size_t kE = align128(sizeof(F) * (TY + 2) * BZ);
  static constexpr size_t kH = align128(sizeof(F) * (TY + 1) * BZ);
  static constexpr size_t kC = align128(sizeof(typename real_of<F>::type) * TY * 32);
  static constexpr size_t kBytes = 3 * kE + 3 * kH + kC;
  // bytes the seven copies deliver (whole boxes, zero-filled where they leave the grid)
  static constexpr unsigned kTx = (unsigned)(3 * sizeof(F) * (TY + 2) * BZ + 3 * sizeof(F) * (TY + 1) * BZ +
                                             sizeof(typename real_of<F>::type) * TY * 32);
};

// dynamic shared memory of the fused passes, from its first 128-byte boundary: the copy ring, the rows of H
// exchanged between warps (two planes), the ring's mbarriers and the tile's halo column of H (two planes)
template <typename F, int TY, int S>
struct TmaLayout {
  static constexpr size_t kRing = S * TmaStage<F, TY>::kBytes;
  static constexpr size_t kRows = 2 * 2 * (TY + 1) * 32 * sizeof(F);
  static constexpr size_t kBars = S * 8;
  static constexpr size_t kCol = (2 * 2 * TY * sizeof(F) + 15) / 16 * 16;
  static constexpr size_t kUsed = kRing + kRows + kBars + kCol;
};

template <typename F, int TY, int S>
constexpr size_t fused_tma_smem_bytes() {
  // + 128: the ring is placed at the first 128-byte boundary of the dynamic shared memory
  return 128 + TmaLayout<F, TY, S>::kUsed;
}

template <typename F, int TY, int S, bool BOX>
__global__ void __launch_bounds__(32 * TY) k_fused_tma(const __grid_constant__ TmaArgs<F> t) {
  using R = typename real_of<F>::type;
  using St = TmaStage<F, TY>;
  constexpr int TZ = 32, BZ = St::BZ;
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  // bulk tensor copies need 128-byte aligned destinations
  unsigned char* smem = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);
  using L = TmaLayout<F, TY, S>;
  F(*sH)[2][TY + 1][TZ] = reinterpret_cast<F(*)[2][TY + 1][TZ]>(smem + L::kRing);
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem + L::kRing + L::kRows);
  F(*zc)[2][TY] = reinterpret_cast<F(*)[2][TY]>(smem + L::kRing + L::kRows + L::kBars);  // [plane][H_x, H_y][row]

  const FusedArgs<F>& a = t.f;
  const YeeArgs<F>& g = a.y;
  const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TZ + tx;
  const int z0 = (BOX ? a.box_lo[2] : 0) + blockIdx.x * TZ, y0 = (BOX ? a.box_lo[1] : 0) + blockIdx.y * TY;
  const int k = z0 + tx, j = y0 + ty;
  const int xs = (BOX ? a.box_lo[0] : 0) + blockIdx.z * a.seg;
  const int xend = BOX ? a.box_hi[0] : n0;
  if (xs >= xend) return;
  const int xe = min(xend, xs + a.seg);
  const int xb = xs > 0 ? xs - 1 : 0;
  const bool own = BOX ? (k < a.box_hi[2] && j < a.box_hi[1]) : (k < n2 && j < n1);
  const long long s1 = n2, s0 = (long long)n1 * n2;

  auto stE = [&](int s, int c) { return reinterpret_cast<F(*)[BZ]>(smem + s * St::kBytes + c * St::kE); };
  auto stH = [&](int s, int c) {
    return reinterpret_cast<F(*)[BZ]>(smem + s * St::kBytes + 3 * St::kE + c * St::kH);
  };
  auto stC = [&](int s) { return reinterpret_cast<R(*)[TZ]>(smem + s * St::kBytes + 3 * St::kE + 3 * St::kH); };

  __shared__ unsigned long long never;  // a barrier nothing completes: the wait of a timeout test
  if (tid == 0) {
    mbar_init(&never, 1);
    for (int s = 0; s < S; ++s) mbar_init(&bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  // plane p goes to stage (p - xb) % S; its fill is that stage's ((p - xb) / S)-th
  auto produce = [&](int p) {
    const int s = (p - xb) % S;
    mbar_expect_tx(&bar[s], St::kTx);
    for (int c = 0; c < 3; ++c) tma_load_3d(stE(s, c), &t.mE[c], z0 - 4, y0 - 1, p, &bar[s]);
    for (int c = 0; c < 3; ++c) tma_load_3d(stH(s, c), &t.mH[c], z0 - 4, y0 - 1, p, &bar[s]);
    tma_load_3d(stC(s), &t.mC, z0, y0, p, &bar[s]);
  };
  auto ready = [&](int p) -> bool {
    if (t.wait_budget < 0) return mbar_wait_bounded(&never, 0, -t.wait_budget);  // a timeout test: see TmaArgs
    return mbar_wait_bounded(&bar[(p - xb) % S], ((p - xb) / S) & 1, t.wait_budget);
  };
  int issued = xb - 1;  // last plane whose copies were issued
  if (tid == 0) {
    for (int p = xb; p < xb + S - 1; ++p) produce(p);
  }
  issued = xb + S - 2;

  // H^{n+1/2}_c of the node at box row `row` (y = y0 - 1 + row) and box column `col` (z = z0 - 4 + col) of
  // plane i, with region and CPML tests (walls and absorbing slabs); stages si (plane i), sn (plane i + 1)
  auto h_checked = [&](int c, int si, int sn, int i, int row, int col, bool store) -> F {
    const int x[3] = {i, y0 - 1 + row, z0 - 4 + col};
    const F h0 = stH(si, c)[row][col];
    const long long p = i * s0 + (long long)x[1] * s1 + x[2];
    if (!in_h_region(c, x, g.n, g.periodic)) {
      if (store) st_global(a.Ho[c] + p, h0);
      return h0;
    }
    F av, bv;
    if (c == 0) {
      av = stE(si, 2)[row + 1][col] - stE(si, 2)[row][col];
      bv = stE(si, 1)[row][col + 1] - stE(si, 1)[row][col];
    } else if (c == 1) {
      av = stE(si, 0)[row][col + 1] - stE(si, 0)[row][col];
      bv = stE(sn, 2)[row][col] - stE(si, 2)[row][col];
    } else {
      av = stE(sn, 1)[row][col] - stE(si, 1)[row][col];
      bv = stE(si, 0)[row + 1][col] - stE(si, 0)[row][col];
    }
    const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    const F curl = g.uniform ? (av - bv) : (av * g.inv_d[d1] - bv * g.inv_d[d2]);
    F h = h0 - curl * g.cH;
    cpml_io<1>(h, a, c, x, av, bv, g.cH, store);
    if (store) st_global(a.Ho[c] + p, h);
    return h;
  };
  // the same for a node inside every component's stepped region and outside every CPML slab
  auto curl = [&](F av, F bv, int d1, int d2) -> F {
    return g.uniform ? (av - bv) : (av * g.inv_d[d1] - bv * g.inv_d[d2]);
  };
  auto hx_fast = [&](int si, int o) -> F {
    const F* ey = &stE(si, 1)[0][0];
    const F* ez = &stE(si, 2)[0][0];
    return stH(si, 0)[0][o] - curl(ez[o + BZ] - ez[o], ey[o + 1] - ey[o], 1, 2) * g.cH;
  };
  auto hy_fast = [&](int si, int sn, int o) -> F {
    const F* ex = &stE(si, 0)[0][0];
    const F* ez = &stE(si, 2)[0][0];
    return stH(si, 1)[0][o] - curl(ex[o + 1] - ex[o], (&stE(sn, 2)[0][0])[o] - ez[o], 2, 0) * g.cH;
  };
  auto hz_fast = [&](int si, int sn, int o) -> F {
    const F* ex = &stE(si, 0)[0][0];
    const F* ey = &stE(si, 1)[0][0];
    return stH(si, 2)[0][o] - curl((&stE(sn, 1)[0][0])[o] - ey[o], ex[o + BZ] - ex[o], 0, 1) * g.cH;
  };

  // per-thread constants: the own node (row ty + 1, column tx + 4 of the boxes), and whether it and the halo
  // nodes this thread computes are interior along y and z
  const unsigned full = 0xffffffffu;
  const int oo = (ty + 1) * BZ + tx + 4;
  const long long off_jk = (long long)j * s1 + k;
  const bool yz_in = own && j >= a.inner_lo[1] && j < a.inner_hi[1] && k >= a.inner_lo[2] && k < a.inner_hi[2];
  const bool yh_in = y0 - 1 >= a.inner_lo[1] && y0 - 1 < a.inner_hi[1] && k >= a.inner_lo[2] && k < a.inner_hi[2];
  // the halo column's node of row y0 + tx (computed by lane tx of warp kColWarp)
  const bool col_in = y0 + tx >= a.inner_lo[1] && y0 + tx < a.inner_hi[1] && z0 - 1 >= a.inner_lo[2] &&
                      z0 - 1 < a.inner_hi[2];
  constexpr int kColWarp = TY > 1 ? 1 : 0;  // warp 0 computes the halo row
  const bool multi_cb = g.cbE[1] != g.cbE[0] || g.cbE[2] != g.cbE[0];

  F prev_hy = zero<F>(), prev_hz = zero<F>();
  bool failed = false;
  int cons = xb - 1;  // planes up to cons have landed and were waited on by every thread
#pragma unroll 1
  for (int i = xb; i < xe; ++i) {
    const bool ok = (i > xb || ready(i)) && ready(i + 1);  // plane i was waited for as plane i + 1 before
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    cons = i + 1;
    if (tid == 0) produce(i + S - 1);  // into the stage of plane i - 1, which every thread has finished with
    issued = i + S - 1;
    const int si = (i - xb) % S, sn = (i + 1 - xb) % S;
    const bool x_in = BOX || (i >= a.inner_lo[0] && i < a.inner_hi[0]);
    const bool fast = BOX || (x_in && yz_in);
    if (i < xs) {  // the plane before the segment: H_y, H_z of the own node, stored by the CTA owning it
      if (own) {
        if (fast) {
          prev_hy = hy_fast(si, sn, oo);
          prev_hz = hz_fast(si, sn, oo);
        } else {
          prev_hy = h_checked(1, si, sn, i, ty + 1, tx + 4, false);
          prev_hz = h_checked(2, si, sn, i, ty + 1, tx + 4, false);
        }
      }
      continue;
    }
    const long long p = i * s0 + off_jk;
    F hx = zero<F>(), hy = zero<F>(), hz = zero<F>();
    if (fast) {
      hx = hx_fast(si, oo);
      hy = hy_fast(si, sn, oo);
      hz = hz_fast(si, sn, oo);
      if (!BOX || own) {  // without BOX, fast implies own
        st_global(a.Ho[0] + p, hx);
        st_global(a.Ho[1] + p, hy);
        st_global(a.Ho[2] + p, hz);
      }
    } else if (own) {
      hx = h_checked(0, si, sn, i, ty + 1, tx + 4, true);
      hy = h_checked(1, si, sn, i, ty + 1, tx + 4, true);
      hz = h_checked(2, si, sn, i, ty + 1, tx + 4, true);
    }
    // y neighbours through shared memory (row 0: the halo row y0 - 1), z neighbours through shuffles
    F(&hs)[2][TY + 1][TZ] = sH[i & 1];
    hs[0][ty + 1][tx] = hx;
    hs[1][ty + 1][tx] = hz;
    if (ty == 0 && y0 > 0 && k < n2) {
      const int o = tx + 4;  // box row 0
      if (BOX || (x_in && yh_in)) {
        hs[0][0][tx] = hx_fast(si, o);
        hs[1][0][tx] = hz_fast(si, sn, o);
      } else {
        hs[0][0][tx] = h_checked(0, si, sn, i, 0, o, false);
        hs[1][0][tx] = h_checked(2, si, sn, i, 0, o, false);
      }
    }
    // the halo column z0 - 1 (H_x, H_y of every row, for lane 0 of each warp): one warp, lane r for row r
    if (ty == kColWarp && tx < TY && z0 > 0 && y0 + tx < n1) {
      const int o = (tx + 1) * BZ + 3;
      if (BOX || (x_in && col_in)) {
        zc[i & 1][0][tx] = hx_fast(si, o);
        zc[i & 1][1][tx] = hy_fast(si, sn, o);
      } else {
        zc[i & 1][0][tx] = h_checked(0, si, sn, i, tx + 1, 3, false);
        zc[i & 1][1][tx] = h_checked(1, si, sn, i, tx + 1, 3, false);
      }
    }
    F hx_zm = shfl_up(full, hx), hy_zm = shfl_up(full, hy);
    __syncthreads();
    if (tx == 0) {
      hx_zm = zc[i & 1][0][ty];
      hy_zm = zc[i & 1][1][ty];
    }
    if (own) {
      const F hz_ym = hs[1][ty][tx], hx_ym = hs[0][ty][tx];
      const R cb = stC(si)[ty][tx];
      const F* ex = &stE(si, 0)[0][0];
      const F* ey = &stE(si, 1)[0][0];
      const F* ez = &stE(si, 2)[0][0];
      // (a, b) per component: E_c += (dH_{d2}/dd1 - dH_{d1}/dd2) cbE_c
      const F a0 = hz - hz_ym, b0 = hy - hy_zm;
      const F a1 = hx - hx_zm, b1 = hz - prev_hz;
      const F a2 = hy - prev_hy, b2 = hx - hx_ym;
      if (fast && !multi_cb) {
        st_global(a.Eo[0] + p, ex[oo] + curl(a0, b0, 1, 2) * cb);
        st_global(a.Eo[1] + p, ey[oo] + curl(a1, b1, 2, 0) * cb);
        st_global(a.Eo[2] + p, ez[oo] + curl(a2, b2, 0, 1) * cb);
      } else {
        const int x[3] = {i, j, k};
        const F av[3] = {a0, a1, a2}, bv[3] = {b0, b1, b2};
        const F* e[3] = {ex, ey, ez};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const F e0 = e[c][oo];
          if (!fast && !in_e_region(c, x, g.n, g.periodic)) {
            st_global(a.Eo[c] + p, e0);
            continue;
          }
          const R cbc = c == 0 ? cb : g.cbE[c][p];
          F ev = e0 + curl(av[c], bv[c], (c + 1) % 3, (c + 2) % 3) * cbc;
          if (!fast) cpml_io<0>(ev, a, c, x, av[c], bv[c], cbc, true);
          st_global(a.Eo[c] + p, ev);
        }
      }
    }
    prev_hy = hy;
    prev_hz = hz;
  }
  // every issued copy must land before the CTA's shared memory is released (each stage has at most one fill
  // in flight beyond the planes consumed, so each wait below targets the stage's latest fill)
  if (tid == 0) {
    for (int p = cons + 1; p <= issued; ++p) mbar_wait_bounded(&bar[(p - xb) % S], ((p - xb) / S) & 1, kDrainBudget);
    if (failed && t.status) atomicExch(t.status, 1);
  }
  __syncthreads();
}

}  // namespace lsfdtd
