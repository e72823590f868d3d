// The fused single pass over the whole grid with lean CPML terms.
//
// Same tiling, copy ring and step as k_fused_tma (fused_tma.cuh): a CTA owns a 32 (z) x TY (y) tile, marches
// through a segment of x planes fed by bulk tensor copies, and computes H^{n+1/2} then E^{n+1} per plane, the
// halo H of its tile recomputed in place. What differs is how nodes near the boundary are stepped.
//
// A warp whose nodes and halo nodes all lie inside every component's stepped region and outside every CPML
// slab takes the region- and CPML-free path (the whole warp, per plane). Any other warp takes the lean path,
// in which each node finds its place in the slabs of each axis from small per-CTA tables built once before
// the x march (rows y0-1 .. y0+TY-1 and columns z0-1 .. z0+31 of the tile, for E and for H) and, along x,
// from one lookup per plane that is uniform across the CTA. Along an axis d the slabs of the two components
// with a psi along d have the same extent, so one entry serves both. A CPML term then costs a predicate, an
// index, a coalesced psi load and store and two multiply-adds; its arithmetic and order are cpml_io's. A lean
// warp issues all psi loads of its own nodes at the top of each plane, ahead of its wait for the plane.
//
// The region tests are those of a grid without periodic axes (the fused pass serves no other): H_c is stepped
// where x_a <= n_a - 2 for every a != c, E_c where 1 <= x_a <= n_a - 2 for a != c and x_c <= n_c - 2; other
// nodes copy the component.
#pragma once

#include "fused_tma.cuh"

namespace lsfdtd {

// a coordinate's place in the CPML slab of one axis and field
template <typename R>
struct SlabInfo {
  int side;  // -1 none, 0 lo, 1 hi
  int st;    // first node of the slab along the axis
  int len;   // its length
  R b, c, k;  // profile values at the coordinate (k: 1/kappa - 1, zero where kappa is 1 everywhere)
};

template <int FLD, typename F>
__device__ __forceinline__ SlabInfo<typename real_of<F>::type> slab_info(const PmlAxis<F>& p, int d, int u) {
  using R = typename real_of<F>::type;
  SlabInfo<R> s;
  s.side = -1;
  s.st = 0;
  s.len = 1;
  s.b = s.c = s.k = R(0);
  if (!p.on) return s;
  const int cr = (d + 1) % 3;  // a component with a psi along d (both have the same slab extents)
#pragma unroll
  for (int sd = 0; sd < 2; ++sd) {
    const int st = p.start[FLD][cr][sd], ln = p.len[FLD][cr][sd];
    if (ln > 0 && u >= st && u < st + ln) {
      s.side = sd;
      s.st = st;
      s.len = ln;
    }
  }
  if (s.side >= 0) {
    s.b = p.b[FLD][u];
    s.c = p.c[FLD][u];
    s.k = p.k[FLD] ? p.k[FLD][u] : R(0);
  }
  return s;
}

template <typename F, int TY>
struct PmlTables {
  using R = typename real_of<F>::type;
  static constexpr int NY = TY + 1, NZ = 33;
  SlabInfo<R> y[2][NY];  // [E, H][row]: y = y0 - 1 + row
  SlabInfo<R> z[2][NZ];  // [E, H][col]: z = z0 - 1 + col
  // the psi of the halo nodes' H CPML terms, per axis, copied ahead of the plane's wait: [plane parity][H_x and
  // H_z of the halo row, H_x and H_y of the halo column][lane][axis]
  F hpsi[2][4][32][3];
};

template <typename F, int TY, int S>
constexpr size_t fused_pml_smem_bytes() {
  return fused_tma_smem_bytes<F, TY, S>() + (sizeof(PmlTables<F, TY>) + 15) / 16 * 16;  // tables after kUsed
}

// index of node x in the psi slab of axis d described by si, in 32-bit arithmetic: the engine takes the lean
// pass only where every slab has fewer than 2^31 nodes
template <typename F>
__device__ __forceinline__ int pml_index(const YeeArgs<F>& g, const SlabInfo<typename real_of<F>::type>& si, int d,
                                         const int* x) {
  if (d == 0) return ((x[0] - si.st) * g.n[1] + x[1]) * g.n[2] + x[2];
  if (d == 1) return (x[0] * si.len + (x[1] - si.st)) * g.n[2] + x[2];
  return (x[0] * g.n[1] + x[1]) * si.len + (x[2] - si.st);
}

// the CPML term along axis d of a value v of field FLD, component c, at psi index q, from psi_prev (the node's
// psi before this step); psi_out == nullptr: a halo node, computed but not stored. UNI: cubic cells (the
// grid's uniform flag, known when the kernel is compiled)
template <int FLD, bool UNI, typename F>
__device__ __forceinline__ void pml_term(F& v, const YeeArgs<F>& g, const SlabInfo<typename real_of<F>::type>& si,
                                         int d, int c, int q, F der, typename real_of<F>::type scale,
                                         F psi_prev, F* psi_out) {
  using R = typename real_of<F>::type;
  const int d1 = (c + 1) % 3;
  R sgn = (d == d1) ? R(1) : R(-1);
  if (FLD == 1) sgn = -sgn;
  R s = UNI ? scale : scale / g.pml[d].div;
  s = sgn * s;
  F psi = psi_prev * si.b;
  if (g.pml[d].k[FLD]) v += (s * si.k) * der;
  psi += der * (s * si.c);
  if (psi_out) st_global(psi_out + q, psi);
  v += psi;
}

// FP32: four CTAs of 8 rows (two of 16) per SM, at most 64 registers per thread, which their shared memory
// allows; FP64 tiles need twice the shared memory and are not constrained. UNI: cubic cells, so the curl
// differences and CPML coefficients carry no per-axis spacing (one instantiation each way).
// ASYNC: the ring is filled by every thread with cp.async copies of whole rows (zero-filled outside the
// grid), completing on the same mbarriers, for grids whose rows the tensor copies cannot stride (not a
// multiple of 16 bytes). A table-fed TF/SF source's corrections of H (FusedArgs::hc) are added to every H
// value the tile computes (its own nodes and its halo) before the E half uses them (HC: compiled in only for
// runs that have such corrections).
// AX: the axes (bit d for axis d) along which the launch's CTAs may meet CPML slabs or walls; a CTA of a
// launch without bit d has its nodes, halo nodes and planes inner along axis d, so that axis's slab lookups
// and terms are compiled out (7: any CTA).
// CLEAN: every CTA of the launch lies in the clean interior (each of its nodes, halo nodes and x planes,
// the plane before its segment included, inside [inner_lo, inner_hi) on every axis): the region tests and
// CPML terms are compiled out, and with them the registers they hold (the lean path's code, though never
// taken there, costs the interior warps a quarter of their speed)
template <typename F, int TY, int S, bool UNI, bool ASYNC = false, bool HC = false, bool CLEAN = false,
          int AX = 7>
__global__ void __launch_bounds__(32 * TY, sizeof(F) == 4 ? (TY == 8 ? 4 : 2) : 1)
    k_fused_pml(const __grid_constant__ TmaArgs<F> t) {
  static_assert(!CLEAN || (!ASYNC && !HC), "the clean interior pass copies by tensor maps and has no sources");
  using R = typename real_of<F>::type;
  using St = TmaStage<F, TY>;
  using Tab = PmlTables<F, TY>;
  constexpr int TZ = 32, BZ = St::BZ, NT = 32 * TY;
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);
  using L = TmaLayout<F, TY, S>;
  F(*sH)[2][TY + 1][TZ] = reinterpret_cast<F(*)[2][TY + 1][TZ]>(smem + L::kRing);
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem + L::kRing + L::kRows);
  F(*zc)[2][TY] = reinterpret_cast<F(*)[2][TY]>(smem + L::kRing + L::kRows + L::kBars);  // [plane][H_x, H_y][row]
  Tab& tab = *reinterpret_cast<Tab*>(smem + L::kUsed);

  const FusedArgs<F>& a = t.f;
  const YeeArgs<F>& g = a.y;
  const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TZ + tx;
  int z0, y0, xs, xe;  // the CTA's tile and x segment, from the launch's box list
  {
    int b = 0;
    while (b + 1 < t.map.n && (int)blockIdx.x >= t.map.box[b + 1].first) ++b;
    const CtaBox& q = t.map.box[b];
    const int l = (int)blockIdx.x - q.first, nz = q.t1[0] - q.t0[0], ny = q.t1[1] - q.t0[1];
    z0 = (q.t0[0] + l % nz) * TZ;
    y0 = (q.t0[1] + (l / nz) % ny) * TY;
    xs = q.x0 + (l / nz / ny) * q.seg;
    xe = min(min(q.x1, n0), xs + q.seg);
  }
  if (xs >= xe) return;
  const int k = z0 + tx, j = y0 + ty;
  const int xb = xs > 0 ? xs - 1 : 0;
  const bool own = k < n2 && j < n1;
  const long long s1 = n2, s0 = (long long)n1 * n2;

  auto stE = [&](int s, int c) { return reinterpret_cast<F(*)[BZ]>(smem + s * St::kBytes + c * St::kE); };
  auto stH = [&](int s, int c) {
    return reinterpret_cast<F(*)[BZ]>(smem + s * St::kBytes + 3 * St::kE + c * St::kH);
  };
  auto stC = [&](int s) { return reinterpret_cast<R(*)[TZ]>(smem + s * St::kBytes + 3 * St::kE + 3 * St::kH); };

  // the slab tables of the tile's rows and columns (halo included)
  for (int e = tid; !CLEAN && e < 2 * (Tab::NY + Tab::NZ); e += NT) {
    const int f = e / (Tab::NY + Tab::NZ), r = e % (Tab::NY + Tab::NZ);
    if (r < Tab::NY ? !(AX & 2) : !(AX & 4)) continue;  // an axis this launch's CTAs are inner along
    if (r < Tab::NY)
      tab.y[f][r] = f ? slab_info<1>(g.pml[1], 1, y0 - 1 + r) : slab_info<0>(g.pml[1], 1, y0 - 1 + r);
    else
      tab.z[f][r - Tab::NY] = f ? slab_info<1>(g.pml[2], 2, z0 - 1 + r - Tab::NY)
                                : slab_info<0>(g.pml[2], 2, z0 - 1 + r - Tab::NY);
  }
  __shared__ unsigned long long never;  // a barrier nothing completes: the wait of a timeout test
  if (tid == 0) {
    mbar_init(&never, 1);
    for (int s = 0; s < S; ++s) mbar_init(&bar[s], ASYNC ? NT : 1);  // cp.async: every thread arrives
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  auto produce = [&](int p) {
    const int s = (int)((unsigned)(p - xb) % S);  // p >= xb: unsigned, so the ring slot is a mask or a multiply
    if constexpr (ASYNC) {
      static_assert(sizeof(F) == sizeof(R), "the fused pass steps real fields");
      // warp ty copies rows ty, ty + TY, ...: E (3 x (TY + 2) rows) and H (3 x (TY + 1) rows) of BZ values
      // from z0 - 4, then the coefficient's TY rows of TZ values from z0; the tensor copies' layout
      constexpr int kRE = TY + 2, kRH = TY + 1, kRows = 3 * kRE + 3 * kRH + TY;
      const bool px = p < n0;
#pragma unroll 1
      for (int rr = ty; rr < kRows; rr += TY) {
        const F* src;
        F* dst;
        int y, z, w;
        if (rr < 3 * kRE) {
          src = g.E[rr / kRE];
          dst = stE(s, rr / kRE)[rr % kRE];
          y = y0 - 1 + rr % kRE;
          z = z0 - 4;
          w = BZ;
        } else if (rr < 3 * kRE + 3 * kRH) {
          const int q = rr - 3 * kRE;
          src = g.H[q / kRH];
          dst = stH(s, q / kRH)[q % kRH];
          y = y0 - 1 + q % kRH;
          z = z0 - 4;
          w = BZ;
        } else {
          const int row = rr - 3 * kRE - 3 * kRH;
          src = reinterpret_cast<const F*>(g.cbE[0]);
          dst = reinterpret_cast<F*>(stC(s)[row]);
          y = y0 + row;
          z = z0;
          w = TZ;
        }
        const bool yin = px && y >= 0 && y < n1;
        const long long base = ((long long)p * n1 + y) * n2;
        for (int col = tx; col < w; col += 32) {
          const int zz = z + col;
          const bool v = yin && zz >= 0 && zz < n2;
          cp_async(dst + col, v ? src + base + zz : src, v);
        }
      }
      asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(smem_u32(&bar[s])) : "memory");
    } else {
      mbar_expect_tx(&bar[s], St::kTx);
      for (int c = 0; c < 3; ++c) tma_load_3d(stE(s, c), &t.mE[c], z0 - 4, y0 - 1, p, &bar[s]);
      for (int c = 0; c < 3; ++c) tma_load_3d(stH(s, c), &t.mH[c], z0 - 4, y0 - 1, p, &bar[s]);
      tma_load_3d(stC(s), &t.mC, z0, y0, p, &bar[s]);
    }
  };
  auto ready = [&](int p) -> bool {
    const unsigned r = (unsigned)(p - xb);
    if (t.wait_budget < 0) return mbar_wait_bounded(&never, 0, -t.wait_budget);  // a timeout test: see TmaArgs
    return mbar_wait_bounded(&bar[r % S], (r / S) & 1, t.wait_budget);
  };
  // the planes a segment reads are xb .. xe (plane xe as the next plane of the last one), and no others are
  // copied
  const int first_fill = min(xb + S - 2, xe);
  if (ASYNC || tid == 0) {
    for (int p = xb; p <= first_fill; ++p) produce(p);
  }
  int issued = first_fill;

  auto curl = [&](F av, F bv, int d1, int d2) -> F {
    if constexpr (UNI) return av - bv;
    else return av * g.inv_d[d1] - bv * g.inv_d[d2];
  };
  // region- and CPML-free H at stage offset o (row-major in the 40-wide boxes)
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

  // H^{n+1/2}_c of the tile node at table row yy (y = y0 - 1 + yy) and column zz (z = z0 - 1 + zz) of plane i,
  // with region test and CPML terms; xs_h: the plane's x slab info (H); store: an own node (H and psi out)
  // pre: the node's psi per axis, loaded ahead (own nodes), or nullptr to load it here (halo nodes)
  auto h_lean = [&](int c, int si, int sn, int i, int yy, int zz, const SlabInfo<R>& xs_h, bool store,
                    const F* pre) -> F {
    const int row = yy, col = zz + 3;
    const int x[3] = {i, y0 - 1 + yy, z0 - 1 + zz};
    const F h0 = stH(si, c)[row][col];
    const long long p = i * s0 + (long long)x[1] * s1 + x[2];
    bool in = true;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax)
      if (ax != c && x[ax] > g.n[ax] - 2) in = false;
    if (!in) {
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
    F h = h0 - curl(av, bv, d1, d2) * g.cH;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (d == c) continue;
      if (!(AX >> d & 1)) continue;
      const SlabInfo<R>& sl = d == 0 ? xs_h : (d == 1 ? tab.y[1][yy] : tab.z[1][zz]);
      if (sl.side < 0) continue;
      const int q = pml_index(g, sl, d, x);
      const F prev = pre ? pre[d] : ro(g.pml[d].psi[1][c][sl.side] + q);
      F* pout = store ? a.psiHo[d][c][sl.side] : nullptr;
      pml_term<1, UNI>(h, g, sl, d, c, q, d == d1 ? av : bv, g.cH, prev, pout);
    }
    if (store) st_global(a.Ho[c] + p, h);
    return h;
  };

  const unsigned full = 0xffffffffu;
  const int oo = (ty + 1) * BZ + tx + 4;
  const long long off_jk = (long long)j * s1 + k;
  auto y_in = [&](int y) { return y >= a.inner_lo[1] && y < a.inner_hi[1]; };
  // the warp's nodes, its halo column (lane 0: z0 - 1) and, for warp 0, the halo row y0 - 1 are all inner
  // along y and z (warp-uniform: every lane of a warp shares its row)
  const bool warp_clean = y_in(j) && (ty != 0 || y_in(y0 - 1)) && z0 - 1 >= a.inner_lo[2] &&
                          z0 + TZ <= a.inner_hi[2];
  const bool multi_cb = g.cbE[1] != g.cbE[0] || g.cbE[2] != g.cbE[0];
  // the halo column z0 - 1 and all the tile's rows are inner along y and z
  const bool col_clean = z0 - 1 >= a.inner_lo[2] && z0 - 1 < a.inner_hi[2] && y_in(y0) && y0 + TY <= a.inner_hi[1];
  constexpr int kColWarp = TY > 1 ? 1 : 0;  // warp 0 computes the halo row, this warp the halo column
  // own node: components stepped as far as y and z decide (bit c), for H and for E; the x part per plane
  unsigned yz_hm = 0, yz_em = 0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const bool hy_ok = c == 1 || j <= n1 - 2, hz_ok = c == 2 || k <= n2 - 2;
    const bool ey_ok = j <= n1 - 2 && (c == 1 || j >= 1), ez_ok = k <= n2 - 2 && (c == 2 || k >= 1);
    yz_hm |= (hy_ok && hz_ok ? 1u : 0u) << c;
    yz_em |= (ey_ok && ez_ok ? 1u : 0u) << c;
  }

  // the TF/SF correction boxes of H that meet the tile (rows y0 - 1 .. y0 + TY - 1, columns z0 - 1 .. z0 + 31)
  unsigned tile_hc = 0;
  for (int b = 0; HC && b < a.hc.n; ++b) {
    const HCorrBox& q = a.hc.box[b];
    if (q.lo[1] < y0 + TY && q.hi[1] > y0 - 1 && q.lo[2] < z0 + TZ && q.hi[2] > z0 - 1) tile_hc |= 1u << b;
  }
  // H_c at (x, y, z) plus the corrections of the boxes in pm that hold it, in box order
  auto hcorr = [&](F h, int c, int x, int y, int z, unsigned pm) -> F {
    for (; pm; pm &= pm - 1) {
      const HCorrBox& q = a.hc.box[__ffs(pm) - 1];
      if (q.c == c && y >= q.lo[1] && y < q.hi[1] && z >= q.lo[2] && z < q.hi[2])
        h = h + static_cast<const F*>(a.hc.vals)[q.off + ((long long)(x - q.lo[0]) * (q.hi[1] - q.lo[1]) +
                                                          (y - q.lo[1])) * (q.hi[2] - q.lo[2]) + (z - q.lo[2])];
    }
    return h;
  };

  F prev_hy = zero<F>(), prev_hz = zero<F>();
  bool failed = false;
  int cons = xb - 1;
#pragma unroll 1
  for (int i = xb; i < xe; ++i) {
    const bool fast = CLEAN || (warp_clean && i >= a.inner_lo[0] && i < a.inner_hi[0]);
    SlabInfo<R> xs_h, xs_e;
    // a lean warp issues the psi loads of its own nodes for this plane before it waits for the plane's
    // copies, so that their latency overlaps the wait and each other: [component][axis], with the psi index
    // per axis (H, E)
    F pre_h[3][3], pre_e[3][3];
    int qh[3] = {0, 0, 0}, qe[3] = {0, 0, 0};
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int d = 0; d < 3; ++d) pre_h[c][d] = pre_e[c][d] = zero<F>();
    if (!fast) {
      if (!(AX & 1) || (i >= a.inner_lo[0] && i < a.inner_hi[0])) {  // a plane outside the x slabs
        xs_h.side = xs_e.side = -1;
        xs_h.st = xs_e.st = 0;
        xs_h.len = xs_e.len = 1;
        xs_h.b = xs_h.c = xs_h.k = xs_e.b = xs_e.c = xs_e.k = R(0);
      } else {
        xs_h = slab_info<1>(g.pml[0], 0, i);
        xs_e = slab_info<0>(g.pml[0], 0, i);
      }
      if (own) {
        const int x[3] = {i, j, k};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          if (!(AX >> d & 1)) continue;
          const SlabInfo<R>& sh = d == 0 ? xs_h : (d == 1 ? tab.y[1][ty + 1] : tab.z[1][tx + 1]);
          const SlabInfo<R>& se = d == 0 ? xs_e : (d == 1 ? tab.y[0][ty + 1] : tab.z[0][tx + 1]);
          const int c1 = (d + 1) % 3, c2 = (d + 2) % 3;  // the components with a psi along d
          if (sh.side >= 0) {
            qh[d] = pml_index(g, sh, d, x);
            pre_h[c1][d] = ro(g.pml[d].psi[1][c1][sh.side] + qh[d]);
            pre_h[c2][d] = ro(g.pml[d].psi[1][c2][sh.side] + qh[d]);
          }
          if (se.side >= 0 && i >= xs) {
            qe[d] = pml_index(g, se, d, x);
            pre_e[c1][d] = g.pml[d].psi[0][c1][se.side][qe[d]];
            pre_e[c2][d] = g.pml[d].psi[0][c2][se.side][qe[d]];
          }
        }
      }
    }
    // the psi of the halo nodes that take the lean path (warp 0: the halo row, warp kColWarp: the halo column),
    // copied into shared memory ahead of the plane's wait like the own nodes' loads above (tensor-copy ring
    // only: the cp.async ring's copies share the wait that these need)
    const bool x_in = i >= a.inner_lo[0] && i < a.inner_hi[0];
    const bool row_lean = !CLEAN && ty == 0 && !fast && y0 > 0 && k < n2 && i >= xs;
    const bool col_lean = !CLEAN && ty == kColWarp && tx < TY && z0 > 0 && y0 + tx < n1 && i >= xs &&
                          !(col_clean && x_in);
    if constexpr (!ASYNC && !CLEAN) {
      if (row_lean || col_lean) {
        const SlabInfo<R> xh = fast && (AX & 1) ? slab_info<1>(g.pml[0], 0, i) : xs_h;
        const int yy = row_lean ? 0 : tx + 1, zz = row_lean ? tx + 1 : 0;
        const int x[3] = {i, y0 - 1 + yy, z0 - 1 + zz};
#pragma unroll
        for (int w = 0; w < 2; ++w) {
          const int c = row_lean ? 2 * w : w;  // the row's H_x and H_z, the column's H_x and H_y
          F* dst = tab.hpsi[i & 1][row_lean ? w : 2 + w][tx];
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            if (d == c || !(AX >> d & 1)) continue;
            const SlabInfo<R>& sl = d == 0 ? xh : (d == 1 ? tab.y[1][yy] : tab.z[1][zz]);
            if (sl.side >= 0) cp_async(dst + d, g.pml[d].psi[1][c][sl.side] + pml_index(g, sl, d, x), true);
          }
        }
      }
    }
    const bool ok = (i > xb || ready(i)) && ready(i + 1);  // plane i was waited for as plane i + 1 before
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    cons = i + 1;
    if (i + S - 1 <= xe) {
      if (ASYNC || tid == 0) produce(i + S - 1);
      issued = i + S - 1;
    }
    const int si = (int)((unsigned)(i - xb) % S), sn = (int)((unsigned)(i + 1 - xb) % S);
    const long long p = i * s0 + off_jk;
    unsigned pm = 0;  // the correction boxes of H that hold nodes of this plane and tile
    for (unsigned m = tile_hc; HC && m; m &= m - 1) {
      const HCorrBox& q = a.hc.box[__ffs(m) - 1];
      if (i >= q.lo[0] && i < q.hi[0]) pm |= m & (0u - m);
    }
    F hx = zero<F>(), hy = zero<F>(), hz = zero<F>();
    if (fast) {
      hx = hx_fast(si, oo);
      hy = hy_fast(si, sn, oo);
      hz = hz_fast(si, sn, oo);
      if (HC && pm) {
        hx = hcorr(hx, 0, i, j, k, pm);
        hy = hcorr(hy, 1, i, j, k, pm);
        hz = hcorr(hz, 2, i, j, k, pm);
      }
      if (i >= xs) {
        st_global(a.Ho[0] + p, hx);
        st_global(a.Ho[1] + p, hy);
        st_global(a.Ho[2] + p, hz);
      }
    } else if (own) {
      // the fast formulas, then the region mask and the CPML terms of the axes whose slab holds the node
      // (x: uniform per plane, y: per warp, z: per lane), in cpml_io's order; nothing stored before xs
      const bool st = i >= xs;
      const F* ex = &stE(si, 0)[0][0];
      const F* ey = &stE(si, 1)[0][0];
      const F* ez = &stE(si, 2)[0][0];
      const F av[3] = {ez[oo + BZ] - ez[oo], ex[oo + 1] - ex[oo], (&stE(sn, 1)[0][0])[oo] - ey[oo]};
      const F bv[3] = {ey[oo + 1] - ey[oo], (&stE(sn, 2)[0][0])[oo] - ez[oo], ex[oo + BZ] - ex[oo]};
      const unsigned hm = yz_hm & (i <= n0 - 2 ? 7u : 1u);
      const SlabInfo<R>& yh = tab.y[1][ty + 1];
      const SlabInfo<R>& zh = tab.z[1][tx + 1];
      F hv[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
        const F h0 = stH(si, c)[0][oo];
        F h = h0;
        if (hm >> c & 1u) {
          h = h0 - curl(av[c], bv[c], d1, d2) * g.cH;
          if ((AX & 1) && c != 0 && xs_h.side >= 0)
            pml_term<1, UNI>(h, g, xs_h, 0, c, qh[0], d1 == 0 ? av[c] : bv[c], g.cH, pre_h[c][0],
                        st ? a.psiHo[0][c][xs_h.side] : nullptr);
          if ((AX & 2) && c != 1 && yh.side >= 0)
            pml_term<1, UNI>(h, g, yh, 1, c, qh[1], d1 == 1 ? av[c] : bv[c], g.cH, pre_h[c][1],
                        st ? a.psiHo[1][c][yh.side] : nullptr);
          if ((AX & 4) && c != 2 && zh.side >= 0)
            pml_term<1, UNI>(h, g, zh, 2, c, qh[2], d1 == 2 ? av[c] : bv[c], g.cH, pre_h[c][2],
                        st ? a.psiHo[2][c][zh.side] : nullptr);
        }
        if (HC && pm) h = hcorr(h, c, i, j, k, pm);
        if (st) st_global(a.Ho[c] + p, h);
        hv[c] = h;
      }
      hx = hv[0];
      hy = hv[1];
      hz = hv[2];
    }
    if (i < xs) {  // the plane before the segment: H_y, H_z of the own node only
      prev_hy = hy;
      prev_hz = hz;
      continue;
    }
    F(&hs)[2][TY + 1][TZ] = sH[i & 1];
    hs[0][ty + 1][tx] = hx;
    hs[1][ty + 1][tx] = hz;
    if (ty == 0 && y0 > 0 && k < n2) {  // the halo row y0 - 1
      F hxr, hzr;
      if (fast) {
        hxr = hx_fast(si, tx + 4);
        hzr = hz_fast(si, sn, tx + 4);
      } else {
        if constexpr (!ASYNC) asm volatile("cp.async.wait_all;\n" ::: "memory");  // this lane's halo psi
        hxr = h_lean(0, si, sn, i, 0, tx + 1, xs_h, false, ASYNC ? nullptr : tab.hpsi[i & 1][0][tx]);
        hzr = h_lean(2, si, sn, i, 0, tx + 1, xs_h, false, ASYNC ? nullptr : tab.hpsi[i & 1][1][tx]);
      }
      if (HC && pm) {
        hxr = hcorr(hxr, 0, i, y0 - 1, k, pm);
        hzr = hcorr(hzr, 2, i, y0 - 1, k, pm);
      }
      hs[0][0][tx] = hxr;
      hs[1][0][tx] = hzr;
    }
    // the halo column z0 - 1 (H_x, H_y of every row, for lane 0 of each warp): one warp, lane r for row r
    if (ty == kColWarp && tx < TY && z0 > 0 && y0 + tx < n1) {
      F hxc, hyc;
      if (CLEAN || (col_clean && i >= a.inner_lo[0] && i < a.inner_hi[0])) {
        const int o = (tx + 1) * BZ + 3;
        hxc = hx_fast(si, o);
        hyc = hy_fast(si, sn, o);
      } else {
        SlabInfo<R> xc_h = fast && (AX & 1) ? slab_info<1>(g.pml[0], 0, i) : xs_h;  // this warp may be fast itself
        if constexpr (!ASYNC) asm volatile("cp.async.wait_all;\n" ::: "memory");
        hxc = h_lean(0, si, sn, i, tx + 1, 0, xc_h, false, ASYNC ? nullptr : tab.hpsi[i & 1][2][tx]);
        hyc = h_lean(1, si, sn, i, tx + 1, 0, xc_h, false, ASYNC ? nullptr : tab.hpsi[i & 1][3][tx]);
      }
      if (HC && pm) {
        hxc = hcorr(hxc, 0, i, y0 + tx, z0 - 1, pm);
        hyc = hcorr(hyc, 1, i, y0 + tx, z0 - 1, pm);
      }
      zc[i & 1][0][tx] = hxc;
      zc[i & 1][1][tx] = hyc;
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
      const F a0 = hz - hz_ym, b0 = hy - hy_zm;
      const F a1 = hx - hx_zm, b1 = hz - prev_hz;
      const F a2 = hy - prev_hy, b2 = hx - hx_ym;
      if (fast && !multi_cb) {
        st_global(a.Eo[0] + p, ex[oo] + curl(a0, b0, 1, 2) * cb);
        st_global(a.Eo[1] + p, ey[oo] + curl(a1, b1, 2, 0) * cb);
        st_global(a.Eo[2] + p, ez[oo] + curl(a2, b2, 0, 1) * cb);
      } else {
        const F av[3] = {a0, a1, a2}, bv[3] = {b0, b1, b2};
        const F* e[3] = {ex, ey, ez};
        const unsigned em = fast ? 7u : yz_em & ((i <= n0 - 2 ? 1u : 0u) | (i >= 1 && i <= n0 - 2 ? 6u : 0u));
        const SlabInfo<R>& ye = tab.y[0][ty + 1];
        const SlabInfo<R>& ze = tab.z[0][tx + 1];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const F e0 = e[c][oo];
          if (!(em >> c & 1u)) {
            st_global(a.Eo[c] + p, e0);
            continue;
          }
          const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
          const R cbc = (c == 0 || !multi_cb) ? cb : ro(g.cbE[c] + p);
          F ev = e0 + curl(av[c], bv[c], d1, d2) * cbc;
          if (!fast) {
            if ((AX & 1) && c != 0 && xs_e.side >= 0)
              pml_term<0, UNI>(ev, g, xs_e, 0, c, qe[0], d1 == 0 ? av[c] : bv[c], cbc, pre_e[c][0],
                          g.pml[0].psi[0][c][xs_e.side]);
            if ((AX & 2) && c != 1 && ye.side >= 0)
              pml_term<0, UNI>(ev, g, ye, 1, c, qe[1], d1 == 1 ? av[c] : bv[c], cbc, pre_e[c][1],
                          g.pml[1].psi[0][c][ye.side]);
            if ((AX & 4) && c != 2 && ze.side >= 0)
              pml_term<0, UNI>(ev, g, ze, 2, c, qe[2], d1 == 2 ? av[c] : bv[c], cbc, pre_e[c][2],
                          g.pml[2].psi[0][c][ze.side]);
          }
          st_global(a.Eo[c] + p, ev);
        }
      }
    }
    prev_hy = hy;
    prev_hz = hz;
  }
  if (tid == 0) {
    for (int p = cons + 1; p <= issued; ++p)
      mbar_wait_bounded(&bar[(unsigned)(p - xb) % S], ((unsigned)(p - xb) / S) & 1, kDrainBudget);
    if (failed && t.status) atomicExch(t.status, 1);
  }
  // every thread's own copies landed (the ring's with cp.async, or the halo psi)
  if constexpr (!CLEAN) asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
}

}  // namespace lsfdtd
