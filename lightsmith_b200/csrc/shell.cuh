// The shell of the split fused step: one FDTD step of every node outside the interior box.
//
// The split step runs the fused pass (k_fused_tma with BOX) over an interior box whose nodes need neither
// region nor CPML tests, and these kernels over the rest: the CPML slabs, the PEC walls and the few nodes
// between them and the box. All read the "in" buffers (E^n, H^n, H-side psi) and write the "out" buffers,
// each its own nodes.
//
// The shell takes two launches, one thread per shell node in each: k_shell_h computes H^{n+1/2} (with its
// psi, in to out), then k_shell_e computes E^{n+1} from the new H of the node and of its neighbours below,
// which the fused pass has written where they lie in the box (so k_shell_e follows both). E-side psi is
// updated in place: only the node's own E update touches it. Nodes outside a component's stepped region copy
// that component. The arithmetic per value is that of update_h_node / update_e_node (yee.cuh).
//
// The shell is at most six boxes (the two x slabs over the whole y-z plane, the two y slabs over the box's x
// range, the two z slabs over the box's x and y ranges), enumerated with z fastest so that consecutive
// threads read consecutive nodes.
#pragma once

#include "common.cuh"
#include "fused.cuh"
#include "yee.cuh"

namespace lsfdtd {

struct ShellBoxes {
  int nbox;
  int lo[6][3];
  int ext[6][3];
  unsigned first[7];         // nodes in the boxes before box b; first[nbox] = all shell nodes
  unsigned long long total;  // all shell nodes (the kernel needs fewer than 2^32)
};

// Where a node lies in the CPML slabs of one field (E or H), per axis. Along an axis d, the slab of every
// component c != d has the same extent (the components' stepped regions along d agree), so one lookup per
// axis serves both components with a psi along d.
template <typename F>
struct SlabPoint {
  using R = typename real_of<F>::type;
  int side[3];   // 0 lo, 1 hi, -1 none
  long long q[3];  // psi index within the slab
  R b[3], c[3], k[3];
};

template <int FLD, typename F>
__device__ __forceinline__ void slab_point(const YeeArgs<F>& g, const int* x, SlabPoint<F>& sp) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    sp.side[d] = -1;
    const PmlAxis<F>& p = g.pml[d];
    if (!p.on) continue;
    const int cr = (d + 1) % 3;  // a component with a psi along d
    const int u = x[d];
    int side = -1;
#pragma unroll
    for (int s = 0; s < 2; ++s)
      if (u >= p.start[FLD][cr][s] && u < p.start[FLD][cr][s] + p.len[FLD][cr][s]) side = s;
    if (side < 0) continue;
    sp.side[d] = side;
    sp.q[d] = psi_index(x, g.n, d, u - p.start[FLD][cr][side], p.len[FLD][cr][side]);
    sp.b[d] = p.b[FLD][u];
    sp.c[d] = p.c[FLD][u];
    sp.k[d] = p.k[FLD] ? p.k[FLD][u] : typename real_of<F>::type(0);
  }
}

// psi of component c before its update, per axis d != c with a slab at this node (zero elsewhere)
template <int FLD, typename F>
__device__ __forceinline__ void slab_psi(const YeeArgs<F>& g, const SlabPoint<F>& sp, int c, F* psi_in) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    psi_in[d] = zero<F>();
    if (d == c || sp.side[d] < 0) continue;
    const F* src = g.pml[d].psi[FLD][c][sp.side[d]] + sp.q[d];
    psi_in[d] = FLD == 1 ? ro(src) : *src;  // E-side psi is updated in place
  }
}

// the CPML terms of component c at a node whose slab lookup is sp: cpml_io's arithmetic, in its order
template <int FLD, typename F>
__device__ __forceinline__ void slab_terms(F& v, const FusedArgs<F>& a, const SlabPoint<F>& sp, int c, F der1,
                                           F der2, typename real_of<F>::type scale, const F* psi_in) {
  using R = typename real_of<F>::type;
  const YeeArgs<F>& g = a.y;
  const int d1 = (c + 1) % 3;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d == c || sp.side[d] < 0) continue;
    const PmlAxis<F>& p = g.pml[d];
    const F der = d == d1 ? der1 : der2;
    R sgn = (d == d1) ? R(1) : R(-1);
    if (FLD == 1) sgn = -sgn;
    R s = g.uniform ? scale : scale / p.div;
    s = sgn * s;
    const int side = sp.side[d];
    F psi = psi_in[d] * sp.b[d];
    if (p.k[FLD]) v += (s * sp.k[d]) * der;
    psi += der * (s * sp.c[d]);
    F* dst = FLD == 1 ? a.psiHo[d][c][side] : p.psi[FLD][c][side];
    st_global(dst + sp.q[d], psi);
    v += psi;
  }
}

// node of shell thread q (z fastest within each box); false past the last shell node
__device__ __forceinline__ bool shell_node(const ShellBoxes& sb, int* x) {
  const unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= sb.first[sb.nbox]) return false;
  int b = 0;
#pragma unroll 1
  while (b + 1 < sb.nbox && q >= sb.first[b + 1]) ++b;
  const unsigned r = q - sb.first[b];
  const unsigned ez = (unsigned)sb.ext[b][2], ey = (unsigned)sb.ext[b][1];
  const unsigned t = r / ez;
  x[0] = sb.lo[b][0] + (int)(t / ey);
  x[1] = sb.lo[b][1] + (int)(t % ey);
  x[2] = sb.lo[b][2] + (int)(r % ez);
  return true;
}

// H^{n+1/2} of the shell nodes: in buffers to out buffers, H psi in to out (update_h_node's arithmetic).
// Every load is issued before the first store.
template <typename F>
__global__ void __launch_bounds__(256) k_shell_h(const __grid_constant__ FusedArgs<F> a,
                                                 const __grid_constant__ ShellBoxes sb) {
  int x[3];
  if (!shell_node(sb, x)) return;
  const YeeArgs<F>& g = a.y;
  const long long s1 = g.n[2], s0 = (long long)g.n[1] * g.n[2];
  const long long p = x[0] * s0 + x[1] * s1 + x[2];
  const long long step[3] = {s0, s1, 1};
  SlabPoint<F> sp;
  slab_point<1>(g, x, sp);
  bool in[3];
  F h0[3], av[3], bv[3], psi[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    in[c] = in_h_region(c, x, g.n, g.periodic);
    h0[c] = ro(g.H[c] + p);
    av[c] = bv[c] = zero<F>();
    if (in[c]) {
      const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
      av[c] = ro(g.E[d2] + p + step[d1]) - ro(g.E[d2] + p);
      bv[c] = ro(g.E[d1] + p + step[d2]) - ro(g.E[d1] + p);
    }
    slab_psi<1>(g, sp, c, psi[c]);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    F h = h0[c];
    if (in[c]) {
      const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
      const F curl = g.uniform ? (av[c] - bv[c]) : (av[c] * g.inv_d[d1] - bv[c] * g.inv_d[d2]);
      h = h0[c] - curl * g.cH;
      slab_terms<1>(h, a, sp, c, av[c], bv[c], g.cH, psi[c]);
    }
    st_global(a.Ho[c] + p, h);
  }
}

// E^{n+1} of the shell nodes from E^n and the new H (out buffers: the interior box's nodes written by the
// fused pass, the shell's by k_shell_h); E psi in place (update_e_node's arithmetic). Every load is issued
// before the first store.
template <typename F>
__global__ void __launch_bounds__(256) k_shell_e(const __grid_constant__ FusedArgs<F> a,
                                                 const __grid_constant__ ShellBoxes sb) {
  using R = typename real_of<F>::type;
  int x[3];
  if (!shell_node(sb, x)) return;
  const YeeArgs<F>& g = a.y;
  const long long s1 = g.n[2], s0 = (long long)g.n[1] * g.n[2];
  const long long p = x[0] * s0 + x[1] * s1 + x[2];
  const long long step[3] = {s0, s1, 1};
  SlabPoint<F> sp;
  slab_point<0>(g, x, sp);
  bool in[3];
  F e0[3], av[3], bv[3], psi[3][3];
  R cb[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    in[c] = in_e_region(c, x, g.n, g.periodic);
    e0[c] = ro(g.E[c] + p);
    av[c] = bv[c] = zero<F>();
    cb[c] = R(0);
    if (in[c]) {
      const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
      av[c] = ro(a.Ho[d2] + p) - ro(a.Ho[d2] + p - step[d1]);
      bv[c] = ro(a.Ho[d1] + p) - ro(a.Ho[d1] + p - step[d2]);
      cb[c] = ro(g.cbE[c] + p);
    }
    slab_psi<0>(g, sp, c, psi[c]);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    F ev = e0[c];
    if (in[c]) {
      const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
      const F curl = g.uniform ? (av[c] - bv[c]) : (av[c] * g.inv_d[d1] - bv[c] * g.inv_d[d2]);
      ev = e0[c] + curl * cb[c];
      slab_terms<0>(ev, a, sp, c, av[c], bv[c], cb[c], psi[c]);
    }
    st_global(a.Eo[c] + p, ev);
  }
}

// The shell of the box [lo, hi) in a grid of n nodes per axis (empty boxes dropped)
inline ShellBoxes shell_boxes(const int* n, const int* lo, const int* hi) {
  ShellBoxes s{};
  auto add = [&](int x0, int x1, int y0, int y1, int z0, int z1) {
    if (x1 <= x0 || y1 <= y0 || z1 <= z0) return;
    const int b = s.nbox++;
    s.lo[b][0] = x0;
    s.lo[b][1] = y0;
    s.lo[b][2] = z0;
    s.ext[b][0] = x1 - x0;
    s.ext[b][1] = y1 - y0;
    s.ext[b][2] = z1 - z0;
  };
  add(0, lo[0], 0, n[1], 0, n[2]);
  add(hi[0], n[0], 0, n[1], 0, n[2]);
  add(lo[0], hi[0], 0, lo[1], 0, n[2]);
  add(lo[0], hi[0], hi[1], n[1], 0, n[2]);
  add(lo[0], hi[0], lo[1], hi[1], 0, lo[2]);
  add(lo[0], hi[0], lo[1], hi[1], hi[2], n[2]);
  unsigned long long acc = 0;
  for (int b = 0; b < s.nbox; ++b) {
    s.first[b] = (unsigned)acc;
    acc += (unsigned long long)s.ext[b][0] * s.ext[b][1] * s.ext[b][2];
  }
  s.first[s.nbox] = (unsigned)acc;
  s.total = acc;
  return s;
}

}  // namespace lsfdtd
