// Vectorised in-place Yee updates (FP32): each thread updates four consecutive z nodes with 16-byte loads and
// stores. y and x neighbours are read from global memory (the neighbouring rows and planes are read by other
// threads at about the same time, so they come from L1/L2); z neighbours come from the adjacent lane by
// shuffle, and from one scalar load at the ends of a warp. A thread whose four nodes are all interior (stepped
// for every component, outside every CPML slab) runs the straight-line update; any other thread updates its
// nodes one at a time with update_h_node / update_e_node (region tests and CPML terms). The arithmetic per
// value is the same in both paths. Rows must be a multiple of four nodes (16-byte aligned float4 access).
#pragma once

#include "yee.cuh"

namespace lsfdtd {

struct VecBounds {
  int lo[3], hi[3];          // interior nodes [lo, hi) per axis: stepped for every component, outside CPML slabs
  int pml_lo[3], pml_hi[3];  // CPML cells per axis and side (0: none)
};

// nodes 1 <= u < n - 1 along every axis are stepped for every component
__device__ __forceinline__ bool in_all_regions(const YeeArgs<float>& g, int i, int j, int k0, int k1) {
  return i >= 1 && i < g.n[0] - 1 && j >= 1 && j < g.n[1] - 1 && k0 >= 1 && k1 < g.n[2] - 1;
}

// CPML terms of node (i, j, k) inside every stepped region for component c (FLD 0 E, 1 H, in place): the
// node's slab positions along each axis are derived from the CPML cell counts
__device__ __forceinline__ void cpml_node(float& v, const YeeArgs<float>& g, const VecBounds& b, int fld, int c,
                                          int i, int j, int k, float der1, float der2, float scale) {
  const int x[3] = {i, j, k};
  const int d1 = (c + 1) % 3;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d == c) continue;
    const PmlAxis<float>& p = g.pml[d];
    if (!p.on) continue;
    const int u = x[d];
    const int lo = b.pml_lo[d], hi = b.pml_hi[d];
    const bool in_lo = lo && u <= lo, in_hi = hi && u >= g.n[d] - 2 - hi;
    if (!in_lo && !in_hi) continue;
    const float der = d == d1 ? der1 : der2;
    float sgn = (d == d1) ? 1.f : -1.f;
    if (fld == 1) sgn = -sgn;
    float sc = g.uniform ? scale : scale / p.div;
    sc = sgn * sc;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      if (side == 0 ? !in_lo : !in_hi) continue;
      const int off = side ? u - (g.n[d] - 2 - hi) : (fld ? u : u - 1);
      const int ln = p.len[fld][c][side];
      const long long q = d == 0 ? ((long long)off * g.n[1] + j) * g.n[2] + k
                                 : (d == 1 ? ((long long)i * ln + off) * g.n[2] + k
                                           : ((long long)i * g.n[1] + j) * ln + off);
      float* ps = p.psi[fld][c][side] + q;
      float psi = *ps * p.b[fld][u];
      if (p.k[fld]) v += (sc * p.k[fld][u]) * der;
      psi += der * (sc * p.c[fld][u]);
      *ps = psi;
      v += psi;
    }
  }
}

// the per-node paths, kept out of line so that the vector path's registers stay few
__device__ __noinline__ void h_nodes4(const YeeArgs<float>& g, int i, int j, int k4) {
  for (int q = 0; q < 4; ++q) update_h_node(g, i, j, k4 + q);
}
__device__ __noinline__ void e_nodes4(const YeeArgs<float>& g, int i, int j, int k4) {
  for (int q = 0; q < 4; ++q) update_e_node(g, i, j, k4 + q);
}

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }

__global__ void __launch_bounds__(256) k_update_h_v4(const __grid_constant__ YeeArgs<float> g,
                                                     const __grid_constant__ VecBounds b) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x;
  const int k4 = (blockIdx.x * 32 + lane) * 4;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  const int n1 = g.n[1], n2 = g.n[2];
  const bool act = k4 < n2 && j < n1;
  const long long s1 = n2, s0 = (long long)n1 * n2;
  const long long p = i * s0 + j * s1 + k4;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 ex = act ? ld4(g.E[0] + p) : z4;
  const float4 ey = act ? ld4(g.E[1] + p) : z4;
  // E_x, E_y one node past the thread's last node
  float nex = __shfl_down_sync(full, ex.x, 1), ney = __shfl_down_sync(full, ey.x, 1);
  if (lane == 31 && act && k4 + 4 < n2) {
    nex = g.E[0][p + 4];
    ney = g.E[1][p + 4];
  }
  const bool fast = act && i >= b.lo[0] && i < b.hi[0] && j >= b.lo[1] && j < b.hi[1] && k4 >= b.lo[2] &&
                    k4 + 4 <= b.hi[2];
  const bool mid = !fast && act && in_all_regions(g, i, j, k4, k4 + 3);
  if (mid) {
    // inside every stepped region, some node in a CPML slab: the vector curl, then each node's psi terms
    const float4 ez = ld4(g.E[2] + p);
    const float4 ez_y = ld4(g.E[2] + p + s1), ex_y = ld4(g.E[0] + p + s1);
    const float4 ey_x = ld4(g.E[1] + p + s0), ez_x = ld4(g.E[2] + p + s0);
    float4 hx = ld4(g.H[0] + p), hy = ld4(g.H[1] + p), hz = ld4(g.H[2] + p);
    const float exa[5] = {ex.x, ex.y, ex.z, ex.w, nex}, eya[5] = {ey.x, ey.y, ey.z, ey.w, ney};
    const float eza[4] = {ez.x, ez.y, ez.z, ez.w}, ezy[4] = {ez_y.x, ez_y.y, ez_y.z, ez_y.w};
    const float exy[4] = {ex_y.x, ex_y.y, ex_y.z, ex_y.w}, eyx[4] = {ey_x.x, ey_x.y, ey_x.z, ey_x.w};
    const float ezx[4] = {ez_x.x, ez_x.y, ez_x.z, ez_x.w};
    float hxa[4] = {hx.x, hx.y, hx.z, hx.w}, hya[4] = {hy.x, hy.y, hy.z, hy.w}, hza[4] = {hz.x, hz.y, hz.z, hz.w};
    const float cH = g.cH;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      float av = ezy[q] - eza[q], bv = eya[q + 1] - eya[q];
      hxa[q] = hxa[q] - (g.uniform ? (av - bv) : (av * g.inv_d[1] - bv * g.inv_d[2])) * cH;
      cpml_node(hxa[q], g, b, 1, 0, i, j, k4 + q, av, bv, cH);
      av = exa[q + 1] - exa[q];
      bv = ezx[q] - eza[q];
      hya[q] = hya[q] - (g.uniform ? (av - bv) : (av * g.inv_d[2] - bv * g.inv_d[0])) * cH;
      cpml_node(hya[q], g, b, 1, 1, i, j, k4 + q, av, bv, cH);
      av = eyx[q] - eya[q];
      bv = exy[q] - exa[q];
      hza[q] = hza[q] - (g.uniform ? (av - bv) : (av * g.inv_d[0] - bv * g.inv_d[1])) * cH;
      cpml_node(hza[q], g, b, 1, 2, i, j, k4 + q, av, bv, cH);
    }
    st4(g.H[0] + p, make_float4(hxa[0], hxa[1], hxa[2], hxa[3]));
    st4(g.H[1] + p, make_float4(hya[0], hya[1], hya[2], hya[3]));
    st4(g.H[2] + p, make_float4(hza[0], hza[1], hza[2], hza[3]));
  } else if (fast) {
    const float4 ez = ld4(g.E[2] + p);
    const float4 ez_y = ld4(g.E[2] + p + s1), ex_y = ld4(g.E[0] + p + s1);
    const float4 ey_x = ld4(g.E[1] + p + s0), ez_x = ld4(g.E[2] + p + s0);
    float4 hx = ld4(g.H[0] + p), hy = ld4(g.H[1] + p), hz = ld4(g.H[2] + p);
    const float cH = g.cH;
    auto cu = [&](float a, float bb, int d1, int d2) {
      return g.uniform ? (a - bb) : (a * g.inv_d[d1] - bb * g.inv_d[d2]);
    };
    // H_x: dEz/dy - dEy/dz; H_y: dEx/dz - dEz/dx; H_z: dEy/dx - dEx/dy
    hx.x = hx.x - cu(ez_y.x - ez.x, ey.y - ey.x, 1, 2) * cH;
    hx.y = hx.y - cu(ez_y.y - ez.y, ey.z - ey.y, 1, 2) * cH;
    hx.z = hx.z - cu(ez_y.z - ez.z, ey.w - ey.z, 1, 2) * cH;
    hx.w = hx.w - cu(ez_y.w - ez.w, ney - ey.w, 1, 2) * cH;
    hy.x = hy.x - cu(ex.y - ex.x, ez_x.x - ez.x, 2, 0) * cH;
    hy.y = hy.y - cu(ex.z - ex.y, ez_x.y - ez.y, 2, 0) * cH;
    hy.z = hy.z - cu(ex.w - ex.z, ez_x.z - ez.z, 2, 0) * cH;
    hy.w = hy.w - cu(nex - ex.w, ez_x.w - ez.w, 2, 0) * cH;
    hz.x = hz.x - cu(ey_x.x - ey.x, ex_y.x - ex.x, 0, 1) * cH;
    hz.y = hz.y - cu(ey_x.y - ey.y, ex_y.y - ex.y, 0, 1) * cH;
    hz.z = hz.z - cu(ey_x.z - ey.z, ex_y.z - ex.z, 0, 1) * cH;
    hz.w = hz.w - cu(ey_x.w - ey.w, ex_y.w - ex.w, 0, 1) * cH;
    st4(g.H[0] + p, hx);
    st4(g.H[1] + p, hy);
    st4(g.H[2] + p, hz);
  } else if (act) {
    h_nodes4(g, i, j, k4);
  }
}

__global__ void __launch_bounds__(256) k_update_e_v4(const __grid_constant__ YeeArgs<float> g,
                                                     const __grid_constant__ VecBounds b) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x;
  const int k4 = (blockIdx.x * 32 + lane) * 4;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  const int n1 = g.n[1], n2 = g.n[2];
  const bool act = k4 < n2 && j < n1;
  const long long s1 = n2, s0 = (long long)n1 * n2;
  const long long p = i * s0 + j * s1 + k4;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 hx = act ? ld4(g.H[0] + p) : z4;
  const float4 hy = act ? ld4(g.H[1] + p) : z4;
  // H_x, H_y one node before the thread's first node
  float phx = __shfl_up_sync(full, hx.w, 1), phy = __shfl_up_sync(full, hy.w, 1);
  if (lane == 0 && act && k4 > 0) {
    phx = g.H[0][p - 1];
    phy = g.H[1][p - 1];
  }
  const bool fast = act && i >= b.lo[0] && i < b.hi[0] && j >= b.lo[1] && j < b.hi[1] && k4 >= b.lo[2] &&
                    k4 + 4 <= b.hi[2];
  const bool mid = !fast && act && in_all_regions(g, i, j, k4, k4 + 3);
  if (mid) {
    const float4 hz = ld4(g.H[2] + p);
    const float4 hz_y = ld4(g.H[2] + p - s1), hx_y = ld4(g.H[0] + p - s1);
    const float4 hz_x = ld4(g.H[2] + p - s0), hy_x = ld4(g.H[1] + p - s0);
    const float4 ex = ld4(g.E[0] + p), ey = ld4(g.E[1] + p), ez = ld4(g.E[2] + p);
    const float4 c0 = ld4(g.cbE[0] + p);
    const float4 c1 = g.cbE[1] == g.cbE[0] ? c0 : ld4(g.cbE[1] + p);
    const float4 c2 = g.cbE[2] == g.cbE[0] ? c0 : ld4(g.cbE[2] + p);
    const float hxa[5] = {phx, hx.x, hx.y, hx.z, hx.w}, hya[5] = {phy, hy.x, hy.y, hy.z, hy.w};
    const float hza[4] = {hz.x, hz.y, hz.z, hz.w}, hzy[4] = {hz_y.x, hz_y.y, hz_y.z, hz_y.w};
    const float hxy[4] = {hx_y.x, hx_y.y, hx_y.z, hx_y.w}, hzx[4] = {hz_x.x, hz_x.y, hz_x.z, hz_x.w};
    const float hyx[4] = {hy_x.x, hy_x.y, hy_x.z, hy_x.w};
    float exa[4] = {ex.x, ex.y, ex.z, ex.w}, eya[4] = {ey.x, ey.y, ey.z, ey.w}, eza[4] = {ez.x, ez.y, ez.z, ez.w};
    const float c0a[4] = {c0.x, c0.y, c0.z, c0.w}, c1a[4] = {c1.x, c1.y, c1.z, c1.w};
    const float c2a[4] = {c2.x, c2.y, c2.z, c2.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      float av = hza[q] - hzy[q], bv = hya[q + 1] - hya[q];
      exa[q] = exa[q] + (g.uniform ? (av - bv) : (av * g.inv_d[1] - bv * g.inv_d[2])) * c0a[q];
      cpml_node(exa[q], g, b, 0, 0, i, j, k4 + q, av, bv, c0a[q]);
      av = hxa[q + 1] - hxa[q];
      bv = hza[q] - hzx[q];
      eya[q] = eya[q] + (g.uniform ? (av - bv) : (av * g.inv_d[2] - bv * g.inv_d[0])) * c1a[q];
      cpml_node(eya[q], g, b, 0, 1, i, j, k4 + q, av, bv, c1a[q]);
      av = hya[q + 1] - hyx[q];
      bv = hxa[q + 1] - hxy[q];
      eza[q] = eza[q] + (g.uniform ? (av - bv) : (av * g.inv_d[0] - bv * g.inv_d[1])) * c2a[q];
      cpml_node(eza[q], g, b, 0, 2, i, j, k4 + q, av, bv, c2a[q]);
    }
    st4(g.E[0] + p, make_float4(exa[0], exa[1], exa[2], exa[3]));
    st4(g.E[1] + p, make_float4(eya[0], eya[1], eya[2], eya[3]));
    st4(g.E[2] + p, make_float4(eza[0], eza[1], eza[2], eza[3]));
  } else if (fast) {
    const float4 hz = ld4(g.H[2] + p);
    const float4 hz_y = ld4(g.H[2] + p - s1), hx_y = ld4(g.H[0] + p - s1);
    const float4 hz_x = ld4(g.H[2] + p - s0), hy_x = ld4(g.H[1] + p - s0);
    float4 ex = ld4(g.E[0] + p), ey = ld4(g.E[1] + p), ez = ld4(g.E[2] + p);
    const float4 c0 = ld4(g.cbE[0] + p);
    const float4 c1 = g.cbE[1] == g.cbE[0] ? c0 : ld4(g.cbE[1] + p);
    const float4 c2 = g.cbE[2] == g.cbE[0] ? c0 : ld4(g.cbE[2] + p);
    auto cu = [&](float a, float bb, int d1, int d2) {
      return g.uniform ? (a - bb) : (a * g.inv_d[d1] - bb * g.inv_d[d2]);
    };
    // E_x: dHz/dy - dHy/dz; E_y: dHx/dz - dHz/dx; E_z: dHy/dx - dHx/dy
    ex.x = ex.x + cu(hz.x - hz_y.x, hy.x - phy, 1, 2) * c0.x;
    ex.y = ex.y + cu(hz.y - hz_y.y, hy.y - hy.x, 1, 2) * c0.y;
    ex.z = ex.z + cu(hz.z - hz_y.z, hy.z - hy.y, 1, 2) * c0.z;
    ex.w = ex.w + cu(hz.w - hz_y.w, hy.w - hy.z, 1, 2) * c0.w;
    ey.x = ey.x + cu(hx.x - phx, hz.x - hz_x.x, 2, 0) * c1.x;
    ey.y = ey.y + cu(hx.y - hx.x, hz.y - hz_x.y, 2, 0) * c1.y;
    ey.z = ey.z + cu(hx.z - hx.y, hz.z - hz_x.z, 2, 0) * c1.z;
    ey.w = ey.w + cu(hx.w - hx.z, hz.w - hz_x.w, 2, 0) * c1.w;
    ez.x = ez.x + cu(hy.x - hy_x.x, hx.x - hx_y.x, 0, 1) * c2.x;
    ez.y = ez.y + cu(hy.y - hy_x.y, hx.y - hx_y.y, 0, 1) * c2.y;
    ez.z = ez.z + cu(hy.z - hy_x.z, hx.z - hx_y.z, 0, 1) * c2.z;
    ez.w = ez.w + cu(hy.w - hy_x.w, hx.w - hx_y.w, 0, 1) * c2.w;
    st4(g.E[0] + p, ex);
    st4(g.E[1] + p, ey);
    st4(g.E[2] + p, ez);
  } else if (act) {
    e_nodes4(g, i, j, k4);
  }
}

}  // namespace lsfdtd
