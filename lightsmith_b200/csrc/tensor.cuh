// The vertex-tensor ADE of conformal interfaces with dispersive media (backends/_fdtd/engine.py:140-175,
// 796-923), on the index tables lightsmith_b200/plan.py:tensor_plan builds.
//
// Per step, after the E curl update, the sources' E corrections and the D-form groups:
//   nodes:    D += E - E_prev
//   vertices: per axis d the mean D~_d of the vertex's two d-nodes (each times its Bloch phase and mirror
//             parity), and s = n . D~
//   slots:    a tensor slot (a node next to a vertex) takes sigma = s + n_c (D_p - D~_c) and
//             out = (1/2) (b[D_p - n_c sigma] + n_c a[sigma]) (times the conjugate phase under a Bloch
//             wavevector); a (harmonic, <1/eps>) and b (arithmetic, 1/<eps>) are ADE operators with the vertex's
//             medium fractions and their own pole states; a plain slot takes out = (1/2) m[D] of its one medium
//   nodes:    E = E_prev = out[slot 0] + out[slot 1]
// Each kernel runs one thread per node, vertex or slot; the state is structure-of-arrays in one buffer.
#pragma once

#include "ade.cuh"
#include "common.cuh"

namespace lsfdtd {

template <typename F>
struct TensorArgs {
  using R = typename real_of<F>::type;
  F* E;                 // flat fields
  const long long* idx;  // (nN) flat E indices of the nodes
  long long nN, nV, nT, nP;
  const long long* vn;   // (nV * 6) node number of each vertex's (minus, plus) d-node, per d
  const F* scale;        // (nV * 6) phase and parity of each of those node positions, or null
  const R* normal;       // (nV * 3)
  const long long *t_pos, *t_v, *t_vc, *t_g;  // (nT) output slot, vertex, vertex * 3 + c, its node position
  const R* t_nc;         // (nT) the normal's component along the node's
  const F* t_conj;       // (nT) conjugate phase, or null
  const R* frac;         // (S, nT) medium fractions of the slot's vertex
  const long long *p_pos, *p_node, *p_medium;  // (nP) plain slots
  int n_media;
  int n_poles[kMaxMedia];
  R inv_inf[kMaxMedia], eps_inf[kMaxMedia];
  R c1[kMaxMedia][kMaxPoles], c2[kMaxMedia][kMaxPoles], c3[kMaxMedia][kMaxPoles];
  // state (field precision): D, E_prev, out (2 nN), D~ (nV * 3), s (nV); per medium s: the harmonic E_s (nT)
  // and (P, P') per pole (nT each); the arithmetic y (nT) and per medium (P, P') per pole; per medium the
  // plain slots' E_s (nP) and (P, P') per pole
  F *D, *Ep, *out, *dbar, *sv;
  F* ha_E[kMaxMedia];
  F* ha_P[kMaxMedia];  // [pole][2][nT]
  F* ar_y;
  F* ar_P[kMaxMedia];
  F* pl_E[kMaxMedia];  // [nP]
  F* pl_P[kMaxMedia];  // [pole][2][nP]
};

// points the state arrays of `a` into one buffer of lsfdtd_tensor_state_len field scalars (sizes and media
// set): D, E_prev, out (2 nN), D~ (3 nV), s (nV); per medium the harmonic E_s and its poles; the arithmetic y;
// per medium its poles; per medium the plain slots' E_s and poles
template <typename F>
inline void tm_bind_state(TensorArgs<F>& a, F* st) {
  a.D = st;
  st += a.nN;
  a.Ep = st;
  st += a.nN;
  a.out = st;
  st += 2 * a.nN;
  a.dbar = st;
  st += 3 * a.nV;
  a.sv = st;
  st += a.nV;
  for (int s = 0; s < a.n_media; ++s) {
    a.ha_E[s] = st;
    st += a.nT;
    a.ha_P[s] = st;
    st += 2LL * a.n_poles[s] * a.nT;
  }
  a.ar_y = st;
  st += a.nT;
  for (int s = 0; s < a.n_media; ++s) {
    a.ar_P[s] = st;
    st += 2LL * a.n_poles[s] * a.nT;
  }
  for (int s = 0; s < a.n_media; ++s) {
    a.pl_E[s] = st;
    st += a.nP;
    a.pl_P[s] = st;
    st += 2LL * a.n_poles[s] * a.nP;
  }
}

// P_k <- c1 P_k + c2 P'_k + c3 drive, P'_k <- old P_k, for every pole of medium s at slot t of n; the sum of
// the new P_k (_Group._advance, engine.py:759-767)
template <typename F>
__device__ __forceinline__ F tm_poles(const TensorArgs<F>& g, int s, F* P, long long t, long long n, F drive) {
  F tot = zero<F>();
  for (int k = 0; k < g.n_poles[s]; ++k) {
    F* pk = P + (2 * k) * n;
    F* pp = P + (2 * k + 1) * n;
    const F p0 = pk[t], p1 = pp[t];
    const F nw = g.c1[s][k] * p0 + g.c2[s][k] * p1 + g.c3[s][k] * drive;
    pp[t] = p0;
    pk[t] = nw;
    tot = k == 0 ? nw : tot + nw;
  }
  return tot;
}

template <typename F>
__global__ void k_tm_nodes_d(TensorArgs<F> g) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.nN) return;
  g.D[i] = g.D[i] + (g.E[g.idx[i]] - g.Ep[i]);
}

template <typename F>
__global__ void k_tm_vertices(TensorArgs<F> g) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= g.nV) return;
  F s = zero<F>();
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    F a = g.D[g.vn[v * 6 + 2 * d]], b = g.D[g.vn[v * 6 + 2 * d + 1]];
    if (g.scale) {
      a = a * g.scale[v * 6 + 2 * d];
      b = b * g.scale[v * 6 + 2 * d + 1];
    }
    const F m = (a + b) * typename real_of<F>::type(0.5);
    g.dbar[v * 3 + d] = m;
    s = d == 0 ? g.normal[v * 3] * m : s + g.normal[v * 3 + d] * m;
  }
  g.sv[v] = s;
}

template <typename F>
__global__ void k_tm_slots(TensorArgs<F> g) {
  using R = typename real_of<F>::type;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.nT) return;
  const long long gp = g.t_g[t];
  F dp = g.D[g.vn[gp]];
  if (g.scale) dp = dp * g.scale[gp];
  const R nc = g.t_nc[t];
  const F sigma = g.sv[g.t_v[t]] + nc * (dp - g.dbar[g.t_vc[t]]);
  // a = <1/eps>[sigma]: u h0 plus each dispersive medium's E_s, driven by its own E_s of the step before
  const F ua = sigma;
  R h0 = R(0);
  for (int s = 0; s < g.n_media; ++s)
    if (!g.n_poles[s]) h0 += g.frac[s * g.nT + t] / g.eps_inf[s];
  F ya = ua * h0;
  for (int s = 0; s < g.n_media; ++s) {
    if (!g.n_poles[s]) continue;
    const F tot = tm_poles(g, s, g.ha_P[s], t, g.nT, g.ha_E[s][t]);
    const F es = (ua - tot) * g.inv_inf[s];
    g.ha_E[s][t] = es;
    ya = ya + g.frac[s * g.nT + t] * es;
  }
  // b = (1/<eps>)[D_p - n_c sigma]: every pole driven by the y of the step before
  const F ub = dp - nc * sigma;
  const F yprev = g.ar_y[t];
  F acc = ub;
  R den = R(0);
  for (int s = 0; s < g.n_media; ++s) den += g.frac[s * g.nT + t] * g.eps_inf[s];
  for (int s = 0; s < g.n_media; ++s) {
    if (!g.n_poles[s]) continue;
    acc = acc - g.frac[s * g.nT + t] * tm_poles(g, s, g.ar_P[s], t, g.nT, yprev);
  }
  const F yb = acc * (R(1) / den);
  g.ar_y[t] = yb;
  F c = (yb + nc * ya) * R(0.5);
  if (g.t_conj) c = c * g.t_conj[t];
  g.out[g.t_pos[t]] = c;
}

template <typename F>
__global__ void k_tm_plain(TensorArgs<F> g) {
  using R = typename real_of<F>::type;
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.nP) return;
  const int m = (int)g.p_medium[p];
  const F u = g.D[g.p_node[p]];
  F y;
  if (!g.n_poles[m]) {
    y = u * (R(1) / g.eps_inf[m]);
  } else {  // its one dispersive medium: y = E_m
    const F tot = tm_poles(g, m, g.pl_P[m], p, g.nP, g.pl_E[m][p]);
    y = (u - tot) * g.inv_inf[m];
    g.pl_E[m][p] = y;
  }
  g.out[g.p_pos[p]] = y * R(0.5);
}

template <typename F>
__global__ void k_tm_nodes_e(TensorArgs<F> g) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.nN) return;
  const F e = g.out[i] + g.out[g.nN + i];
  g.E[g.idx[i]] = e;
  g.Ep[i] = e;
}

}  // namespace lsfdtd
