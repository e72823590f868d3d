// Dispersive (Drude-Lorentz) nodes integrated in D-form with auxiliary differential equations.
//
// Per node, after the E curl and the sources' E corrections (backends/_fdtd/engine.py:722-793):
//   D += E_now - E_prev
//   pure node:   P_k <- c1 P_k + c2 P_k' + c3 E_prev (P_k' <- old P_k);  E = (D - sum_k P_k) / eps_inf
//   mixed node:  harmonic path, per dispersive medium s its own E_s driving its poles,
//                  harm = h0 D + sum_s f_s E_s,  E_s = (D - sum P^h_s) / eps_inf_s
//                arithmetic path, all poles driven by E_a, E_a = (D - sum_s f_s sum P^a_s) * inv_a
//                E = w harm + (1 - w) E_a      (only the paths the group uses at all are run)
//   E_prev = E.
// State is structure-of-arrays (coalesced per field of the state) in one caller-owned buffer.
#pragma once

#include "common.cuh"

namespace lsfdtd {

constexpr int kMaxMedia = 4;
constexpr int kMaxPoles = 6;

template <typename F>
struct AdeArgs {
  using R = typename real_of<F>::type;
  long long n;
  const long long* idx;
  F* E;  // flat E (component-stacked)
  int n_media;                     // dispersive media (1 for a pure group)
  int n_poles[kMaxMedia];
  R c1[kMaxMedia][kMaxPoles], c2[kMaxMedia][kMaxPoles], c3[kMaxMedia][kMaxPoles];
  R inv_inf[kMaxMedia];
  int mixed, has_h, has_a;
  const R* h0;
  const R* inv_a;
  const R* w;
  const R* frac;  // [n_media][n]
  F* state;
};

// state offsets (in units of n): pure D, Eprev, (P, P') per pole;
// mixed D, Eprev, Ea, Eh[s], (P, P')^h[s][k], (P, P')^a[s][k]
template <typename F>
__global__ void k_ade(AdeArgs<F> g) {
  using R = typename real_of<F>::type;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.n) return;
  const long long n = g.n;
  F* D = g.state;
  F* Ep = g.state + n;
  const long long node = g.idx[t];
  const F e_now = g.E[node];
  F d = D[t] + (e_now - Ep[t]);
  // the reference evaluates D += e_now - E_prev as D + (e_now - E_prev)
  D[t] = d;
  F e_new;
  if (!g.mixed) {
    F* P = g.state + 2 * n;
    const F drive = Ep[t];
    F tot = zero<F>();
    for (int k = 0; k < g.n_poles[0]; ++k) {
      F* pk = P + (2 * k) * n;
      F* pp = P + (2 * k + 1) * n;
      const F p0 = pk[t], p1 = pp[t];
      const F nw = g.c1[0][k] * p0 + g.c2[0][k] * p1 + g.c3[0][k] * drive;
      pp[t] = p0;
      pk[t] = nw;
      tot = k == 0 ? nw : tot + nw;
    }
    e_new = (d - tot) * g.inv_inf[0];
  } else {
    const int S = g.n_media;
    F* Ea = g.state + 2 * n;
    F* Eh = g.state + 3 * n;  // [S][n]
    F* Pbase = g.state + (3 + S) * n;
    int n_tot_poles = 0;
    for (int s = 0; s < S; ++s) n_tot_poles += g.n_poles[s];
    F* Ph = Pbase;                         // [sum poles][2][n]
    F* Pa = Pbase + 2 * n_tot_poles * n;   // same layout
    const R w = g.w[t];
    F part_h = zero<F>(), part_a = zero<F>();
    if (g.has_h) {
      F harm = d * g.h0[t];
      int off = 0;
      for (int s = 0; s < S; ++s) {
        const F drive = Eh[s * n + t];
        F tot = zero<F>();
        for (int k = 0; k < g.n_poles[s]; ++k) {
          F* pk = Ph + (2 * (off + k)) * n;
          F* pp = Ph + (2 * (off + k) + 1) * n;
          const F p0 = pk[t], p1 = pp[t];
          const F nw = g.c1[s][k] * p0 + g.c2[s][k] * p1 + g.c3[s][k] * drive;
          pp[t] = p0;
          pk[t] = nw;
          tot = k == 0 ? nw : tot + nw;
        }
        const F es = (d - tot) * g.inv_inf[s];
        Eh[s * n + t] = es;
        harm = harm + g.frac[s * n + t] * es;
        off += g.n_poles[s];
      }
      part_h = w * harm;
    }
    if (g.has_a) {
      F acc = d;
      const F drive = Ea[t];
      int off = 0;
      for (int s = 0; s < S; ++s) {
        F tot = zero<F>();
        for (int k = 0; k < g.n_poles[s]; ++k) {
          F* pk = Pa + (2 * (off + k)) * n;
          F* pp = Pa + (2 * (off + k) + 1) * n;
          const F p0 = pk[t], p1 = pp[t];
          const F nw = g.c1[s][k] * p0 + g.c2[s][k] * p1 + g.c3[s][k] * drive;
          pp[t] = p0;
          pk[t] = nw;
          tot = k == 0 ? nw : tot + nw;
        }
        acc = acc - g.frac[s * n + t] * tot;
        off += g.n_poles[s];
      }
      const F ea = acc * g.inv_a[t];
      Ea[t] = ea;
      part_a = (R(1) - w) * ea;
    }
    e_new = g.has_h && g.has_a ? part_h + part_a : (g.has_h ? part_h : part_a);
  }
  g.E[node] = e_new;
  Ep[t] = e_new;
}

inline long long ade_state_len(int mixed, int n_media, const int* n_poles) {
  if (!mixed) return 2 + 2LL * n_poles[0];
  long long tot = 0;
  for (int s = 0; s < n_media; ++s) tot += n_poles[s];
  return 3 + n_media + 4 * tot;
}

}  // namespace lsfdtd
