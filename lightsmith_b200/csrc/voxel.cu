// Material on the Yee E grid from lightsmith's particle shapes, on the GPU (the host set-up of a scattering
// solve: backends/_fdtd/setup.py:110-289, voxelise, with the slots of setup.py:707-716, particle_slot_fn, and
// backends/_fdtd/scattering.py:81-90, the substrate below its interface).
//
// Three kernels, each over work the host set-up does point by point:
//   k_vox_lattice     the medium slot at every point of the half-cell lattice origin + (m / 2) dx over the
//                     region of interest (every E position and every corner and edge midpoint of its cell);
//   k_vox_classify    per E_c node of the region: its slot, or -1 where a supersampled mesh sees an interface
//                     (a corner or edge midpoint of the node's cell holds another slot);
//   k_vox_supersample per interface cell (one warp): the slot at samples^3 points of the cell, the media
//                     fractions, the first moment of the dominant medium (the interface normal), the smoothed
//                     1/eps_cc of a cell without dispersive media and its off-diagonal terms.
// Every coordinate, containment test and smoothing formula is evaluated with the operations and the order
// numpy uses on the host (no contractions into fused multiply-adds), so the slots are the same point for
// point. The moment sums are sums of products of dyadic numbers with a power-of-two sample count (the
// default 8): exact, in any order.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "lsfdtd.h"

namespace lsfdtd {
int report_error(int code, const std::string& msg);
}

namespace {

// a point's slot: the first particle (in list order) whose region holds it, else the substrate below its
// interface, else 0 (the host medium)
__device__ int vox_slot(const lsfdtd_vox_scene& s, double x, double y, double z) {
  int out = 0;
  for (int i = 0; i < s.n_particles; ++i) {
    const lsfdtd_vox_particle& p = s.particles[i];
    const double p0 = __dsub_rn(x, p.pos[0]), p1 = __dsub_rn(y, p.pos[1]), p2 = __dsub_rn(z, p.pos[2]);
    const double q0 = __dmul_rn(p0, p0), q1 = __dmul_rn(p1, p1), q2 = __dmul_rn(p2, p2);
    int region = -1;
    switch (p.kind) {
      case LSFDTD_VOX_SPHERE:
        region = __dadd_rn(__dadd_rn(q0, q1), q2) <= __dmul_rn(p.a, p.a) ? 0 : -1;
        break;
      case LSFDTD_VOX_SPHEROID: {
        const double t = __dadd_rn(__ddiv_rn(__dadd_rn(q0, q1), __dmul_rn(p.a, p.a)), __ddiv_rn(q2, __dmul_rn(p.b, p.b)));
        region = t <= 1.0 ? 0 : -1;
        break;
      }
      case LSFDTD_VOX_CYLINDER:
        region = (__dadd_rn(q0, q1) <= __dmul_rn(p.a, p.a) && fabs(p2) <= __ddiv_rn(p.b, 2.0)) ? 0 : -1;
        break;
      case LSFDTD_VOX_LAYERED_SPHERE: {
        const double r = __dsqrt_rn(__dadd_rn(__dadd_rn(q0, q1), q2));
        if (r <= p.radii[p.n_regions - 1]) {
          int k = 0;  // the radii below r (a left-sided search of the sorted radii)
          while (k < p.n_regions && p.radii[k] < r) ++k;
          region = k;
        }
        break;
      }
      default:
        break;
    }
    if (region >= 0 && region < p.n_regions && out == 0) out = p.slot[region];
  }
  if (s.has_substrate && out == 0 && z < s.z_int) out = s.sub_slot;
  return out;
}

// the half-cell lattice point m (per axis, from 2 roi_lo - 1) in nm
__device__ __forceinline__ double lattice_coord(const lsfdtd_vox_scene& s, int a, long long m) {
  return __dadd_rn(s.origin[a], __dmul_rn((double)(2LL * s.roi_lo[a] - 1 + m) * 0.5, s.dx[a]));
}

__global__ void k_vox_lattice(const lsfdtd_vox_scene s, long long l1, long long l2, long long n, int16_t* lat) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / (l1 * l2), r = t % (l1 * l2), j = r / l2, k = r % l2;
    lat[t] = (int16_t)vox_slot(s, lattice_coord(s, 0, i), lattice_coord(s, 1, j), lattice_coord(s, 2, k));
  }
}

// per node of the region (i, j, k from roi_lo): lattice index of the node's E_c position is 1 + (a == c) + 2 i
// per axis, and of its 26 neighbours that plus -1, 0 or 1
__global__ void k_vox_classify(const lsfdtd_vox_scene s, const int16_t* lat, int c, int subpixel, int16_t* cls) {
  const long long n0 = s.roi_hi[0] - s.roi_lo[0], n1 = s.roi_hi[1] - s.roi_lo[1], n2 = s.roi_hi[2] - s.roi_lo[2];
  const long long l1 = 2 * n1 + 2, l2 = 2 * n2 + 2, n = n0 * n1 * n2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / (n1 * n2), r = t % (n1 * n2), j = r / n2, k = r % n2;
    const long long li = 1 + (c == 0) + 2 * i, lj = 1 + (c == 1) + 2 * j, lk = 1 + (c == 2) + 2 * k;
    const int16_t ctr = lat[(li * l1 + lj) * l2 + lk];
    bool mixed = false;
    if (subpixel) {
      for (int o = 0; o < 27 && !mixed; ++o) {
        const int di = o / 9 - 1, dj = (o / 3) % 3 - 1, dk = o % 3 - 1;
        if (o == 13) continue;
        mixed = lat[((li + di) * l1 + (lj + dj)) * l2 + (lk + dk)] != ctr;
      }
    }
    cls[t] = mixed ? (int16_t)-1 : ctr;
  }
}

constexpr int kVoxMaxMedia = LSFDTD_VOX_MAX_MEDIA;

// one warp per interface cell: node (i, j, k) of the region for component c. out per cell (row q of n):
// frac[s * n + q] (S media), nhat[3 q + d], w[q], part[q] (holds a medium outside the background set),
// has_disp[q], inv[q] (smoothed 1/eps_cc, cells without dispersive media), od[3 q + d] (off-diagonal terms,
// conformal mode; column c zero)
__global__ void k_vox_supersample(const lsfdtd_vox_scene s, lsfdtd_vox_media m, int c, const int64_t* cells,
                                  long long n, double* frac, double* nhat, double* w_out, int8_t* part,
                                  int8_t* has_disp, double* inv, double* od) {
  const int lane = threadIdx.x & 31;
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
  const long long n1 = s.roi_hi[1] - s.roi_lo[1], n2 = s.roi_hi[2] - s.roi_lo[2];
  const int ns = m.samples, ns3 = ns * ns * ns;
  for (long long q = warp; q < n; q += warps) {
    const long long t = cells[q];
    const long long i = t / (n1 * n2), r = t % (n1 * n2), j = r / n2, k = r % n2;
    const long long idx[3] = {s.roi_lo[0] + i, s.roi_lo[1] + j, s.roi_lo[2] + k};
    double ctr[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
      ctr[a] = __dadd_rn(s.origin[a], __dmul_rn((double)idx[a] + (a == c ? 0.5 : 0.0), s.dx[a]));
    // the slot of every sample, counted per medium (each lane its samples; the counts are exact)
    int cnt[kVoxMaxMedia];
#pragma unroll
    for (int u = 0; u < kVoxMaxMedia; ++u) cnt[u] = 0;
    for (int e = lane; e < ns3; e += 32) {
      const int a0 = e / (ns * ns), a1 = (e / ns) % ns, a2 = e % ns;
      double pt[3];
      const int ai[3] = {a0, a1, a2};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double sub = __dsub_rn(__ddiv_rn((double)ai[a] + 0.5, (double)ns), 0.5);
        pt[a] = __dadd_rn(ctr[a], __dmul_rn(sub, s.dx[a]));
      }
      const int sl = vox_slot(s, pt[0], pt[1], pt[2]);
#pragma unroll
      for (int u = 0; u < kVoxMaxMedia; ++u) cnt[u] += (sl == u);
    }
#pragma unroll
    for (int u = 0; u < kVoxMaxMedia; ++u)
      for (int o = 16; o; o >>= 1) cnt[u] += __shfl_xor_sync(0xffffffffu, cnt[u], o);
    // the dominant medium (the first of the largest fractions) and the first moment of its indicator
    int dom = 0;
    for (int u = 1; u < m.n; ++u)
      if (cnt[u] > cnt[dom]) dom = u;
    double mom[3] = {0.0, 0.0, 0.0};
    const double mean = __ddiv_rn((double)cnt[dom], (double)ns3);
    for (int e = lane; e < ns3; e += 32) {
      const int a0 = e / (ns * ns), a1 = (e / ns) % ns, a2 = e % ns;
      const int ai[3] = {a0, a1, a2};
      double pt[3], sub[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        sub[a] = __dsub_rn(__ddiv_rn((double)ai[a] + 0.5, (double)ns), 0.5);
        pt[a] = __dadd_rn(ctr[a], __dmul_rn(sub[a], s.dx[a]));
      }
      const double chi = __dsub_rn(vox_slot(s, pt[0], pt[1], pt[2]) == dom ? 1.0 : 0.0, mean);
#pragma unroll
      for (int a = 0; a < 3; ++a) mom[a] = __dadd_rn(mom[a], __dmul_rn(chi, sub[a]));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
      for (int o = 16; o; o >>= 1) mom[a] = __dadd_rn(mom[a], __shfl_xor_sync(0xffffffffu, mom[a], o));
    if (lane != 0) continue;
#pragma unroll
    for (int a = 0; a < 3; ++a) mom[a] = __ddiv_rn(mom[a], s.dx[a]);
    const double nrm = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(mom[0], mom[0]), __dmul_rn(mom[1], mom[1])),
                                            __dmul_rn(mom[2], mom[2])));
    double nh[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) nh[a] = nrm > 1e-12 ? __ddiv_rn(mom[a], nrm > 0 ? nrm : 1.0) : 0.0;
    double w = nrm > 1e-12 ? __dmul_rn(nh[c], nh[c]) : 1.0 / 3.0;
    if (m.mode == LSFDTD_VOX_VOLUME_AVERAGE) w = 0.0;
    bool pm = false, hd = false;
    double harm = 0.0, arit = 0.0;
    for (int u = 0; u < m.n; ++u) {
      const double f = __ddiv_rn((double)cnt[u], (double)ns3);
      frac[(long long)u * n + q] = f;
      pm |= !m.background[u] && f > 0.0;
      hd |= m.dispersive[u] && f > 0.0;
      harm = __dadd_rn(harm, __ddiv_rn(f, m.eps_inf[u]));
      arit = __dadd_rn(arit, __dmul_rn(f, m.eps_inf[u]));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) nhat[3 * q + a] = nh[a];
    w_out[q] = w;
    part[q] = pm ? 1 : 0;
    has_disp[q] = hd ? 1 : 0;
    inv[q] = __dadd_rn(__dmul_rn(w, harm), __ddiv_rn(__dsub_rn(1.0, w), arit));
    const double dh = __dsub_rn(harm, __ddiv_rn(1.0, arit));
#pragma unroll
    for (int a = 0; a < 3; ++a) od[3 * q + a] = a == c ? 0.0 : __dmul_rn(__dmul_rn(nh[a], nh[c]), dh);
  }
}

int fail_v(int code, const char* msg) { return lsfdtd::report_error(code, msg); }

bool scene_ok(const lsfdtd_vox_scene* s) {
  if (!s || s->n_particles < 0 || (s->n_particles > 0 && !s->particles)) return false;
  for (int a = 0; a < 3; ++a)
    if (s->roi_lo[a] < 0 || s->roi_hi[a] <= s->roi_lo[a] || s->roi_hi[a] > s->shape[a] || !(s->dx[a] > 0))
      return false;
  return true;
}

unsigned grid_for(long long n, int threads) {
  const long long b = (n + threads - 1) / threads;
  return (unsigned)(b < 65535LL * 64 ? (b > 0 ? b : 1) : 65535LL * 64);
}

}  // namespace

extern "C" {

int32_t lsfdtd_vox_lattice(const lsfdtd_vox_scene* scene, int16_t* lattice, void* stream) {
  if (!scene_ok(scene) || !lattice) return fail_v(LSFDTD_EINVAL, "voxelise: invalid scene or null lattice");
  const lsfdtd_vox_scene& s = *scene;
  const long long l0 = 2LL * (s.roi_hi[0] - s.roi_lo[0]) + 2, l1 = 2LL * (s.roi_hi[1] - s.roi_lo[1]) + 2,
                  l2 = 2LL * (s.roi_hi[2] - s.roi_lo[2]) + 2, n = l0 * l1 * l2;
  k_vox_lattice<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(s, l1, l2, n, lattice);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LSFDTD_OK : fail_v(LSFDTD_ECUDA, cudaGetErrorString(e));
}

int32_t lsfdtd_vox_classify(const lsfdtd_vox_scene* scene, const int16_t* lattice, int32_t c, int32_t subpixel,
                            int16_t* cls, void* stream) {
  if (!scene_ok(scene) || !lattice || !cls || c < 0 || c > 2)
    return fail_v(LSFDTD_EINVAL, "voxelise: invalid scene, component or null array");
  const lsfdtd_vox_scene& s = *scene;
  const long long n = (long long)(s.roi_hi[0] - s.roi_lo[0]) * (s.roi_hi[1] - s.roi_lo[1]) * (s.roi_hi[2] - s.roi_lo[2]);
  k_vox_classify<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(s, lattice, c, subpixel, cls);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LSFDTD_OK : fail_v(LSFDTD_ECUDA, cudaGetErrorString(e));
}

int32_t lsfdtd_vox_supersample(const lsfdtd_vox_scene* scene, const lsfdtd_vox_media* media, int32_t c,
                               const int64_t* cells, int64_t n, lsfdtd_vox_cells out, void* stream) {
  if (!scene_ok(scene) || !media || c < 0 || c > 2 || n < 0 || (n > 0 && !cells))
    return fail_v(LSFDTD_EINVAL, "voxelise: invalid scene, media, component or cells");
  if (media->n < 1 || media->n > LSFDTD_VOX_MAX_MEDIA || media->samples < 1 || media->samples > 64)
    return fail_v(LSFDTD_EINVAL, "voxelise: 1 to LSFDTD_VOX_MAX_MEDIA media, 1 to 64 samples per axis");
  if (n == 0) return LSFDTD_OK;
  if (!out.frac || !out.nhat || !out.w || !out.part || !out.has_disp || !out.inv || !out.od)
    return fail_v(LSFDTD_EINVAL, "voxelise: null output array");
  const long long threads = n * 32;
  k_vox_supersample<<<grid_for(threads, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      *scene, *media, c, cells, n, out.frac, out.nhat, out.w, out.part, out.has_disp, out.inv, out.od);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LSFDTD_OK : fail_v(LSFDTD_ECUDA, cudaGetErrorString(e));
}

}  // extern "C"
