// lsfdtd: the FDTD engine behind the C ABI of include/lsfdtd.h.
//
// An engine is a host-side list of kernel launches over caller-owned device memory: the step order of
// lightsmith's Engine.step (backends/_fdtd/engine.py:665-678) with the Yee/CPML updates fused per field, then
// the sources' hooks, the dispersive groups and the step counter. Nothing here allocates device memory or
// synchronises the host, so a chunk can be captured once as a CUDA graph and replayed.
#include <algorithm>
#include <cmath>
#include <memory>
#include <cstring>
#include <type_traits>
#include <limits>
#include <string>
#include <vector>

#include "lsfdtd.h"

#include "ade.cuh"
#include "adjoint.cuh"
#include "batch.cuh"
#include "common.cuh"
#include "fused.cuh"
#include "fused_pml.cuh"
#include "fused_tma.cuh"
#include "shell.cuh"
#include "tensor.cuh"
#include "yee_vec.cuh"

#include <cudaTypedefs.h>
#include "monitors.cuh"
#include "sources.cuh"
#include "yee.cuh"

using namespace lsfdtd;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define LS_CUDA(x)                                                                          \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess) return fail(LSFDTD_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define LS_LAUNCHED()                                                                       \
  do {                                                                                      \
    cudaError_t e_ = cudaGetLastError();                                                    \
    if (e_ != cudaSuccess) return fail(LSFDTD_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
  } while (0)

#define LS_TRY(x)                 \
  do {                            \
    int r_ = (x);                 \
    if (r_ != LSFDTD_OK) return r_; \
  } while (0)

// stepped range of a field component along an axis (engine.py:47-66, no mirror planes)
void region(int field, int c, int a, const int32_t* shape, const int32_t* periodic, int* lo, int* hi) {
  const int n = shape[a];
  if (field == 0) {
    *lo = (periodic[a] || a != c) ? 1 : 0;
    *hi = n - 1;
  } else {
    *lo = periodic[a] ? 1 : 0;
    *hi = periodic[a] ? n - 1 : (a == c ? n : n - 1);
  }
}

int slab(const int32_t* shape, const int32_t* periodic, int d, int lo_n, int hi_n, int field, int c, int side,
         int* start, int* len) {
  *start = 0;
  *len = 0;
  if (c == d || (side == 0 && !lo_n) || (side == 1 && !hi_n)) return LSFDTD_OK;
  int st, sp;
  region(field, c, d, shape, periodic, &st, &sp);
  int a, b;
  if (side == 0) {
    a = st;
    b = std::min(sp, lo_n + 1);
  } else {
    a = std::max(st, shape[d] - 2 - hi_n);
    b = sp;
  }
  if (b > a) {
    *start = a;
    *len = b - a;
  }
  return LSFDTD_OK;
}

}  // namespace

namespace lsfdtd {
// the error hook of the library's other translation units (lsfdtd_last_error reports it)
int report_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace lsfdtd

struct lsfdtd_engine {
  lsfdtd_grid_desc desc{};
  int64_t n_host = 0;
  int64_t step_limit = std::numeric_limits<int64_t>::max();
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};  // one captured chunk per starting buffer
  cudaGraph_t graph[2] = {nullptr, nullptr};
  int cur = 0;          // buffer holding the current fields
  int fused = -1;       // -1 undecided, 0 in-place kernels, 1 fused single pass
  // 0: in-place H and E kernels; 1: the fused single pass; 2: in-place four-node kernels; 3: the fused pass
  // split into an interior box without region or CPML code and shell kernels; 4: the fused pass with lean CPML
  // terms (3 and 4 run as 1 where they do not apply); runs the fused pass does not serve take 0
  int variant = 4;
  int tile_y = 8, planes = 0, stages = 4;  // planes 0: chosen per grid (Engine::auto_planes)
  int sm_count = 0;
  int use_tma = 1;      // fused pass copies planes with the Tensor Memory Accelerator where the layout allows
  bool tuned = false;   // a kernel choice was set explicitly (lsfdtd_engine_set_tuning)
  long long wait_budget = lsfdtd::kWaitBudget;  // cycles the fused pass waits for a plane's copies
  // the lean pass steps the clean interior of the grid with a kernel that has no region or CPML code, beside
  // the lean kernel on the CTAs around it (where the grid has such an interior and no source corrects H)
  int split_clean = 1;
  virtual int init_side() = 0;  // the side streams of that split and their fork and join events
  // when set, event pairs around every bulk (Yee) kernel launch are appended here (diagnostic timing)
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>>* timing = nullptr;
  virtual ~lsfdtd_engine() {
    for (int b = 0; b < 2; ++b) {
      if (exec[b]) cudaGraphExecDestroy(exec[b]);
      if (graph[b]) cudaGraphDestroy(graph[b]);
    }
  }
  virtual int set_pml(const lsfdtd_pml_desc* p) = 0;
  virtual int add_group(const lsfdtd_group_desc* g) = 0;
  virtual int add_offdiag(const lsfdtd_offdiag_desc* d) = 0;
  virtual int add_tensor(const lsfdtd_tensor_desc* d) = 0;
  virtual int add_table(const lsfdtd_table_source_desc* s) = 0;
  virtual int set_table_boxes(int table, int n, const int32_t* boxes, const int64_t* perm, int64_t n_entries,
                              void* vals) = 0;
  virtual int add_dipole(const lsfdtd_dipole_desc* s) = 0;
  virtual int add_line(const lsfdtd_line_source_desc* s) = 0;
  virtual int add_column(const lsfdtd_column_source_desc* s) = 0;
  virtual int add_mode(const lsfdtd_mode_source_desc* s) = 0;
  virtual int add_monitor(const lsfdtd_monitor_desc* m) = 0;
  virtual size_t need_scratch() const = 0;
  bool fused_variant() const { return variant == 1 || variant == 3 || variant == 4; }
  virtual int step(cudaStream_t s) = 0;
  virtual int sample(cudaStream_t s) = 0;
  virtual int update_h(cudaStream_t s) = 0;
  virtual int update_e(cudaStream_t s) = 0;
  virtual int64_t launches_per_chunk() const = 0;
  virtual int decide() = 0;
  virtual bool uses_tma() const = 0;
  // the run descriptor of a batched Bloch sweep (BlochRun<F>), run to step `last`
  virtual size_t bloch_desc_bytes() const = 0;
  virtual int bloch_desc(void* out, size_t bytes, int64_t last) = 0;
  // the coefficients of the adjoint (YeeArgs of a real engine) and the current H array
  virtual int adjoint_args(void* yee, size_t bytes, void** H) = 0;
  // the dispersive groups (AdeArgs of a real engine), for the adjoint
  virtual int adjoint_n_groups() const = 0;
  // the conformal off-diagonal terms (rows, entries per row), for the adjoint
  virtual void adjoint_offdiag(long long* rows, int* width) const = 0;
  // the vertex-tensor mesh (TensorArgs of a real engine; nN = 0 without one), for the adjoint
  virtual int adjoint_tensor(void* out, size_t bytes) const = 0;
  virtual int adjoint_group(int gi, void* out, size_t bytes) = 0;
};

namespace {

constexpr size_t kStatusBytes = 256;

enum SrcKind { kTable, kDipole, kLine, kColumn, kMode };

template <typename F>
struct Engine final : lsfdtd_engine {
  using R = typename real_of<F>::type;
  static constexpr bool kComplex = is_cplx<F>::value;

  YeeArgs<F> y{};
  double bloch_re[3][2]{}, bloch_im[3][2]{};  // [axis][low/high ghost]
  std::vector<AdeArgs<F>> groups;
  struct Table {
    TableArgs<R> corr[2];
    bool has[2];
    long long n_entries[2];
    // the H corrections' slab boxes for the fused pass (hc.n = 0: not given), the CSR position of each
    // slab-order entry and the step's values in slab order
    HCorr hc;
    const long long* hperm;
    R* hvals;
    const R* Tinc;
    const long long *inc_base, *inc_i0;
    const R* inc_u0;
    R* view;
  };
  struct Dipole {
    const long long* idx;
    const R* coef;
    const R* wave;
    int n;
  };
  struct Line {
    LineArgs<R> corr[2];
    bool has[2];
    R *E, *H;
    const R *ca, *cb, *da, *db, *wave;
    int M, m_src;
  };
  struct Column {
    lsfdtd_engine* col;
    int k_src, k_launch;
    const F* phase;
    F amp0, amp1;
    const R* wave;
    R cE, cH;
  };
  struct Mode {
    lsfdtd_mode_source_desc d;
  };
  struct Monitor {
    int space;
    MonArgs<F> af;
    MonArgs<R> ar;
    long long blocks;
    int energy;
  };
  std::vector<std::pair<SrcKind, size_t>> order;
  std::vector<Table> tables;
  std::vector<Dipole> dipoles;
  std::vector<Line> lines;
  std::vector<Column> columns;
  std::vector<Mode> modes;
  std::vector<Monitor> monitors;
  long long e_first[2] = {0, 0}, e_count[2] = {0, 0};

  explicit Engine(const lsfdtd_grid_desc& g) {
    desc = g;
    const long long cells = (long long)g.shape[0] * g.shape[1] * g.shape[2];
    for (int a = 0; a < 3; ++a) {
      y.n[a] = g.shape[a];
      y.periodic[a] = g.periodic[a];
      y.mirror[a] = g.mirror[a];
      y.inv_d[a] = R(1.0 / g.spacing[a]);
      y.E[a] = static_cast<F*>(g.E) + a * cells;
      y.H[a] = static_cast<F*>(g.H) + a * cells;
      y.cbE[a] = static_cast<const R*>(g.cbE[a]);
      y.pml[a].on = 0;
      // Bloch ghost phases e^{-+i k L}, L = (n - 2) d (engine.py:606-609)
      const double kl = g.bloch[a] * (g.shape[a] - 2) * g.spacing[a];
      bloch_re[a][0] = std::cos(-kl);
      bloch_im[a][0] = std::sin(-kl);
      bloch_re[a][1] = std::cos(kl);
      bloch_im[a][1] = std::sin(kl);
    }
    Ebuf[0] = static_cast<F*>(g.E);
    Hbuf[0] = static_cast<F*>(g.H);
    Ebuf[1] = static_cast<F*>(g.E_alt);
    Hbuf[1] = static_cast<F*>(g.H_alt);
    y.uniform = (g.spacing[0] == g.spacing[1] && g.spacing[1] == g.spacing[2]) ? 1 : 0;
    y.cH = R(y.uniform ? g.dt / g.spacing[0] : g.dt);
  }

  F* Ebuf[2] = {nullptr, nullptr};
  F* Hbuf[2] = {nullptr, nullptr};
  F* psiH[2][3][3][2] = {};  // H psi slabs per [buffer][axis][component][side]
  int pml_cells[3][2] = {};
  bool attr_set[2] = {false, false};
  bool tma_ok = false;
  int maps_tile_y = 0;  // tile rows the tensor-map boxes were made for
  CUtensorMap mapE[2][3], mapH[2][3], mapC;  // per buffer and component; the coefficient of component 0
  static constexpr int kStages = 4;  // x planes in the fused pass's copy ring
  // the lean pass's boundary classes run on streams of their own, one per class, beside the clean
  // interior's and each other (fork and join events on the caller's stream; made with the engine)
  static constexpr int kSides = 4;
  cudaStream_t side[kSides] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[kSides] = {};
  int init_side() override {
    if constexpr (!kComplex) {
      for (int i = 0; i < kSides; ++i) {
        LS_CUDA(cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking));
        LS_CUDA(cudaEventCreateWithFlags(&ev_join[i], cudaEventDisableTiming));
      }
      LS_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    }
    return LSFDTD_OK;
  }
  ~Engine() override {
    for (int i = 0; i < kSides; ++i) {
      if (side[i]) cudaStreamDestroy(side[i]);
      if (ev_join[i]) cudaEventDestroy(ev_join[i]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
  }

  F* Eflat() const { return Ebuf[cur]; }
  F* Hflat() const { return Hbuf[cur]; }

  // the fused single pass needs the second buffers, no periodic axis and sources that only correct E, or
  // table-fed TF/SF sources whose H corrections the lean pass applies as it steps (one at most, boxes given)
  int decide() override {
    if (fused >= 0) return fused;
    fused = 0;
    if (kComplex || !Ebuf[1] || !Hbuf[1]) return 0;  // Bloch fields come with periodic axes
    for (int a = 0; a < 3; ++a)
      if (desc.periodic[a] || desc.mirror[a]) return 0;  // the fused pass's region tests know neither
    int h_tables = 0;
    for (auto& o : order) {
      if (o.first == kTable) {
        const Table& t = tables[o.second];
        if (!t.has[1]) continue;
        if (t.hc.n == 0 || variant != 4 || ++h_tables > 1) return 0;
        continue;
      }
      if (o.first != kDipole) return 0;
    }
    for (int d = 0; d < 3; ++d) {
      if (!y.pml[d].on) continue;
      for (int c = 0; c < 3; ++c)
        for (int sd = 0; sd < 2; ++sd)
          if (y.pml[d].len[1][c][sd] > 0 && !psiH[1][d][c][sd]) return 0;
    }
    tma_ok = use_tma && make_maps() == LSFDTD_OK;
    // rows the tensor copies cannot take (not a multiple of 16 bytes): both fused passes then fill their rings
    // with cp.async copies, which run slower than the in-place kernels (measured on B200, CPML 12: the generic
    // pass 607 against 296 us per step at 214^3, 226 against 74 us at 129^3; the lean pass 224 against 73 us
    // on the 129^3 sphere, issue-bound on its copies), so the default steps in place there; an explicit kernel
    // choice keeps the fused pass
    if (use_tma && !tma_ok && !tuned) return 0;
    fused = 1;
    return 1;
  }

  // 3D tensor maps (z fastest) of the field buffers and the coefficient, boxes as k_fused_tma copies them
  bool uses_tma() const override { return tma_ok; }

  template <int TY, int S, bool BOX>
  int launch_tma_box(dim3 grid, const TmaArgs<F>& ta, cudaStream_t s) {
    if constexpr (!kComplex) {
      constexpr size_t sm = fused_tma_smem_bytes<F, TY, S>();
      static bool attr = false;  // per instantiation: the attribute belongs to the kernel, not the engine
      if (!attr) {
        LS_CUDA(cudaFuncSetAttribute(k_fused_tma<F, TY, S, BOX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
        attr = true;
      }
      k_fused_tma<F, TY, S, BOX><<<grid, dim3(32, TY), sm, s>>>(ta);
    }
    return LSFDTD_OK;
  }
  template <int TY, int S, bool UNI, bool ASYNC, bool HC, bool CLEAN = false, int AX = 7>
  int launch_pml_one(dim3 grid, const TmaArgs<F>& ta, cudaStream_t s) {
    if constexpr (!kComplex) {
      // the clean interior pass reads no slab tables
      constexpr size_t sm = CLEAN ? fused_tma_smem_bytes<F, TY, S>() : fused_pml_smem_bytes<F, TY, S>();
      static bool attr = false;  // per instantiation: the attribute belongs to the kernel, not the engine
      if (!attr) {
        LS_CUDA(cudaFuncSetAttribute(k_fused_pml<F, TY, S, UNI, ASYNC, HC, CLEAN, AX>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        attr = true;
      }
      k_fused_pml<F, TY, S, UNI, ASYNC, HC, CLEAN, AX><<<grid, dim3(32, TY), sm, s>>>(ta);
    }
    return LSFDTD_OK;
  }
  // the lean-CPML pass, one instantiation per cell shape (cubic or not), copy engine (cp.async: rows the
  // tensor copies cannot stride) and whether a table-fed source's H corrections are added as it steps (those
  // two with a ring of 4 only)
  template <int TY, int S, bool ASYNC, bool HC, bool CLEAN = false, int AX = 7>
  int launch_pml_kind(dim3 grid, const TmaArgs<F>& ta, cudaStream_t s) {
    return y.uniform ? launch_pml_one<TY, S, true, ASYNC, HC, CLEAN, AX>(grid, ta, s)
                     : launch_pml_one<TY, S, false, ASYNC, HC, CLEAN, AX>(grid, ta, s);
  }
  // the kernels of the split lean pass (tile rows 8, ring of 4), per class of CTA box: 0 the clean interior,
  // 1, 2, 3 the boxes that meet slabs or walls along x, y, z only, 4 the edges and corners (any axis)
  static constexpr int kClasses = 5;
  int launch_class(int cls, dim3 g, const TmaArgs<F>& ta, cudaStream_t st) {
    switch (cls) {
      case 0: return launch_pml_kind<8, 4, false, false, true, 0>(g, ta, st);
      case 1: return launch_pml_kind<8, 4, false, false, false, 1>(g, ta, st);
      case 2: return launch_pml_kind<8, 4, false, false, false, 2>(g, ta, st);
      case 3: return launch_pml_kind<8, 4, false, false, false, 4>(g, ta, st);
      default: return launch_pml_kind<8, 4, false, false, false, 7>(g, ta, st);
    }
  }
  template <int TY, int S>
  int launch_pml(dim3 grid, const TmaArgs<F>& ta, cudaStream_t s) {
    if (ta.f.hc.n > 0) return launch_pml_kind<TY, 4, false, true>(grid, ta, s);
    return launch_pml_kind<TY, S, false, false>(grid, ta, s);
  }
  template <int TY>
  int launch_pml_async(dim3 grid, const TmaArgs<F>& ta, cudaStream_t s) {
    return ta.f.hc.n > 0 ? launch_pml_kind<TY, 4, true, true>(grid, ta, s)
                         : launch_pml_kind<TY, 4, true, false>(grid, ta, s);
  }
  // kind 0: the fused pass over the grid, 1: over the interior box of the split step, 2: with lean CPML terms
  template <int TY, int S>
  int launch_tma(dim3 grid, const TmaArgs<F>& ta, cudaStream_t s, int kind) {
    if (kind == 2) return launch_pml<TY, S>(grid, ta, s);
    return kind == 1 ? launch_tma_box<TY, S, true>(grid, ta, s) : launch_tma_box<TY, S, false>(grid, ta, s);
  }
  template <int TY, int S>
  static constexpr size_t tma_smem(int kind) {
    return kind == 2 ? fused_pml_smem_bytes<F, TY, S>() : fused_tma_smem_bytes<F, TY, S>();
  }

  // the lean-CPML pass needs its copies by the Tensor Memory Accelerator and, per axis, CPML slabs that do
  // not overlap
  bool lean_ok() const {
    if (variant != 4 || kComplex) return false;
    for (int d = 0; d < 3; ++d) {
      if (!y.pml[d].on) continue;
      // its psi slabs indexed in 32-bit arithmetic: fewer than 2^31 nodes each
      const long long face = (long long)desc.shape[(d + 1) % 3] * desc.shape[(d + 2) % 3];
      for (int f = 0; f < 2; ++f)
        for (int c = 0; c < 3; ++c)
          for (int sd = 0; sd < 2; ++sd)
            if ((long long)y.pml[d].len[f][c][sd] * face >= (1LL << 31)) return false;
      for (int f = 0; f < 2; ++f) {
        const int c = (d + 1) % 3;
        const int lo_end = y.pml[d].start[f][c][0] + y.pml[d].len[f][c][0];
        if (y.pml[d].len[f][c][0] > 0 && y.pml[d].len[f][c][1] > 0 && lo_end > y.pml[d].start[f][c][1]) return false;
      }
    }
    return true;
  }

  // the clean interior of the lean pass: z tiles [zc0, zc1), y tiles [yc0, yc1) (of `rows`), x planes [xc0, xc1)
  void clean_box(int rows, int* zc0, int* zc1, int* yc0, int* yc1, int* xc0, int* xc1) const {
    int lo[3], hi[3];
    inner_bounds(lo, hi);
    *zc0 = (lo[2] + 1 + 31) / 32;
    *zc1 = hi[2] >= 32 ? (hi[2] - 32) / 32 + 1 : 0;
    *yc0 = (lo[1] + 1 + rows - 1) / rows;
    *yc1 = hi[1] >= rows ? (hi[1] - rows) / rows + 1 : 0;
    *xc0 = lo[0] + 1;
    *xc1 = hi[0];
  }
  // whether the lean pass runs as two kernels (clean interior and the rest)
  bool lean_split() const {
    if (kComplex || !tma_ok || !split_clean || !side[kSides - 1] || !lean_ok() || tile_y != 8 || stages != 4)
      return false;
    for (auto& tb : tables)
      if (tb.has[1] && tb.hc.n > 0) return false;
    int zc0, zc1, yc0, yc1, xc0, xc1;
    clean_box(tile_y == 16 ? 16 : 8, &zc0, &zc1, &yc0, &yc1, &xc0, &xc1);
    return zc1 > zc0 && yc1 > yc0 && xc1 > xc0;
  }

  // a box of z tiles [tz0, tz1), y tiles [ty0, ty1) and x planes [x0, x1) in segments of at most seg planes
  // (evened out), appended to m with its CTAs counted in total; nothing for an empty box
  static void add_cta_box(CtaMap& m, long long& total, int tz0, int tz1, int ty0, int ty1, int x0, int x1,
                          int seg) {
    if (tz1 <= tz0 || ty1 <= ty0 || x1 <= x0) return;
    const int len = x1 - x0, nseg = (len + seg - 1) / seg, sg = (len + nseg - 1) / nseg;
    CtaBox& b = m.box[m.n++];
    b.t0[0] = tz0;
    b.t1[0] = tz1;
    b.t0[1] = ty0;
    b.t1[1] = ty1;
    b.x0 = x0;
    b.x1 = x1;
    b.seg = sg;
    b.first = (int)total;
    total += (long long)(tz1 - tz0) * (ty1 - ty0) * ((len + sg - 1) / sg);
  }

  // the lean pass's CTAs (tiles of 32 z nodes by `rows` y nodes, segments of seg x planes) per class (see
  // launch_class): with may_split and a clean interior of whole tiles, that interior in maps[0], the boxes
  // beside it that are inner along all axes but x, y or z in maps[1], [2], [3], and the edges and corners in
  // maps[4] (true); else every CTA in maps[4]. A clean CTA's nodes and halo nodes (row y0 - 1, column z0 - 1)
  // and its x planes, the plane before its segment included, are inner on every axis
  bool lean_plan(int rows, int seg, bool may_split, CtaMap* maps, long long* n) const {
    const int n0 = desc.shape[0], nz = (desc.shape[2] + 31) / 32, ny = (desc.shape[1] + rows - 1) / rows;
    for (int c = 0; c < kClasses; ++c) {
      maps[c].n = 0;
      n[c] = 0;
    }
    int zc0, zc1, yc0, yc1, xc0, xc1;
    clean_box(rows, &zc0, &zc1, &yc0, &yc1, &xc0, &xc1);
    if (!may_split || zc1 <= zc0 || yc1 <= yc0 || xc1 <= xc0) {
      add_cta_box(maps[4], n[4], 0, nz, 0, ny, 0, n0, seg);
      return false;
    }
    const int xr[2][2] = {{0, xc0}, {xc1, n0}}, yr[2][2] = {{0, yc0}, {yc1, ny}}, zr[2][2] = {{0, zc0}, {zc1, nz}};
    add_cta_box(maps[0], n[0], zc0, zc1, yc0, yc1, xc0, xc1, seg);
    for (int s = 0; s < 2; ++s) {
      add_cta_box(maps[1], n[1], zc0, zc1, yc0, yc1, xr[s][0], xr[s][1], seg);
      add_cta_box(maps[2], n[2], zc0, zc1, yr[s][0], yr[s][1], xc0, xc1, seg);
      add_cta_box(maps[3], n[3], zr[s][0], zr[s][1], yc0, yc1, xc0, xc1, seg);
    }
    for (int s = 0; s < 2; ++s)
      for (int t = 0; t < 2; ++t) {
        add_cta_box(maps[4], n[4], 0, nz, yr[t][0], yr[t][1], xr[s][0], xr[s][1], seg);
        add_cta_box(maps[4], n[4], zr[t][0], zr[t][1], yc0, yc1, xr[s][0], xr[s][1], seg);
        add_cta_box(maps[4], n[4], zr[t][0], zr[t][1], yr[s][0], yr[s][1], xc0, xc1, seg);
      }
    return true;
  }
  // launches of the lean pass per step
  int lean_launches() const {
    CtaMap maps[kClasses];
    long long n[kClasses];
    if (!lean_plan(8, 32, lean_split(), maps, n)) return 1;
    int k = 0;
    for (int c = 0; c < kClasses; ++c) k += n[c] > 0;
    return k;
  }

  // nodes [lo, hi) per axis stepped for every component and outside every CPML slab
  void inner_bounds(int* lo_out, int* hi_out) const {
    for (int ax = 0; ax < 3; ++ax) {
      int lo = 1, hi = desc.shape[ax] - 1;
      if (y.pml[ax].on) {
        lo = std::max(lo, pml_cells[ax][0] ? pml_cells[ax][0] + 1 : 1);
        hi = std::min(hi, pml_cells[ax][1] ? desc.shape[ax] - 2 - pml_cells[ax][1] : hi);
      }
      lo_out[ax] = lo;
      hi_out[ax] = std::max(lo, hi);
    }
  }

  // the interior box of the split step and its shell; false when the split does not apply (no TMA copies,
  // an empty box, or a shell of 2^32 nodes or more)
  bool split_box(int* lo, int* hi, ShellBoxes* sb) const {
    if (variant != 3 || !tma_ok) return false;
    int ilo[3], ihi[3];
    inner_bounds(ilo, ihi);
    for (int ax = 0; ax < 3; ++ax) {
      lo[ax] = ilo[ax] + 1;  // the low-side halo node of the box is inner too
      hi[ax] = ihi[ax];
    }
    lo[2] = (lo[2] + 3) / 4 * 4;  // tensor-copy boxes start at z0 - 4 on a 16-byte boundary
    for (int ax = 0; ax < 3; ++ax)
      if (hi[ax] <= lo[ax]) return false;
    *sb = shell_boxes(desc.shape, lo, hi);
    return sb->total > 0 && sb->total < (1ull << 32);
  }

  int make_maps() {
    const size_t es = sizeof(F);
    if ((desc.shape[2] * es) % 16 != 0) return LSFDTD_EUNSUPPORTED;
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
      cudaDriverEntryPointQueryResult q;
      void* fn = nullptr;
      if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
          q != cudaDriverEntryPointSuccess || !fn)
        return LSFDTD_EUNSUPPORTED;
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const CUtensorMapDataType dt = sizeof(R) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const long long cells = (long long)desc.shape[0] * desc.shape[1] * desc.shape[2];
    auto make = [&](CUtensorMap* m, const void* base, unsigned bz, unsigned by) -> bool {
      if (reinterpret_cast<uintptr_t>(base) % 16) return false;
      cuuint64_t dims[3] = {(cuuint64_t)desc.shape[2], (cuuint64_t)desc.shape[1], (cuuint64_t)desc.shape[0]};
      cuuint64_t strides[2] = {(cuuint64_t)desc.shape[2] * es, (cuuint64_t)desc.shape[1] * desc.shape[2] * es};
      cuuint32_t box[3] = {bz, by, 1};
      cuuint32_t estr[3] = {1, 1, 1};
      return encode(m, dt, 3, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    const unsigned ty = (unsigned)tile_y;
    maps_tile_y = tile_y;
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 3; ++c) {
        if (!make(&mapE[b][c], Ebuf[b] + c * cells, 40, ty + 2)) return LSFDTD_EUNSUPPORTED;
        if (!make(&mapH[b][c], Hbuf[b] + c * cells, 40, ty + 1)) return LSFDTD_EUNSUPPORTED;
      }
    if (!make(&mapC, y.cbE[0], 32, ty)) return LSFDTD_EUNSUPPORTED;
    return LSFDTD_OK;
  }

  // x planes per CTA of the fused pass when none is requested: `most`, or fewer where that would give fewer
  // than about three waves of CTAs (resident CTAs per SM as the kernels' launch bounds ask). A small grid
  // steps faster in more, shorter CTAs: measured on B200, a 200 x 200 x 120 grid with 12-cell CPML took 157 us
  // per step at 12 planes and 199 us at 34.
  int auto_planes(int nx, long long columns, int rows, int* seg, int most = 48, int waves = 3) {
    if (sm_count <= 0) {
      int dev = 0;
      LS_CUDA(cudaGetDevice(&dev));
      LS_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev));
    }
    const long long per_sm = sizeof(R) == 4 ? (rows == 8 ? 4 : 2) : 1;
    const long long p = (long long)nx * columns / (waves * per_sm * std::max(sm_count, 1));
    *seg = (int)std::max(4LL, std::min((long long)most, p));
    return LSFDTD_OK;
  }

  int fused_step(cudaStream_t s) {
    const long long cells = (long long)desc.shape[0] * desc.shape[1] * desc.shape[2];
    FusedArgs<F> fa;
    fa.y = y;
    fa.hc.n = 0;
    fa.hc.vals = nullptr;
    for (auto& tb : tables) {  // a table-fed source's H corrections for this step, added by the lean pass
      if (!tb.has[1] || tb.hc.n == 0) continue;
      k_table_values<R><<<cdiv(tb.n_entries[1], 256), 256, 0, s>>>(tb.corr[1], tb.hperm, tb.n_entries[1], tb.hvals);
      LS_LAUNCHED();
      fa.hc = tb.hc;
    }
    const int o = cur ^ 1;
    for (int a = 0; a < 3; ++a) {
      fa.y.E[a] = Ebuf[cur] + a * cells;
      fa.y.H[a] = Hbuf[cur] + a * cells;
      fa.Eo[a] = Ebuf[o] + a * cells;
      fa.Ho[a] = Hbuf[o] + a * cells;
    }
    for (int d = 0; d < 3; ++d)
      for (int c = 0; c < 3; ++c)
        for (int sd = 0; sd < 2; ++sd) {
          fa.y.pml[d].psi[1][c][sd] = psiH[cur][d][c][sd];
          fa.psiHo[d][c][sd] = psiH[o][d][c][sd];
        }
    inner_bounds(fa.inner_lo, fa.inner_hi);
    for (int ax = 0; ax < 3; ++ax) {
      fa.pml_lo[ax] = y.pml[ax].on ? pml_cells[ax][0] : 0;
      fa.pml_hi[ax] = y.pml[ax].on ? pml_cells[ax][1] : 0;
      fa.box_lo[ax] = 0;
      fa.box_hi[ax] = desc.shape[ax];
    }
    if constexpr (!kComplex) {
      if (tma_ok && maps_tile_y != tile_y) tma_ok = make_maps() == LSFDTD_OK;
    }
    ShellBoxes sb{};
    const bool split = split_box(fa.box_lo, fa.box_hi, &sb);
    const int kind = split ? 1 : (lean_ok() ? 2 : 0);
    const int rows = tile_y == 16 ? 16 : 8;
    dim3 grid = split ? dim3(cdiv(fa.box_hi[2] - fa.box_lo[2], 32), cdiv(fa.box_hi[1] - fa.box_lo[1], rows), 1)
                      : dim3(cdiv(desc.shape[2], 32), cdiv(desc.shape[1], rows), 1);
    const int nx = split ? fa.box_hi[0] - fa.box_lo[0] : desc.shape[0];
    fa.seg = planes;
    // the lean pass split by class of box balances its classes better in shorter segments, at least about
    // twelve waves of CTAs (measured on B200: 640^3 at 32 planes 3.32 ms per step, at 48 3.52; 256^3 at 8
    // planes 0.317 ms, at 32 0.421); the lean kernel alone is fastest at 48 planes and three waves
    if (fa.seg <= 0) {
      const bool two = lean_split();
      LS_TRY(auto_planes(nx, (long long)grid.x * grid.y, rows, &fa.seg, two ? 32 : 48, two ? 12 : 3));
    }
    grid.z = (unsigned)cdiv(nx, fa.seg);
    LS_TRY(mark(s, true));
    if constexpr (!kComplex) {
      // the fused passes by tensor copies, with the deepest ring up to the requested depth that fits the
      // device's shared memory per CTA
      auto launch_ring = [&](const TmaArgs<F>& ta, dim3 g, cudaStream_t st) -> int {
        int smax = 0, dev = 0;
        LS_CUDA(cudaGetDevice(&dev));
        LS_CUDA(cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        auto fits = [&](size_t b) { return b <= (size_t)smax; };
        if (tile_y == 16) {
          if (stages >= 8 && fits(tma_smem<16, 8>(kind))) return launch_tma<16, 8>(g, ta, st, kind);
          if (stages >= 6 && fits(tma_smem<16, 6>(kind))) return launch_tma<16, 6>(g, ta, st, kind);
          return launch_tma<16, 4>(g, ta, st, kind);
        }
        if (stages >= 8 && fits(tma_smem<8, 8>(kind))) return launch_tma<8, 8>(g, ta, st, kind);
        if (stages >= 6 && fits(tma_smem<8, 6>(kind))) return launch_tma<8, 6>(g, ta, st, kind);
        return launch_tma<8, 4>(g, ta, st, kind);
      };
      TmaArgs<F> ta;
      ta.f = fa;
      ta.status = static_cast<int*>(scratch);
      ta.wait_budget = wait_budget;
      if (tma_ok) {
        for (int c = 0; c < 3; ++c) {
          ta.mE[c] = mapE[cur][c];
          ta.mH[c] = mapH[cur][c];
        }
        ta.mC = mapC;
      }
      if (kind == 2) {
        // the lean pass: where the grid has a clean interior, one kernel per class of CTA box (launch_class),
        // the interior's on the caller's stream and each other class on a side stream of its own, all at once;
        // else every CTA by the lean kernel
        CtaMap maps[kClasses];
        long long n[kClasses];
        const bool two = lean_plan(rows, fa.seg, lean_split(), maps, n);
        if (!two) {
          ta.map = maps[4];
          const dim3 g((unsigned)n[4]);
          const int r = tma_ok ? launch_ring(ta, g, s)
                               : (tile_y == 16 ? launch_pml_async<16>(g, ta, s) : launch_pml_async<8>(g, ta, s));
          if (r != LSFDTD_OK) return r;
        } else {
          LS_CUDA(cudaEventRecord(ev_fork, s));
          for (int c = kClasses - 1; c >= 1; --c) {  // class c on side stream c - 1
            if (n[c] == 0) continue;
            LS_CUDA(cudaStreamWaitEvent(side[c - 1], ev_fork, 0));
            ta.map = maps[c];
            LS_TRY(launch_class(c, dim3((unsigned)n[c]), ta, side[c - 1]));
            LS_LAUNCHED();
            LS_CUDA(cudaEventRecord(ev_join[c - 1], side[c - 1]));
          }
          ta.map = maps[0];
          LS_TRY(launch_class(0, dim3((unsigned)n[0]), ta, s));
          LS_LAUNCHED();
          for (int c = 1; c < kClasses; ++c)
            if (n[c] > 0) LS_CUDA(cudaStreamWaitEvent(s, ev_join[c - 1], 0));
        }
      } else if (tma_ok) {
        LS_TRY(launch_ring(ta, grid, s));
        if (split) {
          LS_LAUNCHED();
          const unsigned blocks = (unsigned)cdiv((long long)sb.total, 256);
          k_shell_h<F><<<blocks, 256, 0, s>>>(fa, sb);
          LS_LAUNCHED();
          k_shell_e<F><<<blocks, 256, 0, s>>>(fa, sb);
        }
      } else if (tile_y == 16) {
        constexpr size_t sm = fused_smem_bytes<F, 16, kStages>();  // cp.async ring
        if (!attr_set[1]) {
          LS_CUDA(cudaFuncSetAttribute(k_fused_step<F, 16, kStages>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sm));
          attr_set[1] = true;
        }
        k_fused_step<F, 16, kStages><<<grid, dim3(32, 16), sm, s>>>(fa);
      } else {
        constexpr size_t sm = fused_smem_bytes<F, 8, kStages>();
        if (!attr_set[0]) {
          LS_CUDA(cudaFuncSetAttribute(k_fused_step<F, 8, kStages>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sm));
          attr_set[0] = true;
        }
        k_fused_step<F, 8, kStages><<<grid, dim3(32, 8), sm, s>>>(fa);
      }
    }
    LS_LAUNCHED();
    LS_TRY(mark(s, false));
    cur = o;
    return LSFDTD_OK;
  }

  size_t bloch_desc_bytes() const override { return kComplex ? sizeof(BlochRun<F>) : 0; }

  int adjoint_n_groups() const override { return (int)groups.size(); }
  int adjoint_group(int gi, void* out, size_t bytes) override {
    if (gi < 0 || gi >= (int)groups.size() || bytes != sizeof(AdeArgs<F>)) return fail(LSFDTD_EINVAL, "adjoint: group");
    AdeArgs<F> ga = groups[gi];
    ga.E = Eflat();
    std::memcpy(out, &ga, sizeof ga);
    return LSFDTD_OK;
  }

  int adjoint_args(void* yee, size_t bytes, void** H) override {
    if (kComplex) return fail(LSFDTD_EUNSUPPORTED, "adjoint: real fields only");
    if (bytes != sizeof(YeeArgs<F>)) return fail(LSFDTD_EINVAL, "adjoint: argument size");
    const YeeArgs<F> a = current_args();
    std::memcpy(yee, &a, sizeof a);
    *H = Hflat();
    return LSFDTD_OK;
  }

  void adjoint_offdiag(long long* rows, int* width) const override {
    *rows = od_n;
    *width = od_width;
  }
  int adjoint_tensor(void* out, size_t bytes) const override {
    if (kComplex || bytes != sizeof(TensorArgs<F>)) return fail(LSFDTD_EINVAL, "adjoint: tensor argument size");
    TensorArgs<F> a = has_tensor ? tm : TensorArgs<F>{};
    std::memcpy(out, &a, sizeof a);
    return LSFDTD_OK;
  }

  int bloch_desc(void* out, size_t bytes, int64_t last) override {
    if constexpr (!kComplex) {
      (void)out;
      (void)bytes;
      (void)last;
      return fail(LSFDTD_EUNSUPPORTED, "a batched Bloch run needs complex fields");
    } else {
      if (bytes != sizeof(BlochRun<F>)) return fail(LSFDTD_EINVAL, "batch: descriptor size");
      if (!desc.periodic[0] || !desc.periodic[1] || desc.periodic[2])
        return fail(LSFDTD_EUNSUPPORTED, "batch: a run must be periodic along x and y, not z");
      if (desc.mirror[2]) return fail(LSFDTD_EUNSUPPORTED, "batch: no mirror plane");
      if (has_tensor) return fail(LSFDTD_EUNSUPPORTED, "batch: no vertex-tensor mesh");
      if (y.pml[0].on || y.pml[1].on) return fail(LSFDTD_EUNSUPPORTED, "batch: CPML along z only");
      if (!groups.empty()) return fail(LSFDTD_EUNSUPPORTED, "batch: dispersive groups have no batched path");
      if (order.size() != 1 || order[0].first != kColumn)
        return fail(LSFDTD_EUNSUPPORTED, "batch: a run needs exactly one Bloch column source");
      if (monitors.size() > (size_t)kBatchMaxMon) return fail(LSFDTD_EUNSUPPORTED, "batch: at most four monitors");
      for (auto& m : monitors)
        if (m.space == 1) return fail(LSFDTD_EUNSUPPORTED, "batch: monitors on the grid or the column only");
      if (last < n_host || last > step_limit)
        return fail(LSFDTD_ERANGE, "batch: the last step lies before the run's step or past its source waveform");
      const Column& c = columns[0];
      auto* col = static_cast<Engine<F>*>(c.col);
      if (col->desc.shape[2] != desc.shape[2] || col->y.pml[0].on || col->y.pml[1].on || !col->order.empty() ||
          !col->groups.empty())
        return fail(LSFDTD_EUNSUPPORTED, "batch: the column must match the grid along z with CPML along z only");
      if (c.k_src < 1 || c.k_src >= desc.shape[2] - 1 || c.k_launch < 0 || c.k_launch >= desc.shape[2])
        return fail(LSFDTD_EINVAL, "batch: source planes out of range");
      BlochRun<F> r{};
      r.g = y;
      r.col = col->y;
      for (int a = 0; a < 2; ++a)
        for (int sd = 0; sd < 2; ++sd) {
          r.gph[a][sd] = F{(R)bloch_re[a][sd], (R)bloch_im[a][sd]};
          r.cph[a][sd] = F{(R)col->bloch_re[a][sd], (R)col->bloch_im[a][sd]};
        }
      r.phase = c.phase;
      r.amp0 = c.amp0;
      r.amp1 = c.amp1;
      r.wave = c.wave;
      r.cE = c.cE;
      r.cH = c.cH;
      r.k_src = c.k_src;
      r.k_launch = c.k_launch;
      r.stride = desc.dft_stride;
      r.last = last;
      r.nstep = reinterpret_cast<long long*>(desc.step);
      r.status = static_cast<int*>(scratch);
      r.od_e = od_e;
      r.od_h = od_h;
      r.od_w = od_w;
      r.od_n = od_n;
      r.od_width = od_width;
      if (!r.status) return fail(LSFDTD_EINVAL, "batch: the engine's scratch (its status word) is not set");
      r.div_n2 = udiv_make((unsigned)desc.shape[2]);
      r.div_ny = udiv_make((unsigned)(desc.shape[1] - 2));
      r.n_mon = (int)monitors.size();
      for (size_t i = 0; i < monitors.size(); ++i) {
        MonArgs<F> m = monitors[i].af;
        if (monitors[i].space == 0) {
          m.Esrc = Eflat();
          m.Hsrc = Hflat();
        }
        m.want_energy = 0;
        m.partial = nullptr;
        r.mon[i] = m;
      }
      std::memcpy(out, &r, sizeof r);
      return LSFDTD_OK;
    }
  }

  int set_pml(const lsfdtd_pml_desc* p) override {
    const int d = p->axis;
    if (d < 0 || d > 2) return fail(LSFDTD_EINVAL, "pml axis out of range");
    if (desc.periodic[d]) return fail(LSFDTD_EINVAL, "a periodic axis cannot have a PML");
    if (desc.mirror[d] && p->cells_lo) return fail(LSFDTD_EINVAL, "a mirror axis cannot have a PML on its low side");
    PmlAxis<F>& q = y.pml[d];
    q.on = 1;
    pml_cells[d][0] = p->cells_lo;
    pml_cells[d][1] = p->cells_hi;
    q.div = y.uniform ? R(1) : R(desc.spacing[d]);
    for (int f = 0; f < 2; ++f) {
      q.b[f] = static_cast<const R*>(p->b[f]);
      q.c[f] = static_cast<const R*>(p->c[f]);
      q.k[f] = static_cast<const R*>(p->k[f]);
      if (!q.b[f] || !q.c[f]) return fail(LSFDTD_EINVAL, "pml profiles missing");
      for (int c = 0; c < 3; ++c)
        for (int s = 0; s < 2; ++s) {
          int st, ln;
          slab(desc.shape, desc.periodic, d, p->cells_lo, p->cells_hi, f, c, s, &st, &ln);
          q.start[f][c][s] = st;
          q.len[f][c][s] = ln;
          q.psi[f][c][s] = static_cast<F*>(p->psi[f][c][s]);
          if (ln > 0 && !q.psi[f][c][s]) return fail(LSFDTD_EINVAL, "pml psi slab missing");
          if (f == 1) {
            psiH[0][d][c][s] = q.psi[f][c][s];
            psiH[1][d][c][s] = static_cast<F*>(p->psi_alt[c][s]);
          }
        }
    }
    return LSFDTD_OK;
  }

  // conformal off-diagonal gather (at most one set)
  const long long* od_e = nullptr;
  const long long* od_h = nullptr;
  const F* od_w = nullptr;
  long long od_n = 0;
  int od_width = 0;
  int add_offdiag(const lsfdtd_offdiag_desc* d) override {
    if (od_n) return fail(LSFDTD_EINVAL, "offdiag: one set per engine");
    if (d->n < 0 || d->width < 1 || (d->n > 0 && (!d->e || !d->h || !d->w)))
      return fail(LSFDTD_EINVAL, "offdiag: arrays missing or sizes out of range");
    // index ranges checked here, once (the kernel trusts them)
    const long long flat = 3LL * desc.shape[0] * desc.shape[1] * desc.shape[2];
    std::vector<long long> he(d->n), hh(d->n * (long long)d->width);
    if (d->n > 0) {
      LS_CUDA(cudaMemcpy(he.data(), d->e, he.size() * sizeof(long long), cudaMemcpyDeviceToHost));
      LS_CUDA(cudaMemcpy(hh.data(), d->h, hh.size() * sizeof(long long), cudaMemcpyDeviceToHost));
    }
    for (long long v : he)
      if (v < 0 || v >= flat) return fail(LSFDTD_ERANGE, "offdiag: an E index out of range");
    for (long long v : hh)
      if (v < 0 || v >= flat) return fail(LSFDTD_ERANGE, "offdiag: an H index out of range");
    od_e = reinterpret_cast<const long long*>(d->e);
    od_h = reinterpret_cast<const long long*>(d->h);
    od_w = static_cast<const F*>(d->w);
    od_n = d->n;
    od_width = d->width;
    return LSFDTD_OK;
  }
  int offdiag(cudaStream_t s) {
    if (od_n <= 0) return LSFDTD_OK;
    k_offdiag<F><<<cdiv(od_n, 256), 256, 0, s>>>(od_e, od_h, od_w, od_n, od_width, Eflat(), Hflat());
    LS_LAUNCHED();
    return LSFDTD_OK;
  }

  // the vertex-tensor mesh (at most one)
  bool has_tensor = false;
  TensorArgs<F> tm{};
  int add_tensor(const lsfdtd_tensor_desc* d) override {
    if (has_tensor) return fail(LSFDTD_EINVAL, "tensor: one mesh per engine");
    if (d->n_media < 1 || d->n_media > kMaxMedia) return fail(LSFDTD_EINVAL, "tensor: media count out of range");
    if (d->n_nodes < 0 || d->n_vert < 0 || d->n_tslots < 0 || d->n_pslots < 0)
      return fail(LSFDTD_EINVAL, "tensor: sizes out of range");
    if (d->n_nodes > 0 && (!d->idx || !d->state)) return fail(LSFDTD_EINVAL, "tensor: arrays missing");
    if (d->n_vert > 0 && (!d->vn || !d->normal)) return fail(LSFDTD_EINVAL, "tensor: vertex arrays missing");
    if (d->n_tslots > 0 && (!d->t_pos || !d->t_v || !d->t_vc || !d->t_g || !d->t_nc || !d->frac))
      return fail(LSFDTD_EINVAL, "tensor: slot arrays missing");
    if (d->n_pslots > 0 && (!d->p_pos || !d->p_node || !d->p_medium))
      return fail(LSFDTD_EINVAL, "tensor: plain slot arrays missing");
    if (kComplex && d->n_tslots > 0 && !d->t_conj) return fail(LSFDTD_EINVAL, "tensor: complex fields need t_conj");
    // index ranges, once (the kernels trust them)
    const long long flat = 3LL * desc.shape[0] * desc.shape[1] * desc.shape[2];
    auto check = [&](const int64_t* a, long long n, long long hi, const char* what) -> int {
      if (n <= 0) return LSFDTD_OK;
      std::vector<long long> h(n);
      LS_CUDA(cudaMemcpy(h.data(), a, n * sizeof(long long), cudaMemcpyDeviceToHost));
      for (long long v : h)
        if (v < 0 || v >= hi) return fail(LSFDTD_ERANGE, std::string("tensor: an index out of range: ") + what);
      return LSFDTD_OK;
    };
    LS_TRY(check(d->idx, d->n_nodes, flat, "idx"));
    LS_TRY(check(d->vn, 6 * d->n_vert, d->n_nodes, "vn"));
    LS_TRY(check(d->t_pos, d->n_tslots, 2 * d->n_nodes, "t_pos"));
    LS_TRY(check(d->t_v, d->n_tslots, d->n_vert, "t_v"));
    LS_TRY(check(d->t_vc, d->n_tslots, 3 * d->n_vert, "t_vc"));
    LS_TRY(check(d->t_g, d->n_tslots, 6 * d->n_vert, "t_g"));
    LS_TRY(check(d->p_pos, d->n_pslots, 2 * d->n_nodes, "p_pos"));
    LS_TRY(check(d->p_node, d->n_pslots, d->n_nodes, "p_node"));
    LS_TRY(check(d->p_medium, d->n_pslots, d->n_media, "p_medium"));
    TensorArgs<F> a{};
    a.idx = reinterpret_cast<const long long*>(d->idx);
    a.nN = d->n_nodes;
    a.nV = d->n_vert;
    a.nT = d->n_tslots;
    a.nP = d->n_pslots;
    a.vn = reinterpret_cast<const long long*>(d->vn);
    a.scale = static_cast<const F*>(d->scale);
    a.normal = static_cast<const R*>(d->normal);
    a.t_pos = reinterpret_cast<const long long*>(d->t_pos);
    a.t_v = reinterpret_cast<const long long*>(d->t_v);
    a.t_vc = reinterpret_cast<const long long*>(d->t_vc);
    a.t_g = reinterpret_cast<const long long*>(d->t_g);
    a.t_nc = static_cast<const R*>(d->t_nc);
    a.t_conj = static_cast<const F*>(d->t_conj);
    a.frac = static_cast<const R*>(d->frac);
    a.p_pos = reinterpret_cast<const long long*>(d->p_pos);
    a.p_node = reinterpret_cast<const long long*>(d->p_node);
    a.p_medium = reinterpret_cast<const long long*>(d->p_medium);
    a.n_media = d->n_media;
    for (int s = 0; s < d->n_media; ++s) {
      if (d->n_poles[s] < 0 || d->n_poles[s] > kMaxPoles) return fail(LSFDTD_EINVAL, "tensor: pole count out of range");
      if (!(d->eps_inf[s] > 0)) return fail(LSFDTD_EINVAL, "tensor: eps_inf must be positive");
      a.n_poles[s] = d->n_poles[s];
      a.eps_inf[s] = R(d->eps_inf[s]);
      a.inv_inf[s] = R(1.0 / d->eps_inf[s]);
      for (int k = 0; k < d->n_poles[s]; ++k) {
        a.c1[s][k] = R(d->c1[s][k]);
        a.c2[s][k] = R(d->c2[s][k]);
        a.c3[s][k] = R(d->c3[s][k]);
      }
    }
    tm_bind_state(a, static_cast<F*>(d->state));  // the state buffer, in lsfdtd_tensor_state_len's order
    tm = a;
    has_tensor = a.nN > 0;
    return LSFDTD_OK;
  }
  int tensor_step(cudaStream_t s) {
    TensorArgs<F> a = tm;
    a.E = Eflat();
    k_tm_nodes_d<F><<<cdiv(a.nN, 256), 256, 0, s>>>(a);
    LS_LAUNCHED();
    if (a.nV > 0) {
      k_tm_vertices<F><<<cdiv(a.nV, 256), 256, 0, s>>>(a);
      LS_LAUNCHED();
    }
    if (a.nT > 0) {
      k_tm_slots<F><<<cdiv(a.nT, 256), 256, 0, s>>>(a);
      LS_LAUNCHED();
    }
    if (a.nP > 0) {
      k_tm_plain<F><<<cdiv(a.nP, 256), 256, 0, s>>>(a);
      LS_LAUNCHED();
    }
    k_tm_nodes_e<F><<<cdiv(a.nN, 256), 256, 0, s>>>(a);
    LS_LAUNCHED();
    return LSFDTD_OK;
  }

  int add_group(const lsfdtd_group_desc* g) override {
    if (g->n_media < 1 || g->n_media > kMaxMedia) return fail(LSFDTD_EINVAL, "group media count out of range");
    AdeArgs<F> a{};
    a.n = g->n;
    a.idx = reinterpret_cast<const long long*>(g->idx);
    a.E = nullptr;  // the current buffer, set at launch
    a.n_media = g->n_media;
    a.mixed = g->mixed;
    a.has_h = g->has_h;
    a.has_a = g->has_a;
    for (int s = 0; s < g->n_media; ++s) {
      if (g->n_poles[s] < 0 || g->n_poles[s] > kMaxPoles) return fail(LSFDTD_EINVAL, "pole count out of range");
      a.n_poles[s] = g->n_poles[s];
      a.inv_inf[s] = R(g->inv_eps_inf[s]);
      for (int k = 0; k < g->n_poles[s]; ++k) {
        a.c1[s][k] = R(g->c1[s][k]);
        a.c2[s][k] = R(g->c2[s][k]);
        a.c3[s][k] = R(g->c3[s][k]);
      }
    }
    a.h0 = static_cast<const R*>(g->h0);
    a.inv_a = static_cast<const R*>(g->inv_a);
    a.w = static_cast<const R*>(g->w);
    a.frac = static_cast<const R*>(g->frac);
    a.state = static_cast<F*>(g->state);
    if (g->mixed && (!a.w || !a.frac || (g->has_h && !a.h0) || (g->has_a && !a.inv_a)))
      return fail(LSFDTD_EINVAL, "mixed group arrays missing");
    if (a.n > 0 && (!a.idx || !a.state)) return fail(LSFDTD_EINVAL, "group arrays missing");
    groups.push_back(a);
    return LSFDTD_OK;
  }

  int add_table(const lsfdtd_table_source_desc* s) override {
    if (kComplex) return fail(LSFDTD_EUNSUPPORTED, "table-fed sources need real fields");
    if (s->m < 1) return fail(LSFDTD_EINVAL, "table stride m < 1");
    Table t{};
    for (int k = 0; k < 2; ++k) {
      TableArgs<R>& a = t.corr[k];
      t.has[k] = s->pts[k].n_nodes > 0;
      a.T = static_cast<const R*>(s->table);
      a.m = s->m;
      a.cmax = s->cmax;
      a.n_nodes = s->pts[k].n_nodes;
      a.nodes = reinterpret_cast<const long long*>(s->pts[k].nodes);
      a.offsets = reinterpret_cast<const long long*>(s->pts[k].offsets);
      a.base = reinterpret_cast<const long long*>(s->base[k]);
      a.i0 = reinterpret_cast<const long long*>(s->i0[k]);
      a.u0 = static_cast<const R*>(s->u0[k]);
      a.coef = static_cast<const R*>(s->coef[k]);
      a.target = nullptr;  // the current E (k = 0) or H buffer, set at launch
      a.nstep = reinterpret_cast<const long long*>(desc.step);
      t.n_entries[k] = t.has[k] ? s->pts[k].n_entries : 0;
    }
    t.hc.n = 0;
    t.hc.vals = nullptr;
    t.hperm = nullptr;
    t.hvals = nullptr;
    t.Tinc = static_cast<const R*>(s->inc_table);
    t.inc_base = reinterpret_cast<const long long*>(s->inc_base);
    t.inc_i0 = reinterpret_cast<const long long*>(s->inc_i0);
    t.inc_u0 = static_cast<const R*>(s->inc_u0);
    t.view = static_cast<R*>(s->view);
    order.push_back({kTable, tables.size()});
    tables.push_back(t);
    return LSFDTD_OK;
  }

  int set_table_boxes(int table, int n, const int32_t* boxes, const int64_t* perm, int64_t n_entries,
                      void* vals) override {
    if (kComplex) return fail(LSFDTD_EUNSUPPORTED, "table-fed sources need real fields");
    if (table < 0 || table >= (int)tables.size()) return fail(LSFDTD_EINVAL, "table boxes: no such table source");
    Table& t = tables[table];
    if (!t.has[1] || n_entries != t.n_entries[1])
      return fail(LSFDTD_EINVAL, "table boxes: the entry count differs from the source's H corrections");
    if (n < 1 || n > kMaxHBoxes || !boxes || !perm || !vals)
      return fail(LSFDTD_EINVAL, "table boxes: 1 to 24 boxes, a permutation and a value array");
    HCorr hc{};
    hc.n = n;
    long long total = 0;
    for (int b = 0; b < n; ++b) {
      const int32_t* q = boxes + 8 * b;
      HCorrBox& x = hc.box[b];
      x.c = q[0];
      long long vol = 1;
      for (int a = 0; a < 3; ++a) {
        x.lo[a] = q[1 + a];
        x.hi[a] = q[4 + a];
        if (x.lo[a] < 0 || x.hi[a] > desc.shape[a] || x.hi[a] <= x.lo[a])
          return fail(LSFDTD_ERANGE, "table boxes: a box outside the grid or empty");
        vol *= x.hi[a] - x.lo[a];
      }
      x.off = q[7];
      if (x.c < 0 || x.c > 2 || x.off < 0 || x.off + vol > n_entries)
        return fail(LSFDTD_ERANGE, "table boxes: a component or an entry offset out of range");
      total += vol;
    }
    if (total != n_entries) return fail(LSFDTD_EINVAL, "table boxes: the boxes do not cover the entries once");
    // the permutation indexes the CSR entries: checked once here, on the host
    std::vector<long long> h(n_entries);
    LS_CUDA(cudaMemcpy(h.data(), perm, n_entries * sizeof(long long), cudaMemcpyDeviceToHost));
    for (long long v : h)
      if (v < 0 || v >= n_entries) return fail(LSFDTD_ERANGE, "table boxes: a permutation entry out of range");
    hc.vals = vals;
    t.hc = hc;
    t.hperm = reinterpret_cast<const long long*>(perm);
    t.hvals = static_cast<R*>(vals);
    return LSFDTD_OK;
  }

  int add_dipole(const lsfdtd_dipole_desc* s) override {
    if (kComplex) return fail(LSFDTD_EUNSUPPORTED, "a point dipole needs real fields");
    Dipole d{reinterpret_cast<const long long*>(s->idx), static_cast<const R*>(s->coef),
             static_cast<const R*>(s->wave), s->n};
    step_limit = std::min<int64_t>(step_limit, s->wave_len);
    order.push_back({kDipole, dipoles.size()});
    dipoles.push_back(d);
    return LSFDTD_OK;
  }

  int add_line(const lsfdtd_line_source_desc* s) override {
    if (kComplex) return fail(LSFDTD_EUNSUPPORTED, "a 1D-fed source needs real fields");
    Line l{};
    l.E = static_cast<R*>(s->E_line);
    l.H = static_cast<R*>(s->H_line);
    l.ca = static_cast<const R*>(s->ca);
    l.cb = static_cast<const R*>(s->cb);
    l.da = static_cast<const R*>(s->da);
    l.db = static_cast<const R*>(s->db);
    l.wave = static_cast<const R*>(s->wave);
    l.M = s->M;
    l.m_src = s->m_src;
    if (l.m_src < 1 || l.m_src >= l.M - 1) return fail(LSFDTD_EINVAL, "line source node out of range");
    for (int k = 0; k < 2; ++k) {
      LineArgs<R>& a = l.corr[k];
      l.has[k] = s->pts[k].n_nodes > 0;
      a.n_nodes = s->pts[k].n_nodes;
      a.nodes = reinterpret_cast<const long long*>(s->pts[k].nodes);
      a.offsets = reinterpret_cast<const long long*>(s->pts[k].offsets);
      a.i0 = reinterpret_cast<const long long*>(s->i0[k]);
      a.w = static_cast<const R*>(s->w[k]);
      a.coef = static_cast<const R*>(s->coef[k]);
      a.src = k == 0 ? l.H : l.E;  // E corrections read the line's H, H corrections its E
      a.target = nullptr;
    }
    step_limit = std::min<int64_t>(step_limit, s->wave_len);
    order.push_back({kLine, lines.size()});
    lines.push_back(l);
    return LSFDTD_OK;
  }

  int add_column(const lsfdtd_column_source_desc* s) override {
    if (!kComplex) return fail(LSFDTD_EUNSUPPORTED, "a Bloch column source needs complex fields");
    auto* col = dynamic_cast<Engine<F>*>(s->column);
    if (!col) return fail(LSFDTD_EINVAL, "column engine of another precision");
    if (col->desc.shape[0] != 3 || col->desc.shape[1] != 3) return fail(LSFDTD_EINVAL, "column must be 3 x 3 x nz");
    if (s->k_src < 1 || s->k_src >= desc.shape[2] || s->k_src >= col->desc.shape[2] || s->k_launch < 0 ||
        s->k_launch >= col->desc.shape[2])
      return fail(LSFDTD_EINVAL, "column planes out of range");
    Column c{};
    c.col = col;
    c.k_src = s->k_src;
    c.k_launch = s->k_launch;
    c.phase = static_cast<const F*>(s->phase);
    if constexpr (kComplex) {
      c.amp0 = F{R(s->amp[0][0]), R(s->amp[0][1])};
      c.amp1 = F{R(s->amp[1][0]), R(s->amp[1][1])};
    }
    c.wave = static_cast<const R*>(s->wave);
    c.cE = R(s->cE);
    c.cH = R(s->cH);
    step_limit = std::min<int64_t>(step_limit, s->wave_len);
    order.push_back({kColumn, columns.size()});
    columns.push_back(c);
    return LSFDTD_OK;
  }

  int add_mode(const lsfdtd_mode_source_desc* s) override {
    if (kComplex) return fail(LSFDTD_EUNSUPPORTED, "a mode source needs real fields");
    if (s->r_e < 1 || s->r_h < 1) return fail(LSFDTD_EINVAL, "mode source rank < 1");
    step_limit = std::min<int64_t>(step_limit, std::min(s->len_E, s->len_H));
    order.push_back({kMode, modes.size()});
    modes.push_back(Mode{*s});
    return LSFDTD_OK;
  }

  int add_monitor(const lsfdtd_monitor_desc* m) override {
    Monitor q{};
    q.space = m->space;
    q.energy = (m->energy && m->n_h > 0) ? m->energy : 0;
    if (q.energy < 0 || q.energy > 2) return fail(LSFDTD_EINVAL, "monitor energy group must be 0, 1 or 2");
    if (m->space < 0 || m->space > 2) return fail(LSFDTD_EINVAL, "monitor space out of range");
    if (m->space == 2 && !kComplex) return fail(LSFDTD_EINVAL, "a column space needs complex fields");
    auto fill = [&](auto& a, auto* src_e, auto* src_h) {
      a.nf = m->n_freq;
      a.omega = m->omega;
      a.ne = m->n_e;
      a.nh = m->n_h;
      a.e_idx = reinterpret_cast<const long long*>(m->e_idx);
      a.h1 = reinterpret_cast<const long long*>(m->h_idx1);
      a.h2 = reinterpret_cast<const long long*>(m->h_idx2);
      a.acc_e = static_cast<cplx<double>*>(m->acc_e);
      a.acc_h = static_cast<cplx<double>*>(m->acc_h);
      a.Esrc = src_e;
      a.Hsrc = src_h;
      a.dt = desc.dt;
      a.nstep = reinterpret_cast<const long long*>(desc.step);
      a.want_energy = q.energy ? 1 : 0;
      a.partial = nullptr;
      a.blocks_e = cdiv(m->n_e, kMonBlock);
    };
    if (m->space == 1)
      fill(q.ar, static_cast<const R*>(m->E_src), static_cast<const R*>(m->H_src));
    else
      fill(q.af, static_cast<const F*>(m->E_src), static_cast<const F*>(m->H_src));
    q.blocks = (long long)cdiv(m->n_e, kMonBlock) + (m->n_h > 0 ? cdiv(m->n_h, kMonBlock) : 0);
    if (m->n_e <= 0 || m->n_freq <= 0) return fail(LSFDTD_EINVAL, "empty monitor");
    monitors.push_back(q);
    layout_energy();
    return LSFDTD_OK;
  }

  // energy partials: group 1's monitors first, then group 2's, each block one double
  void layout_energy() {
    long long off = 0;
    for (int g = 1; g <= 2; ++g) {
      e_first[g - 1] = off;
      long long cnt = 0;
      for (auto& q : monitors)
        if (q.energy == g) cnt += q.blocks;
      e_count[g - 1] = cnt;
      off += cnt;
    }
  }

  // scratch: a status word (256 bytes reserved), then the energy partials
  size_t need_scratch() const override { return kStatusBytes + (size_t)(e_count[0] + e_count[1]) * sizeof(double); }

  int ghosts(F* f, bool low, cudaStream_t s) {
    for (int a = 0; a < 3; ++a) {
      if (!desc.periodic[a]) continue;
      const int n = desc.shape[a];
      const int dst = low ? 0 : n - 1, src = low ? n - 2 : 1;
      const long long cells = (long long)desc.shape[0] * desc.shape[1] * desc.shape[2];
      const int na = a == 0 ? desc.shape[1] : desc.shape[0], nb = a == 2 ? desc.shape[1] : desc.shape[2];
      const long long tot = 3LL * na * nb;
      k_ghost<F><<<cdiv(tot, 256), 256, 0, s>>>(f, f + cells, f + 2 * cells, desc.shape[0], desc.shape[1],
                                                 desc.shape[2], a, dst, src, bloch_re[a][low ? 0 : 1],
                                                 bloch_im[a][low ? 0 : 1]);
      LS_LAUNCHED();
    }
    return LSFDTD_OK;
  }

  dim3 bulk_grid() const { return dim3(cdiv(desc.shape[2], 32), cdiv(desc.shape[1], 8), desc.shape[0]); }

  int mark(cudaStream_t s, bool begin) {
    if (!timing) return LSFDTD_OK;
    cudaEvent_t ev;
    LS_CUDA(cudaEventCreate(&ev));
    if (begin) {
      timing->push_back({ev, nullptr});
    } else {
      timing->back().second = ev;
    }
    LS_CUDA(cudaEventRecord(ev, s));
    return LSFDTD_OK;
  }

  // the in-place kernels' arguments on the current buffers
  YeeArgs<F> current_args() const {
    YeeArgs<F> a = y;
    const long long cells = (long long)desc.shape[0] * desc.shape[1] * desc.shape[2];
    for (int c = 0; c < 3; ++c) {
      a.E[c] = Ebuf[cur] + c * cells;
      a.H[c] = Hbuf[cur] + c * cells;
    }
    for (int d = 0; d < 3; ++d)
      for (int c = 0; c < 3; ++c)
        for (int sd = 0; sd < 2; ++sd) a.pml[d].psi[1][c][sd] = psiH[cur][d][c][sd];
    // the in-place kernels' inner nodes: stepped for every component and outside every slab (on a mirror
    // axis the stepped range of some components starts at node 2)
    inner_bounds(a.in_lo, a.in_hi);
    for (int ax = 0; ax < 3; ++ax)
      if (desc.mirror[ax]) a.in_lo[ax] = std::min(std::max(a.in_lo[ax], 2), a.in_hi[ax]);
    return a;
  }

  VecBounds interior() const {
    VecBounds b;
    for (int ax = 0; ax < 3; ++ax) {
      int lo = 1, hi = desc.shape[ax] - 1;
      if (y.pml[ax].on) {
        lo = std::max(lo, pml_cells[ax][0] ? pml_cells[ax][0] + 1 : 1);
        hi = std::min(hi, pml_cells[ax][1] ? desc.shape[ax] - 2 - pml_cells[ax][1] : hi);
      }
      b.lo[ax] = lo;
      b.hi[ax] = std::max(lo, hi);
      b.pml_lo[ax] = y.pml[ax].on ? pml_cells[ax][0] : 0;
      b.pml_hi[ax] = y.pml[ax].on ? pml_cells[ax][1] : 0;
    }
    return b;
  }

  // variant 2: FP32 rows of a multiple of four nodes take the four-node vector kernels
  bool vec_ok() const {
    if constexpr (std::is_same<F, float>::value) return variant == 2 && desc.shape[2] % 4 == 0;
    return false;
  }

  // the in-place H (or E) kernel, instantiated for the grid's cell shape
  void launch_inplace(bool h, const YeeArgs<F>& a, cudaStream_t s) {
    if (a.uniform) {
      if (h) k_update_h<F, 1><<<bulk_grid(), dim3(32, 8), 0, s>>>(a);
      else k_update_e<F, 1><<<bulk_grid(), dim3(32, 8), 0, s>>>(a);
    } else {
      if (h) k_update_h<F, 0><<<bulk_grid(), dim3(32, 8), 0, s>>>(a);
      else k_update_e<F, 0><<<bulk_grid(), dim3(32, 8), 0, s>>>(a);
    }
  }

  int update_h(cudaStream_t s) override {
    LS_TRY(ghosts(Eflat(), false, s));
    const YeeArgs<F> a = current_args();
    LS_TRY(mark(s, true));
    if constexpr (std::is_same<F, float>::value) {
      if (vec_ok()) {
        const dim3 grid(cdiv(desc.shape[2], 128), cdiv(desc.shape[1], 8), desc.shape[0]);
        k_update_h_v4<<<grid, dim3(32, 8), 0, s>>>(a, interior());
      } else {
        launch_inplace(true, a, s);
      }
    } else {
      launch_inplace(true, a, s);
    }
    LS_LAUNCHED();
    LS_TRY(mark(s, false));
    return LSFDTD_OK;
  }

  int update_e(cudaStream_t s) override {
    LS_TRY(ghosts(Hflat(), true, s));
    const long long cells = (long long)desc.shape[0] * desc.shape[1] * desc.shape[2];
    for (int a = 0; a < 3; ++a) {  // symmetric mirror planes: tangential H's ghost plane, after the periodic ones
      if (desc.mirror[a] <= 0) continue;
      const long long plane = (long long)desc.shape[0] * desc.shape[1] * desc.shape[2] / desc.shape[a];
      F* h = Hflat();
      k_mirror_ghost<F><<<cdiv(2 * plane, 256), 256, 0, s>>>(h, h + cells, h + 2 * cells, desc.shape[0],
                                                              desc.shape[1], desc.shape[2], a);
      LS_LAUNCHED();
    }
    const YeeArgs<F> a = current_args();
    LS_TRY(mark(s, true));
    if constexpr (std::is_same<F, float>::value) {
      if (vec_ok()) {
        const dim3 grid(cdiv(desc.shape[2], 128), cdiv(desc.shape[1], 8), desc.shape[0]);
        k_update_e_v4<<<grid, dim3(32, 8), 0, s>>>(a, interior());
      } else {
        launch_inplace(false, a, s);
      }
    } else {
      launch_inplace(false, a, s);
    }
    LS_LAUNCHED();
    LS_TRY(mark(s, false));
    return LSFDTD_OK;
  }

  const long long* nstep() const { return reinterpret_cast<const long long*>(desc.step); }

  int hook(int which, cudaStream_t s) {  // 0 correct_H, 1 advance_H, 2 correct_E, 3 advance_E
    for (auto& o : order) {
      switch (o.first) {
        case kTable: {
          Table& t = tables[o.second];
          const int k = which == 0 ? 1 : 0;
          if ((which == 0 || which == 2) && t.has[k]) {
            TableArgs<R> ta = t.corr[k];
            ta.target = reinterpret_cast<R*>(k == 0 ? Eflat() : Hflat());
            k_table_correct<R><<<cdiv(ta.n_nodes, 128), 128, 0, s>>>(ta);
            LS_LAUNCHED();
          }
          if (which == 3 && t.view) {
            k_table_view<R><<<1, 32, 0, s>>>(t.Tinc, t.corr[0].m, t.corr[0].cmax, t.inc_base, t.inc_i0, t.inc_u0,
                                             t.view, nstep());
            LS_LAUNCHED();
          }
          break;
        }
        case kDipole: {
          Dipole& d = dipoles[o.second];
          if (which == 2 && d.n > 0) {
            k_dipole<R><<<cdiv(d.n, 64), 64, 0, s>>>(reinterpret_cast<R*>(Eflat()), d.idx, d.coef, d.n, d.wave,
                                                      nstep());
            LS_LAUNCHED();
          }
          break;
        }
        case kLine: {
          Line& l = lines[o.second];
          const int k = which == 0 ? 1 : 0;
          if ((which == 0 || which == 2) && l.has[k]) {
            LineArgs<R> la = l.corr[k];
            la.target = reinterpret_cast<R*>(k == 0 ? Eflat() : Hflat());
            k_line_correct<R><<<cdiv(la.n_nodes, 128), 128, 0, s>>>(la);
            LS_LAUNCHED();
          }
          if (which == 1) {
            k_line_h<R><<<cdiv(l.M, 128), 128, 0, s>>>(l.E, l.H, l.da, l.db, l.M);
            LS_LAUNCHED();
          }
          if (which == 3) {
            k_line_e<R><<<cdiv(l.M, 128), 128, 0, s>>>(l.E, l.H, l.ca, l.cb, l.M, l.m_src, l.wave, nstep());
            LS_LAUNCHED();
          }
          break;
        }
        case kColumn: {
          Column& c = columns[o.second];
          auto* col = static_cast<Engine<F>*>(c.col);
          const int nx = desc.shape[0] - 2, ny = desc.shape[1] - 2, ncz = col->desc.shape[2];
          const long long ccells = 9LL * ncz;
          if (which == 0 || which == 2) {
            F* t0 = which == 0 ? y.H[0] : y.E[0];
            F* t1 = which == 0 ? y.H[1] : y.E[1];
            const F* src = which == 0 ? col->Eflat() : col->Hflat();
            k_column_plane<F><<<cdiv((long long)nx * ny, 128), 128, 0, s>>>(
                t0, t1, src, src + ccells, c.phase, nx, ny, desc.shape[1], desc.shape[2], c.k_src, ncz,
                which == 0 ? c.cH : c.cE, which == 0 ? 0 : 1);
            LS_LAUNCHED();
          }
          if (which == 1) LS_TRY(col->update_h(s));
          if (which == 3) {
            LS_TRY(col->update_e(s));
            F* e = col->Eflat();
            k_column_sheet<F><<<1, 32, 0, s>>>(e, e + ccells, ncz, c.k_launch, c.amp0, c.amp1, c.wave, nstep());
            LS_LAUNCHED();
          }
          break;
        }
        case kMode: {
          const lsfdtd_mode_source_desc& d = modes[o.second].d;
          if (which == 0 && d.n_h > 0) {
            k_mode<R><<<cdiv(d.n_h, 128), 128, 0, s>>>(reinterpret_cast<R*>(Hflat()),
                                                       reinterpret_cast<const long long*>(d.h_idx),
                                                       static_cast<const R*>(d.mH), static_cast<const R*>(d.tab_E),
                                                       d.n_h, d.r_e, nstep());
            LS_LAUNCHED();
          }
          if (which == 2 && d.n_e > 0) {
            k_mode<R><<<cdiv(d.n_e, 128), 128, 0, s>>>(reinterpret_cast<R*>(Eflat()),
                                                       reinterpret_cast<const long long*>(d.e_idx),
                                                       static_cast<const R*>(d.mE), static_cast<const R*>(d.tab_H),
                                                       d.n_e, d.r_h, nstep());
            LS_LAUNCHED();
          }
          break;
        }
      }
    }
    return LSFDTD_OK;
  }

  int step(cudaStream_t s) override {
    if (scratch_bytes < need_scratch()) return fail(LSFDTD_EINVAL, "scratch not set or too small");
    if (decide() && fused_variant()) {
      LS_TRY(fused_step(s));
    } else {
      LS_TRY(update_h(s));
      LS_TRY(hook(0, s));
      LS_TRY(hook(1, s));
      LS_TRY(update_e(s));
    }
    LS_TRY(offdiag(s));
    LS_TRY(hook(2, s));
    for (auto& g : groups) {
      if (g.n <= 0) continue;
      AdeArgs<F> ga = g;
      ga.E = Eflat();
      k_ade<F><<<cdiv(ga.n, 128), 128, 0, s>>>(ga);
      LS_LAUNCHED();
    }
    if (has_tensor) LS_TRY(tensor_step(s));
    LS_TRY(hook(3, s));
    k_bump<<<1, 32, 0, s>>>(reinterpret_cast<long long*>(desc.step));
    LS_LAUNCHED();
    return LSFDTD_OK;
  }

  int sample(cudaStream_t s) override {
    if (scratch_bytes < need_scratch()) return fail(LSFDTD_EINVAL, "scratch not set or too small");
    double* part = reinterpret_cast<double*>(static_cast<char*>(scratch) + kStatusBytes);
    long long off[2] = {e_first[0], e_first[1]};
    for (auto& q : monitors) {
      double* p = nullptr;
      if (q.energy) {
        p = part + off[q.energy - 1];
        off[q.energy - 1] += q.blocks;
      }
      if (q.space == 1) {
        MonArgs<R> a = q.ar;
        a.partial = p;
        k_monitor<R><<<(unsigned)q.blocks, kMonBlock, 0, s>>>(a);
      } else {
        MonArgs<F> a = q.af;
        a.partial = p;
        if (q.space == 0) {
          a.Esrc = Eflat();
          a.Hsrc = Hflat();
        }
        k_monitor<F><<<(unsigned)q.blocks, kMonBlock, 0, s>>>(a);
      }
      LS_LAUNCHED();
    }
    if (e_count[0] + e_count[1] > 0) {
      k_energy<<<1, 32, 0, s>>>(part, e_first[0], e_count[0], e_first[1], e_count[1], desc.energy);
      LS_LAUNCHED();
    }
    return LSFDTD_OK;
  }

  int64_t launches_per_chunk() const override {
    int64_t per_step = 2 + 1;  // H and E, counter
    if (fused == 1 && fused_variant()) {
      int lo[3], hi[3];
      ShellBoxes sb{};
      // fused pass (interior box, shell H and E; or the lean pass's clean interior and the rest), counter
      per_step = (split_box(lo, hi, &sb) ? 3 : (lean_ok() ? lean_launches() : 1)) + 1;
    }
    int nper = desc.periodic[0] + desc.periodic[1] + desc.periodic[2];
    per_step += 2 * nper;
    for (int a = 0; a < 3; ++a) per_step += desc.mirror[a] > 0;  // mirror ghost planes
    per_step += od_n > 0;  // the off-diagonal gather
    if (has_tensor) per_step += 2 + (tm.nV > 0) + (tm.nT > 0) + (tm.nP > 0);
    for (auto& g : groups) per_step += g.n > 0;
    for (auto& o : order) {
      switch (o.first) {
        // (on the fused pass the H corrections are k_table_values before it, in place of k_table_correct)
        case kTable: per_step += tables[o.second].has[0] + tables[o.second].has[1] + (tables[o.second].view ? 1 : 0); break;
        case kDipole: per_step += 1; break;
        case kLine: per_step += lines[o.second].has[0] + lines[o.second].has[1] + 2; break;
        case kColumn: per_step += 2 + 1 + 2 + 2 * 2; break;  // planes, sheet, column H/E, column ghosts
        case kMode: per_step += 2; break;
      }
    }
    int64_t per_sample = (int64_t)monitors.size() + (e_count[0] + e_count[1] > 0 ? 1 : 0);
    return per_step * desc.dft_stride + per_sample;
  }
};

// a batched Bloch sweep: the engines' run descriptors, the CTAs' run lists, the scratch holding them and
// the captured launch
struct BatchImpl {
  int precision = LSFDTD_F32;
  size_t run_bytes = 0;
  std::vector<lsfdtd_engine*> engines;
  std::vector<int64_t> last;
  std::vector<unsigned char> descs;  // n * run_bytes
  std::vector<int> order, first;     // runs of CTA b: order[first[b] .. first[b + 1])
  int ctas = 0;
  int cluster = kBatchCluster;  // CTAs per run (cluster size, or group size)
  bool group = false;           // more than 16 CTAs per run: a group with barriers in global memory
  int groups = 0;
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  size_t off_order = 0, off_first = 0, off_bar = 0, need = 0;
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  int graph_steps = -1;
};

// clusters of `cl` CTAs of the persistent kernel that fit on the device at once (clusters above the
// portable 8 CTAs are allowed on the kernel first); above 16 CTAs, groups of `cl` CTAs of the cooperative form
template <typename F>
int batch_max_clusters(int cl, int* out) {
  if (cl > 16) {
    int per_sm = 0, dev = 0, sms = 0;
    LS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bloch_batch<F, true>, kBatchThreads, 0));
    LS_CUDA(cudaGetDevice(&dev));
    LS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    *out = per_sm * sms / cl;
    if (*out < 1) return fail(LSFDTD_EUNSUPPORTED, "batch: a group of that many CTAs does not fit the device at once");
    return LSFDTD_OK;
  }
  if (cl > 8) LS_CUDA(cudaFuncSetAttribute(k_bloch_batch<F, false>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cl, 1, 1);
  cfg.blockDim = dim3(kBatchThreads, 1, 1);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaOccupancyMaxActiveClusters(out, k_bloch_batch<F, false>, &cfg);
  if (e != cudaSuccess) return fail(LSFDTD_ECUDA, std::string("batch: cluster occupancy: ") + cudaGetErrorString(e));
  if (*out < 1) return fail(LSFDTD_EUNSUPPORTED, "batch: no cluster of the persistent kernel fits the device");
  return LSFDTD_OK;
}

template <typename F>
int batch_launch(const BatchImpl& b, int steps, cudaStream_t s) {
  const auto* runs = static_cast<const BlochRun<F>*>(b.scratch);
  const int* order = reinterpret_cast<const int*>(static_cast<const char*>(b.scratch) + b.off_order);
  const int* first = reinterpret_cast<const int*>(static_cast<const char*>(b.scratch) + b.off_first);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(b.ctas, 1, 1);  // whole clusters or groups
  cfg.blockDim = dim3(kBatchThreads, 1, 1);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (b.group) {
    // the groups' barrier counters start at zero in every launch; every CTA resident at once
    auto* bar = reinterpret_cast<unsigned long long*>(static_cast<char*>(b.scratch) + b.off_bar);
    LS_CUDA(cudaMemsetAsync(bar, 0, (size_t)b.groups * 128, s));
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    LS_CUDA(cudaLaunchKernelEx(&cfg, k_bloch_batch<F, true>, runs, order, first, steps, b.cluster, bar));
  } else {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = b.cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    LS_CUDA(cudaLaunchKernelEx(&cfg, k_bloch_batch<F, false>, runs, order, first, steps, b.cluster,
                               (unsigned long long*)nullptr));
  }
  LS_LAUNCHED();
  return LSFDTD_OK;
}

lsfdtd_engine* make_engine(const lsfdtd_grid_desc& g) {
  if (g.precision == LSFDTD_F32) {
    if (g.is_complex) return new Engine<cplx<float>>(g);
    return new Engine<float>(g);
  }
  if (g.is_complex) return new Engine<cplx<double>>(g);
  return new Engine<double>(g);
}

int run_chunk(lsfdtd_engine* e, cudaStream_t s) {
  for (int i = 0; i < e->desc.dft_stride; ++i) LS_TRY(e->step(s));
  return e->sample(s);
}

}  // namespace

struct lsfdtd_batch : BatchImpl {};

struct lsfdtd_adjoint {
  lsfdtd_engine* eng = nullptr;
  int precision = LSFDTD_F32;
  lsfdtd_adjoint_desc d{};
  std::vector<unsigned char> yee;  // YeeArgs of the engine's precision
  int buf = 0;                     // psibar buffer holding the current (old) values
  size_t slot_elems = 0;
  AdjFreqs freqs{};                // the objective's frequencies
  std::vector<std::vector<unsigned char>> groups;  // AdeArgs of the engine's dispersive groups
  std::vector<unsigned char> tm;  // TensorArgs of the vertex-tensor mesh, state in tm_bar (nN = 0: none)
};

namespace {

template <typename R>
int adjoint_record(lsfdtd_adjoint* a, int slot, cudaStream_t s) {
  const auto& y = *reinterpret_cast<const YeeArgs<R>*>(a->yee.data());
  void* Hv = nullptr;
  std::vector<unsigned char> tmp(sizeof(YeeArgs<R>));
  LS_TRY(a->eng->adjoint_args(tmp.data(), tmp.size(), &Hv));  // the current H (a fused engine alternates)
  const long long cells = (long long)y.n[0] * y.n[1] * y.n[2];
  const R* H = static_cast<const R*>(Hv);
  const int h0 = a->d.box_hi[0] - a->d.box_lo[0] + 1, h1 = a->d.box_hi[1] - a->d.box_lo[1] + 1,
            h2 = a->d.box_hi[2] - a->d.box_lo[2] + 1;
  R* dst = static_cast<R*>(a->d.hist) + (size_t)slot * a->slot_elems;
  k_adj_hist<R><<<cdiv(3LL * h0 * h1 * h2, 256), 256, 0, s>>>(H, H + cells, H + 2 * cells, dst, y.n[1], y.n[2],
                                                            a->d.box_lo[0], a->d.box_lo[1], a->d.box_lo[2], h0,
                                                            h1, h2);
  LS_LAUNCHED();
  return LSFDTD_OK;
}

template <typename R>
int adjoint_step(lsfdtd_adjoint* a, long long n, int slot, cudaStream_t s) {
  AdjArgs<R> A{};
  A.y = *reinterpret_cast<const YeeArgs<R>*>(a->yee.data());
  const long long cells = (long long)A.y.n[0] * A.y.n[1] * A.y.n[2];
  for (int c = 0; c < 3; ++c) {
    A.Eb[c] = static_cast<R*>(a->d.Eb) + c * cells;
    A.Hb[c] = static_cast<R*>(a->d.Hb) + c * cells;
  }
  const int o = a->buf, w = a->buf ^ 1;
  for (int d = 0; d < 3; ++d)
    for (int c = 0; c < 3; ++c)
      for (int sd = 0; sd < 2; ++sd) {
        A.pe_old[d][c][sd] = static_cast<R*>(a->d.psi_bar[o][0][d][c][sd]);
        A.pe_new[d][c][sd] = static_cast<R*>(a->d.psi_bar[w][0][d][c][sd]);
        A.ph_old[d][c][sd] = static_cast<R*>(a->d.psi_bar[o][1][d][c][sd]);
        A.ph_new[d][c][sd] = static_cast<R*>(a->d.psi_bar[w][1][d][c][sd]);
      }
  for (int ax = 0; ax < 3; ++ax) {
    A.box_lo[ax] = a->d.box_lo[ax];
    A.box_hi[ax] = a->d.box_hi[ax];
  }
  A.hist = static_cast<const R*>(a->d.hist) + (size_t)slot * a->slot_elems;
  A.grad = a->d.grad;
  // inner node ranges per axis: in every component's stepped region and past every slab of the field
  for (int ax = 0; ax < 3; ++ax) {
    const int n = A.y.n[ax], mir = A.y.mirror[ax];
    int elo = mir < 0 ? 2 : 1, ehi = n - 1, hlo = mir < 0 ? 2 : ((A.y.periodic[ax] || mir) ? 1 : 0), hhi = n - 1;
    const PmlAxis<R>& pm = A.y.pml[ax];
    if (pm.on) {
      const int c = (ax + 1) % 3;  // a component with slabs along ax (both share their extent)
      for (int f = 0; f < 2; ++f) {
        int& lo = f ? hlo : elo;
        int& hi = f ? hhi : ehi;
        if (pm.len[f][c][0] > 0) lo = std::max(lo, pm.start[f][c][0] + pm.len[f][c][0]);
        if (pm.len[f][c][1] > 0) hi = std::min(hi, pm.start[f][c][1]);
      }
    }
    A.ein_lo[ax] = elo;
    A.ein_hi[ax] = ehi;
    A.hin_lo[ax] = hlo;
    A.hin_hi[ax] = hhi;
  }
  const auto& desc = a->eng->desc;
  if ((n + 1) % desc.dft_stride == 0 && a->d.n_e + a->d.n_h > 0) {
    if (a->d.inj_work) {  // per point, then per target node in the maps' order
      k_adj_inject_values<<<cdiv(a->d.n_e + a->d.n_h, 256), 256, 0, s>>>(a->d.ge, a->d.n_e, a->d.gh, a->d.n_h,
                                                                         a->freqs, desc.dt, n + 1, a->d.inj_work);
      LS_LAUNCHED();
      using LL = const long long*;
      k_adj_inject_gather<R><<<cdiv(a->d.inj_n_e + a->d.inj_n_h, 256), 256, 0, s>>>(
          A.Eb[0], A.Hb[0], a->d.inj_work, a->d.n_e, reinterpret_cast<LL>(a->d.inj_e_tgt),
          reinterpret_cast<LL>(a->d.inj_e_ptr), reinterpret_cast<LL>(a->d.inj_e_src), a->d.inj_n_e,
          reinterpret_cast<LL>(a->d.inj_h_tgt), reinterpret_cast<LL>(a->d.inj_h_ptr),
          reinterpret_cast<LL>(a->d.inj_h_src), a->d.inj_n_h);
      LS_LAUNCHED();
    } else {
      k_adj_inject<R><<<cdiv(a->d.n_e + a->d.n_h, 256), 256, 0, s>>>(
          A.Eb[0], A.Hb[0], reinterpret_cast<const long long*>(a->d.e_idx), a->d.ge, a->d.n_e,
          reinterpret_cast<const long long*>(a->d.h_idx1), reinterpret_cast<const long long*>(a->d.h_idx2),
          a->d.gh, a->d.n_h, a->freqs, desc.dt, n + 1);
      LS_LAUNCHED();
    }
  }
  // the vertex-tensor mesh ran last in the step (after the groups): its transpose comes first
  const auto& tb = *reinterpret_cast<const TensorArgs<R>*>(a->tm.data());
  if (tb.nN > 0) {
    R* work = static_cast<R*>(a->d.tm_work);
    k_adj_tm_out<R><<<cdiv(tb.nN, 256), 256, 0, s>>>(tb, A.Eb[0]);
    LS_LAUNCHED();
    if (tb.nP > 0) {
      k_adj_tm_plain<R><<<cdiv(tb.nP, 256), 256, 0, s>>>(tb, work);
      LS_LAUNCHED();
    }
    if (tb.nT > 0) {
      k_adj_tm_slots<R><<<cdiv(tb.nT, 256), 256, 0, s>>>(tb, work);
      LS_LAUNCHED();
    }
    if (tb.nV > 0) {
      k_adj_tm_vertices<R><<<cdiv(tb.nV, 256), 256, 0, s>>>(tb, work, reinterpret_cast<const long long*>(a->d.tm_vs_ptr),
                                                            reinterpret_cast<const long long*>(a->d.tm_vs_idx));
      LS_LAUNCHED();
    }
    k_adj_tm_nodes_d<R><<<cdiv(tb.nN, 256), 256, 0, s>>>(tb, A.Eb[0], work,
                                                         reinterpret_cast<const long long*>(a->d.tm_nd_ptr),
                                                         reinterpret_cast<const long long*>(a->d.tm_nd_src));
    LS_LAUNCHED();
  }
  // the dispersive groups ran after the E curl update: their transposes come next
  for (size_t gi = 0; gi < a->groups.size(); ++gi) {
    const auto& ga = *reinterpret_cast<const AdeArgs<R>*>(a->groups[gi].data());
    if (ga.n <= 0) continue;
    k_adj_ade<R><<<cdiv(ga.n, 256), 256, 0, s>>>(ga, A.Eb[0], static_cast<R*>(a->d.group_bar[gi]));
    LS_LAUNCHED();
  }
  const dim3 grid(cdiv(A.y.n[2], 32), cdiv(A.y.n[1], 8), A.y.n[0]);
  // periodic ghost copies of the forward step, transposed in the reverse order (axes 2, 1, 0)
  auto ghosts_t = [&](R* const* f, bool low) -> int {
    for (int ax = 2; ax >= 0; --ax) {
      if (!A.y.periodic[ax]) continue;
      const int n = A.y.n[ax];
      const int na = ax == 0 ? A.y.n[1] : A.y.n[0], nb = ax == 2 ? A.y.n[1] : A.y.n[2];
      k_adj_ghost<R><<<cdiv(3LL * na * nb, 256), 256, 0, s>>>(f[0], f[1], f[2], A.y.n[0], A.y.n[1], A.y.n[2], ax,
                                                            low ? 0 : n - 1, low ? n - 2 : 1);
      LS_LAUNCHED();
    }
    return LSFDTD_OK;
  };
  // the off-diagonal terms were added to E from the H the E update read
  if (a->d.od_rows > 0) {
    k_adj_offdiag<R><<<cdiv(a->d.od_rows, 256), 256, 0, s>>>(
        reinterpret_cast<const long long*>(a->d.od_h), reinterpret_cast<const long long*>(a->d.od_ptr),
        reinterpret_cast<const long long*>(a->d.od_e), static_cast<const R*>(a->d.od_w), a->d.od_rows, A.Eb[0],
        A.Hb[0]);
    LS_LAUNCHED();
  }
  if (A.y.uniform) k_adj_e<R, true><<<grid, dim3(32, 8), 0, s>>>(A);
  else k_adj_e<R, false><<<grid, dim3(32, 8), 0, s>>>(A);
  LS_LAUNCHED();
  // the symmetric mirror planes' ghosts were filled after the periodic ones, before the E update
  for (int ax = 2; ax >= 0; --ax) {
    if (A.y.mirror[ax] <= 0) continue;
    const long long plane = cells / A.y.n[ax];
    k_adj_mirror<R><<<cdiv(2 * plane, 256), 256, 0, s>>>(A.Hb[0], A.Hb[1], A.Hb[2], A.y.n[0], A.y.n[1], A.y.n[2],
                                                        ax);
    LS_LAUNCHED();
  }
  LS_TRY(ghosts_t(A.Hb, true));  // H's low ghosts were filled before the E update
  if (A.y.uniform) k_adj_h<R, true><<<grid, dim3(32, 8), 0, s>>>(A);
  else k_adj_h<R, false><<<grid, dim3(32, 8), 0, s>>>(A);
  LS_LAUNCHED();
  LS_TRY(ghosts_t(A.Eb, false));  // E's high ghosts were filled before the H update
  a->buf = w;
  return LSFDTD_OK;
}

}  // namespace

extern "C" {

int32_t lsfdtd_abi_version(void) { return LSFDTD_ABI_VERSION; }

const char* lsfdtd_last_error(void) { return g_err.c_str(); }

int32_t lsfdtd_cpml_slab(const int32_t shape[3], const int32_t periodic[3], int32_t axis, int32_t cells_lo,
                         int32_t cells_hi, int32_t field, int32_t component, int32_t side, int32_t* start,
                         int32_t* len) {
  if (!shape || !periodic || !start || !len || axis < 0 || axis > 2 || field < 0 || field > 1 || component < 0 ||
      component > 2 || side < 0 || side > 1)
    return fail(LSFDTD_EINVAL, "lsfdtd_cpml_slab: argument out of range");
  int st, ln;
  slab(shape, periodic, axis, cells_lo, cells_hi, field, component, side, &st, &ln);
  *start = st;
  *len = ln;
  return LSFDTD_OK;
}

int64_t lsfdtd_group_state_len(int32_t mixed, int32_t n_media, const int32_t* n_poles) {
  return ade_state_len(mixed, n_media, n_poles);
}

int32_t lsfdtd_engine_create(const lsfdtd_grid_desc* grid, lsfdtd_engine** out) {
  if (!grid || !out) return fail(LSFDTD_EINVAL, "null argument");
  *out = nullptr;
  for (int a = 0; a < 3; ++a) {
    if (grid->shape[a] < 3) return fail(LSFDTD_EINVAL, "every axis needs at least 3 nodes");
    if (!(grid->spacing[a] > 0)) return fail(LSFDTD_EINVAL, "spacing must be positive");
    if (grid->bloch[a] != 0 && !grid->periodic[a]) return fail(LSFDTD_EINVAL, "a Bloch wavevector needs a periodic axis");
    if (grid->mirror[a] < -1 || grid->mirror[a] > 1) return fail(LSFDTD_EINVAL, "mirror must be -1, 0 or +1");
    if (grid->mirror[a] && grid->periodic[a]) return fail(LSFDTD_EINVAL, "a mirror axis cannot be periodic");
  }
  const bool any_bloch = grid->bloch[0] != 0 || grid->bloch[1] != 0 || grid->bloch[2] != 0;
  if (any_bloch && !grid->is_complex) return fail(LSFDTD_EINVAL, "a Bloch wavevector needs complex fields");
  if (grid->precision != LSFDTD_F32 && grid->precision != LSFDTD_F64) return fail(LSFDTD_EINVAL, "unknown precision");
  if (grid->dft_stride < 1) return fail(LSFDTD_EINVAL, "dft_stride < 1");
  if (!grid->E || !grid->H || !grid->cbE[0] || !grid->cbE[1] || !grid->cbE[2] || !grid->step || !grid->energy)
    return fail(LSFDTD_EINVAL, "grid arrays missing");
  const double cells = (double)grid->shape[0] * grid->shape[1] * grid->shape[2];
  if (cells * 3 > 9.0e18) return fail(LSFDTD_EINVAL, "grid too large");
  lsfdtd_engine* e = make_engine(*grid);
  const int r = e->init_side();
  if (r != LSFDTD_OK) {
    delete e;
    return r;
  }
  *out = e;
  return LSFDTD_OK;
}

int32_t lsfdtd_engine_destroy(lsfdtd_engine* eng) {
  delete eng;
  return LSFDTD_OK;
}

#define LS_NEED(p)                                            \
  do {                                                        \
    if (!(p)) return fail(LSFDTD_EINVAL, "null argument"); \
  } while (0)

int32_t lsfdtd_engine_set_pml(lsfdtd_engine* eng, const lsfdtd_pml_desc* p) {
  LS_NEED(eng && p);
  return eng->set_pml(p);
}
int32_t lsfdtd_engine_add_group(lsfdtd_engine* eng, const lsfdtd_group_desc* g) {
  LS_NEED(eng && g);
  return eng->add_group(g);
}
int32_t lsfdtd_engine_add_offdiag(lsfdtd_engine* eng, const lsfdtd_offdiag_desc* d) {
  LS_NEED(eng && d);
  return eng->add_offdiag(d);
}
int64_t lsfdtd_tensor_state_len(int64_t n_nodes, int64_t n_vert, int64_t n_tslots, int64_t n_pslots, int32_t n_media,
                                const int32_t* n_poles) {
  if (n_media < 1 || n_media > kMaxMedia || !n_poles || n_nodes < 0 || n_vert < 0 || n_tslots < 0 || n_pslots < 0)
    return -1;
  int64_t len = 4 * n_nodes + 4 * n_vert + n_tslots;
  for (int s = 0; s < n_media; ++s) {
    if (n_poles[s] < 0 || n_poles[s] > kMaxPoles) return -1;
    len += n_tslots * (1 + 2LL * n_poles[s]) + n_tslots * 2LL * n_poles[s] + n_pslots * (1 + 2LL * n_poles[s]);
  }
  return len;
}
int32_t lsfdtd_engine_add_tensor(lsfdtd_engine* eng, const lsfdtd_tensor_desc* d) {
  LS_NEED(eng && d);
  return eng->add_tensor(d);
}
int32_t lsfdtd_engine_add_table_source(lsfdtd_engine* eng, const lsfdtd_table_source_desc* s) {
  LS_NEED(eng && s);
  return eng->add_table(s);
}
int32_t lsfdtd_engine_add_dipole(lsfdtd_engine* eng, const lsfdtd_dipole_desc* s) {
  LS_NEED(eng && s);
  return eng->add_dipole(s);
}
int32_t lsfdtd_engine_add_line_source(lsfdtd_engine* eng, const lsfdtd_line_source_desc* s) {
  LS_NEED(eng && s);
  return eng->add_line(s);
}
int32_t lsfdtd_engine_add_column_source(lsfdtd_engine* eng, const lsfdtd_column_source_desc* s) {
  LS_NEED(eng && s && s->column);
  return eng->add_column(s);
}
int32_t lsfdtd_engine_add_mode_source(lsfdtd_engine* eng, const lsfdtd_mode_source_desc* s) {
  LS_NEED(eng && s);
  return eng->add_mode(s);
}
int32_t lsfdtd_engine_add_monitor(lsfdtd_engine* eng, const lsfdtd_monitor_desc* m) {
  LS_NEED(eng && m);
  return eng->add_monitor(m);
}
int32_t lsfdtd_engine_scratch_bytes(lsfdtd_engine* eng, size_t* bytes) {
  LS_NEED(eng && bytes);
  *bytes = eng->need_scratch();
  return LSFDTD_OK;
}
int32_t lsfdtd_engine_set_scratch(lsfdtd_engine* eng, void* scratch, size_t bytes) {
  LS_NEED(eng);
  eng->scratch = scratch;
  eng->scratch_bytes = bytes;
  return LSFDTD_OK;
}

int32_t lsfdtd_engine_step(lsfdtd_engine* eng, int32_t n_steps, void* stream) {
  LS_NEED(eng);
  if (n_steps < 0) return fail(LSFDTD_EINVAL, "n_steps < 0");
  if (eng->n_host + n_steps > eng->step_limit)
    return fail(LSFDTD_ERANGE, "the run would read a source waveform past its end");
  auto s = static_cast<cudaStream_t>(stream);
  for (int i = 0; i < n_steps; ++i) {
    LS_TRY(eng->step(s));
    eng->n_host += 1;
  }
  return LSFDTD_OK;
}

int32_t lsfdtd_engine_sample(lsfdtd_engine* eng, void* stream) {
  LS_NEED(eng);
  return eng->sample(static_cast<cudaStream_t>(stream));
}

int32_t lsfdtd_engine_chunk(lsfdtd_engine* eng, int32_t n_chunks, int32_t use_graph, void* stream) {
  LS_NEED(eng);
  if (n_chunks < 0) return fail(LSFDTD_EINVAL, "n_chunks < 0");
  if (eng->n_host + (int64_t)n_chunks * eng->desc.dft_stride > eng->step_limit)
    return fail(LSFDTD_ERANGE, "the run would read a source waveform past its end");
  auto s = static_cast<cudaStream_t>(stream);
  if (!use_graph) {
    for (int c = 0; c < n_chunks; ++c) {
      LS_TRY(run_chunk(eng, s));
      eng->n_host += eng->desc.dft_stride;
    }
    return LSFDTD_OK;
  }
  eng->decide();
  for (int c = 0; c < n_chunks; ++c) {
    const int b = eng->cur;
    if (!eng->exec[b]) {
      if (s == nullptr || s == cudaStreamLegacy) return fail(LSFDTD_EINVAL, "graph capture needs a created stream");
      LS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      int r = run_chunk(eng, s);  // recorded, not run: it also advances the host's buffer index
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(s, &g);
      eng->cur = b;
      if (r != LSFDTD_OK) {
        if (g) cudaGraphDestroy(g);
        return r;
      }
      if (e != cudaSuccess) return fail(LSFDTD_ECUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
      eng->graph[b] = g;
      LS_CUDA(cudaGraphInstantiate(&eng->exec[b], g, 0));
    }
    LS_CUDA(cudaGraphLaunch(eng->exec[b], s));
    eng->n_host += eng->desc.dft_stride;
    if (eng->fused == 1 && eng->fused_variant() && (eng->desc.dft_stride & 1)) eng->cur ^= 1;
  }
  return LSFDTD_OK;
}

int32_t lsfdtd_engine_chunk_timed(lsfdtd_engine* eng, int32_t n_chunks, void* stream, double* bulk_ms,
                                  int64_t* bulk_launches) {
  LS_NEED(eng && bulk_ms && bulk_launches);
  if (n_chunks < 0) return fail(LSFDTD_EINVAL, "n_chunks < 0");
  if (eng->n_host + (int64_t)n_chunks * eng->desc.dft_stride > eng->step_limit)
    return fail(LSFDTD_ERANGE, "the run would read a source waveform past its end");
  auto s = static_cast<cudaStream_t>(stream);
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
  eng->timing = &ev;
  int r = LSFDTD_OK;
  for (int c = 0; c < n_chunks && r == LSFDTD_OK; ++c) {
    r = run_chunk(eng, s);
    if (r == LSFDTD_OK) eng->n_host += eng->desc.dft_stride;
  }
  eng->timing = nullptr;
  cudaError_t e = cudaStreamSynchronize(s);
  double tot = 0.0;
  for (auto& p : ev) {
    float ms = 0.f;
    if (r == LSFDTD_OK && e == cudaSuccess && p.second && cudaEventElapsedTime(&ms, p.first, p.second) == cudaSuccess)
      tot += ms;
    cudaEventDestroy(p.first);
    if (p.second) cudaEventDestroy(p.second);
  }
  if (r != LSFDTD_OK) return r;
  if (e != cudaSuccess) return fail(LSFDTD_ECUDA, std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
  *bulk_ms = tot;
  *bulk_launches = (int64_t)ev.size();
  return LSFDTD_OK;
}

int32_t lsfdtd_engine_buffer(const lsfdtd_engine* eng) { return eng ? eng->cur : -1; }

int32_t lsfdtd_engine_status(lsfdtd_engine* eng, void* stream, int32_t* status) {
  LS_NEED(eng && status);
  *status = 0;
  if (!eng->scratch || eng->scratch_bytes < sizeof(int32_t)) return LSFDTD_OK;
  int32_t v = 0;
  auto s = static_cast<cudaStream_t>(stream);
  LS_CUDA(cudaMemcpyAsync(&v, eng->scratch, sizeof(v), cudaMemcpyDeviceToHost, s));
  LS_CUDA(cudaStreamSynchronize(s));
  *status = v;
  if (v == lsfdtd::kBatchNonFinite) return fail(LSFDTD_ENONFINITE, "the run's fields turned non-finite in a batched launch");
  if (v) return fail(LSFDTD_ETIMEOUT, "a kernel gave up waiting for its copies (status word set)");
  return LSFDTD_OK;
}

int32_t lsfdtd_engine_clear_status(lsfdtd_engine* eng, void* stream) {
  LS_NEED(eng);
  if (!eng->scratch || eng->scratch_bytes < sizeof(int32_t)) return LSFDTD_OK;
  LS_CUDA(cudaMemsetAsync(eng->scratch, 0, sizeof(int32_t), static_cast<cudaStream_t>(stream)));
  return LSFDTD_OK;
}

int32_t lsfdtd_engine_set_wait_budget(lsfdtd_engine* eng, int64_t cycles) {
  LS_NEED(eng);
  if (eng->exec[0] || eng->exec[1])
    return fail(LSFDTD_EINVAL, "the wait budget must be set before the first graph capture");
  eng->wait_budget = cycles != 0 ? (long long)cycles : lsfdtd::kWaitBudget;
  return LSFDTD_OK;
}

int32_t lsfdtd_engine_set_table_boxes(lsfdtd_engine* eng, int32_t table, int32_t n_boxes, const int32_t* boxes,
                                      const int64_t* perm, int64_t n_entries, void* vals) {
  LS_NEED(eng);
  if (eng->fused >= 0) return fail(LSFDTD_EINVAL, "table boxes must be given before the first step");
  return eng->set_table_boxes(table, n_boxes, boxes, perm, n_entries, vals);
}

int32_t lsfdtd_engine_set_copy_engine(lsfdtd_engine* eng, int32_t use_tma) {
  LS_NEED(eng);
  if (eng->fused >= 0) return fail(LSFDTD_EINVAL, "the copy engine must be chosen before the first step");
  eng->use_tma = use_tma ? 1 : 0;
  return LSFDTD_OK;
}

int32_t lsfdtd_engine_uses_tma(lsfdtd_engine* eng) {
  return eng ? (eng->decide() && eng->fused_variant() && eng->uses_tma()) : -1;
}

int32_t lsfdtd_engine_fused(lsfdtd_engine* eng) { return eng ? (eng->decide() && eng->fused_variant()) : -1; }

int32_t lsfdtd_engine_set_tuning(lsfdtd_engine* eng, int32_t variant, int32_t tile_y, int32_t planes,
                                 int32_t stages) {
  LS_NEED(eng);
  const bool ok = variant == 0 || variant == 2 ||
                  ((variant == 1 || variant == 3 || variant == 4) && (tile_y == 8 || tile_y == 16) &&
                   (stages == 4 || stages == 6 || stages == 8) && planes >= 0);
  if (!ok)
    return fail(LSFDTD_EINVAL, "tuning: variant 0 (in-place kernels), 2 (in-place four-node kernels), 1 (fused "
                               "pass), 3 (fused pass split into interior box and shell) or 4 (fused pass with lean "
                               "CPML terms); for 1, 3 and 4 CTA tile rows 8 or 16, ring 4, 6 or 8, planes >= 1 (0: per grid)");
  if (eng->exec[0] || eng->exec[1]) return fail(LSFDTD_EINVAL, "tuning must be set before the first graph capture");
  eng->variant = variant;
  eng->tuned = true;
  eng->tile_y = tile_y;
  eng->planes = planes;
  eng->stages = stages;
  return LSFDTD_OK;
}

int32_t lsfdtd_engine_set_clean_split(lsfdtd_engine* eng, int32_t on) {
  LS_NEED(eng);
  if (eng->exec[0] || eng->exec[1]) return fail(LSFDTD_EINVAL, "the split must be set before the first graph capture");
  eng->split_clean = on ? 1 : 0;
  return LSFDTD_OK;
}

int64_t lsfdtd_engine_steps(const lsfdtd_engine* eng) { return eng ? eng->n_host : -1; }

int64_t lsfdtd_engine_launches_per_chunk(const lsfdtd_engine* eng) { return eng ? eng->launches_per_chunk() : -1; }

int32_t lsfdtd_batch_create(lsfdtd_engine* const* engines, int32_t n, const int64_t* last, lsfdtd_batch** out) {
  return lsfdtd_batch_create_shaped(engines, n, last, 0, 0, out);
}

int32_t lsfdtd_batch_create_shaped(lsfdtd_engine* const* engines, int32_t n, const int64_t* last,
                                   int32_t cluster_ctas, int32_t max_clusters, lsfdtd_batch** out) {
  LS_NEED(engines && last && out && n > 0);
  if (cluster_ctas < 0 || cluster_ctas > 4096 || max_clusters < 0)
    return fail(LSFDTD_EINVAL, "batch: 1 to 16 CTAs per cluster (or up to 4096 per group, 0: the default), a "
                               "non-negative limit");
  *out = nullptr;
  auto b = std::make_unique<lsfdtd_batch>();
  b->precision = engines[0] ? engines[0]->desc.precision : LSFDTD_F32;
  for (int32_t i = 0; i < n; ++i) {
    lsfdtd_engine* e = engines[i];
    if (!e) return fail(LSFDTD_EINVAL, "batch: null engine");
    if (e->desc.precision != b->precision || !e->desc.is_complex)
      return fail(LSFDTD_EINVAL, "batch: engines of one precision with complex fields");
    const size_t rb = e->bloch_desc_bytes();
    if (b->run_bytes == 0) b->run_bytes = rb;
    std::vector<unsigned char> d(rb);
    LS_TRY(e->bloch_desc(d.data(), rb, last[i]));
    b->descs.insert(b->descs.end(), d.begin(), d.end());
    b->engines.push_back(e);
    b->last.push_back(last[i]);
  }
  // the default: groups of half the CTAs resident at once, two runs in flight (measured on B200 over 96
  // metasurface runs of 30-60 x 30-60 x 200 cells: 30.7 Gcell-updates/s, against 29.4 with four groups and
  // 26.9 with clusters of 8 CTAs; the two runs in flight stay in L2, 90 % of sectors hit)
  if (cluster_ctas == 0) {
    int per_sm = 0, dev = 0, sms = 0;
    const cudaError_t e = b->precision == LSFDTD_F32
                              ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bloch_batch<cplx<float>, true>,
                                                                              kBatchThreads, 0)
                              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bloch_batch<cplx<double>, true>,
                                                                              kBatchThreads, 0);
    if (e != cudaSuccess) return fail(LSFDTD_ECUDA, std::string("batch: occupancy: ") + cudaGetErrorString(e));
    LS_CUDA(cudaGetDevice(&dev));
    LS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cluster_ctas = std::max(17, per_sm * sms / 2);
  }
  // one wave of clusters; the runs longest first, each to the cluster with the least work so far
  int clusters = 0;
  LS_TRY(b->precision == LSFDTD_F32 ? batch_max_clusters<cplx<float>>(cluster_ctas, &clusters)
                                    : batch_max_clusters<cplx<double>>(cluster_ctas, &clusters));
  clusters = std::max(1, std::min<int>(n, clusters));
  if (max_clusters > 0) clusters = std::min(clusters, (int)max_clusters);
  b->cluster = cluster_ctas;
  b->group = cluster_ctas > 16;
  b->groups = clusters;
  b->ctas = clusters * cluster_ctas;
  for (int32_t i = 0; i < n; ++i) {
    const auto& d = b->engines[i]->desc;
    // the kernel's node offsets within a component are 32-bit
    if ((double)d.shape[0] * d.shape[1] * d.shape[2] >= 4294967296.0)
      return fail(LSFDTD_EUNSUPPORTED, "batch: a run of 2^32 nodes or more");
  }
  std::vector<double> cost(n);
  for (int32_t i = 0; i < n; ++i) {
    const auto& d = b->engines[i]->desc;
    cost[i] = (double)d.shape[0] * d.shape[1] * d.shape[2] * (double)std::max<int64_t>(0, last[i] - b->engines[i]->n_host);
  }
  std::vector<int> idx(n);
  for (int32_t i = 0; i < n; ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int c) { return cost[a] > cost[c]; });
  std::vector<double> load(clusters, 0.0);
  std::vector<std::vector<int>> lists(clusters);
  for (int i : idx) {
    const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    load[k] += cost[i];
    lists[k].push_back(i);
  }
  b->first.push_back(0);
  for (auto& l : lists) {
    b->order.insert(b->order.end(), l.begin(), l.end());
    b->first.push_back((int)b->order.size());
  }
  auto up = [](size_t x) { return (x + 255) / 256 * 256; };
  b->off_order = up(b->descs.size());
  b->off_first = b->off_order + up(b->order.size() * sizeof(int));
  b->off_bar = b->off_first + up(b->first.size() * sizeof(int));
  b->need = b->off_bar + up((size_t)clusters * 128);  // a 128-byte line per group's barrier counter
  *out = b.release();
  return LSFDTD_OK;
}

int32_t lsfdtd_batch_destroy(lsfdtd_batch* batch) {
  if (!batch) return LSFDTD_OK;
  if (batch->exec) cudaGraphExecDestroy(batch->exec);
  if (batch->graph) cudaGraphDestroy(batch->graph);
  delete batch;
  return LSFDTD_OK;
}

int32_t lsfdtd_batch_scratch_bytes(const lsfdtd_batch* batch, size_t* bytes) {
  LS_NEED(batch && bytes);
  *bytes = batch->need;
  return LSFDTD_OK;
}

int32_t lsfdtd_batch_set_scratch(lsfdtd_batch* batch, void* scratch, size_t bytes) {
  LS_NEED(batch && scratch);
  if (bytes < batch->need) return fail(LSFDTD_EINVAL, "batch: scratch too small");
  if (reinterpret_cast<uintptr_t>(scratch) % 256) return fail(LSFDTD_EINVAL, "batch: scratch must be 256-byte aligned");
  char* base = static_cast<char*>(scratch);
  LS_CUDA(cudaMemcpy(base, batch->descs.data(), batch->descs.size(), cudaMemcpyHostToDevice));
  LS_CUDA(cudaMemcpy(base + batch->off_order, batch->order.data(), batch->order.size() * sizeof(int),
                     cudaMemcpyHostToDevice));
  LS_CUDA(cudaMemcpy(base + batch->off_first, batch->first.data(), batch->first.size() * sizeof(int),
                     cudaMemcpyHostToDevice));
  batch->scratch = scratch;
  batch->scratch_bytes = bytes;
  return LSFDTD_OK;
}

int32_t lsfdtd_batch_run(lsfdtd_batch* batch, int32_t steps, int32_t n_launches, int32_t use_graph, void* stream) {
  LS_NEED(batch);
  if (!batch->scratch) return fail(LSFDTD_EINVAL, "batch: scratch not set");
  if (steps < 0 || n_launches < 0) return fail(LSFDTD_EINVAL, "batch: negative step or launch count");
  auto s = static_cast<cudaStream_t>(stream);
  auto launch = [&](cudaStream_t st) {
    return batch->precision == LSFDTD_F32 ? batch_launch<cplx<float>>(*batch, steps, st)
                                          : batch_launch<cplx<double>>(*batch, steps, st);
  };
  for (int32_t l = 0; l < n_launches; ++l) {
    if (!use_graph) {
      LS_TRY(launch(s));
    } else {
      if (!batch->exec || batch->graph_steps != steps) {
        if (s == nullptr || s == cudaStreamLegacy) return fail(LSFDTD_EINVAL, "graph capture needs a created stream");
        if (batch->exec) cudaGraphExecDestroy(batch->exec);
        if (batch->graph) cudaGraphDestroy(batch->graph);
        batch->exec = nullptr;
        batch->graph = nullptr;
        LS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const int r = launch(s);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s, &g);
        if (r != LSFDTD_OK) {
          if (g) cudaGraphDestroy(g);
          return r;
        }
        if (e != cudaSuccess) return fail(LSFDTD_ECUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
        batch->graph = g;
        LS_CUDA(cudaGraphInstantiate(&batch->exec, g, 0));
        batch->graph_steps = steps;
      }
      LS_CUDA(cudaGraphLaunch(batch->exec, s));
    }
    for (size_t i = 0; i < batch->engines.size(); ++i) {
      lsfdtd_engine* e = batch->engines[i];
      e->n_host = std::min<int64_t>(e->n_host + steps, batch->last[i]);
    }
  }
  return LSFDTD_OK;
}

int32_t lsfdtd_batch_ctas(const lsfdtd_batch* batch) { return batch ? batch->ctas : -1; }

int32_t lsfdtd_adjoint_create(lsfdtd_engine* eng, const lsfdtd_adjoint_desc* d, lsfdtd_adjoint** out) {
  LS_NEED(eng && d && out && d->Eb && d->Hb && d->grad && d->hist && d->hist_slots > 0);
  *out = nullptr;
  auto a = std::make_unique<lsfdtd_adjoint>();
  a->eng = eng;
  a->precision = eng->desc.precision;
  a->d = *d;
  a->yee.resize(a->precision == LSFDTD_F32 ? sizeof(YeeArgs<float>) : sizeof(YeeArgs<double>));
  void* H = nullptr;
  LS_TRY(eng->adjoint_args(a->yee.data(), a->yee.size(), &H));
  if ((d->n_e > 0 && (!d->e_idx || !d->ge)) || (d->n_h > 0 && (!d->h_idx1 || !d->h_idx2 || !d->gh)))
    return fail(LSFDTD_EINVAL, "adjoint: objective arrays missing");
  if (d->n_e + d->n_h > 0) {
    if (!d->omega || d->n_freq < 1 || d->n_freq > kAdjMaxFreq)
      return fail(LSFDTD_EINVAL, "adjoint: 1 to " + std::to_string(kAdjMaxFreq) + " objective frequencies");
    for (int f = 0; f < d->n_freq; ++f) a->freqs.omega[f] = d->omega[f];
    a->freqs.nf = d->n_freq;
  }
  a->d.omega = nullptr;  // copied: the caller's array need not outlive this call
  if (d->inj_work) {  // the injection maps: every target in the field, every listed point one of the objective's
    const long long flat = 3LL * eng->desc.shape[0] * eng->desc.shape[1] * eng->desc.shape[2];
    auto check_map = [&](const int64_t* tgt, const int64_t* ptr, const int64_t* src, long long n_t,
                         long long n_pts) -> int {
      if (n_t < 0 || n_t > flat || (n_t > 0 && (!tgt || !ptr || !src)))
        return fail(LSFDTD_EINVAL, "adjoint: injection map missing or larger than the field");
      if (n_t == 0) return LSFDTD_OK;
      std::vector<long long> t(n_t), p(n_t + 1);
      LS_CUDA(cudaMemcpy(t.data(), tgt, n_t * sizeof(long long), cudaMemcpyDeviceToHost));
      LS_CUDA(cudaMemcpy(p.data(), ptr, (n_t + 1) * sizeof(long long), cudaMemcpyDeviceToHost));
      if (p[0] != 0 || p.back() > 2 * n_pts) return fail(LSFDTD_EINVAL, "adjoint: injection map out of range");
      for (long long r = 0; r < n_t; ++r)  // non-decreasing from 0: every pointer in [0, 2 n_pts]
        if (p[r + 1] < p[r] || t[r] < 0 || t[r] >= flat) return fail(LSFDTD_ERANGE, "adjoint: injection map out of range");
      std::vector<long long> sr(p.back());
      if (!sr.empty()) LS_CUDA(cudaMemcpy(sr.data(), src, sr.size() * sizeof(long long), cudaMemcpyDeviceToHost));
      for (long long v : sr)
        if (v < 0 || v >= n_pts) return fail(LSFDTD_ERANGE, "adjoint: injection map out of range");
      return LSFDTD_OK;
    };
    LS_TRY(check_map(d->inj_e_tgt, d->inj_e_ptr, d->inj_e_src, d->inj_n_e, d->n_e));
    LS_TRY(check_map(d->inj_h_tgt, d->inj_h_ptr, d->inj_h_src, d->inj_n_h, d->n_h));
  }
  if (d->n_groups != eng->adjoint_n_groups() || d->n_groups > LSFDTD_ADJ_MAX_GROUPS)
    return fail(LSFDTD_EINVAL, "adjoint: n_groups must equal the engine's dispersive groups");
  for (int gi = 0; gi < d->n_groups; ++gi) {
    std::vector<unsigned char> ga(a->precision == LSFDTD_F32 ? sizeof(AdeArgs<float>) : sizeof(AdeArgs<double>));
    LS_TRY(eng->adjoint_group(gi, ga.data(), ga.size()));
    const long long gn = a->precision == LSFDTD_F32 ? reinterpret_cast<const AdeArgs<float>*>(ga.data())->n
                                                    : reinterpret_cast<const AdeArgs<double>*>(ga.data())->n;
    if (gn > 0 && !d->group_bar[gi]) return fail(LSFDTD_EINVAL, "adjoint: a group's adjoint state is missing");
    a->groups.push_back(std::move(ga));
  }
  const int32_t* n = eng->desc.shape;
  // inside every E component's stepped region: from node 2 along an antisymmetric mirror plane's axis
  for (int ax = 0; ax < 3; ++ax)
    if (d->box_lo[ax] < (eng->desc.mirror[ax] < 0 ? 2 : 1) || d->box_hi[ax] > n[ax] - 1 ||
        d->box_hi[ax] <= d->box_lo[ax])
      return fail(LSFDTD_EINVAL, "adjoint: gradient box out of range");
  long long od_rows = 0;
  int od_width = 0;
  eng->adjoint_offdiag(&od_rows, &od_width);
  if (od_rows > 0) {
    if (d->od_rows <= 0 || !d->od_h || !d->od_ptr || !d->od_e || !d->od_w)
      return fail(LSFDTD_EINVAL, "adjoint: the engine has conformal off-diagonal terms; give them transposed");
    // index ranges checked here, once (the kernel trusts them)
    const long long flat = 3LL * n[0] * n[1] * n[2];
    if (d->od_rows > flat) return fail(LSFDTD_EINVAL, "adjoint: more off-diagonal rows than H values");
    std::vector<long long> ptr(d->od_rows + 1), hh(d->od_rows);
    LS_CUDA(cudaMemcpy(ptr.data(), d->od_ptr, ptr.size() * sizeof(long long), cudaMemcpyDeviceToHost));
    LS_CUDA(cudaMemcpy(hh.data(), d->od_h, hh.size() * sizeof(long long), cudaMemcpyDeviceToHost));
    if (ptr[0] != 0 || ptr.back() > od_rows * (long long)od_width)
      return fail(LSFDTD_EINVAL, "adjoint: off-diagonal row pointers out of range");
    for (long long r = 0; r < d->od_rows; ++r)
      if (ptr[r + 1] < ptr[r] || hh[r] < 0 || hh[r] >= flat)
        return fail(LSFDTD_ERANGE, "adjoint: an off-diagonal row out of range");
    std::vector<long long> ee(ptr.back());
    if (!ee.empty())
      LS_CUDA(cudaMemcpy(ee.data(), d->od_e, ee.size() * sizeof(long long), cudaMemcpyDeviceToHost));
    for (long long v : ee)
      if (v < 0 || v >= flat) return fail(LSFDTD_ERANGE, "adjoint: an off-diagonal E index out of range");
  } else if (d->od_rows != 0) {
    return fail(LSFDTD_EINVAL, "adjoint: off-diagonal rows given for an engine without such terms");
  }
  // the vertex-tensor mesh: its arguments with the state pointed into tm_bar, and the caller's maps checked
  a->tm.resize(a->precision == LSFDTD_F32 ? sizeof(TensorArgs<float>) : sizeof(TensorArgs<double>));
  LS_TRY(eng->adjoint_tensor(a->tm.data(), a->tm.size()));
  auto bind = [&](auto* ta) -> int {
    if (ta->nN <= 0) {
      if (d->tm_bar) return fail(LSFDTD_EINVAL, "adjoint: tensor adjoint given for an engine without a vertex-tensor mesh");
      return LSFDTD_OK;
    }
    if (!d->tm_bar || !d->tm_work || !d->tm_vs_ptr || !d->tm_nd_ptr || (ta->nT > 0 && !d->tm_vs_idx))
      return fail(LSFDTD_EINVAL, "adjoint: the engine has a vertex-tensor mesh; give its adjoint state and maps");
    auto host = [&](const int64_t* src, long long n, std::vector<long long>& out) -> int {
      out.resize(n);
      if (n > 0) LS_CUDA(cudaMemcpy(out.data(), src, n * sizeof(long long), cudaMemcpyDeviceToHost));
      return LSFDTD_OK;
    };
    std::vector<long long> vp, vi, np_, ns, tv, tvc;
    LS_TRY(host(d->tm_vs_ptr, ta->nV + 1, vp));
    LS_TRY(host(d->tm_nd_ptr, ta->nN + 1, np_));
    LS_TRY(host(reinterpret_cast<const int64_t*>(ta->t_v), ta->nT, tv));
    LS_TRY(host(reinterpret_cast<const int64_t*>(ta->t_vc), ta->nT, tvc));
    if (vp[0] != 0 || vp.back() != ta->nT) return fail(LSFDTD_EINVAL, "adjoint: tensor slot map out of range");
    LS_TRY(host(d->tm_vs_idx, ta->nT, vi));
    for (long long v = 0; v < ta->nV; ++v) {
      if (vp[v + 1] < vp[v]) return fail(LSFDTD_EINVAL, "adjoint: tensor slot map out of range");
      for (long long j = vp[v]; j < vp[v + 1]; ++j)  // the slots listed for v are v's, on one of its components
        if (vi[j] < 0 || vi[j] >= ta->nT || tv[vi[j]] != v || tvc[vi[j]] / 3 != v)
          return fail(LSFDTD_ERANGE, "adjoint: tensor slot map does not match the mesh");
    }
    const long long entries = 6 * ta->nV + ta->nT + ta->nP;
    if (np_[0] != 0 || np_.back() > entries) return fail(LSFDTD_EINVAL, "adjoint: tensor node map out of range");
    for (long long i = 0; i < ta->nN; ++i)  // non-decreasing from 0: every pointer in [0, entries]
      if (np_[i + 1] < np_[i]) return fail(LSFDTD_EINVAL, "adjoint: tensor node map out of range");
    LS_TRY(host(d->tm_nd_src, np_.back(), ns));
    for (long long v : ns)
      if (v < 0 || v >= entries) return fail(LSFDTD_ERANGE, "adjoint: tensor node map out of range");
    using Fld = std::remove_pointer_t<decltype(ta->D)>;
    tm_bind_state(*ta, static_cast<Fld*>(d->tm_bar));
    return LSFDTD_OK;
  };
  LS_TRY(a->precision == LSFDTD_F32 ? bind(reinterpret_cast<TensorArgs<float>*>(a->tm.data()))
                                    : bind(reinterpret_cast<TensorArgs<double>*>(a->tm.data())));
  // every E node of the box outside every E slab (there the E update's coefficient enters only through the
  // curl term; the H values of the box and its halo are recorded, wherever they lie)
  auto slabs_ok = [&](const auto& y) {
    for (int dd = 0; dd < 3; ++dd) {
      if (!y.pml[dd].on) continue;
      for (int f = 0; f < 2; ++f)
        for (int c = 0; c < 3; ++c)
          for (int sd = 0; sd < 2; ++sd) {
            const int st = y.pml[dd].start[f][c][sd], ln = y.pml[dd].len[f][c][sd];
            if (f == 0 && ln > 0 && d->box_lo[dd] < st + ln && d->box_hi[dd] > st) return false;
            const bool need = ln > 0;
            for (int b = 0; b < 2; ++b)
              if (need && !d->psi_bar[b][f][dd][c][sd]) return false;
          }
    }
    return true;
  };
  const bool ok = a->precision == LSFDTD_F32 ? slabs_ok(*reinterpret_cast<const YeeArgs<float>*>(a->yee.data()))
                                             : slabs_ok(*reinterpret_cast<const YeeArgs<double>*>(a->yee.data()));
  if (!ok) return fail(LSFDTD_EINVAL, "adjoint: the box overlaps a CPML slab, or a psibar slab is missing");
  a->slot_elems = 3ull * (d->box_hi[0] - d->box_lo[0] + 1) * (d->box_hi[1] - d->box_lo[1] + 1) *
                  (d->box_hi[2] - d->box_lo[2] + 1);
  *out = a.release();
  return LSFDTD_OK;
}

int32_t lsfdtd_engine_set_steps(lsfdtd_engine* eng, int64_t n) {
  LS_NEED(eng);
  if (n < 0 || n > eng->step_limit) return fail(LSFDTD_ERANGE, "step count out of range");
  eng->n_host = n;
  return LSFDTD_OK;
}

int32_t lsfdtd_adjoint_destroy(lsfdtd_adjoint* adj) {
  delete adj;
  return LSFDTD_OK;
}

int32_t lsfdtd_adjoint_record(lsfdtd_adjoint* adj, int32_t slot, void* stream) {
  LS_NEED(adj);
  if (slot < 0 || slot >= adj->d.hist_slots) return fail(LSFDTD_EINVAL, "adjoint: history slot out of range");
  auto s = static_cast<cudaStream_t>(stream);
  return adj->precision == LSFDTD_F32 ? adjoint_record<float>(adj, slot, s) : adjoint_record<double>(adj, slot, s);
}

int32_t lsfdtd_adjoint_step(lsfdtd_adjoint* adj, int64_t n, int32_t slot, void* stream) {
  LS_NEED(adj);
  if (slot < 0 || slot >= adj->d.hist_slots) return fail(LSFDTD_EINVAL, "adjoint: history slot out of range");
  if (n < 0) return fail(LSFDTD_EINVAL, "adjoint: negative step");
  auto s = static_cast<cudaStream_t>(stream);
  return adj->precision == LSFDTD_F32 ? adjoint_step<float>(adj, n, slot, s) : adjoint_step<double>(adj, n, slot, s);
}

}  // extern "C"
