/*
 * lsfdtd: B200 (sm_100a) kernels for lightsmith's 3D FDTD time-stepping loop, behind a C ABI.
 *
 * The ABI replaces the device-side engine of lightsmith v0.3.0 (src/lightsmith/backends/_fdtd/engine.py):
 * an engine handle is built from plain device pointers and sizes (all device memory is owned by the caller,
 * e.g. PyTorch tensors; the library allocates none), then stepped in chunks of `dft_stride` steps followed by
 * one DFT sample, on a caller stream, optionally replayed as a CUDA graph. Handles are not thread-safe; one
 * handle per run. Every function returns LSFDTD_OK (0) or an error code; lsfdtd_last_error() gives the
 * message of the calling thread's last failure.
 *
 * Field arrays are stacked F[3][N0][N1][N2] (N2 fastest), exactly lightsmith's E/H layout, so the flat
 * indices lightsmith's set-up code produces (monitors, sources, dispersive nodes) are used unchanged.
 * Complex fields (a Bloch wavevector) are interleaved (re, im) pairs of the field precision.
 */
#ifndef LSFDTD_H
#define LSFDTD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LSFDTD_ABI_VERSION 2

enum { LSFDTD_F32 = 0, LSFDTD_F64 = 1 };
enum {
  LSFDTD_OK = 0,
  LSFDTD_EINVAL = 1,      /* bad argument or inconsistent description */
  LSFDTD_ECUDA = 2,       /* a CUDA call failed (the message names it) */
  LSFDTD_EUNSUPPORTED = 3,
  LSFDTD_ERANGE = 4,      /* the run would read a source waveform past its end */
  LSFDTD_ETIMEOUT = 5,    /* a kernel gave up waiting for its own copies (bounded wait, status word set) */
  LSFDTD_ENONFINITE = 6   /* a batched run's fields turned non-finite; the run retired (status word 2) */
};
#define LSFDTD_MAX_MEDIA 4
#define LSFDTD_MAX_POLES 6

typedef struct lsfdtd_engine lsfdtd_engine;

/* Grid, bulk coefficients and run state. Replaces Engine.__init__'s field arrays and curl coefficients
 * (engine.py:231-315): cbE[c] = (dt/dx or dt) * (1/eps)_c over the whole grid (the three may alias one
 * array when eps is isotropic). step: completed-step counter (Engine.n, engine.py:271). energy: the two
 * decay-energy proxies (Engine.energy, engine.py:315). */
typedef struct {
  int32_t shape[3];
  int32_t precision;   /* LSFDTD_F32 or LSFDTD_F64 */
  int32_t is_complex;  /* nonzero under a Bloch wavevector */
  int32_t periodic[3];
  double spacing[3];   /* nm; all equal for cubic cells */
  double dt;           /* nm/c */
  double bloch[3];     /* rad/nm per periodic axis */
  int32_t dft_stride;
  void* E;             /* device, zeroed */
  void* H;             /* device, zeroed */
  const void* cbE[3];  /* device, field precision (real) */
  int64_t* step;       /* device, one int64 */
  double* energy;      /* device, two doubles */
  /* optional second E/H buffers (zeroed, same layout): with them a run without periodic axes whose sources
   * only correct E advances each step in one fused pass, alternating between the two buffers
   * (lsfdtd_engine_buffer tells which holds the current fields); NULL: in-place kernels */
  void* E_alt;
  void* H_alt;
  /* mirror plane per axis at node 1 (engine.py:47-60, the `mirror` argument of lightsmith's Engine): 0 none,
   * +1 symmetric (PMC: tangential H's ghost plane 0 is refreshed as minus plane 1 before each E update), -1
   * antisymmetric (PEC: tangential E vanishes on plane 1); on a non-periodic axis without PML on its low
   * side. Such runs step in place. */
  int32_t mirror[3];
} lsfdtd_grid_desc;

/* One CPML axis (Engine._build_pml, engine.py:344-418). Profiles have one entry per node position along the
 * axis: [0] at the E positions u, [1] at the H positions u + 1/2; b = exp(-(sigma/kappa + alpha) dt),
 * c = sigma (b - 1) / (sigma kappa + kappa^2 alpha), k = 1/kappa - 1 (NULL when kappa is 1 everywhere).
 * psi[field][component][side]: zeroed device slabs sized by lsfdtd_cpml_slab() (NULL where that is empty). */
typedef struct {
  int32_t axis;
  int32_t cells_lo, cells_hi;
  const void* b[2];
  const void* c[2];
  const void* k[2];
  void* psi[2][3][2];
  void* psi_alt[3][2]; /* second H psi slabs, used with the grid's second buffers (else NULL) */
} lsfdtd_pml_desc;

/* D-form ADE nodes (the _Group of engine.py:722-793). Pure group: one dispersive medium. Mixed group
 * (subpixel interface cells): harmonic path weight w, h0 = sum of f_s/eps_inf_s over non-dispersive media,
 * inv_a = 1/sum_s f_s eps_inf_s, frac = [n_media][n] fractions of the dispersive media. Coefficients per
 * dispersive medium and pole: P^{n+1} = c1 P^n + c2 P^{n-1} + c3 E (engine.py:108-111). state: zeroed
 * device buffer of lsfdtd_group_state_len() * n field scalars. */
typedef struct {
  int64_t n;
  const int64_t* idx;
  int32_t mixed, has_h, has_a;
  int32_t n_media;
  int32_t n_poles[LSFDTD_MAX_MEDIA];
  double c1[LSFDTD_MAX_MEDIA][LSFDTD_MAX_POLES];
  double c2[LSFDTD_MAX_MEDIA][LSFDTD_MAX_POLES];
  double c3[LSFDTD_MAX_MEDIA][LSFDTD_MAX_POLES];
  double inv_eps_inf[LSFDTD_MAX_MEDIA];
  const void* h0;
  const void* inv_a;
  const void* w;
  const void* frac;
  void* state;
} lsfdtd_group_desc;

/* Correction points of one kind as a CSR list per target node: entries offsets[t] .. offsets[t+1] of node t
 * are applied in order (a node on two box faces gets both). */
typedef struct {
  int64_t n_nodes;
  const int64_t* nodes;    /* flat E (kind E) or H (kind H) indices */
  const int64_t* offsets;  /* n_nodes + 1 */
  int64_t n_entries;
} lsfdtd_csr;

/* Table-fed TF/SF box (ObliqueLayeredPlaneWave, layered.py:254-482): target += coef * quintic interpolation
 * of the table at fine time (n + i0 + u0) / m; view[3] receives the incident-reference E every step. */
typedef struct {
  const void* table;
  int64_t table_len;
  const void* inc_table;
  int64_t inc_len;
  int32_t m;
  int64_t cmax;
  lsfdtd_csr pts[2];   /* [0]: E targets, [1]: H targets */
  const int64_t* base[2];
  const int64_t* i0[2];
  const void* u0[2];
  const void* coef[2];
  const int64_t* inc_base; /* 3 */
  const int64_t* inc_i0;   /* 3 */
  const void* inc_u0;      /* 3 */
  void* view;              /* device, 3 field-precision scalars */
} lsfdtd_table_source_desc;

/* Point current (PointDipole, emission.py:97-150): E[idx] -= coef * wave[n]. */
typedef struct {
  int32_t n;
  const int64_t* idx;
  const void* coef;
  const void* wave;
  int64_t wave_len;
} lsfdtd_dipole_desc;

/* 1D-fed TF/SF (TFSFPlaneWave, tfsf.py:108-211): line arrays E_line/H_line of M nodes with their update
 * coefficients (full length M), soft source wave at m_src, and the corrections of each kind. */
typedef struct {
  int32_t M, m_src;
  const void* ca;
  const void* cb;
  const void* da;
  const void* db;
  const void* wave;
  int64_t wave_len;
  void* E_line;
  void* H_line;
  lsfdtd_csr pts[2];
  const int64_t* i0[2];
  const void* w[2];
  const void* coef[2];
} lsfdtd_line_source_desc;

/* Bloch column source (BlochPlaneSource, tfsf.py:214-296): `column` is a 3 x 3 x nz engine with the same
 * precision, complex fields and Bloch phases; phase[nx][ny] (complex) maps its field onto the plane. */
typedef struct {
  lsfdtd_engine* column;
  int32_t k_src, k_launch;
  const void* phase;
  double amp[2][2];  /* (re, im) of the E_x and E_y sheet amplitudes */
  const void* wave;
  int64_t wave_len;
  double cE, cH;
} lsfdtd_column_source_desc;

/* Port mode source (ModeSource, ports.py:294-378): H[h_idx] += mH @ tab_E[n], E[e_idx] += mE @ tab_H[n]. */
typedef struct {
  int32_t n_h, r_e;
  const int64_t* h_idx;
  const void* mH;     /* [n_h][r_e] */
  const void* tab_E;  /* [len_E][r_e] */
  int64_t len_E;
  int32_t n_e, r_h;
  const int64_t* e_idx;
  const void* mE;     /* [n_e][r_h] */
  const void* tab_H;  /* [len_H][r_h] */
  int64_t len_H;
} lsfdtd_mode_source_desc;

/* Running-DFT monitor (DFTMonitor, engine.py:194-210): acc_e [n_freq][n_e] and acc_h [n_freq][n_h] are
 * complex128 (interleaved doubles). The sampled arrays are the grid's (space 0), a 1D line's or the
 * incident view's (space 1: real field-precision arrays), or a Bloch column's (space 2). energy: 0, or
 * group 1 / 2 of the decay-energy proxy (monitors without H contribute none, as in the reference). */
typedef struct {
  int32_t n_freq;
  const double* omega;
  int64_t n_e;
  const int64_t* e_idx;
  int64_t n_h;
  const int64_t* h_idx1;
  const int64_t* h_idx2;
  void* acc_e;
  void* acc_h;
  int32_t energy;
  int32_t space;
  const void* E_src;
  const void* H_src;
} lsfdtd_monitor_desc;

int32_t lsfdtd_abi_version(void);
const char* lsfdtd_last_error(void);

/* Stepped range [start, start + len) along `axis` of the CPML slab of `field` (0 E, 1 H), `component`,
 * `side` (0 low, 1 high): the slab's psi array holds the grid with that axis cut to len. */
int32_t lsfdtd_cpml_slab(const int32_t shape[3], const int32_t periodic[3], int32_t axis, int32_t cells_lo,
                         int32_t cells_hi, int32_t field, int32_t component, int32_t side, int32_t* start,
                         int32_t* len);
/* field scalars of state per node of a dispersive group */
int64_t lsfdtd_group_state_len(int32_t mixed, int32_t n_media, const int32_t* n_poles);

int32_t lsfdtd_engine_create(const lsfdtd_grid_desc* grid, lsfdtd_engine** out);
int32_t lsfdtd_engine_destroy(lsfdtd_engine* eng);
int32_t lsfdtd_engine_set_pml(lsfdtd_engine* eng, const lsfdtd_pml_desc* pml);
int32_t lsfdtd_engine_add_group(lsfdtd_engine* eng, const lsfdtd_group_desc* g);

/* Conformal off-diagonal 1/eps terms (Engine._build_offdiag and _update_E, engine.py:421-518, 653-655): row r
 * adds sum_k w[r][k] * H_flat[h[r][k]] to E_flat[e[r]] after each E curl update, before the sources' E
 * corrections. The tables are built on the host (lightsmith_b200/plan.py:offdiag_tables restates the
 * reference's construction). At most one set per engine. */
typedef struct {
  const int64_t* e;  /* device (n): distinct flat E indices */
  const int64_t* h;  /* device (n, width): flat H indices */
  const void* w;     /* device (n, width): weights in the field precision (complex under a Bloch wavevector) */
  int64_t n;
  int32_t width;
} lsfdtd_offdiag_desc;
int32_t lsfdtd_engine_add_offdiag(lsfdtd_engine* eng, const lsfdtd_offdiag_desc* d);

/* The vertex-tensor ADE of conformal interfaces with dispersive media (TensorMesh and _Tensor,
 * engine.py:140-175, 796-923), stepped after the D-form groups, as index tables
 * (lightsmith_b200/plan.py:tensor_plan): nodes (their flat E indices), vertices (each one's six d-node numbers
 * with their phase and parity, and its normal), tensor slots (output position, vertex, vertex * 3 + c, the node
 * position among the vertex's six, the normal's component, the conjugate phase, the vertex's medium fractions)
 * and plain slots (output position, node, medium). Device arrays in the field's (real) precision where not
 * int64; `state` is zeroed, lsfdtd_tensor_state_len() field scalars. At most one mesh per engine. */
typedef struct {
  const int64_t* idx;
  int64_t n_nodes;
  const int64_t* vn;      /* (n_vert * 6) */
  const void* scale;      /* (n_vert * 6) field precision, or NULL (no Bloch phase and no mirror) */
  const void* normal;     /* (n_vert * 3) real */
  int64_t n_vert;
  const int64_t* t_pos;   /* (n_tslots) */
  const int64_t* t_v;
  const int64_t* t_vc;
  const int64_t* t_g;
  const void* t_nc;       /* (n_tslots) real */
  const void* t_conj;     /* (n_tslots) field precision, or NULL for real fields */
  const void* frac;       /* (n_media, n_tslots) real */
  int64_t n_tslots;
  const int64_t* p_pos;   /* (n_pslots) */
  const int64_t* p_node;
  const int64_t* p_medium;
  int64_t n_pslots;
  int32_t n_media;
  int32_t n_poles[LSFDTD_MAX_MEDIA];
  double eps_inf[LSFDTD_MAX_MEDIA];
  double c1[LSFDTD_MAX_MEDIA][LSFDTD_MAX_POLES];
  double c2[LSFDTD_MAX_MEDIA][LSFDTD_MAX_POLES];
  double c3[LSFDTD_MAX_MEDIA][LSFDTD_MAX_POLES];
  void* state;
} lsfdtd_tensor_desc;
int64_t lsfdtd_tensor_state_len(int64_t n_nodes, int64_t n_vert, int64_t n_tslots, int64_t n_pslots,
                                int32_t n_media, const int32_t* n_poles);
int32_t lsfdtd_engine_add_tensor(lsfdtd_engine* eng, const lsfdtd_tensor_desc* d);
/* sources act in the order they are added (Engine.step, engine.py:665-678) */
int32_t lsfdtd_engine_add_table_source(lsfdtd_engine* eng, const lsfdtd_table_source_desc* s);
/* The slab boxes of a table-fed source's H corrections (source `table`, counted among the engine's table
 * sources), for the fused single pass to add them as it steps. lightsmith adds them after the whole H update
 * (ObliqueLayeredPlaneWave.correct_H through apply_fused, backends/_fdtd/layered.py:231-242, 469-476); the
 * fused pass computes H and E plane by plane, so the step's values are computed first (one per correction
 * entry, in the source's slab order) and each H value of a tile gets the values of the boxes that hold it
 * before the E half reads it. boxes: host int32 [n_boxes][8] = component, lo[3], hi[3] (node ranges), offset of
 * the box's first entry; a box's entries are its nodes in row-major order. perm: device int64 [n_entries], the
 * position of each slab-order entry among the entries as given in the source's descriptor (grouped by node);
 * vals: device scratch of n_entries values of the field precision. Before the first step. Without boxes a
 * source with H corrections keeps the in-place kernels. */
int32_t lsfdtd_engine_set_table_boxes(lsfdtd_engine* eng, int32_t table, int32_t n_boxes, const int32_t* boxes,
                                      const int64_t* perm, int64_t n_entries, void* vals);
int32_t lsfdtd_engine_add_dipole(lsfdtd_engine* eng, const lsfdtd_dipole_desc* s);
int32_t lsfdtd_engine_add_line_source(lsfdtd_engine* eng, const lsfdtd_line_source_desc* s);
int32_t lsfdtd_engine_add_column_source(lsfdtd_engine* eng, const lsfdtd_column_source_desc* s);
int32_t lsfdtd_engine_add_mode_source(lsfdtd_engine* eng, const lsfdtd_mode_source_desc* s);
int32_t lsfdtd_engine_add_monitor(lsfdtd_engine* eng, const lsfdtd_monitor_desc* m);
/* bytes of zeroed device scratch the engine needs (a status word, then the monitors' energy partials); set it
 * before the first step */
int32_t lsfdtd_engine_scratch_bytes(lsfdtd_engine* eng, size_t* bytes);
int32_t lsfdtd_engine_set_scratch(lsfdtd_engine* eng, void* scratch, size_t bytes);

/* n_steps time steps (Engine.step, engine.py:665-678), no sample */
int32_t lsfdtd_engine_step(lsfdtd_engine* eng, int32_t n_steps, void* stream);
/* one DFT sample of every monitor (Engine._sample, engine.py:568-592) */
int32_t lsfdtd_engine_sample(lsfdtd_engine* eng, void* stream);
/* n_chunks x (dft_stride steps + one sample) (Engine.chunk, engine.py:680-683). With use_graph, the first
 * call captures one chunk as a CUDA graph on `stream` (which must not be the legacy default stream) and every
 * chunk replays it (Engine.make_runner, engine.py:685-709). */
int32_t lsfdtd_engine_chunk(lsfdtd_engine* eng, int32_t n_chunks, int32_t use_graph, void* stream);
/* Diagnostic: n_chunks eager chunks with CUDA events around every bulk Yee-update kernel; synchronises
 * `stream`, then returns the summed kernel time (ms) and the number of such launches. */
int32_t lsfdtd_engine_chunk_timed(lsfdtd_engine* eng, int32_t n_chunks, void* stream, double* bulk_ms,
                                  int64_t* bulk_launches);
/* which buffer holds the current E/H: 0 the grid's E/H, 1 its E_alt/H_alt */
int32_t lsfdtd_engine_buffer(const lsfdtd_engine* eng);
/* whether steps run as the fused single pass (1) or the in-place H and E kernels (0); valid once the
 * engine is fully described (eligibility is decided at the first step) */
int32_t lsfdtd_engine_fused(lsfdtd_engine* eng);
/* kernel choice and launch shape. variant 0: in-place H and E kernels, one node per thread; variant 2: the
 * same with four-node vector kernels for FP32 rows of a multiple of four nodes (the other arguments are
 * ignored for both). variant 1: the fused single pass where the
 * run allows it (second buffers given, no periodic axis, sources that only correct E): CTA tiles of 32 x
 * tile_y nodes (8 or 16), x planes per tile (>= 1), copy ring of `stages` x planes (4, 6 or 8). variant 3:
 * variant 1 split in two launches where its planes are copied by the Tensor Memory Accelerator: the fused
 * pass over an interior box that needs no region or CPML tests, and shell kernels over the CPML slabs and
 * walls. variant 4: variant 1 with region tests as bit masks and each axis's CPML terms under warp-uniform
 * branches. Variants 3 and 4 compute the values of variant 1 up to the contraction of multiplies and adds
 * into fused multiply-adds. planes 0 chooses per grid: 48, or fewer where 48 would leave fewer than about
 * three waves of CTAs. Default: variant 4, tile_y 8, planes 0, ring 4 (the in-place kernels where the fused
 * pass does not apply). */
int32_t lsfdtd_engine_set_tuning(lsfdtd_engine* eng, int32_t variant, int32_t tile_y, int32_t planes,
                                 int32_t stages);
/* variant 4 with tensor copies: on (the default) steps the clean interior of the grid (the tiles and x planes
 * whose nodes and halo nodes all lie outside every CPML slab and inside every component's stepped region)
 * with a kernel compiled without region or CPML code, on a second stream beside the lean kernel that steps
 * the CTAs around it, where the grid has such an interior and no source corrects H; off steps every CTA with
 * the lean kernel. The values are the same either way. Set before the first graph capture. */
int32_t lsfdtd_engine_set_clean_split(lsfdtd_engine* eng, int32_t on);
/* reads the status word (synchronises `stream`): LSFDTD_ETIMEOUT with *status = 1 if a kernel gave up waiting
 * for its copies, LSFDTD_ENONFINITE with *status = 2 if the run's fields turned non-finite in a batched launch
 * (the run retired then), else LSFDTD_OK */
int32_t lsfdtd_engine_status(lsfdtd_engine* eng, void* stream, int32_t* status);
/* clear the status word on `stream` (after a reported timeout, before the engine's arrays are rebuilt) */
int32_t lsfdtd_engine_clear_status(lsfdtd_engine* eng, void* stream);
/* clock cycles a CTA of the fused pass waits for one plane's copies before it gives up (records the status
 * word, waits a bounded time for its own copies still in flight and returns): the default, about 2 s, when
 * cycles == 0. Negative: a test of that path, in which every wait is on a barrier that nothing completes and
 * gives up after -cycles cycles, while the copies the pass issued still complete and are drained. Set before
 * the first graph capture. */
int32_t lsfdtd_engine_set_wait_budget(lsfdtd_engine* eng, int64_t cycles);
/* whether the fused pass may copy planes with the Tensor Memory Accelerator (default 1); before the first
 * step. With 0, or where the layout rules it out (rows not a multiple of 16 bytes), it uses cp.async. */
int32_t lsfdtd_engine_set_copy_engine(lsfdtd_engine* eng, int32_t use_tma);
/* 1 when steps run the fused pass with TMA copies */
int32_t lsfdtd_engine_uses_tma(lsfdtd_engine* eng);
/* steps completed so far, as the host has launched them */
int64_t lsfdtd_engine_steps(const lsfdtd_engine* eng);

/* One running-DFT sample of one monitor, allocating nothing (no counterpart in lightsmith: its engine samples
 * monitors with array operations of the array library it runs on). For callers that cannot allocate device
 * memory: a host runtime that only lends the library the buffers it owns, or a process whose device memory
 * all comes from one external pool. The caller passes the monitor's inputs (sampled arrays, indices,
 * frequencies) and outputs (accumulators, updated in place) in `m`, the device step counter `step` (the
 * sample time is step * dt, H at half a step earlier) and `energy`, a device double that receives the
 * monitor's sum |E|^2 + |H_avg|^2 when m->energy is set and the monitor has H (else it is left alone).
 * precision / is_complex describe the sampled arrays as for the grid (m->space 1: real arrays).
 * The energy reduction's scratch is a static device array of 8192 doubles (64 KiB, held by every GPU that
 * loads the library until exit): a monitor may span at most 8192 blocks of 256 points (E points and H points
 * rounded up separately), and larger ones are rejected with LSFDTD_EINVAL. The array's device address belongs
 * to the CUDA context that is current at the call (the device's primary context for runtime-API callers, or
 * a caller's own context): the first call in each context looks it up (cudaGetSymbolAddress) and keeps it
 * under that context's unique id, so a context made after cudaDeviceReset, or another context on the same
 * device, gets its own lookup. Make the first call in each context before any stream capture in it.
 * All calls share the array: calls whose GPU work overlaps (for example on two streams) race on it; nothing
 * in it needs clearing between calls. */
int32_t lsfdtd_dft_sample_noalloc(const lsfdtd_monitor_desc* m, int32_t precision, int32_t is_complex,
                                  const int64_t* step, double dt, double* energy, void* stream);
/* kernel launches one chunk issues (for launch accounting) */
int64_t lsfdtd_engine_launches_per_chunk(const lsfdtd_engine* eng);

/* ---- batched Bloch-periodic sweeps ------------------------------------------------------------------
 * Replaces the sequential loop over oblique runs of lightsmith's periodic driver
 * (backends/_fdtd/periodic.py:503-518, each run `_run_oblique`, periodic.py:426-459): many independent runs
 * of uneven grid size advanced by one persistent kernel. Each run is an engine built as usual (complex
 * fields; periodic x and y, CPML along z only; exactly one Bloch column source; no dispersive groups; at
 * most four monitors on the grid or the column). The batch keeps the engines' own device state and step
 * counters: after a batch run each engine is where its own chunks would have left it. */
typedef struct lsfdtd_batch lsfdtd_batch;

/* a batch of n engines of one precision; last[i]: the step count run i stops at (at most what its source
 * waveform covers). The runs are spread over the kernel's CTAs longest first. */
int32_t lsfdtd_batch_create(lsfdtd_engine* const* engines, int32_t n, const int64_t* last, lsfdtd_batch** out);
/* the same with the launch's shape: cluster_ctas CTAs of 512 threads per run and at most max_clusters runs in
 * flight (0: as many as fit). 1 to 16 CTAs: a thread-block cluster per run (above 8 the GPU must allow
 * non-portable clusters). 17 to 4096: a group of CTAs per run that meet at barriers in global memory, in a
 * cooperative launch (every CTA resident at once); a barrier wait is bounded, and a CTA that gives up sets
 * its run's status word to 1 (lsfdtd_engine_status: LSFDTD_ETIMEOUT) and the launch ends. Fewer, larger
 * groups step fewer runs at a time, whose state then stays in L2 through the steps of a launch. 0: the
 * default, groups of half the CTAs resident at once (two runs in flight), which lsfdtd_batch_create takes */
int32_t lsfdtd_batch_create_shaped(lsfdtd_engine* const* engines, int32_t n, const int64_t* last,
                                   int32_t cluster_ctas, int32_t max_clusters, lsfdtd_batch** out);
int32_t lsfdtd_batch_destroy(lsfdtd_batch* batch);
/* device scratch the batch needs (run descriptors and the CTAs' run lists), set once; set_scratch copies
 * the descriptors in (synchronously) */
int32_t lsfdtd_batch_scratch_bytes(const lsfdtd_batch* batch, size_t* bytes);
int32_t lsfdtd_batch_set_scratch(lsfdtd_batch* batch, void* scratch, size_t bytes);
/* n_launches launches of the persistent kernel on `stream`; in each, every run advances `steps` steps (or to
 * its last step), sampling its monitors after every dft_stride steps. use_graph: the launch is captured once
 * as a CUDA graph (per step count) and replayed. */
int32_t lsfdtd_batch_run(lsfdtd_batch* batch, int32_t steps, int32_t n_launches, int32_t use_graph, void* stream);
/* CTAs of the persistent kernel (one wave) */
int32_t lsfdtd_batch_ctas(const lsfdtd_batch* batch);

/* ---- discrete adjoint ----------------------------------------------------------------------------------
 * No counterpart in lightsmith (its FDTD has no gradient): the transpose of one FDTD step of an engine with
 * real fields (periodic axes allowed: their ghost-plane copies are transposed too), no mirror plane and pure
 * (staircase) dispersive groups, for d(objective)/d(E curl coefficient) of a real objective J of one
 * monitor's DFT accumulators (several monitors' points may be concatenated into one). The caller gives J's adjoint source
 * as G = 2 dJ/d(acc) (the Wirtinger derivative: the conjugate of the gradient torch reports for a complex
 * tensor) per frequency and point; the E samples then receive sum_f Re(G_e[f, p] e^{i w_f t}) at each
 * sampled step. */
typedef struct lsfdtd_adjoint lsfdtd_adjoint;

#define LSFDTD_ADJ_MAX_GROUPS 8

typedef struct lsfdtd_adjoint_desc {
  void* Eb;                          /* adjoint fields (3, n0, n1, n2), the engine's precision, zeroed */
  void* Hb;
  void* psi_bar[2][2][3][3][2];      /* [buffer][E, H][axis][component][side]: zeroed slabs shaped as the
                                        engine's psi (null where the engine has none) */
  int32_t box_lo[3], box_hi[3];      /* gradient box, outside every CPML slab and source node */
  void* hist;                        /* hist_slots boxes of H (3, box + 1 along each axis: the low halo) */
  int32_t hist_slots;
  double* grad;                      /* (3, box): dJ/dcbE_c, accumulated */
  const int64_t* e_idx;              /* the objective's E points (flat indices into the fields) */
  const double* ge;                  /* (re, im) per [frequency][E point]: G_e */
  int64_t n_e;
  const int64_t* h_idx1;             /* its H points (the two H samples averaged) */
  const int64_t* h_idx2;
  const double* gh;                  /* (re, im) per [frequency][H point]: G_h */
  int64_t n_h;
  const double* omega;               /* (n_freq) angular frequencies, host memory (copied at create) */
  int32_t n_freq;
  int32_t n_groups;                  /* the engine's dispersive groups, in the order they were added */
  void* group_bar[LSFDTD_ADJ_MAX_GROUPS]; /* adjoint state per group, shaped as its forward state, zeroed */
  /* the engine's conformal off-diagonal terms (lsfdtd_engine_add_offdiag), transposed: row r < od_rows adds
   * sum_{j in [od_ptr[r], od_ptr[r + 1])} od_w[j] Ebar[od_e[j]] to Hbar[od_h[r]], the od_h distinct (device
   * arrays; od_w in the engine's precision). Required, with od_rows > 0, when the engine has such terms. The
   * gradient holds them fixed: it is the derivative with respect to the diagonal coefficients. */
  const int64_t* od_h;
  const int64_t* od_ptr;             /* (od_rows + 1) */
  const int64_t* od_e;
  const void* od_w;
  int64_t od_rows;
  /* the engine's vertex-tensor mesh (lsfdtd_engine_add_tensor), required when it has one: tm_bar its adjoint
   * state, lsfdtd_tensor_state_len scalars laid out as the forward state, zeroed; tm_work 6 n_vert + 2 n_tslots
   * + n_pslots scalars of scratch; the slots by vertex (tm_vs_ptr (n_vert + 1), tm_vs_idx (n_tslots): the
   * tensor slots of vertex v, ascending) and the contributions by node (tm_nd_ptr (n_nodes + 1), tm_nd_src:
   * for node i the positions, ascending, among the 6 n_vert vertex entries (v * 6 + 2 d + side, the node
   * vn[v * 6 + 2 d + side]), then the n_tslots tensor slots (the node vn[t_g[t]]), then the n_pslots plain
   * slots (the node p_node[p]) that read its D). Device arrays, the engine's precision. */
  void* tm_bar;
  void* tm_work;
  const int64_t* tm_vs_ptr;
  const int64_t* tm_vs_idx;
  const int64_t* tm_nd_ptr;
  const int64_t* tm_nd_src;
  /* the objective's adjoint source by target node, in a fixed order (optional; without it each point adds its
   * value with an atomic add, whose order can change the last bit of a node that several points share): the
   * distinct E targets inj_e_tgt (inj_n_e) with, per target r, the E points inj_e_src[inj_e_ptr[r] ..
   * inj_e_ptr[r + 1]] that sample it, ascending; the distinct H targets inj_h_tgt (inj_n_h) with their H points
   * (a point listed once for each of its two samples at the target); inj_work n_e + n_h doubles of scratch */
  const int64_t* inj_e_tgt;
  const int64_t* inj_e_ptr;
  const int64_t* inj_e_src;
  int64_t inj_n_e;
  const int64_t* inj_h_tgt;
  const int64_t* inj_h_ptr;
  const int64_t* inj_h_src;
  int64_t inj_n_h;
  double* inj_work;
} lsfdtd_adjoint_desc;

/* sets the engine's host step count (after the caller rewinds its device counter and fields to a saved step,
 * e.g. a checkpoint of the adjoint's forward recomputation) */
int32_t lsfdtd_engine_set_steps(lsfdtd_engine* eng, int64_t n);
int32_t lsfdtd_adjoint_create(lsfdtd_engine* eng, const lsfdtd_adjoint_desc* d, lsfdtd_adjoint** out);
int32_t lsfdtd_adjoint_destroy(lsfdtd_adjoint* adj);
/* copies the engine's current H over the box (with its low halo) into history slot `slot` */
int32_t lsfdtd_adjoint_record(lsfdtd_adjoint* adj, int32_t slot, void* stream);
/* the transpose of forward step n (E^n, H^{n-1/2} -> E^{n+1}, H^{n+1/2}), H^{n+1/2} of the box in history
 * slot `slot`: adds the objective's adjoint source when the monitor sampled after that step, then the
 * transposes of the E and H updates, and accumulates the gradient */
int32_t lsfdtd_adjoint_step(lsfdtd_adjoint* adj, int64_t n, int32_t slot, void* stream);

/* ---- host set-up on the GPU: material on the Yee E grid from particle shapes ----------------------------------
 * Replaces the per-point work of lightsmith's voxelise (backends/_fdtd/setup.py:110-289) for the scenes of its
 * scattering driver: particles (spec.py:28-122: sphere, spheroid, cylinder, layered sphere, each at a position,
 * the first listed winning overlaps, setup.py:707-716) over a host medium, optionally above a substrate
 * (scattering.py:81-90). The caller assembles inv_eps, the dispersive groups and the off-diagonal terms from
 * the three results as voxelise does (lightsmith_b200/voxel.py). Every array is device memory. */
#define LSFDTD_VOX_MAX_REGIONS 8
#define LSFDTD_VOX_MAX_MEDIA 16
enum { LSFDTD_VOX_SPHERE = 0, LSFDTD_VOX_SPHEROID = 1, LSFDTD_VOX_CYLINDER = 2, LSFDTD_VOX_LAYERED_SPHERE = 3 };
enum { LSFDTD_VOX_STAIRCASE = 0, LSFDTD_VOX_VOLUME_AVERAGE = 1, LSFDTD_VOX_SUBPIXEL = 2, LSFDTD_VOX_CONFORMAL = 3 };

typedef struct {
  int32_t kind;       /* LSFDTD_VOX_* shape */
  int32_t n_regions;  /* 1, or the core and shells of a layered sphere */
  double pos[3];      /* centre, nm */
  double a, b;        /* sphere: radius; spheroid: semi-axes xy and z; cylinder: radius and length (along z) */
  double radii[LSFDTD_VOX_MAX_REGIONS];  /* layered sphere: outer radius of each region, ascending */
  int32_t slot[LSFDTD_VOX_MAX_REGIONS];  /* medium slot of each region */
} lsfdtd_vox_particle;

typedef struct {
  int32_t n_particles;
  const lsfdtd_vox_particle* particles;  /* device array */
  int32_t has_substrate;                 /* points below z_int that no particle holds take sub_slot */
  double z_int;
  int32_t sub_slot;
  double origin[3], dx[3];               /* node (0, 0, 0) and the cell size, nm */
  int32_t shape[3];
  int32_t roi_lo[3], roi_hi[3];          /* the nodes examined */
} lsfdtd_vox_scene;

typedef struct {
  int32_t n;        /* media: slots 0 .. n - 1 (0 the host medium) */
  int32_t samples;  /* supersamples per axis of an interface cell */
  int32_t mode;     /* LSFDTD_VOX_* mesh refinement */
  double eps_inf[LSFDTD_VOX_MAX_MEDIA];
  int8_t dispersive[LSFDTD_VOX_MAX_MEDIA];
  int8_t background[LSFDTD_VOX_MAX_MEDIA];  /* media of a layered background filled beforehand */
} lsfdtd_vox_media;

typedef struct {  /* per interface cell q of n */
  double* frac;     /* [s * n + q] fraction of medium s */
  double* nhat;     /* [3 q + d] unit normal (first moment of the dominant medium), zero when undefined */
  double* w;        /* [q] n_c^2, 1/3 without a normal, 0 for volume averaging */
  int8_t* part;     /* [q] holds a medium outside the background set */
  int8_t* has_disp; /* [q] holds a dispersive medium */
  double* inv;      /* [q] smoothed 1/eps_cc (w <1/eps> + (1 - w) / <eps>) */
  double* od;       /* [3 q + d] off-diagonal terms n_d n_c (<1/eps> - 1/<eps>), column c zero */
} lsfdtd_vox_cells;

/* the medium slot at every point of the half-cell lattice origin + (m / 2) dx, m from 2 roi_lo - 1 to 2 roi_hi
 * per axis: (2 n0 + 2) x (2 n1 + 2) x (2 n2 + 2) int16 values (n_a = roi_hi - roi_lo), row-major
 * (setup.py:276-289, _half_lattice) */
int32_t lsfdtd_vox_lattice(const lsfdtd_vox_scene* scene, int16_t* lattice, void* stream);
/* per node of the region (row-major from roi_lo) for E component c: the slot of its E_c position, or -1 where
 * subpixel != 0 and a corner or edge midpoint of its cell holds another slot (setup.py:153-177) */
int32_t lsfdtd_vox_classify(const lsfdtd_vox_scene* scene, const int16_t* lattice, int32_t c, int32_t subpixel,
                            int16_t* cls, void* stream);
/* per interface cell (cells[q]: row-major node index of the region, component c): the supersampled fractions,
 * normal, weight and smoothed 1/eps (setup.py:190-234) */
int32_t lsfdtd_vox_supersample(const lsfdtd_vox_scene* scene, const lsfdtd_vox_media* media, int32_t c,
                               const int64_t* cells, int64_t n, lsfdtd_vox_cells out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
