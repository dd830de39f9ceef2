// fdtd_api.cu - the C ABI (include/fdtd_b200.h): context, device memory,
// uploads/downloads and the per-time-step launch sequence.
//
// The step sequence mirrors Scheme::performNStepsForBlock
// (Source/Scheme/Scheme.inc.h:28-473): incident E step, E half-step (skipped
// at t == 0, Scheme.inc.h:1032), E point sources, incident H step, H
// half-step, H point sources.  Time levels of the plain form rotate as
// pointers on the host (Grid::shiftInTime, Source/Grid/Grid.h:1304-1319);
// the fused forms update in place.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fdtd_b200.h"
#include "adjoint.h"
#include "fused3d.h"
#include "sweep2.h"
#include "tfsf2.h"
#include "sweep3d.h"
#include "kernels.h"
#include "ntff.h"
#include "setup.h"

using namespace fdtdb;

namespace {

constexpr double kEta0 = 376.730313461770655;  // sqrt(mu0/eps0) for the reference constants
// per time step on the host and the device: incident-grid source, point
// source on E and on H, J and M current
constexpr int kSrcStride = 5;

thread_local std::string g_last_error;

// device / pinned allocations that still succeed before the injected
// failures of fdtd_inject_alloc_failure (-1: no injection)
std::atomic<long long> g_alloc_budget{-1};

int kind_of (int prec)
{
  return prec == FDTD_PREC_FP64_PLAIN ? 0 : (prec == FDTD_PREC_FP32 ? 1 : 2);
}

size_t elem_size (int kind)
{
  return kind == 0 ? 8 : (kind == 1 ? 4 : 2);
}

}  // namespace

struct fdtd_ctx
{
  Geometry g;
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  int prec = 0;
  int kind = 0;
  int64_t launches = 0;
  int *d_err = nullptr;
  double eta0 = 1.0;

  // incident grids (FP64 in every form); cur = index of level 1
  double *einc[2] = {nullptr, nullptr};
  double *hinc[2] = {nullptr, nullptr};
  int ecur = 0, hcur = 0;

  // per-step source table: [incident, point source E, point source H]
  double *d_src = nullptr;
  double *h_src = nullptr;
  size_t src_cap = 0;
  cudaEvent_t src_ev = nullptr;

  // plain form
  double *f[6][3] = {};
  double *dd[6][3] = {};
  double *d1[6][3] = {};
  double *mat64[6] = {};
  double *sig64[3] = {};
  double *ptab[6][6] = {};   // FP64 plain form: PML coefficient tables per component (PlainTabs)
  // double material precision: eps / mu per component averaged from the fine
  // grid at upload (null until then), sigma per component and axis, and the
  // fine upload buffer
  double *matc64[6] = {};
  float *matc32[6] = {};
  double *sigc64[6][3] = {};
  double *fine_tmp = nullptr;
  AdjointCache adj_cache;      // the adjoint's device memory, kept between calls
  SweepStreams sweep_streams;  // side streams of the sweep's item classes
  // asynchronous host copies: a host-to-device and a device-to-host copy
  // stream, their FP64 staging grids, and the events that order them against
  // the context's stream (an event never recorded is complete)
  cudaStream_t h2d = nullptr, d2h = nullptr;
  double *stage_in = nullptr, *stage_out = nullptr;
  cudaEvent_t in_ready = nullptr, in_free = nullptr, out_ready = nullptr, out_free = nullptr;

  // fused forms: two buffer sets; set fcur holds the current time level.
  // The per-cell path updates set fcur in place; the one-sweep 3-D kernel
  // reads set fcur and writes set 1 - fcur.
  void *ffb[2][6] = {};
  float *auxb[2][6] = {};
  int fcur = 0;
  bool has_second = false;
  void *ff[6] = {};
  float *aux[6] = {};
  float *mat32[2] = {};
  float *drude32[4] = {};                 // omegape, omegapm, gammae, gammam (FP32)
  unsigned char *dflag = nullptr;
  float *xppb[2][6] = {}, *zb[2][6] = {}, *zppb[2][6] = {};
  float *tabs = nullptr;
  size_t tab_off[6][6] = {};
  FastHalf fast_e, fast_h;
  FusedParams fused;
  bool ps_interior = true;
  int cs_mask[2] = {0, 0};     // per family: bit ci = current source on component ci (interior cells only)
  int cs_pos[3] = {0, 0, 0};   // its cell (0 on an axis the mode drops)
  // TMA-pipelined one-sweep kernel: plan built at the first step (and again
  // when the permittivity buffer appears); state 0 = not built, 1 = in use,
  // -1 = not applicable (the register-blocked kernel runs instead)
  SweepPlan sweep;
  int sweep_state = 0;
  const float *sweep_eps = nullptr;
  unsigned long long *sweep_ctr = nullptr;
  std::string sweep_why;
  const char *step_kernel = "not_stepped";
  // two-step (temporally blocked) sweep: used for pairs of steps when it can
  // serve the geometry (tb2_state 1), planned with the single-step sweep
  Sweep2Plan tb2;
  int tb2_state = 0;           // 1: whole grid two-step; 2: two-step core + PML shell in single steps
  std::string tb2_why;
  unsigned long long *tb2_ctr = nullptr;
  // PML shell of the two-step scheme (tb2_state 2): the x / y PML slabs with
  // a 2-cell margin advance by two single steps (step 1 into the third
  // buffer set T over the shell and one more cell, step 2 from T), while the
  // two-step kernel advances the core on its own stream
  SweepPlan shell1, shell2;
  int *shell_list[2] = {nullptr, nullptr};
  unsigned long long *shell_ctr[2] = {nullptr, nullptr};
  void *tfb[6] = {};                      // set T: fields
  float *tauxb[6] = {};                   // set T: PML auxiliaries
  cudaStream_t core_stream = nullptr;
  cudaEvent_t core_fork = nullptr, core_join = nullptr;
  // incident-grid steps of a pair beside the shell and the core
  cudaStream_t inc_stream = nullptr;
  cudaEvent_t inc_free = nullptr, inc_done = nullptr;
  // TF/SF with the two-step scheme: the pair's corrections (tfsf2.cu), and a
  // copy of the incident H level the first step's E corrections read (the
  // second step's H-incident update overwrites it)
  Tf2Pass tf2;
  bool tf2_on = false;
  bool stepped = false;   // a field update has run (the Drude state has a form)
  // FP32 / FP16: keep the previous field level after every fdtd_step call
  // (the NTFF averages H over two levels).  prev_src: where the previous H
  // level is after the last call: 0 nowhere, 1 buffer set 1 - fcur, 2 hprev
  bool keep_prev = false;
  int prev_src = 0;
  void *hprev[3] = {nullptr, nullptr, nullptr};
  long long tf2_cells[4] = {0, 0, 0, 0};   // cells and boxes of each pass's region (verbose plan print)
  int tf2_boxes[4] = {0, 0, 0, 0};
  double *hinc_keep = nullptr;
  TfsfBand band;                          // TF/SF post pass of the sweep (band.cells > 0 when in use)
  std::vector<BandBox> band_host;         // its boxes, on the host
  // metamaterials with the sweep: the box of the Drude cells, fixed up after
  // each sweep step (drude_fix), and its device scratch
  bool drude_fix = false;
  DrudeBox drude_box{};
  int *drude_box_dev = nullptr;

  // running DFT of one component on one plane (dft_comp < 0: none)
  int dft_comp = -1, dft_axis = 0, dft_index = 0, dft_nf = 0;
  std::vector<double> dft_freq;
  double *dft_acc = nullptr;              // (re, re comp., im, im comp.) per frequency and plane cell
  double *dft_phase = nullptr;            // per step of the current fdtd_step call: (cos, sin) per frequency
  size_t dft_phase_cap = 0;               // steps the phase table holds
  std::vector<double> h_dft_phase;

  double *staging = nullptr;
  unsigned long long *d_first_bad = nullptr;   // index of a non-finite material value (check on upload)
  long long wait_limit_ns = 0;                 // grid-barrier wait limit of the adjoint (<= 0: default)
  double *partials = nullptr;
  double *d_out = nullptr;
  int nparts = 0;

  std::vector<void *> allocs;

  // field-kernel timing
  bool profiling = false;
  std::vector<cudaEvent_t> prof_events;   // pairs (start, end)
  size_t prof_used = 0;                   // events used since the last read
};

namespace {

int fail (fdtd_ctx *ctx, int code, const std::string &msg)
{
  (void) ctx;
  g_last_error = msg;
  return code;
}

#define CK(call)                                                                                   \
  do                                                                                               \
  {                                                                                                \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return fail (ctx, e_ == cudaErrorMemoryAllocation ? FDTD_ERR_NOMEM : FDTD_ERR_CUDA,          \
                   std::string (#call) + ": " + cudaGetErrorString (e_));                           \
  } while (0)

int dalloc (fdtd_ctx *ctx, void **p, size_t bytes, bool zero = true)
{
  cudaError_t e = device_malloc (p, bytes ? bytes : 16);
  if (e != cudaSuccess)
  {
    *p = nullptr;
    return fail (ctx, FDTD_ERR_NOMEM, std::string ("cudaMalloc: ") + cudaGetErrorString (e));
  }
  ctx->allocs.push_back (*p);
  if (zero)
  {
    e = cudaMemsetAsync (*p, 0, bytes ? bytes : 16, ctx->stream);
    if (e != cudaSuccess)
      return fail (ctx, FDTD_ERR_CUDA, std::string ("cudaMemset: ") + cudaGetErrorString (e));
  }
  return FDTD_OK;
}

#define DALLOC(ptr, bytes)                                                                         \
  do                                                                                               \
  {                                                                                                \
    int r_ = dalloc (ctx, (void **) &(ptr), (bytes));                                              \
    if (r_ != FDTD_OK)                                                                             \
      return r_;                                                                                   \
  } while (0)

GeomDev make_geom_dev (const Geometry &g)
{
  GeomDev d;
  std::memset (&d, 0, sizeof (d));
  for (int a = 0; a < 3; ++a)
    d.n[a] = g.n[a];
  d.drop = g.drop;
  for (int j = 0; j < 2; ++j)
  {
    d.inc_ax[j] = g.inc_ax[j];
    d.inc_k[j] = g.inc_k[j];
  }
  d.dt = g.dt;
  d.dx = g.dx;
  d.s1 = g.s1;
  d.c1 = g.c1;
  d.s2 = g.s2;
  d.c2 = g.c2;
  for (int a = 0; a < 3; ++a)
    d.zero_inc[a] = g.zero_inc[a];
  for (int k = 0; k < 6; ++k)
  {
    d.proj[k] = g.proj[k];
    for (int a = 0; a < 3; ++a)
      d.min_fp[k][a] = g.comp[k].min_fp[a];
  }
  return d;
}

CompDev make_comp_dev (const Geometry &g, int k)
{
  CompDev c;
  std::memset (&c, 0, sizeof (c));
  const CompLayout &l = g.comp[k];
  c.exists = l.exists ? 1 : 0;
  int base = k >= 3 ? 0 : 3;
  c.opp1 = l.opp1 - base;
  c.opp2 = l.opp2 - base;
  for (int a = 0; a < 3; ++a)
  {
    c.d11[a] = l.d11[a];
    c.d12[a] = l.d12[a];
    c.d21[a] = l.d21[a];
    c.d22[a] = l.d22[a];
  }
  c.sig_cacb = l.sig_cacb;
  c.sig4 = l.sig4;
  c.sig5 = l.sig5;
  // double material precision: the material and sigma arrive pre-averaged
  // per component, a one-point stencil
  c.nmat = g.dmp ? 1 : l.nmat;
  for (int j = 0; j < 4; ++j)
    for (int a = 0; a < 3; ++a)
      c.m[j][a] = g.dmp ? 0 : l.m[j][a];
  c.nterms = 0;
  for (const TfsfTerm &t : g.tfsf)
  {
    if (t.comp != k || c.nterms >= kMaxTerms)
      continue;
    TermDev &d = c.term[c.nterms++];
    for (int a = 0; a < 3; ++a)
    {
      d.lo[a] = t.lo[a];
      d.hi[a] = t.hi[a];
      d.aux[a] = t.aux[a];
    }
    d.slot = t.slot;
    d.inc_comp = t.inc_comp;
    d.negate = t.negate;
  }
  return c;
}


}  // namespace

namespace {

int set_device (fdtd_ctx *ctx)
{
  CK (cudaSetDevice (ctx->device));
  return FDTD_OK;
}

int ensure_staging (fdtd_ctx *ctx)
{
  if (!ctx->staging)
    DALLOC (ctx->staging, (size_t) ctx->g.cells * sizeof (double));
  return FDTD_OK;
}

int ensure_copy_streams (fdtd_ctx *ctx)
{
  if (!ctx->h2d)
  {
    CK (cudaStreamCreateWithFlags (&ctx->h2d, cudaStreamNonBlocking));
    CK (cudaStreamCreateWithFlags (&ctx->d2h, cudaStreamNonBlocking));
    for (cudaEvent_t *e : {&ctx->in_ready, &ctx->in_free, &ctx->out_ready, &ctx->out_free})
      CK (cudaEventCreateWithFlags (e, cudaEventDisableTiming));
  }
  if (!ctx->stage_in)
    DALLOC (ctx->stage_in, (size_t) ctx->g.cells * sizeof (double));
  if (!ctx->stage_out)
    DALLOC (ctx->stage_out, (size_t) ctx->g.cells * sizeof (double));
  return FDTD_OK;
}

// cudaSuccess once the context's stream and both copy streams are idle
cudaError_t query_all (fdtd_ctx *ctx)
{
  cudaStream_t s[3] = {ctx->stream, ctx->h2d, ctx->d2h};
  for (cudaStream_t q : s)
  {
    if (!q)
      continue;
    cudaError_t e = cudaStreamQuery (q);
    if (e != cudaSuccess)
      return e;
  }
  return cudaSuccess;
}

int ensure_src (fdtd_ctx *ctx, size_t steps)
{
  if (steps > ctx->src_cap)
  {
    CK (cudaStreamSynchronize (ctx->stream));
    if (ctx->d_src)
    {
      auto it = std::find (ctx->allocs.begin (), ctx->allocs.end (), (void *) ctx->d_src);
      if (it != ctx->allocs.end ())
        ctx->allocs.erase (it);
      cudaFree (ctx->d_src);
      ctx->d_src = nullptr;
    }
    if (ctx->h_src)
    {
      cudaFreeHost (ctx->h_src);
      ctx->h_src = nullptr;
    }
    size_t cap = std::max<size_t> (steps, 1024);
    DALLOC (ctx->d_src, cap * kSrcStride * sizeof (double));
    CK (pinned_malloc ((void **) &ctx->h_src, cap * kSrcStride * sizeof (double)));
    ctx->src_cap = cap;
  }
  else
  {
    CK (cudaEventSynchronize (ctx->src_ev));
  }
  return FDTD_OK;
}

PlainHalf plain_half (fdtd_ctx *ctx, int h);

int alloc_plain (fdtd_ctx *ctx)
{
  const Geometry &g = ctx->g;
  size_t nb = (size_t) g.cells * sizeof (double);
  for (int k = 0; k < 6; ++k)
  {
    if (!g.comp[k].exists)
      continue;
    for (int l = 0; l < g.levels; ++l)
    {
      DALLOC (ctx->f[k][l], nb);
      if (g.cfg.use_pml)
        DALLOC (ctx->dd[k][l], nb);
      if (g.cfg.use_metamaterials)
        DALLOC (ctx->d1[k][l], nb);
    }
  }
  int nmat = g.cfg.use_metamaterials ? 6 : 2;
  for (int m = 0; m < nmat; ++m)
  {
    DALLOC (ctx->mat64[m], nb);
    if (m < 2)
      ctx->launches += launch_fill (ctx->mat64[m], (size_t) g.cells, 1.0, ctx->stream);
  }
  for (int a = 0; a < 3; ++a)
  {
    DALLOC (ctx->sig64[a], g.sigma[a].size () * sizeof (double));
    CK (cudaMemcpyAsync (ctx->sig64[a], g.sigma[a].data (), g.sigma[a].size () * sizeof (double),
                         cudaMemcpyHostToDevice, ctx->stream));
  }
  if (g.dmp)
  {
    for (int k = 0; k < 6; ++k)
    {
      if (!g.comp[k].exists)
        continue;
      for (int a = 0; a < 3; ++a)
      {
        std::vector<double> s = sigma_at (g, k, a);
        DALLOC (ctx->sigc64[k][a], s.size () * sizeof (double));
        CK (cudaMemcpyAsync (ctx->sigc64[k][a], s.data (), s.size () * sizeof (double), cudaMemcpyHostToDevice,
                             ctx->stream));
        CK (cudaStreamSynchronize (ctx->stream));
      }
    }
  }
  // PML coefficient tables of the per-component kernels (computed on the
  // device by the per-cell expressions)
  if (g.cfg.use_pml)
  {
    const int nmax = std::max (g.n[0], std::max (g.n[1], g.n[2]));
    for (int k = 0; k < 6; ++k)
      if (g.comp[k].exists)
        for (int j = 0; j < 6; ++j)
          DALLOC (ctx->ptab[k][j], (size_t) nmax * sizeof (double));
    for (int h = 0; h < 2; ++h)
    {
      const PlainHalf p = plain_half (ctx, h);
      double *out[3][6];
      for (int ci = 0; ci < 3; ++ci)
        for (int j = 0; j < 6; ++j)
          out[ci][j] = ctx->ptab[ci + 3 * h][j];
      ctx->launches += launch_plain_tables (p, out, ctx->stream);
    }
    CK (cudaGetLastError ());
  }
  CK (cudaStreamSynchronize (ctx->stream));
  return FDTD_OK;
}

// Double material precision: eps (which 0) or mu (which 1) on the fine grid,
// from host or device memory, averaged into every component of its family.
int upload_fine_material (fdtd_ctx *ctx, int which, const double *src, cudaMemcpyKind kind)
{
  const Geometry &g = ctx->g;
  if (!ctx->fine_tmp)
    DALLOC (ctx->fine_tmp, (size_t) g.fine_cells * sizeof (double));
  CK (cudaMemcpyAsync (ctx->fine_tmp, src, (size_t) g.fine_cells * sizeof (double), kind, ctx->stream));
  FineAvg a;
  std::memset (&a, 0, sizeof (a));
  for (int b = 0; b < 3; ++b)
  {
    a.n[b] = g.n[b];
    a.nf[b] = g.nf[b];
    a.mul[b] = ((g.drop >> b) & 1) ? 0 : 2;
  }
  const size_t n = (size_t) g.cells;
  for (int ci = 0; ci < 3; ++ci)
  {
    const int k = ci + 3 * which;
    if (!g.comp[k].exists)
      continue;
    std::memcpy (a.off, g.fine_off[k], sizeof (a.off));
    if (ctx->kind == 0)
    {
      if (!ctx->matc64[k])
        DALLOC (ctx->matc64[k], n * sizeof (double));
      ctx->launches += launch_fine_average (ctx->fine_tmp, ctx->matc64[k], nullptr, a, ctx->sm_count, ctx->stream);
    }
    else
    {
      if (!ctx->matc32[k])
        DALLOC (ctx->matc32[k], n * sizeof (float));
      ctx->launches += launch_fine_average (ctx->fine_tmp, nullptr, ctx->matc32[k], a, ctx->sm_count, ctx->stream);
    }
  }
  CK (cudaGetLastError ());
  CK (cudaStreamSynchronize (ctx->stream));
  return FDTD_OK;
}

int alloc_fast (fdtd_ctx *ctx)
{
  const Geometry &g = ctx->g;
  size_t n = (size_t) g.cells;
  // the one-sweep 3-D kernels (register-blocked and TMA) are written for the
  // E_CENTERED stencil on cell-centred materials; H_CENTERED, double material
  // precision and the 2-D / 1-D modes run the per-cell kernels on one buffer set
  ctx->has_second = g.drop == 0 && g.cfg.layout == 0 && !g.dmp;
  for (int b = 0; b < (ctx->has_second ? 2 : 1); ++b)
  {
    for (int k = 0; k < 6; ++k)
    {
      if (!g.comp[k].exists)
        continue;
      DALLOC (ctx->ffb[b][k], n * elem_size (ctx->kind));
      if (g.cfg.use_pml)
        DALLOC (ctx->auxb[b][k], n * sizeof (float));
    }
  }
  for (int k = 0; k < 6; ++k)
  {
    ctx->ff[k] = ctx->ffb[0][k];
    ctx->aux[k] = ctx->auxb[0][k];
  }
  if (g.cfg.use_metamaterials)
  {
    for (int m = 0; m < 4; ++m)
      DALLOC (ctx->drude32[m], n * sizeof (float));
    DALLOC (ctx->dflag, n);
    for (int b = 0; b < 2; ++b)
      for (int k = 0; k < 6; ++k)
      {
        DALLOC (ctx->xppb[b][k], n * sizeof (float));
        DALLOC (ctx->zb[b][k], n * sizeof (float));
        DALLOC (ctx->zppb[b][k], n * sizeof (float));
      }
  }
  // 1-D coefficient tables per component (see fast_kernels.cu)
  std::vector<float> tabs;
  const double S = kC * g.dt / g.dx;
  for (int k = 0; k < 6; ++k)
  {
    const CompLayout &c = g.comp[k];
    if (!c.exists)
      continue;
    int axes[6] = {c.sig_cacb, c.sig_cacb, c.sig5, c.sig5, c.sig4, c.sig4};
    for (int j = 0; j < 6; ++j)
    {
      std::vector<double> s = sigma_at (g, k, axes[j]);
      ctx->tab_off[k][j] = tabs.size ();
      for (double sv : s)
      {
        double r = sv * g.dt / (2 * kEps0);
        double v;
        switch (j)
        {
          case 0: v = (1 - r) / (1 + r); break;
          case 1: v = S / (1 + r); break;
          case 2: v = (1 - r) / (1 + r); break;
          case 3: v = 1 / (1 + r); break;
          case 4: v = 1 + r; break;
          default: v = 1 - r; break;
        }
        tabs.push_back ((float) v);
      }
    }
  }
  DALLOC (ctx->tabs, tabs.size () * sizeof (float));
  CK (cudaMemcpyAsync (ctx->tabs, tabs.data (), tabs.size () * sizeof (float), cudaMemcpyHostToDevice, ctx->stream));

  for (int h = 0; h < 2; ++h)
  {
    FastHalf &p = h ? ctx->fast_h : ctx->fast_e;
    std::memset (&p, 0, sizeof (p));
    p.g = make_geom_dev (g);
    p.is_h = h;
    p.use_pml = g.cfg.use_pml;
    p.use_tfsf = g.cfg.use_tfsf;
    p.fp16 = ctx->kind == 2;
    p.courant = (float) S;
    for (int k = 0; k < 6; ++k)
      p.inc_scale[k] = (float) (k >= 3 ? kEta0 : 1.0);
    p.inc_len = g.inc_len;
    p.cs_mask = ctx->cs_mask[h];
    for (int a = 0; a < 3; ++a)
      p.cs[a] = ctx->cs_pos[a];
    p.cs_scale = (float) (h ? 1.0 : kEta0);
    p.meta = g.cfg.use_metamaterials && g.cfg.use_pml;
    p.dt = (float) g.dt;
    p.om = ctx->drude32[h];       // omegape (E) / omegapm (H)
    p.ga = ctx->drude32[2 + h];   // gammae (E) / gammam (H)
    for (int ci = 0; ci < 3; ++ci)
    {
      int k = ci + 3 * h;
      p.xpp[ci] = ctx->xppb[0][k];
      p.zd[ci] = ctx->zb[0][k];
      p.zpp[ci] = ctx->zppb[0][k];
      p.comp[ci] = make_comp_dev (g, k);
      p.f[ci] = ctx->ff[k];
      p.aux[ci] = ctx->aux[k];
      p.opp[ci] = ctx->ff[ci + 3 * (1 - h)];
      const CompLayout &c = g.comp[k];
      for (int j = 0; j < 6; ++j)
        p.tab[ci][j] = c.exists ? ctx->tabs + ctx->tab_off[k][j] : nullptr;
      for (int a = 0; a < 3; ++a)
      {
        std::vector<double> s = sigma_at (g, k, a);
        int lo = 0, hi = g.n[a];
        if (g.cfg.use_pml)
        {
          lo = 0;
          while (lo < g.n[a] && s[lo] != 0.0)
            ++lo;
          hi = lo;
          while (hi < g.n[a] && s[hi] == 0.0)
            ++hi;
        }
        p.ilo[ci][a] = lo;
        p.ihi[ci][a] = hi;
      }
    }
  }
  CK (cudaStreamSynchronize (ctx->stream));
  return FDTD_OK;
}

// Points ff/aux and the per-cell kernel parameters at buffer set fcur.
void select_fast_set (fdtd_ctx *ctx)
{
  for (int k = 0; k < 6; ++k)
  {
    ctx->ff[k] = ctx->ffb[ctx->fcur][k];
    ctx->aux[k] = ctx->auxb[ctx->fcur][k];
  }
  for (int h = 0; h < 2; ++h)
  {
    FastHalf &p = h ? ctx->fast_h : ctx->fast_e;
    for (int ci = 0; ci < 3; ++ci)
    {
      p.f[ci] = ctx->ff[ci + 3 * h];
      p.aux[ci] = ctx->aux[ci + 3 * h];
      p.opp[ci] = ctx->ff[ci + 3 * (1 - h)];
      p.xpp[ci] = ctx->xppb[ctx->fcur][ci + 3 * h];
      p.zd[ci] = ctx->zb[ctx->fcur][ci + 3 * h];
      p.zpp[ci] = ctx->zppb[ctx->fcur][ci + 3 * h];
    }
  }
}

void init_fused (fdtd_ctx *ctx)
{
  const Geometry &g = ctx->g;
  FusedParams &f = ctx->fused;
  std::memset (&f, 0, sizeof (f));
  f.g = make_geom_dev (g);
  f.use_pml = g.cfg.use_pml;
  f.use_tfsf = g.cfg.use_tfsf;
  f.fp16 = ctx->kind == 2;
  f.courant = ctx->fast_e.courant;
  for (int k = 0; k < 6; ++k)
  {
    f.inc_scale[k] = ctx->fast_e.inc_scale[k];
    f.comp[k] = make_comp_dev (g, k);
    const FastHalf &h = k >= 3 ? ctx->fast_h : ctx->fast_e;
    for (int j = 0; j < 6; ++j)
      f.tab[k][j] = h.tab[k % 3][j];
    for (int a = 0; a < 3; ++a)
    {
      f.ilo[k][a] = h.ilo[k % 3][a];
      f.ihi[k][a] = h.ihi[k % 3][a];
    }
  }
  // TF/SF face planes for the kernel's quick rejection: every term box is
  // one cell thick along some axis; a cell can only need a correction when
  // its coordinate equals one of those planes
  int nf[3] = {0, 0, 0};
  for (int a = 0; a < 3; ++a)
    for (int j = 0; j < 4; ++j)
      f.face[a][j] = -1;
  bool overflow = false;
  for (const TfsfTerm &t : g.tfsf)
  {
    int best = 0;
    for (int a = 1; a < 3; ++a)
      if (t.hi[a] - t.lo[a] < t.hi[best] - t.lo[best])
        best = a;
    if (t.hi[best] - t.lo[best] != 1)
    {
      overflow = true;
      continue;
    }
    bool seen = false;
    for (int j = 0; j < nf[best]; ++j)
      seen = seen || f.face[best][j] == t.lo[best];
    if (seen)
      continue;
    if (nf[best] == 4)
    {
      overflow = true;
      continue;
    }
    f.face[best][nf[best]++] = t.lo[best];
  }
  if (overflow)
  {
    // no quick rejection possible: make every y coordinate a face plane
    // would need more slots, so fall back to the per-cell kernel instead
    ctx->has_second = false;
  }
  f.inc_len = g.inc_len;
  // tile / occupancy variant of the register-blocked one-sweep kernel
  // (shape 3 measured fastest)
  f.shape = 3;
  int tyv = fused_rows_per_cta (f.shape);
  int tiles = ((g.n[2] - 2 + 30) / 31) * ((g.n[1] - 2 + tyv - 1) / tyv);
  int64_t want = (int64_t) ctx->sm_count * 8 * 4;
  int64_t chunk = ((int64_t) (g.n[0] - 2) * tiles) / std::max<int64_t> (want, 1);
  f.x_chunk = (int) std::min<int64_t> (128, std::max<int64_t> (16, chunk));
  const int *ps = g.cfg.point_source;
  f.ps_mask = g.cfg.point_source_mask;
  for (int a = 0; a < 3; ++a)
    f.ps[a] = ps[a];
  ctx->ps_interior = true;
  if (f.ps_mask)
    for (int a = 0; a < 3; ++a)
      ctx->ps_interior = ctx->ps_interior && ps[a] >= 1 && ps[a] <= g.n[a] - 2;
  f.ps_scale_h = (float) kEta0;
  f.use_meta = g.cfg.use_metamaterials;
  f.dt = (float) g.dt;
  f.dflag = ctx->dflag;
  f.omega[0] = ctx->drude32[0];
  f.omega[1] = ctx->drude32[1];
  f.gamma[0] = ctx->drude32[2];
  f.gamma[1] = ctx->drude32[3];
}

// x chunk of the TMA sweep: every item streams its planes plus one halo
// plane, one recomputed E plane and about two planes' worth of pipeline fill
// (measured: 64-plane chunks beat 48 by 2 % at 512^3) over the persistent
// CTAs, and the last item to start sets the tail; ties go to the shorter
// chunk.  `overlap`
// class launches in flight together (side streams) share the tail: only
// the last one's is exposed.
int sweep_chunk (const FusedParams &p, int wy, int ctas, int overlap)
{
  static const int cand[] = {16, 24, 32, 48, 64};
  int best = 32;
  double best_t = 1e300;
  for (int c : cand)
  {
    SweepWork w{};
    sweep3d_items (p, wy, c, w);
    double planes = 0;
    for (int j = 0; j < w.nch; ++j)
      planes += w.xcut[j + 1] - w.xcut[j] + 4;
    const double t = planes * w.nzt * w.nyt / std::max (ctas, 1) + (w.chunk + 4) / (double) std::max (overlap, 1);
    if (t < best_t * 0.999)
    {
      best_t = t;
      best = c;
    }
  }
  return best;
}

// x chunk of the two-step sweep; FDTDB_TB2_CHUNK overrides it (a test hook:
// short chunks put chunk seams into small grids)
int tb2_chunk ()
{
  if (const char *v = std::getenv ("FDTDB_TB2_CHUNK"))
    return std::max (1, std::atoi (v));
  return kTb2Chunk;
}

// Plans the PML shell of the two-step scheme and the two-step core.  The core
// owns the planes cx0 .. cx1 - 1 and rows cy0 .. cy1 - 1 (all z) that are at
// least two cells from every x / y PML cell (so the two-step kernel never
// evaluates an x / y PML cell for it); cy0 and cy1 sit on the single-step
// sweep's 7-row tile boundaries.  The shell (the rest) takes two single
// steps: step 1 over the shell and the cells next to it into set T, step 2
// from T over the shell.  Returns "" or why the scheme does not apply.
std::string plan_shell (fdtd_ctx *ctx, void *const e[2][3], void *const h[2][3], float *const aux[2][6])
{
  const Geometry &g = ctx->g;
  const FusedParams &f = ctx->fused;
  const int nx = g.n[0], ny = g.n[1];
  int X0 = 1, X1 = nx - 1, Y0 = 1, Y1 = ny - 1;
  for (int k = 0; k < 6; ++k)
  {
    X0 = std::max (X0, f.ilo[k][0]);
    X1 = std::min (X1, f.ihi[k][0]);
    Y0 = std::max (Y0, f.ilo[k][1]);
    Y1 = std::min (Y1, f.ihi[k][1]);
  }
  const int cx0 = X0 + 2, cx1 = X1 - 2;
  const int ty = kSweepTileY;
  const int cy0 = 1 + ty * ((Y0 + 2 - 1 + ty - 1) / ty);
  const int cy1 = 1 + ty * ((Y1 - 2 - 1) / ty);
  if (cx1 - cx0 < 1 || cy1 - cy0 < 1)
    return "the PML shell leaves no core";
  // set T (fields as the step stores them, PML auxiliaries), starting as a
  // copy of the current set (its never-updated faces must hold the fields)
  const size_t n = (size_t) g.cells;
  for (int k = 0; k < 6; ++k)
  {
    if (!ctx->tfb[k])
    {
      if (dalloc (ctx, &ctx->tfb[k], n * elem_size (ctx->kind), false) != FDTD_OK)
        return "allocation of the shell buffer set failed";
      if (dalloc (ctx, (void **) &ctx->tauxb[k], n * sizeof (float)) != FDTD_OK)
        return "allocation of the shell buffer set failed";
    }
    if (cudaMemcpyAsync (ctx->tfb[k], ctx->ffb[ctx->fcur][k], n * elem_size (ctx->kind), cudaMemcpyDeviceToDevice,
                         ctx->stream) != cudaSuccess)
      return "shell buffer copy failed";
  }
  // x cuts: step 1 owns planes < cx0 + 1 and >= cx1 - 1 of the x slabs, step
  // 2 those < cx0 and >= cx1; the core planes in chunks of at most 64
  auto cuts_for = [&] (int a, int b) {
    std::vector<int> c = {1};
    auto add = [&] (int v) {
      if (v > c.back () && v < nx - 1)
        c.push_back (v);
    };
    for (int v = 1 + 64; v < a; v += 64)
      add (v);
    add (a);
    const int len = b - a, m = std::max (1, (len + 63) / 64);
    for (int j = 1; j < m; ++j)
      add (a + (int) ((long long) len * j / m));
    add (b);
    for (int v = b + 64; v < nx - 1; v += 64)
      add (v);
    c.push_back (nx - 1);
    return c;
  };
  const std::vector<int> c1 = cuts_for (cx0 + 1, cx1 - 1), c2 = cuts_for (cx0, cx1);
  const int nzt = (g.n[2] - 1 + kSweepTileZ - 1) / kSweepTileZ;
  const int nyt = (ny - 2 + ty - 1) / ty;
  // items: x-slab chunks with every y tile, core chunks with the y-slab tiles
  auto items_for = [&] (const std::vector<int> &c, int xa, int xb, int ya, int yb) {
    std::vector<int> it;
    const int nch = (int) c.size () - 1;
    for (int ch = 0; ch < nch; ++ch)
    {
      const bool xslab = c[ch + 1] <= xa || c[ch] >= xb;
      for (int yt = 0; yt < nyt; ++yt)
      {
        const int r0 = 1 + ty * yt, r1 = std::min (r0 + ty, ny - 1);   // rows r0 .. r1 - 1
        const bool yslab = r1 <= ya || r0 >= yb;
        if (!xslab && !yslab)
          continue;
        for (int zt = 0; zt < nzt; ++zt)
          it.push_back ((ch * nyt + yt) * nzt + zt);
      }
    }
    return it;
  };
  // step 1 rows: the shell rows and the first core row on each side
  const std::vector<int> l1 = items_for (c1, cx0 + 1, cx1 - 1, cy0 + ty, cy1 - ty);
  const std::vector<int> l2 = items_for (c2, cx0, cx1, cy0, cy1);
  for (int q = 0; q < 2; ++q)
  {
    const size_t len = q == 0 ? l1.size () : l2.size ();
    if (!ctx->shell_list[q])
    {
      const size_t cap = (size_t) nzt * nyt * (kMaxChunks + 1);
      if (len > cap || dalloc (ctx, (void **) &ctx->shell_list[q], cap * sizeof (int)) != FDTD_OK)
        return "allocation of the shell item lists failed";
      if (dalloc (ctx, (void **) &ctx->shell_ctr[q], 8 * sizeof (unsigned long long)) != FDTD_OK)
        return "allocation of the shell counters failed";
    }
  }
  std::string why = sweep3d_plan_list (ctx->shell1, f, e, h, aux, ctx->mat32[0], ctx->sm_count, c1, l1,
                                       ctx->shell_list[0], ctx->shell_ctr[0], ctx->stream);
  if (!why.empty ())
    return "shell step 1: " + why;
  void *te[2][3], *th[2][3];
  float *ta[2][6];
  for (int b = 0; b < 2; ++b)
  {
    for (int c = 0; c < 3; ++c)
    {
      te[b][c] = ctx->tfb[c];
      th[b][c] = ctx->tfb[c + 3];
    }
    for (int k = 0; k < 6; ++k)
      ta[b][k] = ctx->tauxb[k];
  }
  why = sweep3d_plan_list (ctx->shell2, f, te, th, ta, ctx->mat32[0], ctx->sm_count, c2, l2, ctx->shell_list[1],
                           ctx->shell_ctr[1], ctx->stream);
  if (!why.empty ())
    return "shell step 2: " + why;
  why = sweep2_plan (ctx->tb2, f, e, h, aux, ctx->mat32[0], ctx->sm_count, tb2_chunk (), ctx->tb2_ctr, cx0, cx1, cy0, cy1);
  if (!why.empty ())
    return "core: " + why;
  if (!ctx->core_stream)
  {
    if (cudaStreamCreateWithFlags (&ctx->core_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags (&ctx->core_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags (&ctx->core_join, cudaEventDisableTiming) != cudaSuccess)
      return "core stream creation failed";
  }
  if (cudaStreamSynchronize (ctx->stream) != cudaSuccess)
    return "shell set-up failed";
  return "";
}

// TF/SF with the two-step scheme: the supports of the pair's corrections
// (which must keep two cells clear of the PML shell the single steps take)
// and the correction kernel's tiles.
std::string plan_tfsf2 (fdtd_ctx *ctx)
{
  std::vector<Tf2Box> rg[4];
  std::string why = tfsf2_regions (ctx->fused, rg);
  if (!why.empty ())
    return why;
  if (ctx->tb2_state == 2)
  {
    const Sweep2Work &w = ctx->tb2.work;
    const int cx0 = w.xcut[0], cx1 = w.xcut[w.nch], cy0 = w.yoff + 1, cy1 = w.yend;
    for (int q = 0; q < 4; ++q)
      for (const Tf2Box &b : rg[q])
        if (b.lo[0] < cx0 + 2 || b.hi[0] > cx1 - 2 || b.lo[1] < cy0 + 2 || b.hi[1] > cy1 - 2)
          return "the TF/SF corrections reach the PML shell";
  }
  for (int q = 0; q < 4; ++q)
  {
    ctx->tf2_cells[q] = 0;
    ctx->tf2_boxes[q] = (int) rg[q].size ();
    for (const Tf2Box &b : rg[q])
      ctx->tf2_cells[q] += (long long) (b.hi[0] - b.lo[0]) * (b.hi[1] - b.lo[1]) * (b.hi[2] - b.lo[2]);
  }
  std::vector<Tf2Tile> tiles;
  unsigned smem = 0;
  if (!(why = tfsf2_tiles (ctx->fused, rg, tiles, smem)).empty () || !(why = tfsf2_configure (smem)).empty ())
    return why;
  Tf2Pass &t = ctx->tf2;
  const Geometry &g = ctx->g;
  if (!ctx->hinc_keep && dalloc (ctx, (void **) &ctx->hinc_keep, (size_t) g.inc_len * sizeof (double)) != FDTD_OK)
    return "allocation of the TF/SF incident copy failed";
  // the tile table (re)allocated at its size
  if (!tiles.empty ())
  {
    const size_t bytes = tiles.size () * sizeof (Tf2Tile);
    if (dalloc (ctx, (void **) &t.tiles, bytes, false) != FDTD_OK ||
        cudaMemcpyAsync (t.tiles, tiles.data (), bytes, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
      return "upload of the TF/SF tiles failed";
  }
  t.ntiles = (int) tiles.size ();
  t.smem = smem;
  if (cudaStreamSynchronize (ctx->stream) != cudaSuccess)
    return "TF/SF set-up failed";
  ctx->tf2_on = true;
  return "";
}

// (Re)builds the TMA sweep plan for the current buffers.  FDTDB_SWEEP=0
// keeps the register-blocked kernel; FDTDB_SWEEP_CHUNK overrides the x
// chunk and FDTDB_SWEEP_VERBOSE=1 prints the plan, for tuning runs.
int plan_sweep (fdtd_ctx *ctx)
{
  const Geometry &g = ctx->g;
  ctx->sweep_state = -1;
  if (const char *v = std::getenv ("FDTDB_SWEEP"))
    if (std::atoi (v) == 0)
    {
      ctx->sweep_why = "disabled by FDTDB_SWEEP=0";
      return FDTD_OK;
    }
  const int wy = 8;
  if (!ctx->sweep_streams.side[0])
  {
    // the item classes on side streams (measured faster: 1.80 -> 1.72 ms
    // per step at 512^3)
    SweepStreams &ss = ctx->sweep_streams;
    for (cudaStream_t &q : ss.side)
      CK (cudaStreamCreateWithFlags (&q, cudaStreamNonBlocking));
    for (cudaEvent_t *e : {&ss.fork, &ss.join[0], &ss.join[1]})
      CK (cudaEventCreateWithFlags (e, cudaEventDisableTiming));
  }
  const bool lean = true;   // item classes (false: every item in the general class)
  if (!ctx->sweep_ctr)
    DALLOC (ctx->sweep_ctr, 8 * sizeof (unsigned long long));
  void *e[2][3], *h[2][3];
  float *aux[2][6];
  for (int b = 0; b < 2; ++b)
  {
    for (int c = 0; c < 3; ++c)
    {
      e[b][c] = ctx->ffb[b][c];
      h[b][c] = ctx->ffb[b][c + 3];
    }
    for (int k = 0; k < 6; ++k)
      aux[b][k] = ctx->auxb[b][k];
  }
  // TF/SF as a post pass over the face band when the band is PML-free
  // (FDTDB_TFSF_POST=0 keeps the corrections inside the sweep).  Decided
  // before the plan: the item classes depend on it.
  bool post = g.cfg.use_tfsf && ctx->band.cells == 0;
  if (const char *v = std::getenv ("FDTDB_TFSF_POST"))
    post = post && std::atoi (v) != 0;
  if (post)
  {
    std::vector<BandBox> boxes;
    std::vector<int2> blk;
    std::string bwhy = tfsf_band_boxes (ctx->fused, boxes, blk);
    if (bwhy.empty () && !boxes.empty ())
    {
      DALLOC (ctx->band.boxes, boxes.size () * sizeof (BandBox));
      CK (cudaMemcpyAsync (ctx->band.boxes, boxes.data (), boxes.size () * sizeof (BandBox), cudaMemcpyHostToDevice,
                           ctx->stream));
      DALLOC (ctx->band.blk, blk.size () * sizeof (int2));
      CK (cudaMemcpyAsync (ctx->band.blk, blk.data (), blk.size () * sizeof (int2), cudaMemcpyHostToDevice,
                           ctx->stream));
      ctx->band.nblk = (int) blk.size ();
      CK (cudaStreamSynchronize (ctx->stream));
      ctx->band.nbox = (int) boxes.size ();
      ctx->band_host = boxes;
      long long cells = 0;
      for (const BandBox &bb : boxes)
        cells += (long long) (bb.hi[0] - bb.lo[0]) * (bb.hi[1] - bb.lo[1]) * (bb.hi[2] - bb.lo[2]);
      ctx->band.cells = cells;
    }
  }
  ctx->fused.tfsf_post = ctx->band.cells > 0 ? 1 : 0;   // read only by the sweep kernels
  // a first plan gives the CTA count the chunk choice depends on
  std::string why = sweep3d_plan (ctx->sweep, ctx->fused, e, h, aux, ctx->mat32[0], ctx->sm_count, wy, 32,
                                  ctx->sweep_ctr, lean);
  if (why.empty ())
  {
    int chunk = sweep_chunk (ctx->fused, wy, ctx->sweep.ctas, ctx->sweep_streams.side[0] ? 3 : 1);
    if (const char *v = std::getenv ("FDTDB_SWEEP_CHUNK"))
      chunk = std::max (1, std::atoi (v));
    why = sweep3d_plan (ctx->sweep, ctx->fused, e, h, aux, ctx->mat32[0], ctx->sm_count, wy, chunk,
                        ctx->sweep_ctr, lean);
  }
  // Drude cells: fixed up after each sweep step when their box (and the H
  // cells one step below it) holds no PML cell, no TF/SF band cell and no
  // point source, and the TF/SF corrections (if any) run as the post pass
  ctx->drude_fix = false;
  if (why.empty () && g.cfg.use_metamaterials)
  {
    if (!ctx->drude_box_dev)
      DALLOC (ctx->drude_box_dev, 6 * sizeof (int));
    ctx->launches += launch_drude_box (ctx->dflag, g.n[0], g.n[1], g.n[2], ctx->drude_box_dev, ctx->stream);
    int hb[6];
    CK (cudaMemcpyAsync (hb, ctx->drude_box_dev, sizeof (hb), cudaMemcpyDeviceToHost, ctx->stream));
    CK (cudaStreamSynchronize (ctx->stream));
    if (hb[3] >= 0)
    {
      DrudeBox b;
      for (int a = 0; a < 3; ++a)
      {
        b.lo[a] = hb[a];
        b.hi[a] = hb[3 + a] + 1;
      }
      int ext_lo[3];
      for (int a = 0; a < 3; ++a)
        ext_lo[a] = std::max (b.lo[a] - 1, 1);
      for (int k = 0; k < 6 && why.empty (); ++k)
        for (int a = 0; a < 3; ++a)
          if (ext_lo[a] < ctx->fused.ilo[k][a] || b.hi[a] > ctx->fused.ihi[k][a])
            why = "Drude cells next to the PML";
      if (why.empty () && g.cfg.use_tfsf && !ctx->fused.tfsf_post)
        why = "Drude cells with TF/SF corrections inside the sweep";
      for (const BandBox &bb : ctx->band_host)
      {
        bool hit = true;
        for (int a = 0; a < 3; ++a)
          hit = hit && bb.lo[a] < b.hi[a] && ext_lo[a] < bb.hi[a];
        if (hit && why.empty ())
          why = "Drude cells on the TF/SF band";
      }
      if (why.empty () && g.cfg.point_source_mask)
      {
        bool in = true;
        for (int a = 0; a < 3; ++a)
          in = in && g.cfg.point_source[a] >= ext_lo[a] && g.cfg.point_source[a] < b.hi[a];
        if (in)
          why = "a point source among the Drude cells";
      }
      if (why.empty ())
      {
        ctx->drude_box = b;
        ctx->drude_fix = true;
      }
    }
  }
  ctx->sweep_why = why;
  if (why.empty ())
  {
    ctx->sweep_state = 1;
    ctx->sweep_eps = ctx->mat32[0];
  }
  // the two-step sweep for pairs of steps (FDTDB_TB2=0 keeps single steps:
  // a test hook)
  ctx->tb2_state = -1;
  ctx->tb2_why = "the single-step sweep is not in use";
  if (ctx->sweep_state == 1)
  {
    bool tb2 = true;
    if (const char *v = std::getenv ("FDTDB_TB2"))
      tb2 = std::atoi (v) != 0;
    if (!tb2)
      ctx->tb2_why = "disabled by FDTDB_TB2=0";
    else
    {
      if (!ctx->tb2_ctr)
        DALLOC (ctx->tb2_ctr, 6 * sizeof (unsigned long long));
      if (g.cfg.use_pml)
      {
        // PML: the x / y PML shell in single steps beside the two-step core
        ctx->tb2_why = plan_shell (ctx, e, h, aux);
        if (ctx->tb2_why.empty ())
          ctx->tb2_state = 2;
      }
      else
      {
        ctx->tb2_why = sweep2_plan (ctx->tb2, ctx->fused, e, h, aux, ctx->mat32[0], ctx->sm_count, tb2_chunk (),
                                     ctx->tb2_ctr);
        if (ctx->tb2_why.empty ())
          ctx->tb2_state = 1;
      }
      if (ctx->tb2_state >= 1 && g.cfg.use_tfsf)
      {
        ctx->tb2_why = plan_tfsf2 (ctx);
        if (!ctx->tb2_why.empty ())
          ctx->tb2_state = -1;
      }
    }
  }
  if (const char *v = std::getenv ("FDTDB_SWEEP_VERBOSE"))
    if (std::atoi (v) != 0)
    {
      const SweepWork &w = ctx->sweep.work;
      std::fprintf (stderr, "sweep3d: %s wy=%d ctas=%d smem=%u tiles z=%d y=%d chunks=%d (x chunk %d) items=%d "
                    "items lean/z-edge/full/PML=%d/%d/%d/%d tfsf band boxes=%d cells=%lld\n",
                    why.empty () ? "in use" : why.c_str (), ctx->sweep.wy, ctx->sweep.ctas, ctx->sweep.smem, w.nzt,
                    w.nyt, w.nch, w.chunk, w.nitems, ctx->sweep.items[0], ctx->sweep.items[1], ctx->sweep.items[2], ctx->sweep.items[3],
                    ctx->band.nbox, ctx->band.cells);
      std::fprintf (stderr, "sweep2: %s ctas=%d smem=%u tiles z=%d y=%d chunks=%d items=%d lean/PML/z-edge=%d/%d/%d\n",
                    ctx->tb2_state >= 1 ? (ctx->tb2_state == 2 ? "in use (core)" : "in use") : ctx->tb2_why.c_str (),
                    ctx->tb2.ctas, ctx->tb2.smem, ctx->tb2.work.nzt, ctx->tb2.work.nyt, ctx->tb2.work.nch,
                    ctx->tb2.work.nitems, ctx->tb2.items[0], ctx->tb2.items[1], ctx->tb2.items[2]);
      if (ctx->tb2_state == 2)
        std::fprintf (stderr, "shell: step 1 items %d (lean/z-edge/full/PML %d/%d/%d/%d), step 2 items %d "
                      "(%d/%d/%d/%d)\n", ctx->shell1.work.nlist, ctx->shell1.items[0], ctx->shell1.items[1],
                      ctx->shell1.items[2], ctx->shell1.items[3], ctx->shell2.work.nlist, ctx->shell2.items[0],
                      ctx->shell2.items[1], ctx->shell2.items[2], ctx->shell2.items[3]);
      if (ctx->tb2_state >= 1 && ctx->tf2_on)
        std::fprintf (stderr, "tfsf2: support boxes %d/%d/%d/%d cells %lld/%lld/%lld/%lld tiles %d smem %u\n",
                      ctx->tf2_boxes[0], ctx->tf2_boxes[1], ctx->tf2_boxes[2], ctx->tf2_boxes[3], ctx->tf2_cells[0],
                      ctx->tf2_cells[1], ctx->tf2_cells[2], ctx->tf2_cells[3], ctx->tf2.ntiles, ctx->tf2.smem);
    }
  return FDTD_OK;
}

int create_impl (const fdtd_config *cfg, int device, fdtd_ctx *ctx)
{
  std::string err = build_geometry (*cfg, ctx->g);
  if (!err.empty ())
    return fail (ctx, FDTD_ERR_ARG, err);
  int ndev = 0;
  if (cudaGetDeviceCount (&ndev) != cudaSuccess || ndev <= 0)
    return fail (ctx, FDTD_ERR_CUDA, "no CUDA device available");
  if (device < 0 || device >= ndev)
    return fail (ctx, FDTD_ERR_ARG, "device index out of range");
  ctx->device = device;
  ctx->prec = cfg->precision;
  {
    // a current source acts on interior cells only: the reference's
    // precomputed Cb is zero on the outer shell, and a cell outside the grid
    // is skipped (InternalScheme.inc.h:2439-2448)
    // (a mode's dropped axes ignore the coordinate, as initAxesCoordinate does)
    const Geometry &g = ctx->g;
    bool inside = true;
    for (int a = 0; a < 3; ++a)
    {
      const bool dropped = (g.drop >> a) & 1;
      const int c = dropped ? 0 : g.cfg.current_source[a];
      ctx->cs_pos[a] = c;
      inside = inside && (dropped || (c >= 1 && c <= g.n[a] - 2));
    }
    for (int k = 0; k < 6; ++k)
      if (inside && ((g.cfg.current_source_mask >> k) & 1) && g.comp[k].exists)
        ctx->cs_mask[k / 3] |= 1 << (k % 3);
  }
  ctx->kind = kind_of (cfg->precision);
  ctx->eta0 = ctx->kind == 0 ? 1.0 : kEta0;
  CK (cudaSetDevice (device));
  CK (cudaDeviceGetAttribute (&ctx->sm_count, cudaDevAttrMultiProcessorCount, device));
  CK (cudaStreamCreateWithFlags (&ctx->stream, cudaStreamNonBlocking));
  CK (cudaEventCreateWithFlags (&ctx->src_ev, cudaEventDisableTiming));
  DALLOC (ctx->d_err, sizeof (int));
  const Geometry &g = ctx->g;
  if (g.cfg.use_tfsf)
  {
    for (int l = 0; l < 2; ++l)
    {
      DALLOC (ctx->einc[l], (size_t) g.inc_len * sizeof (double));
      DALLOC (ctx->hinc[l], (size_t) g.inc_len * sizeof (double));
    }
  }
  ctx->nparts = ctx->sm_count * 4;
  DALLOC (ctx->partials, (size_t) ctx->nparts * 2 * sizeof (double));
  DALLOC (ctx->d_out, 16 * sizeof (double));
  int r = ctx->kind == 0 ? alloc_plain (ctx) : alloc_fast (ctx);
  if (r != FDTD_OK)
    return r;
  if (ctx->kind != 0)
  {
    select_fast_set (ctx);
    init_fused (ctx);
  }
  CK (cudaStreamSynchronize (ctx->stream));
  return FDTD_OK;
}

void release (fdtd_ctx *ctx)
{
  if (!ctx)
    return;
  cudaSetDevice (ctx->device);
  if (ctx->stream)
    cudaStreamSynchronize (ctx->stream);
  for (cudaStream_t q : {ctx->h2d, ctx->d2h})
    if (q)
    {
      cudaStreamSynchronize (q);
      cudaStreamDestroy (q);
    }
  for (cudaEvent_t e : {ctx->in_ready, ctx->in_free, ctx->out_ready, ctx->out_free})
    if (e)
      cudaEventDestroy (e);
  if (ctx->adj_cache.base)
    cudaFree (ctx->adj_cache.base);
  for (cudaStream_t q : ctx->sweep_streams.side)
    if (q)
    {
      cudaStreamSynchronize (q);
      cudaStreamDestroy (q);
    }
  if (ctx->core_stream)
  {
    cudaStreamSynchronize (ctx->core_stream);
    cudaStreamDestroy (ctx->core_stream);
  }
  if (ctx->inc_stream)
  {
    cudaStreamSynchronize (ctx->inc_stream);
    cudaStreamDestroy (ctx->inc_stream);
  }
  for (cudaEvent_t e : {ctx->core_fork, ctx->core_join, ctx->inc_free, ctx->inc_done})
    if (e)
      cudaEventDestroy (e);
  for (cudaEvent_t e : {ctx->sweep_streams.fork, ctx->sweep_streams.join[0], ctx->sweep_streams.join[1]})
    if (e)
      cudaEventDestroy (e);
  for (void *p : ctx->allocs)
    cudaFree (p);
  ctx->allocs.clear ();
  if (ctx->h_src)
    cudaFreeHost (ctx->h_src);
  for (cudaEvent_t e : ctx->prof_events)
    cudaEventDestroy (e);
  if (ctx->src_ev)
    cudaEventDestroy (ctx->src_ev);
  if (ctx->stream)
    cudaStreamDestroy (ctx->stream);
  delete ctx;
}

size_t cell_index (const Geometry &g, int x, int y, int z)
{
  return ((size_t) x * g.n[1] + y) * g.n[2] + z;
}

bool point_source_index (const Geometry &g, size_t *idx)
{
  int p[3];
  for (int a = 0; a < 3; ++a)
  {
    p[a] = ((g.drop >> a) & 1) ? 0 : g.cfg.point_source[a];
    if (p[a] < 0 || p[a] >= g.n[a])
      return false;
  }
  *idx = cell_index (g, p[0], p[1], p[2]);
  return true;
}

void rotate (double **lv, int levels)
{
  if (!lv[0])
    return;
  double *oldest = lv[levels - 1];
  for (int i = levels - 1; i >= 1; --i)
    lv[i] = lv[i - 1];
  lv[0] = oldest;
}

PlainHalf plain_half (fdtd_ctx *ctx, int h)
{
  const Geometry &g = ctx->g;
  PlainHalf p;
  std::memset (&p, 0, sizeof (p));
  p.g = make_geom_dev (g);
  p.is_h = h;
  p.use_pml = g.cfg.use_pml;
  p.use_tfsf = g.cfg.use_tfsf;
  p.use_meta = g.cfg.use_metamaterials;
  p.mat_modifier = h ? kMu0 : kEps0;
  for (int ci = 0; ci < 3; ++ci)
  {
    int k = ci + 3 * h;
    p.comp[ci] = make_comp_dev (g, k);
    for (int l = 0; l < 3; ++l)
    {
      p.f[ci][l] = ctx->f[k][l];
      p.dd[ci][l] = ctx->dd[k][l];
      p.d1[ci][l] = ctx->d1[k][l];
    }
    p.opp[ci] = ctx->f[ci + 3 * (1 - h)][1];
  }
  p.mat = ctx->mat64[h ? 1 : 0];
  p.omega = ctx->mat64[h ? 3 : 2];
  p.gamma = ctx->mat64[h ? 5 : 4];
  for (int a = 0; a < 3; ++a)
    p.sigma[a] = ctx->sig64[a];
  p.inc = h ? ctx->einc[ctx->ecur] : ctx->hinc[ctx->hcur];
  p.cs_mask = ctx->cs_mask[h];
  for (int a = 0; a < 3; ++a)
    p.cs[a] = ctx->cs_pos[a];
  for (int ci = 0; ci < 3; ++ci)
  {
    const int k = ci + 3 * h;
    p.dmp = g.dmp ? 1 : 0;
    p.matc[ci] = ctx->matc64[k] ? ctx->matc64[k] : p.mat;
    for (int a = 0; a < 3; ++a)
      p.sigc[ci][a] = ctx->sigc64[k][a] ? ctx->sigc64[k][a] : p.sigma[a];
  }
  return p;
}

// The side stream of a pair's incident-grid steps and its two events.
int ensure_inc_stream (fdtd_ctx *ctx)
{
  if (ctx->inc_stream)
    return FDTD_OK;
  CK (cudaStreamCreateWithFlags (&ctx->inc_stream, cudaStreamNonBlocking));
  CK (cudaEventCreateWithFlags (&ctx->inc_free, cudaEventDisableTiming));
  CK (cudaEventCreateWithFlags (&ctx->inc_done, cudaEventDisableTiming));
  return FDTD_OK;
}

int prof_begin (fdtd_ctx *ctx, cudaEvent_t *end_out)
{
  *end_out = nullptr;
  if (!ctx->profiling)
    return FDTD_OK;
  while (ctx->prof_events.size () < ctx->prof_used + 2)
  {
    cudaEvent_t e;
    CK (cudaEventCreate (&e));
    ctx->prof_events.push_back (e);
  }
  CK (cudaEventRecord (ctx->prof_events[ctx->prof_used], ctx->stream));
  *end_out = ctx->prof_events[ctx->prof_used + 1];
  ctx->prof_used += 2;
  return FDTD_OK;
}

int prof_end (fdtd_ctx *ctx, cudaEvent_t end)
{
  if (end)
    CK (cudaEventRecord (end, ctx->stream));
  return FDTD_OK;
}

// Phase table of the running DFT for steps t_start .. t_start + n - 1: E is
// taken at (t + 1/2) dt and H at (t + 1) dt, the times of the point
// sources of the same step.
int dft_prepare (fdtd_ctx *ctx, uint32_t t_start, uint32_t n)
{
  if (ctx->dft_comp < 0)
    return FDTD_OK;
  const size_t need = (size_t) n * ctx->dft_nf * 2;
  if (n > ctx->dft_phase_cap)
  {
    CK (cudaStreamSynchronize (ctx->stream));
    if (ctx->dft_phase)
    {
      cudaFree (ctx->dft_phase);
      ctx->allocs.erase (std::remove (ctx->allocs.begin (), ctx->allocs.end (), (void *) ctx->dft_phase),
                         ctx->allocs.end ());
      ctx->dft_phase = nullptr;
    }
    DALLOC (ctx->dft_phase, need * sizeof (double));
    ctx->dft_phase_cap = n;
    ctx->h_dft_phase.resize (need);
  }
  const double shift = ctx->dft_comp >= 3 ? 1.0 : 0.5;
  for (uint32_t i = 0; i < n; ++i)
    for (int j = 0; j < ctx->dft_nf; ++j)
    {
      const double ph = 2 * kPi * ctx->dft_freq[j] * ((double) (t_start + i) + shift) * ctx->g.dt;
      ctx->h_dft_phase[((size_t) i * ctx->dft_nf + j) * 2] = std::cos (ph);
      ctx->h_dft_phase[((size_t) i * ctx->dft_nf + j) * 2 + 1] = std::sin (ph);
    }
  CK (cudaMemcpyAsync (ctx->dft_phase, ctx->h_dft_phase.data (), need * sizeof (double), cudaMemcpyHostToDevice,
                       ctx->stream));
  return FDTD_OK;
}

// adds step i of the current call to the running DFT
void dft_step (fdtd_ctx *ctx, uint32_t i)
{
  if (ctx->dft_comp < 0)
    return;
  const int k = ctx->dft_comp;
  const void *src = ctx->kind == 0 ? (const void *) ctx->f[k][1] : (const void *) ctx->ff[k];
  const double scale = k >= 3 ? 1.0 / ctx->eta0 : 1.0;
  ctx->launches += launch_dft (src, ctx->kind, ctx->dft_axis, ctx->dft_index, ctx->g.n, scale,
                               ctx->dft_phase + (size_t) i * ctx->dft_nf * 2, ctx->dft_nf, ctx->dft_acc,
                               ctx->sm_count, ctx->stream);
}

int step_impl (fdtd_ctx *ctx, uint32_t t_start, uint32_t n)
{
  const Geometry &g = ctx->g;
  int r = ensure_src (ctx, n);
  if (r != FDTD_OK)
    return r;
  for (uint32_t i = 0; i < n; ++i)
  {
    uint32_t t = t_start + i;
    double *hs = ctx->h_src + kSrcStride * i;
    hs[0] = incident_source (g, t);
    hs[1] = point_source (g, t, false);
    hs[2] = point_source (g, t, true);
    hs[3] = current_source (g, t, false);
    hs[4] = current_source (g, t, true);
  }
  CK (cudaMemcpyAsync (ctx->d_src, ctx->h_src, (size_t) n * kSrcStride * sizeof (double), cudaMemcpyHostToDevice,
                       ctx->stream));
  CK (cudaEventRecord (ctx->src_ev, ctx->stream));
  if ((r = dft_prepare (ctx, t_start, n)) != FDTD_OK)
    return r;
  if (n > 1 || t_start > 0)
    ctx->stepped = true;
  size_t ps_idx = 0;
  bool ps_ok = g.cfg.point_source_mask && point_source_index (g, &ps_idx);
  cudaStream_t s = ctx->stream;
  // a current source runs with the one-sweep kernels as a fix-up after each
  // step (launch_current_fix) when its cell and the cells around it update
  // outside the PML, else with the per-cell kernels
  const bool has_cs = ctx->cs_mask[0] || ctx->cs_mask[1];
  bool cs_fix = has_cs && !g.cfg.use_metamaterials;
  if (cs_fix && g.cfg.use_pml)
    for (int k = 0; k < 6; ++k)
      for (int a = 0; a < 3; ++a)
        cs_fix = cs_fix && ctx->cs_pos[a] - 1 >= ctx->fused.ilo[k][a] && ctx->cs_pos[a] + 1 < ctx->fused.ihi[k][a];
  const bool fused = ctx->kind != 0 && ctx->has_second && !ctx->mat32[1] && ctx->ps_interior && (!has_cs || cs_fix);
  CurrentFix cfix{};
  if (has_cs)
  {
    for (int a = 0; a < 3; ++a)
      cfix.pos[a] = ctx->cs_pos[a];
    cfix.mask_e = ctx->cs_mask[0];
    cfix.mask_h = ctx->cs_mask[1];
    cfix.scale_e = (float) kEta0;
    cfix.scale_h = 1.f;
  }

  for (uint32_t i = 0; i < n; ++i)
  {
    uint32_t t = t_start + i;
    if (fused && t > 0)
    {
      // incident E then H steps, then one sweep for both field families
      int hprev = ctx->hcur;
      FusedParams &f = ctx->fused;
      int o = ctx->fcur, nw = 1 - ctx->fcur;
      for (int c = 0; c < 3; ++c)
      {
        f.e_old[c] = ctx->ffb[o][c];
        f.h_old[c] = ctx->ffb[o][c + 3];
        f.e_new[c] = ctx->ffb[nw][c];
        f.h_new[c] = ctx->ffb[nw][c + 3];
      }
      for (int k = 0; k < 6; ++k)
      {
        f.aux_old[k] = ctx->auxb[o][k];
        f.aux_new[k] = ctx->auxb[nw][k];
        f.xpp_old[k] = ctx->xppb[o][k];
        f.xpp_new[k] = ctx->xppb[nw][k];
        f.z_old[k] = ctx->zb[o][k];
        f.z_new[k] = ctx->zb[nw][k];
        f.zpp_old[k] = ctx->zppb[o][k];
        f.zpp_new[k] = ctx->zppb[nw][k];
      }
      f.eps = ctx->mat32[0];
      f.src = ctx->d_src;
      f.src_index = kSrcStride * i + 1;
      if (ctx->sweep_state == 0 || (ctx->sweep_state == 1 && ctx->sweep_eps != ctx->mat32[0]))
        if ((r = plan_sweep (ctx)) != FDTD_OK)
          return r;
      const bool pair = ctx->tb2_state >= 1 && i + (ctx->keep_prev ? 2 : 1) < n && ctx->dft_comp < 0 && !has_cs;
      // On the two-step path with a PML shell only the pair's TF/SF kernel
      // reads the incident grid: its steps run on a stream of their own
      // beside the shell and the core, after every earlier reader (all on s
      // or joined into s), and the TF/SF kernel waits for them
      const bool inc_side = pair && ctx->tb2_state == 2 && g.cfg.use_tfsf;
      cudaStream_t si = s;
      if (inc_side)
      {
        if ((r = ensure_inc_stream (ctx)) != FDTD_OK)
          return r;
        si = ctx->inc_stream;
        CK (cudaEventRecord (ctx->inc_free, s));
        CK (cudaStreamWaitEvent (si, ctx->inc_free, 0));
      }
      if (g.cfg.use_tfsf)
      {
        ctx->launches += launch_incident_e (ctx->einc[1 - ctx->ecur], ctx->einc[ctx->ecur], ctx->hinc[ctx->hcur],
                                            g.inc_len, g.mod_e, ctx->d_src, kSrcStride * i, si);
        ctx->ecur ^= 1;
        ctx->launches += launch_incident_h (ctx->hinc[1 - ctx->hcur], ctx->hinc[ctx->hcur], ctx->einc[ctx->ecur],
                                            g.inc_len, g.mod_h, si);
        ctx->hcur ^= 1;
      }
      f.inc_h = ctx->hinc[hprev];
      f.inc_e = ctx->einc[ctx->ecur];
      cudaEvent_t pe;
      if (pair)
      {
        // steps t and t + 1 in one pass (no point source or Drude medium).
        // With TF/SF the incident grid takes both steps first (this step's
        // E and H updates were issued above), keeping the levels the pair's
        // corrections read
        const double *inc_h1 = nullptr, *inc_e1 = nullptr, *inc_h2 = nullptr, *inc_e2 = nullptr;
        if (g.cfg.use_tfsf)
        {
          CK (cudaMemcpyAsync (ctx->hinc_keep, ctx->hinc[hprev], (size_t) g.inc_len * sizeof (double),
                               cudaMemcpyDeviceToDevice, si));
          inc_h1 = ctx->hinc_keep;
          inc_e1 = ctx->einc[ctx->ecur];
          inc_h2 = ctx->hinc[ctx->hcur];
          ctx->launches += launch_incident_e (ctx->einc[1 - ctx->ecur], ctx->einc[ctx->ecur], ctx->hinc[ctx->hcur],
                                              g.inc_len, g.mod_e, ctx->d_src, kSrcStride * (i + 1), si);
          ctx->ecur ^= 1;
          inc_e2 = ctx->einc[ctx->ecur];
          ctx->launches += launch_incident_h (ctx->hinc[1 - ctx->hcur], ctx->hinc[ctx->hcur], ctx->einc[ctx->ecur],
                                              g.inc_len, g.mod_h, si);
          ctx->hcur ^= 1;
          if (inc_side)
            CK (cudaEventRecord (ctx->inc_done, si));
        }
        if ((r = prof_begin (ctx, &pe)) != FDTD_OK)
          return r;
        if (ctx->tb2_state == 1)
          ctx->launches += launch_sweep2 (ctx->tb2, o, f, ctx->d_err, s, ctx->sweep_streams);
        else
        {
          // the shell's two single steps on s, the core on its own stream
          // (launched after the shell's first step, so that its CTAs take
          // the SMs that step leaves as it drains)
          CK (cudaEventRecord (ctx->core_fork, s));
          CK (cudaStreamWaitEvent (ctx->core_stream, ctx->core_fork, 0));
          FusedParams f1 = f;
          for (int c = 0; c < 3; ++c)
          {
            f1.e_new[c] = ctx->tfb[c];
            f1.h_new[c] = ctx->tfb[c + 3];
          }
          for (int k = 0; k < 6; ++k)
            f1.aux_new[k] = ctx->tauxb[k];
          ctx->launches += launch_sweep3d (ctx->shell1, o, f1, ctx->d_err, s, ctx->sweep_streams);
          ctx->launches += launch_sweep2 (ctx->tb2, o, f, ctx->d_err, ctx->core_stream);
          ctx->launches += launch_sweep3d (ctx->shell2, 0, f, ctx->d_err, s, ctx->sweep_streams);
          // the TF/SF corrections touch only core cells two cells clear of
          // the shell (plan_tfsf2): they follow the core on its stream,
          // beside the shell's second step, once the incident levels they
          // read are in place
          if (g.cfg.use_tfsf)
          {
            CK (cudaStreamWaitEvent (ctx->core_stream, ctx->inc_done, 0));
            ctx->launches += launch_tfsf2 (ctx->tf2, f, inc_h1, inc_e1, inc_h2, inc_e2, ctx->d_err, ctx->core_stream);
          }
          CK (cudaEventRecord (ctx->core_join, ctx->core_stream));
          CK (cudaStreamWaitEvent (s, ctx->core_join, 0));
        }
        if (g.cfg.use_tfsf && ctx->tb2_state == 1)
          ctx->launches += launch_tfsf2 (ctx->tf2, f, inc_h1, inc_e1, inc_h2, inc_e2, ctx->d_err, s);
        ctx->step_kernel = "sweep2_tma";
        if ((r = prof_end (ctx, pe)) != FDTD_OK)
          return r;
        ctx->fcur = nw;
        ctx->prev_src = 0;   // set 1 - fcur holds two steps back
        select_fast_set (ctx);
        ++i;
        continue;
      }
      if ((r = prof_begin (ctx, &pe)) != FDTD_OK)
        return r;
      if (ctx->sweep_state == 1)
      {
        ctx->launches += launch_sweep3d (ctx->sweep, o, f, ctx->d_err, s, ctx->sweep_streams);
        if (ctx->drude_fix)
          ctx->launches += launch_drude_fixup (f, ctx->drude_box, s);
        if (f.tfsf_post)
          ctx->launches += launch_tfsf_post (ctx->band, f, ctx->d_err, s);
        ctx->step_kernel = "sweep3d_tma";
      }
      else
      {
        ctx->launches += launch_fused3d (f, ctx->d_err, s);
        ctx->step_kernel = "fused3d_regblock";
      }
      if (has_cs)
        ctx->launches += launch_current_fix (f, cfix, ctx->d_src + kSrcStride * i + 3, s);
      if ((r = prof_end (ctx, pe)) != FDTD_OK)
        return r;
      ctx->fcur = nw;
      ctx->prev_src = 1;   // set 1 - fcur holds the previous level
      select_fast_set (ctx);
      dft_step (ctx, i);
      continue;
    }
    for (int h = 0; h < 2; ++h)
    {
      if (g.cfg.use_tfsf)
      {
        if (!h)
        {
          ctx->launches += launch_incident_e (ctx->einc[1 - ctx->ecur], ctx->einc[ctx->ecur],
                                              ctx->hinc[ctx->hcur], g.inc_len, g.mod_e, ctx->d_src, kSrcStride * i, s);
          ctx->ecur ^= 1;
        }
        else
        {
          ctx->launches += launch_incident_h (ctx->hinc[1 - ctx->hcur], ctx->hinc[ctx->hcur],
                                              ctx->einc[ctx->ecur], g.inc_len, g.mod_h, s);
          ctx->hcur ^= 1;
        }
      }
      if (ctx->kind == 0)
      {
        if (t > 0)
        {
          PlainHalf p = plain_half (ctx, h);
          p.cs_val = ctx->d_src + kSrcStride * i + 3 + h;
          cudaEvent_t pe;
          if ((r = prof_begin (ctx, &pe)) != FDTD_OK)
            return r;
          if (p.cs_mask == 0 && (!g.cfg.use_pml || ctx->ptab[3 * h][0] || ctx->ptab[3 * h + 1][0] ||
                                 ctx->ptab[3 * h + 2][0]))
          {
            PlainTabs tb;
            for (int ci = 0; ci < 3; ++ci)
              for (int j = 0; j < 6; ++j)
                tb.t[ci][j] = ctx->ptab[ci + 3 * h][j];
            ctx->launches += launch_plain_fast (p, tb, g.inc_len, ctx->d_err, ctx->sm_count, s);
          }
          else
            ctx->launches += launch_plain_half (p, g.inc_len, ctx->d_err, ctx->sm_count, s);
          ctx->step_kernel = "plain_fp64";
          if ((r = prof_end (ctx, pe)) != FDTD_OK)
            return r;
        }
        for (int ci = 0; ci < 3; ++ci)
        {
          int k = ci + 3 * h;
          if (ps_ok && (g.cfg.point_source_mask & (1 << k)) && g.comp[k].exists)
            ctx->launches += launch_point_source (ctx->f[k][0], ps_idx, ctx->d_src, kSrcStride * i + 1 + h, s);
        }
        for (int ci = 0; ci < 3; ++ci)
        {
          int k = ci + 3 * h;
          if (!g.comp[k].exists)
            continue;
          rotate (ctx->f[k], g.levels);
          rotate (ctx->dd[k], g.levels);
          rotate (ctx->d1[k], g.levels);
        }
      }
      else
      {
        if (h == 1)
        {
          // the per-cell kernels update in place: with keep_prev the last
          // step of the call copies H before its H update
          ctx->prev_src = 0;
          if (ctx->keep_prev && i + 1 == n && ctx->hprev[0])
          {
            for (int ci = 0; ci < 3; ++ci)
              if (g.comp[3 + ci].exists)
                CK (cudaMemcpyAsync (ctx->hprev[ci], ctx->ff[3 + ci], (size_t) g.cells * elem_size (ctx->kind),
                                     cudaMemcpyDeviceToDevice, s));
            ctx->prev_src = 2;
          }
        }
        if (t > 0)
        {
          FastHalf &p = h ? ctx->fast_h : ctx->fast_e;
          p.inc = h ? ctx->einc[ctx->ecur] : ctx->hinc[ctx->hcur];
          p.mat = ctx->mat32[h];
          for (int ci = 0; ci < 3; ++ci)
            p.matc[ci] = ctx->matc32[ci + 3 * h];
          p.cs_val = ctx->d_src + kSrcStride * i + 3 + h;
          cudaEvent_t pe;
          if ((r = prof_begin (ctx, &pe)) != FDTD_OK)
            return r;
          ctx->launches += launch_fast_half (p, ctx->d_err, ctx->sm_count, s);
          ctx->step_kernel = "per_cell";
          if ((r = prof_end (ctx, pe)) != FDTD_OK)
            return r;
        }
        for (int ci = 0; ci < 3; ++ci)
        {
          int k = ci + 3 * h;
          if (ps_ok && (g.cfg.point_source_mask & (1 << k)) && g.comp[k].exists)
            ctx->launches += launch_fast_point_source (ctx->ff[k], ctx->kind == 2, ps_idx, ctx->d_src,
                                                       kSrcStride * i + 1 + h, (float) (h ? kEta0 : 1.0), s);
        }
      }
    }
    dft_step (ctx, i);
  }
  CK (cudaGetLastError ());
  return FDTD_OK;
}

}  // namespace

// --------------------------------------------------------------------------
// public C ABI

extern "C" {

int fdtd_create (const fdtd_config *cfg, int device, fdtd_ctx **out)
{
  if (!cfg || !out)
  {
    g_last_error = "null argument";
    return FDTD_ERR_ARG;
  }
  *out = nullptr;
  fdtd_ctx *ctx = new (std::nothrow) fdtd_ctx ();
  if (!ctx)
  {
    g_last_error = "host allocation failed";
    return FDTD_ERR_NOMEM;
  }
  int r = create_impl (cfg, device, ctx);
  if (r != FDTD_OK)
  {
    std::string keep = g_last_error;
    release (ctx);
    g_last_error = keep;
    return r;
  }
  *out = ctx;
  return FDTD_OK;
}

int fdtd_upload_material (fdtd_ctx *ctx, int which, const double *host)
{
  if (!ctx || !host || which < 0 || which > 5)
    return fail (ctx, FDTD_ERR_ARG, "bad argument");
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  size_t n = (size_t) ctx->g.cells;
  if (ctx->g.dmp && which < 2)
    return upload_fine_material (ctx, which, host, cudaMemcpyHostToDevice);
  if (ctx->kind == 0 && !ctx->mat64[which])
    return fail (ctx, FDTD_ERR_UNSUPPORTED, "Drude grids need use_metamaterials");
  // staged on the device and checked there: a NaN or an infinity is refused
  // before anything the step reads changes
  if ((r = ensure_staging (ctx)) != FDTD_OK)
    return r;
  if (!ctx->d_first_bad)
    DALLOC (ctx->d_first_bad, sizeof (unsigned long long));
  CK (cudaMemcpyAsync (ctx->staging, host, n * sizeof (double), cudaMemcpyHostToDevice, ctx->stream));
  CK (cudaMemsetAsync (ctx->d_first_bad, 0xff, sizeof (unsigned long long), ctx->stream));
  ctx->launches += launch_find_nonfinite (ctx->staging, n, ctx->d_first_bad, ctx->stream);
  unsigned long long first = 0;
  CK (cudaMemcpyAsync (&first, ctx->d_first_bad, sizeof (first), cudaMemcpyDeviceToHost, ctx->stream));
  CK (cudaStreamSynchronize (ctx->stream));
  if (first < n)
    return fail (ctx, FDTD_ERR_ARG, std::string ("material ") + std::to_string (which) +
                                        " holds a non-finite value (cell " + std::to_string (first) +
                                        "); nothing was uploaded");
  r = fdtd_upload_material_device (ctx, which, ctx->staging);
  if (r != FDTD_OK)
    return r;
  CK (cudaStreamSynchronize (ctx->stream));
  return FDTD_OK;
}

int fdtd_upload_material_device (fdtd_ctx *ctx, int which, const double *dev)
{
  if (!ctx || !dev || which < 0 || which > 5)
    return fail (ctx, FDTD_ERR_ARG, "bad argument");
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  size_t n = (size_t) ctx->g.cells;
  if (ctx->g.dmp && which < 2)
    return upload_fine_material (ctx, which, dev, cudaMemcpyDeviceToDevice);
  if (ctx->kind == 0)
  {
    if (!ctx->mat64[which])
      return fail (ctx, FDTD_ERR_UNSUPPORTED, "Drude grids need use_metamaterials");
    CK (cudaMemcpyAsync (ctx->mat64[which], dev, n * sizeof (double), cudaMemcpyDeviceToDevice, ctx->stream));
    return FDTD_OK;
  }
  if (which == 1 && ctx->g.cfg.use_metamaterials && ctx->stepped && !ctx->mat32[1] && ctx->has_second)
    return fail (ctx, FDTD_ERR_UNSUPPORTED, "a 3-D FP32 / FP16 Drude run takes its mu map before its first step "
                                            "(the map moves the run from the one-sweep to the per-cell kernels, "
                                            "whose Drude state differs)");
  if (which > 1)
  {
    if (!ctx->dflag)
      return fail (ctx, FDTD_ERR_UNSUPPORTED, "Drude grids need use_metamaterials");
    // FDTD_MAT_OMEGAPE..GAMMAM = 2..5 -> omegape, omegapm, gammae, gammam
    ctx->launches += launch_convert_in (ctx->drude32[which - 2], 1, dev, n, 1.0, ctx->stream);
    ctx->launches += launch_drude_flags (ctx->dflag, ctx->drude32[0], ctx->drude32[2], ctx->drude32[1],
                                         ctx->drude32[3], ctx->g.n[0], ctx->g.n[1], ctx->g.n[2], ctx->stream);
    CK (cudaGetLastError ());
    if (ctx->sweep_state != 0)
      ctx->sweep_state = 0;   // the Drude cells changed: plan again at the next step
    return FDTD_OK;
  }
  if (!ctx->mat32[which])
    DALLOC (ctx->mat32[which], n * sizeof (float));
  ctx->launches += launch_convert_in (ctx->mat32[which], 1, dev, n, 1.0, ctx->stream);
  CK (cudaGetLastError ());
  return FDTD_OK;
}

int fdtd_upload_field (fdtd_ctx *ctx, int component, const double *host)
{
  if (!ctx || !host || component < 0 || component > 5 || !ctx->g.comp[component].exists)
    return fail (ctx, FDTD_ERR_ARG, "bad argument");
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  size_t n = (size_t) ctx->g.cells;
  if (ctx->kind == 0)
  {
    CK (cudaMemcpyAsync (ctx->f[component][1], host, n * sizeof (double), cudaMemcpyHostToDevice, ctx->stream));
  }
  else
  {
    if ((r = ensure_staging (ctx)) != FDTD_OK)
      return r;
    CK (cudaMemcpyAsync (ctx->staging, host, n * sizeof (double), cudaMemcpyHostToDevice, ctx->stream));
    // every buffer set (the two of the one-sweep kernels and the shell's
    // set T): cells the step never updates must keep these values
    for (int b = 0; b < 3; ++b)
    {
      void *dst = b < 2 ? ctx->ffb[b][component] : ctx->tfb[component];
      if (dst)
        ctx->launches += launch_convert_in (dst, ctx->kind, ctx->staging, n, component >= 3 ? kEta0 : 1.0,
                                            ctx->stream);
    }
  }
  CK (cudaStreamSynchronize (ctx->stream));
  return FDTD_OK;
}

int fdtd_step (fdtd_ctx *ctx, uint32_t t_start, uint32_t n_steps)
{
  if (!ctx)
    return FDTD_ERR_ARG;
  if (n_steps == 0)
    return FDTD_OK;
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  return step_impl (ctx, t_start, n_steps);
}

int fdtd_sync (fdtd_ctx *ctx, int64_t timeout_ns)
{
  if (!ctx)
    return FDTD_ERR_ARG;
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  if (timeout_ns < 0)
  {
    CK (cudaStreamSynchronize (ctx->stream));
    if (ctx->h2d)
    {
      CK (cudaStreamSynchronize (ctx->h2d));
      CK (cudaStreamSynchronize (ctx->d2h));
    }
  }
  else
  {
    auto t0 = std::chrono::steady_clock::now ();
    for (;;)
    {
      cudaError_t e = query_all (ctx);
      if (e == cudaSuccess)
        break;
      if (e != cudaErrorNotReady)
        return fail (ctx, FDTD_ERR_CUDA, std::string ("cudaStreamQuery: ") + cudaGetErrorString (e));
      auto dt = std::chrono::duration_cast<std::chrono::nanoseconds> (std::chrono::steady_clock::now () - t0);
      if (dt.count () >= timeout_ns)
        return fail (ctx, FDTD_ERR_TIMEOUT, "sync timed out");
      std::this_thread::sleep_for (std::chrono::microseconds (50));
    }
  }
  int flag = 0;
  CK (cudaMemcpy (&flag, ctx->d_err, sizeof (int), cudaMemcpyDeviceToHost));
  if (flag)
    return fail (ctx, FDTD_ERR_DEVICE,
                 (flag & 4) ? "a sweep kernel gave up waiting for its tensor copies (pipeline timeout)"
                            : "a kernel reported an out-of-range incident-grid index");
  return FDTD_OK;
}

int fdtd_download_field_device (fdtd_ctx *ctx, int component, double *dev)
{
  if (!ctx || !dev || component < 0 || component > 5 || !ctx->g.comp[component].exists)
    return fail (ctx, FDTD_ERR_ARG, "bad argument");
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  size_t n = (size_t) ctx->g.cells;
  if (ctx->kind == 0)
  {
    CK (cudaMemcpyAsync (dev, ctx->f[component][1], n * sizeof (double), cudaMemcpyDeviceToDevice, ctx->stream));
  }
  else
  {
    ctx->launches += launch_convert_out (dev, ctx->ff[component], ctx->kind, n,
                                         component >= 3 ? 1.0 / kEta0 : 1.0, ctx->stream);
    CK (cudaGetLastError ());
  }
  return FDTD_OK;
}

int fdtd_upload_material_async (fdtd_ctx *ctx, int which, const double *host)
{
  if (!ctx || !host || which < 0 || which > 5)
    return fail (ctx, FDTD_ERR_ARG, "bad argument");
  if (ctx->g.dmp && which < 2)
    return fdtd_upload_material (ctx, which, host);   // the fine grid takes the synchronous path
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  if ((r = ensure_copy_streams (ctx)) != FDTD_OK)
    return r;
  const size_t bytes = (size_t) ctx->g.cells * sizeof (double);
  // the staging grid is free once the previous upload has been applied
  CK (cudaStreamWaitEvent (ctx->h2d, ctx->in_free, 0));
  CK (cudaMemcpyAsync (ctx->stage_in, host, bytes, cudaMemcpyHostToDevice, ctx->h2d));
  CK (cudaEventRecord (ctx->in_ready, ctx->h2d));
  CK (cudaStreamWaitEvent (ctx->stream, ctx->in_ready, 0));
  if ((r = fdtd_upload_material_device (ctx, which, ctx->stage_in)) != FDTD_OK)
    return r;
  CK (cudaEventRecord (ctx->in_free, ctx->stream));
  return FDTD_OK;
}

int fdtd_download_field_async (fdtd_ctx *ctx, int component, double *host)
{
  if (!ctx || !host || component < 0 || component > 5 || !ctx->g.comp[component].exists)
    return fail (ctx, FDTD_ERR_ARG, "bad argument");
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  if ((r = ensure_copy_streams (ctx)) != FDTD_OK)
    return r;
  const size_t bytes = (size_t) ctx->g.cells * sizeof (double);
  // snapshot on the context's stream once the previous copy-out has read the
  // staging grid, then copy out while later steps run
  CK (cudaStreamWaitEvent (ctx->stream, ctx->out_free, 0));
  if ((r = fdtd_download_field_device (ctx, component, ctx->stage_out)) != FDTD_OK)
    return r;
  CK (cudaEventRecord (ctx->out_ready, ctx->stream));
  CK (cudaStreamWaitEvent (ctx->d2h, ctx->out_ready, 0));
  CK (cudaMemcpyAsync (host, ctx->stage_out, bytes, cudaMemcpyDeviceToHost, ctx->d2h));
  CK (cudaEventRecord (ctx->out_free, ctx->d2h));
  return FDTD_OK;
}

int fdtd_incident_length (const fdtd_ctx *ctx)
{
  return ctx && ctx->g.cfg.use_tfsf ? ctx->g.inc_len : 0;
}

int fdtd_download_incident (fdtd_ctx *ctx, int family, double *host, int len)
{
  if (!ctx || !host || (family != 0 && family != 1))
    return fail (ctx, FDTD_ERR_ARG, "bad argument");
  if (!ctx->g.cfg.use_tfsf)
    return fail (ctx, FDTD_ERR_STATE, "no incident grid without TF/SF");
  if (len != ctx->g.inc_len)
    return fail (ctx, FDTD_ERR_ARG, "the incident grid holds fdtd_incident_length () values");
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  const double *src = family ? ctx->hinc[ctx->hcur] : ctx->einc[ctx->ecur];
  CK (cudaMemcpyAsync (host, src, (size_t) len * sizeof (double), cudaMemcpyDeviceToHost, ctx->stream));
  CK (cudaStreamSynchronize (ctx->stream));
  return FDTD_OK;
}

int fdtd_download_field_scattered (fdtd_ctx *ctx, int component, double *host)
{
  if (!ctx || !host || component < 0 || component > 5 || !ctx->g.comp[component].exists)
    return fail (ctx, FDTD_ERR_ARG, "bad argument");
  const Geometry &g = ctx->g;
  if (!g.cfg.use_tfsf)
    return fail (ctx, FDTD_ERR_STATE, "the scattered field needs TF/SF");
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  if ((r = ensure_staging (ctx)) != FDTD_OK)
    return r;
  if ((r = fdtd_download_field_device (ctx, component, ctx->staging)) != FDTD_OK)
    return r;
  double left[3], right[3];
  for (int a = 0; a < 3; ++a)
  {
    left[a] = (double) g.cfg.tfsf_left[a];
    right[a] = (double) (g.n[a] - g.cfg.tfsf_right[a]);
  }
  const double *inc = component >= 3 ? ctx->hinc[ctx->hcur] : ctx->einc[ctx->ecur];
  ctx->launches += launch_scattered (ctx->staging, make_geom_dev (g), component, inc, g.inc_len, left, right,
                                     ctx->d_err, ctx->sm_count, ctx->stream);
  CK (cudaGetLastError ());
  const size_t n = (size_t) g.cells;
  CK (cudaMemcpyAsync (host, ctx->staging, n * sizeof (double), cudaMemcpyDeviceToHost, ctx->stream));
  CK (cudaStreamSynchronize (ctx->stream));
  return FDTD_OK;
}

int fdtd_download_field (fdtd_ctx *ctx, int component, double *host)
{
  if (!ctx || !host || component < 0 || component > 5 || !ctx->g.comp[component].exists)
    return fail (ctx, FDTD_ERR_ARG, "bad argument");
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  size_t n = (size_t) ctx->g.cells;
  if (ctx->kind == 0)
  {
    CK (cudaMemcpyAsync (host, ctx->f[component][1], n * sizeof (double), cudaMemcpyDeviceToHost, ctx->stream));
  }
  else
  {
    if ((r = ensure_staging (ctx)) != FDTD_OK)
      return r;
    if ((r = fdtd_download_field_device (ctx, component, ctx->staging)) != FDTD_OK)
      return r;
    CK (cudaMemcpyAsync (host, ctx->staging, n * sizeof (double), cudaMemcpyDeviceToHost, ctx->stream));
  }
  CK (cudaStreamSynchronize (ctx->stream));
  return FDTD_OK;
}

int fdtd_reduce (fdtd_ctx *ctx, int what, double *out)
{
  if (!ctx || !out || (what != FDTD_REDUCE_ENERGY && what != FDTD_REDUCE_L2))
    return fail (ctx, FDTD_ERR_ARG, "bad argument");
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  size_t n = (size_t) ctx->g.cells;
  for (int k = 0; k < 6; ++k)
  {
    if (!ctx->g.comp[k].exists)
    {
      CK (cudaMemsetAsync (ctx->d_out + k, 0, sizeof (double), ctx->stream));
      continue;
    }
    const void *src = ctx->kind == 0 ? (const void *) ctx->f[k][1] : (const void *) ctx->ff[k];
    const void *w = nullptr;
    int wkind = 0;
    double scale = 1.0;
    bool isH = k >= 3;
    if (what == FDTD_REDUCE_ENERGY)
    {
      // (double material precision: the component's own averaged material)
      if (ctx->kind == 0)
      {
        w = ctx->matc64[k] ? ctx->matc64[k] : ctx->mat64[isH ? 1 : 0];
        wkind = 2;
        scale = isH ? kEta0 * kEta0 : 1.0;
      }
      else
      {
        w = ctx->matc32[k] ? ctx->matc32[k] : ctx->mat32[isH ? 1 : 0];
        wkind = w ? 1 : 0;
      }
    }
    else if (ctx->kind != 0 && isH)
    {
      scale = 1.0 / (kEta0 * kEta0);
    }
    ctx->launches += launch_reduce_sq (src, ctx->kind, n, w, wkind, scale, ctx->partials, ctx->nparts, ctx->stream);
    ctx->launches += launch_reduce_final (ctx->partials, ctx->nparts, ctx->d_out + k, ctx->stream);
  }
  double vals[6];
  CK (cudaMemcpyAsync (vals, ctx->d_out, 6 * sizeof (double), cudaMemcpyDeviceToHost, ctx->stream));
  CK (cudaStreamSynchronize (ctx->stream));
  if (what == FDTD_REDUCE_L2)
  {
    for (int k = 0; k < 6; ++k)
      out[k] = vals[k];
  }
  else
  {
    double s = 0.0, c = 0.0;
    for (int k = 0; k < 6; ++k)
    {
      double t = s + vals[k];
      c += std::fabs (s) >= std::fabs (vals[k]) ? (s - t) + vals[k] : (vals[k] - t) + s;
      s = t;
    }
    out[0] = s + c;
  }
  return FDTD_OK;
}

int fdtd_scalars (const fdtd_ctx *ctx, double out[3])
{
  if (!ctx || !out)
    return FDTD_ERR_ARG;
  out[0] = ctx->g.dt;
  out[1] = ctx->g.freq;
  out[2] = ctx->g.rpv;
  return FDTD_OK;
}

namespace {

int adjoint_entry (fdtd_ctx *ctx, const fdtd_adjoint_cfg *cfg, double *objective, double *grad)
{
  if (!ctx || !cfg || !objective)
    return fail (ctx, FDTD_ERR_ARG, "null argument");
  if (cfg->precision != FDTD_PREC_FP32 && cfg->precision != FDTD_PREC_FP64_PLAIN)
    return fail (ctx, FDTD_ERR_ARG, "adjoint precision must be FP32 or FP64");
  const Geometry &g = ctx->g;
  if (!g.tmz || g.cfg.use_tfsf || g.cfg.use_metamaterials || g.cfg.layout != 0 || g.dmp)
    return fail (ctx, FDTD_ERR_UNSUPPORTED, "the adjoint covers 2-D TMz point-source runs (E_CENTERED)");
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  AdjointRun run;
  run.steps = cfg->steps;
  run.every = cfg->checkpoint_every;
  run.cache = &ctx->adj_cache;
  for (int a = 0; a < 2; ++a)
  {
    run.probe_lo[a] = cfg->probe_lo[a];
    run.probe_hi[a] = cfg->probe_hi[a];
  }
  run.fp64 = cfg->precision == FDTD_PREC_FP64_PLAIN;
  run.wait_limit_ns = ctx->wait_limit_ns;
  // eps as the context holds it: FP64 (plain form) or FP32 (null = uniform 1)
  const void *eps = ctx->kind == 0 ? (const void *) ctx->mat64[0] : (const void *) ctx->mat32[0];
  CK (cudaStreamSynchronize (ctx->stream));
  std::string why = adjoint_run (g, eps, ctx->kind == 0, run, objective, grad, ctx->sm_count, ctx->stream);
  if (!why.empty ())
    return fail (ctx,
                 why.find ("timed out") != std::string::npos
                     ? FDTD_ERR_DEVICE
                     : (why.find ("allocation") != std::string::npos
                            ? FDTD_ERR_NOMEM
                            : (why.find ("failed") != std::string::npos ? FDTD_ERR_CUDA : FDTD_ERR_ARG)),
                 why);
  return FDTD_OK;
}

}  // namespace

int fdtd_objective (fdtd_ctx *ctx, const fdtd_adjoint_cfg *cfg, double *objective)
{
  return adjoint_entry (ctx, cfg, objective, nullptr);
}

int fdtd_backward (fdtd_ctx *ctx, const fdtd_adjoint_cfg *cfg, double *objective, double *dobj_deps)
{
  if (!dobj_deps)
    return fail (ctx, FDTD_ERR_ARG, "null gradient buffer");
  return adjoint_entry (ctx, cfg, objective, dobj_deps);
}

int fdtd_dft_setup (fdtd_ctx *ctx, int component, int axis, int index, int nfreq, const double *freq_hz)
{
  if (!ctx || component < 0 || component > 5 || !ctx->g.comp[component].exists || axis < 0 || axis > 2 ||
      index < 0 || index >= ctx->g.n[axis] || nfreq < 1 || nfreq > 64 || !freq_hz)
    return fail (ctx, FDTD_ERR_ARG, "bad DFT plane, component or frequency list");
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  const int *n = ctx->g.n;
  const size_t cells = (size_t) (axis == 0 ? n[1] : n[0]) * (axis == 2 ? n[1] : n[2]);
  CK (cudaStreamSynchronize (ctx->stream));
  if (ctx->dft_acc)
  {
    cudaFree (ctx->dft_acc);
    ctx->allocs.erase (std::remove (ctx->allocs.begin (), ctx->allocs.end (), (void *) ctx->dft_acc),
                       ctx->allocs.end ());
    ctx->dft_acc = nullptr;
  }
  DALLOC (ctx->dft_acc, cells * nfreq * 4 * sizeof (double));
  ctx->dft_comp = component;
  ctx->dft_axis = axis;
  ctx->dft_index = index;
  ctx->dft_nf = nfreq;
  ctx->dft_freq.assign (freq_hz, freq_hz + nfreq);
  CK (cudaStreamSynchronize (ctx->stream));
  return FDTD_OK;
}

int fdtd_dft_read (fdtd_ctx *ctx, double *out)
{
  if (!ctx || !out)
    return fail (ctx, FDTD_ERR_ARG, "bad argument");
  if (ctx->dft_comp < 0)
    return fail (ctx, FDTD_ERR_STATE, "no DFT set up");
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  const int *n = ctx->g.n;
  const int axis = ctx->dft_axis;
  const size_t cells = (size_t) (axis == 0 ? n[1] : n[0]) * (axis == 2 ? n[1] : n[2]);
  std::vector<double> acc (cells * ctx->dft_nf * 4);
  CK (cudaMemcpyAsync (acc.data (), ctx->dft_acc, acc.size () * sizeof (double), cudaMemcpyDeviceToHost,
                       ctx->stream));
  CK (cudaStreamSynchronize (ctx->stream));
  for (size_t q = 0; q < cells * ctx->dft_nf; ++q)
  {
    out[2 * q] = acc[4 * q] + acc[4 * q + 1];
    out[2 * q + 1] = acc[4 * q + 2] + acc[4 * q + 3];
  }
  return FDTD_OK;
}

int fdtd_ntff (fdtd_ctx *re, fdtd_ctx *im, const int left[3], const int right[3], double teta, int nphi,
               const double *phi, double *out)
{
  if (!re || !im || !left || !right || !phi || !out || nphi < 1 || re == im)
    return fail (re, FDTD_ERR_ARG, "bad argument");
  const Geometry &g = re->g;
  const Geometry &gi = im->g;
  if (re->kind != im->kind)
    return fail (re, FDTD_ERR_ARG, "the two runs must have the same form");
  if (re->kind != 0 && (re->prev_src == 0 || im->prev_src == 0))
    return fail (re, FDTD_ERR_STATE, "the NTFF needs the previous H level: call fdtd_keep_previous_level before "
                                     "stepping an FP32 / FP16 run");
  if (g.cfg.mode != FDTD_MODE_DIM3 || gi.cfg.mode != FDTD_MODE_DIM3)
    return fail (re, FDTD_ERR_UNSUPPORTED, "the NTFF is 3-D (the reference's 2-D and 1-D forms are unreachable)");
  if (re->device != im->device || g.cfg.layout != gi.cfg.layout)
    return fail (re, FDTD_ERR_ARG, "the two runs must share the device and the layout");
  for (int a = 0; a < 3; ++a)
  {
    if (g.n[a] != gi.n[a])
      return fail (re, FDTD_ERR_ARG, "the two runs must have the same grid");
    if (left[a] < 1 || right[a] <= left[a] || right[a] > g.n[a] - 1)
      return fail (re, FDTD_ERR_ARG, "NTFF box out of range (1 <= left < right <= size - 1)");
  }
  fdtd_ctx *ctx = re;   // errors are reported on the first run
  int r = set_device (re);
  if (r != FDTD_OK)
    return r;
  CK (cudaStreamSynchronize (im->stream));
  NtffParams p;
  std::memset (&p, 0, sizeof (p));
  int64_t len[3];
  for (int a = 0; a < 3; ++a)
  {
    p.n[a] = g.n[a];
    p.left[a] = left[a];
    p.right[a] = right[a];
    p.diff0[a] = (double) (g.n[a] / 2);
    len[a] = right[a] - left[a];
  }
  p.points = 2 * (len[1] * len[2] + len[0] * len[2] + len[0] * len[1]);
  p.dx = g.cfg.dx;
  p.k = 2 * kPi / g.cfg.wavelength;
  p.teta = teta;
  p.h_centered = g.cfg.layout == 1;
  p.kind = re->kind;
  fdtd_ctx *runs[2] = {re, im};
  for (int k = 0; k < 6; ++k)
  {
    for (int a = 0; a < 3; ++a)
      p.min_fp[k][a] = g.comp[k].min_fp[a];
    for (int q = 0; q < 2; ++q)
    {
      const fdtd_ctx *c = runs[q];
      if (c->kind == 0)
      {
        // after a step the current level is 1 and the previous one 0 (two
        // levels) or 2 (three), the reference's "after shift" accessors
        p.cur[q][k] = c->f[k][1];
        p.prev[q][k] = c->f[k][g.levels == 3 ? 2 : 0];
      }
      else
      {
        // FP32 / FP16 storage: the current set, the previous H where the
        // last call left it (the E sums read the current level only)
        p.cur[q][k] = c->ffb[c->fcur][k];
        p.prev[q][k] = k < 3 ? nullptr : (c->prev_src == 1 ? c->ffb[1 - c->fcur][k] : c->hprev[k - 3]);
      }
    }
    p.scale[k] = k < 3 ? 1.0 : 1.0 / kEta0;
  }
  const int blocks = (int) std::max<int64_t> (1, std::min<int64_t> ((p.points + 255) / 256, 4 * re->sm_count));
  double *phi_dev = nullptr, *partial = nullptr, *sums = nullptr;
  struct Free
  {
    double **p[3];
    ~Free ()
    {
      for (double **q : p)
        if (*q)
          cudaFree (*q);
    }
  } release{{&phi_dev, &partial, &sums}};
  CK (device_malloc ((void **) &phi_dev, (size_t) nphi * sizeof (double)));
  CK (device_malloc ((void **) &partial, (size_t) nphi * blocks * 8 * sizeof (double)));
  CK (device_malloc ((void **) &sums, (size_t) nphi * 8 * sizeof (double)));
  CK (cudaMemcpyAsync (phi_dev, phi, (size_t) nphi * sizeof (double), cudaMemcpyHostToDevice, re->stream));
  re->launches += launch_ntff (p, phi_dev, nphi, partial, blocks, sums, re->stream);
  CK (cudaGetLastError ());
  std::vector<double> h ((size_t) nphi * 8);
  CK (cudaMemcpyAsync (h.data (), sums, h.size () * sizeof (double), cudaMemcpyDeviceToHost, re->stream));
  CK (cudaStreamSynchronize (re->stream));
  // Pointing_scat over Pointing_inc (Scheme.inc.h:4080-4095)
  const double k = 2 * kPi / g.cfg.wavelength;
  const double n0 = std::sqrt (kMu0 / kEps0);
  for (int i = 0; i < nphi; ++i)
  {
    const double *v = &h[(size_t) i * 8];
    const double f_re = v[6] + v[0] * n0, f_im = v[7] + v[1] * n0;   // L.phi + N.teta n0
    const double s_re = v[4] - v[2] * n0, s_im = v[5] - v[3] * n0;   // L.teta - N.phi n0
    const double first_abs2 = f_re * f_re + f_im * f_im;
    const double second_abs2 = s_re * s_re + s_im * s_im;
    double val = (k * k) / (8 * kPi * n0) * (first_abs2 + second_abs2);
    val /= std::sqrt (kEps0 / kMu0) / 2;
    out[i] = val;
  }
  return FDTD_OK;
}

int fdtd_keep_previous_level (fdtd_ctx *ctx, int on)
{
  if (!ctx)
    return fail (ctx, FDTD_ERR_ARG, "bad argument");
  if (ctx->kind == 0)
    return FDTD_OK;   // the FP64 plain form keeps its time levels anyway
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  if (on && !ctx->hprev[0])
    for (int ci = 0; ci < 3; ++ci)
      if ((r = dalloc (ctx, &ctx->hprev[ci], (size_t) ctx->g.cells * elem_size (ctx->kind))) != FDTD_OK)
        return r;
  ctx->keep_prev = on != 0;
  ctx->prev_src = 0;
  return FDTD_OK;
}

const char *fdtd_step_kernel (const fdtd_ctx *ctx)
{
  return ctx ? ctx->step_kernel : nullptr;
}

int64_t fdtd_launch_count (const fdtd_ctx *ctx)
{
  return ctx ? ctx->launches : -1;
}

void *fdtd_stream (const fdtd_ctx *ctx)
{
  return ctx ? (void *) ctx->stream : nullptr;
}

int fdtd_profile (fdtd_ctx *ctx, int enable)
{
  if (!ctx)
    return FDTD_ERR_ARG;
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  CK (cudaStreamSynchronize (ctx->stream));
  ctx->profiling = enable != 0;
  ctx->prof_used = 0;
  return FDTD_OK;
}

int fdtd_kernel_time (fdtd_ctx *ctx, double *ms, int64_t *launches)
{
  if (!ctx || !ms || !launches)
    return FDTD_ERR_ARG;
  int r = set_device (ctx);
  if (r != FDTD_OK)
    return r;
  CK (cudaStreamSynchronize (ctx->stream));
  double total = 0.0;
  for (size_t i = 0; i + 1 < ctx->prof_used; i += 2)
  {
    float t = 0.f;
    CK (cudaEventElapsedTime (&t, ctx->prof_events[i], ctx->prof_events[i + 1]));
    total += t;
  }
  *ms = total;
  *launches = (int64_t) (ctx->prof_used / 2);
  ctx->prof_used = 0;
  return FDTD_OK;
}

void fdtd_destroy (fdtd_ctx *ctx)
{
  release (ctx);
}

const char *fdtd_status_str (int status)
{
  switch (status)
  {
    case FDTD_OK: return "ok";
    case FDTD_ERR_ARG: return "invalid argument or configuration";
    case FDTD_ERR_CUDA: return "CUDA runtime error";
    case FDTD_ERR_NOMEM: return "out of memory";
    case FDTD_ERR_TIMEOUT: return "timed out";
    case FDTD_ERR_UNSUPPORTED: return "unsupported mode or option";
    case FDTD_ERR_STATE: return "call out of order";
    case FDTD_ERR_DEVICE: return "device-side error flag";
    default: return "unknown status";
  }
}

const char *fdtd_last_error (void)
{
  return g_last_error.c_str ();
}

int fdtd_set_wait_limit (fdtd_ctx *ctx, int64_t limit_ns)
{
  if (!ctx)
    return FDTD_ERR_ARG;
  ctx->wait_limit_ns = limit_ns > 0 ? limit_ns : 0;
  return FDTD_OK;
}

int fdtd_inject_alloc_failure (int64_t after)
{
  g_alloc_budget.store (after < 0 ? -1 : after);
  return FDTD_OK;
}

}  // extern "C"

void fdtdb::set_last_error (const char *msg)
{
  g_last_error = msg ? msg : "";
}

namespace {

bool injected_alloc_failure ()
{
  long long b = g_alloc_budget.load ();
  while (b > 0 && !g_alloc_budget.compare_exchange_weak (b, b - 1))
    ;
  return b == 0;
}

}  // namespace

cudaError_t fdtdb::device_malloc (void **p, size_t bytes)
{
  if (injected_alloc_failure ())
  {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc (p, bytes);
}

cudaError_t fdtdb::pinned_malloc (void **p, size_t bytes)
{
  if (injected_alloc_failure ())
  {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocHost (p, bytes);
}

extern "C" {

}  // extern "C"
