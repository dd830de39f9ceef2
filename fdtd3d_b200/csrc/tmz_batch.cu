// tmz_batch.cu - many 2-D TMz simulations of uneven sizes in one persistent
// kernel launch (captured in a CUDA graph), FP32.
//
// Every instance is an fdtd3d Dim2_TMz E_CENTERED run (Ez, Hx, Hy) with PML,
// its own eps map and a point source at its centre; they share dx, Courant
// factor, PML width and source.  The formulation per instance is the FP32
// form of fast_kernels.cu (H stored as eta0*H, PML auxiliaries only in PML
// cells); the step semantics are the reference's (no field update at t = 0,
// Source/Scheme/Scheme.inc.h:1032; hard point source after the E update).
//
// Work decomposition: a work list of tiles (instance, 30-cell y strip,
// x chunk).  One warp owns a tile: lane 0 holds the y-1 halo, lanes 1..30
// the owned cells, lane 31 the y+1 ring whose Ez it recomputes; neighbours
// along y move by warp shuffles, along x by registers as the warp marches.
// E and H of one time step are done in that single sweep (fields double
// buffered, so tiles need no mutual ordering inside a step).  Warps take
// tiles from a per-step atomic counter; a grid-wide barrier separates time
// steps.  The barrier is a bounded spin on a global generation counter
// (globaltimer timeout -> error flag, every CTA leaves); the kernel is
// launched cooperatively so all CTAs are co-resident.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fdtd_b200.h"
#include "kernels.h"
#include "setup.h"

namespace fdtdb {

namespace {

constexpr int kStrip = 30;            // owned y cells per warp tile
constexpr double kEta0B = 376.730313461770655;

struct InstDev
{
  long long off;                      // first cell of the instance in every arena
  int nx, ny;
  int tab;                            // first entry of the instance's 1-D tables
  int ilo[3][2], ihi[3][2];           // per component (Ez, Hx, Hy): sigma == 0 range in x, y
  int ps;                             // 1: point source at the centre
};

// per instance, 12 tables laid out back to back:
//   Ez: ca1(x) sq1(x) p5(y) q5(y)    Hx: g4p(x) g4m(x) ca1(y) sq1(y)    Hy: p5(x) q5(x) g4p(y) g4m(y)
// each of length nx or ny, in that order

struct TileDev
{
  int inst, y0, xa, xb;
};

struct BatchParams
{
  const InstDev *inst;
  const TileDev *tiles;
  int ntiles;
  const float *tab;
  float *ez[2], *hx[2], *hy[2];
  float *aez[2], *ahx[2], *ahy[2];
  const float *eps;
  const double *src;                  // E source value per step of this launch
  float courant;
  int use_pml;
  unsigned *counters;                 // [0], [1]: tile counters by step parity; [2]: barrier arrivals
  unsigned *generation;
  int *err;
  long long timeout_ns;
  // per launch
  unsigned t_start;
  unsigned nsteps;
  int cur;                            // buffer set holding the current time level
};

__device__ __forceinline__ long long globaltimer ()
{
  long long t;
  asm volatile ("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier with a time limit.  Returns false if any CTA gave up.
__device__ bool grid_barrier (const BatchParams &p)
{
  __shared__ int ok;
  __syncthreads ();
  if (threadIdx.x == 0)
  {
    volatile unsigned *gen = p.generation;
    unsigned g = *gen;
    __threadfence ();
    unsigned arrived = atomicAdd (&p.counters[2], 1u);
    if (arrived == gridDim.x - 1)
    {
      atomicExch (&p.counters[2], 0u);
      __threadfence ();
      atomicAdd ((unsigned *) p.generation, 1u);
    }
    else
    {
      long long t0 = globaltimer ();
      while (*gen == g)
      {
        if (*((volatile int *) p.err) != 0 || globaltimer () - t0 > p.timeout_ns)
        {
          atomicExch (p.err, 2);
          break;
        }
        __nanosleep (64);
      }
    }
    __threadfence ();
    ok = *((volatile int *) p.err) == 0;
  }
  __syncthreads ();
  return ok != 0;
}

__device__ __forceinline__ float pml_update (bool interior, float f, float curl, float inv_m, float ca1, float sq1,
                                             float p5, float q5, float g4p, float g4m, const float *ao, float *an,
                                             long long id, bool store, float courant)
{
  if (interior)
    return f + courant * inv_m * curl;
  const float xo = ao[id];
  const float xn = ca1 * xo + sq1 * curl;
  if (store)
    an[id] = xn;
  return p5 * f + (g4p * xn - g4m * xo) * q5 * inv_m;
}

__global__ void __launch_bounds__ (512) tmz_batch_kernel (BatchParams p)
{
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  __shared__ int s_tile[32];
  int cur = p.cur;
  for (unsigned s = 0; s < p.nsteps; ++s)
  {
    const unsigned t = p.t_start + s;
    const int o = cur, nw = 1 - cur;
    if (t == 0)
    {
      // no field update at t = 0; the hard source still sets Ez
      if (blockIdx.x == 0)
      {
        for (int i = threadIdx.x; i < p.ntiles; i += blockDim.x)
        {
          const TileDev td = p.tiles[i];
          const InstDev in = p.inst[td.inst];
          if (in.ps && td.y0 == 1 && td.xa == 1)
          {
            long long id = in.off + (long long) (in.nx / 2) * in.ny + in.ny / 2;
            p.ez[o][id] = (float) p.src[s];
          }
        }
      }
      if (!grid_barrier (p))
        return;
      continue;
    }
    const int warp = threadIdx.x >> 5;
    for (;;)
    {
      int tile;
      if (lane == 0)
        tile = (int) atomicAdd (&p.counters[t & 1], 1u);
      tile = __shfl_sync (0xffffffffu, tile, 0);
      if (tile >= p.ntiles)
        break;
      const TileDev td = p.tiles[tile];
      const InstDev in = p.inst[td.inst];
      const int nx = in.nx, ny = in.ny;
      const int y = td.y0 - 1 + lane;
      const bool valid = y <= ny - 1;
      const bool inner = y >= 1 && y <= ny - 2;
      const bool own = lane >= 1 && lane <= kStrip && inner;
      const long long base = in.off + y;
      const float *T = p.tab + in.tab;
      const float *ez_ca1 = T, *ez_sq1 = T + nx, *ez_p5 = T + 2 * nx, *ez_q5 = T + 2 * nx + ny;
      const float *hx_g4p = T + 2 * nx + 2 * ny, *hx_g4m = T + 3 * nx + 2 * ny, *hx_ca1 = T + 4 * nx + 2 * ny,
                  *hx_sq1 = T + 4 * nx + 3 * ny;
      const float *hy_p5 = T + 4 * nx + 4 * ny, *hy_q5 = T + 5 * nx + 4 * ny, *hy_g4p = T + 6 * nx + 4 * ny,
                  *hy_g4m = T + 6 * nx + 5 * ny;
      const bool ps_col = in.ps && y == ny / 2;
      const int psx = nx / 2;
      const bool y_in_ez = y >= in.ilo[0][1] && y < in.ihi[0][1];
      const bool y_in_hx = y >= in.ilo[1][1] && y < in.ihi[1][1];
      const bool y_in_hy = y >= in.ilo[2][1] && y < in.ihi[2][1];
      const float ez_p5y = valid ? ez_p5[y] : 1.f, ez_q5y = valid ? ez_q5[y] : 1.f;
      const float hx_ca1y = valid ? hx_ca1[y] : 1.f, hx_sq1y = valid ? hx_sq1[y] : 0.f;
      const float hy_g4py = valid ? hy_g4p[y] : 1.f, hy_g4my = valid ? hy_g4m[y] : 1.f;

      // state of plane xa - 1
      float hy_prev = 0.f, hx_prev = 0.f, ez_prev = 0.f;
      if (valid)
      {
        const long long id = base + (long long) (td.xa - 1) * ny;
        hy_prev = p.hy[o][id];
        hx_prev = p.hx[o][id];
      }
      // the old fields of plane x are loaded three planes ahead (a register
      // ring), so each warp keeps four planes of loads in flight; loads read
      // only the old buffers and stores go to the new ones
      const float *Hx = p.hx[o], *Hy = p.hy[o], *Ez = p.ez[o];
      auto load = [&] (int x, float &a, float &b, float &c, float &d) {
        a = b = c = 0.f;
        d = 1.f;
        if (valid && x <= td.xb + 1)
        {
          const long long id = base + (long long) x * ny;
          a = Hx[id];
          b = Hy[id];
          c = Ez[id];
          if (p.eps)
            d = p.eps[id];
        }
      };
      float c_hx, c_hy, c_ez, c_ep, n1_hx, n1_hy, n1_ez, n1_ep, n2_hx, n2_hy, n2_ez, n2_ep, n3_hx, n3_hy, n3_ez,
          n3_ep;
      load (td.xa, c_hx, c_hy, c_ez, c_ep);
      load (td.xa + 1, n1_hx, n1_hy, n1_ez, n1_ep);
      load (td.xa + 2, n2_hx, n2_hy, n2_ez, n2_ep);
      load (td.xa + 3, n3_hx, n3_hy, n3_ez, n3_ep);
      for (int x = td.xa; x <= td.xb + 1; ++x)
      {
        const long long id = base + (long long) x * ny;
        const float hx = c_hx, hy = c_hy, ez = c_ez, ep = c_ep;
        c_hx = n1_hx, c_hy = n1_hy, c_ez = n1_ez, c_ep = n1_ep;
        n1_hx = n2_hx, n1_hy = n2_hy, n1_ez = n2_ez, n1_ep = n2_ep;
        n2_hx = n3_hx, n2_hy = n3_hy, n2_ez = n3_ez, n2_ep = n3_ep;
        load (x + 4, n3_hx, n3_hy, n3_ez, n3_ep);
        const float hx_m = __shfl_up_sync (0xffffffffu, hx, 1);
        float ezn = ez;
        if (lane >= 1 && inner && x <= nx - 2)
        {
          const float curl = (hy - hy_prev) - (hx - hx_m);
          const bool interior = !p.use_pml || (y_in_ez && x >= in.ilo[0][0] && x < in.ihi[0][0]);
          ezn = pml_update (interior, ez, curl, 1.f / ep, ez_ca1[x], ez_sq1[x], ez_p5y, ez_q5y, 1.f, 1.f,
                            p.aez[o], p.aez[nw], id, own && x <= td.xb, p.courant);
          if (ps_col && x == psx)
            ezn = (float) p.src[s];
          if (own && x <= td.xb)
            p.ez[nw][id] = ezn;
        }
        // H at x - 1 from Ez_new(x - 1) (this lane and lane + 1) and Ez_new(x)
        const float ezp_dn = __shfl_down_sync (0xffffffffu, ez_prev, 1);
        const int xh = x - 1;
        if (own && xh >= td.xa && xh <= nx - 2)
        {
          const long long hid = id - ny;
          const float cx = ez_prev - ezp_dn;      // Hx: Ez(y) - Ez(y + 1)
          const float cy = ezn - ez_prev;         // Hy: Ez(x + 1) - Ez(x)
          const bool ix = !p.use_pml || (y_in_hx && xh >= in.ilo[1][0] && xh < in.ihi[1][0]);
          const bool iy = !p.use_pml || (y_in_hy && xh >= in.ilo[2][0] && xh < in.ihi[2][0]);
          const float hxn = pml_update (ix, hx_prev, cx, 1.f, hx_ca1y, hx_sq1y, 1.f, 1.f, hx_g4p[xh], hx_g4m[xh],
                                        p.ahx[o], p.ahx[nw], hid, true, p.courant);
          const float hyn = pml_update (iy, hy_prev, cy, 1.f, 1.f, p.courant, hy_p5[xh], hy_q5[xh], hy_g4py,
                                        hy_g4my, p.ahy[o], p.ahy[nw], hid, true, p.courant);
          p.hx[nw][hid] = hxn;
          p.hy[nw][hid] = hyn;
        }
        hx_prev = hx;
        hy_prev = hy;
        ez_prev = ezn;
      }
    }
    (void) warp;
    (void) s_tile;
    // the counter of the next step (same parity as the previous one) is idle now
    if (blockIdx.x == 0 && threadIdx.x == 0)
      atomicExch (&p.counters[(t + 1) & 1], 0u);
    if (!grid_barrier (p))
      return;
    cur = nw;
  }
}

}  // namespace

}  // namespace fdtdb

// --------------------------------------------------------------------------
// host side

struct fdtd_batch
{
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  fdtd_config base;
  std::vector<fdtdb::Geometry> geo;
  std::vector<fdtdb::InstDev> inst;
  long long cells = 0;
  int ntab = 0;
  std::vector<float> tab_host;
  fdtdb::InstDev *d_inst = nullptr;
  fdtdb::TileDev *d_tiles = nullptr;
  int ntiles = 0;
  float *d_tab = nullptr;
  float *ez[2] = {}, *hx[2] = {}, *hy[2] = {}, *aez[2] = {}, *ahx[2] = {}, *ahy[2] = {};
  float *eps = nullptr;
  double *d_src = nullptr, *h_src = nullptr;
  size_t src_cap = 0;
  unsigned *d_counters = nullptr;
  unsigned *d_generation = nullptr;
  int *d_err = nullptr;
  int cur = 0;
  // launch shape (autotuned)
  int x_chunk = 64;
  int warps_per_cta = 8;
  int ctas_per_sm = 2;
  // graph of (source upload, counter reset, persistent kernel)
  cudaGraphExec_t graph = nullptr;
  unsigned graph_steps = 0;
  unsigned graph_t = 0;
  int graph_cur = -1;
  bool use_graph = true;
  bool graph_ok = false;
  double last_ms = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  long long wait_limit_ns = 0;        // grid-barrier wait limit (<= 0: 5 s)
  std::string err;
  std::vector<void *> allocs;
};

namespace {

using fdtdb::BatchParams;

int bfail (fdtd_batch *b, int code, const std::string &m)
{
  if (b)
    b->err = m;
  return code;
}

#define BCK(call)                                                                                  \
  do                                                                                               \
  {                                                                                                \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return bfail (b, e_ == cudaErrorMemoryAllocation ? FDTD_ERR_NOMEM : FDTD_ERR_CUDA,           \
                    std::string (#call) + ": " + cudaGetErrorString (e_));                          \
  } while (0)

int balloc (fdtd_batch *b, void **p, size_t bytes)
{
  cudaError_t e = fdtdb::device_malloc (p, bytes ? bytes : 16);
  if (e != cudaSuccess)
    return bfail (b, FDTD_ERR_NOMEM, std::string ("cudaMalloc: ") + cudaGetErrorString (e));
  b->allocs.push_back (*p);
  e = cudaMemsetAsync (*p, 0, bytes ? bytes : 16, b->stream);
  return e == cudaSuccess ? FDTD_OK : bfail (b, FDTD_ERR_CUDA, cudaGetErrorString (e));
}

#define BALLOC(ptr, bytes)                                                                         \
  do                                                                                               \
  {                                                                                                \
    int r_ = balloc (b, (void **) &(ptr), (bytes));                                                \
    if (r_ != FDTD_OK)                                                                             \
      return r_;                                                                                   \
  } while (0)

int build_tiles (fdtd_batch *b, int x_chunk)
{
  std::vector<fdtdb::TileDev> tiles;
  // large instances first so the atomic work queue ends on small tiles
  std::vector<int> order (b->inst.size ());
  for (size_t i = 0; i < order.size (); ++i)
    order[i] = (int) i;
  std::sort (order.begin (), order.end (), [&] (int a, int c) {
    return (long long) b->inst[a].nx * b->inst[a].ny > (long long) b->inst[c].nx * b->inst[c].ny;
  });
  for (int i : order)
  {
    const fdtdb::InstDev &in = b->inst[i];
    for (int xa = 1; xa <= in.nx - 2; xa += x_chunk)
      for (int y0 = 1; y0 <= in.ny - 2; y0 += fdtdb::kStrip)
        tiles.push_back ({i, y0, xa, std::min (xa + x_chunk - 1, in.nx - 2)});
  }
  if (b->d_tiles)
  {
    auto it = std::find (b->allocs.begin (), b->allocs.end (), (void *) b->d_tiles);
    if (it != b->allocs.end ())
      b->allocs.erase (it);
    BCK (cudaStreamSynchronize (b->stream));
    cudaFree (b->d_tiles);
    b->d_tiles = nullptr;
  }
  BALLOC (b->d_tiles, tiles.size () * sizeof (fdtdb::TileDev));
  BCK (cudaMemcpyAsync (b->d_tiles, tiles.data (), tiles.size () * sizeof (fdtdb::TileDev), cudaMemcpyHostToDevice,
                        b->stream));
  BCK (cudaStreamSynchronize (b->stream));
  b->ntiles = (int) tiles.size ();
  b->x_chunk = x_chunk;
  return FDTD_OK;
}

void drop_graph (fdtd_batch *b)
{
  if (b->graph)
    cudaGraphExecDestroy (b->graph);
  b->graph = nullptr;
  b->graph_steps = 0;
  b->graph_cur = -1;
}

BatchParams params (fdtd_batch *b, uint32_t t_start, uint32_t n)
{
  BatchParams p;
  std::memset (&p, 0, sizeof (p));
  p.inst = b->d_inst;
  p.tiles = b->d_tiles;
  p.ntiles = b->ntiles;
  p.tab = b->d_tab;
  for (int s = 0; s < 2; ++s)
  {
    p.ez[s] = b->ez[s];
    p.hx[s] = b->hx[s];
    p.hy[s] = b->hy[s];
    p.aez[s] = b->aez[s];
    p.ahx[s] = b->ahx[s];
    p.ahy[s] = b->ahy[s];
  }
  p.eps = b->eps;
  p.src = b->d_src;
  p.courant = (float) (fdtdb::kC * b->geo[0].dt / b->geo[0].dx);
  p.use_pml = b->base.use_pml;
  p.counters = b->d_counters;
  p.generation = b->d_generation;
  p.err = b->d_err;
  p.timeout_ns = b->wait_limit_ns > 0 ? b->wait_limit_ns : 5000000000LL;
  p.t_start = t_start;
  p.nsteps = n;
  p.cur = b->cur;
  return p;
}

int max_ctas (fdtd_batch *b, int warps)
{
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor (&per_sm, fdtdb::tmz_batch_kernel, warps * 32, 0)
      != cudaSuccess)
    return 0;
  return per_sm;
}

// Enqueues one launch (source upload, counter reset, cooperative kernel).
int enqueue (fdtd_batch *b, uint32_t t_start, uint32_t n)
{
  BCK (cudaMemcpyAsync (b->d_src, b->h_src, (size_t) n * sizeof (double), cudaMemcpyHostToDevice, b->stream));
  BCK (cudaMemsetAsync (b->d_counters, 0, 3 * sizeof (unsigned), b->stream));
  BatchParams p = params (b, t_start, n);
  void *args[] = {&p};
  int ctas = std::min (b->ctas_per_sm, max_ctas (b, b->warps_per_cta)) * b->sm_count;
  if (ctas <= 0)
    return bfail (b, FDTD_ERR_CUDA, "batch kernel does not fit on the device");
  cudaLaunchConfig_t lc;
  std::memset (&lc, 0, sizeof (lc));
  lc.gridDim = dim3 (ctas);
  lc.blockDim = dim3 (b->warps_per_cta * 32);
  lc.stream = b->stream;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeCooperative;
  attr.val.cooperative = 1;
  lc.attrs = &attr;
  lc.numAttrs = 1;
  BCK (cudaLaunchKernelExC (&lc, (const void *) fdtdb::tmz_batch_kernel, args));
  return FDTD_OK;
}

}  // namespace

namespace fdtdb {
namespace {

__global__ void fill_float_kernel (float *p, size_t n, float v)
{
  for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
    p[i] = v;
}

}  // namespace
}  // namespace fdtdb

namespace {

int create_batch (fdtd_batch *b, const fdtd_config *base, int count, const int *sizes, int device)
{
  using namespace fdtdb;
  if (base->mode != FDTD_MODE_TMZ || base->precision != FDTD_PREC_FP32)
    return bfail (b, FDTD_ERR_UNSUPPORTED, "batches are 2-D TMz, FP32");
  if (base->use_tfsf || base->use_metamaterials)
    return bfail (b, FDTD_ERR_UNSUPPORTED, "batches provide PML and a centred point source (no TF/SF, no Drude)");
  if (base->layout != 0 || base->double_material_precision || base->current_source_mask)
    return bfail (b, FDTD_ERR_UNSUPPORTED,
                  "batches use the E_CENTERED layout, cell-centred materials and no current source");
  if (count < 1 || !sizes)
    return bfail (b, FDTD_ERR_ARG, "empty batch");
  int ndev = 0;
  if (cudaGetDeviceCount (&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return bfail (b, FDTD_ERR_CUDA, "no such CUDA device");
  b->device = device;
  b->base = *base;
  BCK (cudaSetDevice (device));
  BCK (cudaDeviceGetAttribute (&b->sm_count, cudaDevAttrMultiProcessorCount, device));
  int coop = 0;
  BCK (cudaDeviceGetAttribute (&coop, cudaDevAttrCooperativeLaunch, device));
  if (!coop)
    return bfail (b, FDTD_ERR_UNSUPPORTED, "device cannot launch cooperative kernels");
  BCK (cudaStreamCreateWithFlags (&b->stream, cudaStreamNonBlocking));
  BCK (cudaEventCreate (&b->ev0));
  BCK (cudaEventCreate (&b->ev1));
  b->geo.resize (count);
  b->inst.resize (count);
  const double S_unused = 0;
  (void) S_unused;
  for (int i = 0; i < count; ++i)
  {
    fdtd_config c = *base;
    c.size[0] = sizes[2 * i];
    c.size[1] = sizes[2 * i + 1];
    c.size[2] = 1;
    c.point_source[0] = c.size[0] / 2;
    c.point_source[1] = c.size[1] / 2;
    c.point_source[2] = 0;
    c.point_source_mask &= 1 << FDTD_EZ;
    std::string e = build_geometry (c, b->geo[i]);
    if (!e.empty ())
      return bfail (b, FDTD_ERR_ARG, "instance " + std::to_string (i) + ": " + e);
    const Geometry &g = b->geo[i];
    InstDev &in = b->inst[i];
    std::memset (&in, 0, sizeof (in));
    in.off = b->cells;
    in.nx = g.n[0];
    in.ny = g.n[1];
    in.tab = (int) b->tab_host.size ();
    in.ps = c.point_source_mask ? 1 : 0;
    b->cells += (long long) in.nx * in.ny;
    const double S = kC * g.dt / g.dx;
    // tables: Ez ca1(x) sq1(x) p5(y) q5(y); Hx g4p(x) g4m(x) ca1(y) sq1(y); Hy p5(x) q5(x) g4p(y) g4m(y)
    struct Spec
    {
      int comp, axis, kind;
    };
    static const Spec spec[12] = {{EZ, 0, 0}, {EZ, 0, 1}, {EZ, 1, 2}, {EZ, 1, 3}, {HX, 0, 4}, {HX, 0, 5},
                                  {HX, 1, 0}, {HX, 1, 1}, {HY, 0, 2}, {HY, 0, 3}, {HY, 1, 4}, {HY, 1, 5}};
    for (const Spec &sp : spec)
    {
      std::vector<double> sg = sigma_at (g, sp.comp, sp.axis);
      for (double sv : sg)
      {
        double r = sv * g.dt / (2 * kEps0);
        double v;
        switch (sp.kind)
        {
          case 0: v = (1 - r) / (1 + r); break;
          case 1: v = S / (1 + r); break;
          case 2: v = (1 - r) / (1 + r); break;
          case 3: v = 1 / (1 + r); break;
          case 4: v = 1 + r; break;
          default: v = 1 - r; break;
        }
        b->tab_host.push_back ((float) v);
      }
    }
    const int comps[3] = {EZ, HX, HY};
    for (int ci = 0; ci < 3; ++ci)
      for (int a = 0; a < 2; ++a)
      {
        std::vector<double> sg = sigma_at (g, comps[ci], a);
        int lo = 0, hi = g.n[a];
        if (base->use_pml)
        {
          while (lo < g.n[a] && sg[lo] != 0.0)
            ++lo;
          hi = lo;
          while (hi < g.n[a] && sg[hi] == 0.0)
            ++hi;
        }
        in.ilo[ci][a] = lo;
        in.ihi[ci][a] = hi;
      }
  }
  size_t cells = (size_t) b->cells;
  for (int s = 0; s < 2; ++s)
  {
    BALLOC (b->ez[s], cells * sizeof (float));
    BALLOC (b->hx[s], cells * sizeof (float));
    BALLOC (b->hy[s], cells * sizeof (float));
    if (base->use_pml)
    {
      BALLOC (b->aez[s], cells * sizeof (float));
      BALLOC (b->ahx[s], cells * sizeof (float));
      BALLOC (b->ahy[s], cells * sizeof (float));
    }
  }
  BALLOC (b->eps, cells * sizeof (float));
  fdtdb::fill_float_kernel<<<b->sm_count * 8, 256, 0, b->stream>>> (b->eps, cells, 1.f);
  BALLOC (b->d_tab, b->tab_host.size () * sizeof (float));
  BCK (cudaMemcpyAsync (b->d_tab, b->tab_host.data (), b->tab_host.size () * sizeof (float), cudaMemcpyHostToDevice,
                        b->stream));
  BALLOC (b->d_inst, b->inst.size () * sizeof (fdtdb::InstDev));
  BCK (cudaMemcpyAsync (b->d_inst, b->inst.data (), b->inst.size () * sizeof (fdtdb::InstDev), cudaMemcpyHostToDevice,
                        b->stream));
  BALLOC (b->d_counters, 4 * sizeof (unsigned));
  BALLOC (b->d_generation, sizeof (unsigned));
  BALLOC (b->d_err, sizeof (int));
  BCK (cudaStreamSynchronize (b->stream));
  return build_tiles (b, b->x_chunk);
}

int ensure_src (fdtd_batch *b, size_t n)
{
  BCK (cudaStreamSynchronize (b->stream));   // the previous launch may still read the pinned table
  if (n <= b->src_cap)
    return FDTD_OK;
  if (b->h_src)
    cudaFreeHost (b->h_src);
  b->h_src = nullptr;
  if (b->d_src)
  {
    auto it = std::find (b->allocs.begin (), b->allocs.end (), (void *) b->d_src);
    if (it != b->allocs.end ())
      b->allocs.erase (it);
    cudaFree (b->d_src);
    b->d_src = nullptr;
  }
  size_t cap = std::max<size_t> (n, 1024);
  BALLOC (b->d_src, cap * sizeof (double));
  BCK (fdtdb::pinned_malloc ((void **) &b->h_src, cap * sizeof (double)));
  b->src_cap = cap;
  drop_graph (b);
  return FDTD_OK;
}

// One call = one persistent launch; captured into a CUDA graph (source
// upload, counter reset, kernel) unless capture is refused, in which case
// the same three operations are issued directly.
int step_batch (fdtd_batch *b, uint32_t t_start, uint32_t n, bool allow_graph)
{
  int r = ensure_src (b, n);
  if (r != FDTD_OK)
    return r;
  for (uint32_t s = 0; s < n; ++s)
    b->h_src[s] = fdtdb::point_source (b->geo[0], t_start + s, false);
  BCK (cudaEventRecord (b->ev0, b->stream));
  bool launched = false;
  if (allow_graph && b->use_graph)
  {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture (b->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess)
    {
      int er = enqueue (b, t_start, n);
      cudaError_t ee = cudaStreamEndCapture (b->stream, &g);
      if (er == FDTD_OK && ee == cudaSuccess && g)
      {
        cudaError_t ie;
        if (b->graph)
        {
          cudaGraphExecUpdateResultInfo info;
          ie = cudaGraphExecUpdate (b->graph, g, &info);
          if (ie != cudaSuccess)
          {
            cudaGetLastError ();
            drop_graph (b);
          }
        }
        if (!b->graph)
          ie = cudaGraphInstantiate (&b->graph, g, 0);
        if (ie == cudaSuccess && cudaGraphLaunch (b->graph, b->stream) == cudaSuccess)
        {
          launched = true;
          b->graph_ok = true;
        }
      }
      if (g)
        cudaGraphDestroy (g);
      if (!launched)
      {
        cudaGetLastError ();
        drop_graph (b);
        b->use_graph = false;
        b->graph_ok = false;
      }
    }
    else
    {
      cudaGetLastError ();
      b->use_graph = false;
    }
  }
  if (!launched)
  {
    r = enqueue (b, t_start, n);
    if (r != FDTD_OK)
      return r;
  }
  BCK (cudaEventRecord (b->ev1, b->stream));
  for (uint32_t s = 0; s < n; ++s)
    if (t_start + s > 0)
      b->cur ^= 1;
  return FDTD_OK;
}

}  // namespace

extern "C" {

int fdtd_batch_create (const fdtd_config *base, int count, const int *sizes, int device, fdtd_batch **out)
{
  if (!base || !out)
    return FDTD_ERR_ARG;
  *out = nullptr;
  fdtd_batch *b = new (std::nothrow) fdtd_batch ();
  if (!b)
    return FDTD_ERR_NOMEM;
  int r = create_batch (b, base, count, sizes, device);
  if (r != FDTD_OK)
  {
    fdtd_batch_destroy (b);
    return r;
  }
  *out = b;
  return FDTD_OK;
}

int fdtd_batch_upload_eps (fdtd_batch *b, int instance, const double *host)
{
  if (!b || !host || instance < 0 || instance >= (int) b->inst.size ())
    return FDTD_ERR_ARG;
  BCK (cudaSetDevice (b->device));
  const fdtdb::InstDev &in = b->inst[instance];
  size_t n = (size_t) in.nx * in.ny;
  std::vector<float> f (n);
  for (size_t i = 0; i < n; ++i)
    f[i] = (float) host[i];
  BCK (cudaMemcpyAsync (b->eps + in.off, f.data (), n * sizeof (float), cudaMemcpyHostToDevice, b->stream));
  BCK (cudaStreamSynchronize (b->stream));
  return FDTD_OK;
}

int fdtd_batch_step (fdtd_batch *b, uint32_t t_start, uint32_t n_steps)
{
  if (!b)
    return FDTD_ERR_ARG;
  if (n_steps == 0)
    return FDTD_OK;
  BCK (cudaSetDevice (b->device));
  return step_batch (b, t_start, n_steps, true);
}

int fdtd_batch_sync (fdtd_batch *b, int64_t timeout_ns)
{
  if (!b)
    return FDTD_ERR_ARG;
  BCK (cudaSetDevice (b->device));
  if (timeout_ns < 0)
  {
    BCK (cudaStreamSynchronize (b->stream));
  }
  else
  {
    auto t0 = std::chrono::steady_clock::now ();
    for (;;)
    {
      cudaError_t e = cudaStreamQuery (b->stream);
      if (e == cudaSuccess)
        break;
      if (e != cudaErrorNotReady)
        return bfail (b, FDTD_ERR_CUDA, cudaGetErrorString (e));
      if (std::chrono::duration_cast<std::chrono::nanoseconds> (std::chrono::steady_clock::now () - t0).count ()
          >= timeout_ns)
        return bfail (b, FDTD_ERR_TIMEOUT, "sync timed out");
    }
  }
  float ms = 0.f;
  if (cudaEventElapsedTime (&ms, b->ev0, b->ev1) == cudaSuccess)
    b->last_ms = ms;
  int flag = 0;
  BCK (cudaMemcpy (&flag, b->d_err, sizeof (int), cudaMemcpyDeviceToHost));
  if (flag)
    return bfail (b, FDTD_ERR_DEVICE, "a grid barrier timed out");
  return FDTD_OK;
}

int fdtd_batch_download (fdtd_batch *b, int instance, int component, double *host)
{
  if (!b || !host || instance < 0 || instance >= (int) b->inst.size ()
      || (component != FDTD_EZ && component != FDTD_HX && component != FDTD_HY))
    return FDTD_ERR_ARG;
  int r = fdtd_batch_sync (b, -1);
  if (r != FDTD_OK)
    return r;
  const fdtdb::InstDev &in = b->inst[instance];
  size_t n = (size_t) in.nx * in.ny;
  const float *src = component == FDTD_EZ ? b->ez[b->cur] : (component == FDTD_HX ? b->hx[b->cur] : b->hy[b->cur]);
  std::vector<float> f (n);
  BCK (cudaMemcpy (f.data (), src + in.off, n * sizeof (float), cudaMemcpyDeviceToHost));
  double scale = component == FDTD_EZ ? 1.0 : 1.0 / fdtdb::kEta0B;
  for (size_t i = 0; i < n; ++i)
    host[i] = (double) f[i] * scale;
  return FDTD_OK;
}

int fdtd_batch_tune (fdtd_batch *b, int steps, int *choice)
{
  if (!b || steps < 1)
    return FDTD_ERR_ARG;
  BCK (cudaSetDevice (b->device));
  static const int chunks[] = {16, 32, 64, 128};
  static const int warps[] = {4, 8, 16};
  static const int per_sm[] = {1, 2, 4};
  double best = 1e30;
  int bc = b->x_chunk, bw = b->warps_per_cta, bs = b->ctas_per_sm;
  for (int c : chunks)
  {
    int r = build_tiles (b, c);
    if (r != FDTD_OK)
      return r;
    for (int w : warps)
      for (int s : per_sm)
      {
        if (s > max_ctas (b, w))
          continue;
        b->warps_per_cta = w;
        b->ctas_per_sm = s;
        r = step_batch (b, 1, (uint32_t) steps, false);
        if (r != FDTD_OK)
          return r;
        BCK (cudaStreamSynchronize (b->stream));
        float ms = 0.f;
        BCK (cudaEventElapsedTime (&ms, b->ev0, b->ev1));
        int flag = 0;
        BCK (cudaMemcpy (&flag, b->d_err, sizeof (int), cudaMemcpyDeviceToHost));
        if (flag)
          return bfail (b, FDTD_ERR_DEVICE, "a grid barrier timed out while tuning");
        if (ms < best)
        {
          best = ms;
          bc = c;
          bw = w;
          bs = s;
        }
      }
  }
  // back to the state before tuning: zero fields and auxiliaries, t = 0
  size_t bytes = (size_t) b->cells * sizeof (float);
  for (int s = 0; s < 2; ++s)
  {
    float *arr[6] = {b->ez[s], b->hx[s], b->hy[s], b->aez[s], b->ahx[s], b->ahy[s]};
    for (float *a : arr)
      if (a)
        BCK (cudaMemsetAsync (a, 0, bytes, b->stream));
  }
  b->cur = 0;
  b->warps_per_cta = bw;
  b->ctas_per_sm = bs;
  int r = build_tiles (b, bc);
  if (r != FDTD_OK)
    return r;
  drop_graph (b);
  b->use_graph = true;
  if (choice)
  {
    choice[0] = bc;
    choice[1] = bw;
    choice[2] = bs;
  }
  return FDTD_OK;
}

int fdtd_batch_info (const fdtd_batch *b, int64_t *cells, int *graph_used, double *last_ms)
{
  if (!b)
    return FDTD_ERR_ARG;
  if (cells)
    *cells = b->cells;
  if (graph_used)
    *graph_used = b->graph_ok ? 1 : 0;
  if (last_ms)
    *last_ms = b->last_ms;
  return FDTD_OK;
}

void fdtd_batch_destroy (fdtd_batch *b)
{
  if (!b)
    return;
  cudaSetDevice (b->device);
  if (b->stream)
    cudaStreamSynchronize (b->stream);
  drop_graph (b);
  for (void *p : b->allocs)
    cudaFree (p);
  if (b->h_src)
    cudaFreeHost (b->h_src);
  if (b->ev0)
    cudaEventDestroy (b->ev0);
  if (b->ev1)
    cudaEventDestroy (b->ev1);
  if (b->stream)
    cudaStreamDestroy (b->stream);
  delete b;
}

int fdtd_batch_set_wait_limit (fdtd_batch *b, int64_t limit_ns)
{
  if (!b)
    return FDTD_ERR_ARG;
  b->wait_limit_ns = limit_ns > 0 ? limit_ns : 0;
  return FDTD_OK;
}

const char *fdtd_batch_last_error (const fdtd_batch *b)
{
  return b ? b->err.c_str () : "";
}

}  // extern "C"
