// adjoint.cu - checkpointed reverse-mode differentiation of the 2-D TMz
// step (see adjoint.h).
//
// Forward step k (k = 0 .. steps - 1), as the library's FP32 TMz step:
//   k > 0: Ez cells: curl of H; interior Ez += S * im * curl, PML cells
//          X_new = ca1 X + sq1 curl, Ez = p5 Ez + (g4p X_new - g4m X) q5 im
//          (im = 1 / averaged eps); Ez point source overwrites its cell;
//   k > 0: Hx, Hy the same with im = 1; H point source overwrites its cell;
//   J += sum over the probe of Ez_k^2.
// Reverse sweep, for k = steps - 1 .. 0 with the adjoint state (aE, aH, aX)
// of the state after step k:
//   aE += 2 Ez_k on the probe;
//   k > 0: transpose of the H half-step (aH, aX of H; a curl adjoint per H
//          cell gathered into aE), then of the E half-step (gradient of im
//          += aE * dEz/dim, a curl adjoint per Ez cell gathered into aH).
// Point-source cells carry no adjoint into the step before (their value is
// overwritten).  dJ/d eps = sum over the Ez cells whose average includes
// the cell of dJ/d im * (-im^2 / n_points).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "adjoint.h"

namespace fdtdb {

namespace {

constexpr int kEz = 0, kHx = 1, kHy = 2;   // local component slots
constexpr double kEta0Adj = 376.730313461770655;

template <typename R>
struct AdjDev
{
  int nx, ny;
  R S;
  int ilo[3][2], ihi[3][2];    // sigma == 0 range per component and axis
  int tax[3][3];               // axis of the (ca1, sq1), (p5, q5), (g4p, g4m) pairs
  const R *tab[3][6];          // tables indexed by the coordinate along the pair's axis
  int o1[3], o2[3];            // curl sources (local slots, -1 = absent)
  int d11[3][2], d12[3][2], d21[3][2], d22[3][2];
  const R *im;                 // 1 / averaged eps of Ez
  int ps[2];
  int ps_on[3];                // point source on Ez / Hx / Hy
  const R *src;                // [2k] E value, [2k + 1] H value of step k
  int pr_lo[2], pr_hi[2];
};

template <typename R>
__device__ __forceinline__ bool interior (const AdjDev<R> &p, int c, int x, int y)
{
  return x >= p.ilo[c][0] && x < p.ihi[c][0] && y >= p.ilo[c][1] && y < p.ihi[c][1];
}

template <typename R>
__device__ __forceinline__ R tabv (const AdjDev<R> &p, int c, int j, int x, int y)
{
  const int ax = p.tax[c][j / 2];
  return p.tab[c][j][ax == 0 ? x : (ax == 1 ? y : 0)];   // z has one (sigma = 0) entry in 2-D
}

template <typename R>
__device__ __forceinline__ R curl_of (const AdjDev<R> &p, int c, const R *const F[3], int x, int y)
{
  R v0 = 0, v1 = 0, v2 = 0, v3 = 0;
  const int ny = p.ny;
  if (p.o1[c] >= 0)
  {
    const R *f = F[p.o1[c]];
    v0 = f[(x + p.d11[c][0]) * ny + y + p.d11[c][1]];
    v1 = f[(x + p.d12[c][0]) * ny + y + p.d12[c][1]];
  }
  if (p.o2[c] >= 0)
  {
    const R *f = F[p.o2[c]];
    v2 = f[(x + p.d21[c][0]) * ny + y + p.d21[c][1]];
    v3 = f[(x + p.d22[c][0]) * ny + y + p.d22[c][1]];
  }
  return (v1 - v0) - (v3 - v2);
}

// one component update at (x, y); returns dF/d(im) for the gradient
template <typename R>
__device__ __forceinline__ R update_cell (const AdjDev<R> &p, int c, R *F, R *X, R cu, R im, int x, int y)
{
  const int id = x * p.ny + y;
  R f = F[id];
  R dfdm;
  if (interior (p, c, x, y))
  {
    f += p.S * im * cu;
    dfdm = p.S * cu;
  }
  else
  {
    const R ca1 = tabv (p, c, 0, x, y), sq1 = tabv (p, c, 1, x, y);
    const R p5 = tabv (p, c, 2, x, y), q5 = tabv (p, c, 3, x, y);
    const R g4p = tabv (p, c, 4, x, y), g4m = tabv (p, c, 5, x, y);
    const R xo = X[id];
    const R xn = ca1 * xo + sq1 * cu;
    X[id] = xn;
    dfdm = (g4p * xn - g4m * xo) * q5;
    f = p5 * f + (g4p * xn - g4m * xo) * q5 * im;
  }
  F[id] = f;
  return dfdm;
}

// ---- forward

template <typename R>
__global__ void fwd_e_kernel (AdjDev<R> p, R *Ez, R *Hx, R *Hy, R *Xz, R *dedm, int k, int do_update)
{
  const int n = (p.nx - 2) * (p.ny - 2);
  const R *F[3] = {Ez, Hx, Hy};
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
  {
    const int x = 1 + t / (p.ny - 2), y = 1 + t % (p.ny - 2);
    const int id = x * p.ny + y;
    R d = 0;
    if (do_update)
      d = update_cell (p, kEz, Ez, Xz, curl_of (p, kEz, F, x, y), p.im[id], x, y);
    if (p.ps_on[kEz] && x == p.ps[0] && y == p.ps[1])
      Ez[id] = p.src[2 * k];
    if (dedm)
      dedm[id] = d;
  }
}

__device__ __forceinline__ void kahan_add (double &s, double &c, double v);

// J += sum of Ez^2 over the probe, by one block; probe values optionally kept
template <typename R>
__device__ void probe_sum (const AdjDev<R> &p, const R *Ez, double *acc, double *keep)
{
  __shared__ double part[256];
  const int w = p.pr_hi[1] - p.pr_lo[1];
  const int n = (p.pr_hi[0] - p.pr_lo[0]) * w;
  double s = 0.0;
  for (int t = threadIdx.x; t < n; t += blockDim.x)
  {
    const int x = p.pr_lo[0] + t / w, y = p.pr_lo[1] + t % w;
    const double v = (double) Ez[x * p.ny + y];
    if (keep)
      keep[t] = v;
    s += v * v;
  }
  part[threadIdx.x] = s;
  __syncthreads ();
  for (int h = 128; h > 0; h >>= 1)
  {
    if (threadIdx.x < h)
      part[threadIdx.x] += part[threadIdx.x + h];
    __syncthreads ();
  }
  if (threadIdx.x == 0 && acc)
    kahan_add (acc[0], acc[1], part[0]);
}

// H half-step (and H point source); block 0 first adds the probe term of
// Ez_k, which the E kernel before it completed
template <typename R>
__global__ void __launch_bounds__ (256) fwd_h_kernel (AdjDev<R> p, const R *Ez, R *Hx, R *Hy, R *Xx, R *Xy, int k,
                                                      int do_update, double *acc, double *keep)
{
  if (blockIdx.x == 0)
    probe_sum (p, Ez, acc, keep);
  const int n = (p.nx - 2) * (p.ny - 2);
  const R *F[3] = {Ez, Hx, Hy};
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
  {
    const int x = 1 + t / (p.ny - 2), y = 1 + t % (p.ny - 2);
    const int id = x * p.ny + y;
    // both curls read Ez only, which this kernel does not write
    if (do_update)
    {
      const R cx = curl_of (p, kHx, F, x, y), cy = curl_of (p, kHy, F, x, y);
      update_cell (p, kHx, Hx, Xx, cx, R (1), x, y);
      update_cell (p, kHy, Hy, Xy, cy, R (1), x, y);
    }
    if (x == p.ps[0] && y == p.ps[1])
    {
      if (p.ps_on[kHx])
        Hx[id] = p.src[2 * k + 1];
      if (p.ps_on[kHy])
        Hy[id] = p.src[2 * k + 1];
    }
  }
}

__device__ __forceinline__ void kahan_add (double &s, double &c, double v)
{
  const double t = s + v;
  if (fabs (s) >= fabs (v))
    c += (s - t) + v;
  else
    c += (v - t) + s;
  s = t;
}

// ---- reverse
//
// Each reverse half-step is one kernel over all cells with double-buffered
// adjoint fields: a thread updates its own cell from the old buffers and
// gathers the curl adjoints of its neighbours by recomputing them (they are
// pointwise in the old buffers), so no thread reads what another writes.

template <typename R>
struct CurlAdj
{
  R acu, a_new, x_new;
};

// transpose of one H half-step at an updated H cell (point source included)
template <typename R>
__device__ __forceinline__ CurlAdj<R> h_adj (const AdjDev<R> &p, int c, R a, R ax, int x, int y)
{
  if (x == p.ps[0] && y == p.ps[1] && p.ps_on[c])
    a = 0;
  if (interior (p, c, x, y))
    return {p.S * a, a, ax};
  const R ca1 = tabv (p, c, 0, x, y), sq1 = tabv (p, c, 1, x, y);
  const R p5 = tabv (p, c, 2, x, y), q5 = tabv (p, c, 3, x, y);
  const R g4p = tabv (p, c, 4, x, y), g4m = tabv (p, c, 5, x, y);
  const R t1 = ax + g4p * q5 * a;
  return {sq1 * t1, p5 * a, ca1 * t1 - g4m * q5 * a};
}

// transpose of one E half-step at an updated Ez cell (point source included)
template <typename R>
__device__ __forceinline__ CurlAdj<R> e_adj (const AdjDev<R> &p, R a, R ax, R im, int x, int y)
{
  if (x == p.ps[0] && y == p.ps[1] && p.ps_on[kEz])
    a = 0;
  if (interior (p, kEz, x, y))
    return {p.S * im * a, a, ax};
  const R ca1 = tabv (p, kEz, 0, x, y), sq1 = tabv (p, kEz, 1, x, y);
  const R p5 = tabv (p, kEz, 2, x, y), q5 = tabv (p, kEz, 3, x, y);
  const R g4p = tabv (p, kEz, 4, x, y), g4m = tabv (p, kEz, 5, x, y);
  const R t1 = ax + g4p * q5 * im * a;
  return {sq1 * t1, p5 * a, ca1 * t1 - g4m * q5 * im * a};
}

template <typename R>
__device__ __forceinline__ bool updated (const AdjDev<R> &p, int x, int y)
{
  return x >= 1 && x <= p.nx - 2 && y >= 1 && y <= p.ny - 2;
}

// transpose of the H half-step: new aH, aX of H; aE += curl-of-E adjoint
// gathers + 2 Ez_k on the probe
template <typename R>
__global__ void __launch_bounds__ (256) adj_h_kernel (AdjDev<R> p, const R *aHx0, const R *aHy0, const R *aXx0,
                                                      const R *aXy0, R *aHx1, R *aHy1, R *aXx1, R *aXy1, R *aE,
                                                      const double *probe)
{
  const int n = p.nx * p.ny;
  const int pw = p.pr_hi[1] - p.pr_lo[1];
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
  {
    const int x = t / p.ny, y = t % p.ny;
    R g = 0;
#pragma unroll
    for (int q = 0; q < 2; ++q)
    {
      const int c = q ? kHy : kHx;
      const R *aH0 = q ? aHy0 : aHx0;
      const R *aX0 = q ? aXy0 : aXx0;
      if (updated (p, x, y))
      {
        const CurlAdj<R> r = h_adj (p, c, aH0[t], aX0[t], x, y);
        (q ? aHy1 : aHx1)[t] = r.a_new;
        (q ? aXy1 : aXx1)[t] = r.x_new;
      }
      // Ez (x, y) is read by the H cell h = (x, y) - d of each Ez term
      auto take = [&] (const int d[2], R sgn) {
        const int hx = x - d[0], hy = y - d[1];
        if (updated (p, hx, hy))
        {
          const int h = hx * p.ny + hy;
          g += sgn * h_adj (p, c, aH0[h], aX0[h], hx, hy).acu;
        }
      };
      if (p.o1[c] == kEz)
      {
        take (p.d12[c], R (1));
        take (p.d11[c], R (-1));
      }
      if (p.o2[c] == kEz)
      {
        take (p.d22[c], R (-1));
        take (p.d21[c], R (1));
      }
    }
    R v = aE[t] + g;
    if (x >= p.pr_lo[0] && x < p.pr_hi[0] && y >= p.pr_lo[1] && y < p.pr_hi[1])
      v += (R) (2.0 * probe[(x - p.pr_lo[0]) * pw + (y - p.pr_lo[1])]);
    aE[t] = v;
  }
}

// transpose of the E half-step: gradient of im, new aE, aXz; aH += curl-of-H
// adjoint gathers
template <typename R>
__global__ void __launch_bounds__ (256) adj_e_kernel (AdjDev<R> p, const R *aE0, const R *aXz0, R *aE1, R *aXz1,
                                                      R *aHx, R *aHy, const R *dedm, double *gim)
{
  const int n = p.nx * p.ny;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
  {
    const int x = t / p.ny, y = t % p.ny;
    if (updated (p, x, y))
    {
      R a = aE0[t];
      if (x == p.ps[0] && y == p.ps[1] && p.ps_on[kEz])
        a = 0;
      gim[t] += (double) a * (double) dedm[t];
      const CurlAdj<R> r = e_adj (p, aE0[t], aXz0[t], p.im[t], x, y);
      aE1[t] = r.a_new;
      aXz1[t] = r.x_new;
    }
    auto take = [&] (const int d[2], R sgn) -> R {
      const int ex = x - d[0], ey = y - d[1];
      if (!updated (p, ex, ey))
        return R (0);
      const int e = ex * p.ny + ey;
      return sgn * e_adj (p, aE0[e], aXz0[e], p.im[e], ex, ey).acu;
    };
    R g[2] = {0, 0};
#pragma unroll
    for (int q = 0; q < 2; ++q)
    {
      const int slot = q ? kHy : kHx;
      if (p.o1[kEz] == slot)
        g[q] += take (p.d12[kEz], R (1)) + take (p.d11[kEz], R (-1));
      if (p.o2[kEz] == slot)
        g[q] += take (p.d22[kEz], R (-1)) + take (p.d21[kEz], R (1));
    }
    aHx[t] += g[0];
    aHy[t] += g[1];
  }
}

// dJ/d eps from dJ/d im (gather over the Ez cells that average the cell)
template <typename R>
__global__ void grad_eps_kernel (AdjDev<R> p, const double *gim, const double *imd, int nmat, int m0x, int m0y,
                                 int m1x, int m1y, int m2x, int m2y, int m3x, int m3y, double *out)
{
  const int n = p.nx * p.ny;
  const int mx[4] = {m0x, m1x, m2x, m3x}, my[4] = {m0y, m1y, m2y, m3y};
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
  {
    const int x = t / p.ny, y = t % p.ny;
    double g = 0.0;
    for (int j = 0; j < nmat; ++j)
    {
      const int cx = x - mx[j], cy = y - my[j];
      if (cx >= 1 && cx <= p.nx - 2 && cy >= 1 && cy <= p.ny - 2)
      {
        const int c = cx * p.ny + cy;
        g -= gim[c] * imd[c] * imd[c] / (double) nmat;
      }
    }
    out[t] = g;
  }
}

}  // namespace

// ------------------------------------------------------------------ host side

namespace {

// inverse averaged eps of Ez (as the per-cell kernel computes it) in R and double
template <typename R, typename E>
__global__ void invm_kernel (const E *eps, int nx, int ny, int nmat, int m1x, int m1y, int m2x, int m2y, int m3x,
                             int m3y, R *im, double *imd)
{
  const int n = nx * ny;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
  {
    const int x = t / ny, y = t % ny;
    auto at = [&] (int dx, int dy) -> E {
      const int xx = min (x + dx, nx - 1), yy = min (y + dy, ny - 1);
      return eps ? eps[xx * ny + yy] : E (1);
    };
    R m;
    double md;
    if (nmat == 2)
    {
      m = R (0.5) * ((R) at (0, 0) + (R) at (m1x, m1y));
      md = 0.5 * ((double) at (0, 0) + (double) at (m1x, m1y));
    }
    else
    {
      m = R (0.25) * ((R) at (0, 0) + (R) at (m1x, m1y) + (R) at (m2x, m2y) + (R) at (m3x, m3y));
      md = 0.25 * ((double) at (0, 0) + (double) at (m1x, m1y) + (double) at (m2x, m2y) + (double) at (m3x, m3y));
    }
    im[t] = R (1) / m;
    imd[t] = 1.0 / md;
  }
}

struct DevMem
{
  std::vector<void *> ptr;
  ~DevMem ()
  {
    for (void *q : ptr)
      cudaFree (q);
  }
  template <typename Q>
  Q *get (size_t count)
  {
    void *q = nullptr;
    if (cudaMalloc (&q, std::max<size_t> (count, 1) * sizeof (Q)) != cudaSuccess)
      return nullptr;
    ptr.push_back (q);
    return (Q *) q;
  }
};

int local_slot (int k)
{
  return k == EZ ? kEz : (k == HX ? kHx : (k == HY ? kHy : -1));
}

template <typename R>
std::string run_t (const Geometry &g, const void *eps_dev, bool eps_is_double, const AdjointRun &run,
                   double *objective, double *grad_host, int sm_count, cudaStream_t s)
{
  if (!g.tmz)
    return "the adjoint covers 2-D TMz grids";
  if (g.cfg.use_tfsf)
    return "the adjoint covers point-source runs (no TF/SF)";
  if (g.cfg.use_metamaterials)
    return "the adjoint does not cover metamaterials";
  const int nx = g.n[0], ny = g.n[1];
  const size_t N = (size_t) nx * ny;
  if (run.steps < 1 || run.every < 1)
    return "steps and checkpoint interval must be positive";
  for (int a = 0; a < 2; ++a)
    if (run.probe_lo[a] < 1 || run.probe_hi[a] > g.n[a] - 1 || run.probe_lo[a] >= run.probe_hi[a])
      return "probe box outside the updated cells";
  const int npr = (run.probe_hi[0] - run.probe_lo[0]) * (run.probe_hi[1] - run.probe_lo[1]);

  DevMem mem;
  AdjDev<R> p{};
  p.nx = nx;
  p.ny = ny;
  const double S = 299792458.0 * g.dt / g.dx;
  p.S = (R) S;
  const int kmap[3] = {EZ, HX, HY};
  for (int c = 0; c < 3; ++c)
  {
    const int k = kmap[c];
    const CompLayout &L = g.comp[k];
    p.o1[c] = g.comp[L.opp1].exists ? local_slot (L.opp1) : -1;
    p.o2[c] = g.comp[L.opp2].exists ? local_slot (L.opp2) : -1;
    for (int a = 0; a < 2; ++a)
    {
      p.d11[c][a] = L.d11[a];
      p.d12[c][a] = L.d12[a];
      p.d21[c][a] = L.d21[a];
      p.d22[c][a] = L.d22[a];
    }
    const int axes[3] = {L.sig_cacb, L.sig5, L.sig4};
    for (int q = 0; q < 3; ++q)
      p.tax[c][q] = axes[q];
    for (int j = 0; j < 6; ++j)
    {
      std::vector<double> sg = sigma_at (g, k, axes[j / 2]);
      std::vector<R> v (sg.size ());
      for (size_t i = 0; i < sg.size (); ++i)
      {
        // the coefficient tables of the FP32 step (sigma = 0 gives 1, S, 1, 1, 1, 1)
        const double r = sg[i] * g.dt / (2 * kEps0);
        double w;
        switch (j)
        {
          case 0: w = (1 - r) / (1 + r); break;
          case 1: w = S / (1 + r); break;
          case 2: w = (1 - r) / (1 + r); break;
          case 3: w = 1 / (1 + r); break;
          case 4: w = 1 + r; break;
          default: w = 1 - r; break;
        }
        v[i] = (R) w;
      }
      R *d = mem.get<R> (v.size ());
      if (!d)
        return "cudaMalloc failed";
      if (cudaMemcpyAsync (d, v.data (), v.size () * sizeof (R), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return "cudaMemcpyAsync failed";
      p.tab[c][j] = d;
    }
    for (int a = 0; a < 2; ++a)
    {
      int lo = 0, hi = g.n[a];
      if (g.cfg.use_pml)
      {
        std::vector<double> sg = sigma_at (g, k, a);
        lo = 0;
        while (lo < g.n[a] && sg[lo] != 0.0)
          ++lo;
        hi = lo;
        while (hi < g.n[a] && sg[hi] == 0.0)
          ++hi;
      }
      p.ilo[c][a] = lo;
      p.ihi[c][a] = hi;
    }
  }
  // point source: E value as the E half-step writes it, H value times eta0 in
  // the stored precision
  p.ps[0] = g.cfg.point_source_mask ? g.cfg.point_source[0] : -1;
  p.ps[1] = g.cfg.point_source_mask ? g.cfg.point_source[1] : -1;
  for (int c = 0; c < 3; ++c)
    p.ps_on[c] = (g.cfg.point_source_mask >> kmap[c]) & 1;
  {
    std::vector<R> src (2 * (size_t) run.steps);
    for (uint32_t k = 0; k < run.steps; ++k)
    {
      src[2 * k] = (R) point_source (g, k, false);
      src[2 * k + 1] = (R) point_source (g, k, true) * (R) kEta0Adj;
    }
    R *d = mem.get<R> (src.size ());
    if (!d || cudaMemcpyAsync (d, src.data (), src.size () * sizeof (R), cudaMemcpyHostToDevice, s) != cudaSuccess)
      return "source table upload failed";
    p.src = d;
  }
  for (int a = 0; a < 2; ++a)
  {
    p.pr_lo[a] = run.probe_lo[a];
    p.pr_hi[a] = run.probe_hi[a];
  }

  // state, inverse eps, objective accumulator
  R *F[6];
  for (int q = 0; q < 6; ++q)
  {
    F[q] = mem.get<R> (N);
    if (!F[q] || cudaMemsetAsync (F[q], 0, N * sizeof (R), s) != cudaSuccess)
      return "state allocation failed";
  }
  R *Ez = F[0], *Hx = F[1], *Hy = F[2], *Xz = F[3], *Xx = F[4], *Xy = F[5];
  R *im = mem.get<R> (N);
  double *imd = mem.get<double> (N);
  double *acc = mem.get<double> (2);
  if (!im || !imd || !acc || cudaMemsetAsync (acc, 0, 2 * sizeof (double), s) != cudaSuccess)
    return "allocation failed";
  const CompLayout &LE = g.comp[EZ];
  const int blocks = (int) std::min<size_t> ((N + 255) / 256, (size_t) sm_count * 8);
  if (eps_is_double)
    invm_kernel<R, double><<<blocks, 256, 0, s>>> ((const double *) eps_dev, nx, ny, LE.nmat, LE.m[1][0], LE.m[1][1],
                                                   LE.m[2][0], LE.m[2][1], LE.m[3][0], LE.m[3][1], im, imd);
  else
    invm_kernel<R, float><<<blocks, 256, 0, s>>> ((const float *) eps_dev, nx, ny, LE.nmat, LE.m[1][0], LE.m[1][1],
                                                  LE.m[2][0], LE.m[2][1], LE.m[3][0], LE.m[3][1], im, imd);
  p.im = im;

  const uint32_t K = run.every;
  const uint32_t nck = (run.steps + K - 1) / K;
  R *ck = nullptr;
  if (grad_host)
  {
    ck = mem.get<R> ((size_t) nck * 6 * N);
    if (!ck)
      return "checkpoint allocation failed";
  }
  auto save = [&] (uint32_t j) {
    for (int q = 0; q < 6; ++q)
      cudaMemcpyAsync (ck + ((size_t) j * 6 + q) * N, F[q], N * sizeof (R), cudaMemcpyDeviceToDevice, s);
  };
  auto restore = [&] (uint32_t j) {
    for (int q = 0; q < 6; ++q)
      cudaMemcpyAsync (F[q], ck + ((size_t) j * 6 + q) * N, N * sizeof (R), cudaMemcpyDeviceToDevice, s);
  };
  auto step = [&] (uint32_t k, R *dedm, double *keep, double *a) {
    fwd_e_kernel<R><<<blocks, 256, 0, s>>> (p, Ez, Hx, Hy, Xz, dedm, (int) k, k > 0);
    fwd_h_kernel<R><<<blocks, 256, 0, s>>> (p, Ez, Hx, Hy, Xx, Xy, (int) k, k > 0, a, keep);
  };

  for (uint32_t k = 0; k < run.steps; ++k)
  {
    if (grad_host && k % K == 0)
      save (k / K);
    step (k, nullptr, nullptr, acc);
  }
  double hacc[2];
  if (cudaMemcpyAsync (hacc, acc, sizeof (hacc), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize (s) != cudaSuccess)
    return std::string ("forward run failed: ") + cudaGetErrorString (cudaGetLastError ());
  if (objective)
    *objective = hacc[0] + hacc[1];
  if (!grad_host)
    return "";

  // reverse sweep, one checkpoint segment at a time; adjoint fields double
  // buffered (index 0 / 1 of each pair is swapped every half-step)
  R *A[12];
  for (int q = 0; q < 12; ++q)
  {
    A[q] = mem.get<R> (N);
    if (!A[q] || cudaMemsetAsync (A[q], 0, N * sizeof (R), s) != cudaSuccess)
      return "adjoint allocation failed";
  }
  R *aE[2] = {A[0], A[1]}, *aXz[2] = {A[2], A[3]}, *aHx[2] = {A[4], A[5]}, *aHy[2] = {A[6], A[7]},
    *aXx[2] = {A[8], A[9]}, *aXy[2] = {A[10], A[11]};
  int ie = 0, ih = 0;
  double *gim = mem.get<double> (N);
  double *gout = mem.get<double> (N);
  R *dedm = mem.get<R> ((size_t) K * N);
  double *probe = mem.get<double> ((size_t) K * npr);
  if (!gim || !gout || !dedm || !probe || cudaMemsetAsync (gim, 0, N * sizeof (double), s) != cudaSuccess)
    return "adjoint allocation failed";
  for (int64_t j = (int64_t) nck - 1; j >= 0; --j)
  {
    restore ((uint32_t) j);
    const uint32_t k0 = (uint32_t) j * K, k1 = std::min (k0 + K, run.steps);
    for (uint32_t k = k0; k < k1; ++k)
      step (k, dedm + (size_t) (k - k0) * N, probe + (size_t) (k - k0) * npr, nullptr);
    for (int64_t k = (int64_t) k1 - 1; k >= (int64_t) k0 && k > 0; --k)
    {
      const size_t off = (size_t) (k - k0);
      adj_h_kernel<R><<<blocks, 256, 0, s>>> (p, aHx[ih], aHy[ih], aXx[ih], aXy[ih], aHx[1 - ih], aHy[1 - ih],
                                              aXx[1 - ih], aXy[1 - ih], aE[ie], probe + off * npr);
      ih ^= 1;
      adj_e_kernel<R><<<blocks, 256, 0, s>>> (p, aE[ie], aXz[ie], aE[1 - ie], aXz[1 - ie], aHx[ih], aHy[ih],
                                              dedm + off * N, gim);
      ie ^= 1;
    }
  }
  grad_eps_kernel<R><<<blocks, 256, 0, s>>> (p, gim, imd, LE.nmat, LE.m[0][0], LE.m[0][1], LE.m[1][0], LE.m[1][1],
                                             LE.m[2][0], LE.m[2][1], LE.m[3][0], LE.m[3][1], gout);
  if (cudaMemcpyAsync (grad_host, gout, N * sizeof (double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize (s) != cudaSuccess)
    return std::string ("reverse run failed: ") + cudaGetErrorString (cudaGetLastError ());
  return "";
}

}  // namespace

std::string adjoint_run (const Geometry &g, const void *eps_dev, bool eps_is_double, const AdjointRun &run,
                         double *objective, double *grad_host, int sm_count, cudaStream_t s)
{
  return run.fp64 ? run_t<double> (g, eps_dev, eps_is_double, run, objective, grad_host, sm_count, s)
                  : run_t<float> (g, eps_dev, eps_is_double, run, objective, grad_host, sm_count, s);
}

}  // namespace fdtdb
