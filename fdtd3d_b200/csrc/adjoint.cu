// adjoint.cu - checkpointed reverse-mode differentiation of the 2-D TMz
// step (see adjoint.h).
//
// Forward step k (k = 0 .. steps - 1), as the library's FP32 TMz step:
//   k > 0: Ez cells: curl of H; interior Ez += S * im * curl, PML cells
//          X_new = ca1 X + sq1 curl, Ez = p5 Ez + (g4p X_new - g4m X) q5 im
//          (im = 1 / averaged eps); Ez point source overwrites its cell;
//   k > 0: Hx, Hy the same with im = 1; H point source overwrites its cell;
//   J += sum over the probe of Ez_k^2.
// Reverse step k (k = steps - 1 .. 1), two phases:
//   H phase: aH += (curl of H)^T acz (acz stored by the E phase of step
//            k + 1), then the transpose of the H half-step of step k at each
//            H cell, storing its curl adjoints acx, acy;
//   E phase: aE += (curl of E)^T (acx, acy) + 2 Ez_k on the probe, the
//            gradient of im += aE * dEz/dim, then the transpose of the E
//            half-step of step k at each Ez cell, storing its curl adjoint acz.
// Point-source cells carry no adjoint into the step before (their value is
// overwritten).  dJ/d eps = sum over the Ez cells whose average includes
// the cell of dJ/d im * (-im^2 / n_points).
//
// Execution: one persistent cooperative kernel runs many half-steps with a
// bounded grid barrier between them (a 512^2 grid is a few MB per field and
// lives in L2, so a half-step is far shorter than a kernel launch).  The
// forward run is one launch that also stores the checkpoints (the state
// before every K-th step) and, for the last segment, dEz/dim and the probe
// values the reverse sweep needs.  Every reverse launch splits its CTAs in
// two groups with a barrier each: one group reverses segment j from the
// stored per-step data while the other recomputes segment j - 1 from its
// checkpoint into the other half of the double buffer.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "adjoint.h"
#include "kernels.h"

namespace fdtdb {

namespace {

constexpr int kEz = 0, kHx = 1, kHy = 2;   // local component slots
constexpr double kEta0Adj = 376.730313461770655;
constexpr int kThreads = 512;
constexpr int kBarStride = 64;             // words per group barrier: arrivals at [0], generation at [32]
constexpr long long kDefaultBarrierLimitNs = 2000000000LL;   // 2 s

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

// One persistent launch.  CTAs [0, fwd_ctas) run forward steps fk0 .. fk1 - 1,
// the others reverse steps rk1 - 1 .. max(rk0, 1).
template <typename R>
struct Launch
{
  AdjDev<R> p;
  int N, npr;
  // forward group
  int fwd_ctas;
  uint32_t fk0, fk1;
  R *F[6];                     // Ez, Hx, Hy, Xz, Xx, Xy
  const R *load;               // state to start from (6 N values) or null
  R *ck;                       // state before step k stored at ck + (k / every) 6 N when k % every == 0, or null
  uint32_t every;
  R *dedm;                     // dEz/dim of step k at dedm + (k - keep0) N for k >= keep0, or null
  double *keep;                // probe Ez of step k at keep + (k - keep0) npr
  uint32_t keep0;
  double *acc;                 // compensated J (sum, compensation) or null
  // reverse group
  uint32_t rk0, rk1;
  R *aE, *aXz, *aHx, *aHy, *aXx, *aXy;
  R *acx, *acy, *acz;          // curl adjoints of the H cells and of the Ez cells
  const R *rdedm;              // dEz/dim of step k at rdedm + (k - rk0) N
  const double *rprobe;        // probe Ez of step k at rprobe + (k - rk0) npr
  double *gim;
  // barriers: arrivals at [0] and generation at [32] for the forward group,
  // the same from [kBarStride] for the reverse group (each word in its own
  // 128-byte line, so polling does not slow the arrivals)
  unsigned *bar;
  int *err;
  long long limit_ns;          // time limit of one barrier wait
};

// values that other CTAs of the launch write are read through L2
template <typename R>
__device__ __forceinline__ R ld (const R *q)
{
  return __ldcg (q);
}

__device__ __forceinline__ long long globaltimer ()
{
  long long t;
  asm volatile ("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Barrier over the `ctas` CTAs of one group, with a time limit.  Returns
// false (and sets *err) when any CTA gave up; every CTA then leaves.
__device__ bool group_barrier (unsigned *bar, unsigned ctas, int *err, long long limit_ns)
{
  __shared__ int ok;
  __syncthreads ();
  if (threadIdx.x == 0)
  {
    volatile unsigned *gen = bar + 32;
    const unsigned g = *gen;
    __threadfence ();
    if (atomicAdd (bar, 1u) == ctas - 1)
    {
      atomicExch (bar, 0u);
      __threadfence ();
      atomicAdd (bar + 32, 1u);
    }
    else
    {
      const long long t0 = globaltimer ();
      while (*gen == g)
      {
        if (*((volatile int *) err) != 0 || globaltimer () - t0 > limit_ns)
        {
          atomicExch (err, 1);
          break;
        }
        __nanosleep (20);
      }
    }
    __threadfence ();
    ok = *((volatile int *) err) == 0;
  }
  __syncthreads ();
  return ok != 0;
}

template <typename R>
__device__ __forceinline__ bool interior (const AdjDev<R> &p, int c, int x, int y)
{
  return x >= p.ilo[c][0] && x < p.ihi[c][0] && y >= p.ilo[c][1] && y < p.ihi[c][1];
}

template <typename R>
__device__ __forceinline__ bool updated (const AdjDev<R> &p, int x, int y)
{
  return x >= 1 && x <= p.nx - 2 && y >= 1 && y <= p.ny - 2;
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
    v0 = ld (f + (x + p.d11[c][0]) * ny + y + p.d11[c][1]);
    v1 = ld (f + (x + p.d12[c][0]) * ny + y + p.d12[c][1]);
  }
  if (p.o2[c] >= 0)
  {
    const R *f = F[p.o2[c]];
    v2 = ld (f + (x + p.d21[c][0]) * ny + y + p.d21[c][1]);
    v3 = ld (f + (x + p.d22[c][0]) * ny + y + p.d22[c][1]);
  }
  return (v1 - v0) - (v3 - v2);
}

// one component update at (x, y); returns dF/d(im) for the gradient
template <typename R>
__device__ __forceinline__ R update_cell (const AdjDev<R> &p, int c, R *F, R *X, R cu, R im, int x, int y)
{
  const int id = x * p.ny + y;
  R f = ld (F + id);
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
    const R xo = ld (X + id);
    const R xn = ca1 * xo + sq1 * cu;
    X[id] = xn;
    dfdm = (g4p * xn - g4m * xo) * q5;
    f = p5 * f + (g4p * xn - g4m * xo) * q5 * im;
  }
  F[id] = f;
  return dfdm;
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

// sum over the probe of Ez^2 by one CTA (the result is valid in thread 0);
// the probe values are optionally kept
template <typename R>
__device__ double probe_sum (const AdjDev<R> &p, const R *Ez, double *keep)
{
  __shared__ double part[kThreads / 32];
  const int w = p.pr_hi[1] - p.pr_lo[1];
  const int n = (p.pr_hi[0] - p.pr_lo[0]) * w;
  double s = 0.0;
  for (int t = threadIdx.x; t < n; t += blockDim.x)
  {
    const int x = p.pr_lo[0] + t / w, y = p.pr_lo[1] + t % w;
    const double v = (double) ld (Ez + x * p.ny + y);
    if (keep)
      keep[t] = v;
    s += v * v;
  }
  for (int o = 16; o > 0; o >>= 1)
    s += __shfl_down_sync (0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0)
    part[threadIdx.x >> 5] = s;
  __syncthreads ();
  double tot = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int) (blockDim.x >> 5); ++i)
      tot += part[i];
  return tot;
}

// ---- forward group

template <typename R>
__device__ void forward_part (const Launch<R> &L, int cta, int ctas)
{
  const AdjDev<R> &p = L.p;
  const int N = L.N;
  const int tid = cta * blockDim.x + threadIdx.x, stride = ctas * blockDim.x;
  unsigned *bar = L.bar;
  R *Ez = L.F[0], *Hx = L.F[1], *Hy = L.F[2], *Xz = L.F[3], *Xx = L.F[4], *Xy = L.F[5];
  const R *Fc[3] = {Ez, Hx, Hy};
  if (L.load)
  {
    for (int i = tid; i < N; i += stride)
      for (int q = 0; q < 6; ++q)
        L.F[q][i] = L.load[(size_t) q * N + i];
    if (!group_barrier (bar, ctas, L.err, L.limit_ns))
      return;
  }
  const bool accum = L.acc && cta == 0 && threadIdx.x == 0;
  double js = 0.0, jc = 0.0;
  if (accum)
  {
    js = L.acc[0];
    jc = L.acc[1];
  }
  for (uint32_t k = L.fk0; k < L.fk1; ++k)
  {
    const bool upd = k > 0;
    const bool kept = L.dedm && k >= L.keep0;
    R *dd = kept ? L.dedm + (size_t) (k - L.keep0) * N : nullptr;
    R *save = (L.ck && k % L.every == 0) ? L.ck + (size_t) (k / L.every) * 6 * N : nullptr;
    // E half-step (and the checkpoint of the state before it)
    for (int i = tid; i < N; i += stride)
    {
      if (save)
        for (int q = 0; q < 6; ++q)
          save[(size_t) q * N + i] = ld (L.F[q] + i);
      const int x = i / p.ny, y = i % p.ny;
      if (!updated (p, x, y))
        continue;
      R d = 0;
      if (upd)
        d = update_cell (p, kEz, Ez, Xz, curl_of (p, kEz, Fc, x, y), p.im[i], x, y);
      if (p.ps_on[kEz] && x == p.ps[0] && y == p.ps[1])
        Ez[i] = p.src[2 * k];
      if (dd)
        dd[i] = d;
    }
    if (!group_barrier (bar, ctas, L.err, L.limit_ns))
      return;
    // probe term of Ez_k, then the H half-step
    if (cta == 0 && (L.acc || kept))
    {
      const double v = probe_sum (p, Ez, kept ? L.keep + (size_t) (k - L.keep0) * L.npr : nullptr);
      if (accum)
        kahan_add (js, jc, v);
    }
    for (int i = tid; i < N; i += stride)
    {
      const int x = i / p.ny, y = i % p.ny;
      if (!updated (p, x, y))
        continue;
      if (upd)
      {
        const R cx = curl_of (p, kHx, Fc, x, y), cy = curl_of (p, kHy, Fc, x, y);
        update_cell (p, kHx, Hx, Xx, cx, R (1), x, y);
        update_cell (p, kHy, Hy, Xy, cy, R (1), x, y);
      }
      if (x == p.ps[0] && y == p.ps[1])
      {
        if (p.ps_on[kHx])
          Hx[i] = p.src[2 * k + 1];
        if (p.ps_on[kHy])
          Hy[i] = p.src[2 * k + 1];
      }
    }
    if (!group_barrier (bar, ctas, L.err, L.limit_ns))
      return;
  }
  if (accum)
  {
    L.acc[0] = js;
    L.acc[1] = jc;
  }
}

// ---- reverse group

// H phase at H cell t: gather acz, transpose of the H update and H source
template <typename R>
__device__ __forceinline__ void adj_h_cell (const Launch<R> &L, int t)
{
  const AdjDev<R> &p = L.p;
  const int x = t / p.ny, y = t % p.ny;
  // Ez's curl reads H comp o at e + d: the H cell (x, y) is read by e = (x, y) - d
  auto take = [&] (const int d[2], R sgn) -> R {
    const int ex = x - d[0], ey = y - d[1];
    return updated (p, ex, ey) ? sgn * ld (L.acz + ex * p.ny + ey) : R (0);
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
  if (!updated (p, x, y))
    return;
  const bool at_src = x == p.ps[0] && y == p.ps[1];
#pragma unroll
  for (int q = 0; q < 2; ++q)
  {
    const int c = q ? kHy : kHx;
    R *aH = q ? L.aHy : L.aHx;
    R *aX = q ? L.aXy : L.aXx;
    R a = ld (aH + t) + g[q];
    if (at_src && p.ps_on[c])
      a = 0;
    R acu;
    if (interior (p, c, x, y))
    {
      acu = p.S * a;
      aH[t] = a;
    }
    else
    {
      const R ca1 = tabv (p, c, 0, x, y), sq1 = tabv (p, c, 1, x, y);
      const R p5 = tabv (p, c, 2, x, y), q5 = tabv (p, c, 3, x, y);
      const R g4p = tabv (p, c, 4, x, y), g4m = tabv (p, c, 5, x, y);
      const R t1 = ld (aX + t) + g4p * q5 * a;
      acu = sq1 * t1;
      aX[t] = ca1 * t1 - g4m * q5 * a;
      aH[t] = p5 * a;
    }
    (q ? L.acy : L.acx)[t] = acu;
  }
}

// E phase at Ez cell t: gather acx, acy, probe term, gradient of im,
// transpose of the E update and E source
template <typename R>
__device__ __forceinline__ void adj_e_cell (const Launch<R> &L, int t, const R *dedm, const double *probe)
{
  const AdjDev<R> &p = L.p;
  const int x = t / p.ny, y = t % p.ny;
  if (!updated (p, x, y))
    return;
  R g = 0;
#pragma unroll
  for (int q = 0; q < 2; ++q)
  {
    const int c = q ? kHy : kHx;
    const R *acu = q ? L.acy : L.acx;
    // H cell h reads Ez at h + d: the Ez cell (x, y) is read by h = (x, y) - d
    auto take = [&] (const int d[2], R sgn) {
      const int hx = x - d[0], hy = y - d[1];
      if (updated (p, hx, hy))
        g += sgn * ld (acu + hx * p.ny + hy);
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
  R a = ld (L.aE + t) + g;
  if (x >= p.pr_lo[0] && x < p.pr_hi[0] && y >= p.pr_lo[1] && y < p.pr_hi[1])
    a += (R) (2.0 * probe[(x - p.pr_lo[0]) * (p.pr_hi[1] - p.pr_lo[1]) + (y - p.pr_lo[1])]);
  if (x == p.ps[0] && y == p.ps[1] && p.ps_on[kEz])
    a = 0;
  L.gim[t] += (double) a * (double) dedm[t];
  const R im = p.im[t];
  if (interior (p, kEz, x, y))
  {
    L.acz[t] = p.S * im * a;
    L.aE[t] = a;
  }
  else
  {
    const R ca1 = tabv (p, kEz, 0, x, y), sq1 = tabv (p, kEz, 1, x, y);
    const R p5 = tabv (p, kEz, 2, x, y), q5 = tabv (p, kEz, 3, x, y);
    const R g4p = tabv (p, kEz, 4, x, y), g4m = tabv (p, kEz, 5, x, y);
    const R t1 = ld (L.aXz + t) + g4p * q5 * im * a;
    L.acz[t] = sq1 * t1;
    L.aXz[t] = ca1 * t1 - g4m * q5 * im * a;
    L.aE[t] = p5 * a;
  }
}

template <typename R>
__device__ void reverse_part (const Launch<R> &L, int cta, int ctas)
{
  const int N = L.N;
  const int tid = cta * blockDim.x + threadIdx.x, stride = ctas * blockDim.x;
  unsigned *bar = L.bar + kBarStride;
  for (int64_t k = (int64_t) L.rk1 - 1; k >= (int64_t) L.rk0 && k > 0; --k)
  {
    const size_t off = (size_t) (k - L.rk0);
    for (int t = tid; t < N; t += stride)
      adj_h_cell (L, t);
    if (!group_barrier (bar, ctas, L.err, L.limit_ns))
      return;
    const R *dedm = L.rdedm + off * N;
    const double *probe = L.rprobe + off * L.npr;
    for (int t = tid; t < N; t += stride)
      adj_e_cell (L, t, dedm, probe);
    if (!group_barrier (bar, ctas, L.err, L.limit_ns))
      return;
  }
}

template <typename R>
__global__ void __launch_bounds__ (kThreads) adjoint_kernel (Launch<R> L)
{
  if ((int) blockIdx.x < L.fwd_ctas)
    forward_part (L, blockIdx.x, L.fwd_ctas);
  else
    reverse_part (L, blockIdx.x - L.fwd_ctas, gridDim.x - L.fwd_ctas);
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

}  // namespace

// ------------------------------------------------------------------ host side

namespace {

// One device allocation carved into 256-byte aligned pieces: reserve() every
// piece first, then allocate() once and take the pointers with at().
struct Arena
{
  std::vector<size_t> off;
  size_t total = 0;
  char *base = nullptr;
  AdjointCache *cache = nullptr;   // when set, the allocation outlives the run
  ~Arena ()
  {
    if (base && !cache)
      cudaFree (base);
  }
  template <typename Q>
  int reserve (size_t count)
  {
    off.push_back (total);
    total += (std::max<size_t> (count, 1) * sizeof (Q) + 255) & ~(size_t) 255;
    return (int) off.size () - 1;
  }
  bool allocate ()
  {
    const size_t need = std::max<size_t> (total, 256);
    if (cache && cache->base && cache->bytes >= need)
    {
      base = (char *) cache->base;
      return true;
    }
    if (cache && cache->base)
    {
      cudaFree (cache->base);
      cache->base = nullptr;
      cache->bytes = 0;
    }
    if (device_malloc ((void **) &base, need) != cudaSuccess)
      return false;
    if (cache)
    {
      cache->base = base;
      cache->bytes = need;
    }
    return true;
  }
  template <typename Q>
  Q *at (int i) const
  {
    return (Q *) (base + off[i]);
  }
};

int local_slot (int k)
{
  return k == EZ ? kEz : (k == HX ? kHx : (k == HY ? kHy : -1));
}

template <typename R>
cudaError_t launch (const Launch<R> &L, int ctas, cudaStream_t s)
{
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3 (ctas);
  lc.blockDim = dim3 (kThreads);
  lc.stream = s;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeCooperative;
  attr.val.cooperative = 1;
  lc.attrs = &attr;
  lc.numAttrs = 1;
  return cudaLaunchKernelEx (&lc, adjoint_kernel<R>, L);
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
  if (N > (size_t) 1 << 30)
    return "grid too large for the adjoint";
  if (run.steps < 1 || run.every < 1)
    return "steps and checkpoint interval must be positive";
  for (int a = 0; a < 2; ++a)
    if (run.probe_lo[a] < 1 || run.probe_hi[a] > g.n[a] - 1 || run.probe_lo[a] >= run.probe_hi[a])
      return "probe box outside the updated cells";
  const int npr = (run.probe_hi[0] - run.probe_lo[0]) * (run.probe_hi[1] - run.probe_lo[1]);

  // co-resident CTAs of the cooperative kernel (at most three per SM: each
  // half-step is latency-bound, so more resident threads help)
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor (&per_sm, adjoint_kernel<R>, kThreads, 0) != cudaSuccess ||
      per_sm < 1)
    return "the adjoint kernel does not fit on an SM";
  // 3 CTAs per SM and an even split between the reversing and the
  // recomputing group measured fastest
  const int cap = 3;
  const int ctas = sm_count * std::min (per_sm, cap);
  const double split = 0.5;
  const int fwd_split = std::max (1, std::min (ctas - 1, (int) std::lround (ctas * split)));

  AdjDev<R> p{};
  p.nx = nx;
  p.ny = ny;
  const double S = 299792458.0 * g.dt / g.dx;
  p.S = (R) S;
  const int kmap[3] = {EZ, HX, HY};

  // host copies of the tables and the source values
  std::vector<std::vector<R>> tabs;
  for (int c = 0; c < 3; ++c)
  {
    const int k = kmap[c];
    const CompLayout &CL = g.comp[k];
    p.o1[c] = g.comp[CL.opp1].exists ? local_slot (CL.opp1) : -1;
    p.o2[c] = g.comp[CL.opp2].exists ? local_slot (CL.opp2) : -1;
    for (int a = 0; a < 2; ++a)
    {
      p.d11[c][a] = CL.d11[a];
      p.d12[c][a] = CL.d12[a];
      p.d21[c][a] = CL.d21[a];
      p.d22[c][a] = CL.d22[a];
    }
    const int axes[3] = {CL.sig_cacb, CL.sig5, CL.sig4};
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
      tabs.push_back (std::move (v));
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
  std::vector<R> src (2 * (size_t) run.steps);
  for (uint32_t k = 0; k < run.steps; ++k)
  {
    src[2 * k] = (R) point_source (g, k, false);
    src[2 * k + 1] = (R) point_source (g, k, true) * (R) kEta0Adj;
  }
  for (int a = 0; a < 2; ++a)
  {
    p.pr_lo[a] = run.probe_lo[a];
    p.pr_hi[a] = run.probe_hi[a];
  }

  // device memory, one allocation
  const bool grad = grad_host != nullptr;
  const uint32_t K = std::min (run.every, run.steps);
  const uint32_t nck = (run.steps + K - 1) / K;
  Arena ar;
  ar.cache = run.cache;
  std::vector<int> i_tab;
  for (const auto &v : tabs)
    i_tab.push_back (ar.reserve<R> (v.size ()));
  const int i_src = ar.reserve<R> (src.size ());
  const int i_state = ar.reserve<R> (6 * N);
  const int i_im = ar.reserve<R> (N);
  const int i_imd = ar.reserve<double> (N);
  const int i_acc = ar.reserve<double> (2);
  const int i_bar = ar.reserve<unsigned> (2 * kBarStride);
  const int i_err = ar.reserve<int> (1);
  int i_ck = -1, i_dedm[2] = {-1, -1}, i_probe[2] = {-1, -1}, i_adj = -1, i_gim = -1, i_gout = -1;
  if (grad)
  {
    i_ck = ar.reserve<R> ((size_t) nck * 6 * N);
    for (int b = 0; b < 2; ++b)
    {
      i_dedm[b] = ar.reserve<R> ((size_t) K * N);
      i_probe[b] = ar.reserve<double> ((size_t) K * npr);
    }
    i_adj = ar.reserve<R> (9 * N);
    i_gim = ar.reserve<double> (N);
    i_gout = ar.reserve<double> (N);
  }
  if (!ar.allocate ())
    return "device allocation failed";
  for (size_t t = 0; t < tabs.size (); ++t)
  {
    R *d = ar.at<R> (i_tab[t]);
    if (cudaMemcpyAsync (d, tabs[t].data (), tabs[t].size () * sizeof (R), cudaMemcpyHostToDevice, s) != cudaSuccess)
      return "table upload failed";
    p.tab[t / 6][t % 6] = d;
  }
  if (cudaMemcpyAsync (ar.at<R> (i_src), src.data (), src.size () * sizeof (R), cudaMemcpyHostToDevice, s) !=
      cudaSuccess)
    return "source table upload failed";
  p.src = ar.at<R> (i_src);
  R *imw = ar.at<R> (i_im);
  p.im = imw;
  R *state = ar.at<R> (i_state);
  double *acc = ar.at<double> (i_acc);
  unsigned *bar = ar.at<unsigned> (i_bar);
  int *err = ar.at<int> (i_err);
  if (cudaMemsetAsync (state, 0, 6 * N * sizeof (R), s) != cudaSuccess ||
      cudaMemsetAsync (acc, 0, 2 * sizeof (double), s) != cudaSuccess ||
      cudaMemsetAsync (bar, 0, 2 * kBarStride * sizeof (unsigned), s) != cudaSuccess ||
      cudaMemsetAsync (err, 0, sizeof (int), s) != cudaSuccess)
    return "device initialisation failed";
  const CompLayout &LE = g.comp[EZ];
  const int blocks = (int) std::min<size_t> ((N + 255) / 256, (size_t) sm_count * 8);
  double *imd = ar.at<double> (i_imd);
  if (eps_is_double)
    invm_kernel<R, double><<<blocks, 256, 0, s>>> ((const double *) eps_dev, nx, ny, LE.nmat, LE.m[1][0], LE.m[1][1],
                                                   LE.m[2][0], LE.m[2][1], LE.m[3][0], LE.m[3][1], imw, imd);
  else
    invm_kernel<R, float><<<blocks, 256, 0, s>>> ((const float *) eps_dev, nx, ny, LE.nmat, LE.m[1][0], LE.m[1][1],
                                                  LE.m[2][0], LE.m[2][1], LE.m[3][0], LE.m[3][1], imw, imd);

  Launch<R> L{};
  L.p = p;
  L.N = (int) N;
  L.npr = npr;
  L.bar = bar;
  L.err = err;
  L.limit_ns = run.wait_limit_ns > 0 ? run.wait_limit_ns : kDefaultBarrierLimitNs;
  for (int q = 0; q < 6; ++q)
    L.F[q] = state + (size_t) q * N;

  // forward run: checkpoints, and the per-step data of the last segment
  const uint32_t last0 = (nck - 1) * K;
  L.fwd_ctas = ctas;
  L.fk0 = 0;
  L.fk1 = run.steps;
  L.acc = acc;
  L.every = K;
  if (grad)
  {
    L.ck = ar.at<R> (i_ck);
    L.dedm = ar.at<R> (i_dedm[0]);
    L.keep = ar.at<double> (i_probe[0]);
    L.keep0 = last0;
  }
  if (launch (L, ctas, s) != cudaSuccess)
    return std::string ("adjoint forward launch failed: ") + cudaGetErrorString (cudaGetLastError ());
  double hacc[2];
  int herr = 0;
  if (cudaMemcpyAsync (hacc, acc, sizeof (hacc), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync (&herr, err, sizeof (int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize (s) != cudaSuccess)
    return std::string ("forward run failed: ") + cudaGetErrorString (cudaGetLastError ());
  if (herr)
    return "a grid barrier of the adjoint forward run timed out";
  if (objective)
    *objective = hacc[0] + hacc[1];
  if (!grad)
    return "";

  // reverse sweep: launch idx reverses segment j = nck - 1 - idx from buffer
  // idx & 1 and recomputes segment j - 1 into the other buffer
  R *adj = ar.at<R> (i_adj);
  double *gim = ar.at<double> (i_gim);
  if (cudaMemsetAsync (adj, 0, 9 * N * sizeof (R), s) != cudaSuccess ||
      cudaMemsetAsync (gim, 0, N * sizeof (double), s) != cudaSuccess)
    return "device initialisation failed";
  R *A[9];
  for (int q = 0; q < 9; ++q)
    A[q] = adj + (size_t) q * N;
  L.aE = A[0];
  L.aXz = A[1];
  L.aHx = A[2];
  L.aHy = A[3];
  L.aXx = A[4];
  L.aXy = A[5];
  L.acx = A[6];
  L.acy = A[7];
  L.acz = A[8];
  L.gim = gim;
  L.acc = nullptr;
  L.ck = nullptr;
  const R *ck = ar.at<R> (i_ck);
  for (uint32_t idx = 0; idx < nck; ++idx)
  {
    const uint32_t j = nck - 1 - idx;
    const int b = (int) (idx & 1u);
    L.rk0 = j * K;
    L.rk1 = std::min (L.rk0 + K, run.steps);
    L.rdedm = ar.at<R> (i_dedm[b]);
    L.rprobe = ar.at<double> (i_probe[b]);
    if (j > 0)
    {
      L.fwd_ctas = fwd_split;
      L.fk0 = (j - 1) * K;
      L.fk1 = j * K;
      L.load = ck + (size_t) (j - 1) * 6 * N;
      L.dedm = ar.at<R> (i_dedm[1 - b]);
      L.keep = ar.at<double> (i_probe[1 - b]);
      L.keep0 = L.fk0;
    }
    else
    {
      L.fwd_ctas = 0;
      L.load = nullptr;
      L.dedm = nullptr;
      L.keep = nullptr;
    }
    if (launch (L, ctas, s) != cudaSuccess)
      return std::string ("adjoint reverse launch failed: ") + cudaGetErrorString (cudaGetLastError ());
  }
  double *gout = ar.at<double> (i_gout);
  grad_eps_kernel<R><<<blocks, 256, 0, s>>> (p, gim, imd, LE.nmat, LE.m[0][0], LE.m[0][1], LE.m[1][0], LE.m[1][1],
                                             LE.m[2][0], LE.m[2][1], LE.m[3][0], LE.m[3][1], gout);
  if (cudaMemcpyAsync (grad_host, gout, N * sizeof (double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync (&herr, err, sizeof (int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize (s) != cudaSuccess)
    return std::string ("reverse run failed: ") + cudaGetErrorString (cudaGetLastError ());
  if (herr)
    return "a grid barrier of the adjoint reverse sweep timed out";
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
