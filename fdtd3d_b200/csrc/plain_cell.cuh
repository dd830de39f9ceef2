// plain_cell.cuh - per-cell arithmetic of the FP64 plain form.
//
// The plain form restates fdtd3d's step with the reference's formulation
// (D/B everywhere when PML is on, D -> D1 -> E with metamaterials, two or
// three stored time levels) and the reference's operation order.  Its
// translation unit is compiled with --fmad=false so every multiply and add
// rounds separately, as the reference's x86-64 build does; FP64 division is
// IEEE round-to-nearest on the device.  With the set-up scalars computed on
// the host by the same libm calls, the results are bit-identical to the
// reference CPU double build.
//
//   calcField ...................... Source/Scheme/InternalScheme.inc.h:766-772
//   calculateFieldStepIteration .... InternalScheme.inc.h:2351-2417
//   computeCaCb .................... InternalScheme.inc.h:2297-2349
//   calculateTFSF .................. InternalScheme.inc.h:1386-1835
//   approximateIncidentWave ........ InternalScheme.inc.h:500-515, InternalScheme.cpp:293-324
//   ...PMLMetamaterials / calcFieldDrude  InternalScheme.inc.h:2452-2549, 775-780
//   ...PML / calcFieldFromDOrB ..... InternalScheme.inc.h:2551-2640, 783-787
//   getMaterial / getMetaMaterial .. InternalScheme.inc.h:2897-3213
//   J / M current sources .......... Scheme.inc.h:1171-1260, InternalScheme.inc.h:2423-2449
#pragma once

#include "params.h"

namespace fdtdb {

constexpr double kEps0Dev = 1 / ((4 * 3.14159265358979323846 * 0.0000001) * (299792458.0 * 299792458.0));

FDTDB_HD inline size_t lin (const GeomDev &g, int x, int y, int z)
{
  return ((size_t) x * g.n[1] + y) * g.n[2] + z;
}

// Average of a component's 1, 2 or 4 material points (v1 .. v3 unused
// below their count).  Helpers here keep their values in scalars, never in
// indexed local arrays, so that nothing goes through local memory.
FDTDB_HD inline double avg_points (int nmat, double v0, double v1, double v2, double v3)
{
  if (nmat == 1)
    return v0;
  if (nmat == 2)
    return (v0 + v1) / 2.0;
  return ((v0 + v1) / 2.0 + (v2 + v3) / 2.0) / 2.0;
}

FDTDB_HD inline double material_at (const GeomDev &g, const CompDev &c, const double *m, int j, int x, int y, int z)
{
  return m[lin (g, x + c.m[j][0], y + c.m[j][1], z + c.m[j][2])];
}

FDTDB_HD inline double material_avg (const GeomDev &g, const CompDev &c, const double *m, int x, int y, int z)
{
  const double v0 = material_at (g, c, m, 0, x, y, z);
  const double v1 = c.nmat > 1 ? material_at (g, c, m, 1, x, y, z) : 0.0;
  const double v2 = c.nmat > 2 ? material_at (g, c, m, 2, x, y, z) : 0.0;
  const double v3 = c.nmat > 3 ? material_at (g, c, m, 3, x, y, z) : 0.0;
  return avg_points (c.nmat, v0, v1, v2, v3);
}

FDTDB_HD inline double sigma_avg (const CompDev &c, const double *s, int axis, int x, int y, int z)
{
  const int q = axis == 0 ? x : (axis == 1 ? y : z);
  const double v0 = s[q + c.m[0][axis]];
  const double v1 = c.nmat > 1 ? s[q + c.m[1][axis]] : 0.0;
  const double v2 = c.nmat > 2 ? s[q + c.m[2][axis]] : 0.0;
  const double v3 = c.nmat > 3 ? s[q + c.m[3][axis]] : 0.0;
  return avg_points (c.nmat, v0, v1, v2, v3);
}

// Drude averaging of plasma frequency / collision rate: the two-point form
// divides by 2.0, the four-point form divides the plain sum by 4.0
// (Source/Layout/Approximation.cpp:58-165).
FDTDB_HD inline double drude_avg (const GeomDev &g, const CompDev &c, const double *m, int x, int y, int z)
{
  const double v0 = material_at (g, c, m, 0, x, y, z);
  const double v1 = material_at (g, c, m, 1, x, y, z);
  if (c.nmat == 2)
    return (v0 + v1) / 2.0;
  const double v2 = material_at (g, c, m, 2, x, y, z);
  const double v3 = material_at (g, c, m, 3, x, y, z);
  return (v0 + v1 + v2 + v3) / 4.0;
}

// Incident value of absolute component `k` at integer cell position pos,
// projected onto k (incident grid at level 1).  Out-of-range indices never
// happen for valid geometry; they read as 0 and raise the error flag.
FDTDB_HD inline double incident_value (const GeomDev &g, const double *inc, int inc_len, int *err,
                                       int k, int px, int py, int pz)
{
  double d_diff = k >= 3 ? 0.5 : 0.0;
  double d;
  if (g.drop == 0)
  {
    double x = ((double) px + g.min_fp[k][0]) - g.zero_inc[0];
    double y = ((double) py + g.min_fp[k][1]) - g.zero_inc[1];
    double z = ((double) pz + g.min_fp[k][2]) - g.zero_inc[2];
    d = x * g.s1 * g.c2 + y * g.s1 * g.s2 + z * g.c1 - d_diff;
  }
  else
  {
    // 2-D / 1-D: the mode's own form (InternalScheme.cpp:110-307)
    const int a0 = g.inc_ax[0], a1 = g.inc_ax[1];
    const int p0 = a0 == 0 ? px : (a0 == 1 ? py : pz), p1 = a1 == 0 ? px : (a1 == 1 ? py : pz);
    double u = ((double) p0 + g.min_fp[k][a0]) - g.zero_inc[a0];
    double v = ((double) p1 + g.min_fp[k][a1]) - g.zero_inc[a1];
    d = u * g.inc_k[0] + v * g.inc_k[1] - d_diff;
  }
  double cd1 = (double) ((int) d);
  double cd2 = cd1 + 1;
  double pr2 = d - cd1;
  double pr1 = 1 - pr2;
  int i1 = (int) cd1;
  int i2 = (int) cd2;
  if (i1 < 0 || i2 >= inc_len)
  {
    if (err)
      *err = 1;
    return 0.0;
  }
  double v = inc[i1] * pr1 + inc[i2] * pr2;
  return v * g.proj[k];
}

// One component of one half-step at one interior cell: curl (+ TF/SF) into
// level 0 of E/H (no PML) or D/B (PML), then Drude and E-from-D.
// DMP: per-component material and sigma arrays (double material precision);
// CS: a current source on this family.  Both are template switches so the
// common form keeps the shared arrays and no extra test.
template <bool DMP, bool CS>
FDTDB_HD inline void plain_component (const PlainHalf &p, int ci, int inc_len, int *err, int x, int y, int z)
{
  const GeomDev &g = p.g;
  const CompDev &c = p.comp[ci];
  const size_t id = lin (g, x, y, z);
  const double eps0 = kEps0Dev;
  const double dt = g.dt;
  const double dx = g.dx;

  double *const *grid = p.use_pml ? p.dd[ci] : p.f[ci];
  const double *mat = DMP ? p.matc[ci] : p.mat;
  const double *const *sig = DMP ? p.sigc[ci] : p.sigma;
  double val = grid[1][id];
  double ca, cb;
  if (p.use_pml)
  {
    double material = sigma_avg (c, sig[c.sig_cacb], c.sig_cacb, x, y, z);
    double dd = (2 * eps0 * 1.0 + material * dt);
    ca = (2 * eps0 * 1.0 - material * dt) / dd;
    cb = (2 * eps0 * dt / dx) / dd;
  }
  else
  {
    double material = material_avg (g, c, mat, x, y, z);
    ca = 1.0;
    cb = dt / (material * p.mat_modifier * dx);
  }

  double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
  const double *o1 = p.opp[c.opp1];
  const double *o2 = p.opp[c.opp2];
  if (o1)
  {
    v0 = o1[lin (g, x + c.d11[0], y + c.d11[1], z + c.d11[2])];
    v1 = o1[lin (g, x + c.d12[0], y + c.d12[1], z + c.d12[2])];
  }
  if (o2)
  {
    v2 = o2[lin (g, x + c.d21[0], y + c.d21[1], z + c.d21[2])];
    v3 = o2[lin (g, x + c.d22[0], y + c.d22[1], z + c.d22[2])];
  }
  if (p.use_tfsf)
  {
    for (int t = 0; t < c.nterms; ++t)
    {
      const TermDev &tm = c.term[t];
      if (x >= tm.lo[0] && x < tm.hi[0] && y >= tm.lo[1] && y < tm.hi[1] && z >= tm.lo[2] && z < tm.hi[2])
      {
        double diff = incident_value (g, p.inc, inc_len, err, tm.inc_comp, x + tm.aux[0], y + tm.aux[1],
                                      z + tm.aux[2]);
        if (tm.negate < 0)
          diff *= -1.0;
        if (tm.slot == 0)
          v0 -= diff;
        else if (tm.slot == 1)
          v1 -= diff;
        else if (tm.slot == 2)
          v2 -= diff;
        else
          v3 -= diff;
      }
    }
  }
  double tmp = v1 - v0 - v3 + v2 - 0.0 * dx;
  double nv = val * ca + tmp * cb;
  // J / M current source: -= (I dx) Cb on the freshly updated value, before
  // D -> E (Scheme.inc.h:1171-1260, InternalScheme.inc.h:792-795, 2423-2449)
  if (CS && ((p.cs_mask >> ci) & 1) && x == p.cs[0] && y == p.cs[1] && z == p.cs[2])
    nv -= *p.cs_val * dx * cb;
  grid[0][id] = nv;

  if (!p.use_pml)
    return;

  const double mm = p.mat_modifier;
  if (p.use_meta)
  {
    double cur = p.dd[ci][0][id], prev = p.dd[ci][1][id], pprev = p.dd[ci][2][id];
    double prev1 = p.d1[ci][1][id], pprev1 = p.d1[ci][2][id];
    double material = material_avg (g, c, mat, x, y, z);
    double omega = drude_avg (g, c, p.omega, x, y, z);
    double gamma = drude_avg (g, c, p.gamma, x, y, z);
    double sq = dt * omega;
    double A = 4 * mm * material + 2 * dt * mm * material * gamma + mm * (sq * sq);
    double b0 = (4 + 2 * dt * gamma) / A;
    double b1 = -8 / A;
    double b2 = (4 - 2 * dt * gamma) / A;
    double a1 = (2 * mm * (sq * sq) - 8 * mm * material) / A;
    double a2 = (4 * mm * material - 2 * dt * mm * material * gamma + mm * (sq * sq)) / A;
    p.d1[ci][0][id] = cur * b0 + prev * b1 + pprev * b2 - prev1 * a1 - pprev1 * a2;
  }

  double prev_eh = p.f[ci][1][id];
  double *const *src = p.use_meta ? p.d1[ci] : p.dd[ci];
  double cur_db = src[0][id];
  double prev_db = src[1][id];
  double material1 = material_avg (g, c, mat, x, y, z);
  double material4 = sigma_avg (c, sig[c.sig4], c.sig4, x, y, z);
  double material5 = sigma_avg (c, sig[c.sig5], c.sig5, x, y, z);
  double modifier = material1 * mm;
  if (p.use_meta)
    modifier = 1;
  double dd5 = (2 * eps0 * 1.0 + material5 * dt);
  double ca2 = (2 * eps0 * 1.0 - material5 * dt) / dd5;
  double cb2 = ((2 * eps0 * 1.0 + material4 * dt) / (modifier)) / dd5;
  double cc2 = ((2 * eps0 * 1.0 - material4 * dt) / (modifier)) / dd5;
  p.f[ci][0][id] = prev_eh * ca2 + cur_db * cb2 - prev_db * cc2;
}

}  // namespace fdtdb
