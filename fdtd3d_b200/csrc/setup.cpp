// setup.cpp - geometry, physics scalars and TF/SF terms of the fdtd3d step.
//
// Reference behaviour followed (zer011b/fdtd3d, paths under Source/):
//   dt, frequency, relPhaseVelocity ... Scheme/InternalScheme.inc.h:3359-3394
//   numerical phase velocity .......... Layout/Approximation.cpp:259-359
//   sigma profiles (x vs y/z quirk) ... Scheme/SchemeHelper.h:574-718
//   Yee offsets / circuit diffs ....... Layout/YeeGridLayout.cpp:1937-2035
//                                       (E_CENTERED and H_CENTERED)
//   TF/SF border predicates ........... Layout/YeeGridLayout.h:498-512,
//                                       Layout/YeeGridLayout.cpp:257-1720
//   incident projections .............. Layout/YeeGridLayout.h:2227-2357
//   zeroIncCoordFP .................... Layout/YeeGridLayout.cpp:2600-2660
//   TF/SF slot selection .............. Scheme/InternalScheme.inc.h:1386-1835
#include "setup.h"

#include <cmath>
#include <cstring>

namespace fdtdb {

namespace {

constexpr double kApproxAcc = 0.0000001;   // Layout/Approximation.h:27
constexpr double kFpExact = 0.0000001;     // Kernels/FieldValue.h:153 (double)

bool fp_exact (double a, double b)
{
  return (a > b ? a - b : b - a) < kFpExact;
}

bool axis_angle (double a)
{
  return a == 0 || a == kPi / 2 || a == kPi || a == 3 * kPi / 2;
}

bool diag_angle (double a)
{
  return a == kPi / 4 || a == 3 * kPi / 4 || a == 5 * kPi / 4 || a == 7 * kPi / 4;
}

double wave_number (double delta, double lambda, double courant, double n_lambda, double a1, double a2)
{
  if (axis_angle (a1) && axis_angle (a2))
  {
    return 2.0 / delta * std::asin (std::sin (kPi * courant / n_lambda) / courant);
  }
  if ((axis_angle (a1) && diag_angle (a2)) || (diag_angle (a1) && axis_angle (a2)))
  {
    return 2.0 * std::sqrt (2.0) / delta
           * std::asin (std::sin (kPi * courant / n_lambda) / (courant * std::sqrt (2.0)));
  }
  // Newton iteration on the 3-D numerical dispersion relation
  double k = 2 * kPi;
  double k_prev = k + 2 * std::sqrt (kApproxAcc);
  double nd = delta / lambda;
  double A = nd * std::sin (a1) * std::cos (a2) / 2;
  double B = nd * std::sin (a1) * std::sin (a2) / 2;
  double C = nd * std::cos (a1) / 2;
  double s = std::sin (kPi * courant / n_lambda);
  double D = (s * s) / (courant * courant);
  int guard = 0;
  while ((k_prev - k) * (k_prev - k) >= kApproxAcc && guard++ < 100000)
  {
    k_prev = k;
    double sa = std::sin (A * k), sb = std::sin (B * k), sc = std::sin (C * k);
    double f = sa * sa + sb * sb + sc * sc - D;
    double df = A * std::sin (2 * A * k) + B * std::sin (2 * B * k) + C * std::sin (2 * C * k);
    k -= f / df;
  }
  return k / lambda;
}

double phase_velocity (double delta, double lambda, double courant, double n_lambda, double a1, double a2)
{
  return kC * 2 * kPi / lambda / wave_number (delta, lambda, courant, n_lambda, a1, a2);
}

double sigma_value (double dist, double boundary, double step)
{
  const uint32_t m = 6;
  const double r_err = 1e-16;
  double sigma_max = -std::log (r_err) * (m + 1.0) / (2.0 * std::sqrt (kMu0 / kEps0) * boundary);
  double factor = sigma_max / (step * (std::pow (boundary, m)) * (m + 1));
  double x1 = (dist + 1) * step;
  double x2 = dist * step;
  return factor * (std::pow (x1, (m + 1)) - std::pow (x2, (m + 1)));
}

// Axis 0 keeps the fractional distance and compares against size; axes 1, 2
// truncate the distance and compare against size + 0.5 (the reference's
// initSigmaX / initSigmaY / initSigmaZ differ exactly this way).
// Sigma profile of one axis.  first_variant: the reference's initSigmaX
// form (FP distance, grid size as is), which it applies to the first axis
// of the grid's coordinates (x in 3-D, the plane's first axis in 2-D); the
// other axes take the initSigmaY/Z form (distance truncated to an integer,
// size + 0.5).  SchemeHelper.h:596-718, Scheme.cpp:141-330.
void sigma_profile (std::vector<double> &out, bool first_variant, int n, int pml, double dx)
{
  out.assign (n, 0.0);
  double p = (double) pml;
  double boundary = p * dx;
  for (int i = 0; i < n; ++i)
  {
    double pos = i + 0.5;
    if (first_variant)
    {
      double size = (double) n;
      if (pos < p)
        out[i] = sigma_value (p - pos, boundary, dx);
      else if (pos >= size - p)
        out[i] = sigma_value (pos - (size - p), boundary, dx);
    }
    else
    {
      double size = n + 0.5;
      if (pos < p)
        out[i] = sigma_value ((int32_t) (p - pos), boundary, dx);
      else if (pos >= size - p)
        out[i] = sigma_value ((int32_t) (pos - (size - p)), boundary, dx);
    }
  }
}

void set3 (int *v, int a, int b, int c)
{
  v[0] = a;
  v[1] = b;
  v[2] = c;
}

// Axis tests of one TF/SF border predicate.
enum { T_ANY, T_EXL, T_EXR, T_RANGE };
struct AxisTest
{
  int kind, o1, o2;
};
struct Pred
{
  bool valid;
  AxisTest ax[3];
};
enum { DL, DR, DD, DU, DB, DF, DNONE };

Pred pred (int k0, int a0, int b0, int k1, int a1, int b1, int k2, int a2, int b2)
{
  Pred p;
  p.valid = true;
  p.ax[0] = {k0, a0, b0};
  p.ax[1] = {k1, a1, b1};
  p.ax[2] = {k2, a2, b2};
  return p;
}

}  // namespace

namespace {

// One mode of the reference (SchemeType): the axes it drops, its
// components, and how the incident wave enters (Source/Scheme/InternalScheme.cpp:
// 110-324 distance along the wave vector, Source/Layout/YeeGridLayout.h:
// 1240-2270 projections, Source/Layout/YeeGridLayout.cpp:2050-2580 origin).
enum IncForm
{
  INC_3D,        // x sin(teta) cos(phi) + y sin(teta) sin(phi) + z cos(teta)
  INC_TETA,      // 2-D: u sin(teta) + v cos(teta)
  INC_PHI,       // 2-D: u cos(phi) + v sin(phi)
  INC_1D         // 1-D: the coordinate itself
};

struct ModeSpec
{
  int mode;
  unsigned drop;     // bit a: axis a has size 1
  unsigned comps;    // bit k: component k exists
  IncForm form;
};

constexpr unsigned bit (int k)
{
  return 1u << k;
}

const ModeSpec kModes[] = {
    {FDTD_MODE_DIM3, 0, 0x3f, INC_3D},
    {FDTD_MODE_TMZ, bit (2), bit (EZ) | bit (HX) | bit (HY), INC_PHI},
    {FDTD_MODE_TEZ, bit (2), bit (EX) | bit (EY) | bit (HZ), INC_PHI},
    {FDTD_MODE_TEX, bit (0), bit (EY) | bit (EZ) | bit (HX), INC_TETA},
    {FDTD_MODE_TMX, bit (0), bit (EX) | bit (HY) | bit (HZ), INC_TETA},
    {FDTD_MODE_TEY, bit (1), bit (EX) | bit (EZ) | bit (HY), INC_TETA},
    {FDTD_MODE_TMY, bit (1), bit (EY) | bit (HX) | bit (HZ), INC_TETA},
    {FDTD_MODE_EXHY, bit (0) | bit (1), bit (EX) | bit (HY), INC_1D},
    {FDTD_MODE_EXHZ, bit (0) | bit (2), bit (EX) | bit (HZ), INC_1D},
    {FDTD_MODE_EYHX, bit (0) | bit (1), bit (EY) | bit (HX), INC_1D},
    {FDTD_MODE_EYHZ, bit (1) | bit (2), bit (EY) | bit (HZ), INC_1D},
    {FDTD_MODE_EZHX, bit (0) | bit (2), bit (EZ) | bit (HX), INC_1D},
    {FDTD_MODE_EZHY, bit (1) | bit (2), bit (EZ) | bit (HY), INC_1D},
};

const ModeSpec *mode_spec (int mode)
{
  for (const ModeSpec &m : kModes)
    if (m.mode == mode)
      return &m;
  return nullptr;
}

// Dim3 layout of component k; a 2-D or 1-D mode then drops its axes
// (YeeGridLayout's initAxesCoordinate keeps the coordinates of the kept axes
// of every offset and position).
//
// E_CENTERED (YeeGridLayout.cpp:1937-1990): E_a sits at 1.0 on its own axis
// and 0.5 on the others, H_a at 0.5 / 1.0.  H_CENTERED (YeeGridLayout.cpp:
// 1990-2035) swaps the two families: E_a takes E_CENTERED H_a's position,
// material stencil (YeeGridLayout.h:866-1030) and TF/SF border predicates
// (YeeGridLayout.cpp:257-1720, checked component by component), and H_a
// takes E_CENTERED E_a's.  The circuits keep their partners and directions
// (InternalScheme.inc.h:1840-1895) but their offsets move to the other side:
// an E circuit spans (0, +1) and an H circuit (-1, 0).
void init_components (Geometry &g, unsigned comps, bool h_centered, Pred preds[6][6], int slot_dir[6][4])
{
  for (int k = 0; k < 6; ++k)
  {
    CompLayout &c = g.comp[k];
    std::memset (&c, 0, sizeof (c));
    int a = k % 3;
    // "edge" components sit at 1.0 on their own axis (E in E_CENTERED, H in
    // H_CENTERED) and average two material cells along it; the others sit at
    // 0.5 on their own axis and average four
    bool edge = (k >= 3) == h_centered;
    for (int ax = 0; ax < 3; ++ax)
      c.min_fp[ax] = edge ? (ax == a ? 1.0 : 0.5) : (ax == a ? 0.5 : 1.0);
    c.sig_cacb = (a + 1) % 3;
    c.sig4 = a;
    c.sig5 = (a + 2) % 3;
    if (edge)
    {
      c.nmat = 2;
      c.m[1][a] = 1;
    }
    else
    {
      int lo = a == 0 ? 1 : 0;
      int hi = a == 2 ? 1 : 2;
      c.nmat = 4;
      c.m[1][hi] = 1;
      c.m[2][lo] = 1;
      c.m[3][lo] = 1;
      c.m[3][hi] = 1;
    }
    for (int d = 0; d < 6; ++d)
      preds[k][d].valid = false;
  }
  // predicates are written for E_CENTERED; H_CENTERED reads them with the
  // families swapped (Ex <-> Hx, ...)
  const int pe[3] = {h_centered ? HX : EX, h_centered ? HY : EY, h_centered ? HZ : EZ};
  const int ph[3] = {h_centered ? EX : HX, h_centered ? EY : HY, h_centered ? EZ : HZ};
  // circuit offset of the lower and the upper neighbour
  const int elo = h_centered ? 0 : -1, ehi = h_centered ? 1 : 0;
  const int hlo = h_centered ? -1 : 0, hhi = h_centered ? 0 : 1;
  CompLayout *c;
  c = &g.comp[EX];
  c->opp1 = HZ; c->opp2 = HY;
  set3 (c->d11, 0, elo, 0); set3 (c->d12, 0, ehi, 0); set3 (c->d21, 0, 0, elo); set3 (c->d22, 0, 0, ehi);
  slot_dir[EX][0] = DD; slot_dir[EX][1] = DU; slot_dir[EX][2] = DB; slot_dir[EX][3] = DF;
  preds[pe[0]][DD] = pred (T_RANGE, -1, 1, T_EXL, -5, 0, T_RANGE, 4, -4);
  preds[pe[0]][DU] = pred (T_RANGE, -1, 1, T_EXR, 5, 0, T_RANGE, 4, -4);
  preds[pe[0]][DB] = pred (T_RANGE, -1, 1, T_RANGE, 4, -4, T_EXL, -5, 0);
  preds[pe[0]][DF] = pred (T_RANGE, -1, 1, T_RANGE, 4, -4, T_EXR, 5, 0);
  c = &g.comp[EY];
  c->opp1 = HX; c->opp2 = HZ;
  set3 (c->d11, 0, 0, elo); set3 (c->d12, 0, 0, ehi); set3 (c->d21, elo, 0, 0); set3 (c->d22, ehi, 0, 0);
  slot_dir[EY][0] = DB; slot_dir[EY][1] = DF; slot_dir[EY][2] = DL; slot_dir[EY][3] = DR;
  preds[pe[1]][DL] = pred (T_EXL, -5, 0, T_RANGE, -1, 1, T_RANGE, 4, -4);
  preds[pe[1]][DR] = pred (T_EXR, 5, 0, T_RANGE, -1, 1, T_RANGE, 4, -4);
  preds[pe[1]][DB] = pred (T_RANGE, 4, -4, T_RANGE, -1, 1, T_EXL, -5, 0);
  preds[pe[1]][DF] = pred (T_RANGE, 4, -4, T_RANGE, -1, 1, T_EXR, 5, 0);
  c = &g.comp[EZ];
  c->opp1 = HY; c->opp2 = HX;
  set3 (c->d11, elo, 0, 0); set3 (c->d12, ehi, 0, 0); set3 (c->d21, 0, elo, 0); set3 (c->d22, 0, ehi, 0);
  slot_dir[EZ][0] = DL; slot_dir[EZ][1] = DR; slot_dir[EZ][2] = DD; slot_dir[EZ][3] = DU;
  preds[pe[2]][DL] = pred (T_EXL, -5, 0, T_RANGE, 4, -4, T_RANGE, -1, 1);
  preds[pe[2]][DR] = pred (T_EXR, 5, 0, T_RANGE, 4, -4, T_RANGE, -1, 1);
  preds[pe[2]][DD] = pred (T_RANGE, 4, -4, T_EXL, -5, 0, T_RANGE, -1, 1);
  preds[pe[2]][DU] = pred (T_RANGE, 4, -4, T_EXR, 5, 0, T_RANGE, -1, 1);
  c = &g.comp[HX];
  c->opp1 = EY; c->opp2 = EZ;
  set3 (c->d11, 0, 0, hlo); set3 (c->d12, 0, 0, hhi); set3 (c->d21, 0, hlo, 0); set3 (c->d22, 0, hhi, 0);
  slot_dir[HX][0] = DB; slot_dir[HX][1] = DF; slot_dir[HX][2] = DD; slot_dir[HX][3] = DU;
  preds[ph[0]][DD] = pred (T_RANGE, 4, -4, T_EXL, 0, 0, T_RANGE, -1, 1);
  preds[ph[0]][DU] = pred (T_RANGE, 4, -4, T_EXR, 0, 0, T_RANGE, -1, 1);
  preds[ph[0]][DB] = pred (T_RANGE, 4, -4, T_RANGE, -1, 1, T_EXL, 0, 0);
  preds[ph[0]][DF] = pred (T_RANGE, 4, -4, T_RANGE, -1, 1, T_EXR, 0, 0);
  c = &g.comp[HY];
  c->opp1 = EZ; c->opp2 = EX;
  set3 (c->d11, hlo, 0, 0); set3 (c->d12, hhi, 0, 0); set3 (c->d21, 0, 0, hlo); set3 (c->d22, 0, 0, hhi);
  slot_dir[HY][0] = DL; slot_dir[HY][1] = DR; slot_dir[HY][2] = DB; slot_dir[HY][3] = DF;
  preds[ph[1]][DL] = pred (T_EXL, 0, 0, T_RANGE, 4, -4, T_RANGE, -1, 1);
  preds[ph[1]][DR] = pred (T_EXR, 0, 0, T_RANGE, 4, -4, T_RANGE, -1, 1);
  preds[ph[1]][DB] = pred (T_RANGE, -1, 1, T_RANGE, 4, -4, T_EXL, 0, 0);
  preds[ph[1]][DF] = pred (T_RANGE, -1, 1, T_RANGE, 4, -4, T_EXR, 0, 0);
  c = &g.comp[HZ];
  c->opp1 = EX; c->opp2 = EY;
  set3 (c->d11, 0, hlo, 0); set3 (c->d12, 0, hhi, 0); set3 (c->d21, hlo, 0, 0); set3 (c->d22, hhi, 0, 0);
  slot_dir[HZ][0] = DD; slot_dir[HZ][1] = DU; slot_dir[HZ][2] = DL; slot_dir[HZ][3] = DR;
  preds[ph[2]][DL] = pred (T_EXL, 0, 0, T_RANGE, -1, 1, T_RANGE, 4, -4);
  preds[ph[2]][DR] = pred (T_EXR, 0, 0, T_RANGE, -1, 1, T_RANGE, 4, -4);
  preds[ph[2]][DD] = pred (T_RANGE, -1, 1, T_EXL, 0, 0, T_RANGE, 4, -4);
  preds[ph[2]][DU] = pred (T_RANGE, -1, 1, T_EXR, 0, 0, T_RANGE, 4, -4);

  for (int k = 0; k < 6; ++k)
    g.comp[k].exists = (comps >> k) & 1u;
  // border directions along each axis: x left/right, y down/up, z back/front
  const int dir_lo[3] = {DL, DD, DB}, dir_hi[3] = {DR, DU, DF};
  for (int f = 0; f < 3; ++f)
  {
    if (!((g.drop >> f) & 1u))
      continue;
    for (int k = 0; k < 6; ++k)
    {
      CompLayout &cc = g.comp[k];
      cc.d11[f] = cc.d12[f] = cc.d21[f] = cc.d22[f] = 0;
      for (int j = 0; j < 4; ++j)
        cc.m[j][f] = 0;
      cc.min_fp[f] = 0.0;
      for (int d = 0; d < 6; ++d)
        preds[k][d].ax[f].kind = T_ANY;
      preds[k][dir_lo[f]].valid = false;
      preds[k][dir_hi[f]].valid = false;
    }
  }
}

// The eight fine cells a component averages with double material precision,
// as offsets from (2i, 2j, 2k), in the order of the reference's absPos11,
// 12, 21, 22, 31, 32, 41, 42 (YeeGridLayout.h:866-1030): "edge" components
// (E in E_CENTERED, H in H_CENTERED) along x, y, z, then the others.
const int kFineEdge[3][8][3] = {
    {{1, 0, 0}, {1, 1, 0}, {2, 0, 0}, {2, 1, 0}, {1, 0, 1}, {1, 1, 1}, {2, 0, 1}, {2, 1, 1}},
    {{0, 1, 0}, {1, 1, 0}, {0, 2, 0}, {1, 2, 0}, {0, 1, 1}, {1, 1, 1}, {0, 2, 1}, {1, 2, 1}},
    {{0, 0, 1}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}, {0, 0, 2}, {0, 1, 2}, {1, 0, 2}, {1, 1, 2}},
};
const int kFineFace[3][8][3] = {
    {{0, 1, 1}, {1, 1, 1}, {0, 1, 2}, {1, 1, 2}, {0, 2, 1}, {1, 2, 1}, {0, 2, 2}, {1, 2, 2}},
    {{1, 0, 1}, {1, 1, 1}, {1, 0, 2}, {1, 1, 2}, {2, 0, 1}, {2, 1, 1}, {2, 0, 2}, {2, 1, 2}},
    {{1, 1, 0}, {1, 1, 1}, {1, 2, 0}, {1, 2, 1}, {2, 1, 0}, {2, 1, 1}, {2, 2, 0}, {2, 2, 1}},
};

bool axis_ok (const AxisTest &t, double coord, double left, double right)
{
  switch (t.kind)
  {
    case T_ANY:
      return true;
    case T_EXL:
      return fp_exact (coord, left + t.o1 * 1.0 / 10.0);
    case T_EXR:
      return fp_exact (coord, right + t.o1 * 1.0 / 10.0);
    default:
      return coord > left + t.o1 * 1.0 / 10.0 && coord < right + t.o2 * 1.0 / 10.0;
  }
}

}  // namespace

std::string build_geometry (const fdtd_config &cfg, Geometry &g)
{
  g = Geometry ();
  g.cfg = cfg;
  const ModeSpec *ms = mode_spec (cfg.mode);
  if (!ms)
    return "unknown mode (FDTD_MODE_DIM3, a 2-D or a 1-D mode)";
  if (cfg.layout != 0 && cfg.layout != 1)
    return "unknown layout (0 = E_CENTERED, 1 = H_CENTERED)";
  if (cfg.precision < FDTD_PREC_FP64_PLAIN || cfg.precision > FDTD_PREC_FP16S)
    return "unknown precision";
  if (cfg.use_metamaterials && !cfg.use_pml)
    return "metamaterials require PML (as in the reference)";
  if (cfg.point_source_kind != FDTD_SOURCE_SINE && cfg.point_source_kind != FDTD_SOURCE_GAUSSIAN)
    return "unknown point-source kind";
  if (cfg.point_source_kind == FDTD_SOURCE_GAUSSIAN && !(cfg.point_source_bandwidth > 0))
    return "Gaussian point source needs a positive bandwidth";
  if (cfg.source_phase != 0 && cfg.source_phase != 1)
    return "source_phase must be 0 (sine) or 1 (cosine)";
  if (cfg.current_phase < 0 || cfg.current_phase > 2)
    return "current_phase must be 0 (sin), 1 (complex real part) or 2 (complex imaginary part)";
  if (cfg.current_source_mask & ~0x3f)
    return "current_source_mask has bits beyond the six components";
  if (cfg.double_material_precision && cfg.use_metamaterials)
    return "double material precision with metamaterials is not provided (the reference's eight-point Drude "
           "average is unreachable, Approximation.cpp:167-197)";
  g.tmz = cfg.mode == FDTD_MODE_TMZ;
  g.drop = (int) ms->drop;
  auto active = [&] (int a) { return !((g.drop >> a) & 1); };
  for (int a = 0; a < 3; ++a)
    g.n[a] = active (a) ? cfg.size[a] : 1;
  for (int a = 0; a < 3; ++a)
  {
    if (!active (a))
      continue;
    if (g.n[a] < 3 || g.n[a] > (1 << 20))
      return "grid size out of range";
    if (cfg.use_pml && (cfg.pml[a] < 0 || 2 * cfg.pml[a] >= g.n[a]))
      return "PML size out of range";
    // a right size of 0 puts that face on the grid's last node, where no
    // interior cell takes its terms (the reference's own tests run
    // --tfsf-size-right x:0 for one-sided incidence, Tests/suite/t7.4)
    if (cfg.use_tfsf && (cfg.tfsf_left[a] < 1 || cfg.tfsf_right[a] < 0
                         || cfg.tfsf_left[a] + cfg.tfsf_right[a] >= g.n[a]))
      return "TF/SF size out of range";
  }
  if (!(cfg.dx > 0) || !(cfg.wavelength > 0) || !(cfg.courant > 0))
    return "dx, wavelength and courant factor must be positive";
  g.cells = (int64_t) g.n[0] * g.n[1] * g.n[2];
  g.dmp = cfg.double_material_precision != 0;
  for (int a = 0; a < 3; ++a)
    g.nf[a] = (g.dmp && active (a)) ? 2 * g.n[a] : g.n[a];
  g.fine_cells = (int64_t) g.nf[0] * g.nf[1] * g.nf[2];
  g.levels = (cfg.use_metamaterials && cfg.use_pml) ? 3 : 2;
  g.dx = cfg.dx;

  // InternalScheme::initScheme
  g.freq = kC / cfg.wavelength;
  g.dt = cfg.dx * cfg.courant / kC;
  g.a1 = cfg.angle_teta * kPi / 180.0;
  g.a2 = cfg.angle_phi * kPi / 180.0;
  g.a3 = cfg.angle_psi * kPi / 180.0;
  double n_lambda = cfg.wavelength / cfg.dx;
  double pv0 = phase_velocity (cfg.dx, cfg.wavelength, cfg.courant, n_lambda, kPi / 2, 0);
  double pv = phase_velocity (cfg.dx, cfg.wavelength, cfg.courant, n_lambda, g.a1, g.a2);
  g.rpv = pv0 / pv;
  if (!std::isfinite (g.rpv) || !(g.rpv > 0))
    return "phase-velocity correction did not converge";
  g.mod_e = g.dt / (g.rpv * kEps0 * g.dx);
  g.mod_h = g.dt / (g.rpv * kMu0 * g.dx);
  g.s1 = std::sin (g.a1);
  g.c1 = std::cos (g.a1);
  g.s2 = std::sin (g.a2);
  g.c2 = std::cos (g.a2);
  double s3 = std::sin (g.a3), c3 = std::cos (g.a3);
  for (int k = 0; k < 6; ++k)
    g.proj[k] = 0;
  if (ms->form == INC_3D)
  {
    // the Hz projection carries the reference's leading minus sign
    g.proj[EX] = c3 * g.s2 - s3 * g.c1 * g.c2;
    g.proj[EY] = -c3 * g.c2 - s3 * g.c1 * g.s2;
    g.proj[EZ] = s3 * g.s1;
    g.proj[HX] = s3 * g.s2 + c3 * g.c1 * g.c2;
    g.proj[HY] = -s3 * g.c2 + c3 * g.c1 * g.s2;
    g.proj[HZ] = -(c3 * g.s1);
    g.zero_inc[0] = cfg.tfsf_left[0] - 2.5 * std::sin (g.a1) * std::cos (g.a2);
    g.zero_inc[1] = cfg.tfsf_left[1] - 2.5 * std::sin (g.a1) * std::sin (g.a2);
    g.zero_inc[2] = cfg.tfsf_left[2] - 2.5 * std::cos (g.a1);
  }
  else if (ms->form == INC_1D)
  {
    // the one kept axis; the origin is 2.5 cells before the left TF/SF border
    int a0 = 0;
    while (!active (a0))
      ++a0;
    g.inc_ax[0] = g.inc_ax[1] = a0;
    g.inc_k[0] = 1.0;
    g.inc_k[1] = 0.0;
    g.zero_inc[0] = g.zero_inc[1] = g.zero_inc[2] = 0;
    g.zero_inc[a0] = cfg.tfsf_left[a0] - 2.5;
    switch (cfg.mode)
    {
      case FDTD_MODE_EXHY: g.proj[EX] = -1.0; g.proj[HY] = -1.0; break;
      case FDTD_MODE_EXHZ: g.proj[EX] = 1.0; g.proj[HZ] = -1.0; break;
      case FDTD_MODE_EYHX: g.proj[EY] = -1.0; g.proj[HX] = 1.0; break;
      case FDTD_MODE_EYHZ: g.proj[EY] = -1.0; g.proj[HZ] = -1.0; break;
      case FDTD_MODE_EZHX: g.proj[EZ] = 1.0; g.proj[HX] = 1.0; break;
      default: g.proj[EZ] = 1.0; g.proj[HY] = -1.0; break;   // FDTD_MODE_EZHY
    }
  }
  else
  {
    // plane axes (a0, a1) in x, y, z order; the origin is the left TF/SF
    // corner moved back 2.5 cells along the in-plane wave vector
    const int a0 = active (0) ? 0 : 1, a1 = active (2) ? 2 : 1;
    g.inc_ax[0] = a0;
    g.inc_ax[1] = a1;
    g.zero_inc[0] = g.zero_inc[1] = g.zero_inc[2] = 0;
    if (ms->form == INC_TETA)
    {
      g.inc_k[0] = std::sin (g.a1);
      g.inc_k[1] = std::cos (g.a1);
      g.zero_inc[a0] = cfg.tfsf_left[a0] - 2.5 * std::sin (g.a1);
      g.zero_inc[a1] = cfg.tfsf_left[a1] - 2.5 * std::cos (g.a1);
    }
    else
    {
      g.inc_k[0] = std::cos (g.a2);
      g.inc_k[1] = std::sin (g.a2);
      g.zero_inc[a0] = cfg.tfsf_left[a0] - 2.5 * std::cos (g.a2);
      g.zero_inc[a1] = cfg.tfsf_left[a1] - 2.5 * std::sin (g.a2);
    }
    switch (cfg.mode)
    {
      case FDTD_MODE_TMZ:
        g.proj[EZ] = 1.0;
        g.proj[HX] = std::sin (g.a2);
        g.proj[HY] = -std::cos (g.a2);
        break;
      case FDTD_MODE_TEZ:
        g.proj[EX] = std::sin (g.a2);
        g.proj[EY] = -std::cos (g.a2);
        g.proj[HZ] = -1.0;
        break;
      case FDTD_MODE_TEX:
        g.proj[EY] = -std::cos (g.a1);
        g.proj[EZ] = std::sin (g.a1);
        g.proj[HX] = 1.0;
        break;
      case FDTD_MODE_TMX:
        g.proj[EX] = 1.0;
        g.proj[HY] = std::cos (g.a1);
        g.proj[HZ] = -std::sin (g.a1);
        break;
      case FDTD_MODE_TEY:
        g.proj[EX] = -std::cos (g.a1);
        g.proj[EZ] = std::sin (g.a1);
        g.proj[HY] = -1.0;
        break;
      default:   // FDTD_MODE_TMY
        g.proj[EY] = -1.0;
        g.proj[HX] = std::cos (g.a1);
        g.proj[HZ] = -std::sin (g.a1);
        break;
    }
  }
  // 500 times the grid's first coordinate: x in 3-D, the first kept axis of
  // a 2-D or 1-D mode (InternalScheme.specific.h:105-106)
  g.inc_len = 500 * g.n[active (0) ? 0 : (active (1) ? 1 : 2)];

  // with double material precision the sigma grids are the fine ones:
  // 2 n cells, a PML of 2 p cells, the same dx (SchemeHelper.h:596-718)
  const int fmul = g.dmp ? 2 : 1;
  for (int a = 0; a < 3; ++a)
  {
    g.sigma[a].assign (g.nf[a], 0.0);
    if (cfg.use_pml && active (a))
      sigma_profile (g.sigma[a], a == (active (0) ? 0 : (active (1) ? 1 : 2)), g.nf[a], fmul * cfg.pml[a], cfg.dx);
  }

  Pred preds[6][6];
  int slot_dir[6][4];
  const bool h_centered = cfg.layout == 1;
  init_components (g, ms->comps, h_centered, preds, slot_dir);
  for (int k = 0; k < 6; ++k)
  {
    const bool edge = (k >= 3) == h_centered;
    const int(*tab)[3] = edge ? kFineEdge[k % 3] : kFineFace[k % 3];
    for (int j = 0; j < 8; ++j)
      for (int a = 0; a < 3; ++a)
        g.fine_off[k][j][a] = active (a) ? tab[j][a] : 0;
  }

  if (cfg.use_tfsf)
  {
    double left[3], right[3];
    for (int a = 0; a < 3; ++a)
    {
      left[a] = 0.0 + (double) cfg.tfsf_left[a];
      right[a] = 0.0 + (double) (g.n[a] - cfg.tfsf_right[a]);
    }
    for (int k = 0; k < 6; ++k)
    {
      const CompLayout &c = g.comp[k];
      if (!c.exists)
        continue;
      bool isH = k >= 3;
      int slot_box[4][2][3];
      bool slot_on[4] = {false, false, false, false};
      for (int s = 0; s < 4; ++s)
      {
        const Pred &p = preds[k][slot_dir[k][s]];
        if (!p.valid)
          continue;
        bool empty = false;
        for (int a = 0; a < 3; ++a)
        {
          int lo_r = active (a) ? 1 : 0;
          int hi_r = active (a) ? g.n[a] - 1 : 1;
          int first = -1, last = -2, count = 0;
          for (int i = lo_r; i < hi_r; ++i)
          {
            if (axis_ok (p.ax[a], i + c.min_fp[a], left[a], right[a]))
            {
              if (first < 0)
                first = i;
              last = i;
              ++count;
            }
          }
          if (count == 0)
          {
            empty = true;
            break;
          }
          if (count != last - first + 1)
            return "TF/SF border set is not a box";
          slot_box[s][0][a] = first;
          slot_box[s][1][a] = last + 1;
        }
        slot_on[s] = !empty;
      }
      for (int s = 0; s < 4; ++s)
      {
        if (!slot_on[s])
          continue;
        // slots 11/12 (and 21/22) never hold on the same cell; keep the
        // reference's "if 11 ... else if 12" priority explicit anyway
        int partner = s ^ 1;
        if (slot_on[partner] && partner < s)
        {
          bool overlap = true;
          for (int a = 0; a < 3; ++a)
            overlap = overlap && slot_box[s][0][a] < slot_box[partner][1][a]
                      && slot_box[partner][0][a] < slot_box[s][1][a];
          if (overlap)
            return "TF/SF slots overlap";
        }
        // the reference's isRevertVals: the correction lands on the far
        // neighbour for E in E_CENTERED and for H in H_CENTERED, and the
        // incident value is negated for H in E_CENTERED and for E in
        // H_CENTERED (InternalScheme.inc.h:1386-1835)
        const bool revert = isH == h_centered;
        TfsfTerm t;
        t.comp = k;
        t.slot = revert ? (s ^ 1) : s;
        t.inc_comp = s < 2 ? c.opp1 : c.opp2;
        const int *diffs[4] = {c.d11, c.d12, c.d21, c.d22};
        for (int a = 0; a < 3; ++a)
        {
          t.lo[a] = slot_box[s][0][a];
          t.hi[a] = slot_box[s][1][a];
          t.aux[a] = diffs[t.slot][a];
        }
        t.negate = isH != h_centered ? -1.0 : 1.0;
        if (!g.comp[t.inc_comp].exists)
          continue;
        g.tfsf.push_back (t);
      }
    }
  }
  return "";
}

std::vector<double> sigma_at (const Geometry &g, int k, int b)
{
  const std::vector<double> &s = g.sigma[b];
  int n = g.n[b];
  std::vector<double> out (n, 0.0);
  int a = k % 3;
  if (g.dmp)
  {
    // the eight fine cells span two fine cells on every kept axis, starting
    // at 2i + 1 where the component sits at i + 1.0 and at 2i where it sits
    // at i + 0.5; a sigma grid varies along one axis, so the reference's
    // eight-point average reduces to this pair exactly
    if ((g.drop >> b) & 1)
      return std::vector<double> (n, s[0]);
    const int shift = g.comp[k].min_fp[b] == 1.0 ? 1 : 0;
    for (int i = 0; i < n; ++i)
    {
      const int lo = 2 * i + shift;
      out[i] = lo + 1 < (int) s.size () ? (s[lo] + s[lo + 1]) / 2.0 : s[lo];
    }
    return out;
  }
  // sigma grids vary along one axis: the two-cell material average of an
  // edge component spans its own axis, the four-cell one the other two
  bool averaged = g.comp[k].nmat == 2 ? (b == a) : (b != a);
  if ((g.drop >> b) & 1)
    averaged = false;
  for (int i = 0; i < n; ++i)
    out[i] = (averaged && i + 1 < n) ? (s[i] + s[i + 1]) / 2.0 : s[i];
  return out;
}

double incident_source (const Geometry &g, uint32_t t)
{
  const double arg = g.dt * t * 2 * kPi * g.freq;
  return g.cfg.source_phase ? std::cos (arg) : std::sin (arg);
}

double point_source (const Geometry &g, uint32_t t, bool h)
{
  double ts = t + (h ? 1.0 : 0.5);
  if (g.cfg.point_source_kind == FDTD_SOURCE_GAUSSIAN)
  {
    // Gaussian-modulated pulse: spectral FWHM = bandwidth * f
    double w = 4.0 * std::sqrt (std::log (2.0)) / (kPi * g.freq * g.cfg.point_source_bandwidth);
    double tau = g.dt * ts - 3.0 * w;
    const double carrier = g.cfg.source_phase ? std::cos (2 * kPi * g.freq * tau) : std::sin (2 * kPi * g.freq * tau);
    return std::exp (-(tau / w) * (tau / w)) * carrier;
  }
  const double arg = g.dt * ts * 2 * kPi * g.freq;
  return g.cfg.source_phase ? std::cos (arg) : std::sin (arg);
}

// Scheme.inc.h:1228-1236: the component's time (t on E, t + 1/2 on H), the
// real build's sin or the complex build's cos(w (t - 1)) - i sin(w (t - 1)),
// times mu0 / dt / 2 (mu0 for J as for M, as the reference has it).
double current_source (const Geometry &g, uint32_t t, bool h)
{
  const double ts = h ? t + 0.5 : (double) t;
  double s;
  if (g.cfg.current_phase == 0)
    s = std::sin (g.dt * ts * 2.0 * kPi * g.freq);
  else if (g.cfg.current_phase == 1)
    s = std::cos (g.dt * (ts - 1) * 2.0 * kPi * g.freq);
  else
    s = -std::sin (g.dt * (ts - 1) * 2.0 * kPi * g.freq);
  return s * kMu0 / g.dt / 2.0;
}

}  // namespace fdtdb
