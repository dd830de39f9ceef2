/*
 * fdtd_oracle.c - CPU restatement of the fdtd3d leapfrog time step.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product.  Compiled with
 * -ffp-contract=off so every multiply and add rounds separately, in the order
 * the reference writes them.  References are to zer011b/fdtd3d source files.
 *
 * Scope: E_CENTERED layout, modes Dim3 and Dim2_TMz, real FP64 fields.
 *
 *   time loop ...................... Source/Scheme/Scheme.inc.h:28-473
 *   t > 0 guard .................... Source/Scheme/Scheme.inc.h:1032
 *   curl update (calcField) ........ Source/Scheme/InternalScheme.inc.h:766-772, 2351-2417
 *   PML E from D (calcFieldFromDOrB)  InternalScheme.inc.h:783-787, 2551-2640
 *   Drude ADE (calcFieldDrude) ..... InternalScheme.inc.h:775-780, 2452-2549
 *   Ca/Cb .......................... InternalScheme.inc.h:2297-2349
 *   TF/SF correction ............... InternalScheme.inc.h:1386-1835
 *   incident interpolation ......... InternalScheme.inc.h:500-515;
 *                                    Source/Scheme/InternalScheme.cpp:293-324
 *   incident 1-D grid steps ........ InternalScheme.inc.h:3276-3357
 *   point source ................... InternalScheme.inc.h:2818-2895
 *   dt, frequency, phase velocity .. InternalScheme.inc.h:3359-3394;
 *                                    Source/Layout/Approximation.cpp:259-359
 *   material averaging ............. Source/Layout/YeeGridLayout.h:655-1041;
 *                                    Source/Layout/Approximation.cpp:35-130
 *   sigma profiles ................. Source/Scheme/SchemeHelper.h:574-718
 *   Yee offsets, circuit diffs ..... Source/Layout/YeeGridLayout.cpp:1937-1990
 *   TF/SF predicates ............... YeeGridLayout.h:498-512, YeeGridLayout.cpp:257-1720
 *   incident projections ........... YeeGridLayout.h:2227-2357
 *   zeroIncCoordFP ................. YeeGridLayout.cpp:2600-2660
 *   time-level rotation ............ Source/Grid/Grid.h:1304-1319
 *   constants ...................... Source/Physics/PhysicsConst.h:28-32
 */
#include "fdtd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.14159265358979323846
#define ORC_C 299792458.0
#define ORC_MU0 (4 * ORC_PI * 0.0000001)
#define ORC_EPS0 (1 / (ORC_MU0 * (ORC_C * ORC_C)))
#define ORC_FPEXACT 0.0000001
#define ORC_APPROX_ACC 0.0000001

enum { EX, EY, EZ, HX, HY, HZ };
enum { DIR_L, DIR_R, DIR_D, DIR_U, DIR_B, DIR_F, DIR_NONE };

/* one axis test of a TF/SF border predicate (YeeGridLayoutHelper::tfsfBorder) */
enum { T_ANY, T_EXL, T_EXR, T_RANGE };
typedef struct { int kind; int o1; int o2; } axis_test;
typedef struct { int valid; axis_test ax[3]; } border_pred;

typedef struct
{
  int exists;
  double min_fp[3];          /* minimum real coordinate (Yee offset) */
  int opp1, opp2;            /* opposite components (-1 = absent) */
  int d11[3], d12[3], d21[3], d22[3];
  int dir11, dir12, dir21, dir22;
  int sig_cacb, sig4, sig5;  /* sigma axes for Ca/Cb, material4, material5 */
  int nmat;                  /* 2- or 4-point material average */
  int m[4][3];               /* material offsets 11, 12, 21, 22 */
  border_pred pred[6];       /* by direction L R D U B F */
} comp_desc;

struct fdtd_oracle
{
  fdtd_oracle_cfg cfg;
  int nx, ny, nz;
  size_t n;
  int levels;
  double dt, freq, rpv, dx;
  double a1, a2, a3;
  double s1, c1, s2, c2;
  double proj[6];
  double zero_inc[3];
  double left_fp[3], right_fp[3];
  comp_desc comp[6];
  double *f[6][3];           /* fields E/H */
  double *d[6][3];           /* D/B (PML) */
  double *d1[6][3];          /* D1/B1 (metamaterials) */
  double *mat[6];            /* eps mu omegape omegapm gammae gammam */
  double *sig1d[3];          /* sigma profiles along x, y, z */
  int inc_len;
  double *einc[2], *hinc[2];
};

static size_t idx (const struct fdtd_oracle *o, int x, int y, int z)
{
  return ((size_t) x * o->ny + y) * o->nz + z;
}

static int is_fp_exact (double a, double b)
{
  return ((a > b ? a - b : b - a) < ORC_FPEXACT);
}

static void set3 (int *v, int a, int b, int c) { v[0] = a; v[1] = b; v[2] = c; }

/* ------------------------------------------------------------------------- */
/* phase velocity: Approximation.cpp:259-359                                 */

static double approximate_wave_number_general (double delta, double lambda, double courant,
                                               double n_lambda, double a1, double a2)
{
  double k = 2 * ORC_PI;
  double k_prev = k + 2 * sqrt (ORC_APPROX_ACC);
  double nd = delta / lambda;
  double A = nd * sin (a1) * cos (a2) / 2;
  double B = nd * sin (a1) * sin (a2) / 2;
  double C = nd * cos (a1) / 2;
  double sq = sin (ORC_PI * courant / n_lambda);
  double D = (sq * sq) / (courant * courant);
  while ((k_prev - k) * (k_prev - k) >= ORC_APPROX_ACC)
  {
    k_prev = k;
    double sa = sin (A * k), sb = sin (B * k), sc = sin (C * k);
    double diff1 = sa * sa + sb * sb + sc * sc - D;
    double diff2 = A * sin (2 * A * k) + B * sin (2 * B * k) + C * sin (2 * C * k);
    double diff = diff1 / diff2;
    k -= diff;
  }
  return k / lambda;
}

static int is_axis_angle (double a)
{
  return a == 0 || a == ORC_PI / 2 || a == ORC_PI || a == 3 * ORC_PI / 2;
}

static int is_diag_angle (double a)
{
  return a == ORC_PI / 4 || a == 3 * ORC_PI / 4 || a == 5 * ORC_PI / 4 || a == 7 * ORC_PI / 4;
}

static double approximate_wave_number (double delta, double lambda, double courant,
                                       double n_lambda, double a1, double a2)
{
  if (is_axis_angle (a1) && is_axis_angle (a2))
  {
    return 2.0 / delta * asin (sin (ORC_PI * courant / n_lambda) / courant);
  }
  if ((is_axis_angle (a1) && is_diag_angle (a2)) || (is_diag_angle (a1) && is_axis_angle (a2)))
  {
    return 2.0 * sqrt (2.0) / delta * asin (sin (ORC_PI * courant / n_lambda) / (courant * sqrt (2.0)));
  }
  return approximate_wave_number_general (delta, lambda, courant, n_lambda, a1, a2);
}

static double phase_velocity (double delta, double lambda, double courant, double n_lambda,
                              double a1, double a2)
{
  return ORC_C * 2 * ORC_PI / lambda
         / approximate_wave_number (delta, lambda, courant, n_lambda, a1, a2);
}

/* ------------------------------------------------------------------------- */
/* sigma profiles: SchemeHelper.h:574-718                                    */

static double sigma_value (double dist, double boundary, double grid_step)
{
  double eps0 = ORC_EPS0;
  double mu0 = ORC_MU0;
  uint32_t exponent = 6;
  double r_err = 1e-16;
  double sigma_max_1 = -log (r_err) * (exponent + 1.0) / (2.0 * sqrt (mu0 / eps0) * boundary);
  double boundary_factor = sigma_max_1 / (grid_step * (pow (boundary, exponent)) * (exponent + 1));
  double x1 = (dist + 1) * grid_step;
  double x2 = dist * grid_step;
  return boundary_factor * (pow (x1, (exponent + 1)) - pow (x2, (exponent + 1)));
}

/* axis 0 keeps a fractional distance against size; axes 1 and 2 truncate it
 * and compare against size + 0.5 (initSigmaX vs initSigmaY/Z) */
static void build_sigma (double *out, int axis, int n, int pml, double dx)
{
  double p = (double) pml;
  double boundary = p * dx;
  for (int i = 0; i < n; ++i)
  {
    double pos = i + 0.5;
    double val = 0;
    if (axis == 0)
    {
      double size = (double) n;
      if (pos < p)
      {
        val = sigma_value (p - pos, boundary, dx);
      }
      else if (pos >= size - p)
      {
        val = sigma_value (pos - (size - p), boundary, dx);
      }
    }
    else
    {
      double size = n + 0.5;
      if (pos < p)
      {
        int dist = (int) (p - pos);
        val = sigma_value (dist, boundary, dx);
      }
      else if (pos >= size - p)
      {
        int dist = (int) (pos - (size - p));
        val = sigma_value (dist, boundary, dx);
      }
    }
    out[i] = val;
  }
}

/* ------------------------------------------------------------------------- */
/* layout tables                                                             */

static void pred_set (border_pred *p, int k0, int a0, int b0, int k1, int a1, int b1,
                      int k2, int a2, int b2)
{
  p->valid = 1;
  p->ax[0].kind = k0; p->ax[0].o1 = a0; p->ax[0].o2 = b0;
  p->ax[1].kind = k1; p->ax[1].o1 = a1; p->ax[1].o2 = b1;
  p->ax[2].kind = k2; p->ax[2].o1 = a2; p->ax[2].o2 = b2;
}

/* Dim3 E_CENTERED circuit diffs (YeeGridLayout.cpp:1937-1960) and TF/SF
 * predicates (YeeGridLayout.cpp:272, 558, 844, 1130, 1416, 1702); Dim2_TMz
 * predicates (YeeGridLayout.cpp:817, 1103, 1389) are the same tests with the
 * z axis dropped. */
static void init_layout (struct fdtd_oracle *o)
{
  comp_desc *c;
  int tmz = o->cfg.mode == 2;
  memset (o->comp, 0, sizeof (o->comp));

  for (int k = 0; k < 6; ++k)
  {
    int a = k % 3;
    int isH = k >= 3;
    c = &o->comp[k];
    for (int ax = 0; ax < 3; ++ax)
    {
      c->min_fp[ax] = isH ? (ax == a ? 0.5 : 1.0) : (ax == a ? 1.0 : 0.5);
    }
    c->sig_cacb = (a + 1) % 3;
    c->sig4 = a;
    c->sig5 = (a + 2) % 3;
    memset (c->m, 0, sizeof (c->m));
    if (!isH)
    {
      c->nmat = 2;
      c->m[1][a] = 1;
    }
    else
    {
      int lo = a == 0 ? 1 : 0;
      int hi = a == 2 ? 1 : 2;
      c->nmat = 4;
      c->m[1][hi] = 1;
      c->m[2][lo] = 1;
      c->m[3][lo] = 1;
      c->m[3][hi] = 1;
    }
    c->dir11 = c->dir12 = c->dir21 = c->dir22 = DIR_NONE;
  }

  /* Ex */
  c = &o->comp[EX];
  c->opp1 = HZ; c->opp2 = HY;
  set3 (c->d11, 0, -1, 0); set3 (c->d12, 0, 0, 0); set3 (c->d21, 0, 0, -1); set3 (c->d22, 0, 0, 0);
  c->dir11 = DIR_D; c->dir12 = DIR_U; c->dir21 = DIR_B; c->dir22 = DIR_F;
  pred_set (&c->pred[DIR_D], T_RANGE, -1, 1, T_EXL, -5, 0, T_RANGE, 4, -4);
  pred_set (&c->pred[DIR_U], T_RANGE, -1, 1, T_EXR, 5, 0, T_RANGE, 4, -4);
  pred_set (&c->pred[DIR_B], T_RANGE, -1, 1, T_RANGE, 4, -4, T_EXL, -5, 0);
  pred_set (&c->pred[DIR_F], T_RANGE, -1, 1, T_RANGE, 4, -4, T_EXR, 5, 0);
  /* Ey */
  c = &o->comp[EY];
  c->opp1 = HX; c->opp2 = HZ;
  set3 (c->d11, 0, 0, -1); set3 (c->d12, 0, 0, 0); set3 (c->d21, -1, 0, 0); set3 (c->d22, 0, 0, 0);
  c->dir11 = DIR_B; c->dir12 = DIR_F; c->dir21 = DIR_L; c->dir22 = DIR_R;
  pred_set (&c->pred[DIR_L], T_EXL, -5, 0, T_RANGE, -1, 1, T_RANGE, 4, -4);
  pred_set (&c->pred[DIR_R], T_EXR, 5, 0, T_RANGE, -1, 1, T_RANGE, 4, -4);
  pred_set (&c->pred[DIR_B], T_RANGE, 4, -4, T_RANGE, -1, 1, T_EXL, -5, 0);
  pred_set (&c->pred[DIR_F], T_RANGE, 4, -4, T_RANGE, -1, 1, T_EXR, 5, 0);
  /* Ez */
  c = &o->comp[EZ];
  c->opp1 = HY; c->opp2 = HX;
  set3 (c->d11, -1, 0, 0); set3 (c->d12, 0, 0, 0); set3 (c->d21, 0, -1, 0); set3 (c->d22, 0, 0, 0);
  c->dir11 = DIR_L; c->dir12 = DIR_R; c->dir21 = DIR_D; c->dir22 = DIR_U;
  pred_set (&c->pred[DIR_L], T_EXL, -5, 0, T_RANGE, 4, -4, T_RANGE, -1, 1);
  pred_set (&c->pred[DIR_R], T_EXR, 5, 0, T_RANGE, 4, -4, T_RANGE, -1, 1);
  pred_set (&c->pred[DIR_D], T_RANGE, 4, -4, T_EXL, -5, 0, T_RANGE, -1, 1);
  pred_set (&c->pred[DIR_U], T_RANGE, 4, -4, T_EXR, 5, 0, T_RANGE, -1, 1);
  /* Hx */
  c = &o->comp[HX];
  c->opp1 = EY; c->opp2 = EZ;
  set3 (c->d11, 0, 0, 0); set3 (c->d12, 0, 0, 1); set3 (c->d21, 0, 0, 0); set3 (c->d22, 0, 1, 0);
  c->dir11 = DIR_B; c->dir12 = DIR_F; c->dir21 = DIR_D; c->dir22 = DIR_U;
  pred_set (&c->pred[DIR_D], T_RANGE, 4, -4, T_EXL, 0, 0, T_RANGE, -1, 1);
  pred_set (&c->pred[DIR_U], T_RANGE, 4, -4, T_EXR, 0, 0, T_RANGE, -1, 1);
  pred_set (&c->pred[DIR_B], T_RANGE, 4, -4, T_RANGE, -1, 1, T_EXL, 0, 0);
  pred_set (&c->pred[DIR_F], T_RANGE, 4, -4, T_RANGE, -1, 1, T_EXR, 0, 0);
  /* Hy */
  c = &o->comp[HY];
  c->opp1 = EZ; c->opp2 = EX;
  set3 (c->d11, 0, 0, 0); set3 (c->d12, 1, 0, 0); set3 (c->d21, 0, 0, 0); set3 (c->d22, 0, 0, 1);
  c->dir11 = DIR_L; c->dir12 = DIR_R; c->dir21 = DIR_B; c->dir22 = DIR_F;
  pred_set (&c->pred[DIR_L], T_EXL, 0, 0, T_RANGE, 4, -4, T_RANGE, -1, 1);
  pred_set (&c->pred[DIR_R], T_EXR, 0, 0, T_RANGE, 4, -4, T_RANGE, -1, 1);
  pred_set (&c->pred[DIR_B], T_RANGE, -1, 1, T_RANGE, 4, -4, T_EXL, 0, 0);
  pred_set (&c->pred[DIR_F], T_RANGE, -1, 1, T_RANGE, 4, -4, T_EXR, 0, 0);
  /* Hz */
  c = &o->comp[HZ];
  c->opp1 = EX; c->opp2 = EY;
  set3 (c->d11, 0, 0, 0); set3 (c->d12, 0, 1, 0); set3 (c->d21, 0, 0, 0); set3 (c->d22, 1, 0, 0);
  c->dir11 = DIR_D; c->dir12 = DIR_U; c->dir21 = DIR_L; c->dir22 = DIR_R;
  pred_set (&c->pred[DIR_L], T_EXL, 0, 0, T_RANGE, -1, 1, T_RANGE, 4, -4);
  pred_set (&c->pred[DIR_R], T_EXR, 0, 0, T_RANGE, -1, 1, T_RANGE, 4, -4);
  pred_set (&c->pred[DIR_D], T_RANGE, -1, 1, T_EXL, 0, 0, T_RANGE, 4, -4);
  pred_set (&c->pred[DIR_U], T_RANGE, -1, 1, T_EXR, 0, 0, T_RANGE, 4, -4);

  for (int k = 0; k < 6; ++k)
  {
    o->comp[k].exists = tmz ? (k == EZ || k == HX || k == HY) : 1;
  }
  if (tmz)
  {
    /* 2-D: z offsets vanish and z tests are dropped */
    for (int k = 0; k < 6; ++k)
    {
      c = &o->comp[k];
      c->d11[2] = c->d12[2] = c->d21[2] = c->d22[2] = 0;
      for (int j = 0; j < 4; ++j)
      {
        c->m[j][2] = 0;
      }
      for (int dd = 0; dd < 6; ++dd)
      {
        c->pred[dd].ax[2].kind = T_ANY;
      }
      c->pred[DIR_B].valid = 0;
      c->pred[DIR_F].valid = 0;
    }
  }
}

static int axis_ok (const struct fdtd_oracle *o, const axis_test *t, int ax, double coord)
{
  switch (t->kind)
  {
    case T_ANY:
      return 1;
    case T_EXL:
      return is_fp_exact (coord, o->left_fp[ax] + t->o1 * 1.0 / 10.0);
    case T_EXR:
      return is_fp_exact (coord, o->right_fp[ax] + t->o1 * 1.0 / 10.0);
    default:
      return coord > o->left_fp[ax] + t->o1 * 1.0 / 10.0
             && coord < o->right_fp[ax] + t->o2 * 1.0 / 10.0;
  }
}

static int need_update (const struct fdtd_oracle *o, int k, int dir, int x, int y, int z)
{
  if (dir == DIR_NONE)
  {
    return 0;
  }
  const border_pred *p = &o->comp[k].pred[dir];
  if (!p->valid)
  {
    return 0;
  }
  int pos[3] = { x, y, z };
  for (int ax = 0; ax < 3; ++ax)
  {
    double coord = pos[ax] + o->comp[k].min_fp[ax];
    if (!axis_ok (o, &p->ax[ax], ax, coord))
    {
      return 0;
    }
  }
  return 1;
}

/* incident value at the real coordinate of component k at cell pos */
static double incident_at (const struct fdtd_oracle *o, int k, const int *pos)
{
  const comp_desc *c = &o->comp[k];
  int isH = k >= 3;
  double d_diff = isH ? 0.5 : 0.0;
  double d;
  if (o->cfg.mode == 3)
  {
    double x = (pos[0] + c->min_fp[0]) - o->zero_inc[0];
    double y = (pos[1] + c->min_fp[1]) - o->zero_inc[1];
    double z = (pos[2] + c->min_fp[2]) - o->zero_inc[2];
    d = x * o->s1 * o->c2 + y * o->s1 * o->s2 + z * o->c1 - d_diff;
  }
  else
  {
    double x = (pos[0] + c->min_fp[0]) - o->zero_inc[0];
    double y = (pos[1] + c->min_fp[1]) - o->zero_inc[1];
    d = x * o->c2 + y * o->s2 - d_diff;
  }
  const double *inc = isH ? o->hinc[1] : o->einc[1];
  double coord_d1 = (double) ((int32_t) d);
  double coord_d2 = coord_d1 + 1;
  double prop_d2 = d - coord_d1;
  double prop_d1 = 1 - prop_d2;
  int32_t i1 = (int32_t) coord_d1;
  int32_t i2 = (int32_t) coord_d2;
  double v = inc[i1] * prop_d1 + inc[i2] * prop_d2;
  if (o->cfg.mode == 2 && k == EZ)
  {
    return v;
  }
  if (o->cfg.mode == 3 && k == HZ)
  {
    return -v * o->proj[HZ];
  }
  return v * o->proj[k];
}

static double material_avg (const struct fdtd_oracle *o, const double *m, int k, int x, int y, int z)
{
  const comp_desc *c = &o->comp[k];
  double v[4];
  for (int j = 0; j < c->nmat; ++j)
  {
    v[j] = m[idx (o, x + c->m[j][0], y + c->m[j][1], z + c->m[j][2])];
  }
  if (c->nmat == 2)
  {
    return (v[0] + v[1]) / 2.0;
  }
  return ((v[0] + v[1]) / 2.0 + (v[2] + v[3]) / 2.0) / 2.0;
}

static double sigma_avg (const struct fdtd_oracle *o, int axis, int k, int x, int y, int z)
{
  const comp_desc *c = &o->comp[k];
  double v[4];
  for (int j = 0; j < c->nmat; ++j)
  {
    int p[3] = { x + c->m[j][0], y + c->m[j][1], z + c->m[j][2] };
    v[j] = o->sig1d[axis][p[axis]];
  }
  if (c->nmat == 2)
  {
    return (v[0] + v[1]) / 2.0;
  }
  return ((v[0] + v[1]) / 2.0 + (v[2] + v[3]) / 2.0) / 2.0;
}

static int has_sigma (const struct fdtd_oracle *o, int axis)
{
  return o->cfg.mode == 3 || axis != 2;
}

/* ------------------------------------------------------------------------- */

static double *zalloc (size_t n)
{
  return (double *) calloc (n, sizeof (double));
}

fdtd_oracle *fdtd_oracle_create (const fdtd_oracle_cfg *cfg, const double *const materials[6])
{
  struct fdtd_oracle *o = (struct fdtd_oracle *) calloc (1, sizeof (struct fdtd_oracle));
  if (!o)
  {
    return NULL;
  }
  o->cfg = *cfg;
  o->nx = cfg->size[0];
  o->ny = cfg->size[1];
  o->nz = cfg->mode == 2 ? 1 : cfg->size[2];
  o->n = (size_t) o->nx * o->ny * o->nz;
  o->levels = (cfg->use_metamaterials && cfg->use_pml) ? 3 : 2;
  o->dx = cfg->dx;

  /* InternalScheme::initScheme */
  o->freq = ORC_C / cfg->wavelength;
  o->dt = cfg->dx * cfg->courant / ORC_C;
  o->a1 = cfg->angle_teta * ORC_PI / 180.0;
  o->a2 = cfg->angle_phi * ORC_PI / 180.0;
  o->a3 = cfg->angle_psi * ORC_PI / 180.0;
  {
    double n_lambda = cfg->wavelength / cfg->dx;
    double pv0 = phase_velocity (cfg->dx, cfg->wavelength, cfg->courant, n_lambda, ORC_PI / 2, 0);
    double pv = phase_velocity (cfg->dx, cfg->wavelength, cfg->courant, n_lambda, o->a1, o->a2);
    o->rpv = pv0 / pv;
  }
  o->s1 = sin (o->a1); o->c1 = cos (o->a1);
  o->s2 = sin (o->a2); o->c2 = cos (o->a2);
  {
    double s3 = sin (o->a3), c3 = cos (o->a3);
    double s1 = o->s1, c1 = o->c1, s2 = o->s2, c2 = o->c2;
    if (cfg->mode == 3)
    {
      o->proj[EX] = c3 * s2 - s3 * c1 * c2;
      o->proj[EY] = -c3 * c2 - s3 * c1 * s2;
      o->proj[EZ] = s3 * s1;
      o->proj[HX] = s3 * s2 + c3 * c1 * c2;
      o->proj[HY] = -s3 * c2 + c3 * c1 * s2;
      o->proj[HZ] = c3 * s1;
      o->zero_inc[0] = cfg->tfsf_left[0] - 2.5 * sin (o->a1) * cos (o->a2);
      o->zero_inc[1] = cfg->tfsf_left[1] - 2.5 * sin (o->a1) * sin (o->a2);
      o->zero_inc[2] = cfg->tfsf_left[2] - 2.5 * cos (o->a1);
    }
    else
    {
      o->proj[EZ] = 1.0;
      o->proj[HX] = sin (o->a2);
      o->proj[HY] = -cos (o->a2);
      o->zero_inc[0] = cfg->tfsf_left[0] - 2.5 * cos (o->a2);
      o->zero_inc[1] = cfg->tfsf_left[1] - 2.5 * sin (o->a2);
      o->zero_inc[2] = 0;
    }
  }
  int sz[3] = { o->nx, o->ny, o->nz };
  for (int ax = 0; ax < 3; ++ax)
  {
    o->left_fp[ax] = 0.0 + (double) cfg->tfsf_left[ax];
    o->right_fp[ax] = 0.0 + (double) (sz[ax] - cfg->tfsf_right[ax]);
  }
  init_layout (o);

  static const double defaults[6] = { 1, 1, 0, 0, 0, 0 };
  for (int m = 0; m < 6; ++m)
  {
    o->mat[m] = zalloc (o->n);
    for (size_t i = 0; i < o->n; ++i)
    {
      o->mat[m][i] = (materials && materials[m]) ? materials[m][i] : defaults[m];
    }
  }
  for (int ax = 0; ax < 3; ++ax)
  {
    o->sig1d[ax] = zalloc (sz[ax]);
    if (cfg->use_pml && has_sigma (o, ax))
    {
      build_sigma (o->sig1d[ax], ax, sz[ax], cfg->pml[ax], cfg->dx);
    }
  }
  for (int k = 0; k < 6; ++k)
  {
    if (!o->comp[k].exists)
    {
      continue;
    }
    for (int l = 0; l < o->levels; ++l)
    {
      o->f[k][l] = zalloc (o->n);
      if (cfg->use_pml)
      {
        o->d[k][l] = zalloc (o->n);
      }
      if (cfg->use_metamaterials)
      {
        o->d1[k][l] = zalloc (o->n);
      }
    }
  }
  o->inc_len = 500 * o->nx;
  for (int l = 0; l < 2; ++l)
  {
    o->einc[l] = zalloc (o->inc_len);
    o->hinc[l] = zalloc (o->inc_len);
  }
  return o;
}

void fdtd_oracle_destroy (fdtd_oracle *o)
{
  if (!o)
  {
    return;
  }
  for (int k = 0; k < 6; ++k)
  {
    for (int l = 0; l < 3; ++l)
    {
      free (o->f[k][l]);
      free (o->d[k][l]);
      free (o->d1[k][l]);
    }
    free (o->mat[k]);
  }
  for (int ax = 0; ax < 3; ++ax)
  {
    free (o->sig1d[ax]);
  }
  for (int l = 0; l < 2; ++l)
  {
    free (o->einc[l]);
    free (o->hinc[l]);
  }
  free (o);
}

/* Grid::shiftInTime: the oldest level becomes the new current one */
static void shift_levels (double **lv, int levels)
{
  double *oldest = lv[levels - 1];
  for (int i = levels - 1; i >= 1; --i)
  {
    lv[i] = lv[i - 1];
  }
  lv[0] = oldest;
}

static double value_at (const struct fdtd_oracle *o, int k, int x, int y, int z)
{
  return o->f[k][1][idx (o, x, y, z)];
}

/* curl step of component k at one cell (calculateFieldStepIteration) */
static void curl_cell (struct fdtd_oracle *o, int k, int x, int y, int z)
{
  const comp_desc *c = &o->comp[k];
  int isH = k >= 3;
  int use_pml = o->cfg.use_pml;
  double **grid = use_pml ? o->d[k] : o->f[k];
  size_t id = idx (o, x, y, z);
  double val = grid[1][id];
  double ca, cb;
  if (use_pml)
  {
    double material = has_sigma (o, c->sig_cacb) ? sigma_avg (o, c->sig_cacb, k, x, y, z) : 0;
    double eps0 = ORC_EPS0;
    double dd = (2 * eps0 * 1.0 + material * o->dt);
    ca = (2 * eps0 * 1.0 - material * o->dt) / dd;
    cb = (2 * eps0 * o->dt / o->dx) / dd;
  }
  else
  {
    double material = material_avg (o, isH ? o->mat[1] : o->mat[0], k, x, y, z);
    double modifier = isH ? ORC_MU0 : ORC_EPS0;
    ca = 1.0;
    cb = o->dt / (material * modifier * o->dx);
  }
  double p11 = 0, p12 = 0, p21 = 0, p22 = 0;
  int pos11[3] = { x + c->d11[0], y + c->d11[1], z + c->d11[2] };
  int pos12[3] = { x + c->d12[0], y + c->d12[1], z + c->d12[2] };
  int pos21[3] = { x + c->d21[0], y + c->d21[1], z + c->d21[2] };
  int pos22[3] = { x + c->d22[0], y + c->d22[1], z + c->d22[2] };
  if (o->comp[c->opp1].exists)
  {
    p11 = value_at (o, c->opp1, pos11[0], pos11[1], pos11[2]);
    p12 = value_at (o, c->opp1, pos12[0], pos12[1], pos12[2]);
  }
  if (o->comp[c->opp2].exists)
  {
    p21 = value_at (o, c->opp2, pos21[0], pos21[1], pos21[2]);
    p22 = value_at (o, c->opp2, pos22[0], pos22[1], pos22[2]);
  }
  if (o->cfg.use_tfsf)
  {
    int u11 = need_update (o, k, c->dir11, x, y, z);
    int u12 = need_update (o, k, c->dir12, x, y, z);
    int u21 = need_update (o, k, c->dir21, x, y, z);
    int u22 = need_update (o, k, c->dir22, x, y, z);
    int revert = !isH;
    double diff1 = 0, diff2 = 0;
    if (u11 || u12)
    {
      const int *aux = revert ? (u11 ? pos12 : pos11) : (u11 ? pos11 : pos12);
      diff1 = incident_at (o, c->opp1, aux);
      if (isH)
      {
        diff1 *= -1.0;
      }
    }
    if (u21 || u22)
    {
      const int *aux = revert ? (u21 ? pos22 : pos21) : (u21 ? pos21 : pos22);
      diff2 = incident_at (o, c->opp2, aux);
      if (isH)
      {
        diff2 *= -1.0;
      }
    }
    if (revert)
    {
      if (u11) p12 -= diff1; else if (u12) p11 -= diff1;
      if (u21) p22 -= diff2; else if (u22) p21 -= diff2;
    }
    else
    {
      if (u11) p11 -= diff1; else if (u12) p12 -= diff1;
      if (u21) p21 -= diff2; else if (u22) p22 -= diff2;
    }
  }
  double tmp = p12 - p11 - p22 + p21 - 0.0 * o->dx;
  grid[0][id] = val * ca + tmp * cb;
}

/* Drude ADE at one cell (calculateFieldStepIterationPMLMetamaterials) */
static void drude_cell (struct fdtd_oracle *o, int k, int x, int y, int z)
{
  int isH = k >= 3;
  size_t id = idx (o, x, y, z);
  double cur = o->d[k][0][id], prev = o->d[k][1][id], pprev = o->d[k][2][id];
  double prev1 = o->d1[k][1][id], pprev1 = o->d1[k][2][id];
  double material = material_avg (o, isH ? o->mat[1] : o->mat[0], k, x, y, z);
  double omega = material_avg (o, isH ? o->mat[3] : o->mat[2], k, x, y, z);
  double gamma = material_avg (o, isH ? o->mat[5] : o->mat[4], k, x, y, z);
  /* 4-point Drude averaging divides the sum of four by 4.0 */
  if (o->comp[k].nmat == 4)
  {
    const comp_desc *c = &o->comp[k];
    const double *om = isH ? o->mat[3] : o->mat[2];
    const double *ga = isH ? o->mat[5] : o->mat[4];
    double w[4], g[4];
    for (int j = 0; j < 4; ++j)
    {
      size_t q = idx (o, x + c->m[j][0], y + c->m[j][1], z + c->m[j][2]);
      w[j] = om[q];
      g[j] = ga[q];
    }
    omega = (w[0] + w[1] + w[2] + w[3]) / 4.0;
    gamma = (g[0] + g[1] + g[2] + g[3]) / 4.0;
  }
  double mm = isH ? ORC_MU0 : ORC_EPS0;
  double dt = o->dt;
  double sq = dt * omega;
  double A = 4 * mm * material + 2 * dt * mm * material * gamma + mm * (sq * sq);
  double b0 = (4 + 2 * dt * gamma) / A;
  double b1 = -8 / A;
  double b2 = (4 - 2 * dt * gamma) / A;
  double a1 = (2 * mm * (sq * sq) - 8 * mm * material) / A;
  double a2 = (4 * mm * material - 2 * dt * mm * material * gamma + mm * (sq * sq)) / A;
  o->d1[k][0][id] = cur * b0 + prev * b1 + pprev * b2 - prev1 * a1 - pprev1 * a2;
}

/* E (H) from D (B) at one cell (calculateFieldStepIterationPML) */
static void pml_cell (struct fdtd_oracle *o, int k, int x, int y, int z)
{
  int isH = k >= 3;
  const comp_desc *c = &o->comp[k];
  size_t id = idx (o, x, y, z);
  double prev_eh = o->f[k][1][id];
  double **src = o->cfg.use_metamaterials ? o->d1[k] : o->d[k];
  double cur_db = src[0][id];
  double prev_db = src[1][id];
  double eps0 = ORC_EPS0;
  double material1 = material_avg (o, isH ? o->mat[1] : o->mat[0], k, x, y, z);
  double material4 = has_sigma (o, c->sig4) ? sigma_avg (o, c->sig4, k, x, y, z) : 0;
  double material5 = has_sigma (o, c->sig5) ? sigma_avg (o, c->sig5, k, x, y, z) : 0;
  double modifier = material1 * (isH ? ORC_MU0 : ORC_EPS0);
  if (o->cfg.use_metamaterials)
  {
    modifier = 1;
  }
  double dd = (2 * eps0 * 1.0 + material5 * o->dt);
  double ca = (2 * eps0 * 1.0 - material5 * o->dt) / dd;
  double cb = ((2 * eps0 * 1.0 + material4 * o->dt) / (modifier)) / dd;
  double cc = ((2 * eps0 * 1.0 - material4 * o->dt) / (modifier)) / dd;
  o->f[k][0][id] = prev_eh * ca + cur_db * cb - prev_db * cc;
}

static void field_half_step (struct fdtd_oracle *o, int k, uint32_t t)
{
  if (!o->comp[k].exists)
  {
    return;
  }
  int x1 = o->nx - 1, y1 = o->ny - 1;
  int z0 = o->cfg.mode == 3 ? 1 : 0;
  int z1 = o->cfg.mode == 3 ? o->nz - 1 : 1;
  if (t > 0 || !o->cfg.skip_first_update)
  {
    for (int x = 1; x < x1; ++x)
      for (int y = 1; y < y1; ++y)
        for (int z = z0; z < z1; ++z)
          curl_cell (o, k, x, y, z);
    if (o->cfg.use_pml)
    {
      if (o->cfg.use_metamaterials)
      {
        for (int x = 1; x < x1; ++x)
          for (int y = 1; y < y1; ++y)
            for (int z = z0; z < z1; ++z)
              drude_cell (o, k, x, y, z);
      }
      for (int x = 1; x < x1; ++x)
        for (int y = 1; y < y1; ++y)
          for (int z = z0; z < z1; ++z)
            pml_cell (o, k, x, y, z);
    }
  }
  if (o->cfg.point_source_mask & (1 << k))
  {
    const int *ps = o->cfg.point_source;
    int pz = o->cfg.mode == 3 ? ps[2] : 0;
    if (ps[0] >= 0 && ps[0] < o->nx && ps[1] >= 0 && ps[1] < o->ny && pz >= 0 && pz < o->nz)
    {
      double ts = t + (k >= 3 ? 1.0 : 0.5);
      double v;
      if (o->cfg.point_source_kind == 1)
      {
        /* project-defined Gaussian-modulated pulse (no reference counterpart) */
        double w = 4.0 * sqrt (log (2.0)) / (ORC_PI * o->freq * o->cfg.point_source_bandwidth);
        double tau = o->dt * ts - 3.0 * w;
        v = exp (-(tau / w) * (tau / w)) * sin (2 * ORC_PI * o->freq * tau);
      }
      else
      {
        v = sin (o->dt * ts * 2 * ORC_PI * o->freq);
      }
      o->f[k][0][idx (o, ps[0], ps[1], pz)] = v;
    }
  }
}

static void shift_component (struct fdtd_oracle *o, int k)
{
  if (!o->comp[k].exists)
  {
    return;
  }
  shift_levels (o->f[k], o->levels);
  if (o->cfg.use_pml)
  {
    shift_levels (o->d[k], o->levels);
  }
  if (o->cfg.use_metamaterials)
  {
    shift_levels (o->d1[k], o->levels);
  }
}

static void swap2 (double **p)
{
  double *t = p[0];
  p[0] = p[1];
  p[1] = t;
}

void fdtd_oracle_step (fdtd_oracle *o, uint32_t t_start, uint32_t n)
{
  double mod_e = o->dt / (o->rpv * ORC_EPS0 * o->dx);
  double mod_h = o->dt / (o->rpv * ORC_MU0 * o->dx);
  for (uint32_t t = t_start; t < t_start + n; ++t)
  {
    if (o->cfg.use_tfsf)
    {
      for (int i = 1; i < o->inc_len; ++i)
      {
        o->einc[0][i] = o->einc[1][i] + (o->hinc[1][i - 1] - o->hinc[1][i]) * mod_e;
      }
      o->einc[0][0] = sin (o->dt * t * 2 * ORC_PI * o->freq);
      swap2 (o->einc);
    }
    for (int k = EX; k <= EZ; ++k)
    {
      field_half_step (o, k, t);
    }
    for (int k = EX; k <= EZ; ++k)
    {
      shift_component (o, k);
    }
    if (o->cfg.use_tfsf)
    {
      for (int i = 0; i < o->inc_len - 1; ++i)
      {
        o->hinc[0][i] = o->hinc[1][i] + (o->einc[1][i] - o->einc[1][i + 1]) * mod_h;
      }
      swap2 (o->hinc);
    }
    for (int k = HX; k <= HZ; ++k)
    {
      field_half_step (o, k, t);
    }
    for (int k = HX; k <= HZ; ++k)
    {
      shift_component (o, k);
    }
  }
}

int fdtd_oracle_get (const fdtd_oracle *o, int c, int level, double *out)
{
  if (c < 0 || c > 5 || !o->comp[c].exists || level < 0 || level >= o->levels)
  {
    return -1;
  }
  memcpy (out, o->f[c][level], o->n * sizeof (double));
  return 0;
}

void fdtd_oracle_scalars (const fdtd_oracle *o, double out[3])
{
  out[0] = o->dt;
  out[1] = o->freq;
  out[2] = o->rpv;
}

void fdtd_oracle_incident (const fdtd_oracle *o, double *einc, double *hinc)
{
  if (einc)
  {
    memcpy (einc, o->einc[1], o->inc_len * sizeof (double));
  }
  if (hinc)
  {
    memcpy (hinc, o->hinc[1], o->inc_len * sizeof (double));
  }
}

/* ------------------------------------------------------------------------- */
/* 1-D ExHy with the unit-test driver: Source/UnitTests/unit-test-internalscheme.cpp:42-841,
 * layout Dim1_ExHy along z (YeeGridLayout.cpp:30-40, 1176-1185, 2062;
 * YeeGridLayout.h:1250-1311; InternalScheme.cpp:114-124).                  */

static void exhy_run (int size, int tfsf, double dx, double lambda, double courant,
                      uint32_t steps, int cosine, double *ex_out)
{
  double freq = ORC_C / lambda;
  double dt = dx * courant / ORC_C;
  double n_lambda = lambda / dx;
  double pv0 = phase_velocity (dx, lambda, courant, n_lambda, ORC_PI / 2, 0);
  double pv = phase_velocity (dx, lambda, courant, n_lambda, 0 * ORC_PI / 180.0, 0 * ORC_PI / 180.0);
  double rpv = pv0 / pv;
  int inc_len = 500 * size;
  double *ex[2], *hy[2], *einc[2], *hinc[2];
  for (int l = 0; l < 2; ++l)
  {
    ex[l] = zalloc (size);
    hy[l] = zalloc (size);
    einc[l] = zalloc (inc_len);
    hinc[l] = zalloc (inc_len);
  }
  double left = tfsf, right = size - tfsf;
  double zero_inc = tfsf - 2.5;
  double cb_e = dt / (((1.0 + 1.0) / 2.0) * ORC_EPS0 * dx);
  double cb_h = dt / (((1.0 + 1.0) / 2.0) * ORC_MU0 * dx);
  double mod_e = dt / (rpv * ORC_EPS0 * dx);
  double mod_h = dt / (rpv * ORC_MU0 * dx);
  for (uint32_t t = 0; t < steps; ++t)
  {
    for (int i = 1; i < inc_len; ++i)
    {
      einc[0][i] = einc[1][i] + (hinc[1][i - 1] - hinc[1][i]) * mod_e;
    }
    double arg = dt * t * 2 * ORC_PI * freq;
    einc[0][0] = cosine ? cos (arg) : sin (arg);
    swap2 (einc);
    for (int k = 1; k < size - 1; ++k)
    {
      double p21 = hy[1][k - 1], p22 = hy[1][k];
      double c = k + 0.5;
      int back = is_fp_exact (c, left + -5 * 1.0 / 10.0);
      int front = is_fp_exact (c, right + 5 * 1.0 / 10.0);
      if (back || front)
      {
        int aux = back ? k : k - 1;
        double d = ((aux + 1.0) - zero_inc) - 0.5;
        double d1 = (double) ((int32_t) d);
        double pr2 = d - d1, pr1 = 1 - pr2;
        double v = hinc[1][(int32_t) d1] * pr1 + hinc[1][(int32_t) (d1 + 1)] * pr2;
        double diff2 = -v;
        if (back) p22 -= diff2; else p21 -= diff2;
      }
      double tmp = 0.0 - 0.0 - p22 + p21 - 0.0 * dx;
      ex[0][k] = ex[1][k] * 1.0 + tmp * cb_e;
    }
    swap2 (ex);
    for (int i = 0; i < inc_len - 1; ++i)
    {
      hinc[0][i] = hinc[1][i] + (einc[1][i] - einc[1][i + 1]) * mod_h;
    }
    swap2 (hinc);
    for (int k = 1; k < size - 1; ++k)
    {
      double p21 = ex[1][k], p22 = ex[1][k + 1];
      double c = k + 1.0;
      int back = is_fp_exact (c, left + 0 * 1.0 / 10.0);
      int front = is_fp_exact (c, right + 0 * 1.0 / 10.0);
      if (back || front)
      {
        int aux = back ? k : k + 1;
        double d = ((aux + 0.5) - zero_inc) - 0.0;
        double d1 = (double) ((int32_t) d);
        double pr2 = d - d1, pr1 = 1 - pr2;
        double v = einc[1][(int32_t) d1] * pr1 + einc[1][(int32_t) (d1 + 1)] * pr2;
        double diff2 = -v;
        diff2 *= -1.0;
        if (back) p21 -= diff2; else p22 -= diff2;
      }
      double tmp = 0.0 - 0.0 - p22 + p21 - 0.0 * dx;
      hy[0][k] = hy[1][k] * 1.0 + tmp * cb_h;
    }
    swap2 (hy);
  }
  memcpy (ex_out, ex[1], size * sizeof (double));
  for (int l = 0; l < 2; ++l)
  {
    free (ex[l]);
    free (hy[l]);
    free (einc[l]);
    free (hinc[l]);
  }
}

void fdtd_oracle_exhy_1d (int size, int tfsf, double dx, double lambda, double courant,
                          uint32_t steps, double *ex_sin, double *ex_cos)
{
  exhy_run (size, tfsf, dx, lambda, courant, steps, 0, ex_sin);
  exhy_run (size, tfsf, dx, lambda, courant, steps, 1, ex_cos);
}
