// setup.h - host-side set-up of the fdtd3d leapfrog step for the B200 kernels.
//
// Everything here runs once per context on the host, in FP64, with the same
// operation order as the reference so that the FP64 plain form can be
// bit-faithful.  The kernels receive the results as plain numbers, 1-D tables
// and integer boxes (no per-cell predicate evaluation on the device).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/fdtd_b200.h"

namespace fdtdb {

// Source/Physics/PhysicsConst.h:28-32
constexpr double kPi = 3.14159265358979323846;
constexpr double kC = 299792458.0;
constexpr double kMu0 = 4 * kPi * 0.0000001;
constexpr double kEps0 = 1 / (kMu0 * (kC * kC));

enum Comp { EX = 0, EY = 1, EZ = 2, HX = 3, HY = 4, HZ = 5 };

// One TF/SF correction term: on the cells of `box`, the curl of component
// `comp` uses neighbour slot `slot` (0 = p11, 1 = p12, 2 = p21, 3 = p22)
// minus the incident value of component `inc_comp` taken at the real
// coordinate of cell + aux.  InternalScheme.inc.h:1386-1835.
struct TfsfTerm
{
  int comp;
  int slot;
  int inc_comp;
  int lo[3];
  int hi[3];       // exclusive
  int aux[3];
  double negate;   // -1 for H in E_CENTERED and for E in H_CENTERED, else +1
};

// Per-component layout (E_CENTERED or H_CENTERED).  YeeGridLayout.cpp:1937-2035.
struct CompLayout
{
  bool exists;
  double min_fp[3];
  int opp1, opp2;
  int d11[3], d12[3], d21[3], d22[3];
  int sig_cacb, sig4, sig5;   // sigma axes
  int nmat;                   // 2 or 4 point material average
  int m[4][3];                // material offsets
};

struct Geometry
{
  fdtd_config cfg;
  int n[3];                   // grid size (1 along the axis a 2-D mode drops)
  int64_t cells;
  bool tmz;                   // Dim2_TMz (the mode of the adjoint and the batches)
  int drop = 0;               // bit a: axis a has size 1 (one axis in 2-D, two in 1-D)
  // 2-D / 1-D modes: distance of the incident wave along the wave vector is
  // u k0 + v k1 with u, v the positions along inc_ax[0], inc_ax[1]
  // (InternalScheme.cpp:110-307)
  int inc_ax[2] = {0, 1};
  double inc_k[2] = {0, 0};
  int levels;                 // stored time levels (2, or 3 with metamaterials)
  double dt, freq, rpv, dx;
  double a1, a2, a3;
  double s1, c1, s2, c2;
  double proj[6];
  double zero_inc[3];
  int inc_len;
  double mod_e, mod_h;        // incident-grid update modifiers
  CompLayout comp[6];
  // --use-double-material-precision: eps, mu and sigma on a grid of twice
  // the resolution (nf = 2 n on a kept axis, 1 on a dropped one); component
  // k averages the fine cells (2i, 2j, 2k) + fine_off[k][0..7] in the
  // reference's order (YeeGridLayout.h:866-1030)
  bool dmp = false;
  int nf[3] = {1, 1, 1};
  int64_t fine_cells = 0;
  int fine_off[6][8][3] = {};
  std::vector<double> sigma[3];   // 1-D sigma profiles (zero when PML off; on the fine grid with dmp)
  std::vector<TfsfTerm> tfsf;     // every TF/SF correction term
};

// Builds the geometry; returns an error message or "" on success.
std::string build_geometry (const fdtd_config &cfg, Geometry &g);

// Sigma profile of axis b averaged at the position of component k, as the
// reference's getMaterial averages the sigma grids (two points along an
// edge component's own axis, along the other two axes for the others).
std::vector<double> sigma_at (const Geometry &g, int k, int b);

// sin(2 pi f dt t) hard source of the incident grid at time step t.
double incident_source (const Geometry &g, uint32_t t);
// point-source value for an E (h = false) or H (h = true) component.
double point_source (const Geometry &g, uint32_t t, bool h);
// current I of the J (h = false) or M (h = true) current sources at time
// step t; the cell takes -= I dx Cb after its curl update.
double current_source (const Geometry &g, uint32_t t, bool h);

}  // namespace fdtdb
