// cli.cpp - fdtd3d-b200: command-line drop-in for fdtd3d's step path.
//
// Accepts fdtd3d's own flags for the modes this library provides
// (Source/Settings/Settings.inc.h; coordinate syntax "x:N,y:N,z:N",
// Source/Settings/Settings.cpp:74-131; float flags parsed with std::stof as
// the reference does, Settings.cpp:186-191), runs the time loop through the
// C ABI and writes the reference's outputs: "Total time = ... seconds"
// around the step loop (Source/main.cpp:1175-1213) and --save-as-txt dumps
// named previous-1_[timestep=T]_[pid=0]_[name=F].txt with 15 significant
// digits (Source/File-Management/Commons.h:63-120,
// Source/File-Management/Dumper/TXTDumper.h:60-84).  --save-as-dat writes the
// same region as raw FP64 values, z fastest, to previous-1_[...].dat
// (Source/File-Management/Dumper/DATDumper.h:52-90); the reference's DAT
// dumper names one file but opens the second name and writes nothing
// (DATDumper.h:129 passes the time level as the file count), so this takes
// the TXT dumper's naming, the evident intent.  Material files load by
// extension like GridFileManager::getFileType (Commons.cpp:46-67): .txt
// through the TXT loader, .dat as raw FP64 values of the whole grid, z
// fastest, with nothing after them (DATLoader.h:52-90).  The default save region
// is the reference's: the whole grid, one z slice at size/2 in 3-D
// (Source/Scheme/SchemeHelper.h:870-889).  The --same-size* flags copy x
// to y and z at the point where they are parsed, so a later coordinate flag
// overrides them (Source/Settings/Settings.cpp:249-261).
//
// Extra flags: --precision fp64|fp32|fp16s (default fp64 = the plain form);
// --complex-field-values writes what the reference's complex-field build
// (COMPLEX_FIELD_VALUES) writes: two runs, sine and cosine sources, give
// the real and imaginary parts ("coords re im" in TXT dumps, (re, im)
// pairs in DAT dumps); material files then hold complex values, of which
// the step uses the real parts, as the reference's does.  With it, --use-ntff (3-D) writes the
// reference's NTFF files from the two runs (fdtd_ntff; with --precision fp32
// or fp16s from the fast forms' fields).
// Flags of subsystems outside the step path (MPI, BMP output, test
// callbacks) are rejected with a message instead of being ignored.
#include <sys/time.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <limits>
#include <map>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/fdtd_b200.h"

namespace {

struct Opts
{
  fdtd_config cfg;
  int steps = 100;
  bool save_res = false, save_txt = false, save_dat = false, manual = false;
  bool complex_values = false;   // --complex-field-values: the reference's complex-field build
  int save_start[3] = {0, 0, 0}, save_end[3] = {0, 0, 0};
  std::string mat_file[6];
  int device = 0;
  // --use-ntff and its settings, with the reference's defaults
  // (Source/Settings/Settings.inc.h:83-88, 124, 181-187)
  bool use_ntff = false, ntff_reverse = false, ntff_stdout = false;
  int ntff_size[3] = {3, 3, 3};
  int ntff_diff = 1;
  double ntff_angle_step = 10.0;
  int ntff_interm = 100;
  std::string ntff_file = "ntff-res";
  // dump options of Scheme::saveGrids (Settings.inc.h:199-217, 279-281)
  bool save_interm = false, scattered_res = false, scattered_interm = false, save_no_pml = false;
  bool save_einc = false, save_hinc = false, save_materials = false;
  int interm_save_step = 100;
  bool orth[3] = {false, false, false};
  // material spheres: eps, mu, omegape, omegapm (Settings.inc.h:232-249);
  // a sphere is set when its value differs from the default (1, 1, 0, 0)
  struct Sphere
  {
    double value;
    int center[3] = {0, 0, 0};
    int radius = 0;
  } sphere[4] = {{1.0}, {1.0}, {0.0}, {0.0}};
  bool stair_sphere = false;
  int sphere_accuracy = 100;
};

// Axes a mode drops (bit a) and the components it keeps (bit k).
unsigned dropped_axes (int mode)
{
  switch (mode)
  {
    case FDTD_MODE_TEX:
    case FDTD_MODE_TMX:
      return 1u;
    case FDTD_MODE_TEY:
    case FDTD_MODE_TMY:
      return 2u;
    case FDTD_MODE_TEZ:
    case FDTD_MODE_TMZ:
      return 4u;
    case FDTD_MODE_EXHY:
    case FDTD_MODE_EYHX:
      return 3u;
    case FDTD_MODE_EXHZ:
    case FDTD_MODE_EZHX:
      return 5u;
    case FDTD_MODE_EYHZ:
    case FDTD_MODE_EZHY:
      return 6u;
    default:
      return 0u;
  }
}

unsigned mode_components (int mode)
{
  switch (mode)
  {
    case FDTD_MODE_TMZ: return (1u << FDTD_EZ) | (1u << FDTD_HX) | (1u << FDTD_HY);
    case FDTD_MODE_TEZ: return (1u << FDTD_EX) | (1u << FDTD_EY) | (1u << FDTD_HZ);
    case FDTD_MODE_TEX: return (1u << FDTD_EY) | (1u << FDTD_EZ) | (1u << FDTD_HX);
    case FDTD_MODE_TMX: return (1u << FDTD_EX) | (1u << FDTD_HY) | (1u << FDTD_HZ);
    case FDTD_MODE_TEY: return (1u << FDTD_EX) | (1u << FDTD_EZ) | (1u << FDTD_HY);
    case FDTD_MODE_TMY: return (1u << FDTD_EY) | (1u << FDTD_HX) | (1u << FDTD_HZ);
    case FDTD_MODE_EXHY: return (1u << FDTD_EX) | (1u << FDTD_HY);
    case FDTD_MODE_EXHZ: return (1u << FDTD_EX) | (1u << FDTD_HZ);
    case FDTD_MODE_EYHX: return (1u << FDTD_EY) | (1u << FDTD_HX);
    case FDTD_MODE_EYHZ: return (1u << FDTD_EY) | (1u << FDTD_HZ);
    case FDTD_MODE_EZHX: return (1u << FDTD_EZ) | (1u << FDTD_HX);
    case FDTD_MODE_EZHY: return (1u << FDTD_EZ) | (1u << FDTD_HY);
    default: return 0x3fu;
  }
}

int fail (const std::string &m)
{
  std::fprintf (stderr, "fdtd3d-b200: %s\n", m.c_str ());
  return 1;
}

bool parse_coord (const std::string &s, int out[3])
{
  std::stringstream ss (s);
  std::string tok;
  while (std::getline (ss, tok, ','))
  {
    if (tok.size () < 3 || tok[1] != ':')
      return false;
    int axis = tok[0] == 'x' ? 0 : (tok[0] == 'y' ? 1 : (tok[0] == 'z' ? 2 : -1));
    if (axis < 0)
      return false;
    out[axis] = std::atoi (tok.c_str () + 2);
  }
  return true;
}

double stof_like (const std::string &s)
{
  return (double) std::stof (s);
}

// --eps-sphere / --mu-sphere / --omegape-sphere / --omegapm-sphere and their
// -center / -radius flags.  Returns true when `a` is one of them; `ok`
// tells whether its argument parsed.
bool sphere_flag (const std::string &a, Opts &o, const std::vector<std::string> &args, size_t &i, std::string &v,
                  bool &ok)
{
  static const char *names[4] = {"--eps-sphere", "--mu-sphere", "--omegape-sphere", "--omegapm-sphere"};
  for (int m = 0; m < 4; ++m)
  {
    const std::string base = names[m];
    const int what = a == base ? 0 : (a == base + "-center" ? 1 : (a == base + "-radius" ? 2 : -1));
    if (what < 0)
      continue;
    ok = i + 1 < args.size ();
    if (!ok)
      return true;
    v = args[++i];
    if (what == 0)
      o.sphere[m].value = stof_like (v);
    else if (what == 1)
      ok = parse_coord (v, o.sphere[m].center);
    else
      o.sphere[m].radius = std::atoi (v.c_str ());
    return true;
  }
  return false;
}

// Fraction of the unit cell centred at mid (its `dim` kept coordinates)
// inside the sphere (centre c, radius r): the reference's column
// integration with `steps` samples per axis, the height of the sphere's
// surface above (or below) the cell's face clamped to the cell
// (Approximation::approximateSphereAccurate, Source/Layout/Approximation.cpp:
// 387-668; its 1-D form takes the interval overlap with the reference's
// tests as written).  The arithmetic follows the reference expression by
// expression, so the values agree bit for bit.
double sphere_volume (int dim, const double mid[3], const double c[3], double r, int steps)
{
  double lo[3], hi[3];
  for (int k = 0; k < dim; ++k)
  {
    lo[k] = mid[k] - 0.5;
    hi[k] = mid[k] + 0.5;
  }
  double volume = 0;
  if (dim == 1)
  {
    const double left = c[0] - r, right = c[0] + r;
    if (hi[0] <= left || lo[0] >= right)
      volume = 0;
    else if (lo[0] >= left || hi[0] <= right)
      volume = 1;
    else if (lo[0] < left)
      volume = hi[0] - left;
    else if (hi[0] > right)
      volume = right - lo[0];
  }
  else
  {
    // the last kept axis is the one solved for; the others are sampled
    const int h = dim - 1;
    const double step = 1.0 / steps;
    const double cell = dim == 2 ? step : step * step;
    const int n2 = dim == 2 ? 1 : steps;
    for (int i = 0; i < steps; ++i)
      for (int j = 0; j < n2; ++j)
      {
        const double u = lo[0] + i * step;
        double rest = r * r - (u - c[0]) * (u - c[0]);
        if (dim == 3)
        {
          const double w = lo[1] + j * step;
          rest = rest - (w - c[1]) * (w - c[1]);
        }
        double height = 0.0;
        if (rest >= 0)
        {
          const bool above = mid[h] > c[h];
          height = above ? c[h] + std::sqrt (rest) : c[h] - std::sqrt (rest);
          if (height < lo[h])
            height = lo[h];
          else if (height > hi[h])
            height = hi[h];
          height = above ? height - lo[h] : hi[h] - height;
        }
        volume += height * cell;
      }
  }
  if (volume > 1)
    volume = 1;
  return volume;
}

// Whether every corner of the unit cell centred at mid lies in the sphere
// (Approximation::approximateSphereStair, Approximation.cpp:678-764).
bool sphere_stair (int dim, const double mid[3], const double c[3], double r)
{
  for (int corner = 0; corner < (1 << dim); ++corner)
  {
    double d2 = 0;
    for (int k = 0; k < dim; ++k)
    {
      const double q = mid[k] + (((corner >> k) & 1) ? 0.5 : -0.5) - c[k];
      d2 = d2 + q * q;
    }
    if (!(std::sqrt (d2) <= r))
      return false;
  }
  return true;
}

// Fills a material grid (x-major over n[0] x n[1] x n[2], a mode's dropped
// axes of size 1) with a sphere as Scheme::initGrids does for the
// --*-sphere flags (Source/Scheme/Scheme.inc.h:2980-3160): every cell, at
// its real position (index + 0.5 on each kept axis, YeeGridLayout's
// minEpsCoordFP), gets value * volume + outside * (1 - volume), or value /
// outside by the stair test; the centre is centre * modifier + 0.5 and the
// radius radius * modifier (modifier 2 on the doubled grid of
// --use-double-material-precision).
void fill_sphere (std::vector<double> &grid, const int n[3], unsigned drop, const Opts::Sphere &sp, double value,
                  double outside, double modifier, bool stair, int steps)
{
  int axes[3], dim = 0;
  for (int a = 0; a < 3; ++a)
    if (!((drop >> a) & 1u))
      axes[dim++] = a;
  double c[3];
  for (int k = 0; k < dim; ++k)
    c[k] = sp.center[axes[k]] * modifier + 0.5;
  const double r = sp.radius * modifier;
  size_t id = 0;
  for (int x = 0; x < n[0]; ++x)
    for (int y = 0; y < n[1]; ++y)
      for (int z = 0; z < n[2]; ++z, ++id)
      {
        const int pos[3] = {x, y, z};
        double mid[3];
        for (int k = 0; k < dim; ++k)
          mid[k] = (double) pos[axes[k]] + 0.5;
        if (stair)
          grid[id] = sphere_stair (dim, mid, c, r) ? value : outside;
        else
        {
          const double vol = sphere_volume (dim, mid, c, r, steps);
          grid[id] = value * vol + outside * (1 - vol);
        }
      }
}

std::vector<std::string> read_cmd_file (const std::string &path)
{
  std::vector<std::string> out;
  std::ifstream f (path);
  std::string line;
  while (std::getline (f, line))
  {
    size_t b = line.find_first_not_of (" \t\r");
    if (b == std::string::npos)
      continue;
    line = line.substr (b);
    if (line[0] == '#' || line.compare (0, 2, "//") == 0)
      continue;
    size_t e = line.find_last_not_of (" \t\r");
    out.push_back (line.substr (0, e + 1));
  }
  return out;
}

int parse (std::vector<std::string> args, Opts &o)
{
  std::memset (&o.cfg, 0, sizeof (o.cfg));
  fdtd_config &c = o.cfg;
  c.mode = FDTD_MODE_DIM3;
  for (int a = 0; a < 3; ++a)
  {
    c.size[a] = 100;
    c.pml[a] = 2;
    c.tfsf_left[a] = 4;
    c.tfsf_right[a] = 4;
  }
  // defaults are the reference's double literals, used as they are; only
  // values given on the command line pass through stof
  // (Source/Settings/Settings.inc.h:192-194, Settings.h:200-215)
  c.dx = 0.0005;
  c.wavelength = 0.02;
  c.courant = 0.5;
  c.angle_teta = 90.0;
  c.angle_phi = 0.0;
  c.angle_psi = 90.0;
  c.precision = FDTD_PREC_FP64_PLAIN;
  static const char *mat_flags[6] = {"--load-eps-from-file", "--load-mu-from-file", "--load-omegape-from-file",
                                     "--load-omegapm-from-file", "--load-gammae-from-file",
                                     "--load-gammam-from-file"};
  static const char *ps_flags[6] = {"--point-source-ex", "--point-source-ey", "--point-source-ez",
                                    "--point-source-hx", "--point-source-hy", "--point-source-hz"};
  static const char *cs_flags[6] = {"--current-source-jx", "--current-source-jy", "--current-source-jz",
                                    "--current-source-mx", "--current-source-my", "--current-source-mz"};
  static const char *ignored[] = {"--use-ca-cb", "--use-ca-cb-pml", "--use-ca-cb-pml-metamaterials", "--use-cuda",
                                  nullptr};
  static const char *ignored_arg[] = {"--log-level", "--cuda-buffer-size", "--num-cuda-threads", "--layout-type",
                                      nullptr};
  for (size_t i = 0; i < args.size (); ++i)
  {
    const std::string &a = args[i];
    auto next = [&] (std::string &v) -> bool {
      if (i + 1 >= args.size ())
        return false;
      v = args[++i];
      return true;
    };
    std::string v;
    bool handled = true;
    if (a == "--3d")
      c.mode = FDTD_MODE_DIM3;
    else if (a == "--2d-tmz")
      c.mode = FDTD_MODE_TMZ;
    else if (a == "--2d-tez")
      c.mode = FDTD_MODE_TEZ;
    else if (a == "--2d-tex")
      c.mode = FDTD_MODE_TEX;
    else if (a == "--2d-tmx")
      c.mode = FDTD_MODE_TMX;
    else if (a == "--2d-tey")
      c.mode = FDTD_MODE_TEY;
    else if (a == "--2d-tmy")
      c.mode = FDTD_MODE_TMY;
    else if (a == "--1d-exhy")
      c.mode = FDTD_MODE_EXHY;
    else if (a == "--1d-exhz")
      c.mode = FDTD_MODE_EXHZ;
    else if (a == "--1d-eyhx")
      c.mode = FDTD_MODE_EYHX;
    else if (a == "--1d-eyhz")
      c.mode = FDTD_MODE_EYHZ;
    else if (a == "--1d-ezhx")
      c.mode = FDTD_MODE_EZHX;
    else if (a == "--1d-ezhy")
      c.mode = FDTD_MODE_EZHY;
    else if (a == "--size" && next (v))
    {
      if (!parse_coord (v, c.size))
        return fail ("bad --size");
    }
    else if (a == "--same-size")
      c.size[1] = c.size[2] = c.size[0];   // applied when parsed, as the reference does
    else if (a == "--pml-size" && next (v))
    {
      if (!parse_coord (v, c.pml))
        return fail ("bad --pml-size");
    }
    else if (a == "--same-size-pml")
      c.pml[1] = c.pml[2] = c.pml[0];
    else if (a == "--tfsf-size-left" && next (v))
    {
      if (!parse_coord (v, c.tfsf_left))
        return fail ("bad --tfsf-size-left");
    }
    else if (a == "--tfsf-size-right" && next (v))
    {
      if (!parse_coord (v, c.tfsf_right))
        return fail ("bad --tfsf-size-right");
    }
    else if (a == "--same-size-tfsf")
    {
      c.tfsf_left[1] = c.tfsf_left[2] = c.tfsf_left[0];
      c.tfsf_right[1] = c.tfsf_right[2] = c.tfsf_right[0];
    }
    else if (a == "--time-steps" && next (v))
      o.steps = std::atoi (v.c_str ());
    else if (a == "--angle-teta" && next (v))
      c.angle_teta = stof_like (v);
    else if (a == "--angle-phi" && next (v))
      c.angle_phi = stof_like (v);
    else if (a == "--angle-psi" && next (v))
      c.angle_psi = stof_like (v);
    else if (a == "--dx" && next (v))
      c.dx = stof_like (v);
    else if (a == "--wavelength" && next (v))
      c.wavelength = stof_like (v);
    else if (a == "--courant-factor" && next (v))
      c.courant = stof_like (v);
    else if (a == "--use-pml")
      c.use_pml = 1;
    else if (a == "--use-tfsf")
      c.use_tfsf = 1;
    else if (a == "--use-metamaterials")
      c.use_metamaterials = 1;
    else if (a == "--use-double-material-precision")
      c.double_material_precision = 1;
    else if (a == "--point-source" && next (v))
    {
      if (!parse_coord (v, c.point_source))
        return fail ("bad --point-source");
    }
    else if (a == "--current-source" && next (v))
    {
      if (!parse_coord (v, c.current_source))
        return fail ("bad --current-source");
    }
    else if (a == "--save-res")
      o.save_res = true;
    else if (a == "--save-interm-res")
      o.save_interm = true;
    else if (a == "--interm-save-step" && next (v))
      o.interm_save_step = std::atoi (v.c_str ());
    else if (a == "--save-scattered-field-res")
      o.scattered_res = true;
    else if (a == "--save-scattered--field-interm")   // the reference's spelling
      o.scattered_interm = true;
    else if (a == "--save-tfsf-e-incident")
      o.save_einc = true;
    else if (a == "--save-tfsf-h-incident")
      o.save_hinc = true;
    else if (a == "--save-no-pml")
      o.save_no_pml = true;
    else if (a == "--save-materials")
      o.save_materials = true;
    else if (a == "--orth-axis-x" || a == "--orth-axis-y" || a == "--orth-axis-z")
      o.orth[a.back () - 'x'] = true;
    else if (a == "--save-as-txt")
      o.save_txt = true;
    else if (a == "--save-as-dat")
      o.save_dat = true;
    else if (a == "--complex-field-values")
      o.complex_values = true;
    else if (a == "--use-ntff")
      o.use_ntff = true;
    else if (a == "--ntff-size" && next (v))
    {
      if (!parse_coord (v, o.ntff_size))
        return fail ("bad --ntff-size");
    }
    else if (a == "--same-size-ntff")
      o.ntff_size[1] = o.ntff_size[2] = o.ntff_size[0];
    else if (a == "--ntff-diff" && next (v))
      o.ntff_diff = std::atoi (v.c_str ());
    else if (a == "--ntff-reverse")
      o.ntff_reverse = true;
    else if (a == "--ntff-filename" && next (v))
      o.ntff_file = v;
    else if (a == "--ntff-to-stdout")
      o.ntff_stdout = true;
    else if (a == "--ntff-step-angle" && next (v))
      o.ntff_angle_step = stof_like (v);
    else if (a == "--interm-ntff-step" && next (v))
      o.ntff_interm = std::atoi (v.c_str ());
    else if (a == "--manual-save-coords")
      o.manual = true;
    else if (a == "--save-start-coord" && next (v))
    {
      if (!parse_coord (v, o.save_start))
        return fail ("bad --save-start-coord");
    }
    else if (a == "--save-end-coord" && next (v))
    {
      if (!parse_coord (v, o.save_end))
        return fail ("bad --save-end-coord");
    }
    else if (a == "--cuda-gpus" && next (v))
      o.device = std::atoi (v.c_str ());
    else if (a == "--precision" && next (v))
    {
      if (v == "fp64")
        c.precision = FDTD_PREC_FP64_PLAIN;
      else if (v == "fp32")
        c.precision = FDTD_PREC_FP32;
      else if (v == "fp16s")
        c.precision = FDTD_PREC_FP16S;
      else
        return fail ("--precision must be fp64, fp32 or fp16s");
    }
    else if (a == "--stair-sphere-approx")
      o.stair_sphere = true;
    else if (a == "--sphere-accuracy" && next (v))
      o.sphere_accuracy = std::atoi (v.c_str ());
    else if (sphere_flag (a, o, args, i, v, handled))
    {
      if (!handled)
        return fail ("bad " + a);
    }
    else if (a == "--cmd-from-file" && next (v))
    {
      std::vector<std::string> more = read_cmd_file (v);
      args.insert (args.begin () + i + 1, more.begin (), more.end ());
    }
    else
      handled = false;
    if (handled)
      continue;
    bool done = false;
    for (int m = 0; m < 6 && !done; ++m)
    {
      if (a == mat_flags[m] && next (v))
      {
        o.mat_file[m] = v;
        done = true;
      }
      else if (a == ps_flags[m])
      {
        c.point_source_mask |= 1 << m;
        done = true;
      }
      else if (a == cs_flags[m])
      {
        c.current_source_mask |= 1 << m;
        done = true;
      }
    }
    for (int m = 0; ignored[m] && !done; ++m)
      done = a == ignored[m];
    for (int m = 0; ignored_arg[m] && !done; ++m)
    {
      if (a == ignored_arg[m])
      {
        if (a == "--layout-type")
        {
          // Settings.inc.h: 0 = E_CENTERED, 1 = H_CENTERED (main.cpp asserts one of the two)
          if (!next (v) || (v != "0" && v != "1"))
            return fail ("--layout-type takes 0 (E_CENTERED) or 1 (H_CENTERED)");
          c.layout = std::atoi (v.c_str ());
        }
        else
          next (v);
        done = true;
      }
    }
    if (!done)
      return fail ("unsupported flag " + a + " (outside the step path this binary provides)");
  }
  for (int a = 0; a < 3; ++a)
    if ((dropped_axes (c.mode) >> a) & 1u)
      c.size[a] = 1;
  return 0;
}

// TXT grid loader: "x y [z] value" per line, z fastest; values through stof
// (Source/File-Management/Loader/TXTLoader.h:60-100).
bool load_txt (const std::string &path, size_t n, int coords, bool complex_values, std::vector<double> &out,
               std::vector<double> &im_out)
{
  std::ifstream f (path);
  if (!f)
    return false;
  out.assign (n, 0.0);
  im_out.assign (complex_values ? n : 0, 0.0);
  std::string line;
  size_t i = 0;
  while (i < n && std::getline (f, line))
  {
    std::stringstream ss (line);
    std::string tok;
    for (int k = 0; k <= coords; ++k)
      ss >> tok;
    out[i] = (double) std::stof (tok);
    if (complex_values)
    {
      // complex build: "coords re im"; the step reads the real part of every
      // material value (Approximation::getMaterial, Approximation.cpp:250-255),
      // --save-materials writes both
      std::string im;
      if (!(ss >> im))
        return false;
      im_out[i] = (double) std::stof (im);
    }
    ++i;
  }
  return i == n;
}

// DAT grid loader: raw FP64 values of the whole grid, z fastest, and
// nothing after them (Source/File-Management/Loader/DATLoader.h:52-90);
// (re, im) pairs in the complex build, of which the step reads the real part.
bool load_dat (const std::string &path, size_t n, bool complex_values, std::vector<double> &out,
               std::vector<double> &im_out)
{
  std::ifstream f (path, std::ios::binary);
  if (!f)
    return false;
  const size_t per = complex_values ? 2 : 1;
  std::vector<double> raw (n * per);
  f.read (reinterpret_cast<char *> (raw.data ()), (std::streamsize) (raw.size () * sizeof (double)));
  if (!f || (size_t) f.gcount () != raw.size () * sizeof (double))
    return false;
  f.peek ();
  if (!f.eof ())
    return false;
  out.assign (n, 0.0);
  im_out.assign (complex_values ? n : 0, 0.0);
  for (size_t i = 0; i < n; ++i)
  {
    out[i] = raw[i * per];
    if (complex_values)
      im_out[i] = raw[i * per + 1];
  }
  return true;
}

// Material file by extension (GridFileManager::getFileType, Commons.cpp:46-67).
bool load_material (const std::string &path, size_t n, int coords, bool complex_values, std::vector<double> &out,
                    std::vector<double> &im, std::string &why)
{
  const size_t dot = path.find_last_of ('.');
  const std::string ext = dot == std::string::npos ? "" : path.substr (dot + 1);
  const std::string note = complex_values ? " (complex values: coordinates, real and imaginary part)" : "";
  if (ext == "txt")
    return load_txt (path, n, coords, complex_values, out, im) || (why = "cannot read " + path + note, false);
  if (ext == "dat")
    return load_dat (path, n, complex_values, out, im) ||
           (why = "cannot read " + path + " (expects " + std::to_string (n) + " FP64 values)" + note, false);
  why = path + ": material files are .txt or .dat";
  return false;
}

// im: imaginary parts (complex build: (re, im) pairs), or null
bool save_dat (const std::string &name, const std::vector<double> &v, const std::vector<double> *im, const int n[3],
               const int lo[3], const int hi[3])
{
  std::ofstream f (name, std::ios::binary);
  if (!f)
    return false;
  for (int x = lo[0]; x < hi[0]; ++x)
    for (int y = lo[1]; y < hi[1]; ++y)
    {
      const size_t id = ((size_t) x * n[1] + y) * n[2] + lo[2];
      if (!im)
      {
        f.write (reinterpret_cast<const char *> (v.data () + id), (std::streamsize) ((hi[2] - lo[2]) * sizeof (double)));
        continue;
      }
      for (int z = lo[2]; z < hi[2]; ++z)
      {
        const double pair[2] = {v[id + (z - lo[2])], (*im)[id + (z - lo[2])]};
        f.write (reinterpret_cast<const char *> (pair), sizeof (pair));
      }
    }
  return (bool) f;
}

bool save_txt (const std::string &name, const std::vector<double> &v, const std::vector<double> *im, const int n[3],
               unsigned drop, const int lo[3], const int hi[3])
{
  std::ofstream f (name);
  if (!f)
    return false;
  f << std::setprecision (std::numeric_limits<double>::digits10);
  for (int x = lo[0]; x < hi[0]; ++x)
    for (int y = lo[1]; y < hi[1]; ++y)
      for (int z = lo[2]; z < hi[2]; ++z)
      {
        size_t id = ((size_t) x * n[1] + y) * n[2] + z;
        const int c[3] = {x, y, z};
        bool first = true;
        for (int a = 0; a < 3; ++a)
          if (!((drop >> a) & 1u))
          {
            f << (first ? "" : " ") << c[a];
            first = false;
          }
        f << " " << v[id];
        if (im)
          f << " " << (*im)[id];
        f << std::endl;
      }
  return true;
}

}  // namespace

// First position of component k on axis a (Source/Layout/YeeGridLayout.cpp:
// 1937-2035): an "edge" component (E in E_CENTERED, H in H_CENTERED) sits at
// 1.0 on its own axis and 0.5 on the others; the other family the reverse.
double min_fp (int layout, int k, int a)
{
  const bool edge = (k >= 3) == (layout == 1);
  return edge ? (a == k % 3 ? 1.0 : 0.5) : (a == k % 3 ? 0.5 : 1.0);
}

// Scheme::saveGrids (Source/Scheme/Scheme.inc.h:4367-4530) at time t: every
// component of the mode over the save region (manual coordinates; else the
// whole grid, inside the PML with --save-no-pml, one slice across the
// orthogonal axis in 3-D), the scattered field when asked
// (makeGridScattered), and the 1-D incident grids when asked, to
// previous-1_[timestep=t]_[pid=0]_[name=F].{txt,dat}.
bool save_grids (const Opts &o, std::vector<fdtd_ctx *> &ctx, uint32_t t, bool scattered, std::string &why)
{
  static const char *names[6] = {"Ex", "Ey", "Ez", "Hx", "Hy", "Hz"};
  const unsigned drop = dropped_axes (o.cfg.mode);
  int n[3];
  for (int a = 0; a < 3; ++a)
    n[a] = ((drop >> a) & 1u) ? 1 : o.cfg.size[a];
  const size_t cells = (size_t) n[0] * n[1] * n[2];
  const int nrun = (int) ctx.size ();
  const int orth = o.orth[0] ? 0 : (o.orth[1] ? 1 : 2);
  std::vector<double> buf[2];
  for (int k = 0; k < 6; ++k)
  {
    if (!((mode_components (o.cfg.mode) >> k) & 1u))
      continue;
    int lo[3] = {0, 0, 0}, hi[3] = {n[0], n[1], n[2]};
    if (o.manual)
    {
      for (int a = 0; a < 3; ++a)
      {
        lo[a] = o.save_start[a];
        hi[a] = o.save_end[a];
      }
      for (int a = 0; a < 3; ++a)
        if ((drop >> a) & 1u)
        {
          lo[a] = 0;
          hi[a] = 1;
        }
    }
    else
    {
      if (o.save_no_pml && o.cfg.use_pml)
      {
        // getStartCoord / getEndCoord (Scheme.inc.h:4645-4790): the PML
        // borders less the component's position, truncated; the start one
        // cell further in
        for (int a = 0; a < 3; ++a)
          if (!((drop >> a) & 1u))
          {
            lo[a] = (int) ((double) o.cfg.pml[a] - min_fp (o.cfg.layout, k, a)) + 1;
            hi[a] = (int) ((double) (n[a] - o.cfg.pml[a]) - min_fp (o.cfg.layout, k, a));
          }
      }
      if (drop == 0)
      {
        lo[orth] = n[orth] / 2;
        hi[orth] = n[orth] / 2 + 1;
      }
    }
    for (int r = 0; r < nrun; ++r)
    {
      buf[r].resize (cells);
      const int st = scattered ? fdtd_download_field_scattered (ctx[r], k, buf[r].data ())
                               : fdtd_download_field (ctx[r], k, buf[r].data ());
      if (st)
        return why = std::string ("download: ") + fdtd_last_error (), false;
    }
    const std::vector<double> *im = o.complex_values ? &buf[1] : nullptr;
    const std::string base = "previous-1_[timestep=" + std::to_string (t) + "]_[pid=0]_[name=" + names[k] + "]";
    if (o.save_txt && !save_txt (base + ".txt", buf[0], im, n, drop, lo, hi))
      return why = "cannot write " + base + ".txt", false;
    if (o.save_dat && !save_dat (base + ".dat", buf[0], im, n, lo, hi))
      return why = "cannot write " + base + ".dat", false;
  }
  // the 1-D incident grids (a grid of one axis, dumped whole)
  for (int fam = 0; fam < 2; ++fam)
  {
    if (!(fam ? o.save_hinc : o.save_einc) || !o.cfg.use_tfsf)
      continue;
    const int len = fdtd_incident_length (ctx[0]);
    for (int r = 0; r < nrun; ++r)
    {
      buf[r].resize (len);
      if (fdtd_download_incident (ctx[r], fam, buf[r].data (), len))
        return why = std::string ("download_incident: ") + fdtd_last_error (), false;
    }
    const std::vector<double> *im = o.complex_values ? &buf[1] : nullptr;
    const int n1[3] = {1, 1, len}, lo1[3] = {0, 0, 0}, hi1[3] = {1, 1, len};
    const std::string base = std::string ("previous-1_[timestep=") + std::to_string (t) + "]_[pid=0]_[name="
                             + (fam ? "HInc" : "EInc") + "]";
    if (o.save_txt && !save_txt (base + ".txt", buf[0], im, n1, 3u, lo1, hi1))
      return why = "cannot write " + base + ".txt", false;
    if (o.save_dat && !save_dat (base + ".dat", buf[0], im, n1, lo1, hi1))
      return why = "cannot write " + base + ".dat", false;
  }
  return true;
}

// --save-materials (Source/Scheme/Scheme.inc.h:3168-3225): the material
// grids as set, before the first step, to previous-0_[timestep=0]_[pid=0]_
// [name=Eps|Mu|OmegaPE|OmegaPM|GammaE|GammaM] (the Drude grids with
// metamaterials only), over the save region of a grid with no component
// offset (the doubled grid with double material precision).
bool save_materials (const Opts &o, const std::vector<double> mat[6], const std::vector<double> mat_im[6],
                     std::string &why)
{
  static const char *names[6] = {"Eps", "Mu", "OmegaPE", "OmegaPM", "GammaE", "GammaM"};
  const unsigned drop = dropped_axes (o.cfg.mode);
  const int orth = o.orth[0] ? 0 : (o.orth[1] ? 1 : 2);
  for (int m = 0; m < (o.cfg.use_metamaterials ? 6 : 2); ++m)
  {
    const int mul = (m < 2 && o.cfg.double_material_precision) ? 2 : 1;
    int n[3];
    for (int a = 0; a < 3; ++a)
      n[a] = ((drop >> a) & 1u) ? 1 : mul * o.cfg.size[a];
    int lo[3] = {0, 0, 0}, hi[3] = {n[0], n[1], n[2]};
    if (o.manual)
    {
      for (int a = 0; a < 3; ++a)
        if (!((drop >> a) & 1u))
        {
          lo[a] = o.save_start[a];
          hi[a] = o.save_end[a];
        }
    }
    else
    {
      if (o.save_no_pml && o.cfg.use_pml)
        for (int a = 0; a < 3; ++a)
          if (!((drop >> a) & 1u))
          {
            lo[a] = o.cfg.pml[a] + 1;
            hi[a] = n[a] - o.cfg.pml[a];
          }
      if (drop == 0)
      {
        lo[orth] = n[orth] / 2;
        hi[orth] = n[orth] / 2 + 1;
      }
    }
    const std::vector<double> *im = o.complex_values ? &mat_im[m] : nullptr;
    const std::string base = std::string ("previous-0_[timestep=0]_[pid=0]_[name=") + names[m] + "]";
    if (o.save_txt && !save_txt (base + ".txt", mat[m], im, n, drop, lo, hi))
      return why = "cannot write " + base + ".txt", false;
    if (o.save_dat && !save_dat (base + ".dat", mat[m], im, n, lo, hi))
      return why = "cannot write " + base + ".dat", false;
  }
  return true;
}

// Scheme::saveNTFF (Source/Scheme/Scheme.inc.h:4535-4645): for every box of
// --ntff-diff (moved in by one cell each), the forward diagram (azimuths 0 ..
// 2 pi + pi / 180 by --ntff-step-angle at the incident polar angle) or the
// reverse one (the incident azimuth), to ntff-res_[timestep=T]_[step=S].txt
// or to stdout, in the reference's words and default stream formatting.
bool save_ntff (const Opts &o, fdtd_ctx *re, fdtd_ctx *im, uint32_t t, std::string &why)
{
  const double pi = 3.14159265358979323846;
  const double a1 = o.cfg.angle_teta * pi / 180.0;
  const double a2 = o.cfg.angle_phi * pi / 180.0;
  const double a3 = o.cfg.angle_psi * pi / 180.0;
  for (int s = 0; s < o.ntff_diff; ++s)
  {
    int left[3], right[3];
    for (int a = 0; a < 3; ++a)
    {
      left[a] = o.ntff_size[a] + s;
      right[a] = o.cfg.size[a] - o.ntff_size[a] + 1 - s;
    }
    double start, end, step;
    const char *name;
    if (o.ntff_reverse)
    {
      name = "Reverse diagram";
      start = end = a2;
      step = 1.0;
    }
    else
    {
      name = "Forward diagram";
      start = 0.0;
      end = 2 * pi + pi / 180;
      step = pi * o.ntff_angle_step / 180;
    }
    std::vector<double> phi;
    for (double angle = start; angle <= end; angle += step)
      phi.push_back (angle);
    std::vector<double> val (phi.size ());
    if (fdtd_ntff (re, im, left, right, a1, (int) phi.size (), phi.data (), val.data ()))
      return why = std::string ("fdtd_ntff: ") + fdtd_last_error (), false;
    std::ofstream file;
    std::ostream *out = &std::cout;
    if (!o.ntff_stdout)
    {
      const std::string fname = o.ntff_file + "_[timestep=" + std::to_string (t) + "]_[step=" + std::to_string (s)
                                + "].txt";
      file.open (fname);
      if (!file)
        return why = "cannot write " + fname, false;
      out = &file;
    }
    (*out) << "==== NTFF (step=" << s << ") ====" << std::endl;
    (*out) << name << std::endl << std::endl;
    for (size_t i = 0; i < phi.size (); ++i)
      (*out) << "timestep = " << t << ", incident wave angle=(" << a1 << "," << a2 << "," << a3 << ","
             << "), angle NTFF = " << phi[i] << ", NTFF value = " << val[i] << std::endl;
  }
  return true;
}

int main (int argc, char **argv)
{
  Opts o;
  std::vector<std::string> args (argv + 1, argv + argc);
  if (parse (args, o))
    return 1;
  if (o.save_no_pml && !o.manual && o.cfg.use_pml)
  {
    // the reference's getStartCoord expands the PML border to 3-D and
    // narrows it back by position, which matches the grid's axes only when
    // a mode keeps the leading ones; otherwise it indexes out of its grid
    const unsigned d = dropped_axes (o.cfg.mode);
    if (d != 0 && d != 4u && d != 6u)
      return fail ("--save-no-pml: the reference's save region is defined for 3-D and for modes that keep x "
                   "(and y); for this mode it indexes outside its grid");
  }
  if ((o.scattered_res || o.scattered_interm) && !o.cfg.use_tfsf)
    return fail ("the scattered field needs --use-tfsf");
  if (o.use_ntff && (!o.complex_values || o.cfg.mode != FDTD_MODE_DIM3))
    return fail ("--use-ntff needs --3d and --complex-field-values (the reference computes the NTFF in its "
                 "complex-field build only, for 3-D grids)");
  // the complex-field build's run is the sine-source run (real part) plus i
  // times the cosine-source run (imaginary part): one context for each
  const int nrun = o.complex_values ? 2 : 1;
  std::vector<fdtd_ctx *> ctx (nrun, nullptr);
  struct Release
  {
    std::vector<fdtd_ctx *> &c;
    ~Release ()
    {
      for (fdtd_ctx *x : c)
        if (x)
          fdtd_destroy (x);
    }
  } release{ctx};
  int st = 0;
  for (int r = 0; r < nrun; ++r)
  {
    fdtd_config cfg = o.cfg;
    cfg.source_phase = r;
    // the complex build's current is cos(w (t - 1)) - i sin(w (t - 1))
    cfg.current_phase = o.complex_values ? 1 + r : 0;
    st = fdtd_create (&cfg, o.device, &ctx[r]);
    if (st)
      return fail (std::string ("fdtd_create: ") + fdtd_status_str (st) + ": " + fdtd_last_error ());
    // the NTFF of an FP32 / FP16 run reads the previous H level
    if (o.use_ntff && (st = fdtd_keep_previous_level (ctx[r], 1)))
      return fail (std::string ("fdtd_keep_previous_level: ") + fdtd_last_error ());
  }
  const unsigned drop = dropped_axes (o.cfg.mode);
  int n[3] = {o.cfg.size[0], o.cfg.size[1], o.cfg.size[2]};
  int kept = 0;
  for (int a = 0; a < 3; ++a)
  {
    if ((drop >> a) & 1u)
      n[a] = 1;
    else
      ++kept;
  }
  size_t cells = (size_t) n[0] * n[1] * n[2];
  // --use-double-material-precision: eps and mu files hold the grid of twice
  // the resolution on every kept axis
  size_t fine = cells;
  if (o.cfg.double_material_precision)
    for (int a = 0; a < kept; ++a)
      fine *= 2;
  // material grids as set (defaults eps = mu = 1, Drude terms 0), kept for
  // --save-materials
  std::vector<double> mat[6], mat_im[6];
  for (int m = 0; m < 6; ++m)
  {
    mat[m].assign (m < 2 ? fine : cells, m < 2 ? 1.0 : 0.0);
    if (o.complex_values)
      mat_im[m].assign (mat[m].size (), 0.0);
    // a material sphere replaces every value of its grid, the file's too
    // (Scheme::initGrids: file first, then the sphere); the Drude spheres
    // hold omega * 2 pi * (c / lambda) and only with --use-metamaterials
    const bool sphere = m < 4 && o.sphere[m].value != (m < 2 ? 1.0 : 0.0) && (m < 2 || o.cfg.use_metamaterials);
    if (o.mat_file[m].empty () && !sphere)
      continue;
    std::string why;
    if (!o.mat_file[m].empty () &&
        !load_material (o.mat_file[m], m < 2 ? fine : cells, kept, o.complex_values, mat[m], mat_im[m], why))
      return fail (why);
    if (sphere)
    {
      int nm[3] = {n[0], n[1], n[2]};
      if (m < 2 && o.cfg.double_material_precision)
        for (int a = 0; a < 3; ++a)
          if (!((drop >> a) & 1u))
            nm[a] *= 2;
      double value = o.sphere[m].value;
      if (m >= 2)
        value = value * 2 * M_PI * (299792458.0 / o.cfg.wavelength);
      fill_sphere (mat[m], nm, drop, o.sphere[m], value, m < 2 ? 1.0 : 0.0,
                   o.cfg.double_material_precision ? 2.0 : 1.0, o.stair_sphere, o.sphere_accuracy);
      if (o.complex_values)
        std::fill (mat_im[m].begin (), mat_im[m].end (), 0.0);
    }
    for (int r = 0; r < nrun; ++r)
    {
      st = fdtd_upload_material (ctx[r], m, mat[m].data ());
      if (st)
        return fail (std::string ("fdtd_upload_material: ") + fdtd_last_error ());
    }
  }
  if (o.save_materials && (o.save_txt || o.save_dat))
  {
    std::string why;
    if (!save_materials (o, mat, mat_im, why))
      return fail (why);
  }
  struct timeval tv1, tv2;
  gettimeofday (&tv1, nullptr);
  // the reference saves the NTFF after every step that ends on a multiple
  // of --interm-ntff-step (SchemeHelper.h:100-104): step in chunks up to
  // those times
  uint32_t done = 0;
  while (!st && done < (uint32_t) o.steps)
  {
    uint32_t stop = (uint32_t) o.steps;
    if (o.use_ntff && o.ntff_interm > 0)
      stop = std::min<uint32_t> (stop, (done / o.ntff_interm + 1) * o.ntff_interm);
    if (o.save_interm && o.interm_save_step > 0)
      stop = std::min<uint32_t> (stop, (done / o.interm_save_step + 1) * o.interm_save_step);
    for (int r = 0; r < nrun && !st; ++r)
      st = fdtd_step (ctx[r], done, stop - done);
    for (int r = 0; r < nrun && !st; ++r)
      st = fdtd_sync (ctx[r], -1);
    done = stop;
    std::string why;
    if (!st && o.use_ntff && o.ntff_interm > 0 && done % o.ntff_interm == 0)
      if (!save_ntff (o, ctx[0], ctx[1], done, why))
        return fail (why);
    // intermediate dumps after the NTFF, as performNSteps orders them
    // (SchemeHelper.h:100-120)
    if (!st && o.save_interm && o.interm_save_step > 0 && done % o.interm_save_step == 0 &&
        (o.save_txt || o.save_dat))
      if (!save_grids (o, ctx, done, o.scattered_interm, why))
        return fail (why);
  }
  gettimeofday (&tv2, nullptr);
  if (st)
    return fail (std::string ("step: ") + fdtd_status_str (st) + ": " + fdtd_last_error ());
  std::printf ("Total time = %f seconds\n",
               (double) (tv2.tv_usec - tv1.tv_usec) / 1000000 + (double) (tv2.tv_sec - tv1.tv_sec));
  if (o.save_res && (o.save_txt || o.save_dat))
  {
    std::string why;
    if (!save_grids (o, ctx, (uint32_t) o.steps, o.scattered_res, why))
      return fail (why);
  }
  return 0;
}
