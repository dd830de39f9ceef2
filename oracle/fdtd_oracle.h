/*
 * fdtd_oracle.h - CPU restatement of the fdtd3d leapfrog time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the parity tests, smoke()
 * and the cpu_baseline leg of bench.py compare the CUDA product against.
 * Nothing in the product (fdtd3d_b200/, include/) links or calls it.
 *
 * It restates, in plain C with the reference's operation order, the
 * E_CENTERED layout of fdtd3d for the Dim3 and Dim2_TMz modes:
 * Yee curl update, PML D/B formulation, Drude ADE (metamaterials), TF/SF
 * correction with the 1-D incident grid, point source, sigma profiles,
 * material averaging and the numerical phase-velocity correction.
 * Pinned against the reference binary built from its own sources
 * (oracle/_ref/fdtd3d) by tests/test_oracle_pin.py.
 */
#ifndef FDTD_ORACLE_H
#define FDTD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct
{
  int mode;                   /* 3 = Dim3, 2 = Dim2_TMz */
  int size[3];                /* grid size; size[2] = 1 for TMz */
  int pml[3];
  int tfsf_left[3];
  int tfsf_right[3];
  double dx;                  /* metres, float-rounded like std::stof */
  double wavelength;          /* metres, float-rounded */
  double courant;             /* float-rounded */
  double angle_teta;          /* degrees, float-rounded */
  double angle_phi;
  double angle_psi;
  int use_pml;
  int use_tfsf;
  int use_metamaterials;
  int point_source[3];
  int point_source_mask;      /* bit c set -> hard source on component c (Ex..Hz) */
  int skip_first_update;      /* 1 = fdtd3d driver (no field update at t == 0) */
  int point_source_kind;      /* 0 = reference sine, 1 = Gaussian-modulated pulse */
  double point_source_bandwidth;
} fdtd_oracle_cfg;

typedef struct fdtd_oracle fdtd_oracle;

/* materials: eps, mu, omegape, omegapm, gammae, gammam; each size-N array
 * (x-major, z fastest) or NULL for the default (1, 1, 0, 0, 0, 0). */
fdtd_oracle *fdtd_oracle_create (const fdtd_oracle_cfg *cfg, const double *const materials[6]);
void fdtd_oracle_destroy (fdtd_oracle *o);
/* advance time steps t_start .. t_start + n - 1 */
void fdtd_oracle_step (fdtd_oracle *o, uint32_t t_start, uint32_t n);
/* copy component c (0..5 = Ex,Ey,Ez,Hx,Hy,Hz) at time level `level` into out
 * (N doubles); returns 0, or -1 if the component does not exist in the mode */
int fdtd_oracle_get (const fdtd_oracle *o, int c, int level, double *out);
/* scalars computed at set-up: [0] dt, [1] frequency, [2] relPhaseVelocity */
void fdtd_oracle_scalars (const fdtd_oracle *o, double out[3]);
/* copy the incident grids at level 1 (length 500*size[0] each) */
void fdtd_oracle_incident (const fdtd_oracle *o, double *einc, double *hinc);

/* 1-D ExHy run of the reference unit-test driver (no t == 0 skip, no PML):
 * size, tfsf size (both sides), dx, lambda, courant, steps; writes Ex
 * level 1 for sine and cosine hard sources (the real and imaginary parts of
 * the reference's complex-valued run). */
void fdtd_oracle_exhy_1d (int size, int tfsf, double dx, double lambda, double courant,
                          uint32_t steps, double *ex_sin, double *ex_cos);

#ifdef __cplusplus
}
#endif

#endif /* FDTD_ORACLE_H */
