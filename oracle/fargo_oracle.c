/*
 * fargo_oracle.c -- CPU restatement of the reference's hydro timestep
 * (MatiasFloresS/CudaProtoplanetaryDisksFloat, AlgoGas and everything it
 * calls).  TEST INFRASTRUCTURE ONLY: the checker of the CUDA path, never part
 * of the product.  See fargo_oracle.h for the two builds.
 *
 * Every function names the reference code it restates (file:line, paths
 * relative to the reference project).  Expression typing follows the
 * reference: a float operand meeting a double literal (2.0, 0.5, PI, 1e-20 ...)
 * is promoted to double and the result rounded back on assignment, exactly as
 * nvcc compiles the reference's kernels.  In the f64 build "real" is double
 * throughout.
 *
 * Deviations, all deliberate:
 *   - Force, Hill-mass and lost-mass sums accumulate in double (the reference
 *     sums the FP32 per-cell values with an FP32 tree, Kernels.cu:270-557);
 *     the per-cell values themselves are the reference's.
 *   - Uninitialised host table entries of the reference (Rmed[NRAD], ...,
 *     SourceEuler.cu:139-157) are 0 here; the reference multiplies Rmed[NRAD]
 *     by a zero slope (Kernels.cu:941), so the value never matters.
 *   - Update_sgvelocityKernel reads SG_Acct[-1] for ring 0, sector 0
 *     (Kernels.cu:1039); here that one read takes the last sector of ring 0.
 */
#include "fargo_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORC_F64
typedef double real;
#define RSQRT sqrt
#define REXP exp
#define RLOG log
#define RPOW pow
#define RCOS cos
#define RSIN sin
#define RFABS fabs
#define RCOSH cosh
#else
typedef float real;
#define RSQRT sqrtf
#define REXP expf
#define RLOG logf
#define RPOW powf
#define RCOS cosf
#define RSIN sinf
#define RFABS fabsf
#define RCOSH coshf
#endif

/* Fondam.cuh:1-10 */
#define G 1.0
#define PI 3.14159265358979323844
#define MU 1.0
#define RGAS 1.0
#define CFLSECURITY 0.5
#define CVNR 1.41

#define YES 1
#define NO 0

#define MAXSUB 4096

typedef struct { real x, y; } pairr;

struct orc {
  fargo_params p;
  int nrad, nsec, size_grid;
  /* 1-D tables, NRAD+1 entries (SourceEuler.cu:88-104) */
  double *Radii2, *Rmed2;
  real *Radii, *Rinf, *Rsup, *Rmed, *Surf, *invRinf, *invSurf, *invRmed, *invdiffRsup,
      *invdiffRmed, *powRmed;
  real *SigmaMed, *SigmaInf, *EnergyMed, *CoolingTimeMed, *QplusMed, *viscosity_array;
  real *supp_torque, *dxtheta, *GLOBAL_bufarray, *GLOBAL_AxiSGAccr;
  real *Vmoy, *newDT, *DT1D, *VMed;
  int *Nshift;
  /* grid fields, (NRAD+1)*NSEC */
  real *Dens, *Vrad, *Vtheta, *Energy, *SoundSpeed, *Pressure, *Temperature, *Potential;
  real *VradInt, *VthetaInt, *VradNew, *VthetaNew, *EnergyInt, *EnergyNew, *DensInt, *TemperInt;
  real *DRR, *DPP, *DRP, *DivergenceVelocity, *TAURR, *TAUPP, *TAURP, *Qplus;
  real *CellAbscissa, *CellOrdinate;
  real *RadMomP, *RadMomM, *ThetaMomP, *ThetaMomM, *Work, *QRStar, *DensStar, *dq, *VthetaRes,
      *TempShift, *LostByDisk;
  /* self-gravity */
  real *Kr_aux, *Kt_aux, *SG_Accr, *SG_Acct;
  double *Kr_hat, *Kt_hat; /* FFT of the kernels, complex interleaved, 2*NRAD*NSEC */
  double *cbuf0, *cbuf1;
  real SGP_eps, SGP_rstep, SGP_tstep;
  /* scalars */
  float PhysicalTime, PhysicalTimeInitial, OmegaFrame, MassTaper, HillRadius, LostMass, mdcp1;
  real invdphi, onethird, dphi;
  float Xplanet_mark, Yplanet_mark; /* Psys.cu:79 static float Xplanet, Yplanet */
  int bc_angle[2];                   /* NonReflectingBoundary's i_angle, i_angle2 (last call) */
  fargo_planets sys, sys0;
  pairr DiskOnPrimaryAcceleration, IndirectTerm;
  /* precision mode (orc_set_precision): 0 the reference's arithmetic,
     1 accurate (FP64 star-potential gradient, compensated ring means, FP64
     self-gravity kernel table) */
  int accurate;
  real* star_grad; /* G / (Rmed[i] Rmed[i-1]) from the FP64 radii, accurate mode */
  /* substep log */
  int nsub;
  int* log_nshift;
  double log_dt[MAXSUB];
  int nsub_total;
  double last_dt;
};

static real* zr(size_t n) { return (real*)calloc(n ? n : 1, sizeof(real)); }

/* ------------------------------------------------------------------------ */
/* Small helpers                                                             */
/* ------------------------------------------------------------------------ */

/* Kernels.cu:1459-1470 */
static real max2(real a, real b) { return (b > a) ? b : a; }
static real min2(real a, real b) { return (b < a) ? b : a; }
static real device_reduce(const real* in, int n);

/* AspectRatioDevice, Kernels.cu:1473-1488 (float math on the device). */
static real aspect_ratio_dev(const orc* o, real r) {
  const fargo_params* p = &o->p;
  real aspectratio, rmin, rmax, scale;
  aspectratio = p->ASPECTRATIO;
  rmin = (real)(p->TRANSITIONRADIUS - p->TRANSITIONWIDTH * p->ASPECTRATIO);
  rmax = (real)(p->TRANSITIONRADIUS + p->TRANSITIONWIDTH * p->ASPECTRATIO);
  scale = 1.0 + (o->PhysicalTime - o->PhysicalTimeInitial) * p->LAMBDADOUBLING;
  rmin *= scale;
  rmax *= scale;
  if (r < rmin) aspectratio *= p->TRANSITIONRATIO;
  if ((r >= rmin) && (r <= rmax))
    aspectratio *= REXP((rmax - r) / (rmax - rmin) * RLOG((real)p->TRANSITIONRATIO));
  return aspectratio;
}

/* AspectRatioHost, Viscosity.cu:39-52 (double math on the host). */
static real aspect_ratio_host(const orc* o, real r) {
  const fargo_params* p = &o->p;
  real aspectratio, rmin, rmax, scale;
  aspectratio = p->ASPECTRATIO;
  rmin = (real)(p->TRANSITIONRADIUS - p->TRANSITIONWIDTH * p->ASPECTRATIO);
  rmax = (real)(p->TRANSITIONRADIUS + p->TRANSITIONWIDTH * p->ASPECTRATIO);
  scale = 1.0 + (o->PhysicalTime - o->PhysicalTimeInitial) * p->LAMBDADOUBLING;
  rmin *= scale;
  rmax *= scale;
  if (r < rmin) aspectratio *= p->TRANSITIONRATIO;
  if ((r >= rmin) && (r <= rmax))
    aspectratio *= exp((rmax - r) / (rmax - rmin) * log(p->TRANSITIONRATIO));
  return aspectratio;
}

/* FViscosity, Viscosity.cu:19-37. */
static real fviscosity(const orc* o, real r) {
  const fargo_params* p = &o->p;
  real viscosity, rmin, rmax, scale;
  int i = 0;
  viscosity = p->VISCOSITY;
  if (p->ViscosityAlpha) {
    while (o->Rmed[i] < r) i++;
    viscosity = p->ALPHAVISCOSITY * o->GLOBAL_bufarray[i] * o->GLOBAL_bufarray[i] * pow(r, 1.5);
  }
  rmin = (real)(p->CAVITYRADIUS - p->CAVITYWIDTH * p->ASPECTRATIO);
  rmax = (real)(p->CAVITYRADIUS + p->CAVITYWIDTH * p->ASPECTRATIO);
  scale = 1.0 + (o->PhysicalTime - o->PhysicalTimeInitial) * p->LAMBDADOUBLING;
  rmin *= scale;
  rmax *= scale;
  if (r < rmin) viscosity *= p->CAVITYRATIO;
  if ((r >= rmin) && (r <= rmax)) viscosity *= exp((rmax - r) / (rmax - rmin) * log(p->CAVITYRATIO));
  return viscosity;
}

/* Compute_smoothing, Force.cu:69-74. */
static double compute_smoothing(const orc* o, double r) {
  return o->p.THICKNESSSMOOTHING * aspect_ratio_host(o, (real)r) * pow(r, 1.0 + o->p.FLARINGINDEX);
}

/* Sigma / Energy / CoolingTime / Qplusinit, Theo.cu:13-78. */
static real sigma_profile(const orc* o, real r) {
  const fargo_params* p = &o->p;
  real cavity = 1.0;
  if (r < p->CAVITYRADIUS) cavity = 1.0 / p->CAVITYRATIO;
  return cavity * p->ScalingFactor * p->SIGMA0 * pow(r, -p->SIGMASLOPE);
}
static real energy_profile(const orc* o, real r) {
  const fargo_params* p = &o->p;
  return RGAS / MU / (p->ADIABATICINDEX - 1.0) * p->SIGMA0 * pow(p->ASPECTRATIO, 2.0) *
         pow(r, -p->SIGMASLOPE - 1.0 + 2.0 * p->FLARINGINDEX);
}
static real cooling_time(const orc* o, real r) {
  return o->p.COOLINGTIME0 * pow(r, 2.0 + 2.0 * o->p.FLARINGINDEX);
}
static real qplus_init(const orc* o, real r) {
  real viscosity = fviscosity(o, r);
  return 2.25 * viscosity * o->p.SIGMA0 * pow(r, -o->p.SIGMASLOPE - 3.0);
}

/* Serial ring mean of a grid field: Make1DprofileKernel (Kernels.cu:726-738),
   ComputeAverageThetaVelocitiesKernel (Kernels.cu:1177-1188) and
   ConditionCFLKernel1D (Kernels.cu:1363-1377) all add the sectors one by one
   in order into one float. */
static void ring_mean(const orc* o, const real* f, real* out) {
  int nsec = o->nsec;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < o->nrad; i++) {
    real moy = 0.0;
    if (o->accurate) {
      /* accurate mode: Kahan-compensated sum in the same order */
      real comp = 0.0;
      for (int j = 0; j < nsec; j++) {
        real y = f[i * nsec + j] - comp;
        real t = moy + y;
        comp = (t - moy) - y;
        moy = t;
      }
    } else {
      for (int j = 0; j < nsec; j++) moy += f[i * nsec + j];
    }
    out[i] = moy / (real)nsec;
  }
}

/* ------------------------------------------------------------------------ */
/* Setup                                                                    */
/* ------------------------------------------------------------------------ */

/* FillPolar1DArrays, SourceEuler.cu:76-157 (used_rad.dat is written by the
   driver, not here). */
static void fill_polar_1d(orc* o, const double* radii_in) {
  const fargo_params* p = &o->p;
  int NRAD = o->nrad, NSEC = o->nsec, i;
  float drrsep = (p->RMAX - p->RMIN) / (float)NRAD;
  for (i = 0; i <= NRAD; i++) {
    if (radii_in)
      o->Radii2[i] = radii_in[i];
    else if (p->LogGrid == YES)
      o->Radii2[i] = (double)p->RMIN * exp((double)i / (double)NRAD * log((double)p->RMAX / (double)p->RMIN));
    else
      o->Radii2[i] = p->RMIN + drrsep * (double)i;
    o->Radii[i] = (real)o->Radii2[i];
  }
  for (i = 0; i < NRAD; i++) {
    double* R2 = o->Radii2;
    o->Rinf[i] = R2[i];
    o->Rsup[i] = R2[i + 1];
    o->Rmed2[i] = 2.0 / 3.0 * (R2[i + 1] * R2[i + 1] * R2[i + 1] - R2[i] * R2[i] * R2[i]);
    o->Rmed2[i] = o->Rmed2[i] / (R2[i + 1] * R2[i + 1] - R2[i] * R2[i]);
    o->Rmed[i] = o->Rmed2[i];
    o->Surf[i] = PI * (R2[i + 1] * R2[i + 1] - R2[i] * R2[i]) / (double)NSEC;
    o->invRmed[i] = 1.0 / o->Rmed2[i];
    o->invSurf[i] = 1.0 / o->Surf[i];
    o->invdiffRsup[i] = 1.0 / (R2[i + 1] - R2[i]);
    o->invRinf[i] = 1.0 / R2[i];
  }
  o->Rinf[NRAD] = o->Radii2[NRAD];
  for (i = 0; i < NRAD; i++) {
    if (i > 0) o->invdiffRmed[i] = 1.0 / (o->Rmed2[i] - o->Rmed2[i - 1]);
    o->powRmed[i] = pow(o->Rmed2[i], -2.5 + p->SIGMASLOPE);
  }
}

/* Main.cu:259-268: dphi, invdphi, onethird, supp_torque, dxtheta. */
static void fill_misc_tables(orc* o) {
  const fargo_params* p = &o->p;
  o->dphi = 2.0 * PI / (float)o->nsec;
  o->invdphi = 1.0 / o->dphi;
  o->onethird = 1.0 / 3.0;
  for (int i = 0; i < o->nrad; i++) {
    o->supp_torque[i] = p->IMPOSEDDISKDRIFT * 0.5 * pow(o->Rmed[i], -2.5 + p->SIGMASLOPE);
    o->dxtheta[i] = 2.0 * PI / (float)o->nsec * o->Rmed[i];
  }
}

/* InitComputeAccelKernel, Kernels.cu:164-173. */
static void init_cell_coords(orc* o) {
  int nsec = o->nsec;
  for (int i = 0; i < o->nrad; i++)
    for (int j = 0; j < nsec; j++) {
      o->CellAbscissa[i * nsec + j] = o->Rmed[i] * RCOS(2.0 * PI * (float)j / (float)nsec);
      o->CellOrdinate[i * nsec + j] = o->Rmed[i] * RSIN(2.0 * PI * (float)j / (float)nsec);
    }
}

/* ComputeSoundSpeedKernel, Kernels.cu:176-193. */
static void compute_sound_speed(orc* o) {
  const fargo_params* p = &o->p;
  int nsec = o->nsec;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < o->nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j;
      if (!p->Adiabatic) {
        real ar = aspect_ratio_dev(o, o->Rmed[i]);
        o->SoundSpeed[l] = ar * RSQRT(G * 1.0 / o->Rmed[i]) * RPOW(o->Rmed[i], p->FLARINGINDEX);
      } else {
        o->SoundSpeed[l] =
            RSQRT(p->ADIABATICINDEX * (p->ADIABATICINDEX - 1.0) * o->Energy[l] / o->Dens[l]);
      }
    }
}

/* ComputePressureFieldKernel, Kernels.cu:196-208. */
static void compute_pressure(orc* o) {
  const fargo_params* p = &o->p;
  int n = o->nrad * o->nsec;
#pragma omp parallel for schedule(static)
  for (int l = 0; l < n; l++) {
    if (!p->Adiabatic)
      o->Pressure[l] = o->Dens[l] * o->SoundSpeed[l] * o->SoundSpeed[l];
    else
      o->Pressure[l] = (p->ADIABATICINDEX - 1.0) * o->Energy[l];
  }
}

/* ComputeTemperatureFieldKernel, Kernels.cu:211-223. */
static void compute_temperature(orc* o) {
  const fargo_params* p = &o->p;
  int n = o->nrad * o->nsec;
#pragma omp parallel for schedule(static)
  for (int l = 0; l < n; l++) {
    if (!p->Adiabatic)
      o->Temperature[l] = MU / RGAS * o->Pressure[l] / o->Dens[l];
    else
      o->Temperature[l] = MU / RGAS * (p->ADIABATICINDEX - 1.0) * o->Energy[l] / o->Dens[l];
  }
}

/* Viscosity table as ComputeViscousTerms rebuilds it (Viscosity.cu:79-86):
   ring-mean sound speed first when the viscosity is of alpha type. */
static void refresh_viscosity(orc* o) {
  if (o->p.ViscosityAlpha) ring_mean(o, o->SoundSpeed, o->GLOBAL_bufarray);
  for (int i = 0; i < o->nrad; i++) o->viscosity_array[i] = fviscosity(o, o->Rmed[i]);
}

/* InitGasVelocitiesKernel, Kernels.cu:759-800.  The kernel's ViscosityAlpha
   argument is the int global read through an `extern float` declaration
   (Pframeforce.cu:20): 1 becomes 1.4e-45f, converted to int 0, so the kernel
   always takes its constant-viscosity branch. */
static void init_gas_velocities_kernel(orc* o) {
  const fargo_params* p = &o->p;
  int nrad = o->nrad, nsec = o->nsec;
  for (int i = 0; i <= nrad; i++)
    for (int j = 0; j < nsec; j++) {
      real omega, r, ri;
      int l = i * nsec + j;
      if (i == nrad) {
        r = o->Rmed[nrad - 1];
        ri = o->Rinf[nrad - 1];
      } else {
        r = o->Rmed[i];
        ri = o->Rinf[i];
      }
      if (!p->SelfGravity) {
        omega = RSQRT(G * 1.0 / r / r / r);
        o->Vtheta[l] = omega * r *
                       RSQRT(1.0 - RPOW(p->ASPECTRATIO, 2.0) * RPOW(r, 2.0 * p->FLARINGINDEX) *
                                       (1. + p->SIGMASLOPE - 2.0 * p->FLARINGINDEX));
      }
      o->Vtheta[l] -= o->OmegaFrame * r;
      if (i == nrad)
        o->Vrad[l] = 0.0;
      else {
        o->Vrad[l] = p->IMPOSEDDISKDRIFT * p->SIGMA0 / o->SigmaInf[i] / ri;
        o->Vrad[l] -= 3.0 * o->viscosity_array[i] / r * (-p->SIGMASLOPE + .5);
      }
    }
  for (int j = 0; j < nsec; j++) o->Vrad[j] = o->Vrad[nrad * nsec + j] = 0.0;
}

/* ------------------------------------------------------------------------ */
/* Self-gravity: log-polar convolution (SgMain.cu:23-162)                   */
/* ------------------------------------------------------------------------ */

/* In-place complex DFT of length n with stride s (mixed radix 2/3/5, O(n^2)
   fallback for other factors), double precision.  sign = -1 forward. */
static void dft_1d(double* a, int n, int s, int sign, double* tmp) {
  if (n == 1) return;
  int radix = 0;
  if (n % 2 == 0) radix = 2;
  else if (n % 3 == 0) radix = 3;
  else if (n % 5 == 0) radix = 5;
  if (!radix) {
    for (int k = 0; k < n; k++) {
      double re = 0, im = 0;
      for (int t = 0; t < n; t++) {
        double ang = sign * 2.0 * PI * (double)((long)k * t % n) / n;
        double c = cos(ang), sn = sin(ang);
        double xr = a[2 * t * s], xi = a[2 * t * s + 1];
        re += xr * c - xi * sn;
        im += xr * sn + xi * c;
      }
      tmp[2 * k] = re;
      tmp[2 * k + 1] = im;
    }
    for (int k = 0; k < n; k++) {
      a[2 * k * s] = tmp[2 * k];
      a[2 * k * s + 1] = tmp[2 * k + 1];
    }
    return;
  }
  int m = n / radix;
  /* split into radix sub-sequences, transform each */
  double* sub = (double*)malloc(sizeof(double) * 2 * n);
  for (int r = 0; r < radix; r++)
    for (int t = 0; t < m; t++) {
      sub[2 * (r * m + t)] = a[2 * (t * radix + r) * s];
      sub[2 * (r * m + t) + 1] = a[2 * (t * radix + r) * s + 1];
    }
  for (int r = 0; r < radix; r++) dft_1d(sub + 2 * r * m, m, 1, sign, tmp);
  for (int k = 0; k < n; k++) {
    double re = 0, im = 0;
    for (int r = 0; r < radix; r++) {
      double ang = sign * 2.0 * PI * (double)((long)r * k % n) / n;
      double c = cos(ang), sn = sin(ang);
      double xr = sub[2 * (r * m + k % m)], xi = sub[2 * (r * m + k % m) + 1];
      re += xr * c - xi * sn;
      im += xr * sn + xi * c;
    }
    a[2 * k * s] = re;
    a[2 * k * s + 1] = im;
  }
  free(sub);
}

/* 2-D C2C transform of a (2*NRAD) x NSEC array, unnormalised (cufftPlan2d +
   cufftExecC2C as Main.cu:186-196 and SgMain.cu:115-162 use them). */
static void fft2d(orc* o, double* a, int sign) {
  int nx = 2 * o->nrad, ny = o->nsec;
#pragma omp parallel
  {
    double* tmp = (double*)malloc(sizeof(double) * 2 * (nx > ny ? nx : ny));
#pragma omp for schedule(static)
    for (int i = 0; i < nx; i++) dft_1d(a + 2 * (size_t)i * ny, ny, 1, sign, tmp);
#pragma omp for schedule(static)
    for (int j = 0; j < ny; j++) dft_1d(a + 2 * j, nx, ny, sign, tmp);
    free(tmp);
  }
}

/* compute_kernel, SgMain.cu:49-81 (host float math), then the forward FFTs
   of Kr and Kt that the reference repeats every call (SgMain.cu:124,138). */
static void sg_init_kernel(orc* o) {
  int NRAD = o->nrad, NSEC = o->nsec;
  real u, theta, Kr, Kt, base;
  for (int i = 0; i < 2 * NRAD; i++) {
    if (i < NRAD)
      u = RLOG(o->Radii[i] / o->Radii[0]);
    else
      u = -RLOG(o->Radii[2 * NRAD - i] / o->Radii[0]);
    for (int j = 0; j < NSEC; j++) {
      theta = 2.0 * PI * (float)j / (float)NSEC;
      Kr = 1.0 + o->SGP_eps * o->SGP_eps - RCOS(theta) * REXP(-u);
      base = o->SGP_eps * o->SGP_eps * REXP(u) + 2.0 * (RCOSH(u) - RCOS(theta));
      Kr *= RPOW(base, -1.5);
      Kt = RSIN(theta);
      Kt *= RPOW(base, -1.5);
      o->Kr_aux[i * NSEC + j] = Kr;
      o->Kt_aux[i * NSEC + j] = Kt;
    }
  }
  size_t n = (size_t)2 * NRAD * NSEC;
  for (size_t l = 0; l < n; l++) {
    o->Kr_hat[2 * l] = o->Kr_aux[l];
    o->Kr_hat[2 * l + 1] = 0;
    o->Kt_hat[2 * l] = o->Kt_aux[l];
    o->Kt_hat[2 * l + 1] = 0;
  }
  if (o->accurate) {
    /* accurate mode: the same kernel tabulated in FP64 from the FP64 radii */
    double eps = o->SGP_eps;
    for (int i = 0; i < 2 * NRAD; i++) {
      double ud = i < NRAD ? log(o->Radii2[i] / o->Radii2[0]) : -log(o->Radii2[2 * NRAD - i] / o->Radii2[0]);
      for (int j = 0; j < NSEC; j++) {
        double th = 2.0 * PI * (double)j / (double)NSEC;
        double b = eps * eps * exp(ud) + 2.0 * (cosh(ud) - cos(th));
        size_t l = (size_t)i * NSEC + j;
        o->Kr_hat[2 * l] = (1.0 + eps * eps - cos(th) * exp(-ud)) * pow(b, -1.5);
        o->Kt_hat[2 * l] = sin(th) * pow(b, -1.5);
      }
    }
  }
  fft2d(o, o->Kr_hat, -1);
  fft2d(o, o->Kt_hat, -1);
}

/* compute_selfgravity (SgMain.cu:23-45): ComputeFFTKernel (Kernels.cu:949-977),
   forward FFTs, ComputeConvolutionKernel (Kernels.cu:980-999), inverse FFTs,
   ComputeSgAccKernel (Kernels.cu:1002-1021); the FFT runs in double here. */
static void sg_accelerations(orc* o) {
  int nrad = o->nrad, nsec = o->nsec;
  size_t n2 = (size_t)2 * nrad * nsec;
  double *Sr = o->cbuf0, *St = o->cbuf1;
  for (int i = 0; i < 2 * nrad; i++)
    for (int j = 0; j < nsec; j++) {
      size_t l = (size_t)i * nsec + j;
      real var;
      if (i < nrad) {
        var = o->Dens[l] * RSQRT(o->Rmed[i] / o->Rmed[0]);
        Sr[2 * l] = var;
        St[2 * l] = (real)(var * o->Rmed[i] / o->Rmed[0]);
      } else {
        Sr[2 * l] = 0.;
        St[2 * l] = 0.;
      }
      Sr[2 * l + 1] = 0.;
      St[2 * l + 1] = 0.;
    }
  fft2d(o, St, -1);
  fft2d(o, Sr, -1);
  for (size_t l = 0; l < n2; l++) {
    double ktr = o->Kt_hat[2 * l], kti = o->Kt_hat[2 * l + 1];
    double krr = o->Kr_hat[2 * l], kri = o->Kr_hat[2 * l + 1];
    double str = St[2 * l], sti = St[2 * l + 1], srr = Sr[2 * l], sri = Sr[2 * l + 1];
    St[2 * l] = -G * (ktr * str - kti * sti);
    St[2 * l + 1] = -G * (ktr * sti + kti * str);
    Sr[2 * l] = -G * (krr * srr - kri * sri);
    Sr[2 * l + 1] = -G * (krr * sri + kri * srr);
  }
  fft2d(o, St, +1); /* Gphi */
  fft2d(o, Sr, +1); /* Gr */
  for (int i = 0; i < nrad; i++) {
    real normaccr, normacct, divRmed;
    divRmed = o->Rmed[i] / o->Rmed[0];
    normaccr = o->SGP_rstep * o->SGP_tstep / ((float)(2 * nrad) * (float)nsec);
    normacct = normaccr;
    normaccr /= RSQRT(divRmed);
    normacct /= (divRmed * RSQRT(divRmed));
    for (int j = 0; j < nsec; j++) {
      size_t l = (size_t)i * nsec + j;
      o->SG_Acct[l] = (real)St[2 * l] * normacct;
      o->SG_Accr[l] = (real)Sr[2 * l] * normaccr;
      o->SG_Accr[l] += G * o->Dens[l] * o->SGP_rstep * o->SGP_tstep / o->SGP_eps;
    }
  }
}

/* Update_sgvelocityKernel, Kernels.cu:1024-1041, on VradInt/VthetaInt
   (Substep1 copies them through Vradial/Vazimutal, SourceEuler.cu:319-329). */
static void sg_kick(orc* o, real dt) {
  int nrad = o->nrad, nsec = o->nsec;
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j;
      if (i > 0)
        o->VradInt[l] += dt * ((o->Rinf[i] - o->Rmed[i - 1]) * o->SG_Accr[l] +
                               (o->Rmed[i] - o->Rinf[i]) * o->SG_Accr[(i - 1) * nsec + j]) *
                         o->invdiffRmed[i];
      /* reference index i*nsec + (j-1)%nsec: ring i-1's last sector when j=0 */
      int lm = (j > 0) ? l - 1 : (i > 0 ? l - 1 : nsec - 1);
      o->VthetaInt[l] += 0.5 * dt * (o->SG_Acct[l] + o->SG_Acct[lm]);
    }
}

/* Init_azimutalvelocity_withSG (SourceEuler.cu:428-437) with
   Azimutalvelocity_withSGKernel (Kernels.cu:1044-1059). */
static void init_vtheta_with_sg(orc* o) {
  const fargo_params* p = &o->p;
  int nrad = o->nrad, nsec = o->nsec;
  ring_mean(o, o->SG_Accr, o->GLOBAL_AxiSGAccr);
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      real omegakep, omega, invr;
      invr = 1. / o->Rmed[i];
      omegakep = RSQRT(G * 1.0 * invr * invr * invr);
      omega = RSQRT(omegakep * omegakep *
                        (1.0 - (1. + p->SIGMASLOPE - 2.0 * p->FLARINGINDEX) * RPOW(p->ASPECTRATIO, 2.0) *
                                   RPOW(o->Rmed[i], 2.0 * p->FLARINGINDEX)) -
                    invr * o->GLOBAL_AxiSGAccr[i]);
      o->Vtheta[i * nsec + j] = o->Rmed[i] * omega;
    }
}

/* Init_planetarysys_withSG, SgMain.cu:166-195. */
static void init_planets_with_sg(orc* o) {
  ring_mean(o, o->SG_Accr, o->GLOBAL_AxiSGAccr);
  for (int k = 0; k < o->sys.nb; k++) {
    real r, dist, ri, rip1, dr, sgacc;
    int ipl;
    r = o->sys.x[k];
    dist = (real)(r / (1. + o->p.ECCENTRICITY));
    ipl = 0;
    while (o->Rmed[ipl] <= dist) ipl++;
    ri = o->Rmed[ipl];
    rip1 = o->Rmed[ipl + 1];
    dr = rip1 - ri;
    sgacc = (dist - ri) * o->GLOBAL_AxiSGAccr[ipl + 1] + (rip1 - dist) * o->GLOBAL_AxiSGAccr[ipl];
    sgacc /= dr;
    o->sys.vy[k] *= (real)RSQRT(1. - dist * dist * sgacc);
  }
}

/* ------------------------------------------------------------------------ */
/* Planets (host FP64 in the reference)                                     */
/* ------------------------------------------------------------------------ */

/* DerivMotionRK5, RungeKutta.cu:9-46 (planet-planet term uses the star
   distance of the perturber, as the reference does). */
static void deriv_motion_rk5(const orc* o, const double* q_init, const double* masses, double* deriv,
                             int nb, float dt, const int* feelothers) {
  const double *x = q_init, *y = x + nb, *vx = y + nb, *vy = vx + nb;
  double *derivx = deriv, *derivy = derivx + nb, *derivvx = derivy + nb, *derivvy = derivvx + nb;
  double Dist[FARGO_MAXPLANETS];
  for (int i = 0; i < nb; i++) Dist[i] = sqrt(x[i] * x[i] + y[i] * y[i]);
  for (int i = 0; i < nb; i++) {
    derivx[i] = vx[i];
    derivy[i] = vy[i];
    derivvx[i] = -G * 1.0 / Dist[i] / Dist[i] / Dist[i] * x[i];
    derivvy[i] = -G * 1.0 / Dist[i] / Dist[i] / Dist[i] * y[i];
    for (int j = 0; j < nb; j++) {
      if (o->p.Indirect_Term == YES) {
        derivvx[i] -= G * masses[j] / Dist[j] / Dist[j] / Dist[j] * x[j];
        derivvy[i] -= G * masses[j] / Dist[j] / Dist[j] / Dist[j] * y[j];
      }
      if ((j != i) && (feelothers[i] == YES)) {
        derivvx[i] += G * masses[j] / Dist[j] / Dist[j] / Dist[j] * (x[j] - x[i]);
        derivvy[i] += G * masses[j] / Dist[j] / Dist[j] / Dist[j] * (y[j] - y[i]);
      }
    }
  }
  for (int i = 0; i < 4 * nb; i++) deriv[i] *= dt;
}

/* RungeKutta + TranslatePlanetRK5, RungeKutta.cu:48-74. */
static void runge_kutta(const orc* o, const double* q0, float timestep, const double* masses, double* q1,
                        int nb, const int* feelothers) {
  static const double c[5][5] = {{0.2, 0.0, 0.0, 0.0, 0.0},
                                 {0.075, 0.225, 0.0, 0.0, 0.0},
                                 {0.3, -0.9, 1.2, 0.0, 0.0},
                                 {-11.0 / 54.0, 2.5, -70.0 / 27.0, 35.0 / 27.0, 0.0},
                                 {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0,
                                  253.0 / 4096.0}};
  double k[6][4 * FARGO_MAXPLANETS];
  memset(k, 0, sizeof(k));
  deriv_motion_rk5(o, q0, masses, k[0], nb, timestep, feelothers);
  for (int s = 0; s < 5; s++) {
    for (int i = 0; i < 4 * nb; i++)
      q1[i] = q0[i] + c[s][0] * k[0][i] + c[s][1] * k[1][i] + c[s][2] * k[2][i] + c[s][3] * k[3][i] +
              c[s][4] * k[4][i];
    deriv_motion_rk5(o, q1, masses, k[s + 1], nb, timestep, feelothers);
  }
  for (int i = 0; i < 4 * nb; i++)
    q1[i] = q0[i] + 37.0 / 378.0 * k[0][i] + 250.0 / 621.0 * k[2][i] + 125.0 / 594.0 * k[3][i] +
            512.0 / 1771.0 * k[5][i];
}

/* AdvanceSystemRK5, Pframeforce.cu:94-157. */
static void advance_system_rk5(orc* o, float dt) {
  fargo_planets* sys = &o->sys;
  const fargo_params* p = &o->p;
  int nb = sys->nb;
  double q0[4 * FARGO_MAXPLANETS], q1[4 * FARGO_MAXPLANETS];
  double dtheta, omega, rdot, x, y, r, new_r, vx, vy, theta, denom;
  if (!p->ForcedCircular) {
    for (int k = 0; k < nb; k++) {
      q0[k] = sys->x[k];
      q0[k + nb] = sys->y[k];
      q0[k + 2 * nb] = sys->vx[k];
      q0[k + 3 * nb] = sys->vy[k];
    }
    runge_kutta(o, q0, dt, sys->mass, q1, nb, sys->feelothers);
  }
  for (int i = 1 - (o->PhysicalTime >= p->RELEASEDATE); i < nb; i++) {
    if (!p->ForcedCircular) {
      sys->x[i] = q1[i];
      sys->y[i] = q1[i + nb];
      sys->vx[i] = q1[i + 2 * nb];
      sys->vy[i] = q1[i + 3 * nb];
    } else {
      x = sys->x[i];
      y = sys->y[i];
      theta = atan2(y, x);
      vx = sys->vx[i];
      vy = sys->vy[i];
      r = sqrt(x * x + y * y);
      omega = (-y * vx + x * vy) / r / r;
      dtheta = omega * dt;
      sys->x[i] = r * cos(theta + dtheta);
      sys->y[i] = r * sin(theta + dtheta);
      sys->vx[i] = vx * cos(dtheta + theta) - vy * sin(dtheta + theta);
      sys->vy[i] = vx * sin(dtheta + theta) + vy * cos(dtheta + theta);
    }
  }
  if (o->PhysicalTime < p->RELEASEDATE) {
    x = sys->x[0];
    y = sys->y[0];
    r = sqrt(x * x + y * y);
    theta = atan2(y, x);
    rdot = (p->RELEASERADIUS - r) / (p->RELEASEDATE - o->PhysicalTime);
    omega = sqrt((1. + sys->mass[0]) / r / r / r);
    new_r = r + rdot * dt;
    denom = r - new_r;
    if (denom != 0.0)
      dtheta = 2. * dt * r * omega / denom * (sqrt(r / new_r) - 1.);
    else
      dtheta = omega * dt;
    vx = rdot;
    vy = new_r * sqrt((1. + sys->mass[0]) / new_r / new_r / new_r);
    sys->x[0] = new_r * cos(dtheta + theta);
    sys->y[0] = new_r * sin(dtheta + theta);
    sys->vx[0] = vx * cos(dtheta + theta) - vy * sin(dtheta + theta);
    sys->vy[0] = vx * sin(dtheta + theta) + vx * cos(dtheta + theta);
  }
}

/* GetPsysInfo, Psys.cu:236-306. */
static float get_psys_info(orc* o, int action) {
  const fargo_planets* sys = &o->sys;
  double d1, d2, cross;
  double x, y, vx, vy, m, h, d, Ax, Ay, e, a, E, M;
  double xc, yc, vxc, vyc, omega;
  double arg, PerihelionPA;
  xc = x = sys->x[0];
  yc = y = sys->y[0];
  vxc = vx = sys->vx[0];
  vyc = vy = sys->vy[0];
  m = sys->mass[0] + 1.;
  h = x * vy - y * vx;
  d = sqrt(x * x + y * y);
  Ax = x * vy * vy - y * vx * vy - G * m * x / d;
  Ay = y * vx * vx - x * vx * vy - G * m * y / d;
  e = sqrt(Ax * Ax + Ay * Ay) / m;
  a = h * h / G / m / (1. - e * e);
  if (e == 0.0)
    arg = 1.0;
  else
    arg = (1.0 - d / a) / e;
  if (fabs(arg) >= 1.0)
    E = PI * (1. - arg / fabs(arg)) / 2.;
  else
    E = acos((1.0 - d / a) / e);
  if ((x * y * (vy * vy - vx * vx) + vx * vy * (x * x - y * y)) < 0) E = -E;
  M = E - e * sin(E);
  omega = sqrt(m / a / a / a);
  PerihelionPA = atan2(Ay, Ax);
  if (o->p.GuidingCenter == YES) {
    xc = a * cos(M + PerihelionPA);
    yc = a * sin(M + PerihelionPA);
    vxc = -a * omega * sin(M + PerihelionPA);
    vyc = a * omega * cos(M + PerihelionPA);
  }
  if (e < 1e-8) {
    xc = x;
    yc = y;
    vxc = vx;
    vyc = vy;
  }
  (void)vxc;
  (void)vyc;
  switch (action) {
    case 1:
      o->Xplanet_mark = xc;
      o->Yplanet_mark = yc;
      return 0.;
    case 0:
      x = xc;
      y = yc;
      d2 = sqrt(x * x + y * y);
      d1 = sqrt((double)o->Xplanet_mark * o->Xplanet_mark + (double)o->Yplanet_mark * o->Yplanet_mark);
      cross = o->Xplanet_mark * y - x * o->Yplanet_mark;
      o->Xplanet_mark = x;
      o->Yplanet_mark = y;
      return asin(cross / (d1 * d2));
    case 2:
      return omega;
  }
  return 0.0;
}

/* RotatePsys, Psys.cu:308-325 (rotation by -angle). */
static void rotate_psys(orc* o, float angle) {
  fargo_planets* sys = &o->sys;
  double sint = sin(angle), cost = cos(angle), xt, yt;
  for (int i = 0; i < sys->nb; i++) {
    xt = sys->x[i];
    yt = sys->y[i];
    sys->x[i] = xt * cost + yt * sint;
    sys->y[i] = -xt * sint + yt * cost;
    xt = sys->vx[i];
    yt = sys->vy[i];
    sys->vx[i] = xt * cost + yt * sint;
    sys->vy[i] = -xt * sint + yt * cost;
  }
}

/* ------------------------------------------------------------------------ */
/* Disk forces (Force.cu:31-67, ComputeForceKernel Kernels.cu:804-839)      */
/* ------------------------------------------------------------------------ */

/* The four sums (fx inner, fx outer, fy inner, fy outer) of one Hill-cut
   level k for a body at (x, y).  Kernel arguments are floats. */
static void force_level(orc* o, real x, real y, real rsmoothing, real rh, real a, int k, int dimfxy,
                        double out[4]) {
  int nrad = o->nrad, nsec = o->nsec;
  double sxi = 0, sxo = 0, syi = 0, syo = 0;
#pragma omp parallel for reduction(+ : sxi, sxo, syi, syo) schedule(static)
  for (int i = 0; i < nrad; i++) {
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j;
      real cellmass, dx, dy, d2, InvDist3, dist2, distance, hillcutfactor, hill_cut, rhk = rh;
      cellmass = o->Surf[i] * o->Dens[l];
      dx = o->CellAbscissa[l] - x;
      dy = o->CellOrdinate[l] - y;
      d2 = dx * dx + dy * dy;
      dist2 = d2 + rsmoothing * rsmoothing;
      distance = RSQRT(dist2);
      InvDist3 = 1.0 / dist2 / distance;
      hillcutfactor = (real)k / (real)(dimfxy - 1);
      if (k != 0) {
        rhk *= hillcutfactor;
        hill_cut = 1. - REXP(-d2 / (rhk * rhk));
      } else
        hill_cut = 1.;
      real fx = G * cellmass * dx * InvDist3 * hill_cut;
      real fy = G * cellmass * dy * InvDist3 * hill_cut;
      if (o->Rmed[i] < a) {
        sxi += fx;
        syi += fy;
      } else {
        sxo += fx;
        syo += fy;
      }
    }
  }
  out[0] = sxi;
  out[1] = sxo;
  out[2] = syi;
  out[3] = syo;
}

/* ComputeForce restricted to the levels ComputeAccel reads (Force.cu:330-337,
   SideEuler.cu:151-164).  Returns the float acceleration pair. */
static pairr compute_accel(orc* o, real x, real y, real rsmoothing, real mass) {
  double a = sqrt((double)x * x + (double)y * y);
  double rh = pow((double)mass / 3., 1. / 3.) * a + 1e-15;
  int dimfxy = FARGO_DIMFXY;
  int k = o->p.ExcludeHill ? dimfxy - 1 : 0;
  double s[4];
  force_level(o, x, y, rsmoothing, (real)rh, (real)a, k, dimfxy, s);
  pairr acc;
  real fxi = s[0], fxo = s[1], fyi = s[2], fyo = s[3];
  acc.x = fxi + fxo;
  acc.y = fyi + fyo;
  return acc;
}

void orc_disk_force(orc* o, double x, double y, double rsmoothing, double mass, int dimfxy,
                    double* globalforce) {
  double a = sqrt(x * x + y * y);
  double rh = pow(mass / 3., 1. / 3.) * a + 1e-15;
  for (int k = 0; k < dimfxy; k++) {
    double s[4];
    force_level(o, (real)x, (real)y, (real)rsmoothing, (real)rh, (real)a, k, dimfxy, s);
    globalforce[k] = s[0];
    globalforce[k + dimfxy] = s[1];
    globalforce[k + 2 * dimfxy] = s[2];
    globalforce[k + 3 * dimfxy] = s[3];
  }
}

/* ------------------------------------------------------------------------ */
/* Potential (FillForcesArrays Pframeforce.cu:27-66, kernel Kernels.cu:1322) */
/* ------------------------------------------------------------------------ */

static void fill_forces_arrays(orc* o) {
  const fargo_params* p = &o->p;
  const fargo_planets* sys = &o->sys;
  int nrad = o->nrad, nsec = o->nsec;
  /* ComputeIndirectTerm, Pframeforce.cu:27-35 */
  o->IndirectTerm.x = -o->DiskOnPrimaryAcceleration.x;
  o->IndirectTerm.y = -o->DiskOnPrimaryAcceleration.y;
  if (!p->Indirect_Term) {
    o->IndirectTerm.x = 0.0;
    o->IndirectTerm.y = 0.0;
  }
  memset(o->Potential, 0, sizeof(real) * o->size_grid);
  for (int k = 0; k < sys->nb; k++) {
    double xplanet = sys->x[k], yplanet = sys->y[k], mplanet = sys->mass[k] * o->MassTaper;
    double PlanetDistance = sqrt(xplanet * xplanet + yplanet * yplanet);
    double InvPlanetDistance3 = 1.0 / PlanetDistance / PlanetDistance / PlanetDistance;
    double RRoche = PlanetDistance * pow((1.0 / 3.0 * mplanet), 1.0 / 3.0);
    double smoothing = p->RocheSmoothing ? RRoche * p->ROCHESMOOTHING : compute_smoothing(o, PlanetDistance);
    double smooth = smoothing * smoothing;
    /* kernel arguments are floats */
    real xp = xplanet, yp = yplanet, sm = smooth, mp = mplanet, ipd3 = InvPlanetDistance3;
    real itx = o->IndirectTerm.x, ity = o->IndirectTerm.y;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nrad; i++)
      for (int j = 0; j < nsec; j++) {
        real InvDistance, angle, x, y, distance, distancesmooth, pot;
        InvDistance = 1.0 / o->Rmed[i];
        angle = (real)j / (real)nsec * 2.0 * PI;
        x = o->Rmed[i] * RCOS(angle);
        y = o->Rmed[i] * RSIN(angle);
        distance = (x - xp) * (x - xp) + (y - yp) * (y - yp);
        distancesmooth = RSQRT(distance + sm);
        pot = -G * mp / distancesmooth;
        if (p->Indirect_Term) pot += G * mp * ipd3 * (x * xp + y * yp);
        o->Potential[i * nsec + j] += pot;
        if (k == 0) {
          /* accurate mode: the star's -G/r enters Substep1 as its exact
             radial difference (star_grad) instead */
          pot = o->accurate ? 0.0 : -G * 1.0 * InvDistance;
          pot -= itx * x + ity * y;
          o->Potential[i * nsec + j] += pot;
        }
      }
  }
}

/* AdvanceSystemFromDisk, Pframeforce.cu:68-92 (ComputeAccel takes floats). */
static void advance_system_from_disk(orc* o, float dt) {
  const fargo_params* p = &o->p;
  fargo_planets* sys = &o->sys;
  for (int k = 0; k < sys->nb; k++) {
    if (sys->feeldisk[k]) {
      double m = sys->mass[k], x = sys->x[k], y = sys->y[k], r = sqrt(x * x + y * y), smoothing;
      if (p->RocheSmoothing)
        smoothing = r * pow(m / 3., 1. / 3.) * p->ROCHESMOOTHING;
      else
        smoothing = compute_smoothing(o, r);
      pairr gamma = compute_accel(o, (real)x, (real)y, (real)smoothing, (real)m);
      sys->vx[k] += (real)(dt * gamma.x);
      sys->vy[k] += (real)(dt * gamma.y);
      sys->vx[k] += (real)(dt * o->IndirectTerm.x);
      sys->vy[k] += (real)(dt * o->IndirectTerm.y);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* CFL (ConditionCFL SourceEuler.cu:494-536, kernels Kernels.cu:1363-1429)  */
/* ------------------------------------------------------------------------ */

static int condition_cfl(orc* o, float DeltaT) {
  const fargo_params* p = &o->p;
  int nrad = o->nrad, nsec = o->nsec;
  ring_mean(o, o->Vtheta, o->Vmoy);
#pragma omp parallel for schedule(static)
  for (int i = 1; i < nrad; i++) {
    real newdt = 1e30;
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j;
      real dxrad, invdt1, invdt2, invdt3, invdt4, dvr, dvt, vres, dt2d;
      dxrad = o->Rsup[i] - o->Rinf[i];
      if (p->FastTransport)
        vres = o->Vtheta[l] - o->Vmoy[i];
      else
        vres = o->Vtheta[l];
      invdt1 = o->SoundSpeed[l] / (min2(dxrad, o->dxtheta[i]));
      invdt2 = RFABS(o->Vrad[l]) / dxrad;
      invdt3 = RFABS(vres) / o->dxtheta[i];
      dvr = o->Vrad[l + nsec] - o->Vrad[l];
      dvt = o->Vtheta[i * nsec + (j + 1) % nsec] - o->Vtheta[l];
      if (dvr >= 0.0)
        dvr = 1e-10;
      else
        dvr = -dvr;
      if (dvt >= 0.0)
        dvt = 1e-10;
      else
        dvt = -dvt;
      invdt4 = max2(dvr / dxrad, dvt / o->dxtheta[i]);
      invdt4 *= 4.0 * CVNR * CVNR;
      dt2d = CFLSECURITY / RSQRT(invdt1 * invdt1 + invdt2 * invdt2 + invdt3 * invdt3 + invdt4 * invdt4);
      if (dt2d < newdt) newdt = dt2d;
    }
    o->newDT[i] = newdt;
  }
  for (int i = 0; i < nrad - 1; i++)
    o->DT1D[i] = 2.0 * PI * CFLSECURITY / (float)nsec /
                 RFABS(o->Vmoy[i] * o->invRmed[i] - o->Vmoy[i + 1] * o->invRmed[i + 1]);
  real newdt = o->newDT[1];
  for (int i = 2; i < nrad; i++)
    if (o->newDT[i] < newdt) newdt = o->newDT[i];
  for (int i = 0; i < nrad - 1; i++)
    if (o->DT1D[i] < newdt) newdt = o->DT1D[i];
  if (DeltaT < newdt) newdt = DeltaT;
  return (int)(ceil((real)(DeltaT / newdt)));
}

/* ------------------------------------------------------------------------ */
/* Source steps                                                             */
/* ------------------------------------------------------------------------ */

/* Substep1KernelVrad / Substep1KernelVtheta, Kernels.cu:52-88. */
static void substep1_kernels(orc* o, real dt) {
  int nrad = o->nrad, nsec = o->nsec;
  real* P = o->Pressure;
  real* D = o->Dens;
  real* Phi = o->Potential;
  real* Vt = o->Vtheta;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j, jp = i * nsec + (j + 1) % nsec, jm = i * nsec + ((j - 1) + nsec) % nsec;
      real gradp, gradphi, vt2;
      if (i > 0) {
        gradp = (P[l] - P[l - nsec]) * 2.0 / (D[l] + D[l - nsec]) * o->invdiffRmed[i];
        gradphi = (Phi[l] - Phi[l - nsec]) * o->invdiffRmed[i];
        if (o->accurate && o->sys.nb > 0) gradphi += o->star_grad[i];
        vt2 = Vt[l] + Vt[jp] + Vt[l - nsec] + Vt[jp - nsec];
        vt2 = vt2 / 4.0 + o->Rinf[i] * o->OmegaFrame;
        vt2 = vt2 * vt2;
        o->VradInt[l] = o->Vrad[l] + dt * (-gradp - gradphi + vt2 * o->invRinf[i]);
      }
      real dxtheta, invdxtheta;
      dxtheta = 2.0 * PI / (float)nsec * o->Rmed[i];
      invdxtheta = 1.0 / dxtheta;
      gradp = (P[l] - P[jm]) * 2.0 / (D[l] + D[jm]) * invdxtheta;
      gradphi = (Phi[l] - Phi[jm]) * invdxtheta;
      o->VthetaInt[l] = Vt[l] - dt * (gradp + gradphi);
      o->VthetaInt[l] += dt * o->supp_torque[i];
    }
}

/* ViscousTermsKernelDRP + ViscousTermsKernelTAURP, Kernels.cu:843-880.
   TAURP's third density sample is dens[i*nsec] for every j: the reference
   writes ((j-1)*nsec)%nsec, which is 0 (Kernels.cu:876). */
static void compute_viscous_terms(orc* o, const real* Vradial, const real* Vazimutal) {
  int nrad = o->nrad, nsec = o->nsec;
  refresh_viscosity(o);
  const real* D = o->Dens;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j, jp = i * nsec + (j + 1) % nsec, jm = i * nsec + ((j - 1) + nsec) % nsec;
      o->DRR[l] = (Vradial[l + nsec] - Vradial[l]) * o->invdiffRsup[i];
      o->DPP[l] = (Vazimutal[jp] - Vazimutal[l]) * o->invdphi * o->invRmed[i] +
                  0.5 * (Vradial[l + nsec] + Vradial[l]) * o->invRmed[i];
      o->DivergenceVelocity[l] =
          (Vradial[l + nsec] * o->Rsup[i] - Vradial[l] * o->Rinf[i]) * o->invdiffRsup[i] * o->invRmed[i];
      o->DivergenceVelocity[l] += (Vazimutal[jp] - Vazimutal[l]) * o->invdphi * o->invRmed[i];
      if (i > 0)
        o->DRP[l] = 0.5 * (o->Rinf[i] *
                               (Vazimutal[l] * o->invRmed[i] - Vazimutal[l - nsec] * o->invRmed[i - 1]) *
                               o->invdiffRmed[i] +
                           (Vradial[l] - Vradial[jm]) * o->invdphi * o->invRinf[i]);
    }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j;
      real nu = o->viscosity_array[i];
      o->TAURR[l] = 2.0 * D[l] * nu * (o->DRR[l] - o->onethird * o->DivergenceVelocity[l]);
      o->TAUPP[l] = 2.0 * D[l] * nu * (o->DPP[l] - o->onethird * o->DivergenceVelocity[l]);
      if (i > 0)
        o->TAURP[l] = 2.0 * 0.25 *
                      (D[l] + D[l - nsec] + D[i * nsec] + D[(i - 1) * nsec + ((j - 1) + nsec) % nsec]) * nu *
                      o->DRP[l];
    }
}

/* UpdateVelocitiesKernel, Kernels.cu:142-160. */
static void update_velocities_with_viscosity(orc* o, real DeltaT) {
  int nrad = o->nrad, nsec = o->nsec;
  const real *D = o->Dens, *TRR = o->TAURR, *TRP = o->TAURP, *TPP = o->TAUPP;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j, jp = i * nsec + (j + 1) % nsec, jm = i * nsec + ((j - 1) + nsec) % nsec;
      if (i < nrad - 1)
        o->VthetaInt[l] += DeltaT * o->invRmed[i] *
                           ((o->Rsup[i] * TRP[l + nsec] - o->Rinf[i] * TRP[l]) * o->invdiffRsup[i] +
                            (TPP[l] - TPP[jm]) * o->invdphi + 0.5 * (TRP[l] + TRP[l + nsec])) /
                           (0.5 * (D[l] + D[jm]));
      o->VradInt[l] += DeltaT * o->invRinf[i] *
                       ((o->Rmed[i] * TRR[l] - o->Rmed[i - 1] * TRR[l - nsec]) * o->invdiffRmed[i] +
                        (TRP[jp] - TRP[l]) * o->invdphi - 0.5 * (TPP[l] + TPP[l - nsec])) /
                       (0.5 * (D[l] + D[l - nsec]));
    }
}

/* ApplySubKeplerianBoundary, SideEuler.cu:250-272 + kernel Kernels.cu:1490. */
static void apply_sub_keplerian_boundary(orc* o) {
  const fargo_params* p = &o->p;
  int nrad = o->nrad, nsec = o->nsec;
  double VKepIn, VKepOut;
  real r0 = o->Rmed[0], r1 = o->Rmed[nrad - 1];
  if (!p->SelfGravity) {
    VKepIn = sqrt(G * 1.0 / r0 *
                  (1.0 - (1.0 + p->SIGMASLOPE - 2.0 * p->FLARINGINDEX) * pow(aspect_ratio_host(o, r0), 2.0) *
                             pow(r0, 2.0 * p->FLARINGINDEX)));
    VKepOut = sqrt(G * 1.0 / r1 *
                   (1.0 - (1.0 + p->SIGMASLOPE - 2.0 * p->FLARINGINDEX) * pow(aspect_ratio_host(o, r1), 2.0) *
                              pow(r1, 2.0 * p->FLARINGINDEX)));
  } else {
    ring_mean(o, o->SG_Accr, o->GLOBAL_AxiSGAccr);
    VKepIn = sqrt(G * 1.0 / r0 *
                      (1.0 - (1.0 + p->SIGMASLOPE - 2.0 * p->FLARINGINDEX) *
                                 pow(aspect_ratio_host(o, r0), 2.0) * pow(r0, 2.0 * p->FLARINGINDEX)) -
                  r0 * o->GLOBAL_AxiSGAccr[0]);
    VKepOut = sqrt(G * 1.0 / r1 *
                       (1.0 - (1.0 + p->SIGMASLOPE - 2.0 * p->FLARINGINDEX) *
                                  pow(aspect_ratio_host(o, r1), 2.0) * pow(r1, 2.0 * p->FLARINGINDEX)) -
                   r1 * o->GLOBAL_AxiSGAccr[nrad - 1]);
  }
  real vin = VKepIn, vout = VKepOut;
  for (int j = 0; j < nsec; j++) {
    o->VthetaInt[j] = vin - o->Rmed[0] * o->OmegaFrame;
    o->VthetaInt[(nrad - 1) * nsec + j] = vout - o->Rmed[nrad - 1] * o->OmegaFrame;
  }
}

/* Substep1, SourceEuler.cu:305-335. */
static void substep1(orc* o, real dt) {
  substep1_kernels(o, dt);
  if (o->p.SelfGravity) {
    sg_accelerations(o);
    sg_kick(o, dt);
  }
  compute_viscous_terms(o, o->VradInt, o->VthetaInt);
  update_velocities_with_viscosity(o, dt);
  if (!o->p.Evanescent) apply_sub_keplerian_boundary(o);
}

/* Substep2Kernel / Substep2Kernel2 (Kernels.cu:570-621), then the
   ActualiseGasVrad/Vtheta copies (SourceEuler.cu:466-477). */
static void substep2(orc* o, real dt) {
  const fargo_params* p = &o->p;
  int nrad = o->nrad, nsec = o->nsec;
  const real *D = o->Dens, *VRI = o->VradInt, *VTI = o->VthetaInt;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j, jp = i * nsec + (j + 1) % nsec;
      real dv = VRI[l + nsec] - VRI[l];
      if (dv < 0.0)
        o->DensInt[l] = CVNR * CVNR * D[l] * dv * dv;
      else
        o->DensInt[l] = 0.0;
      dv = VTI[jp] - VTI[l];
      if (dv < 0.0)
        o->TemperInt[l] = CVNR * CVNR * D[l] * dv * dv;
      else
        o->TemperInt[l] = 0.0;
    }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j, jp = i * nsec + (j + 1) % nsec, jm = i * nsec + ((j - 1) + nsec) % nsec;
      if (i > 0)
        o->VradNew[l] = VRI[l] - dt * 2.0 / (D[l] + D[l - nsec]) * (o->DensInt[l] - o->DensInt[l - nsec]) *
                                     o->invdiffRmed[i];
      real dxtheta = 2.0 * PI / (float)nsec * o->Rmed[i];
      real invdxtheta = 1.0 / dxtheta;
      o->VthetaNew[l] =
          VTI[l] - dt * 2.0 / (D[l] + D[jm]) * (o->TemperInt[l] - o->TemperInt[jm]) * invdxtheta;
      if (p->Adiabatic)
        o->EnergyInt[l] = o->Energy[l] - dt * o->DensInt[l] * (VRI[l + nsec] - VRI[l]) * o->invdiffRsup[i] -
                          dt * o->TemperInt[l] * (VTI[jp] - VTI[l]) * invdxtheta;
    }
  memcpy(o->Vrad, o->VradNew, sizeof(real) * o->size_grid);
  memcpy(o->Vtheta, o->VthetaNew, sizeof(real) * o->size_grid);
}

/* Substep3Kernel / Substep3Kernel2 (Kernels.cu:91-139) with the viscosity
   table rebuilt on the host (SourceEuler.cu:348-362), then ActualiseGasEnergy. */
static void substep3(orc* o, real dt) {
  const fargo_params* p = &o->p;
  int nrad = o->nrad, nsec = o->nsec;
  const real* D = o->Dens;
  real* Q = o->Qplus;
  for (int i = 0; i < nrad; i++) o->viscosity_array[i] = fviscosity(o, o->Rmed[i]);
#pragma omp parallel for schedule(static)
  for (int i = 1; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j;
      real nu = o->viscosity_array[i];
      if (nu != 0.0) {
        Q[l] = 0.5 / nu / D[l] *
               (o->TAURR[l] * o->TAURR[l] + +o->TAURP[l] * o->TAURP[l] + o->TAUPP[l] * o->TAUPP[l]);
        Q[l] += (2.0 / 9.0) * nu * D[l] * o->DivergenceVelocity[l] * o->DivergenceVelocity[l];
      } else
        Q[l] = 0.0;
    }
  for (int j = 0; j < nsec; j++) {
    if (o->viscosity_array[nrad - 1] != 0.0)
      Q[j] = Q[nsec + j] * REXP(RLOG(Q[nsec + j] / Q[2 * nsec + j]) * RLOG(o->Rmed[0] / o->Rmed[1]) /
                                RLOG(o->Rmed[1] / o->Rmed[2]));
    else
      Q[j] = 0.0;
  }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j;
      real num, den;
      if (!p->Cooling) {
        num = dt * Q[l] + o->EnergyInt[l];
        den = 1.0 + (p->ADIABATICINDEX - 1.0) * dt * o->DivergenceVelocity[l];
        o->EnergyNew[l] = num / den;
      } else {
        num = o->EnergyMed[i] * dt * D[l] / o->SigmaMed[i] + o->CoolingTimeMed[i] * o->EnergyInt[l] +
              dt * o->CoolingTimeMed[i] * (Q[l] - o->QplusMed[i] * D[l] / o->SigmaMed[i]);
        den = dt + o->CoolingTimeMed[i] + (p->ADIABATICINDEX - 1.0) * dt * o->CoolingTimeMed[i] *
                                              o->DivergenceVelocity[l];
        o->EnergyNew[l] = num / den;
      }
    }
  memcpy(o->Energy, o->EnergyNew, sizeof(real) * o->size_grid);
}

/* ------------------------------------------------------------------------ */
/* Transport (TransportEuler.cu:24-263)                                     */
/* ------------------------------------------------------------------------ */

/* LRMomentaKernel, Kernels.cu:883-896. */
static void compute_lr_momenta(orc* o) {
  int nrad = o->nrad, nsec = o->nsec;
  const real *D = o->Dens, *Vr = o->Vrad, *Vt = o->Vtheta;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j, jp = i * nsec + (j + 1) % nsec;
      real rm = o->Rmed[i];
      o->RadMomP[l] = D[l] * Vr[l + nsec];
      o->RadMomM[l] = D[l] * Vr[l];
      o->ThetaMomP[l] = D[l] * (Vt[jp] + rm * o->OmegaFrame) * rm;
      o->ThetaMomM[l] = D[l] * (Vt[l] + rm * o->OmegaFrame) * rm;
    }
}

/* DivisePolarGridKernel, Kernels.cu:1127-1134 (element-wise; only the
   active rings are ever read back). */
static void divise_polar_grid(orc* o, const real* Qb, const real* Dint, real* Work) {
  int n = o->nrad * o->nsec;
#pragma omp parallel for schedule(static)
  for (int l = 0; l < n; l++) Work[l] = Qb[l] / (Dint[l] + 1e-20);
}

/* StarRadKernel + StarRadKernel2, Kernels.cu:909-947. */
static void compute_star_rad(orc* o, const real* Qb, real* QStar, real dt) {
  int nrad = o->nrad, nsec = o->nsec;
  real* dq = o->dq;
  const real* Vr = o->Vrad;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j;
      if (i == 0 || i == nrad - 1)
        dq[l] = 0.0;
      else {
        real dqm = (Qb[l] - Qb[l - nsec]) * o->invdiffRmed[i];
        real dqp = (Qb[l + nsec] - Qb[l]) * o->invdiffRmed[i + 1];
        if (dqp * dqm > 0.0)
          dq[l] = 2.0 * dqp * dqm / (dqp + dqm);
        else
          dq[l] = 0.0;
      }
    }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j;
      if (Vr[l] > 0.0 && i > 0)
        QStar[l] = Qb[l - nsec] + (o->Rmed[i] - o->Rmed[i - 1] - Vr[l] * dt) * 0.5 * dq[l - nsec];
      else
        QStar[l] = Qb[l] - (o->Rmed[i + 1] - o->Rmed[i] + Vr[l] * dt) * 0.5 * dq[l];
    }
  for (int j = 0; j < nsec; j++) QStar[j] = QStar[j + nsec * nrad] = 0.0;
}

/* VanLeerRadialKernel, Kernels.cu:1137-1154. */
static void van_leer_radial_kernel(orc* o, real* Qb, real dt, int return_lost) {
  int nrad = o->nrad, nsec = o->nsec;
  const real *QR = o->QRStar, *DS = o->DensStar, *Vr = o->Vrad;
  real dtheta = 2.0 * PI / (float)nsec;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j;
      real varq = dt * dtheta * o->Rinf[i] * QR[l] * DS[l] * Vr[l];
      varq -= dt * dtheta * o->Rsup[i] * QR[l + nsec] * DS[l + nsec] * Vr[l + nsec];
      Qb[l] += varq * o->invSurf[i];
      if (i == 0 && o->p.OpenInner) o->LostByDisk[j] = varq;
    }
  (void)return_lost;
}

/* VanLeerRadial, TransportEuler.cu:100-150. */
static real van_leer_radial(orc* o, real* Qb, real dt, int return_lost) {
  divise_polar_grid(o, Qb, o->DensInt, o->Work);
  compute_star_rad(o, o->Work, o->QRStar, dt);
  van_leer_radial_kernel(o, Qb, dt, return_lost);
  return return_lost ? device_reduce(o->LostByDisk, o->nsec) : (real)0;
}

/* OneWindRad, TransportEuler.cu:54-73. */
static void one_wind_rad(orc* o, real dt) {
  compute_star_rad(o, o->Dens, o->DensStar, dt);
  memcpy(o->DensInt, o->Dens, sizeof(real) * o->size_grid);
  van_leer_radial(o, o->RadMomP, dt, 0);
  van_leer_radial(o, o->RadMomM, dt, 0);
  van_leer_radial(o, o->ThetaMomP, dt, 0);
  van_leer_radial(o, o->ThetaMomM, dt, 0);
  if (o->p.Adiabatic) van_leer_radial(o, o->Energy, dt, 0);
  o->LostMass += van_leer_radial(o, o->Dens, dt, 1);
}

/* StarThetaKernel + StarThetaKernel2, Kernels.cu:1235-1273. */
static void compute_star_theta(orc* o, const real* Qb, const real* Vaz, real* QStar, real dt) {
  int nrad = o->nrad, nsec = o->nsec;
  real* dq = o->dq;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++) {
    real dxtheta = 2.0 * PI / (float)nsec * o->Rmed[i];
    real invdxtheta = 1.0 / dxtheta;
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j, jp = i * nsec + (j + 1) % nsec, jm = i * nsec + ((j - 1) + nsec) % nsec;
      real dqm = (Qb[l] - Qb[jm]);
      real dqp = (Qb[jp] - Qb[l]);
      if (dqp * dqm > 0.0)
        dq[l] = dqp * dqm / (dqp + dqm) * invdxtheta;
      else
        dq[l] = 0.0;
    }
  }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++) {
    real dxtheta = 2.0 * PI / (float)nsec * o->Rmed[i];
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j, jm = i * nsec + ((j - 1) + nsec) % nsec;
      real ksi = Vaz[l] * dt;
      if (ksi > 0.0)
        QStar[l] = Qb[jm] + (dxtheta - ksi) * dq[jm];
      else
        QStar[l] = Qb[l] - (dxtheta + ksi) * dq[l];
    }
  }
}

/* VanLeerTheta + VanLeerThetaKernel, TransportEuler.cu:243-251,
   Kernels.cu:1157-1174 (the wrapper passes UniformTransport = 0, so every
   ring is advected). */
static void van_leer_theta(orc* o, const real* Vaz, real* Qb, real dt) {
  int nrad = o->nrad, nsec = o->nsec;
  divise_polar_grid(o, Qb, o->DensInt, o->Work);
  compute_star_theta(o, o->Work, Vaz, o->QRStar, dt);
  const real *QR = o->QRStar, *DS = o->DensStar;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++) {
    real invsurf = 1.0 / o->Surf[i];
    real dxrad = (o->Rsup[i] - o->Rinf[i]) * dt;
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j, jp = i * nsec + (j + 1) % nsec;
      real varq = dxrad * QR[l] * DS[l] * Vaz[l];
      varq -= dxrad * QR[jp] * DS[jp] * Vaz[jp];
      Qb[l] += varq * invsurf;
    }
  }
}

/* QuantitiesAdvection, TransportEuler.cu:223-239. */
static void quantities_advection(orc* o, const real* Vaz, real dt) {
  compute_star_theta(o, o->Dens, Vaz, o->DensStar, dt);
  memcpy(o->DensInt, o->Dens, sizeof(real) * o->size_grid);
  van_leer_theta(o, Vaz, o->RadMomP, dt);
  van_leer_theta(o, Vaz, o->RadMomM, dt);
  van_leer_theta(o, Vaz, o->ThetaMomP, dt);
  van_leer_theta(o, Vaz, o->ThetaMomM, dt);
  if (o->p.Adiabatic) van_leer_theta(o, Vaz, o->Energy, dt);
  van_leer_theta(o, Vaz, o->Dens, dt);
}

/* AdvectSHIFTKernel + copy back, Kernels.cu:1276-1289, TransportEuler.cu:204-210. */
static void advect_shift(orc* o, real* a) {
  int nrad = o->nrad, nsec = o->nsec;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int ji = j - o->Nshift[i];
      while (ji < 0) ji += nsec;
      while (ji >= nsec) ji -= nsec;
      o->TempShift[i * nsec + j] = a[i * nsec + ji];
    }
  memcpy(a, o->TempShift, sizeof(real) * nrad * nsec);
}

/* OneWindTheta, TransportEuler.cu:171-219, with
   ComputeAverageThetaVelocitiesKernel, ComputeResidualsKernel and
   ComputeConstantResidualKernel (Kernels.cu:1177-1232). */
static void one_wind_theta(orc* o, real dt) {
  const fargo_params* p = &o->p;
  int nrad = o->nrad, nsec = o->nsec;
  ring_mean(o, o->Vtheta, o->VMed);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) o->VthetaRes[i * nsec + j] = o->Vtheta[i * nsec + j] - o->VMed[i];
  for (int i = 0; i < nrad; i++) {
    real maxfrac = p->FastTransport ? 1.0 : 0.0;
    real invdt = 1.0 / dt;
    real dpinvns = 2.0 * PI / (float)nsec;
    real Ntilde = o->VMed[i] * o->invRmed[i] * dt * (float)nsec / 2.0 / PI;
    real Nround = floor(Ntilde + 0.5);
    long nitemp = (long)Nround;
    o->Nshift[i] = (int)nitemp;
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j;
      o->Vtheta[l] = (Ntilde - Nround) * o->Rmed[i] * invdt * dpinvns;
      if (maxfrac < 0.5) {
        o->VthetaRes[l] = o->Vtheta[l] + o->VthetaRes[l];
        o->Vtheta[l] = 0.0;
      }
    }
  }
  quantities_advection(o, o->VthetaRes, dt);
  quantities_advection(o, o->Vtheta, dt);
  advect_shift(o, o->RadMomP);
  advect_shift(o, o->RadMomM);
  advect_shift(o, o->ThetaMomP);
  advect_shift(o, o->ThetaMomM);
  if (p->Adiabatic) advect_shift(o, o->Energy);
  advect_shift(o, o->Dens);
}

/* ComputeVelocitiesKernel, Kernels.cu:1292-1306. */
static void compute_velocities(orc* o) {
  int nrad = o->nrad, nsec = o->nsec;
  const real* D = o->Dens;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j, jm = i * nsec + ((j - 1) + nsec) % nsec;
      if (i == 0)
        o->Vrad[l] = 0.0;
      else
        o->Vrad[l] = (o->RadMomP[l - nsec] + o->RadMomM[l]) / (D[l] + D[l - nsec] + 1e-20);
      o->Vtheta[l] = (o->ThetaMomP[jm] + o->ThetaMomM[l]) / (D[l] + D[jm] + 1e-15) / o->Rmed[i] -
                     o->Rmed[i] * o->OmegaFrame;
    }
}

/* Transport, TransportEuler.cu:24-35. */
static void transport(orc* o, real dt) {
  compute_lr_momenta(o);
  one_wind_rad(o, dt);
  one_wind_theta(o, dt);
  compute_velocities(o);
}

/* CircumPlanetaryMass + kernel, SourceEuler.cu:539-553, Kernels.cu:245-261. */
static float circum_planetary_mass(orc* o) {
  int nrad = o->nrad, nsec = o->nsec;
  real xpl = o->sys.x[0], ypl = o->sys.y[0], hill = o->HillRadius;
  double s = 0;
  if (o->sys.nb < 1) return 0.0f;
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j;
      real dist = RSQRT((o->CellAbscissa[l] - xpl) * (o->CellAbscissa[l] - xpl) +
                        (o->CellOrdinate[l] - ypl) * (o->CellOrdinate[l] - ypl));
      if (dist < hill) s += (real)(o->Surf[i] * o->Dens[l]);
    }
  return (float)s;
}

/* CorrectVthetaKernel, Kernels.cu:1352-1359. */
static void correct_vtheta(orc* o, real domega) {
  for (int i = 0; i < o->nrad; i++)
    for (int j = 0; j < o->nsec; j++) o->Vtheta[i * o->nsec + j] -= domega * o->Rmed[i];
}

/* ------------------------------------------------------------------------ */
/* AlgoGas, SourceEuler.cu:208-301                                          */
/* ------------------------------------------------------------------------ */

/* ------------------------------------------------------------------------ */
/* Boundary conditions (SideEuler.cu:64-182)                                */
/* ------------------------------------------------------------------------ */

static long nearest_pow2(long n) {
  long x = 1;
  if (!n) return n;
  while (x < n) x <<= 1;
  return x;
}

/* DeviceReduce<float> (Kernels.cu:431-557) in its own order of operations:
   getNumBlocksAndThreads (Kernels.cu:404-429) picks the block count and size,
   each block reduces with deviceReduceKernel (Kernels.cu:269-383; IsPow2 is
   always false for n > 1 because of its operator precedence, so the bounds-
   checked form runs), the final warp by shuffles, and the host adds the block
   sums in order.  The reference launches no block for n <= 128 and stops
   there with an error; the caller refuses such grids. */
static real device_reduce(const real* in, int n) {
  long maxBlocks = nearest_pow2(n) / 256;
  int threads = (n < 256 * 2) ? (int)nearest_pow2((n + 1) / 2) : 256;
  long blocks = (n + (threads * 2 - 1)) / (threads * 2);
  if (blocks > maxBlocks) blocks = maxBlocks;
  real s[512], w[32];
  real sum = 0;
  for (long b = 0; b < blocks; b++) {
    long gridSize = (long)threads * 2 * blocks;
    for (int t = 0; t < threads; t++) {
      real mySum = 0;
      long i = b * threads * 2 + t;
      while (i < n) {
        mySum += in[i];
        if (i + threads < n) mySum += in[i + threads];
        i += gridSize;
      }
      s[t] = mySum;
    }
    for (int stride = 256; stride >= 64; stride >>= 1)
      if (threads >= 2 * stride)
        for (int t = 0; t < stride; t++) s[t] = s[t] + s[t + stride];
    for (int t = 0; t < 32; t++) w[t] = (threads >= 64) ? s[t] + s[t + 32] : s[t];
    for (int off = 16; off > 0; off >>= 1) {
      real nw[32];
      for (int t = 0; t < 32; t++) nw[t] = (t + off < 32) ? w[t] + w[t + off] : w[t];
      memcpy(w, nw, sizeof(w));
    }
    sum += w[0];
  }
  return sum;
}

/* OpenBoundaryKernel, Kernels.cu:623-637. */
static void open_boundary(orc* o) {
  int nsec = o->nsec, i = 1;
  real* D = o->Dens;
  real* E = o->Energy;
  real* V = o->Vrad;
  real SigmaMed = (float)o->SigmaMed[0];
  for (int j = 0; j < nsec; j++) {
    D[(i - 1) * nsec + j] = D[i * nsec + j];
    E[(i - 1) * nsec + j] = E[i * nsec + j];
    if (V[(i + 1) * nsec + j] > 0.0 || (D[i * nsec + j] < SigmaMed))
      V[i * nsec + j] = 0.0;
    else
      V[i * nsec + j] = V[(i + 1) * nsec + j];
  }
}

/* NonReflectingBoundary (SideEuler.cu:70-101) with ReduceCs, ReduceMean
   (SideEuler.cu:103-122) and the kernels NonReflectingBoundaryKernel,
   MinusMeanKernel (Kernels.cu:676-722). */
static void non_reflecting_boundary(orc* o) {
  int nsec = o->nsec, nrad = o->nrad, i, i_angle, i_angle2;
  double dangle, dangle2;
  real* D = o->Dens;
  real* E = o->Energy;
  real* V = o->Vrad;
  const real* cs = o->SoundSpeed;
  real cs0_r = device_reduce(cs, nsec) / (float)nsec;
  real cs1_r = device_reduce(cs + nsec, nsec) / (float)nsec;
  real csnrm1_r = device_reduce(cs + (size_t)(nrad - 1) * nsec, nsec) / (float)nsec;
  real csnrm2_r = device_reduce(cs + (size_t)(nrad - 2) * nsec, nsec) / (float)nsec;
  i = 1;
  dangle = (pow(o->Rinf[i], -1.5) - 1.0) / (.5 * (cs0_r + cs1_r));
  dangle *= (o->Rmed[i] - o->Rmed[i - 1]);
  i_angle = (int)(dangle / 2.0 / PI * (float)nsec + .5);
  i = nrad - 1;
  dangle2 = (pow(o->Rinf[i - 1], -1.5) - 1.0) / (.5 * (csnrm1_r + csnrm2_r));
  dangle2 *= (o->Rmed[i] - o->Rmed[i - 1]);
  i_angle2 = (int)(dangle2 / 2.0 / PI * (float)nsec + .5);
  o->bc_angle[0] = i_angle;
  o->bc_angle[1] = i_angle2;
  real SigmaMed = (float)o->SigmaMed[1], SigmaMed2 = (float)o->SigmaMed[nrad - 2];
  for (int j = 0; j < nsec; j++) {
    int jp;
    real Vrad_med;
    i = 1;
    jp = j + i_angle;
    if (jp >= nsec) jp -= nsec;
    if (jp < 0) jp += nsec;
    D[jp] = D[i * nsec + j];
    E[jp] = E[i * nsec + j];
    Vrad_med = -cs[i * nsec + j] * (D[i * nsec + j] - SigmaMed) / SigmaMed;
    V[i * nsec + j] = 2. * Vrad_med - V[(i + 1) * nsec + j];
    i = nrad - 1;
    jp = j - i_angle2;
    if (jp >= nsec) jp -= nsec;
    if (jp < 0) jp += nsec;
    D[i * nsec + j] = D[jp + (i - 1) * nsec];
    E[i * nsec + j] = E[jp + (i - 1) * nsec];
    Vrad_med = cs[i * nsec + j] * (D[(i - 1) * nsec + j] - SigmaMed2) / SigmaMed2;
    V[i * nsec + j] = 2. * Vrad_med - V[(i - 1) * nsec + j];
  }
  real mean_dens_r = device_reduce(D, nsec) / (float)nsec;
  real mean_dens_r2 = device_reduce(D + (size_t)(nrad - 1) * nsec, nsec) / (float)nsec;
  real mean_energy_r = device_reduce(E, nsec) / (float)nsec;
  real mean_energy_r2 = device_reduce(E + (size_t)(nrad - 1) * nsec, nsec) / (float)nsec;
  real sm0 = (float)o->SigmaMed[0], sm1 = (float)o->SigmaMed[nrad - 1];
  real em0 = (float)o->EnergyMed[0], em1 = (float)o->EnergyMed[nrad - 1];
  for (int j = 0; j < nsec; j++) {
    D[j] += sm0 - mean_dens_r;
    E[j] += em0 - mean_energy_r;
    D[(nrad - 1) * nsec + j] += sm1 - mean_dens_r2;
    E[(nrad - 1) * nsec + j] += em1 - mean_energy_r2;
  }
}

/* EvanescentBoundary (SideEuler.cu:124-141) and EvanescentBoundaryKernel
   (Kernels.cu:1076-1124).  The kernel's GLOBAL_bufarray_d is never filled by
   the reference (a fresh, zeroed allocation): its self-gravity term is 0. */
static void evanescent_boundary(orc* o, real step) {
  const fargo_params* p = &o->p;
  int nrad = o->nrad, nsec = o->nsec;
  double Tin_d = 2.0 * PI * pow(o->Rmed[0], 3. / 2);
  double Tout_d = 2.0 * PI * pow(o->Rmed[nrad - 1], 3. / 2);
  float DRMIN = o->Rmed[0] * 1.25, DRMAX = o->Rmed[nrad - 1] * 0.84;
  float Tin = (float)Tin_d, Tout = (float)Tout_d;
  for (int i = 0; i < nrad; i++) o->viscosity_array[i] = fviscosity(o, o->Rmed[i]);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nrad; i++) {
    real Rm = o->Rmed[i];
    if (!((Rm < DRMIN) || (Rm > DRMAX))) continue;
    real damping, lambda = 0.0, vtheta0, vrad0, energy0, dens0, AspectRatio;
    if (Rm < DRMIN) {
      damping = (Rm - DRMIN) / (o->Rmed[0] - DRMIN);
      lambda = damping * damping * 10.0 * step / Tin;
    }
    if (Rm > DRMAX) {
      damping = (Rm - DRMAX) / (o->Rmed[nrad - 1] - DRMAX);
      lambda = damping * damping * 10.0 * step / Tout;
    }
    AspectRatio = aspect_ratio_dev(o, Rm);
    /* the self-gravity branch subtracts Rmed * GLOBAL_bufarray_d[i] = 0 */
    vtheta0 = RSQRT(G * 1.0 / Rm *
                    (1.0 - (1.0 + p->SIGMASLOPE - 2.0 * p->FLARINGINDEX) * RPOW(AspectRatio, 2.0) *
                               RPOW(Rm, 2.0 * p->FLARINGINDEX)));
    vtheta0 -= Rm * o->OmegaFrame;
    vrad0 = -3.0 * o->viscosity_array[i] / Rm * (-p->SIGMASLOPE + .5);
    dens0 = o->SigmaMed[i];
    energy0 = o->EnergyMed[i];
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j;
      o->Vrad[l] = (o->Vrad[l] + lambda * vrad0) / (1.0 + lambda);
      o->Vtheta[l] = (o->Vtheta[l] + lambda * vtheta0) / (1.0 + lambda);
      o->Dens[l] = (o->Dens[l] + lambda * dens0) / (1.0 + lambda);
      if (p->Adiabatic) o->Energy[l] = (o->Energy[l] + lambda * energy0) / (1.0 + lambda);
    }
  }
}

/* ApplyBoundaryCondition, SideEuler.cu:172-182. */
static void apply_boundary_condition(orc* o, real step) {
  const fargo_params* p = &o->p;
  if (p->OpenInner) open_boundary(o);
  if (p->NonReflecting) {
    if (p->Adiabatic) compute_sound_speed(o);
    non_reflecting_boundary(o);
  }
  if (p->Evanescent) evanescent_boundary(o, step);
}

int orc_advance_dt(orc* o) {
  const fargo_params* p = &o->p;
  double dt, dtemp = 0.0;
  double OmegaNew, domega;
  int gastimestepcfl = 1;
  o->nsub = 0;
  if (p->Adiabatic) compute_sound_speed(o);
  if (p->IsDisk == YES && p->SloppyCFL == YES) gastimestepcfl = condition_cfl(o, (float)(p->DT - dtemp));
  dt = p->DT / (double)gastimestepcfl;
  while (dtemp < 0.999999999 * p->DT) {
    o->MassTaper = o->PhysicalTime / (p->MASSTAPER * 2.0 * M_PI);
    o->MassTaper = (o->MassTaper > 1.0 ? 1.0 : pow(sin(o->MassTaper * M_PI / 2.0), 2.0));
    if (p->IsDisk == YES) {
      if (p->SloppyCFL == NO) {
        gastimestepcfl = condition_cfl(o, (float)(p->DT - dtemp));
        dt = (p->DT - dtemp) / (double)gastimestepcfl;
      }
    }
    dtemp += dt;
    o->DiskOnPrimaryAcceleration.x = 0.0;
    o->DiskOnPrimaryAcceleration.y = 0.0;
    if (p->Corotating == YES) get_psys_info(o, 1);
    if (p->IsDisk == YES) {
      o->DiskOnPrimaryAcceleration = compute_accel(o, 0.0, 0.0, 0.0, 0.0);
      fill_forces_arrays(o);
      advance_system_from_disk(o, (float)dt);
    }
    advance_system_rk5(o, (float)dt);
    if (p->Corotating == YES) {
      OmegaNew = get_psys_info(o, 0) / dt;
      domega = OmegaNew - o->OmegaFrame;
      if (p->IsDisk == YES) correct_vtheta(o, (real)domega);
      o->OmegaFrame = OmegaNew;
    }
    rotate_psys(o, (float)(o->OmegaFrame * dt));
    if (p->IsDisk == YES) {
      real dtr = (real)(float)dt;
      apply_boundary_condition(o, dtr);
      compute_pressure(o);
      substep1(o, dtr);
      substep2(o, dtr);
      apply_boundary_condition(o, dtr);
      if (p->Adiabatic) {
        compute_viscous_terms(o, o->Vrad, o->Vtheta);
        substep3(o, dtr);
      }
      transport(o, dtr);
      apply_boundary_condition(o, dtr);
      compute_temperature(o);
      o->mdcp1 = circum_planetary_mass(o);
    }
    if (o->nsub < MAXSUB) {
      memcpy(o->log_nshift + (size_t)o->nsub * o->nrad, o->Nshift, sizeof(int) * o->nrad);
      o->log_dt[o->nsub] = dt;
    }
    o->nsub++;
    o->nsub_total++;
    o->last_dt = dt;
    o->PhysicalTime += dt;
  }
  return o->nsub;
}

/* ------------------------------------------------------------------------ */
/* Creation: the setup part of main() (Main.cu:198-344)                     */
/* ------------------------------------------------------------------------ */

int orc_create(const fargo_params* pin, const fargo_planets* planets, const double* radii, orc** out) {
  orc* o = (orc*)calloc(1, sizeof(orc));
  if (!o) return 1;
  o->p = *pin;
  const fargo_params* p = &o->p;
  int nrad = p->NRAD, nsec = p->NSEC;
  if (nrad < 3 || nsec < 3 || (p->NonReflecting && nsec <= 128)) {
    free(o);
    return 1;
  }
  o->nrad = nrad;
  o->nsec = nsec;
  o->size_grid = (nrad + 1) * nsec;
  size_t n1 = nrad + 1, ng = o->size_grid;
  o->Radii2 = (double*)calloc(n1, sizeof(double));
  o->Rmed2 = (double*)calloc(n1, sizeof(double));
  real** t1[] = {&o->Radii, &o->Rinf, &o->Rsup, &o->Rmed, &o->Surf, &o->invRinf, &o->invSurf, &o->invRmed,
                 &o->invdiffRsup, &o->invdiffRmed, &o->powRmed, &o->SigmaMed, &o->SigmaInf, &o->EnergyMed,
                 &o->CoolingTimeMed, &o->QplusMed, &o->viscosity_array, &o->supp_torque, &o->dxtheta,
                 &o->GLOBAL_bufarray, &o->GLOBAL_AxiSGAccr, &o->Vmoy, &o->newDT, &o->DT1D, &o->VMed};
  for (size_t k = 0; k < sizeof(t1) / sizeof(t1[0]); k++) *t1[k] = zr(n1 + 1);
  o->Nshift = (int*)calloc(n1, sizeof(int));
  o->log_nshift = (int*)calloc((size_t)MAXSUB * nrad, sizeof(int));
  real** t2[] = {&o->Dens, &o->Vrad, &o->Vtheta, &o->Energy, &o->SoundSpeed, &o->Pressure, &o->Temperature,
                 &o->Potential, &o->VradInt, &o->VthetaInt, &o->VradNew, &o->VthetaNew, &o->EnergyInt,
                 &o->EnergyNew, &o->DensInt, &o->TemperInt, &o->DRR, &o->DPP, &o->DRP,
                 &o->DivergenceVelocity, &o->TAURR, &o->TAUPP, &o->TAURP, &o->Qplus, &o->CellAbscissa,
                 &o->CellOrdinate, &o->RadMomP, &o->RadMomM, &o->ThetaMomP, &o->ThetaMomM, &o->Work,
                 &o->QRStar, &o->DensStar, &o->dq, &o->VthetaRes, &o->TempShift, &o->SG_Accr, &o->SG_Acct};
  for (size_t k = 0; k < sizeof(t2) / sizeof(t2[0]); k++) *t2[k] = zr(ng);
  o->LostByDisk = zr(nsec);

  fill_polar_1d(o, radii);
  fill_misc_tables(o);
  o->sys0 = *planets;
  /* FillSigma / FillEnergy profiles, Theo.cu:23-29,42-51 */
  for (int i = 0; i < nrad; i++) {
    o->SigmaMed[i] = sigma_profile(o, o->Rmed[i]);
    o->SigmaInf[i] = sigma_profile(o, o->Rinf[i]);
    if (p->Adiabatic) o->EnergyMed[i] = energy_profile(o, o->Rmed[i]);
  }
  if (p->SelfGravity) {
    size_t n2 = (size_t)2 * nrad * nsec;
    o->Kr_aux = zr(n2);
    o->Kt_aux = zr(n2);
    o->Kr_hat = (double*)calloc(2 * n2, sizeof(double));
    o->Kt_hat = (double*)calloc(2 * n2, sizeof(double));
    o->cbuf0 = (double*)calloc(2 * n2, sizeof(double));
    o->cbuf1 = (double*)calloc(2 * n2, sizeof(double));
    /* Main.cu:308-310 */
    o->SGP_eps = p->THICKNESSSMOOTHING * p->ASPECTRATIO;
    o->SGP_rstep = RLOG(o->Radii[nrad] / o->Radii[0]) / (float)nrad;
    o->SGP_tstep = 2.0 * PI / (float)nsec;
    sg_init_kernel(o);
  }
  *out = o;
  orc_init_state(o, NULL, NULL);
  return 0;
}

/* The initialisation of main() from InitGasDensity on (Main.cu:292-344),
   with an optional perturbed density / energy in place of the profiles. */
void orc_init_state(orc* o, const float* dens, const float* energy) {
  const fargo_params* p = &o->p;
  int nrad = o->nrad, nsec = o->nsec;
  size_t ng = o->size_grid;
  for (size_t l = 0; l < ng; l++) {
    o->Dens[l] = 0;
    o->Energy[l] = 0;
    o->Vrad[l] = 0;
    o->Vtheta[l] = 0;
  }
  /* InitGasDensity / InitGasEnergy, Pframeforce.cu:173-192 */
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      o->Dens[j + i * nsec] = o->SigmaMed[i];
      if (p->Adiabatic) o->Energy[i * nsec + j] = o->EnergyMed[i];
    }
  if (dens)
    for (size_t l = 0; l < ng; l++) o->Dens[l] = dens[l];
  if (energy)
    for (size_t l = 0; l < ng; l++) o->Energy[l] = energy[l];
  o->sys = o->sys0;
  o->PhysicalTime = 0.0f;
  o->PhysicalTimeInitial = 0.0f;
  o->LostMass = 0.0f;
  o->nsub = 0;
  o->nsub_total = 0;
  if (o->sys.nb > 0) o->HillRadius = o->sys.x[0] * pow(o->sys.mass[0] / 3., 1. / 3.); /* Psys.cu:206 */
  if (p->SelfGravity) {
    /* compute_selfgravity(..., init=1) without the velocity update, then
       Init_planetarysys_withSG (Main.cu:322-328) */
    sg_accelerations(o);
    init_planets_with_sg(o);
  }
  /* OmegaFrame (Main.cu:332-333) */
  o->OmegaFrame = p->OMEGAFRAME;
  if (p->Corotating) o->OmegaFrame = get_psys_info(o, 2);
  /* Initialization -> InitEuler (SourceEuler.cu:177-204) */
  init_cell_coords(o);
  compute_sound_speed(o);
  compute_pressure(o);
  compute_temperature(o);
  /* InitGasVelocities (Pframeforce.cu:194-255) */
  if (p->SelfGravity) init_vtheta_with_sg(o);
  if (p->ViscosityAlpha) ring_mean(o, o->SoundSpeed, o->GLOBAL_bufarray);
  if (p->Cooling) {
    for (int i = 0; i < nrad; i++) o->CoolingTimeMed[i] = cooling_time(o, o->Rmed[i]);
    for (int i = 0; i < nrad; i++) o->QplusMed[i] = qplus_init(o, o->Rmed[i]);
  }
  /* InitVelocities, Pframeforce.cu:258-272 */
  for (int i = 0; i < nrad; i++) o->viscosity_array[i] = fviscosity(o, o->Rmed[i]);
  o->viscosity_array[nrad] = fviscosity(o, o->Rmed[nrad - 1]);
  init_gas_velocities_kernel(o);
  o->PhysicalTimeInitial = o->PhysicalTime;
}


void orc_destroy(orc* o) {
  if (!o) return;
  real** t[] = {&o->Radii, &o->Rinf, &o->Rsup, &o->Rmed, &o->Surf, &o->invRinf, &o->invSurf, &o->invRmed,
                &o->invdiffRsup, &o->invdiffRmed, &o->powRmed, &o->SigmaMed, &o->SigmaInf, &o->EnergyMed,
                &o->CoolingTimeMed, &o->QplusMed, &o->viscosity_array, &o->supp_torque, &o->dxtheta,
                &o->GLOBAL_bufarray, &o->GLOBAL_AxiSGAccr, &o->Vmoy, &o->newDT, &o->DT1D, &o->VMed,
                &o->Dens, &o->Vrad, &o->Vtheta, &o->Energy, &o->SoundSpeed, &o->Pressure, &o->Temperature,
                &o->Potential, &o->VradInt, &o->VthetaInt, &o->VradNew, &o->VthetaNew, &o->EnergyInt,
                &o->EnergyNew, &o->DensInt, &o->TemperInt, &o->DRR, &o->DPP, &o->DRP,
                &o->DivergenceVelocity, &o->TAURR, &o->TAUPP, &o->TAURP, &o->Qplus, &o->CellAbscissa,
                &o->CellOrdinate, &o->RadMomP, &o->RadMomM, &o->ThetaMomP, &o->ThetaMomM, &o->Work,
                &o->QRStar, &o->DensStar, &o->dq, &o->VthetaRes, &o->TempShift, &o->SG_Accr, &o->SG_Acct,
                &o->LostByDisk, &o->Kr_aux, &o->Kt_aux};
  for (size_t k = 0; k < sizeof(t) / sizeof(t[0]); k++) free(*t[k]);
  free(o->Radii2);
  free(o->Rmed2);
  free(o->Nshift);
  free(o->log_nshift);
  free(o->Kr_hat);
  free(o->Kt_hat);
  free(o->cbuf0);
  free(o->star_grad);
  free(o->cbuf1);
  free(o);
}

int orc_real_size(void) { return (int)sizeof(real); }

void orc_set_fields(orc* o, const void* dens, const void* vrad, const void* vtheta, const void* energy) {
  size_t b = sizeof(real) * o->size_grid;
  if (dens) memcpy(o->Dens, dens, b);
  if (vrad) memcpy(o->Vrad, vrad, b);
  if (vtheta) memcpy(o->Vtheta, vtheta, b);
  if (energy) memcpy(o->Energy, energy, b);
}

void orc_get_fields(const orc* o, void* dens, void* vrad, void* vtheta, void* energy, void* temperature,
                    void* qplus) {
  size_t b = sizeof(real) * o->size_grid;
  if (dens) memcpy(dens, o->Dens, b);
  if (vrad) memcpy(vrad, o->Vrad, b);
  if (vtheta) memcpy(vtheta, o->Vtheta, b);
  if (energy) memcpy(energy, o->Energy, b);
  if (temperature) memcpy(temperature, o->Temperature, b);
  if (qplus) memcpy(qplus, o->Qplus, b);
}

static void cp_in(real* dst, const float* src, size_t n) {
  if (src)
    for (size_t l = 0; l < n; l++) dst[l] = src[l];
}
static void cp_out(float* dst, const real* src, size_t n) {
  if (dst)
    for (size_t l = 0; l < n; l++) dst[l] = (float)src[l];
}

void orc_set_fields_f32(orc* o, const float* dens, const float* vrad, const float* vtheta, const float* energy) {
  size_t n = o->size_grid;
  cp_in(o->Dens, dens, n);
  cp_in(o->Vrad, vrad, n);
  cp_in(o->Vtheta, vtheta, n);
  cp_in(o->Energy, energy, n);
}

void orc_get_fields_f32(const orc* o, float* dens, float* vrad, float* vtheta, float* energy, float* temperature,
                        float* qplus) {
  size_t n = o->size_grid;
  cp_out(dens, o->Dens, n);
  cp_out(vrad, o->Vrad, n);
  cp_out(vtheta, o->Vtheta, n);
  cp_out(energy, o->Energy, n);
  cp_out(temperature, o->Temperature, n);
  cp_out(qplus, o->Qplus, n);
}

/* The self-gravity accelerations (SG_Accr, SG_Acct; NRAD*NSEC each) of the
   current density, as compute_selfgravity leaves them (SgMain.cu:23-45).
   Returns -1 when the run has no self-gravity. */
int orc_sg_accelerations(orc* o, double* accr, double* acct) {
  if (!o->p.SelfGravity) return -1;
  sg_accelerations(o);
  size_t n = (size_t)o->nrad * o->nsec;
  for (size_t l = 0; l < n; l++) {
    accr[l] = o->SG_Accr[l];
    acct[l] = o->SG_Acct[l];
  }
  return 0;
}

/* Precision mode: 0 the reference's arithmetic (default), 1 accurate.  Call
   before the first DT (re-tabulates the self-gravity kernel). */
void orc_set_precision(orc* o, int mode) {
  o->accurate = mode == 1;
  if (!o->star_grad) o->star_grad = zr(o->nrad + 1);
  for (int i = 1; i < o->nrad; i++) o->star_grad[i] = (real)(G / (o->Rmed2[i] * o->Rmed2[i - 1]));
  if (o->p.SelfGravity) sg_init_kernel(o);
}

void orc_get_planets(const orc* o, fargo_planets* out) { *out = o->sys; }
void orc_set_planets(orc* o, const fargo_planets* in) { o->sys = *in; }

int orc_substep_log(const orc* o, int cap, int* nshift, double* dt) {
  int n = o->nsub < MAXSUB ? o->nsub : MAXSUB;
  if (n > cap) n = cap;
  if (nshift) memcpy(nshift, o->log_nshift, sizeof(int) * (size_t)n * o->nrad);
  if (dt) memcpy(dt, o->log_dt, sizeof(double) * n);
  return o->nsub;
}

void orc_get_scalars(orc* o, fargo_scalars* s) {
  memset(s, 0, sizeof(*s));
  s->physical_time = o->PhysicalTime;
  s->omega_frame = o->OmegaFrame;
  s->mdcp1 = circum_planetary_mass(o);
  s->lost_mass = o->LostMass;
  s->nsub_last_dt = o->nsub;
  s->nsub_total = o->nsub_total;
  s->last_dt = o->last_dt;
  double m = 0, am = 0;
  int nsec = o->nsec;
  for (int i = 0; i < o->nrad; i++)
    for (int j = 0; j < nsec; j++) {
      int l = i * nsec + j, jp = i * nsec + (j + 1) % nsec;
      double cm = (double)o->Surf[i] * (double)o->Dens[l];
      m += cm;
      am += cm * (double)o->Rmed[i] *
            (0.5 * ((double)o->Vtheta[l] + (double)o->Vtheta[jp]) + (double)o->Rmed[i] * o->OmegaFrame);
    }
  s->mass = m;
  s->angular_momentum = am;
}

void orc_get_table(const orc* o, int which, double* out) {
  const real* t = NULL;
  switch (which) {
    case 0: t = o->Radii; break;
    case 1: t = o->Rinf; break;
    case 2: t = o->Rsup; break;
    case 3: t = o->Rmed; break;
    case 4: t = o->Surf; break;
    case 5: t = o->invRinf; break;
    case 6: t = o->invSurf; break;
    case 7: t = o->invRmed; break;
    case 8: t = o->invdiffRsup; break;
    case 9: t = o->invdiffRmed; break;
    case 10: t = o->SigmaMed; break;
    case 11: t = o->SigmaInf; break;
    case 12: t = o->EnergyMed; break;
    case 13: t = o->viscosity_array; break;
    case 14:
      for (int i = 0; i <= o->nrad; i++) out[i] = o->SoundSpeed[(size_t)i * o->nsec];
      return;
    default: return;
  }
  for (int i = 0; i <= o->nrad; i++) out[i] = t[i];
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
