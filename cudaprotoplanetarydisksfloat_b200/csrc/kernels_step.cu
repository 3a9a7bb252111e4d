// kernels_step.cu -- sm_100a kernels of one FARGO hydro substep, batched over disks.
//
// The reference runs ~120 single-purpose kernels, ~50 host-side reductions
// (each with cudaMalloc/cudaFree) and ~15 full-grid device copies per
// substep, with a device synchronisation after every launch
// (SourceEuler.cu:230-299).  Here one substep of an isothermal batch is 10
// launches that read and write only the disk state and a few scratch fields,
// with the CFL count, the disk forces and the planet integrator kept on the
// device:
//
//   k_ring_mean<0>   serial FP32 ring means of v_theta for the CFL
//   k_cfl_force      CFL minimum, disk-on-body forces on 4096-cell tiles; the
//                    last block of each disk finishes the substep's scalar
//                    work (dt, mass taper, potential parameters, planet kicks,
//                    FP64 RK5, frame rotation, per-ring viscosity)
//   k_potential      star and planet potential of every cell
//   k_source1        Substep1 (pressure + potential + centrifugal kick) +
//                    self-gravity kick; one instance per kind of disk
//   k_viscosity      viscous stress tensor + velocity update + sub-Keplerian
//                    boundary on 16x64 tiles staged in shared memory
//   k_source2        artificial viscosity (Substep2) + energy predictor
//   k_energy         viscous heating and implicit energy update (Substep3)
//   k_ring_mean<1>   ring means of v_theta for FARGO: Nshift, residual
//   k_transport      a band of 8 rings x one segment of source sectors per
//                    CTA: momenta + radial van Leer from staged rows, residual
//                    and constant azimuthal van Leer sweeps (quantities in
//                    pairs of FP32 lanes), shift applied on the store
//   k_velocities     velocities from the transported momenta
//   k_substep_end    disks still inside their DT -> graph loop condition
//
// The cell kernels take four consecutive cells per thread (quads).
//
// Arithmetic per cell follows the reference kernels expression by expression
// (a float meeting a double literal is promoted and rounded back on
// assignment); where the reference computes one IEEE operation in double on
// two float operands and rounds to float, the float operation is used, which
// gives the same bits.  Per-cell quotients (Substep1, Substep2, the viscous
// update, the viscous heating and energy update, the velocities) use div_refined
// (fast_div.cuh): the IEEE quotient but within ~2^-22 ulp of a rounding
// boundary, one ulp from it there.
#include <cuda_runtime.h>

#include <cmath>
#include <algorithm>
#include <cstdio>
#include <type_traits>

#include "fargo_internal.h"
#include "fast_div.cuh"

#define PI_D FARGO_PI
#define CVNR FARGO_CVNR
#define CFLSEC FARGO_CFLSECURITY

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int disk_of_cell(const BatchDev& B, long long c) {
  int lo = 0, hi = B.ndisk - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (B.cell_off[mid] <= c)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int disk_of_ring(const BatchDev& B, int r) {
  int lo = 0, hi = B.ndisk - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (B.ring_off[mid] <= r)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int jwrap_m(int j, int nsec) { return j == 0 ? nsec - 1 : j - 1; }
__device__ __forceinline__ int jwrap_p(int j, int nsec) { return j + 1 == nsec ? 0 : j + 1; }

// max2 / min2, Kernels.cu:1459-1470
__device__ __forceinline__ float max2(float a, float b) { return (b > a) ? b : a; }

// Kahan-compensated FP32 sum (accurate mode's ring means): the same order as
// the plain sum, with the rounding error of every addition carried into the
// next one.  No multiplications, so no contraction into fused multiply-adds.
struct KahanSum {
  float s = 0.0f, c = 0.0f;
  __device__ __forceinline__ void add(float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
  }
};
__device__ __forceinline__ float min2(float a, float b) { return (b < a) ? b : a; }

// AspectRatioDevice, Kernels.cu:1473-1488
__device__ float aspect_ratio_dev(const DiskDev& D, float r, float PT, float PTI) {
  float aspectratio, rmin, rmax, scale;
  aspectratio = D.ASPECTRATIO;
  rmin = D.TRANSITIONRADIUS - D.TRANSITIONWIDTH * D.ASPECTRATIO;
  rmax = D.TRANSITIONRADIUS + D.TRANSITIONWIDTH * D.ASPECTRATIO;
  scale = 1.0 + (PT - PTI) * D.LAMBDADOUBLING;
  rmin *= scale;
  rmax *= scale;
  if (r < rmin) aspectratio *= D.TRANSITIONRATIO;
  if ((r >= rmin) && (r <= rmax)) aspectratio *= expf((rmax - r) / (rmax - rmin) * logf(D.TRANSITIONRATIO));
  return aspectratio;
}

// AspectRatioHost, Viscosity.cu:39-52 (double math)
__device__ float aspect_ratio_host(const DiskDev& D, float r, float PT, float PTI) {
  float aspectratio, rmin, rmax, scale;
  aspectratio = D.ASPECTRATIO;
  rmin = D.TRANSITIONRADIUS - D.TRANSITIONWIDTH * D.ASPECTRATIO;
  rmax = D.TRANSITIONRADIUS + D.TRANSITIONWIDTH * D.ASPECTRATIO;
  scale = 1.0 + (PT - PTI) * D.LAMBDADOUBLING;
  rmin *= scale;
  rmax *= scale;
  if (r < rmin) aspectratio *= D.TRANSITIONRATIO;
  if ((r >= rmin) && (r <= rmax))
    aspectratio *= exp((rmax - r) / (rmax - rmin) * log((double)D.TRANSITIONRATIO));
  return aspectratio;
}

// FViscosity, Viscosity.cu:19-37.  The ring search `while (Rmed[k] < r) k++`
// ends at k = i for r = Rmed[i] on a strictly increasing grid.
__device__ float fviscosity_ring(const DiskDev& D, int i, float PT, float PTI) {
  float r = D.Rmed[i];
  float viscosity, rmin, rmax, scale;
  viscosity = D.VISCOSITY;
  if (D.ViscosityAlpha) {
    float g = D.csmean[i];
    viscosity = D.ALPHAVISCOSITY * g * g * D.pow15[i];
  }
  rmin = D.CAVITYRADIUS - D.CAVITYWIDTH * D.ASPECTRATIO;
  rmax = D.CAVITYRADIUS + D.CAVITYWIDTH * D.ASPECTRATIO;
  scale = 1.0 + (PT - PTI) * D.LAMBDADOUBLING;
  rmin *= scale;
  rmax *= scale;
  if (r < rmin) viscosity *= D.CAVITYRATIO;
  if ((r >= rmin) && (r <= rmax)) viscosity *= exp((rmax - r) / (rmax - rmin) * log((double)D.CAVITYRATIO));
  return viscosity;
}

// Compute_smoothing, Force.cu:69-74 (AspectRatioHost takes a float radius)
__device__ double compute_smoothing(const DiskDev& D, double r, float PT, float PTI) {
  return D.THICKNESSSMOOTHING * aspect_ratio_host(D, (float)r, PT, PTI) * pow(r, 1.0 + D.FLARINGINDEX);
}

// ---------------------------------------------------------------- planets (FP64)

// The planet integrator runs on the 32 lanes of one warp: lane l takes
// planets l, l+32, ... in the derivative and elements l, l+32, ... of the
// Runge-Kutta combinations, each with the reference's expression, so the
// result is the one thread's result bit for bit (nothing is reassociated);
// __syncwarp orders the phases.

// DerivMotionRK5, RungeKutta.cu:9-46; the planet-planet term divides by the
// cube of the perturber's distance to the star, as the reference does.
__device__ void deriv_motion(const DiskDev& D, const DiskCtl* C, const double* q, double* deriv, int nb,
                             float dt, double* Dist, int lane) {
  const double *x = q, *y = q + nb, *vx = q + 2 * nb, *vy = q + 3 * nb;
  double *dx = deriv, *dy = deriv + nb, *dvx = deriv + 2 * nb, *dvy = deriv + 3 * nb;
  // m_j / d_j / d_j / d_j depends on j alone: formed once per perturber (the
  // same expression, so the same bits), not once per pair; Dist holds the
  // distances in [0, nb) and these quotients in [nb, 2 nb)
  double* mD3 = Dist + nb;
  for (int i = lane; i < nb; i += 32) {
    Dist[i] = sqrt(x[i] * x[i] + y[i] * y[i]);
    mD3[i] = 1.0 * C->mass[i] / Dist[i] / Dist[i] / Dist[i];
  }
  __syncwarp();
  for (int i = lane; i < nb; i += 32) {
    double ax = -1.0 * 1.0 / Dist[i] / Dist[i] / Dist[i] * x[i];
    double ay = -1.0 * 1.0 / Dist[i] / Dist[i] / Dist[i] * y[i];
    for (int j = 0; j < nb; j++) {
      if (D.Indirect_Term) {
        ax -= mD3[j] * x[j];
        ay -= mD3[j] * y[j];
      }
      if ((j != i) && C->feelothers[i]) {
        ax += mD3[j] * (x[j] - x[i]);
        ay += mD3[j] * (y[j] - y[i]);
      }
    }
    dx[i] = vx[i] * dt;
    dy[i] = vy[i] * dt;
    dvx[i] = ax * dt;
    dvy[i] = ay * dt;
  }
  __syncwarp();
}

// RungeKutta, RungeKutta.cu:55-74 (Cash-Karp coefficients of the reference)
__device__ void runge_kutta(const DiskDev& D, const DiskCtl* C, const double* q0, float dt, double* q1,
                            double* k, int nb, double* Dist, int lane) {
  const double c[5][5] = {{0.2, 0.0, 0.0, 0.0, 0.0},
                          {0.075, 0.225, 0.0, 0.0, 0.0},
                          {0.3, -0.9, 1.2, 0.0, 0.0},
                          {-11.0 / 54.0, 2.5, -70.0 / 27.0, 35.0 / 27.0, 0.0},
                          {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0}};
  int n4 = 4 * nb;
  for (int s = lane; s < 6 * n4; s += 32) k[s] = 0.0;
  __syncwarp();
  deriv_motion(D, C, q0, k, nb, dt, Dist, lane);
  for (int s = 0; s < 5; s++) {
    for (int i = lane; i < n4; i += 32)
      q1[i] = q0[i] + c[s][0] * k[i] + c[s][1] * k[n4 + i] + c[s][2] * k[2 * n4 + i] +
              c[s][3] * k[3 * n4 + i] + c[s][4] * k[4 * n4 + i];
    __syncwarp();
    deriv_motion(D, C, q1, k + (s + 1) * n4, nb, dt, Dist, lane);
  }
  for (int i = lane; i < n4; i += 32)
    q1[i] = q0[i] + 37.0 / 378.0 * k[i] + 250.0 / 621.0 * k[2 * n4 + i] + 125.0 / 594.0 * k[3 * n4 + i] +
            512.0 / 1771.0 * k[5 * n4 + i];
  __syncwarp();
}

// AdvanceSystemRK5, Pframeforce.cu:94-157; work holds FARGO_RK_WORK(nb)
// doubles.  Called by the 32 lanes of one warp (the Runge-Kutta step is
// lane-parallel, the rest runs on lane 0).
__device__ void advance_system_rk5(const DiskDev& D, DiskCtl* C, float dt, float PT, double* work, int lane) {
  int nb = C->nb;
  double dtheta, omega, rdot, x, y, r, new_r, vx, vy, theta, denom;
  double* q0 = work;
  double* q1 = work + 4 * nb;
  double* k = work + 8 * nb;
  double* Dist = work + 32 * nb;
  if (!D.ForcedCircular && nb > 0) {
    for (int i = lane; i < nb; i += 32) {
      q0[i] = C->x[i];
      q0[i + nb] = C->y[i];
      q0[i + 2 * nb] = C->vx[i];
      q0[i + 3 * nb] = C->vy[i];
    }
    __syncwarp();
    runge_kutta(D, C, q0, dt, q1, k, nb, Dist, lane);
  }
  if (lane != 0) return;
  for (int i = 1 - (PT >= D.RELEASEDATE); i < nb; i++) {
    if (!D.ForcedCircular) {
      C->x[i] = q1[i];
      C->y[i] = q1[i + nb];
      C->vx[i] = q1[i + 2 * nb];
      C->vy[i] = q1[i + 3 * nb];
    } else {
      x = C->x[i];
      y = C->y[i];
      theta = atan2(y, x);
      vx = C->vx[i];
      vy = C->vy[i];
      r = sqrt(x * x + y * y);
      omega = (-y * vx + x * vy) / r / r;
      dtheta = omega * dt;
      C->x[i] = r * cos(theta + dtheta);
      C->y[i] = r * sin(theta + dtheta);
      C->vx[i] = vx * cos(dtheta + theta) - vy * sin(dtheta + theta);
      C->vy[i] = vx * sin(dtheta + theta) + vy * cos(dtheta + theta);
    }
  }
  if (PT < D.RELEASEDATE && nb > 0) {
    x = C->x[0];
    y = C->y[0];
    r = sqrt(x * x + y * y);
    theta = atan2(y, x);
    rdot = (D.RELEASERADIUS - r) / (D.RELEASEDATE - PT);
    omega = sqrt((1. + C->mass[0]) / r / r / r);
    new_r = r + rdot * dt;
    denom = r - new_r;
    if (denom != 0.0)
      dtheta = 2. * dt * r * omega / denom * (sqrt(r / new_r) - 1.);
    else
      dtheta = omega * dt;
    vx = rdot;
    vy = new_r * sqrt((1. + C->mass[0]) / new_r / new_r / new_r);
    C->x[0] = new_r * cos(dtheta + theta);
    C->y[0] = new_r * sin(dtheta + theta);
    C->vx[0] = vx * cos(dtheta + theta) - vy * sin(dtheta + theta);
    C->vy[0] = vx * sin(dtheta + theta) + vx * cos(dtheta + theta);  // Pframeforce.cu:154 uses vx twice
  }
}

// GetPsysInfo, Psys.cu:236-306 (0 = GET, 1 = MARK, 2 = FREQUENCY)
__device__ float get_psys_info(const DiskDev& D, DiskCtl* C, int action) {
  double d1, d2, cross;
  double x, y, vx, vy, m, h, d, Ax, Ay, e, a, E, M;
  double xc, yc, omega;
  double arg, PerihelionPA;
  xc = x = C->x[0];
  yc = y = C->y[0];
  vx = C->vx[0];
  vy = C->vy[0];
  m = C->mass[0] + 1.;
  h = x * vy - y * vx;
  d = sqrt(x * x + y * y);
  Ax = x * vy * vy - y * vx * vy - 1.0 * m * x / d;
  Ay = y * vx * vx - x * vx * vy - 1.0 * m * y / d;
  e = sqrt(Ax * Ax + Ay * Ay) / m;
  a = h * h / 1.0 / m / (1. - e * e);
  if (e == 0.0)
    arg = 1.0;
  else
    arg = (1.0 - d / a) / e;
  if (fabs(arg) >= 1.0)
    E = PI_D * (1. - arg / fabs(arg)) / 2.;
  else
    E = acos((1.0 - d / a) / e);
  if ((x * y * (vy * vy - vx * vx) + vx * vy * (x * x - y * y)) < 0) E = -E;
  M = E - e * sin(E);
  omega = sqrt(m / a / a / a);
  PerihelionPA = atan2(Ay, Ax);
  if (D.GuidingCenter) {
    xc = a * cos(M + PerihelionPA);
    yc = a * sin(M + PerihelionPA);
  }
  if (e < 1e-8) {
    xc = x;
    yc = y;
  }
  switch (action) {
    case 1:
      C->Xplanet_mark = xc;
      C->Yplanet_mark = yc;
      return 0.;
    case 0:
      x = xc;
      y = yc;
      d2 = sqrt(x * x + y * y);
      d1 = sqrt((double)C->Xplanet_mark * C->Xplanet_mark + (double)C->Yplanet_mark * C->Yplanet_mark);
      cross = C->Xplanet_mark * y - x * C->Yplanet_mark;
      C->Xplanet_mark = x;
      C->Yplanet_mark = y;
      return asin(cross / (d1 * d2));
    case 2:
      return omega;
  }
  return 0.0;
}

// RotatePsys, Psys.cu:308-325
__device__ void rotate_psys(DiskCtl* C, float angle) {
  double sint = sin((double)angle), cost = cos((double)angle), xt, yt;
  for (int i = 0; i < C->nb; i++) {
    xt = C->x[i];
    yt = C->y[i];
    C->x[i] = xt * cost + yt * sint;
    C->y[i] = -xt * sint + yt * cost;
    xt = C->vx[i];
    yt = C->vy[i];
    C->vx[i] = xt * cost + yt * sint;
    C->vy[i] = -xt * sint + yt * cost;
  }
}

// Arguments of the force kernel for the star and every FeelDisk planet at
// the planets' current positions (ComputeAccel takes floats, SideEuler.cu:151;
// ComputeForce derives a and rh from them, Force.cu:311-312).
__device__ void prepare_bodies(const DiskDev& D, DiskCtl* C) {
  int nbody = 0;
  C->bx[0] = 0.0f;
  C->by[0] = 0.0f;
  C->brs[0] = 0.0f;
  C->ba[0] = 0.0f;
  C->brh[0] = (float)(pow(0.0 / 3., 1. / 3.) * 0.0 + 1e-15);
  C->body_planet[0] = -1;
  nbody = 1;
  for (int k = 0; k < C->nb && nbody < FARGO_MAXBODY; k++) {
    if (!C->feeldisk[k]) continue;
    double m = C->mass[k], x = C->x[k], y = C->y[k];
    double r = sqrt(x * x + y * y), smoothing;
    if (D.RocheSmoothing)
      smoothing = r * pow(m / 3., 1. / 3.) * D.ROCHESMOOTHING;
    else
      smoothing = compute_smoothing(D, r, C->PhysicalTime, C->PhysicalTimeInitial);
    float xf = (float)x, yf = (float)y, rsf = (float)smoothing, mf = (float)m;
    double a = sqrt((double)xf * xf + (double)yf * yf);
    double rh = pow((double)mf / 3., 1. / 3.) * a + 1e-15;
    C->bx[nbody] = xf;
    C->by[nbody] = yf;
    C->brs[nbody] = rsf;
    C->brh[nbody] = (float)rh;
    C->ba[nbody] = (float)a;
    C->body_planet[nbody] = k;
    nbody++;
  }
  C->nbody = nbody;
}


// Binary search in a prefix array off[0..n] (off[0] = 0): the a with off[a] <= x < off[a+1].
template <class T>
__device__ __forceinline__ int find_range(const T* off, int n, T x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= x)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Walk over the cells of the disks still inside their DT, in tiles of
// kThreads consecutive cells of one disk.  Each block takes a contiguous run
// of tiles, so it meets few disks; on entering a disk the block copies its
// DiskDev to shared memory, and the body's field reads then neither chase
// global pointers nor reload after its stores.
static_assert(sizeof(DiskDev) % 4 == 0, "DiskDev copy by words");
__device__ __forceinline__ void copy_words(void* dst, const void* src, int bytes) {
  const int* s = reinterpret_cast<const int*>(src);
  int* d = reinterpret_cast<int*>(dst);
  for (int k = threadIdx.x; k < bytes / 4; k += blockDim.x) d[k] = s[k];
}

// Four consecutive cells c0 .. c0+3 of one disk (c0 a multiple of 4).  With
// vec (NSEC a multiple of 4) they share a ring, start at a sector multiple
// of 4, and their fields load and store as 16-byte vectors; otherwise each
// cell is addressed on its own and may lie past the disk's end (!ok).
template <bool V>
struct Quad {
  static constexpr bool vec = V;
  int i[4], j[4], l[4];
  bool ok[4];
};

// Walk over the cells of the disks still inside their DT in tiles of
// FARGO_QTILE cells, four per thread.  Each block takes a contiguous run of
// tiles, so it meets few disks; on entering a disk the block copies its
// DiskDev to shared memory.  A thread's quad advances by FARGO_QTILE cells
// from one tile to the next (no division after the disk's first tile); the
// tiles of one disk form an inner loop without barriers.  kAdi, kSg (0 or 1;
// -1: any): only the disks whose Adiabatic / SelfGravity flags match (the
// energy kernel takes adiabatic disks, the Substep1 instances one kind each).
static_assert(FARGO_QTILE == 4 * kThreads, "four cells per thread");
template <int kAdi, int kSg, class Body>
__device__ __forceinline__ void for_active_quads(const BatchDev& B, Body body) {
  __shared__ DiskDev sD;
  const int na = B.act[0];
  if (na <= 0) return;
  const int ntile = B.act_tile_off[na];
  const int per = (ntile + gridDim.x - 1) / gridDim.x;
  const int t0 = blockIdx.x * per, t1 = min(t0 + per, ntile);
  int t = t0;
  while (t < t1) {  // block-uniform: one disk per pass
    const int a = find_range(B.act_tile_off, na, t);
    const int lo = B.act_tile_off[a], te = min(t1, B.act_tile_off[a + 1]);
    __syncthreads();
    copy_words(&sD, B.disks + B.act_disk[a], sizeof(DiskDev));
    __syncthreads();
    if (!sD.IsDisk || (kAdi >= 0 && (sD.Adiabatic != 0) != (kAdi == 1)) ||
        (kSg >= 0 && (sD.SelfGravity != 0) != (kSg == 1))) {  // nothing to do on this disk
      t = te;
      continue;
    }
    const int nsec = sD.nsec, nrad = sD.nrad;
    const int c0 = (t - lo) * FARGO_QTILE + 4 * threadIdx.x;
    int i = c0 / nsec, j = c0 - i * nsec;
    if ((nsec & 3) == 0) {
      for (; t < te; t++) {
        if (i < nrad) {
          Quad<true> q;
#pragma unroll
          for (int u = 0; u < 4; u++) {
            q.i[u] = i;
            q.j[u] = j + u;
            q.l[u] = i * nsec + j + u;
            q.ok[u] = true;
          }
          body(sD, sD.ctl, q);
        }
        j += FARGO_QTILE;
        while (j >= nsec) {
          j -= nsec;
          i++;
        }
      }
    } else {
      for (; t < te; t++) {
        Quad<false> q;
        int ii = i, jj = j;
#pragma unroll
        for (int u = 0; u < 4; u++) {
          q.ok[u] = ii < nrad;
          q.i[u] = q.ok[u] ? ii : 0;
          q.j[u] = q.ok[u] ? jj : 0;
          q.l[u] = q.i[u] * nsec + q.j[u];
          if (++jj == nsec) {
            jj = 0;
            ii++;
          }
        }
        if (q.ok[0]) body(sD, sD.ctl, q);
        j += FARGO_QTILE;
        while (j >= nsec) {
          j -= nsec;
          i++;
        }
      }
    }
  }
}

// Store to global memory for the cell kernels.  None of them reads back in
// the same launch what it stores, so the store is not ordered against the
// compiler's loads (no memory clobber): loads of the disk's fields from
// shared memory need not be repeated after it.
__device__ __forceinline__ void stg(float* p, float v) {
  asm volatile("st.global.f32 [%0], %1;\n" ::"l"(p), "f"(v));
}

__device__ __forceinline__ void stg4(float* p, float a, float b, float c, float d) {
  asm volatile("st.global.v4.f32 [%0], {%1, %2, %3, %4};\n" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d));
}

// Quad loads and stores.  Row offsets: 0 (ring i), +nsec (ring i+1, the
// ghost row for the last ring), -nsec (ring i-1: zero where i == 0).
template <bool V>
__device__ __forceinline__ void qld(float (&v)[4], const float* p, const Quad<V>& q, int roff = 0) {
  if (V) {
    if (roff < 0 && q.i[0] == 0) {
      v[0] = v[1] = v[2] = v[3] = 0.0f;
      return;
    }
    const float4 t = __ldg(reinterpret_cast<const float4*>(p + q.l[0] + roff));
    v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
  } else {
#pragma unroll
    for (int u = 0; u < 4; u++) v[u] = (q.ok[u] && (roff >= 0 || q.i[u] > 0)) ? __ldg(p + q.l[u] + roff) : 0.0f;
  }
}
// values at (i, j-1) of each cell, given the same row's values c at (i, j)
template <bool V>
__device__ __forceinline__ void qld_jm(float (&v)[4], const float (&c)[4], const float* p, const Quad<V>& q, int nsec,
                                       int roff = 0) {
  if (V) {
    v[0] = (roff < 0 && q.i[0] == 0) ? 0.0f : __ldg(p + q.i[0] * nsec + jwrap_m(q.j[0], nsec) + roff);
    v[1] = c[0], v[2] = c[1], v[3] = c[2];
  } else {
#pragma unroll
    for (int u = 0; u < 4; u++)
      v[u] = (q.ok[u] && (roff >= 0 || q.i[u] > 0)) ? __ldg(p + q.i[u] * nsec + jwrap_m(q.j[u], nsec) + roff) : 0.0f;
  }
}
// values at (i, j+1) of each cell, given the same row's values c at (i, j)
template <bool V>
__device__ __forceinline__ void qld_jp(float (&v)[4], const float (&c)[4], const float* p, const Quad<V>& q, int nsec,
                                       int roff = 0) {
  if (V) {
    v[0] = c[1], v[1] = c[2], v[2] = c[3];
    v[3] = (roff < 0 && q.i[0] == 0) ? 0.0f : __ldg(p + q.i[0] * nsec + jwrap_p(q.j[3], nsec) + roff);
  } else {
#pragma unroll
    for (int u = 0; u < 4; u++)
      v[u] = (q.ok[u] && (roff >= 0 || q.i[u] > 0)) ? __ldg(p + q.i[u] * nsec + jwrap_p(q.j[u], nsec) + roff) : 0.0f;
  }
}
// sector-table values (index j) of each cell
template <bool V>
__device__ __forceinline__ void qld_sector(float (&v)[4], const float* p, const Quad<V>& q) {
  if (V) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p + q.j[0]));
    v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
  } else {
#pragma unroll
    for (int u = 0; u < 4; u++) v[u] = __ldg(p + q.j[u]);
  }
}
template <bool V>
__device__ __forceinline__ void qst(float* p, const Quad<V>& q, const float (&v)[4], int roff = 0) {
  if (V) {
    stg4(p + q.l[0] + roff, v[0], v[1], v[2], v[3]);
  } else {
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (q.ok[u]) stg(p + q.l[u] + roff, v[u]);
  }
}

#define QUAD_BEGIN_T(kAdi, kSg)                                                                         \
  for_active_quads<kAdi, kSg>(B, [&](const DiskDev& D, const DiskCtl* C, const auto& q) {              \
    constexpr bool V = std::decay_t<decltype(q)>::vec;                                                 \
    (void)V;                                                                                           \
    const int nsec = D.nsec, nrad = D.nrad;                                                            \
    (void)nsec;                                                                                        \
    (void)nrad;
#define QUAD_BEGIN QUAD_BEGIN_T(-1, -1)
#define QUAD_END \
  });

// -------------------------------------------------------------- reductions

// DeviceReduce<float> (Kernels.cu:431-557) of f(0) .. f(n-1) in the
// reference's order of operations, for the whole block (kThreads threads):
// getNumBlocksAndThreads (Kernels.cu:404-429) picks the reference's block
// count and size, each of its blocks is reduced in turn as deviceReduceKernel
// does (Kernels.cu:269-383: the bounds-checked form, since IsPow2 is false
// for every n > 1; shared-memory tree down to 64, the last warp by shuffles),
// and the block sums are added in order as its host loop does.  Result in
// every thread.  n > 128 (the reference launches no block below that).
template <class F>
__device__ float ref_device_reduce(F f, int n, float* sm) {
  long np2 = 1;
  while (np2 < n) np2 <<= 1;
  const long maxBlocks = np2 / 256;
  long h = (n + 1) / 2, T2 = 1;
  while (T2 < h) T2 <<= 1;
  const int T = (n < 512) ? (int)T2 : 256;
  long blocks = (n + (2L * T - 1)) / (2L * T);
  if (blocks > maxBlocks) blocks = maxBlocks;
  const int t = threadIdx.x;
  float total = 0.0f;
  for (long b = 0; b < blocks; b++) {
    float my = 0.0f;
    __syncthreads();
    if (t < T) {
      const long gridSize = 2L * T * blocks;
      for (long i = b * 2L * T + t; i < n; i += gridSize) {
        my += f(i);
        if (i + T < n) my += f(i + T);
      }
      sm[t] = my;
    }
    __syncthreads();
    for (int stride = 256; stride >= 64; stride >>= 1) {
      if (T >= 2 * stride && t < stride) sm[t] = my = my + sm[t + stride];
      __syncthreads();
    }
    if (t < 32) {
      if (T >= 64) my = my + sm[t + 32];
      for (int off = 16; off > 0; off >>= 1) my += __shfl_down_sync(0xffffffffu, my, off);
      if (t == 0) total += my;
    }
  }
  __syncthreads();
  if (t == 0) sm[0] = total;
  __syncthreads();
  const float r = sm[0];
  __syncthreads();
  return r;
}

__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_min_f(float v) {
  for (int o = 16; o > 0; o >>= 1) {
    float w = __shfl_down_sync(0xffffffffu, v, o);
    if (w < v) v = w;
  }
  return v;
}

// Minimum over the block with the reference's ordered comparison
// (`if (x < m) m = x`, so NaNs are skipped).  All threads get the result.
__device__ float block_min_f(float v, float* sh) {
  v = warp_min_f(v);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (l < (int)(blockDim.x >> 5)) ? sh[l] : 1e30f;
    v = warp_min_f(v);
    if (l == 0) sh[0] = v;
  }
  __syncthreads();
  float r = sh[0];
  __syncthreads();
  return r;
}

// -------------------------------------------------------------- CFL + forces

// The scalar part of the substep (SourceEuler.cu:231-264), run by the block
// that completed a disk's last CFL tile (or, for a radial stripe, by
// k_stripe_finish once every stripe's partials are gathered).
constexpr int kRkShared = 16;  // planets whose RK5 scratch fits in shared memory
__device__ bool finish_serial(const DiskDev& D, DiskCtl* C, float newdt, const double* s_sum);
__device__ void finish_serial_tail(const DiskDev& D, DiskCtl* C);

// ConditionCFL host part (SourceEuler.cu:513-535): the shear limit DT1D
// (ConditionCFLKernel2D2, Kernels.cu:1425-1428) of the ring pairs (i, i+1),
// i in [i0, i1), folded into a thread's running minimum.
__device__ __forceinline__ float dt1d_min(const DiskDev& D, int i0, int i1, int tid, int nt, float m) {
#pragma unroll 4
  for (int i = i0 + tid; i < i1; i += nt) {
    float dt1 = 2.0 * PI_D * CFLSEC / (float)D.nsec / fabsf(D.vmoy[i] * D.invRmed[i] - D.vmoy[i + 1] * D.invRmed[i + 1]);
    if (dt1 < m) m = dt1;
  }
  return m;
}

// Inputs of the finishing sums of a whole disk: its CFL tiles' minima and
// force partials ([sum][tile]), written by the blocks of this launch (read
// through L2), and the shear limit of every ring pair.
struct DiskTiles {
  const DiskDev& D;
  int nct;
  __device__ float thread_min(int tid, int nt) const {
    float m = 1e30f;
#pragma unroll 4
    for (int t = tid; t < nct; t += nt) {
      float v = __ldcg(D.ringmin + t);
      if (v < m) m = v;
    }
    return dt1d_min(D, 0, D.nrad - 1, tid, nt, m);
  }
  __device__ int ntiles() const { return nct; }
  __device__ double partial(int q, int t) const { return __ldcg(D.partials + (size_t)q * nct + t); }
};

// Inputs of the finishing sums of a radially decomposed disk: one block per
// stripe, gathered from every stripe in stripe order (k_stripe_block writes
// them): [0] the minimum over the stripe's tiles and own ring pairs, [1] its
// CFL tile count, [2] its body count, then its force partials [sum][tile].
// The stripes' tiles, concatenated, are the whole disk's tiles (stripe
// boundaries on tile boundaries), so the sums below add the same partials in
// the same order as DiskTiles does.
constexpr int kStripeHead = FARGO_STRIPE_HEAD;
struct StripeBlocks {
  const double* blk;
  int nstripe, stride;
  const int* t0;  // shared: first tile of each stripe, t0[nstripe] = all tiles
  __device__ float thread_min(int tid, int nt) const {
    float m = 1e30f;
    for (int s = tid; s < nstripe; s += nt) {
      float v = (float)blk[(size_t)s * stride];
      if (v < m) m = v;
    }
    return m;
  }
  __device__ int ntiles() const { return t0[nstripe]; }
  __device__ double partial(int q, int t) const {
    int lo = 0, hi = nstripe - 1;  // the stripe s with t0[s] <= t < t0[s+1]
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (t0[mid] <= t)
        lo = mid;
      else
        hi = mid - 1;
    }
    const int n = t0[lo + 1] - t0[lo];
    return blk[(size_t)lo * stride + kStripeHead + (size_t)q * n + (t - t0[lo])];
  }
};

// Substep scalars of one disk, run by one block: the CFL minimum, the disk
// forces summed over the tiles in a fixed order, the viscosity per ring and
// the serial part (on a shared-memory copy of the disk's control block, sC,
// written back at the end).
template <int NB, class Src>
__device__ void finish_cfl_and_planets(const DiskDev& D, DiskCtl* Cg, DiskCtl* sC, float* shf, double* s_sum,
                                       double* s_work, const Src& src) {
  const int nrad = D.nrad, tid = threadIdx.x;
  const int nct = src.ntiles();
  float newdt = block_min_f(src.thread_min(tid, blockDim.x), shf);
  // disk-force sums over the tiles in a fixed order: every thread a strided
  // share of the tiles for all sums at once, the warps by shuffle, then the
  // warps in order (s_work is free until the planet update)
  const int nbody = min(Cg->nbody, NB), nsum = 4 * nbody;
  const int w = tid >> 5, l = tid & 31, nw = blockDim.x >> 5;
  double acc[4 * NB];
#pragma unroll
  for (int q = 0; q < 4 * NB; q++) acc[q] = 0.0;
#pragma unroll 2
  for (int t = tid; t < nct; t += blockDim.x) {
#pragma unroll
    for (int q = 0; q < 4 * NB; q++)
      if (q < nsum) acc[q] += src.partial(q, t);
  }
#pragma unroll
  for (int q = 0; q < 4 * NB; q++) {
    if (q < nsum) {
      const double v = warp_sum_d(acc[q]);
      if (l == 0) s_work[q * nw + w] = v;
    }
  }
  __syncthreads();
  if (tid < nsum) {
    double acc = 0.0;
    for (int u = 0; u < nw; u++) acc += s_work[tid * nw + u];
    s_sum[tid] = acc;
  }
  // FViscosity per ring for this substep (Viscosity.cu:84-85, SourceEuler.cu:350)
  const float PT = Cg->PhysicalTime;
  for (int i = tid; i < nrad; i += blockDim.x) D.visc[i] = fviscosity_ring(D, i, PT, Cg->PhysicalTimeInitial);
  {
    const int* src = reinterpret_cast<const int*>(Cg);
    int* dst = reinterpret_cast<int*>(sC);
    for (int k = tid; k < (int)(sizeof(DiskCtl) / 4); k += blockDim.x) dst[k] = src[k];
  }
  __syncthreads();
  // the serial part on thread 0, the planet integrator on warp 0, the rest
  // on thread 0 again
  __shared__ int s_go;
  if (tid == 0) s_go = finish_serial(D, sC, newdt, s_sum) ? 1 : 0;
  __syncthreads();
  if (s_go && tid < 32)
    advance_system_rk5(D, sC, sC->dtf, sC->PhysicalTime, sC->nb <= kRkShared ? s_work : D.rk_work, tid);
  __syncthreads();
  if (s_go && tid == 0) finish_serial_tail(D, sC);
  __syncthreads();
  {
    const int* src = reinterpret_cast<const int*>(sC);
    int* dst = reinterpret_cast<int*>(Cg);
    for (int k = tid; k < (int)(sizeof(DiskCtl) / 4); k += blockDim.x) dst[k] = src[k];
  }
}

// ... through AdvanceSystemFromDisk; false: the DT stopped (non-finite or
// non-positive CFL step), nothing more to do
__device__ bool finish_serial(const DiskDev& D, DiskCtl* C, float newdt, const double* s_sum) {
  const int nbody = C->nbody;
  const float PT = C->PhysicalTime;
  double DTd = (double)D.DT;
  // MassTaper, SourceEuler.cu:231-232
  float mt = PT / (D.MASSTAPER * 2.0 * M_PI);
  mt = (mt > 1.0 ? 1.0 : pow(sin(mt * M_PI / 2.0), 2.0));
  C->MassTaper = mt;
  // substep count and dt (SourceEuler.cu:236-241, 535)
  double dt = C->dt;
  if (D.IsDisk && (!D.SloppyCFL || C->nsub == 0)) {
    float DeltaT = DTd - C->dtemp;
    if (DeltaT < newdt) newdt = DeltaT;
    float q = DeltaT / newdt;
    if (!(newdt > 0.0f) || !(q < 1.0e5f)) {
      C->error = 1;
      C->more = 0;
      C->active = 0;
      C->counter = 0;
      return false;
    }
    int n = (int)ceilf(q);
    dt = (DTd - C->dtemp) / (double)n;
  } else if (!D.IsDisk && C->nsub == 0) {
    dt = DTd;
  }
  C->dt = dt;
  C->dtf = (float)dt;
  C->dtemp += dt;
  if (C->nsub < FARGO_MAXLOG) D.log_dt[C->nsub] = dt;
  float dtf = (float)dt;
  if (D.Corotating) get_psys_info(D, C, 1);
  // DiskOnPrimaryAcceleration (ComputeAccel for the star, SideEuler.cu:151-164):
  // the Force fields are floats, their sum is a float.
  float ax = 0.0f, ay = 0.0f;
  if (D.IsDisk) {
    ax = (float)s_sum[0] + (float)s_sum[1];
    ay = (float)s_sum[2] + (float)s_sum[3];
  }
  // ComputeIndirectTerm, Pframeforce.cu:27-35
  C->itx = -ax;
  C->ity = -ay;
  if (!D.Indirect_Term) {
    C->itx = 0.0f;
    C->ity = 0.0f;
  }
  // FillForcesArrays arguments (Pframeforce.cu:49-61)
  for (int k = 0; k < C->nb; k++) {
    double xplanet = C->x[k], yplanet = C->y[k], mplanet = C->mass[k] * mt;
    double PlanetDistance = sqrt(xplanet * xplanet + yplanet * yplanet);
    double InvPlanetDistance3 = 1.0 / PlanetDistance / PlanetDistance / PlanetDistance;
    double RRoche = PlanetDistance * pow((1.0 / 3.0 * mplanet), 1.0 / 3.0);
    double smoothing = D.RocheSmoothing ? RRoche * D.ROCHESMOOTHING
                                        : compute_smoothing(D, PlanetDistance, PT, C->PhysicalTimeInitial);
    double smooth = smoothing * smoothing;
    C->pxp[k] = (float)xplanet;
    C->pyp[k] = (float)yplanet;
    C->psmooth[k] = (float)smooth;
    C->pmass[k] = (float)mplanet;
    C->pipd3[k] = (float)InvPlanetDistance3;
  }
  // AdvanceSystemFromDisk, Pframeforce.cu:68-92
  if (D.IsDisk) {
    for (int b = 1; b < nbody; b++) {
      int k = C->body_planet[b];
      float gx = (float)s_sum[4 * b] + (float)s_sum[4 * b + 1];
      float gy = (float)s_sum[4 * b + 2] + (float)s_sum[4 * b + 3];
      C->vx[k] += dtf * gx;
      C->vy[k] += dtf * gy;
      C->vx[k] += dtf * C->itx;
      C->vy[k] += dtf * C->ity;
    }
  }
  return true;
}

// The rest of the substep's scalars, after the planet integrator.
__device__ void finish_serial_tail(const DiskDev& D, DiskCtl* C) {
  const double dt = C->dt, DTd = (double)D.DT;
  const float PT = C->PhysicalTime;
  C->domega = 0.0f;
  if (D.Corotating) {
    double OmegaNew = get_psys_info(D, C, 0) / dt;
    double domega = OmegaNew - C->OmegaFrame;
    if (D.IsDisk) C->domega = (float)domega;
    C->OmegaFrame = (float)OmegaNew;
  }
  rotate_psys(C, (float)(C->OmegaFrame * dt));
  C->time_start = PT;
  C->PhysicalTime = PT + dt;
  C->nsub++;
  C->nsub_total++;
  C->more = (C->dtemp < 0.999999999 * DTd) ? 1 : 0;
  if (C->more && C->nsub >= D.max_sub) {
    C->error = 2;
    C->more = 0;
  }
  prepare_bodies(D, C);
  C->counter = 0;
}

// ConditionCFLKernel1D + ConditionCFLKernel2D1 + the cell minimum of
// ConditionCFLKernel2D2 (Kernels.cu:1363-1422), and the disk force of
// ComputeForceKernel (Kernels.cu:804-839) for the star and every FeelDisk
// planet, accumulated in double, on CFL tiles of D.cfl_tile consecutive
// cells (four consecutive cells per thread and step, their loads issued
// together).  Each tile
// writes its minimum and its force partials (inner / outer by the ring of
// each cell), so that the finishing sums run in a fixed order.  Each block
// takes a contiguous run of tiles; the block that completes a disk's last
// tile finishes the substep's scalar work.
// NB >= every disk's body count (star + FeelDisk planets): the per-thread
// FP64 force accumulators are sized for it.
static_assert(FARGO_CFL_TILE_SMALL == 4 * kThreads && FARGO_CFL_TILE % FARGO_CFL_TILE_SMALL == 0,
              "a CFL tile is whole quads of every thread");
// The per-cell limit CFLSECURITY / s (s = sqrtf(...), a float) is a double
// division rounded to float.  For CFLSECURITY = 2^-1 it equals 0.5f times the
// correctly rounded float reciprocal of s: scaling by a power of two commutes
// with rounding (normal range), and rounding the double quotient 1/s to float
// gives the correctly rounded float quotient, since 53 >= 2*24 + 2 makes the
// double rounding innocuous for a quotient of two floats (Figueroa, "When is
// double rounding innocuous?", SIGNUM 1995).
static_assert(CFLSEC == 0.5, "the CFL limit's reciprocal form needs CFLSECURITY = 0.5");
template <int NB>
__global__ void __launch_bounds__(kThreads, NB <= 1 ? 3 : 2) k_cfl_force(BatchDev B) {
  __shared__ DiskDev sD;
  __shared__ DiskCtl sC;
  __shared__ float s_b[5][NB];
  __shared__ float s_min[2][32];                     // double-buffered by tile parity
  __shared__ double s_red[2][4 * NB][kThreads / 32];
  __shared__ double s_sum[4 * FARGO_MAXBODY];
  __shared__ double s_work[FARGO_RK_WORK(kRkShared)];
  __shared__ unsigned s_ticket;
  __shared__ int s_nbody;
  const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
  const int na = B.act[0];
  const int ntile = na > 0 ? B.act_ctile_off[na] : 0;
  const int per = (ntile + gridDim.x - 1) / gridDim.x;
  const int t0 = blockIdx.x * per, t1 = min(t0 + per, ntile);
  int lo = 0, hi = -1, run = 0;
  // A run of tiles of one disk is done: count it on the disk's ticket; the
  // block that completes the disk's last tile finishes the substep.  Warp 0
  // wrote the run's results and fences them before the ticket.
  // A radial stripe takes no ticket: k_stripe_finish finishes it.
  auto finish_run = [&]() {
    if (run == 0 || sD.stripe) {  // block-uniform
      run = 0;
      return;
    }
    DiskCtl* Cr = sD.ctl;
    if (w == 0) {
      __threadfence();
      __syncwarp();
      if (l == 0) s_ticket = atomicAdd(&Cr->counter, (unsigned)run);
    }
    __syncthreads();
    const int nct = fargo_cfl_tiles_own(sD);
    if (s_ticket + (unsigned)run == (unsigned)nct) {
      __threadfence();
      finish_cfl_and_planets<NB>(sD, Cr, &sC, s_min[0], s_sum, s_work, DiskTiles{sD, nct});
    }
    run = 0;
    __syncthreads();
  };
  for (int t = t0; t < t1; t++) {
    if (t >= hi) {  // block-uniform: entering a disk
      finish_run();
      const int a = find_range(B.act_ctile_off, na, t);
      lo = B.act_ctile_off[a];
      hi = B.act_ctile_off[a + 1];
      __syncthreads();
      copy_words(&sD, B.disks + B.act_disk[a], sizeof(DiskDev));
      __syncthreads();
      const DiskCtl* C = sD.ctl;
      const int nb = min(C->nbody, NB);
      if (tid == 0) s_nbody = nb;
      if (tid < nb) {
        s_b[0][tid] = C->bx[tid];
        s_b[1][tid] = C->by[tid];
        s_b[2][tid] = C->brs[tid];
        s_b[3][tid] = C->brh[tid];
        s_b[4][tid] = C->ba[tid];
      }
      __syncthreads();
    }
    const DiskDev& D = sD;
    const int nbody = s_nbody;
    const int nsec = D.nsec, nrad = D.nrad;
    const int k = t - lo;  // tile of this disk
    float lmin = 1e30f;
    double acc[NB][4];     // x inner, x outer, y inner, y outer
#pragma unroll
    for (int b = 0; b < NB; b++) acc[b][0] = acc[b][1] = acc[b][2] = acc[b][3] = 0.0;
    if (D.IsDisk) {
      const int kh = D.ExcludeHill ? FARGO_DIMFXY - 1 : 0;
      const float hillcutfactor = (float)kh / (float)(FARGO_DIMFXY - 1);
      const int iend = D.own_hi;
      // One cell (ring ic, sector cj): its CFL limit (rings > 0) and its
      // force on every body.  Ring constants come in rt (dxrad, dxtheta,
      // their three reciprocals, the ring-mean velocity, Rmed, Surf).
      auto cell = [&](int ic, int cj, float v0, float vr0, float dn, float vrp, float vtp, float csv, float cth,
                      float sth, const float (&rt)[8]) {
        // a NaN or Inf in the state: a NaN dt2d would be skipped by the
        // minimum below (as the reference's is) and the step would go on
        // with it; mark the tile instead, so that the DT stops with
        // FARGO_ENONFINITE (finite values leave lmin as it is)
        if (!(fabsf(v0) + fabsf(vr0) + fabsf(dn) + fabsf(csv) <= 3.4028235e38f)) lmin = -1.0f;
        if (ic > 0) {
          const float dxrad = rt[0], dxt = rt[1];
          float cs = csv;
          float vres = D.FastTransport ? v0 - rt[5] : v0;  // vmoy: k_ring_mean<0>
          // the IEEE quotients by the ring's divisors, from their correctly
          // rounded reciprocals (Markstein's method, fast_div.cuh)
          const float rdr = rt[2], rdt = rt[3];
          float invdt1 = div_by_recip(cs, min2(dxrad, dxt), rt[4]);
          float invdt2 = div_by_recip(fabsf(vr0), dxrad, rdr);
          float invdt3 = div_by_recip(fabsf(vres), dxt, rdt);
          float dvr = vrp - vr0;
          float dvt = vtp - v0;
          if (dvr >= 0.0)
            dvr = 1e-10;
          else
            dvr = -dvr;
          if (dvt >= 0.0)
            dvt = 1e-10;
          else
            dvt = -dvt;
          float invdt4 = max2(div_by_recip(dvr, dxrad, rdr), div_by_recip(dvt, dxt, rdt));
          invdt4 *= 4.0 * CVNR * CVNR;
          // CFLSECURITY / sqrtf(..) divides in double; with CFLSECURITY = 0.5
          // that is 0.5 * the float IEEE reciprocal, bit for bit (see below)
          float dt2d =
              0.5f * __frcp_rn(sqrtf(invdt1 * invdt1 + invdt2 * invdt2 + invdt3 * invdt3 + invdt4 * invdt4));
          if (dt2d < lmin) lmin = dt2d;
        }
        const float Rm = rt[6];
        float cellmass = rt[7] * dn;
        float cx = Rm * cth;
        float cy = Rm * sth;
#pragma unroll
        for (int b = 0; b < NB; b++) {
          if (b < nbody) {
            float dx = cx - s_b[0][b];
            float dy = cy - s_b[1][b];
            float rs = s_b[2][b];
            float d2 = dx * dx + dy * dy;
            float dist2 = d2 + rs * rs;
            float distance = sqrtf(dist2);
            // 1.0/dist2/distance, as one float reciprocal
            float InvDist3 = div_refined(1.0f, dist2 * distance);
            float hill_cut;
            if (kh != 0) {
              float rh = s_b[3][b] * hillcutfactor;
              hill_cut = 1. - expf(-d2 / (rh * rh));
            } else
              hill_cut = 1.;
            const double fx = cellmass * dx * InvDist3 * hill_cut;
            const double fy = cellmass * dy * InvDist3 * hill_cut;
            if (Rm < s_b[4][b]) {  // f*_inner (constant indices: the sums stay in registers)
              acc[b][0] += fx;
              acc[b][2] += fy;
            } else {  // f*_outer
              acc[b][1] += fx;
              acc[b][3] += fy;
            }
          }
        }
      };
      auto ring_consts = [&](int ic, float (&rt)[8]) {
        rt[0] = D.Rsup[ic] - D.Rinf[ic];
        rt[1] = D.dxtheta[ic];
        rt[2] = D.cfl_rdr[ic];
        rt[3] = D.cfl_rdt[ic];
        rt[4] = D.cfl_rmd[ic];
        rt[5] = D.FastTransport ? D.vmoy[ic] : 0.0f;
        rt[6] = D.Rmed[ic];
        rt[7] = D.Surf[ic];
      };
      if ((nsec & 3) == 0) {
        // four consecutive cells of one ring per thread and step (16-byte
        // loads; the ring's constants once per four cells): the tile's 1024
        // quads, thread tid takes quads tid, tid + 256, ...
        const int c0 = D.own_lo * nsec + k * D.cfl_tile + 4 * tid;
        int i = c0 / nsec, j = c0 - i * nsec;
        const int nq = D.cfl_tile / (4 * kThreads);
#pragma unroll 1
        for (int g = 0; g < nq; g++) {
          if (i >= iend) break;
          const int q = i * nsec + j;
          const float4 V0 = __ldg(reinterpret_cast<const float4*>(D.vtheta + q));
          const float4 VR0 = __ldg(reinterpret_cast<const float4*>(D.vrad + q));
          const float4 DN = __ldg(reinterpret_cast<const float4*>(D.dens + q));
          const float4 VRP = __ldg(reinterpret_cast<const float4*>(D.vrad + q + nsec));
          const float vt4 = __ldg(D.vtheta + q - j + (j + 4 == nsec ? 0 : j + 4));
          const float4 CS = D.Adiabatic ? __ldg(reinterpret_cast<const float4*>(D.cs + q))
                                        : make_float4(D.cs_ring[i], D.cs_ring[i], D.cs_ring[i], D.cs_ring[i]);
          const float4 CT = __ldg(reinterpret_cast<const float4*>(D.cos_cell + j));
          const float4 ST = __ldg(reinterpret_cast<const float4*>(D.sin_cell + j));
          float rt[8];
          ring_consts(i, rt);
          cell(i, j, V0.x, VR0.x, DN.x, VRP.x, V0.y, CS.x, CT.x, ST.x, rt);
          cell(i, j + 1, V0.y, VR0.y, DN.y, VRP.y, V0.z, CS.y, CT.y, ST.y, rt);
          cell(i, j + 2, V0.z, VR0.z, DN.z, VRP.z, V0.w, CS.z, CT.z, ST.z, rt);
          cell(i, j + 3, V0.w, VR0.w, DN.w, VRP.w, vt4, CS.w, CT.w, ST.w, rt);
          j += 4 * kThreads;
          while (j >= nsec) {
            j -= nsec;
            i++;
          }
        }
      } else {
        const int c0 = D.own_lo * nsec + k * D.cfl_tile + tid;
        int i = c0 / nsec, j = c0 - i * nsec;
        const int ncell = D.cfl_tile / kThreads;
        // kG cells at a time: their loads are issued together (cells past
        // the disk's end read cell 0 and are skipped); fewer with more bodies,
        // whose accumulators take the registers
        constexpr int kG = NB <= 2 ? 4 : (NB <= 4 ? 2 : 1);
        for (int g = 0; g < ncell; g += kG) {
          int ci[kG], cj[kG];
          bool ok[kG];
#pragma unroll
          for (int u = 0; u < kG; u++) {
            ok[u] = i < iend;
            ci[u] = ok[u] ? i : 0;
            cj[u] = ok[u] ? j : 0;
            j += kThreads;
            while (j >= nsec) {
              j -= nsec;
              i++;
            }
          }
          float v0[kG], vr0[kG], dn[kG], vrp[kG], vtp[kG], csv[kG], cth[kG], sth[kG];
#pragma unroll
          for (int u = 0; u < kG; u++) {
            const int q = ci[u] * nsec + cj[u];
            v0[u] = D.vtheta[q];
            vr0[u] = D.vrad[q];
            dn[u] = D.dens[q];
            vrp[u] = D.vrad[q + nsec];
            vtp[u] = D.vtheta[q - cj[u] + jwrap_p(cj[u], nsec)];
            csv[u] = D.Adiabatic ? D.cs[q] : D.cs_ring[ci[u]];
            cth[u] = D.cos_cell[cj[u]];
            sth[u] = D.sin_cell[cj[u]];
          }
#pragma unroll
          for (int u = 0; u < kG; u++) {
            if (!ok[u]) continue;
            float rt[8];
            ring_consts(ci[u], rt);
            cell(ci[u], cj[u], v0[u], vr0[u], dn[u], vrp[u], vtp[u], csv[u], cth[u], sth[u], rt);
          }
        }
      }
    }
    // tile minimum and force sums: warps by shuffle, then warp 0 over the
    // warps (buffers alternate by tile, so one barrier per tile suffices)
    const int pb = t & 1;
    lmin = warp_min_f(lmin);
    if (l == 0) s_min[pb][w] = lmin;
#pragma unroll
    for (int b = 0; b < NB; b++) {
      if (b < nbody) {
#pragma unroll
        for (int u = 0; u < 4; u++) {
          double v = warp_sum_d(acc[b][u]);
          if (l == 0) s_red[pb][4 * b + u][w] = v;
        }
      }
    }
    __syncthreads();
    if (w == 0) {
      if (l == 0) {
        float m = s_min[pb][0];
        for (int u = 1; u < kThreads / 32; u++)
          if (s_min[pb][u] < m) m = s_min[pb][u];
        D.ringmin[k] = m;
      }
      const int nct = fargo_cfl_tiles_own(D);
      for (int u = l; u < 4 * nbody; u += 32) {
        double v = 0.0;
        for (int x = 0; x < kThreads / 32; x++) v += s_red[pb][u][x];
        D.partials[(size_t)u * nct + k] = v;  // [sum][tile]
      }
    }
    run++;
  }
  finish_run();
}

// ----------------------------------------------------------- radial stripes

// A radial stripe's block for the gather across stripes (StripeBlocks): the
// minimum over its CFL tiles and over the shear limits of its own ring pairs
// (i, i+1) (the disk's last ring has none), its tile count, its body count
// and its force partials [sum][tile].  One block; the stripe is disk 0 of
// its batch.
__global__ void __launch_bounds__(kThreads) k_stripe_block(BatchDev B, double* out) {
  __shared__ float shf[32];
  const DiskDev& D = B.disks[0];
  const int tid = threadIdx.x;
  const int nct = fargo_cfl_tiles_own(D);
  float m = 1e30f;
  for (int t = tid; t < nct; t += blockDim.x) {
    const float v = D.ringmin[t];
    if (v < m) m = v;
  }
  m = dt1d_min(D, D.own_lo, D.own_hi < D.nrad ? D.own_hi : D.nrad - 1, tid, blockDim.x, m);
  m = block_min_f(m, shf);
  const int nbody = D.ctl->nbody;
  if (tid == 0) {
    out[0] = m;
    out[1] = nct;
    out[2] = nbody;
  }
  for (int u = tid; u < 4 * nbody * nct; u += blockDim.x) out[kStripeHead + u] = D.partials[u];
}

// The substep scalars of a radial stripe from every stripe's block (the
// same minimum and the same sums, in the same order, as the whole disk's
// finishing block forms): every stripe runs it on the same blocks, so every
// stripe takes the same dt, planet update and substep count.
constexpr int kMaxStripes = 256;
template <int NB>
__global__ void __launch_bounds__(kThreads) k_stripe_finish(BatchDev B, const double* blk, int nstripe, int stride) {
  __shared__ DiskDev sD;
  __shared__ DiskCtl sC;
  __shared__ float shf[32];
  __shared__ double s_sum[4 * FARGO_MAXBODY];
  __shared__ double s_work[FARGO_RK_WORK(kRkShared)];
  __shared__ int s_t0[kMaxStripes + 1];
  const int tid = threadIdx.x;
  copy_words(&sD, B.disks, sizeof(DiskDev));
  if (tid == 0) {
    int t = 0;
    for (int k = 0; k < nstripe; k++) {
      s_t0[k] = t;
      t += (int)blk[(size_t)k * stride + 1];
    }
    s_t0[nstripe] = t;
  }
  __syncthreads();
  finish_cfl_and_planets<NB>(sD, sD.ctl, &sC, shf, s_sum, s_work, StripeBlocks{blk, nstripe, stride, s_t0});
}

// ----------------------------------------------------------- source terms

// FillForcesArrays (Pframeforce.cu:37-66): the potential of every cell, once
// per substep (Substep1 reads it at three cells each), summed over the
// planets in the reference's order (FillForcesArraysKernel,
// Kernels.cu:1322-1349); each planet's parameters are read once per quad.
__global__ void __launch_bounds__(kThreads) k_potential(BatchDev B) {
  QUAD_BEGIN
  float cp[4], sp[4], x[4], y[4], P[4];
  qld_sector(cp, D.cos_pot, q);
  qld_sector(sp, D.sin_pot, q);
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const float Rm = D.Rmed[q.i[u]];
    x[u] = Rm * cp[u];
    y[u] = Rm * sp[u];
    P[u] = 0.0f;
  }
  const int nb = C->nb;
  const bool ind = D.Indirect_Term;
  for (int k = 0; k < nb; k++) {
    const float xp = C->pxp[k], yp = C->pyp[k], mp = C->pmass[k], sm = C->psmooth[k], ip3 = C->pipd3[k];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      float distance = (x[u] - xp) * (x[u] - xp) + (y[u] - yp) * (y[u] - yp);
      float distancesmooth = sqrtf(distance + sm);
      float pot = div_refined(-mp, distancesmooth);  // -G*mplanet/distancesmooth
      if (ind) pot += mp * ip3 * (x[u] * xp + y[u] * yp);
      P[u] += pot;
    }
    if (k == 0) {  // the star
      const float itx = C->itx, ity = C->ity;
      // accurate mode: the star's -G/r enters Substep1 as its exact radial
      // difference quotient (star_grad) instead of a difference of FP32 values
      const bool star = !D.accurate;
#pragma unroll
      for (int u = 0; u < 4; u++) {
        float InvDistance = __fdiv_rn(1.0f, D.Rmed[q.i[u]]);
        float pot = star ? -InvDistance : 0.0f;
        pot -= itx * x[u] + ity * y[u];
        P[u] += pot;
      }
    }
  }
  qst(D.phi, q, P);
  QUAD_END
}

// Substep1KernelVrad / Substep1KernelVtheta (Kernels.cu:52-88), with
// CorrectVthetaKernel (Kernels.cu:1352-1359) applied on the fly, and the
// self-gravity kick of Update_sgvelocityKernel (Kernels.cu:1024-1041).
// One instance per kind of disk (kAdi: adiabatic, kSg: self-gravity), so
// that the isothermal form without self-gravity holds no energy or
// acceleration samples and runs with more warps per SM.
template <int kAdi, int kSg>
__global__ void __launch_bounds__(kThreads, (kAdi == 0 && kSg == 0) ? 3 : 2) k_source1(BatchDev B) {
  QUAD_BEGIN_T(kAdi, kSg)
  const float dt = C->dtf;
  const float OmegaFrame = C->OmegaFrame;
  // CorrectVtheta (SideEuler.cu:184-188) on the fly; evanescent disks had it
  // applied in place by the boundary pass that precedes this kernel
  const float dom = D.Evanescent ? 0.0f : C->domega;
  constexpr bool adi = kAdi == 1, sg = kSg == 1;
  auto vth = [&](float v, int r) -> float { return dom != 0.0f ? v - dom * D.Rmed[r] : v; };
  // (i, j), (i-1, j) and (i, j-1) samples; v_theta also at (i, j+1), (i-1, j+1)
  float Dn0[4], Dnm[4], Dna[4], E0[4], Em[4], Ea[4], Ph0[4], Phm[4], Pha[4];
  float Vt0[4], Vtp[4], Vtm[4], Vtmp[4], Vr0[4];
  qld(Dn0, D.dens, q);
  qld(Dnm, D.dens, q, -nsec);
  qld_jm(Dna, Dn0, D.dens, q, nsec);
  if (adi) {
    qld(E0, D.energy, q);
    qld(Em, D.energy, q, -nsec);
    qld_jm(Ea, E0, D.energy, q, nsec);
  }
  qld(Ph0, D.phi, q);  // k_potential
  qld(Phm, D.phi, q, -nsec);
  qld_jm(Pha, Ph0, D.phi, q, nsec);
  qld(Vt0, D.vtheta, q);
  qld_jp(Vtp, Vt0, D.vtheta, q, nsec);
  qld(Vtm, D.vtheta, q, -nsec);
  qld_jp(Vtmp, Vtm, D.vtheta, q, nsec, -nsec);
  qld(Vr0, D.vrad, q);
  float ar0[4], arm[4], at0[4], atq[4];
  if (sg) {
    qld(ar0, D.sg_accr, q);
    qld(arm, D.sg_accr, q, -nsec);
    qld(at0, D.sg_acct, q);
    // the reference reads SG_Acct[i*nsec + (j-1)%nsec]: for j = 0 that is
    // the last sector of ring i-1 (ring 0: taken from ring 0 itself), i.e.
    // the cell before in memory
#pragma unroll
    for (int u = 0; u < 4; u++) {
      if (V && u > 0) {
        atq[u] = at0[u - 1];
      } else {
        const int lq = q.l[u] > 0 ? q.l[u] - 1 : nsec - 1;
        atq[u] = q.ok[u] ? __ldg(D.sg_acct + lq) : 0.0f;
      }
    }
  }
  float vri[4], vti[4], P0s[4];
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const int i = q.i[u];
    const float cs = adi ? 0.0f : D.cs_ring[i];
    // pressure: isothermal Sigma cs^2 per ring, adiabatic (gamma - 1) e
    const float P0 = adi ? (D.ADIABATICINDEX - 1.0f) * E0[u] : Dn0[u] * cs * cs;
    P0s[u] = P0;
    if (i > 0) {
      const float csm = adi ? 0.0f : D.cs_ring[i - 1];
      const float Pm = adi ? (D.ADIABATICINDEX - 1.0f) * Em[u] : Dnm[u] * csm * csm;
      float gradp = div_refined((P0 - Pm) * 2.0f, Dn0[u] + Dnm[u]) * D.invdiffRmed[i];
      float gradphi = (Ph0[u] - Phm[u]) * D.invdiffRmed[i];
      if (D.accurate && C->nb > 0) gradphi += D.star_grad[i];
      float vt2 = vth(Vt0[u], i) + vth(Vtp[u], i) + vth(Vtm[u], i - 1) + vth(Vtmp[u], i - 1);
      vt2 = vt2 * 0.25f + D.Rinf[i] * OmegaFrame;
      vt2 = vt2 * vt2;
      float v = Vr0[u] + dt * (-gradp - gradphi + vt2 * D.invRinf[i]);
      if (sg)
        v += dt * ((D.Rinf[i] - D.Rmed[i - 1]) * ar0[u] + (D.Rmed[i] - D.Rinf[i]) * arm[u]) * D.invdiffRmed[i];
      vri[u] = v;
    } else {
      vri[u] = 0.0f;  // VradInt's ring 0 is never written by the reference: zero
    }
    float dxtheta = 2.0f * (float)PI_D / (float)nsec * D.Rmed[i];
    float invdxtheta = 1.0f / dxtheta;
    const float Pa = adi ? (D.ADIABATICINDEX - 1.0f) * Ea[u] : Dna[u] * cs * cs;
    float gradp = div_refined((P0 - Pa) * 2.0f, Dn0[u] + Dna[u]) * invdxtheta;
    float gradphi = (Ph0[u] - Pha[u]) * invdxtheta;
    float v = vth(Vt0[u], i) - dt * (gradp + gradphi);
    v += dt * D.supp_torque[i];
    if (sg) v += 0.5f * dt * (at0[u] + atq[u]);
    vti[u] = v;
  }
  // ComputeTemperatureField divides the pressure of the substep start by the
  // final density (SourceEuler.cu:280,293): keep the last substep's pressure
  if (!adi && !C->more) qst(D.pres, q, P0s);
  qst(D.vri, q, vri);
  qst(D.vti, q, vti);
  QUAD_END
}

// ViscousTermsKernelDRP + ViscousTermsKernelTAURP (Kernels.cu:843-880) on
// (Vradial, Vazimutal); TAURP's third density sample is dens[i*nsec]
// because the reference indexes ((j-1)*nsec)%nsec (Kernels.cu:876).
struct Tau {
  float rr, pp, rp, divv;
};

__device__ __forceinline__ Tau viscous_terms(const DiskDev& D, const float* Vr, const float* Va, int i, int j,
                                             int nsec) {
  const int l = i * nsec + j;
  const int jp = jwrap_p(j, nsec), jm = jwrap_m(j, nsec);
  const int lp = i * nsec + jp;
  const float* Dn = D.dens;
  const float nu = D.visc[i];
  Tau t;
  float DRR = (Vr[l + nsec] - Vr[l]) * D.invdiffRsup[i];
  float DPP = (Va[lp] - Va[l]) * D.invdphi * D.invRmed[i] + 0.5f * (Vr[l + nsec] + Vr[l]) * D.invRmed[i];
  float divV = (Vr[l + nsec] * D.Rsup[i] - Vr[l] * D.Rinf[i]) * D.invdiffRsup[i] * D.invRmed[i];
  divV += (Va[lp] - Va[l]) * D.invdphi * D.invRmed[i];
  t.divv = divV;
  t.rr = 2.0f * Dn[l] * nu * (DRR - D.onethird * divV);
  t.pp = 2.0f * Dn[l] * nu * (DPP - D.onethird * divV);
  t.rp = 0.0f;
  if (i > 0) {
    const int lm = i * nsec + jm;
    float DRP = 0.5f * (D.Rinf[i] * (Va[l] * D.invRmed[i] - Va[l - nsec] * D.invRmed[i - 1]) * D.invdiffRmed[i] +
                        (Vr[l] - Vr[lm]) * D.invdphi * D.invRinf[i]);
    t.rp = 0.5f * (Dn[l] + Dn[l - nsec] + Dn[i * nsec] + Dn[lm - nsec]) * nu * DRP;
  }
  return t;
}

// Sub-Keplerian boundary speeds (SideEuler.cu:250-268), device double math
// when they change with time or self-gravity.
__device__ void vkep_pair(const DiskDev& D, const DiskCtl* C, float* vin, float* vout) {
  if (D.vkep_const) {
    *vin = D.VKepIn;
    *vout = D.VKepOut;
    return;
  }
  const int nrad = D.nrad;
  float PT = C->time_start, PTI = C->PhysicalTimeInitial;
  float r0 = D.Rmed[0], r1 = D.Rmed[nrad - 1];
  double f = (1.0 + D.SIGMASLOPE - 2.0 * D.FLARINGINDEX);
  double a0 = 1.0 / r0 * (1.0 - f * pow((double)aspect_ratio_host(D, r0, PT, PTI), 2.0) * pow(r0, 2.0 * D.FLARINGINDEX));
  double a1 = 1.0 / r1 * (1.0 - f * pow((double)aspect_ratio_host(D, r1, PT, PTI), 2.0) * pow(r1, 2.0 * D.FLARINGINDEX));
  if (D.SelfGravity) {
    a0 -= r0 * C->axisg_in;
    a1 -= r1 * C->axisg_out;
  }
  *vin = sqrt(a0);
  *vout = sqrt(a1);
}

// ComputeViscousTerms + UpdateVelocitiesWithViscosity + the sub-Keplerian
// boundary (Viscosity.cu:77-102, Kernels.cu:142-160, 843-880, 1490-1503)
// fused on radial x azimuthal tiles of kVR x kVC cells.  The block stages
// VradInt, VthetaInt and Sigma for the tile and a 2-cell halo in shared
// memory (azimuth periodic), computes the stress tensor once for the tile
// and a 1-cell halo into shared memory (the same arithmetic as
// viscous_terms), then the updated velocities of its own cells.  They go to
// the trr / tpp buffers (the stresses never reach HBM), which Substep2 then
// reads as VradInt / VthetaInt: writing them in place would race with the
// neighbouring tiles' halo reads.
constexpr int kVR = 16, kVC = 64;                       // tile rows, columns
constexpr int kSO = 4;                                  // staged columns left of the tile
constexpr int kSR = kVR + 4, kSC = kVC + 2 * kSO;       // staged rows, columns (whole 16-byte chunks)
constexpr int kTR = kVR + 2, kTC = kVC + 2;             // stress rows, columns
constexpr int kTQ = (kTC + 3) / 4;                      // stress quads per row
constexpr int kRuns = 14;                               // stress runs per row: 12 of 5 columns, 2 of 3
static_assert(12 * 5 + 2 * 3 == kTC && kTR * kRuns <= kThreads, "stress runs cover a tile's rows in one pass");
constexpr int kTCp = 4 * kTQ;                           // stress row length in shared memory
static_assert(kVR * kVC == 4 * kThreads, "one quad of the tile per thread in the update");
__device__ __forceinline__ int vtiles_of(const DiskDev& D) {
  return ((D.nrad + kVR - 1) / kVR) * ((D.nsec + kVC - 1) / kVC);
}

// 4-byte asynchronous global -> shared copy (zero-filled when !valid)
__device__ __forceinline__ void cp_async4(float* smem, const float* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = valid ? 4 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz) : "memory");
}
// 16-byte asynchronous global -> shared copy, both addresses 16-byte
// aligned (zero-filled when !valid)
__device__ __forceinline__ void cp_async16(float* smem, const float* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int n>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(n) : "memory");
}

constexpr size_t kViscSmem = sizeof(float) * 3 * 2 * kSR * kSC;  // dynamic: the staged tiles
__global__ void __launch_bounds__(kThreads, 3) k_viscosity(BatchDev B) {
  __shared__ DiskDev sD;
  extern __shared__ __align__(16) float vs_sm[];
  float(*sVrb)[kSR][kSC] = reinterpret_cast<float(*)[kSR][kSC]>(vs_sm);  // [2][kSR][kSC] each
  float(*sVab)[kSR][kSC] = sVrb + 2;
  float(*sDnb)[kSR][kSC] = sVab + 2;
  __shared__ float sD0b[2][kSR];
  __shared__ float sTrr[kTR][kTCp], sTpp[kTR][kTCp], sTrp[kTR][kTCp];
  const int tid = threadIdx.x;
  const int na = B.act[0];
  const int ntile = na > 0 ? B.act_vtile_off[na] : 0;
  const int per = (ntile + gridDim.x - 1) / gridDim.x;
  const int t0 = blockIdx.x * per, t1 = min(t0 + per, ntile);
  // issue the asynchronous staging of tile lt of the disk in sD into buffer bf:
  // rows i0-2 .. i0+kVR+1 (row NRAD is the ghost row), columns j0-kSO ..
  // j0+kVC+kSO-1 (azimuth periodic).  With NSEC a multiple of 4 every
  // 4-column chunk is one aligned 16-byte copy (j0 is a multiple of 64 and a
  // wrap moves a chunk by NSEC); otherwise column by column.
  auto stage = [&](int lt, int bf) {
    const int nsec = sD.nsec, nrad = sD.nrad;
    const int ncol = (nsec + kVC - 1) / kVC;
    const int i0 = (lt / ncol) * kVR, j0 = (lt % ncol) * kVC;
    if ((nsec & 3) == 0) {
      constexpr int kCh = kSC / 4;  // chunks per staged row
      for (int q = tid; q < kSR * kCh; q += kThreads) {
        const int r = q / kCh, c = 4 * (q - r * kCh);
        const int i = i0 - 2 + r;
        int j = j0 - kSO + c;  // j0 - kSO >= -kSO: at most one wrap below
        if (j < 0) j += nsec;
        while (j >= nsec) j -= nsec;
        const bool ok = i >= 0 && i <= nrad;
        const int l = ok ? i * nsec + j : 0;
        cp_async16(&sVrb[bf][r][c], sD.vri + l, ok);
        cp_async16(&sVab[bf][r][c], sD.vti + l, ok);
        cp_async16(&sDnb[bf][r][c], sD.dens + l, ok);
      }
    } else {
      for (int q = tid; q < kSR * kSC; q += kThreads) {
        const int r = q / kSC, c = q - r * kSC;
        const int i = i0 - 2 + r;
        int j = (j0 - kSO + c) % nsec;
        if (j < 0) j += nsec;
        const bool ok = i >= 0 && i <= nrad;
        const int l = ok ? i * nsec + j : 0;
        cp_async4(&sVrb[bf][r][c], sD.vri + l, ok);
        cp_async4(&sVab[bf][r][c], sD.vti + l, ok);
        cp_async4(&sDnb[bf][r][c], sD.dens + l, ok);
      }
    }
    if (tid < kSR) {
      const int i = i0 - 2 + tid;
      const bool ok = i >= 0 && i <= nrad;
      cp_async4(&sD0b[bf][tid], sD.dens + (ok ? i * nsec : 0), ok);
    }
    cp_async_commit();
  };
  int lo = 0, hi = -1, bf = 0;
  bool have = false;  // tile t already staged (prefetched) in buffer bf
  for (int t = t0; t < t1; t++) {
    if (t >= hi) {  // block-uniform: entering a disk
      const int a = find_range(B.act_vtile_off, na, t);
      lo = B.act_vtile_off[a];
      hi = B.act_vtile_off[a + 1];
      __syncthreads();
      copy_words(&sD, B.disks + B.act_disk[a], sizeof(DiskDev));
      __syncthreads();
      have = false;
    }
    if (!have) stage(t - lo, bf);
    // prefetch the next tile of the same disk while this one is computed
    const bool pre = (t + 1 < t1) && (t + 1 < hi);
    if (pre) {
      stage(t + 1 - lo, bf ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    float(*sVr)[kSC] = sVrb[bf];
    float(*sVa)[kSC] = sVab[bf];
    float(*sDn)[kSC] = sDnb[bf];
    const float* sD0 = sD0b[bf];
    const DiskDev& D = sD;
    const DiskCtl* C = D.ctl;
    const int nsec = D.nsec, nrad = D.nrad;
    const int ncol = (nsec + kVC - 1) / kVC;
    const int lt = t - lo;
    const int i0 = (lt / ncol) * kVR, j0 = (lt % ncol) * kVC;
    const float invdphi = D.invdphi, onethird = D.onethird;
    if (D.IsDisk) {
      // stresses at rows i0-1 .. i0+kVR, columns j0-1 .. j0+kVC (viscous_terms),
      // one run of consecutive columns of one row per thread (each row in 12
      // runs of 5 and 2 of 3: all 18 rows in one pass of the block): the
      // row's tables are read once and neighbouring samples are shared in
      // registers
      if (tid < kTR * kRuns) {
        const int r = tid / kRuns, m = tid - r * kRuns;
        const int c0 = m < 12 ? 5 * m : 60 + 3 * (m - 12);
        const int len = m < 12 ? 5 : 3;
        const int i = i0 - 1 + r;
        if (i >= 0 && i < nrad) {
          const int rr = r + 1, cc = c0 + kSO - 1;  // staged indices of (i, j) for the first column
          const float nu = D.visc[i];
          const float iRm = D.invRmed[i];
          const float idRs = D.invdiffRsup[i], Rs = D.Rsup[i], Ri = D.Rinf[i];
          float vr[6], vr1[5], va[6], vam[5], dn[5], dnm[6];
#pragma unroll
          for (int u = 0; u < 6; u++) {
            vr[u] = sVr[rr][cc - 1 + u];   // columns c0-1 .. c0+4
            va[u] = sVa[rr][cc + u];       // columns c0 .. c0+5
            dnm[u] = sDn[rr - 1][cc - 1 + u];
          }
#pragma unroll
          for (int u = 0; u < 5; u++) {
            vr1[u] = sVr[rr + 1][cc + u];
            vam[u] = sVa[rr - 1][cc + u];
            dn[u] = sDn[rr][cc + u];
          }
          const float d0 = sD0[rr];
          const float iRm1 = i > 0 ? D.invRmed[i - 1] : 0.0f;
          const float idRm = D.invdiffRmed[i], iRi = D.invRinf[i];
#pragma unroll
          for (int u = 0; u < 5; u++) {
            if (u >= len) break;
            const int c = c0 + u;
            const float v0 = vr[u + 1], vp = vr1[u], a0 = va[u], ap = va[u + 1];
            float DRR = (vp - v0) * idRs;
            float DPP = (ap - a0) * invdphi * iRm + 0.5f * (vp + v0) * iRm;
            float divV = (vp * Rs - v0 * Ri) * idRs * iRm;
            divV += (ap - a0) * invdphi * iRm;
            sTrr[r][c] = 2.0f * dn[u] * nu * (DRR - onethird * divV);
            sTpp[r][c] = 2.0f * dn[u] * nu * (DPP - onethird * divV);
            float rp = 0.0f;  // TAURP's ring 0 is never written: zero
            if (i > 0) {
              float DRP = 0.5f * (Ri * (a0 * iRm - vam[u] * iRm1) * idRm + (v0 - vr[u]) * invdphi * iRi);
              // TAURP's third density sample is dens[i*nsec] (Kernels.cu:876)
              rp = 0.5f * (dn[u] + dnm[u + 1] + d0 + dnm[u]) * nu * DRP;
            }
            sTrp[r][c] = rp;
          }
        }
      }
    }
    __syncthreads();
    // updated velocities of the tile's cells: one quad per thread
    const float DeltaT = C->dtf;
    float vin = 0.0f, vout = 0.0f;
    const bool kep = !D.Evanescent && (i0 == 0 || i0 + kVR >= nrad);
    if (kep) vkep_pair(D, C, &vin, &vout);
    {
      const int r = tid / (kVC / 4), c0 = 4 * (tid - r * (kVC / 4));
      const int i = i0 + r, j = j0 + c0;
      if (i < nrad && j < nsec) {
        const int R = r + 1, Cc = c0 + 1;   // stress index of (i, j)
        const int rr = r + 2, cc = c0 + kSO;  // staged index of (i, j)
        float vti[4], vri[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          vti[u] = sVa[rr][cc + u];
          vri[u] = sVr[rr][cc + u];
        }
        if (D.IsDisk) {
          const float iRm = D.invRmed[i], Rs = D.Rsup[i], Ri = D.Rinf[i], idRs = D.invdiffRsup[i];
          const float iRi = D.invRinf[i], Rm = D.Rmed[i];
          const float Rm1 = i > 0 ? D.Rmed[i - 1] : 0.0f, idRm = D.invdiffRmed[i];
          float trp0[5], trp1[4], tpp0[5], tpp1[4], trr0[4], trr1[4], dn[5], dnm[4];
#pragma unroll
          for (int u = 0; u < 5; u++) {
            trp0[u] = sTrp[R][Cc + u];       // columns c0 .. c0+4
            tpp0[u] = sTpp[R][Cc - 1 + u];   // columns c0-1 .. c0+3
            dn[u] = sDn[rr][cc - 1 + u];     // columns c0-1 .. c0+3
          }
#pragma unroll
          for (int u = 0; u < 4; u++) {
            trp1[u] = sTrp[R + 1][Cc + u];
            tpp1[u] = sTpp[R - 1][Cc + u];
            trr0[u] = sTrr[R][Cc + u];
            trr1[u] = sTrr[R - 1][Cc + u];
            dnm[u] = sDn[rr - 1][cc + u];
          }
#pragma unroll
          for (int u = 0; u < 4; u++) {
            if (i > 0 && i < nrad - 1) {
              vti[u] += div_refined(DeltaT * iRm *
                                        ((Rs * trp1[u] - Ri * trp0[u]) * idRs + (tpp0[u + 1] - tpp0[u]) * invdphi +
                                         0.5f * (trp0[u] + trp1[u])),
                                    0.5f * (dn[u + 1] + dn[u]));
            }
            if (i > 0) {
              vri[u] += div_refined(DeltaT * iRi *
                                        ((Rm * trr0[u] - Rm1 * trr1[u]) * idRm + (trp0[u + 1] - trp0[u]) * invdphi -
                                         0.5f * (tpp0[u + 1] + tpp1[u])),
                                    0.5f * (dn[u + 1] + dnm[u]));
            }
            if (kep && i == 0) vti[u] = vin - D.Rmed[0] * C->OmegaFrame;
            if (kep && i == nrad - 1) vti[u] = vout - D.Rmed[nrad - 1] * C->OmegaFrame;
          }
        }
        const int l = i * nsec + j;
        if ((nsec & 3) == 0) {  // the quad lies inside the ring, 16-byte aligned
          stg4(D.trr + l, vri[0], vri[1], vri[2], vri[3]);
          stg4(D.tpp + l, vti[0], vti[1], vti[2], vti[3]);
        } else {
#pragma unroll
          for (int u = 0; u < 4; u++) {
            if (j + u < nsec) {
              stg(D.trr + l + u, vri[u]);
              stg(D.tpp + l + u, vti[u]);
            }
          }
        }
      }
    }
    __syncthreads();  // buffer bf is restaged two tiles on
    bf ^= 1;
    have = pre;
  }
}

// Substep2Kernel + Substep2Kernel2 (Kernels.cu:570-621), then the
// ActualiseGasVrad/Vtheta copies become direct stores into the state.
__device__ __forceinline__ float qvisc(float dv, float dens) {
  if (dv < 0.0f) return (float)(CVNR * CVNR) * dens * dv * dv;
  return 0.0f;
}

// One instance per kind of disk (kAdi: adiabatic): the isothermal form holds
// no energy samples.
template <int kAdi>
__global__ void __launch_bounds__(kThreads, kAdi ? 3 : 4) k_source2(BatchDev B) {
  QUAD_BEGIN_T(kAdi, -1)
  const float dt = C->dtf;
  constexpr bool adi = kAdi == 1;
  // viscosity-updated VradInt / VthetaInt (k_viscosity) and the density
  float R0[4], Ru[4], Rd[4], T0[4], Tp[4], Tm[4], N0[4], Nd[4], Nm[4], E0[4];
  qld(R0, D.trr, q);
  qld(Ru, D.trr, q, nsec);
  qld(Rd, D.trr, q, -nsec);
  qld(T0, D.tpp, q);
  qld_jp(Tp, T0, D.tpp, q, nsec);
  qld_jm(Tm, T0, D.tpp, q, nsec);
  qld(N0, D.dens, q);
  qld(Nd, D.dens, q, -nsec);
  qld_jm(Nm, N0, D.dens, q, nsec);
  if (adi) qld(E0, D.energy, q);
  float vrn[4], vtn[4], ein[4];
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const int i = q.i[u];
    float qr = qvisc(Ru[u] - R0[u], N0[u]);
    float qt = qvisc(Tp[u] - T0[u], N0[u]);
    float vr_new = 0.0f;
    if (i > 0) {
      float qrm = qvisc(R0[u] - Rd[u], Nd[u]);
      vr_new = R0[u] - div_refined(dt * 2.0f, N0[u] + Nd[u]) * (qr - qrm) * D.invdiffRmed[i];
    }
    float qtm = qvisc(T0[u] - Tm[u], Nm[u]);
    float dxtheta = 2.0f * (float)PI_D / (float)nsec * D.Rmed[i];
    float invdxtheta = 1.0f / dxtheta;
    vtn[u] = T0[u] - div_refined(dt * 2.0f, N0[u] + Nm[u]) * (qt - qtm) * invdxtheta;
    vrn[u] = vr_new;
    // EnergyInt goes to scratch: the boundary pass before Substep3 still sees the state energy
    if (adi) ein[u] = E0[u] - dt * qr * (Ru[u] - R0[u]) * D.invdiffRsup[i] - dt * qt * (Tp[u] - T0[u]) * invdxtheta;
  }
  if (adi) qst(D.a1, q, ein);
  qst(D.vrad, q, vrn);
  qst(D.vtheta, q, vtn);
  // VthetaNew's ghost row is zero
  if (V) {
    if (q.i[0] == nrad - 1) stg4(D.vtheta + q.l[0] + nsec, 0.0f, 0.0f, 0.0f, 0.0f);
  } else {
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (q.ok[u] && q.i[u] == nrad - 1) stg(D.vtheta + q.l[u] + nsec, 0.0f);
  }
  QUAD_END
}

// Substep3Kernel + Substep3Kernel2 (Kernels.cu:91-139) with the viscous
// terms of the new velocities (SourceEuler.cu:286-289) evaluated per cell.
__device__ __forceinline__ float qplus_at(const DiskDev& D, int i, int j, int nsec, float* divv) {
  Tau t = viscous_terms(D, D.vrad, D.vtheta, i, j, nsec);
  *divv = t.divv;
  const int l = i * nsec + j;
  const float nu = D.visc[i];
  float q;
  if (nu != 0.0f) {
    q = div_refined(div_refined(0.5f, nu), D.dens[l]) * (t.rr * t.rr + +t.rp * t.rp + t.pp * t.pp);
    q += (float)(2.0 / 9.0) * nu * D.dens[l] * t.divv * t.divv;
  } else
    q = 0.0f;
  return q;
}

// qplus_at for the four cells of a quad in one ring i >= 1 (vector path):
// the same expressions, the neighbours loaded as 16-byte rows and shifted
// lanes instead of ten scalar loads per cell.
template <bool V>
__device__ __forceinline__ void qplus_quad(const DiskDev& D, const Quad<V>& q, int nsec, float (&qp)[4],
                                           float (&dv)[4]) {
  const int i = q.i[0];
  float Vr0[4], Vrp[4], Vrj[4], Va0[4], Vap[4], Vam[4], Dn0[4], Dnm[4], Dnmj[4];
  qld(Vr0, D.vrad, q);
  qld(Vrp, D.vrad, q, nsec);
  qld_jm(Vrj, Vr0, D.vrad, q, nsec);
  qld(Va0, D.vtheta, q);
  qld_jp(Vap, Va0, D.vtheta, q, nsec);
  qld(Vam, D.vtheta, q, -nsec);
  qld(Dn0, D.dens, q);
  qld(Dnm, D.dens, q, -nsec);
  qld_jm(Dnmj, Dnm, D.dens, q, nsec, -nsec);
  const float Di = __ldg(D.dens + i * nsec);  // TAURP's third density sample (Kernels.cu:876)
  const float nu = D.visc[i], iRm = D.invRmed[i], iRm1 = D.invRmed[i - 1], idRs = D.invdiffRsup[i];
  const float Rs = D.Rsup[i], Ri = D.Rinf[i], idRm = D.invdiffRmed[i], iRi = D.invRinf[i];
  const float invdphi = D.invdphi, onethird = D.onethird;
#pragma unroll
  for (int u = 0; u < 4; u++) {
    float DRR = (Vrp[u] - Vr0[u]) * idRs;
    float DPP = (Vap[u] - Va0[u]) * invdphi * iRm + 0.5f * (Vrp[u] + Vr0[u]) * iRm;
    float divV = (Vrp[u] * Rs - Vr0[u] * Ri) * idRs * iRm;
    divV += (Vap[u] - Va0[u]) * invdphi * iRm;
    const float rr = 2.0f * Dn0[u] * nu * (DRR - onethird * divV);
    const float pp = 2.0f * Dn0[u] * nu * (DPP - onethird * divV);
    float DRP = 0.5f * (Ri * (Va0[u] * iRm - Vam[u] * iRm1) * idRm + (Vr0[u] - Vrj[u]) * invdphi * iRi);
    const float rp = 0.5f * (Dn0[u] + Dnm[u] + Di + Dnmj[u]) * nu * DRP;
    dv[u] = divV;
    if (nu != 0.0f) {
      qp[u] = div_refined(div_refined(0.5f, nu), Dn0[u]) * (rr * rr + +rp * rp + pp * pp);
      qp[u] += (float)(2.0 / 9.0) * nu * Dn0[u] * divV * divV;
    } else {
      qp[u] = 0.0f;
    }
  }
}

__global__ void __launch_bounds__(kThreads, 3) k_energy(BatchDev B) {
  QUAD_BEGIN_T(1, -1)
  const float dt = C->dtf;
  float qv[4], ev[4], dvq[4];
  const bool quad = V && q.i[0] > 0;
  if (quad) qplus_quad(D, q, nsec, qv, dvq);
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const int i = q.i[u], j = q.j[u], l = q.l[u];
    if (!q.ok[u]) {
      qv[u] = ev[u] = 0.0f;
      continue;
    }
    float divv;
    float qp = 0.0f;
    if (quad) {
      qp = qv[u];
      divv = dvq[u];
    } else if (i > 0) {
      qp = qplus_at(D, i, j, nsec, &divv);
    } else {
      float dv1, dv2;
      float q1 = qplus_at(D, 1, j, nsec, &dv1);
      float q2 = qplus_at(D, 2, j, nsec, &dv2);
      Tau t0 = viscous_terms(D, D.vrad, D.vtheta, 0, j, nsec);
      divv = t0.divv;
      if (D.visc[nrad - 1] != 0.0)
        qp = q1 * expf(logf(q1 / q2) * logf(D.Rmed[0] / D.Rmed[1]) / logf(D.Rmed[1] / D.Rmed[2]));
      else
        qp = 0.0;
    }
    const float e_int = D.a1[l];  // EnergyInt from k_source2
    const float Dl = D.dens[l];
    float num, den;
    if (!D.Cooling) {
      num = dt * qp + e_int;
      den = 1.0f + (D.ADIABATICINDEX - 1.0f) * dt * divv;
    } else {
      num = D.EnergyMed[i] * dt * Dl / D.SigmaMed[i] + D.CoolingTimeMed[i] * e_int +
            dt * D.CoolingTimeMed[i] * (qp - D.QplusMed[i] * Dl / D.SigmaMed[i]);
      den = dt + D.CoolingTimeMed[i] + (D.ADIABATICINDEX - 1.0f) * dt * D.CoolingTimeMed[i] * divv;
    }
    qv[u] = qp;
    ev[u] = div_refined(num, den);
  }
  qst(D.qplus, q, qv);
  qst(D.energy, q, ev);
  // EnergyNew's ghost row is zero
  if (V) {
    if (q.i[0] == nrad - 1) stg4(D.energy + q.l[0] + nsec, 0.0f, 0.0f, 0.0f, 0.0f);
  } else {
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (q.ok[u] && q.i[u] == nrad - 1) stg(D.energy + q.l[u] + nsec, 0.0f);
  }
  QUAD_END
}

// ------------------------------------------------------------- transport

// Transport arithmetic is FP32 throughout, and free of multiply-add
// contraction: every product that meets an addition is an explicit
// round-to-nearest multiply (fm), so each cell's result does not depend on
// how the work is cut into bands, segments and unrolled steps (the compiler
// may contract the same expression differently in different code paths).
// The reference's own arithmetic, and the oracle's, is uncontracted too.
//
// Transport arithmetic is FP32 throughout.  The reference writes several
// of these expressions with double literals (0.5, 2.0, 1e-20), which
// promotes them to double; here each is the same expression in float, the
// quotient Q / (Sigma + 1e-20) is Q times the float reciprocal, and the
// results differ by at most a few ulps per operation, the size of the
// fused-multiply-add differences between two builds of the reference
// itself.  (FP64 conversions and divisions run on the SM's transcendental
// pipe at 1/8 of the FP32 rate and made this kernel issue-bound.)  Slope
// quotients use the fast reciprocal division (2 ulp): their operands are
// differences of O(1e-12 .. 1) quantities, far from the range where it
// differs from IEEE division by more than that.

// van Leer slope of StarRadKernel (Kernels.cu:917-927)
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }

// Paired FP32 arithmetic (Blackwell's two-lane FADD2 / FMUL2, round to
// nearest): a pair of quantities goes through one instruction, each lane
// rounding as the scalar operation (no difference on 8.4 M operand pairs,
// subnormals included).  Whole builds still differ in the last bits: the
// paired azimuthal sweeps and the earlier scalar ones give fields ~5e-6
// apart (rel-L2 of Sigma after 5 DTs), within the parity tolerances.
__device__ __forceinline__ float2 bc2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 m2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 a2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 s2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 sel2(bool c, float2 a, float2 b) { return c ? a : b; }

__device__ __forceinline__ float vl_rad_slope(float qm, float q0, float qp, float invdm, float invdp) {
  float dqm = fm(q0 - qm, invdm);
  float dqp = fm(qp - q0, invdp);
  if (fm(dqp, dqm) > 0.0f) return __fdividef(fm(fm(2.0f, dqp), dqm), dqp + dqm);
  return 0.0f;
}
// the same for two quantities at once
__device__ __forceinline__ float2 vl_rad_slope2(float2 qm, float2 q0, float2 qp, float invdm, float invdp) {
  const float2 dqm = m2(s2(q0, qm), bc2(invdm));
  const float2 dqp = m2(s2(qp, q0), bc2(invdp));
  const float2 t = m2(dqp, dqm);
  const float2 num = m2(m2(bc2(2.0f), dqp), dqm);
  const float2 den = a2(dqp, dqm);
  return make_float2(t.x > 0.0f ? __fdividef(num.x, den.x) : 0.0f, t.y > 0.0f ? __fdividef(num.y, den.y) : 0.0f);
}

// One row sample of the radial half of Transport at column g: the
// LRMomentaKernel quantities (Kernels.cu:883-896) RadMomP, RadMomM,
// ThetaMomP, ThetaMomM, [energy], density, and their DivisePolarGridKernel
// quotients by the density (Kernels.cu:1127-1134).  Quantity c is lane
// c % 2 of pair c / 2; with an odd count the last pair's second lane is a
// zero that no result reads.
template <int nq>
struct RadRow {
  static constexpr int np = (nq + 1) / 2;
  float S;         // density
  float2 Q[np];    // quantities, quantity nq-1 = S
  float2 W[np];    // quotients Q / (S + 1e-20)
};
template <int nq>
__device__ __forceinline__ float lane_of(const float2 (&v)[(nq + 1) / 2], int c) {
  return (c & 1) ? v[c >> 1].y : v[c >> 1].x;
}

// The disk fields and ring tables the radial half reads, loaded once per
// band into registers (the band's shared-memory stores then cannot force
// reloads of the disk's pointers); 32-bit cell offsets, as the reference's.
struct TrView {
  const float *dens, *vrad, *vtheta, *energy;
  const float *Rmed, *invdiffRmed, *Rinf, *Rsup, *invSurf;
  int nsec, nrad;
};

// van Leer slopes at row r from rows r-1, r, r+1 (StarRadKernel; zero on the
// first and last ring): g[] for the quotients, gs for the density.
template <int nq>
__device__ __forceinline__ void rad_slopes(const TrView& V, int r, const RadRow<nq>& A, const RadRow<nq>& Bm,
                                           const RadRow<nq>& Cp, float2* g, float& gs) {
  constexpr int np = RadRow<nq>::np;
  if (r <= 0 || r >= V.nrad - 1) {
#pragma unroll
    for (int c = 0; c < np; c++) g[c] = bc2(0.0f);
    gs = 0.0f;
    return;
  }
  const float im = __ldg(V.invdiffRmed + r), ip = __ldg(V.invdiffRmed + r + 1);
#pragma unroll
  for (int c = 0; c < np; c++) g[c] = vl_rad_slope2(A.W[c], Bm.W[c], Cp.W[c], im, ip);
  gs = vl_rad_slope(A.S, Bm.S, Cp.S, im, ip);
}

// Upwind interface values at the boundary b between rows b-1 (lo) and b
// (hi) for radial velocity vr (StarRadKernel2, Kernels.cu:929-947); zero on
// the inner edge and beyond the outer ring.
template <int nq>
__device__ __forceinline__ void rad_face(const TrView& V, int b, float vr, float dt, const RadRow<nq>& lo,
                                         const RadRow<nq>& hi, const float2* glo, float gslo, const float2* ghi,
                                         float gshi, float2* qs, float& ds) {
  constexpr int np = RadRow<nq>::np;
  const int nrad = V.nrad;
  if (b <= 0 || b >= nrad) {
#pragma unroll
    for (int c = 0; c < np; c++) qs[c] = bc2(0.0f);
    ds = 0.0f;
    return;
  }
  // upwind side by selection (columns differ in sign): vr > 0 takes row b-1
  // at + h, else row b at -h; a - fm(h, g) = a + fm(-h, g)
  const bool pos = vr > 0.0f;
  const float rm = __ldg(V.Rmed + b), rl = __ldg(V.Rmed + b - 1);
  const float rp = (b + 1 <= nrad - 1) ? __ldg(V.Rmed + b + 1) : 0.0f;  // only meets a zero slope
  const float h = pos ? fm(rm - rl - fm(vr, dt), 0.5f) : fm(rp - rm + fm(vr, dt), 0.5f);
  const float hs = pos ? h : -h;
#pragma unroll
  for (int c = 0; c < np; c++) qs[c] = a2(sel2(pos, lo.W[c], hi.W[c]), m2(bc2(hs), sel2(pos, glo[c], ghi[c])));
  ds = (pos ? lo.S : hi.S) + fm(hs, pos ? gslo : gshi);
}

// The band's input rows staged in shared memory (k_transport): logical row
// k holds ring i0-2+k on the window's columns (L + 1 of them: v_theta is
// also read one column to the right); dens and v_theta rings i0-2 ..
// i0+kBR+1, v_r rings i0-2 .. i0+kBR+2 (its ghost row NRAD included).
// Rings outside the disk are zero-filled: they only feed zero slopes and
// zero interface fluxes, whose values do not depend on them.
constexpr int kRow = FARGO_TR_ROW;           // staged row length (>= window + 1; one TMA box)
constexpr int kInD = 0, kInR = 12, kInT = 25;  // first staged row of dens, v_r, v_theta
constexpr int kInRows = 37;
static_assert(kInR - kInD == FARGO_TR_ROWS_D && kInT - kInR == FARGO_TR_ROWS_R &&
                  kInRows - kInT == FARGO_TR_ROWS_T, "staged rows of one band");
static_assert(FARGO_SEG_MAX + 9 <= kRow && (FARGO_SEG_MAX & 3) == 0, "a window fits one staged row");
static_assert((kInR * kRow * 4) % 128 == 0 && (kInT * kRow * 4) % 128 == 0, "TMA destinations 128-byte aligned");
// bytes one band's three TMA boxes deliver (zero-filled parts included)
constexpr unsigned kTmaBytes = 4u * kRow * kInRows;

template <int nq>
__device__ __forceinline__ RadRow<nq> rad_row_s(const TrView& V, const float* sIn, int r, int k, int p, int g,
                                                float Om) {
  constexpr int np = RadRow<nq>::np;
  const int rc = r < 0 ? 0 : (r > V.nrad - 1 ? V.nrad - 1 : r);
  RadRow<nq> R;
  const float sg = sIn[(kInD + k) * kRow + p];
  const float rm = __ldg(V.Rmed + rc);
  R.S = sg;
  // RadMomP, RadMomM = Sigma v_r(i+1), Sigma v_r(i)
  R.Q[0] = m2(bc2(sg), make_float2(sIn[(kInR + k + 1) * kRow + p], sIn[(kInR + k) * kRow + p]));
  // ThetaMomP, ThetaMomM = Sigma (v_theta(j+1) + r Omega) r, Sigma (v_theta(j) + r Omega) r
  const float2 vt = make_float2(sIn[(kInT + k) * kRow + p + 1], sIn[(kInT + k) * kRow + p]);
  R.Q[1] = m2(m2(bc2(sg), a2(vt, bc2(fm(rm, Om)))), bc2(rm));
  if (nq == 6)
    R.Q[2] = make_float2(__ldg(V.energy + rc * V.nsec + g), sg);
  else
    R.Q[2] = make_float2(sg, 0.0f);
  const float rden = __fdividef(1.0f, sg + 1e-20f);
#pragma unroll
  for (int c = 0; c < np; c++) R.W[c] = m2(R.Q[c], bc2(rden));
  return R;
}

// Radial half of Transport (VanLeerRadialKernel, Kernels.cu:1137-1154) for
// rings ia .. ib-1 at column g, marching outwards: each ring loads one new
// row, one new slope and one new interface.  out[k][c] at stride ostride.
// lost0 (may be null): receives the density's varq at ring 0, the mass that
// leaves through the inner edge (LostByDisk, Kernels.cu:941-944).
// The rows come from the band's staged rows (ia = i0): window column p,
// global column g.
template <int nq>
__device__ __forceinline__ void rad_march_s(const TrView& V, const float* sIn, int ia, int ib, int p, int g,
                                            float dt, float Om, float dtheta, float* out, int ostride_c,
                                            int ostride_r, float* lost0) {
  constexpr int np = RadRow<nq>::np;
  RadRow<nq> R0 = rad_row_s<nq>(V, sIn, ia - 1, 1, p, g, Om);  // row i-1 for the first slope
  RadRow<nq> R1 = rad_row_s<nq>(V, sIn, ia, 2, p, g, Om);      // row i
  RadRow<nq> R2 = rad_row_s<nq>(V, sIn, ia + 1, 3, p, g, Om);  // row i+1
  float2 G0[np], G1[np], qs[np];
  float gs0, gs1, ds;
  {
    RadRow<nq> Rm = rad_row_s<nq>(V, sIn, ia - 2, 0, p, g, Om);
    rad_slopes<nq>(V, ia - 1, Rm, R0, R1, G0, gs0);  // slope at row i-1
  }
  rad_slopes<nq>(V, ia, R0, R1, R2, G1, gs1);  // slope at row i
  float vr0 = sIn[(kInR + 2) * kRow + p];
  rad_face<nq>(V, ia, vr0, dt, R0, R1, G0, gs0, G1, gs1, qs, ds);
  const float dtdth = fm(dt, dtheta);
#pragma unroll
  for (int k = 0; k < FARGO_BAND; k++) {
    const int i = ia + k;
    if (i >= ib) break;
    RadRow<nq> R3 = rad_row_s<nq>(V, sIn, i + 2, k + 4, p, g, Om);
    float2 G2[np], qs1[np];
    float gs2, ds1;
    rad_slopes<nq>(V, i + 1, R1, R2, R3, G2, gs2);  // slope at row i+1
    const float vr1 = sIn[(kInR + k + 3) * kRow + p];  // row nrad is the zero ghost row
    rad_face<nq>(V, i + 1, vr1, dt, R1, R2, G1, gs1, G2, gs2, qs1, ds1);
    const float Ri = __ldg(V.Rinf + i), Rs = __ldg(V.Rsup + i), iS = __ldg(V.invSurf + i);
    const float fi = fm(dtdth, Ri), fs = fm(dtdth, Rs);
    float* o = out + k * ostride_r;
    float2 varq[np];
#pragma unroll
    for (int c = 0; c < np; c++) {
      varq[c] = m2(m2(m2(bc2(fi), qs[c]), bc2(ds)), bc2(vr0));
      varq[c] = s2(varq[c], m2(m2(m2(bc2(fs), qs1[c]), bc2(ds1)), bc2(vr1)));
      const float2 r = a2(R1.Q[c], m2(varq[c], bc2(iS)));
      o[(2 * c) * ostride_c] = r.x;
      if (2 * c + 1 < nq) o[(2 * c + 1) * ostride_c] = r.y;
    }
    if (i == 0 && lost0) *lost0 = lane_of<nq>(varq, nq - 1);
    R1 = R2;
    R2 = R3;
#pragma unroll
    for (int c = 0; c < np; c++) {
      G1[c] = G2[c];
      qs[c] = qs1[c];
    }
    gs1 = gs2;
    ds = ds1;
    vr0 = vr1;
  }
}

// ---------------------------------------------------------- ring means

// Serial FP32 ring means of v_theta, j = 0 .. NSEC-1 in order as one thread
// of ConditionCFLKernel1D (Kernels.cu:352-356) and of
// ComputeAverageThetaVelocitiesKernel (Kernels.cu:1184-1198) sum them: the
// FARGO shift floor(Ntilde + 0.5) and the CFL dt depend on the last bit.
// One CTA takes kRMR rings of one disk.  All its threads stream the rings
// through shared memory in chunks of kRMW sectors (coalesced, kRMR loads in
// flight per thread) while warp 0, lane r owning ring i0 + r, adds the
// previous chunk's row in order.  The chain of one ring (NSEC dependent
// additions) bounds the kernel, so a few rings per CTA spread the chains over
// every SM in one wave.
//   mode 0: vmoy[i] (CFL, substep start)
//   mode 1: transport VMed, Nshift and constant residual (OneWindTheta,
//           TransportEuler.cu:171-219 with ComputeConstantResidualKernel,
//           Kernels.cu:1201-1232), and the Nshift log of the DT.
constexpr int kRMT = 256;             // threads
constexpr int kRMW = 256;             // sectors per chunk
constexpr int kRMR = FARGO_RM_RINGS;  // rings per CTA (one serial chain each)
// shared row stride: 16-byte aligned rows, and the kRMR lanes' 16-byte reads
// at the same offset fall on disjoint banks (260 = 4 mod 32)
constexpr int kRMS = kRMW + 4;
static_assert(kRMR <= 32 && kRMR * 4 <= 32, "one lane of warp 0 per ring, conflict-free 16-byte reads");
static_assert(kRMW % 32 == 0 && kRMS % 4 == 0, "chunks of whole 32-sector blocks, 16-byte rows");
size_t fargo_ring_mean_smem_bytes() { return sizeof(float) * 2 * kRMR * kRMS; }
template <int mode>
__global__ void __launch_bounds__(kRMT) k_ring_mean(BatchDev B) {
  extern __shared__ __align__(16) float rm_sm[];  // [2][kRMR][kRMS]
  const int na = B.act[0];
  const int ng = na > 0 ? B.act_grp_off[na] : 0;
  const int tid = threadIdx.x, lane = tid & 31;
  for (int g = blockIdx.x; g < ng; g += gridDim.x) {
    const int a = find_range(B.act_grp_off, na, g);
    const DiskDev& D = B.disks[B.act_disk[a]];
    const int i0 = (g - B.act_grp_off[a]) * kRMR;
    const int nsec = D.nsec, nrad = D.nrad;
    const int nr = min(kRMR, nrad - i0);
    const float* base = D.vtheta + (size_t)i0 * nsec;
    const int nchunk = (nsec + kRMW - 1) / kRMW;
    float r[kRMR];
    auto load = [&](int c) {
      const int col = c * kRMW + tid;
#pragma unroll
      for (int k = 0; k < kRMR; k++)
        r[k] = (c < nchunk && k < nr && col < nsec) ? __ldg(base + (size_t)k * nsec + col) : 0.0f;
    };
    auto store = [&](int c) {
      float* buf = rm_sm + (c & 1) * kRMR * kRMS;
#pragma unroll
      for (int k = 0; k < kRMR; k++) buf[k * kRMS + tid] = r[k];
    };
    float moy = 0.0f;
    KahanSum ks;  // accurate mode
    const bool acc = D.accurate;
    __syncthreads();
    load(0);
    store(0);
    __syncthreads();
    for (int c = 0; c < nchunk; c++) {
      load(c + 1);
      if (tid < kRMR) {
        const float* row = rm_sm + (c & 1) * kRMR * kRMS + lane * kRMS;
        const int w = min(kRMW, nsec - c * kRMW);
        if (acc) {
          for (int k = 0; k < w; k++) ks.add(row[k]);
        } else if (w == kRMW) {
          // the chain in sector order, its operands read 32 ahead as 16-byte
          // words, so that the shared-memory latency stays off the chain
          const float4* r4 = reinterpret_cast<const float4*>(row);
          float4 a[8], b[8];
#pragma unroll
          for (int k = 0; k < 8; k++) a[k] = r4[k];
#pragma unroll
          for (int blk = 0; blk < kRMW / 32; blk++) {
            if (blk + 1 < kRMW / 32) {
#pragma unroll
              for (int k = 0; k < 8; k++) b[k] = r4[(blk + 1) * 8 + k];
            }
#pragma unroll
            for (int k = 0; k < 8; k++) {
              moy += a[k].x;
              moy += a[k].y;
              moy += a[k].z;
              moy += a[k].w;
            }
#pragma unroll
            for (int k = 0; k < 8; k++) a[k] = b[k];
          }
        } else {
          for (int k = 0; k < w; k++) moy += row[k];
        }
      }
      if (c + 1 < nchunk) store(c + 1);
      __syncthreads();
    }
    const int i = i0 + lane;
    if (acc) moy = ks.s;
    if (tid < 32 && lane < nr) {
      if (mode == 0) {
        D.vmoy[i] = moy / (float)nsec;
      } else {
        const DiskCtl* C = D.ctl;
        const float dt = C->dtf;
        float VMed = moy / (float)nsec;
        float invdt = 1.0 / dt;
        float dpinvns = 2.0 * PI_D / (float)nsec;
        float Ntilde = VMed * D.invRmed[i] * dt * (float)nsec / 2.0 / PI_D;
        float Nround = floor(Ntilde + 0.5);
        long nitemp = (long)Nround;
        D.tvmed[i] = VMed;
        D.tvconst[i] = (Ntilde - Nround) * D.Rmed[i] * invdt * dpinvns;
        D.nshift[i] = (int)nitemp;
        int sidx = C->nsub - 1;
        if (sidx >= 0 && sidx < FARGO_MAXLOG) D.log_nshift[(size_t)sidx * nrad + i] = (int)nitemp;
      }
    }
  }
}

constexpr int kTT = 256;         // threads of the transport kernel
constexpr int kBR = FARGO_BAND;  // rings per transport band: one warp each in the sweeps
constexpr int kPad = kTT + kTT / 8;  // shared row with a padding word after every 8
static_assert(FARGO_SEG_OUT + 8 <= kTT, "transport window must fit the CTA");
static_assert(kBR * 32 == kTT, "one warp per ring of the band");

// padded shared-memory index: 8 consecutive points per lane read without
// bank conflicts, 32 consecutive points per warp too
__device__ __forceinline__ int pidx(int t) { return t + (t >> 3); }

size_t fargo_transport_smem_bytes(int adiabatic) {
  const int nq = adiabatic ? 6 : 5;
  // + 128: the staged rows start on a 128-byte boundary
  return sizeof(float) * ((size_t)kPad * (size_t)(kBR * (nq + 1) + 1) + (size_t)kInRows * kRow) + 128;
}
static_assert((kPad * 4) % 16 == 0 && (kRow * 4) % 16 == 0, "staged rows 16-byte aligned");

#ifndef FARGO_NOFMA
// One van Leer pass of OneWindTheta on the window (see sweep_ring).  kind 0:
// every point's own velocity v[k] (the residual sweep); kind 1 / 2: one
// velocity vu for the whole ring (the constant-residual sweep), whose
// interfaces all take their upwind value from the left (1: vu dt > 0) or
// from the right (2), at the same distance h: no per-point selects.
// The quantities stay in the ring's shared-memory rows (each lane reads and
// writes only its own 8 points there); they are processed two at a time as
// the lanes of paired FP32 operations (each lane rounds as the scalar
// operation); with an odd count the last quantity, the density, shares a
// pair with its own star value.
template <int nq, int kind>
__device__ __forceinline__ void sweep_pass(float* sRr, int b0, const float (&v)[8], float vu, float dt,
                                           float dxtheta, float invdxtheta, float invsurf, float dxrad) {
  auto slope = [&](float wm, float w0, float wp) -> float {
    float dqm = (w0 - wm);
    float dqp = (wp - w0);
    if (fm(dqp, dqm) > 0.0f) return fm(__fdividef(fm(dqp, dqm), dqp + dqm), invdxtheta);
    return 0.0f;
  };
  auto slope2 = [&](float2 wm, float2 w0, float2 wp) -> float2 {
    const float2 dqm = s2(w0, wm);
    const float2 dqp = s2(wp, w0);
    const float2 t = m2(dqp, dqm);
    const float2 den = a2(dqp, dqm);
    const float2 g = m2(make_float2(__fdividef(t.x, den.x), __fdividef(t.y, den.y)), bc2(invdxtheta));
    return make_float2(t.x > 0.0f ? g.x : 0.0f, t.y > 0.0f ? g.y : 0.0f);
  };
  auto shup2 = [](float2 x) -> float2 {
    return make_float2(__shfl_up_sync(0xffffffffu, x.x, 1), __shfl_up_sync(0xffffffffu, x.y, 1));
  };
  auto shdn2 = [](float2 x) -> float2 {
    return make_float2(__shfl_down_sync(0xffffffffu, x.x, 1), __shfl_down_sync(0xffffffffu, x.y, 1));
  };
  // upwind side of each point's left interface and the distance to it:
  // ksi > 0 takes point k-1 at dxtheta - ksi, else point k at -(dxtheta + ksi)
  float vv[8], rr[8], S[8], GS[8], sD[8], h[8];
  unsigned up = 0;
  const float ksu = fm(vu, dt);
  const float hu = (kind == 1) ? dxtheta - ksu : dxtheta + ksu;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    vv[k] = (kind == 0) ? v[k] : vu;
    S[k] = sRr[(nq - 1) * kPad + b0 + k];
    rr[k] = __fdividef(1.0f, S[k] + 1e-20f);
    if (kind == 0) {
      const float ksi = fm(vv[k], dt);
      if (ksi > 0.0f) up |= 1u << k;
      h[k] = (ksi > 0.0f) ? dxtheta - ksi : dxtheta + ksi;
    } else {
      h[k] = hu;
    }
  }
  auto is_left = [&](int k) -> bool { return kind == 0 ? ((up >> k) & 1u) != 0 : kind == 1; };
  if constexpr ((nq & 1) == 0) {
    const float Sl = __shfl_up_sync(0xffffffffu, S[7], 1);
    const float Sr = __shfl_down_sync(0xffffffffu, S[0], 1);
#pragma unroll
    for (int k = 0; k < 8; k++) GS[k] = slope(k ? S[k - 1] : Sl, S[k], k < 7 ? S[k + 1] : Sr);
    const float GSl = (kind == 2) ? 0.0f : __shfl_up_sync(0xffffffffu, GS[7], 1);
    // DensStar (StarThetaKernel2 on the density); a - fm(h, g) = a + fm(h, -g)
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const bool u = is_left(k);
      const float su = u ? (k ? S[k - 1] : Sl) : S[k];
      const float gu = u ? (k ? GS[k - 1] : GSl) : -GS[k];
      sD[k] = su + fm(h[k], gu);
    }
  } else {
    // odd count (the isothermal density last): DensStar and the density's own
    // interface value are the same slope and upwind expressions, on Sigma and
    // on Sigma / (Sigma + 1e-20): the two lanes of one pair.  The density row
    // is updated at once (the pairs below read only their own rows).
    float2 X[8], GX[8], FX[8];
#pragma unroll
    for (int k = 0; k < 8; k++) X[k] = make_float2(S[k], fm(S[k], rr[k]));
    const float2 Xl = shup2(X[7]);
    const float2 Xr = shdn2(X[0]);
#pragma unroll
    for (int k = 0; k < 8; k++) GX[k] = slope2(k ? X[k - 1] : Xl, X[k], k < 7 ? X[k + 1] : Xr);
    const float2 GXl = (kind == 2) ? bc2(0.0f) : shup2(GX[7]);
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const bool u = is_left(k);
      const float2 xu = u ? (k ? X[k - 1] : Xl) : X[k];
      const float2 gu = u ? (k ? GX[k - 1] : GXl) : make_float2(-GX[k].x, -GX[k].y);
      const float2 st = a2(xu, m2(bc2(h[k]), gu));  // (DensStar, the density's QRStar)
      sD[k] = st.x;
      FX[k].x = fm(fm(fm(dxrad, st.y), st.x), vv[k]);  // the density's flux, left interface
    }
    const float Fr = __shfl_down_sync(0xffffffffu, FX[0].x, 1);
    float* rd = sRr + (nq - 1) * kPad + b0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      float varq = FX[k].x;
      varq -= (k < 7 ? FX[k + 1].x : Fr);
      rd[k] = S[k] + fm(varq, invsurf);
    }
  }
  // the paired quantities (with an even count the last pair holds the
  // density); all quotients use the pre-sweep density
  constexpr int npair = nq / 2;
#pragma unroll
  for (int c2 = 0; c2 < npair; c2++) {
    float* r0 = sRr + (2 * c2) * kPad + b0;
    float* r1 = r0 + kPad;
    float2 W[8], G[8], F[8];
#pragma unroll
    for (int k = 0; k < 8; k++) W[k] = m2(make_float2(r0[k], r1[k]), bc2(rr[k]));
    const float2 Wl = shup2(W[7]);
    const float2 Wr = shdn2(W[0]);
#pragma unroll
    for (int k = 0; k < 8; k++) G[k] = slope2(k ? W[k - 1] : Wl, W[k], k < 7 ? W[k + 1] : Wr);
    const float2 Gl = (kind == 2) ? bc2(0.0f) : shup2(G[7]);
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const bool u = is_left(k);
      const float2 wu = u ? (k ? W[k - 1] : Wl) : W[k];
      const float2 gu = u ? (k ? G[k - 1] : Gl) : make_float2(-G[k].x, -G[k].y);
      const float2 qr = a2(wu, m2(bc2(h[k]), gu));
      F[k] = m2(m2(m2(bc2(dxrad), qr), bc2(sD[k])), bc2(vv[k]));  // flux through the left interface
    }
    const float2 Fr = shdn2(F[0]);
    asm volatile("" ::: "memory");  // reread the rows rather than keep them in registers
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const float2 varq = s2(F[k], k < 7 ? F[k + 1] : Fr);
      const float2 q = a2(make_float2(r0[k], r1[k]), m2(varq, bc2(invsurf)));  // unchanged rows: reread
      r0[k] = q.x;
      r1[k] = q.y;
    }
  }
}

// The residual and constant-residual van Leer sweeps of OneWindTheta
// (StarThetaKernel, StarThetaKernel2, VanLeerThetaKernel, Kernels.cu:1157-1273)
// on one ring's window of 256 points, by one warp: lane l holds points
// 8l .. 8l+7 and takes its neighbours' edge values by shuffle.
// sRr: the ring's radial results [nq][kPad] and v_theta [kPad] (point x at
// pidx(x)); the swept values go back to the same places.  The window's
// points 0..3 and L-4.. (and any beyond L) are halo: each sweep's result at
// a point depends on the points within two of it, so after the two sweeps
// the values at 4 .. L-5 do not depend on anything outside the window and
// the edges need no special case (their values are never stored).
// The second sweep's velocity is the ring's constant residual: one upwind
// side for the whole ring (a warp-uniform branch), and none of it when that
// residual is exactly zero (every flux is then zero: the quantities are
// unchanged, as the reference's q + 0 leaves them).
template <int nq>
__device__ __forceinline__ void sweep_ring(float* sRr, float VMed, float vconst, bool fast, float dt,
                                           float dxtheta, float invdxtheta, float invsurf, float dxrad) {
  const int lane = threadIdx.x & 31;
  const int b0 = 9 * lane;  // pidx(8 * lane): points 8l .. 8l+7 are contiguous
  float v[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    float vres = sRr[nq * kPad + b0 + k] - VMed;
    if (!fast) vres = vconst + vres;
    v[k] = vres;
  }
  if (!fast) vconst = 0.0f;
  sweep_pass<nq, 0>(sRr, b0, v, 0.0f, dt, dxtheta, invdxtheta, invsurf, dxrad);
  if (fm(vconst, dt) > 0.0f)
    sweep_pass<nq, 1>(sRr, b0, v, vconst, dt, dxtheta, invdxtheta, invsurf, dxrad);
  else if (vconst != 0.0f)
    sweep_pass<nq, 2>(sRr, b0, v, vconst, dt, dxtheta, invdxtheta, invsurf, dxrad);
  __syncwarp();  // the ring's swept values, lane by lane, before the shifted store
}

#else
// The accurate mode's kernel set keeps the scalar sweeps with the
// quantities in registers, the form its FP64 error was measured with.
// One van Leer pass of OneWindTheta on the window (see sweep_ring).  kind 0:
// every point's own velocity v[k] (the residual sweep); kind 1 / 2: one
// velocity vu for the whole ring (the constant-residual sweep), whose
// interfaces all take their upwind value from the left (1: vu dt > 0) or
// from the right (2), at the same distance h: no per-point selects.
template <int nq, int kind>
__device__ __forceinline__ void sweep_pass(float (&q)[nq][8], const float (&v)[8], float vu, float dt,
                                           float dxtheta, float invdxtheta, float invsurf, float dxrad) {
  auto slope = [&](float wm, float w0, float wp) -> float {
    float dqm = (w0 - wm);
    float dqp = (wp - w0);
    if (fm(dqp, dqm) > 0.0f) return fm(__fdividef(fm(dqp, dqm), dqp + dqm), invdxtheta);
    return 0.0f;
  };
  // upwind side of each point's left interface and the distance to it:
  // ksi > 0 takes point k-1 at dxtheta - ksi, else point k at -(dxtheta + ksi)
  float vv[8], rr[8], S[8], GS[8], sD[8], h[8];
  unsigned up = 0;
  const float ksu = fm(vu, dt);
  const float hu = (kind == 1) ? dxtheta - ksu : dxtheta + ksu;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    vv[k] = (kind == 0) ? v[k] : vu;
    S[k] = q[nq - 1][k];
    rr[k] = __fdividef(1.0f, S[k] + 1e-20f);
    if (kind == 0) {
      const float ksi = fm(vv[k], dt);
      if (ksi > 0.0f) up |= 1u << k;
      h[k] = (ksi > 0.0f) ? dxtheta - ksi : dxtheta + ksi;
    } else {
      h[k] = hu;
    }
  }
  auto is_left = [&](int k) -> bool { return kind == 0 ? ((up >> k) & 1u) != 0 : kind == 1; };
  const float Sl = __shfl_up_sync(0xffffffffu, S[7], 1);
  const float Sr = __shfl_down_sync(0xffffffffu, S[0], 1);
#pragma unroll
  for (int k = 0; k < 8; k++) GS[k] = slope(k ? S[k - 1] : Sl, S[k], k < 7 ? S[k + 1] : Sr);
  const float GSl = (kind == 2) ? 0.0f : __shfl_up_sync(0xffffffffu, GS[7], 1);
  // DensStar (StarThetaKernel2 on the density); a - fm(h, g) = a + fm(h, -g)
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const bool u = is_left(k);
    const float su = u ? (k ? S[k - 1] : Sl) : S[k];
    const float gu = u ? (k ? GS[k - 1] : GSl) : -GS[k];
    sD[k] = su + fm(h[k], gu);
  }
  // every quantity, density last; all quotients use the pre-sweep density
#pragma unroll
  for (int c = 0; c < nq; c++) {
    float W[8], G[8], F[8];
#pragma unroll
    for (int k = 0; k < 8; k++) W[k] = fm(q[c][k], rr[k]);
    const float Wl = __shfl_up_sync(0xffffffffu, W[7], 1);
    const float Wr = __shfl_down_sync(0xffffffffu, W[0], 1);
#pragma unroll
    for (int k = 0; k < 8; k++) G[k] = slope(k ? W[k - 1] : Wl, W[k], k < 7 ? W[k + 1] : Wr);
    const float Gl = (kind == 2) ? 0.0f : __shfl_up_sync(0xffffffffu, G[7], 1);
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const bool u = is_left(k);
      const float wu = u ? (k ? W[k - 1] : Wl) : W[k];
      const float gu = u ? (k ? G[k - 1] : Gl) : -G[k];
      const float qr = wu + fm(h[k], gu);
      F[k] = fm(fm(fm(dxrad, qr), sD[k]), vv[k]);  // flux through the left interface of point k
    }
    const float Fr = __shfl_down_sync(0xffffffffu, F[0], 1);
#pragma unroll
    for (int k = 0; k < 8; k++) {
      float varq = F[k];
      varq -= (k < 7 ? F[k + 1] : Fr);
      q[c][k] += fm(varq, invsurf);
    }
  }
}

// The residual and constant-residual van Leer sweeps of OneWindTheta
// (StarThetaKernel, StarThetaKernel2, VanLeerThetaKernel, Kernels.cu:1157-1273)
// on one ring's window of 256 points, by one warp: lane l holds points
// 8l .. 8l+7 in registers and takes its neighbours' edge values by shuffle.
// sRr: the ring's radial results [nq][kPad] and v_theta [kPad] (point x at
// pidx(x)); the swept values go back to the same places.  The window's
// points 0..3 and L-4.. (and any beyond L) are halo: each sweep's result at
// a point depends on the points within two of it, so after the two sweeps
// the values at 4 .. L-5 do not depend on anything outside the window and
// the edges need no special case (their values are never stored).
// The second sweep's velocity is the ring's constant residual: one upwind
// side for the whole ring (a warp-uniform branch), and none of it when that
// residual is exactly zero (every flux is then zero: the quantities are
// unchanged, as the reference's q + 0 leaves them).
template <int nq>
__device__ __forceinline__ void sweep_ring(float* sRr, float VMed, float vconst, bool fast, float dt,
                                           float dxtheta, float invdxtheta, float invsurf, float dxrad) {
  const int lane = threadIdx.x & 31;
  const int b0 = 9 * lane;  // pidx(8 * lane): points 8l .. 8l+7 are contiguous
  float q[nq][8], v[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
#pragma unroll
    for (int c = 0; c < nq; c++) q[c][k] = sRr[c * kPad + b0 + k];
    float vres = sRr[nq * kPad + b0 + k] - VMed;
    if (!fast) vres = vconst + vres;
    v[k] = vres;
  }
  if (!fast) vconst = 0.0f;
  sweep_pass<nq, 0>(q, v, 0.0f, dt, dxtheta, invdxtheta, invsurf, dxrad);
  if (fm(vconst, dt) > 0.0f)
    sweep_pass<nq, 1>(q, v, vconst, dt, dxtheta, invdxtheta, invsurf, dxrad);
  else if (vconst != 0.0f)
    sweep_pass<nq, 2>(q, v, vconst, dt, dxtheta, invdxtheta, invsurf, dxrad);
  __syncwarp();
#pragma unroll
  for (int k = 0; k < 8; k++)
#pragma unroll
    for (int c = 0; c < nq; c++) sRr[c * kPad + b0 + k] = q[c][k];
  __syncwarp();
}

#endif

// ---- TMA staging: mbarrier and bulk tensor copy (one CTA, no cluster) ----
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for the phase of the given parity, polling at most kSpin times (each
// poll itself blocks for a bounded, hardware-defined time): false when the
// wait gave up, so that a copy that never lands cannot hang the GPU.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
  constexpr int kSpin = 1 << 20;
  for (int k = 0; k < kSpin; k++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// 2-D tiled TMA load of one box at coordinates (x, y) of the tensor map
// (global memory of this GPU) into shared memory, completing on `bar`.
// x is a column index (multiple of 4: 16 bytes); x and y may be negative or
// beyond the tensor: those elements are zero-filled.
__device__ __forceinline__ void tma_load_2d(float* dst, const void* tmap, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          smem_u32(dst)),
      "l"(tmap), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Issue the asynchronous staging of transport item t's input rows (see
// kRow).  With the disk's tensor maps (NSEC a multiple of 4, >= 64) one
// thread issues three TMA box loads (Sigma, v_r, v_theta rows; rings outside
// the disk come zero-filled) that complete on `bar`, and the call returns
// true; columns of the window that wrap around the ring are then filled in
// by tr_fixup once the copies have landed.  Otherwise every thread issues
// cp.async copies (16-byte when NSEC and the segment start are multiples of
// 4, so that every 4-column chunk lies inside the ring, else 4-byte), which
// follow the azimuthal wrap themselves, and the call returns false.  The
// choice depends only on the item and the disk: it is block-uniform.
template <int nq>
__device__ __forceinline__ bool tr_stage(const BatchDev& B, const int4* __restrict__ items, int t, float* sIn,
                                         uint64_t* bar) {
  const int nak = (nq == 5) ? B.act[1] : B.act[2];
  const int* aoff = (nq == 5) ? B.act_iso_off : B.act_adi_off;
  const int* adisk = (nq == 5) ? B.act_iso_disk : B.act_adi_disk;
  const int a = find_range(aoff, nak, t);
  const DiskDev& D = B.disks[adisk[a]];
  const int4 it = items[D.item0 + (t - aoff[a])];
  const int i0 = it.y, g0 = it.z, W = it.w + 9;  // window + 1 columns
  const int nsec = D.nsec, nrad = D.nrad;
  if (D.tmap && (nsec & 3) == 0 && nsec >= 64 && (g0 & 3) == 0 && (smem_u32(sIn) & 127) == 0) {
    if (threadIdx.x == 0) {
      const char* tm = static_cast<const char*>(D.tmap);
      // the previous item's reads of sIn (generic proxy) are complete (the
      // block passed a barrier): order them before the copies' writes
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      mbar_expect_tx(bar, kTmaBytes);
      tma_load_2d(sIn + kInD * kRow, tm, g0 - 4, i0 - 2, bar);
      tma_load_2d(sIn + kInR * kRow, tm + 128, g0 - 4, i0 - 2, bar);
      tma_load_2d(sIn + kInT * kRow, tm + 256, g0 - 4, i0 - 2, bar);
    }
    return true;
  }
  const float *dens = D.dens, *vrad = D.vrad, *vth = D.vtheta;
  auto src = [&](int row, int& r, int& lim) -> const float* {
    if (row < kInR) {
      r = i0 - 2 + row - kInD;
      lim = nrad - 1;
      return dens;
    }
    if (row < kInT) {
      r = i0 - 2 + row - kInR;
      lim = nrad;  // the ghost row
      return vrad;
    }
    r = i0 - 2 + row - kInT;
    lim = nrad - 1;
    return vth;
  };
  if ((nsec & 3) == 0 && (g0 & 3) == 0) {
    constexpr int nch = kRow / 4;  // whole staged rows: a constant divisor
    for (int q = threadIdx.x; q < kInRows * nch; q += kTT) {
      const int row = q / nch, ch = q - row * nch;
      int r, lim;
      const float* base = src(row, r, lim);
      const bool ok = r >= 0 && r <= lim;
      int g = g0 - 4 + 4 * ch;
      if (g < 0) g += nsec;
      while (g >= nsec) g -= nsec;
      cp_async16(sIn + row * kRow + 4 * ch, base + (ok ? r * nsec + g : 0), ok);
    }
  } else {
    for (int q = threadIdx.x; q < kInRows * W; q += kTT) {
      const int row = q / W, c = q - row * W;
      int r, lim;
      const float* base = src(row, r, lim);
      const bool ok = r >= 0 && r <= lim;
      int g = (g0 - 4 + c) % nsec;
      if (g < 0) g += nsec;
      cp_async4(sIn + row * kRow + c, base + (ok ? r * nsec + g : 0), ok);
    }
  }
  cp_async_commit();
  return false;
}

// After a TMA staging has landed: the window's columns left of sector 0 or
// right of sector NSEC-1 were zero-filled by the copy (the tensor map does
// not wrap); fill them from the other end of the ring, as the reference's
// periodic azimuth reads them.  At most 4 columns on the left and 5 on the
// right (the segment lies inside the ring).
__device__ __forceinline__ void tr_fixup(const DiskDev& D, int4 it, float* sIn) {
  const int i0 = it.y, g0 = it.z, W = it.w + 9;
  const int nsec = D.nsec, nrad = D.nrad;
  const int nl = g0 < 4 ? 4 - g0 : 0;
  const int nr = max(0, g0 - 4 + W - nsec);
  const int nw = nl + nr;
  for (int q = threadIdx.x; q < kInRows * nw; q += kTT) {
    const int row = q / nw, k = q - row * nw;
    const int c = k < nl ? k : W - nr + (k - nl);
    int g = g0 - 4 + c;
    g = g < 0 ? g + nsec : (g >= nsec ? g - nsec : g);
    const float* base;
    int r, lim;
    if (row < kInR) {
      r = i0 - 2 + row - kInD;
      lim = nrad - 1;
      base = D.dens;
    } else if (row < kInT) {
      r = i0 - 2 + row - kInR;
      lim = nrad;  // the ghost row
      base = D.vrad;
    } else {
      r = i0 - 2 + row - kInT;
      lim = nrad - 1;
      base = D.vtheta;
    }
    sIn[row * kRow + c] = (r >= 0 && r <= lim) ? __ldg(base + r * nsec + g) : 0.0f;
  }
}

// Transport (TransportEuler.cu:24-35) of a band of up to kBR rings i0 ..
// and one azimuthal segment of source sectors g0 .. g0+S-1.  The tile is
// taken in source coordinates: the radial half (rad_march_s) runs over the
// window g0-4 .. g0+S+3 of every ring of the band, one thread per column
// marching outwards, on input rows staged in shared memory, into shared
// memory; then one warp per ring runs the azimuthal sweeps (sweep_ring) on
// that window, whose 4-point halo covers the sweeps' stencils.  The next
// item's rows are staged while the sweeps run.  Source sector g of ring i
// is then stored at output sector g + Nshift_i (AdvectSHIFTKernel,
// Kernels.cu:1276-1289: output j takes source j - Nshift): per ring a
// contiguous run, and the segments of a ring map one to one onto its output
// sectors.  VMed, Nshift and the constant residual come from
// k_ring_mean<1>.  Final density / energy go to scratch (a0 / a1) because
// neighbouring bands still read the old ones; the velocity kernel moves
// them into the state.
template <int nq>
__global__ void __launch_bounds__(kTT, 2) k_transport(BatchDev B, const int4* __restrict__ items) {
  extern __shared__ __align__(16) float tr_sm[];
  float* sR = tr_sm;                         // [kBR][nq + 1][kPad] radial results + v_theta
  float* sL = sR + kBR * (nq + 1) * kPad;    // [kPad] mass through the inner edge (OPEN)
  // [kInRows][kRow] staged input rows, 128-byte aligned (TMA destination)
  float* sIn = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(sL + kPad) + 127) & ~uintptr_t(127));
  __shared__ int s_jb[kBR];
  __shared__ float s_vmed[kBR], s_vc[kBR];
  __shared__ __align__(8) uint64_t s_bar;  // completion of the TMA staging
  __shared__ int s_gaveup;
  const int nak = (nq == 5) ? B.act[1] : B.act[2];
  const int* aoff = (nq == 5) ? B.act_iso_off : B.act_adi_off;
  const int* adisk = (nq == 5) ? B.act_iso_disk : B.act_adi_disk;
  const int nai = nak > 0 ? aoff[nak] : 0;
  const int p = threadIdx.x, warp = p >> 5, lane = p & 31;
  if (p == 0) {
    mbar_init(&s_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_gaveup = 0;
  }
  __syncthreads();
  unsigned phase = 0;  // parity of the staging barrier's next phase
  bool pend = false;   // a TMA staging is in flight
  if ((int)blockIdx.x < nai) pend = tr_stage<nq>(B, items, blockIdx.x, sIn, &s_bar);
  for (int t = blockIdx.x; t < nai; t += gridDim.x) {
    const int tn = t + gridDim.x;  // this block's next item
    const int a = find_range(aoff, nak, t);
    const DiskDev& D = B.disks[adisk[a]];
    const int4 it = items[D.item0 + (t - aoff[a])];
    if (pend) {
      if (mbar_wait_bounded(&s_bar, phase)) {
        tr_fixup(D, it, sIn);
      } else {
        s_gaveup = 1;
      }
    }
    cp_async_wait<0>();
    __syncthreads();  // staged rows visible; the previous item's sweeps are done
    if (s_gaveup) {
      // the staged rows never arrived: report it on the disk (the host maps
      // it to FARGO_ETIMEOUT), wait once more for the copies, and stop
      if (p == 0) const_cast<DiskCtl*>(D.ctl)->error = 3;
      mbar_wait_bounded(&s_bar, phase);
      return;
    }
    if (pend) phase ^= 1;
    pend = false;
    if (!D.IsDisk) {
      if (tn < nai) pend = tr_stage<nq>(B, items, tn, sIn, &s_bar);
      continue;
    }
    const DiskCtl* C = D.ctl;
    const int i0 = it.y, g0 = it.z, S = it.w;
    const int nsec = D.nsec, nrad = D.nrad;
    const int nb = min(kBR, nrad - i0);
    const int L = S + 8;
    const float dt = C->dtf;
    const float Om = C->OmegaFrame;
    const bool fast = D.FastTransport;
    const float dtheta = 2.0f * (float)PI_D / (float)nsec;
    if (p < nb) {
      int jb = (g0 + D.nshift[i0 + p]) % nsec;  // output sector of source sector g0
      s_jb[p] = jb < 0 ? jb + nsec : jb;
      s_vmed[p] = D.tvmed[i0 + p];
      s_vc[p] = D.tvconst[i0 + p];
    }
    if (p < L) {
      const TrView V = {D.dens, D.vrad, D.vtheta, D.energy, D.Rmed, D.invdiffRmed, D.Rinf, D.Rsup, D.invSurf,
                        nsec, nrad};
      int g = (g0 - 4 + p) % nsec;
      if (g < 0) g += nsec;
      float* o = sR + pidx(p);
      rad_march_s<nq>(V, sIn, i0, i0 + nb, p, g, dt, Om, dtheta, o, kPad, (nq + 1) * kPad,
                      (D.OpenInner && i0 == 0) ? sL + pidx(p) : nullptr);
      for (int r = 0; r < nb; r++) o[(r * (nq + 1) + nq) * kPad] = sIn[(kInT + r + 2) * kRow + p];
    }
    __syncthreads();  // radial results complete; the staged rows are free
    if (tn < nai) pend = tr_stage<nq>(B, items, tn, sIn, &s_bar);
    const int r = warp;
    if (r < nb) {
      const int i = i0 + r;
      float* sRr = sR + (size_t)r * (nq + 1) * kPad;
      const float Rm = D.Rmed[i];
      const float dxtheta = fm(dtheta, Rm);
      sweep_ring<nq>(sRr, s_vmed[r], s_vc[r], fast, dt, dxtheta, 1.0f / dxtheta, 1.0f / D.Surf[i],
                     fm(D.Rsup[i] - D.Rinf[i], dt));
      // window point x is source sector g0 + x - 4, stored at output sector
      // jb + x - 4 (jb < nsec and x - 4 < S <= nsec: one wrap at most)
      float* dsts[6] = {D.vri, D.vti, D.trr, D.tpp, D.a1, D.a0};
      const int row = i * nsec;
      const int jb = s_jb[r] - 4;
      for (int x = 4 + lane; x < L - 4; x += 32) {
        int j = jb + x;
        if (j >= nsec) j -= nsec;
#pragma unroll
        for (int c = 0; c < nq; c++) dsts[c == nq - 1 ? 5 : c][row + j] = sRr[c * kPad + pidx(x)];
        if (i == 0 && D.OpenInner) D.lost[g0 + x - 4] = sL[pidx(x)];
      }
    }
  }
  cp_async_wait<0>();
}

// ComputeVelocitiesKernel, Kernels.cu:1292-1306, from the transported
// momenta (vri, vti, trr, tpp) and density (a0); then the transported
// density (and energy, a1) become the state.
// One instance per kind of disk (kAdi: adiabatic, which also moves the
// transported energy into the state).
template <int kAdi>
__global__ void __launch_bounds__(kThreads, kAdi ? 4 : 5) k_velocities(BatchDev B) {
  QUAD_BEGIN_T(kAdi, -1)
  const float Om = C->OmegaFrame;
  float A0[4], Ad[4], Am[4], Rd[4], T0[4], P0[4], Pm[4], S0[4], E1[4];
  qld(A0, D.a0, q);  // transported density
  qld(Ad, D.a0, q, -nsec);
  qld_jm(Am, A0, D.a0, q, nsec);
  qld(Rd, D.vri, q, -nsec);
  qld(T0, D.vti, q);
  qld(P0, D.trr, q);
  qld_jm(Pm, P0, D.trr, q, nsec);
  qld(S0, D.tpp, q);
  if (kAdi == 1) qld(E1, D.a1, q);
  float vr[4], vt[4];
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const int i = q.i[u];
    if (i == 0)
      vr[u] = 0.0;
    else
      vr[u] = div_refined(Rd[u] + T0[u], A0[u] + Ad[u] + 1e-20f);
    vt[u] = div_refined(div_refined(Pm[u] + S0[u], A0[u] + Am[u] + 1e-15f), D.Rmed[i]) - D.Rmed[i] * Om;
  }
  qst(D.vrad, q, vr);
  qst(D.vtheta, q, vt);
  qst(D.dens, q, A0);
  if (kAdi == 1) qst(D.energy, q, E1);
  QUAD_END
}

// Compacted lists of the disks inside their DT, by the whole block (at most
// kThreads threads): the threads gather each disk's flags and sizes into
// shared memory, a chunk of blockDim.x disks at a time, and thread 0 then
// runs the prefix sums over shared memory (the disks' global reads are thus
// issued in parallel, not one dependent chain per disk).
__device__ void compact_active(const BatchDev& B) {
  __shared__ int s_act[kThreads], s_adi[kThreads], s_items[kThreads], s_nrad[kThreads];
  __shared__ int s_tiles[kThreads], s_ctiles[kThreads], s_vtiles[kThreads];
  __shared__ long long s_cells[kThreads];
  __shared__ long long s_cc;
  __shared__ int s_cnt[10];  // na, ni, nd, rr, ii, ia, gg, tt, ct, vt
  const int tid = threadIdx.x;
  if (tid == 0) {
    s_cc = 0;
    for (int k = 0; k < 10; k++) s_cnt[k] = 0;
  }
  for (int d0 = 0; d0 < B.ndisk; d0 += blockDim.x) {
    const int d = d0 + tid;
    if (d < B.ndisk) {
      const DiskDev& D = B.disks[d];
      const long long cells = (long long)D.nrad * D.nsec;
      s_act[tid] = D.ctl->active;
      s_adi[tid] = D.Adiabatic;
      s_items[tid] = D.nitems;
      s_nrad[tid] = D.nrad;
      s_cells[tid] = cells;
      s_tiles[tid] = (int)((cells + FARGO_QTILE - 1) / FARGO_QTILE);
      s_ctiles[tid] = fargo_cfl_tiles_own(D);
      s_vtiles[tid] = vtiles_of(D);
    }
    __syncthreads();
    if (tid == 0) {
      int na = s_cnt[0], ni = s_cnt[1], nd = s_cnt[2], rr = s_cnt[3], ii = s_cnt[4], ia = s_cnt[5];
      int gg = s_cnt[6], tt = s_cnt[7], ct = s_cnt[8], vt = s_cnt[9];
      long long cc = s_cc;
      const int n = min((int)blockDim.x, B.ndisk - d0);
      for (int k = 0; k < n; k++) {
        if (!s_act[k]) continue;
        const int d = d0 + k;
        B.act_disk[na] = d;
        B.act_cell_off[na] = cc;
        B.act_ring_off[na] = rr;
        B.act_grp_off[na] = gg;
        B.act_tile_off[na] = tt;
        B.act_ctile_off[na] = ct;
        B.act_vtile_off[na] = vt;
        cc += s_cells[k];
        rr += s_nrad[k];
        gg += (s_nrad[k] + FARGO_RM_RINGS - 1) / FARGO_RM_RINGS;
        tt += s_tiles[k];
        ct += s_ctiles[k];
        vt += s_vtiles[k];
        na++;
        if (s_adi[k]) {
          B.act_adi_disk[nd] = d;
          B.act_adi_off[nd] = ia;
          ia += s_items[k];
          nd++;
        } else {
          B.act_iso_disk[ni] = d;
          B.act_iso_off[ni] = ii;
          ii += s_items[k];
          ni++;
        }
      }
      s_cnt[0] = na, s_cnt[1] = ni, s_cnt[2] = nd, s_cnt[3] = rr, s_cnt[4] = ii, s_cnt[5] = ia;
      s_cnt[6] = gg, s_cnt[7] = tt, s_cnt[8] = ct, s_cnt[9] = vt;
      s_cc = cc;
    }
    __syncthreads();
  }
  if (tid == 0) {
    const int na = s_cnt[0], ni = s_cnt[1], nd = s_cnt[2];
    B.act_cell_off[na] = s_cc;
    B.act_ring_off[na] = s_cnt[3];
    B.act_grp_off[na] = s_cnt[6];
    B.act_tile_off[na] = s_cnt[7];
    B.act_ctile_off[na] = s_cnt[8];
    B.act_vtile_off[na] = s_cnt[9];
    B.act_iso_off[ni] = s_cnt[4];
    B.act_adi_off[nd] = s_cnt[5];
    B.act[0] = na;
    B.act[1] = ni;
    B.act[2] = nd;
  }
}

// End of a substep: which disks take another one; drives the graph's loop.
__global__ void k_substep_end(BatchDev B, cudaGraphConditionalHandle h, int use_handle) {
  __shared__ float sm[kThreads];
  // LostMass += VanLeerRadial's DeviceReduce of LostByDisk (TransportEuler.cu:72, 145)
  if (B.any_bc) {
    for (int d = 0; d < B.ndisk; d++) {
      const DiskDev& D = B.disks[d];
      if (!D.OpenInner || !D.IsDisk || !D.ctl->active) continue;  // block-uniform
      const float lost = ref_device_reduce([&](long j) { return D.lost[j]; }, D.nsec, sm);
      if (threadIdx.x == 0) D.ctl->LostMass += lost;
    }
    __syncthreads();
  }
  int any = 0;
  for (int d = threadIdx.x; d < B.ndisk; d += blockDim.x) {
    DiskCtl* C = B.disks[d].ctl;
    if (C->active) C->active = C->more;
    any |= C->active;
  }
  any = __syncthreads_or(any);
  compact_active(B);
  if (threadIdx.x == 0) {
    B.flags[0] = any;
    if (use_handle) cudaGraphSetConditional(h, any ? 1u : 0u);
  }
}

// Start of a DT (AlgoGas entry, SourceEuler.cu:211-229) for every disk.
__global__ void k_dt_begin(BatchDev B) {
  for (int d = threadIdx.x; d < B.ndisk; d += blockDim.x) {
    const DiskDev& D = B.disks[d];
    DiskCtl* C = D.ctl;
    C->dtemp = 0.0;
    C->nsub = 0;
    C->error = 0;  // an error is reported at the end of the DT it stopped
    C->active = 1;
    C->more = 1;
    C->counter = 0;
    prepare_bodies(D, C);
  }
  __syncthreads();
  compact_active(B);
}

// ComputeSoundSpeedKernel, adiabatic branch (Kernels.cu:190-191)
__global__ void __launch_bounds__(kThreads) k_cs_adiabatic(BatchDev B, int only_disk) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= B.ncell) return;
  const int d = disk_of_cell(B, c);
  const DiskDev& D = B.disks[d];
  if (!D.Adiabatic) return;
  if (only_disk >= 0 ? d != only_disk : !D.ctl->active) return;
  const int loc = (int)(c - D.cell0);
  const long long l = loc;
  D.cs[l] = sqrtf(D.ADIABATICINDEX * (D.ADIABATICINDEX - 1.0) * D.energy[l] / D.dens[l]);
}

// ComputeSoundSpeedKernel, isothermal branch (Kernels.cu:185-188): one value per ring.
__global__ void k_cs_isothermal(BatchDev B, int only_disk) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= B.nring) return;
  const int d = disk_of_ring(B, r);
  const DiskDev& D = B.disks[d];
  if (D.Adiabatic) return;
  if (only_disk >= 0 && d != only_disk) return;
  const int i = r - D.ring0;
  const DiskCtl* C = D.ctl;
  float AspectRatio = aspect_ratio_dev(D, D.Rmed[i], C->PhysicalTime, C->PhysicalTimeInitial);
  D.cs_ring[i] = AspectRatio * sqrtf(1.0 * 1.0 / D.Rmed[i]) * powf(D.Rmed[i], D.FLARINGINDEX);
}

// Make1DprofileKernel on the sound speed (Kernels.cu:726-738): GLOBAL_bufarray.
// One warp per ring, lane 0 adds the sectors in order.
__global__ void k_cs_ringmean(BatchDev B, int only_disk) {
  int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (r >= B.nring) return;
  const int d = disk_of_ring(B, r);
  const DiskDev& D = B.disks[d];
  if (only_disk >= 0 ? d != only_disk : !D.ctl->active) return;
  if (lane != 0) return;
  const int i = r - D.ring0, nsec = D.nsec;
  float sum = 0.0f;
  KahanSum ks;  // accurate mode
  if (D.Adiabatic) {
    const float* f = D.cs + (size_t)i * nsec;
    if (D.accurate) {
      for (int j = 0; j < nsec; j++) ks.add(f[j]);
    } else {
      for (int j = 0; j < nsec; j++) sum += f[j];
    }
  } else {
    const float v = D.cs_ring[i];
    if (D.accurate) {
      for (int j = 0; j < nsec; j++) ks.add(v);
    } else {
      for (int j = 0; j < nsec; j++) sum += v;
    }
  }
  if (D.accurate) sum = ks.s;
  D.csmean[i] = sum / (float)nsec;
}

// ------------------------------------------------------- boundary conditions

// ApplyBoundaryCondition (SideEuler.cu:172-182), ring-local part, one block
// per ring of the disks inside their DT (contiguous runs, DiskDev in shared
// memory):
//  - NONREFLECTING, adiabatic: ComputeSoundSpeed first (SideEuler.cu:176-177),
//    then, for alpha viscosity, the ring-mean sound speed and the viscosity
//    that the next ComputeViscousTerms rebuilds from it (Viscosity.cu:79-86);
//  - EVANESCENT: EvanescentBoundaryKernel (Kernels.cu:1076-1124) in the
//    damping zones; at the first call of a substep it is preceded by
//    CorrectVtheta, applied here in place (k_source1 then skips it).
// stage 0, 1, 2: the calls before Substep1, before Substep3, after Transport
// (SourceEuler.cu:267, 285, 292).
template <int stage>
__global__ void __launch_bounds__(kThreads) k_bc_rings(BatchDev B) {
  __shared__ DiskDev sD;
  const int tid = threadIdx.x;
  const int na = B.act[0];
  const int ntile = na > 0 ? B.act_ring_off[na] : 0;
  const int per = (ntile + gridDim.x - 1) / gridDim.x;
  const int t0 = blockIdx.x * per, t1 = min(t0 + per, ntile);
  int lo = 0, hi = -1;
  for (int t = t0; t < t1; t++) {
    if (t >= hi) {  // block-uniform: entering a disk
      const int a = find_range(B.act_ring_off, na, t);
      lo = B.act_ring_off[a];
      hi = B.act_ring_off[a + 1];
      __syncthreads();
      copy_words(&sD, B.disks + B.act_disk[a], sizeof(DiskDev));
      __syncthreads();
    }
    const DiskDev& D = sD;
    const DiskCtl* C = D.ctl;
    if (!D.IsDisk) continue;
    const int i = t - lo, nsec = D.nsec;
    const size_t r0 = (size_t)i * nsec;
    if (D.NonReflecting && D.Adiabatic) {
      for (int j = tid; j < nsec; j += kThreads)
        D.cs[r0 + j] = sqrtf(D.ADIABATICINDEX * (D.ADIABATICINDEX - 1.0) * D.energy[r0 + j] / D.dens[r0 + j]);
      if (D.ViscosityAlpha) {
        __syncthreads();
        if (tid == 0) {
          float sum = 0.0f;  // Make1DprofileKernel: sectors in order
          if (D.accurate) {
            KahanSum ks;
            for (int j = 0; j < nsec; j++) ks.add(D.cs[r0 + j]);
            sum = ks.s;
          } else {
            for (int j = 0; j < nsec; j++) sum += D.cs[r0 + j];
          }
          D.csmean[i] = sum / (float)nsec;
          D.visc[i] = fviscosity_ring(D, i, C->time_start, C->PhysicalTimeInitial);
        }
      }
    }
    if (D.Evanescent) {
      const float Rm = D.Rmed[i];
      if (stage == 0 && C->domega != 0.0f)
        for (int j = tid; j < nsec; j += kThreads) D.vtheta[r0 + j] = D.vtheta[r0 + j] - C->domega * Rm;
      const float DRMIN = D.ev_DRMIN, DRMAX = D.ev_DRMAX;
      if ((Rm < DRMIN) || (Rm > DRMAX)) {
        float damping, lambda = 0.0f;
        if (Rm < DRMIN) {
          damping = (Rm - DRMIN) / (D.Rmed[0] - DRMIN);
          lambda = damping * damping * 10.0 * C->dtf / D.ev_Tin;
        }
        if (Rm > DRMAX) {
          damping = (Rm - DRMAX) / (D.Rmed[D.nrad - 1] - DRMAX);
          lambda = damping * damping * 10.0 * C->dtf / D.ev_Tout;
        }
        // the self-gravity form subtracts Rmed * GLOBAL_bufarray_d[i], an
        // array the reference never fills (zero)
        const float AspectRatio = aspect_ratio_dev(D, Rm, C->time_start, C->PhysicalTimeInitial);
        float vtheta0 = sqrtf(1.0 * 1.0 / Rm *
                              (1.0 - (1.0 + D.SIGMASLOPE - 2.0 * D.FLARINGINDEX) * powf(AspectRatio, 2.0f) *
                                         powf(Rm, (float)(2.0 * D.FLARINGINDEX))));
        vtheta0 -= Rm * C->OmegaFrame;
        const float vrad0 = -3.0 * D.visc[i] / Rm * (-D.SIGMASLOPE + .5);
        const float dens0 = D.SigmaMed[i];
        const float energy0 = D.EnergyMed[i];
        for (int j = tid; j < nsec; j += kThreads) {
          const size_t l = r0 + j;
          D.vrad[l] = (D.vrad[l] + lambda * vrad0) / (1.0 + lambda);
          D.vtheta[l] = (D.vtheta[l] + lambda * vtheta0) / (1.0 + lambda);
          D.dens[l] = (D.dens[l] + lambda * dens0) / (1.0 + lambda);
          if (D.Adiabatic) D.energy[l] = (D.energy[l] + lambda * energy0) / (1.0 + lambda);
        }
      }
    }
  }
}

// ApplyBoundaryCondition, edge-ring part, one block per disk inside its DT:
// OpenBoundaryKernel (Kernels.cu:623-637) and NonReflectingBoundary
// (SideEuler.cu:70-101: ReduceCs, the angular offsets i_angle / i_angle2,
// NonReflectingBoundaryKernel, ReduceMean, MinusMeanKernel,
// Kernels.cu:640-722), with the ring means reduced in DeviceReduce's order.
__global__ void __launch_bounds__(kThreads) k_bc_disk(BatchDev B) {
  __shared__ float sm[kThreads];
  __shared__ int s_angle[2];
  const int tid = threadIdx.x;
  const int na = B.act[0];
  for (int a = blockIdx.x; a < na; a += gridDim.x) {
    const DiskDev& D = B.disks[B.act_disk[a]];
    if (!D.IsDisk || !(D.OpenInner || D.NonReflecting)) continue;
    const int nsec = D.nsec, nrad = D.nrad;
    float* Dn = D.dens;
    float* En = D.energy;
    float* Vr = D.vrad;
    if (D.OpenInner) {
      const float SigmaMed = D.SigmaMed[0];
      for (int j = tid; j < nsec; j += kThreads) {
        const int i = 1;
        Dn[(i - 1) * nsec + j] = Dn[i * nsec + j];
        En[(i - 1) * nsec + j] = En[i * nsec + j];
        if (Vr[(i + 1) * nsec + j] > 0.0 || (Dn[i * nsec + j] < SigmaMed))
          Vr[i * nsec + j] = 0.0;
        else
          Vr[i * nsec + j] = Vr[(i + 1) * nsec + j];
      }
    }
    if (D.NonReflecting) {
      auto csr = [&](int r) {
        return [&, r](long j) -> float {
          return D.Adiabatic ? D.cs[(size_t)r * nsec + j] : D.cs_ring[r];
        };
      };
      const float cs0_r = ref_device_reduce(csr(0), nsec, sm) / (float)nsec;
      const float cs1_r = ref_device_reduce(csr(1), nsec, sm) / (float)nsec;
      const float csnrm1_r = ref_device_reduce(csr(nrad - 1), nsec, sm) / (float)nsec;
      const float csnrm2_r = ref_device_reduce(csr(nrad - 2), nsec, sm) / (float)nsec;
      if (tid == 0) {
        // host arithmetic of NonReflectingBoundary, pow() of the radii from the host
        double dangle = (D.nr_pow_in - 1.0) / (.5 * (cs0_r + cs1_r));
        dangle *= (D.Rmed[1] - D.Rmed[0]);
        s_angle[0] = (int)(dangle / 2.0 / PI_D * (float)nsec + .5);
        double dangle2 = (D.nr_pow_out - 1.0) / (.5 * (csnrm1_r + csnrm2_r));
        dangle2 *= (D.Rmed[nrad - 1] - D.Rmed[nrad - 2]);
        s_angle[1] = (int)(dangle2 / 2.0 / PI_D * (float)nsec + .5);
      }
      __syncthreads();
      const int i_angle = s_angle[0], i_angle2 = s_angle[1];
      const float* cs = D.cs;
      const float SigmaMed = D.SigmaMed[1], SigmaMed2 = D.SigmaMed[nrad - 2];
      for (int j = tid; j < nsec; j += kThreads) {
        int i = 1, jp = j + i_angle;
        if (jp >= nsec) jp -= nsec;
        if (jp < 0) jp += nsec;
        float csv = D.Adiabatic ? cs[(size_t)i * nsec + j] : D.cs_ring[i];
        Dn[jp] = Dn[i * nsec + j];
        En[jp] = En[i * nsec + j];
        float Vrad_med = -csv * (Dn[i * nsec + j] - SigmaMed) / SigmaMed;
        Vr[i * nsec + j] = 2. * Vrad_med - Vr[(i + 1) * nsec + j];
        i = nrad - 1;
        jp = j - i_angle2;
        if (jp >= nsec) jp -= nsec;
        if (jp < 0) jp += nsec;
        csv = D.Adiabatic ? cs[(size_t)i * nsec + j] : D.cs_ring[i];
        Dn[i * nsec + j] = Dn[jp + (i - 1) * nsec];
        En[i * nsec + j] = En[jp + (i - 1) * nsec];
        Vrad_med = csv * (Dn[(i - 1) * nsec + j] - SigmaMed2) / SigmaMed2;
        Vr[i * nsec + j] = 2. * Vrad_med - Vr[(i - 1) * nsec + j];
      }
      __syncthreads();
      const size_t lo = (size_t)(nrad - 1) * nsec;
      const float mean_dens_r = ref_device_reduce([&](long j) { return Dn[j]; }, nsec, sm) / (float)nsec;
      const float mean_dens_r2 = ref_device_reduce([&](long j) { return Dn[lo + j]; }, nsec, sm) / (float)nsec;
      const float mean_energy_r = ref_device_reduce([&](long j) { return En[j]; }, nsec, sm) / (float)nsec;
      const float mean_energy_r2 = ref_device_reduce([&](long j) { return En[lo + j]; }, nsec, sm) / (float)nsec;
      const float sm0 = D.SigmaMed[0], sm1 = D.SigmaMed[nrad - 1];
      const float em0 = D.EnergyMed[0], em1 = D.EnergyMed[nrad - 1];
      for (int j = tid; j < nsec; j += kThreads) {
        Dn[j] += sm0 - mean_dens_r;
        En[j] += em0 - mean_energy_r;
        Dn[lo + j] += sm1 - mean_dens_r2;
        En[lo + j] += em1 - mean_energy_r2;
      }
    }
    __syncthreads();
  }
}

// Sector tables: the angle formulas of FillForcesArraysKernel
// (Kernels.cu:1332) and InitComputeAccelKernel (Kernels.cu:170-171).
__global__ void k_sector_tables(BatchDev B) {
  int d = blockIdx.y;
  if (d >= B.ndisk) return;
  const DiskDev& D = B.disks[d];
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= D.nsec) return;
  int nsec = D.nsec;
  float angle = (float)j / (float)nsec * 2.0 * PI_D;
  const_cast<float*>(D.cos_pot)[j] = cosf(angle);
  const_cast<float*>(D.sin_pot)[j] = sinf(angle);
  const_cast<float*>(D.cos_cell)[j] = cosf(2.0 * PI_D * (float)j / (float)nsec);
  const_cast<float*>(D.sin_cell)[j] = sinf(2.0 * PI_D * (float)j / (float)nsec);
}

// InitGasVelocitiesKernel (Kernels.cu:759-800).  Its ViscosityAlpha argument
// is always 0 in the reference (int global read as float, then converted
// back, Pframeforce.cu:20,269), so the constant-viscosity drift is used.
__global__ void __launch_bounds__(kThreads) k_init_velocities(BatchDev B, int disk) {
  // cells of one disk including the ghost row
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int d = disk;
  const DiskDev& D = B.disks[d];
  if (c >= (long long)(D.nrad + 1) * D.nsec) return;
  const long long base = 0;
  const DiskCtl* C = D.ctl;
  const int nsec = D.nsec, nrad = D.nrad;
  const int loc = (int)(c - base), i = loc / nsec;
  const long long l = loc;
  float omega, r, ri;
  if (i == nrad) {
    r = D.Rmed[nrad - 1];
    ri = D.Rinf[nrad - 1];
  } else {
    r = D.Rmed[i];
    ri = D.Rinf[i];
  }
  float vt = D.vtheta[l];
  if (!D.SelfGravity) {
    omega = sqrtf(1.0 * 1.0 / r / r / r);
    vt = omega * r *
         sqrtf(1.0 - powf(D.ASPECTRATIO, 2.0) * powf(r, 2.0 * D.FLARINGINDEX) *
                         (1. + D.SIGMASLOPE - 2.0 * D.FLARINGINDEX));
  }
  vt -= C->OmegaFrame * r;
  D.vtheta[l] = vt;
  float vr;
  if (i == nrad)
    vr = 0.0;
  else {
    vr = D.IMPOSEDDISKDRIFT * D.SIGMA0 / D.SigmaInf[i] / ri;
    vr -= 3.0 * D.visc[i] / r * (-D.SIGMASLOPE + .5);
  }
  if (i == 0) vr = 0.0;
  D.vrad[l] = vr;
  // initial pressure (ComputePressureField in InitEuler) for the temperature output
  if (!D.Adiabatic && i < nrad) {
    float cs = D.cs_ring[i];
    D.pres[l] = D.dens[l] * cs * cs;
  }
}

// ComputeForce for one body at every Hill-cut level (Force.cu:314-328), as
// UpdateLog uses it: 44 double sums.
__global__ void __launch_bounds__(kThreads) k_disk_force(BatchDev B, int disk, float x, float y, float rs,
                                                         float rh0, float a, double* out) {
  const DiskDev& D = B.disks[disk];
  const int nsec = D.nsec, nrad = D.nrad;
  long long n = (long long)nrad * nsec;
  double s[4 * FARGO_DIMFXY];
  for (int q = 0; q < 4 * FARGO_DIMFXY; q++) s[q] = 0.0;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    int i = (int)(c / nsec), j = (int)(c - (long long)i * nsec);
    float cellmass = D.Surf[i] * D.dens[c];
    float dx = D.Rmed[i] * D.cos_cell[j] - x;
    float dy = D.Rmed[i] * D.sin_cell[j] - y;
    float d2 = dx * dx + dy * dy;
    float dist2 = d2 + rs * rs;
    float distance = sqrtf(dist2);
    float InvDist3 = 1.0 / dist2 / distance;  // two FP64 divisions, as Kernels.cu:821
    bool inner = D.Rmed[i] < a;
    for (int k = 0; k < FARGO_DIMFXY; k++) {
      float hillcutfactor = (float)k / (float)(FARGO_DIMFXY - 1);
      float hill_cut;
      if (k != 0) {
        float rh = rh0 * hillcutfactor;
        hill_cut = 1. - expf(-d2 / (rh * rh));
      } else
        hill_cut = 1.;
      float fx = 1.0 * cellmass * dx * InvDist3 * hill_cut;
      float fy = 1.0 * cellmass * dy * InvDist3 * hill_cut;
      if (inner) {
        s[k] += fx;
        s[k + 2 * FARGO_DIMFXY] += fy;
      } else {
        s[k + FARGO_DIMFXY] += fx;
        s[k + 3 * FARGO_DIMFXY] += fy;
      }
    }
  }
  __shared__ double red[kThreads / 32];
  for (int q = 0; q < 4 * FARGO_DIMFXY; q++) {
    double v = warp_sum_d(s[q]);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double acc = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) acc += red[w];
      out[(size_t)blockIdx.x * 4 * FARGO_DIMFXY + q] = acc;
    }
    __syncthreads();
  }
}

// FP64 diagnostics: mass, angular momentum, Hill-sphere mass of planet 0
// (CircumPlanetaryMassKernel, Kernels.cu:245-261).
__global__ void __launch_bounds__(kThreads) k_diagnostics(BatchDev B, int disk, double* out) {
  const DiskDev& D = B.disks[disk];
  const DiskCtl* C = D.ctl;
  const int nsec = D.nsec, nrad = D.nrad;
  long long n = (long long)nrad * nsec;
  float xpl = C->nb > 0 ? (float)C->x[0] : 0.0f, ypl = C->nb > 0 ? (float)C->y[0] : 0.0f;
  double m = 0, am = 0, hill = 0;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    int i = (int)(c / nsec), j = (int)(c - (long long)i * nsec);
    int jp = jwrap_p(j, nsec);
    double cm = (double)D.Surf[i] * (double)D.dens[c];
    m += cm;
    am += cm * (double)D.Rmed[i] *
          (0.5 * ((double)D.vtheta[c] + (double)D.vtheta[(long long)i * nsec + jp]) + (double)D.Rmed[i] * C->OmegaFrame);
    float cx = D.Rmed[i] * D.cos_cell[j], cy = D.Rmed[i] * D.sin_cell[j];
    float dist = sqrtf((cx - xpl) * (cx - xpl) + (cy - ypl) * (cy - ypl));
    if (C->nb > 0 && dist < D.HillRadius) hill += (double)(float)(D.Surf[i] * D.dens[c]);
  }
  __shared__ double red[3][kThreads / 32];
  m = warp_sum_d(m);
  am = warp_sum_d(am);
  hill = warp_sum_d(hill);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = m;
    red[1][threadIdx.x >> 5] = am;
    red[2][threadIdx.x >> 5] = hill;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double acc = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) acc += red[threadIdx.x][w];
    out[(size_t)blockIdx.x * 3 + threadIdx.x] = acc;
  }
}

}  // namespace

// ------------------------------------------------------------------ launchers
// This file is compiled twice: with contraction of a*b+c into fused
// multiply-adds (fargo_k) and, with FARGO_NOFMA defined, without
// (fargo_k_nofma, nvcc -fmad=false); fargo_internal.h has the dispatch.
#ifdef FARGO_NOFMA
#define FARGO_KNS fargo_k_nofma
#else
#define FARGO_KNS fargo_k
#endif
namespace FARGO_KNS {

static inline unsigned cell_blocks(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }


void fargo_launch_dt_begin(const BatchDev& b, cudaStream_t s) { k_dt_begin<<<1, 128, 0, s>>>(b); }

void fargo_launch_cs_refresh(const BatchDev& b, int only_disk, cudaStream_t s) {
  k_cs_adiabatic<<<cell_blocks(b.ncell), kThreads, 0, s>>>(b, only_disk);
  k_cs_ringmean<<<(unsigned)((b.nring * 32 + kThreads - 1) / kThreads), kThreads, 0, s>>>(b, only_disk);
}

void fargo_launch_cs_isothermal(const BatchDev& b, int only_disk, cudaStream_t s) {
  k_cs_isothermal<<<(unsigned)((b.nring + 127) / 128), 128, 0, s>>>(b, only_disk);
}


const char* fargo_substep_kernel_name(int k) {
  static const char* names[] = {"k_ring_mean_cfl", "k_cfl_force",    "k_potential",  "k_boundary_0",
                                "k_source1",       "k_viscosity",    "k_source2",    "k_boundary_1",
                                "k_energy",        "k_ring_mean_tr", "k_transport",  "k_velocities",
                                "k_boundary_2",    "k_substep_end"};
  return (k >= 0 && k < FARGO_NKERNELS) ? names[k] : "";
}

void fargo_launch_substep(const BatchDev& b, cudaGraphConditionalHandle h, int use_handle, cudaStream_t s,
                          int max_nsec, long long* launches, cudaEvent_t* ev, int part) {
  (void)max_nsec;
  int k = 0;
#define REC()                                  \
  do {                                         \
    if (ev) cudaEventRecord(ev[k], s);         \
    k++;                                       \
  } while (0)
  if (part & FARGO_PART_HEAD) {
    REC();
    k_ring_mean<0><<<b.grp_grid, kRMT, fargo_ring_mean_smem_bytes(), s>>>(b);
    REC();
    if (b.max_body <= 1)
      k_cfl_force<1><<<b.g_cfl, kThreads, 0, s>>>(b);
    else if (b.max_body <= 2)
      k_cfl_force<2><<<b.g_cfl, kThreads, 0, s>>>(b);
    else if (b.max_body <= 4)
      k_cfl_force<4><<<b.g_cfl, kThreads, 0, s>>>(b);
    else
      k_cfl_force<FARGO_MAXBODY><<<b.g_cfl, kThreads, 0, s>>>(b);
  } else {
    k = 2;
  }
  if (!(part & FARGO_PART_TAIL)) {
    if (launches) *launches += 2;
    return;
  }
  REC();
  k_potential<<<b.g_potential, kThreads, 0, s>>>(b);
  REC();
  if (b.any_bc) {
    k_bc_rings<0><<<b.ring_grid, kThreads, 0, s>>>(b);
    k_bc_disk<<<b.ndisk, kThreads, 0, s>>>(b);
  }
  REC();
  if (b.src1_classes & 1) k_source1<0, 0><<<b.g_source1[0], kThreads, 0, s>>>(b);
  if (b.src1_classes & 2) k_source1<0, 1><<<b.g_source1[1], kThreads, 0, s>>>(b);
  if (b.src1_classes & 4) k_source1<1, 0><<<b.g_source1[2], kThreads, 0, s>>>(b);
  if (b.src1_classes & 8) k_source1<1, 1><<<b.g_source1[3], kThreads, 0, s>>>(b);
  REC();
  k_viscosity<<<b.g_viscosity, kThreads, kViscSmem, s>>>(b);
  REC();
  if (b.ntheta_iso) k_source2<0><<<b.g_source2[0], kThreads, 0, s>>>(b);
  if (b.ntheta_adi) k_source2<1><<<b.g_source2[1], kThreads, 0, s>>>(b);
  REC();
  if (b.any_bc) {
    k_bc_rings<1><<<b.ring_grid, kThreads, 0, s>>>(b);
    k_bc_disk<<<b.ndisk, kThreads, 0, s>>>(b);
  }
  REC();
  if (b.ntheta_adi) k_energy<<<b.g_energy, kThreads, 0, s>>>(b);  // adiabatic disks only
  REC();
  k_ring_mean<1><<<b.grp_grid, kRMT, fargo_ring_mean_smem_bytes(), s>>>(b);
  REC();
  if (b.ntheta_iso)
    k_transport<5><<<std::min(b.g_transport, b.ntheta_iso), kTT, fargo_transport_smem_bytes(0), s>>>(b, b.theta_iso);
  if (b.ntheta_adi)
    k_transport<6><<<std::min(b.g_transport, b.ntheta_adi), kTT, fargo_transport_smem_bytes(1), s>>>(b, b.theta_adi);
  REC();
  if (b.ntheta_iso) k_velocities<0><<<b.g_velocities[0], kThreads, 0, s>>>(b);
  if (b.ntheta_adi) k_velocities<1><<<b.g_velocities[1], kThreads, 0, s>>>(b);
  REC();
  if (b.any_bc) {
    k_bc_rings<2><<<b.ring_grid, kThreads, 0, s>>>(b);
    k_bc_disk<<<b.ndisk, kThreads, 0, s>>>(b);
  }
  REC();
  k_substep_end<<<1, kThreads, 0, s>>>(b, h, use_handle);
  REC();
#undef REC
  if (launches) *launches += FARGO_KNS::fargo_substep_launches(b) - ((part & FARGO_PART_HEAD) ? 0 : 2);
}

void fargo_launch_stripe_block(const BatchDev& b, double* out, cudaStream_t s) {
  k_stripe_block<<<1, kThreads, 0, s>>>(b, out);
}

int fargo_launch_stripe_finish(const BatchDev& b, const double* blk, int nstripe, int stride, cudaStream_t s) {
  if (nstripe < 1 || nstripe > kMaxStripes) return 1;
  if (b.max_body <= 1)
    k_stripe_finish<1><<<1, kThreads, 0, s>>>(b, blk, nstripe, stride);
  else if (b.max_body <= 2)
    k_stripe_finish<2><<<1, kThreads, 0, s>>>(b, blk, nstripe, stride);
  else if (b.max_body <= 4)
    k_stripe_finish<4><<<1, kThreads, 0, s>>>(b, blk, nstripe, stride);
  else
    k_stripe_finish<FARGO_MAXBODY><<<1, kThreads, 0, s>>>(b, blk, nstripe, stride);
  return 0;
}

// The transport kernels alone (both forms), for the autotuner: they read the
// state and the last substep's ring means and write only scratch.
void fargo_launch_transport(const BatchDev& b, cudaStream_t s) {
  if (b.ntheta_iso)
    k_transport<5><<<std::min(b.g_transport, b.ntheta_iso), kTT, fargo_transport_smem_bytes(0), s>>>(b, b.theta_iso);
  if (b.ntheta_adi)
    k_transport<6><<<std::min(b.g_transport, b.ntheta_adi), kTT, fargo_transport_smem_bytes(1), s>>>(b, b.theta_adi);
}

// The CFL/force kernel instance for up to max_body bodies.
const void* fargo_cfl_kernel(int max_body) {
  return max_body <= 1   ? (const void*)k_cfl_force<1>
         : max_body <= 2 ? (const void*)k_cfl_force<2>
         : max_body <= 4 ? (const void*)k_cfl_force<4>
                         : (const void*)k_cfl_force<FARGO_MAXBODY>;
}

// Grids of the substep kernels: one wave of resident blocks (the kernels walk
// contiguous runs of tiles, so a second partial wave would idle most SMs),
// never more blocks than work items.
cudaError_t fargo_size_grids(BatchDev& b, int nsm, long long ncell_tiles, int nitems) {
  auto wave = [&](const void* fn, int threads, size_t smem, long long work, int* out) -> cudaError_t {
    int per = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem);
    if (e != cudaSuccess) return e;
    long long g = (long long)nsm * (per > 0 ? per : 1);
    *out = (int)std::max<long long>(1, std::min<long long>(g, work));
    return cudaSuccess;
  };
  cudaError_t e;
  if ((e = wave(fargo_cfl_kernel(b.max_body), kThreads, 0, b.ncfl, &b.g_cfl))) return e;
  if ((e = wave((const void*)k_source1<0, 0>, kThreads, 0, ncell_tiles, &b.g_source1[0]))) return e;
  if ((e = wave((const void*)k_source1<0, 1>, kThreads, 0, ncell_tiles, &b.g_source1[1]))) return e;
  if ((e = wave((const void*)k_source1<1, 0>, kThreads, 0, ncell_tiles, &b.g_source1[2]))) return e;
  if ((e = wave((const void*)k_source1<1, 1>, kThreads, 0, ncell_tiles, &b.g_source1[3]))) return e;
  if ((e = wave((const void*)k_potential, kThreads, 0, ncell_tiles, &b.g_potential))) return e;
  if ((e = wave((const void*)k_viscosity, kThreads, kViscSmem, ncell_tiles, &b.g_viscosity))) return e;
  if ((e = wave((const void*)k_source2<0>, kThreads, 0, ncell_tiles, &b.g_source2[0]))) return e;
  if ((e = wave((const void*)k_source2<1>, kThreads, 0, ncell_tiles, &b.g_source2[1]))) return e;
  if ((e = wave((const void*)k_energy, kThreads, 0, ncell_tiles, &b.g_energy))) return e;
  if ((e = wave((const void*)k_velocities<0>, kThreads, 0, ncell_tiles, &b.g_velocities[0]))) return e;
  if ((e = wave((const void*)k_velocities<1>, kThreads, 0, ncell_tiles, &b.g_velocities[1]))) return e;
  return wave((const void*)k_transport<6>, kTT, fargo_transport_smem_bytes(1), nitems, &b.g_transport);
}

// Launches of one substep: 6 kernels, one Substep1 instance per kind of disk
// present, the energy kernel when a disk is adiabatic, the isothermal and the
// adiabatic forms of Substep2, transport and the velocity update when the
// batch holds both, two per boundary call when a disk has a non-rigid
// boundary.
int fargo_substep_launches(const BatchDev& b) {
  return 6 + __builtin_popcount((unsigned)b.src1_classes) + (b.ntheta_adi ? 1 : 0) +
         3 * ((b.ntheta_iso && b.ntheta_adi) ? 2 : 1) + (b.any_bc ? 6 : 0);
}

void fargo_launch_sector_tables(const BatchDev& b, int max_nsec, cudaStream_t s) {
  dim3 g((max_nsec + 255) / 256, b.ndisk);
  k_sector_tables<<<g, 256, 0, s>>>(b);
}

void fargo_launch_init_velocities(const BatchDev& b, int disk, long long ncell_ghost, cudaStream_t s) {
  k_init_velocities<<<cell_blocks(ncell_ghost), kThreads, 0, s>>>(b, disk);
}

void fargo_launch_disk_force(const BatchDev& b, int disk, float x, float y, float rs, float rh, float a,
                             double* out44, int nblocks, cudaStream_t s) {
  k_disk_force<<<nblocks, kThreads, 0, s>>>(b, disk, x, y, rs, rh, a, out44);
}

void fargo_launch_diagnostics(const BatchDev& b, int disk, double* out3, int nblocks, cudaStream_t s) {
  k_diagnostics<<<nblocks, kThreads, 0, s>>>(b, disk, out3);
}

cudaError_t fargo_kernel_attributes(int max_nsec) {
  (void)max_nsec;
  cudaError_t e = cudaFuncSetAttribute(k_ring_mean<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)fargo_ring_mean_smem_bytes());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_ring_mean<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)fargo_ring_mean_smem_bytes());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_viscosity, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kViscSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_transport<5>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)fargo_transport_smem_bytes(0));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_transport<6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)fargo_transport_smem_bytes(1));
}

}  // namespace FARGO_KNS
