// fargo_internal.h -- device-side data layout of the B200 FARGO step.
//
// A "batch" is a list of independent disks (a single disk is a batch of
// one).  Every kernel takes the batch descriptor and walks a flat work list,
// so one launch advances every disk that is still inside its DT.
//
// Per disk, in HBM:
//   grid fields   float32, ring-major, (nrad+1)*nsec, element [i*nsec+j]
//   ring tables   float32, nrad+1 entries (host-built in double, rounded
//                 to float exactly as FillPolar1DArrays does)
//   sector tables float32, nsec entries (cosf/sinf of the two angle
//                 formulas the reference uses)
//   DiskCtl       mutable scalars: DT bookkeeping, planets (FP64),
//                 potential parameters, force sums, logs.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define FARGO_PI 3.14159265358979323844
#define FARGO_CFLSECURITY 0.5
#define FARGO_CVNR 1.41
#define FARGO_MAXLOG 2048  // substeps logged per DT (Nshift + dt)

#include "../../include/fargo_b200.h"

// planets integrated on the device (the reference's limit, RungeKutta.cu:4)
#define FARGO_MAXPLANETS_DEV FARGO_MAXPLANETS
// bodies whose disk force is summed every substep: the star and up to 7
// FeelDisk planets (each carries 2 double accumulators per thread)
#define FARGO_MAXBODY 8

struct DiskCtl {
  // DT bookkeeping (SourceEuler.cu:211-241)
  double dtemp;        // time advanced inside the current DT
  double dt;           // current substep dt (double, as in AlgoGas)
  float dtf;           // (float)dt, the value every kernel receives
  int active;          // 1 while this disk is inside a substep of the current DT
  int more;            // set by the CFL finalize: another substep follows
  int nsub;            // substeps taken in the current DT
  int nsub_total;
  int error;           // nonzero: 1 non-finite CFL, 2 too many substeps
  unsigned int counter;        // last-block ticket of the CFL/force kernel
  float PhysicalTime;          // advanced at the end of each substep
  float time_start;            // PhysicalTime at the start of this substep
  float PhysicalTimeInitial;
  float OmegaFrame;
  float MassTaper;
  float domega;                // CorrectVtheta amount of this substep (0 if not corotating)
  float LostMass;
  // potential parameters of this substep (FillForcesArraysKernel arguments, floats)
  float itx, ity;              // IndirectTerm
  float pxp[FARGO_MAXPLANETS_DEV], pyp[FARGO_MAXPLANETS_DEV], psmooth[FARGO_MAXPLANETS_DEV];
  float pmass[FARGO_MAXPLANETS_DEV], pipd3[FARGO_MAXPLANETS_DEV];
  // planets, FP64 (Types.cuh:2-15)
  int nb;
  double mass[FARGO_MAXPLANETS_DEV], x[FARGO_MAXPLANETS_DEV], y[FARGO_MAXPLANETS_DEV];
  double vx[FARGO_MAXPLANETS_DEV], vy[FARGO_MAXPLANETS_DEV];
  int feeldisk[FARGO_MAXPLANETS_DEV], feelothers[FARGO_MAXPLANETS_DEV];
  float Xplanet_mark, Yplanet_mark;  // Psys.cu:79 static floats of GetPsysInfo
  // bodies whose disk force the CFL/force kernel sums this substep:
  // body 0 = star, then FeelDisk planets; coordinates as ComputeAccel floats
  int nbody;
  int body_planet[FARGO_MAXBODY];
  float bx[FARGO_MAXBODY], by[FARGO_MAXBODY], brs[FARGO_MAXBODY];
  float brh[FARGO_MAXBODY], ba[FARGO_MAXBODY];
  // self-gravity axisymmetric accelerations at rings 0 and NRAD-1
  float axisg_in, axisg_out;
};

// cell tiles of the cell kernels: FARGO_QTILE consecutive cells of one disk,
// four per thread
#define FARGO_QTILE 1024

// CFL/force tiles: DiskDev::cfl_tile consecutive cells of one disk, each with
// its own minimum and force partials: FARGO_CFL_TILE, or FARGO_CFL_TILE_SMALL
// in a batch too small to give every SM two tiles of the large size (more
// blocks share the per-cell work of a small disk)
#define FARGO_CFL_TILE 4096
#define FARGO_CFL_TILE_SMALL 1024
inline __host__ __device__ int fargo_cfl_tiles(int nrad, int nsec, int tile) {
  return (int)(((long long)nrad * nsec + tile - 1) / tile);
}

// CFL tiles of a disk's own rings (every ring unless it is a radial stripe)
#define fargo_cfl_tiles_own(D) fargo_cfl_tiles((D).own_hi - (D).own_lo, (D).nsec, (D).cfl_tile)

// scratch of the device RK5 (q0, q1, k1..k6, distances, perturber quotients):
// 34 doubles per planet
#define FARGO_RK_WORK(nb) (34 * (nb))

struct DiskDev {
  int nrad, nsec;
  long long cell0;  // first active cell of this disk in the batch's flat index
  int ring0;        // first ring of this disk in the batch's flat ring index
  int item0, nitems;  // its transport items in the isothermal or adiabatic list
  // parameters (floats, as the reference's globals)
  float DT, ADIABATICINDEX, ASPECTRATIO, FLARINGINDEX, SIGMASLOPE, SIGMA0;
  float TRANSITIONRADIUS, TRANSITIONRATIO, TRANSITIONWIDTH, LAMBDADOUBLING;
  float VISCOSITY, ALPHAVISCOSITY, CAVITYRADIUS, CAVITYRATIO, CAVITYWIDTH;
  float MASSTAPER, RELEASEDATE, RELEASERADIUS, THICKNESSSMOOTHING, ROCHESMOOTHING;
  float IMPOSEDDISKDRIFT;
  int Adiabatic, Cooling, ViscosityAlpha, FastTransport, Indirect_Term, ExcludeHill;
  int ForcedCircular, Corotating, GuidingCenter, RocheSmoothing, SelfGravity, Evanescent;
  int OpenInner, NonReflecting, SloppyCFL, IsDisk;
  int max_sub;  // substeps one DT may take before it stops with FARGO_ETIMEOUT
  // Radial stripe of a decomposed disk: the rings own_lo .. own_hi-1 are this
  // context's own, the others are ghost rings refreshed from the neighbouring
  // stripes after every substep.  The CFL limit and the disk forces cover the
  // own rings only, and with stripe = 1 the CFL kernel leaves the substep's
  // scalar work to k_stripe_finish, which reads every stripe's partials.
  // A whole disk: own_lo = 0, own_hi = nrad, stripe = 0.
  int own_lo, own_hi, stripe;
  int cfl_tile;  // cells per CFL/force tile (FARGO_CFL_TILE or FARGO_CFL_TILE_SMALL)
  int accurate;  // precision mode: 0 the reference's arithmetic, 1 accurate (FARGO_PRECISION_*)
  // three CUtensorMap (Sigma, v_r, v_theta; 2-D, FARGO_TR_ROW-column boxes)
  // for the transport's TMA staging, or null (NSEC not a multiple of 4, or
  // below 64): then the rows are staged by 16- or 4-byte cp.async copies
  const void* tmap;
  // boundary constants computed on the host as the reference does:
  // pow(Rinf[1], -1.5), pow(Rinf[NRAD-2], -1.5) of NonReflectingBoundary;
  // damping zones and orbital periods of EvanescentBoundary (SideEuler.cu:127-132)
  double nr_pow_in, nr_pow_out;
  float ev_DRMIN, ev_DRMAX, ev_Tin, ev_Tout;
  float invdphi, onethird;
  float HillRadius;
  // constant sub-Keplerian boundary speeds (host double -> float) when they
  // do not depend on time or self-gravity; otherwise computed on device
  int vkep_const;
  float VKepIn, VKepOut;
  // state
  float *dens, *vrad, *vtheta, *energy;
  float *cs;  // per cell (adiabatic); isothermal uses cs_ring
  float *pres;  // isothermal: pressure at the start of the DT's last substep (temperature output)
  // scratch
  float *vri, *vti, *trr, *tpp, *trp, *qplus;
  float *a0, *a1;  // transported density and energy, moved into the state by k_velocities
  float* phi;      // gravitational potential of the substep (k_potential)
  // self-gravity accelerations (NRAD*NSEC), may be null
  float *sg_accr, *sg_acct;
  // ring tables
  const float *Rinf, *Rsup, *Rmed, *Surf, *invRinf, *invSurf, *invRmed, *invdiffRsup, *invdiffRmed;
  const float *dxtheta, *supp_torque, *SigmaMed, *SigmaInf, *EnergyMed, *CoolingTimeMed, *QplusMed;
  const double* pow15;   // pow(Rmed[i], 1.5) from the host (FViscosity)
  const float* star_grad;  // accurate mode: G / (Rmed[i] Rmed[i-1]) (FP64 radii)
  const float *cfl_rdr, *cfl_rdt, *cfl_rmd;  // RN(1/(Rsup-Rinf)), RN(1/dxtheta), RN(1/min of the two)
  float* visc;           // viscosity_array of this substep
  float* cs_ring;        // isothermal sound speed per ring
  float* csmean;         // GLOBAL_bufarray: ring-mean sound speed
  float* vmoy;           // ConditionCFLKernel1D ring mean
  float* ringmin;        // newDT per CFL tile
  int* nshift;           // Nshift per ring of the current substep
  float* tvmed;          // transport: ring-mean v_theta of the current substep
  float* tvconst;        // transport: constant residual per ring
  int* log_nshift;       // [FARGO_MAXLOG][nrad]
  float* lost;           // [nsec] mass through the inner edge this substep (OPEN inner boundary)
  double* partials;      // [4*FARGO_MAXBODY][CFL tiles] force partial sums per tile
  double* log_dt;        // [FARGO_MAXLOG] substep dt of the current DT
  double* rk_work;       // [FARGO_RK_WORK(FARGO_MAXPLANETS_DEV)] RK5 scratch of large systems
  // sector tables
  const float *cos_pot, *sin_pot;    // cosf/sinf of (float)j/(float)nsec*2.0*PI
  const float *cos_cell, *sin_cell;  // cosf/sinf of 2.0*PI*(float)j/(float)nsec
  DiskCtl* ctl;
};

struct BatchDev {
  int ndisk;
  long long ncell;       // total active cells
  int nring;             // total rings
  int ncfl;              // total CFL tiles
  const long long* cell_off;  // [ndisk+1]
  const int* ring_off;        // [ndisk+1]
  DiskDev* disks;
  // transport work items (disk, ring, first sector, sectors), one per CTA,
  // separate lists for isothermal and adiabatic disks
  const int4* theta_iso;
  const int4* theta_adi;
  int ntheta_iso, ntheta_adi;
  int theta_seg;          // largest azimuthal segment (sectors)
  int* flags;             // [0] OR of the disks' "more" flags after a substep
  // compacted lists of the disks inside their DT (rebuilt on the device at the
  // start of a DT and after every substep): act[0] active disks, act[1] active
  // isothermal disks, act[2] active adiabatic disks
  int* act;
  int* act_disk;             // [ndisk] disk id of active index a
  long long* act_cell_off;   // [ndisk+1] prefix of active cells
  int* act_ring_off;         // [ndisk+1] prefix of active rings
  int* act_iso_disk;         // [ndisk] isothermal active disks
  int* act_iso_off;          // [ndisk+1] prefix of their transport items
  int* act_adi_disk;
  int* act_adi_off;
  int* act_grp_off;          // [ndisk+1] prefix of FARGO_RM_RINGS-ring groups of active disks
  int* act_tile_off;         // [ndisk+1] prefix of cell tiles (FARGO_QTILE cells) of active disks
  int* act_ctile_off;        // [ndisk+1] prefix of CFL tiles (FARGO_CFL_TILE cells) of active disks
  int* act_vtile_off;        // [ndisk+1] prefix of viscosity tiles (8 x 64 cells) of active disks
  int cell_grid, ring_grid, item_grid, grp_grid;  // fixed grid sizes of the grid-stride kernels
  int any_bc;                // some disk has an OPEN, NONREFLECTING or EVANESCENT boundary
  int src1_classes;          // bit 2*Adiabatic + SelfGravity set for every kind of disk present
  int accurate;              // precision mode of the batch's disks: which kernel set runs (FARGO_LAUNCHERS)
  int max_body;              // largest body count of the force sums (star + FeelDisk planets)
  // one-wave grids of the substep kernels (fargo_size_grids)
  int g_cfl, g_source1[4], g_potential, g_viscosity, g_source2[2], g_energy, g_velocities[2], g_transport;
};

// kernel entry points (kernels_step.cu), launched by fargo_api.cu
#define FARGO_NKERNELS 14  // profiled slots per substep (boundary slots empty for rigid boundaries)
#define FARGO_SEG_OUT 192  // largest azimuthal transport segment (output sectors per CTA)
#define FARGO_BAND 8       // rings per transport CTA
#define FARGO_RM_RINGS 8   // rings per ring-mean CTA (serial FP32 chain per ring)
#define FARGO_SEG_MAX 244  // widest segment the autotuner may pick: window + 1 = 253 <= FARGO_TR_ROW
// Transport staging: each band's input rows are copied into shared memory as
// rows of FARGO_TR_ROW columns (one TMA box of a 2-D tensor map per field):
// Sigma and v_theta rings i0-2 .. i0+FARGO_BAND+1, v_r rings i0-2 ..
// i0+FARGO_BAND+2.
#define FARGO_TR_ROW 256
#define FARGO_TR_ROWS_D (FARGO_BAND + 4)
#define FARGO_TR_ROWS_R (FARGO_BAND + 5)
#define FARGO_TR_ROWS_T (FARGO_BAND + 4)
// ev (optional): FARGO_NKERNELS+1 events, before each kernel and after the last.
// part: FARGO_PART_HEAD (ring means and CFL/forces), FARGO_PART_TAIL (the
// rest: potential ... end of substep) or both.
#define FARGO_PART_HEAD 1
#define FARGO_PART_TAIL 2
#define FARGO_STRIPE_HEAD 3
// The kernels and their launchers are compiled twice (kernels_step.cu):
// fargo_k with the compiler's contraction of a*b+c into fused multiply-adds
// (the reference-arithmetic precision mode, as the reference's own build)
// and fargo_k_nofma without it (the accurate mode: each product rounded
// before it is added, as the FP64-checked restatement does).  The
// unqualified launchers below pick the set by BatchDev::accurate
// (kernels_dispatch.cu).
#define FARGO_LAUNCHERS                                                                                        \
  cudaError_t fargo_kernel_attributes(int max_nsec);                                                          \
  void fargo_launch_dt_begin(const BatchDev& b, cudaStream_t s);                                              \
  /* only_disk >= 0: that disk; -1: every disk still inside its DT */                                         \
  void fargo_launch_cs_refresh(const BatchDev& b, int only_disk, cudaStream_t s);                             \
  void fargo_launch_cs_isothermal(const BatchDev& b, int only_disk, cudaStream_t s);                          \
  void fargo_launch_substep(const BatchDev& b, cudaGraphConditionalHandle h, int use_handle, cudaStream_t s,   \
                            int max_nsec, long long* launches, cudaEvent_t* ev = nullptr,                     \
                            int part = FARGO_PART_HEAD | FARGO_PART_TAIL);                                     \
  /* radial stripes: the stripe's block for the gather (3 + 4 * bodies * own CFL tiles doubles), and the     \
     substep scalars from the gathered blocks (nonzero return: nstripe out of range) */                       \
  void fargo_launch_stripe_block(const BatchDev& b, double* out, cudaStream_t s);                             \
  int fargo_launch_stripe_finish(const BatchDev& b, const double* blk, int nstripe, int stride, cudaStream_t s); \
  const char* fargo_substep_kernel_name(int k);                                                               \
  void fargo_launch_sector_tables(const BatchDev& b, int max_nsec, cudaStream_t s);                           \
  void fargo_launch_init_velocities(const BatchDev& b, int disk, long long ncell_ghost, cudaStream_t s);      \
  void fargo_launch_disk_force(const BatchDev& b, int disk, float x, float y, float rs, float rh, float a,     \
                               double* out44, int nblocks, cudaStream_t s);                                   \
  void fargo_launch_diagnostics(const BatchDev& b, int disk, double* out3, int nblocks, cudaStream_t s);      \
  int fargo_substep_launches(const BatchDev& b);                                                              \
  cudaError_t fargo_size_grids(BatchDev& b, int nsm, long long ncell_tiles, int nitems);                      \
  const void* fargo_cfl_kernel(int max_body);                                                                 \
  void fargo_launch_transport(const BatchDev& b, cudaStream_t s);
namespace fargo_k {
FARGO_LAUNCHERS
}
namespace fargo_k_nofma {
FARGO_LAUNCHERS
}
FARGO_LAUNCHERS
