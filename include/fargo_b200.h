/*
 * fargo_b200.h -- C ABI of the B200-native FARGO / FARGO_ADSG disk-hydro timestep.
 *
 * The reference (MatiasFloresS/CudaProtoplanetaryDisksFloat) has no library
 * interface: its hot path is the set of host functions that AlgoGas calls,
 * acting on ~60 process-global device arrays.  This header replaces exactly
 * that path.  Every entry point names the reference code it stands in for.
 *
 * Conventions
 *   - Plain C types, caller-owned host buffers (copied in/out), no torch types.
 *   - Every call returns a fargo_status; nothing calls exit().  On error,
 *     fargo_last_error(ctx) returns a one-line description.
 *   - One context = one disk (or one batch of disks) on one CUDA device,
 *     with its own stream.  Contexts are independent; a context must be used
 *     from one host thread at a time.
 *   - Grid fields are ring-major float32, (NRAD+1)*NSEC values, element
 *     [i*NSEC + j] = ring i, sector j; row NRAD is the outer ghost row of the
 *     reference (used by v_r).
 */
#ifndef FARGO_B200_H
#define FARGO_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FARGO_ABI_VERSION 1
#define FARGO_MAXPLANETS 100   /* RungeKutta.cu:4 static arrays of 100 */
#define FARGO_DIMFXY 11        /* Main.cu:71 dimfxy: Hill-cut levels of ComputeForce */
#define FARGO_NOALLOC_MAXRAD 4096 /* largest NRAD of fargo_disk_force_noalloc */
#define FARGO_STRLEN 512
#define FARGO_MAX_SUBSTEPS 100000 /* default substep limit of one DT */

typedef enum fargo_status {
  FARGO_OK = 0,
  FARGO_EINVAL = 1,      /* bad argument or parameter combination          */
  FARGO_ECUDA = 2,       /* CUDA runtime error                             */
  FARGO_ECUFFT = 3,      /* cuFFT error (self-gravity)                     */
  FARGO_ENONFINITE = 4,  /* NaN/Inf or non-positive density detected       */
  FARGO_ETIMEOUT = 5,    /* a bounded device-side wait gave up             */
  FARGO_EOOM = 6,        /* device allocation failed                       */
  FARGO_EIO = 7,         /* file missing / unreadable / unwritable         */
  FARGO_ENODEV = 8       /* no CUDA device, or the kernels are not loaded  */
} fargo_status;

/*
 * Parameters of a run: the .par variables of the reference with the same
 * names and defaults (Param.cuh:9-63 declarations, Interpret.cu:35-95
 * parsing), the switches that ReadVariables derives from them
 * (Interpret.cu:23-31,126-202) and the command-line switches that matter on
 * the hot path (Main.cu:101-174).
 */
typedef struct fargo_params {
  /* numeric .par variables */
  float DT, SIGMA0;
  int NINTERM, NTOT;
  float MASSTAPER;
  int NRAD, NSEC;
  float RMIN, RMAX, THICKNESSSMOOTHING, ROCHESMOOTHING, ASPECTRATIO;
  float VISCOSITY, ALPHAVISCOSITY, SIGMASLOPE, RELEASERADIUS, RELEASEDATE;
  float OMEGAFRAME, IMPOSEDDISKDRIFT, FLARINGINDEX, ECCENTRICITY;
  float CAVITYRADIUS, CAVITYRATIO, CAVITYWIDTH;
  float TRANSITIONRADIUS, TRANSITIONRATIO, TRANSITIONWIDTH, LAMBDADOUBLING;
  float ADIABATICINDEX, COOLINGTIME0;
  /* string .par variables (first token after the key, as sscanf %s reads it) */
  char OUTPUTDIR[FARGO_STRLEN];
  char PLANETCONFIG[FARGO_STRLEN];
  char INNERBOUNDARY[64], LABELADVECTION[64], TRANSPORT[64], RADIALSPACING[64];
  char DISK[64], FRAME[64], OUTERSOURCEMASS[64], WRITEDENSITY[64], WRITEVELOCITY[64];
  char WRITEENERGY[64], WRITETEMPERATURE[64], WRITEQPLUS[64], INDIRECTTERM[64];
  char EXCLUDEHILL[64], SELFGRAVITY[64], CICPLANET[64], FORCEDCIRCULAR[64];
  char ZMPLUS[64], ADIABATIC[64], COOLING[64];
  /* switches derived by ReadVariables (Interpret.cu:126-202); 1 = YES */
  int AdvecteLabel, OuterSourceMass, FastTransport, OpenInner, NonReflecting;
  int Evanescent, LogGrid, IsDisk, Corotating, GuidingCenter;
  int Write_Density, Write_Velocity, Write_Energy, Write_Temperature, Write_DivV;
  int Write_Qplus, Indirect_Term, SelfGravity, SGZeroMode, ZMPluss;
  int Adiabatic, Cooling, ExcludeHill, CICPlanet, ForcedCircular;
  int ViscosityAlpha, RocheSmoothing;
  /* command-line switches (Main.cu:110-174) */
  int SloppyCFL;        /* -c */
  float ScalingFactor;  /* -f */
} fargo_params;

/* Planetary system, FP64 (Types.cuh:2-15 planetary_system). */
typedef struct fargo_planets {
  int nb;
  double mass[FARGO_MAXPLANETS], x[FARGO_MAXPLANETS], y[FARGO_MAXPLANETS];
  double vx[FARGO_MAXPLANETS], vy[FARGO_MAXPLANETS], acc[FARGO_MAXPLANETS];
  int feeldisk[FARGO_MAXPLANETS], feelothers[FARGO_MAXPLANETS];
  char name[FARGO_MAXPLANETS][64];
} fargo_planets;

/* Scalars of the last advanced DT (for logs, bigplanet files and tests). */
typedef struct fargo_scalars {
  float physical_time;      /* PhysicalTime (Viscosity.cu:15), float as in the reference */
  float omega_frame;        /* OmegaFrame */
  float mdcp1;              /* CircumPlanetaryMass of planet 0 (SourceEuler.cu:539-553) */
  float lost_mass;          /* LostMass (TransportEuler.cu:17,71) */
  int nsub_last_dt;         /* hydro substeps taken by the last DT */
  int nsub_total;           /* hydro substeps since fargo_create */
  double mass;              /* FP64 sum of Sigma*Surf over active cells */
  double angular_momentum;  /* FP64 sum of Sigma*Surf*r*(v_theta + r*OmegaFrame) (cell-centred) */
  double last_dt;           /* dt of the last substep */
} fargo_scalars;

typedef struct fargo_ctx fargo_ctx;

/* ---- parameter / configuration handling (host only, no GPU needed) ---- */

/* Reference defaults of every variable (Param.cuh:9-63, Interpret.cu:23-31). */
fargo_status fargo_params_default(fargo_params* p);

/* ReadVariables (Interpret.cu:97-208) + SearchVariable (Interpret.cu:35-95):
   case-insensitive keys, first token as value, unknown keys ignored, the
   same consistency checks (reported as FARGO_EINVAL instead of exit(1)). */
fargo_status fargo_params_read(const char* parfile, fargo_params* p);

/* Re-derive the YES/NO switches from the string variables
   (Interpret.cu:126-202); use after editing strings by hand. */
fargo_status fargo_params_derive(fargo_params* p);

/* InitPlanetarySystem (Psys.cu:159-208) with FindNumberOfPlanets
   (Psys.cu:83-99).  p supplies ECCENTRICITY and the grid for CICPLANET. */
fargo_status fargo_planets_read(const char* cfgfile, const fargo_params* p,
                                fargo_planets* out);

/* FillPolar1DArrays (SourceEuler.cu:76-173): interface radii, NRAD+1 doubles
   (the values written to used_rad.dat) and the float tables used on device. */
fargo_status fargo_grid_radii(const fargo_params* p, double* radii_out /* NRAD+1 */);

/* ---- context lifetime ---- */

/* Everything main() does between ReadVariables and the DT loop
   (Main.cu:198-344): grid tables, initial Sigma/energy/velocities, sound
   speed, pressure, per-ring viscosity, planets; device memory, stream and
   graphs.  radii may be NULL (computed from RMIN/RMAX/RadialSpacing) or
   point to NRAD+1 interface radii (the reference's radii.dat path).
   device < 0 selects the current device. */
fargo_status fargo_create(const fargo_params* p, const fargo_planets* planets,
                          const double* radii, int device, fargo_ctx** out);
void fargo_destroy(fargo_ctx* ctx);
const char* fargo_last_error(const fargo_ctx* ctx);

/* Re-run the initialisation of main() from InitGasDensity on (Main.cu:292-344:
   self-gravity start-up, OmegaFrame, sound speed, viscosity table, initial
   velocities) with the given surface density and energy in place of the
   reference's axisymmetric profiles.  This is where the reference would see
   a perturbed initial density.  dens/energy may be NULL (profiles). */
fargo_status fargo_init_state(fargo_ctx* ctx, const float* dens, const float* energy);

/* Replace the disk state (H2D), e.g. seeded noisy initial conditions.
   Any pointer may be NULL to keep that field.  (Cudamalloc, Main.cu:700-867) */
fargo_status fargo_upload(fargo_ctx* ctx, const float* dens, const float* vrad,
                          const float* vtheta, const float* energy);

/* Read the disk state (D2H).  Any pointer may be NULL.  temperature and
   qplus are the reference's output-only fields (DeviceToHostcudaMemcpy,
   Main.cu:643-654; ComputeTemperatureField, SourceEuler.cu:458-463). */
fargo_status fargo_download(fargo_ctx* ctx, float* dens, float* vrad, float* vtheta,
                            float* energy, float* temperature, float* qplus);

fargo_status fargo_get_planets(fargo_ctx* ctx, fargo_planets* out);
fargo_status fargo_set_planets(fargo_ctx* ctx, const fargo_planets* in);

/* One DT of the hydro loop: the body of AlgoGas (SourceEuler.cu:208-301),
   all CFL substeps, planet kicks and RK5 on the device.  nsub_out (may be
   NULL) receives the number of substeps taken. */
fargo_status fargo_advance_dt(fargo_ctx* ctx, int* nsub_out);

/* ndt DTs back to back without host synchronisation in between (one CUDA
   graph launch per DT), then wait.  Scalars are those of the last DT. */
fargo_status fargo_advance(fargo_ctx* ctx, int ndt);
/* Same without the final wait (pair with fargo_sync). */
fargo_status fargo_advance_async(fargo_ctx* ctx, int ndt);

/* Wait for the context's stream. */
fargo_status fargo_sync(fargo_ctx* ctx);

/* ComputeForce (Force.cu:31-67) as UpdateLog uses it (Force.cu:102):
   disk force on a body at (x,y), all FARGO_DIMFXY Hill-cut levels.
   globalforce[k + m*dimfxy], m = 0 fx_inner, 1 fx_outer, 2 fy_inner,
   3 fy_outer; FP64 sums of the FP32 per-cell forces. */
fargo_status fargo_disk_force(fargo_ctx* ctx, double x, double y, double rsmoothing,
                              double mass, int dimfxy, double* globalforce);

/* compute_selfgravity (SgMain.cu:23-45) on the current density, between
   DTs: the radial and azimuthal self-gravity accelerations SG_Accr, SG_Acct
   (NRAD*NSEC each, host memory), as the next substep would use them.
   FARGO_EINVAL when the run has no self-gravity. */
fargo_status fargo_sg_accelerations(fargo_ctx* ctx, float* accr, float* acct);

/* No counterpart in the reference: fargo_disk_force for callers that keep
   their disk in their own device arrays and must not allocate device memory
   (they manage it themselves, or cannot afford cudaMalloc's device-wide
   synchronisation mid-step).  Allocates nothing: its only scratch is a fixed
   static device array of (FARGO_NOALLOC_MAXRAD + 1) * 44 doubles (1.4 MB,
   held by every GPU that loads the library until exit); NRAD above
   FARGO_NOALLOC_MAXRAD is rejected with FARGO_EINVAL.  Inputs are device
   pointers in the reference's layout: dens, cell_x, cell_y [NRAD*NSEC]
   (Dens, CellAbscissa, CellOrdinate), surf, rmed [NRAD]; globalforce is
   host memory, filled as by fargo_disk_force.  Runs on `stream` (a
   cudaStream_t, NULL for the default stream) on the current device, copies
   the result to globalforce and synchronises that stream before returning.
   The first call on a device looks up the scratch address there: make it
   before any stream capture.  Calls share the scratch, so calls that
   overlap on the GPU race.  A CUDA error already pending when the call
   starts is reported (FARGO_ECUDA) and left pending.  err/errlen (may be
   NULL/0) receive a message on failure. */
fargo_status fargo_disk_force_noalloc(const float* dens, const float* cell_x, const float* cell_y,
                                      const float* surf, const float* rmed, int nrad, int nsec,
                                      double x, double y, double rsmoothing, double mass,
                                      int dimfxy, double* globalforce, void* stream, char* err,
                                      int errlen);

/* Checkpoint / restart (new: the reference parses -s N, Main.cu:147-155, but
   never restores a state).  A checkpoint is the device state a later DT
   reads: control block (time, frame, planets in FP64), fields with their
   ghost rows and the per-ring sound speed and viscosity.  Save and load
   between DTs; loading into a context of the same grid and build continues
   the run bit for bit. */
size_t fargo_checkpoint_bytes(fargo_ctx* ctx);
fargo_status fargo_checkpoint_save(fargo_ctx* ctx, void* buf, size_t bytes);
fargo_status fargo_checkpoint_load(fargo_ctx* ctx, const void* buf, size_t bytes);

/* Scalars after the last DT (also recomputes mdcp1, mass, angular momentum). */
fargo_status fargo_get_scalars(fargo_ctx* ctx, fargo_scalars* out);

/* Per-substep record of the last DT, for bit-exact parity checks:
   nshift[s*NRAD + i] = FARGO integer shift of ring i in substep s
   (ComputeConstantResidualKernel, Kernels.cu:1218-1221), dt[s] = substep dt.
   cap = room in substeps; *nsub receives the count. */
fargo_status fargo_get_substep_log(fargo_ctx* ctx, int cap, int* nshift, double* dt, int* nsub);

/* ---- batched form: many independent disks, one launch per kernel ---- */

/* n contexts' worth of disks in one batch (different NRAD/NSEC/parameters).
   Each disk keeps its own CFL substep sequence; one fargo_batch_advance_dt
   advances every disk by its own DT. */
typedef struct fargo_batch fargo_batch;
fargo_status fargo_batch_create(int n, const fargo_params* params, const fargo_planets* planets,
                                int device, fargo_batch** out);
void fargo_batch_destroy(fargo_batch* b);
const char* fargo_batch_last_error(const fargo_batch* b);
fargo_status fargo_batch_upload(fargo_batch* b, int disk, const float* dens, const float* vrad,
                                const float* vtheta, const float* energy);
fargo_status fargo_batch_download(fargo_batch* b, int disk, float* dens, float* vrad,
                                  float* vtheta, float* energy);
fargo_status fargo_batch_init_state(fargo_batch* b, int disk, const float* dens, const float* energy);
fargo_status fargo_batch_advance(fargo_batch* b, int ndt);
fargo_status fargo_batch_advance_async(fargo_batch* b, int ndt);
fargo_status fargo_batch_sync(fargo_batch* b);
fargo_status fargo_batch_get_scalars(fargo_batch* b, int disk, fargo_scalars* out);
fargo_status fargo_batch_get_planets(fargo_batch* b, int disk, fargo_planets* out);

/* Library facts for tests and tools. */
int fargo_abi_version(void);
/* Kernel launches of this library on the context outside the DT graph. */
long long fargo_kernel_launches(const fargo_ctx* ctx);
/* All kernel launches of this library on the batch since creation,
   including those inside the DT graphs (substeps x kernels per substep). */
long long fargo_batch_count_launches(fargo_batch* b);
long long fargo_batch_kernel_launches(const fargo_batch* b);
/* The CUDA stream (cudaStream_t) every call of the context/batch uses, so a
   caller can order its own work or record timing events on it. */
void* fargo_stream(fargo_ctx* ctx);
void* fargo_batch_stream(fargo_batch* b);
/* The one-disk batch inside a context (to use the batch calls on it). */
fargo_batch* fargo_ctx_batch(fargo_ctx* ctx);
/* Copies without the final wait; host buffers must stay valid until
   fargo_batch_sync (page-locked buffers let them overlap). */
fargo_status fargo_batch_upload_async(fargo_batch* b, int disk, const float* dens, const float* vrad,
                                      const float* vtheta, const float* energy);
fargo_status fargo_batch_download_async(fargo_batch* b, int disk, float* dens, float* vrad,
                                        float* vtheta, float* energy);
/* Per-kernel device time of ndt DTs run with one CUDA event pair per kernel
   launch (host loop over substeps): ms[k] for the fargo_profile_kernel_count()
   slots named by fargo_profile_kernel_name(k): the substep kernels in launch
   order, then the self-gravity pipeline. */
fargo_status fargo_batch_profile(fargo_batch* b, int ndt, double* ms /* >= 16 */, int* nsub);
int fargo_profile_kernel_count(void);
const char* fargo_profile_kernel_name(int k);
/* 1 (default): one CUDA graph launch per DT with a device-driven WHILE node
   over the substeps; 0: host loop with one wait per substep. */
fargo_status fargo_set_graph_mode(fargo_ctx* ctx, int use_graph);
fargo_status fargo_batch_set_graph_mode(fargo_batch* b, int use_graph);
/* (new) Largest number of CFL substeps one DT may take (default
   FARGO_MAX_SUBSTEPS).  A DT that needs more stops after that many substeps
   and fargo_advance* return FARGO_ETIMEOUT; the context stays usable (upload
   a state and advance again).  A NaN or Inf in the density, velocities or
   sound speed (checked on every cell by the CFL kernel at the start of each
   substep), or a CFL step that is not positive, stops the DT in the same
   way with FARGO_ENONFINITE.  Call between DTs. */
fargo_status fargo_set_max_substeps(fargo_ctx* ctx, int n);
fargo_status fargo_batch_set_max_substeps(fargo_batch* b, int n);
/* (new) Precision mode of every disk of the context / batch.
   FARGO_PRECISION_REFERENCE (default): the reference's FP32 arithmetic, so
   that substep counts, every dt and every FARGO shift match its build bit
   for bit.  FARGO_PRECISION_ACCURATE: closer to an FP64 run of the same
   algorithm, at the same FP32 storage:
   - the star's potential -G/r is left out of the stored potential and its
     radial difference quotient enters Substep1 (SourceEuler.cu:305-335,
     Kernels.cu:52-70) as G/(Rmed[i] Rmed[i-1]) from the FP64 radii: the
     reference differences two FP32 values of -G/r ~ 1 across a ring
     spacing of ~1%, which costs ~1e-5 of the radial gravity each substep;
   - ring means (FARGO VMed, CFL mean, alpha-viscosity sound speed) are
     Kahan-compensated FP32 sums in the same order;
   - the self-gravity kernel is tabulated in FP64 (the reference's float
     table is not exactly antisymmetric in azimuth);
   - the step kernels run as a second build without contraction of a*b+c
     into fused multiply-adds (every product rounded before it is added).
   Integer outcomes may then differ from the reference's build.  Call
   between DTs, before the first one for a reproducible run. */
#define FARGO_PRECISION_REFERENCE 0
#define FARGO_PRECISION_ACCURATE 1
fargo_status fargo_set_precision(fargo_ctx* ctx, int mode);
fargo_status fargo_batch_set_precision(fargo_batch* b, int mode);
/* (new) Tile autotuner: times the transport kernels on the current state for
   azimuthal segment widths 96..244 sectors, first one width for every disk,
   then each class of disk (NSEC, adiabatic, precision mode; largest share of
   cells first) in turn with the others fixed, and keeps the fastest.
   *seg_out: the width of the class with the most cells.  The widths are kept
   for the life of the process per class: batches created later (and a change
   of precision mode) start from them.  Results do not depend on the widths.
   Call between DTs; the state is not advanced.  fargo_batch_segments gives
   each disk's width (cap entries). */
fargo_status fargo_batch_autotune(fargo_batch* b, int reps, int* seg_out);
fargo_status fargo_autotune(fargo_ctx* ctx, int reps, int* seg_out);
fargo_status fargo_batch_segments(fargo_batch* b, int cap, int* seg_per_disk);

/* (new) Radial decomposition of one disk over several contexts, usually one
   per GPU (the loop of AlgoGas, SourceEuler.cu:208-301, split by rings).
   A stripe owns the rings [ring_lo, ring_hi) of the whole disk (p->NRAD
   rings on `radii`, NRAD+1 values, or on fargo_grid_radii(p) when null) and
   computes `ghost` more rings on each side (fewer at the disk's edges) as a
   disk of its own.  One DT, driven by the caller:
     fargo_stripe_dt_begin
     do {
       [self-gravity: fargo_stripe_sg_rows(rows) -> gather every stripe's
        rows in stripe order -> fargo_stripe_sg_apply(gathered): the whole
        disk's convolution on the whole density, this stripe's rings of it]
       fargo_stripe_forces(block)       CFL minimum and force partials of the
                                        own rings -> this stripe's block
       gather every stripe's block, in stripe order, each `stride` doubles
       fargo_stripe_substep(blocks)     the substep's scalars from all blocks
                                        (the same on every stripe), then the
                                        rest of the substep
       fargo_stripe_halo_pack(lo, hi)   own edge rings -> send buffers
       fargo_stripe_more(&more)         waits; more = another substep follows
       send lo to the stripe below, hi to the stripe above, receive theirs
       fargo_stripe_halo_unpack(lo, hi) received rings -> ghost rings
     } while (more)
   With every stripe boundary a multiple of 4096 / gcd(NSEC, 4096) rings
   (whole CFL tiles) and ghost >= FARGO_STRIPE_GHOST, the own rings end
   every substep with the bits of the undecomposed disk: the tiles and the
   finishing sums are the same, and the cut edges' boundary treatment
   reaches fewer than FARGO_STRIPE_GHOST rings into the ghosts in one
   substep (4 to 5 rings, measured).  Stripes need RIGID boundaries
   (FARGO_EINVAL otherwise), at least `ghost` own rings each, and the same
   parameters, radii and planets.  Self-gravity couples every ring: each
   stripe runs the whole disk's log-polar convolution on the whole density,
   gathered from the stripes' own rings before every substep, and keeps its
   own rings' accelerations; the result stays bit-identical to the whole
   disk's.  Start with fargo_stripe_init_state (the whole grid's arrays; the
   stripe takes its rings, a self-gravitating one the whole density too) or
   upload the stripe's rings base .. base+nrad (the local grid, ghost row
   included) with fargo_upload, then exchange halos once before the first
   DT.  fargo_advance*, the CUDA graph and fargo_sg_accelerations are not
   available on a stripe. */
#define FARGO_STRIPE_GHOST 8
#define FARGO_STRIPE_MAX_GHOST 64
typedef struct {
  int base;        /* whole-disk ring of the stripe's local ring 0 */
  int nrad, nsec;  /* local grid: nrad rings (ghosts included) */
  int own_lo, own_hi;      /* own rings, local indices */
  int ghost_lo, ghost_hi;  /* ghost rings below / above (0 at the disk's edges) */
  int nfields;             /* fields in a halo: Sigma, v_r, v_theta (+ energy) */
  int halo_floats_lo, halo_floats_hi;  /* floats of each side's halo buffer */
  int block_doubles;       /* doubles of this stripe's block (the stride must
                              be at least the largest over the stripes) */
} fargo_stripe_layout;
fargo_status fargo_stripe_create(const fargo_params* p, const fargo_planets* planets, const double* radii,
                                 int ring_lo, int ring_hi, int ghost, int device, fargo_ctx** out);
fargo_status fargo_stripe_info(fargo_ctx* ctx, fargo_stripe_layout* out);
/* dens / energy: (NRAD+1)*NSEC host arrays of the whole grid, or NULL for
   the reference's profiles (as fargo_init_state) */
fargo_status fargo_stripe_init_state(fargo_ctx* ctx, const float* dens, const float* energy);
/* self-gravity: the density of the own rings -> out ((own_hi-own_lo)*NSEC
   floats, device); the gathered rows of every stripe (stripe k's at
   gathered + k*stride, its rings cuts[k] .. cuts[k+1]-1; cuts: host array of
   nstripe+1 rings) -> the whole disk's convolution, this stripe's rings of
   it.  Asynchronous on the stripe's stream. */
fargo_status fargo_stripe_sg_rows(fargo_ctx* ctx, float* out);
fargo_status fargo_stripe_sg_apply(fargo_ctx* ctx, const float* gathered, int nstripe, int stride,
                                   const int* cuts);
fargo_status fargo_stripe_dt_begin(fargo_ctx* ctx);
/* device pointers; the calls are asynchronous on the context's stream
   (fargo_stream) except fargo_stripe_more */
fargo_status fargo_stripe_forces(fargo_ctx* ctx, double* block);
fargo_status fargo_stripe_substep(fargo_ctx* ctx, const double* blocks, int nstripe, int stride);
fargo_status fargo_stripe_halo_pack(fargo_ctx* ctx, float* lo, float* hi);
fargo_status fargo_stripe_halo_unpack(fargo_ctx* ctx, const float* lo, const float* hi);
/* waits for the stripe's stream; at the end of the DT (more = 0) reports
   its errors as fargo_advance_dt does */
fargo_status fargo_stripe_more(fargo_ctx* ctx, int* more);

#ifdef __cplusplus
}
#endif

#endif /* FARGO_B200_H */
