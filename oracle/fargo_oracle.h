/*
 * fargo_oracle.h -- CPU restatement of the reference's hydro timestep.
 *
 * TEST INFRASTRUCTURE ONLY.  This code is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it.  The product never links, imports or calls it.
 *
 * Two builds of the same source:
 *   liboracle_f32.so  -- every float of the reference is a float and every
 *                        double literal promotes as in the reference's
 *                        FP32 build (the parity oracle);
 *   liboracle_f64.so  -- every float becomes a double (the FP64 reference
 *                        against which per-field errors are stated).
 *
 * Pinning: the f32 build is checked against outputs of the reference's own
 * CUDA build (compiled from its unmodified sources by oracle/Makefile.ref and
 * run on a B200), committed under tests/golden/ with the script that made them.
 */
#ifndef FARGO_ORACLE_H
#define FARGO_ORACLE_H

#include "../include/fargo_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc;

/* Setup as main() does it (Main.cu:198-344).  radii may be NULL. */
int orc_create(const fargo_params* p, const fargo_planets* planets, const double* radii, orc** out);
void orc_destroy(orc* o);
/* Re-run the initialisation from InitGasDensity on (Main.cu:292-344) with a
   perturbed density / energy (float32, (NRAD+1)*NSEC; NULL = profile). */
void orc_init_state(orc* o, const float* dens, const float* energy);

/* Element size of the grid fields of this build (4 or 8). */
int orc_real_size(void);

/* State access; buffers hold (NRAD+1)*NSEC values of the build's real type.
   NULL pointers are skipped. */
void orc_set_fields(orc* o, const void* dens, const void* vrad, const void* vtheta, const void* energy);
void orc_get_fields(const orc* o, void* dens, void* vrad, void* vtheta, void* energy,
                    void* temperature, void* qplus);
/* Same, converting to/from float32. */
void orc_set_fields_f32(orc* o, const float* dens, const float* vrad, const float* vtheta,
                        const float* energy);
void orc_get_fields_f32(const orc* o, float* dens, float* vrad, float* vtheta, float* energy,
                        float* temperature, float* qplus);

/* SG_Accr / SG_Acct of the current density (NRAD*NSEC each, in the
   build's precision widened to double); -1 without self-gravity. */
int orc_sg_accelerations(orc* o, double* accr, double* acct);
/* 0: the reference's arithmetic (default); 1: accurate mode (FP64 star
   potential gradient, Kahan ring means, FP64 self-gravity kernel table). */
void orc_set_precision(orc* o, int mode);
void orc_get_planets(const orc* o, fargo_planets* out);
void orc_set_planets(orc* o, const fargo_planets* in);

/* One AlgoGas call (SourceEuler.cu:208-301); returns the substep count. */
int orc_advance_dt(orc* o);

/* Per-substep log of the last DT: nshift[s*NRAD+i], dt[s]. Returns count. */
int orc_substep_log(const orc* o, int cap, int* nshift, double* dt);

/* ComputeForce (Force.cu:31-67): globalforce[k + m*dimfxy]. */
void orc_disk_force(orc* o, double x, double y, double rsmoothing, double mass, int dimfxy,
                    double* globalforce);

/* Scalars after the last DT (same meaning as fargo_scalars). */
void orc_get_scalars(orc* o, fargo_scalars* out);

/* Grid tables (float or double per build), NRAD+1 values each.
   which: 0 Radii 1 Rinf 2 Rsup 3 Rmed 4 Surf 5 invRinf 6 invSurf 7 invRmed
          8 invdiffRsup 9 invdiffRmed 10 SigmaMed 11 SigmaInf 12 EnergyMed
          13 viscosity_array 14 SoundSpeed ring 0.. (per ring, first sector) */
void orc_get_table(const orc* o, int which, double* out);

/* OpenMP threads used by the oracle loops (0 = leave the default). */
void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif

#endif
