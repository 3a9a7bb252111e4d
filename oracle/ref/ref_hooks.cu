/*
 * Link-level hooks around the reference's own code, used only to make the
 * reference produce golden data (test infrastructure).  oracle/ref/Makefile.ref
 * compiles the reference sources unmodified; in Main.cu it maps the names
 * InitGasDensity and AlgoGas, and in SourceEuler.cu the name Transport, to the
 * functions below with -D, and each of them calls the reference's real
 * function.  None of them changes the reference's arithmetic.
 *
 * Environment:
 *   FARGO_REF_NOISE_SEED  seed of the multiplicative density noise applied
 *                         right after InitGasDensity (Main.cu:292):
 *                         Sigma *= 1 + FARGO_REF_NOISE_AMP * u, u in [-1, 1)
 *                         from splitmix64 (same generator as the tests).
 *   FARGO_REF_NOISE_AMP   noise amplitude (default 1e-3).
 *   FARGO_REF_DUMP        path prefix: <prefix>nshift.bin gets, per hydro
 *                         substep, the substep dt (double) and Nshift[NRAD]
 *                         (int32) right after Transport (a device-to-host
 *                         copy and a file write per substep: golden data
 *                         only, never in a timed run); <prefix>algogas.txt
 *                         gets the line of every AlgoGas call (below).
 *   FARGO_REF_TIMES       file that gets, for every AlgoGas call, the line
 *                         "<iteration> <wall seconds> <substeps>".  The
 *                         substep count is a host counter that the Transport
 *                         hook increments (one Transport call per substep):
 *                         no device copy and no I/O inside AlgoGas, so the
 *                         timed call is the reference's own.
 */
#include "Main.cuh"
#include <time.h>
#include <stdint.h>

extern int NRAD, NSEC;
extern int* Nshift_d;

__host__ void fargo_hook_InitGasDensity(float* Dens);
__host__ void fargo_hook_AlgoGas(Force* force, float* Dens, float* Vrad, float* Vtheta, float* Energy,
                                 float* Label, PlanetarySystem* sys, int iteracion);
__host__ void fargo_hook_Transport(float* Dens, float* Vrad, float* Vtheta, float* Energy, float* Label,
                                   float dt);

static uint64_t splitmix64_next(uint64_t* s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

__host__ void fargo_hook_InitGasDensity(float* Dens) {
  InitGasDensity(Dens);
  const char* seed = getenv("FARGO_REF_NOISE_SEED");
  if (!seed) return;
  const char* amps = getenv("FARGO_REF_NOISE_AMP");
  float amp = amps ? (float)atof(amps) : 1e-3f;
  uint64_t s = strtoull(seed, NULL, 10);
  for (int i = 0; i < NRAD; i++)
    for (int j = 0; j < NSEC; j++) {
      uint64_t x = splitmix64_next(&s);
      float u = (float)((x >> 40) & 0xFFFFFFULL) / 8388608.0f - 1.0f;
      float f = 1.0f + amp * u;
      Dens[i * NSEC + j] = Dens[i * NSEC + j] * f;
    }
}

static FILE* dump_file(const char* suffix, const char* mode) {
  const char* pre = getenv("FARGO_REF_DUMP");
  if (!pre) return NULL;
  char name[1024];
  snprintf(name, sizeof(name), "%s%s", pre, suffix);
  return fopen(name, mode);
}

static long transport_calls = 0;

__host__ void fargo_hook_Transport(float* Dens, float* Vrad, float* Vtheta, float* Energy, float* Label,
                                   float dt) {
  Transport(Dens, Vrad, Vtheta, Energy, Label, dt);
  transport_calls++;
  static FILE* f = NULL;
  static int opened = 0;
  if (!opened) {
    f = dump_file("nshift.bin", "wb");
    opened = 1;
  }
  if (!f) return;
  int* ns = (int*)malloc(sizeof(int) * NRAD);
  cudaMemcpy(ns, Nshift_d, sizeof(int) * NRAD, cudaMemcpyDeviceToHost);
  double d = dt;
  fwrite(&d, sizeof(double), 1, f);
  fwrite(ns, sizeof(int), NRAD, f);
  fflush(f);
  free(ns);
}

__host__ void fargo_hook_AlgoGas(Force* force, float* Dens, float* Vrad, float* Vtheta, float* Energy,
                                 float* Label, PlanetarySystem* sys, int iteracion) {
  static FILE* f = NULL;
  static int opened = 0;
  if (!opened) {
    const char* times = getenv("FARGO_REF_TIMES");
    f = times ? fopen(times, "w") : dump_file("algogas.txt", "w");
    opened = 1;
  }
  long calls0 = transport_calls;
  cudaDeviceSynchronize();
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  AlgoGas(force, Dens, Vrad, Vtheta, Energy, Label, sys, iteracion);
  cudaDeviceSynchronize();
  clock_gettime(CLOCK_MONOTONIC, &t1);
  double s = (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
  if (f) {
    fprintf(f, "%d %.9f %ld\n", iteracion, s, transport_calls - calls0);
    fflush(f);
  }
}
