// fargo_main.cpp -- drop-in replacement of the reference's bin/fargoGPU.
//
// Same command line (Main.cu:108-182), same .par/.cfg reading, same output
// files (Output.cu, Force.cu:76-138, SourceEuler.cu:159-171), with the hot
// path (AlgoGas) running through the C ABI of libfargo_b200.so.  Output
// formats are kept byte-compatible on purpose, so the reference's
// post-processing (plot2d.py and friends) reads them unchanged.
//
// Two additions: every output also writes checkpointN.bin (the device state,
// fargo_checkpoint_save), so that -s N, which the reference parses but never
// acts on, restarts from output N and continues the run bit for bit; and
// output files are written by a writer thread while the next DTs run (the
// console messages stay in the reference's order, printed by the main
// thread).
#include <sys/stat.h>
#include <sys/types.h>

#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fargo_b200.h"

#define PI 3.14159265358979323844

static void usage(const char* exe) {
  std::printf("Usage : %s [-abcdeimnptvz] [-(0-9)] [-s number] [-f scaling] parameters file\n", exe);
  std::printf("\n-a : Monitor mass and angular momentum at each timestep\n");
  std::printf("-b : Adjust azimuthal velocity to impose strict centrifugal balance at t=0\n");
  std::printf("-c : Sloppy CFL condition (checked at each DT, not at each timestep)\n");
  std::printf("-d : Print some debugging information on 'stdout' at each timestep\n");
  std::printf("-e : Activate EU test problem torque file output\n");
  std::printf("-f : Scale density array by 'scaling'. Useful to increase/decrease\n");
  std::printf("     disk surface density after a restart, for instance.            \n");
  std::printf("-i : tabulate Sigma profile as given by restart files\n");
  std::printf("-m : Merge output files from different CPUs\n");
  std::printf("-n : Disable simulation. The program just reads parameters file\n");
  std::printf("-o : Overrides output directory of input file.\n");
  std::printf("-p : Give profiling information at each time step\n");
  std::printf("-s : Restart simulation, taking #'number' files as initial conditions\n");
  std::printf("-t : Monitor CPU time usage at each time step\n");
  std::printf("-v : Verbose mode. Tells everything about parameters file\n");
  std::printf("-z : fake sequential built when evaluating sums on HD meshes\n");
  std::printf("-(0-9) : only write initial (or restart) HD meshes,\n");
  std::printf("     proceed to the next nth output and exit\n");
  std::printf("     This option must stand alone on one switch (-va -4 is legal, -v4a is not)\n");
  std::exit(1);
}

// TellNbOrbits / TellNbOutputs / TellEverything (Interpret.cu:235-306)
static float nb_orbits(float time) { return time / 2.0 / PI * std::sqrt(1.0 * 1.0 / 1.0 / 1.0 / 1.0); }
static float nb_outputs(const fargo_params& p, float time) { return (time / p.DT / p.NINTERM); }

static void tell_everything(const fargo_params& p) {
  float temp, nbfileoutput;
  float RMIN = p.RMIN, RMAX = p.RMAX, SIGMA0 = p.SIGMA0, SIGMASLOPE = p.SIGMASLOPE, AR = p.ASPECTRATIO;
  std::printf("\nDisc properties:\n");
  std::printf("----------------\n");
  std::printf("Inner Radius          : %g\n", RMIN);
  std::printf("Outer Radius          : %g\n", RMAX);
  std::printf("Aspect Ratio          : %g\n", AR);
  std::printf("VKep at inner edge    : %.3g\n", std::sqrt(1.0 * 1.0 * (1. - 0.0) / RMIN));
  std::printf("VKep at outer edge    : %.3g\n", std::sqrt(1.0 * 1.0 / RMAX));
  temp = 2.0 * PI * SIGMA0 / (2.0 - SIGMASLOPE) * (std::pow(RMAX, 2.0 - SIGMASLOPE) - std::pow(RMIN, 2.0 - SIGMASLOPE));
  std::printf("Initial Disk Mass             : %g\n", temp);
  temp = 2.0 * PI * SIGMA0 / (2.0 - SIGMASLOPE) * (1.0 - std::pow(RMIN, 2.0 - SIGMASLOPE));
  std::printf("Initial Mass inner to r=1.0  : %g \n", temp);
  temp = 2.0 * PI * SIGMA0 / (2.0 - SIGMASLOPE) * (std::pow(RMAX, 2.0 - SIGMASLOPE) - 1.0);
  std::printf("Initial Mass outer to r=1.0  : %g \n", temp);
  std::printf("Travelling time for acoustic density waves :\n");
  temp = 2.0 / 3.0 / AR * (std::pow(RMAX, 1.5) - std::pow(RMIN, 1.5));
  std::printf(" * From Rmin to Rmax  : %.2g = %.2f orbits ~ %.1f outputs\n", temp, nb_orbits(temp), nb_outputs(p, temp));
  temp = 2.0 / 3.0 / AR * (std::pow(RMAX, 1.5) - std::pow(1.0, 1.5));
  std::printf(" * From r=1.0 to Rmax: %.2g = %.2f orbits ~ %.1f outputs\n", temp, nb_orbits(temp), nb_outputs(p, temp));
  temp = 2.0 / 3.0 / AR * (std::pow(1.0, 1.5) - std::pow(RMIN, 1.5));
  std::printf(" * From r=1.0 to Rmin: %.2g = %.2f orbits ~ %.1f outputs\n", temp, nb_orbits(temp), nb_outputs(p, temp));
  temp = 2.0 * PI * std::sqrt(RMIN * RMIN * RMIN / 1.0 / 1.0);
  std::printf("Orbital time at Rmin  : %.3g ~ %.2f outputs\n", temp, nb_outputs(p, temp));
  temp = 2.0 * PI * std::sqrt(RMAX * RMAX * RMAX / 1.0 / 1.0);
  std::printf("Orbital time at Rmax  : %.3g ~ %.2f outputs\n", temp, nb_outputs(p, temp));
  std::printf("Sound speed :\n");
  std::printf(" * At unit radius     : %.3g\n", AR * std::sqrt(1.0 * 1.0));
  std::printf(" * At outer edge      : %.3g\n", AR * std::sqrt(1.0 * 1.0 / RMAX));
  std::printf(" * At inner edge      : %.3g\n", AR * std::sqrt(1.0 * 1.0 / RMIN));
  std::printf("\nGrid properties:\n");
  std::printf("----------------\n");
  std::printf("Number of rings       : %d\n", p.NRAD);
  std::printf("Number of sectors     : %d\n", p.NSEC);
  std::printf("Total cells           : %d\n", p.NRAD * p.NSEC);
  std::printf("\nOutputs properties:\n");
  std::printf("-------------------\n");
  std::printf("Time increment between outputs : %.3f = %.3f orbits\n", p.NINTERM * p.DT, nb_orbits(p.NINTERM * p.DT));
  std::printf("At each output #i, the following files are written:\n");
  std::printf("gasdens[i].dat : %d bytes\n", (int)(p.NRAD * p.NSEC * sizeof(float)));
  std::printf("gasvrad[i].dat : %d bytes\n", (int)(p.NRAD * p.NSEC * sizeof(float)));
  std::printf("gasvtheta[i].dat : %d bytes\n", (int)(p.NRAD * p.NSEC * sizeof(float)));
  if (p.Adiabatic) std::printf("gasTemperature[i].dat : %d bytes\n", (int)(p.NRAD * p.NSEC * sizeof(float)));
  if (p.AdvecteLabel) std::printf("gaslabel[i].dat : %d bytes\n", (int)(p.NRAD * p.NSEC * sizeof(float)));
  std::printf("There will be in total %d outputs\n", p.NTOT / p.NINTERM);
  std::printf("(which correspond to an elapsed time = %.3f or to %.2f orbits)\n", p.NTOT * p.DT, nb_orbits(p.NTOT * p.DT));
  nbfileoutput = 3.0;
  if (p.Adiabatic) nbfileoutput += 1.0;
  if (p.AdvecteLabel) nbfileoutput += 1.0;
  temp = nbfileoutput * p.NRAD * p.NSEC * sizeof(float);
  temp *= (float)p.NTOT / (float)p.NINTERM;
  temp /= 1024.0 * 1024.0;
  std::printf("So the code will produce ~%.2f Mbytes of data\n", temp);
  std::printf("Check (eg by issuing a 'df' command) that you have enough disk space,\n");
  std::printf("otherwise you will get a system full and the code will stop.\n");
  std::fflush(stdout);
}

static void die(fargo_ctx* ctx, fargo_status st, const char* what) {
  std::fprintf(stderr, "%s failed (status %d): %s\n", what, (int)st, ctx ? fargo_last_error(ctx) : "");
  std::exit(1);
}

// Output files are written here, in order, while the main thread advances.
class Writer {
 public:
  Writer() : t_([this] { loop(); }) {}
  ~Writer() {
    {
      std::lock_guard<std::mutex> lk(m_);
      done_ = true;
    }
    cv_.notify_one();
    t_.join();
  }
  void push(std::function<void()> job) {
    {
      std::lock_guard<std::mutex> lk(m_);
      q_.push_back(std::move(job));
    }
    cv_.notify_one();
  }

 private:
  void loop() {
    for (;;) {
      std::function<void()> job;
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [this] { return done_ || !q_.empty(); });
        if (q_.empty()) return;
        job = std::move(q_.front());
        q_.pop_front();
      }
      job();
    }
  }
  std::mutex m_;
  std::condition_variable cv_;
  std::deque<std::function<void()>> q_;
  bool done_ = false;
  std::thread t_;
};

static void write_file(const std::string& fn, const void* data, size_t bytes) {
  FILE* f = std::fopen(fn.c_str(), "wb");
  if (!f) {
    std::fprintf(stderr, "Unable to open '%s'\n", fn.c_str());
    std::exit(1);
  }
  std::fwrite(data, 1, bytes, f);
  std::fclose(f);
}

// WriteDiskPolar, Output.cu:104-135: the message now, the file by the writer
static void write_disk_polar(Writer& w, const std::string& outdir, const std::vector<float>& a, const char* name,
                             int number, int nrad, int nsec) {
  std::string url = outdir + name;
  struct stat st;
  if (stat(url.c_str(), &st) == -1) mkdir(url.c_str(), 0700);
  char fn[1024];
  std::snprintf(fn, sizeof(fn), "%s%s/%s%d.dat", outdir.c_str(), name, name, number);
  std::printf("Writting '%s%d.dat'... ", name, number);
  auto copy = std::make_shared<std::vector<float>>(a.begin(), a.begin() + (size_t)nrad * nsec);
  std::string path = fn;
  w.push([copy, path] { write_file(path, copy->data(), copy->size() * sizeof(float)); });
  std::printf("done\n");
}

int main(int argc, char** argv) {
  int disable = 0, verbose = 0, sloppy = 0, restart = 0, overrides = 0, nb_restart = 0;
  float scaling = 1.0f;
  char parfile[1024] = "";
  std::string newout;
  if (argc == 1) usage(argv[0]);
  for (int i = 1; i < argc; i++) {
    if (argv[i][0] == '-') {
      if (std::strspn(argv[i], "-secndovtpfamzib0123456789") != std::strlen(argv[i])) usage(argv[0]);
      if (std::strchr(argv[i], 'n')) disable = 1;
      if (std::strchr(argv[i], 'v')) verbose = 1;
      if (std::strchr(argv[i], 'c')) sloppy = 1;
      if (std::strchr(argv[i], 's')) {
        restart = 1;
        i++;
        if (i >= argc || std::atoi(argv[i]) < 0) {
          std::printf("Incorrect restart number\n");
          usage(argv[0]);
        }
        nb_restart = std::atoi(argv[i]);
      }
      if (std::strchr(argv[i], 'o')) {
        overrides = 1;
        i++;
        if (i < argc) newout = argv[i];
      } else if (std::strchr(argv[i], 'f')) {
        i++;
        scaling = (i < argc) ? (float)std::atof(argv[i]) : 0.0f;
        std::printf("Scaling factor = %g\n", scaling);
        if (scaling <= 0) {
          std::printf("Incorrect scaling factor\n");
          usage(argv[0]);
        }
      }
    } else {
      std::snprintf(parfile, sizeof(parfile), "%s", argv[i]);
    }
  }
  if (parfile[0] == 0) usage(argv[0]);
  fargo_params p;
  fargo_status st = fargo_params_read(parfile, &p);
  if (st == FARGO_EIO) {
    std::printf("Unable to read %s . Program stopped. \n", parfile);
    return 1;
  }
  // the messages and checks of ReadVariables, in its order (Interpret.cu:152-201)
  if (std::strcmp(p.ZMPLUS, "YES") == 0 && !p.SGZeroMode)
    std::printf("This is not very meaningfull to involve the anisotropic pressure model (ZMPluss=Yes) \
      without taking into account the axisymmetric component of the disk self-gravity. I decided to \
      put ZMPluss = No. Please check again!");
  if (std::strcmp(p.ADIABATIC, "YES") == 0 && p.ADIABATICINDEX == 1.0f)
    std::printf("You cannot have Adiabatic = YES and AdiabatcIndex = 1. I decided to put Adiabatic = No,\
       to simulate a locally isothermal equation of state. Please check that it what you really wanted to do!\n");
  if (p.ALPHAVISCOSITY != 0.0f && p.VISCOSITY != 0.0f) {
    std::printf("You cannot use at the same time\n");
    std::printf("VISCOSITY and ALPHAVISCOSITY.\n");
    std::printf("Edit the parameter file so as to remove\n");
    std::printf("one of these variables and run again.\n");
    return 1;
  }
  if (p.ALPHAVISCOSITY != 0.0f) std::printf("Viscosity is of alpha type\n");
  if (p.THICKNESSSMOOTHING != 0.0f && p.ROCHESMOOTHING != 0.0f) {
    std::printf("You cannot use at the same time\n");
    std::printf("ThicknessSmoothing and RocheSmoothing.\n");
    std::printf("Edit the parameter file so as to remove\n");
    std::printf("one of these variables and run again.\n");
    return 1;
  }
  if (p.THICKNESSSMOOTHING <= 0.0f && p.ROCHESMOOTHING <= 0.0f) {
    std::printf("A non-vanishing potential smoothing length is required.\n");
    std::printf("Please use either of the following variables:\n");
    std::printf("ThicknessSmoothing *or* RocheSmoothing.\n");
    std::printf("before launching the run again.\n");
    return 1;
  }
  if (p.ROCHESMOOTHING != 0.0f) std::printf("Planet potential smoothing scales with their Hill sphere.\n");
  if (st != FARGO_OK) {
    std::printf("Inconsistent parameters in %s. Program stopped.\n", parfile);
    return 1;
  }
  if (overrides) std::snprintf(p.OUTPUTDIR, sizeof(p.OUTPUTDIR), "%s", newout.c_str());
  p.SloppyCFL = sloppy;
  p.ScalingFactor = scaling;
  if (verbose) tell_everything(p);
  if (disable) return 0;
  std::printf("Allocating arrays...\n");
  std::printf("done.\n");
  const std::string outdir = p.OUTPUTDIR;
  const int NRAD = p.NRAD, NSEC = p.NSEC;
  // FillPolar1DArrays: radii.dat in, used_rad.dat out (SourceEuler.cu:84-171)
  std::vector<double> radii(NRAD + 1);
  const double* radii_in = nullptr;
  {
    FILE* in = std::fopen((outdir + "radii.dat").c_str(), "r");
    if (!in) {
      std::printf("Warning : no `radii.dat' file found. Using default.\n");
      fargo_grid_radii(&p, radii.data());
    } else {
      std::printf("Reading 'radii.dat' file.\n");
      for (int i = 0; i <= NRAD; i++) {
        float t = 0;
        if (std::fscanf(in, "%f", &t) != 1) t = 0;
        radii[i] = t;
      }
      std::fclose(in);
      radii_in = radii.data();
    }
    FILE* out = std::fopen((outdir + "used_rad.dat").c_str(), "w");
    if (!out) {
      std::printf("Can't write %sused_rad.dat.\nProgram stopped.\n", outdir.c_str());
      return 1;
    }
    for (int i = 0; i <= NRAD; i++) std::fprintf(out, "%.18g\n", radii[i]);
    std::fclose(out);
  }
  fargo_planets sys;
  st = fargo_planets_read(p.PLANETCONFIG, &p, &sys);
  if (st != FARGO_OK) {
    std::fprintf(stderr, "Error : can't find '%s'.\n", p.PLANETCONFIG);
    return 1;
  }
  std::printf("%d planet(s) found.\n", sys.nb);
  fargo_ctx* ctx = nullptr;
  st = fargo_create(&p, &sys, radii_in, -1, &ctx);
  if (st != FARGO_OK) die(ctx, st, "fargo_create");
  st = fargo_get_planets(ctx, &sys);
  for (int i = 0; i < sys.nb; i++) {  // ListPlanets, Psys.cu:210-234
    std::printf("Planet number %d\n", i);
    std::printf("---------------\n");
    std::printf("x = %.10f\ty = %.10f\n", sys.x[i], sys.y[i]);
    std::printf("vx = %.10f\tvy = %.10f\n", sys.vx[i], sys.vy[i]);
    if (sys.acc[i] == 0.0)
      std::printf("Non-accreting.\n");
    else
      std::printf("accretion time = %.10f\n", 1.0 / (sys.acc[i]));
    std::printf(sys.feeldisk[i] ? "Feels the disk potential\n" : "Doesn't feel the disk potential\n");
    std::printf(sys.feelothers[i] ? "Feels the other planets potential\n"
                                  : "Doesn't feel the other planets potential\n");
    std::printf("\n");
  }
  // WriteDim, Output.cu:137-153
  {
    FILE* dim = std::fopen((outdir + "dims.dat").c_str(), "w");
    if (!dim) {
      std::fprintf(stderr, "Unable to open %sdims.dat. Program stopped\n", outdir.c_str());
      return 1;
    }
    std::fprintf(dim, "%d\t%d\t\t%d\t%d\t%f\t%d\t%d\t%d\n", 0, 0, 0, 0, p.RMAX, p.NTOT / p.NINTERM, NRAD, NSEC);
    std::fclose(dim);
  }
  // EmptyPlanetSystemFile, Output.cu:12-32
  for (int i = 0; i < sys.nb; i++) {
    char fn[1024];
    std::snprintf(fn, sizeof(fn), "%splanet%d.dat", outdir.c_str(), i);
    FILE* f = std::fopen(fn, "w");
    if (!f) {
      std::fprintf(stderr, "Can't write %s file. Aborting\n", fn);
      return 1;
    }
    std::fclose(f);
  }
  // label field (InitLabelKernel, Kernels.cu:226-242), constant: label advection is disabled
  const size_t ng = (size_t)(NRAD + 1) * NSEC;
  std::vector<float> dens(ng), vrad(ng), vtheta(ng), energy(ng), temperature(ng), qplus(ng), label(ng, 0.0f);
  if (sys.nb > 0) {
    std::vector<double> tab(NRAD + 1);
    double xp = sys.x[0], yp = sys.y[0];
    double rp = std::sqrt(xp * xp + yp * yp), rhill = rp * std::pow(sys.mass[0] / 3., 1. / 3);
    std::vector<double> r2(NRAD + 1);
    fargo_grid_radii(&p, r2.data());
    if (radii_in) r2 = radii;
    for (int i = 0; i < NRAD; i++) {
      double m2 = 2.0 / 3.0 * (r2[i + 1] * r2[i + 1] * r2[i + 1] - r2[i] * r2[i] * r2[i]) /
                  (r2[i + 1] * r2[i + 1] - r2[i] * r2[i]);
      float rm = (float)m2;
      for (int j = 0; j < NSEC; j++) {
        float angle = (float)j / float(NSEC) * 2.0 * PI;
        float x = rm * cosf(angle), y = rm * sinf(angle);
        float distance = sqrtf((x - (float)xp) * (x - (float)xp) + (y - (float)yp) * (y - (float)yp));
        label[(size_t)i * NSEC + j] = (distance < (float)rhill) ? 1.0f : 0.0f;
      }
    }
  }
  fargo_scalars sc;
  std::memset(&sc, 0, sizeof(sc));
  float mdcp1 = 0.0f, lost = 0.0f;
  int TimeStep = 0;
  int begin_i = 0;
  if (restart) {
    // the state saved with output nb_restart; the loop resumes at that output
    char fn[1024];
    std::snprintf(fn, sizeof(fn), "%scheckpoint%d.bin", outdir.c_str(), nb_restart);
    FILE* f = std::fopen(fn, "rb");
    if (!f) {
      std::fprintf(stderr, "Can't read restart file %s\n", fn);
      return 1;
    }
    std::vector<char> ck(fargo_checkpoint_bytes(ctx));
    size_t got = std::fread(ck.data(), 1, ck.size(), f);
    std::fclose(f);
    st = fargo_checkpoint_load(ctx, ck.data(), got);
    if (st != FARGO_OK) die(ctx, st, "fargo_checkpoint_load");
    fargo_get_scalars(ctx, &sc);
    mdcp1 = sc.mdcp1;
    lost = sc.lost_mass;
    begin_i = nb_restart * p.NINTERM;
  }
  Writer writer;
  auto start = std::chrono::steady_clock::now();
  for (int i = begin_i; i <= p.NTOT; i++) {
    fargo_get_planets(ctx, &sys);
    // WriteBigPlanetSystemFile (every DT, Main.cu:349-355; Output.cu:70-102):
    // the planet values pass through static floats
    fargo_get_scalars(ctx, &sc);
    for (int k = 0; k < sys.nb; k++) {
      char fn[1024];
      std::snprintf(fn, sizeof(fn), "%sbigplanet%d.dat", outdir.c_str(), k);
      FILE* f = std::fopen(fn, "a");
      if (!f) {
        std::fprintf(stderr, "Can't write 'bigplanet.dat' file. Aborting.\n");
        return 1;
      }
      float X = sys.x[k], Y = sys.y[k], VX = sys.vx[k], VY = sys.vy[k], M = sys.mass[k];
      std::fprintf(f, "%d\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\n", TimeStep, X, Y,
                   VX, VY, M, lost, sc.physical_time, sc.omega_frame, mdcp1, mdcp1);
      std::fclose(f);
    }
    // UpdateLog (Force.cu:348-410)
    for (int k = 0; k < sys.nb; k++) {
      double x = sys.x[k], y = sys.y[k], vx = sys.vx[k], vy = sys.vy[k], m = sys.mass[k];
      double r = std::sqrt(x * x + y * y), smoothing;
      if (p.RocheSmoothing)
        smoothing = r * std::pow(m / 3., 1. / 3.) * p.ROCHESMOOTHING;
      else {
        // Compute_smoothing with AspectRatioHost (no transition by default)
        float ar = p.ASPECTRATIO;
        float rmin = p.TRANSITIONRADIUS - p.TRANSITIONWIDTH * p.ASPECTRATIO;
        float rmax = p.TRANSITIONRADIUS + p.TRANSITIONWIDTH * p.ASPECTRATIO;
        float scale = 1.0 + (sc.physical_time - 0.0f) * p.LAMBDADOUBLING;
        rmin *= scale;
        rmax *= scale;
        float rf = (float)r;
        if (rf < rmin) ar *= p.TRANSITIONRATIO;
        if ((rf >= rmin) && (rf <= rmax)) ar *= std::exp((rmax - rf) / (rmax - rmin) * std::log(p.TRANSITIONRATIO));
        smoothing = p.THICKNESSSMOOTHING * ar * std::pow(r, 1.0 + p.FLARINGINDEX);
      }
      double gf[4 * FARGO_DIMFXY];
      st = fargo_disk_force(ctx, x, y, smoothing, m, FARGO_DIMFXY, gf);
      if (st != FARGO_OK) die(ctx, st, "fargo_disk_force");
      const int d = FARGO_DIMFXY;
      float fxi = gf[0], fxei = gf[d - 1], fxo = gf[d], fxeo = gf[2 * d - 1];
      float fyi = gf[2 * d], fyei = gf[3 * d - 1], fyo = gf[3 * d], fyeo = gf[4 * d - 1];
      double PT = sc.physical_time;
      char fn[1024];
      std::snprintf(fn, sizeof(fn), "%stqwk%d.dat", outdir.c_str(), k);
      FILE* f = std::fopen(fn, "a");
      if (f) {
        std::fprintf(f, "%d\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\n", TimeStep,
                     x * fyi - y * fxi, x * fyo - y * fxo, x * fyei - y * fxei, x * fyeo - y * fxeo,
                     vx * fxi + vy * fyi, vx * fxo + vy * fyo, vx * fxei + vy * fyei, vx * fxeo + vy * fyeo, PT);
        std::fclose(f);
      }
      if (!p.SelfGravity) {
        for (int q = 0; q < d; q++) {
          std::snprintf(fn, sizeof(fn), "%stqwk%d_%d.dat", outdir.c_str(), k, q);
          f = std::fopen(fn, "a");
          if (!f) continue;
          std::fprintf(f, "%d\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\n", TimeStep, x * gf[2 * d + q] - y * gf[q],
                       x * gf[3 * d + q] - y * gf[d + q], vx * gf[q] + vy * gf[2 * d + q],
                       vx * gf[d + q] + vy * gf[3 * d + q], PT);
          std::fclose(f);
        }
      }
    }
    if (p.NINTERM * (TimeStep = (i / p.NINTERM)) == i) {
      st = fargo_download(ctx, dens.data(), vrad.data(), vtheta.data(), energy.data(), temperature.data(),
                          qplus.data());
      if (st != FARGO_OK) die(ctx, st, "fargo_download");
      std::printf("\n*** OUTPUT %d ***\n", TimeStep);
      if (p.IsDisk) {
        if (p.Write_Density) write_disk_polar(writer, outdir, dens, "dens", TimeStep, NRAD, NSEC);
        if (p.Write_Velocity) {
          write_disk_polar(writer, outdir, vrad, "vrad", TimeStep, NRAD, NSEC);
          write_disk_polar(writer, outdir, vtheta, "vtheta", TimeStep, NRAD, NSEC);
        }
        if (p.Write_Energy) write_disk_polar(writer, outdir, energy, "energy", TimeStep, NRAD, NSEC);
        if (p.Write_Temperature) write_disk_polar(writer, outdir, temperature, "temperature", TimeStep, NRAD, NSEC);
        if (p.Write_Qplus) write_disk_polar(writer, outdir, qplus, "qplus", TimeStep, NRAD, NSEC);
        if (p.AdvecteLabel) write_disk_polar(writer, outdir, label, "label", TimeStep, NRAD, NSEC);
      }
      auto ck = std::make_shared<std::vector<char>>(fargo_checkpoint_bytes(ctx));
      st = fargo_checkpoint_save(ctx, ck->data(), ck->size());
      if (st != FARGO_OK) die(ctx, st, "fargo_checkpoint_save");
      char fn[1024];
      std::snprintf(fn, sizeof(fn), "%scheckpoint%d.bin", outdir.c_str(), TimeStep);
      std::string path = fn;
      writer.push([ck, path] { write_file(path, ck->data(), ck->size()); });
    }
    int nsub = 0;
    st = fargo_advance_dt(ctx, &nsub);
    if (st != FARGO_OK) die(ctx, st, "fargo_advance_dt");
    if (p.IsDisk)
      for (int s = 0; s < nsub; s++) std::printf(".");
    std::printf("\n");
    fargo_get_scalars(ctx, &sc);
    mdcp1 = sc.mdcp1;
    lost = sc.lost_mass;
  }
  auto finish = std::chrono::steady_clock::now();
  std::printf("%g\n", std::chrono::duration<double>(finish - start).count());
  fargo_destroy(ctx);
  return 0;
}
