// host_params.cpp -- .par / .cfg handling with the reference's semantics.
//
// ReadVariables + SearchVariable (Interpret.cu:35-208) and
// InitPlanetarySystem (Psys.cu:83-208).  Quirks kept on purpose so that a
// parameter file means the same thing to both programs:
//   - keys are upper-cased, values compared case-sensitively ("YES" only);
//   - the value is the first token after the key (sscanf "%289s");
//   - unknown keys are ignored;
//   - WriteDivV is assigned from a number (Interpret.cu:73), so it is never YES;
//   - an AdiabaticIndex of 1 turns Adiabatic off (Interpret.cu:164-168).
// Fatal checks of the reference (exit(1)) become FARGO_EINVAL.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fargo_b200.h"
#include "host_internal.h"

namespace {

void setstr(char* dst, size_t cap, const char* v) {
  std::snprintf(dst, cap, "%s", v);
}

#define SETS(field, v) setstr(p->field, sizeof(p->field), v)

}  // namespace

extern "C" fargo_status fargo_params_default(fargo_params* p) {
  if (!p) return FARGO_EINVAL;
  std::memset(p, 0, sizeof(*p));
  // Param.cuh:9-63
  p->DT = 1.0f;
  p->SIGMA0 = 173.0f;
  p->NINTERM = 10;
  p->NTOT = 1501;
  SETS(OUTPUTDIR, "~masset");
  SETS(INNERBOUNDARY, "WALL");
  SETS(LABELADVECTION, "NO");
  SETS(TRANSPORT, "FAST");
  SETS(PLANETCONFIG, "Systems/SolarSystem.cfg");
  p->MASSTAPER = 0.0000001f;
  SETS(RADIALSPACING, "ARITHMETIC");
  p->NRAD = 64;
  p->NSEC = 64;
  p->RMIN = 1.0f;
  p->RMAX = 1.0f;
  p->THICKNESSSMOOTHING = 0.0f;
  p->ROCHESMOOTHING = 0.0f;
  p->ASPECTRATIO = 0.05f;
  p->VISCOSITY = 0.0f;
  p->ALPHAVISCOSITY = 0.0f;
  p->SIGMASLOPE = 0.0f;
  p->RELEASERADIUS = 0.0f;
  p->RELEASEDATE = 0.0f;
  p->OMEGAFRAME = 0.0f;
  SETS(DISK, "YES");
  SETS(FRAME, "FIXED");
  SETS(OUTERSOURCEMASS, "NO");
  SETS(WRITEDENSITY, "YES");
  SETS(WRITEVELOCITY, "YES");
  SETS(WRITEENERGY, "NO");
  SETS(WRITETEMPERATURE, "NO");
  SETS(WRITEQPLUS, "NO");
  SETS(INDIRECTTERM, "YES");
  SETS(EXCLUDEHILL, "NO");
  p->IMPOSEDDISKDRIFT = 0.0f;
  p->FLARINGINDEX = 0.0f;
  p->ECCENTRICITY = 0.0f;
  p->CAVITYRADIUS = 0.0f;
  p->CAVITYRATIO = 1.0f;
  p->CAVITYWIDTH = 1.0f;
  p->TRANSITIONRADIUS = 0.0f;
  p->TRANSITIONRATIO = 1.0f;
  p->TRANSITIONWIDTH = 1.0f;
  p->LAMBDADOUBLING = 0.0f;
  SETS(SELFGRAVITY, "NO");
  SETS(CICPLANET, "NO");
  SETS(FORCEDCIRCULAR, "NO");
  SETS(ZMPLUS, "NO");
  SETS(ADIABATIC, "NO");
  p->ADIABATICINDEX = 1.4f;
  SETS(COOLING, "NO");
  p->COOLINGTIME0 = 6.28f;
  // command-line defaults (Main.cu:75, Param.cuh:1)
  p->SloppyCFL = 0;
  p->ScalingFactor = 1.0f;
  // switch defaults (Interpret.cu:23-31)
  p->FastTransport = 1;
  p->Indirect_Term = 1;
  p->IsDisk = 1;
  p->Write_Density = 1;
  p->Write_Velocity = 1;
  fargo_params_derive(p);  // the defaults alone fail the smoothing check; not an error here
  return FARGO_OK;
}

// SearchVariable, Interpret.cu:35-95
static void search_variable(fargo_params* p, const char* name, const char* stringval, double temp) {
#define NUMF(KEY) \
  if (std::strcmp(name, #KEY) == 0) p->KEY = (float)(temp);
#define NUMI(KEY) \
  if (std::strcmp(name, #KEY) == 0) p->KEY = (int)(temp);
#define STR(KEY) \
  if (std::strcmp(name, #KEY) == 0) SETS(KEY, stringval);
  NUMF(DT)
  NUMF(SIGMA0)
  NUMI(NINTERM)
  NUMI(NTOT)
  STR(OUTPUTDIR)
  STR(INNERBOUNDARY)
  STR(LABELADVECTION)
  STR(TRANSPORT)
  STR(PLANETCONFIG)
  NUMF(MASSTAPER)
  STR(RADIALSPACING)
  NUMI(NRAD)
  NUMI(NSEC)
  NUMF(RMIN)
  NUMF(RMAX)
  NUMF(THICKNESSSMOOTHING)
  NUMF(ROCHESMOOTHING)
  NUMF(ASPECTRATIO)
  NUMF(VISCOSITY)
  NUMF(ALPHAVISCOSITY)
  NUMF(SIGMASLOPE)
  NUMF(RELEASERADIUS)
  NUMF(RELEASEDATE)
  NUMF(OMEGAFRAME)
  STR(DISK)
  STR(FRAME)
  STR(OUTERSOURCEMASS)
  STR(WRITEDENSITY)
  STR(WRITEVELOCITY)
  STR(WRITEENERGY)
  STR(WRITETEMPERATURE)
  // WRITEDIVV = temp (Interpret.cu:73): a one-character string, never "YES"
  STR(WRITEQPLUS)
  STR(INDIRECTTERM)
  STR(EXCLUDEHILL)
  NUMF(IMPOSEDDISKDRIFT)
  NUMF(FLARINGINDEX)
  NUMF(ECCENTRICITY)
  NUMF(CAVITYRADIUS)
  NUMF(CAVITYRATIO)
  NUMF(CAVITYWIDTH)
  NUMF(TRANSITIONRADIUS)
  NUMF(TRANSITIONRATIO)
  NUMF(TRANSITIONWIDTH)
  NUMF(LAMBDADOUBLING)
  STR(SELFGRAVITY)
  STR(CICPLANET)
  STR(FORCEDCIRCULAR)
  STR(ZMPLUS)
  STR(ADIABATIC)
  NUMF(ADIABATICINDEX)
  STR(COOLING)
  NUMF(COOLINGTIME0)
#undef NUMF
#undef NUMI
#undef STR
}

static bool eq(const char* a, const char* b) { return std::strcmp(a, b) == 0; }

// The derived switches of ReadVariables (Interpret.cu:126-201).
extern "C" fargo_status fargo_params_derive(fargo_params* p) {
  if (!p) return FARGO_EINVAL;
  p->AdvecteLabel = eq(p->LABELADVECTION, "YES");
  p->OuterSourceMass = eq(p->OUTERSOURCEMASS, "YES");
  p->FastTransport = !eq(p->TRANSPORT, "STANDARD");
  p->OpenInner = eq(p->INNERBOUNDARY, "OPEN");
  p->NonReflecting = eq(p->INNERBOUNDARY, "NONREFLECTING");
  p->Evanescent = eq(p->INNERBOUNDARY, "EVANESCENT");
  p->LogGrid = eq(p->RADIALSPACING, "LOGARITHM");
  p->IsDisk = !eq(p->DISK, "NO");
  p->Corotating = eq(p->FRAME, "COROTATING");
  p->GuidingCenter = 0;
  if (eq(p->FRAME, "GUIDING-CENTER")) {
    p->GuidingCenter = 1;
    p->Corotating = 1;
  }
  p->Write_Velocity = !eq(p->WRITEVELOCITY, "NO");
  p->Write_Density = !eq(p->WRITEDENSITY, "NO");
  p->Write_Energy = eq(p->WRITEENERGY, "YES");
  p->Write_Temperature = eq(p->WRITETEMPERATURE, "YES");
  p->Write_DivV = 0;
  p->Write_Qplus = eq(p->WRITEQPLUS, "YES");
  p->Indirect_Term = !eq(p->INDIRECTTERM, "NO");
  p->SelfGravity = 0;
  p->SGZeroMode = 0;
  if (eq(p->SELFGRAVITY, "YES")) p->SelfGravity = 1;
  if (eq(p->SELFGRAVITY, "Z")) {
    p->SelfGravity = 1;
    p->SGZeroMode = 1;
  }
  p->ZMPluss = eq(p->ZMPLUS, "YES");
  if (p->ZMPluss && !p->SGZeroMode) p->ZMPluss = 0;
  p->Adiabatic = 0;
  if (eq(p->ADIABATIC, "YES")) {
    p->Adiabatic = 1;
    p->Write_Temperature = 1;
  }
  p->Cooling = eq(p->COOLING, "YES");
  if (p->Adiabatic && p->ADIABATICINDEX == 1.0f) p->Adiabatic = 0;
  if (eq(p->WRITEENERGY, "NO")) p->Write_Energy = 0;
  p->ExcludeHill = eq(p->EXCLUDEHILL, "YES");
  p->CICPlanet = eq(p->CICPLANET, "YES");
  p->ForcedCircular = eq(p->FORCEDCIRCULAR, "YES");
  if (p->ALPHAVISCOSITY != 0.0f && p->VISCOSITY != 0.0f) return FARGO_EINVAL;
  p->ViscosityAlpha = (p->ALPHAVISCOSITY != 0.0f);
  if (p->THICKNESSSMOOTHING != 0.0f && p->ROCHESMOOTHING != 0.0f) return FARGO_EINVAL;
  if (p->THICKNESSSMOOTHING <= 0.0f && p->ROCHESMOOTHING <= 0.0f) return FARGO_EINVAL;
  p->RocheSmoothing = (p->ROCHESMOOTHING != 0.0f);
  return FARGO_OK;
}

// ReadVariables, Interpret.cu:97-124
extern "C" fargo_status fargo_params_read(const char* parfile, fargo_params* p) {
  if (!parfile || !p) return FARGO_EINVAL;
  fargo_params_default(p);
  FILE* input = std::fopen(parfile, "r");
  if (!input) return FARGO_EIO;
  char nm[300], s[350], stringval[290];
  while (std::fgets(s, 349, input) != NULL) {
    int success = std::sscanf(s, "%299s ", nm);
    if (success == 1 && nm[0] != '#') {
      const char* s1 = s + std::strlen(nm);
      s1 += std::strspn(s1, "\t :=>_");
      stringval[0] = 0;
      std::sscanf(s1, "%289s ", stringval);
      // SearchVariable parses the value token as a number; a failed parse
      // keeps an indeterminate value in the reference, which is only ever
      // assigned to string variables (or WriteDivV) -- 0 here.
      double temp = 0.0;
      std::sscanf(stringval, "%lf", &temp);
      for (size_t i = 0; i < std::strlen(nm); i++) nm[i] = (char)std::toupper((unsigned char)nm[i]);
      search_variable(p, nm, stringval, temp);
    }
  }
  std::fclose(input);
  return fargo_params_derive(p);
}

// FillPolar1DArrays radii (SourceEuler.cu:113-130), in double.
extern "C" fargo_status fargo_grid_radii(const fargo_params* p, double* radii) {
  if (!p || !radii || p->NRAD < 1) return FARGO_EINVAL;
  int NRAD = p->NRAD;
  float drrsep = (p->RMAX - p->RMIN) / (float)NRAD;
  for (int i = 0; i <= NRAD; i++) {
    if (p->LogGrid)
      radii[i] = (double)p->RMIN * std::exp((double)i / (double)NRAD * std::log((double)p->RMAX / (double)p->RMIN));
    else
      radii[i] = p->RMIN + drrsep * (double)i;
  }
  return FARGO_OK;
}

// InitPlanetarySystem + FindNumberOfPlanets, Psys.cu:83-208
extern "C" fargo_status fargo_planets_read(const char* cfgfile, const fargo_params* p, fargo_planets* out) {
  if (!cfgfile || !p || !out) return FARGO_EINVAL;
  std::memset(out, 0, sizeof(*out));
  FILE* input = std::fopen(cfgfile, "r");
  if (!input) return FARGO_EIO;
  char s[512], nm[512], test1[512], test2[512];
  int nb = 0;
  while (std::fgets(s, 510, input) != NULL)
    if (std::isalpha((unsigned char)s[0])) nb++;
  if (nb > FARGO_MAXPLANETS) {
    std::fclose(input);
    return FARGO_EINVAL;
  }
  std::rewind(input);
  std::vector<double> rmed, radii;
  if (p->CICPlanet) host_grid_rmed(p, nullptr, &radii, &rmed);
  int i = 0;
  while (std::fgets(s, 510, input) != NULL) {
    nm[0] = 0;
    std::sscanf(s, "%511s ", nm);
    if (std::isalpha((unsigned char)s[0])) {
      const char* s1 = s + std::strlen(nm);
      double dist = 0, mass = 0, accret = 0;
      test1[0] = test2[0] = 0;
      std::sscanf(s1 + std::strspn(s1, "\t :=>_"), "%lf %lf %lf %511s %511s", &dist, &mass, &accret, test1, test2);
      if (p->CICPlanet) {
        int j = 0;
        while ((float)rmed[j] < dist) j++;
        dist = (float)radii[j + 1];
      }
      out->mass[i] = mass;
      int feeldis = 1, feelothers = 1;
      if (std::tolower((unsigned char)test1[0]) == 'n') feeldis = 0;
      if (std::tolower((unsigned char)test2[0]) == 'n') feelothers = 0;
      out->x[i] = dist * (1.0 + p->ECCENTRICITY);
      out->y[i] = 0.0;
      out->vy[i] = std::sqrt(1.0 * (1.0 + mass) / dist) * std::sqrt((1.0 - p->ECCENTRICITY) / (1.0 + p->ECCENTRICITY));
      out->vx[i] = -0.0000000001 * out->vy[i];
      out->acc[i] = accret;
      out->feeldisk[i] = feeldis;
      out->feelothers[i] = feelothers;
      std::snprintf(out->name[i], sizeof(out->name[i]), "%s", nm);
      i++;
    }
  }
  out->nb = nb;
  std::fclose(input);
  return FARGO_OK;
}
