// host_internal.h -- host-side setup shared by the C ABI and the driver.
#pragma once
#include <vector>

#include "../../include/fargo_b200.h"

// 1-D tables of FillPolar1DArrays (SourceEuler.cu:76-157) and Main.cu:259-268,
// computed in double and rounded to float exactly as the reference does.
struct HostTables {
  int nrad = 0, nsec = 0;
  std::vector<double> Radii2, Rmed2;
  std::vector<float> Radii, Rinf, Rsup, Rmed, Surf, invRinf, invSurf, invRmed, invdiffRsup, invdiffRmed;
  std::vector<float> powRmed, dxtheta, supp_torque, SigmaMed, SigmaInf, EnergyMed, CoolingTimeMed, QplusMed;
  std::vector<double> pow15;  // pow(Rmed[i], 1.5) as FViscosity evaluates it
  // accurate mode: the star potential's radial difference quotient
  // (-G/Rmed[i] + G/Rmed[i-1]) / (Rmed[i] - Rmed[i-1]) = G / (Rmed[i] Rmed[i-1]),
  // from the FP64 radii, rounded once
  std::vector<float> star_grad;
  // the CFL's per-ring divisors Rsup-Rinf, dxtheta and their minimum
  // (ConditionCFLKernel2D1, Kernels.cu:1380-1400), as correctly rounded FP32
  // reciprocals: the quotients are then formed by Markstein's method
  std::vector<float> cfl_rdr, cfl_rdt, cfl_rmd;
  float invdphi = 0, onethird = 0;
};

void host_grid_rmed(const fargo_params* p, const double* radii_in, std::vector<double>* radii2,
                    std::vector<double>* rmed2);
void host_build_tables(const fargo_params* p, const double* radii_in, HostTables* t);
float host_aspect_ratio(const fargo_params* p, float r, float PT, float PTI);
float host_fviscosity(const fargo_params* p, const HostTables& t, const float* csmean, float r, float PT,
                      float PTI);
void host_vkep(const fargo_params* p, const HostTables& t, float PT, float PTI, double* vin, double* vout);
float host_get_psys_frequency(const fargo_planets* sys);
