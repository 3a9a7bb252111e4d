// host_setup.cpp -- host-side setup with the reference's arithmetic:
// FillPolar1DArrays (SourceEuler.cu:76-157), Main.cu:259-268, Theo.cu:13-78
// profiles, FViscosity / AspectRatioHost (Viscosity.cu:19-52), the
// sub-Keplerian boundary speeds (SideEuler.cu:250-259) and GetPsysInfo's
// FREQUENCY branch (Psys.cu:236-306).
#include <cmath>
#include <cstring>

#include "host_internal.h"

#define PI 3.14159265358979323844

void host_grid_rmed(const fargo_params* p, const double* radii_in, std::vector<double>* radii2,
                    std::vector<double>* rmed2) {
  int NRAD = p->NRAD;
  radii2->assign(NRAD + 1, 0.0);
  rmed2->assign(NRAD + 1, 0.0);
  if (radii_in) {
    for (int i = 0; i <= NRAD; i++) (*radii2)[i] = radii_in[i];
  } else {
    fargo_grid_radii(p, radii2->data());
  }
  const std::vector<double>& R2 = *radii2;
  for (int i = 0; i < NRAD; i++) {
    double v = 2.0 / 3.0 * (R2[i + 1] * R2[i + 1] * R2[i + 1] - R2[i] * R2[i] * R2[i]);
    (*rmed2)[i] = v / (R2[i + 1] * R2[i + 1] - R2[i] * R2[i]);
  }
}

void host_build_tables(const fargo_params* p, const double* radii_in, HostTables* t) {
  int NRAD = p->NRAD, NSEC = p->NSEC;
  t->nrad = NRAD;
  t->nsec = NSEC;
  host_grid_rmed(p, radii_in, &t->Radii2, &t->Rmed2);
  std::vector<float>* f1[] = {&t->Radii,    &t->Rinf,         &t->Rsup,         &t->Rmed,       &t->Surf,
                              &t->invRinf,  &t->invSurf,      &t->invRmed,      &t->invdiffRsup, &t->invdiffRmed,
                              &t->powRmed,  &t->dxtheta,      &t->supp_torque,  &t->SigmaMed,   &t->SigmaInf,
                              &t->EnergyMed, &t->CoolingTimeMed, &t->QplusMed};
  for (auto* v : f1) v->assign(NRAD + 1, 0.0f);  // entries the reference leaves unset are 0
  t->pow15.assign(NRAD + 1, 0.0);
  t->star_grad.assign(NRAD + 1, 0.0f);
  t->cfl_rdr.assign(NRAD + 1, 0.0f);
  t->cfl_rdt.assign(NRAD + 1, 0.0f);
  t->cfl_rmd.assign(NRAD + 1, 0.0f);
  const std::vector<double>& R2 = t->Radii2;
  const std::vector<double>& M2 = t->Rmed2;
  for (int i = 0; i <= NRAD; i++) t->Radii[i] = (float)R2[i];
  for (int i = 0; i < NRAD; i++) {
    t->Rinf[i] = R2[i];
    t->Rsup[i] = R2[i + 1];
    t->Rmed[i] = M2[i];
    t->Surf[i] = PI * (R2[i + 1] * R2[i + 1] - R2[i] * R2[i]) / (double)NSEC;
    t->invRmed[i] = 1.0 / M2[i];
    t->invSurf[i] = 1.0 / t->Surf[i];
    t->invdiffRsup[i] = 1.0 / (R2[i + 1] - R2[i]);
    t->invRinf[i] = 1.0 / R2[i];
  }
  t->Rinf[NRAD] = R2[NRAD];
  for (int i = 0; i < NRAD; i++) {
    if (i > 0) t->invdiffRmed[i] = 1.0 / (M2[i] - M2[i - 1]);
    if (i > 0) t->star_grad[i] = (float)(1.0 / (M2[i] * M2[i - 1]));
    t->powRmed[i] = std::pow(M2[i], -2.5 + p->SIGMASLOPE);
    t->pow15[i] = std::pow((double)t->Rmed[i], 1.5);
  }
  // Main.cu:259-268
  float dphi = 2.0 * PI / (float)NSEC;
  t->invdphi = 1.0 / dphi;
  t->onethird = 1.0 / 3.0;
  for (int i = 0; i < NRAD; i++) {
    t->supp_torque[i] = p->IMPOSEDDISKDRIFT * 0.5 * std::pow(t->Rmed[i], -2.5 + p->SIGMASLOPE);
    t->dxtheta[i] = 2.0 * PI / (float)NSEC * t->Rmed[i];
  }
  // RN(1/d) in FP32: the FP64 quotient rounded to float (double rounding is
  // innocuous for a quotient of floats: 53 >= 2*24 + 2)
  for (int i = 0; i < NRAD; i++) {
    const float dxr = t->Rsup[i] - t->Rinf[i];  // the device's float subtraction
    const float dxt = t->dxtheta[i];
    const float md = (dxt < dxr) ? dxt : dxr;  // min2(dxrad, dxtheta)
    t->cfl_rdr[i] = (float)(1.0 / (double)dxr);
    t->cfl_rdt[i] = (float)(1.0 / (double)dxt);
    t->cfl_rmd[i] = (float)(1.0 / (double)md);
  }
  // FillSigma / FillEnergy / FillCoolingTime (Theo.cu:23-61), Sigma(r)
  for (int i = 0; i < NRAD; i++) {
    float r = t->Rmed[i], ri = t->Rinf[i];
    float cav = 1.0, cavi = 1.0;
    if (r < p->CAVITYRADIUS) cav = 1.0 / p->CAVITYRATIO;
    if (ri < p->CAVITYRADIUS) cavi = 1.0 / p->CAVITYRATIO;
    t->SigmaMed[i] = cav * p->ScalingFactor * p->SIGMA0 * std::pow(r, -p->SIGMASLOPE);
    t->SigmaInf[i] = cavi * p->ScalingFactor * p->SIGMA0 * std::pow(ri, -p->SIGMASLOPE);
    if (p->ADIABATICINDEX != 1.0f)
      t->EnergyMed[i] = 1.0 / 1.0 / (p->ADIABATICINDEX - 1.0) * p->SIGMA0 * std::pow(p->ASPECTRATIO, 2.0) *
                        std::pow(r, -p->SIGMASLOPE - 1.0 + 2.0 * p->FLARINGINDEX);
    t->CoolingTimeMed[i] = p->COOLINGTIME0 * std::pow(r, 2.0 + 2.0 * p->FLARINGINDEX);
  }
}

float host_aspect_ratio(const fargo_params* p, float r, float PT, float PTI) {
  float aspectratio, rmin, rmax, scale;
  aspectratio = p->ASPECTRATIO;
  rmin = p->TRANSITIONRADIUS - p->TRANSITIONWIDTH * p->ASPECTRATIO;
  rmax = p->TRANSITIONRADIUS + p->TRANSITIONWIDTH * p->ASPECTRATIO;
  scale = 1.0 + (PT - PTI) * p->LAMBDADOUBLING;
  rmin *= scale;
  rmax *= scale;
  if (r < rmin) aspectratio *= p->TRANSITIONRATIO;
  if ((r >= rmin) && (r <= rmax)) aspectratio *= std::exp((rmax - r) / (rmax - rmin) * std::log(p->TRANSITIONRATIO));
  return aspectratio;
}

float host_fviscosity(const fargo_params* p, const HostTables& t, const float* csmean, float r, float PT,
                      float PTI) {
  float viscosity, rmin, rmax, scale;
  int i = 0;
  viscosity = p->VISCOSITY;
  if (p->ViscosityAlpha) {
    while (t.Rmed[i] < r) i++;
    viscosity = p->ALPHAVISCOSITY * csmean[i] * csmean[i] * std::pow(r, 1.5);
  }
  rmin = p->CAVITYRADIUS - p->CAVITYWIDTH * p->ASPECTRATIO;
  rmax = p->CAVITYRADIUS + p->CAVITYWIDTH * p->ASPECTRATIO;
  scale = 1.0 + (PT - PTI) * p->LAMBDADOUBLING;
  rmin *= scale;
  rmax *= scale;
  if (r < rmin) viscosity *= p->CAVITYRATIO;
  if ((r >= rmin) && (r <= rmax)) viscosity *= std::exp((rmax - r) / (rmax - rmin) * std::log(p->CAVITYRATIO));
  return viscosity;
}

void host_vkep(const fargo_params* p, const HostTables& t, float PT, float PTI, double* vin, double* vout) {
  int NRAD = t.nrad;
  float r0 = t.Rmed[0], r1 = t.Rmed[NRAD - 1];
  *vin = std::sqrt(1.0 * 1.0 / r0 *
                   (1.0 - (1.0 + p->SIGMASLOPE - 2.0 * p->FLARINGINDEX) *
                              std::pow(host_aspect_ratio(p, r0, PT, PTI), 2.0) * std::pow(r0, 2.0 * p->FLARINGINDEX)));
  *vout = std::sqrt(1.0 * 1.0 / r1 *
                    (1.0 - (1.0 + p->SIGMASLOPE - 2.0 * p->FLARINGINDEX) *
                               std::pow(host_aspect_ratio(p, r1, PT, PTI), 2.0) * std::pow(r1, 2.0 * p->FLARINGINDEX)));
}

float host_get_psys_frequency(const fargo_planets* sys) {
  double x = sys->x[0], y = sys->y[0], vx = sys->vx[0], vy = sys->vy[0];
  double m = sys->mass[0] + 1.;
  double h = x * vy - y * vx;
  double d = std::sqrt(x * x + y * y);
  double Ax = x * vy * vy - y * vx * vy - 1.0 * m * x / d;
  double Ay = y * vx * vx - x * vx * vy - 1.0 * m * y / d;
  double e = std::sqrt(Ax * Ax + Ay * Ay) / m;
  double a = h * h / 1.0 / m / (1. - e * e);
  return std::sqrt(m / a / a / a);
}
