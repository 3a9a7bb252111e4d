// fargo_api.cu -- the C ABI (include/fargo_b200.h): contexts, batches,
// device memory, the per-DT CUDA graph and the host-visible operations.
//
// One DT (the body of AlgoGas, SourceEuler.cu:208-301) is
//   k_dt_begin [+ adiabatic sound speed refresh]  -> stream launches
//   WHILE(any disk inside its DT) { one substep }  -> one CUDA graph launch
// The WHILE node's condition is written by the last kernel of the substep
// (cudaGraphSetConditional), so the host never waits inside a DT.
#include <cuda.h>  // CUtensorMap (encoded through the runtime's driver entry point; no libcuda link)
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "fargo_internal.h"
#include "host_internal.h"
#include "sg.h"

namespace {


struct DiskHost {
  int seg_out = FARGO_SEG_OUT;  // transport segment width of this disk (autotuned per NSEC class)
  fargo_params p;
  fargo_planets planets0;
  HostTables t;
  DiskDev dev{};  // device pointers + parameters
  std::vector<void*> allocs;
  SelfGravity* sg = nullptr;
};

}  // namespace

struct fargo_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<DiskHost> disks;
  BatchDev bd{};
  DiskDev* d_disks = nullptr;
  DiskCtl* d_ctl = nullptr;
  long long* d_cell_off = nullptr;
  int* d_ring_off = nullptr;
  int4* d_theta = nullptr;
  int seg_out = FARGO_SEG_OUT;  // transport segment width in use (autotuned)
  int* d_flags = nullptr;
  int* d_act = nullptr;  // every compacted-list array in one allocation
  long long* d_act_cell = nullptr;
  double* d_red = nullptr;  // reduction scratch for force/diagnostic kernels
  int red_blocks = 0;
  int max_nsec = 0;
  int any_adiabatic = 0;
  int n_sg = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphConditionalHandle handle = 0;
  bool use_graph = true;
  long long launches = 0;
  long long ncell_ghost = 0;
  // radial stripe (fargo_stripe_create): global ring of local ring 0, the
  // whole disk's ring count, ghost rings below and above the own rings
  int stripe = 0, stripe_base = 0, stripe_nrad = 0, ghost_lo = 0, ghost_hi = 0;
  // self-gravity of a self-gravitating stripe: the whole disk's convolution
  // (gsg) on a view gv of the whole grid, whose density is gathered from
  // every stripe's own rings before each substep; gt: the whole disk's tables
  SelfGravity* gsg = nullptr;
  DiskDev gv{};
  HostTables gt;
  std::vector<void*> gallocs;
  std::string err;
};

struct fargo_ctx {
  fargo_batch b;
};

namespace {

fargo_status set_err(fargo_batch* b, fargo_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (b) b->err = buf;
  return st;
}

#define CK(call)                                                                               \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) {                                                                   \
      fargo_status st_ = (e_ == cudaErrorMemoryAllocation) ? FARGO_EOOM : FARGO_ECUDA;         \
      return set_err(b, st_, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    }                                                                                          \
  } while (0)

template <class T>
fargo_status dalloc(fargo_batch* b, DiskHost& h, T** ptr, size_t count) {
  void* p = nullptr;
  CK(cudaMalloc(&p, sizeof(T) * (count ? count : 1)));
  CK(cudaMemsetAsync(p, 0, sizeof(T) * (count ? count : 1), b->stream));
  h.allocs.push_back(p);
  *ptr = (T*)p;
  return FARGO_OK;
}

template <class T>
fargo_status dupload(fargo_batch* b, DiskHost& h, const T** ptr, const std::vector<T>& v) {
  T* p = nullptr;
  fargo_status st = dalloc(b, h, &p, v.size());
  if (st) return st;
  CK(cudaMemcpyAsync(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, b->stream));
  *ptr = p;
  return FARGO_OK;
}

// bodies of the per-substep force sums: the star and every FeelDisk planet
int body_count(const fargo_planets* pl) {
  int n = 1;
  for (int k = 0; k < pl->nb; k++) n += pl->feeldisk[k] ? 1 : 0;
  return n;
}

fargo_status check_params(fargo_batch* b, const fargo_params* p, const fargo_planets* pl) {
  if (p->NRAD < 4 || p->NSEC < 4) return set_err(b, FARGO_EINVAL, "NRAD and NSEC must be >= 4");
  if (p->NSEC > 16384) return set_err(b, FARGO_EINVAL, "NSEC > 16384 is not supported");
  if ((long long)(p->NRAD + 1) * p->NSEC > 0x7fffffffLL)
    return set_err(b, FARGO_EINVAL, "(NRAD+1)*NSEC must fit a 32-bit cell index, as in the reference's kernels");
  if (p->NonReflecting && p->NSEC <= 128)
    return set_err(b, FARGO_EINVAL,
                   "InnerBoundary NONREFLECTING needs NSEC > 128 (the reference's DeviceReduce launches no block "
                   "for 128 or fewer values)");
  if (p->SelfGravity && !p->LogGrid)
    return set_err(b, FARGO_EINVAL, "self-gravity needs RadialSpacing LOGARITHM (Main.cu:302-306)");
  if (p->SelfGravity && p->SGZeroMode) return set_err(b, FARGO_EINVAL, "SelfGravity Z is not implemented");
  if (pl->nb < 0 || pl->nb > FARGO_MAXPLANETS) return set_err(b, FARGO_EINVAL, "bad planet count %d", pl->nb);
  int nfeel = 0;
  for (int k = 0; k < pl->nb; k++) nfeel += pl->feeldisk[k] ? 1 : 0;
  if (nfeel > FARGO_MAXBODY - 1)
    return set_err(b, FARGO_EINVAL, "at most %d planets may feel the disk", FARGO_MAXBODY - 1);
  if (p->Corotating && pl->nb < 1) return set_err(b, FARGO_EINVAL, "a corotating frame needs a planet");
  return FARGO_OK;
}

// Device memory and constant tables of one disk.
// cuTensorMapEncodeTiled, looked up once through the runtime (null when the
// driver does not provide it: the transport then stages by cp.async).
PFN_cuTensorMapEncodeTiled_v12000 tensormap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  });
  return fn;
}

// The transport's three tensor maps of one disk (Sigma, v_r, v_theta):
// 2-D, NSEC columns x rows (NRAD for Sigma and v_theta, NRAD + 1 for v_r
// with its ghost row), boxes of FARGO_TR_ROW columns x the band's staged
// rows, FP32, no swizzle, zero fill outside.  Needs NSEC a multiple of 4
// (16-byte row pitch) and >= 64; D.tmap stays null otherwise.
fargo_status make_tensor_maps(fargo_batch* b, DiskHost& h, DiskDev& D);

fargo_status alloc_disk(fargo_batch* b, DiskHost& h, const double* radii) {
  const fargo_params* p = &h.p;
  host_build_tables(p, radii, &h.t);
  DiskDev& D = h.dev;
  std::memset(&D, 0, sizeof(D));
  D.nrad = p->NRAD;
  D.nsec = p->NSEC;
  D.DT = p->DT;
  D.ADIABATICINDEX = p->ADIABATICINDEX;
  D.ASPECTRATIO = p->ASPECTRATIO;
  D.FLARINGINDEX = p->FLARINGINDEX;
  D.SIGMASLOPE = p->SIGMASLOPE;
  D.SIGMA0 = p->SIGMA0;
  D.TRANSITIONRADIUS = p->TRANSITIONRADIUS;
  D.TRANSITIONRATIO = p->TRANSITIONRATIO;
  D.TRANSITIONWIDTH = p->TRANSITIONWIDTH;
  D.LAMBDADOUBLING = p->LAMBDADOUBLING;
  D.VISCOSITY = p->VISCOSITY;
  D.ALPHAVISCOSITY = p->ALPHAVISCOSITY;
  D.CAVITYRADIUS = p->CAVITYRADIUS;
  D.CAVITYRATIO = p->CAVITYRATIO;
  D.CAVITYWIDTH = p->CAVITYWIDTH;
  D.MASSTAPER = p->MASSTAPER;
  D.RELEASEDATE = p->RELEASEDATE;
  D.RELEASERADIUS = p->RELEASERADIUS;
  D.THICKNESSSMOOTHING = p->THICKNESSSMOOTHING;
  D.ROCHESMOOTHING = p->ROCHESMOOTHING;
  D.IMPOSEDDISKDRIFT = p->IMPOSEDDISKDRIFT;
  D.Adiabatic = p->Adiabatic;
  D.Cooling = p->Cooling;
  D.ViscosityAlpha = p->ViscosityAlpha;
  D.FastTransport = p->FastTransport;
  D.Indirect_Term = p->Indirect_Term;
  D.ExcludeHill = p->ExcludeHill;
  D.ForcedCircular = p->ForcedCircular;
  D.Corotating = p->Corotating;
  D.GuidingCenter = p->GuidingCenter;
  D.RocheSmoothing = p->RocheSmoothing;
  D.SelfGravity = p->SelfGravity;
  D.Evanescent = p->Evanescent;
  D.OpenInner = p->OpenInner;
  D.NonReflecting = p->NonReflecting;
  if (p->NRAD >= 3) {
    D.nr_pow_in = std::pow((double)h.t.Rinf[1], -1.5);
    D.nr_pow_out = std::pow((double)h.t.Rinf[p->NRAD - 2], -1.5);
  }
  D.ev_Tin = (float)(2.0 * FARGO_PI * std::pow((double)h.t.Rmed[0], 3. / 2));
  D.ev_Tout = (float)(2.0 * FARGO_PI * std::pow((double)h.t.Rmed[p->NRAD - 1], 3. / 2));
  D.ev_DRMIN = (float)(h.t.Rmed[0] * 1.25);
  D.ev_DRMAX = (float)(h.t.Rmed[p->NRAD - 1] * 0.84);
  D.SloppyCFL = p->SloppyCFL;
  D.IsDisk = p->IsDisk;
  D.max_sub = FARGO_MAX_SUBSTEPS;
  D.accurate = 0;
  D.own_lo = 0;
  D.own_hi = p->NRAD;
  D.stripe = 0;
  D.cfl_tile = FARGO_CFL_TILE;  // set per batch by set_cfl_tiles
  D.invdphi = h.t.invdphi;
  D.onethird = h.t.onethird;
  size_t ng = (size_t)(p->NRAD + 1) * p->NSEC;
  size_t n1 = (size_t)p->NRAD + 1;
  fargo_status st;
#define A(ptr, n)                          \
  if ((st = dalloc(b, h, &(ptr), (n)))) \
    return st;
  A(D.dens, ng) A(D.vrad, ng) A(D.vtheta, ng) A(D.energy, ng) A(D.vri, ng) A(D.vti, ng) A(D.trr, ng)
  A(D.tpp, ng) A(D.trp, ng) A(D.qplus, ng) A(D.a0, ng)
  if (p->Adiabatic) {
    A(D.cs, ng) A(D.a1, ng)
  } else {
    D.cs = nullptr;
    D.a1 = D.a0;  // never written in isothermal runs
  }
  A(D.pres, ng) A(D.phi, ng)
  size_t nct = std::max<size_t>(n1, (size_t)fargo_cfl_tiles(p->NRAD, p->NSEC, FARGO_CFL_TILE_SMALL));
  A(D.visc, n1) A(D.cs_ring, n1) A(D.csmean, n1) A(D.vmoy, n1) A(D.ringmin, nct) A(D.nshift, n1)
  A(D.tvmed, n1) A(D.tvconst, n1)
  A(D.log_nshift, (size_t)FARGO_MAXLOG * p->NRAD) A(D.partials, nct * 4 * FARGO_MAXBODY)
  A(D.log_dt, (size_t)FARGO_MAXLOG) A(D.rk_work, (size_t)FARGO_RK_WORK(FARGO_MAXPLANETS_DEV))
  if (p->OpenInner) {
    A(D.lost, (size_t)p->NSEC)
  } else {
    D.lost = nullptr;
  }
  float *cp, *sp, *cc, *sc;
  A(cp, (size_t)p->NSEC) A(sp, (size_t)p->NSEC) A(cc, (size_t)p->NSEC) A(sc, (size_t)p->NSEC)
#undef A
  D.cos_pot = cp;
  D.sin_pot = sp;
  D.cos_cell = cc;
  D.sin_cell = sc;
  if ((st = make_tensor_maps(b, h, D))) return st;
#define U(ptr, vec)                            \
  if ((st = dupload(b, h, &(ptr), (vec)))) \
    return st;
  U(D.Rinf, h.t.Rinf) U(D.Rsup, h.t.Rsup) U(D.Rmed, h.t.Rmed) U(D.Surf, h.t.Surf) U(D.invRinf, h.t.invRinf)
  U(D.invSurf, h.t.invSurf) U(D.invRmed, h.t.invRmed) U(D.invdiffRsup, h.t.invdiffRsup)
  U(D.invdiffRmed, h.t.invdiffRmed) U(D.dxtheta, h.t.dxtheta) U(D.supp_torque, h.t.supp_torque)
  U(D.SigmaMed, h.t.SigmaMed) U(D.SigmaInf, h.t.SigmaInf) U(D.EnergyMed, h.t.EnergyMed)
  U(D.CoolingTimeMed, h.t.CoolingTimeMed) U(D.pow15, h.t.pow15) U(D.star_grad, h.t.star_grad)
  U(D.cfl_rdr, h.t.cfl_rdr) U(D.cfl_rdt, h.t.cfl_rdt) U(D.cfl_rmd, h.t.cfl_rmd)
#undef U
  // QplusMed is filled at initialisation (it needs the viscosity)
  float* qpm;
  if ((st = dalloc(b, h, &qpm, n1))) return st;
  D.QplusMed = qpm;
  if (p->SelfGravity) {
    st = sg_create(&h.sg, p, h.t, b->stream, &D, b->err);
    if (D.sg_accr) h.allocs.push_back(D.sg_accr);
    if (D.sg_acct) h.allocs.push_back(D.sg_acct);
    if (st) return st;
  }
  return FARGO_OK;
}

fargo_status make_tensor_maps(fargo_batch* b, DiskHost& h, DiskDev& D) {
  D.tmap = nullptr;
  const int nrad = h.p.NRAD, nsec = h.p.NSEC;
  if ((nsec & 3) != 0 || nsec < 64) return FARGO_OK;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensormap_encoder();
  if (!enc) return FARGO_OK;
  static_assert(sizeof(CUtensorMap) == 128, "three maps at 128-byte strides");
  CUtensorMap m[3];
  const float* base[3] = {D.dens, D.vrad, D.vtheta};
  const int rows[3] = {nrad, nrad + 1, nrad};
  const int box_rows[3] = {FARGO_TR_ROWS_D, FARGO_TR_ROWS_R, FARGO_TR_ROWS_T};
  for (int k = 0; k < 3; k++) {
    cuuint64_t dim[2] = {(cuuint64_t)nsec, (cuuint64_t)rows[k]};
    cuuint64_t stride[1] = {(cuuint64_t)nsec * sizeof(float)};
    cuuint32_t box[2] = {FARGO_TR_ROW, (cuuint32_t)box_rows[k]};
    cuuint32_t es[2] = {1, 1};
    CUresult r = enc(&m[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base[k]), dim, stride, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return FARGO_OK;  // staged by cp.async instead
  }
  CUtensorMap* dm = nullptr;
  fargo_status st = dalloc(b, h, &dm, 3);
  if (st) return st;
  CK(cudaMemcpy(dm, m, sizeof(m), cudaMemcpyHostToDevice));
  D.tmap = dm;
  return FARGO_OK;
}

DiskCtl ctl_header(const fargo_batch* b, int d, cudaError_t* e) {
  DiskCtl c;
  *e = cudaMemcpy(&c, b->d_ctl + d, sizeof(DiskCtl), cudaMemcpyDeviceToHost);
  return c;
}

fargo_status put_ctl_header(fargo_batch* b, int d, const DiskCtl& c) {
  CK(cudaMemcpyAsync(b->d_ctl + d, &c, sizeof(DiskCtl), cudaMemcpyHostToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return FARGO_OK;
}

void planets_to_ctl(const fargo_planets* pl, DiskCtl* c) {
  c->nb = pl->nb;
  for (int k = 0; k < pl->nb; k++) {
    c->mass[k] = pl->mass[k];
    c->x[k] = pl->x[k];
    c->y[k] = pl->y[k];
    c->vx[k] = pl->vx[k];
    c->vy[k] = pl->vy[k];
    c->feeldisk[k] = pl->feeldisk[k];
    c->feelothers[k] = pl->feelothers[k];
  }
}

void ctl_to_planets(const DiskCtl& c, const fargo_planets& names, fargo_planets* out) {
  *out = names;
  out->nb = c.nb;
  for (int k = 0; k < c.nb; k++) {
    out->mass[k] = c.mass[k];
    out->x[k] = c.x[k];
    out->y[k] = c.y[k];
    out->vx[k] = c.vx[k];
    out->vy[k] = c.vy[k];
    out->feeldisk[k] = c.feeldisk[k];
    out->feelothers[k] = c.feelothers[k];
  }
}

// The initialisation part of main() between InitGasDensity and the DT loop
// (Main.cu:292-344): self-gravity start-up, OmegaFrame, InitEuler's sound
// speed, viscosity and velocities.  dens/energy: NULL = the reference's
// axisymmetric profiles (InitGasDensity / InitGasEnergy, Pframeforce.cu:173-192).
fargo_status init_disk_state(fargo_batch* b, int d, const float* dens, const float* energy) {
  DiskHost& h = b->disks[d];
  DiskDev& D = h.dev;
  const fargo_params* p = &h.p;
  const int nrad = p->NRAD, nsec = p->NSEC;
  const size_t ng = (size_t)(nrad + 1) * nsec;
  std::vector<float> S(ng, 0.0f), E(ng, 0.0f);
  for (int i = 0; i < nrad; i++)
    for (int j = 0; j < nsec; j++) {
      S[(size_t)i * nsec + j] = h.t.SigmaMed[i];
      if (p->Adiabatic) E[(size_t)i * nsec + j] = h.t.EnergyMed[i];
    }
  if (dens) std::memcpy(S.data(), dens, sizeof(float) * ng);
  if (energy) std::memcpy(E.data(), energy, sizeof(float) * ng);
  CK(cudaMemcpyAsync(D.dens, S.data(), sizeof(float) * ng, cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(D.energy, E.data(), sizeof(float) * ng, cudaMemcpyHostToDevice, b->stream));
  float* scratch[] = {D.vrad, D.vtheta, D.vri, D.vti, D.trr, D.tpp, D.trp, D.qplus, D.a0, D.a1};
  for (float* f : scratch) CK(cudaMemsetAsync(f, 0, sizeof(float) * ng, b->stream));
  // scalars and planets
  DiskCtl c;
  std::memset(&c, 0, sizeof(DiskCtl));
  fargo_planets pl = h.planets0;
  c.PhysicalTime = 0.0f;
  c.PhysicalTimeInitial = 0.0f;
  planets_to_ctl(&pl, &c);
  D.HillRadius = pl.nb > 0 ? (float)(pl.x[0] * std::pow(pl.mass[0] / 3., 1. / 3.)) : 0.0f;  // Psys.cu:206
  fargo_status st;
  if ((st = put_ctl_header(b, d, c))) return st;
  CK(cudaMemcpy(b->d_disks + d, &D, sizeof(DiskDev), cudaMemcpyHostToDevice));
  if (p->SelfGravity) {
    // compute_selfgravity(init) + Init_planetarysys_withSG (Main.cu:302-329);
    // a radial stripe takes the whole disk's convolution on the whole
    // density (gathered into gv.dens by fargo_stripe_init_state), its
    // tables, and the profile's values at its own rings
    SelfGravity* sg = b->gsg ? b->gsg : h.sg;
    DiskDev* G = b->gsg ? &b->gv : &D;
    const HostTables& T = b->gsg ? b->gt : h.t;
    const int base = b->gsg ? b->stripe_base : 0;
    st = sg_accelerations(sg, b->bd, d, G, b->stream, b->err);
    if (st) return st;
    std::vector<float> axi(G->nrad);
    st = sg_axisymmetric(sg, G, axi.data(), b->stream, b->err);
    if (st) return st;
    for (int k = 0; k < pl.nb; k++) {
      float r, dist, ri, rip1, dr, sgacc;
      int ipl;
      r = pl.x[k];
      dist = (float)(r / (1. + p->ECCENTRICITY));
      ipl = 0;
      while (T.Rmed[ipl] <= dist) ipl++;
      ri = T.Rmed[ipl];
      rip1 = T.Rmed[ipl + 1];
      dr = rip1 - ri;
      sgacc = (dist - ri) * axi[ipl + 1] + (rip1 - dist) * axi[ipl];
      sgacc /= dr;
      pl.vy[k] *= (float)sqrtf(1. - dist * dist * sgacc);
    }
    planets_to_ctl(&pl, &c);
    // Init_azimutalvelocity_withSG (SourceEuler.cu:428-437)
    st = sg_init_vtheta(sg, &D, axi.data() + base, b->stream, b->err);
    if (st) return st;
  }
  // OmegaFrame (Main.cu:332-333)
  c.OmegaFrame = p->OMEGAFRAME;
  if (p->Corotating) c.OmegaFrame = host_get_psys_frequency(&pl);
  if ((st = put_ctl_header(b, d, c))) return st;
  // InitEuler's ComputeSoundSpeed, then Make1Dprofile(1) (SourceEuler.cu:199, Pframeforce.cu:242-245)
  fargo_launch_cs_isothermal(b->bd, d, b->stream);
  fargo_launch_cs_refresh(b->bd, d, b->stream);
  CK(cudaGetLastError());
  std::vector<float> csmean(nrad + 1, 0.0f);
  CK(cudaMemcpyAsync(csmean.data(), D.csmean, sizeof(float) * (nrad + 1), cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  // InitVelocities' viscosity table (Pframeforce.cu:262-265) and FillQplus (Theo.cu:299-311)
  std::vector<float> visc(nrad + 1, 0.0f), qpm(nrad + 1, 0.0f);
  for (int i = 0; i < nrad; i++) visc[i] = host_fviscosity(p, h.t, csmean.data(), h.t.Rmed[i], 0.0f, 0.0f);
  visc[nrad] = host_fviscosity(p, h.t, csmean.data(), h.t.Rmed[nrad - 1], 0.0f, 0.0f);
  if (p->Cooling)
    for (int i = 0; i < nrad; i++) {
      float r = h.t.Rmed[i];
      float vis = host_fviscosity(p, h.t, csmean.data(), r, 0.0f, 0.0f);
      qpm[i] = 2.25 * vis * p->SIGMA0 * std::pow(r, -p->SIGMASLOPE - 3.0);
    }
  CK(cudaMemcpyAsync(D.visc, visc.data(), sizeof(float) * (nrad + 1), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync((void*)D.QplusMed, qpm.data(), sizeof(float) * (nrad + 1), cudaMemcpyHostToDevice, b->stream));
  // constant sub-Keplerian speeds
  D.vkep_const = (!p->SelfGravity && p->LAMBDADOUBLING == 0.0f) ? 1 : 0;
  if (D.vkep_const) {
    double vin, vout;
    host_vkep(p, h.t, 0.0f, 0.0f, &vin, &vout);
    D.VKepIn = (float)vin;
    D.VKepOut = (float)vout;
  }
  CK(cudaMemcpyAsync(b->d_disks + d, &D, sizeof(DiskDev), cudaMemcpyHostToDevice, b->stream));
  // InitGasVelocitiesKernel
  fargo_launch_init_velocities(b->bd, d, (long long)(nrad + 1) * nsec, b->stream);
  CK(cudaGetLastError());
  // pressure of the initial state for the isothermal temperature output
  CK(cudaStreamSynchronize(b->stream));
  return FARGO_OK;
}

fargo_status build_graph(fargo_batch* b) {
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  if (!b->use_graph) return FARGO_OK;
  CK(cudaGraphCreate(&b->graph, 0));
  CK(cudaGraphConditionalHandleCreate(&b->handle, b->graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = b->handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, b->graph, nullptr, 0, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  CK(cudaStreamBeginCaptureToGraph(b->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  for (int d = 0; d < (int)b->disks.size(); d++)
    if (b->disks[d].sg) sg_capture_substep(b->disks[d].sg, b->bd, d, &b->disks[d].dev, b->stream);
  fargo_launch_substep(b->bd, b->handle, 1, b->stream, b->max_nsec, nullptr);
  cudaError_t ec = cudaStreamEndCapture(b->stream, &body);
  if (ec != cudaSuccess) return set_err(b, FARGO_ECUDA, "graph capture: %s", cudaGetErrorString(ec));
  CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return FARGO_OK;
}

// Segment widths chosen by the autotuner, kept for the life of the process
// per class of disk (NSEC, adiabatic, precision mode): a batch created later
// with disks of a tuned class starts from the tuned width.  The transport's
// results do not depend on the width (its arithmetic is contraction-free and
// per cell), only its speed does.
using SegKey = std::tuple<int, int, int>;
std::mutex g_seg_mutex;
std::map<SegKey, int> g_seg_cache;
SegKey seg_key(const DiskHost& h) { return SegKey(h.p.NSEC, h.p.Adiabatic ? 1 : 0, h.dev.accurate); }
void apply_seg_cache(fargo_batch* b) {
  std::lock_guard<std::mutex> lock(g_seg_mutex);
  for (auto& h : b->disks) {
    auto it = g_seg_cache.find(seg_key(h));
    if (it != g_seg_cache.end()) h.seg_out = it->second;
  }
}

// Transport work items of every disk: bands of FARGO_BAND rings, each in
// nseg near-equal azimuthal segments of at most the disk's seg_out source
// sectors (the sectors a band reads; each ring stores them shifted by its
// Nshift); isothermal and adiabatic disks in separate lists.  Sets each
// disk's item0 / nitems (host copy) and returns the widest segment.
int build_items(fargo_batch* b, std::vector<int4>& theta_iso, std::vector<int4>& theta_adi) {
  int seg_max = 0;
  theta_iso.clear();
  theta_adi.clear();
  for (int d = 0; d < (int)b->disks.size(); d++) {
    DiskHost& h = b->disks[d];
    const int nrad = h.p.NRAD, nsec = h.p.NSEC, seg_out = h.seg_out;
    std::vector<int4>& theta = h.p.Adiabatic ? theta_adi : theta_iso;
    h.dev.item0 = (int)theta.size();
    const int nseg = (nsec + seg_out - 1) / seg_out;
    int seg = (nsec + nseg - 1) / nseg;
    // segment starts on 4-sector boundaries when NSEC allows: the transport
    // kernel then stages its rows by 16-byte copies (seg_out is a multiple of 4)
    if ((nsec & 3) == 0 && (seg_out & 3) == 0) seg = (seg + 3) & ~3;
    for (int i = 0; i < nrad; i += FARGO_BAND) {
      for (int j0 = 0; j0 < nsec; j0 += seg) {
        int S = std::min(seg, nsec - j0);
        theta.push_back(make_int4(d, i, j0, S));
        seg_max = std::max(seg_max, S);
      }
    }
    h.dev.nitems = (int)theta.size() - h.dev.item0;
  }
  return seg_max;
}

// Replace the batch's transport items (device list, per-disk item0/nitems,
// grid) with those of the disks' current segment widths.
fargo_status install_items(fargo_batch* b) {
  std::vector<int4> theta_iso, theta_adi;
  int seg_max = build_items(b, theta_iso, theta_adi);
  CK(cudaStreamSynchronize(b->stream));
  if (b->d_theta) CK(cudaFree(b->d_theta));
  b->d_theta = nullptr;
  CK(cudaMalloc(&b->d_theta, sizeof(int4) * (theta_iso.size() + theta_adi.size() + 1)));
  if (!theta_iso.empty())
    CK(cudaMemcpy(b->d_theta, theta_iso.data(), sizeof(int4) * theta_iso.size(), cudaMemcpyHostToDevice));
  if (!theta_adi.empty())
    CK(cudaMemcpy(b->d_theta + theta_iso.size(), theta_adi.data(), sizeof(int4) * theta_adi.size(),
                  cudaMemcpyHostToDevice));
  for (int d = 0; d < (int)b->disks.size(); d++)
    CK(cudaMemcpy(&b->d_disks[d].item0, &b->disks[d].dev.item0, 2 * sizeof(int), cudaMemcpyHostToDevice));
  BatchDev& bd = b->bd;
  bd.theta_iso = b->d_theta;
  bd.theta_adi = b->d_theta + theta_iso.size();
  bd.ntheta_iso = (int)theta_iso.size();
  bd.ntheta_adi = (int)theta_adi.size();
  bd.theta_seg = seg_max;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
  long long tiles = 0;
  for (auto& h : b->disks) tiles += ((long long)h.dev.nrad * h.dev.nsec + FARGO_QTILE - 1) / FARGO_QTILE;
  CK(fargo_size_grids(bd, nsm, tiles, (int)(theta_iso.size() + theta_adi.size())));
  return FARGO_OK;
}

// CFL/force tile size of every disk of the batch: the small tile when the
// large one would give fewer than two tiles per SM over `cells` (the whole
// disk's cells for a radial stripe, so that its tiles are the whole disk's),
// and the batch's tile count.  Host copies only; the caller uploads.
void set_cfl_tiles(fargo_batch* b, long long cells, int device) {
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  const int tile = cells < 2LL * nsm * FARGO_CFL_TILE ? FARGO_CFL_TILE_SMALL : FARGO_CFL_TILE;
  b->bd.ncfl = 0;
  for (auto& h : b->disks) {
    h.dev.cfl_tile = tile;
    b->bd.ncfl += fargo_cfl_tiles_own(h.dev);
  }
}

fargo_status batch_create(fargo_batch* b, int n, const fargo_params* params, const fargo_planets* planets,
                          const double* const* radii, int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_err(b, FARGO_ENODEV, "no CUDA device available");
  if (device < 0) CK(cudaGetDevice(&device));
  CK(cudaSetDevice(device));
  b->device = device;
  CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  b->disks.resize(n);
  std::vector<long long> cell_off(n + 1, 0);
  std::vector<int> ring_off(n + 1, 0);
  std::vector<int4> theta_iso, theta_adi;
  int seg_max = 0, any_bc = 0, max_body = 1, src1_classes = 0;
  for (int d = 0; d < n; d++) {
    fargo_status st = check_params(b, &params[d], &planets[d]);
    if (st) return st;
    DiskHost& h = b->disks[d];
    h.p = params[d];
    h.planets0 = planets[d];
    st = alloc_disk(b, h, radii ? radii[d] : nullptr);
    if (st) return st;
    int nrad = h.p.NRAD, nsec = h.p.NSEC;
    h.dev.cell0 = cell_off[d];
    h.dev.ring0 = ring_off[d];
    cell_off[d + 1] = cell_off[d] + (long long)nrad * nsec;
    ring_off[d + 1] = ring_off[d] + nrad;
    b->ncell_ghost += (long long)(nrad + 1) * nsec;
    b->max_nsec = std::max(b->max_nsec, nsec);
    b->any_adiabatic |= h.p.Adiabatic;
    b->n_sg += h.p.SelfGravity ? 1 : 0;
    any_bc |= (h.p.OpenInner || h.p.NonReflecting || h.p.Evanescent) ? 1 : 0;
    src1_classes |= 1 << (2 * (h.p.Adiabatic ? 1 : 0) + (h.p.SelfGravity ? 1 : 0));
    max_body = std::max(max_body, body_count(&planets[d]));
  }
  apply_seg_cache(b);
  seg_max = build_items(b, theta_iso, theta_adi);
  CK(cudaMalloc(&b->d_disks, sizeof(DiskDev) * n));
  CK(cudaMalloc(&b->d_ctl, sizeof(DiskCtl) * n));
  CK(cudaMemsetAsync(b->d_ctl, 0, sizeof(DiskCtl) * n, b->stream));
  CK(cudaMalloc(&b->d_cell_off, sizeof(long long) * (n + 1)));
  CK(cudaMalloc(&b->d_ring_off, sizeof(int) * (n + 1)));
  CK(cudaMalloc(&b->d_theta, sizeof(int4) * (theta_iso.size() + theta_adi.size() + 1)));
  CK(cudaMalloc(&b->d_flags, sizeof(int) * 4));
  // compacted active lists: act[4] + 3 disk lists + 3 int prefix arrays, and the cell prefix
  CK(cudaMalloc(&b->d_act, sizeof(int) * (4 + 3 * n + 7 * (n + 1))));
  CK(cudaMemsetAsync(b->d_act, 0, sizeof(int) * (4 + 3 * n + 7 * (n + 1)), b->stream));
  CK(cudaMalloc(&b->d_act_cell, sizeof(long long) * (n + 1)));
  CK(cudaMemsetAsync(b->d_act_cell, 0, sizeof(long long) * (n + 1), b->stream));
  b->red_blocks = 296;
  CK(cudaMalloc(&b->d_red, sizeof(double) * b->red_blocks * 4 * FARGO_DIMFXY));
  CK(cudaMemcpyAsync(b->d_cell_off, cell_off.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->d_ring_off, ring_off.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, b->stream));
  if (!theta_iso.empty())
    CK(cudaMemcpyAsync(b->d_theta, theta_iso.data(), sizeof(int4) * theta_iso.size(), cudaMemcpyHostToDevice,
                       b->stream));
  if (!theta_adi.empty())
    CK(cudaMemcpyAsync(b->d_theta + theta_iso.size(), theta_adi.data(), sizeof(int4) * theta_adi.size(),
                       cudaMemcpyHostToDevice, b->stream));
  for (int d = 0; d < n; d++) b->disks[d].dev.ctl = b->d_ctl + d;
  set_cfl_tiles(b, cell_off[n], device);  // sets bd.ncfl
  for (int d = 0; d < n; d++)
    CK(cudaMemcpyAsync(b->d_disks + d, &b->disks[d].dev, sizeof(DiskDev), cudaMemcpyHostToDevice, b->stream));
  BatchDev& bd = b->bd;
  bd.ndisk = n;
  bd.any_bc = any_bc;
  bd.src1_classes = src1_classes;
  bd.max_body = max_body;
  bd.ncell = cell_off[n];
  bd.nring = ring_off[n];
  bd.cell_off = b->d_cell_off;
  bd.ring_off = b->d_ring_off;
  bd.disks = b->d_disks;
  bd.theta_iso = b->d_theta;
  bd.theta_adi = b->d_theta + theta_iso.size();
  bd.ntheta_iso = (int)theta_iso.size();
  bd.ntheta_adi = (int)theta_adi.size();
  bd.theta_seg = seg_max;
  bd.flags = b->d_flags;
  bd.act = b->d_act;
  bd.act_disk = b->d_act + 4;
  bd.act_iso_disk = bd.act_disk + n;
  bd.act_adi_disk = bd.act_iso_disk + n;
  bd.act_ring_off = bd.act_adi_disk + n;
  bd.act_iso_off = bd.act_ring_off + (n + 1);
  bd.act_adi_off = bd.act_iso_off + (n + 1);
  bd.act_grp_off = bd.act_adi_off + (n + 1);
  bd.act_tile_off = bd.act_grp_off + (n + 1);
  bd.act_ctile_off = bd.act_tile_off + (n + 1);
  bd.act_vtile_off = bd.act_ctile_off + (n + 1);
  bd.act_cell_off = b->d_act_cell;
  {
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    long long cg = (bd.ncell + 255) / 256;
    bd.cell_grid = (int)std::min<long long>(cg, (long long)nsm * 8);
    bd.ring_grid = std::min(bd.nring, nsm * 6);
    bd.item_grid = std::min((int)(theta_iso.size() + theta_adi.size()), nsm * 8);
    bd.grp_grid = std::min((bd.nring + (FARGO_RM_RINGS - 1) * (n + 1)) / FARGO_RM_RINGS, nsm * 8);
  }
  CK(fargo_kernel_attributes(b->max_nsec));
  {
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    long long tiles = 0;
    for (int d = 0; d < n; d++)
      tiles += ((long long)b->disks[d].dev.nrad * b->disks[d].dev.nsec + FARGO_QTILE - 1) / FARGO_QTILE;
    CK(fargo_size_grids(bd, nsm, tiles, (int)(theta_iso.size() + theta_adi.size())));
  }
  fargo_launch_sector_tables(bd, b->max_nsec, b->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(b->stream));
  for (int d = 0; d < n; d++) {
    fargo_status st = init_disk_state(b, d, nullptr, nullptr);
    if (st) return st;
  }
  return build_graph(b);
}

void batch_free(fargo_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto& h : b->disks) {
    if (h.sg) sg_destroy(h.sg);
    for (void* p : h.allocs) cudaFree(p);
  }
  if (b->gsg) sg_destroy(b->gsg);
  for (void* p : b->gallocs) cudaFree(p);
  void* ps[] = {b->d_disks, b->d_ctl, b->d_cell_off, b->d_ring_off, b->d_theta, b->d_flags, b->d_red,
                b->d_act, b->d_act_cell};
  for (void* p : ps)
    if (p) cudaFree(p);
  if (b->stream) cudaStreamDestroy(b->stream);
}

fargo_status advance_dt_async(fargo_batch* b) {
  if (b->stripe) return set_err(b, FARGO_EINVAL, "a radial stripe advances through fargo_stripe_*");
  CK(cudaSetDevice(b->device));
  fargo_launch_dt_begin(b->bd, b->stream);
  b->launches += 1;
  if (b->any_adiabatic) {
    fargo_launch_cs_refresh(b->bd, -1, b->stream);
    b->launches += 2;
  }
  CK(cudaGetLastError());
  if (b->use_graph) {
    CK(cudaGraphLaunch(b->exec, b->stream));
  } else {
    int more = 1;
    int* hflag = nullptr;
    CK(cudaMallocHost(&hflag, sizeof(int)));
    while (more) {
      for (int d = 0; d < (int)b->disks.size(); d++)
        if (b->disks[d].sg) sg_capture_substep(b->disks[d].sg, b->bd, d, &b->disks[d].dev, b->stream);
      fargo_launch_substep(b->bd, 0, 0, b->stream, b->max_nsec, nullptr);
      CK(cudaMemcpyAsync(hflag, b->d_flags, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
      CK(cudaStreamSynchronize(b->stream));
      more = *hflag;
    }
    cudaFreeHost(hflag);
  }
  return FARGO_OK;
}

fargo_status finish_dts(fargo_batch* b) {
  CK(cudaStreamSynchronize(b->stream));
  CK(cudaGetLastError());
  for (int d = 0; d < (int)b->disks.size(); d++) {
    cudaError_t e;
    DiskCtl c = ctl_header(b, d, &e);
    if (e != cudaSuccess) return set_err(b, FARGO_ECUDA, "ctl read: %s", cudaGetErrorString(e));
    if (c.error == 1) return set_err(b, FARGO_ENONFINITE, "disk %d: non-finite or non-positive CFL time step", d);
    if (c.error == 3)
      return set_err(b, FARGO_ETIMEOUT, "disk %d: a transport block gave up waiting for its staged rows", d);
    if (c.error == 2)
      return set_err(b, FARGO_ETIMEOUT, "disk %d: the DT needs more than %d substeps (the substep limit)", d,
                     b->disks[d].dev.max_sub);
  }
  return FARGO_OK;
}

}  // namespace

// =============================================================== C ABI

extern "C" {

int fargo_abi_version(void) { return FARGO_ABI_VERSION; }

fargo_status fargo_create(const fargo_params* p, const fargo_planets* planets, const double* radii, int device,
                          fargo_ctx** out) {
  if (!p || !planets || !out) return FARGO_EINVAL;
  *out = nullptr;
  fargo_ctx* ctx = new fargo_ctx();
  const double* r[1] = {radii};
  fargo_status st = batch_create(&ctx->b, 1, p, planets, r, device);
  *out = ctx;  // returned even on failure so that fargo_last_error can explain
  return st;
}

void fargo_destroy(fargo_ctx* ctx) {
  if (!ctx) return;
  batch_free(&ctx->b);
  delete ctx;
}

const char* fargo_last_error(const fargo_ctx* ctx) { return ctx ? ctx->b.err.c_str() : "null context"; }

fargo_status fargo_init_state(fargo_ctx* ctx, const float* dens, const float* energy) {
  if (!ctx) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  if (b->gsg)
    return set_err(b, FARGO_EINVAL, "a self-gravitating stripe starts from the whole density: fargo_stripe_init_state");
  CK(cudaSetDevice(b->device));
  return init_disk_state(b, 0, dens, energy);
}

fargo_status fargo_batch_init_state(fargo_batch* b, int disk, const float* dens, const float* energy) {
  if (!b || disk < 0 || disk >= (int)b->disks.size()) return FARGO_EINVAL;
  CK(cudaSetDevice(b->device));
  return init_disk_state(b, disk, dens, energy);
}

static fargo_status upload_impl(fargo_batch* b, int d, const float* dens, const float* vrad, const float* vtheta,
                                const float* energy) {
  if (!b || d < 0 || d >= (int)b->disks.size()) return FARGO_EINVAL;
  CK(cudaSetDevice(b->device));
  const DiskDev& D = b->disks[d].dev;
  size_t bytes = sizeof(float) * (size_t)(D.nrad + 1) * D.nsec;
  if (dens) CK(cudaMemcpyAsync(D.dens, dens, bytes, cudaMemcpyHostToDevice, b->stream));
  if (vrad) CK(cudaMemcpyAsync(D.vrad, vrad, bytes, cudaMemcpyHostToDevice, b->stream));
  if (vtheta) CK(cudaMemcpyAsync(D.vtheta, vtheta, bytes, cudaMemcpyHostToDevice, b->stream));
  if (energy) CK(cudaMemcpyAsync(D.energy, energy, bytes, cudaMemcpyHostToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return FARGO_OK;
}

// ComputeTemperatureFieldKernel (Kernels.cu:211-223) on the host copy.
static void temperature_host(const fargo_params* p, const float* dens, const float* pres, const float* energy,
                             float* T, size_t n, size_t nact) {
  for (size_t l = 0; l < n; l++) {
    if (l >= nact) {
      T[l] = 0.0f;
      continue;
    }
    if (!p->Adiabatic)
      T[l] = 1.0 / 1.0 * pres[l] / dens[l];
    else
      T[l] = 1.0 / 1.0 * (p->ADIABATICINDEX - 1.0) * energy[l] / dens[l];
  }
}

static fargo_status download_impl(fargo_batch* b, int d, float* dens, float* vrad, float* vtheta, float* energy,
                                  float* temperature, float* qplus) {
  if (!b || d < 0 || d >= (int)b->disks.size()) return FARGO_EINVAL;
  CK(cudaSetDevice(b->device));
  const DiskHost& h = b->disks[d];
  const DiskDev& D = h.dev;
  size_t n = (size_t)(D.nrad + 1) * D.nsec;
  size_t bytes = sizeof(float) * n;
  std::vector<float> S, P, E;
  if (dens) CK(cudaMemcpyAsync(dens, D.dens, bytes, cudaMemcpyDeviceToHost, b->stream));
  if (vrad) CK(cudaMemcpyAsync(vrad, D.vrad, bytes, cudaMemcpyDeviceToHost, b->stream));
  if (vtheta) CK(cudaMemcpyAsync(vtheta, D.vtheta, bytes, cudaMemcpyDeviceToHost, b->stream));
  if (energy) CK(cudaMemcpyAsync(energy, D.energy, bytes, cudaMemcpyDeviceToHost, b->stream));
  if (qplus) {
    if (h.p.Adiabatic)
      CK(cudaMemcpyAsync(qplus, D.qplus, bytes, cudaMemcpyDeviceToHost, b->stream));
    else
      std::memset(qplus, 0, bytes);
  }
  if (temperature) {
    S.resize(n);
    P.resize(n);
    E.resize(n);
    CK(cudaMemcpyAsync(S.data(), D.dens, bytes, cudaMemcpyDeviceToHost, b->stream));
    CK(cudaMemcpyAsync(P.data(), D.pres, bytes, cudaMemcpyDeviceToHost, b->stream));
    CK(cudaMemcpyAsync(E.data(), D.energy, bytes, cudaMemcpyDeviceToHost, b->stream));
  }
  CK(cudaStreamSynchronize(b->stream));
  if (temperature) temperature_host(&h.p, S.data(), P.data(), E.data(), temperature, n, (size_t)D.nrad * D.nsec);
  return FARGO_OK;
}

fargo_status fargo_upload(fargo_ctx* ctx, const float* dens, const float* vrad, const float* vtheta,
                          const float* energy) {
  if (!ctx) return FARGO_EINVAL;
  return upload_impl(&ctx->b, 0, dens, vrad, vtheta, energy);
}

fargo_status fargo_download(fargo_ctx* ctx, float* dens, float* vrad, float* vtheta, float* energy,
                            float* temperature, float* qplus) {
  if (!ctx) return FARGO_EINVAL;
  return download_impl(&ctx->b, 0, dens, vrad, vtheta, energy, temperature, qplus);
}

// ---------------------------------------------------------------- checkpoints

// Everything a later DT reads from the device that the next DT does not
// rebuild itself: the control block (time, frame, planets, DT bookkeeping),
// the state fields with their ghost rows, the temperature-output pressure,
// Q+, the adiabatic sound speed and the per-ring sound speed, mean sound
// speed and viscosity.
struct CkptPart {
  void* dev;
  size_t bytes;
};
static std::vector<CkptPart> ckpt_parts(fargo_batch* b, int d) {
  const DiskHost& h = b->disks[d];
  const DiskDev& D = h.dev;
  const size_t ng = sizeof(float) * (size_t)(D.nrad + 1) * D.nsec, n1 = sizeof(float) * (size_t)(D.nrad + 1);
  std::vector<CkptPart> v = {{b->d_ctl + d, sizeof(DiskCtl)}, {D.dens, ng},  {D.vrad, ng},    {D.vtheta, ng},
                             {D.energy, ng},                 {D.pres, ng},  {D.qplus, ng},   {D.visc, n1},
                             {D.cs_ring, n1},                {D.csmean, n1}};
  if (h.p.Adiabatic) v.push_back({D.cs, ng});
  return v;
}
static const unsigned kCkptMagic = 0x43324246u;  // "FB2C"
struct CkptHeader {
  unsigned magic, version;
  int nrad, nsec, adiabatic, ctl_bytes;
};
static size_t ckpt_bytes(fargo_batch* b, int d) {
  size_t n = sizeof(CkptHeader);
  for (auto& p : ckpt_parts(b, d)) n += p.bytes;
  return n;
}

size_t fargo_checkpoint_bytes(fargo_ctx* ctx) { return ctx ? ckpt_bytes(&ctx->b, 0) : 0; }

fargo_status fargo_checkpoint_save(fargo_ctx* ctx, void* buf, size_t bytes) {
  if (!ctx || !buf) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  if (bytes < ckpt_bytes(b, 0)) return set_err(b, FARGO_EINVAL, "checkpoint buffer too small");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  const DiskHost& h = b->disks[0];
  CkptHeader hd = {kCkptMagic, 1u, h.p.NRAD, h.p.NSEC, h.p.Adiabatic, (int)sizeof(DiskCtl)};
  char* o = static_cast<char*>(buf);
  std::memcpy(o, &hd, sizeof(hd));
  o += sizeof(hd);
  for (auto& p : ckpt_parts(b, 0)) {
    CK(cudaMemcpy(o, p.dev, p.bytes, cudaMemcpyDeviceToHost));
    o += p.bytes;
  }
  return FARGO_OK;
}

fargo_status fargo_checkpoint_load(fargo_ctx* ctx, const void* buf, size_t bytes) {
  if (!ctx || !buf) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  const DiskHost& h = b->disks[0];
  CkptHeader hd;
  if (bytes < sizeof(hd)) return set_err(b, FARGO_EINVAL, "checkpoint truncated");
  std::memcpy(&hd, buf, sizeof(hd));
  if (hd.magic != kCkptMagic || hd.version != 1u)
    return set_err(b, FARGO_EINVAL, "not a checkpoint of this library");
  if (hd.nrad != h.p.NRAD || hd.nsec != h.p.NSEC || hd.adiabatic != h.p.Adiabatic ||
      hd.ctl_bytes != (int)sizeof(DiskCtl))
    return set_err(b, FARGO_EINVAL, "checkpoint of a different grid or build (%dx%d)", hd.nrad, hd.nsec);
  if (bytes < ckpt_bytes(b, 0)) return set_err(b, FARGO_EINVAL, "checkpoint truncated");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  const char* in = static_cast<const char*>(buf) + sizeof(hd);
  for (auto& p : ckpt_parts(b, 0)) {
    CK(cudaMemcpy(p.dev, in, p.bytes, cudaMemcpyHostToDevice));
    in += p.bytes;
  }
  return FARGO_OK;
}

static fargo_status get_planets_impl(fargo_batch* b, int d, fargo_planets* out) {
  if (!b || !out || d < 0 || d >= (int)b->disks.size()) return FARGO_EINVAL;
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  cudaError_t e;
  DiskCtl c = ctl_header(b, d, &e);
  if (e != cudaSuccess) return set_err(b, FARGO_ECUDA, "%s", cudaGetErrorString(e));
  ctl_to_planets(c, b->disks[d].planets0, out);
  return FARGO_OK;
}

fargo_status fargo_get_planets(fargo_ctx* ctx, fargo_planets* out) {
  if (!ctx) return FARGO_EINVAL;
  return get_planets_impl(&ctx->b, 0, out);
}

fargo_status fargo_set_planets(fargo_ctx* ctx, const fargo_planets* in) {
  if (!ctx || !in || in->nb != ctx->b.disks[0].planets0.nb) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  cudaError_t e;
  DiskCtl c = ctl_header(b, 0, &e);
  if (e != cudaSuccess) return set_err(b, FARGO_ECUDA, "%s", cudaGetErrorString(e));
  if (body_count(in) > FARGO_MAXBODY) return set_err(b, FARGO_EINVAL, "at most %d planets may feel the disk", FARGO_MAXBODY - 1);
  planets_to_ctl(in, &c);
  fargo_status st = put_ctl_header(b, 0, c);
  if (st) return st;
  if (body_count(in) > b->bd.max_body) {  // the force kernel was built for fewer bodies
    b->bd.max_body = FARGO_MAXBODY;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
    int per = 1;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fargo_cfl_kernel(FARGO_MAXBODY), 256, 0));
    b->bd.g_cfl = std::max(1, std::min(b->bd.ncfl, nsm * std::max(per, 1)));
    return build_graph(b);
  }
  return FARGO_OK;
}

fargo_status fargo_advance_dt(fargo_ctx* ctx, int* nsub_out) {
  if (!ctx) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  fargo_status st = advance_dt_async(b);
  if (st) return st;
  st = finish_dts(b);
  if (st) return st;
  if (nsub_out) {
    cudaError_t e;
    DiskCtl c = ctl_header(b, 0, &e);
    *nsub_out = c.nsub;
  }
  return FARGO_OK;
}

fargo_status fargo_advance(fargo_ctx* ctx, int ndt) {
  if (!ctx) return FARGO_EINVAL;
  return fargo_batch_advance(&ctx->b, ndt);
}

fargo_status fargo_sync(fargo_ctx* ctx) {
  if (!ctx) return FARGO_EINVAL;
  return finish_dts(&ctx->b);
}

fargo_status fargo_advance_async(fargo_ctx* ctx, int ndt) {
  if (!ctx) return FARGO_EINVAL;
  for (int k = 0; k < ndt; k++) {
    fargo_status st = advance_dt_async(&ctx->b);
    if (st) return st;
  }
  return FARGO_OK;
}

static fargo_status disk_force_impl(fargo_batch* b, int d, double x, double y, double rsmoothing, double mass,
                                    int dimfxy, double* gf) {
  if (!b || !gf || dimfxy != FARGO_DIMFXY) return set_err(b, FARGO_EINVAL, "dimfxy must be %d", FARGO_DIMFXY);
  CK(cudaSetDevice(b->device));
  // ComputeForce (Force.cu:311-312): a and rh in double, kernel arguments float
  double a = std::sqrt(x * x + y * y);
  double rh = std::pow(mass / 3., 1. / 3.) * a + 1e-15;
  fargo_launch_disk_force(b->bd, d, (float)x, (float)y, (float)rsmoothing, (float)rh, (float)a, b->d_red,
                          b->red_blocks, b->stream);
  CK(cudaGetLastError());
  std::vector<double> part((size_t)b->red_blocks * 4 * FARGO_DIMFXY);
  CK(cudaMemcpyAsync(part.data(), b->d_red, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  b->launches += 1;
  for (int q = 0; q < 4 * FARGO_DIMFXY; q++) {
    double s = 0;
    for (int k = 0; k < b->red_blocks; k++) s += part[(size_t)k * 4 * FARGO_DIMFXY + q];
    gf[q] = s;
  }
  return FARGO_OK;
}

fargo_status fargo_disk_force(fargo_ctx* ctx, double x, double y, double rsmoothing, double mass, int dimfxy,
                              double* globalforce) {
  if (!ctx) return FARGO_EINVAL;
  return disk_force_impl(&ctx->b, 0, x, y, rsmoothing, mass, dimfxy, globalforce);
}

fargo_status fargo_sg_accelerations(fargo_ctx* ctx, float* accr, float* acct) {
  if (!ctx || !accr || !acct) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  DiskHost& h = b->disks[0];
  if (!h.sg) return set_err(b, FARGO_EINVAL, "fargo_sg_accelerations: the run has no self-gravity");
  if (b->stripe) return set_err(b, FARGO_EINVAL, "fargo_sg_accelerations: not on a radial stripe");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  fargo_status st = sg_accelerations(h.sg, b->bd, 0, &h.dev, b->stream, b->err);
  if (st) return st;
  size_t n = (size_t)h.dev.nrad * h.dev.nsec;
  CK(cudaMemcpy(accr, h.dev.sg_accr, sizeof(float) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(acct, h.dev.sg_acct, sizeof(float) * n, cudaMemcpyDeviceToHost));
  return FARGO_OK;
}

static fargo_status scalars_impl(fargo_batch* b, int d, fargo_scalars* out) {
  if (!b || !out || d < 0 || d >= (int)b->disks.size()) return FARGO_EINVAL;
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  cudaError_t e;
  DiskCtl c = ctl_header(b, d, &e);
  if (e != cudaSuccess) return set_err(b, FARGO_ECUDA, "%s", cudaGetErrorString(e));
  fargo_launch_diagnostics(b->bd, d, b->d_red, b->red_blocks, b->stream);
  CK(cudaGetLastError());
  std::vector<double> part((size_t)b->red_blocks * 3);
  CK(cudaMemcpyAsync(part.data(), b->d_red, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  b->launches += 1;
  double m = 0, am = 0, hill = 0;
  for (int k = 0; k < b->red_blocks; k++) {
    m += part[3 * k];
    am += part[3 * k + 1];
    hill += part[3 * k + 2];
  }
  std::memset(out, 0, sizeof(*out));
  out->physical_time = c.PhysicalTime;
  out->omega_frame = c.OmegaFrame;
  out->mdcp1 = (float)hill;
  out->lost_mass = c.LostMass;
  out->nsub_last_dt = c.nsub;
  out->nsub_total = c.nsub_total;
  out->mass = m;
  out->angular_momentum = am;
  out->last_dt = c.dt;
  return FARGO_OK;
}

fargo_status fargo_get_scalars(fargo_ctx* ctx, fargo_scalars* out) {
  if (!ctx) return FARGO_EINVAL;
  return scalars_impl(&ctx->b, 0, out);
}

fargo_status fargo_get_substep_log(fargo_ctx* ctx, int cap, int* nshift, double* dt, int* nsub) {
  if (!ctx) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  cudaError_t e;
  DiskCtl c = ctl_header(b, 0, &e);
  if (e != cudaSuccess) return set_err(b, FARGO_ECUDA, "%s", cudaGetErrorString(e));
  int n = std::min(c.nsub, std::min(cap, FARGO_MAXLOG));
  const DiskDev& D = b->disks[0].dev;
  if (nshift && n > 0)
    CK(cudaMemcpy(nshift, D.log_nshift, sizeof(int) * (size_t)n * D.nrad, cudaMemcpyDeviceToHost));
  if (dt && n > 0)
    CK(cudaMemcpy(dt, D.log_dt, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (nsub) *nsub = c.nsub;
  return FARGO_OK;
}

long long fargo_kernel_launches(const fargo_ctx* ctx) { return ctx ? ctx->b.launches : 0; }

// ---------------------------------------------------------------- batches

fargo_status fargo_batch_create(int n, const fargo_params* params, const fargo_planets* planets, int device,
                                fargo_batch** out) {
  if (n < 1 || !params || !planets || !out) return FARGO_EINVAL;
  fargo_batch* b = new fargo_batch();
  fargo_status st = batch_create(b, n, params, planets, nullptr, device);
  *out = b;
  return st;
}

void fargo_batch_destroy(fargo_batch* b) {
  if (!b) return;
  batch_free(b);
  delete b;
}

const char* fargo_batch_last_error(const fargo_batch* b) { return b ? b->err.c_str() : "null batch"; }

fargo_status fargo_batch_upload(fargo_batch* b, int disk, const float* dens, const float* vrad, const float* vtheta,
                                const float* energy) {
  return upload_impl(b, disk, dens, vrad, vtheta, energy);
}

fargo_status fargo_batch_download(fargo_batch* b, int disk, float* dens, float* vrad, float* vtheta, float* energy) {
  return download_impl(b, disk, dens, vrad, vtheta, energy, nullptr, nullptr);
}

fargo_status fargo_batch_advance(fargo_batch* b, int ndt) {
  if (!b || ndt < 0) return FARGO_EINVAL;
  for (int k = 0; k < ndt; k++) {
    fargo_status st = advance_dt_async(b);
    if (st) return st;
  }
  return finish_dts(b);
}

fargo_status fargo_batch_advance_async(fargo_batch* b, int ndt) {
  if (!b || ndt < 0) return FARGO_EINVAL;
  for (int k = 0; k < ndt; k++) {
    fargo_status st = advance_dt_async(b);
    if (st) return st;
  }
  return FARGO_OK;
}

fargo_status fargo_batch_sync(fargo_batch* b) {
  if (!b) return FARGO_EINVAL;
  return finish_dts(b);
}

fargo_status fargo_batch_get_scalars(fargo_batch* b, int disk, fargo_scalars* out) {
  return scalars_impl(b, disk, out);
}

fargo_status fargo_batch_get_planets(fargo_batch* b, int disk, fargo_planets* out) {
  return get_planets_impl(b, disk, out);
}

long long fargo_batch_kernel_launches(const fargo_batch* b) { return b ? b->launches : 0; }

void* fargo_batch_stream(fargo_batch* b) { return b ? (void*)b->stream : nullptr; }
void* fargo_stream(fargo_ctx* ctx) { return ctx ? (void*)ctx->b.stream : nullptr; }
fargo_batch* fargo_ctx_batch(fargo_ctx* ctx) { return ctx ? &ctx->b : nullptr; }

// Asynchronous copies (no wait): the host buffers must stay valid and, to
// overlap, be page-locked; pair with fargo_batch_sync.
fargo_status fargo_batch_upload_async(fargo_batch* b, int d, const float* dens, const float* vrad,
                                      const float* vtheta, const float* energy) {
  if (!b || d < 0 || d >= (int)b->disks.size()) return FARGO_EINVAL;
  const DiskDev& D = b->disks[d].dev;
  size_t bytes = sizeof(float) * (size_t)(D.nrad + 1) * D.nsec;
  if (dens) CK(cudaMemcpyAsync(D.dens, dens, bytes, cudaMemcpyHostToDevice, b->stream));
  if (vrad) CK(cudaMemcpyAsync(D.vrad, vrad, bytes, cudaMemcpyHostToDevice, b->stream));
  if (vtheta) CK(cudaMemcpyAsync(D.vtheta, vtheta, bytes, cudaMemcpyHostToDevice, b->stream));
  if (energy) CK(cudaMemcpyAsync(D.energy, energy, bytes, cudaMemcpyHostToDevice, b->stream));
  return FARGO_OK;
}

fargo_status fargo_batch_download_async(fargo_batch* b, int d, float* dens, float* vrad, float* vtheta,
                                        float* energy) {
  if (!b || d < 0 || d >= (int)b->disks.size()) return FARGO_EINVAL;
  const DiskDev& D = b->disks[d].dev;
  size_t bytes = sizeof(float) * (size_t)(D.nrad + 1) * D.nsec;
  if (dens) CK(cudaMemcpyAsync(dens, D.dens, bytes, cudaMemcpyDeviceToHost, b->stream));
  if (vrad) CK(cudaMemcpyAsync(vrad, D.vrad, bytes, cudaMemcpyDeviceToHost, b->stream));
  if (vtheta) CK(cudaMemcpyAsync(vtheta, D.vtheta, bytes, cudaMemcpyDeviceToHost, b->stream));
  if (energy) CK(cudaMemcpyAsync(energy, D.energy, bytes, cudaMemcpyDeviceToHost, b->stream));
  return FARGO_OK;
}

// Per-kernel timing: ndt DTs in host-loop mode with a CUDA event before and
// after every kernel of every substep.  ms[k] accumulates the time of
// substep kernel k (fargo_profile_kernel_name order), the last slot the
// self-gravity pipeline; *nsub receives the substeps run.
int fargo_profile_kernel_count(void) { return FARGO_NKERNELS + 1; }

fargo_status fargo_batch_profile(fargo_batch* b, int ndt, double* ms, int* nsub) {
  if (!b || !ms || ndt < 1 || b->stripe) return FARGO_EINVAL;
  CK(cudaSetDevice(b->device));
  const int NK = FARGO_NKERNELS;
  cudaEvent_t ev[FARGO_NKERNELS + 1], sg0, sg1;
  for (int k = 0; k <= NK; k++) CK(cudaEventCreate(&ev[k]));
  CK(cudaEventCreate(&sg0));
  CK(cudaEventCreate(&sg1));
  for (int k = 0; k <= NK; k++) ms[k] = 0.0;
  int* hflag = nullptr;
  CK(cudaMallocHost(&hflag, sizeof(int)));
  int subs = 0;
  for (int t = 0; t < ndt; t++) {
    fargo_launch_dt_begin(b->bd, b->stream);
    if (b->any_adiabatic) fargo_launch_cs_refresh(b->bd, -1, b->stream);
    int more = 1;
    while (more) {
      CK(cudaEventRecord(sg0, b->stream));
      for (int d = 0; d < (int)b->disks.size(); d++)
        if (b->disks[d].sg) sg_capture_substep(b->disks[d].sg, b->bd, d, &b->disks[d].dev, b->stream);
      CK(cudaEventRecord(sg1, b->stream));
      fargo_launch_substep(b->bd, 0, 0, b->stream, b->max_nsec, nullptr, ev);
      CK(cudaMemcpyAsync(hflag, b->d_flags, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
      CK(cudaStreamSynchronize(b->stream));
      for (int k = 0; k < NK; k++) {
        float x = 0;
        CK(cudaEventElapsedTime(&x, ev[k], ev[k + 1]));
        ms[k] += x;
      }
      float y = 0;
      CK(cudaEventElapsedTime(&y, sg0, sg1));
      ms[NK] += y;
      subs++;
      more = *hflag;
    }
  }
  cudaFreeHost(hflag);
  for (int k = 0; k <= NK; k++) cudaEventDestroy(ev[k]);
  cudaEventDestroy(sg0);
  cudaEventDestroy(sg1);
  if (nsub) *nsub = subs;
  return finish_dts(b);
}

const char* fargo_profile_kernel_name(int k) {
  return k == FARGO_NKERNELS ? "self_gravity" : fargo_substep_kernel_name(k);
}

// Launch counting needs the substep counts: total launches of the batch's
// own kernels so far (pre-DT launches + substeps x kernels per substep).
long long fargo_batch_count_launches(fargo_batch* b) {
  if (!b) return 0;
  cudaStreamSynchronize(b->stream);
  long long subs = 0;
  for (int d = 0; d < (int)b->disks.size(); d++) {
    cudaError_t e;
    DiskCtl c = ctl_header(b, d, &e);
    subs = std::max<long long>(subs, c.nsub_total);
  }
  return b->launches + subs * fargo_substep_launches(b->bd);
}

fargo_status fargo_set_graph_mode(fargo_ctx* ctx, int use_graph) {
  if (!ctx) return FARGO_EINVAL;
  return fargo_batch_set_graph_mode(&ctx->b, use_graph);
}

// Autotuner of the transport tile: the azimuthal segment width (output
// sectors per CTA) decides the threads left idle in the last segment of a
// ring, the halo overhead and the number of CTAs.  Each candidate is
// installed and the transport kernels are timed on the current state (they
// write only scratch); the fastest stays and the graph is rebuilt.
fargo_status batch_autotune(fargo_batch* b, int reps, int* chosen) {
  if (!b || reps < 1) return FARGO_EINVAL;
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  static const int cand[] = {96, 128, 160, 192, 224, FARGO_SEG_MAX};
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  // install the disks' current widths and time the transport kernels on the
  // current state (every disk active, the compacted item prefixes rebuilt
  // for these items, as the next DT starts; the kernels write only scratch)
  auto timed = [&](float* ms) -> fargo_status {
    fargo_status st = install_items(b);
    if (st) return st;
    fargo_launch_dt_begin(b->bd, b->stream);
    fargo_launch_transport(b->bd, b->stream);
    CK(cudaEventRecord(e0, b->stream));
    for (int r = 0; r < reps; r++) fargo_launch_transport(b->bd, b->stream);
    CK(cudaEventRecord(e1, b->stream));
    CK(cudaEventSynchronize(e1));
    CK(cudaGetLastError());
    CK(cudaEventElapsedTime(ms, e0, e1));
    return FARGO_OK;
  };
  // the classes of disk, largest share of cells first
  std::map<SegKey, long long> cells;
  for (auto& h : b->disks) cells[seg_key(h)] += (long long)h.p.NRAD * h.p.NSEC;
  std::vector<std::pair<long long, SegKey>> classes;
  for (auto& kv : cells) classes.push_back({kv.second, kv.first});
  std::sort(classes.begin(), classes.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
  auto set_class = [&](const SegKey& k, int w) {
    for (auto& h : b->disks)
      if (seg_key(h) == k) h.seg_out = w;
  };
  // one width for every disk, then each class in turn with the others fixed
  float best_ms = 1e30f;
  int best = FARGO_SEG_OUT;
  fargo_status st = FARGO_OK;
  for (int c : cand) {
    for (auto& h : b->disks) h.seg_out = c;
    float ms = 0.0f;
    if ((st = timed(&ms))) return st;
    if (ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  for (auto& h : b->disks) h.seg_out = best;
  if (classes.size() > 1) {
    for (auto& cl : classes) {
      int keep = best;
      for (int c : cand) {
        if (c == keep) continue;
        set_class(cl.second, c);
        float ms = 0.0f;
        if ((st = timed(&ms))) return st;
        if (ms < best_ms) {
          best_ms = ms;
          keep = c;
        }
      }
      set_class(cl.second, keep);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if ((st = install_items(b))) return st;
  {
    std::lock_guard<std::mutex> lock(g_seg_mutex);
    for (auto& h : b->disks) g_seg_cache[seg_key(h)] = h.seg_out;
  }
  b->seg_out = best;
  if (chosen) {  // the width of the class with the most cells
    for (auto& h : b->disks)
      if (seg_key(h) == classes[0].second) *chosen = h.seg_out;
  }
  return build_graph(b);
}

fargo_status fargo_batch_segments(fargo_batch* b, int cap, int* seg_per_disk) {
  if (!b || cap < 0 || (cap && !seg_per_disk)) return FARGO_EINVAL;
  for (int d = 0; d < (int)b->disks.size() && d < cap; d++) seg_per_disk[d] = b->disks[d].seg_out;
  return FARGO_OK;
}

fargo_status fargo_batch_autotune(fargo_batch* b, int reps, int* seg_out) { return batch_autotune(b, reps, seg_out); }

fargo_status fargo_autotune(fargo_ctx* ctx, int reps, int* seg_out) {
  if (!ctx) return FARGO_EINVAL;
  return batch_autotune(&ctx->b, reps, seg_out);
}

fargo_status fargo_batch_set_max_substeps(fargo_batch* b, int n) {
  if (!b || n < 1) return FARGO_EINVAL;
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  for (int d = 0; d < (int)b->disks.size(); d++) {
    b->disks[d].dev.max_sub = n;
    CK(cudaMemcpy(&b->d_disks[d].max_sub, &n, sizeof(int), cudaMemcpyHostToDevice));
  }
  return FARGO_OK;
}

fargo_status fargo_batch_set_precision(fargo_batch* b, int mode) {
  if (!b || (mode != FARGO_PRECISION_REFERENCE && mode != FARGO_PRECISION_ACCURATE)) return FARGO_EINVAL;
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  const int acc = mode == FARGO_PRECISION_ACCURATE;
  for (int d = 0; d < (int)b->disks.size(); d++) {
    DiskHost& h = b->disks[d];
    h.dev.accurate = acc;
    CK(cudaMemcpy(&b->d_disks[d].accurate, &acc, sizeof(int), cudaMemcpyHostToDevice));
    if (h.sg) {
      fargo_status st = sg_tabulate(h.sg, h.t, acc, b->stream, b->err);
      if (st) return st;
    }
  }
  if (b->gsg) {
    b->gv.accurate = acc;
    fargo_status st = sg_tabulate(b->gsg, b->gt, acc, b->stream, b->err);
    if (st) return st;
  }
  b->bd.accurate = acc;  // the accurate mode runs the kernel set without fused multiply-adds
  apply_seg_cache(b);    // the segment widths tuned for this mode, if any
  fargo_status st = install_items(b);
  if (st) return st;
  return build_graph(b);  // whose launches the graph must capture
}

fargo_status fargo_set_precision(fargo_ctx* ctx, int mode) {
  if (!ctx) return FARGO_EINVAL;
  return fargo_batch_set_precision(&ctx->b, mode);
}

fargo_status fargo_set_max_substeps(fargo_ctx* ctx, int n) {
  if (!ctx) return FARGO_EINVAL;
  return fargo_batch_set_max_substeps(&ctx->b, n);
}

fargo_status fargo_batch_set_graph_mode(fargo_batch* b, int use_graph) {
  if (!b) return FARGO_EINVAL;
  if (b->stripe && use_graph) return set_err(b, FARGO_EINVAL, "a radial stripe runs its substeps from the host");
  b->use_graph = use_graph != 0;
  return build_graph(b);
}

// ------------------------------------------------------------ radial stripes
// One stripe of a disk decomposed by rings over several contexts (usually
// one per GPU): its own rings ring_lo .. ring_hi-1 plus `ghost` rings on
// each side (fewer at the disk's edges), computed as a disk of its own on the
// whole disk's radii.  After every substep the ghost rings are refreshed from
// the neighbours' own rings (halo pack / unpack), so that the boundary
// treatment at the stripe's cut edges, which is not the whole disk's, only
// ever reaches ghost rings.  The substep's scalars come from every stripe's
// partials (fargo_stripe_forces, gathered by the caller, then
// fargo_stripe_substep), so all stripes take the same dt and planet update.

static int stripe_nfields(const fargo_batch* b) { return b->disks[0].p.Adiabatic ? 4 : 3; }

fargo_status fargo_stripe_create(const fargo_params* p, const fargo_planets* planets, const double* radii,
                                 int ring_lo, int ring_hi, int ghost, int device, fargo_ctx** out) {
  if (!p || !planets || !out) return FARGO_EINVAL;
  *out = nullptr;
  fargo_ctx* ctx = new fargo_ctx();
  *out = ctx;  // returned even on failure so that fargo_last_error can explain
  fargo_batch* b = &ctx->b;
  const int NRAD = p->NRAD;
  if (ring_lo < 0 || ring_hi > NRAD || ring_lo >= ring_hi)
    return set_err(b, FARGO_EINVAL, "stripe rings [%d, %d) outside the disk's %d rings", ring_lo, ring_hi, NRAD);
  if (ghost < 1 || ghost > FARGO_STRIPE_MAX_GHOST)
    return set_err(b, FARGO_EINVAL, "ghost rings must be 1 .. %d", FARGO_STRIPE_MAX_GHOST);
  if (ring_hi - ring_lo < ghost && !(ring_lo == 0 && ring_hi == NRAD))
    return set_err(b, FARGO_EINVAL, "a stripe needs at least as many own rings (%d) as ghost rings (%d)",
                   ring_hi - ring_lo, ghost);
  if (p->OpenInner || p->NonReflecting || p->Evanescent)
    return set_err(b, FARGO_EINVAL, "radial stripes need RIGID inner and outer boundaries");
  std::vector<double> R(NRAD + 1);
  if (radii) {
    std::memcpy(R.data(), radii, sizeof(double) * (NRAD + 1));
  } else {
    fargo_status st = fargo_grid_radii(p, R.data());
    if (st) return set_err(b, st, "grid radii");
  }
  const int base = std::max(0, ring_lo - ghost), top = std::min(NRAD, ring_hi + ghost);
  fargo_params q = *p;
  q.NRAD = top - base;
  q.RMIN = (float)R[base];
  q.RMAX = (float)R[top];
  const double* r[1] = {R.data() + base};
  fargo_status st = batch_create(b, 1, &q, planets, r, device);
  if (st) return st;
  DiskDev& D = b->disks[0].dev;
  D.own_lo = ring_lo - base;
  D.own_hi = ring_hi - base;
  D.stripe = 1;
  b->stripe = 1;
  b->stripe_base = base;
  b->stripe_nrad = NRAD;
  b->ghost_lo = ring_lo - base;
  b->ghost_hi = top - ring_hi;
  set_cfl_tiles(b, (long long)NRAD * p->NSEC, b->device);  // the whole disk's tiles; sets bd.ncfl
  CK(cudaMemcpy(b->d_disks, &D, sizeof(DiskDev), cudaMemcpyHostToDevice));
  if (p->SelfGravity) {
    // the whole disk's convolution: a view of the whole grid with its own
    // density buffer and ring tables, this stripe's control block
    host_build_tables(p, R.data(), &b->gt);
    DiskDev& G = b->gv;
    G = D;
    G.nrad = NRAD;
    G.own_lo = 0;
    G.own_hi = NRAD;
    G.sg_accr = G.sg_acct = nullptr;
    float *gd = nullptr, *gr = nullptr;
    CK(cudaMalloc(&gd, sizeof(float) * (size_t)NRAD * p->NSEC));
    b->gallocs.push_back(gd);
    CK(cudaMalloc(&gr, sizeof(float) * (NRAD + 1)));
    b->gallocs.push_back(gr);
    CK(cudaMemcpy(gr, b->gt.Rmed.data(), sizeof(float) * (NRAD + 1), cudaMemcpyHostToDevice));
    G.dens = gd;
    G.Rmed = gr;
    fargo_status sst = sg_create(&b->gsg, p, b->gt, b->stream, &G, b->err);
    if (G.sg_accr) b->gallocs.push_back(G.sg_accr);
    if (G.sg_acct) b->gallocs.push_back(G.sg_acct);
    if (sst) return sst;
  }
  b->use_graph = false;
  return build_graph(b);
}

fargo_status fargo_stripe_init_state(fargo_ctx* ctx, const float* dens, const float* energy) {
  if (!ctx || !ctx->b.stripe) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  CK(cudaSetDevice(b->device));
  const DiskDev& D = b->disks[0].dev;
  const int nsec = D.nsec, NRAD = b->stripe_nrad;
  const size_t off = (size_t)b->stripe_base * nsec;
  if (b->gsg) {
    // the whole density, for the initial convolution (the profile by default)
    std::vector<float> S;
    const float* src = dens;
    if (!src) {
      S.resize((size_t)NRAD * nsec);
      for (int i = 0; i < NRAD; i++)
        for (int j = 0; j < nsec; j++) S[(size_t)i * nsec + j] = b->gt.SigmaMed[i];
      src = S.data();
    }
    CK(cudaMemcpy(b->gv.dens, src, sizeof(float) * (size_t)NRAD * nsec, cudaMemcpyHostToDevice));
  }
  return init_disk_state(b, 0, dens ? dens + off : nullptr, energy ? energy + off : nullptr);
}

fargo_status fargo_stripe_sg_rows(fargo_ctx* ctx, float* out) {
  if (!ctx || !ctx->b.stripe || !out) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  if (!b->gsg) return set_err(b, FARGO_EINVAL, "the stripe has no self-gravity");
  CK(cudaSetDevice(b->device));
  const DiskDev& D = b->disks[0].dev;
  CK(cudaMemcpyAsync(out, D.dens + (size_t)D.own_lo * D.nsec, sizeof(float) * (size_t)(D.own_hi - D.own_lo) * D.nsec,
                     cudaMemcpyDeviceToDevice, b->stream));
  return FARGO_OK;
}

fargo_status fargo_stripe_sg_apply(fargo_ctx* ctx, const float* gathered, int nstripe, int stride,
                                   const int* cuts) {
  if (!ctx || !ctx->b.stripe || !gathered || !cuts || nstripe < 1) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  if (!b->gsg) return set_err(b, FARGO_EINVAL, "the stripe has no self-gravity");
  const DiskDev& D = b->disks[0].dev;
  const int nsec = D.nsec, NRAD = b->stripe_nrad;
  if (cuts[0] != 0 || cuts[nstripe] != NRAD) return set_err(b, FARGO_EINVAL, "stripe cuts must span 0 .. NRAD");
  for (int k = 0; k < nstripe; k++)
    if (cuts[k + 1] <= cuts[k] || (long long)(cuts[k + 1] - cuts[k]) * nsec > stride)
      return set_err(b, FARGO_EINVAL, "stripe %d: rows %d .. %d do not fit a stride of %d floats", k, cuts[k],
                     cuts[k + 1], stride);
  CK(cudaSetDevice(b->device));
  for (int k = 0; k < nstripe; k++)
    CK(cudaMemcpyAsync(b->gv.dens + (size_t)cuts[k] * nsec, gathered + (size_t)k * stride,
                       sizeof(float) * (size_t)(cuts[k + 1] - cuts[k]) * nsec, cudaMemcpyDeviceToDevice, b->stream));
  sg_capture_substep(b->gsg, b->bd, 0, &b->gv, b->stream);
  const size_t n = (size_t)D.nrad * nsec, o = (size_t)b->stripe_base * nsec;
  CK(cudaMemcpyAsync(D.sg_accr, b->gv.sg_accr + o, sizeof(float) * n, cudaMemcpyDeviceToDevice, b->stream));
  CK(cudaMemcpyAsync(D.sg_acct, b->gv.sg_acct + o, sizeof(float) * n, cudaMemcpyDeviceToDevice, b->stream));
  b->launches += 6;
  CK(cudaGetLastError());
  return FARGO_OK;
}

fargo_status fargo_stripe_info(fargo_ctx* ctx, fargo_stripe_layout* out) {
  if (!ctx || !out || !ctx->b.stripe) return FARGO_EINVAL;
  const fargo_batch* b = &ctx->b;
  const DiskDev& D = b->disks[0].dev;
  out->base = b->stripe_base;
  out->nrad = D.nrad;
  out->nsec = D.nsec;
  out->own_lo = D.own_lo;
  out->own_hi = D.own_hi;
  out->ghost_lo = b->ghost_lo;
  out->ghost_hi = b->ghost_hi;
  out->nfields = stripe_nfields(b);
  out->halo_floats_lo = out->nfields * b->ghost_lo * D.nsec;
  out->halo_floats_hi = out->nfields * b->ghost_hi * D.nsec;
  out->block_doubles = FARGO_STRIPE_HEAD + 4 * FARGO_MAXBODY * fargo_cfl_tiles_own(D);
  return FARGO_OK;
}

fargo_status fargo_stripe_dt_begin(fargo_ctx* ctx) {
  if (!ctx || !ctx->b.stripe) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  CK(cudaSetDevice(b->device));
  fargo_launch_dt_begin(b->bd, b->stream);
  b->launches += 1;
  if (b->any_adiabatic) {
    fargo_launch_cs_refresh(b->bd, -1, b->stream);
    b->launches += 2;
  }
  CK(cudaGetLastError());
  return FARGO_OK;
}

fargo_status fargo_stripe_forces(fargo_ctx* ctx, double* block) {
  if (!ctx || !ctx->b.stripe || !block) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  CK(cudaSetDevice(b->device));
  fargo_launch_substep(b->bd, 0, 0, b->stream, b->max_nsec, &b->launches, nullptr, FARGO_PART_HEAD);
  fargo_launch_stripe_block(b->bd, block, b->stream);
  b->launches += 1;
  CK(cudaGetLastError());
  return FARGO_OK;
}

fargo_status fargo_stripe_substep(fargo_ctx* ctx, const double* blocks, int nstripe, int stride) {
  if (!ctx || !ctx->b.stripe || !blocks || nstripe < 1 || stride < FARGO_STRIPE_HEAD) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  CK(cudaSetDevice(b->device));
  if (fargo_launch_stripe_finish(b->bd, blocks, nstripe, stride, b->stream))
    return set_err(b, FARGO_EINVAL, "stripe count %d out of range", nstripe);
  b->launches += 1;
  fargo_launch_substep(b->bd, 0, 0, b->stream, b->max_nsec, &b->launches, nullptr, FARGO_PART_TAIL);
  CK(cudaGetLastError());
  return FARGO_OK;
}

// ghost rows of one side: [field][rows][nsec], fields Sigma, v_r, v_theta (+ e)
static fargo_status stripe_halo(fargo_batch* b, int row0, int rows, float* buf, bool pack) {
  if (rows == 0) return FARGO_OK;
  const DiskDev& D = b->disks[0].dev;
  float* f[4] = {D.dens, D.vrad, D.vtheta, D.energy};
  const size_t n = (size_t)rows * D.nsec;
  for (int k = 0; k < stripe_nfields(b); k++) {
    float* grid = f[k] + (size_t)row0 * D.nsec;
    if (pack)
      CK(cudaMemcpyAsync(buf + k * n, grid, sizeof(float) * n, cudaMemcpyDeviceToDevice, b->stream));
    else
      CK(cudaMemcpyAsync(grid, buf + k * n, sizeof(float) * n, cudaMemcpyDeviceToDevice, b->stream));
  }
  return FARGO_OK;
}

fargo_status fargo_stripe_halo_pack(fargo_ctx* ctx, float* lo, float* hi) {
  if (!ctx || !ctx->b.stripe) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  if ((b->ghost_lo && !lo) || (b->ghost_hi && !hi)) return set_err(b, FARGO_EINVAL, "missing halo buffer");
  CK(cudaSetDevice(b->device));
  const DiskDev& D = b->disks[0].dev;
  fargo_status st = stripe_halo(b, D.own_lo, b->ghost_lo, lo, true);
  if (st) return st;
  return stripe_halo(b, D.own_hi - b->ghost_hi, b->ghost_hi, hi, true);
}

fargo_status fargo_stripe_halo_unpack(fargo_ctx* ctx, const float* lo, const float* hi) {
  if (!ctx || !ctx->b.stripe) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  if ((b->ghost_lo && !lo) || (b->ghost_hi && !hi)) return set_err(b, FARGO_EINVAL, "missing halo buffer");
  CK(cudaSetDevice(b->device));
  const DiskDev& D = b->disks[0].dev;
  fargo_status st = stripe_halo(b, D.own_lo - b->ghost_lo, b->ghost_lo, const_cast<float*>(lo), false);
  if (st) return st;
  return stripe_halo(b, D.own_hi, b->ghost_hi, const_cast<float*>(hi), false);
}

fargo_status fargo_stripe_more(fargo_ctx* ctx, int* more) {
  if (!ctx || !ctx->b.stripe || !more) return FARGO_EINVAL;
  fargo_batch* b = &ctx->b;
  CK(cudaSetDevice(b->device));
  int h = 0;
  CK(cudaMemcpyAsync(&h, b->d_flags, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  *more = h;
  return h ? FARGO_OK : finish_dts(b);
}

}  // extern "C"
