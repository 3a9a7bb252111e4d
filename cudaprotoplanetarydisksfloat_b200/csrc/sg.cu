// sg.cu -- self-gravity (SgMain.cu:23-195) on B200: cuFFT as the FFT engine,
// hand-written fused kernels for the pad, the kernel-spectrum multiply and
// the unpad/normalise/acceleration step.
//
// Differences in method from the reference, all exact in arithmetic:
//   - the kernel spectra K^r, K^t are transformed once, in FP64 (D2Z), at
//     creation; the reference re-transforms the constant kernels in FP32
//     every call (SgMain.cu:124,138);
//   - the density transforms are real-to-complex and the inverse
//     complex-to-real (the inputs are real, so the reference's C2C result
//     is the same Hermitian spectrum);
//   - the 2-D transforms are done as their row and column passes, pruned:
//     the density occupies rows 0 .. NRAD-1 of the zero-padded 2 NRAD rows,
//     so the forward azimuthal (row) transforms run on those rows only, into
//     a spectrum buffer whose rows NRAD .. 2 NRAD-1 stay zero, and the
//     inverse ones only on the rows the accelerations use; the radial
//     (column) transforms take all 2 NRAD rows, strided, one column per
//     transform of the batch;
//   - the velocity kick (Update_sgvelocityKernel) is fused into the
//     Substep1 kernel, so the accelerations are stored once and read once.
#include <cufft.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "sg.h"

#define PI_D FARGO_PI

struct SelfGravity {
  int nrad = 0, nsec = 0, nx = 0, nyh = 0;
  cufftHandle rowf = 0, rowi = 0, col = 0;  // row R2C / C2R on nrad rows, column C2C on 2 nrad rows
  // the two fields (Sr, St; then Gr, Gphi) interleaved by row, so that one
  // transform call takes both: element (row i, field f, column j)
  float* real2 = nullptr;     // [nrad][2][nsec]
  float2* rows2 = nullptr;    // [2*nrad][2][nsec/2+1]: row spectra, rows nrad.. zero
  float2* spec2 = nullptr;    // [2*nrad][2][nsec/2+1]: 2-D spectra
  float2* khat = nullptr;     // [2*nrad][2][nsec/2+1]: K^r, K^t spectra
  float eps = 0, rstep = 0, tstep = 0;
  bool plans = false;
};

namespace {

// ComputeFFTKernel's density part (Kernels.cu:957-976) as real arrays, on
// the rows that hold the density (the padding rows are the zero rows of the
// row-spectrum buffer).
__global__ void k_sg_pad(DiskDev D, float* real2) {
  const int nrad = D.nrad, nsec = D.nsec;
  long long n = (long long)nrad * nsec;
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  if (!D.ctl->active) return;
  int i = (int)(c / nsec), j = (int)(c - (long long)i * nsec);
  float var = D.dens[c] * sqrtf(D.Rmed[i] / D.Rmed[0]);
  float* row = real2 + 2LL * i * nsec + j;
  row[0] = var;
  row[nsec] = var * D.Rmed[i] / D.Rmed[0];
}

// ComputeConvolutionKernel, Kernels.cu:980-999 (half spectrum): G = -K S
// for both fields, element by element (spectra and kernels share a layout)
__global__ void k_sg_mul(const DiskCtl* C, float2* spec2, const float2* khat, long long n) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  if (!C->active) return;
  const float2 sv = spec2[c], k = khat[c];
  float2 g;
  g.x = -1.0 * (k.x * sv.x - k.y * sv.y);
  g.y = -1.0 * (k.x * sv.y + k.y * sv.x);
  spec2[c] = g;
}

// ComputeSgAccKernel, Kernels.cu:1002-1021 (the C2R output is unnormalised,
// as cufftExecC2C INVERSE is in the reference).
__global__ void k_sg_acc(DiskDev D, const float* real2, float rstep, float tstep, float eps) {
  const int nrad = D.nrad, nsec = D.nsec;
  long long n = (long long)nrad * nsec;
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  if (!D.ctl->active) return;
  int i = (int)(c / nsec), j = (int)(c - (long long)i * nsec);
  const float* row = real2 + 2LL * i * nsec + j;  // Gr, then Gphi one row on
  float normaccr, normacct, divRmed;
  divRmed = D.Rmed[i] / D.Rmed[0];
  normaccr = rstep * tstep / ((float)(2 * nrad) * (float)nsec);
  normacct = normaccr;
  normaccr /= sqrtf(divRmed);
  normacct /= (divRmed * sqrtf(divRmed));
  D.sg_acct[c] = row[nsec] * normacct;
  float a = row[0] * normaccr;
  a += 1.0 * D.dens[c] * rstep * tstep / eps;
  D.sg_accr[c] = a;
}

// Make1Dprofile(2) at rings 0 and NRAD-1 (SideEuler.cu:261-267 needs only these)
__global__ void k_sg_axi_edges(DiskDev D) {
  if (!D.ctl->active) return;
  int t = threadIdx.x;
  if (t > 1) return;
  int i = (t == 0) ? 0 : D.nrad - 1;
  const float* f = D.sg_accr + (size_t)i * D.nsec;
  float s = 0.0f;
  for (int j = 0; j < D.nsec; j++) s += f[j];
  s /= (float)D.nsec;
  if (t == 0)
    D.ctl->axisg_in = s;
  else
    D.ctl->axisg_out = s;
}

// Make1Dprofile(2), all rings (initialisation only)
__global__ void k_sg_axi_all(DiskDev D, float* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D.nrad) return;
  const float* f = D.sg_accr + (size_t)i * D.nsec;
  float s = 0.0f;
  for (int j = 0; j < D.nsec; j++) s += f[j];
  out[i] = s / (float)D.nsec;
}

// Azimutalvelocity_withSGKernel, Kernels.cu:1044-1059
__global__ void k_sg_vtheta(DiskDev D, const float* axi) {
  long long n = (long long)D.nrad * D.nsec;
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  int i = (int)(c / D.nsec);
  float omegakep, omega, invr;
  invr = 1. / D.Rmed[i];
  omegakep = sqrt(1.0 * 1.0 * invr * invr * invr);
  omega = sqrt(omegakep * omegakep *
                   (1.0 - (1. + D.SIGMASLOPE - 2.0 * D.FLARINGINDEX) * powf(D.ASPECTRATIO, 2.0) *
                              powf(D.Rmed[i], 2.0 * D.FLARINGINDEX)) -
               invr * axi[i]);
  D.vtheta[c] = D.Rmed[i] * omega;
}

// [2][rows][nyh] FP64 spectra -> [rows][2][nyh] FP32 (fields interleaved by row)
__global__ void k_to_complex_float(const double2* in, float2* out, long long rows, int nyh) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= 2 * rows * nyh) return;
  const long long nh = rows * nyh;
  const long long f = c / nh, r = (c - f * nh) / nyh, m = c - f * nh - r * nyh;
  out[(r * 2 + f) * nyh + m] = make_float2((float)in[c].x, (float)in[c].y);
}

inline unsigned blocks(long long n) { return (unsigned)((n + 255) / 256); }

fargo_status fail(std::string& err, fargo_status st, const char* what, int code) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "self-gravity: %s failed (%d)", what, code);
  err = buf;
  return st;
}

}  // namespace

fargo_status sg_create(SelfGravity** out, const fargo_params* p, const HostTables& t, cudaStream_t s, DiskDev* D,
                       std::string& err) {
  SelfGravity* sg = new SelfGravity();
  *out = sg;
  const int NRAD = p->NRAD, NSEC = p->NSEC;
  sg->nrad = NRAD;
  sg->nsec = NSEC;
  sg->nx = 2 * NRAD;
  sg->nyh = NSEC / 2 + 1;
  // Main.cu:308-310
  sg->eps = p->THICKNESSSMOOTHING * p->ASPECTRATIO;
  sg->rstep = logf(t.Radii[NRAD] / t.Radii[0]) / (float)NRAD;
  sg->tstep = 2.0 * PI_D / (float)NSEC;
  long long nr = (long long)NRAD * NSEC, nh = (long long)sg->nx * sg->nyh;
  cudaError_t e;
  if ((e = cudaMalloc(&sg->real2, sizeof(float) * 2 * nr))) return fail(err, FARGO_EOOM, "cudaMalloc", e);
  if ((e = cudaMalloc(&sg->rows2, sizeof(float2) * 2 * nh))) return fail(err, FARGO_EOOM, "cudaMalloc", e);
  if ((e = cudaMalloc(&sg->spec2, sizeof(float2) * 2 * nh))) return fail(err, FARGO_EOOM, "cudaMalloc", e);
  if ((e = cudaMalloc(&sg->khat, sizeof(float2) * 2 * nh))) return fail(err, FARGO_EOOM, "cudaMalloc", e);
  if ((e = cudaMalloc(&D->sg_accr, sizeof(float) * (size_t)NRAD * NSEC))) return fail(err, FARGO_EOOM, "cudaMalloc", e);
  if ((e = cudaMalloc(&D->sg_acct, sizeof(float) * (size_t)NRAD * NSEC))) return fail(err, FARGO_EOOM, "cudaMalloc", e);
  cudaMemsetAsync(sg->rows2, 0, sizeof(float2) * 2 * nh, s);  // the padding rows stay zero
  cudaMemsetAsync(D->sg_accr, 0, sizeof(float) * (size_t)NRAD * NSEC, s);
  cudaMemsetAsync(D->sg_acct, 0, sizeof(float) * (size_t)NRAD * NSEC, s);
  // row transforms: the 2 NRAD rows (both fields) of the density;
  // column transforms: the 2 nyh columns (both fields), 2 NRAD long
  int nsec1[1] = {NSEC}, nx1[1] = {sg->nx};
  int rin[1] = {NSEC}, rout[1] = {sg->nyh}, cemb[1] = {sg->nx};
  const int ncol = 2 * sg->nyh;
  cufftResult r;
  if ((r = cufftPlanMany(&sg->rowf, 1, nsec1, rin, 1, NSEC, rout, 1, sg->nyh, CUFFT_R2C, 2 * NRAD)))
    return fail(err, FARGO_ECUFFT, "cufftPlanMany R2C", r);
  if ((r = cufftPlanMany(&sg->rowi, 1, nsec1, rout, 1, sg->nyh, rin, 1, NSEC, CUFFT_C2R, 2 * NRAD)))
    return fail(err, FARGO_ECUFFT, "cufftPlanMany C2R", r);
  if ((r = cufftPlanMany(&sg->col, 1, nx1, cemb, ncol, 1, cemb, ncol, 1, CUFFT_C2C, ncol)))
    return fail(err, FARGO_ECUFFT, "cufftPlanMany C2C", r);
  sg->plans = true;
  cufftSetStream(sg->rowf, s);
  cufftSetStream(sg->rowi, s);
  cufftSetStream(sg->col, s);
  return sg_tabulate(sg, t, 0, s, err);
}

// compute_kernel (SgMain.cu:49-81): the kernels K^r, K^t on the padded
// (2 NRAD) x NSEC grid, tabulated with the reference's host float math
// (accurate = 0) or in FP64 from the FP64 radii (accurate = 1), then
// transformed once in FP64 (D2Z) and kept as FP32 spectra.
fargo_status sg_tabulate(SelfGravity* sg, const HostTables& t, int accurate, cudaStream_t s, std::string& err) {
  const int NRAD = sg->nrad, NSEC = sg->nsec;
  long long nr = (long long)sg->nx * NSEC, nh = (long long)sg->nx * sg->nyh;
  int n[2] = {sg->nx, NSEC};
  cudaError_t e;
  cufftResult r;
  std::vector<double> K(2 * (size_t)nr);
  float eps = sg->eps;
  for (int i = 0; i < 2 * NRAD; i++) {
    if (accurate) {
      const double ed = eps;
      const double u = i < NRAD ? std::log(t.Radii2[i] / t.Radii2[0]) : -std::log(t.Radii2[2 * NRAD - i] / t.Radii2[0]);
      for (int j = 0; j < NSEC; j++) {
        const double th = 2.0 * PI_D * (double)j / (double)NSEC;
        const double base = ed * ed * std::exp(u) + 2.0 * (std::cosh(u) - std::cos(th));
        K[(size_t)i * NSEC + j] = (1.0 + ed * ed - std::cos(th) * std::exp(-u)) * std::pow(base, -1.5);
        K[nr + (size_t)i * NSEC + j] = std::sin(th) * std::pow(base, -1.5);
      }
      continue;
    }
    float u;
    if (i < NRAD)
      u = logf(t.Radii[i] / t.Radii[0]);
    else
      u = -logf(t.Radii[2 * NRAD - i] / t.Radii[0]);
    for (int j = 0; j < NSEC; j++) {
      float theta = 2.0 * PI_D * (float)j / (float)NSEC;
      float Kr = 1.0 + eps * eps - cosf(theta) * expf(-u);
      float base = eps * eps * expf(u) + 2.0 * (coshf(u) - cosf(theta));
      Kr *= powf(base, -1.5);
      float Kt = sinf(theta);
      Kt *= powf(base, -1.5);
      K[(size_t)i * NSEC + j] = Kr;
      K[nr + (size_t)i * NSEC + j] = Kt;
    }
  }
  // FP64 transform of the kernels, once
  double* dK = nullptr;
  double2* dKh = nullptr;
  if ((e = cudaMalloc(&dK, sizeof(double) * 2 * nr))) return fail(err, FARGO_EOOM, "cudaMalloc", e);
  if ((e = cudaMalloc(&dKh, sizeof(double2) * 2 * nh))) {
    cudaFree(dK);
    return fail(err, FARGO_EOOM, "cudaMalloc", e);
  }
  cudaMemcpyAsync(dK, K.data(), sizeof(double) * 2 * nr, cudaMemcpyHostToDevice, s);
  cufftHandle pd;
  if ((r = cufftPlanMany(&pd, 2, n, nullptr, 1, (int)nr, nullptr, 1, (int)nh, CUFFT_D2Z, 2))) {
    cudaFree(dK);
    cudaFree(dKh);
    return fail(err, FARGO_ECUFFT, "cufftPlanMany D2Z", r);
  }
  cufftSetStream(pd, s);
  r = cufftExecD2Z(pd, dK, dKh);
  k_to_complex_float<<<blocks(2 * nh), 256, 0, s>>>(dKh, sg->khat, sg->nx, sg->nyh);
  cudaStreamSynchronize(s);
  cufftDestroy(pd);
  cudaFree(dK);
  cudaFree(dKh);
  if (r) return fail(err, FARGO_ECUFFT, "cufftExecD2Z", r);
  return FARGO_OK;
}

void sg_destroy(SelfGravity* sg) {
  if (!sg) return;
  if (sg->plans) {
    cufftDestroy(sg->rowf);
    cufftDestroy(sg->rowi);
    cufftDestroy(sg->col);
  }
  cudaFree(sg->real2);
  cudaFree(sg->rows2);
  cudaFree(sg->spec2);
  cudaFree(sg->khat);
  delete sg;
}

void sg_capture_substep(SelfGravity* sg, const BatchDev& b, int d, DiskDev* D, cudaStream_t s) {
  (void)b;
  (void)d;
  const long long nr = (long long)sg->nrad * sg->nsec, nh = (long long)sg->nx * sg->nyh;
  cufftSetStream(sg->rowf, s);
  cufftSetStream(sg->rowi, s);
  cufftSetStream(sg->col, s);
  cufftComplex* rows = reinterpret_cast<cufftComplex*>(sg->rows2);
  cufftComplex* spec = reinterpret_cast<cufftComplex*>(sg->spec2);
  k_sg_pad<<<blocks(nr), 256, 0, s>>>(*D, sg->real2);
  cufftExecR2C(sg->rowf, sg->real2, rows);                    // rows 0 .. nrad-1 of both fields
  cufftExecC2C(sg->col, rows, spec, CUFFT_FORWARD);          // all 2 nrad rows
  k_sg_mul<<<blocks(2 * nh), 256, 0, s>>>(D->ctl, sg->spec2, sg->khat, 2 * nh);
  cufftExecC2C(sg->col, spec, spec, CUFFT_INVERSE);
  cufftExecC2R(sg->rowi, spec, sg->real2);                    // rows 0 .. nrad-1 of both fields
  k_sg_acc<<<blocks(nr), 256, 0, s>>>(*D, sg->real2, sg->rstep, sg->tstep, sg->eps);
  k_sg_axi_edges<<<1, 32, 0, s>>>(*D);
}

fargo_status sg_accelerations(SelfGravity* sg, const BatchDev& b, int d, DiskDev* D, cudaStream_t s,
                              std::string& err) {
  // the per-substep kernels check ctl->active: mark the disk active for this call
  int one = 1;
  cudaMemcpyAsync(&D->ctl->active, &one, sizeof(int), cudaMemcpyHostToDevice, s);
  sg_capture_substep(sg, b, d, D, s);
  int zero = 0;
  cudaMemcpyAsync(&D->ctl->active, &zero, sizeof(int), cudaMemcpyHostToDevice, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(err, FARGO_ECUDA, "accelerations", e);
  return FARGO_OK;
}

fargo_status sg_axisymmetric(SelfGravity* sg, DiskDev* D, float* axi, cudaStream_t s, std::string& err) {
  float* dax = nullptr;
  cudaError_t e = cudaMalloc(&dax, sizeof(float) * sg->nrad);
  if (e) return fail(err, FARGO_EOOM, "cudaMalloc", e);
  k_sg_axi_all<<<(sg->nrad + 127) / 128, 128, 0, s>>>(*D, dax);
  cudaMemcpyAsync(axi, dax, sizeof(float) * sg->nrad, cudaMemcpyDeviceToHost, s);
  e = cudaStreamSynchronize(s);
  cudaFree(dax);
  if (e) return fail(err, FARGO_ECUDA, "axisymmetric profile", e);
  return FARGO_OK;
}

fargo_status sg_init_vtheta(SelfGravity* sg, DiskDev* D, const float* axi, cudaStream_t s, std::string& err) {
  (void)sg;
  float* dax = nullptr;
  cudaError_t e = cudaMalloc(&dax, sizeof(float) * D->nrad);
  if (e) return fail(err, FARGO_EOOM, "cudaMalloc", e);
  cudaMemcpyAsync(dax, axi, sizeof(float) * D->nrad, cudaMemcpyHostToDevice, s);
  k_sg_vtheta<<<blocks((long long)D->nrad * D->nsec), 256, 0, s>>>(*D, dax);
  e = cudaStreamSynchronize(s);
  cudaFree(dax);
  if (e) return fail(err, FARGO_ECUDA, "vtheta init", e);
  return FARGO_OK;
}
