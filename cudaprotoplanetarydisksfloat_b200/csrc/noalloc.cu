// noalloc.cu -- disk force on one body from caller-owned device fields,
// with no device allocation of any kind.
//
// Who needs it: a program that already holds its disk on the GPU in its own
// arrays (as the reference's main() does) but may not call cudaMalloc in
// the middle of its step -- because it manages device memory itself (its
// own pool, or a fixed budget shared with other work), or because
// cudaMalloc/cudaFree synchronise the whole device and would stall its other
// streams.  fargo_disk_force needs a context, and creating one allocates.
//
// The only scratch is the file-scope array g_force_scratch below, a fixed
// 1.4 MB that every GPU which loads this library holds until the process
// exits.  Its device address is looked up once per device, with that device
// current, by the first call made on that device.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "../../include/fargo_b200.h"

namespace {

constexpr int kNQ = 4 * FARGO_DIMFXY;  // sums per ring: fx/fy, inner/outer, every Hill-cut level
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

// Per-ring partial sums [FARGO_NOALLOC_MAXRAD][kNQ], then the kNQ totals.
// Every slot a call reads is written earlier by the same call, so nothing
// has to start at zero and nothing is cleared; two calls whose kernels
// overlap on the GPU (different streams, or host threads) race on it.
static __device__ __align__(256) double g_force_scratch[(FARGO_NOALLOC_MAXRAD + 1) * kNQ];

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// ComputeForceKernel (Kernels.cu:804-839) for every Hill-cut level k at once,
// one block per ring; the block's FP64 sums of the FP32 per-cell forces go to
// part[i * kNQ + q].  Each thread keeps all 44 FP64 sums, more than fit in
// registers beside the rest (ptxas spills part of them to local memory):
// acceptable for a diagnostic call made once per output, not per substep.  The same arithmetic as the library's context-based
// disk force, reading the cell coordinates from the caller's
// CellAbscissa/CellOrdinate arrays.
__global__ void __launch_bounds__(kThreads) k_disk_force_rings(const float* __restrict__ dens,
                                                                const float* __restrict__ cell_x,
                                                                const float* __restrict__ cell_y,
                                                                const float* __restrict__ surf,
                                                                const float* __restrict__ rmed, int nrad,
                                                                int nsec, float x, float y, float rs,
                                                                float rh0, float a, double* part) {
  __shared__ double red[kThreads / 32];
  for (int i = blockIdx.x; i < nrad; i += gridDim.x) {
    double s[kNQ];
#pragma unroll
    for (int q = 0; q < kNQ; q++) s[q] = 0.0;
    const bool inner = rmed[i] < a;
    const float sf = surf[i];
    for (int j = threadIdx.x; j < nsec; j += blockDim.x) {
      const long long c = (long long)i * nsec + j;
      float cellmass = sf * dens[c];
      float dx = cell_x[c] - x;
      float dy = cell_y[c] - y;
      float d2 = dx * dx + dy * dy;
      float dist2 = d2 + rs * rs;
      float distance = sqrtf(dist2);
      float InvDist3 = 1.0 / dist2 / distance;  // two FP64 divisions, as Kernels.cu:821
#pragma unroll
      for (int k = 0; k < FARGO_DIMFXY; k++) {
        float hillcutfactor = (float)k / (float)(FARGO_DIMFXY - 1);
        float hill_cut;
        if (k != 0) {
          float rh = rh0 * hillcutfactor;
          hill_cut = 1. - expf(-d2 / (rh * rh));
        } else
          hill_cut = 1.;
        float fx = 1.0 * cellmass * dx * InvDist3 * hill_cut;
        float fy = 1.0 * cellmass * dy * InvDist3 * hill_cut;
        if (inner) {
          s[k] += fx;
          s[k + 2 * FARGO_DIMFXY] += fy;
        } else {
          s[k + FARGO_DIMFXY] += fx;
          s[k + 3 * FARGO_DIMFXY] += fy;
        }
      }
    }
    for (int q = 0; q < kNQ; q++) {
      double v = warp_sum(s[q]);
      __syncthreads();
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
      __syncthreads();
      if (threadIdx.x == 0) {
        double acc = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) acc += red[w];
        part[(size_t)i * kNQ + q] = acc;
      }
    }
  }
}

// Totals over the rings in a fixed order (one warp per sum) into out[kNQ].
__global__ void __launch_bounds__(kThreads) k_disk_force_total(const double* part, int nrad, double* out) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int q = w; q < kNQ; q += blockDim.x >> 5) {
    double acc = 0.0;
    for (int r = l; r < nrad; r += 32) acc += part[(size_t)r * kNQ + q];
    acc = warp_sum(acc);
    if (l == 0) out[q] = acc;
  }
}

std::mutex g_mu;
double* g_addr[kMaxDevices];  // device address of g_force_scratch, per device

fargo_status fail(char* err, int errlen, fargo_status st, const char* fmt, ...) {
  if (err && errlen > 0) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(err, (size_t)errlen, fmt, ap);
    va_end(ap);
  }
  return st;
}

}  // namespace

extern "C" fargo_status fargo_disk_force_noalloc(const float* dens, const float* cell_x, const float* cell_y,
                                                 const float* surf, const float* rmed, int nrad, int nsec,
                                                 double x, double y, double rsmoothing, double mass,
                                                 int dimfxy, double* globalforce, void* stream, char* err,
                                                 int errlen) {
  if (err && errlen > 0) err[0] = '\0';
  if (!dens || !cell_x || !cell_y || !surf || !rmed || !globalforce)
    return fail(err, errlen, FARGO_EINVAL, "fargo_disk_force_noalloc: null pointer argument");
  if (dimfxy != FARGO_DIMFXY)
    return fail(err, errlen, FARGO_EINVAL, "fargo_disk_force_noalloc: dimfxy must be %d", FARGO_DIMFXY);
  if (nsec < 1 || nrad < 1)
    return fail(err, errlen, FARGO_EINVAL, "fargo_disk_force_noalloc: NRAD and NSEC must be >= 1");
  if (nrad > FARGO_NOALLOC_MAXRAD)
    return fail(err, errlen, FARGO_EINVAL,
                "fargo_disk_force_noalloc: NRAD = %d exceeds the fixed scratch of %d rings; "
                "use fargo_disk_force for larger grids",
                nrad, FARGO_NOALLOC_MAXRAD);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return fail(err, errlen, e == cudaErrorNoDevice ? FARGO_ENODEV : FARGO_ECUDA,
                "fargo_disk_force_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return fail(err, errlen, FARGO_EINVAL, "fargo_disk_force_noalloc: device %d beyond %d", dev, kMaxDevices);
  double* scratch = nullptr;
  {
    // set-up, once per device, with that device current
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_force_scratch);
      if (e != cudaSuccess)
        return fail(err, errlen, FARGO_ECUDA, "fargo_disk_force_noalloc: cudaGetSymbolAddress: %s",
                    cudaGetErrorString(e));
      g_addr[dev] = static_cast<double*>(p);
    }
    scratch = g_addr[dev];
  }
  // ComputeForce (Force.cu:39-40): a and rh in double, kernel arguments float
  const double a = std::sqrt(x * x + y * y);
  const double rh = std::pow(mass / 3., 1. / 3.) * a + 1e-15;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // an error left pending by the caller's own launches is reported as such
  // and left in place (peek), so it is neither blamed on this call nor lost
  e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return fail(err, errlen, FARGO_ECUDA, "fargo_disk_force_noalloc: an earlier CUDA error is pending: %s",
                cudaGetErrorString(e));
  double* totals = scratch + (size_t)FARGO_NOALLOC_MAXRAD * kNQ;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int grid = nrad < 4 * nsm ? nrad : 4 * nsm;
  k_disk_force_rings<<<grid, kThreads, 0, s>>>(dens, cell_x, cell_y, surf, rmed, nrad, nsec, (float)x, (float)y,
                                               (float)rsmoothing, (float)rh, (float)a, scratch);
  k_disk_force_total<<<1, kThreads, 0, s>>>(scratch, nrad, totals);
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(globalforce, totals, sizeof(double) * kNQ, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess)
    return fail(err, errlen, FARGO_ECUDA, "fargo_disk_force_noalloc: %s", cudaGetErrorString(e));
  return FARGO_OK;
}
