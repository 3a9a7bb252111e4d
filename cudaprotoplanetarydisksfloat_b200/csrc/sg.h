// sg.h -- self-gravity of one disk: the log-polar convolution of
// compute_selfgravity (SgMain.cu:23-162) with cuFFT as the FFT engine.
#pragma once
#include <string>

#include "fargo_internal.h"
#include "host_internal.h"

struct SelfGravity;

fargo_status sg_create(SelfGravity** out, const fargo_params* p, const HostTables& t, cudaStream_t s, DiskDev* D,
                       std::string& err);
void sg_destroy(SelfGravity* sg);
// compute_kernel (SgMain.cu:49-81) tabulated in the reference's float math
// (accurate = 0) or in FP64 (accurate = 1), transformed once in FP64
fargo_status sg_tabulate(SelfGravity* sg, const HostTables& t, int accurate, cudaStream_t s, std::string& err);
// pad -> R2C -> kernel-spectrum multiply -> C2R -> accelerations (SG_Accr/SG_Acct)
fargo_status sg_accelerations(SelfGravity* sg, const BatchDev& b, int d, DiskDev* D, cudaStream_t s,
                              std::string& err);
// Make1Dprofile(2): ring means of SG_Accr, copied to the host (nrad values)
fargo_status sg_axisymmetric(SelfGravity* sg, DiskDev* D, float* axi, cudaStream_t s, std::string& err);
// Init_azimutalvelocity_withSG (SourceEuler.cu:428-437) on the rings of D,
// axi[i] the axisymmetric acceleration at ring i of D (D->nrad values)
fargo_status sg_init_vtheta(SelfGravity* sg, DiskDev* D, const float* axi, cudaStream_t s, std::string& err);
// enqueue the per-substep pipeline (capturable)
void sg_capture_substep(SelfGravity* sg, const BatchDev& b, int d, DiskDev* D, cudaStream_t s);
