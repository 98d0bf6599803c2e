// ns_sensor.h -- learned troubled-face sensor gating the characteristic
// projection (internal interface).
#pragma once

#include <cuda_runtime.h>

#include "ns_common.cuh"

namespace nsb {

struct SensorState;

ns_status sensor_create(SensorState** out, const Box& b, const FaceBox fb[3], cudaStream_t s);
void sensor_destroy(SensorState* st);
// Gated face fluxes along axis dir: component-wise FP32 WENO on every face, the
// characteristic-wise flux recomputed on the faces the sensor flags.
ns_status sensor_face_flux(SensorState* st, int dir, const double* W, const double* U, const Box& b,
                           const Consts& c, double threshold, bool borges, bool phys, void* F,
                           const FaceBox& fb, cudaStream_t s, long long* launches);
// Per-step flags along axis dir for the fused stage kernel: the network on every
// face of the step's start state U0, one byte per face (FaceBox order).  The
// call for dir 0 (always the first of a step) also forms the FP32 primitive
// planes the three axes read.
ns_status sensor_step_mask(SensorState* st, int dir, const double* U0, const Box& b, const Consts& c,
                           double threshold, const FaceBox& fb, cudaStream_t s, long long* launches);
const unsigned char* sensor_mask(const SensorState* st, int dir);
// fraction of evaluated faces the sensor flagged since the context was created
double sensor_last_fraction(SensorState* st);
ns_status sensor_set_weights(SensorState* st, const float* w, cudaStream_t s);
// features + labels of the faces along dir into feat/label starting at row base
// (labels from the FP64 fluxes of the given semantics)
ns_status sensor_harvest(int dir, bool borges, bool phys, const double* W, const double* U, const Box& b,
                         const Consts& c, const FaceBox& fb, long long base, double thr, float* feat,
                         float* label, cudaStream_t s);

}  // namespace nsb
