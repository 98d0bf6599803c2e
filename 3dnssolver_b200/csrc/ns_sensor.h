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
                           const Consts& c, void* F, const FaceBox& fb, cudaStream_t s,
                           long long* launches);
double sensor_last_fraction(SensorState* st);

}  // namespace nsb
