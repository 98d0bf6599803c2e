// ns_sensor.h -- learned troubled-face sensor gating the characteristic
// projection (internal interface).
#pragma once

#include <cuda_runtime.h>

#include "ns_common.cuh"
#include "ns_kernels.h"

namespace nsb {

struct SensorState;

ns_status sensor_create(SensorState** out, const Box& b, const FaceBox fb[3], cudaStream_t s);
void sensor_destroy(SensorState* st);
// Gated face fluxes along axis dir: component-wise FP32 WENO on every face, the
// characteristic-wise flux recomputed on the faces the sensor flags.
ns_status sensor_face_flux(SensorState* st, int dir, const double* W, const double* U, const Box& b,
                           const Consts& c, double threshold, bool borges, bool phys, void* F,
                           const FaceBox& fb, cudaStream_t s, long long* launches);
// The flags of a step from its start state U0: the network on every face of the
// convected axes (one byte per face, FaceBox order), the compacted lists of the
// flagged faces and of the cells next to them (GateLists).
ns_status sensor_step_flags(SensorState* st, const double* U0, const Box& b, const Consts& c, double threshold,
                            const FaceBox fb[3], int conv_dims, cudaStream_t s, long long* launches);
GateLists sensor_gate_lists(const SensorState* st);
// NS_ERR_TIMEOUT if a tensor-core wait of the flag kernels ran out of polls (waits for the device)
ns_status sensor_status(SensorState* st);
// fraction of evaluated faces the sensor flagged since the context was created
double sensor_last_fraction(SensorState* st);
ns_status sensor_set_weights(SensorState* st, const float* w, cudaStream_t s);
// features + labels of the faces along dir into feat/label starting at row base
// (labels from the FP64 fluxes of the given semantics)
ns_status sensor_harvest(int dir, bool borges, bool phys, const double* W, const double* U, const Box& b,
                         const Consts& c, const FaceBox& fb, long long base, double thr, float* feat,
                         float* label, cudaStream_t s);

}  // namespace nsb
