// ns_sensor.cu -- learned troubled-face sensor (placeholder until the MLP lands).
#include "ns_sensor.h"

namespace nsb {

struct SensorState {
    double fraction = 0.0;
};

ns_status sensor_create(SensorState** out, const Box&, const FaceBox*, cudaStream_t) {
    *out = nullptr;
    return NS_ERR_UNSUPPORTED;
}
void sensor_destroy(SensorState* st) { delete st; }
ns_status sensor_face_flux(SensorState*, int, const double*, const double*, const Box&, const Consts&,
                           void*, const FaceBox&, cudaStream_t, long long*) {
    return NS_ERR_UNSUPPORTED;
}
double sensor_last_fraction(SensorState* st) { return st ? st->fraction : 0.0; }

}  // namespace nsb
