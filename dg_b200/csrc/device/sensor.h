// Troubled-cell sensors on the device (SENSOR::sensing, code/src/sensors/sensor.cc:11-35, with
// calc_sensors, code/src/sensors/sensor_kernels.cu:19-165).  Host-side launcher; the kernels live
// in dgb_sensor.cu, which is compiled without floating-point contraction so that every threshold
// decision is taken on the same IEEE-rounded values as the reference's CPU arithmetic.
#pragma once
#include <cuda_runtime.h>

namespace dgb {

struct SensorLaunch {
  int D, ns, nf, n_elem, ld, n_nbr;
  const double* U;      // state, internal layout U[(f*ns + t)*ld + e]
  const int* iperm;     // reference node i -> internal node t (sums in the reference's node order)
  const int* nbr;       // nbr[k*ld + e]
  int on[3];            // sensors 1..3 switched on (deck thresholds present)
  double th[3];         // their thresholds
  // work arrays (device): cell means nf*ld doubles; target, type, processed, in-edge mask,
  // edge list: ld ints each; edge count: 1 int
  double* mean;
  int *target, *type, *processed, *mask, *list, *count;
  int* sens;            // output flags (0 = not flagged, 1..3 = the sensor that fired)
};

// Enqueues the sensor evaluation on `st`; returns 0 or a cudaError_t value.
int launch_sensors(const SensorLaunch& s, cudaStream_t st);
// Same, from cell means already in s.mean (mean[f*ld + e]); s.U and s.iperm are not used.
int launch_sensors_from_means(const SensorLaunch& s, cudaStream_t st);

}  // namespace dgb
