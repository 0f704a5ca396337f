/* prc_data.h -- synthetic measurement data on the device.
 *
 * The reference makes its test data on the host: a phantom blurred by the projector, scaled to a
 * total count and Poisson-sampled (tests/test_solver.py builds its phantoms from a seed).  This
 * header adds the sampling step on the GPU, so that data for large grids and many frames never
 * leave the device.  Return codes and prc_last_error() are those of prc_b200.h.
 */
#ifndef PRC_DATA_H
#define PRC_DATA_H

#include <stdint.h>

#include "prc_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* out[i] ~ Poisson(scale * mean[i]) for i < n (device arrays of floats; means that are negative
 * or not finite count as 0), enqueued on `stream` (NULL: the default stream).  The random
 * numbers are Philox4x32-10 keyed by `seed` with the index as counter, so each count depends
 * only on (mean[i], scale, seed, i).  Means below 10 are sampled by inversion, larger ones by
 * the transformed rejection method PTRS (Hormann 1993).  No counterpart in the reference's C
 * code: it replaces the host-side NumPy sampling of its test data. */
int prc_poisson(const float* d_mean, int64_t n, double scale, uint64_t seed, float* d_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PRC_DATA_H */
