/*
 * prc_surrogate.h -- the learned range-kernel surrogate of libprc_b200.so.
 *
 * No counterpart in the reference (jlherraiz/PRC_MLEM): a 3D CNN that maps a voxel's 21^3 density
 * patch and its isotope to per-direction radial far-field kernel coefficients (128 ray
 * directions x 16 radial bins), trained on kernels produced by the plain ray tracer, with
 * bf16 tensor-core (tcgen05) implicit-GEMM kernels and fp32 accumulation.  Conventions as in
 * prc_b200.h: int status, device pointers, stream as void* (NULL = default stream).
 */
#ifndef PRC_SURROGATE_H
#define PRC_SURROGATE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* C[M][N] (fp32) = A[M][K] . B[N][K]^T on the tensor cores; A and B bf16 row-major with K
 * contiguous.  *d_error (device) is set non-zero if an MMA completion wait gave up.  The GEMM
 * engine of the network, exposed for testing. */
int prc_nn_gemm_bf16(const void* d_a, const void* d_b, float* d_c, int M, int N, int K, unsigned int* d_error,
                     void* stream);

/* The network: four valid 3x3x3 convolutions (32 channels, ReLU) with tap spacings (dilations)
 * 1, 2, 3 and 4 over a 21^3 patch of channels-last bf16 input [density / 2, 1 inside the volume
 * (0 beyond it, where the density reads as air), one-hot 18F, 68Ga, 82Rb, 0, 0, 0] (sides
 * 21 -> 19 -> 15 -> 9 -> 1), then a linear head to 2048 = 128 directions x 16 radial bins.
 * fp32 master weights, bf16 copies for the tensor cores, Adam (beta 0.9 / 0.999, eps 1e-8).
 * Parameter order for get/set: w1, b1, w2, b2, w3, b3, w4, b4, wh, bh with conv weights
 * [32][3][3][3][cin] (cin 8, then 32) and head weights [2048][32]. */
typedef struct prc_net prc_net;

/* Side of the input patch (21). */
int prc_nn_patch_side(void);

int prc_nn_create(int max_batch, prc_net** out);
void prc_nn_destroy(prc_net* net);
int64_t prc_nn_param_count(void);
int prc_nn_set_params(prc_net* net, const float* host_params);
/* what = 0: parameters, 1: gradients of the last prc_nn_backward.  Synchronises. */
int prc_nn_get(prc_net* net, int what, float* host_out);
/* d_x0: [batch][21][21][21][8] bf16 patches; d_y: [batch][2048] fp32 or NULL (internal buffer). */
int prc_nn_forward(prc_net* net, const void* d_x0, int batch, float* d_y, void* stream);
/* MSE against d_target after prc_nn_forward (d_y NULL), all gradients, an Adam step if lr > 0;
 * *loss (host, optional) receives the MSE (sum of squared errors / (batch x 2048)).  Outputs
 * whose target is negative are masked: no error, no gradient. */
int prc_nn_backward(prc_net* net, const float* d_target, int batch, float lr, double* loss, void* stream);

/* Training data on the device: n_vol random volumes of side^3 voxels of spacing_mm, each air
 * plus up to 10 ellipsoids (ellipsoids: host [n_vol][10][8] = cx, cy, cz, rx, ry, rz in voxels,
 * density, used flag) with Gaussian multiplicative density jitter of relative spread `jitter`
 * (0 to 0.5; seeded); per_vol (a multiple of 32)
 * tissue sources per volume.  Outputs the sources' input patches (d_patches,
 * [n][21][21][21][8] bf16) and their traced radial far-field kernels times target_scale
 * (d_targets, [n][2048] fp32, direction-major), for isotope 18F, 68Ga or 82Rb.  Targets a
 * surrogate field never takes from the network are -1 (masked in the loss): the bins past the
 * water range (the last 4 of every ray), and all bins of a ray with more than 2 % of its mass
 * past it.  Synchronises. */
int prc_nn_make_samples(const char* isotope, int n_vol, int side, float spacing_mm, const float* ellipsoids,
                        uint64_t seed, int per_vol, void* d_patches, float* d_targets, float target_scale,
                        float jitter, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PRC_SURROGATE_H */
