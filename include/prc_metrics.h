/* prc_metrics.h -- reference-based image-quality metrics on the device.
 *
 * Replaces the per-image work of the reference's scorer, tools/evaluate.py (class Evaluator,
 * tools/evaluate.py:47-154): the evaluator is built once from the truth and its masks
 * (Evaluator.__init__, :48-103), and each reconstruction is reduced on the GPU to the FP64
 * sums below (Evaluator.__call__, :105-154), from which the host forms the metric values.
 * Return codes and prc_last_error() are those of prc_b200.h.
 */
#ifndef PRC_METRICS_H
#define PRC_METRICS_H

#include "prc_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Voxel classes (bit flags of the per-voxel class volume). */
#define PRC_CLASS_BODY 1       /* tissue mask (truth > 0, or the explicit mask)            :56-66 */
#define PRC_CLASS_HOT 2        /* hot regions (truth > 1.5 x background, or explicit)      :77-89 */
#define PRC_CLASS_BACKGROUND 4 /* background interior (eroded 4 times, 3x3x3)              :97-99 */
#define PRC_CLASS_EDGE 8       /* edge band: 5-voxel max filter > 5-voxel min filter       :100-103 */
#define PRC_CLASS_HALO 16      /* shell 2-3 voxels around hot regions, in background      :104-107 */
#define PRC_CLASS_ROI 32       /* inside the bounding box of the body dilated 4 times      :95 */

/* Indices of the FP64 sums (over all voxels unless a class is named; d = f - truth). */
enum {
    PRC_EVAL_D2 = 0,      /* sum d^2 */
    PRC_EVAL_T2,          /* sum truth^2 */
    PRC_EVAL_D2_BODY,     /* sum d^2, body */
    PRC_EVAL_T2_BODY,     /* sum truth^2, body */
    PRC_EVAL_ABS_BODY,    /* sum |d|, body */
    PRC_EVAL_N_BODY,      /* body voxels */
    PRC_EVAL_F,           /* sum f */
    PRC_EVAL_T,           /* sum truth */
    PRC_EVAL_D2_ROI,      /* sum d^2, ROI box */
    PRC_EVAL_N_ROI,       /* ROI voxels */
    PRC_EVAL_F_HOT,       /* sum f, hot */
    PRC_EVAL_T_HOT,       /* sum truth, hot */
    PRC_EVAL_F_BG,        /* sum f, background interior */
    PRC_EVAL_F2_BG,       /* sum f^2, background interior */
    PRC_EVAL_N_BG,        /* background interior voxels */
    PRC_EVAL_RING2,       /* sum (over + under)^2, edge band */
    PRC_EVAL_OVER2,       /* sum max(f - hi, 0)^2, edge band */
    PRC_EVAL_UNDER2,      /* sum max(lo - f, 0)^2, edge band */
    PRC_EVAL_N_EDGE,      /* edge-band voxels */
    PRC_EVAL_D2_EDGE,     /* sum d^2, edge band */
    PRC_EVAL_T2_EDGE,     /* sum truth^2, edge band */
    PRC_EVAL_F_HALO,      /* sum f, halo shell */
    PRC_EVAL_N_HALO,      /* halo voxels */
    PRC_EVAL_NONFINITE,   /* voxels of f that are not finite (then nothing else is meaningful) */
    PRC_EVAL_SSIM_SUM,    /* SSIM map summed over the valid interior of the ROI box (5 voxels
                             from every face); the next five: that count, the sum and count
                             over body voxels, the sum and count over edge-band voxels.
                             All six stay 0 when a side of the box is shorter than 11. */
    PRC_EVAL_NUM_SUMS = PRC_EVAL_SSIM_SUM + 6
};
/* After the PRC_EVAL_NUM_SUMS fixed sums: for hot region l = 1..n_labels, sum f then sum truth. */

typedef struct prc_eval prc_eval;

/* Builds an evaluator for one truth volume (nz*ny*nx doubles, x fastest; all arrays are host
 * memory): classes = per-voxel PRC_CLASS_* flags; labels = hot-region label per voxel (0 =
 * none, 1..n_labels; may be NULL when n_labels is 0); lo / hi = the truth's 5-voxel minimum and
 * maximum filters; roi = {z0, z1, y0, y1, x0, x1} (half-open); data_range = the SSIM / PSNR
 * range.  The device copies are owned by the evaluator. */
int prc_eval_create(int nz, int ny, int nx, const double* truth, const unsigned char* classes, const int* labels,
                    int n_labels, const double* lo, const double* hi, const int* roi, double data_range,
                    prc_eval** out);

/* Scores the reconstruction d_f (device, nz*ny*nx floats) on `stream` (NULL: the default
 * stream) and writes PRC_EVAL_NUM_SUMS + 2 * n_labels FP64 sums to host memory `sums`
 * (synchronises with the stream). */
int prc_eval_sums(prc_eval* e, const float* d_f, double* sums, void* stream);

/* The same for a reconstruction held in doubles. */
int prc_eval_sums_f64(prc_eval* e, const double* d_f, double* sums, void* stream);

void prc_eval_destroy(prc_eval* e);

#ifdef __cplusplus
}
#endif

#endif /* PRC_METRICS_H */
