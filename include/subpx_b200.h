/*
 * libsubpx_b200 — C ABI of the B200 (sm_100a) subpixel-metrology hot path.
 *
 * Conventions
 *   - Every buffer argument is a DEVICE pointer owned by the caller (cudaMalloc, a torch tensor,
 *     CuPy, ...). Images are row-major [y][x]; coordinates are [x, y] pixels with pixel centres
 *     at integers, as in subpx (docs/conventions.md).
 *   - `stream` is a cudaStream_t passed as void*; all work is enqueued on it, nothing synchronises
 *     unless the function says so.
 *   - Scratch memory comes from a caller-provided workspace sized by the matching
 *     *_workspace_bytes() query. Nothing allocates device memory behind the caller's back.
 *   - Return value: SPX_OK (0) or a negative error code; spx_last_error() gives the message of
 *     the calling thread's last failure.
 *   - Per-cell failures are not errors: they are status codes (SPX_ST_*), NaN geometry.
 */
#ifndef SUBPX_B200_H
#define SUBPX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    SPX_OK = 0,
    SPX_ERR_ARGUMENT = -1,
    SPX_ERR_CUDA = -2,
    SPX_ERR_CAPACITY = -3,
    SPX_ERR_UNSUPPORTED = -4
};

/* Pixel dtypes of input images. */
enum { SPX_U8 = 0, SPX_U16 = 1, SPX_F32 = 2, SPX_F64 = 3 };

/* Centre refinement methods (subpx/_cpu/centers.py:225-244 refine_centers_cpu). */
enum { SPX_REFINE_NONE = 0, SPX_REFINE_WEIGHTED = 1, SPX_REFINE_LOGQUAD = 2, SPX_REFINE_EDGE = 3,
       SPX_REFINE_AUTO = 4 };

/* Per-cell statuses (subpx/_cpu/cd.py:64-87, 226-264; subpx/_cpu/deblend.py:262-277). */
enum {
    SPX_ST_OK = 0,
    SPX_ST_NO_SIGNAL = 1,
    SPX_ST_INSUFFICIENT_CELL_PIXELS = 2,
    SPX_ST_INSUFFICIENT_FIT_PIXELS = 3,
    SPX_ST_SINGULAR_FIT = 4,
    SPX_ST_NON_GAUSSIAN_FIT = 5,
    SPX_ST_CONTOUR_OUTSIDE_CELL = 6,
    SPX_ST_INCOMPLETE_RAYS = 7,
    SPX_ST_FIT_DIVERGED = 8,
    SPX_ST_CENTER_OUTSIDE_CELL = 9
};

const char* spx_last_error(void);
int spx_version(void);
/* Number of SMs of the current device, and whether it is an sm_100 part (1) or not (0). */
int spx_device_info(int* sm_count, int* is_sm100);

/* ------------------------------------------------------------------------------------------------
 * Segmentation: Otsu threshold, binarisation, 8/4-connected components with stats.
 * Replaces cv2.threshold(THRESH_OTSU) in subpx/_cpu/centers.py:247-266 (_segment_binary),
 * subpx/_gpu/centers.py:1789-1796 (global Otsu of img[::ds, ::ds] for the tiled path) and
 * cv2.connectedComponentsWithStats in subpx/_cpu/components.py:18-32.
 * ---------------------------------------------------------------------------------------------- */

size_t spx_otsu_workspace_bytes(int dtype);
/* Otsu threshold of img[::step, ::step] (u8: 256 bins, u16: 65536 bins), as OpenCV's THRESH_OTSU.
 * Writes the threshold (a whole number, as double) to *threshold (device). */
int spx_otsu(const void* img, int dtype, int height, int width, int step, double* threshold,
             void* workspace, size_t workspace_bytes, void* stream);

/* Triangle threshold of a uint8 image, as OpenCV's THRESH_TRIANGLE (uses the Otsu workspace). */
int spx_triangle(const void* img, int dtype, int height, int width, double* threshold,
                 void* workspace, size_t workspace_bytes, void* stream);

size_t spx_ccl_workspace_bytes(int height, int width);
/* Binarise (img > t, or img <= t with invert; t = *threshold_dev when threshold_dev is non-null,
 * else fixed_threshold) and label the foreground with `connectivity` 8 or 4. Writes provisional
 * labels into `labels` (H*W int32) and the component count K to *count (device int).
 * Label numbering follows OpenCV: components ordered by their first 2x2 block in row-pair scan
 * order (8-connectivity) or their first pixel in raster order (4-connectivity).
 * The workspace holds state that spx_ccl_finish reads: pass the same workspace to both. */
int spx_ccl_label(const void* img, int dtype, int height, int width, const double* threshold_dev,
                  double fixed_threshold, int invert, int connectivity, int* labels, int* count,
                  void* workspace, size_t workspace_bytes, void* stream);
/* Final labels (0 background, 1..K) in place, plus per-label stats [x, y, w, h, area] int32
 * ((K+1) x 5, row 0 = background) and centroids [cx, cy] double ((K+1) x 2), as
 * cv2.connectedComponentsWithStats. */
int spx_ccl_finish(int* labels, int height, int width, int connectivity, int num_components,
                   int* stats, double* centroids, void* workspace, size_t workspace_bytes,
                   void* stream);

/* ------------------------------------------------------------------------------------------------
 * Component selection and centre refinement.
 * Replaces the per-label Python loops of subpx/_cpu/centers.py:376-391 and
 * subpx/_gpu/centers.py:1636-1650 (area filter, refine="auto" bucketing), and the refiners
 * refine_weighted_centroid_cpu (:45-64), refine_logquadratic_cpu (:67-107),
 * refine_edge_moment_cpu (:153-223) and method "none" (:239-243).
 * ---------------------------------------------------------------------------------------------- */

size_t spx_select_workspace_bytes(int num_components);
/* Keeps labels 1..K with area_min <= area <= area_max, in label order. rows_out receives
 * [x, y, w, h, label] int32 per kept component, methods_out the refine method (auto resolved by
 * max(w, h) <= small_feature_max -> logquad else edge), *kept the count (device int). */
int spx_select_components(const int* stats, int num_components, int area_min, int area_max,
                          int refine, double small_feature_max, int* rows_out,
                          uint8_t* methods_out, int* kept, void* workspace,
                          size_t workspace_bytes, void* stream);

/* One centre per row: ROI = bbox +- pad clipped to the image, mask = labels == label.
 * centers_out (n x 2 double) gets global [x, y] or NaN where the refiner fails. */
int spx_refine_centers(const void* img, int dtype, int height, int width, const int* labels,
                       const int* rows, const uint8_t* methods, int n, int pad,
                       double* centers_out, void* stream);

/* ------------------------------------------------------------------------------------------------
 * Voronoi partition. Replaces subpx/_cpu/cells.py:8-33 (compute_voronoi_labels_cpu, cKDTree) and
 * subpx/_gpu/voronoi.py:124-151 (_labels_device): nearest seed by FP64 squared distance
 * dx*dx + dy*dy (no FMA), exact ties to the lowest seed index; -1 everywhere without seeds.
 * ---------------------------------------------------------------------------------------------- */

size_t spx_voronoi_workspace_bytes(int n, int height, int width);
int spx_voronoi_labels(const double* seeds, int n, int height, int width, int* labels,
                       void* workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SUBPX_B200_H */
