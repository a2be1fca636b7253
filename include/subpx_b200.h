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
    SPX_ST_CENTER_OUTSIDE_CELL = 9,
    SPX_ST_EDGE_AT_CELL_BORDER = 10,
    SPX_ST_REGION_AT_CELL_BORDER = 11
};

const char* spx_last_error(void);
int spx_version(void);
/* Number of kernel launches this library has issued in the process (for launch accounting). */
unsigned long long spx_launch_count(void);
/* Launch-shape knobs (process-wide, chosen by the autotuner; none changes a result):
 * "fit_warps" (2, 4, 8 cells in flight per block of the LM fit kernels), "fit_blocks_per_sm"
 * (2..32 persistent fit blocks per SM), "render_tile" (16, 32 or 64 pixel model-render tiles),
 * "radial_rays" (one ray per thread: 0 with a cached spline window, 2 reading the window at every
 * sample). No reference counterpart. */
int spx_tune_set(const char* knob, int value);
int spx_tune_get(const char* knob, int* value);
/* Number of SMs of the current device, and whether it is an sm_100 part (1) or not (0). */
int spx_device_info(int* sm_count, int* is_sm100);
/* FP64 FMA throughput probe (no reference counterpart): `blocks` x 256 threads each run eight
 * independent FP64 FMA chains of `iters` steps; *flops (host) = the launch's floating-point
 * operations (2 per FMA), so that a caller timing the launch gets the device's FP64 rate, the
 * denominator of an FP64-bound kernel's roofline. sink: blocks x 256 doubles. */
int spx_fp64_fma_rate(int blocks, int iters, double* sink, double* flops, void* stream);

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

/* Allocation-free Otsu threshold, for callers that cannot allocate device memory or pass a
 * workspace: code running inside CUDA stream capture or a real-time acquisition loop, where
 * cudaMalloc would synchronise the device or fail under a fixed memory budget, and hosts whose own
 * allocator owns every device byte. No counterpart in the reference: it is spx_otsu with its scratch
 * in a 2.3 MiB file-scope device array that every GPU loading the library holds until exit.
 * Limit: at most 4294967295 sampled pixels (ceil(H/step) * ceil(W/step)), the range of the 32-bit
 * histogram counts; larger images are rejected with SPX_ERR_ARGUMENT. The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress), so make it before any stream capture;
 * the address is kept until the process exits, so do not call it after a cudaDeviceReset.
 * All calls share the one array: calls that overlap on the GPU (other streams, other host threads)
 * race and must be serialised by the caller. Allocates nothing (no cudaMalloc, cudaFree or
 * allocating library call). */
int spx_otsu_static(const void* img, int dtype, int height, int width, int step, double* threshold, void* stream);

/* Histogram of img[::step, ::step] into hist (65536 uint32 counts, absolute grey levels) and its
 * [min, max] into range[2]. With spx_otsu_from_histogram this splits spx_otsu so that row shards of
 * one page on several GPUs can sum their histograms (and min / max their ranges) before the global
 * Otsu of subpx/_gpu/centers.py:1789-1796. */
int spx_histogram(const void* img, int dtype, int height, int width, int step, unsigned int* hist,
                  unsigned int* range, void* stream);
/* Otsu threshold (OpenCV THRESH_OTSU) of a histogram of `total` pixels with value range `range`;
 * the workspace is spx_otsu_workspace_bytes(dtype). */
int spx_otsu_from_histogram(const unsigned int* hist, int dtype, const unsigned int* range, long long total,
                            double* threshold, void* workspace, size_t workspace_bytes, void* stream);

/* Triangle threshold of a uint8 image, as OpenCV's THRESH_TRIANGLE (uses the Otsu workspace). */
int spx_triangle(const void* img, int dtype, int height, int width, double* threshold,
                 void* workspace, size_t workspace_bytes, void* stream);

/* bw (H x W uint8) = 255 where img > t (img <= t with invert), else 0, t = *threshold_dev or
 * fixed_threshold when threshold_dev is null: cv2.threshold(THRESH_BINARY[_INV]) as
 * subpx/_cpu/centers.py:257-258 and subpx/_gpu/centers.py:1515-1516 use it before morphology. */
int spx_binarize(const void* img, int dtype, int height, int width, const double* threshold_dev,
                 double fixed_threshold, int invert, uint8_t* out, void* stream);
/* In place on the 0/255 image bw: open_iterations x (erode) then open_iterations x (dilate)
 * (MORPH_OPEN), then close_iterations x (dilate) and close_iterations x (erode) (MORPH_CLOSE), each
 * with the 3x3 cross and image-border pixels ignored; tmp is an H x W scratch image.
 * subpx/_cpu/centers.py:260-265 (cv2.morphologyEx with MORPH_ELLIPSE (3, 3)). */
int spx_morphology(uint8_t* bw, int height, int width, int open_iterations, int close_iterations, uint8_t* tmp,
                   void* stream);

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

/* measure_cds cells (subpx/cd.py:485-500): the components 1..K with area_min <= area <= area_max in
 * label order as rows_out [x, y, w, h, cx, cy] (double), ids_out their labels, interior_out whether
 * the bbox keeps off the image border (x > 0, y > 0, x + w < width, y + h < height); oversized_out
 * (K + 1 bytes) flags labels with area > area_max. counts_out (device, 2 ints) = [kept, oversized].
 * Workspace: spx_select_workspace_bytes(K). */
int spx_component_rows(const int* stats, const double* centroids, int num_components, int area_min, int area_max,
                       int width, int height, double* rows_out, int* ids_out, uint8_t* interior_out,
                       uint8_t* oversized_out, int* counts_out, void* workspace, size_t workspace_bytes,
                       void* stream);

/* One centre per row: ROI = bbox +- pad clipped to the image, mask = labels == label.
 * centers_out (n x 2 double) gets global [x, y] or NaN where the refiner fails. */
int spx_refine_centers(const void* img, int dtype, int height, int width, const int* labels,
                       const int* rows, const uint8_t* methods, int n, int pad,
                       double* centers_out, void* stream);
/* spx_refine_centers for the first min(*n_dev, capacity) of `capacity` rows, the count read on the
 * device (rows past it get NaN centres), so a pipeline that selects and refines needs no host
 * read-back of the count and can be captured in a CUDA graph. */
int spx_refine_centers_counted(const void* img, int dtype, int height, int width, const int* labels,
                               const int* rows, const uint8_t* methods, const int* n_dev, int capacity, int pad,
                               double* centers_out, void* stream);

/* ------------------------------------------------------------------------------------------------
 * Tiled detection (detect_centers(tile_h=...), subpx/_gpu/centers.py:1778-1862 and
 * subpx/legacy.py:93-95): band keep rule and dedupe_centers (subpx/centers.py:335-378).
 * ---------------------------------------------------------------------------------------------- */

size_t spx_keep_band_workspace_bytes(int n);
/* Appends the finite centres of one band (band-local y) whose global y = y + y_offset lies in
 * [keep_lo, keep_hi) to out at the device counter *count (zero it before the first band), in order. */
int spx_keep_band(const double* centers, int n, double y_offset, double keep_lo, double keep_hi, double* out,
                  int* count, int capacity, void* workspace, size_t workspace_bytes, void* stream);
size_t spx_dedupe_workspace_bytes(int n, double xmin, double ymin, double xmax, double ymax, double eps);
/* Clusters of centres linked by squared distance <= eps^2 (union-find), each replaced by the mean
 * of its members summed in index order; clusters ordered by their smallest member; *count (device)
 * = number of clusters. out needs n rows. [xmin, xmax] x [ymin, ymax] bounds the centres. */
int spx_dedupe_centers(const double* centers, int n, double xmin, double ymin, double xmax, double ymax, double eps,
                       double* out, int* count, void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------------------------------
 * Voronoi partition. Replaces subpx/_cpu/cells.py:8-33 (compute_voronoi_labels_cpu, cKDTree) and
 * subpx/_gpu/voronoi.py:124-151 (_labels_device): nearest seed by FP64 squared distance
 * dx*dx + dy*dy (no FMA), exact ties to the lowest seed index; -1 everywhere without seeds.
 * ---------------------------------------------------------------------------------------------- */

size_t spx_voronoi_workspace_bytes(int n, int height, int width);
int spx_voronoi_labels(const double* seeds, int n, int height, int width, int* labels,
                       void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------------------------------
 * Deblending: smooth background map + one 2-D Gaussian per hole, fitted by Levenberg-Marquardt.
 * Replaces subpx/_cpu/deblend.py:421-522 (deblend) with subpx/_gpu/deblend.py:453-585 as the
 * reference GPU driver: fit_gaussians_batch (:174-254) / lm_fit, initial_params (:152-171),
 * fit_status (:262-277), clean_cells (:136-149), render_models (:87-107) / render_fixed,
 * _tile_medians (:280-291) / tile_medians, _upsample_tiles (:294-320). Cells are the Voronoi cells
 * of subpx/_gpu/cells.py:11-38 (box = bbox +- pad clipped; mask = box & labels == j), stored as
 * boxes (int4 x0, y0, w, h) over the label image instead of a mask stack. Params are ROI-local
 * [A, x0, y0, u1, u2, u3] as double[6] per cell.
 * ---------------------------------------------------------------------------------------------- */

enum { SPX_BG_MAP = 0, SPX_BG_FIXED = 1 };
/* Background map: bg(y, x) = (1 - t[y]) rows[j1[y]-1][x] + t[y] rows[j1[y]][x] (ny > 1),
 * rows[0][x] (ny == 1), or `fixed` (mode SPX_BG_FIXED). rows: ny x width; j1, t: one per image row. */
typedef struct spx_bgmap {
    const double* rows;
    const int* j1;
    const double* t;
    int ny;
    int width;
    double fixed;
    int mode;
} spx_bgmap;

/* Cell boxes, mask pixel counts and sigma caps max(1, sqrt(count / pi)) from rows (n x 6 double
 * [x, y, w, h, cx, cy]) and the Voronoi labels. */
int spx_cells_setup(const double* rows, int n, int pad, int height, int width, const int* voronoi,
                    int* boxes, int* counts, double* caps, void* stream);

/* Arithmetic of the LM fits (no reference counterpart; a null options pointer means FP64 with the
 * reference's rule). SPX_FIT_F64: every sum and the solve in FP64, as subpx/_cpu/deblend.py:174-254.
 * SPX_FIT_F32: the staged cell values, residuals, model, Jacobian and per-lane sums in FP32 (J^T J by
 * FMA, J^T r and the cost Kahan-compensated), lane totals added in FP64, and the damped solve, the
 * clipping, the step acceptance and the stop rule in FP64. cost_tol: relative cost drop at or below
 * which an accepted step ends a plain-start fit (1e-12 is the reference's rule; FP32 residuals
 * resolve cost changes down to a few 1e-7 of the cost). */
enum { SPX_FIT_F64 = 0, SPX_FIT_F32 = 1 };
typedef struct spx_fit_options {
    int precision;
    double cost_tol;
    int rows_per_image; /* 0: one image; > 0: the image is a stack of images this many rows high
                         * (boxes in stack rows, seeds in each cell's own image rows) */
} spx_fit_options;

size_t spx_fit_workspace_bytes(int max_cell_pixels);
/* Initial fits: 10th-percentile cell-border background (or background_level when has_level),
 * initial_params, LM (max_iter), fit_status. `sign` is -1 for inverted images. */
int spx_deblend_initial(const void* img, int dtype, double sign, int height, int width, const int* voronoi,
                        const int* boxes, const double* caps, const double* seeds, int n, int hm, int wm,
                        int max_cell_pixels, double background_level, int has_level, int max_iter,
                        double* params, uint8_t* status, int* iterations, void* workspace,
                        size_t workspace_bytes, void* stream);
/* spx_deblend_initial with a warm start: where init_params (n x 6, ROI-local) is given and
 * init_ok[j] is set (or init_ok is null), cell j's LM starts from init_params[j] and stops when
 * an accepted step lowers the cost by at most warm_cost_tol relative (1e-12 is the plain rule),
 * max |step| < 1e-7 or the damping exceeds 1e12; that fit is kept when it stops within max_iter and ends "ok", otherwise
 * the plain start runs as well (fallback_out[j] = 1; iterations counts both). background_out[j]
 * receives the cell-border background the fit subtracted and cost_out[j] (may be null) the LM cost
 * (sum of squared residuals) at the returned params, so that a caller can compare a warm-started
 * fit's converged cost with the plain fit's. options (null: FP64, cost_tol 1e-12) sets the fits'
 * arithmetic and the plain-start fits' stop rule. No reference counterpart (learned warm start). */
int spx_deblend_initial_warm(const void* img, int dtype, double sign, int height, int width, const int* voronoi,
                             const int* boxes, const double* caps, const double* seeds, int n, int hm, int wm,
                             int max_cell_pixels, double background_level, int has_level, int max_iter,
                             const double* init_params, const uint8_t* init_ok, double warm_cost_tol,
                             double* params, uint8_t* status, int* iterations, double* background_out,
                             uint8_t* fallback_out, double* cost_out, const spx_fit_options* options,
                             void* workspace, size_t workspace_bytes, void* stream);
/* One outer iteration: clean every cell against `model` and `background`, LM from `params`,
 * params_out = params + relaxation * (fitted - params), status of params_out, and maxstep =
 * max |step[1:]| (NaN unless the cell is ok with a finite fit). The cleaning is FP64 in both
 * arithmetics; options as for spx_deblend_initial_warm. */
int spx_deblend_iteration(const void* img, int dtype, double sign, int height, int width, const int* voronoi,
                          const int* boxes, const double* caps, int n, int hm, int wm, int max_cell_pixels,
                          const spx_bgmap* background, const double* model, int radius_cap,
                          const double* params, double relaxation, int max_iter, double* params_out,
                          uint8_t* status_out, double* maxstep, int* iterations, const spx_fit_options* options,
                          void* workspace, size_t workspace_bytes, void* stream);

size_t spx_render_workspace_bytes(int n, int height, int width);
/* Sum of every cell's truncated Gaussian (radius clip(ceil(4 sigma_major), 2, radius_cap)) into
 * model (H x W double), in increasing cell order per pixel (see spx_render_overflow). */
int spx_render_model(const double* params, const int* boxes, int n, int height, int width, int radius_cap,
                     double* model, void* workspace, size_t workspace_bytes, void* stream);
/* Render overflow flag kept in the render workspace (more than 2048 truncated Gaussians reaching
 * one 16x16 tile leaves that tile unrendered): reset = 1 clears it, reset = 0 copies it to the host
 * int *flag_out and synchronises the stream. */
int spx_render_overflow(void* workspace, int n, int height, int width, int* flag_out, int reset, void* stream);
/* Centre re-refinement on deblended cells (detect_centers(background="model"), subpx/centers.py:
 * 224-268): labels (n*hm x wm int32) marks, in cell j's window of the cleaned stack (rows j*hm ..
 * j*hm + hm - 1), the pixels of the cell's mask above 0.2 x its peak (fitted amplitude, else the
 * largest cleaned value) with j + 1; rows_out (n x 5) = [0, j*hm, wm, hm, j + 1], so that
 * spx_refine_centers on the stack as an (n*hm x wm) double image with pad 0 refines every cell. */
int spx_support_labels(const double* cleaned, const int* voronoi, const int* boxes, const double* params, int n,
                       int hm, int wm, int width, int* labels, int* rows_out, void* stream);
/* Cleaned cells of `which` (n_out indices; all cells when null) as an (n_out, hm, wm) stack. */
int spx_clean_cells(const void* img, int dtype, double sign, int height, int width, const int* voronoi,
                    const int* boxes, const double* params, int radius_cap, const spx_bgmap* background,
                    const double* model, const int* which, int n_out, int hm, int wm, double* out, void* stream);

enum { SPX_TILE_FREE = 0, SPX_TILE_USABLE = 1, SPX_TILE_ALL = 2 };
/* Per tile (ny x nx, row-major): median (mean of the middle pair; NaN if none) and count of the
 * residual sign*img - model over the selected pixels: SPX_TILE_FREE = usable & model < thr_model &
 * sqrt(dist2) >= thr_dist; SPX_TILE_USABLE = usable; SPX_TILE_ALL = every pixel. usable may be null. */
int spx_tile_medians(const void* img, int dtype, double sign, int height, int width, const double* model,
                     const unsigned int* dist2, const uint8_t* usable, int mode, double thr_model, double thr_dist,
                     int tile, double* medians, long long* counts, void* stream);
/* rows[j][x] = np.interp(x, tile-centre columns, medians[j]) (ny x width). */
int spx_background_rows(const double* medians, int ny, int nx, int tile, int width, double* rows, void* stream);
/* Order statistics on the device (np.median / np.percentile 'linear' of a selection), one request
 * per block: requests is a device array of n_requests structs {const double* values; int stride;
 * const uint8_t* mask; int finite_only; int n; int mode (0 median, 1 percentile); double q} laid
 * out as in C; out[2 b] = value (NaN if none selected), out[2 b + 1] = count. Replaces the host
 * medians and percentile of deblend (subpx/_cpu/deblend.py:463-464, 517). */
int spx_quantiles(const void* requests, int n_requests, double* out, void* stream);
/* fwhm[j] = 2 sqrt(2 ln 2) sigma_major(params[j]); good[j] = status ok and A > 0. */
int spx_cell_stats(const double* params, const uint8_t* status, int n, double* fwhm, uint8_t* good, void* stream);
/* sign * map_coordinates(background, [y, x], order=1, mode="nearest") at n points [x, y]
 * (the per-hole "background" metric, subpx/cd.py:719-721). */
int spx_background_at(const spx_bgmap* background, int height, int width, const double* points, int n,
                      double sign, double* out, void* stream);
/* out = sign*img - background - model (H x W double). */
int spx_residual(const void* img, int dtype, double sign, int height, int width, const spx_bgmap* background,
                 const double* model, double* out, void* stream);

/* Squared distance (uint32) from every pixel to the nearest rint()-ed, clipped seed pixel, as
 * scipy.ndimage.distance_transform_edt of the seed-pixel mask squared (subpx/_cpu/deblend.py:452-457).
 * Uses the Voronoi workspace. */
int spx_seed_distance_map(const double* seeds, int n, int height, int width, unsigned int* dist2,
                          void* workspace, size_t workspace_bytes, void* stream);
/* Distance from each query point to the nearest of `points` (excluding the same index when
 * exclude_self), as cKDTree.query (auto_tile's pitch, subpx/_cpu/deblend.py:396-403, and the
 * new-seed spacing test of revise_seeds, :564-566). Uses the Voronoi workspace sized for n points. */
int spx_nearest_distances(const double* points, int n, const double* queries, int nq, int exclude_self,
                          int height, int width, double* out, void* workspace, size_t workspace_bytes,
                          void* stream);

/* ------------------------------------------------------------------------------------------------
 * Seed revision and feature masks. Replaces the SciPy filters of revise_seeds
 * (subpx/_cpu/deblend.py:555-558: gaussian_filter / maximum_filter, mode "nearest"; the CuPy
 * variants in the reference GPU path), _unmodelled_features (subpx/cd.py:411-421) and the oversized
 * exclusion (subpx/cd.py:489-491).
 * ---------------------------------------------------------------------------------------------- */

/* Separable Gaussian filter (weights of length 2 radius + 1, symmetric), axis 0 then axis 1,
 * nearest edges; tmp is an H x W scratch image distinct from in and out. */
int spx_gaussian_filter(const double* in, int height, int width, const double* weights, int radius, double* tmp,
                        double* out, void* stream);
/* Separable maximum filter of size 2 radius + 1, nearest edges. */
int spx_maximum_filter(const double* in, int height, int width, int radius, double* tmp, double* out, void* stream);
/* Separable minimum filter of size 2 radius + 1, nearest edges (detect_peaks' prominence window,
 * subpx/_cpu/deblend.py:620). */
int spx_minimum_filter(const double* in, int height, int width, int radius, double* tmp, double* out, void* stream);
/* Pixels where smooth == maxf, smooth > level and not exclude[i] (exclude may be null), appended as
 * (y, x) int pairs in any order; *count (device) receives the total (may exceed capacity). */
int spx_find_peaks(const double* smooth, const double* maxf, const uint8_t* exclude, int height, int width,
                   double level, int* out_yx, int capacity, int* count, void* stream);
/* out[i] = flags[labels[i]] for labels > 0 (else 0), then `dilations` dilations with the 3x3 cross
 * (zero outside the image); tmp is an H x W byte scratch. */
int spx_label_mask(const int* labels, const uint8_t* flags, int height, int width, int dilations, uint8_t* out,
                   uint8_t* tmp, void* stream);

/* ------------------------------------------------------------------------------------------------
 * Peak seeds for arrays too dense to threshold: measure_cds(seeds="peaks") (subpx/cd.py:502-511)
 * with estimate_pitch and detect_peaks (subpx/_cpu/deblend.py:570-630).
 * ---------------------------------------------------------------------------------------------- */

/* out = sign * img as double (H x W), the signal the peak search and the pitch read. */
int spx_signal_image(const void* img, int dtype, double sign, int height, int width, double* out, void* stream);
size_t spx_pitch_workspace_bytes(int height, int width, int max_size);
/* The centred crop of estimate_pitch (at most max_size x max_size, offsets max(0, (H - max_size) / 2)
 * and likewise in x) times sign, minus its mean, in the top-left corner of `padded`, a zero
 * (2 ch) x (2 cw) double array (ch, cw = the crop's size): the input of the caller's FFT. */
int spx_pitch_crop(const void* img, int dtype, double sign, int height, int width, int max_size, double* padded,
                   void* workspace, size_t workspace_bytes, void* stream);
/* Pitch from the autocorrelation `autoc` (height2 x width2, zero lag at [0, 0], periodic, i.e. the
 * inverse FFT of the padded crop's power spectrum before fftshift): means of the lags in integer
 * radius bins 0..r_max (r_max = min(ch, cw) / 2), the first bin k >= 2 above its predecessor, at
 * least its successor and positive, refined by a parabola. *pitch (device) = NaN when none is
 * found. Uses the workspace of spx_pitch_crop. */
int spx_pitch_from_autocorrelation(const double* autoc, int height2, int width2, int r_max, double* pitch,
                                   void* workspace, size_t workspace_bytes, void* stream);
size_t spx_peak_workspace_bytes(int height, int width);
/* Pixels with smooth == maxf and prominence smooth - minf > 0, as (y, x) int pairs with their
 * prominence, in row-major order; *count (device) receives the total (may exceed capacity). */
int spx_peak_candidates(const double* smooth, const double* maxf, const double* minf, int height, int width,
                        int* out_yx, double* out_prom, int capacity, int* count, void* workspace,
                        size_t workspace_bytes, void* stream);
size_t spx_peak_select_workspace_bytes(int n);
/* Candidates with prom >= fraction * (*level) (level: a device double, e.g. the 90th percentile of
 * spx_quantiles), kept in order as [x, y] seeds moved by the parabola vertex of their row and column
 * neighbours in `smooth`, clipped to +-0.5 px; *count (device) = the number kept. */
int spx_peak_select(const int* yx, const double* prom, int n, const double* level, double fraction,
                    const double* smooth, int height, int width, double* out_xy, int* count, void* workspace,
                    size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------------------------------
 * CD measurements of cleaned cells (an (n, hm, wm) stack, zero outside each cell; cell i is cell
 * which[i] of the Voronoi labels / boxes, or i when which is null). Replaces subpx/_cpu/cd.py
 * measure_cells (:267-322: logquad, gradient, halfmax) and gaussian_method (:144-192), with the GPU
 * reference subpx/_gpu/cd.py (:31-131 rays, :147-207 logquad sums, :465-522 gaussian) as the
 * batched counterpart. Metric columns: 0 area_px2, 1 cd_equivalent_px, 2 cd_x_px, 3 cd_y_px,
 * 4 perimeter_px, 5 background, 6 peak_signal, then for the ellipse methods 7 sigma_major_px,
 * 8 sigma_minor_px, 9 fwhm_major_px, 10 fwhm_minor_px, 11 angle_deg, 12 log_fit_rmse (logquad) or
 * fit_rmse (gaussian); for the radial methods 7 ray_coverage.
 * ---------------------------------------------------------------------------------------------- */

typedef struct spx_method_out {
    double* centers;       /* n x 2 global [x, y] */
    double* contours;      /* n x (n_angles + 1) x 2 global, or null (metrics only) */
    uint8_t* status;       /* n status codes */
    double* metrics;       /* n x n_metrics (row-major), or n_metrics columns of n (metric_col_stride) */
    double* center_local;  /* n x 2 (radial, logquad) */
    double* edge_px;       /* n x n_angles (radial) */
    double* eigenvalues;   /* n x 2 (ellipse methods) */
    double* axes;          /* n x 2 x 2 (ellipse methods) */
    int n_metrics;
    long long metric_col_stride;  /* 0: row-major; else metric q of cell i at metrics[i + q * stride] */
} spx_method_out;

/* Status text of per-cell result codes as the reference's "U32" string arrays hold it: 32 UCS-4
 * code points per cell (text: n x 32 uint32), zero-padded, so a host copy can be viewed as a
 * NumPy "<U32" array. spx_status_name(code) is the same name as a C string (null for an unknown
 * code). No reference counterpart (the reference builds its string arrays on the host). */
const char* spx_status_name(int code);
int spx_status_text(const uint8_t* codes, int n, uint32_t* text, void* stream);

/* Half-maximum ellipses of the deblended Gaussian fits (params of cells `which`, ROI-local). */
int spx_gaussian_method(const double* params, const uint8_t* status_in, const double* cleaned, const int* voronoi,
                        const int* boxes, const int* which, int n, int hm, int wm, int width, int n_angles,
                        const spx_method_out* out, void* stream);
/* Weighted log-quadratic fit of log(signal) over pixels above fit_fraction x peak (background 0). */
int spx_logquad_cd(const double* cleaned, const int* voronoi, const int* boxes, const int* which, const double* seeds,
                   int n, int hm, int wm, int width, int n_angles, double fit_fraction, const spx_method_out* out,
                   void* stream);
/* The "projection" CD (subpx/_cpu/invariant_cd.py:365-421 _projection; 320-336 _set_ellipses): per
 * reported cell the x and y profiles of the cleaned cell summed over its mask, their not-a-knot
 * cubic splines (value_op_* / slope_op_*: size x g operators from the host, size wm for x and hm for
 * y, evaluated at k * step for k < g), the highest value inside each profile's span and the steepest
 * rise before / fall after it: widths cd_x, cd_y and the centre; drawn as the axis-aligned ellipse of
 * the two widths (edge_px, contours), area pi a b, cd_equivalent a + b (a, b the half widths),
 * Ramanujan's perimeter. Status ok, edge_at_cell_border (a rise or fall not strictly inside its span,
 * geometry metrics NaN, ellipse still drawn) or no_signal (peak <= 0). n_metrics >= 7. */
int spx_projection_cd(const double* cleaned, const int* voronoi, const int* boxes, const int* which, int n, int hm,
                      int wm, int width, int n_angles, double step, const double* value_op_x,
                      const double* slope_op_x, int gx, const double* value_op_y, const double* slope_op_y, int gy,
                      const spx_method_out* out, void* stream);

/* The half_area family (subpx/_cpu/invariant_cd.py:551-799, 802-875): half_area (median local level,
 * highest-pixel peak), half_area_min (minimum level) and half_area_min_avg (minimum level, peak =
 * mean of the n_top highest sub-pixels). Per reported cell the local level b (median = 1: median,
 * else minimum of the mask pixels with a 4-neighbour outside the mask or on the stack's edge), the
 * cell minus b enlarged factor times by zoom_y ((hm factor) x hm) and zoom_x ((wm factor) x wm),
 * the host's cubic zoom operators; the region = the 8-connected sub-pixels above b + level x peak
 * around the highest one; area, centroid, the equal-area ellipse's x / y diameters (cd_x, cd_y),
 * metrics local_level, threshold, mean_signal (columns 7-9; n_metrics >= 10) and, with outlines, the
 * display outline (edge_px, contours, perimeter). `single` gets the highest-pixel peak, `averaged`
 * the averaged one (either may be null; both share one enlargement). Status ok,
 * region_at_cell_border or no_signal. (hm factor) x (wm factor) <= 32768; workspace:
 * spx_half_area_workspace_bytes. */
size_t spx_half_area_workspace_bytes(int hm, int wm, int factor);
int spx_half_area_cd(const double* cleaned, const int* voronoi, const int* boxes, const int* which, int n, int hm,
                     int wm, int width, int n_angles, const double* zoom_y, const double* zoom_x, int factor,
                     double level, int median, int n_top, int outlines, const spx_method_out* single,
                     const spx_method_out* averaged, void* workspace, size_t workspace_bytes, void* stream);
/* Windows of the tail family (subpx/_cpu/invariant_cd.py:878-964, _wide_cells; replaces its CPU
 * branch and subpx/_gpu/windows.py wide_cells): for each reported hole rows[i] (of n_all modelled holes
 * with ROI-local Gaussian params (n_all, 6) and cell boxes (n_all, 4) of an hm x wm stack) the
 * (2 radius + 1)^2 window around its rounded fitted centre (box centre when not finite): cells =
 * float32((sign img - background) x own model / (model + floor)) inside the image, 0 outside; inside;
 * territory = inside and no farther from the hole than from its 8 nearest modelled holes (ties in
 * distance to the lower index; neighbours found in buckets of `bucket` px); level = the territory
 * pixels at or beyond the keep-th largest distance, keep = clip(max(count // 10, 4), 1, area) - 1;
 * origins = window origins (x, y). neighbours_out (optional, (n_rep, 9) ints) receives each row's hole
 * and its neighbours (-1 where fewer). 2 radius + 1 <= 64; workspace: spx_wide_cells_workspace_bytes. */
size_t spx_wide_cells_workspace_bytes(int n_all, int n_rep, int height, int width, double bucket);
int spx_wide_cells(const void* img, int dtype, double sign, int height, int width, const spx_bgmap* background,
                   const double* model, const double* params, const int* boxes, int n_all, int hm, int wm,
                   const int* rows, int n_rep, int radius, double bucket, double floor, float* cells, uint8_t* inside,
                   uint8_t* level, uint8_t* territory, int* origins, int* neighbours_out, void* workspace,
                   size_t workspace_bytes, void* stream);
/* The tail family on those windows (subpx/_cpu/invariant_cd.py:551-875 with measure_invariant's
 * tail branch 1009-1068): per window the local level (tail: median of the level pixels inside the
 * window; the others none), the window minus it enlarged factor times by zoom_y ((side factor) x side)
 * and zoom_x_t (side x (side factor), the x operator transposed), the averaged peak (n_top highest
 * sub-pixels), and the threshold: level x peak (tail = tail_area, norm = tail_area_norm), the
 * steepness-weighted mean of the core sub-pixels (edge = edge_area), the curvature-weighted mean below
 * the steepest level inside the territory (foot = foot_area; its steepest level in metric column 10,
 * n_metrics >= 11), or cuts[i] (given = foot_area_ratio). Region, metrics (columns 7-9: local_level,
 * threshold, mean_signal) and outline as spx_half_area_cd; centres and contours in image pixels,
 * center_local relative to cell_origins. Outputs may be null; (side factor)^2 <= 65536; workspace:
 * spx_tail_area_workspace_bytes. */
size_t spx_tail_area_workspace_bytes(int side, int factor, int n_angles);
int spx_tail_area_cd(const float* cells, const uint8_t* inside, const uint8_t* level_pixels, const uint8_t* territory,
                     const int* window_origins, const int* cell_origins, int n, int side, int n_angles,
                     const double* zoom_y, const double* zoom_x_t, int factor, double level, int n_top, int outlines,
                     const double* cuts, const spx_method_out* tail, const spx_method_out* norm,
                     const spx_method_out* edge, const spx_method_out* foot, const spx_method_out* given,
                     void* workspace, size_t workspace_bytes, void* stream);
size_t spx_radial_workspace_bytes(int hm, int wm, int smooth);
/* Cubic-spline radial profiles; half-height crossings (halfmax) and gradient maxima (gradient).
 * Either output may be null. smooth_weights (device, 2 smooth_radius + 1 symmetric Gaussian
 * weights, scipy's gaussian_filter kernel for smooth_sigma) selects the mask-normalised smoothing
 * of the profiles (subpx/_cpu/cd.py:206-208); null for smooth_sigma = 0. */
int spx_radial_cd(const double* cleaned, const int* voronoi, const int* boxes, const int* which, int n, int hm,
                  int wm, int width, int n_angles, double radial_step, const double* smooth_weights,
                  int smooth_radius, const spx_method_out* halfmax, const spx_method_out* gradient, void* workspace,
                  size_t workspace_bytes, void* stream);


/* ------------------------------------------------------------------------------------------------
 * Compact result files (save_cd_results(compact=True) / load_cd_results, subpx/cd.py:878-1131): the
 * arrays a compact file leaves out are rebuilt on the device from what it keeps.
 * ---------------------------------------------------------------------------------------------- */

/* Measured cells from their stored masks (n x hm x wm bytes), origins (n x 2 int [x, y]) and global
 * params (n x 6): image - background - (model - own truncated Gaussian) on the mask, 0 elsewhere
 * (subpx/cd.py:1116-1131 _rebuild_rois; the same arithmetic as spx_clean_cells). */
int spx_clean_masked(const void* img, int dtype, double sign, int height, int width, const uint8_t* masks,
                     const int* origins, const double* params_global, int radius_cap, const spx_bgmap* background,
                     const double* model, int n, int hm, int wm, double* out, void* stream);
/* Closed contours (n x (n_angles + 1) x 2) from stored geometry with the measurement kernels'
 * arithmetic (subpx/_cpu/cd.py:110-128 radial_contours / ellipse_contours): kind 0 gaussian
 * (centers, eigenvalues, axes), 1 logquad (center_local, eigenvalues, axes, origins), 2 radial
 * (center_local, edge_px, origins). */
int spx_rebuild_contours(int kind, const double* centers, const double* center_local, const double* eigenvalues,
                         const double* axes, const double* edge_px, const int* origins, int n, int n_angles,
                         double* contours, void* stream);

/* ------------------------------------------------------------------ learned warm start (MLP) */

/* Epilogue of spx_gemm_bf16: x = scale * acc (+ bias[n]); x = 0 where mask_act[m, n] <= 0 (the
 * ReLU derivative of a forward activation, bf16, row stride ld_mask) when mask_act is set;
 * x = max(x, 0) when relu; then any of: out_f32[m, n] (= or += with accumulate), out_bf16[m, n],
 * out_bf16_t[n, m] (transposed). */
typedef struct spx_gemm_epilogue {
    float scale;
    const float* bias;
    int relu;
    const void* mask_act;
    int ld_mask;
    float* out_f32;
    int ld_f32;
    int accumulate;
    void* out_bf16;
    int ld_bf16;
    void* out_bf16_t;
    int ld_t;
} spx_gemm_epilogue;

/* C (M x N) = A (M x K) B^T (B: N x K), bf16 operands with K contiguous (row strides lda, ldb,
 * multiples of 8 elements, 16-byte aligned), f32 accumulation in TMEM by tcgen05.mma, then the
 * epilogue. *error_flag (device int) is set to 1 if a completion wait gave up. No reference
 * counterpart: this and the MLP entry points below implement the learned warm start of the LM fits. */
int spx_gemm_bf16(const void* A, int lda, const void* B, int ldb, int M, int N, int K, const spx_gemm_epilogue* epi,
                  int* error_flag, void* stream);


/* Weighted MSE gradient of the MLP outputs y (batch x n_out f32) against t: dy (batch x ld_grad
 * bf16, zero padding columns) and its transpose (ld_grad x batch); *loss (device double) +=
 * mean_b sum_j w_j (y - t)^2. */
int spx_mlp_loss_grad(const float* y, const float* t, const float* weights, int batch, int n_out, int ld_grad,
                      void* dy, void* dy_t, double* loss, void* stream);
/* out[r] = sum of row r of a bf16 rows x cols matrix (f32): bias gradients from transposed
 * activation gradients. */
int spx_rowsum_bf16(const void* src, int rows, int cols, float* out, void* stream);
/* AdamW (decoupled weight decay, bias-corrected moments, step >= 1) on f32 params (rows x cols),
 * then optional bf16 copies: row-major with rows padded by zeros to out_rows, and transposed
 * (cols x ld_t, ld_t >= rows). */
int spx_adamw(float* param, const float* grad, float* m, float* v, int rows, int cols, int step, float lr, float beta1,
              float beta2, float eps, float weight_decay, void* out_bf16, int out_rows, void* out_bf16_t, int ld_t,
              void* stream);
/* dst (cols x rows) = src (rows x cols)^T, bf16. */
int spx_transpose_bf16(const void* src, int rows, int cols, void* dst, void* stream);
/* Standardised MLP outputs y (n x 7 f32) -> ROI-local LM starting params (n x 6): t = y * std +
 * mean; A = t0 amp, x0 = (origin x - box x) + 16 + t1, y0 = (origin y - box y) + 16 + t2, u = t3..t5,
 * with norm rows [origin x, origin y, bg, amp] of spx_extract_patches; ok = finite and A > 0. */
int spx_mlp_outputs_to_params(const float* y, const double* out_mean, const double* out_std, const double* norm,
                              const int* boxes, int n, double* params, uint8_t* ok, void* stream);
/* 32 x 32 signal patches (sign x image) centred on the rounded seeds [x, y], edges replicated,
 * normalised to (v - bg) / amp with bg the smallest mean of the 2 x 2 blocks along the border and
 * amp = max - bg, as bf16 (n x 1024); norm (n x 4 doubles) = [origin x, origin y, bg, amp]. */
int spx_extract_patches(const void* img, int dtype, double sign, int height, int width, const double* seeds, int n,
                        void* out, double* norm, void* stream);
/* spx_extract_patches over a stack of `images` images of height x width stored one after another
 * (images * height rows): boxes (n x 4 int [x, y, w, h], y in stack rows; may be null for one image)
 * give each cell's image, seeds are in that image's rows, each patch replicates the edges of its
 * cell's image (the patch the cell has in its own image), and norm's origin y is in stack rows. */
int spx_extract_patches_stack(const void* img, int dtype, double sign, int images, int height, int width,
                              const double* seeds, const int* boxes, int n, void* out, double* norm, void* stream);
/* Training pages: coverage (H x W doubles) of rotated superellipse holes (rows of [cx, cy, a, b,
 * theta, exponent]) sampled on samples x samples points per pixel, holes found through a CSR grid
 * of cell size `cell` (grid_start: grid_w * grid_h + 1 offsets into grid_ids). */
int spx_hole_coverage(int height, int width, const double* holes, const int* grid_start, const int* grid_ids,
                      int grid_w, int grid_h, double cell, int samples, double* coverage, void* stream);
/* page = clip(rint(background + amplitude x coverage + noise x N(0, 1)), 0, 65535) as uint16, the
 * normal deviates from a counter-based hash of (seed, pixel). */
int spx_page_finish(const double* coverage, long long n, double background, double amplitude, double noise,
                    unsigned long long seed, uint16_t* page, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SUBPX_B200_H */
