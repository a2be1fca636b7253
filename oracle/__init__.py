"""CPU oracle of the subpx metrology hot path — TEST INFRASTRUCTURE, never the product.

A restatement, in NumPy/SciPy, of the reference algorithms that the CUDA library replaces
(ywk3484/ImageProcessor_new, package ``subpx``). Each function cites the reference file:line it
follows. Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
import this package, and only as the checker / the timed CPU baseline.

Parity is pinned: ``tests/golden/`` holds fixtures produced by running the reference's own CPU path
(OpenCV 4.13, SciPy, NumPy) in a container where it is importable (``tests/golden/make_golden.py``),
and ``tests/test_oracle_golden.py`` checks this oracle against every fixture.

Third-party arithmetic the reference delegates and how it is restated here:
  * cv2.threshold(THRESH_OTSU / THRESH_TRIANGLE): OpenCV's published histogram scans, restated
    step by step (same FP64 operation order), see ``segment.py``.
  * cv2.connectedComponentsWithStats: components are the 8/4-connected sets of foreground pixels
    (scipy.ndimage.label finds them); OpenCV's numbering is restated (first 2x2 block in row-pair
    scan order for 8-connectivity, raster order for 4).
  * scipy.spatial.cKDTree nearest seed: the exact rule argmin (d2, index) evaluated directly.
"""
