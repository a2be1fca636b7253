"""B200-native (sm_100a) subpixel-metrology hot path with the subpx API.

Drop-in for the GPU backend of ``subpx`` (ywk3484/ImageProcessor_new): Otsu thresholding,
connected components, per-blob centre refinement, the Voronoi cell partition and per-cell CD
measurement run as hand-written CUDA kernels in ``libsubpx_b200.so`` behind a C ABI
(``include/subpx_b200.h``). There is no CPU fallback.
"""

from .types import CDMethodResult, CDResult, CDSummary, CenterResult, ComponentStatsResult
from .centers import (
    choose_refine_method_for_bbox,
    detect_centers,
    detect_centers_batch,
    detect_centers_tiled,
    detect_centers_tiled_global_otsu,
    filter_centers,
    recommend_refine_method,
)
from .cd import METHOD_LABELS, measure_cds
from .results import load_cd_results, save_cd_arrays, save_cd_results, save_cd_tables
from .segment import connected_components_stats
from .voronoi import compute_voronoi_labels, compute_voronoi_labels_gpu

__version__ = "0.1.0"

__all__ = [
    "CDMethodResult", "CDResult", "CDSummary", "CenterResult", "ComponentStatsResult", "METHOD_LABELS",
    "measure_cds", "load_cd_results", "save_cd_arrays", "save_cd_results", "save_cd_tables",
    "choose_refine_method_for_bbox", "compute_voronoi_labels", "compute_voronoi_labels_gpu",
    "connected_components_stats", "detect_centers", "detect_centers_batch", "detect_centers_tiled",
    "detect_centers_tiled_global_otsu", "filter_centers", "recommend_refine_method",
]
