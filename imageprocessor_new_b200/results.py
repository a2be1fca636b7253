"""Result files of measure_cds: save_cd_results / load_cd_results (drop-in for subpx/cd.py:872-1131).

A results folder holds measurements.csv (one row per cell and method, pixel and calibrated
values), cells.csv (one row per cell), contours.csv (every contour vertex; not in compact
exports), raw_data.npz (the arrays of the CDResult, loadable with allow_pickle=False) and
manifest.json (parameters, definitions, calibration, per-method counts). The file names, CSV
columns, NPZ keys and manifest keys are the reference's, so that folders written by either package
load in the other.

``compact=True`` (batches of large pages) writes no contours.csv and an uncompressed NPZ without
the arrays that load_cd_results rebuilds: each method's contours (from its stored geometry, by
spx_rebuild_contours), the measured cells ``rois`` (from masks, origins, the deblended params and
the background tiles, by spx_render_model / spx_background_rows / spx_clean_masked), the component
labels (spx_ccl_* on the stored binary image) and the background map (from its tile medians). The
rebuilds run on the device with the measurement kernels' own arithmetic.
"""

from __future__ import annotations

import csv
import json
from pathlib import Path

import numpy as np

from .types import CDMethodResult, CDResult, CDSummary

CELL_ARRAYS = ("image", "binary", "component_labels", "component_ids", "boxes_xywh", "seeds_xy", "cell_labels",
               "cell_areas_px2", "mean_intensity", "origins_xy", "rois", "masks")
METHOD_ARRAYS = ("centers_xy", "contours_xy", "valid", "status")
# Length metrics and their calibrated CSV names (areas scale with the pixel size squared).
CALIBRATED = {"area_px2": "area", "cd_equivalent_px": "cd_equivalent", "cd_x_px": "cd_x", "cd_y_px": "cd_y",
              "perimeter_px": "perimeter", "fwhm_major_px": "fwhm_major", "fwhm_minor_px": "fwhm_minor",
              "cd_uncertainty_px": "cd_uncertainty"}
DEFINITIONS = {
    "gaussian": "Half-maximum ellipse of a 2-D Gaussian fitted by least squares jointly with a smooth background "
                "map and every neighbouring hole (deblended); FWHM = 2 sqrt(2 ln 2) sigma.",
    "logquad": "Half-maximum ellipse of a weighted log-quadratic fit of the background-subtracted cell; "
               "FWHM = 2 sqrt(2 ln 2) sigma.",
    "gradient": "Closed polygon through the subpixel maxima of the outward decrease of the radial profiles.",
    "halfmax": "Closed polygon through the first outward crossings of half the central signal.",
    "cd_equivalent": "2 sqrt(contour area / pi): analytic ellipse area for the ellipse methods, polygon area "
                     "otherwise.",
    "cd_x_cd_y": "Axis-aligned extents of the contour; analytic ellipse projections for the ellipse methods.",
    "failed_cells": "Kept with valid=False, their status and NaN geometric metrics.",
    "calibration": "NPZ geometry is in pixels; unsuffixed CSV lengths are in `unit`, areas in unit squared; "
                   "cell areas are Voronoi areas.",
    "background_map": "Fitted background in original intensity units; rois are the measured cells with the "
                      "background and the neighbours' models removed, in polarity-normalised units.",
    "mean_intensity": "Mean of the original pixels over the full Voronoi cell (background included).",
    "deblend": "deblend_params: global [amplitude, x0, y0, u1, u2, u3] of every modelled hole (precision L L^T, "
               "L = [[e^u1, 0], [u2, e^u3]]); deblend_report: the measured cells among them; deblend_tile_medians "
               "and deblend_tile_px: the background map's tiles.",
    "compact": "A compact raw_data.npz omits contours_xy, rois, component_labels and (when tile medians exist) "
               "background_map; load_cd_results rebuilds them from <method>_geometry_*, deblend_* and masks.",
}


def _names(compact: bool) -> tuple[str, ...]:
    return ("measurements.csv", "cells.csv") + (() if compact else ("contours.csv",)) + ("raw_data.npz",
                                                                                          "manifest.json")


def _require_full(result, compact: bool):
    if isinstance(result, CDSummary):
        raise ValueError("image exports require summary_only=False")
    if compact and result.meta.get("metrics_only"):
        raise ValueError("compact geometry export requires metrics_only=False; save tables or a full NPZ instead")


def save_cd_results(result: CDResult, output, *, compact: bool = False) -> dict[str, Path]:
    """measurements.csv, cells.csv, contours.csv (unless compact), raw_data.npz and manifest.json
    in the folder `output` (subpx/cd.py:877-897)."""
    _require_full(result, compact)
    return {**save_cd_tables(result, output, compact=compact), **save_cd_arrays(result, output, compact=compact)}


def save_cd_tables(result: CDResult, output, *, compact: bool = False) -> dict[str, Path]:
    """The CSV files of save_cd_results (subpx/cd.py:904-953)."""
    if isinstance(result, CDSummary):
        raise ValueError("cell tables require summary_only=False; batch page tables accept a summary")
    out = Path(output)
    out.mkdir(parents=True, exist_ok=True)
    paths = {name: out / name for name in _names(compact) if name.endswith(".csv")}
    scale = float(result.pixel_size)
    metric_names = sorted({k for m in result.measurements.values() for k in m.metrics})
    n = len(result.seeds_xy)
    cell_ids = list(range(n))
    comp = np.asarray(result.component_ids).tolist()
    sx, sy = result.seeds_xy[:, 0].tolist(), result.seeds_xy[:, 1].tolist()
    means = result.mean_intensity.tolist()
    nan_col = [np.nan] * n
    header = ["cell_id", "component_id", "method", "valid", "status", "seed_x_px", "seed_y_px", "center_x_px",
              "center_y_px", "center_x", "center_y", "unit", "pixel_size", "mean_intensity"]
    with paths["measurements.csv"].open("w", newline="", encoding="utf-8") as fh:
        wr = csv.writer(fh)
        wr.writerow(header + metric_names + list(CALIBRATED.values()))
        for method, m in result.measurements.items():
            cx, cy = m.centers_xy[:, 0], m.centers_xy[:, 1]
            cols = [cell_ids, comp, [method] * n, m.valid.tolist(), m.status.tolist(), sx, sy, cx.tolist(),
                    cy.tolist(), (cx * scale).tolist(), (cy * scale).tolist(), [result.unit] * n, [scale] * n,
                    means]
            cols += [m.metrics[k].tolist() if k in m.metrics else nan_col for k in metric_names]
            for k in CALIBRATED:
                if k in m.metrics:
                    factor = scale ** 2 if k == "area_px2" else scale
                    cols.append(np.where(m.valid, m.metrics[k] * factor, np.nan).tolist())
                else:
                    cols.append(nan_col)
            wr.writerows(zip(*cols))
    with paths["cells.csv"].open("w", newline="", encoding="utf-8") as fh:
        wr = csv.writer(fh)
        wr.writerow(["cell_id", "component_id", "seed_x_px", "seed_y_px", "cell_area_px2", "mean_intensity"])
        wr.writerows(zip(cell_ids, comp, sx, sy, np.asarray(result.cell_areas_px2).tolist(), means))
    if not compact:
        with paths["contours.csv"].open("w", newline="", encoding="utf-8") as fh:
            wr = csv.writer(fh)
            wr.writerow(["cell_id", "component_id", "method", "valid", "vertex", "x_px", "y_px", "x", "y", "unit"])
            for method, m in result.measurements.items():
                nv = m.contours_xy.shape[1]
                for lo in range(0, n, 4096):  # bounded Python lists on large pages
                    block = m.contours_xy[lo:lo + 4096]
                    cells = np.repeat(np.arange(lo, lo + len(block)), nv)
                    x, y = block[..., 0].ravel(), block[..., 1].ravel()
                    wr.writerows(zip(cells.tolist(), np.asarray(result.component_ids)[cells].tolist(),
                                     [method] * len(cells), np.repeat(m.valid[lo:lo + len(block)], nv).tolist(),
                                     np.tile(np.arange(nv), len(block)).tolist(), x.tolist(), y.tolist(),
                                     (x * scale).tolist(), (y * scale).tolist(), [result.unit] * len(cells)))
    return paths


def save_cd_arrays(result: CDResult, output, *, compact: bool = False) -> dict[str, Path]:
    """raw_data.npz and manifest.json of save_cd_results (subpx/cd.py:956-1047)."""
    _require_full(result, compact)
    out = Path(output)
    out.mkdir(parents=True, exist_ok=True)
    names = _names(compact)
    paths = {name: out / name for name in names[-2:]}
    model = result.deblend_model or {}
    if compact and result.meta.get("background") == "model" and "params" not in model:
        raise ValueError("compact export of background='model' results needs result.deblend_model")
    dropped = ("component_labels", "rois") if compact else ()
    arrays = {name: getattr(result, name) for name in CELL_ARRAYS if name not in dropped}
    arrays.update(pixel_size=np.asarray(float(result.pixel_size)), unit=np.asarray(result.unit),
                  methods=np.asarray(list(result.measurements)))
    for key, value in model.items():
        arrays[f"deblend_{key}"] = np.asarray(value)
    if result.background_map is not None and not (compact and "tile_medians" in model):
        arrays["background_map"] = result.background_map
    summary = {}
    for method, m in result.measurements.items():
        for name in METHOD_ARRAYS:
            if not (compact and name == "contours_xy"):
                arrays[f"{method}_{name}"] = getattr(m, name)
        for key, values in m.metrics.items():
            arrays[f"{method}_{key}"] = values
        if compact:
            if not m.geometry:
                raise ValueError(f"compact export needs the contour geometry of method {method!r}")
            for key, values in m.geometry.items():
                arrays[f"{method}_geometry_{key}"] = values
        statuses, counts = np.unique(m.status, return_counts=True)
        cds = m.metrics["cd_equivalent_px"][m.valid]
        summary[method] = {"valid": int(m.valid.sum()), "failed": int((~m.valid).sum()),
                           "status_counts": dict(zip(statuses.tolist(), counts.tolist())),
                           "median_cd_px": float(np.median(cds)) if cds.size else None,
                           "mean_cd_px": float(cds.mean()) if cds.size else None,
                           "std_cd_px": float(cds.std()) if cds.size else None}
    if compact:
        arrays["compact"] = np.asarray(True)
        np.savez(paths["raw_data.npz"], **arrays)  # uncompressed: zlib costs more time than it saves
    else:
        np.savez_compressed(paths["raw_data.npz"], **arrays)
    definitions = dict(DEFINITIONS, background=result.meta.get("background_definition", ""))
    manifest = {"schema_version": 2, "compact": bool(compact), "shape_hw": list(result.image.shape),
                "cells": int(len(result.seeds_xy)), "pixel_size": float(result.pixel_size), "unit": result.unit,
                "parameters": _jsonable(result.meta), "definitions": definitions, "methods": summary,
                "files": list(names)}
    paths["manifest.json"].write_text(json.dumps(manifest, indent=2, allow_nan=False) + "\n", encoding="utf-8")
    return paths


def _jsonable(value):
    """meta as strict JSON: NumPy scalars and arrays as Python values, non-finite floats as null."""
    if isinstance(value, dict):
        return {str(k): _jsonable(v) for k, v in value.items()}
    if isinstance(value, (list, tuple)):
        return [_jsonable(v) for v in value]
    if isinstance(value, np.ndarray):
        return _jsonable(value.tolist())
    if isinstance(value, np.generic):
        value = value.item()
    if isinstance(value, float) and not np.isfinite(value):
        return None
    return value


def load_cd_results(path, *, rois: bool = True) -> CDResult:
    """A results folder (or its raw_data.npz) written by save_cd_results, full or compact, as a
    CDResult (subpx/cd.py:1050-1113); meta from manifest.json beside the NPZ. Compact files have
    their contours, rois, component labels and background map rebuilt on the device; rois=False
    skips the measured cells (result.rois is then None)."""
    path = Path(path)
    npz = path / "raw_data.npz" if path.is_dir() else path
    manifest = npz.parent / "manifest.json"
    meta = json.loads(manifest.read_text(encoding="utf-8")).get("parameters", {}) if manifest.exists() else {}
    with np.load(npz, allow_pickle=False) as data:
        arrays = {name: data[name] for name in data.files}
    compact = bool(arrays.pop("compact", False))
    methods = arrays.pop("methods").tolist()
    model = {name[len("deblend_"):]: arrays.pop(name) for name in list(arrays) if name.startswith("deblend_")}
    if "tile_px" in model:
        model["tile_px"] = int(model["tile_px"])
    origins = arrays["origins_xy"]
    n_angles = int(meta.get("n_angles", 128))
    # Per-method arrays, each name to the longest method name that prefixes it.
    owned = {m: {} for m in methods}
    for name in list(arrays):
        owners = [m for m in methods if name.startswith(f"{m}_")]
        if owners:
            owner = max(owners, key=len)
            owned[owner][name[len(owner) + 1:]] = arrays.pop(name)
    measurements = {}
    for method in methods:
        own = owned[method]
        fields = {k: own.pop(k) for k in METHOD_ARRAYS if k in own}
        geometry = {k[len("geometry_"):]: own.pop(k) for k in list(own) if k.startswith("geometry_")}
        if "contours_xy" not in fields:
            fields["contours_xy"] = _rebuild_contours(method, fields, geometry, origins, n_angles)
        measurements[method] = CDMethodResult(method=method, metrics=own, geometry=geometry, **fields)
    shape = arrays["image"].shape
    sign = -1.0 if meta.get("invert") else 1.0
    if "background_map" not in arrays and "tile_medians" in model:
        arrays["background_map"] = sign * _background_from_tiles(model["tile_medians"], model["tile_px"], shape)
    if compact:
        arrays["component_labels"] = _component_labels(arrays["binary"])
        arrays["rois"] = _rebuild_rois(arrays, model, sign) if rois else None
    scalars = {"pixel_size": float(arrays.pop("pixel_size")), "unit": str(arrays.pop("unit"))}
    arrays.pop("mean_intensity", None)  # CDResult recomputes it from the image and the cell labels
    return CDResult(measurements=measurements, deblend_model=model or None, meta=meta,
                    background_map=arrays.pop("background_map", None), **scalars, **arrays)


def _rebuild_contours(method, fields, geometry, origins, n_angles) -> np.ndarray:
    import torch

    from . import _device as dev
    from . import _lib

    n = len(fields["valid"])
    out = dev.empty((max(n, 1), n_angles + 1, 2), torch.float64)
    up = {k: dev.upload(np.ascontiguousarray(v, dtype=np.float64)) for k, v in geometry.items()}
    org = dev.upload(np.ascontiguousarray(origins, dtype=np.int32))
    if "edge_px" in geometry:
        kind, centers = 2, None
    elif method == "logquad":
        kind, centers = 1, None
    else:
        kind, centers = 0, dev.upload(np.ascontiguousarray(fields["centers_xy"], dtype=np.float64))
    _lib.call("spx_rebuild_contours", kind, dev.ptr(centers), dev.ptr(up.get("center_local")),
              dev.ptr(up.get("eigenvalues")), dev.ptr(up.get("axes")), dev.ptr(up.get("edge_px")), org.data_ptr(), n,
              n_angles, out.data_ptr(), dev.stream_ptr())
    return out[:n].cpu().numpy()


def _background_from_tiles(medians, tile, shape) -> np.ndarray:
    from .deblend import Background

    return Background(shape, int(tile)).set_medians(np.asarray(medians, dtype=np.float64)).host_map()


def _component_labels(binary) -> np.ndarray:
    import torch

    from . import _device as dev
    from . import segment

    binary = np.asarray(binary)
    if not binary.any():
        return np.zeros(binary.shape, np.int32)
    img = dev.upload(binary.astype(np.uint8))
    comp = segment.label(img, fixed_threshold=0.0, connectivity=8)
    torch.cuda.current_stream().synchronize()
    return comp.labels.cpu().numpy()


def _rebuild_rois(arrays, model, sign) -> np.ndarray:
    """The measured cells as measure_cds stored them in CDResult.rois (subpx/cd.py:1116-1131)."""
    import torch

    from . import _device as dev
    from . import _lib
    from .deblend import Background

    masks, origins = arrays["masks"], arrays["origins_xy"]
    n, hm, wm = masks.shape
    if n == 0:
        return np.zeros((0, hm, wm))
    img = arrays["image"]
    img_d = dev.upload(img if img.dtype in _lib.DTYPES else img.astype(np.float64))
    h, w = img.shape
    params = np.ascontiguousarray(model["params"], dtype=np.float64)
    report = np.asarray(model["report"], dtype=np.int64)
    radius_cap = int(max(hm, wm))
    # The model image of every modelled hole (global params, zero box origins).
    m = len(params)
    params_d = dev.upload(params)
    zero_boxes = dev.upload(np.zeros((max(m, 1), 4), np.int32))
    ws = dev.workspace(_lib.size("spx_render_workspace_bytes", m, h, w))
    model_d = dev.empty((h, w), torch.float64)
    _lib.call("spx_render_model", params_d.data_ptr(), zero_boxes.data_ptr(), m, h, w, max(radius_cap, 2),
              model_d.data_ptr(), ws.data_ptr(), ws.numel(), dev.stream_ptr())
    if "tile_medians" in model:
        bg = Background((h, w), int(model["tile_px"])).set_medians(np.asarray(model["tile_medians"], np.float64))
    else:  # a full map of one level (background_level given) or without tiles
        bg = Background((h, w), max(h, w)).set_fixed(float(sign * np.asarray(arrays["background_map"]).flat[0]))
    out = dev.empty((n, hm, wm), torch.float64)
    # Uploads held in names until the launch: a temporary's block could be reused by the next upload
    # (enqueued before the kernel) on the same stream.
    masks_d = dev.upload(masks.astype(np.uint8))
    origins_d = dev.upload(np.ascontiguousarray(origins, np.int32))
    own_d = dev.upload(params[report])
    _lib.call("spx_clean_masked", img_d.data_ptr(), dev.dtype_code(img_d), float(sign), h, w, masks_d.data_ptr(),
              origins_d.data_ptr(), own_d.data_ptr(), max(radius_cap, 2), bg.struct(), model_d.data_ptr(), n, hm, wm,
              out.data_ptr(), dev.stream_ptr())
    return out.cpu().numpy()
