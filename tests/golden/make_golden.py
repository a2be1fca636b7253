"""Generates the golden fixtures of tests/golden/ by running the REFERENCE's own CPU path.

Run in a container where the reference checkout (ywk3484/ImageProcessor_new, package ``subpx``) and
its CPU dependencies (OpenCV, SciPy) are importable:

    python tests/golden/make_golden.py --reference /path/to/ImageProcessor_new [--only NAME]

Inputs are seeded synthetic images built with imageprocessor_new_b200.synthetic (or small random
arrays); outputs are whatever the reference functions return. The fixtures are small .npz files;
tests compare the oracle (CPU) and the CUDA library against them.
"""

from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))


def _ref(path: str):
    sys.path.insert(0, path)
    import subpx  # noqa: F401

    return subpx


def threshold_images():
    from imageprocessor_new_b200 import synthetic as S

    rng = np.random.default_rng(0)
    imgs = []
    for t in range(12):
        kind = t % 4
        if kind == 0:
            imgs.append(rng.integers(0, 65536, (37, 53)).astype(np.uint16))
        elif kind == 1:
            img = rng.normal(1000, 50, (64, 64)) + (rng.random((64, 64)) < 0.3) * 3000
            imgs.append(img.clip(0, 65535).astype(np.uint16))
        elif kind == 2:
            imgs.append(rng.integers(0, 256, (31, 29)).astype(np.uint8))
        else:
            imgs.append(rng.integers(990, 1010, (20, 33)).astype(np.uint16))
    page = S.page_square(0).image
    imgs.append(np.ascontiguousarray(page[:256, :256]))
    imgs.append(np.ascontiguousarray(page[::4, ::4]))
    u8 = (page[:200, :300] >> 4).astype(np.uint8)
    imgs.append(u8)
    return imgs


def make_thresholds(out: Path):
    import cv2

    imgs = threshold_images()
    otsu = [cv2.threshold(im, 0, 255, cv2.THRESH_BINARY | cv2.THRESH_OTSU)[0] for im in imgs]
    tri = [cv2.threshold(im, 0, 255, cv2.THRESH_BINARY | cv2.THRESH_TRIANGLE)[0] if im.dtype == np.uint8
           else np.nan for im in imgs]
    arrays = {f"img{i}": im for i, im in enumerate(imgs)}
    np.savez_compressed(out / "thresholds.npz", otsu=np.array(otsu), triangle=np.array(tri), n=len(imgs), **arrays)


def make_ccl(out: Path):
    import cv2
    from scipy import ndimage

    rng = np.random.default_rng(1)
    arrays = {}
    cases = []
    for t in range(10):
        h, w = int(rng.integers(1, 70)), int(rng.integers(1, 70))
        mask = rng.random((h, w)) < rng.uniform(0.05, 0.7)
        cases.append(mask)
    blobs = ndimage.binary_dilation(rng.random((300, 257)) < 0.01, iterations=3) | (rng.random((300, 257)) < 0.02)
    cases.append(blobs)
    big = rng.random((1100, 900)) < 0.45
    cases.append(big)
    for i, mask in enumerate(cases):
        bw = mask.astype(np.uint8) * 255
        arrays[f"mask{i}"] = np.packbits(mask, axis=None)
        arrays[f"shape{i}"] = np.array(mask.shape)
        for conn in (8, 4):
            n, lab, stats, cents = cv2.connectedComponentsWithStats(bw, connectivity=conn)
            arrays[f"labels{i}_{conn}"] = lab.astype(np.int32)
            arrays[f"stats{i}_{conn}"] = stats.astype(np.int32)
            arrays[f"cent{i}_{conn}"] = cents
    np.savez_compressed(out / "ccl.npz", n=len(cases), **arrays)


def center_images():
    from imageprocessor_new_b200 import synthetic as S

    page = S.page_square(0).image
    dots, _ = S.dot_grid(rows=5, cols=6, spacing=17, dot_size=4, margin=9)
    rng = np.random.default_rng(5)
    small = S.render((160, 200), S.square_grid((160, 200), 20.0, rng), 8.0 + rng.normal(0, 0.3, 80), 1.2,
                     amplitude=2000.0, background=500.0)
    small = S.add_noise(small, rng, read_noise=15.0)
    return {
        "page": (np.ascontiguousarray(page[:384, :512]), dict(threshold="otsu", area_max=400)),
        "dots": (dots, dict(threshold="otsu", area_max=50)),
        "small": (small, dict(threshold="otsu", area_max=200)),
        "dots_tri": (dots, dict(threshold="triangle", area_max=50)),
        "small_morph": (small, dict(threshold="otsu", area_max=200, morph_open=1, morph_close=1)),
        "page_morph": (np.ascontiguousarray(page[:256, :384]), dict(threshold="otsu", area_max=400, morph_open=2,
                                                                    morph_close=1)),
    }


def make_centers(out: Path, ref):
    from subpx._cpu.centers import detect_centers_cpu

    arrays = {}
    names = []
    for name, (img, kw) in center_images().items():
        arrays[f"{name}_img"] = img
        for refine in ("weighted", "logquad", "edge_gradmoment", "none", "auto"):
            for invert in (False,):
                res = detect_centers_cpu(img, refine=refine, invert=invert, **kw)
                arrays[f"{name}_{refine}"] = res.centers_xy
        names.append(name)
    np.savez_compressed(out / "centers.npz", names=np.array(names), **arrays)


def voronoi_cases():
    rng = np.random.default_rng(3)
    shape = (130, 170)
    return {
        "uniform": (rng.uniform(0, [170, 130], (500, 2)), shape),
        "clustered": (rng.uniform(0, [60, 40], (400, 2)), shape),
        "integer_ties": (np.column_stack(np.nonzero(np.ones((20, 20))))[:, ::-1] * 6.0 + 3, shape),
        "few": (rng.uniform(0, [170, 130], (5, 2)), shape),
        "two": (np.array([[10.0, 10.0], [100.0, 50.0]]), shape),
        "outside": (rng.uniform(-20, [190, 150], (300, 2)), shape),
    }


def make_voronoi(out: Path, ref):
    from subpx._cpu.cells import compute_voronoi_labels_cpu

    arrays = {}
    for name, (seeds, shape) in voronoi_cases().items():
        arrays[f"{name}_seeds"] = seeds
        arrays[f"{name}_shape"] = np.array(shape)
        arrays[f"{name}_labels"] = compute_voronoi_labels_cpu(seeds, shape)
    np.savez_compressed(out / "voronoi.npz", names=np.array(list(voronoi_cases())), **arrays)


def make_tiled(out: Path, ref):
    """The reference GPU tiled driver's rules composed from reference CPU pieces (cv2 threshold and
    CCL, refine_centers_cpu, dedupe_centers), since the GPU driver itself needs CuPy."""
    import cv2
    from subpx._cpu.centers import refine_centers_cpu
    from subpx._cpu.components import connected_components_stats_cpu
    from subpx.centers import dedupe_centers

    from imageprocessor_new_b200 import synthetic as S

    rng = np.random.default_rng(9)
    shape = (700, 300)
    centers = S.square_grid(shape, 20.0, rng)
    img = S.add_noise(S.render(shape, centers, 10.0 * (1 + rng.uniform(-0.04, 0.04, len(centers))), 1.0,
                               amplitude=3000.0, background=1000.0), rng, read_noise=30.0)
    tile_h, overlap, ds, scale = 256, 64, 4, 0.8
    otsu, _ = cv2.threshold(np.ascontiguousarray(img[::ds, ::ds]), 0, 255, cv2.THRESH_BINARY | cv2.THRESH_OTSU)
    pre = float(otsu) * scale
    H, W = img.shape
    step = tile_h - overlap
    kept = []
    y0 = 0
    while y0 < H:
        y1 = min(H, y0 + tile_h)
        tile = img[y0:y1]
        _, bw = cv2.threshold(tile, pre, 255, cv2.THRESH_BINARY)
        comp = connected_components_stats_cpu(bw, connectivity=8)
        pts = []
        for lab in range(1, comp.num_labels):
            x, y, w, h, area = comp.stats[lab]
            if area < 1 or area > 200:
                continue
            xa, ya = max(0, int(x) - 3), max(0, int(y) - 3)
            xb, yb = min(W, int(x + w) + 3), min(y1 - y0, int(y + h) + 3)
            cx, cy = refine_centers_cpu(tile[ya:yb, xa:xb], comp.labels[ya:yb, xa:xb] == lab, method="logquad")
            if np.isfinite(cx) and np.isfinite(cy):
                pts.append([xa + cx, ya + cy + y0])
        pts = np.asarray(pts).reshape(-1, 2)
        half = overlap // 2
        lo = y0 if y0 == 0 else y0 + half
        hi = y1 if y1 == H else y1 - half
        kept.append(pts[(pts[:, 1] >= lo) & (pts[:, 1] < hi)])
        if y1 == H:
            break
        y0 += step
    merged = dedupe_centers(np.vstack(kept), eps=1.5)
    raw = np.vstack(kept)
    np.savez_compressed(out / "tiled.npz", img=img, pre_threshold=pre, raw=raw, centers=merged,
                        tile_h=tile_h, overlap=overlap)


def cd_cases():
    from imageprocessor_new_b200 import synthetic as S

    lat2, _ = S.gaussian_lattice(2.0, shape=(120, 240))
    lat14, _ = S.gaussian_lattice(1.4, shape=(120, 240), seed=1)
    page = np.ascontiguousarray(S.page_square(0).image[:256, :320])
    rng = np.random.default_rng(11)
    cen = S.staggered_grid((192, 256), 24.0, rng)
    stag = S.add_noise(S.render((192, 256), cen, 12.0 * (1 + rng.uniform(-0.05, 0.05, len(cen))), 1.2,
                                amplitude=3000.0, background=1000.0), rng, read_noise=100.0, poisson=False)
    # Seed revision: faint spots found by peak seeding and dropped after the first pass; narrow spots
    # that thresholding misses (below area_min) and the residual check adds.
    drop, _ = S.gaussian_lattice(2.0, faint=6, faint_amplitude=0.26, seed=3)
    add, _ = S.gaussian_lattice(1.8, small=6, faint=6, faint_amplitude=0.26, seed=3)
    clean20, _ = S.gaussian_lattice(2.0, snr=0)
    return {
        "lattice2": (lat2, dict(area_max=400)),
        # pitch / FWHM 1.4: too dense to threshold; peak seeding (subpx/cd.py:502-511).
        "lattice14": (lat14, dict(area_max=400, seeds="peaks", methods=("gaussian", "halfmax"))),
        "page": (page, dict(area_max=400)),
        "staggered": (stag, dict(area_max=400)),
        "page_invert": ((65535 - page).astype(np.uint16), dict(area_max=400, invert=True,
                                                               methods=("gaussian", "logquad"))),
        "drop_peaks": (drop, dict(seeds="peaks", methods=("gaussian", "gradient"), area_max=400)),
        "add_threshold": (add, dict(methods=("gaussian", "halfmax"), area_min=10, area_max=400)),
        "dark_peaks_fixed": (100 - clean20, dict(invert=True, seeds="peaks", methods=("gaussian", "halfmax"),
                                                  background_level=80.0)),
        "page_smooth": (page, dict(area_max=400, smooth_sigma=1.0, methods=("gaussian", "gradient", "halfmax"))),
    }


def make_cd(out: Path, ref):
    from subpx import measure_cds

    arrays = {}
    names = []
    for name, (img, kw) in cd_cases().items():
        res = measure_cds(img, backend="cpu", **kw)
        arrays[f"{name}_img"] = img
        arrays[f"{name}_kwargs"] = np.array(json.dumps(kw))
        arrays[f"{name}_seeds"] = res.seeds_xy
        arrays[f"{name}_cell_labels"] = res.cell_labels
        arrays[f"{name}_params"] = res.deblend_model["params"]
        arrays[f"{name}_report"] = res.deblend_model["report"]
        arrays[f"{name}_bgmap"] = res.background_map.astype(np.float32)
        arrays[f"{name}_meta"] = np.array([res.meta["deblend_iterations_used"], res.meta["deblend_passes"],
                                           res.meta["seeds_added_from_residual"],
                                           res.meta["seeds_dropped_as_insignificant"]])
        arrays[f"{name}_source"] = np.array(res.meta["background_source"])
        arrays[f"{name}_pitch"] = np.array(np.nan if res.meta.get("pitch_px") is None else res.meta["pitch_px"])
        arrays[f"{name}_passes"] = np.array(res.meta["deblend_pass_iterations"])
        meths = list(res.measurements)
        arrays[f"{name}_methods"] = np.array(meths)
        for m, r in res.measurements.items():
            arrays[f"{name}_{m}_status"] = r.status
            arrays[f"{name}_{m}_centers"] = r.centers_xy
            arrays[f"{name}_{m}_contours"] = r.contours_xy
            for metric, v in r.metrics.items():
                arrays[f"{name}_{m}_m_{metric}"] = v
        names.append(name)
    np.savez_compressed(out / "cd.npz", names=np.array(names), **arrays)


def invariant_cases():
    cases = cd_cases()
    stag, _ = cases["staggered"]
    page, _ = cases["page"]
    lat2, _ = cases["lattice2"]
    return {
        "staggered": (stag, dict(area_max=400, methods=("projection", "gaussian"))),
        "page": (page, dict(area_max=400, methods=("gaussian", "projection"))),
        "lattice2": (lat2, dict(area_max=400, methods=("projection",))),
        "page_invert": ((65535 - page).astype(np.uint16), dict(area_max=400, invert=True, methods=("projection",))),
        # Dense holes (pitch / FWHM 1.4): profiles whose steepest points reach the cell border.
        "lattice14": (cases["lattice14"][0], dict(area_max=400, seeds="peaks", methods=("projection", "halfmax"))),
        # The half_area family: median and minimum local levels, the averaged peak.
        "staggered_half": (stag, dict(area_max=400, methods=("half_area", "half_area_min", "half_area_min_avg",
                                                            "projection"))),
        "page_half": (page, dict(area_max=400, methods=("gaussian", "half_area_min_avg", "half_area"))),
        "lattice14_half": (cases["lattice14"][0], dict(area_max=400, seeds="peaks",
                                                       methods=("half_area", "half_area_min_avg"))),
    }


def make_invariant(out: Path, ref):
    """measure_cds with the projection method (subpx/_cpu/invariant_cd.py:365-421) beside others."""
    from subpx import measure_cds

    arrays = {}
    names = []
    for name, (img, kw) in invariant_cases().items():
        res = measure_cds(img, backend="cpu", **kw)
        arrays[f"{name}_img"] = img
        arrays[f"{name}_kwargs"] = np.array(json.dumps(kw))
        arrays[f"{name}_seeds"] = res.seeds_xy
        arrays[f"{name}_methods"] = np.array(list(res.measurements))
        for m, r in res.measurements.items():
            arrays[f"{name}_{m}_status"] = r.status
            arrays[f"{name}_{m}_centers"] = r.centers_xy
            arrays[f"{name}_{m}_contours"] = r.contours_xy
            if "edge_px" in r.geometry:
                arrays[f"{name}_{m}_edge_px"] = r.geometry["edge_px"]
            for metric, v in r.metrics.items():
                arrays[f"{name}_{m}_m_{metric}"] = v
        names.append(name)
    np.savez_compressed(out / "invariant.npz", names=np.array(names), **arrays)


def make_results(out: Path, ref):
    """Result folders written by the reference's own save_cd_results (full and compact) for a small
    lattice page measured by its CPU path: the file format the loader must read."""
    from subpx import measure_cds
    from subpx.cd import save_cd_results

    from imageprocessor_new_b200 import synthetic as S

    img, _ = S.gaussian_lattice(2.0, shape=(64, 112), seed=6)
    res = measure_cds(img, backend="cpu", methods=("gaussian", "halfmax"), area_max=400)
    for compact in (False, True):
        save_cd_results(res, out / ("results_compact" if compact else "results_full"), compact=compact)


def make_centers_model(out: Path, ref):
    """detect_centers(background="model") of the reference's CPU path: centres re-refined on
    deblended cells, for the refiners that support it."""
    from subpx import detect_centers

    from imageprocessor_new_b200 import synthetic as S

    page = np.ascontiguousarray(S.page_square(4).image[:256, :320])
    lat, _ = S.gaussian_lattice(2.2, shape=(96, 160), seed=8)
    lat = np.clip(np.rint(lat), 0, 255).astype(np.uint8)
    arrays = {"page_img": page, "lattice_img": lat}
    for name, img, kw in (("page", page, dict(threshold="otsu", area_max=400)),
                          ("lattice", lat, dict(threshold="otsu", area_max=400))):
        for refine in ("weighted", "logquad", "none"):
            res = detect_centers(img, backend="cpu", refine=refine, background="model", **kw)
            arrays[f"{name}_{refine}"] = res.centers_xy
            arrays[f"{name}_{refine}_used"] = np.array(res.meta["deblend_iterations_used"])
    np.savez_compressed(out / "centers_model.npz", **arrays)


TAIL = ("tail_area", "tail_area_norm", "edge_area", "foot_area", "foot_area_ratio")


def tail_cases():
    cases = cd_cases()
    stag, _ = cases["staggered"]
    page, _ = cases["page"]
    lat2, _ = cases["lattice2"]
    return {
        # Windows of 1.2 pitches holding each hole's share of the light; the five threshold rules.
        "staggered_tail": (stag, dict(area_max=400, methods=TAIL)),
        "lattice2_tail": (lat2, dict(area_max=400, methods=TAIL + ("half_area_min_avg",))),
        # Options: a lower level on narrower windows, no display outlines.
        "page_tail": (page, dict(area_max=400, methods=("tail_area", "foot_area_ratio", "edge_area"),
                                 tail_area_level=0.3, tail_window=0.8, outlines=False)),
        # Dense holes seeded by peaks: windows reaching past several neighbours.
        "lattice14_tail": (cases["lattice14"][0], dict(area_max=400, seeds="peaks",
                                                       methods=("tail_area", "tail_area_norm", "foot_area"))),
    }


def make_tail(out: Path, ref):
    """measure_cds with the tail family (subpx/_cpu/invariant_cd.py:878-1068)."""
    from subpx import measure_cds

    arrays = {}
    names = []
    for name, (img, kw) in tail_cases().items():
        res = measure_cds(img, backend="cpu", **kw)
        arrays[f"{name}_img"] = img
        arrays[f"{name}_kwargs"] = np.array(json.dumps(kw))
        arrays[f"{name}_seeds"] = res.seeds_xy
        arrays[f"{name}_meta"] = np.array(json.dumps({k: res.meta.get(k) for k in ("tail_window_px", "foot_ratio")}))
        for m, r in res.measurements.items():
            arrays[f"{name}_{m}_status"] = r.status
            arrays[f"{name}_{m}_centers"] = r.centers_xy
            arrays[f"{name}_{m}_center_local"] = r.geometry["center_local"]
            # Outline radii are k / 8 + 1 / 16 px: exact in float32. Contours are centre + radius x
            # (cos, sin) + origin and are not stored.
            arrays[f"{name}_{m}_edge_px"] = r.geometry["edge_px"].astype(np.float32)
            for metric, v in r.metrics.items():
                arrays[f"{name}_{m}_m_{metric}"] = v
        names.append(name)
    np.savez_compressed(out / "tail.npz", names=np.array(names), **arrays)


def disk_cases():
    from imageprocessor_new_b200 import synthetic as S

    small, _ = S.gaussian_lattice(2.0, shape=(60, 120))
    stag, _ = cd_cases()["staggered"]
    return {
        # Blur given: the disk table of that Airy FWHM, two rounds of fits.
        "lattice_psf": (small, dict(area_max=400, methods=("disk", "flux_ratio"), psf_fwhm=2.0)),
        # Blur calibrated by bisection so that the median disk diameter equals nominal_cd; flux ratios
        # scaled to it.
        "lattice_nominal": (small, dict(area_max=400, methods=("disk", "flux_ratio"), nominal_cd=3.0)),
        # Wide holes of a staggered page; dark level and a given flux-ratio scale.
        "staggered_disk": (stag, dict(area_max=400, methods=("flux_ratio", "disk"), psf_fwhm=3.0, dark_level=100.0,
                                      flux_ratio_scale=1.5)),
    }


def make_disk(out: Path, ref):
    """measure_cds with the disk and flux_ratio methods (subpx/_cpu/invariant_cd.py:94-306, 1069-1206)."""
    from subpx import measure_cds

    arrays = {}
    names = []
    for name, (img, kw) in disk_cases().items():
        res = measure_cds(img, backend="cpu", **kw)
        arrays[f"{name}_img"] = img
        arrays[f"{name}_kwargs"] = np.array(json.dumps(kw))
        arrays[f"{name}_seeds"] = res.seeds_xy
        arrays[f"{name}_meta"] = np.array(json.dumps({k: res.meta.get(k) for k in (
            "psf_fwhm_px", "psf_source", "disk_median_cd_px", "flux_ratio_scale")}))
        for m, r in res.measurements.items():
            arrays[f"{name}_{m}_status"] = r.status
            arrays[f"{name}_{m}_centers"] = r.centers_xy
            arrays[f"{name}_{m}_edge_px"] = r.geometry["edge_px"]
            for metric, v in r.metrics.items():
                arrays[f"{name}_{m}_m_{metric}"] = v
        names.append(name)
    np.savez_compressed(out / "disk.npz", names=np.array(names), **arrays)


MAKERS = {"thresholds": make_thresholds, "ccl": make_ccl, "centers": make_centers, "voronoi": make_voronoi,
          "tiled": make_tiled, "cd": make_cd, "results": make_results, "centers_model": make_centers_model,
          "invariant": make_invariant, "tail": make_tail, "disk": make_disk}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    ref = _ref(args.reference)
    for name, fn in MAKERS.items():
        if args.only and name != args.only:
            continue
        if fn in (make_thresholds, make_ccl):
            fn(HERE)
        else:
            fn(HERE, ref)
        print("wrote", name)


if __name__ == "__main__":
    main()
