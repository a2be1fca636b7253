"""Kernel-level reference bar: the reference's own CUDA kernels beside this library's, on one B200 —
MEASUREMENT INFRASTRUCTURE (like the rest of oracle/), never the product.

The reference's GPU path (subpx/_gpu, run through CuPy, which this image lacks) keeps its kernels
as CUDA source strings that CuPy compiles at run time. ``build`` reads those strings out of the
reference checkout's module text (parsed with ``ast``; nothing of the reference is imported), writes
them to ``oracle/_ref/*.cu`` and compiles each for sm_100a with nvcc and the reference's own options
(subpx/_gpu/_cuda.py:18-29: ``--std=c++14``; ``--fmad=false`` for the kernels it marks exact; the
defines its launcher picks). The sources and cubins stay in ``oracle/_ref/`` (git-ignored).

``bench`` (needs the GPU) loads the cubins through the CUDA driver API (cuda-python), builds the
inputs of one deblending iteration, one render, the radial profiles and the Voronoi labels of a
synthetic page of the benchmark's kind with this library, launches the reference kernels with the
reference's launch shapes on exactly those inputs and this library's kernels beside them, times
both with CUDA events on the same stream (after a warm-up launch, the median of a few repeats),
checks that they agree, and prints one JSON line. Where the reference does part of a stage outside
its kernels (CuPy array operations: the spline prefilter and centroids of the radial profiles, the
relaxation and statuses after the LM, the conversion of the fixed-point render), only its kernels
are timed, which favours the reference.

  python -m oracle.ref_kernels build [--reference PATH]
  python -m oracle.ref_kernels bench [--page 4096] [--repeats 5]
"""

from __future__ import annotations

import argparse
import ast
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
ROOT = HERE.parent

# name -> (module file in the reference, source variable, kernel name, exact, defines)
KERNELS = {
    "lm_fit_shared": ("subpx/_gpu/deblend.py", "_LM_SRC", "lm_fit", False, ("CELL_IN_SHARED",)),
    "lm_fit_cached": ("subpx/_gpu/deblend.py", "_LM_SRC", "lm_fit", False, ("CELL_IN_SHARED", "CACHE_SHAPES")),
    "lm_fit_global": ("subpx/_gpu/deblend.py", "_LM_SRC", "lm_fit", False, ()),
    "clean_cells": ("subpx/_gpu/deblend.py", "_CLEAN_SRC", "clean_cells", False, ()),
    "render_fixed": ("subpx/_gpu/deblend.py", "_RENDER_SRC", "render_fixed", False, ()),
    "radial_edges": ("subpx/_gpu/cd.py", "_RAY_SRC", "radial_edges", True, ()),
    "voronoi_ring": ("subpx/_gpu/voronoi.py", "_KERNEL_SRC", "voronoi_ring", True, ()),
}


def _source_strings(path: Path) -> dict[str, str]:
    """Module-level string constants (plain assignments of a string literal) of a Python file."""
    tree = ast.parse(path.read_text())
    out = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and isinstance(node.value, ast.Constant) and isinstance(node.value.value, str):
            for target in node.targets:
                if isinstance(target, ast.Name):
                    out[target.id] = node.value.value
    return out


def build(reference: str | Path = "/root/reference", nvcc: str = "/usr/local/cuda/bin/nvcc") -> list[Path]:
    """Extracts and compiles the reference kernels into oracle/_ref/ (one cubin per variant)."""
    reference = Path(reference)
    OUT.mkdir(exist_ok=True)
    built = []
    for name, (module, var, _, exact, defines) in KERNELS.items():
        src = _source_strings(reference / module)[var]
        cu = OUT / f"{name}.cu"
        cu.write_text(src)
        cubin = OUT / f"{name}.cubin"
        cmd = [nvcc, "-cubin", "-gencode", "arch=compute_100a,code=sm_100a", "--std=c++14", "-o", str(cubin),
               str(cu)] + (["--fmad=false"] if exact else []) + [f"-D{d}" for d in defines]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"nvcc failed on {name}:\n{proc.stderr}")
        built.append(cubin)
    return built


# ----------------------------------------------------------------------------------- GPU side

class _Module:
    """One reference cubin loaded with the driver API; launch() takes torch tensors and numpy scalars."""

    def __init__(self, name: str):
        from cuda.bindings import driver as cu

        self.cu = cu
        _check(cu.cuInit(0))
        data = (OUT / f"{name}.cubin").read_bytes()
        self.mod = _check(cu.cuModuleLoadData(data))
        self.fn = _check(cu.cuModuleGetFunction(self.mod, KERNELS[name][2].encode()))

    def launch(self, grid: int, block: int, args, shared: int = 0):
        import torch

        cu = self.cu
        if shared > 48 * 1024:
            _check(cu.cuFuncSetAttribute(self.fn, cu.CUfunction_attribute.CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES,
                                         int(shared)))
        holders = []
        for a in args:
            if isinstance(a, torch.Tensor):
                holders.append(np.array([a.data_ptr()], dtype=np.uint64))
            else:
                holders.append(np.array([a], dtype=np.asarray(a).dtype))
        ptrs = np.array([h.ctypes.data for h in holders], dtype=np.uint64)
        stream = cu.CUstream(torch.cuda.current_stream().cuda_stream)
        _check(cu.cuLaunchKernel(self.fn, int(grid), 1, 1, int(block), 1, 1, int(shared), stream, ptrs.ctypes.data, 0))


def _check(res):
    err, *rest = res if isinstance(res, tuple) else (res,)
    if int(err) != 0:
        raise RuntimeError(f"CUDA driver call failed: {err}")
    return rest[0] if len(rest) == 1 else (rest or None)


def _time(fn, repeats: int) -> float:
    """Median CUDA-event time (ms) of fn() on the current stream, after one untimed call."""
    import torch

    fn()
    times = []
    for _ in range(repeats):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        torch.cuda.synchronize()
        times.append(s.elapsed_time(e))
    return float(np.median(times))


def bench(page_size: int = 4096, repeats: int = 5, radial_cells: int = 20000) -> dict:
    import torch
    from scipy.ndimage import binary_erosion, spline_filter1d

    sys.path.insert(0, str(ROOT))
    from imageprocessor_new_b200 import _device as dev
    from imageprocessor_new_b200 import _lib, synthetic, warmstart
    from imageprocessor_new_b200.cd import _mask_stack, _method_buffers
    from imageprocessor_new_b200.deblend import Deblender, sigma_major
    from imageprocessor_new_b200.voronoi import labels_device

    torch.cuda.set_device(0)
    page = synthetic.page_staggered(0, shape=(page_size, page_size)).image
    page_d = dev.upload(page)
    h, w = page.shape
    cells = warmstart.page_cells(page_d, area_min=3, area_max=400, pad=3)
    n, hm, wm = cells.n, cells.hm, cells.wm
    out = {"page": f"{page_size}x{page_size} staggered uint16 (pitch 24, d 12)", "cells": int(n),
           "cell_box": [int(hm), int(wm)], "repeats": repeats}

    # Voronoi labels (subpx/_gpu/voronoi.py:86-116): host binning as the reference does it.
    seeds = np.ascontiguousarray(cells.seeds, dtype=np.float64)
    cell = max(1, int(np.sqrt(h * w / n)))
    gw, gh = -(-w // cell), -(-h // cell)
    bx = np.clip(np.floor(seeds[:, 0]).astype(np.int64) // cell, 0, gw - 1)
    by = np.clip(np.floor(seeds[:, 1]).astype(np.int64) // cell, 0, gh - 1)
    bins = by * gw + bx
    order = np.argsort(bins, kind="stable").astype(np.int32)
    start = np.zeros(gw * gh + 1, dtype=np.int32)
    np.cumsum(np.bincount(bins, minlength=gw * gh), out=start[1:])
    seeds_d, order_d, start_d = dev.upload(seeds), dev.upload(order), dev.upload(start)
    ref_labels = dev.empty((h, w), torch.int32)
    vor = _Module("voronoi_ring")
    ref_ms = _time(lambda: vor.launch(-(-(h * w) // 256), 256, (seeds_d, order_d, start_d, ref_labels, np.int64(h * w),
                                                              np.int32(w), np.int32(gw), np.int32(gh),
                                                              np.int32(cell))), repeats)
    ours = {}
    our_ms = _time(lambda: ours.__setitem__("labels", labels_device(seeds_d, (h, w))), repeats)
    out["voronoi"] = {"reference_kernel": "voronoi_ring", "ours": "k_voronoi", "ref_ms": ref_ms, "ours_ms": our_ms,
                      "speedup": ref_ms / our_ms,
                      "labels_equal": bool(torch.equal(ref_labels, ours["labels"]))}

    # One deblending iteration: the reference's clean_cells + lm_fit (subpx/_gpu/deblend.py:519-536,
    # 243-286) against k_fit_iteration, from the same params, model and background map.
    dbl = Deblender(page_d, 1.0, cells)
    params_d, status_d, _ = dbl.initial(30)
    stats = dbl.stats(params_d, status_d)
    model = dbl.render(params_d)
    bg, _ = dbl.background_of(model, stats)
    res = {}
    our_ms = _time(lambda: res.__setitem__("it", dbl.iteration(params_d, model, bg)), repeats)
    ours_params = res["it"][0].cpu().numpy()
    p = params_d.cpu().numpy()
    origins = np.asarray(cells.origins, dtype=np.int64)
    pg = p.copy()
    pg[:, 1:3] += origins
    radius = np.clip(np.ceil(4.0 * sigma_major(pg)), 2, dbl.radius_cap).astype(np.int32)
    image_d = page_d.to(torch.float64)
    bg_d = dev.upload(bg.host_map())
    masks = _mask_stack(cells, np.arange(n)).astype(np.uint8)
    masks_d = dev.upload(masks)
    pg_d, radius_d, origins_d = dev.upload(pg), dev.upload(radius), dev.upload(origins)
    cleaned_d = dev.empty((n, hm, wm), torch.float64)
    clean = _Module("clean_cells")
    total = n * hm * wm

    def ref_clean():
        clean.launch(-(-total // 256), 256, (image_d, bg_d, model, pg_d, radius_d, masks_d, origins_d, cleaned_d,
                                             np.int64(total), np.int32(hm), np.int32(wm), np.int32(h), np.int32(w)))

    cached = hm * wm <= 256
    shared = 4 * hm * wm * (25 if cached else 9)
    variant = "lm_fit_cached" if cached else ("lm_fit_shared" if shared <= 96 * 1024 else "lm_fit_global")
    if variant == "lm_fit_global":
        shared = 0
    lm = _Module(variant)
    fit_d = dev.empty((n, 6), torch.float64)

    def ref_fit():
        fit_d.copy_(params_d)
        lm.launch(-(-n // 4), 128, (cleaned_d, masks_d, fit_d, np.int32(n), np.int32(hm), np.int32(wm), np.int32(30),
                                    np.float64(0.5)), shared)

    clean_ms = _time(ref_clean, repeats)
    fit_ms = _time(ref_fit, repeats)
    fitted = fit_d.cpu().numpy()
    step = np.where(np.isfinite(fitted), fitted - p, 0.0)
    relaxed = p + 0.6 * step
    fin = np.isfinite(relaxed).all(axis=1) & np.isfinite(ours_params).all(axis=1)
    out["lm_iteration"] = {"reference_kernels": ["clean_cells", variant], "ours": "k_fit_iteration",
                           "ref_ms": clean_ms + fit_ms, "ref_clean_ms": clean_ms, "ref_lm_ms": fit_ms,
                           "ours_ms": our_ms, "speedup": (clean_ms + fit_ms) / our_ms,
                           "max_param_diff": float(np.abs(relaxed[fin] - ours_params[fin]).max())}

    # Render (subpx/_gpu/deblend.py:289-307): render_fixed + its conversion against k_render.
    top = float(np.max(np.abs(pg[:, 0]))) * n
    scale = 2.0 ** int(np.clip(62 - np.ceil(np.log2(top)), -1000, 1000)) if top > 0 else 1.0
    acc = torch.zeros(h * w, dtype=torch.int64, device="cuda")
    rend = _Module("render_fixed")

    def ref_render():
        acc.zero_()
        rend.launch(n, 128, (pg_d, radius_d, acc, np.int32(n), np.int32(h), np.int32(w), np.float64(scale)))
        return acc.to(torch.float64) / scale

    ref_ms = _time(ref_render, repeats)
    got = {}
    our_ms = _time(lambda: got.__setitem__("m", dbl.render(params_d)), repeats)
    diff = float((ref_render().reshape(h, w) - got["m"]).abs().max())
    out["render"] = {"reference_kernel": "render_fixed (+ fixed-point conversion)", "ours": "k_render",
                     "ref_ms": ref_ms, "ours_ms": our_ms, "speedup": ref_ms / our_ms, "max_abs_diff": diff,
                     "max_amplitude": float(np.abs(pg[:, 0]).max())}

    # Radial profiles (subpx/_gpu/cd.py:258-303): the reference kernel on its prefiltered spline
    # coefficients (computed here with SciPy on the host, untimed) against k_radial_cd (prefilter
    # included) on the same cleaned cells.
    m = min(n, radial_cells)
    rois = cleaned_d[:m].cpu().numpy()
    mk = masks[:m].astype(bool)
    signal = np.where(mk, rois, 0.0)
    topv = signal.reshape(m, -1).max(axis=1)[:, None, None]
    wgt = np.where(mk & (signal > 0.1 * topv), signal, 0.0)
    yy, xx = np.indices((hm, wm), dtype=np.float64)
    center = np.stack(((wgt * xx).sum(axis=(1, 2)), (wgt * yy).sum(axis=(1, 2))), axis=1) / wgt.sum(axis=(1, 2))[:, None]
    coef = np.pad(signal, ((0, 0), (12, 12), (12, 12)), mode="edge")
    coef = spline_filter1d(coef, 3, axis=1, output=np.float64, mode="nearest")
    coef = np.ascontiguousarray(spline_filter1d(coef, 3, axis=2, output=np.float64, mode="nearest"))
    safe = binary_erosion(mk, structure=np.array([[[0, 1, 0], [1, 1, 1], [0, 1, 0]]], bool),
                          border_value=0).astype(np.uint8)
    n_angles, radial_step = 128, 0.1
    radii = np.arange(0, np.hypot(hm, wm) + radial_step, radial_step)
    angles = np.arange(n_angles) * (2 * np.pi / n_angles)
    dirs = np.ascontiguousarray(np.column_stack((np.cos(angles), np.sin(angles))))
    coef_d, safe_d, center_d = dev.upload(coef), dev.upload(safe), dev.upload(np.ascontiguousarray(center))
    radii_d, dirs_d = dev.upload(radii), dev.upload(dirs)
    peak_d, half_d, grad_d = dev.empty((m,), torch.float64), dev.empty((m, n_angles), torch.float64), \
        dev.empty((m, n_angles), torch.float64)
    ray = _Module("radial_edges")
    ref_ms = _time(lambda: ray.launch(-(-(m * n_angles) // 128), 128, (
        coef_d, safe_d, center_d, radii_d, np.int32(len(radii)), dirs_d, np.int32(n_angles), peak_d, half_d, grad_d,
        np.int32(m), np.int32(hm), np.int32(wm), np.float64(max(0.35, 2 * radial_step)))), repeats)
    which_d = dev.upload(np.arange(m, dtype=np.int32))
    hb, hs = _method_buffers(m, n_angles, "halfmax", False)
    gb, gs = _method_buffers(m, n_angles, "gradient", False)
    ws = dev.workspace(_lib.size("spx_radial_workspace_bytes", hm, wm, 0))
    our_ms = _time(lambda: _lib.call("spx_radial_cd", cleaned_d.data_ptr(), cells.voronoi.data_ptr(),
                                     cells.boxes.data_ptr(), which_d.data_ptr(), m, hm, wm, w, n_angles, radial_step,
                                     None, 0, hs, gs, ws.data_ptr(), ws.numel(), dev.stream_ptr()), repeats)
    a, b = half_d.cpu().numpy(), hb["edge_px"].cpu().numpy()
    both = np.isfinite(a) & np.isfinite(b)
    ga, gb_ = grad_d.cpu().numpy(), gb["edge_px"].cpu().numpy()
    gboth = np.isfinite(ga) & np.isfinite(gb_)
    out["radial"] = {"reference_kernel": "radial_edges (prefilter and centroids outside, untimed)",
                     "ours": "k_radial_cd (prefilter and centroids included)", "cells": int(m), "ref_ms": ref_ms,
                     "ours_ms": our_ms, "speedup": ref_ms / our_ms,
                     "halfmax_same_found": float((np.isfinite(a) == np.isfinite(b)).mean()),
                     "halfmax_edge_max_diff_px": float(np.abs(a[both] - b[both]).max(initial=0.0)),
                     "gradient_same_found": float((np.isfinite(ga) == np.isfinite(gb_)).mean()),
                     "gradient_edge_p99_diff_px": float(np.percentile(np.abs(ga[gboth] - gb_[gboth]), 99))
                     if gboth.any() else 0.0}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m oracle.ref_kernels")
    sub = ap.add_subparsers(dest="cmd", required=True)
    b = sub.add_parser("build")
    b.add_argument("--reference", default="/root/reference")
    r = sub.add_parser("bench")
    r.add_argument("--page", type=int, default=4096)
    r.add_argument("--repeats", type=int, default=5)
    args = ap.parse_args(argv)
    if args.cmd == "build":
        for p in build(args.reference):
            print(p)
    else:
        print(json.dumps(bench(args.page, args.repeats)), flush=True)


if __name__ == "__main__":
    main()
