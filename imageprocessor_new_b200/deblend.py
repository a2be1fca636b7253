"""Deblending driver: background map + one Gaussian per hole, every per-pixel / per-cell step on the
device (libsubpx_b200), the outer iteration and the tile interpolation on the host.

Follows subpx/_cpu/deblend.py:421-522 (deblend) and the reference GPU driver subpx/_gpu/deblend.py:
453-585: all cells update at once against the previous iteration's neighbours, relaxation 0.6,
status of the relaxed parameters, stop when the 99th percentile of the centre / log-width steps of
the "ok" cells is below the tolerance. Background tiles: median residual over pixels far from every
hole where the model is faint; unmeasured tiles are interpolated linearly over a Delaunay
triangulation of the measured tile centres (nearest measured tile outside it), as
subpx/_cpu/deblend.py:346-393 does — on the host, with SciPy, as the reference's GPU path does.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _device as dev
from . import _lib
from .voronoi import labels_device

FWHM_K = float(np.sqrt(2 * np.log(2)))
STATUS = np.array(_lib.STATUS_NAMES, dtype="U32")
OK = 0


def _ptr(t):
    return None if t is None else t.data_ptr()


@dataclass
class Cells:
    """Voronoi cells of the seeds: cell j = box j intersected with Voronoi label j (device arrays)."""

    rows: np.ndarray          # (N, 6) [x, y, w, h, cx, cy]
    seeds: np.ndarray         # (N, 2) host
    seeds_d: torch.Tensor     # (N, 2) f64
    voronoi: torch.Tensor     # (H, W) int32
    boxes: torch.Tensor       # (N, 4) int32 x0, y0, w, h
    counts: torch.Tensor      # (N,) int32 mask pixels
    caps: torch.Tensor        # (N,) f64 sigma caps
    origins: np.ndarray       # (N, 2) int32 host
    sizes: np.ndarray         # (N, 2) int32 host (w, h)
    hm: int
    wm: int
    max_px: int

    @property
    def n(self) -> int:
        return len(self.rows)


def build_cells(rows, shape, pad: int, rows_d: torch.Tensor | None = None) -> Cells:
    """Voronoi labels of the row centres and the padded boxes (subpx/_gpu/cells.py:11-38).

    With ``rows_d`` (the rows already on the device) ``rows`` may be a host array whose copy from
    the device is still in flight on the current stream: it is read only after the stream syncs."""
    h, w = shape
    if rows_d is None:
        rows = np.asarray(rows, dtype=np.float64).reshape(-1, 6)
        n = len(rows)
        rows_d = dev.upload(rows) if n else None
    else:
        n = rows_d.shape[0]
    seeds_d = rows_d[:, 4:6].contiguous() if n else dev.empty((0, 2), torch.float64)
    vor = labels_device(seeds_d if n else None, shape)
    boxes = dev.empty((max(n, 1), 4), torch.int32)
    counts = dev.empty((max(n, 1),), torch.int32)
    caps = dev.empty((max(n, 1),), torch.float64)
    _lib.call("spx_cells_setup", _ptr(rows_d) if n else None, n, int(pad), h, w, vor.data_ptr(), boxes.data_ptr(),
              counts.data_ptr(), caps.data_ptr(), dev.stream_ptr())
    host = dev.start_download(boxes[:n])
    host_counts = dev.start_download(counts[:n])
    torch.cuda.current_stream().synchronize()
    rows = np.asarray(rows, dtype=np.float64).reshape(-1, 6)
    hm = int(host[:, 3].max()) if n else 0
    wm = int(host[:, 2].max()) if n else 0
    max_px = int(host_counts.max()) if n else 1
    # Seeds, origins and sizes are views of the downloaded arrays (new host arrays of this size
    # cost more in first-touch page faults than the copies themselves).
    return Cells(rows, rows[:, 4:6], seeds_d, vor, boxes[:n], counts[:n], caps[:n], host[:, :2], host[:, 2:4], hm,
                 wm, max(max_px, 1))


def auto_tile(seeds_d: torch.Tensor, n: int, shape) -> tuple[int, float]:
    """Tile of about four pitches; pitch = median nearest-seed distance (subpx/_cpu/deblend.py:396-403)."""
    if n < 2:
        return int(max(shape)), float("nan")
    h, w = shape
    out = dev.empty((n,), torch.float64)
    ws = dev.workspace(_lib.size("spx_voronoi_workspace_bytes", n, h, w))
    _lib.call("spx_nearest_distances", seeds_d.data_ptr(), n, seeds_d.data_ptr(), n, 1, h, w, out.data_ptr(),
              ws.data_ptr(), ws.numel(), dev.stream_ptr())
    res = quantiles([_lib.QuantileReq(out.data_ptr(), 1, None, 0, n, 0, 0.0)])
    pitch = float(res[0, 0])
    return int(np.clip(round(4 * pitch), 16, max(shape))), pitch


def quantile_device(*reqs) -> torch.Tensor:
    """Run spx_quantiles on _lib.QuantileReq requests; a (len, 2) device array of (value, count),
    left on the device (nothing synchronises)."""
    arr = (_lib.QuantileReq * len(reqs))(*reqs)
    raw = dev.upload(np.frombuffer(bytes(arr), dtype=np.uint8))
    out = dev.empty((len(reqs), 2), torch.float64)
    _lib.call("spx_quantiles", raw.data_ptr(), len(reqs), out.data_ptr(), dev.stream_ptr())
    return out


def quantiles(reqs) -> np.ndarray:
    """Run spx_quantiles on a list of _lib.QuantileReq; (len, 2) array of (value, count)."""
    return quantile_device(*reqs).cpu().numpy()


def sigma_major(params: np.ndarray) -> np.ndarray:
    """Closed form of the precision's smaller eigenvalue (det / larger), as 1 / sqrt."""
    e1, u2, e3 = np.exp(params[:, 3]), params[:, 4], np.exp(params[:, 5])
    a, b, c = e1 * e1, e1 * u2, u2 * u2 + e3 * e3
    half = (a - c) / 2
    larger = (a + c) / 2 + np.sqrt(half * half + b * b)
    with np.errstate(divide="ignore", invalid="ignore"):
        smaller = np.where(larger > 0, (e1 * e3) ** 2 / larger, 0.0)
    return 1 / np.sqrt(np.maximum(smaller, 1e-300))


FIT_PRECISIONS = ("fp64", "fp32")
# Relative cost drop that ends an FP32 fit. FP32 residuals resolve cost changes down to a few 1e-7
# of the cost (a tighter rule only adds rejected trials); 1e-7 keeps the fitted sigmas within about
# 1e-3 px of the FP64 fit on holes up to 20 px.
FP32_COST_TOL = 1e-7


def fit_options(precision: str = "fp64", cost_tol: float | None = None) -> _lib.FitOptions:
    """spx_fit_options for an LM arithmetic: "fp64" (the reference's, stop rule 1e-12) or "fp32"
    (FP32 per-pixel arithmetic and lane sums, FP64 totals, solve and acceptance)."""
    if precision not in FIT_PRECISIONS:
        raise ValueError(f"fit_precision must be one of {FIT_PRECISIONS}, got {precision!r}")
    if cost_tol is None:
        cost_tol = 1e-12 if precision == "fp64" else FP32_COST_TOL
    return _lib.FitOptions(_lib.FIT_F32 if precision == "fp32" else _lib.FIT_F64, float(cost_tol))


def tile_centers(tile: int, shape):
    h, w = shape
    yc = np.array([(j * tile + min((j + 1) * tile, h) - 1) / 2 for j in range(-(-h // tile))])
    xc = np.array([(i * tile + min((i + 1) * tile, w) - 1) / 2 for i in range(-(-w // tile))])
    return yc, xc


_INTERPOLATORS: dict = {}


def interpolate_tiles(free_med, measured, tile, shape):
    """Unmeasured tiles from the measured ones: linear over their Delaunay triangulation, the
    nearest measured tile outside it (subpx/_cpu/deblend.py:359-385)."""
    from scipy.spatial import Delaunay, cKDTree

    key = (tuple(shape), tile, measured.shape, measured.tobytes())
    if key not in _INTERPOLATORS:
        yc, xc = tile_centers(tile, shape)
        grid = np.stack(np.meshgrid(yc, xc, indexing="ij"), axis=-1)
        known, query = grid[measured], grid[~measured]
        try:
            tri = Delaunay(known) if len(known) >= 3 else None
        except Exception:  # collinear measured tiles
            tri = None
        # LinearNDInterpolator's barycentric weights of the unmeasured tile centres, kept for the
        # next calls with the same measured tiles (only the values change between deblending
        # iterations); evaluated below with its arithmetic, so the results are the same bits.
        bary = None
        if tri is not None:
            simplex = tri.find_simplex(query)
            inside = simplex >= 0
            t = tri.transform[simplex[inside]]
            d = query[inside] - t[:, 2]
            c0 = t[:, 0, 0] * d[:, 0] + t[:, 0, 1] * d[:, 1]
            c1 = t[:, 1, 0] * d[:, 0] + t[:, 1, 1] * d[:, 1]
            bary = (inside, tri.simplices[simplex[inside]], c0, c1, 1.0 - c0 - c1)
        if len(_INTERPOLATORS) >= 32:
            _INTERPOLATORS.clear()
        _INTERPOLATORS[key] = (bary, cKDTree(known), query)
    bary, tree, query = _INTERPOLATORS[key]
    values = free_med[measured]
    medians = free_med.copy()
    missing = ~measured
    interp = np.full(len(query), np.nan)
    if bary is not None:
        inside, vert, c0, c1, c2 = bary
        interp[inside] = values[vert[:, 0]] * c0 + values[vert[:, 1]] * c1 + values[vert[:, 2]] * c2
    still = np.isnan(interp)
    if still.any():
        interp[still] = values[tree.query(query[still])[1]]
    medians[missing] = interp
    return medians


class Background:
    """Device background map (tile rows + per-row interpolation) with its host metadata."""

    def __init__(self, shape, tile: int):
        self.shape = tuple(shape)
        self.tile = int(tile)
        h, w = self.shape
        self.ny, self.nx = -(-h // self.tile), -(-w // self.tile)
        yc, _ = tile_centers(self.tile, self.shape)
        if self.ny > 1:
            y = np.arange(h, dtype=float)
            j1 = np.clip(np.searchsorted(yc, y), 1, self.ny - 1)
            t = np.clip((y - yc[j1 - 1]) / (yc[j1] - yc[j1 - 1]), 0, 1)
            self.j1 = dev.upload(j1.astype(np.int32))
            self.t = dev.upload(t.astype(np.float64))
        else:
            self.j1 = self.t = None
        self.rows = None
        self.medians = None
        self.fixed = None

    def set_fixed(self, level: float):
        self.fixed = float(level)
        self.medians = None
        return self

    def set_medians(self, medians: np.ndarray):
        self.fixed = None
        self.medians = np.asarray(medians, dtype=np.float64).reshape(self.ny, self.nx)
        md = dev.upload(self.medians)
        if self.rows is None:
            self.rows = dev.empty((self.ny, self.shape[1]), torch.float64)
        _lib.call("spx_background_rows", md.data_ptr(), self.ny, self.nx, self.tile, self.shape[1],
                  self.rows.data_ptr(), dev.stream_ptr())
        return self

    def struct(self) -> _lib.BgMap:
        if self.fixed is not None:
            return _lib.BgMap(None, None, None, 1, self.shape[1], self.fixed, _lib.BG_FIXED)
        return _lib.BgMap(self.rows.data_ptr(), _ptr(self.j1), _ptr(self.t), self.ny, self.shape[1], 0.0,
                          _lib.BG_MAP)

    def host_map(self) -> np.ndarray:
        """The (H, W) map (subpx _upsample_tiles), built on the device and copied back."""
        h, w = self.shape
        if self.fixed is not None:
            return np.full(self.shape, self.fixed)
        img = torch.zeros((h, w), dtype=torch.uint8, device="cuda")  # residual of a zero image = -bg
        model = torch.zeros((h, w), dtype=torch.float64, device="cuda")
        out = dev.empty((h, w), torch.float64)
        bg = self.struct()
        _lib.call("spx_residual", img.data_ptr(), 0, 1.0, h, w, bg, model.data_ptr(), out.data_ptr(),
                  dev.stream_ptr())
        return -out.cpu().numpy()

    def at_points(self, xy_d: torch.Tensor, sign: float = 1.0) -> np.ndarray:
        """sign * map_coordinates(map, [y, x], order=1, mode="nearest") at device points (N, 2) [x, y]."""
        n = int(xy_d.shape[0])
        if n == 0:
            return np.zeros(0)
        out = dev.empty((n,), torch.float64)
        _lib.call("spx_background_at", self.struct(), self.shape[0], self.shape[1],
                  xy_d.contiguous().data_ptr(), n, float(sign), out.data_ptr(), dev.stream_ptr())
        return out.cpu().numpy()


@dataclass
class DeblendState:
    """Deblending of one image (subpx/_cpu/deblend.py:29-45), device-resident where large."""

    background: Background
    model: torch.Tensor          # (H, W) f64
    params: np.ndarray           # (N, 6) ROI-local
    params_d: torch.Tensor
    status_codes: np.ndarray     # (N,) uint8
    status_d: torch.Tensor
    tile_px: int
    iterations: int
    background_info: dict
    converged: bool = False
    fit_iterations: list = field(default_factory=list)  # LM iterations per pass (device, int32)
    amplitude_median: float = float("nan")  # median A of the "ok" cells with A > 0 (NaN if none)

    @property
    def status(self) -> np.ndarray:
        return STATUS[self.status_codes]


class Deblender:
    """One image's deblending context: the signal, the cells and their device workspaces."""

    def __init__(self, image_d: torch.Tensor, sign: float, cells: Cells, *, exclude_d=None, tile=None,
                 background_level=None, free_fraction=0.05, free_distance_fwhm=1.25, relaxation=0.6,
                 tolerance=1e-3, max_iter=30, fit_precision="fp64", fit_cost_tol=None):
        self.img = image_d
        self.fit_precision = fit_precision
        self.fit_options = fit_options(fit_precision, fit_cost_tol)
        self.dtype = dev.dtype_code(image_d)
        self.sign = float(sign)
        self.shape = tuple(image_d.shape)
        self.cells = cells
        self.n = cells.n
        self.exclude_d = exclude_d
        self.usable_d = None if exclude_d is None else (exclude_d == 0).to(torch.uint8)
        self.background_level = background_level
        self.free_fraction = free_fraction
        self.free_distance_fwhm = free_distance_fwhm
        self.relaxation = relaxation
        self.tolerance = tolerance
        self.max_iter = int(max_iter)
        h, w = self.shape
        if tile is None:
            tile = auto_tile(cells.seeds_d, self.n, self.shape)[0]
        self.tile = int(tile)
        self.radius_cap = int(max(cells.hm, cells.wm)) if self.n else 2
        self.fit_ws = dev.workspace(_lib.size("spx_fit_workspace_bytes", cells.max_px))
        self.render_ws = dev.workspace(_lib.size("spx_render_workspace_bytes", self.n, h, w))
        if self.n:
            _lib.call("spx_render_overflow", self.render_ws.data_ptr(), self.n, h, w, ctypes.byref(ctypes.c_int(0)), 1,
                      dev.stream_ptr())
        if self.n:
            self.dist2 = dev.empty((h, w), torch.int32)
            ws = dev.workspace(_lib.size("spx_voronoi_workspace_bytes", self.n, h, w))
            _lib.call("spx_seed_distance_map", cells.seeds_d.data_ptr(), self.n, h, w, self.dist2.data_ptr(),
                      ws.data_ptr(), ws.numel(), dev.stream_ptr())
        else:
            # No seeds: every pixel is "far" (the reference's distance map is +inf; the FWHM threshold
            # is then 0, which any distance meets).
            self.dist2 = torch.zeros((h, w), dtype=torch.int32, device="cuda")
        self.bg = Background(self.shape, self.tile)

    # ---------------------------------------------------------------------------- pieces
    def render(self, params_d: torch.Tensor) -> torch.Tensor:
        h, w = self.shape
        model = dev.empty((h, w), torch.float64)
        _lib.call("spx_render_model", _ptr(params_d) if self.n else None, self.cells.boxes.data_ptr() if self.n else None,
                  self.n, h, w, max(self.radius_cap, 2), model.data_ptr(), self.render_ws.data_ptr(),
                  self.render_ws.numel(), dev.stream_ptr())
        return model

    def _tile_medians(self, model, mode, thr_model=0.0, thr_dist=0.0, tile=None):
        h, w = self.shape
        tile = self.tile if tile is None else tile
        ny, nx = -(-h // tile), -(-w // tile)
        med = dev.empty((ny * nx,), torch.float64)
        cnt = dev.empty((ny * nx,), torch.int64)
        _lib.call("spx_tile_medians", self.img.data_ptr(), self.dtype, self.sign, h, w, _ptr(model),
                  _ptr(self.dist2), _ptr(self.usable_d), mode, float(thr_model), float(thr_dist), int(tile),
                  med.data_ptr(), cnt.data_ptr(), dev.stream_ptr())
        return med.cpu().numpy().reshape(ny, nx), cnt.cpu().numpy().reshape(ny, nx)

    def stats(self, params_d, status_d, maxstep_d=None):
        """Median amplitude and FWHM of the good cells (subpx/_cpu/deblend.py:463-464) and, given the
        steps, the 99th percentile of the finite ones (:517), computed on the device; one download.
        Returns (amplitude, fwhm, p99, n_finite, n_good)."""
        n = self.n
        if n == 0:
            return 1.0, 0.0, np.nan, 0, 0
        fwhm = dev.empty((n,), torch.float64)
        good = dev.empty((n,), torch.uint8)
        _lib.call("spx_cell_stats", params_d.data_ptr(), status_d.data_ptr(), n, fwhm.data_ptr(), good.data_ptr(),
                  dev.stream_ptr())
        reqs = [_lib.QuantileReq(params_d.data_ptr(), 6, good.data_ptr(), 0, n, 0, 0.0),
                _lib.QuantileReq(fwhm.data_ptr(), 1, good.data_ptr(), 0, n, 0, 0.0)]
        if maxstep_d is not None:
            reqs.append(_lib.QuantileReq(maxstep_d.data_ptr(), 1, None, 1, n, 1, 99 / 100))
        res = quantiles(reqs)
        amplitude = float(res[0, 0]) if res[0, 1] > 0 else 1.0
        width = float(res[1, 0]) if res[1, 1] > 0 else 0.0
        if maxstep_d is None:
            return amplitude, width, np.nan, 0, int(res[0, 1])
        return amplitude, width, float(res[2, 0]), int(res[2, 1]), int(res[0, 1])

    def background_of(self, model, stats):
        """Background map and info (subpx/_cpu/deblend.py:459-466 background_of, 323-393); stats =
        (median amplitude, median FWHM) of the good cells."""
        if self.background_level is not None:
            return self.bg.set_fixed(self.background_level), {"source": "fixed"}
        amplitude, fwhm = stats[0], stats[1]
        tile = self.tile
        free_med, free_count = self._tile_medians(model, _lib.TILE_FREE, self.free_fraction * amplitude,
                                                  self.free_distance_fwhm * fwhm)
        measured = free_count >= max(16, int(0.1 * tile * tile))
        info = {"tiles": int(measured.size), "measured_tiles": int(measured.sum())}
        if measured.all():
            medians, info["source"] = free_med, "measured"
        elif measured.any():
            medians, info["source"] = interpolate_tiles(free_med, measured, tile, self.shape), "interpolated"
        else:
            medians, _ = self._tile_medians(model, _lib.TILE_USABLE)
            info["source"] = "inferred"
            if np.isnan(medians).all():
                whole, _ = self._tile_medians(model, _lib.TILE_ALL, tile=max(self.shape))
                return self.bg.set_fixed(float(whole.ravel()[0])), info
            medians = np.where(np.isnan(medians), np.nanmedian(medians), medians)
        info["tile_medians"] = medians
        return self.bg.set_medians(medians), info

    def initial(self, max_iter, warm_params=None, warm_ok=None, extras=False, warm_cost_tol=1e-12):
        """Initial fits (subpx/_cpu/deblend.py:152-171 + LM). With warm_params (n x 6, ROI-local,
        device) the LM starts there and falls back to the plain start per cell (learned warm
        start); extras=True also returns the cell-border backgrounds and the fallback flags."""
        h, w = self.shape
        c = self.cells
        params = dev.empty((self.n, 6), torch.float64)
        status = dev.empty((self.n,), torch.uint8)
        iters = dev.empty((self.n,), torch.int32)
        bg0 = dev.empty((self.n,), torch.float64) if extras else None
        fell = dev.empty((self.n,), torch.uint8) if extras else None
        has = self.background_level is not None
        warm_cost_tol = max(float(warm_cost_tol), self.fit_options.cost_tol)
        _lib.call("spx_deblend_initial_warm", self.img.data_ptr(), self.dtype, self.sign, h, w, c.voronoi.data_ptr(),
                  c.boxes.data_ptr(), c.caps.data_ptr(), c.seeds_d.data_ptr(), self.n, c.hm, c.wm, c.max_px,
                  float(self.background_level) if has else 0.0, int(has), int(max_iter), _ptr(warm_params),
                  _ptr(warm_ok), float(warm_cost_tol), params.data_ptr(), status.data_ptr(), iters.data_ptr(),
                  _ptr(bg0), _ptr(fell), None, self.fit_options,
                  self.fit_ws.data_ptr(), self.fit_ws.numel(), dev.stream_ptr())
        if extras:
            return params, status, iters, bg0, fell
        return params, status, iters

    def iteration(self, params_d, model, bg: Background):
        h, w = self.shape
        c = self.cells
        out = dev.empty((self.n, 6), torch.float64)
        status = dev.empty((self.n,), torch.uint8)
        maxstep = dev.empty((self.n,), torch.float64)
        iters = dev.empty((self.n,), torch.int32)
        st = bg.struct()
        _lib.call("spx_deblend_iteration", self.img.data_ptr(), self.dtype, self.sign, h, w, c.voronoi.data_ptr(),
                  c.boxes.data_ptr(), c.caps.data_ptr(), self.n, c.hm, c.wm, c.max_px, st, model.data_ptr(),
                  max(self.radius_cap, 2), params_d.data_ptr(), float(self.relaxation), self.max_iter,
                  out.data_ptr(), status.data_ptr(), maxstep.data_ptr(), iters.data_ptr(), self.fit_options,
                  self.fit_ws.data_ptr(), self.fit_ws.numel(), dev.stream_ptr())
        return out, status, maxstep, iters

    def cleaned(self, state: DeblendState, which: np.ndarray | None = None) -> torch.Tensor:
        """(n_out, hm, wm) cleaned cells of `which` (all cells when None)."""
        h, w = self.shape
        c = self.cells
        n_out = self.n if which is None else len(which)
        out = dev.empty((n_out, c.hm, c.wm), torch.float64)
        which_d = None if which is None else dev.upload(np.asarray(which, dtype=np.int32))
        if n_out and c.hm and c.wm:
            _lib.call("spx_clean_cells", self.img.data_ptr(), self.dtype, self.sign, h, w, c.voronoi.data_ptr(),
                      c.boxes.data_ptr(), state.params_d.data_ptr(), max(self.radius_cap, 2),
                      state.background.struct(), state.model.data_ptr(), _ptr(which_d), n_out, c.hm, c.wm,
                      out.data_ptr(), dev.stream_ptr())
        return out

    # ------------------------------------------------------------------------------- run
    def run(self, *, iterations: int = 30, init: np.ndarray | None = None) -> DeblendState:
        """deblend() of subpx/_cpu/deblend.py:421-522."""
        if self.n == 0:
            model = torch.zeros(self.shape, dtype=torch.float64, device="cuda")
            bg, info = self.background_of(model, (1.0, 0.0))
            return DeblendState(bg, model, np.zeros((0, 6)), dev.empty((0, 6), torch.float64),
                                np.zeros(0, np.uint8), dev.empty((0,), torch.uint8), self.tile, 0, info, False)
        fit_iters = []
        if init is None:
            from . import warmstart

            net = warmstart.active()
            if net is not None and self.n:
                p0, ok = warmstart.predict_init(net, self.img, self.sign, self.cells.seeds_d, self.cells.boxes,
                                                self.n)
                params_d, status_d, it = self.initial(self.max_iter, warm_params=p0, warm_ok=ok,
                                                      warm_cost_tol=net.cost_tol)
            else:
                params_d, status_d, it = self.initial(self.max_iter)
            fit_iters.append(it)
        else:
            init = np.asarray(init, dtype=np.float64)
            params_d = dev.upload(init)
            status_d = self._status_of(params_d)
        stats = self.stats(params_d, status_d)
        model = self.render(params_d)
        used, converged = 0, False
        for used in range(1, int(iterations) + 1):
            bg, info = self.background_of(model, stats)
            params_d, status_d, maxstep_d, it = self.iteration(params_d, model, bg)
            fit_iters.append(it)
            model = self.render(params_d)
            stats = self.stats(params_d, status_d, maxstep_d)
            if stats[3] == 0:
                break
            if stats[2] < self.tolerance:
                converged = True
                break
        bg, info = self.background_of(model, stats)
        self.check_render()
        # Host copies through pinned memory (cached blocks, no fresh pageable arrays to fault in).
        params_h, status_h = dev.start_download(params_d), dev.start_download(status_d)
        torch.cuda.current_stream().synchronize()
        return DeblendState(bg, model, params_h, params_d, status_h, status_d, self.tile,
                            used, info, converged, fit_iters, stats[0] if stats[4] else float("nan"))

    def check_render(self):
        """Raise if a render since the last check overflowed a tile's Gaussian list."""
        if not self.n:
            return
        h, w = self.shape
        flag = ctypes.c_int(0)
        _lib.call("spx_render_overflow", self.render_ws.data_ptr(), self.n, h, w, ctypes.byref(flag), 0,
                  dev.stream_ptr())
        if flag.value:
            raise RuntimeError("render: more than 2048 truncated Gaussians reach one 16x16 tile")

    def _status_of(self, params_d):
        """fit_status of given params: an iteration pass with relaxation 0 returns the params unchanged
        (finite steps times 0) and the status of those params."""
        h, w = self.shape
        c = self.cells
        out = dev.empty((self.n, 6), torch.float64)
        status = dev.empty((self.n,), torch.uint8)
        maxstep = dev.empty((self.n,), torch.float64)
        # relaxation 0 leaves the params unchanged; the LM result is discarded.
        zero_model = torch.zeros(self.shape, dtype=torch.float64, device="cuda")
        st = self.bg.set_fixed(0.0).struct()
        _lib.call("spx_deblend_iteration", self.img.data_ptr(), self.dtype, self.sign, h, w, c.voronoi.data_ptr(),
                  c.boxes.data_ptr(), c.caps.data_ptr(), self.n, c.hm, c.wm, c.max_px, st, zero_model.data_ptr(),
                  max(self.radius_cap, 2), params_d.data_ptr(), 0.0, 1, out.data_ptr(), status.data_ptr(),
                  maxstep.data_ptr(), None, None, self.fit_ws.data_ptr(), self.fit_ws.numel(), dev.stream_ptr())
        return status
