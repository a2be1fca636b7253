"""Multi-GPU sharding of the centre-detection path: one process per GPU, torch.distributed.

Two ways the work splits (no exchange on the data path except the two listed collectives):

* Independent units -- pages of a batch, frames of a stack (``detect_centers_batch``,
  subpx/batch.py:22-24): each rank takes a contiguous run of them (``units_of_rank``).
* One large page (``detect_centers(tile_h=...)``, subpx/_gpu/centers.py:1778-1862): the row bands of
  tile_h rows stepping tile_h - overlap are dealt round-robin to the ranks. Two collectives:

  - the global Otsu threshold of img[::ds, ::ds]: every rank histograms a contiguous share of the
    sampled rows; the 65,536-bin histograms are summed and the value ranges min/max-reduced with
    ``all_reduce``, then each rank runs the same Otsu scan (identical thresholds everywhere);
  - the kept centres of every band are ``all_gather``-ed, put back in band order, and deduplicated
    (every rank ends with the same result).

The per-band work and the histogram are behind a small ``ops`` object so that the same driver runs
on the GPU (``GpuBandOps``, NCCL) and, for tests of the sharding on the CPU, over ``gloo``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch
import torch.distributed as dist

NBINS = 65536


@dataclass(frozen=True)
class Band:
    index: int
    y0: int
    y1: int
    keep_lo: int
    keep_hi: int


def band_plan(height: int, tile_h: int, overlap: int) -> list[Band]:
    """Bands of subpx/_gpu/centers.py:1812-1835: rows [y0, y0 + tile_h) stepping tile_h - overlap;
    a band keeps centres with keep_lo <= y < keep_hi (overlap // 2 inside its cut edges)."""
    if overlap >= tile_h:
        raise ValueError("overlap must be < tile_h")
    step, half = tile_h - overlap, overlap // 2
    bands, y0 = [], 0
    while y0 < height:
        y1 = min(height, y0 + tile_h)
        bands.append(Band(len(bands), y0, y1, y0 if y0 == 0 else y0 + half, y1 if y1 == height else y1 - half))
        if y1 == height:
            break
        y0 += step
    return bands


def bands_of_rank(bands: list[Band], rank: int, world: int) -> list[Band]:
    """Round-robin: band b goes to rank b % world (neighbouring bands land on different GPUs, so a
    page's density gradient spreads over all of them)."""
    return [b for b in bands if b.index % world == rank]


def units_of_rank(n: int, rank: int, world: int) -> range:
    """Contiguous share [lo, hi) of n independent units (pages, frames) for this rank."""
    base, extra = divmod(int(n), int(world))
    lo = rank * base + min(rank, extra)
    return range(lo, lo + base + (1 if rank < extra else 0))


def sampled_rows_of_rank(height: int, ds: int, rank: int, world: int) -> tuple[int, int]:
    """This rank's share of the rows of img[::ds, ::ds], as image rows [r0, r1) with r0 % ds == 0,
    so that img[r0:r1][::ds] are exactly those sampled rows."""
    n_sampled = -(-height // ds)
    share = units_of_rank(n_sampled, rank, world)
    return share.start * ds, min(height, share.stop * ds)


def allreduce_histogram(hist: torch.Tensor, value_range: torch.Tensor, group=None):
    """Sums int64 histograms over the ranks and reduces the [min, max] value ranges (int64) in place."""
    dist.all_reduce(hist, op=dist.ReduceOp.SUM, group=group)
    lo, hi = value_range[0:1].clone(), value_range[1:2].clone()
    dist.all_reduce(lo, op=dist.ReduceOp.MIN, group=group)
    dist.all_reduce(hi, op=dist.ReduceOp.MAX, group=group)
    value_range[0:1] = lo
    value_range[1:2] = hi
    return hist, value_range


def gather_band_centres(pieces: dict[int, np.ndarray], device: str, group=None) -> list[np.ndarray]:
    """All-gathers {band index: (n, 2) centres} from every rank; returns every band's centres in
    band order (the order the single-GPU driver concatenates them in)."""
    world = dist.get_world_size(group)
    rows = [np.column_stack((np.full(len(c), b, np.float64), np.asarray(c, np.float64).reshape(-1, 2)))
            for b, c in sorted(pieces.items())]
    local = np.vstack(rows) if rows else np.zeros((0, 3))
    count = torch.tensor([len(local)], dtype=torch.int64, device=device)
    counts = [torch.zeros_like(count) for _ in range(world)]
    dist.all_gather(counts, count, group=group)
    n_max = max(int(c.item()) for c in counts)
    buf = torch.zeros((max(n_max, 1), 3), dtype=torch.float64, device=device)
    buf[: len(local)] = torch.from_numpy(local).to(device)
    bufs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf, group=group)
    allrows = np.vstack([b[: int(c.item())].cpu().numpy() for b, c in zip(bufs, counts)])
    by_band: dict[int, np.ndarray] = {}
    for b in np.unique(allrows[:, 0]).astype(int) if len(allrows) else []:
        by_band[int(b)] = allrows[allrows[:, 0] == b, 1:]
    return [by_band[b] for b in sorted(by_band)]


class GpuBandOps:
    """The per-rank work on this process's GPU through libsubpx_b200 (collectives over NCCL)."""

    device = "cuda"

    def __init__(self, **detect_kw):
        self.kw = detect_kw

    def histogram(self, rows: np.ndarray, step: int):
        """(hist int64[65536], [min, max] int64, sampled pixel count) of rows[::step, ::step]."""
        from . import _device as dev
        from . import _lib

        img = dev.upload(np.ascontiguousarray(rows))
        h, w = img.shape
        hist = dev.empty((NBINS,), torch.int32)
        rng = dev.empty((2,), torch.int32)
        _lib.call("spx_histogram", img.data_ptr(), dev.dtype_code(img), h, w, int(step), hist.data_ptr(),
                  rng.data_ptr(), dev.stream_ptr())
        n = (-(-h // step)) * (-(-w // step))
        # The uint32 counts and values, widened exactly to int64 for the reduction.
        return hist.to(torch.int64) & 0xFFFFFFFF, rng.to(torch.int64) & 0xFFFFFFFF, n

    def otsu(self, hist: torch.Tensor, value_range: torch.Tensor, total: int, dtype) -> float:
        from . import _device as dev
        from . import _lib

        if total >= 1 << 32:
            raise ValueError("the global Otsu sample exceeds 2^32 pixels; raise otsu_downsample")
        code = _lib.DTYPES[np.dtype(dtype)]
        # Back to the uint32 bit patterns the kernel reads (two's-complement wrap of int64 -> int32).
        h32 = hist.to(torch.int64).to(torch.int32).contiguous()
        r32 = value_range.to(torch.int64).to(torch.int32).contiguous()
        out = dev.empty((1,), torch.float64)
        ws = dev.workspace(_lib.size("spx_otsu_workspace_bytes", code))
        _lib.call("spx_otsu_from_histogram", h32.data_ptr(), code, r32.data_ptr(), int(total), out.data_ptr(),
                  ws.data_ptr(), ws.numel(), dev.stream_ptr())
        return float(out.item())

    def detect(self, band: np.ndarray, fixed_threshold: float | None) -> np.ndarray:
        """Finite refined centres of one band (band-local coordinates, label order)."""
        from . import _device as dev
        from . import segment
        from .centers import _centers_on_device, _finite

        kw = dict(self.kw)
        method = kw.pop("threshold", "otsu")
        img = dev.upload(np.ascontiguousarray(band))
        thr = segment.binarize_threshold(img, method, kw["invert"]) if fixed_threshold is None else None
        c = _centers_on_device(img, threshold_dev=thr,
                               fixed_threshold=0.0 if fixed_threshold is None else float(fixed_threshold), **kw)
        return _finite(c)

    def dedupe(self, points: np.ndarray, eps: float) -> np.ndarray:
        from .tiled import dedupe_centers

        return dedupe_centers(points, eps=eps)


def detect_tiled_sharded(image: np.ndarray, *, tile_h: int, overlap: int = 128, threshold_mode: str = "auto",
                         otsu_downsample: int = 4, thr_scale: float = 0.8, dedupe_eps: float = 1.5, ops=None,
                         group=None) -> np.ndarray:
    """Tiled detection of one page with its bands spread over the process group (every rank passes
    the same host page and gets the same (N, 2) centres back). ``ops`` does the per-rank work:
    GpuBandOps by default."""
    if threshold_mode not in ("auto", "global", "per_tile"):
        raise ValueError("threshold_mode must be 'auto', 'global' or 'per_tile'")
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    img = np.asarray(image)
    height = img.shape[0]
    bands = band_plan(height, int(tile_h), int(overlap))
    pre = None
    if threshold_mode in ("global", "auto"):
        ds = max(1, int(otsu_downsample))
        r0, r1 = sampled_rows_of_rank(height, ds, rank, world)
        if r1 > r0:
            hist, value_range, n = ops.histogram(img[r0:r1], ds)
        else:  # more ranks than sampled rows
            hist = torch.zeros(NBINS, dtype=torch.int64, device=ops.device)
            value_range = torch.tensor([np.iinfo(np.int64).max, 0], dtype=torch.int64, device=ops.device)
            n = 0
        hist, value_range = hist.to(ops.device), value_range.to(ops.device)
        allreduce_histogram(hist, value_range, group)
        total = torch.tensor([n], dtype=torch.int64, device=ops.device)
        dist.all_reduce(total, group=group)
        pre = ops.otsu(hist, value_range, int(total.item()), img.dtype) * float(thr_scale)
    pieces = {}
    for b in bands_of_rank(bands, rank, world):
        c = ops.detect(img[b.y0:b.y1], pre)
        if len(c):
            c = np.asarray(c, np.float64).copy()
            c[:, 1] += b.y0
            c = c[(c[:, 1] >= b.keep_lo) & (c[:, 1] < b.keep_hi)]
        pieces[b.index] = np.asarray(c, np.float64).reshape(-1, 2)
    kept = [c for c in gather_band_centres(pieces, ops.device, group) if len(c)]
    if not kept:
        return np.zeros((0, 2))
    return ops.dedupe(np.vstack(kept), float(dedupe_eps))


def measure_cds_sharded(pages, *, measure=None, group=None, dst: int | None = 0, **measure_kw):
    """measure_cds of a batch of pages (a sequence or an (N, H, W) stack, e.g. the images of an
    uneven stack or the pages of a TIFF batch) spread over the process group: rank r measures the
    contiguous run units_of_rank(N, r, world) of pages (each page once, no exchange while
    measuring), and the per-page results are gathered in page order, as the reference's batch
    pipeline runs one worker process per GPU over its share of the pages and collects their
    summaries (scripts/cd_batch.py:369-420, 705-728).

    ``measure`` maps one page to its result (default: ``measure_cds(page, backend="gpu",
    summary_only=True, **measure_kw)`` on this rank's GPU). Results are gathered to rank ``dst``
    (other ranks return None), or to every rank when ``dst`` is None. Every rank must call this
    with the same number of pages."""
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    if measure is None:
        from .cd import measure_cds

        kw = dict(summary_only=True, **measure_kw)

        def measure(page):
            return measure_cds(page, backend="gpu", **kw)

    n = len(pages)
    local = [(i, measure(pages[i])) for i in units_of_rank(n, rank, world)]
    if dst is None:
        parts = [None] * world
        dist.all_gather_object(parts, local, group=group)
    else:
        parts = [None] * world if rank == dst else None
        dist.gather_object(local, parts, dst=dst, group=group)
        if rank != dst:
            return None
    out = [None] * n
    for part in parts:
        for i, res in part:
            out[i] = res
    return out
