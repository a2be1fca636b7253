"""Learned warm start of the initial LM fits (no reference counterpart).

A 1024 -> 256 -> 256 -> 7 MLP (ReLU) reads a cell's 32 x 32 signal patch (normalised by its border
level and peak, ``spx_extract_patches``) and predicts the parameters the plain initial fit ends
at, relative to the patch: [A / amp, x0 - cx, y0 - cy, u1, u2, u3, (bg0 - bg) / amp] with (cx, cy)
the patch centre and bg0 the cell-border background the fit subtracts. The LM then starts there
(``spx_deblend_initial_warm``) and falls back to the plain start for every cell whose warm fit does
not meet the stop rule within the iteration cap or does not end "ok".

Everything runs on the GPU through the library: bf16 GEMMs on the tensor cores (tcgen05, f32
accumulation in TMEM) for the forward pass and both backward products, the weighted-MSE gradient,
the bias-gradient row sums and AdamW on f32 master weights. Outputs are standardised by the
training set's mean and standard deviation, which are part of the saved model.

Training data: synthetic pages of superellipse holes (random pitch, diameter, ellipticity,
rotation, corner rounding, blur and SNR) rendered on the GPU, run through the same detection and
plain initial fit as production; each "ok" cell gives one (patch, fit) example.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _device as dev
from . import _lib

IN, HID, OUT, OUT_PAD = 1024, 256, 7, 16
IN_CENTRE = 16.0  # the patch's centre pixel, (16, 16) from its origin
DEFAULT_MODEL = Path(__file__).resolve().parent / "data" / "warmstart_mlp.npz"


def _gemm(a, b, m, n, k, *, lda=None, ldb=None, scale=1.0, bias=None, relu=False, mask=None, ld_mask=0,
          out_f32=None, ld_f32=0, accumulate=False, out_bf16=None, ld_bf16=0, out_t=None, ld_t=0, err=None):
    ep = _lib.GemmEpilogue()
    ep.scale = scale
    ep.bias = None if bias is None else bias.data_ptr()
    ep.relu = int(relu)
    ep.mask_act = None if mask is None else mask.data_ptr()
    ep.ld_mask = ld_mask
    ep.out_f32 = None if out_f32 is None else out_f32.data_ptr()
    ep.ld_f32 = ld_f32
    ep.accumulate = int(accumulate)
    ep.out_bf16 = None if out_bf16 is None else out_bf16.data_ptr()
    ep.ld_bf16 = ld_bf16
    ep.out_bf16_t = None if out_t is None else out_t.data_ptr()
    ep.ld_t = ld_t
    _lib.call("spx_gemm_bf16", a.data_ptr(), lda or k, b.data_ptr(), ldb or k, m, n, k, ep, err.data_ptr(),
              dev.stream_ptr())


@dataclass
class _Param:
    w: torch.Tensor   # f32 master
    m: torch.Tensor
    v: torch.Tensor
    g: torch.Tensor


class WarmStartNet:
    """The MLP with its f32 master weights, AdamW state and bf16 working copies on the device."""

    def __init__(self, seed: int = 0):
        rng = np.random.default_rng(seed)

        def he(rows, cols):
            return rng.normal(0.0, np.sqrt(2.0 / cols), (rows, cols)).astype(np.float32)

        host = {"w1": he(HID, IN), "b1": np.zeros(HID, np.float32), "w2": he(HID, HID),
                "b2": np.zeros(HID, np.float32), "w3": (he(OUT, HID) * 0.1).astype(np.float32),
                "b3": np.zeros(OUT, np.float32)}
        self._setup(host)
        self.set_output_scale(np.zeros(OUT), np.ones(OUT))

    def _setup(self, host):
        self.p = {}
        for name, arr in host.items():
            w = dev.upload(np.ascontiguousarray(arr, dtype=np.float32))
            self.p[name] = _Param(w, torch.zeros_like(w), torch.zeros_like(w), torch.zeros_like(w))
        bf = torch.bfloat16
        self.w1 = dev.empty((HID, IN), bf)
        self.w2 = dev.empty((HID, HID), bf)
        self.w2t = dev.empty((HID, HID), bf)
        self.w3 = torch.zeros((OUT_PAD, HID), dtype=bf, device="cuda")
        self.w3t = torch.zeros((HID, OUT_PAD), dtype=bf, device="cuda")
        self.step = 0
        self.err = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.w1.copy_(self.p["w1"].w.to(bf))
        self.w2.copy_(self.p["w2"].w.to(bf))
        self.w2t.copy_(self.p["w2"].w.t().to(bf))
        self.w3[:OUT].copy_(self.p["w3"].w.to(bf))
        self.w3t[:, :OUT].copy_(self.p["w3"].w.t().to(bf))

    # Stop rule of the warm-started fits: an accepted step that lowers the cost by at most this
    # fraction ends the fit (the plain rule is 1e-12). Chosen on held-out pages so that the warm
    # fits stay far inside the 1e-3 px accuracy they are held to against the plain FP64 fit.
    cost_tol = 1e-7

    def set_output_scale(self, mean, std):
        self.out_mean = np.asarray(mean, dtype=np.float64)
        self.out_std = np.asarray(std, dtype=np.float64)
        self.mean_d = dev.upload(self.out_mean)
        self.std_d = dev.upload(self.out_std)

    # ---------------------------------------------------------------------------- forward
    def forward(self, x: torch.Tensor, keep: bool = False):
        """x: (B, 1024) bf16 on the device -> standardised outputs (B, 7) f32 (and activations)."""
        b = x.shape[0]
        bf = torch.bfloat16
        h1 = dev.empty((b, HID), bf)
        h2 = dev.empty((b, HID), bf)
        h1t = dev.empty((HID, b), bf) if keep else None
        h2t = dev.empty((HID, b), bf) if keep else None
        y = dev.empty((b, OUT), torch.float32)
        _gemm(x, self.w1, b, HID, IN, bias=self.p["b1"].w, relu=True, out_bf16=h1, ld_bf16=HID, out_t=h1t, ld_t=b,
              err=self.err)
        _gemm(h1, self.w2, b, HID, HID, bias=self.p["b2"].w, relu=True, out_bf16=h2, ld_bf16=HID, out_t=h2t, ld_t=b,
              err=self.err)
        _gemm(h2, self.w3, b, OUT, HID, bias=self.p["b3"].w, out_f32=y, ld_f32=OUT, err=self.err)
        if keep:
            return y, (h1, h1t, h2, h2t)
        return y

    # ---------------------------------------------------------------------------- training
    def train_step(self, x: torch.Tensor, xt: torch.Tensor, t: torch.Tensor, weights: torch.Tensor, *, lr: float,
                   weight_decay: float = 1e-4, loss_acc: torch.Tensor | None = None) -> torch.Tensor:
        """One AdamW step on the batch (x: B x 1024 bf16, xt: its transpose, t: B x 7 standardised
        targets f32; B a multiple of 8). Returns the device loss accumulator (f64)."""
        b = x.shape[0]
        bf = torch.bfloat16
        y, (h1, h1t, h2, h2t) = self.forward(x, keep=True)
        if loss_acc is None:
            loss_acc = torch.zeros(1, dtype=torch.float64, device="cuda")
        dy = dev.empty((b, OUT_PAD), bf)
        dyt = dev.empty((OUT_PAD, b), bf)
        _lib.call("spx_mlp_loss_grad", y.data_ptr(), t.data_ptr(), weights.data_ptr(), b, OUT, OUT_PAD, dy.data_ptr(),
                  dyt.data_ptr(), loss_acc.data_ptr(), dev.stream_ptr())
        p = self.p
        # dW3 = dY^T H2, db3 = row sums of dY^T.
        _gemm(dyt, h2t, OUT, HID, b, out_f32=p["w3"].g, ld_f32=HID, err=self.err)
        _lib.call("spx_rowsum_bf16", dyt.data_ptr(), OUT, b, p["b3"].g.data_ptr(), dev.stream_ptr())
        # dH2 = (dY W3) * (H2 > 0), kept transposed for dW2 and row-major for dH1.
        dh2 = dev.empty((b, HID), bf)
        dh2t = dev.empty((HID, b), bf)
        _gemm(dy, self.w3t, b, HID, OUT_PAD, mask=h2, ld_mask=HID, out_bf16=dh2, ld_bf16=HID, out_t=dh2t, ld_t=b,
              err=self.err)
        _gemm(dh2t, h1t, HID, HID, b, out_f32=p["w2"].g, ld_f32=HID, err=self.err)
        _lib.call("spx_rowsum_bf16", dh2t.data_ptr(), HID, b, p["b2"].g.data_ptr(), dev.stream_ptr())
        # dH1 = (dH2 W2) * (H1 > 0), transposed only.
        dh1t = dev.empty((HID, b), bf)
        _gemm(dh2, self.w2t, b, HID, HID, mask=h1, ld_mask=HID, out_t=dh1t, ld_t=b, err=self.err)
        _gemm(dh1t, xt, HID, IN, b, out_f32=p["w1"].g, ld_f32=IN, err=self.err)
        _lib.call("spx_rowsum_bf16", dh1t.data_ptr(), HID, b, p["b1"].g.data_ptr(), dev.stream_ptr())
        self.step += 1
        self._adamw(lr, weight_decay)
        return loss_acc

    def _adamw(self, lr, weight_decay, beta1=0.9, beta2=0.999, eps=1e-8):
        s = dev.stream_ptr()
        p = self.p
        for name, out, out_rows, out_t, ld_t in (("w1", self.w1, HID, None, 0), ("w2", self.w2, HID, self.w2t, HID),
                                                 ("w3", self.w3, OUT_PAD, self.w3t, OUT_PAD), ("b1", None, 0, None, 0),
                                                 ("b2", None, 0, None, 0), ("b3", None, 0, None, 0)):
            q = p[name]
            rows, cols = (q.w.shape[0], q.w.shape[1]) if q.w.dim() == 2 else (1, q.w.shape[0])
            wd = weight_decay if name.startswith("w") else 0.0
            _lib.call("spx_adamw", q.w.data_ptr(), q.g.data_ptr(), q.m.data_ptr(), q.v.data_ptr(), rows, cols,
                      self.step, ctypes.c_float(lr), ctypes.c_float(beta1), ctypes.c_float(beta2),
                      ctypes.c_float(eps), ctypes.c_float(wd), None if out is None else out.data_ptr(),
                      out_rows, None if out_t is None else out_t.data_ptr(), ld_t, s)

    def check_errors(self):
        if int(self.err.item()):
            raise RuntimeError("a tensor-core GEMM gave up waiting for its MMAs")

    # ---------------------------------------------------------------------------- persistence
    def state(self) -> dict:
        out = {name: q.w.cpu().numpy() for name, q in self.p.items()}
        out["out_mean"] = self.out_mean
        out["out_std"] = self.out_std
        return out

    def save(self, path):
        Path(path).parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(path, **self.state())

    @classmethod
    def load(cls, path=DEFAULT_MODEL) -> "WarmStartNet":
        z = np.load(path)
        net = cls.__new__(cls)
        net._setup({k: z[k] for k in ("w1", "b1", "w2", "b2", "w3", "b3")})
        net.set_output_scale(z["out_mean"], z["out_std"])
        return net


# ------------------------------------------------------------------------------- switch

_ACTIVE: "WarmStartNet | None" = None


def use(model=DEFAULT_MODEL) -> "WarmStartNet | None":
    """Turns the warm start of every later measure_cds / deblend on (a WarmStartNet or a saved
    model path; the packaged model by default) or off (None / False). Returns the active net."""
    global _ACTIVE
    if model is None or model is False:
        _ACTIVE = None
    elif isinstance(model, WarmStartNet):
        _ACTIVE = model
    else:
        _ACTIVE = WarmStartNet.load(model)
    return _ACTIVE


def active() -> "WarmStartNet | None":
    return _ACTIVE


# ---------------------------------------------------------------------------------- inference

def patches(image_d: torch.Tensor, sign: float, seeds_d: torch.Tensor, n: int, images: int = 1,
            boxes_d: torch.Tensor | None = None):
    """(n, 1024) bf16 patches and (n, 4) [origin x, origin y, bg, amp] around the seeds. With
    images > 1 the (rows, W) image is a stack of that many images of rows / images rows each, the
    cell boxes (y in stack rows) say which image each cell is in, the seeds are in that image's rows,
    and each patch replicates the edges of its cell's image."""
    h, w = image_d.shape
    if images < 1 or h % images or (images > 1 and boxes_d is None):
        raise ValueError(f"{h} rows do not split into {images} images with cell boxes")
    out = dev.empty((max(n, 1), IN), torch.bfloat16)
    norm = dev.empty((max(n, 1), 4), torch.float64)
    if n:
        _lib.call("spx_extract_patches_stack", image_d.data_ptr(), dev.dtype_code(image_d), float(sign), images,
                  h // images, w, seeds_d.data_ptr(), None if images == 1 else boxes_d.data_ptr(), n,
                  out.data_ptr(), norm.data_ptr(), dev.stream_ptr())
    return out[:n], norm[:n]


def predict_init(net: WarmStartNet, image_d: torch.Tensor, sign: float, seeds_d: torch.Tensor, boxes_d: torch.Tensor,
                 n: int, batch: int | None = None, images: int = 1):
    """ROI-local LM starting params (n, 6) f64 and validity flags for the cells, on the device.
    All cells go through each layer in one GEMM launch unless `batch` bounds the rows per launch
    (the activations take 1 KB per row); a row's outputs do not depend on the batching. `images` as
    in `patches`."""
    x, norm = patches(image_d, sign, seeds_d, n, images, boxes_d)
    if n and (batch is None or batch >= n):
        y = net.forward(x)
    else:
        y = dev.empty((max(n, 1), OUT), torch.float32)
        for b0 in range(0, n, batch or 1):
            y[b0:b0 + batch] = net.forward(x[b0:b0 + batch])
    params = dev.empty((max(n, 1), 6), torch.float64)
    ok = dev.empty((max(n, 1),), torch.uint8)
    _lib.call("spx_mlp_outputs_to_params", y.data_ptr(), net.mean_d.data_ptr(), net.std_d.data_ptr(),
              norm.data_ptr(), boxes_d.data_ptr(), n, params.data_ptr(), ok.data_ptr(), dev.stream_ptr())
    return params[:n], ok[:n]


def targets(params: torch.Tensor, bg0: torch.Tensor, norm: torch.Tensor, boxes_d: torch.Tensor) -> torch.Tensor:
    """Training targets (n, 7) f64 from plain fits (ROI-local params), their backgrounds and the
    patches' normalisation."""
    box = boxes_d.double()
    amp = norm[:, 3]
    gx = params[:, 1] + box[:, 0]
    gy = params[:, 2] + box[:, 1]
    return torch.stack([params[:, 0] / amp, gx - (norm[:, 0] + IN_CENTRE), gy - (norm[:, 1] + IN_CENTRE),
                        params[:, 3], params[:, 4], params[:, 5], (bg0 - norm[:, 2]) / amp], dim=1)


# ------------------------------------------------------------------------------- training set

def synth_page(seed: int, size: int = 2048):
    """A synthetic page of superellipse holes rendered on the device: (uint16 page, info)."""
    rng = np.random.default_rng(seed)
    pitch = rng.uniform(16.0, 40.0)
    d = float(np.clip(pitch * rng.uniform(0.4, 0.6), 8.0, 20.0))
    staggered = bool(rng.random() < 0.5)
    dy = pitch * (np.sqrt(3.0) / 2.0 if staggered else 1.0)
    ys = np.arange(-pitch, size + pitch, dy)
    rows = []
    for r, y in enumerate(ys):
        off = (pitch / 2.0) if (staggered and r % 2) else 0.0
        xs = np.arange(-pitch + off, size + pitch, pitch)
        rows.append(np.column_stack((xs, np.full(len(xs), y))))
    c = np.vstack(rows)
    c = c + rng.uniform(-0.5, 0.5, c.shape)
    c = c[rng.random(len(c)) >= 0.05]                       # 5 % missing holes
    merge = rng.random(len(c)) < 0.02                        # 2 % moved to touch their +x neighbour
    c[merge, 0] += pitch - 0.9 * d
    n = len(c)
    di = d * (1.0 + rng.uniform(-0.05, 0.05, n))
    e = rng.uniform(0.0, 0.1, n)
    holes = np.column_stack((c, di / 2 * (1 + e / 2), di / 2 * (1 - e / 2), rng.uniform(0, np.pi, n),
                             rng.uniform(2.0, 6.0, n)))
    sigma = rng.uniform(0.8, 2.5)
    amp, bg = rng.uniform(1500.0, 4000.0), rng.uniform(500.0, 1500.0)
    noise = amp / rng.uniform(10.0, 100.0)
    cell = float(np.ceil(pitch))
    gw = int(np.ceil(size / cell)) + 1
    gx = np.clip(np.floor(holes[:, 0] / cell).astype(np.int64), 0, gw - 1)
    gy = np.clip(np.floor(holes[:, 1] / cell).astype(np.int64), 0, gw - 1)
    key = gy * gw + gx
    order = np.argsort(key, kind="stable")
    start = np.zeros(gw * gw + 1, np.int64)
    np.add.at(start, key + 1, 1)
    start = np.cumsum(start).astype(np.int32)
    holes_d = dev.upload(np.ascontiguousarray(holes))
    start_d, ids_d = dev.upload(start), dev.upload(order.astype(np.int32))
    cov = dev.empty((size, size), torch.float64)
    s = dev.stream_ptr()
    _lib.call("spx_hole_coverage", size, size, holes_d.data_ptr(), start_d.data_ptr(), ids_d.data_ptr(), gw, gw, cell,
              4, cov.data_ptr(), s)
    radius = int(4.0 * sigma + 0.5)
    x = np.arange(-radius, radius + 1)
    phi = np.exp(-0.5 / (sigma * sigma) * x ** 2)
    wts = dev.upload(phi / phi.sum())
    tmp = dev.empty((size, size), torch.float64)
    blur = dev.empty((size, size), torch.float64)
    _lib.call("spx_gaussian_filter", cov.data_ptr(), size, size, wts.data_ptr(), radius, tmp.data_ptr(),
              blur.data_ptr(), s)
    page = dev.empty((size, size), torch.uint16)
    _lib.call("spx_page_finish", blur.data_ptr(), size * size, float(bg), float(amp), float(noise),
              ctypes.c_ulonglong(int(rng.integers(0, 2 ** 63))), page.data_ptr(), s)
    info = dict(pitch=pitch, d=d, staggered=staggered, sigma=sigma, amp=amp, bg=bg, noise=noise, holes=n)
    return page, info


def page_cells(page_d: torch.Tensor, *, area_min: int = 10, area_max: int = 2000, pad: int = 3):
    """Otsu + CCL + area filter + Voronoi cells of a page, as measure_cds builds them."""
    from .cd import _segment
    from .deblend import build_cells

    comp, _ = _segment(page_d, "otsu", False)
    k = comp.count
    stats = comp.stats.cpu().numpy()[1:k + 1].astype(np.int64)
    cents = comp.centroids.cpu().numpy()[1:k + 1]
    area = stats[:, 4]
    keep = (area >= area_min) & (area <= area_max)
    rows = np.column_stack((stats[:, :4], cents)).astype(np.float64)[keep]
    return build_cells(rows, tuple(page_d.shape), pad)


def initial_fits(page_d: torch.Tensor, cells, *, sign: float = 1.0, max_iter: int = 30, warm=None,
                 cost_tol: float = 1e-12, precision: str = "fp64", rows_per_image: int = 0,
                 plain_cost_tol: float | None = None, costs: torch.Tensor | None = None):
    """The initial LM fits of the cells (plain, or warm-started with (params, ok)) in the given LM
    arithmetic: params, status, iterations, cell-border backgrounds and fallback flags (device).
    rows_per_image > 0: the page is a stack of such images (boxes in stack rows, seeds in image rows).
    plain_cost_tol: the plain-start fits' relative cost-drop stop rule (default: the arithmetic's,
    1e-12 in FP64, the reference's); costs: a (n,) float64 device tensor that receives each fit's
    converged LM cost."""
    from .deblend import fit_options

    opts = fit_options(precision, plain_cost_tol)
    opts.rows_per_image = int(rows_per_image)
    cost_tol = max(float(cost_tol), opts.cost_tol)
    n = cells.n
    h, w = page_d.shape
    ws = dev.workspace(_lib.size("spx_fit_workspace_bytes", cells.max_px))
    params = dev.empty((max(n, 1), 6), torch.float64)
    status = dev.empty((max(n, 1),), torch.uint8)
    iters = dev.empty((max(n, 1),), torch.int32)
    bg0 = dev.empty((max(n, 1),), torch.float64)
    fell = dev.empty((max(n, 1),), torch.uint8)
    wp, wo = (None, None) if warm is None else warm
    _lib.call("spx_deblend_initial_warm", page_d.data_ptr(), dev.dtype_code(page_d), float(sign), h, w,
              cells.voronoi.data_ptr(), cells.boxes.data_ptr(), cells.caps.data_ptr(), cells.seeds_d.data_ptr(), n,
              cells.hm, cells.wm, cells.max_px, 0.0, 0, int(max_iter), None if wp is None else wp.data_ptr(),
              None if wo is None else wo.data_ptr(), float(cost_tol), params.data_ptr(), status.data_ptr(),
              iters.data_ptr(),
              bg0.data_ptr(), fell.data_ptr(), None if costs is None else costs.data_ptr(), opts, ws.data_ptr(),
              ws.numel(), dev.stream_ptr())
    return params[:n], status[:n], iters[:n], bg0[:n], fell[:n]


def training_set(pages: int, *, size: int = 2048, seed: int = 0, max_iter: int = 30):
    """Patches (N, 1024) bf16 and targets (N, 7) f64 on the device from `pages` synthetic pages
    (the "ok" plain initial fits)."""
    xs, ts = [], []
    for k in range(pages):
        page, _ = synth_page(seed * 100003 + k, size)
        cells = page_cells(page)
        if cells.n == 0:
            continue
        params, status, _, bg0, _ = initial_fits(page, cells, max_iter=max_iter)
        x, norm = patches(page, 1.0, cells.seeds_d, cells.n)
        t = targets(params, bg0, norm, cells.boxes)
        ok = (status == 0) & torch.isfinite(t).all(dim=1)
        xs.append(x[ok])
        ts.append(t[ok])
    return torch.cat(xs), torch.cat(ts)


def train(net: WarmStartNet, x: torch.Tensor, t: torch.Tensor, *, epochs: int = 30, batch: int = 4096,
          lr: float = 2e-3, weight_decay: float = 1e-4, seed: int = 0, log=None) -> list[float]:
    """Trains on (x, t) (standardising t, holding out 2 % for the per-output report); returns the
    mean training loss of every epoch."""
    n = x.shape[0]
    mean = t.mean(dim=0)
    std = t.std(dim=0).clamp_min(1e-6)
    net.set_output_scale(mean.cpu().numpy(), std.cpu().numpy())
    ts = ((t - mean) / std).float().contiguous()
    order = torch.randperm(n, device="cuda", generator=torch.Generator(device="cuda").manual_seed(seed + 1))
    n_val = max(n // 50, 1)
    val, keep = order[:n_val], order[n_val:]
    x_val, t_val = x[val].contiguous(), ts[val]
    x, ts, n = x[keep].contiguous(), ts[keep].contiguous(), n - n_val
    if n < batch:
        raise ValueError(f"need at least one batch of {batch} examples, got {n}")
    weights = torch.ones(OUT, dtype=torch.float32, device="cuda")
    gen = torch.Generator(device="cuda").manual_seed(seed)
    steps_per_epoch = n // batch
    total = epochs * steps_per_epoch
    xt = dev.empty((IN, batch), torch.bfloat16)
    history = []
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=gen)
        acc = torch.zeros(1, dtype=torch.float64, device="cuda")
        for s in range(steps_per_epoch):
            idx = perm[s * batch:(s + 1) * batch]
            xb = x[idx].contiguous()
            tb = ts[idx].contiguous()
            _lib.call("spx_transpose_bf16", xb.data_ptr(), batch, IN, xt.data_ptr(), dev.stream_ptr())
            step = ep * steps_per_epoch + s
            rate = lr * 0.5 * (1.0 + np.cos(np.pi * step / total))  # cosine decay
            net.train_step(xb, xt, tb, weights, lr=float(rate), weight_decay=weight_decay, loss_acc=acc)
        history.append(float(acc.item()) / steps_per_epoch)
        net.check_errors()
        if log:
            rmse = ((net.forward(x_val) - t_val) ** 2).mean(dim=0).sqrt().cpu().numpy()
            log(f"epoch {ep + 1}/{epochs}: loss {history[-1]:.5f}; held-out RMSE per output (standardised) "
                + " ".join(f"{v:.3f}" for v in rmse))
    return history


# -------------------------------------------------------------------------------- evaluation

def compare_on_page(net: WarmStartNet, page_d: torch.Tensor, *, max_iter: int = 30, repeats: int = 3,
                    cells=None, precision: str = "fp64") -> dict:
    """The initial-fit stage of one page's cells in three arms, timed by CUDA events:

      plain_ref   plain start, the reference's stop rule (relative cost drop 1e-12);
      plain_loose plain start, the warm fits' stop rule (net.cost_tol, 1e-7): the like-for-like arm,
                  so warm over plain_loose is what the network alone gains;
      warm        patches + MLP + warm-started LM (net.cost_tol) with the plain-start fallback.

    Reported: LM iterations per arm, the fallback share, centre deviations of the loose arms from
    plain_ref ("ok" in both), and the fallback rule's miss rate: the share of kept warm fits whose
    converged LM cost exceeds the plain-start fit's under the same stop rule by more than ten times
    that rule's relative drop (both fits stop within about one such drop of the optimum), i.e. cells
    where "fall back whenever the warm fit's converged residual exceeds the plain fit's" would have
    refitted but the cheaper rule used here (stop within max_iter and end "ok") did not."""
    cells = page_cells(page_d) if cells is None else cells
    n = cells.n
    costs = {k: dev.empty((max(n, 1),), torch.float64) for k in ("plain_ref", "plain_loose", "warm")}

    def plain_ref():
        return initial_fits(page_d, cells, max_iter=max_iter, costs=costs["plain_ref"])

    def plain_loose():
        return initial_fits(page_d, cells, max_iter=max_iter, plain_cost_tol=net.cost_tol,
                            costs=costs["plain_loose"])

    def warm():
        p0, ok = predict_init(net, page_d, 1.0, cells.seeds_d, cells.boxes, n)
        return initial_fits(page_d, cells, max_iter=max_iter, warm=(p0, ok), cost_tol=net.cost_tol,
                            precision=precision, costs=costs["warm"])

    arms = {"plain_ref": plain_ref, "plain_loose": plain_loose, "warm": warm}
    for fn in arms.values():
        fn()
    t = {k: 0.0 for k in arms}
    res = {}
    for _ in range(repeats):
        for which, fn in arms.items():
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            res[which] = fn()
            e.record()
            torch.cuda.synchronize()
            t[which] += s.elapsed_time(e) / repeats
    net.check_errors()
    host = {k: [a.cpu().numpy() for a in v] for k, v in res.items()}
    cost = {k: v[:n].cpu().numpy() for k, v in costs.items()}
    pp, sp, ip = host["plain_ref"][:3]
    out = {"cells": int(n)}
    for k in ("plain_loose", "warm"):
        pk, sk = host[k][:2]
        both = (sp == 0) & (sk == 0)
        dc = np.abs(pk[both, 1:3] - pp[both, 1:3]).max(axis=1) if both.any() else np.zeros(0)
        out[f"{k}_centre_dev_max_px"] = float(dc.max()) if len(dc) else 0.0
        out[f"{k}_within_1e-3_px"] = float((dc <= 1e-3).mean()) if len(dc) else 1.0
        out[f"{k}_same_status"] = float((sp == sk).mean())
    fw = host["warm"][4].astype(bool)
    kept = ~fw & (host["warm"][1] == 0) & (host["plain_loose"][1] == 0)
    excess = (cost["warm"] - cost["plain_loose"]) / np.maximum(cost["plain_loose"], 1e-300)
    for k in arms:
        out[f"{k}_iterations_mean"] = float(host[k][2].mean())
        out[f"{k}_ms"] = t[k]
        out[f"{k}_cells_per_s"] = n / (t[k] / 1e3)
    out.update(
        fallback_fraction=float(fw.mean()),
        fallback_miss_rate=float((excess[kept] > 10 * net.cost_tol).mean()) if kept.any() else 0.0,
        fallback_miss_excess_max=float(excess[kept].max()) if kept.any() else 0.0,
        speedup_vs_plain_ref=t["plain_ref"] / t["warm"],
        speedup_vs_plain_loose=t["plain_loose"] / t["warm"],
        # names kept from the two-arm report: plain = the reference's stop rule
        plain_ms=t["plain_ref"], warm_ms=t["warm"], speedup=t["plain_ref"] / t["warm"],
        centre_dev_max_px=out["warm_centre_dev_max_px"],
    )
    return out


def evaluate(net: WarmStartNet, *, pages: int = 2, size: int = 2048, seed: int = 999, max_iter: int = 30,
             repeats: int = 3) -> dict:
    """compare_on_page over held-out synthetic pages, pooled (times summed, means cell-weighted,
    maxima over pages)."""
    rows = [compare_on_page(net, synth_page(seed * 7919 + k, size)[0], max_iter=max_iter, repeats=repeats)
            for k in range(pages)]
    n = sum(r["cells"] for r in rows)
    out = {"cells": n}
    arms = ("plain_ref", "plain_loose", "warm")
    means = [f"{k}_iterations_mean" for k in arms] + ["fallback_fraction", "fallback_miss_rate"] + [
        f"{k}_{q}" for k in arms[1:] for q in ("within_1e-3_px", "same_status")]
    for key in means:
        out[key] = sum(r[key] * r["cells"] for r in rows) / max(n, 1)
    for key in ["fallback_miss_excess_max"] + [f"{k}_centre_dev_max_px" for k in arms[1:]]:
        out[key] = max(r[key] for r in rows)
    for k in arms:
        out[f"{k}_ms"] = sum(r[f"{k}_ms"] for r in rows)
        out[f"{k}_cells_per_s"] = n / (out[f"{k}_ms"] / 1e3)
    out["speedup_vs_plain_ref"] = out["plain_ref_ms"] / out["warm_ms"]
    out["speedup_vs_plain_loose"] = out["plain_loose_ms"] / out["warm_ms"]
    return out


def bench_page() -> torch.Tensor:
    """The 8192 x 8192 staggered benchmark page (pitch 24, d 12, sigma 1.2, read noise 100)."""
    from .synthetic import page_staggered

    return dev.upload(page_staggered(0).image)


def main(argv=None):
    import argparse
    import json
    import time

    ap = argparse.ArgumentParser(prog="python -m imageprocessor_new_b200.warmstart")
    sub = ap.add_subparsers(dest="cmd", required=True)
    tr = sub.add_parser("train", help="build a synthetic training set on the GPU and train the MLP")
    tr.add_argument("--pages", type=int, default=200)
    tr.add_argument("--size", type=int, default=2048)
    tr.add_argument("--epochs", type=int, default=60)
    tr.add_argument("--batch", type=int, default=4096)
    tr.add_argument("--lr", type=float, default=2e-3)
    tr.add_argument("--seed", type=int, default=0)
    tr.add_argument("--out", default=str(DEFAULT_MODEL))
    tr.add_argument("--bench-page", action="store_true", help="also compare on the 8192 x 8192 benchmark page")
    ev = sub.add_parser("eval", help="plain vs warm-started initial fits on held-out pages")
    ev.add_argument("--model", default=str(DEFAULT_MODEL))
    ev.add_argument("--pages", type=int, default=2)
    ev.add_argument("--bench-page", action="store_true", help="also compare on the 8192 x 8192 benchmark page")
    args = ap.parse_args(argv)
    if args.cmd == "train":
        t0 = time.perf_counter()
        x, t = training_set(args.pages, size=args.size, seed=args.seed)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        print(f"training set: {x.shape[0]} cells from {args.pages} pages in {t1 - t0:.1f} s", flush=True)
        net = WarmStartNet(seed=args.seed)
        hist = train(net, x, t, epochs=args.epochs, batch=args.batch, lr=args.lr, seed=args.seed,
                     log=lambda m: print(m, flush=True))
        torch.cuda.synchronize()
        print(f"trained in {time.perf_counter() - t1:.1f} s; final loss {hist[-1]:.5f}", flush=True)
        net.save(args.out)
    else:
        net = WarmStartNet.load(args.model)
    print(json.dumps(evaluate(net, pages=2 if args.cmd == "train" else args.pages)), flush=True)
    if args.bench_page:
        print(json.dumps(compare_on_page(net, bench_page())), flush=True)


if __name__ == "__main__":
    main()
