"""Learned read scheduling for the SMEM path: a per-read cost model and the schedule it
drives (no counterpart in the reference; the reference runs reads in input order).

The exact SMEM kernel logs each read's work (hfm_sched.d_work_log: Occ touches, MemHits,
positions).  ReadCostModel is a 258 -> 128 -> 128 -> 3 MLP over 4-mer composition, the
share of ambiguous 4-mers and length that predicts log1p of those three counters; it is
trained on the GPU by the library's own forward / backward kernels (hfm_mlp_*).  LearnedSmem bins reads by
predicted cost (costliest first, warp-uniform runs of similar cost) and sends reads
predicted to report many MemHits straight to the warp-per-read kernel.  The schedule only
reorders work: results are byte-identical to the plain path for any model, which is its
fallback and its yardstick.

Device arrays are torch CUDA tensors (plumbing only; every kernel is the library's).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib as L

NPARAM = 128 * 272 + 128 + 128 * 128 + 128 + 3 * 128 + 3
IN_PAD = 272


def _torch():
    import torch
    return torch


def torch_ones_like(t):
    return _torch().ones_like(t)


def torch_expm1_sum(y) -> np.ndarray:
    """Sum over reads of expm1 of the log1p predictions -> float64[3] (host)."""
    torch = _torch()
    return torch.expm1(y.double().clamp(max=40.0)).clamp_min(0).sum(dim=0).cpu().numpy()


def work_targets(log) -> "torch.Tensor":
    """Work log rows (u32 touches, MemHits, positions, flags) -> float32 log1p targets [n, 3]."""
    torch = _torch()
    if isinstance(log, np.ndarray):
        log = torch.from_numpy(np.ascontiguousarray(log.astype(np.int64)))
    t = log[:, :3].to(torch.int64)
    t = torch.where(t < 0, t + (1 << 32), t)            # u32 stored in int32 tensors
    return torch.log1p(t.to(torch.float64)).to(torch.float32).contiguous()


class ReadCostModel:
    """Owns one hfm_mlp (weights and Adam state on `device`)."""

    def __init__(self, device: int = 0, seed: int = 0):
        self.device = device
        h = C.c_void_p()
        L.check(L.lib().hfm_mlp_create(device, seed, C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None) and self.h.value and L._lib is not None:
            L._lib.hfm_mlp_free(self.h)
            self.h = None

    # -- parameters --------------------------------------------------------------------
    def get_params(self) -> np.ndarray:
        p = np.zeros(NPARAM, dtype=np.float32)
        L.check(L.lib().hfm_mlp_get_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.shape == (NPARAM,)
        L.check(L.lib().hfm_mlp_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))))

    def save(self, path: str):
        np.save(path, self.get_params())

    def load(self, path: str):
        self.set_params(np.load(path))

    # -- kernels -------------------------------------------------------------------------
    def features(self, q_d, off_d, nq: int):
        """-> int16 tensor [nq, 272] holding BF16 bits."""
        torch = _torch()
        x = torch.empty((max(nq, 1), IN_PAD), dtype=torch.int16, device=q_d.device)
        L.check(L.lib().hfm_mlp_features(self.h, q_d.data_ptr(), off_d.data_ptr(), nq, x.data_ptr()))
        return x[:nq]

    def forward(self, x):
        torch = _torch()
        n = x.shape[0]
        y = torch.empty((max(n, 1), 3), dtype=torch.float32, device=x.device)
        L.check(L.lib().hfm_mlp_forward(self.h, x.data_ptr(), n, y.data_ptr()))
        return y[:n]

    def predict(self, q_d, off_d, nq: int, out=None):
        torch = _torch()
        y = out if out is not None else torch.empty((max(nq, 1), 3), dtype=torch.float32, device=q_d.device)
        L.check(L.lib().hfm_mlp_predict(self.h, q_d.data_ptr(), off_d.data_ptr(), nq, y.data_ptr()))
        return y[:nq]

    def grad(self, x, t):
        """-> (grad float32[NPARAM] numpy, loss) over all rows as one batch."""
        torch = _torch()
        g = torch.empty(NPARAM, dtype=torch.float32, device=x.device)
        loss = C.c_float()
        L.check(L.lib().hfm_mlp_grad(self.h, x.data_ptr(), t.data_ptr(), x.shape[0], g.data_ptr(), C.byref(loss)))
        return g.cpu().numpy(), loss.value

    def train(self, x, t, epochs: int = 4, batch: int = 8192, lr: float = 1e-3, seed: int = 0):
        """Adam over shuffled mini-batches; -> per-epoch training MSE."""
        losses = np.zeros(max(epochs, 1), dtype=np.float32)
        L.check(L.lib().hfm_mlp_train(self.h, x.data_ptr(), t.data_ptr(), x.shape[0], epochs, batch, lr, seed,
                                      losses.ctypes.data_as(C.POINTER(C.c_float))))
        return losses[:epochs]

    def init_output_bias(self, t):
        """Start the output biases at the targets' means (faster convergence)."""
        p = self.get_params()
        p[NPARAM - 3:] = t.mean(dim=0).cpu().numpy()
        self.set_params(p)

    def schedule(self, y, warp_min_hits: float = 0.0, order=None):
        """-> (order int32 tensor [nq] (a permutation), n_warp)."""
        torch = _torch()
        nq = y.shape[0]
        if order is None:
            order = torch.empty(max(nq, 1), dtype=torch.int32, device=y.device)
        nw = C.c_uint32()
        L.check(L.lib().hfm_mlp_schedule(self.h, y.data_ptr(), nq, warp_min_hits, order.data_ptr(), C.byref(nw)))
        return order[:nq], nw.value


@dataclass
class PredictionError:
    """Prediction quality on one read set (log1p space)."""
    mae: np.ndarray        # mean absolute error per output
    r2: np.ndarray         # coefficient of determination per output
    spearman_touches: float

    def as_dict(self):
        return {"mae_log1p": [round(float(v), 4) for v in self.mae], "r2": [round(float(v), 4) for v in self.r2],
                "spearman_touches": round(float(self.spearman_touches), 4)}


def prediction_error(y, t) -> PredictionError:
    y = y.detach().cpu().numpy().astype(np.float64) if hasattr(y, "detach") else np.asarray(y, np.float64)
    t = t.detach().cpu().numpy().astype(np.float64) if hasattr(t, "detach") else np.asarray(t, np.float64)
    mae = np.abs(y - t).mean(axis=0)
    var = t.var(axis=0)
    r2 = 1.0 - ((y - t) ** 2).mean(axis=0) / np.where(var > 0, var, 1.0)
    ry = np.argsort(np.argsort(y[:, 0])).astype(np.float64)
    rt = np.argsort(np.argsort(t[:, 0])).astype(np.float64)
    sp = float(np.corrcoef(ry, rt)[0, 1]) if len(ry) > 1 else 0.0
    return PredictionError(mae, r2, sp)


class LearnedSmem:
    """SMEM/MEM search on a BidirFmIndex handle with the learned schedule.

    fit(): run the exact kernel with its work log on training reads, train the model on
    the log.  run(): predict, bin, and search through hfm_mems_batch_device_sched."""

    def __init__(self, handle, device: int = 0, seed: int = 0, warp_min_hits: float = 0.0,
                 min_spearman: float = 0.3):
        self.handle = handle
        self.model = ReadCostModel(device, seed)
        self.warp_min_hits = warp_min_hits
        self.min_spearman = min_spearman
        self.enabled = True            # False: the model does not rank work; run the plain order
        self.holdout_error: Optional[PredictionError] = None
        self.calibration: Optional[dict] = None
        self._order = None
        self._y = None
        self.presize = True            # reserve pools and outputs from the predicted totals
        self.total_scale = np.ones(3)  # actual / predicted totals on the training reads
        self.margin = 1.15

    def log_work(self, q_d, off_d, nq, min_len, mode, bounds, max_hits):
        torch = _torch()
        log = torch.zeros(4 * max(nq, 1), dtype=torch.int32, device=q_d.device)
        sc = L.HfmSched(None, 0, 0, log.data_ptr())
        dm = L.HfmDevMems()
        rb = np.ascontiguousarray(bounds, dtype=np.uint32)
        L.check(L.lib().hfm_mems_batch_device_sched(self.handle.h, q_d.data_ptr(), off_d.data_ptr(), nq, min_len,
                                                    mode, L.ptr(rb, L.u32p) if len(rb) else None, len(rb),
                                                    max_hits, C.byref(sc), C.byref(dm)))
        return log[:4 * nq].view(nq, 4)

    def fit(self, q_d, off_d, nq, min_len, mode, bounds, max_hits, epochs=4, batch=8192, lr=1e-3, seed=0,
            holdout: float = 0.1, calibrate: bool = True, calibrate_all: bool = False):
        """Log the exact kernel's work on the training reads, train on the first
        (1 - holdout) of them (MSE of standardised targets; per-epoch losses are in those
        units), and evaluate the model on the rest: the learned order is used
        only when its predicted Occ touches rank the held-out reads' true touches with
        Spearman >= min_spearman and (calibrate) the learned order runs the held-out reads
        at least 2% faster than the plain order; otherwise run() keeps the plain order."""
        log = self.log_work(q_d, off_d, nq, min_len, mode, bounds, max_hits)
        t = work_targets(log).to(q_d.device)
        x = self.model.features(q_d, off_d, nq)
        ntr = nq - int(nq * holdout) if nq > 10 else nq
        # train on standardised targets, then fold the scale into the output layer
        mu = t[:ntr].mean(dim=0)
        sd = t[:ntr].std(dim=0).clamp_min(1e-3) if ntr > 1 else torch_ones_like(mu)
        tz = ((t - mu) / sd).contiguous()
        p = self.model.get_params()
        p[NPARAM - 3:] = 0.0
        self.model.set_params(p)
        losses = self.model.train(x[:ntr].contiguous(), tz[:ntr].contiguous(), epochs, batch, lr, seed)
        p = self.model.get_params()
        sd_h, mu_h = sd.cpu().numpy().astype(np.float32), mu.cpu().numpy().astype(np.float32)
        w3 = p[NPARAM - 3 - 3 * 128:NPARAM - 3].reshape(3, 128)
        w3 *= sd_h[:, None]
        p[NPARAM - 3:] = p[NPARAM - 3:] * sd_h + mu_h
        self.model.set_params(p)
        # totals: the model's summed predictions against the logged totals (pre-sizing)
        pred_tot = torch_expm1_sum(self.model.forward(x))
        true_tot = log[:, :3].to(_torch().int64).clamp_min(0).sum(dim=0).double().cpu().numpy()
        self.total_scale = np.where(pred_tot > 0, true_tot / np.maximum(pred_tot, 1e-9), 1.0)
        if ntr < nq:
            self.holdout_error = prediction_error(self.model.forward(x[ntr:].contiguous()), t[ntr:])
            self.enabled = self.holdout_error.spearman_touches >= self.min_spearman
            if self.enabled and calibrate:
                # the order's effect depends on the batch size (how many reads share a warp's
                # prefix, how long the queue's tail is): calibrate_all times it on every
                # training read, a batch the size of the one it will run on
                a = 0 if calibrate_all else ntr
                self.calibrate(q_d, off_d, a, nq, min_len, mode, bounds, max_hits)
        return losses, x, t

    def calibrate(self, q_d, off_d, a, b, min_len, mode, bounds, max_hits, reps=2):
        """Time the plain and the learned order on reads a..b (held out from training);
        keep the learned order only when it is at least 2% faster."""
        import time
        torch = _torch()
        base = int(off_d[a].item())
        q = q_d[base:int(off_d[b].item())]
        o = (off_d[a:b + 1] - base).contiguous()
        n = b - a
        rb = np.ascontiguousarray(bounds, dtype=np.uint32)
        bp = L.ptr(rb, L.u32p) if len(rb) else None

        def plain():
            dm = L.HfmDevMems()
            L.check(L.lib().hfm_mems_batch_device(self.handle.h, q.data_ptr(), o.data_ptr(), n, min_len, mode, bp,
                                                  len(rb), max_hits, C.byref(dm)))

        def learned():
            self.run(q, o, n, min_len, mode, bp, len(rb), max_hits)

        def best(f):
            ts = []
            for _ in range(reps + 1):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                f()
                torch.cuda.synchronize()
                ts.append(time.perf_counter() - t0)
            return min(ts[1:]) * 1e3

        self.enabled = True
        tp, tl = best(plain), best(learned)
        self.calibration = {"reads": n, "plain_ms": round(tp, 3), "learned_ms": round(tl, 3)}
        self.enabled = tl < 0.98 * tp

    def plan(self, q_d, off_d, nq):
        """Predict and bin: -> (order tensor, n_warp, predictions)."""
        torch = _torch()
        if self._y is None or self._y.shape[0] < nq:
            self._y = torch.empty((max(nq, 1), 3), dtype=torch.float32, device=q_d.device)
            self._order = torch.empty(max(nq, 1), dtype=torch.int32, device=q_d.device)
        y = self.model.predict(q_d, off_d, nq, out=self._y)
        order, nw = self.model.schedule(y, self.warp_min_hits, order=self._order)
        return order, nw, y

    def reserve_from(self, y, nq):
        """Pre-size the handle's pools and result arrays from the predicted totals (in place
        of a count pass); candidate intervals are reserved at 3 per predicted MemHit."""
        tot = torch_expm1_sum(y) * self.total_scale * self.margin
        hits = int(tot[1]) + nq
        L.check(L.lib().hfm_mems_reserve(self.handle.h, nq, 3 * hits + 4 * nq, hits, int(tot[2]) + nq))

    def run(self, q_d, off_d, nq, min_len, mode, bounds_ptr, n_bounds, max_hits) -> L.HfmDevMems:
        order, nw = None, 0
        if self.enabled or self.presize:
            order, nw, y = self.plan(q_d, off_d, nq)
            if self.presize and nq:
                self.reserve_from(y, nq)
        if self.enabled:
            sc = L.HfmSched(order.data_ptr() if nq else None, nw, 0, None)
        else:
            sc = L.HfmSched(None, 0, 0, None)
        dm = L.HfmDevMems()
        L.check(L.lib().hfm_mems_batch_device_sched(self.handle.h, q_d.data_ptr(), off_d.data_ptr(), nq, min_len,
                                                    mode, bounds_ptr, n_bounds, max_hits, C.byref(sc),
                                                    C.byref(dm)))
        return dm
