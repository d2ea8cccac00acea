"""Learned hypothesis proposal for batched RANSAC plane fitting.

A per-point MLP scores how likely each point lies on the plane that plain
RANSAC picks, from eight features of its 16 nearest neighbours; RANSAC then
draws its three points with probability proportional to the score, and the
exact inlier count over all points still decides (uniform sampling, the
plain rand() stream, stays available as rvp_ransac_frames).

Everything runs on the GPU through the C ABI (rvpoint_b200/csrc/learned.cu):
features, training (forward, backward, Adam), inference and the weighted
RANSAC. Device buffers are torch tensors, used only as memory.

    scorer = PlaneScorer(max_points, max_frames)
    train(scorer, train_batch)                 # labels from plain RANSAC
    lr = LearnedRansac(scorer)
    models, best, iters = lr.run(batch_dev)    # weighted RANSAC
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import check
from .api import Context, default_context

FEATURES = ("abs_nx", "abs_ny", "abs_nz", "curvature", "planarity", "log_r16",
            "plane_offset_over_r", "centroid_offset_over_r")


def _p(t: Optional[torch.Tensor]):
    return None if t is None else C.c_void_p(t.data_ptr())


@dataclass
class DeviceBatch:
    """Frames stored back to back in device memory (SoA float32)."""
    x: torch.Tensor
    y: torch.Tensor
    z: torch.Tensor
    offsets: torch.Tensor          # int64, n_frames + 1, device
    offsets_host: np.ndarray       # the same on the host

    @property
    def n_frames(self) -> int:
        return int(self.offsets_host.shape[0] - 1)

    @property
    def n(self) -> int:
        return int(self.offsets_host[-1])

    @staticmethod
    def from_host(batch, device: int = 0) -> "DeviceBatch":
        dev = torch.device("cuda", device)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        return DeviceBatch(t(batch.x), t(batch.y), t(batch.z),
                           t(np.asarray(batch.offsets, np.int64)),
                           np.asarray(batch.offsets, np.int64).copy())


def candidates(offsets_host: np.ndarray, per_frame: int, seed: int):
    """A uniform random subset of each frame's points (all of a frame with
    fewer), sorted; returns (cand uint32, cand_offsets int64) on the host."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out, offs = [], [0]
    for f in range(offsets_host.shape[0] - 1):
        a, b = int(offsets_host[f]), int(offsets_host[f + 1])
        n = b - a
        if n <= per_frame:
            sel = np.arange(a, b)
        else:
            sel = a + np.sort(rng.choice(n, per_frame, replace=False))
        out.append(sel.astype(np.uint32))
        offs.append(offs[-1] + sel.shape[0])
    return np.concatenate(out), np.asarray(offs, np.int64)


def proposal_features(scorer: "PlaneScorer", b: DeviceBatch, cand: torch.Tensor,
                      cand_offsets: torch.Tensor, cell: float, scope: str) -> torch.Tensor:
    """Features of the candidates. scope "points": neighbours among all of
    the frame's points; "candidates": among the frame's candidates only (a
    coarser neighbourhood, far less kNN work)."""
    if scope not in ("points", "candidates"):
        raise ValueError(scope)
    return scorer.features(b, cell, cand, cand_offsets, scope == "candidates")


class PlaneScorer:
    """Features + MLP (rvp_scorer)."""

    def __init__(self, max_points: int, max_frames: int, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.L = _lib.load()
        h = C.c_void_p()
        check(self.L.rvp_scorer_create(self.ctx.h, int(max_points), int(max_frames),
                                       C.byref(h)), self.ctx.h)
        self.h = h
        self.mean = np.zeros(8, np.float32)
        self.std = np.ones(8, np.float32)

    def features(self, b: DeviceBatch, cell: float, cand: Optional[torch.Tensor] = None,
                 cand_offsets: Optional[torch.Tensor] = None, among_candidates: bool = False):
        self.ctx.use_torch_stream()
        n_cand = b.n if cand is None else int(cand.numel())
        feat = torch.empty((n_cand, 8), dtype=torch.float32, device=b.x.device)
        check(self.L.rvp_scorer_features(self.h, _p(b.x), _p(b.y), _p(b.z), _p(b.offsets),
                                         b.n_frames, b.n, float(cell), _p(cand),
                                         _p(cand_offsets), n_cand, int(among_candidates),
                                         _p(feat)), self.ctx.h)
        return feat

    def set_knn(self, queries_per_warp: int, rfac: float = 1.0) -> None:
        """kNN kernels of the features among candidates: 0 one query per
        lane, 3 a cooperative first pass (rvp_scorer_set_knn)."""
        check(self.L.rvp_scorer_set_knn(self.h, int(queries_per_warp), float(rfac)), self.ctx.h)

    def set_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, np.float32)
        assert p.shape == (_lib.MLP_PARAMS,)
        check(self.L.rvp_mlp_set_params(self.h, p.ctypes.data_as(C.c_void_p)), self.ctx.h)

    def get_params(self) -> np.ndarray:
        p = np.empty(_lib.MLP_PARAMS, np.float32)
        check(self.L.rvp_mlp_get_params(self.h, p.ctypes.data_as(C.c_void_p)), self.ctx.h)
        return p

    def set_norm(self, mean, std) -> None:
        self.mean = np.ascontiguousarray(mean, np.float32)
        self.std = np.ascontiguousarray(std, np.float32)
        check(self.L.rvp_mlp_set_norm(self.h, self.mean.ctypes.data_as(C.c_void_p),
                                      self.std.ctypes.data_as(C.c_void_p)), self.ctx.h)

    def forward(self, feat: torch.Tensor) -> torch.Tensor:
        self.ctx.use_torch_stream()
        out = torch.empty(feat.shape[0], dtype=torch.float32, device=feat.device)
        check(self.L.rvp_mlp_forward(self.h, _p(feat), int(feat.shape[0]), _p(out)), self.ctx.h)
        return out

    def gradients(self, feat: torch.Tensor, labels: torch.Tensor):
        self.ctx.use_torch_stream()
        g = np.empty(_lib.MLP_PARAMS, np.float32)
        loss = C.c_double(0.0)
        check(self.L.rvp_mlp_gradients(self.h, _p(feat), _p(labels), int(feat.shape[0]),
                                       g.ctypes.data_as(C.c_void_p), C.byref(loss)), self.ctx.h)
        return float(loss.value), g

    def train_step(self, feat: torch.Tensor, labels: torch.Tensor, lr: float,
                   want_loss: bool = False, batch: int = 0, seed: int = 1):
        """One Adam step over all rows, or over a minibatch of `batch` rows
        drawn on the device."""
        self.ctx.use_torch_stream()
        loss = C.c_double(0.0)
        check(self.L.rvp_mlp_train_step(self.h, _p(feat), _p(labels), int(feat.shape[0]),
                                        int(batch), int(seed), float(lr),
                                        C.byref(loss) if want_loss else None), self.ctx.h)
        return float(loss.value) if want_loss else None

    def close(self):
        if getattr(self, "h", None):
            self.L.rvp_scorer_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


def ransac_frames(b: DeviceBatch, max_iters: int, thresh: float, collinear: float = 1e-6,
                  probability: float = 0.99, targets: Optional[torch.Tensor] = None,
                  ctx: Optional[Context] = None):
    """Plain RANSAC (the reference's rand() stream) on every frame."""
    ctx = ctx or default_context()
    ctx.use_torch_stream()
    dev = b.x.device
    nf = b.n_frames
    models = torch.empty((nf, 4), dtype=torch.float32, device=dev)
    best = torch.empty(nf, dtype=torch.int32, device=dev)
    iters = torch.empty(nf, dtype=torch.int32, device=dev)
    check(_lib.load().rvp_ransac_frames(ctx.h, _p(b.x), _p(b.y), _p(b.z), _p(b.offsets), nf,
                                        int(max_iters), float(thresh), float(collinear),
                                        float(probability), _p(targets), _p(models), _p(best),
                                        _p(iters)), ctx.h)
    return models, best, iters


def ransac_weighted(b: DeviceBatch, cand: torch.Tensor, cand_offsets: torch.Tensor,
                    weights: torch.Tensor, max_iters: int, thresh: float, seed: int = 1,
                    logit_power: float = 0.0, collinear: float = 1e-6,
                    probability: float = 0.99, targets: Optional[torch.Tensor] = None,
                    ctx: Optional[Context] = None):
    ctx = ctx or default_context()
    ctx.use_torch_stream()
    dev = b.x.device
    nf = b.n_frames
    models = torch.empty((nf, 4), dtype=torch.float32, device=dev)
    best = torch.empty(nf, dtype=torch.int32, device=dev)
    iters = torch.empty(nf, dtype=torch.int32, device=dev)
    check(_lib.load().rvp_ransac_weighted(ctx.h, _p(b.x), _p(b.y), _p(b.z), _p(b.offsets), nf,
                                          _p(cand), _p(cand_offsets), int(cand.numel()),
                                          _p(weights),
                                          float(logit_power), int(seed), int(max_iters),
                                          float(thresh), float(collinear), float(probability),
                                          _p(targets), _p(models), _p(best), _p(iters)), ctx.h)
    return models, best, iters


PREEMPT_GROWTH = 2  # rvp_ransac_preemptive: later rounds draw (and count) this many times more


def preemptive_rounds(max_iters: int, draws: int) -> int:
    """Rounds of rvp_ransac_preemptive whose hypotheses first reach max_iters."""
    rest = max(0, max_iters - draws)
    step = PREEMPT_GROWTH * draws
    return 1 + (rest + step - 1) // step


def ransac_preemptive(b: DeviceBatch, cand: torch.Tensor, cand_offsets: torch.Tensor,
                      weights: torch.Tensor, thresh: float, draws: int = 256,
                      max_rounds: int = 40, seed: int = 1, logit_power: float = 0.0,
                      collinear: float = 1e-6, targets: Optional[torch.Tensor] = None,
                      ctx: Optional[Context] = None):
    """Weighted proposal in preemptive rounds (rvp_ransac_preemptive: the
    first round draws `draws` hypotheses, each later one PREEMPT_GROWTH times
    as many): returns (models, best, hypotheses drawn per frame)."""
    ctx = ctx or default_context()
    ctx.use_torch_stream()
    dev = b.x.device
    nf = b.n_frames
    models = torch.empty((nf, 4), dtype=torch.float32, device=dev)
    best = torch.empty(nf, dtype=torch.int32, device=dev)
    drawn = torch.empty(nf, dtype=torch.int32, device=dev)
    check(_lib.load().rvp_ransac_preemptive(ctx.h, _p(b.x), _p(b.y), _p(b.z), _p(b.offsets), nf,
                                            _p(cand), _p(cand_offsets), int(cand.numel()),
                                            _p(weights), float(logit_power), int(seed),
                                            int(draws), int(max_rounds), float(thresh),
                                            float(collinear), _p(targets), _p(models), _p(best),
                                            _p(drawn)), ctx.h)
    return models, best, drawn


def plane_labels(b: DeviceBatch, models: torch.Tensor, thresh: float,
                 ctx: Optional[Context] = None) -> torch.Tensor:
    ctx = ctx or default_context()
    ctx.use_torch_stream()
    labels = torch.empty(b.n, dtype=torch.float32, device=b.x.device)
    check(_lib.load().rvp_plane_labels(ctx.h, _p(b.x), _p(b.y), _p(b.z), _p(b.offsets),
                                       b.n_frames, b.n, _p(models), float(thresh), _p(labels)),
          ctx.h)
    return labels


@dataclass
class TrainConfig:
    thresh: float = 0.02          # RANSAC inlier distance (m)
    label_iters: int = 10_000     # plain RANSAC hypotheses behind the labels
    cell: float = 2.5             # grid cell of the feature kNN (m; speed only)
    cand_per_frame: int = 1024    # feature points per frame
    scope: str = "candidates"     # feature neighbourhoods: "candidates" or "points"
    steps: int = 400
    batch: int = 32_768
    lr: float = 3e-3
    seed: int = 7
    log: list = field(default_factory=list)


def train(scorer: PlaneScorer, b: DeviceBatch, cfg: TrainConfig = TrainConfig()) -> dict:
    """Labels from plain RANSAC on b, then Adam on the GPU. Returns a summary."""
    t0 = time.perf_counter()
    models, best, _ = ransac_frames(b, cfg.label_iters, cfg.thresh)
    labels_all = plane_labels(b, models, cfg.thresh)
    cand_h, coffs_h = candidates(b.offsets_host, cfg.cand_per_frame, cfg.seed)
    cand = torch.from_numpy(cand_h.view(np.int32)).to(b.x.device)
    coffs = torch.from_numpy(coffs_h).to(b.x.device)
    feat = proposal_features(scorer, b, cand, coffs, cfg.cell, cfg.scope)
    labels = labels_all[cand.long()].contiguous()
    mean = feat.mean(0).cpu().numpy()
    std = feat.std(0).clamp_min(1e-6).cpu().numpy()
    scorer.set_norm(mean, std)
    n = feat.shape[0]
    losses = []
    for step in range(cfg.steps):
        want = step % 50 == 0 or step == cfg.steps - 1
        l_ = scorer.train_step(feat, labels, cfg.lr, want_loss=want,
                               batch=min(cfg.batch, n), seed=cfg.seed)
        if want:
            losses.append((step, l_))
    torch.cuda.synchronize()
    return {"losses": losses, "seconds": time.perf_counter() - t0,
            "positive_fraction": float(labels.mean().item()), "points": int(n)}


class LearnedRansac:
    """features -> MLP -> weighted RANSAC over every frame of a batch."""

    def __init__(self, scorer: PlaneScorer, cell: float = 2.5, cand_per_frame: int = 1024,
                 logit_power: float = 1.0, seed: int = 11, scope: str = "candidates",
                 preemptive: bool = True, draws: int = 512):
        """preemptive: hypotheses ranked among the candidates first, the best
        32 of every `draws` counted exactly (else every hypothesis is counted
        exactly, 32 at a time)."""
        self.preemptive = preemptive
        self.draws = draws
        self.scorer = scorer
        self.cell = cell
        self.cand_per_frame = cand_per_frame
        self.logit_power = logit_power
        self.seed = seed
        self.scope = scope

    def prepare(self, b: DeviceBatch):
        """The candidate subset of every frame (host-side draw, uploaded)."""
        cand_h, coffs_h = candidates(b.offsets_host, self.cand_per_frame, self.seed)
        dev = b.x.device
        self._coffs_h = coffs_h
        return (torch.from_numpy(cand_h.view(np.int32)).to(dev),
                torch.from_numpy(coffs_h).to(dev))

    def run(self, b: DeviceBatch, cand, cand_offsets, max_iters: int, thresh: float,
            targets: Optional[torch.Tensor] = None):
        feat = proposal_features(self.scorer, b, cand, cand_offsets, self.cell, self.scope)
        logits = self.scorer.forward(feat)
        return self.ransac(b, cand, cand_offsets, logits, max_iters, thresh, targets)

    def ransac(self, b: DeviceBatch, cand, cand_offsets, logits, max_iters: int, thresh: float,
               targets: Optional[torch.Tensor] = None):
        if self.preemptive:
            rounds = preemptive_rounds(max_iters, self.draws)
            return ransac_preemptive(b, cand, cand_offsets, logits, thresh, draws=self.draws,
                                     max_rounds=rounds, seed=self.seed,
                                     logit_power=self.logit_power, targets=targets,
                                     ctx=self.scorer.ctx)
        return ransac_weighted(b, cand, cand_offsets, logits, max_iters, thresh,
                               seed=self.seed, logit_power=self.logit_power, targets=targets,
                               ctx=self.scorer.ctx)
