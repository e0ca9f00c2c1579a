"""CUDA-graph capture of a whole ray-casting training step: BVH refit, colour pass, forward
launch, loss, backward launch and gradient assembly replayed as one graph.

Every engine call is stream-ordered, synchronisation-free and (after ``Engine.reserve`` /
the warm-up steps) allocation-free, so the step captures with ``torch.cuda.graph``.  The
captured step refits the LBVH built during warm-up (the reference's
``update_acceleration_structure``); call :meth:`GraphedStep.rebuild` after a change of the number
of Gaussians (densification) to rebuild and re-capture.

Usage::

    step = GraphedStep(params, views, target, loss="mse")
    for it in range(n):
        step.replay()            # grads in step.grads, loss in step.loss (device tensors)
        optimizer_step(params, step.grads)   # in-place updates of the same tensors

With ``tail=FusedTrainTail(...)`` over the same tensors, the Adam steps, the densification
statistics and the parameter clamps are captured too (one more kernel), and with
``activation=point_cloud_data`` the params are the trained tensors of the reference's point cloud:
``replay()`` is then a whole iteration of the reference loop (scripts/train.py:100-181, L1/SSIM loss
aside) without host synchronisation.
"""
from __future__ import annotations

import torch

from .batched import BatchedRenderFunction, BatchedViews
from .losses import views_l1_ssim_loss

_KEYS = ("positions", "scales", "quaternions", "densities", "color_features", "sph_gauss_features",
         "bandwidth_sharpness", "lobe_axis")


class GraphedStep:
    """Capture fwd+bwd of :class:`BatchedRenderFunction` over fixed parameter/target tensors.

    ``params`` are leaf tensors updated in place between replays (their storage must not change);
    ``target`` is the (R, 3) packed target of the views; ``loss`` is "mse", "l1" or "l1_ssim" (the
    reference's 0.8 L1 + 0.2 (1 - SSIM) per view image, averaged over the views).  Without
    ``activation`` the params are the render inputs (positions, scales, ...); with it they are the
    trained tensors and ``activation(params)`` gives the render inputs inside the graph (e.g.
    :func:`ray_gauss_b200.train_tail.point_cloud_data`), and ``grads`` are those of the trained tensors.
    ``tail`` (a :class:`ray_gauss_b200.train_tail.FusedTrainTail` over tensors of ``params``) and its
    ``min_scale`` are captured after the backward.
    """

    def __init__(self, params: dict, views: BatchedViews, target: torch.Tensor, loss: str = "mse",
                 warmup: int = 3, tail=None, min_scale: torch.Tensor | None = None, activation=None):
        self.activation = activation
        self.params = self._select(params)
        self.views = views
        self.target = target
        self.loss_kind = loss
        self.warmup = warmup
        self.graph = None
        self.loss = None
        self.grads = None
        self.tail = tail
        self.min_scale = min_scale
        self._capture()

    def _select(self, params):
        if self.activation is not None:
            return {k: v for k, v in params.items() if v is not None}
        return {k: params[k] for k in _KEYS if params.get(k) is not None}

    def _step(self):
        P = self.params
        X = P if self.activation is None else self.activation(P)
        out = BatchedRenderFunction.apply(*(X.get(k) for k in _KEYS), self.views)
        if self.loss_kind == "mse":
            loss = torch.nn.functional.mse_loss(out, self.target)
        elif self.loss_kind == "l1_ssim":
            loss = views_l1_ssim_loss(out, self.target, self.views)
        else:
            loss = torch.nn.functional.l1_loss(out, self.target)
        grads = torch.autograd.grad(loss, [P[k] for k in P], allow_unused=True)
        return loss.detach(), grads

    def _capture(self):
        for v in self.params.values():
            v.requires_grad_(True)
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            # warm-up builds the LBVH and sizes every scratch buffer outside the capture
            self.views.update = False
            for _ in range(self.warmup):
                self._step()
            self.views.update = True
            self._step()
        torch.cuda.current_stream().wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            loss, grads = self._step()
            if self.tail is not None:
                by_id = {id(v): g for v, g in zip(self.params.values(), grads)}
                missing = [k for k, v in self.tail.params.items() if id(v) not in by_id]
                if missing:
                    raise ValueError(f"tail tensors not among the step's parameters: {missing}")
                self.tail.capture({k: by_id[id(v)] for k, v in self.tail.params.items()}, self.min_scale)
        self.loss = loss
        self.grads = dict(zip(self.params.keys(), grads))

    def replay(self):
        if self.tail is not None:
            self.tail.prepare_replay()
        self.graph.replay()
        return self.loss

    def rebuild(self, params: dict | None = None, tail=None, min_scale: torch.Tensor | None = None):
        """Re-capture after the parameter tensors were replaced (e.g. densification): the warm-up
        rebuilds the LBVH for the new number of Gaussians.  ``tail`` / ``min_scale`` replace the
        captured tail and its lower scale clamp when given."""
        if params is not None:
            self.params = self._select(params)
        if tail is not None:
            self.tail = tail
        if min_scale is not None:
            self.min_scale = min_scale
        self.graph = None
        self._capture()
