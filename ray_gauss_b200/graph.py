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
"""
from __future__ import annotations

import torch

from .batched import BatchedRenderFunction, BatchedViews

_KEYS = ("positions", "scales", "quaternions", "densities", "color_features", "sph_gauss_features",
         "bandwidth_sharpness", "lobe_axis")


class GraphedStep:
    """Capture fwd+bwd of :class:`BatchedRenderFunction` over fixed parameter/target tensors.

    ``params`` are leaf tensors updated in place between replays (their storage must not change);
    ``target`` is the (R, 3) packed target of the views; ``loss`` is "mse" or "l1".
    """

    def __init__(self, params: dict, views: BatchedViews, target: torch.Tensor, loss: str = "mse",
                 warmup: int = 3):
        self.params = {k: params[k] for k in _KEYS if params.get(k) is not None}
        self.views = views
        self.target = target
        self.loss_kind = loss
        self.warmup = warmup
        self.graph = None
        self.loss = None
        self.grads = None
        self._capture()

    def _step(self):
        P = self.params
        out = BatchedRenderFunction.apply(*(P.get(k) for k in _KEYS), self.views)
        if self.loss_kind == "mse":
            loss = torch.nn.functional.mse_loss(out, self.target)
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
        self.loss = loss
        self.grads = dict(zip(self.params.keys(), grads))

    def replay(self):
        self.graph.replay()
        return self.loss

    def rebuild(self, params: dict | None = None):
        """Re-capture after the parameter tensors were replaced (e.g. densification)."""
        if params is not None:
            self.params = {k: params[k] for k in _KEYS if params.get(k) is not None}
        self.graph = None
        self._capture()
