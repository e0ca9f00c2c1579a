"""Fused training-step tail: the reference's optimizer managers and parameter clamps in one launch.

The reference training loop (scripts/train.py:121-181) ends every iteration with
  - the densification statistics of the position gradient (classes/point_cloud.py:633-640),
  - one ``torch.optim.Adam`` step per parameter tensor, each with its own learning-rate schedule,
    ``donotuse_steps`` warm-up and ``eps=1e-15`` (classes/optimizer.py:4-21, 203-231),
  - ``densities[densities < 0] = 0``, quaternion (and optionally lobe-axis) normalisation and the
    log-scale clamp to ``[filter_3D, max_scale]``.
:class:`FusedTrainTail` keeps the Adam moments and schedules of those tensors on the host side and
runs all of it as one kernel (``rg_train_tail_step``), stream-ordered and without host
synchronisation, so it can sit inside the captured step (:class:`ray_gauss_b200.graph.GraphedStep`).
:func:`point_cloud_data` is the reference's ``PointCloud.get_data``: the activations between the
trained tensors and the render inputs.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import torch

from . import _lib
from ._lib import check

RAW_NAMES = ("positions", "scales", "quaternions", "densities", "rgb", "spherical_harmonics", "sph_gauss_features",
             "bandwidth_sharpness", "lobe_axis")


def point_cloud_data(raw: dict, normalized_quaternion: bool = True, normalized_lobe_axis: bool = True) -> dict:
    """Render inputs from the raw trained tensors, as the reference's ``PointCloud.get_data``
    (classes/point_cloud.py:689-739): positions and densities as stored, ``exp(scales)``, quaternions
    divided by their norm when asked, colour features ``cat(rgb[:, :, None], spherical_harmonics)``,
    SG features as stored, ``softplus(bandwidth_sharpness)``, lobe axes divided by their norm when
    asked.  ``raw`` uses the reference's attribute names (:data:`RAW_NAMES`).  Built from torch ops
    without host synchronisation, so it captures in a CUDA graph; a zero lobe axis is rendered as
    (0, 0, 1) without rewriting the stored tensor (the reference overwrites it in place)."""
    q = raw["quaternions"]
    if normalized_quaternion:
        q = q / torch.norm(q, dim=1)[:, None]
    ax = raw["lobe_axis"]
    if normalized_lobe_axis and ax.numel():
        ez = (torch.arange(3, device=ax.device) == 2).to(ax.dtype)   # (0, 0, 1) without a host copy
        ax = torch.where((torch.norm(ax, dim=2) == 0)[:, :, None], ez, ax)
        ax = ax / torch.norm(ax, dim=2)[:, :, None]
    return {"positions": raw["positions"], "scales": torch.exp(raw["scales"]), "quaternions": q,
            "densities": raw["densities"],
            "color_features": torch.cat([raw["rgb"][:, :, None], raw["spherical_harmonics"]], dim=2),
            "sph_gauss_features": raw["sph_gauss_features"],
            "bandwidth_sharpness": torch.nn.functional.softplus(raw["bandwidth_sharpness"]),
            "lobe_axis": ax}


def raw_from_render_inputs(p: dict) -> dict:
    """Raw tensors whose :func:`point_cloud_data` gives the render inputs ``p`` (log scales, colour
    features split into rgb and SH, inverse softplus of the SG bandwidths)."""
    bw = p["bandwidth_sharpness"]
    return {"positions": p["positions"].clone(), "scales": torch.log(p["scales"]),
            "quaternions": p["quaternions"].clone(), "densities": p["densities"].clone(),
            "rgb": p["color_features"][:, :, 0].contiguous(),
            "spherical_harmonics": p["color_features"][:, :, 1:].contiguous(),
            "sph_gauss_features": p["sph_gauss_features"].clone(),
            "bandwidth_sharpness": bw + torch.log(-torch.expm1(-bw)),
            "lobe_axis": p["lobe_axis"].clone()}


@dataclass
class LrSchedule:
    """One tensor's learning rate, as an OptimizerManager (classes/optimizer.py:4-21, 203-231):
    ``gamma`` multiplies the rate after each optimizer step taken at manager step s with
    ``delay <= s < delay + decay`` (ExponentialLR); the first ``donotuse`` manager steps skip the
    optimizer entirely."""
    lr: float
    gamma: float = 1.0
    delay: int = 0
    decay: int = 0
    donotuse: int = 0

    @staticmethod
    def exponential(init_lr, final_lr, decay, delay=0, donotuse=0):
        """init_ExponentialLR without an explicit gamma: gamma = (final / init)^(1 / decay)."""
        return LrSchedule(init_lr, (final_lr / init_lr) ** (1.0 / decay), delay, decay, donotuse)


def unlock_spherical_harmonics(tail: "FusedTrainTail", n_sh: int, name: str = "spherical_harmonics"):
    """``PointCloud.unlock_spherical_harmonics`` (classes/point_cloud.py:518-528): grow the SH
    coefficients to ``n_sh`` per channel (the DC term lives in rgb) with zeros."""
    p = tail.params[name]
    add = n_sh - p.shape[2] - 1
    if add <= 0:
        return p
    return tail.extend(name, torch.zeros((p.shape[0], 3, add), dtype=p.dtype, device=p.device), dim=2)


def unlock_spherical_gaussians(tail: "FusedTrainTail", n_sph_gauss: int, generator: torch.Generator | None = None):
    """``PointCloud.unlock_spherical_gaussians`` (classes/point_cloud.py:530-545): add
    ``n_sph_gauss`` lobes with zero amplitudes and bandwidths and random (unnormalised, standard
    normal) axes.  The tail must hold ``sph_gauss_features``, ``bandwidth_sharpness`` and
    ``lobe_axis`` (zero-width tensors before the first unlock)."""
    n = tail.n
    dev = tail.params["sph_gauss_features"].device
    tail.extend("sph_gauss_features", torch.zeros((n, 3, n_sph_gauss), device=dev), dim=2)
    tail.extend("bandwidth_sharpness", torch.zeros((n, n_sph_gauss), device=dev), dim=1)
    axes = torch.randn((n, n_sph_gauss, 3), device=dev, generator=generator)
    tail.extend("lobe_axis", axes, dim=1)


def reset_density(tail: "FusedTrainTail", max_density: float = 4.0, name: str = "densities"):
    """``PointCloud.reset_density`` (classes/point_cloud.py:1145-1149): densities clamped to at most
    ``max_density``, their Adam moments zeroed."""
    d = tail.params[name].detach()
    return tail.replace(name, torch.min(d, torch.ones_like(d) * max_density))


# configuration sections of the reference's optimisation config (utils/optim_utils.py:4-82) -> the
# trained tensors they drive
CONFIG_SECTIONS = {"position": "positions", "rgb": "rgb", "sh": "spherical_harmonics", "density": "densities",
                   "scale": "scales", "quaternion": "quaternions", "sph_gauss_features": "sph_gauss_features",
                   "bandwidth_sharpness": "bandwidth_sharpness", "lobe_axis": "lobe_axis"}


def _cfg(c, key, default=None):
    if isinstance(c, dict):
        return c.get(key, default)
    return getattr(c, key, default)


def schedules_from_config(config_opti) -> dict:
    """The learning-rate schedules of ``define_optimizer_manager`` (utils/optim_utils.py:4-82,
    classes/optimizer.py:203-218) from the reference's ``training.optimization`` config (a dict,
    OmegaConf node or namespace with one section per tensor): ``scheduler: true`` gives an
    exponential schedule with the section's ``gamma`` or ``(final_lr / init_lr)^(1 / decay_step)``
    over ``[delay_step, delay_step + decay_step)``; otherwise a constant ``init_lr``.  Every section's
    ``donotuse_steps`` carries over.  Keys are the trained tensors' names."""
    out = {}
    for section, name in CONFIG_SECTIONS.items():
        c = _cfg(config_opti, section)
        if c is None:
            continue
        donotuse = int(_cfg(c, "donotuse_steps", 0) or 0)
        init = float(_cfg(c, "init_lr"))
        if _cfg(c, "scheduler", False):
            decay, delay = int(_cfg(c, "decay_step")), int(_cfg(c, "delay_step"))
            gamma = _cfg(c, "gamma")
            gamma = float(gamma) if gamma is not None else (float(_cfg(c, "final_lr")) / init) ** (1 / decay)
            out[name] = LrSchedule(init, gamma, delay, decay, donotuse)
        else:
            out[name] = LrSchedule(init, donotuse=donotuse)
    return out


class FusedTrainTail:
    """Adam + statistics + clamps over the Gaussians' raw parameter tensors.

    ``params`` maps names to leaf tensors of shape (N, ...) (FP32, contiguous, on one GPU), e.g. the
    reference's ``positions, rgb, spherical_harmonics, densities, scales, quaternions,
    sph_gauss_features, bandwidth_sharpness, lobe_axis``; ``schedules`` gives each its
    :class:`LrSchedule`.  Names in ``roles`` (positions, densities, scales, quaternions, lobe_axis)
    select the tensors that the statistics and the clamps apply to.  ``step()`` reads ``p.grad`` (a
    tensor without a gradient is left as it is, like torch's Adam)."""

    ROLES = ("positions", "densities", "scales", "quaternions", "lobe_axis")

    def __init__(self, params: dict, schedules: dict, roles: dict | None = None, betas=(0.9, 0.999), eps=1e-15,
                 normalize_quaternion=True, normalize_lobe_axis=False, max_scale=math.inf, statistics=True):
        if len(params) > _lib.RG_TAIL_MAX_TENSORS:
            raise ValueError(f"at most {_lib.RG_TAIL_MAX_TENSORS} tensors")
        self.names = list(params)
        self.params = params
        n = {int(p.shape[0]) for p in params.values()}
        if len(n) != 1:
            raise ValueError("all tensors need the same number of Gaussians")
        self.n = n.pop()
        dev = next(iter(params.values())).device
        for k, p in params.items():
            if p.dtype != torch.float32 or not p.is_contiguous() or p.device != dev:
                raise ValueError(f"{k}: FP32 contiguous tensors on one device")
        self.schedules = {k: LrSchedule(**vars(schedules[k])) for k in self.names}
        self.lr = {k: float(self.schedules[k].lr) for k in self.names}
        self.manager_step = {k: 0 for k in self.names}
        self.adam_step = {k: 0 for k in self.names}
        self.exp_avg = {k: torch.zeros_like(p) for k, p in params.items()}
        self.exp_avg_sq = {k: torch.zeros_like(p) for k, p in params.items()}
        self.betas, self.eps = betas, eps
        self.roles = dict(roles or {})
        for r in self.roles:
            if r not in self.ROLES or self.roles[r] not in params:
                raise ValueError(f"unknown role or tensor: {r} -> {self.roles[r]}")
        self.normalize_quaternion, self.normalize_lobe_axis = normalize_quaternion, normalize_lobe_axis
        self.max_scale = float(max_scale)
        self.stats = None
        if statistics and "positions" in self.roles:
            z = lambda: torch.zeros(self.n, dtype=torch.float32, device=dev)  # noqa: E731
            self.stats = {"xyz_gradient_accum_norm": z(), "num_accum": z(), "num_accum_gnv": z()}
        self.lib = _lib.load()
        # device scalars of the CUDA-graph form (allocated here: nothing may allocate inside a capture)
        self._dev_scalars = torch.zeros((len(self.names), 4), dtype=torch.float32, device=dev)
        self._host_scalars = None
        self._graph_grads = None
        self._grad_copies = []

    def current_lrs(self) -> dict:
        return dict(self.lr)

    def rebind(self, params: dict, exp_avg: dict, exp_avg_sq: dict, stats: dict | None):
        """Point the tail at new tensors of the same names (after densification changed N): the
        learning rates, manager and Adam step counters carry over, like the reference's optimizers
        whose state is pruned and concatenated in place (classes/optimizer.py:54-83).  A captured
        graph must be re-captured (``GraphedStep.rebuild``)."""
        if list(params) != self.names:
            raise ValueError("rebind needs the same tensor names")
        n = {int(p.shape[0]) for p in params.values()}
        if len(n) != 1:
            raise ValueError("all tensors need the same number of Gaussians")
        self.params, self.exp_avg, self.exp_avg_sq = params, exp_avg, exp_avg_sq
        self.n = n.pop()
        if self.stats is not None:
            self.stats = stats
        self._graph_grads = None
        self._grad_copies = []

    def extend(self, name: str, extension: torch.Tensor, dim: int) -> torch.Tensor:
        """``_cat_tensor`` (classes/optimizer.py:71-83): append ``extension`` to tensor ``name``
        along ``dim`` (e.g. newly unlocked SH coefficients); the Adam moments grow by zeros, the step
        count and learning rate stay.  Returns the new tensor (a captured graph must be re-captured)."""
        p = self.params[name]
        ext = extension.to(device=p.device, dtype=p.dtype)
        newp = torch.cat((p.detach(), ext), dim=dim).contiguous().requires_grad_(p.requires_grad)
        m = torch.cat((self.exp_avg[name], torch.zeros_like(ext)), dim=dim).contiguous()
        v = torch.cat((self.exp_avg_sq[name], torch.zeros_like(ext)), dim=dim).contiguous()
        params = dict(self.params)
        params[name] = newp
        exp_avg, exp_avg_sq = dict(self.exp_avg), dict(self.exp_avg_sq)
        exp_avg[name], exp_avg_sq[name] = m, v
        self.rebind(params, exp_avg, exp_avg_sq, self.stats)
        return newp

    def replace(self, name: str, values: torch.Tensor) -> torch.Tensor:
        """``_replace`` (classes/optimizer.py:97-106): new values for tensor ``name`` with zero Adam
        moments; the step count and learning rate stay."""
        p = self.params[name]
        newp = values.detach().to(device=p.device, dtype=p.dtype).contiguous().requires_grad_(p.requires_grad)
        if newp.shape != p.shape:
            raise ValueError("replace keeps the shape; use extend or densification to change it")
        params = dict(self.params)
        params[name] = newp
        exp_avg, exp_avg_sq = dict(self.exp_avg), dict(self.exp_avg_sq)
        exp_avg[name], exp_avg_sq[name] = torch.zeros_like(newp), torch.zeros_like(newp)
        self.rebind(params, exp_avg, exp_avg_sq, self.stats)
        return newp

    # ---- per-step host scalars (the optimizer managers' step logic) ----
    def _plan(self, has_grad) -> list:
        """(name, use, lr, bias1, bias2_sqrt) of this step for every tensor; advances the counters:
        a manager past its ``donotuse`` steps steps Adam when the tensor has a gradient (torch's Adam
        counts its steps per parameter with a gradient) and steps its scheduler in
        ``[delay, delay + decay)`` either way (classes/optimizer.py:13-21)."""
        b1, b2 = self.betas
        plan = []
        for k in self.names:
            sched = self.schedules[k]
            s = self.manager_step[k]
            past = s >= sched.donotuse
            use = past and has_grad(k)
            if use:
                self.adam_step[k] += 1
                t = self.adam_step[k]
                plan.append((k, True, self.lr[k], 1.0 - b1 ** t, math.sqrt(1.0 - b2 ** t)))
            else:
                plan.append((k, False, self.lr[k], 1.0, 1.0))
            if past and sched.delay <= s < sched.delay + sched.decay:
                self.lr[k] *= sched.gamma
            self.manager_step[k] = s + 1
        return plan

    def _args(self, grads: dict, min_scale, may_step) -> "_lib.rg_train_tail":
        self._grad_copies = []                     # kept alive until the next launch is built
        d = _lib.rg_train_tail()
        d.n = self.n
        d.n_tensors = len(self.names)
        for r in self.ROLES:
            setattr(d, "idx_" + r, self.names.index(self.roles[r]) if r in self.roles else -1)
        d.normalize_quaternions = int(bool(self.normalize_quaternion))
        d.normalize_lobe_axis = int(bool(self.normalize_lobe_axis))
        d.max_scale = self.max_scale
        d.min_scale = min_scale.data_ptr() if min_scale is not None else None
        if self.stats is not None:
            d.grad_norm_accum = self.stats["xyz_gradient_accum_norm"].data_ptr()
            d.num_accum = self.stats["num_accum"].data_ptr()
            d.num_accum_gnv = self.stats["num_accum_gnv"].data_ptr()
        b1, b2 = self.betas
        for i, k in enumerate(self.names):
            p, g = self.params[k], grads.get(k)
            t = d.tensors[i]
            t.param = p.data_ptr()
            t.width = int(p.numel() // max(1, self.n))
            if g is not None:
                if g.dtype != torch.float32 or g.shape != p.shape:
                    raise ValueError(f"{k}: gradient must be FP32 and shaped like the tensor")
                if not g.is_contiguous():          # e.g. rgb's slice of the colour-feature gradient
                    g = g.contiguous()
                    self._grad_copies.append(g)
                t.grad = g.data_ptr()
            t.active = int(bool(may_step(k)) and g is not None and t.width > 0)
            t.exp_avg = self.exp_avg[k].data_ptr()
            t.exp_avg_sq = self.exp_avg_sq[k].data_ptr()
            t.beta1, t.beta2, t.eps = b1, b2, self.eps
            t.one_minus_beta1, t.one_minus_beta2 = 1.0 - b1, 1.0 - b2
        return d

    def _min_scale(self, min_scale):
        if min_scale is None:
            return None
        m = min_scale.reshape(-1)
        if m.dtype != torch.float32 or not m.is_contiguous() or m.numel() != self.n:
            raise ValueError("min_scale: (N,) or (N, 1) FP32 contiguous")
        return m

    def _launch(self, d):
        dev = self.params[self.names[0]].device
        if dev.type != "cuda":
            raise ValueError("the fused tail runs on CUDA tensors")
        with torch.cuda.device(dev):   # the kernel launches on the current CUDA device
            check(self.lib.rg_train_tail_step(ctypes.byref(d), ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)),
                  None, "rg_train_tail_step")

    def step(self, min_scale: torch.Tensor | None = None, grads: dict | None = None):
        """One tail step on the current stream.  ``grads`` maps names to gradients (default: each
        tensor's ``.grad``; a missing or None gradient leaves the tensor as it is, like torch's
        Adam); ``min_scale`` (N,) or (N, 1) is filter_3D (log)."""
        if grads is None:
            grads = {k: self.params[k].grad for k in self.names}
        plan = {k: (use, lr, b1c, b2c) for k, use, lr, b1c, b2c in self._plan(lambda k: grads.get(k) is not None)}
        d = self._args(grads, self._min_scale(min_scale), lambda k: plan[k][0])
        for i, k in enumerate(self.names):
            _, d.tensors[i].lr, d.tensors[i].bias1, d.tensors[i].bias2_sqrt = plan[k]
        self._launch(d)

    # ---- CUDA-graph form ----
    def capture(self, grads: dict, min_scale: torch.Tensor | None = None):
        """Launch the tail reading this step's learning rates and bias corrections from a device
        buffer, for capture inside a CUDA graph; call :meth:`prepare_replay` before each replay.
        ``grads`` and ``min_scale`` are the graph's own tensors (their storage is baked in)."""
        self._graph_grads = {k for k in self.names if grads.get(k) is not None}
        d = self._args(grads, self._min_scale(min_scale), lambda k: True)
        d.step_scalars = self._dev_scalars.data_ptr()
        self._launch(d)

    def prepare_replay(self):
        """Write the next replay's scalars to the captured buffer on the current stream (an
        asynchronous copy from a ring of pinned host buffers) and advance the schedules."""
        if self._graph_grads is None:
            raise RuntimeError("prepare_replay() before capture()")
        if self._host_scalars is None:
            self._host_scalars = [torch.zeros((len(self.names), 4), dtype=torch.float32).pin_memory()
                                  for _ in range(4)]
            self._host_events = [None] * 4
            self._ring = 0
        plan = self._plan(lambda k: k in self._graph_grads)
        j = self._ring % len(self._host_scalars)
        self._ring += 1
        if self._host_events[j] is not None:
            self._host_events[j].synchronize()         # that buffer's copy has run
        h = self._host_scalars[j]
        h.copy_(torch.tensor([[float(use), lr, b1c, b2c] for _, use, lr, b1c, b2c in plan], dtype=torch.float32))
        self._dev_scalars.copy_(h, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        self._host_events[j] = ev
