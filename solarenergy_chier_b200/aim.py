"""Aim-point optimisation of a field with the differentiable pair (qmcrt_fwd / qmcrt_bwd).

Adam over per-heliostat aim offsets (metres, along the receiver's aim axes)
and, optionally, normal offsets (radians), minimising the L2 distance between
the Gaussian-splatted receiver flux and a target flux.  Every step can be
checked by the plain tracer (qmcrt_diff_plain): the same rays binned to the
nearest pixel, smoothed by the same Gaussian, give the loss that the tracer
the reference runs would report for those parameters, and their FP64 power
must equal the forward's (the same hits).

The reference has no derivative of its tracer; its aim points are the
receiver's focus centres (CylinderReceiver.cu:18-31, RectangleReceiver.cu:103-105),
which the aim offsets move.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


def gaussian_weights(sigma_px: float) -> np.ndarray:
    """Taps 0..radius (radius = ceil(3 sigma)) of the normalised Gaussian the pair smooths with."""
    radius = int(math.ceil(3.0 * sigma_px))
    w = np.array([math.exp(-0.5 * k * k / (sigma_px * sigma_px)) for k in range(radius + 1)])
    return (w / (w[0] + 2.0 * w[1:].sum())).astype(np.float32)


def gaussian_smooth(image: np.ndarray, sigma_px: float, wrap_cols: bool) -> np.ndarray:
    """Rows (columns wrapping around a cylinder's image when wrap_cols) then
    columns (zero outside), in FP64: the pair's smoothing of a flux map."""
    w = gaussian_weights(sigma_px).astype(np.float64)
    r = len(w) - 1
    img = np.asarray(image, np.float64)
    h, wd = img.shape
    tmp = np.zeros_like(img)
    for k in range(-r, r + 1):
        if wrap_cols:
            tmp += w[abs(k)] * np.roll(img, -k, axis=1)
        else:
            src = np.zeros_like(img)
            if k >= 0:
                src[:, :wd - k] = img[:, k:]
            else:
                src[:, -k:] = img[:, :wd + k]
            tmp += w[abs(k)] * src
    out = np.zeros_like(img)
    for k in range(-r, r + 1):
        src = np.zeros_like(tmp)
        if k >= 0:
            src[:h - k] = tmp[k:]
        else:
            src[-k:] = tmp[:h + k]
        out += w[abs(k)] * src
    return out


class Adam:
    """Adam (Kingma & Ba 2015) on a numpy array, bias-corrected."""

    def __init__(self, shape, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8):
        self.lr, self.b1, self.b2, self.eps = lr, beta1, beta2, eps
        self.m = np.zeros(shape)
        self.v = np.zeros(shape)
        self.t = 0

    def step(self, x: np.ndarray, grad: np.ndarray) -> np.ndarray:
        self.t += 1
        self.m = self.b1 * self.m + (1 - self.b1) * grad
        self.v = self.b2 * self.v + (1 - self.b2) * grad * grad
        mh = self.m / (1 - self.b1 ** self.t)
        vh = self.v / (1 - self.b2 ** self.t)
        return x - self.lr * mh / (np.sqrt(vh) + self.eps)


@dataclass
class AimResult:
    aim: np.ndarray                      # (H, 2) metres
    normal: np.ndarray                   # (H, 2) radians
    history: list = field(default_factory=list)  # one dict per step


def optimise_aim(diff, target: np.ndarray, steps: int, lr_aim: float = 0.05, lr_normal: float = 0.0,
                 aim0=None, normal0=None, aim_bound: float = 1.0, normal_bound: float = 1e-3,
                 check: bool = True, receiver: int = 0, cylinder: bool = True, sigma_px: float = 2.0,
                 stream=None) -> AimResult:
    """`steps` Adam steps on `diff` (a solarenergy_chier_b200.Diff whose target
    is `target`).  Parameters are kept within +-aim_bound metres and
    +-normal_bound radians.  With `check`, every step also runs the plain
    tracer on the step's parameters and records its smoothed-flux loss
    (`plain_loss`), the relative L1 between that flux and the pair's
    (`plain_vs_splat_l1`) and the forward's and plain tracer's FP64 powers."""
    H = diff.num_heliostats
    aim = np.zeros((H, 2)) if aim0 is None else np.array(aim0, np.float64).reshape(H, 2)
    normal = np.zeros((H, 2)) if normal0 is None else np.array(normal0, np.float64).reshape(H, 2)
    opt_a, opt_n = Adam(aim.shape, lr_aim), Adam(normal.shape, lr_normal)
    target = np.asarray(target, np.float64)
    hist = []
    for k in range(steps):
        diff.set_params(aim, normal)
        loss = diff.forward(stream)
        grad = diff.backward(stream)
        rec = {"step": k, "loss": loss, "grad_norm": float(np.linalg.norm(grad))}
        if check:
            _, fwd_power = diff.power()
            flux = diff.flux(receiver).astype(np.float64)
            diff.plain(stream)
            smoothed = gaussian_smooth(diff.image(receiver), sigma_px, cylinder)
            _, plain_power = diff.power()
            rec.update({"plain_loss": float(((smoothed - target) ** 2).sum()),
                        "plain_vs_splat_l1": float(np.abs(smoothed - flux).sum() / max(np.abs(flux).sum(), 1e-30)),
                        "power": fwd_power, "plain_power": plain_power})
        hist.append(rec)
        aim = np.clip(opt_a.step(aim, grad[:, :2]), -aim_bound, aim_bound)
        if lr_normal > 0.0:
            normal = np.clip(opt_n.step(normal, grad[:, 2:]), -normal_bound, normal_bound)
    return AimResult(aim, normal, hist)


def smooth_target(flux: np.ndarray, seed: int, lit_fraction: float = 0.05) -> np.ndarray:
    """A smooth seeded target over the lit part of `flux` with peak/mean <= 2:
    the lit pixels' mean times 1 + 0.5 cos(3 turns across, random phase) x
    cos(half a turn down, random phase)."""
    h, w = flux.shape
    rows, cols = np.mgrid[0:h, 0:w]
    lit = flux > lit_fraction * flux.max()
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0, 2 * np.pi, 2)
    bump = 1.0 + 0.5 * np.cos(2 * np.pi * cols / w * 3 + ph[0]) * np.cos(np.pi * rows / h + ph[1])
    return (bump * lit * (flux[lit].mean() if lit.any() else 0.0)).astype(np.float32)
