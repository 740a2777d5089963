"""Robust loss functions with ceres-torch's class names and semantics
(``losses.py:13-148``): ``evaluate(s)`` returns (rho(s), rho'(s), rho''(s)).

On the solve path the loss is not evaluated here: ``device_spec`` encodes it
for the CUDA evaluator, which applies the same formulas and the Ceres
corrector per observation.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib


def _t(v: float, like: torch.Tensor) -> torch.Tensor:
    return torch.as_tensor(v, dtype=like.dtype, device=like.device)


class LossFunction:
    def evaluate(self, sq_norm: torch.Tensor):
        raise NotImplementedError

    def __call__(self, sq_norm: torch.Tensor):
        return self.evaluate(sq_norm)

    def device_spec(self) -> tuple[int, float, float, float]:
        """(kind, a, b, scale) for the CUDA evaluator."""
        raise NotImplementedError(f"{type(self).__name__} has no CUDA evaluator")


class TrivialLoss(LossFunction):
    def evaluate(self, s):
        return s, torch.ones_like(s), torch.zeros_like(s)

    def device_spec(self):
        return (_lib.LOSS_TRIVIAL, 0.0, 0.0, 1.0)


@dataclass(frozen=True)
class HuberLoss(LossFunction):
    a: float

    def evaluate(self, s):
        b = self.a * self.a
        inside = s <= b
        root = torch.sqrt(torch.clamp(s, min=torch.finfo(s.dtype).tiny))
        return (torch.where(inside, s, 2.0 * self.a * root - b),
                torch.where(inside, torch.ones_like(s), self.a / root),
                torch.where(inside, torch.zeros_like(s), -0.5 * self.a / (root * s)))

    def device_spec(self):
        return (_lib.LOSS_HUBER, float(self.a), 0.0, 1.0)


@dataclass(frozen=True)
class SoftLOneLoss(LossFunction):
    a: float

    def evaluate(self, s):
        b = self.a * self.a
        z = 1.0 + s / b
        rz = torch.sqrt(z)
        return 2.0 * b * (rz - 1.0), 1.0 / rz, -0.5 / (b * z * rz)

    def device_spec(self):
        return (_lib.LOSS_SOFTLONE, float(self.a), 0.0, 1.0)


@dataclass(frozen=True)
class CauchyLoss(LossFunction):
    a: float

    def evaluate(self, s):
        b = self.a * self.a
        z = 1.0 + s / b
        return b * torch.log(z), 1.0 / z, -1.0 / (b * z * z)

    def device_spec(self):
        return (_lib.LOSS_CAUCHY, float(self.a), 0.0, 1.0)


@dataclass(frozen=True)
class ArctanLoss(LossFunction):
    a: float

    def evaluate(self, s):
        z = s / self.a
        d = 1.0 + z * z
        return self.a * torch.atan(z), 1.0 / d, -2.0 * z / (self.a * d * d)

    def device_spec(self):
        return (_lib.LOSS_ARCTAN, float(self.a), 0.0, 1.0)


@dataclass(frozen=True)
class TolerantLoss(LossFunction):
    a: float
    b: float

    def evaluate(self, s):
        z = (s - self.a) / self.b
        c = self.b * torch.nn.functional.softplus(_t(-self.a / self.b, s))
        r1 = torch.sigmoid(z)
        return self.b * torch.nn.functional.softplus(z) - c, r1, r1 * (1.0 - r1) / self.b

    def device_spec(self):
        return (_lib.LOSS_TOLERANT, float(self.a), float(self.b), 1.0)


@dataclass(frozen=True)
class TukeyLoss(LossFunction):
    a: float

    def evaluate(self, s):
        a2 = self.a * self.a
        inner = 1.0 - s / a2
        inside = s <= a2
        return (torch.where(inside, (a2 / 3.0) * (1.0 - inner ** 3), _t(a2 / 3.0, s)),
                torch.where(inside, inner ** 2, torch.zeros_like(s)),
                torch.where(inside, -2.0 * inner / a2, torch.zeros_like(s)))

    def device_spec(self):
        return (_lib.LOSS_TUKEY, float(self.a), 0.0, 1.0)


@dataclass
class ScaledLoss(LossFunction):
    rho: Optional[LossFunction]
    scale: float

    def evaluate(self, s):
        r0, r1, r2 = (self.rho or TrivialLoss()).evaluate(s)
        return self.scale * r0, self.scale * r1, self.scale * r2

    def device_spec(self):
        kind, a, b, sc = (self.rho or TrivialLoss()).device_spec()
        return (kind, a, b, sc * float(self.scale))


@dataclass
class ComposedLoss(LossFunction):
    outer: LossFunction
    inner: LossFunction

    def evaluate(self, s):
        g0, g1, g2 = self.inner.evaluate(s)
        f0, f1, f2 = self.outer.evaluate(g0)
        return f0, f1 * g1, f2 * g1 * g1 + f1 * g2


class LossFunctionWrapper(LossFunction):
    def __init__(self, rho: Optional[LossFunction]) -> None:
        self.rho = rho

    def reset(self, rho: Optional[LossFunction]) -> None:
        self.rho = rho

    def evaluate(self, s):
        return (self.rho or TrivialLoss()).evaluate(s)

    def device_spec(self):
        return (self.rho or TrivialLoss()).device_spec()


_BY_NAME = {"TrivialLoss": TrivialLoss, "HuberLoss": HuberLoss, "SoftLOneLoss": SoftLOneLoss, "CauchyLoss": CauchyLoss,
            "ArctanLoss": ArctanLoss, "TolerantLoss": TolerantLoss, "TukeyLoss": TukeyLoss}


def as_loss(loss) -> Optional[LossFunction]:
    """This module's loss for ``loss``, which may be a loss object of ceres-torch itself
    (losses.py:13-146: the same class names and fields); None stays None."""
    if loss is None or isinstance(loss, LossFunction):
        return loss
    kind = type(loss).__name__
    if kind in _BY_NAME:
        cls = _BY_NAME[kind]
        return cls() if kind == "TrivialLoss" else cls(*(float(getattr(loss, f)) for f in ("a", "b")
                                                          if hasattr(loss, f)))
    if kind == "ScaledLoss":
        return ScaledLoss(as_loss(loss.rho), float(loss.scale))
    if kind == "ComposedLoss":
        return ComposedLoss(as_loss(loss.outer), as_loss(loss.inner))
    if kind == "LossFunctionWrapper":
        return LossFunctionWrapper(as_loss(loss.rho))
    raise NotImplementedError(f"{kind} has no CUDA evaluator")


def device_loss(loss: Optional[LossFunction]) -> dict:
    """Fields of ceres_b200_ba_t describing ``loss`` (None = trivial; ceres-torch's own
    loss objects are accepted)."""
    loss = as_loss(loss) or TrivialLoss()
    if isinstance(loss, LossFunctionWrapper):
        loss = loss.rho or TrivialLoss()
    scale = 1.0
    if isinstance(loss, ScaledLoss) and isinstance(loss.rho, ComposedLoss):
        scale = float(loss.scale)
        loss = loss.rho
    if isinstance(loss, ComposedLoss):
        ok, oa, ob, osc = loss.outer.device_spec()
        ik, ia, ib, isc = loss.inner.device_spec()
        return dict(loss_kind=ok, loss_a=oa, loss_b=ob, loss_scale=osc * scale, inner_loss_kind=ik,
                    inner_a=ia, inner_b=ib, inner_scale=isc)
    k, a, b, sc = loss.device_spec()
    return dict(loss_kind=k, loss_a=a, loss_b=b, loss_scale=sc * scale, inner_loss_kind=-1, inner_a=0.0,
                inner_b=0.0, inner_scale=1.0)
