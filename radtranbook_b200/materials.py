"""Material callables.

The reference step functions receive Python callables (sigma_a_func(T), cv(T), inv_eos(e),
eos(T)) and call them on NumPy arrays shaped like the temperature field.  The drop-in API
accepts exactly those callables and calls them the same way (a host evaluation of the
user's material model, O(cells) per step; particle work never leaves the GPU).

Callables marked with :func:`device_callable` are called instead with CUDA torch tensors
(float64, same shape) and must return CUDA tensors; then the whole step stays on the
device.  The parametric materials below are device callables.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import TRANSFER


def device_callable(fn):
    """Mark fn as accepting and returning CUDA torch tensors."""
    fn._imc_device = True
    return fn


def is_device(fn) -> bool:
    return bool(getattr(fn, "_imc_device", False))


def evaluate(fn, T_dev: torch.Tensor, T_host_fn, like: torch.Tensor, stage: torch.Tensor | None = None,
             stage_dev: torch.Tensor | None = None) -> torch.Tensor:
    """Evaluate a material callable on the temperature field.

    T_dev: device tensor in the reference's array shape.  T_host_fn: zero-argument
    function returning the same field as a NumPy array (called only for host callables).
    stage: optional pinned host buffer (>= like.numel() doubles) for a host callable's
    result, which then goes to the device by an asynchronous copy (the caller must not
    refill the buffer before the stream has passed that copy); stage_dev: optional device
    buffer of the same size that receives it (no allocation per call; the result is a view of
    it, valid until the buffer's next use).
    Returns a float64 device tensor broadcast to `like`'s shape.
    """
    if is_device(fn):
        out = fn(T_dev)
        if not isinstance(out, torch.Tensor):
            out = torch.as_tensor(np.asarray(out, dtype=np.float64), device=like.device)
        return torch.broadcast_to(out.to(like.device, torch.float64), like.shape)
    out = fn(T_host_fn())
    if stage is not None:
        n = like.numel()
        host = stage[:n].view(tuple(like.shape))
        np.copyto(host.numpy(), np.broadcast_to(np.asarray(out, dtype=np.float64), tuple(like.shape)))
        TRANSFER["h2d"] += n * 8
        if stage_dev is not None:
            out_dev = stage_dev[:n].view(tuple(like.shape))
            out_dev.copy_(host, non_blocking=True)
            return out_dev
        return host.to(like.device, non_blocking=True)
    arr = np.array(np.broadcast_to(np.asarray(out, dtype=np.float64), tuple(like.shape)), order="C", copy=True)
    TRANSFER["h2d"] += arr.nbytes
    return torch.as_tensor(arr, device=like.device)


class PowerLawOpacity:
    """sigma(T) = A * T**(-n), optionally clamped to [lo, hi] (device callable)."""

    _imc_device = True

    def __init__(self, A: float, n: float, lo: float | None = None, hi: float | None = None):
        self.A, self.n, self.lo, self.hi = float(A), float(n), lo, hi

    def __call__(self, T):
        if isinstance(T, torch.Tensor):
            s = self.A * torch.pow(T, -self.n)
            if self.lo is not None or self.hi is not None:
                s = torch.clamp(s, min=self.lo, max=self.hi)
            return s
        s = self.A * np.power(T, -self.n)
        if self.lo is not None or self.hi is not None:
            s = np.clip(s, self.lo, self.hi)
        return s


class Constant:
    """A constant (scalar or per-cell array) material property (device callable)."""

    _imc_device = True

    def __init__(self, value):
        self.value = value
        self._dev = None

    def __call__(self, T):
        if isinstance(T, torch.Tensor):
            if self._dev is None or self._dev.device != T.device:
                self._dev = torch.as_tensor(np.asarray(self.value, dtype=np.float64), device=T.device)
            return torch.broadcast_to(self._dev, T.shape)
        return np.broadcast_to(np.asarray(self.value, dtype=np.float64), np.shape(T))


class _LinearEOSFunction:
    """e = cv T (inverse=False) or T = e / cv (inverse=True), a device callable that carries
    its heat capacity so the step can evaluate it on the device."""

    _imc_device = True

    def __init__(self, cv: Constant, inverse: bool):
        self.cv, self.inverse = cv, inverse

    def __call__(self, x):
        return x / self.cv(x) if self.inverse else self.cv(x) * x


class LinearEOS:
    """e = cv * T and its inverse, for a constant or per-cell cv (device callables)."""

    def __init__(self, cv):
        self.cv = Constant(cv)
        self.eos = _LinearEOSFunction(self.cv, False)
        self.inv_eos = _LinearEOSFunction(self.cv, True)
        self.cv_func = self.cv


def material_law(sigma_a_func, cv, inv_eos, flat, device):
    """The law of a gray material the device evaluates itself (imc_material_law), when the
    callables are a LinearEOS inverse, a Constant heat capacity and a PowerLawOpacity or
    Constant opacity; else None.  flat(tensor) puts a per-cell array in the engine's cell
    order.  Returns (law, tensors the law points to)."""
    from ._lib import ImcMaterialLaw

    if not (isinstance(inv_eos, _LinearEOSFunction) and inv_eos.inverse and isinstance(cv, Constant)
            and isinstance(sigma_a_func, (PowerLawOpacity, Constant))):
        return None
    keep = []

    def scalar_or_array(const):
        v = np.asarray(const.value, dtype=np.float64)
        if v.ndim == 0:
            return float(v), None
        t = flat(torch.as_tensor(v, device=device)).contiguous()
        keep.append(t)
        return 0.0, t.data_ptr()

    law = ImcMaterialLaw()
    law.cv_eos, law.cv_eos_array = scalar_or_array(inv_eos.cv)
    law.cv, law.cv_array = scalar_or_array(cv)
    if isinstance(sigma_a_func, Constant):
        law.sigma_A, law.sigma_array = scalar_or_array(sigma_a_func)
        law.sigma_n = 0.0
    else:
        law.sigma_A, law.sigma_n = sigma_a_func.A, sigma_a_func.n
        law.sigma_lo = float(sigma_a_func.lo) if sigma_a_func.lo is not None else 0.0
        law.sigma_hi = float(sigma_a_func.hi) if sigma_a_func.hi is not None else 0.0
    return law, keep


class GroupedOpacity(list):
    """The per-group opacity callables of a multigroup problem (a list, as MG_IMC2D.step
    takes) together with one device function that evaluates every group at once:
    all_groups(T) -> (G, *T.shape).  The multigroup steps call all_groups (one fused
    expression instead of G small ones); iterating gives the per-group callables, which
    must compute the same numbers."""

    def __init__(self, funcs, all_groups):
        super().__init__(funcs)
        self.all_groups = all_groups


def evaluate_groups(funcs, T_dev: torch.Tensor, T_host_fn, like: torch.Tensor,
                    stage: torch.Tensor | None = None, stage_dev: torch.Tensor | None = None) -> torch.Tensor:
    """Every group's opacity on the temperature field, (G, *like.shape) float64 on the device.
    stage: optional pinned host buffer of G x like.numel() doubles for host callables (see
    evaluate)."""
    if isinstance(funcs, GroupedOpacity):
        out = funcs.all_groups(T_dev)
        return torch.broadcast_to(out.to(like.device, torch.float64), (len(funcs),) + tuple(like.shape))
    n = like.numel()
    return torch.stack([evaluate(f, T_dev, T_host_fn, like, stage=None if stage is None else stage[g * n:(g + 1) * n],
                                 stage_dev=None if stage_dev is None else stage_dev[g * n:(g + 1) * n])
                        for g, f in enumerate(funcs)])
