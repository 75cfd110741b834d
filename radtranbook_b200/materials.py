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
    """The law of a material the device evaluates itself (imc_material_law), when the
    callables are a LinearEOS inverse, a Constant heat capacity and a PowerLawOpacity or
    Constant opacity (gray) or a GroupPowerLawOpacity (multigroup); else None.  flat(tensor)
    puts a per-cell array in the engine's cell order.  Returns (law, tensors the law points
    to)."""
    from ._lib import ImcMaterialLaw

    if not (isinstance(inv_eos, _LinearEOSFunction) and inv_eos.inverse and isinstance(cv, Constant)
            and isinstance(sigma_a_func, (PowerLawOpacity, Constant, GroupPowerLawOpacity))):
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
    if isinstance(sigma_a_func, GroupPowerLawOpacity):
        o = sigma_a_func
        law.sigma_A, law.sigma_n = o.A, o.n
        law.sigma_lo = float(o.lo) if o.lo is not None else 0.0
        law.sigma_hi = float(o.hi) if o.hi is not None else 0.0
        law.sigma_T_floor = float(o.T_floor) if o.T_floor is not None else 0.0
        sc = np.asarray(o.scale, dtype=np.float64)
        if sc.ndim or float(sc) != 1.0:  # a per-cell factor (a scalar one as a constant array)
            t = flat(torch.as_tensor(np.broadcast_to(sc, o.field_shape) if sc.ndim == 0 else sc,
                                     device=device)).contiguous()
            keep.append(t)
            law.sigma_scale = t.data_ptr()
        f = torch.as_tensor(o.factors, device=device)
        keep.append(f)
        law.sigma_group = f.data_ptr()
    elif isinstance(sigma_a_func, Constant):
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


class GroupPowerLawOpacity(GroupedOpacity):
    """Multigroup opacity sigma_g(T) = A * max(T, T_floor)**(-n) * scale * factors[g], clamped
    to [lo, hi] (multiplied in that order; T_floor / lo / hi None for none; scale a scalar or
    a per-cell array shaped like the temperature field).  A GroupedOpacity: its per-group
    callables and all_groups work on host arrays and device tensors alike.  With a LinearEOS
    and a Constant heat capacity the multigroup steps evaluate it on the device themselves,
    in the material update kernel (imc_material_law)."""

    def __init__(self, A: float, n: float, factors, scale=1.0, T_floor: float | None = None,
                 lo: float | None = None, hi: float | None = None, field_shape: tuple | None = None):
        self.A, self.n = float(A), float(n)
        self.factors = np.ascontiguousarray(factors, dtype=np.float64)
        self.scale = scale
        self.T_floor, self.lo, self.hi = T_floor, lo, hi
        sc = np.asarray(scale)
        self.field_shape = tuple(field_shape) if field_shape is not None else sc.shape
        self._dev = {}
        super().__init__([self._one(g) for g in range(len(self.factors))], self._all)

    def _const(self, key, value, like):
        k = (key, like.device)
        if k not in self._dev:
            self._dev[k] = torch.as_tensor(np.asarray(value, dtype=np.float64), device=like.device)
        return self._dev[k]

    def _base(self, T):
        if isinstance(T, torch.Tensor):
            tp = torch.clamp(T, min=self.T_floor) if self.T_floor is not None else T
            b = self.A * torch.pow(tp, -self.n) if self.n != 0.0 else torch.full_like(T, self.A)
            return b * self._const("scale", self.scale, T) if np.ndim(self.scale) else b * float(self.scale)
        T = np.asarray(T, dtype=np.float64)
        tp = np.maximum(T, self.T_floor) if self.T_floor is not None else T
        b = self.A * np.power(tp, -self.n) if self.n != 0.0 else np.full_like(T, self.A)
        return b * np.asarray(self.scale, dtype=np.float64)

    def _clamp(self, s):
        if self.lo is None and self.hi is None:
            return s
        if isinstance(s, torch.Tensor):
            return torch.clamp(s, min=self.lo, max=self.hi)
        return np.clip(s, self.lo, self.hi)

    def _one(self, g):
        f = float(self.factors[g])

        def sigma_g(T):
            return self._clamp(self._base(T) * f)
        sigma_g._imc_device = True
        return sigma_g

    def _all(self, T):
        b = self._base(T)
        if isinstance(b, torch.Tensor):
            f = self._const("factors", self.factors, b).view((-1,) + (1,) * b.dim())
        else:
            f = self.factors.reshape((-1,) + (1,) * b.ndim)
        return self._clamp(b.unsqueeze(0) * f if isinstance(b, torch.Tensor) else b[None] * f)


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
