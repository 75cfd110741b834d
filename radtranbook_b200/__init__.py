"""B200-native implicit Monte Carlo (Fleck-Cummings) time-step engine.

Drop-in modules with the reference (DrRyanMc/RadTranBook) step API:
  radtranbook_b200.imc1d     ~ IMC/IMC1D.py        (slab, spherical)
  radtranbook_b200.imc2d     ~ IMC/IMC2D.py        (xy, rz)
  radtranbook_b200.mg_imc2d  ~ MG_IMC/MG_IMC2D.py  (multigroup xy, rz)
  radtranbook_b200.mg_imc1d  ~ MG_IMC/MG_IMC1D.py  (multigroup sphere)
The compute path is libimcb200.so (hand-written sm_100a CUDA behind the C ABI of
include/imcb200.h); there is no CPU fallback.
"""
from . import _lib  # noqa: F401

__all__ = ["imc1d", "imc2d", "mg_imc2d", "mg_imc1d", "batch", "adjoint", "engine", "materials"]
