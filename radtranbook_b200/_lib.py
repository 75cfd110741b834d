"""ctypes binding of libimcb200.so (the C ABI declared in include/imcb200.h).

The library is loaded from this package directory.  Nothing here falls back to another
implementation: if the shared object is missing, or no CUDA device is present when a
device call is made, the call raises.
"""
from __future__ import annotations

import ctypes
import os
import pathlib
from ctypes import POINTER, c_double, c_int, c_int32, c_int64, c_uint32, c_uint64, c_ulonglong, c_void_p, c_size_t, c_char_p

HERE = pathlib.Path(__file__).resolve().parent
# IMCB200_CHECKED=1 selects the bounds-checked build (radtranbook_b200/build.py)
LIB_PATH = HERE / ("libimcb200_checked.so" if os.environ.get("IMCB200_CHECKED") == "1" else "libimcb200.so")

GEOM = {"slab": 0, "spherical": 1, "xy": 2, "rz": 3}

STATUS = {
    0: "IMC_OK",
    1: "IMC_ERR_BANK_OVERFLOW",
    2: "IMC_ERR_EVENT_CAP",
    3: "IMC_ERR_NONFINITE",
    4: "IMC_ERR_BAD_GEOMETRY",
    5: "IMC_ERR_TIMEOUT",
    6: "IMC_ERR_CUDA",
    7: "IMC_ERR_INVALID_ARG",
    8: "IMC_ERR_WORKSPACE",
    9: "IMC_ERR_BOUNDS",
}
OK, BANK_OVERFLOW = 0, 1

COMB_PER_GROUP, COMB_CONSERVE_RADIATION, COMB_CENSUS_READY, COMB_WRITE_AFTER = 1, 2, 4, 8  # imc_comb flags
CENSUS_BY_CELL, CENSUS_BY_GROUP_CELL = 1, 2  # imc_step_params.census_bins
METHOD_FLECK_CUMMINGS, METHOD_CARTER_FOREST = 0, 1  # imc_step_params.method

STAT_EVENTS, STAT_BOUNDARY, STAT_SCATTER, STAT_CENSUS, STAT_CAPTURE, STAT_FLOOR, STAT_REFLECT, STAT_CAP, STAT_ESCAPE, STAT_N = range(10)


class ImcMesh(ctypes.Structure):
    _fields_ = [
        ("geometry", c_int32), ("nx", c_int32), ("ny", c_int32), ("n_groups", c_int32),
        ("edges1", c_void_p), ("edges2", c_void_p), ("volume", c_void_p), ("group_edges", c_void_p),
    ]


class ImcBank(ctypes.Structure):
    _fields_ = [
        ("pos1", c_void_p), ("pos2", c_void_p), ("dir1", c_void_p), ("dir2", c_void_p),
        ("weight", c_void_p), ("time", c_void_p), ("cell", c_void_p), ("group", c_void_p),
        ("size", c_int64), ("capacity", c_int64),
    ]


class ImcMaterial(ctypes.Structure):
    _fields_ = [("temperature", c_void_p), ("sigma", c_void_p), ("cv", c_void_p), ("source", c_void_p)]


class ImcStepParams(ctypes.Structure):
    _fields_ = [
        ("seed", c_uint64), ("step", c_uint32), ("reflect", c_int32 * 4),
        ("dt", c_double), ("theta", c_double),
        ("n_target", c_int64), ("n_boundary", c_int64), ("n_source", c_int64),
        ("face_T", c_void_p * 4),
        ("max_events", c_int64),
        ("rz_linear_source", c_int32), ("census_bins", c_int32),
        ("t_emit_floor", c_double),
        ("block_size", c_int32), ("blocks_per_sm", c_int32), ("chunk", c_int32), ("reserved", c_int32),
        ("emission_fractions", c_void_p),
        ("n_boundary_side", c_int64 * 4),
        ("method", c_int32), ("id_base", c_uint32), ("cf_fastpath", c_double),
        ("step_dev", c_void_p), ("dt_dev", c_void_p), ("energy_share", c_double),
    ]


class ImcMaterialLaw(ctypes.Structure):
    _fields_ = [("cv_eos", c_double), ("cv_eos_array", c_void_p), ("cv", c_double), ("cv_array", c_void_p),
                ("sigma_A", c_double), ("sigma_n", c_double), ("sigma_lo", c_double), ("sigma_hi", c_double),
                ("sigma_array", c_void_p), ("sigma_scale", c_void_p), ("sigma_T_floor", c_double),
                ("sigma_group", c_void_p)]


class ImcTallies(ctypes.Structure):
    _fields_ = [
        ("dep", c_void_p), ("si", c_void_p), ("emitted", c_void_p), ("sigma_a", c_void_p),
        ("sigma_s", c_void_p), ("escaped", c_void_p), ("stats", c_void_p),
        ("escaped_group", c_void_p), ("boundary_group", c_void_p),
    ]


class ImcStepReport(ctypes.Structure):
    _fields_ = [
        ("n_boundary", c_int64), ("n_source", c_int64), ("n_emission", c_int64),
        ("n_transported", c_int64), ("required_capacity", c_int64),
        ("boundary_emission", c_double), ("source_emission", c_double), ("emission_total", c_double),
        ("weight_floor", c_double),
        ("ms_sources", ctypes.c_float), ("ms_transport", ctypes.c_float),
    ]


class ImcCombReport(ctypes.Structure):
    _fields_ = [
        ("n_in", c_int64), ("n_out", c_int64), ("required_capacity", c_int64),
        ("energy_before", c_double), ("energy_after", c_double),
    ]


FLAG_EVENT_CAP, FLAG_NONFINITE, FLAG_COMB_OVERFLOW, FLAG_BOUNDS = 1, 2, 4, 8


class ImcStepSummary(ctypes.Structure):
    _fields_ = [
        ("n_census", c_int64), ("n_side", c_int64 * 4), ("n_source", c_int64), ("n_emission", c_int64),
        ("base_side", c_int64 * 4), ("base_source", c_int64), ("base_emission", c_int64),
        ("n_bank", c_int64), ("n_out", c_int64), ("flags", c_int32), ("pad", c_int32),
        ("e_side", c_double * 4), ("source_emission", c_double), ("emission_total", c_double),
        ("weight_sum", c_double), ("comb_before", c_double), ("comb_after", c_double),
        ("internal_energy", c_double), ("stats", c_ulonglong * 9), ("escaped", c_double * 4),
    ]


# name -> (restype, argtypes); every symbol declared in include/imcb200.h
# batched 1-D slab problems
(BL_TOTAL, BL_PREV, BL_INTERNAL, BL_RADIATION, BL_BOUNDARY, BL_ESCAPED, BL_EMISSION, BL_COMB_DISC, BL_CLOSURE,
 BL_MAX_REL, BL_EVENTS, BL_N) = range(12)


class ImcBatch(ctypes.Structure):
    _fields_ = [("n_inst", c_int32), ("n_cells", c_int32), ("n_slots", c_int64), ("max_new", c_int64),
                ("dt", c_double), ("theta", c_double),
                ("cell_off", c_void_p), ("edges", c_void_p), ("slot_off", c_void_p), ("seed", c_void_p),
                ("n_target", c_void_p), ("n_boundary", c_void_p), ("n_max", c_void_p), ("face_T", c_void_p),
                ("reflect", c_void_p), ("opacity_a", c_void_p), ("opacity_p", c_void_p), ("cv", c_void_p),
                ("max_cells", c_int32)]


class ImcBatchState(ctypes.Structure):
    _fields_ = [("bank", ImcBank * 2), ("sel", c_void_p), ("step", c_void_p), ("n_census", c_void_p),
                ("T", c_void_p), ("e", c_void_p), ("tr", c_void_p), ("dep", c_void_p), ("si", c_void_p),
                ("emitted", c_void_p), ("ledger", c_void_p), ("stats", c_void_p), ("flags", c_void_p)]


class ImcBatchLaunch(ctypes.Structure):
    _fields_ = [("block_size", c_int32), ("blocks_per_sm", c_int32), ("chunk", c_int32), ("refill_min", c_int32),
                ("form", c_int32)]


SIGNATURES = {
    "imc_workspace_bytes": (c_size_t, [POINTER(ImcMesh), c_int64]),
    "imc_workspace_bytes_event": (c_size_t, [POINTER(ImcMesh), c_int64]),
    "imc_init_census": (c_int, [POINTER(ImcMesh), c_void_p, c_int64, c_double, c_uint64, POINTER(ImcBank),
                                c_void_p, c_size_t, POINTER(c_int64), c_void_p]),
    "imc_step_transport": (c_int, [POINTER(ImcMesh), POINTER(ImcMaterial), POINTER(ImcStepParams),
                                   POINTER(ImcBank), POINTER(ImcTallies), c_void_p, c_size_t,
                                   POINTER(ImcStepReport), c_void_p]),
    "imc_material_update": (c_int, [POINTER(ImcMesh), POINTER(ImcTallies), c_void_p, c_void_p, c_void_p]),
    "imc_material_update_law": (c_int, [POINTER(ImcMesh), POINTER(ImcTallies), POINTER(ImcMaterialLaw), c_void_p,
                                        c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "imc_comb": (c_int, [POINTER(ImcMesh), POINTER(ImcBank), POINTER(ImcBank), c_int64, c_uint64, c_uint32,
                         c_int32, c_void_p, c_void_p, c_size_t, POINTER(ImcCombReport), c_void_p]),
    "imc_comb_noalloc": (c_int, [POINTER(ImcMesh), POINTER(ImcBank), POINTER(ImcBank), c_int64, c_uint64,
                                 c_uint32, c_int32, c_void_p, POINTER(ImcCombReport), c_void_p]),
    "imc_adjoint_vjp": (c_int, [POINTER(ImcMesh), POINTER(ImcMaterial), POINTER(ImcStepParams), POINTER(ImcBank),
                                c_void_p, c_void_p, POINTER(ImcTallies), c_void_p, c_size_t, c_void_p]),
    "imc_batch_workspace_bytes": (c_size_t, [POINTER(ImcBatch)]),
    "imc_batch_init": (c_int, [POINTER(ImcBatch), POINTER(ImcBatchState), c_void_p, c_void_p, c_void_p, c_size_t,
                               c_void_p]),
    "imc_batch_step": (c_int, [POINTER(ImcBatch), POINTER(ImcBatchState), POINTER(ImcBatchLaunch), c_void_p, c_size_t,
                               c_void_p]),
    "imc_source_bound": (c_int64, [POINTER(ImcMesh), POINTER(ImcStepParams)]),
    "imc_step_transport_async": (c_int, [POINTER(ImcMesh), POINTER(ImcMaterial), POINTER(ImcStepParams),
                                         POINTER(ImcBank), POINTER(ImcTallies), c_void_p, c_size_t, c_void_p,
                                         c_void_p]),
    "imc_comb_async": (c_int, [POINTER(ImcMesh), POINTER(ImcBank), POINTER(ImcBank), c_int64, c_uint64, c_uint32,
                               c_int32, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p, c_void_p]),
    "imc_comb_async_dev": (c_int, [POINTER(ImcMesh), POINTER(ImcBank), POINTER(ImcBank), c_int64, c_void_p,
                                   c_uint64, c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p, c_void_p]),
    "imc_mg_report_fields": (c_int, [POINTER(ImcMesh), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                     c_void_p, c_void_p, c_void_p]),
    "imc_bank_energy_by_bin": (c_int, [POINTER(ImcMesh), POINTER(ImcBank), c_void_p, c_int32, c_void_p,
                                       c_void_p]),
    "imc_phase_times": (c_int, [POINTER(ctypes.c_float), POINTER(ctypes.c_float)]),
    "imc_energy_totals": (c_int, [POINTER(ImcMesh), POINTER(ImcBank), c_void_p, POINTER(c_double),
                                  POINTER(c_double), c_void_p, c_size_t, c_void_p]),
    "imc_philox": (c_int, [c_void_p, c_uint32, c_uint32, c_void_p, c_int64, c_void_p]),
    "imc_status_str": (c_char_p, [c_int]),
    "imc_last_cuda_error": (c_int, []),
    "imc_kernel_launches": (c_ulonglong, []),
}

# host<->device bytes moved by the drop-in API (material callables, host mirrors)
TRANSFER = {"h2d": 0, "d2h": 0}

_lib = None


def load() -> ctypes.CDLL:
    """Load libimcb200.so; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                "or `python radtranbook_b200/build.py` (requires nvcc)")
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class ImcError(RuntimeError):
    def __init__(self, call: str, status: int):
        lib = load()
        msg = lib.imc_status_str(status).decode()
        extra = f" (cudaError {lib.imc_last_cuda_error()})" if status == 6 else ""
        super().__init__(f"{call}: {STATUS.get(status, status)}: {msg}{extra}")
        self.status = status


def check(call: str, status: int) -> None:
    if status != OK:
        raise ImcError(call, status)
