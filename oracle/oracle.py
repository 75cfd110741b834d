"""ORACLE — test infrastructure only (never imported by the product package).

ctypes wrapper of oracle/liboracle.so, the FP64 history-based CPU restatement of the
reference IMC step (see imc_oracle.cpp for the reference line citations).  It exposes the
same phases as the device engine (initial census, sources + transport, comb) so a test
can feed both the same inputs, and a small driver (`OracleGray`) that runs whole steps
with the reference's step() semantics for statistical comparisons and CPU baselines.
"""
from __future__ import annotations

import ctypes
import math
import os
from ctypes import POINTER, c_double, c_int, c_int64, c_longlong, c_uint32, c_uint64, c_void_p

import numpy as np

from . import build as _build

GEOM = {"slab": 0, "spherical": 1, "xy": 2, "rz": 3}
S_N = 9
A_RAD = 0.01372
C_LIGHT = 29.98


class StepIn(ctypes.Structure):
    _fields_ = [
        ("step", c_uint32), ("dt", c_double), ("theta", c_double),
        ("T", c_void_p), ("sigma", c_void_p), ("cv", c_void_p),
        ("Ntarget", c_longlong), ("Nboundary", c_longlong), ("Nsource", c_longlong),
        ("source", c_void_p), ("face_T", c_void_p * 4), ("reflect", c_int * 4),
        ("max_events", c_longlong), ("rz_linear_source", c_int), ("T_emit_floor", c_double),
        ("nthreads", c_int), ("sources_only", c_int), ("method", c_int), ("cf_fastpath", c_double),
    ]


class StepOut(ctypes.Structure):
    _fields_ = [
        ("dep", c_void_p), ("si", c_void_p), ("emitted", c_void_p), ("sigma_a", c_void_p), ("sigma_s", c_void_p),
        ("boundary_emission", c_double), ("source_emission", c_double), ("escaped", c_double * 4),
        ("stats", c_longlong * S_N), ("n_transported", c_longlong), ("weight_floor", c_double),
    ]


class MgIn(ctypes.Structure):
    _fields_ = [
        ("step", c_uint32), ("dt", c_double), ("theta", c_double),
        ("T", c_void_p), ("sigma", c_void_p), ("cv", c_void_p),
        ("Ntarget", c_longlong), ("Nboundary", c_longlong), ("Nsource", c_longlong),
        ("source", c_void_p), ("face_T", c_void_p * 4), ("reflect", c_int * 4),
        ("max_events", c_longlong), ("emission_fractions", c_void_p), ("group_edges", c_void_p),
        ("T_emit_floor", c_double), ("nthreads", c_int), ("sources_only", c_int),
    ]


class MgOut(ctypes.Structure):
    _fields_ = [
        ("dep", c_void_p), ("si", c_void_p), ("emitted", c_void_p), ("sigma_a", c_void_p), ("sigma_s", c_void_p),
        ("bnd_by_group", c_void_p), ("esc_by_group", c_void_p),
        ("boundary_emission", c_double), ("source_emission", c_double), ("emission_total", c_double),
        ("bnd_by_side", c_double * 4), ("escaped", c_double * 4), ("stats", c_longlong * S_N),
        ("n_transported", c_longlong), ("weight_floor", c_double),
    ]


_lib = None


def load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(str(_build.build()))
        lib.orc_create.restype = c_void_p
        lib.orc_create.argtypes = [c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_uint64]
        lib.orc_destroy.argtypes = [c_void_p]
        lib.orc_size.restype = c_longlong
        lib.orc_size.argtypes = [c_void_p]
        lib.orc_get_bank.argtypes = [c_void_p] + [c_void_p] * 8
        lib.orc_set_bank.argtypes = [c_void_p, c_longlong] + [c_void_p] * 8
        lib.orc_init_ic.restype = c_longlong
        lib.orc_init_ic.argtypes = [c_void_p, c_longlong, c_void_p, c_double]
        lib.orc_step_transport.restype = c_int
        lib.orc_step_transport.argtypes = [c_void_p, POINTER(StepIn), POINTER(StepOut)]
        lib.orc_adjoint_vjp.restype = c_int
        lib.orc_adjoint_vjp.argtypes = [c_void_p, POINTER(StepIn), c_void_p, c_void_p]
        lib.orc_comb.restype = c_longlong
        lib.orc_comb.argtypes = [c_void_p, c_longlong, c_uint32, c_int, c_void_p]
        lib.orc_comb_with_xi.restype = c_longlong
        lib.orc_comb_with_xi.argtypes = [c_void_p, c_longlong, c_void_p, c_void_p]
        lib.orc_event.argtypes = [c_int, c_void_p, c_void_p]
        lib.orc_event_cf.argtypes = [c_int, c_void_p, c_void_p]
        lib.orc_init_ic_mg.restype = c_longlong
        lib.orc_init_ic_mg.argtypes = [c_void_p, c_longlong, c_void_p, c_void_p, c_double]
        lib.orc_step_transport_mg.restype = c_int
        lib.orc_step_transport_mg.argtypes = [c_void_p, POINTER(MgIn), POINTER(MgOut)]
        lib.orc_init_ic_mg1d.restype = c_longlong
        lib.orc_init_ic_mg1d.argtypes = [c_void_p, c_longlong, c_void_p, c_void_p, c_double]
        lib.orc_step_transport_mg1d.restype = c_int
        lib.orc_step_transport_mg1d.argtypes = [c_void_p, POINTER(MgIn), POINTER(MgOut)]
        lib.orc_comb_mg_with_xi.restype = c_longlong
        lib.orc_comb_mg_with_xi.argtypes = [c_void_p, c_longlong, c_void_p, c_int, c_void_p]
        lib.orc_planck_F.restype = c_double
        lib.orc_planck_F.argtypes = [c_double]
        lib.orc_planck_fractions.argtypes = [c_void_p, c_int, c_double, c_void_p]
        lib.orc_planck_group.restype = c_int
        lib.orc_planck_group.argtypes = [c_double, c_void_p, c_int, c_void_p]
        lib.orc_planck_group_mg1d.restype = c_int
        lib.orc_planck_group_mg1d.argtypes = [c_double, c_void_p, c_int, c_void_p]
        lib.orc_philox.argtypes = [c_void_p, c_void_p, c_void_p]
        for f in ("orc_slab_linear", "orc_sphere_cdf", "orc_rz_r_cdf"):
            getattr(lib, f).restype = c_double
        lib.orc_slab_linear.argtypes = [c_double] * 4
        lib.orc_sphere_cdf.argtypes = [c_double] * 5
        lib.orc_rz_r_cdf.argtypes = [c_double] * 5
        _lib = lib
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def philox(ctr, key):
    lib = load()
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib.orc_philox(_p(c), _p(k), _p(out))
    return out


def event(geometry: str, inp) -> np.ndarray:
    """One reference event.  inp = (w d1 d2 p1 p2 lo1 hi1 lo2 hi2 sa ss dcen u0 u1 u2)."""
    lib = load()
    a = np.ascontiguousarray(inp, dtype=np.float64)
    out = np.zeros(10)
    lib.orc_event(GEOM[geometry], _p(a), _p(out))
    return out


def event_cf(geometry: str, inp) -> np.ndarray:
    """One Carter-Forest event.  inp = (w d1 d2 p1 p2 lo1 hi1 lo2 hi2 sigma_a rate dcen
    fastpath u0 u1 u2 u3); returns (w d1 d2 p1 p2 dep_w dep_i dcen crossed evt)."""
    lib = load()
    a = np.ascontiguousarray(inp, dtype=np.float64)
    out = np.zeros(10)
    lib.orc_event_cf(GEOM[geometry], _p(a), _p(out))
    return out


class Oracle:
    def __init__(self, geometry: str, edges1, edges2, volumes_flat, seed: int, n_groups: int = 1):
        self.lib = load()
        self.geometry = geometry
        self.e1 = np.ascontiguousarray(edges1, dtype=np.float64)
        self.e2 = np.ascontiguousarray(edges2, dtype=np.float64)
        self.nx, self.ny = len(self.e1) - 1, len(self.e2) - 1
        self.nc = self.nx * self.ny
        self.vol = np.ascontiguousarray(volumes_flat, dtype=np.float64).reshape(-1)
        self.ng = int(n_groups)
        self.h = self.lib.orc_create(GEOM[geometry], self.nx, self.ny, n_groups, _p(self.e1), _p(self.e2),
                                     _p(self.vol), int(seed) & 0xFFFFFFFFFFFFFFFF)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    @property
    def size(self) -> int:
        return int(self.lib.orc_size(self.h))

    def init_ic(self, tr_flat, N, t_emit_floor=0.0) -> int:
        tr = np.ascontiguousarray(tr_flat, dtype=np.float64)
        return int(self.lib.orc_init_ic(self.h, int(N), _p(tr), float(t_emit_floor)))

    def get_bank(self) -> dict:
        n = self.size
        f = {k: np.zeros(n) for k in ("weight", "dir1", "dir2", "time", "pos1", "pos2")}
        cell = np.zeros(n, dtype=np.int32)
        grp = np.zeros(n, dtype=np.int32)
        self.lib.orc_get_bank(self.h, _p(f["weight"]), _p(f["dir1"]), _p(f["dir2"]), _p(f["time"]), _p(f["pos1"]),
                              _p(f["pos2"]), _p(cell), _p(grp))
        f["cell"] = cell
        f["group"] = grp
        return f

    def set_bank(self, weight, dir1, dir2, time, pos1, pos2, cell, group=None) -> None:
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (weight, dir1, dir2, time, pos1, pos2)]
        c = np.ascontiguousarray(cell, dtype=np.int32)
        g = None if group is None else np.ascontiguousarray(group, dtype=np.int32)
        self.lib.orc_set_bank(self.h, len(arrs[0]), *[_p(a) for a in arrs], _p(c), _p(g))

    def transport(self, T, sigma, cv, source, step, dt, theta, Ntarget, Nboundary, Nsource, face_T, reflect,
                  max_events=0, rz_linear_source=True, t_emit_floor=0.0, nthreads=None, sources_only=False,
                  method="fc", cf_fastpath=0.0) -> dict:
        """Sources + transport of one step; method 'fc' (Fleck-Cummings) or 'cf' (Carter-Forest)."""
        keep = []

        def arr(x):
            if x is None:
                return None
            a = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
            keep.append(a)
            return _p(a)

        si = StepIn()
        si.step = int(step) & 0xFFFFFFFF
        si.dt, si.theta = float(dt), float(theta)
        si.T, si.sigma, si.cv = arr(T), arr(sigma), arr(cv)
        si.Ntarget, si.Nboundary, si.Nsource = int(Ntarget), int(Nboundary), int(Nsource)
        si.source = arr(source)
        for q in range(4):
            si.face_T[q] = arr(face_T[q]) if q < len(face_T) else None
            si.reflect[q] = int(bool(reflect[q])) if q < len(reflect) else 0
        si.max_events = int(max_events)
        si.rz_linear_source = int(bool(rz_linear_source))
        si.T_emit_floor = float(t_emit_floor)
        si.nthreads = int(nthreads or os.cpu_count() or 1)
        si.sources_only = int(bool(sources_only))
        si.method = {"fc": 0, "cf": 1}[method]
        si.cf_fastpath = float(cf_fastpath)
        out = {k: np.zeros(self.nc) for k in ("dep", "si", "emitted", "sigma_a", "sigma_s")}
        so = StepOut()
        so.dep, so.si, so.emitted, so.sigma_a, so.sigma_s = (_p(out[k]) for k in ("dep", "si", "emitted", "sigma_a", "sigma_s"))
        st = self.lib.orc_step_transport(self.h, ctypes.byref(si), ctypes.byref(so))
        if st != 0:
            raise AssertionError("non-positive temperature in material state")
        out["boundary_emission"] = so.boundary_emission
        out["source_emission"] = so.source_emission
        out["escaped"] = np.array(so.escaped[:])
        out["stats"] = np.array(so.stats[:], dtype=np.int64)
        out["n_transported"] = so.n_transported
        out["weight_floor"] = so.weight_floor
        return out

    def adjoint_vjp(self, T, sigma, cv, step, dt, theta, reflect, cotangent, max_events=0, nthreads=None):
        """d(cot . dep)/d sigma on the current bank (census + the step's sources, e.g. after
        transport(..., sources_only=True)), FP64; the bank is not modified."""
        keep = []

        def arr(x):
            a = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
            keep.append(a)
            return _p(a)

        si = StepIn()
        si.step = int(step) & 0xFFFFFFFF
        si.dt, si.theta = float(dt), float(theta)
        si.T, si.sigma, si.cv = arr(T), arr(sigma), arr(cv)
        for q in range(4):
            si.face_T[q] = None
            si.reflect[q] = int(bool(reflect[q])) if q < len(reflect) else 0
        si.max_events = int(max_events)
        si.nthreads = int(nthreads or os.cpu_count() or 1)
        grad = np.zeros(self.nc)
        st = self.lib.orc_adjoint_vjp(self.h, ctypes.byref(si), arr(cotangent), _p(grad))
        if st != 0:
            raise ValueError("the adjoint covers 2-D gray geometries (xy, rz)")
        return grad

    # ---------------- multigroup ----------------
    def init_ic_mg(self, tr_flat, N, group_edges, t_emit_floor=0.0) -> int:
        tr = np.ascontiguousarray(tr_flat, dtype=np.float64)
        ge = np.ascontiguousarray(group_edges, dtype=np.float64)
        return int(self.lib.orc_init_ic_mg(self.h, int(N), _p(tr), _p(ge), float(t_emit_floor)))

    def init_ic_mg1d(self, tr_flat, N, group_edges, t_emit_floor=0.0) -> int:
        """MG_IMC1D initial census (stratified per shell, Planck group at the shell's Tr)."""
        tr = np.ascontiguousarray(tr_flat, dtype=np.float64)
        ge = np.ascontiguousarray(group_edges, dtype=np.float64)
        return int(self.lib.orc_init_ic_mg1d(self.h, int(N), _p(tr), _p(ge), float(t_emit_floor)))

    def transport_mg1d(self, *args, **kw) -> dict:
        """One MG_IMC1D step up to the material update (same arguments as transport_mg)."""
        return self.transport_mg(*args, _entry="orc_step_transport_mg1d", **kw)

    def transport_mg(self, T, sigma_gc, cv, source_gc, step, dt, theta, Ntarget, Nboundary, Nsource, face_T,
                     reflect, group_edges, max_events=0, emission_fractions=None, t_emit_floor=0.0, nthreads=None,
                     sources_only=False, _entry="orc_step_transport_mg") -> dict:
        keep = []

        def arr(x):
            if x is None:
                return None
            a = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
            keep.append(a)
            return _p(a)

        G = len(group_edges) - 1
        mi = MgIn()
        mi.step = int(step) & 0xFFFFFFFF
        mi.dt, mi.theta = float(dt), float(theta)
        mi.T, mi.sigma, mi.cv = arr(T), arr(sigma_gc), arr(cv)
        mi.Ntarget, mi.Nboundary, mi.Nsource = int(Ntarget), int(Nboundary), int(Nsource)
        mi.source = arr(source_gc)
        for q in range(4):
            mi.face_T[q] = arr(face_T[q]) if q < len(face_T) else None
            mi.reflect[q] = int(bool(reflect[q])) if q < len(reflect) else 0
        mi.max_events = int(max_events)
        mi.emission_fractions = arr(emission_fractions)
        mi.group_edges = arr(group_edges)
        mi.T_emit_floor = float(t_emit_floor)
        mi.nthreads = int(nthreads or os.cpu_count() or 1)
        mi.sources_only = int(bool(sources_only))
        ncg = self.nc * G
        out = {k: np.zeros(ncg) for k in ("dep", "si", "sigma_a", "sigma_s")}
        out["emitted"] = np.zeros(self.nc)
        out["bnd_by_group"] = np.zeros(G)
        out["esc_by_group"] = np.zeros(G)
        mo = MgOut()
        for k in ("dep", "si", "emitted", "sigma_a", "sigma_s", "bnd_by_group", "esc_by_group"):
            setattr(mo, k, _p(out[k]))
        st = getattr(self.lib, _entry)(self.h, ctypes.byref(mi), ctypes.byref(mo))
        if st != 0:
            raise AssertionError("invalid multigroup material state")
        out["boundary_emission"] = mo.boundary_emission
        out["source_emission"] = mo.source_emission
        out["emission_total"] = mo.emission_total
        out["bnd_by_side"] = np.array(mo.bnd_by_side[:])
        out["escaped"] = np.array(mo.escaped[:])
        out["stats"] = np.array(mo.stats[:], dtype=np.int64)
        out["n_transported"] = mo.n_transported
        out["weight_floor"] = mo.weight_floor
        return out

    def comb(self, Nmax, step, per_group=False, conserve_radiation=False) -> np.ndarray:
        """Nmax > 0 combs to Nmax; 0 only drops dead entries; < 0 combs to |Nmax| once at
        least |Nmax| entries are alive.  Returns the per-bin discrepancy (before - after)."""
        disc = np.zeros(self.nc * (self.ng if per_group else 1))
        flags = int(bool(per_group)) | (2 if conserve_radiation else 0)
        self.lib.orc_comb(self.h, int(Nmax), int(step) & 0xFFFFFFFF, flags, _p(disc))
        return disc

    def comb_mg_with_xi(self, Nmax, xi, conserve_radiation=False) -> np.ndarray:
        disc = np.zeros(self.nc * self.ng)
        x = np.ascontiguousarray(xi, dtype=np.float64)
        self.lib.orc_comb_mg_with_xi(self.h, int(Nmax), _p(x), 2 if conserve_radiation else 0, _p(disc))
        return disc

    def comb_with_xi(self, Nmax, xi) -> np.ndarray:
        disc = np.zeros(self.nc)
        x = np.ascontiguousarray(xi, dtype=np.float64)
        self.lib.orc_comb_with_xi(self.h, int(Nmax), _p(x), _p(disc))
        return disc


def flat2d(a):
    """reference (nx, ny) array -> flat c = i + nx*j"""
    a = np.asarray(a, dtype=np.float64)
    return np.ascontiguousarray(a.T).reshape(-1) if a.ndim == 2 else a.reshape(-1)


def grid2d(f, nx, ny):
    return np.asarray(f).reshape(ny, nx).T


class OracleGray:
    """Whole reference steps (IMC1D/IMC2D semantics) on the oracle, in FP64 on the CPU."""

    def __init__(self, geometry, edges1, edges2, volumes_flat, seed, Ntarget, Tinit, Tr_init, eos, inv_eos,
                 Ntarget_ic=None, nthreads=None, T_emit_floor=0.0):
        self.o = Oracle(geometry, edges1, edges2, volumes_flat, seed)
        self.geometry = geometry
        self.dim = 1 if geometry in ("slab", "spherical") else 2
        self.shape = np.shape(Tinit)
        self.nthreads = nthreads
        self.T = flat2d(Tinit)
        self.e = flat2d(eos(np.asarray(Tinit, dtype=np.float64)))
        self.o.init_ic(flat2d(Tr_init), Ntarget if Ntarget_ic is None else Ntarget_ic, T_emit_floor)
        b = self.o.get_bank()
        self.prev = float(np.sum(self.e * self.o.vol) + np.sum(b["weight"]))
        self.count = 0
        self.time = 0.0
        self.Tr = np.zeros(self.o.nc)

    def grid(self, f):
        return f if self.dim == 1 else grid2d(f, self.o.nx, self.o.ny)

    def step(self, Ntarget, Nboundary, Nsource, Nmax, face_T, dt, sigma_a_func, inv_eos, cv, source=None,
             reflect=(False, False, False, False), theta=1.0, conserve_comb_energy=False, max_events=0,
             rz_linear_source=True, method="fc", cf_fastpath=0.0):
        Tg = self.grid(self.T)
        sigma = flat2d(np.broadcast_to(sigma_a_func(Tg), Tg.shape))
        cvv = flat2d(np.broadcast_to(cv(Tg), Tg.shape))
        src = None if source is None else flat2d(source)
        r = self.o.transport(self.T, sigma, cvv, src, self.count, dt, theta, Ntarget, Nboundary, Nsource, face_T,
                             reflect, max_events=max_events, rz_linear_source=rz_linear_source,
                             nthreads=self.nthreads, method=method, cf_fastpath=cf_fastpath)
        self.e = self.e + r["dep"] - r["emitted"] / self.o.vol
        self.T = flat2d(inv_eos(self.grid(self.e)))
        self.Tr = np.sqrt(np.sqrt(np.maximum(r["si"], 0) / A_RAD / C_LIGHT))
        disc = self.o.comb(Nmax, self.count)
        if conserve_comb_energy:
            self.e = self.e + disc / self.o.vol
            self.T = flat2d(inv_eos(self.grid(self.e)))
        b = self.o.get_bank()
        total = float(np.sum(self.e * self.o.vol) + math.fsum(b["weight"]))
        bl = float(np.sum(r["escaped"]))
        loss = total - self.prev - r["boundary_emission"] + bl - r["source_emission"]
        r["energy_loss"] = loss
        r["closure"] = loss + (0.0 if conserve_comb_energy else float(np.sum(disc)))
        r["total_energy"] = total
        r["disc"] = disc
        self.prev = total
        self.count += 1
        self.time += dt
        return r
