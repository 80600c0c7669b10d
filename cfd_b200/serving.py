"""Serving loop front end (include/cfdb_serve.h) and its load generator.

`Server` wraps the library's continuous-batching request loop. `run_load` drives it with
Poisson arrivals of pressure-solve requests over a pool of registered meshes and reports
latency percentiles and throughput.
"""
from __future__ import annotations

import ctypes as C
import threading
import time
from dataclasses import dataclass

import numpy as np

from . import (AmgSettings, AmgSettingsStruct, InvalidArgument, Precision, SolveStats,
               StatsStruct, _check, _dp, _f64, _i32, _ip, _lib)

_i, _d, _vp, _ll = C.c_int, C.c_double, C.c_void_p, C.c_longlong
_pd = C.POINTER(C.c_double)


class ServerConfigStruct(C.Structure):
    _fields_ = [("slots", _i), ("hbm_budget_bytes", _d), ("precision", _i),
                ("settings", AmgSettingsStruct), ("max_age", _i)]


class ServerInfoStruct(C.Structure):
    _fields_ = [("resident_systems", _i), ("resident_bytes", _d), ("queued", _i),
                ("completed", _ll), ("evictions", _ll)]


def _p(name, args, res=_i):
    f = getattr(_lib, name)
    f.argtypes = args
    f.restype = res


_p("cfdb_default_server_config", [C.POINTER(ServerConfigStruct)], None)
_p("cfdb_server_create", [C.POINTER(ServerConfigStruct), C.POINTER(_vp)])
_p("cfdb_server_destroy", [_vp])
_p("cfdb_server_add_mesh", [_vp, _i, _i, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)])
_p("cfdb_server_submit", [_vp, _i, _ll, _pd, _pd, _pd, _pd, _i, _d, _i, C.POINTER(_ll)])
_p("cfdb_server_wait", [_vp, _ll, _pd, C.POINTER(StatsStruct), _pd])
_p("cfdb_server_info", [_vp, C.POINTER(ServerInfoStruct)])


class Server:
    def __init__(self, slots=4, hbm_budget_bytes=150e9, precision=Precision.MIXED,
                 settings: AmgSettings | None = None, max_age=0):
        cfg = ServerConfigStruct()
        _lib.cfdb_default_server_config(C.byref(cfg))
        cfg.slots, cfg.hbm_budget_bytes, cfg.precision = int(slots), float(hbm_budget_bytes), int(precision)
        cfg.settings = (settings or AmgSettings())._c()
        cfg.max_age = int(max_age)
        h = _vp()
        _check(_lib.cfdb_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self.meshes = {}

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            _lib.cfdb_server_destroy(h)
            self._h = None

    __del__ = close

    def add_mesh(self, n_cells, owner, neighbour) -> int:
        nei = _i32(neighbour)
        own = _i32(owner[:len(nei)])
        mid = _i()
        _check(_lib.cfdb_server_add_mesh(self._h, int(n_cells), len(nei), _ip(own), _ip(nei),
                                         C.byref(mid)))
        self.meshes[mid.value] = (int(n_cells), len(nei))
        return mid.value

    def submit(self, mesh_id, matrix_key, diag, upper, lower, rhs, warm_start=False,
               rel_tol=1e-8, max_iterations=500) -> int:
        n, nf = self.meshes[mesh_id]
        diag, upper, lower, rhs = _f64(diag), _f64(upper), _f64(lower), _f64(rhs)
        if len(diag) != n or len(rhs) != n or len(upper) != nf or len(lower) != nf:
            raise InvalidArgument("request arrays do not match the mesh")
        t = _ll()
        _check(_lib.cfdb_server_submit(self._h, int(mesh_id), int(matrix_key), _dp(diag),
                                       _dp(upper), _dp(lower), _dp(rhs), 1 if warm_start else 0,
                                       float(rel_tol), int(max_iterations), C.byref(t)))
        return t.value

    def wait(self, ticket, n_cells=None):
        x = np.zeros(n_cells) if n_cells else None
        st = StatsStruct()
        times = (C.c_double * 3)()
        _check(_lib.cfdb_server_wait(self._h, int(ticket), _dp(x) if x is not None else None,
                                     C.byref(st), times))
        return x, SolveStats._from(st), (times[0], times[1], times[2])

    def info(self) -> dict:
        i = ServerInfoStruct()
        _check(_lib.cfdb_server_info(self._h, C.byref(i)))
        return {"resident_systems": i.resident_systems, "resident_bytes": i.resident_bytes,
                "queued": i.queued, "completed": i.completed, "evictions": i.evictions}


@dataclass
class MeshEntry:
    mesh_id: int
    n: int
    diag: np.ndarray
    upper: np.ndarray
    lower: np.ndarray
    rhs: np.ndarray


def run_load(server: Server, pool: list, rate_hz: float, duration_s: float, repeat_frac=0.3,
             seed=0, coefficient_jitter=0.1, rel_tol=1e-8):
    """Poisson arrivals at rate_hz for duration_s over the meshes in `pool` (MeshEntry). A
    fraction repeat_frac repeats the previous matrix of its mesh with a warm start; the rest
    carry new coefficients (the mesh's base matrix scaled per face by LogNormal(0, jitter)) and
    a new right-hand side. Returns per-request records and summary statistics."""
    rng = np.random.default_rng(seed)
    arrivals = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t > duration_s:
            break
        arrivals.append(t)
    last_key = {}
    key_counter = [0]
    records = []
    lock = threading.Lock()
    pending = []

    def waiter(ticket, meta):
        _, st, times = server.wait(ticket)
        with lock:
            records.append(dict(meta, latency=times[2] - times[0], queue=times[1] - times[0],
                                service=times[2] - times[1], iterations=st.iterations,
                                converged=st.converged, true_residual=st.true_residual))

    t0 = time.perf_counter()
    threads = []
    for ta in arrivals:
        now = time.perf_counter() - t0
        if ta > now:
            time.sleep(ta - now)
        e = pool[int(rng.integers(len(pool)))]
        repeat = e.mesh_id in last_key and rng.random() < repeat_frac
        if repeat:
            key, d, u, l, b = last_key[e.mesh_id]
            warm = True
        else:
            key_counter[0] += 1
            key = key_counter[0]
            s = np.exp(coefficient_jitter * rng.standard_normal(len(e.upper)))
            u, l = e.upper * s, e.lower * s
            d = e.diag - (e.upper - u) - (e.lower - l)
            b = rng.standard_normal(e.n)
            b -= b.mean()
            last_key[e.mesh_id] = (key, d, u, l, b)
            warm = False
        tk = server.submit(e.mesh_id, key, d, u, l, b, warm_start=warm, rel_tol=rel_tol)
        th = threading.Thread(target=waiter, args=(tk, {"mesh": e.mesh_id, "n": e.n, "warm": warm,
                                                        "arrival": ta}))
        th.start()
        threads.append(th)
    for th in threads:
        th.join()
    wall = time.perf_counter() - t0
    lat = np.array([r["latency"] for r in records])
    return records, {
        "requests": len(records), "rate_hz": rate_hz, "wall_s": wall,
        "solves_per_s": len(records) / wall if wall > 0 else 0.0,
        "p50_ms": float(np.percentile(lat, 50) * 1e3) if len(lat) else None,
        "p99_ms": float(np.percentile(lat, 99) * 1e3) if len(lat) else None,
        "mean_service_ms": float(np.mean([r["service"] for r in records]) * 1e3) if records else None,
        "all_converged": all(r["converged"] for r in records),
    }
