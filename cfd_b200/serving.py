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
                ("settings", AmgSettingsStruct), ("max_age", _i), ("pdl", _i),
                ("mixed_sweeps", _i), ("mixed_weight", _d), ("background_rebuild", _i), ("schedule", _i)]


class ServerInfoStruct(C.Structure):
    _fields_ = [("resident_systems", _i), ("resident_bytes", _d), ("queued", _i),
                ("completed", _ll), ("evictions", _ll), ("rebuilds", _ll), ("background_rebuilds", _ll)]


def _p(name, args, res=_i):
    f = getattr(_lib, name)
    f.argtypes = args
    f.restype = res


_p("cfdb_default_server_config", [C.POINTER(ServerConfigStruct)], None)
_p("cfdb_server_create", [C.POINTER(ServerConfigStruct), C.POINTER(_vp)])
_p("cfdb_server_destroy", [_vp])
_p("cfdb_server_add_mesh", [_vp, _i, _i, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)])
_p("cfdb_server_submit", [_vp, _i, _ll, _pd, _pd, _pd, _pd, _pd, _i, _d, _i, C.POINTER(_ll)])
_p("cfdb_server_wait", [_vp, _ll, C.POINTER(StatsStruct), _pd])
_p("cfdb_server_info", [_vp, C.POINTER(ServerInfoStruct)])


class Server:
    def __init__(self, slots=4, hbm_budget_bytes=150e9, precision=Precision.MIXED,
                 settings: AmgSettings | None = None, max_age=0, pdl=0, mixed_schedule=None,
                 background_rebuild=False, schedule="fifo"):
        cfg = ServerConfigStruct()
        _lib.cfdb_default_server_config(C.byref(cfg))
        cfg.slots, cfg.hbm_budget_bytes, cfg.precision = int(slots), float(hbm_budget_bytes), int(precision)
        cfg.settings = (settings or AmgSettings())._c()
        cfg.max_age = int(max_age)
        cfg.pdl = int(pdl)
        if mixed_schedule is not None:  # (sweeps, weight) of the mixed V-cycle
            cfg.mixed_sweeps, cfg.mixed_weight = int(mixed_schedule[0]), float(mixed_schedule[1])
        cfg.background_rebuild = 1 if background_rebuild else 0
        cfg.schedule = {"fifo": 0, "most_work": 1}[schedule]
        h = _vp()
        _check(_lib.cfdb_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self.meshes = {}
        self._borrowed = {}

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

    def submit(self, mesh_id, matrix_key, diag, upper, lower, rhs, x=None, warm_start=False,
               rel_tol=1e-8, max_iterations=500) -> int:
        """Queues a solve. The arrays are borrowed until wait(ticket) returns (the server keeps
        references); x (float64, n_cells) receives the solution, a new array when omitted."""
        n, nf = self.meshes[mesh_id]
        diag, upper, lower, rhs = _f64(diag), _f64(upper), _f64(lower), _f64(rhs)
        if len(diag) != n or len(rhs) != n or len(upper) != nf or len(lower) != nf:
            raise InvalidArgument("request arrays do not match the mesh")
        if x is None:
            x = np.zeros(n)
        elif not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous
                  and x.size == n):
            raise InvalidArgument("x must be a contiguous float64 array of n_cells")
        t = _ll()
        _check(_lib.cfdb_server_submit(self._h, int(mesh_id), int(matrix_key), _dp(diag),
                                       _dp(upper), _dp(lower), _dp(rhs), _dp(x),
                                       1 if warm_start else 0, float(rel_tol),
                                       int(max_iterations), C.byref(t)))
        self._borrowed[t.value] = (diag, upper, lower, rhs, x)
        return t.value

    def wait(self, ticket):
        """(x, SolveStats, (submit, start, finish) seconds since the server started)."""
        st = StatsStruct()
        times = (C.c_double * 3)()
        try:
            _check(_lib.cfdb_server_wait(self._h, int(ticket), C.byref(st), times))
        finally:
            arrays = self._borrowed.pop(ticket, None)
        return arrays[4], SolveStats._from(st), (times[0], times[1], times[2])

    def info(self) -> dict:
        i = ServerInfoStruct()
        _check(_lib.cfdb_server_info(self._h, C.byref(i)))
        return {"resident_systems": i.resident_systems, "resident_bytes": i.resident_bytes,
                "queued": i.queued, "completed": i.completed, "evictions": i.evictions,
                "rebuilds": i.rebuilds, "background_rebuilds": i.background_rebuilds}


def _pinned(shape_or_array):
    """Page-locked float64 numpy array (a copy of the array given, or zeros of a length)."""
    import torch
    if isinstance(shape_or_array, int):
        return torch.zeros(shape_or_array, dtype=torch.float64).pin_memory().numpy()
    a = np.ascontiguousarray(shape_or_array, dtype=np.float64)
    return torch.from_numpy(a.copy()).pin_memory().numpy()


@dataclass
class MeshEntry:
    """One pooled mesh: its server id, kind, size and page-locked request data: `variants`
    coefficient sets (diag, upper, lower) and right-hand sides."""
    mesh_id: int
    kind: str
    n: int
    matrices: list
    rhs: list
    free_x: list


def make_pool(server: Server, pool_cases, variants=3, seed=0, coefficient_jitter=0.1,
              x_buffers=4):
    """Registers the meshes of `pool_cases` [(kind, case, diag, upper, lower, source)] and
    prepares page-locked coefficient variants: the finalized matrix with its face coefficients
    scaled by LogNormal(0, coefficient_jitter) (diagonal adjusted so row sums are kept) and
    zero-mean random right-hand sides; `x_buffers` page-locked solution buffers per mesh (run_load
    adds more before its clock starts when its trace can have more requests of one mesh in
    flight)."""
    rng = np.random.default_rng(seed)
    pool = []
    for kind, c, d, u, l, b in pool_cases:
        mid = server.add_mesh(c.n, c.owner, c.neighbour)
        mats, rhs = [], []
        for v in range(variants):
            if v == 0:
                dv, uv, lv = d, u, l
            else:
                sc = np.exp(coefficient_jitter * rng.standard_normal(len(u)))
                uv, lv = u * sc, l * sc
                dv = d.copy()
                np.add.at(dv, c.owner, -(uv - u))
                np.add.at(dv, c.neighbour, -(lv - l))
            mats.append((_pinned(dv), _pinned(uv), _pinned(lv)))
            r = b if v == 0 else rng.standard_normal(c.n)
            rhs.append(_pinned(r - r.mean()))
        pool.append(MeshEntry(mid, kind, c.n, mats, rhs, [_pinned(c.n) for _ in range(x_buffers)]))
    return pool


def request_trace(pool: list, rate_hz: float, n_requests: int, repeat_frac=0.3, tet_frac=0.25, seed=0,
                  closed_loop=False):
    """The requests run_load submits, drawn from `seed` before any clock starts: a list of
    (arrival s, pool entry, matrix key, variant, right-hand side, repeat). A request picks tet
    meshes with probability tet_frac, then a pool mesh of that kind uniformly; with probability
    repeat_frac it repeats its mesh's previous key and variant, otherwise it carries the next
    key and the variant key % variants. Arrivals are Poisson at rate_hz (all 0 in a closed
    loop). The same arguments give the same trace."""
    rng = np.random.default_rng(seed)
    by_kind = {}
    for e in pool:
        by_kind.setdefault(e.kind, []).append(e)
    kinds = sorted(by_kind)
    last = {}
    key_counter = 0
    trace = []
    ta = 0.0
    for _ in range(n_requests):
        if not closed_loop:
            ta += rng.exponential(1.0 / rate_hz)
        kind = "tet" if ("tet" in by_kind and rng.random() < tet_frac) else \
            ("box" if "box" in by_kind else kinds[0])
        group = by_kind[kind]
        e = group[int(rng.integers(len(group)))]
        rep = e.mesh_id in last and rng.random() < repeat_frac
        if rep:
            key, mi = last[e.mesh_id]
        else:
            key_counter += 1
            key = key_counter
            mi = key % len(e.matrices)
            last[e.mesh_id] = (key, mi)
        bi = int(rng.integers(len(e.rhs)))
        trace.append((ta, e, key, mi, bi, bool(rep)))
    return trace


def run_load(server: Server, pool: list, rate_hz: float, n_requests: int, repeat_frac=0.3,
             tet_frac=0.25, seed=0, rel_tol=1e-8, closed_loop=False, warm_start=True):
    """Open-loop Poisson arrivals at rate_hz (closed_loop: each request submitted when the
    previous one finished) of the n_requests of request_trace over the pool. A repeat carries
    its mesh's previous matrix (same key: no re-upload) with a new right-hand side and, if
    warm_start, starts from the resident solution. Latency = finish - submit on the server
    clock."""
    import queue as _q
    records = []
    pending = _q.Queue()
    lock = threading.Lock()

    def collector():
        while True:
            item = pending.get()
            if item is None:
                return
            ticket, e, x, meta = item
            _, st, times = server.wait(ticket)
            with lock:
                e.free_x.append(x)
                records.append(dict(meta, latency=times[2] - times[0], queue=times[1] - times[0],
                                    service=times[2] - times[1], iterations=st.iterations,
                                    converged=st.converged, residual=st.residual))

    # the request trace, drawn before the clock starts, and enough page-locked solution buffers
    # for every request of a mesh to be in flight at once, so that no buffer is page-locked
    # while the server runs
    trace = request_trace(pool, rate_hz, n_requests, repeat_frac, tet_frac, seed, closed_loop)
    if not closed_loop:
        need = {}
        for _, e, *_ in trace:
            need[e.mesh_id] = need.get(e.mesh_id, 0) + 1
        for e in pool:
            while len(e.free_x) < need.get(e.mesh_id, 0):
                e.free_x.append(_pinned(e.n))
    th = threading.Thread(target=collector, daemon=True)
    th.start()
    t0 = time.perf_counter()
    for i, (ta, e, key, mi, bi, rep) in enumerate(trace):
        if not closed_loop:
            now = time.perf_counter() - t0
            if ta > now:
                time.sleep(ta - now)
        d, u, l = e.matrices[mi]
        with lock:
            x = e.free_x.pop() if e.free_x else _pinned(e.n)
        ticket = server.submit(e.mesh_id, key, d, u, l, e.rhs[bi], x=x,
                               warm_start=bool(rep and warm_start), rel_tol=rel_tol)
        # host-to-device bytes of the request: the matrix unless it repeats the resident key,
        # and the right-hand side; the solution comes back
        h2d = 8 * (e.n + (0 if rep else len(d) + len(u) + len(l)))
        pending.put((ticket, e, x, {"mesh": e.mesh_id, "kind": e.kind, "n": e.n,
                                    "repeat": rep, "h2d": h2d, "d2h": 8 * e.n}))
        if closed_loop:
            while True:
                with lock:
                    if len(records) == i + 1:
                        break
                time.sleep(0.0002)
    pending.put(None)
    th.join()
    wall = time.perf_counter() - t0
    lat = np.array([r["latency"] for r in records])
    cells = sum(r["n"] for r in records)
    return records, {
        "requests": len(records), "rate_hz": None if closed_loop else rate_hz,
        "closed_loop": closed_loop, "wall_s": wall,
        "solves_per_s": len(records) / wall if wall > 0 else 0.0,
        "mcells_per_s": cells / wall / 1e6 if wall > 0 else 0.0,
        "p50_ms": float(np.percentile(lat, 50) * 1e3) if len(lat) else None,
        "p99_ms": float(np.percentile(lat, 99) * 1e3) if len(lat) else None,
        "mean_service_ms": float(np.mean([r["service"] for r in records]) * 1e3) if records else None,
        "repeat_frac": float(np.mean([r["repeat"] for r in records])) if records else None,
        "mean_iterations": float(np.mean([r["iterations"] for r in records])) if records else None,
        "all_converged": all(r["converged"] for r in records),
        "h2d_gbs": sum(r["h2d"] for r in records) / wall / 1e9 if wall > 0 else 0.0,
        "d2h_gbs": sum(r["d2h"] for r in records) / wall / 1e9 if wall > 0 else 0.0,
        "mean_h2d_mb": float(np.mean([r["h2d"] for r in records]) / 1e6) if records else None,
    }
