"""Batched and served execution of independent instances (the orctm_serve_*
and orctm_batch_run entry points of liborctm_gpu.so).

``Server`` admits requests as slots and device memory free up (continuous
batching at step granularity: every admitted instance advances on its own
slot thread and stream, and the device runs the slots' kernels
concurrently); ``run_batch`` submits a whole ensemble at once;
``NodeServer`` spreads requests over the GPUs of a node, one ``Server`` per
device behind a least-outstanding-work scheduler.  Inputs are
instance dicts and state dicts of orctm_b200.configs; outputs come back as
numpy arrays in the reference's layouts.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .api import FIELDS, SHAPES, field_id, make_desc

_D = C.POINTER(C.c_double)


class ServeOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("slots", C.c_int), ("memory_fraction", C.c_double),
                ("solver", C.c_int), ("rtol", C.c_double), ("maxit", C.c_int)]


class Request(C.Structure):
    _fields_ = [("desc", C.POINTER(_lib.Desc)), ("nsteps", C.c_int),
                ("nin", C.c_int), ("in_fields", C.POINTER(C.c_int)), ("in_data", C.POINTER(_D)),
                ("nout", C.c_int), ("out_fields", C.POINTER(C.c_int)),
                ("out_data", C.POINTER(_D))]


class RequestStats(C.Structure):
    _fields_ = [("status", C.c_int), ("steps_done", C.c_int), ("iterations", C.c_int),
                ("relres_max", C.c_double), ("queued_ms", C.c_double), ("run_ms", C.c_double),
                ("step_ms_p50", C.c_double), ("step_ms_p99", C.c_double),
                ("step_ms_max", C.c_double), ("device_bytes", C.c_ulonglong),
                ("estimated_bytes", C.c_ulonglong)]


class ServeStats(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong),
                ("failed", C.c_longlong), ("steps", C.c_longlong), ("cell_steps", C.c_double),
                ("elapsed_ms", C.c_double), ("step_ms_p50", C.c_double),
                ("step_ms_p99", C.c_double), ("peak_in_flight", C.c_int),
                ("peak_reserved_bytes", C.c_ulonglong), ("budget_bytes", C.c_ulonglong)]


def _bind(lib):
    if getattr(lib, "_serve_bound", False):
        return lib
    lib.orctm_serve_create.argtypes = [C.POINTER(ServeOpts), C.POINTER(C.c_void_p)]
    lib.orctm_serve_submit.argtypes = [C.c_void_p, C.POINTER(Request), C.POINTER(C.c_ulonglong)]
    lib.orctm_serve_wait.argtypes = [C.c_void_p, C.c_ulonglong, C.POINTER(RequestStats)]
    lib.orctm_serve_poll.argtypes = [C.c_void_p, C.c_ulonglong, C.POINTER(C.c_int),
                                     C.POINTER(RequestStats)]
    lib.orctm_serve_drain.argtypes = [C.c_void_p]
    lib.orctm_serve_get_stats.argtypes = [C.c_void_p, C.POINTER(ServeStats)]
    lib.orctm_serve_destroy.argtypes = [C.c_void_p]
    lib.orctm_batch_run.argtypes = [C.POINTER(ServeOpts), C.c_int, C.POINTER(Request),
                                    C.POINTER(RequestStats), C.POINTER(ServeStats)]
    lib.orctm_estimate_device_bytes.argtypes = [C.POINTER(_lib.Desc), C.c_int,
                                                C.POINTER(C.c_ulonglong)]
    lib._serve_bound = True
    return lib


def _solver_id(solver: str) -> int:
    return {"fp64": _lib.SOLVER_FP64, "fp32_refined": _lib.SOLVER_FP32_REFINED}[solver]


def opts(device=0, slots=8, memory_fraction=0.9, solver="fp64", rtol=1e-10, maxit=5000):
    return ServeOpts(device, slots, memory_fraction, _solver_id(solver), rtol, maxit)


def _struct(s) -> dict:
    return {k: getattr(s, k) for k, _ in s._fields_}


def _shape(inst, name):
    ie, je, ke = inst["ie"], inst["je"], inst["ke"]
    kind = "p" if name.startswith("tracer") else SHAPES[name]
    return {"p": (ie, je, ke), "u": (ie + 1, je, ke), "v": (ie, je + 1, ke),
            "w": (ie, je, ke + 1), "2": (ie, je)}[kind]


class Job:
    """One request and the host arrays it refers to (kept alive until done)."""

    def __init__(self, inst: dict, state: dict, nsteps: int,
                 outputs=("uoo", "voe", "wno", "pnh", "tracers")):
        self.desc, self._keep = make_desc(inst)
        names_in = [k for k in FIELDS if k in state]
        names_in += [f"tracer{n}" for n in range(len(state.get("tracers", [])))]
        arrs_in = [np.asfortranarray(state[k] if not k.startswith("tracer")
                                     else state["tracers"][int(k[6:])], dtype=np.float64)
                   for k in names_in]
        ntr = self.desc.ntracers
        names_out = []
        for k in outputs:
            names_out += [f"tracer{n}" for n in range(ntr)] if k == "tracers" else [k]
        self.out = {k: np.zeros(_shape(inst, k), dtype=np.float64, order="F") for k in names_out}
        self._in = arrs_in
        self._in_ids = (C.c_int * len(names_in))(*[field_id(k) for k in names_in])
        self._in_ptr = (_D * len(arrs_in))(*[a.ctypes.data_as(_D) for a in arrs_in])
        self._out_ids = (C.c_int * len(names_out))(*[field_id(k) for k in names_out])
        self._out_ptr = (_D * len(names_out))(*[self.out[k].ctypes.data_as(_D)
                                                for k in names_out])
        self.req = Request(C.pointer(self.desc), nsteps, len(names_in), self._in_ids, self._in_ptr,
                           len(names_out), self._out_ids, self._out_ptr)
        self.cells = (inst["ie"] - 2) * (inst["je"] - 2) * inst["ke"]
        self.id = None
        self.stats = None

    def outputs(self) -> dict:
        out = {k: v for k, v in self.out.items() if not k.startswith("tracer")}
        tr = sorted((int(k[6:]), v) for k, v in self.out.items() if k.startswith("tracer"))
        if tr:
            out["tracers"] = [v for _, v in tr]
        return out


class Server:
    """A served loop on one device (orctm_serve_*)."""

    def __init__(self, **kw):
        self.lib = _bind(_lib.load())
        self.opts = opts(**kw)
        h = C.c_void_p()
        _lib.check(self.lib.orctm_serve_create(C.byref(self.opts), C.byref(h)))
        self.h = h
        self.jobs = {}

    def submit(self, job: Job) -> Job:
        i = C.c_ulonglong()
        _lib.check(self.lib.orctm_serve_submit(self.h, C.byref(job.req), C.byref(i)))
        job.id = i.value
        self.jobs[job.id] = job
        return job

    def wait(self, job: Job) -> Job:
        s = RequestStats()
        _lib.check(self.lib.orctm_serve_wait(self.h, job.id, C.byref(s)))
        job.stats = _struct(s)
        self.jobs.pop(job.id, None)
        return job

    def poll(self, job: Job) -> bool:
        s, done = RequestStats(), C.c_int()
        _lib.check(self.lib.orctm_serve_poll(self.h, job.id, C.byref(done), C.byref(s)))
        if done.value:
            job.stats = _struct(s)
            self.jobs.pop(job.id, None)
        return bool(done.value)

    def drain(self):
        _lib.check(self.lib.orctm_serve_drain(self.h))

    def stats(self) -> dict:
        s = ServeStats()
        _lib.check(self.lib.orctm_serve_get_stats(self.h, C.byref(s)))
        return _struct(s)

    def close(self):
        if getattr(self, "h", None):
            self.lib.orctm_serve_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pick_device(outstanding) -> int:
    """The index of the device with the least outstanding work (ties: the
    lowest index)."""
    return min(range(len(outstanding)), key=lambda k: (outstanding[k], k))


class NodeServer:
    """An ensemble's requests spread over the GPUs of one node: one Server
    per device, each with its own slots, admission and memory budget, behind
    a host scheduler that sends every request to the device with the least
    outstanding work (the cell-steps of its requests not yet seen done).
    The instances are independent, so nothing crosses between devices and
    there is no collective.  ``server`` builds the per-device servers (the
    tests pass a stand-in)."""

    def __init__(self, devices=None, server=Server, **kw):
        if devices is None:
            import torch

            devices = list(range(torch.cuda.device_count()))
        if not devices:
            raise ValueError("NodeServer: no device")
        self.devices = list(devices)
        self.servers = [server(device=d, **kw) for d in self.devices]
        self.outstanding = [0] * len(self.devices)
        self._where = {}      # id(job) -> (server index, work, job)
        self._seen_done = set()

    def _finished(self, key):
        k, work, _ = self._where.pop(key)
        self.outstanding[k] -= work

    def _refresh(self):
        for key, (k, _, job) in list(self._where.items()):
            if key not in self._seen_done and self.servers[k].poll(job):
                self._seen_done.add(key)
                self._finished(key)

    def submit(self, job: Job) -> Job:
        self._refresh()
        k = pick_device(self.outstanding)
        self.servers[k].submit(job)
        work = job.cells * job.req.nsteps
        self.outstanding[k] += work
        self._where[id(job)] = (k, work, job)
        job.device = self.devices[k]
        return job

    def poll(self, job: Job) -> bool:
        key = id(job)
        if key in self._seen_done:
            return True
        k = self._where[key][0]
        if self.servers[k].poll(job):
            self._seen_done.add(key)
            self._finished(key)
            return True
        return False

    def wait(self, job: Job) -> Job:
        key = id(job)
        if key not in self._seen_done:
            self.servers[self._where[key][0]].wait(job)
            self._seen_done.add(key)
            self._finished(key)
        return job

    def drain(self):
        for srv in self.servers:
            srv.drain()

    def stats(self) -> dict:
        per = [srv.stats() for srv in self.servers]
        total = {k: sum(p[k] for p in per)
                 for k in ("submitted", "completed", "failed", "steps", "cell_steps")
                 if all(k in p for p in per)}
        return {"devices": dict(zip(self.devices, per)), **total}

    def close(self):
        for srv in self.servers:
            srv.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def run_batch(jobs: list, **kw) -> dict:
    """Runs the jobs submitted together (orctm_batch_run); fills each job's
    outputs and stats and returns the batch totals."""
    lib = _bind(_lib.load())
    o = opts(**kw)
    n = len(jobs)
    reqs = (Request * n)(*[j.req for j in jobs])
    per = (RequestStats * n)()
    tot = ServeStats()
    st = lib.orctm_batch_run(C.byref(o), n, reqs, per, C.byref(tot))
    for j, s in zip(jobs, per):
        j.stats = _struct(s)
    _lib.check(st)
    return _struct(tot)


def estimate_device_bytes(inst: dict, solver="fp64") -> int:
    lib = _bind(_lib.load())
    d, keep = make_desc(inst)
    b = C.c_ulonglong()
    _lib.check(lib.orctm_estimate_device_bytes(C.byref(d), _solver_id(solver), C.byref(b)))
    del keep
    return int(b.value)
