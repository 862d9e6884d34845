"""Batched and served execution on the GPU: every instance's result is the
same, bit for bit, alone and in the mix; admission respects the memory
budget; a failing request does not disturb the others."""
import time

import numpy as np
import pytest

from orctm_b200 import _lib
from orctm_b200 import configs as C
from orctm_b200 import grid
from orctm_b200.api import Instance
from orctm_b200.serve import Job, NodeServer, Server, estimate_device_bytes, run_batch

pytestmark = pytest.mark.gpu

SPECS = [dict(nx=40, ny=33, nz=24), dict(nx=57, ny=21, nz=31), dict(nx=33, ny=48, nz=17),
         dict(nx=64, ny=64, nz=40)]
OUT = ("uoo", "voe", "wno", "pnh")


@pytest.fixture(scope="module")
def insts():
    return [C.make_instance("c4", index=k, builder=grid.build_grid, **sp)
            for k, sp in enumerate(SPECS)]


def _alone(inst, nsteps, solver):
    gpu = Instance(inst)
    gpu.upload_state(C.copy_state(inst))
    gpu.set_solver(solver, rtol=1e-10, maxit=5000)
    for _ in range(nsteps):
        gpu.step_hotpath()
    out = {k: gpu.download(k) for k in OUT}
    out["tracers"] = [gpu.download(f"tracer{n}") for n in range(gpu.ntr)]
    gpu.close()
    return out


def _same(a, b):
    for k in OUT:
        assert np.array_equal(a[k], b[k]), k
    assert len(a["tracers"]) == len(b["tracers"])
    for x, y in zip(a["tracers"], b["tracers"]):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("solver", ["fp64", "fp32_refined"])
def test_served_results_equal_alone(insts, solver):
    nsteps = 3
    alone = [_alone(i, nsteps, solver) for i in insts]
    with Server(slots=4, solver=solver, rtol=1e-10, maxit=5000) as srv:
        first = [srv.submit(Job(i, C.copy_state(i), nsteps)) for i in insts]
        # a second wave arrives while the first is on the device
        second = [srv.submit(Job(i, C.copy_state(i), nsteps)) for i in insts[::-1]]
        for j in first + second:
            srv.wait(j)
            assert j.stats["status"] == 0, j.stats
            assert j.stats["steps_done"] == nsteps
            assert j.stats["relres_max"] <= 1e-10
        st = srv.stats()
    assert st["completed"] == 8 and st["failed"] == 0
    assert st["steps"] == 8 * nsteps
    assert st["peak_in_flight"] >= 2
    assert st["step_ms_p99"] >= st["step_ms_p50"] > 0
    for k, j in enumerate(first):
        _same(j.outputs(), alone[k])
    for k, j in enumerate(second):
        _same(j.outputs(), alone[len(insts) - 1 - k])


def test_node_server_equals_alone(insts):
    """The node scheduler over this box's GPUs (one per call here): every
    request lands on a device and its result is the one alone."""
    nsteps = 2
    with NodeServer(slots=3, solver="fp64", rtol=1e-10, maxit=5000) as node:
        jobs = [node.submit(Job(i, C.copy_state(i), nsteps)) for i in insts]
        node.drain()
        for j in jobs:
            node.wait(j)
            assert j.stats["status"] == 0, j.stats
        st = node.stats()
    assert st["completed"] == len(insts) and st["failed"] == 0
    assert all(j.device in node.devices for j in jobs)
    for j, i in zip(jobs, insts):
        _same(j.outputs(), _alone(i, nsteps, "fp64"))


def test_batch_equals_alone(insts):
    nsteps = 2
    jobs = [Job(i, C.copy_state(i), nsteps) for i in insts]
    tot = run_batch(jobs, slots=len(jobs), solver="fp64")
    assert tot["completed"] == len(jobs)
    assert tot["cell_steps"] == sum(j.cells for j in jobs) * nsteps
    for j, i in zip(jobs, insts):
        _same(j.outputs(), _alone(i, nsteps, "fp64"))


@pytest.mark.parametrize("solver", ["fp64", "fp32_refined"])
def test_memory_estimate_bounds_use(insts, solver):
    inst = insts[3]
    gpu = Instance(inst)
    gpu.upload_state(C.copy_state(inst))
    gpu.set_solver(solver, rtol=1e-10, maxit=5000)
    gpu.step_hotpath()
    gpu.step_hotpath()
    used = gpu.device_bytes()
    gpu.close()
    est = estimate_device_bytes(inst, solver)
    assert used <= est <= 1.5 * used, (used, est)


def test_admission_against_budget(insts):
    # a budget below one instance: requests run one at a time
    with Server(slots=4, memory_fraction=1e-9) as srv:
        jobs = [srv.submit(Job(i, C.copy_state(i), 1)) for i in insts]
        for j in jobs:
            srv.wait(j)
            assert j.stats["status"] == 0
        st = srv.stats()
    assert st["peak_in_flight"] == 1
    assert st["completed"] == len(insts)


def test_failed_request_is_isolated(insts):
    nsteps = 2
    with Server(slots=3) as srv:
        good = [srv.submit(Job(i, C.copy_state(i), nsteps)) for i in insts[:2]]
        early = Job(insts[2], C.copy_state(insts[2]), nsteps)
        early.desc.ntracers = 1  # rejected at submission (no memory estimate)
        with pytest.raises(_lib.OrctmError):
            srv.submit(early)
        bad = Job(insts[2], C.copy_state(insts[2]), nsteps)
        bad.desc.dt = -1.0  # admitted, then rejected by orctm_create in its slot
        srv.submit(bad)
        for j in good:
            srv.wait(j)
        while not srv.poll(bad):
            time.sleep(0.001)
        st = srv.stats()
    assert bad.stats["status"] == -1 and bad.stats["steps_done"] == 0
    assert st["failed"] == 1 and st["completed"] == 2
    for j, i in zip(good, insts[:2]):
        _same(j.outputs(), _alone(i, nsteps, "fp64"))
