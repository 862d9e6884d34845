"""Host side of the batch/serve API without a GPU: argument checks, the
memory estimate, request marshalling, and the node scheduler that spreads
requests over devices (NodeServer, with stand-in per-device servers)."""
import ctypes as C

import numpy as np
import pytest

from orctm_b200 import _lib, configs, grid
from orctm_b200 import serve as S


@pytest.fixture(scope="module")
def inst():
    return configs.make_instance("c4", index=1, builder=grid.build_grid, nx=20, ny=17, nz=9)


def test_estimate_grows_with_size_and_solver(inst):
    e64 = S.estimate_device_bytes(inst, "fp64")
    e32 = S.estimate_device_bytes(inst, "fp32_refined")
    assert e32 > e64 > 0
    big = dict(inst)
    big["ke"] = inst["ke"] * 2
    assert S.estimate_device_bytes(big, "fp64") > e64


def test_estimate_rejects_bad_desc(inst):
    lib = S._bind(_lib.load())
    d, keep = S.make_desc(inst)
    d.ntracers = 1
    b = C.c_ulonglong()
    assert lib.orctm_estimate_device_bytes(C.byref(d), 0, C.byref(b)) == _lib.ORCTM_E_ARG


@pytest.mark.parametrize("kw", [dict(slots=0), dict(memory_fraction=0.0),
                                dict(memory_fraction=1.5), dict(rtol=0.0), dict(maxit=0)])
def test_serve_create_rejects_bad_options(kw):
    lib = S._bind(_lib.load())
    o = S.opts(**kw)
    h = C.c_void_p()
    assert lib.orctm_serve_create(C.byref(o), C.byref(h)) == _lib.ORCTM_E_ARG


def test_serve_create_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = S._bind(_lib.load())
    h = C.c_void_p()
    assert lib.orctm_serve_create(C.byref(S.opts()), C.byref(h)) == -7  # ORCTM_E_NODEVICE


def test_job_marshalling(inst):
    st = configs.copy_state(inst)
    j = S.Job(inst, st, nsteps=4)
    r = j.req
    assert r.nsteps == 4 and r.nin == 13 + len(st["tracers"])
    ids = [r.in_fields[k] for k in range(r.nin)]
    assert sorted(ids) == sorted(set(ids))
    # outputs: uoo, voe, wno, pnh and every tracer, in the reference layouts
    assert r.nout == 4 + inst["ntracers"]
    assert j.out["uoo"].shape == (inst["ie"] + 1, inst["je"], inst["ke"])
    assert j.out["voe"].shape == (inst["ie"], inst["je"] + 1, inst["ke"])
    assert j.out["wno"].shape == (inst["ie"], inst["je"], inst["ke"] + 1)
    assert j.out["pnh"].shape == (inst["ie"], inst["je"], inst["ke"])
    assert j.out["uoo"].flags.f_contiguous
    # the input pointers address the job's own Fortran-ordered copies
    a = np.ctypeslib.as_array(r.in_data[0], shape=(st["uoo"].size,))
    assert np.array_equal(a, st["uoo"].ravel(order="F"))
    out = j.outputs()
    assert len(out["tracers"]) == inst["ntracers"]


def test_serve_submit_rejects_bad_request():
    lib = S._bind(_lib.load())
    assert lib.orctm_serve_submit(None, None, None) == _lib.ORCTM_E_ARG


class _FakeServer:
    """Stands in for one device's Server: records submissions; a request is
    done once the test says so."""

    def __init__(self, device, **kw):
        self.device, self.kw = device, kw
        self.jobs, self.done, self.waited = [], set(), []
        self.closed = False

    def submit(self, job):
        self.jobs.append(job)
        return job

    def poll(self, job):
        if id(job) in self.done:
            self.done.discard(id(job))
            self.jobs.remove(job)
            return True
        return False

    def wait(self, job):
        self.waited.append(job)
        self.jobs.remove(job)
        return job

    def drain(self):
        pass

    def stats(self):
        return {"submitted": len(self.jobs), "completed": 0, "failed": 0, "steps": 0,
                "cell_steps": 0.0}

    def close(self):
        self.closed = True


def _job(cells, nsteps=1):
    from types import SimpleNamespace

    return SimpleNamespace(cells=cells, req=SimpleNamespace(nsteps=nsteps))


def test_pick_device_least_outstanding_lowest_on_ties():
    assert S.pick_device([0, 0, 0]) == 0
    assert S.pick_device([5, 2, 2]) == 1
    assert S.pick_device([3, 7, 1, 1]) == 2


def test_node_server_spreads_by_outstanding_work():
    node = S.NodeServer(devices=[0, 1, 2], server=_FakeServer, slots=4)
    assert [s.device for s in node.servers] == [0, 1, 2]
    assert all(s.kw == {"slots": 4} for s in node.servers)
    big, mid, small = _job(100, 10), _job(50, 10), _job(30, 10)
    for j in (big, mid, small):
        node.submit(j)
    assert (big.device, mid.device, small.device) == (0, 1, 2)
    assert node.outstanding == [1000, 500, 300]
    nxt = node.submit(_job(10, 10))              # the least loaded: device 2
    assert nxt.device == 2 and node.outstanding == [1000, 500, 400]
    # device 0's request finishes: seen at the next submission, which goes there
    node.servers[0].done.add(id(big))
    after = node.submit(_job(20, 10))
    assert after.device == 0 and node.outstanding == [200, 500, 400]
    assert node.poll(big) and node.wait(big) is big   # already seen done
    assert node.servers[0].waited == []
    node.wait(mid)                               # blocks on device 1's server
    assert node.servers[1].waited == [mid] and node.outstanding == [200, 0, 400]
    assert node.stats()["submitted"] == 3
    node.close()
    assert all(s.closed for s in node.servers)


def test_node_server_needs_a_device():
    with pytest.raises(ValueError):
        S.NodeServer(devices=[], server=_FakeServer)

