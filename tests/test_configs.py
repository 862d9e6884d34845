"""Seeded synthetic instance generators of the c1-c5 workloads.  CPU only."""
import numpy as np
import pytest

import oracle as O
from orctm_b200 import configs as C


def test_generators_are_deterministic():
    a = C.make_instance("c2", builder=O.build_grid, nx=20, ny=18, nz=8)
    b = C.make_instance("c2", builder=O.build_grid, nx=20, ny=18, nz=8)
    for k in ("depto", "uoo", "voe", "wno", "dvo", "avo", "zo"):
        assert np.array_equal(a[k], b[k]), k
    for x, y in zip(a["tracers"], b["tracers"]):
        assert np.array_equal(x, y)


def test_instance_seeds_differ():
    a = C.raw_instance("c4", index=0)
    b = C.raw_instance("c4", index=1)
    assert (a["nx"], a["ny"], a["nz"]) != (b["nx"], b["ny"], b["nz"]) or \
        not np.array_equal(a["depto_raw"], b["depto_raw"])


def test_config_shapes():
    for name, shape in (("c1", (512, 1, 60)), ("c2", (256, 256, 60)), ("c3", (1024, 1024, 80))):
        r = C.raw_instance(name)
        assert (r["nx"], r["ny"], r["nz"]) == shape
    for i in range(8):
        r = C.raw_instance("c4", index=i)
        assert 96 <= r["nx"] <= 512 and 96 <= r["ny"] <= 512 and 40 <= r["nz"] <= 100


def test_vertical_grids():
    dz = C.geometric_dz(60, 2.0, 1200.0)
    assert abs(dz.sum() - 1200.0) < 1e-3 and abs(dz[0] - 2.0) < 0.05
    assert np.all(np.diff(dz) > 0)


def test_land_fraction_and_open_boundaries():
    inst = C.make_instance("c2", builder=O.build_grid, nx=64, ny=64, nz=12)
    land = 1.0 - inst["weto"][1:-1, 1:-1, 0].mean()
    assert 0.08 < land < 0.25
    assert inst["ob"]["west"] and inst["ob"]["south"]
    assert inst["weto"][-1, :, 0].max() == 0      # closed east (land halo)
    assert inst["weto"][:, 0, 0].max() == 0       # closed north


def test_cfl_scaling():
    inst = C.make_instance("c2", builder=O.build_grid, nx=20, ny=18, nz=8, cfl=0.45)
    dx, dt = inst["dlxp"][0, 0], inst["dt"]
    c = max(np.abs(inst["uoo"]).max(), np.abs(inst["voe"]).max()) * dt / dx
    assert 0.3 < c <= 0.45 + 1e-12
    # velocities vanish on land faces
    assert np.all(inst["uoo"][inst["amsuo"] == 0] == 0)


@pytest.mark.parametrize("name,over", [("c4", dict(nx=48, ny=40, nz=40)),
                                       ("c2", dict(nx=30, ny=26, nz=20))])
def test_initial_vertical_courant_number_capped(name, over):
    inst = C.make_instance(name, builder=O.build_grid, **over)
    w, d, dt, ke = inst["wno"], inst["ddpo"], inst["dt"], inst["ke"]
    thin = np.where(d > 0.0, d, np.inf)
    cz = (np.abs(w[:, :, 1:ke]) * dt / np.minimum(thin[:, :, :-1], thin[:, :, 1:])).max()
    assert cz <= C.VERTICAL_CFL + 1e-12


def test_workload_state_stays_bounded():
    """Ten hot-path steps of a c4 member keep the tracers within their initial
    range: the workload respects the scheme's stability limit (an uncapped
    state of this member grew T by 1e3 per step)."""
    inst = C.make_instance("c4", index=22, builder=O.build_grid, nx=40, ny=32, nz=30)
    st = C.copy_state(inst)
    lo, hi = st["tracers"][0][inst["weto"] > 0].min(), st["tracers"][0].max()
    orc = O.Oracle(inst)
    for _ in range(10):
        orc.step_hotpath(st, solver="direct")
    t = st["tracers"][0][inst["weto"] > 0]
    assert np.isfinite(t).all()
    assert t.max() <= hi + 1e-3 and t.min() >= lo - 1e-3
