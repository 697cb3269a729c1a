"""Golden fixtures made by the reference itself (tests/golden/make_golden.py,
fvhyper's sources compiled by oracle/Makefile): the oracle restatement and
the GPU FP64_EXACT path must reproduce them bit for bit -- geometry, every
stage function on a seeded random state, and whole time loops.  These need
no fvhyper checkout, so they pin the oracle and the device path on any
machine."""
import glob
import os

import numpy as np
import pytest

import meshgen
from cases import CASES

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))
GEOM_KEYS = ("edge_cells", "edge_nodes", "enx", "eny", "elen", "ecx", "ecy", "area", "ccx", "ccy",
             "bound_edges", "bound_group")


def bits_equal(a, b):
    a = np.ascontiguousarray(a); b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def load(name):
    z = dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
    em = meshgen.ElementMesh(z["nodes_x"], z["nodes_y"], z["cells"], z["bnd_nodes"], z["bnd_group"],
                             [str(s) for s in z["group_names"]])
    return z, em, CASES[name]["phys"]()


def test_fixtures_present():
    assert set(NAMES) == {n for n in CASES if CASES[n]["ref"] is not None}


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden(name, oracle):
    z, em, ph = load(name)
    g = oracle.build_mesh(em)
    for k in GEOM_KEYS:
        assert bits_equal(getattr(g, k), z["geom_" + k].astype(getattr(g, k).dtype)), k
    p = oracle.physics(ph, em.group_names)
    q = z["stage_q"]
    assert bits_equal(oracle.calc_dt(g, p, q, False), z["stage_dt_local"])
    assert bits_equal(oracle.calc_dt(g, p, q, True), z["stage_dt_global"])
    gx, gy = oracle.gradients(g, p, q)
    assert bits_equal(gx, z["stage_gx"]) and bits_equal(gy, z["stage_gy"])
    lim = oracle.limiters(g, p, q, gx, gy)
    if ph.order2:
        assert bits_equal(lim, z["stage_lim"])
    else:
        lim = np.zeros_like(q)
        if not ph.diffusive:  # the gradients feed only the diffusive face gradient
            gx = np.zeros_like(q); gy = np.zeros_like(q)
    assert bits_equal(oracle.time_derivatives(g, p, q, gx, gy, lim), z["stage_qt"])
    assert bits_equal(oracle.update_bounds(g, p, q, gx, gy, lim), z["stage_bounds"])
    r = oracle.run_loop(g, p, z["loop_q0"], z["alpha"], int(z["steps"]))
    assert r["step"] == int(z["loop_step"]) and r["time"] == float(z["loop_time"])
    assert bits_equal(r["q"], z["loop_q"]) and bits_equal(r["R"], z["loop_R"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_reproduces_golden(name):
    import fvgpu

    z, em, ph = load(name)
    mesh = fvgpu.Mesh.from_elements(em)
    s = fvgpu.Solver(mesh, ph, "fp64_exact")
    q = z["stage_q"]
    assert bits_equal(s.stage_dt(q, False), z["stage_dt_local"])
    assert bits_equal(s.stage_dt(q, True), z["stage_dt_global"])
    if ph.order2 or ph.diffusive:
        gx, gy, lim = s.stage_gradients_limiters(q)
        assert bits_equal(gx, z["stage_gx"]) and bits_equal(gy, z["stage_gy"])
        if ph.order2:
            assert bits_equal(lim, z["stage_lim"])
        else:
            assert np.all(lim == 1.0)
    s.set_state(z["loop_q0"])
    got = s.run(int(z["steps"]), alpha=z["alpha"])
    assert got["step"] == int(z["loop_step"]) and got["time"] == float(z["loop_time"])
    assert bits_equal(s.get_state(), z["loop_q"])
    # residual norms: sums over cells, reduced in a fixed but different order
    np.testing.assert_allclose(got["R"], z["loop_R"], rtol=1e-12, atol=0)
    s.close()
