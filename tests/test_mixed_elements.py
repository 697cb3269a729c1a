"""Ragged element sets on the CPU: a mesh whose left half is quadrilaterals
and right half triangles (cells4 rows padded with -1 next to full rows).

The native mesh builder, the C restatement and the reference compiled from
its own sources (oracle/_ref) must agree bit for bit on the geometry, and the
restated time loop must reproduce the reference's over a shock-tube run, in
first order and in second order with Venkatakrishnan's limiter.
"""
import numpy as np
import pytest

import fvgpu
import meshgen
import physics as P
from cases import make_ref
from oracle import ref_available


def bits_equal(a, b):
    a = np.ascontiguousarray(a); b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def mixed_strip(nx=24, ny=6):
    """rect_tri's strip with the triangle pairs of its left half merged back
    into their quadrilaterals (node order n00, n10, n11, n01)."""
    em = meshgen.rect_tri(nx, ny, 1.0, 0.25)
    t = em.cells.reshape(ny, nx, 2, 4)
    cells = []
    for j in range(ny):
        for i in range(nx):
            a, b = t[j, i]
            if i < nx // 2:
                cells.append((a[0], a[1], a[2], b[2]))  # n00, n10, n11, n01
            else:
                cells.extend([tuple(a), tuple(b)])
    em.cells = np.ascontiguousarray(cells, dtype=np.int32)
    return em


CASE_O1 = dict(ref="forwardStep", alias={"ends": ("shockTube", "wall")}, consts=dict(cfl=0.5))
CASE_O2 = dict(ref="forwardStep_o2venk5", alias={"ends": ("shockTube", "wall")}, consts=dict(cfl=0.5))


def _physics(order2):
    return P.Physics(V=4, flux="roe_fs", order2=order2, limiter="venkat" if order2 else "zero",
                     K=5.0 if order2 else 7.5, dt_kind="cfl_sum", cfl=0.5, global_dt=True,
                     bcs={"wall": ("wall", None), "ends": ("copy", None)})


def test_mixed_mesh_native_geometry_matches_oracle(oracle):
    em = mixed_strip()
    quads = int((em.cells[:, 3] >= 0).sum())
    assert 0 < quads < em.n_cells
    m = fvgpu.Mesh.from_elements(em)
    g = m.geometry()
    o = oracle.build_mesh(em)
    assert (m.n_real, m.n_total, m.n_edges, m.n_bound) == (o.n_real, o.n_total, o.n_edges, o.n_bound)
    for k in ("edge_cells", "edge_nodes", "enx", "eny", "elen", "ecx", "ecy", "area", "ccx", "ccy",
              "bound_edges", "bound_group"):
        assert bits_equal(g[k], getattr(o, k)), k
    # Euler's formula for the planar mesh: V - E + F = 1
    assert em.nodes_x.size - m.n_edges + m.n_real == 1


@pytest.mark.skipif(not ref_available("forwardStep_o2venk5"),
                    reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("order2", [False, True])
def test_mixed_mesh_oracle_matches_reference(order2, oracle):
    em = mixed_strip()
    case = CASE_O2 if order2 else CASE_O1
    ref = make_ref(case, em)
    g = oracle.build_mesh(em)
    gr = ref.geometry()
    for k in ("edge_cells", "edge_nodes", "enx", "eny", "elen", "ecx", "ecy", "area", "ccx", "ccy",
              "bound_edges", "bound_group"):
        assert bits_equal(getattr(g, k), getattr(gr, k)), k
    p = oracle.physics(_physics(order2), em.group_names)
    q0 = P.ic_sod(g.ccx).ravel()
    steps = 25
    alpha = P.RK5_ALPHA
    a = oracle.run_loop(g, p, q0, alpha, steps)
    b = ref.run_loop(q0, alpha, steps)
    assert a["step"] == b["step"] == steps
    assert bits_equal(a["q"], b["q"])
    assert bits_equal(a["R"], b["R"]) and a["time"] == b["time"]
    assert np.all(np.isfinite(a["q"])) and not bits_equal(a["q"], q0)
