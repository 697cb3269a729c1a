"""Generates the golden fixtures in this folder from the reference itself.

Each fixture holds one small case of tests/cases.py: the element mesh, the
reference's geometry, its stage-function outputs on a seeded random state and
the state after its time loop, all produced by fvhyper's own sources compiled
by oracle/Makefile (oracle/_ref/libref_<variant>.so).  The fixtures let the
oracle and the GPU path be checked against the reference on machines that
have no fvhyper checkout.

    make -C oracle ref REF_DIR=<fvhyper checkout>
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "finite-volume-2d-cpp_b200"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)

from cases import CASES, make_ref, random_euler_state  # noqa: E402

GEOM_KEYS = ("edge_cells", "edge_nodes", "enx", "eny", "elen", "ecx", "ecy", "area", "ccx", "ccy",
             "bound_edges", "bound_group")


def make(name):
    case = CASES[name]
    em = case["mesh"]()
    ref = make_ref(case, em)
    g = ref.geometry()
    V = ref.V
    out = dict(nodes_x=em.nodes_x, nodes_y=em.nodes_y, cells=em.cells, bnd_nodes=em.bnd_nodes,
               bnd_group=em.bnd_group, group_names=np.array(em.group_names),
               alpha=np.asarray(case["alpha"], np.float64), steps=np.int64(case["steps"]))
    for k in GEOM_KEYS:
        out["geom_" + k] = getattr(g, k)
    # stage functions on a seeded random state
    if V == 4:
        q = random_euler_state(g.n_total, seed=11)
    else:
        q = np.random.default_rng(11).uniform(-1, 1, g.n_total * V)
    flags = ref.flags()
    out["stage_q"] = q
    out["stage_dt_local"] = ref.calc_dt(q, False)
    out["stage_dt_global"] = ref.calc_dt(q, True)
    gx, gy = ref.gradients(q)
    out["stage_gx"], out["stage_gy"] = gx, gy
    lim = ref.limiters(q, gx, gy) if flags["lim"] else np.zeros_like(q)
    out["stage_lim"] = lim
    if not flags["linear"]:
        lim = np.zeros_like(q)
        if not flags["diffusive"]:  # the gradients feed only the diffusive face gradient
            gx = np.zeros_like(q); gy = np.zeros_like(q)
    out["stage_qt"] = ref.time_derivatives(q, gx, gy, lim)
    out["stage_bounds"] = ref.update_bounds(q, gx, gy, lim)
    # the time loop from the example's initial condition family
    q0 = case["ic"](g)
    r = ref.run_loop(q0, case["alpha"], case["steps"])
    out["loop_q0"], out["loop_q"], out["loop_R"] = q0, r["q"], r["R"]
    out["loop_time"], out["loop_step"] = np.float64(r["time"]), np.int64(r["step"])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    return g.n_real


if __name__ == "__main__":
    for name in sorted(n for n in CASES if CASES[n]["ref"] is not None):
        print(name, make(name), "cells")
