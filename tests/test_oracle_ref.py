"""Pin the C restatement (oracle/fvoracle.c) against the reference compiled
from its own sources (oracle/_ref).  Everything must agree bit for bit:
geometry, every stage function and whole runs of the time loop."""
import numpy as np
import pytest

import meshgen
from cases import CASES, make_ref, random_euler_state
from oracle import ref_available

pytestmark = pytest.mark.skipif(not ref_available("naca"),
                                reason="oracle/_ref not built (needs the reference sources)")


def bits_equal(a, b):
    a = np.ascontiguousarray(a); b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def _setup(name, oracle):
    case = CASES[name]
    em = case["mesh"]()
    ref = make_ref(case, em)
    g = oracle.build_mesh(em)
    ph = case["phys"]()
    p = oracle.physics(ph, em.group_names)
    return case, em, ref, g, ph, p


REF_CASES = sorted(n for n in CASES if CASES[n]["ref"] is not None)


@pytest.mark.parametrize("name", REF_CASES)
def test_geometry_bitwise(name, oracle):
    case, em, ref, g, ph, p = _setup(name, oracle)
    gr = ref.geometry()
    for k in ("edge_cells", "edge_nodes", "enx", "eny", "elen", "ecx", "ecy", "area", "ccx", "ccy",
              "bound_edges", "bound_group"):
        assert bits_equal(getattr(g, k), getattr(gr, k)), k


@pytest.mark.parametrize("name", REF_CASES)
def test_stage_functions_bitwise(name, oracle):
    case, em, ref, g, ph, p = _setup(name, oracle)
    if ph.V == 4:
        q = random_euler_state(g.n_total, seed=11)
    else:
        q = np.random.default_rng(11).uniform(-1, 1, g.n_total * ph.V)
    flags = ref.flags()
    assert bits_equal(oracle.calc_dt(g, p, q, False), ref.calc_dt(q, False))
    assert bits_equal(oracle.calc_dt(g, p, q, True), ref.calc_dt(q, True))
    gx, gy = oracle.gradients(g, p, q)
    rgx, rgy = ref.gradients(q)
    assert bits_equal(gx, rgx) and bits_equal(gy, rgy)
    lim = oracle.limiters(g, p, q, gx, gy)
    if flags["lim"]:  # first-order cases never call limiter_func
        assert bits_equal(lim, ref.limiters(q, gx, gy))
    if not flags["linear"]:
        lim = np.zeros_like(q)
        if not flags["diffusive"]:  # the gradients feed only the diffusive face gradient
            gx = np.zeros_like(q); gy = np.zeros_like(q)
    assert bits_equal(oracle.time_derivatives(g, p, q, gx, gy, lim), ref.time_derivatives(q, gx, gy, lim))
    assert bits_equal(oracle.update_bounds(g, p, q, gx, gy, lim), ref.update_bounds(q, gx, gy, lim))


@pytest.mark.parametrize("name", REF_CASES)
def test_time_loop_bitwise(name, oracle):
    case, em, ref, g, ph, p = _setup(name, oracle)
    q0 = case["ic"](g)
    a = oracle.run_loop(g, p, q0, case["alpha"], case["steps"])
    b = ref.run_loop(q0, case["alpha"], case["steps"])
    assert a["step"] == b["step"] == case["steps"]
    assert bits_equal(a["q"], b["q"])
    assert bits_equal(a["R"], b["R"]) and a["time"] == b["time"]
    assert np.all(np.isfinite(a["q"]))


@pytest.mark.parametrize("name", ["naca", "step_o1", "burgers"])
def test_loop_equals_reference_run(name, oracle):
    """The restated loop with the 5-stage set reproduces fvhyper::run itself
    (explicit.cpp:657-817, example initial condition and hard-coded RK5)."""
    case, em, ref, g, ph, p = _setup(name, oracle)
    q_run = ref.run(max_step=12, verbose=False)
    a = oracle.run_loop(g, p, ref.initial_state(), case["alpha"], 12)
    assert bits_equal(a["q"], q_run)


def test_time_and_tolerance_stops(oracle):
    """max_time and tolerance stops follow explicit.cpp:717-726 (time += dt[0])."""
    case, em, ref, g, ph, p = _setup("sod", oracle)
    q0 = case["ic"](g)
    a = oracle.run_loop(g, p, q0, case["alpha"], 10 ** 6, max_time=0.02)
    b = ref.run_loop(q0, case["alpha"], 10 ** 6, max_time=0.02)
    assert a["step"] == b["step"] and a["time"] == b["time"] and a["time"] >= 0.02
    case, em, ref, g, ph, p = _setup("naca", oracle)
    q0 = case["ic"](g)
    a = oracle.run_loop(g, p, q0, case["alpha"], 500, tolerance=0.5)
    b = ref.run_loop(q0, case["alpha"], 500, tolerance=0.5)
    assert a["step"] == b["step"] < 500 and bits_equal(a["q"], b["q"])


def test_flux_and_limiter_functions(oracle):
    from oracle import RefLib
    import physics as P
    r = np.random.default_rng(5)
    for variant, ph in (("forwardStep", P.forward_step(order2=False)), ("naca", P.naca())):
        ref = RefLib(variant)
        p = oracle.physics(ph, sorted(ph.bcs))
        for _ in range(200):
            qi = random_euler_state(1, int(r.integers(1 << 30)))
            qj = random_euler_state(1, int(r.integers(1 << 30)))
            t = r.uniform(0, 2 * np.pi); n = np.array([np.cos(t), np.sin(t)])
            assert bits_equal(oracle.flux(p, qi, qj, n), ref.flux(qi, qj, n))
    ref = RefLib("naca")
    p = oracle.physics(P.naca(), ["airfoil", "farfield"])
    for y in np.concatenate([np.linspace(-3, 3, 61), [2.0, 1e-300, -0.0]]):
        assert oracle.limiter_func(p, y) == ref.lib.ref_limiter_func(float(y))
    ref = RefLib("forwardStep_o2venk5")
    p = oracle.physics(P.forward_step(), ["wall"])
    assert ref.lib.ref_limiter_k() == 5.0
    for y in np.linspace(-3, 3, 61):
        assert oracle.limiter_func(p, y) == ref.lib.ref_limiter_func(float(y))


def test_diffusive_fluxes_with_face_gradients(oracle):
    """calc_flux of the diffusive examples, fed random face gradients: the
    Navier-Stokes flux of flatPlate / nacaTransient and the heatTransfer
    diffusion flux, bit for bit."""
    from oracle import RefLib
    import physics as P
    r = np.random.default_rng(7)
    for variant, ph in (("flatPlate", P.flat_plate()), ("nacaTransient", P.naca_transient()),
                        ("heatTransfer", P.heat())):
        ref = RefLib(variant)
        p = oracle.physics(ph, sorted(ph.bcs))
        V = ph.V
        for _ in range(200):
            if V == 4:
                qi = random_euler_state(1, int(r.integers(1 << 30)))
                qj = random_euler_state(1, int(r.integers(1 << 30)))
            else:
                qi, qj = r.uniform(-1, 1, V), r.uniform(-1, 1, V)
            gx, gy = r.normal(size=V) * 3, r.normal(size=V) * 3
            t = r.uniform(0, 2 * np.pi); n = np.array([np.cos(t), np.sin(t)])
            assert bits_equal(oracle.flux_grad(p, qi, qj, gx, gy, n), ref.flux_grad(qi, qj, gx, gy, n))


def test_residual_smoothing_bitwise(oracle):
    """smooth_residuals (explicit.cpp:32-66) on a random residual, triangle
    and quadrilateral meshes: the restatement equals the reference."""
    for name in ("burgers_diffusion", "flat_plate"):
        case = CASES[name]
        em = case["mesh"]()
        em.bnd_group[:] = 0          # one "wall" group: the only name the test physics defines
        em.group_names = ["wall"]
        ref = make_ref(dict(case, ref="tests", consts={}), em)
        g = oracle.build_mesh(em)
        p = oracle.physics(CASES["burgers_diffusion"]["phys"](), em.group_names)
        qt = np.random.default_rng(3).normal(size=g.n_total * 2)
        qt[g.n_real * 2:] = 0.0   # the time derivative leaves ghosts at 0
        assert bits_equal(oracle.smooth_residuals(g, p, qt), ref.smooth_residuals(qt))


def test_missing_boundary_edge_rejected(oracle):
    em = meshgen.sod_strip(8, 2)
    em.bnd_nodes = em.bnd_nodes.copy()
    em.bnd_nodes[0] = (0, em.nodes_x.size - 1)  # not an edge of the mesh
    with pytest.raises(ValueError):
        oracle.build_mesh(em)


def test_positivity_guard_is_inert_on_physical_states(oracle):
    """The optional guard (not in the reference) changes nothing while every
    MUSCL face state stays physical: the guarded oracle equals the reference."""
    case, em, ref, g, ph, p = _setup("step_o2_venk5", oracle)
    ph.positivity_guard = True
    pg = oracle.physics(ph, em.group_names)
    q0 = case["ic"](g)
    a = oracle.run_loop(g, pg, q0, case["alpha"], case["steps"])
    b = ref.run_loop(q0, case["alpha"], case["steps"])
    assert bits_equal(a["q"], b["q"])
