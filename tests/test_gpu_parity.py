"""GPU parity: the CUDA kernels, called through the C ABI, against the CPU
oracle on the same inputs.  The FP64_EXACT path must match bit for bit
(tolerance 0); residual norms, whose sums are reduced in a different order,
within 1e-12 relative."""
import numpy as np
import pytest

import fvgpu
import physics as P
from cases import CASES, random_euler_state

pytestmark = pytest.mark.gpu

R_RTOL = 1e-12


def bits_equal(a, b):
    a = np.ascontiguousarray(a); b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def setup(name, oracle, precision="fp64_exact"):
    case = CASES[name]
    em = case["mesh"]()
    ph = case["phys"]()
    mesh = fvgpu.Mesh.from_elements(em)
    s = fvgpu.Solver(mesh, ph, precision)
    g = oracle.build_mesh(em)
    p = oracle.physics(ph, em.group_names)
    return case, em, ph, s, g, p


def rand_state(g, ph, seed):
    if ph.V == 4:
        return random_euler_state(g.n_total, seed)
    return np.random.default_rng(seed).uniform(-1, 1, g.n_total * ph.V)


def stage_inputs(oracle, g, p, ph, q):
    """gx, gy, lim as a reference stage sees them: gradients and limiters
    (second order), unlimited gradients (diffusive fluxes: lim is unused and
    the device's is 1), or nothing (first order)."""
    if ph.order2:
        gx, gy = oracle.gradients(g, p, q)
        return gx, gy, oracle.limiters(g, p, q, gx, gy)
    if ph.diffusive:
        gx, gy = oracle.gradients(g, p, q)
        return gx, gy, np.ones_like(q)
    return np.zeros_like(q), np.zeros_like(q), np.zeros_like(q)


@pytest.mark.parametrize("name", sorted(CASES))
def test_stage_dt(name, oracle):
    case, em, ph, s, g, p = setup(name, oracle)
    q = rand_state(g, ph, 3)
    for glob in (False, True):
        assert bits_equal(s.stage_dt(q, glob), oracle.calc_dt(g, p, q, glob))


@pytest.mark.parametrize("name", [n for n in sorted(CASES) if CASES[n]["phys"]().order2 or CASES[n]["phys"]().diffusive])
def test_stage_gradients_limiters(name, oracle):
    case, em, ph, s, g, p = setup(name, oracle)
    q = rand_state(g, ph, 4)
    gx, gy, lim = s.stage_gradients_limiters(q)
    ogx, ogy, olim = stage_inputs(oracle, g, p, ph, q)
    assert bits_equal(gx, ogx) and bits_equal(gy, ogy) and bits_equal(lim, olim)


@pytest.mark.parametrize("name", sorted(CASES))
def test_stage_update_and_ghost_fill(name, oracle):
    case, em, ph, s, g, p = setup(name, oracle)
    qb = rand_state(g, ph, 5)
    qs = rand_state(g, ph, 6)
    gx, gy, lim = stage_inputs(oracle, g, p, ph, qs)
    dt = oracle.calc_dt(g, p, qs, ph.global_dt)
    alpha = 0.2898
    qt = oracle.time_derivatives(g, p, qs, gx, gy, lim)
    expect = qb + qt * np.repeat(dt, ph.V) * alpha            # update_cells
    expect = oracle.update_bounds(g, p, expect, gx, gy, lim)  # update_bounds
    got = s.stage_update(qb, qs, gx, gy, lim, dt, alpha)
    assert bits_equal(got, expect)
    assert bits_equal(s.stage_bounds(qs, gx, gy, lim), oracle.update_bounds(g, p, qs, gx, gy, lim))


@pytest.mark.parametrize("name", sorted(CASES))
def test_time_loop(name, oracle):
    case, em, ph, s, g, p = setup(name, oracle)
    q0 = case["ic"](g)
    steps = case["steps"]
    want = oracle.run_loop(g, p, q0, case["alpha"], steps)
    s.set_state(q0)
    got = s.run(steps, alpha=case["alpha"])
    q = s.get_state()
    assert got["step"] == want["step"] == steps
    assert bits_equal(q, want["q"])
    assert got["time"] == want["time"]
    np.testing.assert_allclose(got["R"], want["R"], rtol=R_RTOL, atol=0)


def test_stopping_criteria(oracle):
    case, em, ph, s, g, p = setup("sod", oracle)
    q0 = case["ic"](g)
    want = oracle.run_loop(g, p, q0, case["alpha"], 10 ** 6, max_time=0.02)
    s.set_state(q0)
    got = s.run(10 ** 6, alpha=case["alpha"], max_time=0.02)
    assert got["step"] == want["step"] and got["time"] == want["time"]
    assert bits_equal(s.get_state(), want["q"])
    case, em, ph, s, g, p = setup("naca", oracle)
    q0 = case["ic"](g)
    want = oracle.run_loop(g, p, q0, case["alpha"], 500, tolerance=0.5)
    s.set_state(q0)
    got = s.run(500, alpha=case["alpha"], tolerance=0.5)
    assert got["step"] == want["step"] < 500
    assert bits_equal(s.get_state(), want["q"])


def test_chunking_and_continuation_invariance(oracle):
    """Graph chunk length and splitting a run into continued runs do not
    change a single bit (RK1 alternates state buffers between steps)."""
    for name in ("sod", "step_o2_venk5"):
        case, em, ph, s, g, p = setup(name, oracle)
        q0 = case["ic"](g)
        want = oracle.run_loop(g, p, q0, case["alpha"], 13)["q"]
        for chunk in (1, 4, 7):
            s.set_chunk(chunk)
            s.set_state(q0)
            s.run(13, alpha=case["alpha"])
            assert bits_equal(s.get_state(), want), (name, chunk)
        s.set_chunk(16)
        s.set_state(q0)
        s.run(5, alpha=case["alpha"])
        r = s.run(13, alpha=case["alpha"], restart=False)
        assert r["step"] == 13
        assert bits_equal(s.get_state(), want)


def test_print_records(oracle):
    case, em, ph, s, g, p = setup("naca", oracle)
    s.set_state(case["ic"](g))
    recs = []
    s.run(25, alpha=case["alpha"], print_interval=10, on_print=lambda st, t, R: recs.append((st, t, R)))
    assert [r[0] for r in recs] == [0, 10, 20]
    assert recs[0][2] == [1.0] * 4 and recs[0][1] == 0.0
    want = oracle.run_loop(g, p, case["ic"](g), case["alpha"], 11, print_interval=10)
    np.testing.assert_allclose(recs[1][2], want["R"], rtol=R_RTOL)


def test_boundary_force(oracle):
    case, em, ph, s, g, p = setup("naca", oracle)
    q = random_euler_state(g.n_total, 9)
    s.set_state(q)
    fx, fy = s.boundary_force("airfoil")
    ox, oy = oracle.boundary_force(g, p, q, em.group_names.index("airfoil"))
    np.testing.assert_allclose([fx, fy], [ox, oy], rtol=1e-12, atol=1e-14)


def test_nonfinite_state_is_reported(oracle):
    case, em, ph, s, g, p = setup("sod", oracle)
    q = case["ic"](g)
    s.set_state(q)
    assert s.check_state() == 0
    q = q.copy(); q[4 * 7] = np.nan
    s.set_state(q)
    assert s.check_state() == -5
    q[4 * 7] = -1.0  # negative density
    s.set_state(q)
    assert s.check_state() == -5


def test_unsupported_physics_rejected():
    em = CASES["sod"]["mesh"]()
    mesh = fvgpu.Mesh.from_elements(em)
    bad = P.sod()
    bad.V = 2
    with pytest.raises(fvgpu.FvError) as e:
        fvgpu.Solver(mesh, bad)
    assert e.value.code == -4


# ---------------------------------------------------------------- FP64 / FP32
def normwise_rel(a, b, V):
    """max over variables k of max|a_k - b_k| / s_k on AoS [n][V] arrays, with
    s_k = max(max|b_k|, 1e-3 * max|b|) so that a variable that is zero up to
    rounding (rho*v in a 1-D problem) is measured against the state's scale.
    Entries that are NaN in both count as equal, NaN in one only as inf."""
    a = a.reshape(-1, V).copy(); b = b.reshape(-1, V).copy()
    na, nb = np.isnan(a), np.isnan(b)
    if np.any(na != nb):
        return float("inf")
    a[na] = 0.0; b[nb] = 0.0
    scale = np.maximum(np.abs(b).max(axis=0), 1e-3 * np.abs(b).max())
    scale = np.maximum(scale, 1e-300)
    return float((np.abs(a - b).max(axis=0) / scale).max())


FP64_STEP_RTOL = 1e-12     # plain FP64 path: max relative error per step
# The near-uniform M 0.2 flat-plate flow has residuals of ~3 % of its face
# fluxes, so cancellation amplifies the rounding of the rearranged Roe flux
# (the fast viscous terms add nothing measurable): up to 2.4e-12 per step.
FP64_STEP_RTOL_CASE = {"flat_plate": 5e-12}


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_stage_functions(name, oracle):
    case, em, ph, s, g, p = setup(name, oracle, "fp64")
    q = rand_state(g, ph, 21)
    e_dt = normwise_rel(s.stage_dt(q, False), oracle.calc_dt(g, p, q, False), 1)
    assert e_dt < FP64_STEP_RTOL, e_dt
    ogx, ogy, olim = stage_inputs(oracle, g, p, ph, q)
    # FP64 keeps the limiter multiplied into the gradients, except for the
    # diffusive fluxes, whose face gradient needs the raw gradients
    dev = (ogx, ogy, olim) if ph.diffusive else (ogx * olim, ogy * olim, olim)
    if ph.order2 or ph.diffusive:
        gx, gy, lim = s.stage_gradients_limiters(q)
        e = (normwise_rel(gx, dev[0], ph.V), normwise_rel(gy, dev[1], ph.V))
        assert max(e) < 1e-9, e
        if ph.diffusive:
            assert normwise_rel(lim, olim, ph.V) < 1e-9
        else:
            assert np.all(lim == 1.0)
    dt = oracle.calc_dt(g, p, q, ph.global_dt)
    qb = rand_state(g, ph, 22)
    qt = oracle.time_derivatives(g, p, q, ogx, ogy, olim)
    want = oracle.update_bounds(g, p, qb + qt * np.repeat(dt, ph.V) * 0.506, ogx, ogy, olim)
    got = s.stage_update(qb, q, dev[0], dev[1], dev[2], dt, 0.506)
    e = normwise_rel(got, want, ph.V)
    assert e < FP64_STEP_RTOL, e


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_per_step_error(name, oracle):
    """Each time step from the oracle's state: normwise relative error of the
    state after one step <= 1e-12; over the whole run the error stays small."""
    case, em, ph, s, g, p = setup(name, oracle, "fp64")
    q = case["ic"](g)
    worst = 0.0
    for k in range(6):
        want = oracle.run_loop(g, p, q, case["alpha"], 1)
        s.set_state(q)
        s.run(1, alpha=case["alpha"])
        got = s.get_state()
        worst = max(worst, normwise_rel(got[: g.n_real * ph.V], want["q"][: g.n_real * ph.V], ph.V))
        q = want["q"]
    assert worst < FP64_STEP_RTOL_CASE.get(name, FP64_STEP_RTOL), worst
    q0 = case["ic"](g)
    want = oracle.run_loop(g, p, q0, case["alpha"], case["steps"])
    s.set_state(q0)
    s.run(case["steps"], alpha=case["alpha"])
    assert normwise_rel(s.get_state()[: g.n_real * ph.V], want["q"][: g.n_real * ph.V], ph.V) < 1e-9


def l2_rel(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def rho_p(q, gamma=1.4):
    q = q.reshape(-1, 4)
    return q[:, 0], (gamma - 1) * (q[:, 3] - 0.5 * (q[:, 1] ** 2 + q[:, 2] ** 2) / q[:, 0])


FP32_L2_TOL = 1e-4         # FP32-bulk path: relative L2 error of density and pressure


@pytest.mark.parametrize("name", ["sod", "step_o1", "step_o2_venk5", "step_o2_mich", "naca", "flat_plate",
                                  "naca_transient"])
def test_fp32_l2_error(name, oracle):
    case, em, ph, s, g, p = setup(name, oracle, "fp32")
    q0 = case["ic"](g)
    want = oracle.run_loop(g, p, q0, case["alpha"], case["steps"])
    s.set_state(q0)
    got = s.run(case["steps"], alpha=case["alpha"])
    assert got["step"] == case["steps"]
    q = s.get_state()
    n = g.n_real * 4
    r1, p1 = rho_p(q[:n]); r0, p0 = rho_p(want["q"][:n])
    assert l2_rel(r1, r0) < FP32_L2_TOL and l2_rel(p1, p0) < FP32_L2_TOL
    assert s.check_state() == 0


@pytest.mark.parametrize("name", ["burgers", "heat"])
def test_fp32_scalar_kinds(name, oracle):
    case, em, ph, s, g, p = setup(name, oracle, "fp32")
    q0 = case["ic"](g)
    want = oracle.run_loop(g, p, q0, case["alpha"], case["steps"])
    s.set_state(q0)
    s.run(case["steps"], alpha=case["alpha"])
    n = g.n_real * ph.V
    assert l2_rel(s.get_state()[:n], want["q"][:n]) < FP32_L2_TOL


@pytest.mark.parametrize("precision", ["fp64_exact", "fp64", "fp32"])
def test_runs_are_bitwise_reproducible(precision, oracle):
    """No atomics in any accumulation: two runs give identical bits."""
    case, em, ph, s, g, p = setup("step_o2_venk5", oracle, precision)
    q0 = case["ic"](g)
    out = []
    for _ in range(2):
        s.set_state(q0)
        r = s.run(20, alpha=case["alpha"])
        out.append((s.get_state(), r["R"]))
    assert out[0][0].tobytes() == out[1][0].tobytes() and out[0][1].tobytes() == out[1][1].tobytes()


def test_solvers_of_different_tile_sizes_coexist(oracle):
    """Two solvers of one process whose tile kernels need different amounts of
    shared memory (FP64_EXACT, 256- and 64-cell tiles): creating the smaller
    one must not lower the limit the larger one launches with."""
    case = CASES["step_o2_venk5"]
    em, ph = case["mesh"](), case["phys"]()
    mesh = fvgpu.Mesh.from_elements(em)
    g = oracle.build_mesh(em)
    p = oracle.physics(ph, em.group_names)
    q0 = case["ic"](g)
    want = oracle.run_loop(g, p, q0, case["alpha"], 10)
    big = fvgpu.Solver(mesh, ph, "fp64_exact", tile_cells=256)
    small = fvgpu.Solver(mesh, ph, "fp64_exact", tile_cells=64)
    for s in (big, small):
        s.set_state(q0)
        s.run(10, alpha=case["alpha"])
        assert s.get_state().tobytes() == want["q"].tobytes()
    big.close()
    small.close()


FUSED_CASES = [n for n in sorted(CASES) if CASES[n]["phys"]().order2 and CASES[n]["phys"]().flux in ("roe_fs", "roe_st")
               and not CASES[n]["phys"]().diffusive]


@pytest.mark.parametrize("precision", ["fp64_exact", "fp64", "fp32"])
@pytest.mark.parametrize("name", FUSED_CASES)
def test_fused_and_split_stage_kernels_agree(name, precision, oracle):
    """The fused stage kernel (gradients, limiter and fluxes of a two-ring
    tile in one launch), with one CTA per tile (one or two threads per cell)
    and with the work-list schedule, the split gradient + flux kernels, and
    the hybrid (split first stage with the time step folded into its
    gradient kernel, fused others) give the same bits in every precision
    mode, and in FP64_EXACT all equal the oracle, at every tile size."""
    case = CASES[name]
    em, ph = case["mesh"](), case["phys"]()
    mesh = fvgpu.Mesh.from_elements(em)
    g = oracle.build_mesh(em)
    p = oracle.physics(ph, em.group_names)
    q0 = case["ic"](g)
    want = oracle.run_loop(g, p, q0, case["alpha"], case["steps"]) if precision == "fp64_exact" else None
    out = {}
    for T in (64, 128, 256):
        for sk, sched in (("split", "tile"), ("fused", "tile"), ("fused", "worklist"), ("fused", "tile2"),
                          ("hybrid", "tile"), ("hybrid", "tile2")):
            if sched == "tile2" and T > 128:
                continue
            s = fvgpu.Solver(mesh, ph, precision, tile_cells=T, stage_kernels=sk, schedule=sched)
            assert s.stage_kernels == sk and s.schedule == sched
            s.set_state(q0)
            r = s.run(case["steps"], alpha=case["alpha"])
            out[(T, sk, sched)] = (s.get_state(), np.asarray(r["R"]), r["time"])
            s.close()
    ref = out[(128, "split", "tile")]
    for k, v in out.items():
        assert bits_equal(v[0], ref[0]), k
        assert v[2] == ref[2], k
        np.testing.assert_allclose(v[1], ref[1], rtol=R_RTOL, atol=0)
    if want is not None:
        assert bits_equal(ref[0], want["q"])


def test_fused_stage_kernel_is_chosen_where_the_physics_allow():
    for name in sorted(CASES):
        case = CASES[name]
        ph = case["phys"]()
        fusable = ph.V == 4 and ph.order2 and ph.flux in ("roe_fs", "roe_st") and not ph.diffusive
        mesh = fvgpu.Mesh.from_elements(case["mesh"]())
        for prec, layout in (("fp64", "fused"), ("fp32", "hybrid")):
            s = fvgpu.Solver(mesh, ph, prec)
            assert s.stage_kernels == (layout if fusable else "split"), (name, prec)
            s.close()
    case = CASES["heat"]
    with pytest.raises(fvgpu.FvError) as e:
        fvgpu.Solver(fvgpu.Mesh.from_elements(case["mesh"]()), case["phys"](), "fp64", stage_kernels="fused")
    assert e.value.code == -4


@pytest.mark.parametrize("precision", ["fp64_exact", "fp32"])
def test_output_fields_on_the_device_equal_the_host_kinds(precision):
    """fv_output_fields (the writeVtk extra fields, evaluated on the device)
    gives the host kinds' bits for every real cell, from a host state and from
    the solver's own state."""
    import ctypes as C
    case = CASES["step_o2_venk5"]
    em = case["mesh"]()
    mesh = fvgpu.Mesh.from_elements(em)
    s = fvgpu.Solver(mesh, case["phys"](), precision)
    q = random_euler_state(mesh.n_total, 31)
    kinds = ["pressure", "mach", "velocity", "state01"]
    L = fvgpu.lib()
    p = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    want = []
    for k in kinds:
        nc = 2 if k in ("velocity", "state01") else 1
        w = np.zeros((mesh.n_real, nc))
        for c in range(mesh.n_real):
            o = np.zeros(2)
            L.fv_kind_output(fvgpu.Solver.OUTPUT_KINDS[k], C.c_double(1.4), p(q[4 * c:4 * c + 4].copy()), p(o))
            w[c] = o[:nc]
        want.append(w if nc == 2 else w[:, 0])
    for got in (s.output_fields(kinds, q), None):
        if got is None:  # the solver's state (FP64 base state, device numbering)
            s.set_state(q)
            got = s.output_fields(kinds)
        for g, w, k in zip(got, want, kinds):
            assert g.tobytes() == w.tobytes(), k
    s.close()
