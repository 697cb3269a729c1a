"""Batched independent cases (the Riemann-strip workload): many strips of
uneven sizes as one mesh (fv_mesh_create_batch), advanced together in the
same launches, each with its own global dt minimum and time.  Every case of
the batch must give exactly what it gives alone -- in FP64_EXACT that is the
oracle's result for that case, bit for bit -- however the tiles fall across
case boundaries."""
import numpy as np
import pytest

import meshgen
import physics as P


def strips(nxs, ny=2, seed=4):
    rng = np.random.default_rng(seed)
    ems = [meshgen.riemann_strip(nx, ny) for nx in nxs]
    states = [(rng.uniform(0.1, 1.0), rng.uniform(-0.5, 0.5), rng.uniform(0.1, 1.0),
               rng.uniform(0.1, 1.0), rng.uniform(-0.5, 0.5), rng.uniform(0.1, 1.0)) for _ in nxs]
    return ems, states


def bits_equal(a, b):
    a = np.ascontiguousarray(a); b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def test_batch_mesh_is_the_disjoint_union():
    import fvgpu

    ems, _ = strips([5, 9, 3, 12])
    parts = [fvgpu.Mesh.from_elements(em) for em in ems]
    b = fvgpu.Mesh.batch(parts)
    assert b.n_cases == 4
    ro, bo = b.case_offsets()
    assert ro.tolist() == np.cumsum([0] + [m.n_real for m in parts]).tolist()
    assert bo.tolist() == np.cumsum([0] + [m.n_bound for m in parts]).tolist()
    assert b.n_real == ro[-1] and b.n_bound == bo[-1] and b.n_edges == sum(m.n_edges for m in parts)
    gb = b.geometry()
    area = b.split(gb["area"], 1)
    ccx = b.split(gb["ccx"], 1)
    e0 = 0
    for k, m in enumerate(parts):
        g = m.geometry()
        assert bits_equal(area[k], g["area"]) and bits_equal(ccx[k], g["ccx"])
        # edges of case k: its own, in order, with cells renumbered into the batch
        ec = gb["edge_cells"][2 * e0: 2 * (e0 + m.n_edges)].astype(np.int64)
        own = g["edge_cells"].astype(np.int64)
        remap = np.where(own < m.n_real, own + ro[k], own - m.n_real + b.n_real + bo[k])
        assert np.array_equal(ec, remap)
        for key in ("enx", "eny", "elen"):
            assert bits_equal(gb[key][e0: e0 + m.n_edges], g[key])
        e0 += m.n_edges
    # device order keeps each case's real cells contiguous
    n2r = b.device_order()[: b.n_real]
    case_of = np.searchsorted(ro, n2r, side="right") - 1
    assert np.all(np.diff(case_of) >= 0)


def test_batch_requires_matching_group_names():
    import fvgpu

    a = meshgen.riemann_strip(4, 2)
    c = meshgen.rect_tri(4, 2, 1.0, 0.5, side_names=("ends", "wall"))
    with pytest.raises(ValueError):
        fvgpu.Mesh.batch([fvgpu.Mesh.from_elements(a), fvgpu.Mesh.from_elements(c)])


@pytest.mark.gpu
@pytest.mark.parametrize("tile_cells", [64, 128, 256])
def test_batch_equals_each_case_alone(tile_cells, oracle):
    import fvgpu

    ems, states = strips([37, 8, 90, 12, 61, 150, 24])
    ph = P.riemann_strip()
    parts = [fvgpu.Mesh.from_elements(em) for em in ems]
    b = fvgpu.Mesh.batch(parts)
    q0s = []
    for em, m, st in zip(ems, parts, states):
        g = m.geometry()
        q0s.append(P.ic_riemann(g["ccx"], st[:3], st[3:]).ravel())
    steps = 25
    wants = []
    for em, q0 in zip(ems, q0s):
        g = oracle.build_mesh(em)
        wants.append(oracle.run_loop(g, oracle.physics(ph, em.group_names), q0, P.RK5_ALPHA, steps))
    # the split kernels, and the fused kernel with both schedules
    for sk, sched in (("split", "tile"), ("fused", "tile"), ("fused", "worklist"), ("fused", "tile2")):
        if sched == "tile2" and tile_cells > 128:
            continue
        sb = fvgpu.Solver(b, ph, "fp64_exact", tile_cells=tile_cells, stage_kernels=sk, schedule=sched)
        sb.set_state(b.join(q0s, 4))
        sb.run(steps, print_interval=10 ** 9)
        got = b.split(sb.get_state(), 4)
        times = sb.case_times()
        for k, want in enumerate(wants):
            assert bits_equal(got[k], want["q"]), (sk, sched, k)
            assert times[k] == want["time"], (sk, sched, k)
        sb.close()
    # FP32-bulk: the batch equals the cases run alone in FP32
    s32 = fvgpu.Solver(b, ph, "fp32", tile_cells=tile_cells)
    s32.set_state(b.join(q0s, 4))
    s32.run(steps, print_interval=10 ** 9)
    got32 = b.split(s32.get_state(), 4)
    for k, (m, q0) in enumerate(zip(parts, q0s)):
        s1 = fvgpu.Solver(m, ph, "fp32", tile_cells=tile_cells)
        s1.set_state(q0)
        s1.run(steps, print_interval=10 ** 9)
        assert bits_equal(got32[k], s1.get_state()), k
        s1.close()
    s32.close()


@pytest.mark.gpu
def test_batch_stage_dt_is_per_case(oracle):
    import fvgpu
    from cases import random_euler_state

    ems, _ = strips([20, 7, 33])
    ph = P.riemann_strip()
    parts = [fvgpu.Mesh.from_elements(em) for em in ems]
    b = fvgpu.Mesh.batch(parts)
    s = fvgpu.Solver(b, ph, "fp64_exact")
    q = random_euler_state(b.n_total, seed=9)
    got = b.split(s.stage_dt(q, True), 1)
    for k, (em, qk) in enumerate(zip(ems, b.split(q, 4))):
        g = oracle.build_mesh(em)
        assert bits_equal(got[k], oracle.calc_dt(g, oracle.physics(ph, em.group_names), qk, True)), k
    s.close()


@pytest.mark.gpu
def test_batch_fp32_error_equals_fp64_error_against_exact_riemann():
    """FP32-bulk and FP64 reach the same L2 density error against the exact
    Riemann solution (area-weighted over the batch) within 1e-4."""
    import fvgpu
    import riemann

    nx = [300, 520, 800, 1250, 2000, 410, 950]
    rng = np.random.default_rng(4)
    states = [(rng.uniform(0.1, 1.0), rng.uniform(-0.5, 0.5), rng.uniform(0.1, 1.0),
               rng.uniform(0.1, 1.0), rng.uniform(-0.5, 0.5), rng.uniform(0.1, 1.0)) for _ in nx]
    parts = [fvgpu.Mesh.from_elements(meshgen.riemann_strip(n, 8)) for n in nx]
    b = fvgpu.Mesh.batch(parts)
    geo = b.geometry()
    ccx, area = b.split(geo["ccx"], 1), b.split(geo["area"], 1)
    q0 = b.join([P.ic_riemann(c, st[:3], st[3:]) for c, st in zip(ccx, states)], 4)
    errs = {}
    for prec in ("fp64", "fp32"):
        s = fvgpu.Solver(b, P.riemann_strip(), prec)
        s.set_state(q0)
        s.run(300, print_interval=10 ** 9)
        qs, times = b.split(s.get_state(), 4), s.case_times()
        num = den = 0.0
        for k, m in enumerate(parts):
            n = m.n_real
            ra, _, _ = riemann.sample(ccx[k][:n], times[k], states[k][:3], states[k][3:])
            num += float(((qs[k].reshape(-1, 4)[:n, 0] - ra) ** 2 * area[k][:n]).sum())
            den += float(area[k][:n].sum())
        errs[prec] = np.sqrt(num / den)
        s.close()
    print(f"batch L2 density error vs exact Riemann: fp64 {errs['fp64']:.4e} fp32 {errs['fp32']:.4e}")
    assert errs["fp64"] < 0.02
    assert abs(errs["fp32"] - errs["fp64"]) <= 1e-4
