"""Domain decomposition on one GPU (fv_group_*): several parts in one
process, their halos exchanged by device copies or through NCCL (a
one-process communicator sending to itself, the transport that links the
processes of a multi-GPU run).  Every part computes its own cells with the
single-solver arithmetic, so the decomposed state equals the single solver's
bit for bit in every precision, and FP64_EXACT equals the oracle."""
import numpy as np
import pytest

import meshgen
import physics as P

pytestmark = pytest.mark.gpu


def _cases():
    fs = P.forward_step(order2=True, limiter="venkat", K=5.0, cfl=0.8)
    fs.positivity_guard = True
    return {
        "forward_step": (lambda: meshgen.forward_step(n=20), lambda: fs, lambda g: P.ic_forward_step(g.n_total),
                         P.RK5_ALPHA, 12),
        "naca_local_dt": (lambda: meshgen.naca_ogrid(48, 12), P.naca, lambda g: P.ic_naca(g.n_total), P.RK5_ALPHA, 12),
        "sod_first_order": (lambda: meshgen.sod_strip(40, 4), P.sod, lambda g: P.ic_sod(g.ccx), P.RK1_ALPHA, 25),
    }


def _single(mesh, ph, prec, q0, alpha, steps):
    import fvgpu
    s = fvgpu.Solver(mesh, ph, prec)
    s.set_state(q0)
    r = s.run(steps, alpha=alpha)
    q = s.get_state()
    s.close()
    return r, q


@pytest.mark.parametrize("case", ["forward_step", "naca_local_dt", "sod_first_order"])
@pytest.mark.parametrize("prec", ["fp64_exact", "fp64", "fp32"])
def test_group_equals_single_solver(case, prec, oracle):
    import fvgpu
    mk_em, mk_ph, ic, alpha, steps = _cases()[case]
    em, ph = mk_em(), mk_ph()
    g = oracle.build_mesh(em)
    q0 = np.ascontiguousarray(ic(g), np.float64).ravel()
    mesh = fvgpu.Mesh.from_elements(em)
    r1, q1 = _single(mesh, ph, prec, q0, alpha, steps)
    if prec == "fp64_exact":
        want = oracle.run_loop(g, oracle.physics(ph, em.group_names), q0, alpha, steps)
        assert q1.tobytes() == want["q"].tobytes()
    for n_parts, serial in ((1, False), (2, False), (3, False), (4, False), (3, True)):
        grp = fvgpu.Group(mesh, ph, prec, n_parts=n_parts, serial_exchange=serial)
        inf = grp.info()
        assert inf["local_parts"] == n_parts and inf["owned_cells"] == mesh.n_real
        # the band-first overlap: fused second-order parts with something to exchange
        assert (inf["band_tiles"] >= 0) == (ph.order2 and not serial and n_parts > 1)
        grp.set_state(q0)
        r = grp.run(steps, alpha=alpha)
        q = grp.get_state()
        grp.close()
        assert r["step"] == r1["step"] == steps
        assert r["time"] == r1["time"]
        assert q.tobytes() == q1.tobytes(), (n_parts, float(np.abs(q - q1).max()))
        np.testing.assert_allclose(r["R"], r1["R"], rtol=1e-12)


@pytest.mark.parametrize("serial", [False, True], ids=["overlapped", "serial"])
@pytest.mark.parametrize("prec", ["fp64_exact", "fp32"])
def test_group_exchange_through_nccl(prec, serial):
    """The same decomposition with every exchange, dt record and residual sum
    going through NCCL (send/recv to this process, all-gathers) instead of
    device copies, with the exchange on its own stream beside the interior
    tiles or after all tiles."""
    import fvgpu
    mk_em, mk_ph, ic, alpha, steps = _cases()["forward_step"]
    em, ph = mk_em(), mk_ph()
    mesh = fvgpu.Mesh.from_elements(em)
    q0 = P.ic_forward_step(mesh.n_total).ravel()
    r1, q1 = _single(mesh, ph, prec, q0, alpha, steps)
    for n_parts in (2, 3):
        grp = fvgpu.Group(mesh, ph, prec, n_parts=n_parts, nccl_local=True, serial_exchange=serial)
        inf = grp.info()
        assert inf["nccl"] and (inf["band_tiles"] < 0) == serial
        grp.set_state(q0)
        r = grp.run(steps, alpha=alpha)
        q = grp.get_state()
        grp.close()
        assert r["step"] == steps and r["time"] == r1["time"]
        assert q.tobytes() == q1.tobytes()


@pytest.mark.parametrize("case", ["forward_step", "naca_local_dt", "sod_first_order"])
@pytest.mark.parametrize("prec", ["fp64_exact", "fp32"])
def test_group_p2p_transport(case, prec):
    """The P2P transport: the states other parts read are stored straight
    into their stage buffers, and an epoch flag is released in each, by the
    fused stage launch itself (second order: its band tiles wait for the
    senders, compute, store and count) or by a push kernel (first order);
    a bounded wait precedes the dt kernel (and, first order, each stage).
    With and without a communicator (dt records and residual sums through
    NCCL), across a continued run: the same bits as the single solver, and no
    wait gives up (fv_group_run would report it)."""
    import fvgpu
    mk_em, mk_ph, ic, alpha, steps = _cases()[case]
    em, ph = mk_em(), mk_ph()
    mesh = fvgpu.Mesh.from_elements(em)
    geo = mesh.geometry()
    q0 = np.ascontiguousarray(ic(type("G", (), {"n_total": mesh.n_total, "ccx": geo["ccx"]})()), np.float64).ravel()
    r1, q1 = _single(mesh, ph, prec, q0, alpha, steps)
    for n_parts, serial, nccl in ((2, False, False), (3, True, False), (4, False, True)):
        grp = fvgpu.Group(mesh, ph, prec, n_parts=n_parts, transport="p2p", serial_exchange=serial,
                          nccl_local=nccl, wait_polls=200000)
        inf = grp.info()
        assert inf["transport"] == "p2p" and inf["nccl"] == nccl
        grp.set_state(q0)
        r = grp.run(steps, alpha=alpha)
        r2 = grp.run(steps + 3, alpha=alpha, restart=False)
        q = grp.get_state()
        grp.close()
        assert r["step"] == steps and r2["step"] == steps + 3
        s = fvgpu.Solver(mesh, ph, prec)
        s.set_state(q0)
        s.run(steps + 3, alpha=alpha)
        q3 = s.get_state()
        s.close()
        assert q.tobytes() == q3.tobytes(), (n_parts, serial, nccl)
    del r1, q1


def test_group_continues_across_runs_and_schedules():
    """run(4) then run(11, restart=False) equals run(11); tile sizes and the
    work-list schedule change nothing."""
    import fvgpu
    mk_em, mk_ph, ic, alpha, steps = _cases()["forward_step"]
    em, ph = mk_em(), mk_ph()
    mesh = fvgpu.Mesh.from_elements(em)
    q0 = P.ic_forward_step(mesh.n_total).ravel()
    r1, q1 = _single(mesh, ph, "fp32", q0, alpha, 11)
    for tile, sched in ((128, "tile"), (64, "worklist"), (256, "tile"), (64, "tile2")):
        grp = fvgpu.Group(mesh, ph, "fp32", n_parts=3, tile_cells=tile, schedule=sched)
        grp.set_state(q0)
        grp.run(4, alpha=alpha)
        r = grp.run(11, alpha=alpha, restart=False)
        q = grp.get_state()
        grp.close()
        assert r["step"] == 11 and r["time"] == r1["time"]
        assert q.tobytes() == q1.tobytes(), (tile, sched)


def test_group_prints_and_stops_like_the_single_solver():
    import fvgpu
    mk_em, mk_ph, ic, alpha, steps = _cases()["naca_local_dt"]
    em, ph = mk_em(), mk_ph()
    mesh = fvgpu.Mesh.from_elements(em)
    q0 = P.ic_naca(mesh.n_total).ravel()
    logs = {}
    for key in ("single", "group"):
        rec = []
        if key == "single":
            s = fvgpu.Solver(mesh, ph, "fp64")
        else:
            s = fvgpu.Group(mesh, ph, "fp64", n_parts=4)
        s.set_state(q0)
        r = s.run(40, max_time=1e10, print_interval=5, on_print=lambda st, t, R: rec.append((st, t, R)))
        logs[key] = (r, rec)
        s.close()
    (r1, rec1), (r2, rec2) = logs["single"], logs["group"]
    assert r1["step"] == r2["step"] == 40
    assert [x[0] for x in rec1] == [x[0] for x in rec2]
    assert [x[1] for x in rec1] == [x[1] for x in rec2]
    np.testing.assert_allclose([x[2] for x in rec2], [x[2] for x in rec1], rtol=1e-11)


def test_group_refuses_what_it_cannot_exchange():
    import fvgpu
    mesh = fvgpu.Mesh.from_elements(meshgen.forward_step(n=20))
    ph = P.forward_step(order2=True)
    with pytest.raises(fvgpu.FvError):
        fvgpu.Group(mesh, ph, "fp64", n_parts=5, n_ranks=2)    # parts not a multiple of processes
    with pytest.raises(fvgpu.FvError):
        fvgpu.Group(mesh, ph, "fp64", n_parts=2, rank=1, n_ranks=2)  # no NCCL id
    for flag in ("diffusive", "smooth"):                            # more than the stage state to exchange
        ph2 = P.forward_step(order2=True)
        setattr(ph2, flag, True)
        with pytest.raises(fvgpu.FvError):
            fvgpu.Group(mesh, ph2, "fp64", n_parts=2)


def test_group_full_size_forward_step():
    """The 998,046-cell bench mesh in 4 parts: FP32-bulk and FP64 states equal
    the single solver's after 5 steps."""
    import fvgpu
    em = meshgen.forward_step()
    mesh = fvgpu.Mesh.from_elements(em)
    ph = P.forward_step(order2=True, limiter="venkat", K=5.0, cfl=0.8)
    ph.positivity_guard = True
    q0 = P.ic_forward_step(mesh.n_total).ravel()
    for prec in ("fp32", "fp64"):
        r1, q1 = _single(mesh, ph, prec, q0, P.RK5_ALPHA, 5)
        grp = fvgpu.Group(mesh, ph, prec, n_parts=4)
        grp.set_state(q0)
        r = grp.run(5)
        q = grp.get_state()
        inf = grp.info()
        grp.close()
        print(f"{prec}: halo cells per stage {inf['halo_cells']} of {mesh.n_real}")
        assert r["time"] == r1["time"]
        assert q.tobytes() == q1.tobytes()


def test_group_with_nccl_leaves_torch_importable():
    """A decomposition that loads NCCL before PyTorch does loads PyTorch's own
    copy (fvgpu.py sets FVGPU_NCCL_LIB), so `import torch` afterwards in the
    same process finds the NCCL it was built for."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (f"import sys; sys.path[:0] = [{os.path.join(root, 'finite-volume-2d-cpp_b200')!r}]\n"
            "import fvgpu, meshgen, physics as P\n"
            "mesh = fvgpu.Mesh.from_elements(meshgen.forward_step(n=20))\n"
            "g = fvgpu.Group(mesh, P.forward_step(order2=True), 'fp64', n_parts=2, nccl_local=True)\n"
            "g.run(2)\n"
            "g.close()\n"
            "import torch\n"
            "print('torch', torch.__version__)\n")
    env = {k: v for k, v in os.environ.items() if k != "FVGPU_NCCL_LIB"}
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0 and "torch" in r.stdout, r.stdout + r.stderr


@pytest.mark.parametrize("transport", ["copy", "p2p"])
def test_group_on_mixed_elements_equals_the_oracle(transport, oracle):
    """A mesh whose left half is quadrilaterals and right half triangles, in
    2 and 3 parts, second order (Venkatakrishnan), FP64_EXACT: the
    decomposed state equals the oracle's whole-mesh run bit for bit."""
    import fvgpu
    from test_mixed_elements import mixed_strip
    em = mixed_strip(32, 8)
    ph = P.Physics(V=4, flux="roe_fs", order2=True, limiter="venkat", K=5.0, dt_kind="cfl_sum", cfl=0.5,
                   global_dt=True, bcs={"wall": ("wall", None), "ends": ("copy", None)})
    g = oracle.build_mesh(em)
    q0 = P.ic_sod(g.ccx).ravel()
    want = oracle.run_loop(g, oracle.physics(ph, em.group_names), q0, P.RK5_ALPHA, 15)
    mesh = fvgpu.Mesh.from_elements(em)
    for n_parts in (2, 3):
        grp = fvgpu.Group(mesh, ph, "fp64_exact", n_parts=n_parts, transport=transport, wait_polls=200000)
        grp.set_state(q0)
        r = grp.run(15)
        q = grp.get_state()
        grp.close()
        assert r["step"] == 15 and r["time"] == want["time"]
        assert q.tobytes() == want["q"].tobytes(), (transport, n_parts)
