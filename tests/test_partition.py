"""Domain decomposition on CPU: the part plans (fv_mesh_partition) and the
exchange schedule of fv_group_run, checked with the oracle.

- Every plan covers the mesh: owned ranges partition the real cells and
  ghosts, each owned and ring-1 cell keeps all its faces in reference edge
  order, and what part p sends to part r is, cell for cell and in order, what
  r expects from p.
- Two gloo ranks run the decomposed time loop with the oracle's stage
  functions on each part's local mesh: per step the dt minimum over the
  parts' own cells and ghosts (all-reduce), per RK stage gradients, limiters,
  time derivatives, update and ghost fill on the local mesh, then the halo
  exchange of the plan.  The owned cells' states equal the oracle's
  whole-mesh run bit for bit (fvhyper's MPI loop, explicit.cpp:729-749,
  exchanges q, gx, gy, limiters and dt of one ring; two rings and one
  exchange of the stage state per stage give the same arithmetic).
"""
import os
import socket

import numpy as np
import pytest

import meshgen
import physics as P


def _cases():
    return {
        "forward_step": (lambda: meshgen.forward_step(n=20), lambda: P.forward_step(order2=True, limiter="venkat", K=5.0),
                         lambda g: P.ic_forward_step(g.n_total), P.RK5_ALPHA),
        "naca_local_dt": (lambda: meshgen.naca_ogrid(48, 12), P.naca, lambda g: P.ic_naca(g.n_total), P.RK5_ALPHA),
        "sod_first_order": (lambda: meshgen.sod_strip(40, 4), P.sod, lambda g: P.ic_sod(g.ccx), P.RK1_ALPHA),
        "mixed_elements": (_mixed_strip, _mixed_physics, lambda g: P.ic_sod(g.ccx), P.RK5_ALPHA),
    }


def _mixed_strip():
    from test_mixed_elements import mixed_strip
    return mixed_strip(32, 8)


def _mixed_physics():
    return P.Physics(V=4, flux="roe_fs", order2=True, limiter="venkat", K=5.0, dt_kind="cfl_sum", cfl=0.5,
                     global_dt=True, bcs={"wall": ("wall", None), "ends": ("copy", None)})


def _local_geom(g, pl):
    """The oracle's mesh arrays of one part's local mesh."""
    from oracle import GeomMesh
    l2r = pl["local2ref"].astype(np.int64)
    E = pl["local_edges"].astype(np.int64)
    nt, nr = pl["n_total"], pl["n_real"]
    r2l = np.full(g.n_total, -1, np.int64)
    r2l[l2r] = np.arange(nt)
    lec = r2l[g.edge_cells.reshape(-1, 2)[E].astype(np.int64)]
    assert (lec >= 0).all(), "an edge of the part reaches outside its local mesh"
    eloc = np.full(g.n_edges, -1, np.int64)
    eloc[E] = np.arange(E.size)
    rb = l2r[nr:] - g.n_real
    be = eloc[g.bound_edges[rb].astype(np.int64)]
    assert (be >= 0).all()
    return GeomMesh(n_nodes=g.n_nodes, n_real=nr, n_total=nt, n_edges=E.size, n_bound=nt - nr,
                    edge_cells=np.ascontiguousarray(lec.ravel(), np.uint32),
                    edge_nodes=np.ascontiguousarray(g.edge_nodes.reshape(-1, 2)[E].ravel(), np.uint32),
                    enx=g.enx[E].copy(), eny=g.eny[E].copy(), elen=g.elen[E].copy(), ecx=g.ecx[E].copy(),
                    ecy=g.ecy[E].copy(), area=g.area[l2r].copy(), ccx=g.ccx[l2r].copy(), ccy=g.ccy[l2r].copy(),
                    bound_edges=be.astype(np.uint32), bound_group=g.bound_group[rb].astype(np.int32))


@pytest.mark.parametrize("case", ["forward_step", "naca_local_dt", "sod_first_order", "mixed_elements"])
@pytest.mark.parametrize("n_parts", [2, 3, 5])
def test_part_plans_cover_the_mesh(case, n_parts, oracle):
    import fvgpu
    mk_em = _cases()[case][0]
    em = mk_em()
    mesh = fvgpu.Mesh.from_elements(em)
    g = oracle.build_mesh(em)
    N, NT = mesh.n_real, mesh.n_total
    plans = [mesh.partition(n_parts, p) for p in range(n_parts)]
    owned_real = np.concatenate([pl["local2ref"][: pl["n_own"]] for pl in plans])
    owned_ghost = np.concatenate([pl["local2ref"][pl["n_real"]: pl["n_real"] + pl["n_own_ghost"]] for pl in plans])
    assert np.array_equal(np.sort(owned_real), np.arange(N))
    assert np.array_equal(np.sort(owned_ghost), np.arange(N, NT))
    assert sum(pl["cell0"] >= 0 for pl in plans) == 1
    assert all(pl["owner0"] == plans[0]["owner0"] for pl in plans)
    ec = g.edge_cells.reshape(-1, 2)
    faces = [[] for _ in range(NT)]
    for e, (i, j) in enumerate(ec):
        faces[i].append(e)
        faces[j].append(e)
    for p, pl in enumerate(plans):
        l2r = pl["local2ref"]
        local_edges = pl["local_edges"]
        assert np.all(np.diff(local_edges) > 0)           # reference edge order
        edge_set = set(local_edges.tolist())
        local = set(l2r.tolist())
        own = set(l2r[: pl["n_own"]].tolist())
        ring1 = {int(c) for r in own for e in faces[r] for c in ec[e] if c < N} - own
        for r in own | ring1:                             # all faces of owned and ring-1 cells
            assert set(faces[r]) <= edge_set
            assert all(int(c) in local for e in faces[r] for c in ec[e])
        for r in range(n_parts):
            if r == p:
                continue
            sent = l2r[pl["send_idx"][pl["send_off"][r]: pl["send_off"][r + 1]]]
            want = plans[r]["local2ref"][plans[r]["recv_idx"][plans[r]["recv_off"][p]: plans[r]["recv_off"][p + 1]]]
            assert np.array_equal(sent, want)
        # the band (owned cells other parts read) comes first
        sent_real = np.unique(pl["send_idx"][pl["send_idx"] < pl["n_real"]])
        assert np.array_equal(sent_real, np.arange(pl["n_band"]))
        # every halo cell and halo ghost arrives from its owner
        recv = np.sort(l2r[pl["recv_idx"]])
        halo = np.sort(np.concatenate([l2r[pl["n_own"]: pl["n_real"]], l2r[pl["n_real"] + pl["n_own_ghost"]:]]))
        assert np.array_equal(recv, halo)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _decomposed_run(rank, world, case, n_parts, steps, out):
    """The decomposed time loop of this rank's parts on the oracle."""
    import torch
    import torch.distributed as dist

    import fvgpu
    from oracle import Oracle

    dist.init_process_group("gloo", rank=rank, world_size=world)
    mk_em, mk_ph, ic, alpha = _cases()[case]
    em = mk_em()
    ph = mk_ph()
    orc = Oracle()
    g = orc.build_mesh(em)
    p = orc.physics(ph, em.group_names)
    mesh = fvgpu.Mesh.from_elements(em)
    V = ph.V
    q0 = np.ascontiguousarray(ic(g), np.float64).reshape(-1, V)
    mine = list(range(rank * n_parts // world, (rank + 1) * n_parts // world))
    parts = {}
    for j in mine:
        pl = mesh.partition(n_parts, j)
        lg = _local_geom(g, pl)
        q = q0[pl["local2ref"]].ravel().copy()
        z = np.zeros_like(q)
        parts[j] = dict(pl=pl, g=lg, q=orc.update_bounds(lg, p, q, z, z, z), gx=z.copy(), gy=z.copy(), lim=z.copy())

    def exchange(states):
        reqs, bufs = [], {}
        for s in range(n_parts):
            for r in range(n_parts):
                if s == r:
                    continue
                rs, rr = s * world // n_parts, r * world // n_parts
                if s in parts:
                    pl = parts[s]["pl"]
                    idx = pl["send_idx"][pl["send_off"][r]: pl["send_off"][r + 1]]
                    data = states[s].reshape(-1, V)[idx].copy()
                    if r in parts:
                        bufs[(s, r)] = data
                    elif idx.size:
                        reqs.append(dist.isend(torch.from_numpy(data), dst=rr))
                if r in parts and s not in parts:
                    pl = parts[r]["pl"]
                    n = pl["recv_off"][s + 1] - pl["recv_off"][s]
                    if n:
                        t = torch.zeros((n, V), dtype=torch.float64)
                        dist.recv(t, src=rs)
                        bufs[(s, r)] = t.numpy()
        for q in reqs:
            q.wait()
        for (s, r), data in bufs.items():
            pl = parts[r]["pl"]
            idx = pl["recv_idx"][pl["recv_off"][s]: pl["recv_off"][s + 1]]
            states[r].reshape(-1, V)[idx] = data

    for _ in range(steps):
        dts = {}
        for j, st in parts.items():
            dts[j] = orc.calc_dt(st["g"], p, st["q"])
        if ph.global_dt:
            m = np.inf
            for j, st in parts.items():
                pl = st["pl"]
                own = np.concatenate([dts[j][: pl["n_own"]], dts[j][pl["n_real"]: pl["n_real"] + pl["n_own_ghost"]]])
                m = min(m, own.min())
            t = torch.tensor([m], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MIN)
            for j in parts:
                dts[j][:] = t.item()
        qk = {j: st["q"].copy() for j, st in parts.items()}
        for a in alpha:
            for j, st in parts.items():
                lg = st["g"]
                if ph.order2:
                    st["gx"], st["gy"] = orc.gradients(lg, p, qk[j])
                    st["lim"] = orc.limiters(lg, p, qk[j], st["gx"], st["gy"])
                qt = orc.time_derivatives(lg, p, qk[j], st["gx"], st["gy"], st["lim"])
                qk[j] = st["q"] + qt * np.repeat(dts[j], V) * a
                qk[j] = orc.update_bounds(lg, p, qk[j], st["gx"], st["gy"], st["lim"])
            exchange(qk)
        for j in parts:
            parts[j]["q"] = qk[j]
    res = {}
    for j, st in parts.items():
        pl = st["pl"]
        keep = np.r_[0: pl["n_own"], pl["n_real"]: pl["n_real"] + pl["n_own_ghost"]]
        res[j] = (pl["local2ref"][keep].copy(), st["q"].reshape(-1, V)[keep].copy())
    out[rank] = res
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("case,n_parts,steps", [("forward_step", 2, 8), ("forward_step", 4, 6),
                                                ("naca_local_dt", 4, 6), ("sod_first_order", 2, 10),
                                                ("mixed_elements", 4, 8)])
def test_decomposed_oracle_run_on_two_gloo_ranks(case, n_parts, steps, oracle):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    procs = [ctx.Process(target=_decomposed_run, args=(r, 2, case, n_parts, steps, out)) for r in range(2)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=300)
        assert pr.exitcode == 0
    mk_em, mk_ph, ic, alpha = _cases()[case]
    em = mk_em()
    ph = mk_ph()
    g = oracle.build_mesh(em)
    want = oracle.run_loop(g, oracle.physics(ph, em.group_names), np.ascontiguousarray(ic(g), np.float64).ravel(),
                           alpha, steps)["q"].reshape(-1, ph.V)
    got = np.full_like(want, np.nan)
    for rank in range(2):
        for j, (refs, q) in out[rank].items():
            got[refs] = q
    assert not np.isnan(got).any()
    assert got.tobytes() == want.tobytes()
