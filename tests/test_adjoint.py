"""Discrete adjoint of the time loop (fv_adjoint_*): the gradient of the
time-integrated pressure force on the step face with respect to the inflow
Mach number and inflow density bins, on the second-order forward-step case
(Green-Gauss + Venkatakrishnan K = 5, Roe, RK5, CFL 0.8, positivity guard).

- its forward run is fv_run's FP64_EXACT step, bit for bit;
- its loss is the loss of an FP64 reference run assembled from the oracle's
  stage functions (CPU), and its gradient matches central finite
  differences of that reference (h = 1e-6);
- over 300 steps with checkpoints every 50 (recomputed segments) the
  gradient matches central finite differences of the GPU loss;
- torch.autograd.gradcheck passes through the autograd wrapper.
"""
import numpy as np
import pytest

import meshgen
import physics as P

pytestmark = pytest.mark.gpu

N_BINS = 8


def setup_case(n=20):
    em = meshgen.forward_step(n=n)
    ph = P.forward_step(order2=True, limiter="venkat", K=5.0, cfl=0.8)
    ph.positivity_guard = True
    return em, ph


def theta0(nb=N_BINS, seed=5):
    return np.concatenate([[3.0], np.random.default_rng(seed).normal(0.0, 0.01, nb)])


def ghost_states(em, geo, ph, theta, nb=N_BINS, lo=0.0, hi=1.0):
    """Reference-order boundary states of the inflow parametrisation."""
    M = theta[0]
    bv = np.array(ph.bcs["inlet"][1])
    rho_inf = bv[0]
    p_inf = (ph.gamma - 1) * (bv[3] - 0.5 * (bv[1] ** 2 + bv[2] ** 2) / bv[0])
    out = np.zeros((em.bnd_group.size, 4))
    for r, gi in enumerate(em.bnd_group):
        name = em.group_names[gi]
        if ph.bcs[name][0] not in ("inlet_outlet", "farfield"):
            continue
        rho = rho_inf
        if name == "inlet":
            y = geo.ecy[geo.bound_edges[r]]
            b = min(max(int(np.floor((y - lo) / (hi - lo) * nb)), 0), nb - 1)
            rho = rho_inf * (1 + theta[1 + b])
        out[r] = (rho, rho * M, 0.0, p_inf / (ph.gamma - 1) + 0.5 * rho * M * M)
    return out, rho_inf, p_inf


def oracle_loss(oracle, em, ph, theta, steps):
    """The loss from the oracle's stage functions: run()'s loop (explicit.cpp:
    657-817) with the inflow states per ghost, summing dt_n * p le over the
    step faces at each step's start."""
    g = oracle.build_mesh(em)
    bvg, rho_inf, p_inf = ghost_states(em, g, ph, theta)
    p = oracle.physics(ph, em.group_names, ghost_bv=bvg)
    M = theta[0]
    q = np.tile([rho_inf, rho_inf * M, 0.0, p_inf / (ph.gamma - 1) + 0.5 * rho_inf * M * M], g.n_total)
    z = np.zeros_like(q)
    q = oracle.update_bounds(g, p, q, z, z, z)
    step = em.group_names.index("step")
    loss = 0.0
    for _ in range(steps):
        dt = oracle.calc_dt(g, p, q, True)[0]
        s = 0.0
        for b in range(g.n_bound):
            if g.bound_group[b] != step:
                continue
            e = g.bound_edges[b]
            c = g.edge_cells[2 * e]
            v = q[4 * c: 4 * c + 4]
            s += (ph.gamma - 1) * (v[3] - 0.5 / v[0] * (v[1] ** 2 + v[2] ** 2)) * g.elen[e]
        loss += s * dt
        qs = q
        for a in P.RK5_ALPHA:
            gx, gy = oracle.gradients(g, p, qs)
            lim = oracle.limiters(g, p, qs, gx, gy)
            qt = oracle.time_derivatives(g, p, qs, gx, gy, lim)
            qn = q + qt * np.repeat(np.full(g.n_total, dt), 4) * a
            qs = oracle.update_bounds(g, p, qn, gx, gy, lim)
        q = qs
    return loss, q


def test_forward_is_the_exact_time_loop_and_the_oracle_loss(oracle):
    import fvgpu

    em, ph = setup_case()
    mesh = fvgpu.Mesh.from_elements(em)
    steps = 30
    th = theta0()
    adj = fvgpu.Adjoint(mesh, ph, n_steps=steps, checkpoint_every=10, n_bins=N_BINS)
    L = adj.loss(th)
    qa = adj.final_state()
    # fv_run with the same initial state and inflow states
    geo = oracle.build_mesh(em)
    bvg, rho_inf, p_inf = ghost_states(em, geo, ph, th)
    M = th[0]
    s = fvgpu.Solver(mesh, ph, "fp64_exact")
    s.set_ghost_states(bvg)
    s.set_state(np.tile([rho_inf, rho_inf * M, 0.0, p_inf / (ph.gamma - 1) + 0.5 * rho_inf * M * M], mesh.n_total))
    s.run(steps, print_interval=10 ** 9)
    assert qa.tobytes() == s.get_state().tobytes()
    s.close()
    # the oracle's loop gives the same state and (summed in another order) the same loss
    Lo, qo = oracle_loss(oracle, em, ph, th, steps)
    assert qa.tobytes() == qo.tobytes()
    assert abs(L - Lo) <= 1e-13 * abs(Lo)
    adj.close()


def test_gradient_matches_fp64_reference_finite_differences(oracle):
    """dL/dM from the adjoint vs central differences of the oracle-built loss."""
    import fvgpu

    em, ph = setup_case()
    mesh = fvgpu.Mesh.from_elements(em)
    steps = 30
    th = theta0()
    adj = fvgpu.Adjoint(mesh, ph, n_steps=steps, checkpoint_every=10, n_bins=N_BINS)
    _, g = adj.gradient(th)
    h = 1e-6
    tp, tm = th.copy(), th.copy()
    tp[0] += h; tm[0] -= h
    fd = (oracle_loss(oracle, em, ph, tp, steps)[0] - oracle_loss(oracle, em, ph, tm, steps)[0]) / (2 * h)
    assert abs(g[0] - fd) <= 1e-6 * abs(fd), (g[0], fd)
    adj.close()


def test_gradient_with_checkpoints_matches_finite_differences():
    import fvgpu

    em, ph = setup_case()
    mesh = fvgpu.Mesh.from_elements(em)
    adj = fvgpu.Adjoint(mesh, ph, n_steps=300, checkpoint_every=50, n_bins=N_BINS)
    th = theta0()
    L, g = adj.gradient(th)
    h = 1e-6
    fd = np.zeros_like(g)
    for i in range(g.size):
        tp, tm = th.copy(), th.copy()
        tp[i] += h; tm[i] -= h
        fd[i] = (adj.loss(tp) - adj.loss(tm)) / (2 * h)
    rel = np.linalg.norm(g - fd) / np.linalg.norm(fd)
    print(f"adjoint vs FD over 300 steps: loss {L:.6e}, |g| {np.linalg.norm(g):.4e}, relative error {rel:.2e}")
    assert rel <= 1e-6
    big = np.abs(fd) > 1e-3 * np.abs(fd).max()
    assert np.all(np.abs(g - fd)[big] <= 5e-6 * np.abs(fd)[big])
    adj.close()


def test_autograd_wrapper_gradcheck():
    import torch

    import fvgpu
    from fv_autograd import inflow_loss

    em, ph = setup_case()
    mesh = fvgpu.Mesh.from_elements(em)
    adj = fvgpu.Adjoint(mesh, ph, n_steps=60, checkpoint_every=20, n_bins=N_BINS)
    th = torch.tensor(theta0(), dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda t: inflow_loss(t, adj), (th,), eps=1e-6, atol=1e-8, rtol=1e-5)
    adj.close()
