"""Small parity cases shared by the oracle, fixture and GPU tests.

Each case is a mesh from ``meshgen``, a ``physics.Physics`` description, an
initial condition and the reference build (oracle/_ref variant) whose
example translation unit defines the same physics.  Sizes are small so the
CPU oracle and the reference finish in well under a second.
"""
import numpy as np

import meshgen
import physics as P


def _prim_to_cons(rho, u, v, p, gamma=1.4):
    return np.stack([rho, rho * u, rho * v, p / (gamma - 1) + 0.5 * rho * (u * u + v * v)], 1)


def random_euler_state(n, seed, rho=(0.5, 1.5), vel=0.5, p=(0.5, 1.5)):
    r = np.random.default_rng(seed)
    return _prim_to_cons(r.uniform(*rho, n), r.uniform(-vel, vel, n), r.uniform(-vel, vel, n),
                         r.uniform(*p, n)).ravel()


def _renamed(em, names):
    em.group_names = list(names)
    return em


def _guarded(ph):
    ph.positivity_guard = True
    return ph


CASES = {
    # name: (mesh builder, physics, ic(geom)->q, alpha, steps, ref variant, ref bc aliases, ref consts)
    "sod": dict(mesh=lambda: meshgen.sod_strip(40, 4), phys=lambda: P.sod(),
                ic=lambda g: P.ic_sod(g.ccx).ravel(), alpha=P.RK1_ALPHA, steps=40,
                ref="forwardStep", alias={"ends": ("shockTube", "wall")}, consts=dict(cfl=0.5)),
    "sod_st": dict(mesh=lambda: meshgen.sod_strip(40, 4),
                   phys=lambda: P.Physics(V=4, flux="roe_st", dt_kind="const", dt_const=2e-5,
                                          bcs={"wall": ("copy", None), "ends": ("copy", None)}),
                   ic=lambda g: P.ic_sod(g.ccx).ravel(), alpha=P.RK5_ALPHA, steps=20,
                   ref="shockTube", alias={"ends": ("shockTube", "wall")}, consts={}),
    "step_o1": dict(mesh=lambda: meshgen.forward_step(n=20), phys=lambda: P.forward_step(order2=False),
                    ic=lambda g: P.ic_forward_step(g.n_total).ravel(), alpha=P.RK5_ALPHA, steps=30,
                    ref="forwardStep", alias={"step": ("forwardStep", "wall")}, consts=dict(cfl=0.8)),
    "step_o2_venk5": dict(mesh=lambda: meshgen.forward_step(n=20),
                          phys=lambda: P.forward_step(order2=True, limiter="venkat", K=5.0),
                          ic=lambda g: P.ic_forward_step(g.n_total).ravel(), alpha=P.RK5_ALPHA, steps=30,
                          ref="forwardStep_o2venk5", alias={"step": ("forwardStep_o2venk5", "wall")},
                          consts=dict(cfl=0.8)),
    "step_o2_guard": dict(mesh=lambda: meshgen.forward_step(n=20),
                          phys=lambda: _guarded(P.forward_step(order2=True, limiter="venkat", K=5.0)),
                          ic=lambda g: P.ic_forward_step(g.n_total).ravel(), alpha=P.RK5_ALPHA, steps=30,
                          ref=None, alias={}, consts=dict(cfl=0.8)),
    "step_o2_mich": dict(mesh=lambda: meshgen.forward_step(n=20),
                         phys=lambda: P.forward_step(order2=True, limiter="michalak", K=7.5),
                         ic=lambda g: P.ic_forward_step(g.n_total).ravel(), alpha=P.RK5_ALPHA, steps=30,
                         ref="forwardStep_o2mich", alias={"step": ("forwardStep_o2mich", "wall")},
                         consts=dict(cfl=0.8)),
    "naca": dict(mesh=lambda: meshgen.naca_ogrid(ni=48, nj=12, r_far=10.0),
                 phys=lambda: P.naca(), ic=lambda g: P.ic_naca(g.n_total).ravel(), alpha=P.RK5_ALPHA,
                 steps=30, ref="naca", alias={}, consts=dict(cfl=1.0)),
    "heat": dict(mesh=lambda: meshgen.rect_tri(16, 16, 1.0, 1.0, side_names=("wall", "wall")),
                 phys=lambda: P.heat(), ic=lambda g: P.ic_heat(g.ccx, g.ccy).ravel(),
                 alpha=P.RK5_ALPHA, steps=30, ref="heatTransfer", alias={}, consts={}),
    "flat_plate": dict(mesh=lambda: meshgen.flat_plate(nx0=6, nx1=18, ny=12),
                       phys=lambda: P.flat_plate(), ic=lambda g: P.ic_forward_step(g.n_total, mach=0.2).ravel(),
                       alpha=P.RK5_ALPHA, steps=30, ref="flatPlate", alias={}, consts={}),
    "naca_transient": dict(mesh=lambda: _renamed(meshgen.naca_ogrid(ni=48, nj=12, r_far=10.0), ["wall", "farfield"]),
                           phys=lambda: P.naca_transient(),
                           ic=lambda g: P.ic_forward_step(g.n_total, mach=0.8).ravel(),
                           alpha=P.RK5_ALPHA, steps=30, ref="nacaTransient", alias={}, consts={}),
    "burgers_diffusion": dict(mesh=lambda: meshgen.rect_tri(16, 16, 1.0, 1.0, side_names=("wall", "wall")),
                              phys=lambda: P.burgers_diffusion(),
                              ic=lambda g: np.zeros(g.n_total * 2), alpha=P.RK5_ALPHA, steps=30, ref="tests",
                              alias={}, consts={}),
    "burgers": dict(mesh=lambda: meshgen.rect_tri(16, 16, 1.0, 1.0, side_names=("wall", "wall")),
                    phys=lambda: P.burgers(), ic=lambda g: P.ic_burgers(g.ccx, g.ccy).ravel(),
                    alpha=P.RK5_ALPHA, steps=30, ref="burgers", alias={}, consts={}),
}


def make_ref(case, em):
    """Load the reference build for a case and read its mesh."""
    from oracle import RefLib
    ref = RefLib(case["ref"])
    others = {}
    for name, (variant, src) in case["alias"].items():
        lib = ref if variant == case["ref"] else others.setdefault(variant, RefLib(variant))
        ref.bc_set(name, lib.bc_get(src))
    ref._keep = others
    if case["consts"]:
        ref.set_consts(**case["consts"])
    ref.read_mesh(em, meshgen.write_msh41)
    return ref
