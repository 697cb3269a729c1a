"""Physics descriptions for the device kernels (the "physics kinds").

fvhyper takes the PDE as link-time user functions (examples/*/main.cpp:
calc_flux, calc_dt, limiter_func, boundaries::bounds).  The GPU path cannot
call host function pointers, so it implements the physics the reference
examples define as device kinds, selected by name:

* flux:     ``roe_fs`` (examples/forwardStep/main.cpp:72-135),
            ``roe_st`` (examples/shockTube/main.cpp:68-135, naca/main.cpp:71-137;
            same Roe-"cures" flux, central part associated differently),
            ``burgers`` (examples/burgers/main.cpp:68-96, V = 2),
            ``diffusion`` (examples/heatTransfer/main.cpp:63-73, V = 1: F = -grad T . n
            with the face gradient of gradient_for_diffusion, explicit.cpp:70-109),
            ``ns`` (examples/flatPlate/main.cpp:126-225 = nacaTransient/main.cpp:130-229:
            the roe_st flux minus viscous stresses and heat conduction from the face
            gradient; constants mu, pr, cp, r),
            ``burgers_diffusion`` (tests/tests.cpp:76-117, V = 2: burgers plus
            -grad q . n per variable from the face gradient)
* limiter:  ``zero`` (shockTube/main.cpp:60-62), ``michalak``
            (forwardStep/main.cpp:57-66), ``minmod`` (burgers/main.cpp:51-53),
            ``venkat`` (Venkatakrishnan 1995, not in the reference)
* dt:       ``cfl_sum`` (forwardStep/main.cpp:140-185), ``cfl_min_signed``
            (naca/main.cpp:142-183), ``const`` (shockTube/main.cpp:140-147),
            ``visc_min`` (flatPlate/main.cpp:230-277), ``visc_sum``
            (nacaTransient/main.cpp:234-285)
* bc:       ``copy`` (shockTube/main.cpp:158-163), ``wall``
            (forwardStep/main.cpp:262-269), ``inlet_outlet``
            (forwardStep/main.cpp:194-261), ``farfield`` (naca/main.cpp:192-259),
            ``farfield_b0`` (flatPlate/main.cpp:286-352: farfield with
            b[2] = b[0]*(...)), ``noslip`` (flatPlate/main.cpp:361-366),
            ``tangent`` (tests/tests.cpp:132-135, V = 2: b = (-n_y, n_x));
            the inflow/far-field kinds take the far-field state bv[4].
"""
from __future__ import annotations

import dataclasses
from typing import Dict, Optional, Sequence, Tuple

RK5_ALPHA = (0.0695, 0.1602, 0.2898, 0.506, 1.0)  # explicit.cpp:681-687
RK1_ALPHA = (1.0,)


@dataclasses.dataclass
class Physics:
    V: int = 4
    flux: str = "roe_fs"
    gamma: float = 1.4
    order2: bool = False
    limiter: str = "zero"
    K: float = 7.5
    dt_kind: str = "cfl_sum"
    cfl: float = 0.5
    dt_const: float = 0.0
    global_dt: bool = True
    bcs: Dict[str, Tuple[str, Optional[Sequence[float]]]] = dataclasses.field(default_factory=dict)
    # not in the reference: fall back to the cell value on MUSCL face states
    # with rho <= 0 or p <= 0 (off = the reference's scheme, bit for bit)
    positivity_guard: bool = False
    # solver::diffusive_gradients: the flux receives the corrected face
    # gradient; with order2 off the gradients are computed without limiter
    # or interpolation (examples/heatTransfer/main.cpp:18-25)
    diffusive: bool = False
    # consts:: of the Navier-Stokes examples (flatPlate/main.cpp:30-37)
    mu: float = 0.0
    pr: float = 1.0
    cp: float = 1.0
    r: float = 1.0
    # solver::smooth_residuals: two Jacobi sweeps of implicit residual
    # smoothing after each stage's time derivatives (explicit.cpp:32-66, 743)
    smooth: bool = False


def euler_state(rho, u, v, p, gamma=1.4):
    return (rho, rho * u, rho * v, p / (gamma - 1) + 0.5 * rho * (u * u + v * v))


def forward_step_bv(mach=3.0, gamma=1.4):
    """Inflow state of examples/forwardStep/main.cpp:196-201 (same arithmetic)."""
    b_pressure = 1.0
    bv0 = 1.4
    bv1 = bv0 * mach
    bv2 = bv0 * 0.0
    bv3 = b_pressure / (gamma - 1) + 0.5 / bv0 * (bv1 * bv1 + bv2 * bv2)
    return (bv0, bv1, bv2, bv3)


def naca_bv(gamma=1.4):
    """Far-field state of examples/naca/main.cpp:194-199 (M 0.8, alpha 1.25 deg)."""
    b_pressure = 1.0
    bv0 = 1.4
    bv1 = bv0 * 0.8
    bv2 = bv0 * 0.0175
    bv3 = b_pressure / (gamma - 1) + 0.5 / bv0 * (bv1 * bv1 + bv2 * bv2)
    return (bv0, bv1, bv2, bv3)


def sod(cfl=0.5, flux="roe_fs"):
    """Sod tube: first-order Roe, CFL-sum global dt, slip walls, copy ends."""
    return Physics(V=4, flux=flux, order2=False, limiter="zero", dt_kind="cfl_sum", cfl=cfl,
                   global_dt=True, bcs={"wall": ("wall", None), "ends": ("copy", None)})


def forward_step(order2=True, limiter="venkat", K=5.0, cfl=0.8, mach=3.0):
    bv = forward_step_bv(mach)
    return Physics(V=4, flux="roe_fs", order2=order2, limiter=limiter if order2 else "michalak",
                   K=K, dt_kind="cfl_sum", cfl=cfl, global_dt=True,
                   bcs={"wall": ("wall", None), "step": ("wall", None),
                        "inlet": ("inlet_outlet", bv), "outlet": ("inlet_outlet", bv)})


def naca(cfl=1.0, K=7.5, limiter="michalak"):
    return Physics(V=4, flux="roe_st", order2=True, limiter=limiter, K=K, dt_kind="cfl_min_signed",
                   cfl=cfl, global_dt=False,
                   bcs={"airfoil": ("wall", None), "farfield": ("farfield", naca_bv())})


def riemann_strip(order2=True, limiter="venkat", K=5.0, cfl=0.8):
    return Physics(V=4, flux="roe_fs", order2=order2, limiter=limiter, K=K, dt_kind="cfl_sum", cfl=cfl,
                   global_dt=True, bcs={"wall": ("wall", None), "ends": ("copy", None)})


def heat(dt=1e-5):
    """examples/heatTransfer/main.cpp: u_t = div(grad u), constant dt, zero-flux walls."""
    return Physics(V=1, flux="diffusion", order2=False, limiter="zero", dt_kind="const", dt_const=dt,
                   global_dt=True, diffusive=True, bcs={"wall": ("copy", None)})


NS_CONSTS = dict(mu=2e-5, pr=0.72, cp=1.0, r=8.3145)   # flatPlate/main.cpp:30-37


def flat_plate(cfl=2.0, mach=0.2):
    """examples/flatPlate: laminar boundary layer, Navier-Stokes with MUSCL +
    Michalak, local viscous dt (min form), far field / slip / no-slip walls."""
    bv = forward_step_bv(mach)   # flatPlate/main.cpp:288-293, the same arithmetic
    return Physics(V=4, flux="ns", order2=True, limiter="michalak", K=7.5, dt_kind="visc_min", cfl=cfl,
                   global_dt=False, diffusive=True, **NS_CONSTS,
                   bcs={"top": ("farfield_b0", bv), "bot0": ("wall", None), "bot1": ("noslip", None),
                        "left": ("farfield_b0", bv), "right": ("farfield_b0", bv)})


def naca_transient(cfl=1.5, mach=0.8):
    """examples/nacaTransient: Navier-Stokes with cell values as face states
    (gradients for the viscous terms only), global viscous dt (sum form)."""
    bv = forward_step_bv(mach)   # nacaTransient/main.cpp:296-301
    return Physics(V=4, flux="ns", order2=False, limiter="michalak", K=7.5, dt_kind="visc_sum", cfl=cfl,
                   global_dt=True, diffusive=True, **NS_CONSTS,
                   bcs={"wall": ("noslip", None), "farfield": ("farfield_b0", bv)})


def burgers_diffusion(dt=1e-3):
    """The reference's regression-test physics (tests/tests.cpp:40-150):
    Burgers advection plus diffusion, MUSCL with minmod, residual smoothing,
    local constant dt, tangential boundary state."""
    return Physics(V=2, flux="burgers_diffusion", order2=True, limiter="minmod", K=7.5, dt_kind="const",
                   dt_const=dt, global_dt=False, diffusive=True, smooth=True, bcs={"wall": ("tangent", None)})


def burgers(dt=1e-4):
    return Physics(V=2, flux="burgers", order2=True, limiter="minmod", K=7.5, dt_kind="const",
                   dt_const=dt, global_dt=True, bcs={"wall": ("copy", None)})


# ---- initial conditions (arrays over all n_total cells, AoS [n_total, V]) ----
def ic_sod(ccx, gamma=1.4):
    """examples/shockTube/main.cpp:40-57."""
    import numpy as np
    q = np.zeros((ccx.size, 4))
    left = ccx < 0.5
    q[left] = (1.0, 0.0, 0.0, 1.0 / (gamma - 1))
    q[~left] = (0.125, 0.0, 0.0, 0.1 / (gamma - 1))
    return q


def ic_uniform(n, state):
    import numpy as np
    q = np.zeros((n, len(state)))
    q[:] = state
    return q


def ic_forward_step(n, mach=3.0, gamma=1.4):
    """examples/forwardStep/main.cpp:44-54."""
    return ic_uniform(n, (1.4, 1.4 * mach, 1.4 * 0.0, 1.0 / (gamma - 1) + 0.5 * 1.4 * (mach * mach + 0.0 * 0.0)))


def ic_naca(n, gamma=1.4):
    """examples/naca/main.cpp:43-53."""
    return ic_uniform(n, (1.4, 1.4 * 0.8, 1.4 * 0.0175, 1.0 / (gamma - 1) + 0.5 * 1.4 * (0.8 * 0.8 + 0.0175 * 0.0175)))


def ic_riemann(ccx, left, right, gamma=1.4):
    """Left/right primitive states (rho, u, p) split at x = 0.5, v = 0."""
    import numpy as np
    q = np.zeros((ccx.size, 4))
    m = ccx < 0.5
    q[m] = euler_state(left[0], left[1], 0.0, left[2], gamma)
    q[~m] = euler_state(right[0], right[1], 0.0, right[2], gamma)
    return q


def ic_heat(ccx, ccy):
    """examples/heatTransfer/main.cpp:32-45 (radius test sqrt(r2) < 0.4*0.4 as written there)."""
    import numpy as np
    q = np.zeros((ccx.size, 1))
    x = ccx - 0.5; y = ccy - 0.5
    q[np.sqrt(x * x + y * y) < 0.4 * 0.4] = 1.0
    return q


def ic_burgers(ccx, ccy):
    """examples/burgers/main.cpp:35-48."""
    import numpy as np
    q = np.zeros((ccx.size, 2))
    x = ccx - 0.5; y = ccy - 0.5
    m = (x * x + y * y) < 0.25 * 0.25
    q[m] = (1.0, -1.0)
    return q
