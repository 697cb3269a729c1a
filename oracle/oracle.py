"""Python access to the test oracles (test infrastructure only).

* ``Oracle``  — the C restatement (oracle/fvoracle.c -> liboracle.so).
* ``RefLib``  — the reference library compiled from its own sources with a
  reference example TU (oracle/_ref/libref_<variant>.so, built by
  ``make -C oracle ref`` when the reference sources are present).

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
use this module, and only as the checker / CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

FLUX = {"roe_fs": 1, "roe_st": 2, "burgers": 3, "diffusion": 4, "ns": 5, "burgers_diffusion": 6}
LIMITER = {"zero": 0, "michalak": 1, "venkat": 2, "minmod": 3}
DT = {"const": 0, "cfl_sum": 1, "cfl_min_signed": 2, "visc_min": 3, "visc_sum": 4}
BC = {"copy": 0, "wall": 1, "inlet_outlet": 2, "farfield": 3, "noslip": 4, "farfield_b0": 5, "tangent": 6}

_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


class _FvoMesh(C.Structure):
    _fields_ = [("n_nodes", C.c_int64), ("n_real", C.c_int64), ("n_total", C.c_int64),
                ("n_edges", C.c_int64), ("n_bound", C.c_int64),
                ("edge_cells", _u32p), ("edge_nodes", _u32p),
                ("enx", _dp), ("eny", _dp), ("elen", _dp), ("ecx", _dp), ("ecy", _dp),
                ("area", _dp), ("ccx", _dp), ("ccy", _dp),
                ("bound_edges", _u32p), ("bound_group", _i32p)]


class _FvoPhysics(C.Structure):
    _fields_ = [("V", C.c_int), ("flux", C.c_int), ("gamma", C.c_double), ("order2", C.c_int),
                ("limiter", C.c_int), ("K", C.c_double), ("dt_kind", C.c_int),
                ("cfl", C.c_double), ("dt_const", C.c_double), ("global_dt", C.c_int),
                ("n_groups", C.c_int), ("group_bc", _i32p), ("group_bv", _dp), ("positivity_guard", C.c_int),
                ("ghost_bv", _dp), ("diffusive", C.c_int), ("mu", C.c_double), ("pr", C.c_double),
                ("cp", C.c_double), ("r", C.c_double), ("smooth", C.c_int)]


def build_oracle():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load_oracle():
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        build_oracle()
    lib = C.CDLL(path)
    lib.fvo_mesh_build.restype = C.c_int
    lib.fvo_limiter_func.restype = C.c_double
    return lib


class GeomMesh:
    """Finite-volume mesh arrays in the reference's numbering (copied to numpy)."""

    FIELDS = ("edge_cells", "edge_nodes", "enx", "eny", "elen", "ecx", "ecy", "area", "ccx", "ccy",
              "bound_edges", "bound_group")

    def __init__(self, **kw):
        for k, v in kw.items():
            setattr(self, k, v)

    def struct(self):
        s = _FvoMesh()
        s.n_nodes, s.n_real, s.n_total = self.n_nodes, self.n_real, self.n_total
        s.n_edges, s.n_bound = self.n_edges, self.n_bound
        s.edge_cells = _ptr(self.edge_cells, _u32p); s.edge_nodes = _ptr(self.edge_nodes, _u32p)
        for k in ("enx", "eny", "elen", "ecx", "ecy", "area", "ccx", "ccy"):
            setattr(s, k, _ptr(getattr(self, k)))
        s.bound_edges = _ptr(self.bound_edges, _u32p); s.bound_group = _ptr(self.bound_group, _i32p)
        return s


class Oracle:
    """The C restatement.  ``phys`` is any object with the fields of
    ``fvgpu.Physics``; ``group_names`` orders its boundary groups."""

    def __init__(self):
        self.lib = _load_oracle()

    # -- mesh ---------------------------------------------------------------
    def build_mesh(self, em) -> GeomMesh:
        s = _FvoMesh()
        cells = np.ascontiguousarray(em.cells, np.int32)
        bn = np.ascontiguousarray(em.bnd_nodes, np.int32)
        bg = np.ascontiguousarray(em.bnd_group, np.int32)
        rc = self.lib.fvo_mesh_build(C.c_int64(em.nodes_x.size), _ptr(em.nodes_x), _ptr(em.nodes_y),
                                     C.c_int64(cells.shape[0]), _ptr(cells, _i32p), C.c_int64(bn.shape[0]),
                                     _ptr(bn, _i32p), _ptr(bg, _i32p), C.byref(s))
        if rc != 0:
            raise ValueError("boundary segment is not a mesh edge")
        E, NT, NB = s.n_edges, s.n_total, s.n_bound

        def cp(p, n, dt):
            return np.ctypeslib.as_array(p, shape=(n,)).astype(dt, copy=True)

        g = GeomMesh(n_nodes=s.n_nodes, n_real=s.n_real, n_total=NT, n_edges=E, n_bound=NB,
                     edge_cells=cp(s.edge_cells, 2 * E, np.uint32), edge_nodes=cp(s.edge_nodes, 2 * E, np.uint32),
                     enx=cp(s.enx, E, np.float64), eny=cp(s.eny, E, np.float64), elen=cp(s.elen, E, np.float64),
                     ecx=cp(s.ecx, E, np.float64), ecy=cp(s.ecy, E, np.float64),
                     area=cp(s.area, NT, np.float64), ccx=cp(s.ccx, NT, np.float64), ccy=cp(s.ccy, NT, np.float64),
                     bound_edges=cp(s.bound_edges, NB, np.uint32), bound_group=cp(s.bound_group, NB, np.int32))
        self.lib.fvo_mesh_free(C.byref(s))
        return g

    # -- physics ------------------------------------------------------------
    @staticmethod
    def physics(phys, group_names, ghost_bv=None):
        """ghost_bv: optional [n_bound, 4] boundary state per ghost (reference
        ghost order) replacing the group's state."""
        p = _FvoPhysics()
        p.V = phys.V; p.flux = FLUX[phys.flux]; p.gamma = phys.gamma; p.order2 = int(phys.order2)
        p.limiter = LIMITER[phys.limiter]; p.K = phys.K; p.dt_kind = DT[phys.dt_kind]
        p.cfl = phys.cfl; p.dt_const = phys.dt_const; p.global_dt = int(phys.global_dt)
        gbc = np.array([BC[phys.bcs[n][0]] for n in group_names], np.int32)
        gbv = np.array([list(phys.bcs[n][1]) if phys.bcs[n][1] is not None else [0.0] * 4
                        for n in group_names], np.float64).reshape(-1)
        p.n_groups = len(group_names)
        p.group_bc = _ptr(gbc, _i32p); p.group_bv = _ptr(gbv)
        p.positivity_guard = int(getattr(phys, "positivity_guard", False))
        p.diffusive = int(getattr(phys, "diffusive", False))
        p.mu, p.pr, p.cp, p.r = phys.mu, phys.pr, phys.cp, phys.r
        p.smooth = int(getattr(phys, "smooth", False))
        gh = None
        if ghost_bv is not None:
            gh = np.ascontiguousarray(ghost_bv, np.float64).reshape(-1)
            p.ghost_bv = _ptr(gh)
        p._keep = (gbc, gbv, gh)
        return p

    # -- stages -------------------------------------------------------------
    def calc_dt(self, g, p, q, global_min=False):
        dt = np.zeros(g.n_total)
        ms = g.struct()
        self.lib.fvo_calc_dt(C.byref(ms), C.byref(p), _ptr(q), _ptr(dt))
        if global_min:
            self.lib.fvo_min_dt(C.byref(ms), _ptr(dt))
        return dt

    def gradients(self, g, p, q):
        gx = np.zeros_like(q); gy = np.zeros_like(q)
        self.lib.fvo_calc_gradients(C.byref(g.struct()), C.byref(p), _ptr(q), _ptr(gx), _ptr(gy))
        return gx, gy

    def limiters(self, g, p, q, gx, gy):
        lim = np.zeros_like(q)
        self.lib.fvo_calc_limiters(C.byref(g.struct()), C.byref(p), _ptr(q), _ptr(gx), _ptr(gy), _ptr(lim))
        return lim

    def time_derivatives(self, g, p, q, gx, gy, lim):
        qt = np.zeros_like(q)
        self.lib.fvo_calc_time_derivatives(C.byref(g.struct()), C.byref(p), _ptr(q), _ptr(gx), _ptr(gy),
                                           _ptr(lim), _ptr(qt))
        return qt

    def update_bounds(self, g, p, q, gx, gy, lim):
        q = q.copy()
        self.lib.fvo_update_bounds(C.byref(g.struct()), C.byref(p), _ptr(q), _ptr(gx), _ptr(gy), _ptr(lim))
        return q

    def residuals(self, g, p, qt):
        R = np.zeros(p.V)
        self.lib.fvo_calc_residuals(C.byref(g.struct()), C.byref(p), _ptr(qt), _ptr(R))
        return R

    def run_loop(self, g, p, q0, alpha, max_step, max_time=1e10, tolerance=1e-16, print_interval=1):
        q = np.ascontiguousarray(q0, np.float64).copy()
        a = np.ascontiguousarray(alpha, np.float64)
        step = C.c_uint64(); t = C.c_double(); R = np.zeros(p.V); qt = np.zeros_like(q)
        self.lib.fvo_run_loop(C.byref(g.struct()), C.byref(p), _ptr(q), _ptr(a), C.c_int(a.size),
                              C.c_uint64(max_step), C.c_double(max_time), C.c_double(tolerance),
                              C.c_uint64(print_interval), C.byref(step), C.byref(t), _ptr(R), _ptr(qt))
        return dict(q=q, step=step.value, time=t.value, R=R, qt=qt)

    def smooth_residuals(self, g, p, qt):
        qt = np.ascontiguousarray(qt, np.float64).copy()
        self.lib.fvo_smooth_residuals(C.byref(g.struct()), C.byref(p), _ptr(qt))
        return qt

    def flux(self, p, qi, qj, n):
        f = np.zeros(p.V)
        self.lib.fvo_flux(C.byref(p), _ptr(f), _ptr(np.ascontiguousarray(qi, np.float64)),
                          _ptr(np.ascontiguousarray(qj, np.float64)), _ptr(np.ascontiguousarray(n, np.float64)))
        return f

    def flux_grad(self, p, qi, qj, gx, gy, n):
        f = np.zeros(p.V)
        a = [np.ascontiguousarray(x, np.float64) for x in (qi, qj, gx, gy, n)]
        self.lib.fvo_flux_grad(C.byref(p), _ptr(f), *[_ptr(x) for x in a])
        return f

    def bc(self, p, group, q, n):
        b = np.zeros(p.V)
        self.lib.fvo_bc(C.byref(p), C.c_int(group), _ptr(b), _ptr(np.ascontiguousarray(q, np.float64)),
                        _ptr(np.ascontiguousarray(n, np.float64)))
        return b

    def limiter_func(self, p, y):
        return self.lib.fvo_limiter_func(C.byref(p), C.c_double(y))

    def boundary_force(self, g, p, q, group):
        fx = C.c_double(); fy = C.c_double()
        self.lib.fvo_boundary_force(C.byref(g.struct()), C.byref(p), _ptr(q), C.c_int(group),
                                    C.byref(fx), C.byref(fy))
        return fx.value, fy.value


# ---------------------------------------------------------------------------
# The reference compiled from its own sources
# ---------------------------------------------------------------------------
def ref_available(variant="shockTube") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{variant}.so"))


class RefLib:
    """One reference build (reference library + one example TU + harness)."""

    def __init__(self, variant: str):
        path = os.path.join(REF_DIR, f"libref_{variant}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.variant = variant
        self.lib = C.CDLL(path)  # RTLD_LOCAL: each variant keeps its own globals
        self.lib.ref_bc_get.restype = C.c_void_p
        self.lib.ref_limiter_k.restype = C.c_double
        self.lib.ref_limiter_func.restype = C.c_double
        self.lib.ref_limiter_func.argtypes = [C.c_double]
        self.V = self.lib.ref_vars()
        self._tmp = tempfile.TemporaryDirectory(prefix="fvref_")

    def flags(self):
        f = np.zeros(6, np.int32)
        self.lib.ref_flags(_ptr(f, _i32p))
        return dict(zip(("grad", "lim", "linear", "diffusive", "global_dt", "smooth"), f.tolist()))

    def set_consts(self, gamma=-1.0, cfl=-1.0, mach=-1.0):
        self.lib.ref_set_consts(C.c_double(gamma), C.c_double(cfl), C.c_double(mach))

    def bc_get(self, name):
        return self.lib.ref_bc_get(name.encode())

    def bc_set(self, name, fn_addr):
        self.lib.ref_bc_set(name.encode(), C.c_void_p(fn_addr))

    def read_mesh(self, em, write_msh):
        base = os.path.join(self._tmp.name, "mesh")
        write_msh(base + ".msh", em)
        if self.lib.ref_read_mesh(base.encode()) != 0:
            raise ValueError("reference reader rejected the mesh")
        s = np.zeros(5, np.int64)
        self.lib.ref_mesh_sizes(_ptr(s, C.POINTER(C.c_int64)))
        self.n_nodes, self.n_real, self.n_total, self.n_edges, self.n_bound = (int(x) for x in s)
        self.nq = self.V * self.n_total

    def geometry(self) -> GeomMesh:
        E, NT, NB = self.n_edges, self.n_total, self.n_bound
        ec = np.zeros(2 * E, np.uint32); en = np.zeros(2 * E, np.uint32)
        f = {k: np.zeros(E) for k in ("enx", "eny", "elen", "ecx", "ecy")}
        a = {k: np.zeros(NT) for k in ("area", "ccx", "ccy")}
        be = np.zeros(NB, np.uint32); bt = np.zeros(NB, np.uint32)
        self.lib.ref_mesh_get(_ptr(ec, _u32p), _ptr(en, _u32p), *[_ptr(f[k]) for k in ("enx", "eny", "elen", "ecx", "ecy")],
                              *[_ptr(a[k]) for k in ("area", "ccx", "ccy")], _ptr(be, _u32p), _ptr(bt, _u32p))
        return GeomMesh(n_nodes=self.n_nodes, n_real=self.n_real, n_total=NT, n_edges=E, n_bound=NB,
                        edge_cells=ec, edge_nodes=en, bound_edges=be, bound_group=bt.astype(np.int32) - 1,
                        **f, **a)

    def initial_state(self):
        q = np.zeros(self.nq); self.lib.ref_initial_state(_ptr(q)); return q

    def calc_dt(self, q, global_min=False):
        dt = np.zeros(self.nq)
        self.lib.ref_calc_dt(_ptr(np.ascontiguousarray(q)), _ptr(dt), C.c_int(int(global_min)))
        return dt[:: self.V].copy()

    def gradients(self, q):
        gx = np.zeros(self.nq); gy = np.zeros(self.nq)
        self.lib.ref_calc_gradients(_ptr(np.ascontiguousarray(q)), _ptr(gx), _ptr(gy))
        return gx, gy

    def limiters(self, q, gx, gy):
        lim = np.zeros(self.nq)
        self.lib.ref_calc_limiters(_ptr(q), _ptr(gx), _ptr(gy), _ptr(lim))
        return lim

    def time_derivatives(self, q, gx, gy, lim):
        qt = np.zeros(self.nq)
        self.lib.ref_calc_time_derivatives(_ptr(q), _ptr(gx), _ptr(gy), _ptr(lim), _ptr(qt))
        return qt

    def update_bounds(self, q, gx, gy, lim):
        q = np.ascontiguousarray(q).copy()
        self.lib.ref_update_bounds(_ptr(q), _ptr(gx), _ptr(gy), _ptr(lim))
        return q

    def flux(self, qi, qj, n):
        f = np.zeros(self.V)
        self.lib.ref_flux(_ptr(f), _ptr(np.ascontiguousarray(qi, np.float64)),
                          _ptr(np.ascontiguousarray(qj, np.float64)), _ptr(np.ascontiguousarray(n, np.float64)))
        return f

    def smooth_residuals(self, qt):
        t = np.ascontiguousarray(qt, np.float64).copy()
        self.lib.ref_smooth_residuals(_ptr(t))
        return t

    def flux_grad(self, qi, qj, gx, gy, n):
        f = np.zeros(self.V)
        a = [np.ascontiguousarray(x, np.float64) for x in (qi, qj, gx, gy, n)]
        self.lib.ref_flux_grad(_ptr(f), *[_ptr(x) for x in a])
        return f

    def run_loop(self, q0, alpha, max_step, max_time=1e10, tolerance=1e-16, print_interval=1):
        q = np.ascontiguousarray(q0, np.float64).copy()
        a = np.ascontiguousarray(alpha, np.float64)
        step = C.c_uint64(); t = C.c_double(); R = np.zeros(self.V); qt = np.zeros(self.nq)
        self.lib.ref_run_loop(_ptr(q), _ptr(a), C.c_int(a.size), C.c_uint64(max_step), C.c_double(max_time),
                              C.c_double(tolerance), C.c_uint64(print_interval), C.byref(step), C.byref(t),
                              _ptr(R), _ptr(qt))
        return dict(q=q, step=step.value, time=t.value, R=R, qt=qt)

    def run(self, max_step, max_time=1e10, tolerance=1e-16, print_interval=1, verbose=False):
        q = np.zeros(self.nq)
        self.lib.ref_run(_ptr(q), C.c_uint64(max_step), C.c_double(max_time), C.c_double(tolerance),
                         C.c_uint64(print_interval), C.c_int(int(verbose)))
        return q
