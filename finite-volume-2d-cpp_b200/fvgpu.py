"""Python binding of the C ABI in include/fvgpu.h (libfvgpu.so).

This is a thin ctypes layer for tests, benchmarks and scripting; the C++
drop-in for fvhyper's own API lives in ``shim/``.  There is no CPU fallback:
if libfvgpu.so is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Callable, Optional, Sequence

import numpy as np

import physics as _phys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfvgpu.so")

FLUX = {"roe_fs": 1, "roe_st": 2, "burgers": 3, "diffusion": 4, "ns": 5, "burgers_diffusion": 6}
LIMITER = {"zero": 0, "michalak": 1, "venkat": 2, "minmod": 3}
DT = {"const": 0, "cfl_sum": 1, "cfl_min_signed": 2, "visc_min": 3, "visc_sum": 4}
BC = {"copy": 0, "wall": 1, "inlet_outlet": 2, "farfield": 3, "noslip": 4, "farfield_b0": 5, "tangent": 6}
PREC = {"fp64_exact": 0, "fp64": 1, "fp32": 2}

_dp = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_u32p = C.POINTER(C.c_uint32)
_i64p = C.POINTER(C.c_int64)


class FvError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"fvgpu error {code}: {msg}")
        self.code = code


class _Physics(C.Structure):
    _fields_ = [("V", C.c_int32), ("flux", C.c_int32), ("order2", C.c_int32), ("limiter", C.c_int32),
                ("dt_kind", C.c_int32), ("global_dt", C.c_int32), ("gamma", C.c_double), ("K", C.c_double),
                ("cfl", C.c_double), ("dt_const", C.c_double), ("n_groups", C.c_int32),
                ("group_bc", _i32p), ("group_bv", _dp), ("positivity_guard", C.c_int32),
                ("diffusive", C.c_int32), ("mu", C.c_double), ("pr", C.c_double), ("cp", C.c_double),
                ("r", C.c_double), ("smooth_residuals", C.c_int32)]


_PRINT_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_uint64, C.c_double, _dp, C.c_int32)


class _RunOptions(C.Structure):
    _fields_ = [("max_step", C.c_uint64), ("max_time", C.c_double), ("tolerance", C.c_double),
                ("print_interval", C.c_uint64), ("n_alpha", C.c_int32), ("alpha", _dp),
                ("restart", C.c_int32), ("on_print", _PRINT_CB), ("user", C.c_void_p)]


class _RunInfo(C.Structure):
    _fields_ = [("step", C.c_uint64), ("time", C.c_double), ("R", C.c_double * 8), ("R0", C.c_double * 8)]


_lib = None


def _torch_nccl():
    """PyTorch's bundled NCCL library (found without importing torch), or None."""
    try:
        import importlib.util
        spec = importlib.util.find_spec("nvidia.nccl")
    except (ImportError, ValueError):
        return None
    for base in (spec.submodule_search_locations or []) if spec else []:
        path = os.path.join(base, "lib", "libnccl.so.2")
        if os.path.exists(path):
            return path
    return None


def lib():
    """Load libfvgpu.so (raises if it is not built: there is no fallback)."""
    global _lib
    if _lib is None:
        # decompositions load NCCL on first use: make it PyTorch's copy, so a
        # later `import torch` in this process finds the NCCL it was built for
        if "FVGPU_NCCL_LIB" not in os.environ:
            path = _torch_nccl()
            if path:
                os.environ["FVGPU_NCCL_LIB"] = path
        if not os.path.exists(LIB_PATH):
            raise FvError(-100, f"{LIB_PATH} is not built; run `make -C {HERE}` (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        L.fv_last_error.restype = C.c_char_p
        for name in ("fv_mesh_create", "fv_mesh_read_msh", "fv_solver_create"):
            getattr(L, name).restype = C.c_int
        L.fv_stage_update.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, _dp]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise FvError(rc, lib().fv_last_error().decode(errors="replace"))


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


class Mesh:
    """FV mesh built by the native library exactly as fvhyper's reader builds it."""

    def __init__(self, handle, group_names):
        self._h = C.c_void_p(handle)
        self.group_names = list(group_names)
        s = np.zeros(5, np.int64)
        _check(lib().fv_mesh_sizes(self._h, _p(s, _i64p)))
        self.n_nodes, self.n_real, self.n_total, self.n_edges, self.n_bound = (int(v) for v in s)

    @classmethod
    def from_elements(cls, em):
        h = C.c_void_p()
        cells = np.ascontiguousarray(em.cells, np.int32)
        bn = np.ascontiguousarray(em.bnd_nodes, np.int32)
        bg = np.ascontiguousarray(em.bnd_group, np.int32)
        x = np.ascontiguousarray(em.nodes_x, np.float64); y = np.ascontiguousarray(em.nodes_y, np.float64)
        _check(lib().fv_mesh_create(C.c_int64(x.size), _p(x), _p(y), C.c_int64(cells.shape[0]), _p(cells, _i32p),
                                    C.c_int64(bn.shape[0]), _p(bn, _i32p), _p(bg, _i32p),
                                    C.c_int32(len(em.group_names)), C.byref(h)))
        return cls(h.value, em.group_names)

    @classmethod
    def read_su2(cls, path):
        """SU2 native ASCII mesh (2D); boundary groups are the marker tags."""
        return cls._read(lib().fv_mesh_read_su2, path)

    @classmethod
    def read_msh(cls, path):
        return cls._read(lib().fv_mesh_read_msh, path)

    @classmethod
    def _read(cls, fn, path):
        h = C.c_void_p()
        _check(fn(os.fsencode(path), C.byref(h)))
        n = lib().fv_mesh_group_count(h)
        names = []
        for i in range(n):
            buf = C.create_string_buffer(256)
            _check(lib().fv_mesh_group_name(h, C.c_int32(i), buf, C.c_int32(256)))
            names.append(buf.value.decode())
        return cls(h.value, names)

    @classmethod
    def batch(cls, meshes):
        """Independent cases as one mesh (fv_mesh_create_batch).  Every case
        must list the same boundary group names in the same order."""
        names = meshes[0].group_names
        for m in meshes:
            if m.group_names != names:
                raise ValueError("batched cases must share their boundary group names")
        arr = (C.c_void_p * len(meshes))(*[m._h.value for m in meshes])
        h = C.c_void_p()
        _check(lib().fv_mesh_create_batch(C.c_int32(len(meshes)), arr, C.byref(h)))
        out = cls(h.value, names)
        out._cases = list(meshes)
        return out

    @property
    def n_cases(self):
        return int(lib().fv_mesh_case_count(self._h))

    def case_offsets(self):
        """(real_off, bound_off), each [n_cases + 1]: case k's real cells are
        reference cells real_off[k]:real_off[k+1], its ghosts n_real + bound_off[k]:bound_off[k+1]."""
        n = self.n_cases
        ro = np.zeros(n + 1, np.int64); bo = np.zeros(n + 1, np.int64)
        _check(lib().fv_mesh_case_offsets(self._h, _p(ro, _i64p), _p(bo, _i64p)))
        return ro, bo

    def split(self, a, V):
        """Per-case arrays ([n_total_k * V], reference order) from a batch array."""
        ro, bo = self.case_offsets()
        a = np.asarray(a).reshape(self.n_total, V)
        return [np.concatenate([a[ro[k]:ro[k + 1]], a[self.n_real + bo[k]:self.n_real + bo[k + 1]]]).ravel()
                for k in range(len(ro) - 1)]

    def join(self, parts, V):
        """Batch array from per-case arrays (the inverse of split)."""
        ro, bo = self.case_offsets()
        out = np.zeros((self.n_total, V))
        for k, p in enumerate(parts):
            p = np.asarray(p).reshape(-1, V)
            nr = ro[k + 1] - ro[k]
            out[ro[k]:ro[k + 1]] = p[:nr]
            out[self.n_real + bo[k]:self.n_real + bo[k + 1]] = p[nr:]
        return out.ravel()

    def __del__(self):
        try:
            if self._h and _lib is not None:
                _lib.fv_mesh_destroy(self._h)
        except Exception:
            pass

    def geometry(self):
        E, NT, NB = self.n_edges, self.n_total, self.n_bound
        out = dict(edge_cells=np.zeros(2 * E, np.uint32), edge_nodes=np.zeros(2 * E, np.uint32),
                   enx=np.zeros(E), eny=np.zeros(E), elen=np.zeros(E), ecx=np.zeros(E), ecy=np.zeros(E),
                   area=np.zeros(NT), ccx=np.zeros(NT), ccy=np.zeros(NT),
                   bound_edges=np.zeros(NB, np.uint32), bound_group=np.zeros(NB, np.int32))
        _check(lib().fv_mesh_geometry(self._h, _p(out["edge_cells"], _u32p), _p(out["edge_nodes"], _u32p),
                                      *[_p(out[k]) for k in ("enx", "eny", "elen", "ecx", "ecy", "area", "ccx", "ccy")],
                                      _p(out["bound_edges"], _u32p), _p(out["bound_group"], _i32p)))
        return out

    def device_order(self):
        a = np.zeros(self.n_total, np.int32)
        _check(lib().fv_mesh_device_order(self._h, _p(a, _i32p)))
        return a

    def partition(self, n_parts, part):
        """Host-only plan of one part of a decomposition (fv_mesh_partition):
        a dict of its sizes and index lists."""
        sz = np.zeros(11, np.int64)
        _check(lib().fv_mesh_partition_sizes(self._h, C.c_int32(n_parts), C.c_int32(part), _p(sz, _i64p)))
        n_real, n_total, n_edges, n_own, n_own_ghost, cell0, owner0, n_recv, n_send, n_bound, n_band = \
            (int(v) for v in sz)
        out = dict(n_real=n_real, n_total=n_total, n_edges=n_edges, n_own=n_own, n_own_ghost=n_own_ghost,
                   cell0=cell0, owner0=owner0, n_bound=n_bound, n_band=n_band,
                   local2ref=np.zeros(n_total, np.int32), local_edges=np.zeros(n_edges, np.int32),
                   recv_off=np.zeros(n_parts + 1, np.int64), recv_idx=np.zeros(n_recv, np.int32),
                   send_off=np.zeros(n_parts + 1, np.int64), send_idx=np.zeros(n_send, np.int32))
        _check(lib().fv_mesh_partition(self._h, C.c_int32(n_parts), C.c_int32(part),
                                       _p(out["local2ref"], _i32p), _p(out["local_edges"], _i32p),
                                       _p(out["recv_off"], _i64p), _p(out["recv_idx"], _i32p),
                                       _p(out["send_off"], _i64p), _p(out["send_idx"], _i32p)))
        return out


def physics_struct(ph: _phys.Physics, group_names: Sequence[str]):
    gbc = np.array([BC[ph.bcs[n][0]] for n in group_names], np.int32)
    gbv = np.array([list(ph.bcs[n][1]) if ph.bcs[n][1] is not None else [0.0] * 4 for n in group_names],
                   np.float64).reshape(-1)
    s = _Physics(V=ph.V, flux=FLUX[ph.flux], order2=int(ph.order2), limiter=LIMITER[ph.limiter],
                 dt_kind=DT[ph.dt_kind], global_dt=int(ph.global_dt), gamma=ph.gamma, K=ph.K, cfl=ph.cfl,
                 dt_const=ph.dt_const, n_groups=len(group_names))
    s.group_bc = _p(gbc, _i32p); s.group_bv = _p(gbv)
    s.positivity_guard = int(getattr(ph, "positivity_guard", False))
    s.diffusive = int(getattr(ph, "diffusive", False))
    s.mu, s.pr, s.cp, s.r = ph.mu, ph.pr, ph.cp, ph.r
    s.smooth_residuals = int(getattr(ph, "smooth", False))
    s._keep = (gbc, gbv)
    return s


class Solver:
    """Device solver for one mesh + physics (one CUDA device)."""

    STAGE_KERNELS = {"auto": 0, "split": 1, "fused": 2, "hybrid": 3}

    SCHEDULES = {"tile": 0, "worklist": 1, "tile2": 2}

    def __init__(self, mesh: Mesh, ph: _phys.Physics, precision: str = "fp64_exact", device: int = 0,
                 tile_cells: int = 0, stage_kernels: str = "auto", schedule: str = "tile"):
        """stage_kernels: "auto" ("hybrid" where the physics allow the fused
        stage kernel, else "split"), "split" (gradient and flux kernels),
        "fused", or "hybrid" (split first stage with the time step folded into
        its gradient kernel, fused others); schedule of
        the fused kernel: "tile" (one CTA per tile), "worklist" or "tile2"
        (one CTA of two threads per cell per tile)."""
        self.mesh = mesh
        self.phys = ph
        self.V = ph.V
        self.precision = precision
        self._ps = physics_struct(ph, mesh.group_names)
        h = C.c_void_p()
        opt = (C.c_int32 * 3)(int(tile_cells), self.STAGE_KERNELS[stage_kernels], self.SCHEDULES[schedule])
        _check(lib().fv_solver_create_ex(mesh._h, C.byref(self._ps), C.c_int32(PREC[precision]), C.c_int32(device),
                                         opt, C.byref(h)))
        self._h = h

    @classmethod
    def create_tuned(cls, mesh: Mesh, ph: _phys.Physics, precision: str, q, alpha=_phys.RK5_ALPHA,
                     steps: int = 5, device: int = 0):
        """The solver with the fastest tile size for this mesh and physics
        (fv_solver_create_tuned); its state is q, step 0."""
        self = cls.__new__(cls)
        self.mesh = mesh
        self.phys = ph
        self.V = ph.V
        self.precision = precision
        self._ps = physics_struct(ph, mesh.group_names)
        q = np.ascontiguousarray(q, np.float64)
        a = np.ascontiguousarray(alpha, np.float64)
        h = C.c_void_p(); t = C.c_int32(); ms = C.c_double()
        _check(lib().fv_solver_create_tuned(mesh._h, C.byref(self._ps), C.c_int32(PREC[precision]),
                                            C.c_int32(device), _p(q), _p(a), C.c_int32(a.size), C.c_int32(steps),
                                            C.byref(h), C.byref(t), C.byref(ms)))
        self._h = h
        self.tile_cells = t.value
        self.tuned_ms_per_step = ms.value
        return self

    OUTPUT_KINDS = {"pressure": 1, "mach": 2, "velocity": 3, "state01": 4}

    def output_fields(self, kinds, q=None):
        """Extra output fields (fv_output_fields) of the real cells in
        reference order: a list of arrays, [n_real] for pressure / mach,
        [n_real, 2] for velocity / state01.  q: a host state (reference
        numbering), or None for the solver's current state."""
        ks = (C.c_int32 * len(kinds))(*[self.OUTPUT_KINDS[k] for k in kinds])
        ncs = [2 if k in ("velocity", "state01") else 1 for k in kinds]
        n_real = self.mesh.n_real
        out = np.zeros(sum(ncs) * n_real)
        qp, n = None, 0
        if q is not None:
            q = np.ascontiguousarray(q, np.float64)
            qp, n = _p(q), q.size // self.V
        _check(lib().fv_output_fields(self._h, qp, C.c_int64(n), C.c_int32(len(kinds)), ks, _p(out)))
        res, o = [], 0
        for nc in ncs:
            a = out[o:o + nc * n_real]
            res.append(a.reshape(n_real, 2) if nc == 2 else a)
            o += nc * n_real
        return res

    @property
    def stage_kernels(self):
        """"fused", "split" or "hybrid" (split first stage, fused others): the
        stage kernels this solver runs."""
        return {3: "hybrid", 2: "fused", 1: "split"}[lib().fv_solver_stage_kernels(self._h)]

    @property
    def schedule(self):
        """"tile", "worklist" or "tile2": the fused stage kernel's schedule."""
        return {0: "tile", 1: "worklist", 2: "tile2"}[lib().fv_solver_schedule(self._h)]

    def close(self):
        if self._h:
            lib().fv_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nq(self):
        return self.mesh.n_total * self.V

    def set_stream(self, stream_ptr: int):
        _check(lib().fv_solver_set_stream(self._h, C.c_void_p(stream_ptr)))

    def sync(self):
        _check(lib().fv_solver_sync(self._h))

    def set_chunk(self, n):
        _check(lib().fv_solver_set_chunk(self._h, C.c_int32(n)))

    # -- state -----------------------------------------------------------
    def set_state(self, q):
        q = np.ascontiguousarray(q, np.float64).reshape(-1)
        assert q.size == self.nq
        _check(lib().fv_set_state(self._h, _p(q)))

    def get_state(self):
        q = np.zeros(self.nq)
        _check(lib().fv_get_state(self._h, _p(q)))
        return q

    def set_state_ptr(self, ptr: int, device: bool):
        fn = lib().fv_set_state_device if device else lib().fv_set_state
        _check(fn(self._h, C.c_void_p(ptr)))

    def get_state_ptr(self, ptr: int, device: bool):
        fn = lib().fv_get_state_device if device else lib().fv_get_state
        _check(fn(self._h, C.c_void_p(ptr)))

    # -- time loop -------------------------------------------------------
    def run(self, max_step, alpha=_phys.RK5_ALPHA, max_time=1e10, tolerance=1e-16, print_interval=1,
            restart=True, on_print: Optional[Callable] = None):
        a = np.ascontiguousarray(alpha, np.float64)
        cb = _PRINT_CB(0)
        if on_print is not None:
            def _cb(user, step, time, R, V):
                on_print(int(step), float(time), [R[k] for k in range(V)])
            cb = _PRINT_CB(_cb)
        o = _RunOptions(max_step=int(max_step), max_time=float(max_time), tolerance=float(tolerance),
                        print_interval=int(print_interval), n_alpha=a.size, alpha=_p(a), restart=int(restart),
                        on_print=cb, user=None)
        info = _RunInfo()
        _check(lib().fv_run(self._h, C.byref(o), C.byref(info)))
        return dict(step=info.step, time=info.time, R=np.array(info.R[: self.V]), R0=np.array(info.R0[: self.V]))

    def set_ghost_states(self, bv):
        """Per-ghost boundary states [n_bound, 4] (reference ghost order) for
        inflow / far-field ghosts; None restores the group states."""
        if bv is None:
            _check(lib().fv_solver_set_ghost_states(self._h, None))
            return
        b = np.ascontiguousarray(bv, np.float64).reshape(-1)
        _check(lib().fv_solver_set_ghost_states(self._h, _p(b)))

    def case_times(self):
        """Each case's accumulated time (one entry for a single mesh)."""
        t = np.zeros(self.mesh.n_cases)
        _check(lib().fv_batch_times(self._h, _p(t)))
        return t

    def continue_from(self, other: "Solver"):
        """Take over another solver's state and run control (same mesh), so
        run(..., restart=False) continues its run in this solver's precision."""
        _check(lib().fv_solver_continue_from(self._h, other._h))

    def last_run_stats(self):
        ms = C.c_double(); n = C.c_int64()
        _check(lib().fv_last_run_stats(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def check_state(self):
        rc = lib().fv_check_state(self._h)
        return rc

    def boundary_force(self, group_name):
        g = self.mesh.group_names.index(group_name)
        fx = C.c_double(); fy = C.c_double()
        _check(lib().fv_boundary_force(self._h, C.c_int32(g), C.byref(fx), C.byref(fy)))
        return fx.value, fy.value

    def residuals(self):
        R = np.zeros(self.V)
        _check(lib().fv_residuals(self._h, _p(R)))
        return R

    # -- stage entry points (reference numbering) -------------------------
    def stage_dt(self, q, global_min=False):
        q = np.ascontiguousarray(q, np.float64); dt = np.zeros(self.mesh.n_total)
        _check(lib().fv_stage_dt(self._h, _p(q), _p(dt), C.c_int32(int(global_min))))
        return dt

    def stage_gradients_limiters(self, q):
        q = np.ascontiguousarray(q, np.float64)
        gx = np.zeros(self.nq); gy = np.zeros(self.nq); lim = np.zeros(self.nq)
        _check(lib().fv_stage_gradients_limiters(self._h, _p(q), _p(gx), _p(gy), _p(lim)))
        return gx, gy, lim

    def stage_update(self, q_base, q_stage, gx, gy, lim, dt, alpha):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (q_base, q_stage, gx, gy, lim, dt)]
        out = np.zeros(self.nq)
        _check(lib().fv_stage_update(self._h, *[_p(a) for a in arrs], C.c_double(alpha), _p(out)))
        return out

    def stage_bounds(self, q, gx, gy, lim):
        q = np.ascontiguousarray(q, np.float64).copy()
        arrs = [np.ascontiguousarray(a, np.float64) for a in (gx, gy, lim)]
        _check(lib().fv_stage_bounds(self._h, _p(q), *[_p(a) for a in arrs]))
        return q


def nccl_id() -> bytes:
    """A fresh 128-byte NCCL id for Group (create on one process, pass to all)."""
    b = C.create_string_buffer(128)
    _check(lib().fv_group_nccl_id(b))
    return b.raw


class Group:
    """A domain decomposition of one mesh (fv_group_*): this process's parts
    on one CUDA device, NCCL between processes.  Create it on every process
    with the same mesh, n_parts and id; set_state takes the whole mesh's
    state, get_state returns it with this process's cells filled in."""

    def __init__(self, mesh: Mesh, ph: _phys.Physics, precision: str = "fp64_exact", n_parts: int = 2,
                 rank: int = 0, n_ranks: int = 1, nccl_id_bytes: Optional[bytes] = None, device: int = 0,
                 nccl_local: bool = False, tile_cells: int = 0, schedule: str = "tile",
                 serial_exchange: bool = False, timeout_ms: float = 0.0, transport: str = "copy",
                 wait_polls: int = 0):
        self.mesh = mesh
        self.V = ph.V
        self._ps = physics_struct(ph, mesh.group_names)
        self._id = C.create_string_buffer(nccl_id_bytes, 128) if nccl_id_bytes is not None else None
        o = _GroupOptions(n_parts=n_parts, rank=rank, n_ranks=n_ranks,
                          nccl_id=C.cast(self._id, C.c_void_p) if self._id is not None else None,
                          nccl_local=int(nccl_local), tile_cells=int(tile_cells), stage_kernels=0,
                          schedule=Solver.SCHEDULES[schedule], serial_exchange=int(serial_exchange),
                          transport={"copy": 0, "p2p": 1}[transport], wait_polls=int(wait_polls),
                          timeout_ms=float(timeout_ms))
        h = C.c_void_p()
        _check(lib().fv_group_create(mesh._h, C.byref(self._ps), C.c_int32(PREC[precision]), C.c_int32(device),
                                     C.byref(o), C.byref(h)))
        self._h = h

    def set_state(self, q):
        q = np.ascontiguousarray(q, np.float64).reshape(-1)
        assert q.size == self.mesh.n_total * self.V
        _check(lib().fv_group_set_state(self._h, _p(q)))

    def get_state(self, q=None):
        q = np.zeros(self.mesh.n_total * self.V) if q is None else np.ascontiguousarray(q, np.float64)
        _check(lib().fv_group_get_state(self._h, _p(q)))
        return q

    def run(self, max_step, alpha=_phys.RK5_ALPHA, max_time=1e10, tolerance=1e-16, print_interval=1,
            restart=True, on_print: Optional[Callable] = None):
        a = np.ascontiguousarray(alpha, np.float64)
        cb = _PRINT_CB(0)
        if on_print is not None:
            def _cb(user, step, time, R, V):
                on_print(int(step), float(time), [R[k] for k in range(V)])
            cb = _PRINT_CB(_cb)
        o = _RunOptions(max_step=int(max_step), max_time=float(max_time), tolerance=float(tolerance),
                        print_interval=int(print_interval), n_alpha=a.size, alpha=_p(a), restart=int(restart),
                        on_print=cb, user=None)
        info = _RunInfo()
        _check(lib().fv_group_run(self._h, C.byref(o), C.byref(info)))
        return dict(step=info.step, time=info.time, R=np.array(info.R[: self.V]), R0=np.array(info.R0[: self.V]))

    def info(self):
        out = np.zeros(8, np.int64)
        _check(lib().fv_group_info(self._h, _p(out, _i64p)))
        return dict(local_parts=int(out[0]), owned_cells=int(out[1]), halo_cells=int(out[2]),
                    sent_cells=int(out[3]), tiles=int(out[4]), nccl=bool(out[5]), band_tiles=int(out[6]),
                    transport={0: "copy", 1: "p2p"}[int(out[7])])

    def last_run_stats(self):
        ms = C.c_double(); n = C.c_int64()
        _check(lib().fv_group_last_run_stats(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def close(self):
        if self._h:
            lib().fv_group_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _GroupOptions(C.Structure):
    _fields_ = [("n_parts", C.c_int32), ("rank", C.c_int32), ("n_ranks", C.c_int32), ("nccl_id", C.c_void_p),
                ("nccl_local", C.c_int32), ("tile_cells", C.c_int32), ("stage_kernels", C.c_int32),
                ("schedule", C.c_int32), ("serial_exchange", C.c_int32), ("transport", C.c_int32),
                ("wait_polls", C.c_int64), ("timeout_ms", C.c_double)]


def solver_info(s: Solver):
    out = np.zeros(6, np.int64)
    _check(lib().fv_solver_info(s._h, _p(out, _i64p)))
    return dict(tiles=int(out[0]), tile_cells=int(out[1]), max_halo=int(out[2]), max_edges=int(out[3]),
                precision=int(out[4]), stage_bytes=int(out[5]))


class _AdjOptions(C.Structure):
    _fields_ = [("n_steps", C.c_int32), ("checkpoint_every", C.c_int32), ("n_alpha", C.c_int32),
                ("alpha", _dp), ("loss_group", C.c_int32), ("param_group", C.c_int32), ("n_bins", C.c_int32),
                ("bin_lo", C.c_double), ("bin_hi", C.c_double)]


class Adjoint:
    """Discrete adjoint of the FP64_EXACT time loop for the inflow-parameter
    problem (fv_adjoint_*): theta = (M, delta_1..delta_nb) sets the free
    stream and the inflow density bins; loss = time integral of the pressure
    force magnitude sum_f p le over `loss_group`'s faces."""

    def __init__(self, mesh: Mesh, ph: _phys.Physics, n_steps: int, checkpoint_every: int = 50,
                 alpha=_phys.RK5_ALPHA, loss_group: str = "step", param_group: str = "inlet", n_bins: int = 64,
                 bin_lo: float = 0.0, bin_hi: float = 1.0, device: int = 0):
        self.mesh = mesh
        self.n_bins = n_bins
        self._ps = physics_struct(ph, mesh.group_names)
        self._alpha = np.ascontiguousarray(alpha, np.float64)
        self._o = _AdjOptions(n_steps=n_steps, checkpoint_every=checkpoint_every, n_alpha=self._alpha.size,
                              alpha=_p(self._alpha), loss_group=mesh.group_names.index(loss_group),
                              param_group=mesh.group_names.index(param_group), n_bins=n_bins,
                              bin_lo=bin_lo, bin_hi=bin_hi)
        h = C.c_void_p()
        _check(lib().fv_adjoint_create(mesh._h, C.byref(self._ps), C.c_int32(device), C.byref(self._o),
                                       C.byref(h)))
        self._h = h

    def loss(self, theta):
        t = np.ascontiguousarray(theta, np.float64)
        out = C.c_double()
        _check(lib().fv_adjoint_run(self._h, _p(t), C.byref(out), None))
        return out.value

    def gradient(self, theta):
        """(loss, dloss/dtheta)"""
        t = np.ascontiguousarray(theta, np.float64)
        out = C.c_double()
        g = np.zeros(1 + self.n_bins)
        _check(lib().fv_adjoint_run(self._h, _p(t), C.byref(out), _p(g)))
        return out.value, g

    def final_state(self):
        q = np.zeros(self.mesh.n_total * 4)
        _check(lib().fv_adjoint_final_state(self._h, _p(q)))
        return q

    def close(self):
        if self._h:
            lib().fv_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
