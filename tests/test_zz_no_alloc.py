"""fv_stage_dt_noalloc: the CFL time step computed without allocating any
device memory, for callers that cannot call cudaMalloc (an application that
reserves all GPU memory for its own pool up front, or one that must not
trigger the device synchronisation an allocation implies between its queued
kernels).  It must give exactly what the allocating entry point fv_stage_dt
gives, call after call: every call reuses one fixed scratch array."""
import ctypes

import numpy as np
import pytest

import fvgpu
import meshgen
import physics as P
from cases import CASES, random_euler_state

pytestmark = pytest.mark.gpu


def noalloc_dt(solver, q_dev, out_dev, global_min):
    return fvgpu.lib().fv_stage_dt_noalloc(solver._h, ctypes.c_void_p(q_dev.data_ptr()),
                                          ctypes.c_void_p(out_dev.data_ptr()),
                                          ctypes.c_int32(int(global_min)), ctypes.c_void_p(None))


@pytest.mark.parametrize("precision", ["fp64_exact", "fp64", "fp32"])
@pytest.mark.parametrize("name", ["step_o2_venk5", "naca"])
def test_noalloc_dt_matches_allocating_entry(name, precision):
    import torch

    case = CASES[name]
    em = case["mesh"]()
    mesh = fvgpu.Mesh.from_elements(em)
    s = fvgpu.Solver(mesh, case["phys"](), precision)
    for call in range(2):  # two calls in a row through the same scratch array
        q = random_euler_state(mesh.n_total, seed=100 + call)
        for glob in (False, True):
            want = s.stage_dt(q, glob)
            q_dev = torch.from_numpy(q).cuda()
            out = torch.full((mesh.n_total,), -1.0, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()  # inputs are on torch's stream; the call uses the solver's
            assert noalloc_dt(s, q_dev, out, glob) == 0, fvgpu.lib().fv_last_error()
            s.sync()
            got = out.cpu().numpy()
            assert got.tobytes() == want.tobytes(), (call, glob, np.abs(got - want).max())
    s.close()


def test_noalloc_dt_rejects_meshes_beyond_its_scratch():
    import torch

    em = meshgen.rect_tri(400, 300, 1.0, 0.75)   # 240,000 cells: more than the fixed scratch holds
    mesh = fvgpu.Mesh.from_elements(em)
    s = fvgpu.Solver(mesh, P.riemann_strip(), "fp64")
    q = torch.zeros(mesh.n_total * 4, dtype=torch.float64, device="cuda")
    out = torch.zeros(mesh.n_total, dtype=torch.float64, device="cuda")
    assert noalloc_dt(s, q, out, True) == -1
    assert b"scratch" in fvgpu.lib().fv_last_error()
    s.close()
