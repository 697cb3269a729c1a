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


def noalloc_dt(solver, q_dev, out_dev, global_min, stream=None):
    return fvgpu.lib().fv_stage_dt_noalloc(solver._h, ctypes.c_void_p(q_dev.data_ptr()),
                                          ctypes.c_void_p(out_dev.data_ptr()),
                                          ctypes.c_int32(int(global_min)), ctypes.c_void_p(stream))


# the Euler time steps (edge-sum CFL, signed-normal CFL) and the viscous one
# of the flat plate (a separate kernel instantiation)
@pytest.mark.parametrize("precision", ["fp64_exact", "fp64", "fp32"])
@pytest.mark.parametrize("name", ["step_o2_venk5", "naca", "flat_plate"])
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


def test_noalloc_dt_on_a_caller_stream():
    """The work is queued on the caller's stream and complete when it is."""
    import torch

    case = CASES["step_o2_venk5"]
    mesh = fvgpu.Mesh.from_elements(case["mesh"]())
    s = fvgpu.Solver(mesh, case["phys"](), "fp64")
    st = torch.cuda.Stream()
    for call in range(2):
        q = random_euler_state(mesh.n_total, seed=200 + call)
        want = s.stage_dt(q, True)
        with torch.cuda.stream(st):
            q_dev = torch.from_numpy(q).cuda(non_blocking=False)
            out = torch.full((mesh.n_total,), -1.0, dtype=torch.float64, device="cuda")
            assert noalloc_dt(s, q_dev, out, True, st.cuda_stream) == 0, fvgpu.lib().fv_last_error()
        st.synchronize()
        assert out.cpu().numpy().tobytes() == want.tobytes(), call
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
