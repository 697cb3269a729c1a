"""Drop-in test of the fvhyper C++ API: fvhyper's own example programs
(examples/<name>/main.cpp), compiled unchanged against include/fvhyper/*.h and
libfvhyper_gpu.a, run on the GPU and must reproduce the reference CPU
program built from the same source on fvhyper's own library
(oracle/_ref/libref_<name>.so, entry point ref_example_main):

- the same log: header, then per printed step the same step and time columns
  and the same residual columns (the seconds column is wall time);
- the same output file: the final VTU, byte for byte, in the reference's
  ASCII layout (FVGPU_VTK_FORMAT=ascii);
- the default binary VTU carries the same cell values.

All seven examples run.  Programs whose physics no device kind implements and
meshes whose boundary names the program does not define must be refused the
way the reference refuses them: an uncaught std::invalid_argument.
"""
import os
import re
import shutil
import struct
import subprocess
import sys

import numpy as np
import pytest

import meshgen
from conftest import PKG, ROOT

EXAMPLES = os.path.join(PKG, "shim", "_examples")
REF = os.path.join(ROOT, "oracle", "_ref")


def _program(name):
    p = os.path.join(EXAMPLES, name)
    if not os.path.exists(p):
        pytest.skip("example programs are built from the fvhyper sources (shim/examples.mk)")
    return p


def _one_group(em, name):
    em.bnd_group[:] = 0
    em.group_names = [name]
    return em


def _renamed(em, names):
    em.group_names = list(names)
    return em


def _step_mesh():
    em = meshgen.forward_step(n=10)
    names = list(em.group_names)            # wall, inlet, outlet, step
    em.bnd_group[em.bnd_group == names.index("step")] = names.index("wall")
    em.group_names = names[:3]
    return em


# example -> (mesh file, mesh builder, VTU written at the end or None)
CASES = {
    "shockTube": ("square.msh", lambda: _one_group(meshgen.rect_tri(40, 4, 1.0, 0.1), "wall"), "square.vtu"),
    "burgers": ("square.msh", lambda: _one_group(meshgen.rect_tri(12, 12, 1.0, 1.0), "wall"), "square.vtu"),
    "naca": ("naca.msh", lambda: meshgen.naca_ogrid(ni=40, nj=10, r_far=10.0, jitter=0.0), "naca.vtu"),
    "forwardStep": ("step.msh", _step_mesh, None),
    "heatTransfer": ("square.msh", lambda: _one_group(meshgen.rect_tri(12, 12, 1.0, 1.0), "wall"), "square.vtu"),
    "flatPlate": ("square.msh", lambda: meshgen.flat_plate(nx0=6, nx1=18, ny=12), "square.vtu"),
    # saves a time series (times/naca0012_<k>.vtu, 334 snapshots) and no final file
    "nacaTransient": ("naca0012.msh", lambda: _renamed(meshgen.naca_ogrid(ni=24, nj=12, r_far=10.0, jitter=0.0),
                                                       ["wall", "farfield"]), None),
}


def _setup(tmp, name):
    fname, build, _ = CASES[name]
    os.makedirs(os.path.join(tmp, "times"), exist_ok=True)  # time-series snapshots go there
    meshgen.write_msh41(os.path.join(tmp, fname), build())


def _outputs(d):
    return sorted(os.path.relpath(os.path.join(r, f), d) for r, _, fs in os.walk(d) for f in fs
                  if f.endswith((".vtu", ".pvtu")))


def _run_gpu(name, cwd, vtk_format="ascii"):
    env = dict(os.environ, FVGPU_VTK_FORMAT=vtk_format, FVGPU_PRECISION="fp64_exact")
    r = subprocess.run([_program(name)], cwd=cwd, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout


def _run_reference(name, cwd):
    lib = os.path.join(REF, f"libref_{name}.so")
    if not os.path.exists(lib):
        pytest.skip("reference build (oracle/_ref) not present")
    code = ("import ctypes, sys; lib = ctypes.CDLL(sys.argv[1]); "
            "sys.exit(lib.ref_example_main())")
    r = subprocess.run([sys.executable, "-c", code, lib], cwd=cwd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout


def _log(out):
    lines = [l for l in out.splitlines() if l.strip()]
    head = lines[0]
    rows = []
    for l in lines[1:]:
        f = [x.strip() for x in l.split(",")]
        rows.append((f[0], f[1], f[3:]))  # step, time, residuals (f[2] = seconds)
    return head, rows


def _num(s):
    return float(s.replace("-nan", "nan"))


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_example_program_matches_reference(name, tmp_path):
    ref_dir, gpu_dir = str(tmp_path / "ref"), str(tmp_path / "gpu")
    _setup(ref_dir, name)
    _setup(gpu_dir, name)
    want = _run_reference(name, ref_dir)
    got = _run_gpu(name, gpu_dir)
    wh, wrows = _log(want)
    gh, grows = _log(got)
    assert gh == wh
    assert len(grows) == len(wrows), (len(grows), len(wrows))
    for (gs, gt, gr), (ws, wt, wr) in zip(grows, wrows):
        assert (gs, gt) == (ws, wt)
        # residual norms are sums over all cells, reduced in a different
        # order on the device: equal to print precision up to the last digit
        assert np.allclose([_num(x) for x in gr], [_num(x) for x in wr], rtol=2e-5, atol=0, equal_nan=True), \
            (gs, gr, wr)
    # every file written (final state, time series), byte for byte
    files = _outputs(ref_dir)
    assert _outputs(gpu_dir) == files and (CASES[name][2] is None or CASES[name][2] in files)
    for f in files:
        a = open(os.path.join(gpu_dir, f), "rb").read()
        b = open(os.path.join(ref_dir, f), "rb").read()
        assert a == b, f


def _read_binary_vtu(path):
    """Cell arrays of a raw-appended VTU written by writeVtk's binary mode."""
    raw = open(path, "rb").read()
    head, _, rest = raw.partition(b'<AppendedData encoding="raw">')
    data = rest[rest.index(b"_") + 1:]
    out = {}
    for m in re.finditer(rb'<DataArray type="(\w+)" (?:Name="([^"]+)" )?(?:NumberOfComponents="3" )?'
                         rb'format="appended" offset="(\d+)"', head):
        typ, nm, off = m.group(1).decode(), (m.group(2) or b"Points").decode(), int(m.group(3))
        nb = struct.unpack_from("<Q", data, off)[0]
        dt = {"Float64": "<f8", "Float32": "<f4", "Int32": "<i4", "UInt8": "u1"}[typ]
        out[nm] = np.frombuffer(data, dt, nb // np.dtype(dt).itemsize, off + 8)
    return out


def _read_ascii_cell_array(path, name):
    txt = open(path).read()
    i = txt.index(f'Name="{name}"')
    body = txt[txt.index(">", i) + 1: txt.index("</DataArray>", i)]
    return np.array([float(x) for x in body.split()])


@pytest.mark.gpu
def test_binary_vtu_holds_the_state(tmp_path):
    d_a, d_b = str(tmp_path / "a"), str(tmp_path / "b")
    _setup(d_a, "shockTube")
    _setup(d_b, "shockTube")
    _run_gpu("shockTube", d_a, "ascii")
    _run_gpu("shockTube", d_b, "binary")
    b = _read_binary_vtu(os.path.join(d_b, "square.vtu"))
    for nm in ("rho", "rhou", "rhoe", "p"):
        a = _read_ascii_cell_array(os.path.join(d_a, "square.vtu"), nm)
        assert b[nm].shape == a.shape
        assert np.abs(b[nm] - a).max() <= 5e-7 * max(1.0, np.abs(a).max())  # ascii keeps 6 decimals
    assert b["types"].tolist() == [5] * b["types"].size
    assert b["offsets"][-1] == b["connectivity"].size


# User programs in the fvhyper API (our own code): VARS variables with
# diffusive fluxes; FLUX is the body of calc_flux, BC of the boundary
# function, SMOOTH the residual-smoothing flag.
_PROGRAM = r"""
#include <fvhyper/mesh.h>
#include <fvhyper/explicit.h>
#include <fvhyper/parallel.h>
#include <fvhyper/post.h>
#include <algorithm>
#include <cmath>
namespace fvhyper {
const int vars = VARS;
const std::vector<std::string> var_names = NAMES;
namespace solver {
const bool do_calc_gradients = true;
const bool do_calc_limiters = ORDER2;
const bool linear_interpolate = ORDER2;
const bool diffusive_gradients = true;
const bool global_dt = false;
const bool smooth_residuals = SMOOTH;
}
void generate_initial_solution(std::vector<double>& q, const mesh& m) {
    for (double& x : q) x = 0.0;
}
double limiter_func(const double& y) { return std::max(0., std::min(1., y)); }
void calc_flux(double* f, const double* qi, const double* qj, const double* gx, const double* gy,
               const double* n) {
    FLUX
}
void calc_dt(std::vector<double>& dt, const std::vector<double>& q, mesh& m) {
    for (double& d : dt) d = 1e-3;
}
namespace boundaries {
void side(double* b, double* q, double* n) { BC }
std::map<std::string, void (*)(double*, double*, double*)> bounds = {{"wall", side}};
}
namespace post {
std::map<std::string, void (*)(double*, double*)> extra_scalars = {};
std::map<std::string, void (*)(double*, double*)> extra_vectors = {};
}
}
int main() {
    fvhyper::mpi_wrapper pool;
    fvhyper::mesh m;
    m.read_file("square", pool);
    fvhyper::solverOptions options;
    options.max_step = STEPS;
    options.print_interval = 10;
    std::vector<double> q;
    fvhyper::run("square", q, pool, m, options);
    fvhyper::writeVtk("square", q, m, pool.rank, pool.size);
    return pool.exit();
}
"""
# upwind advection plus -(grad q . n): the Burgers-diffusion kind
_BURGERS_DIFF = ("double a = qi[0] * n[0] + qi[1] * n[1], c = qj[0] * n[0] + qj[1] * n[1];"
                 "double s = std::max(std::abs(a), std::abs(c));"
                 "for (int k = 0; k < 2; ++k) {"
                 "  f[k] = 0.5 * (a * qi[k] + c * qj[k]) - 0.5 * s * (qj[k] - qi[k]);"
                 "  f[k] += -(gx[k] * n[0] + gy[k] * n[1]); }")


def _build_program(tmp_path, **kw):
    shim = os.path.join(PKG, "libfvhyper_gpu.a")
    if not os.path.exists(shim) or shutil.which("g++") is None:
        pytest.skip("needs the built shim and g++")
    src = _PROGRAM
    for k, v in dict(dict(VARS="2", NAMES='{"u", "v"}', ORDER2="true", SMOOTH="true", STEPS="30",
                          FLUX=_BURGERS_DIFF, BC="b[0] = -n[1]; b[1] = n[0];"), **kw).items():
        src = src.replace(k, v)
    (tmp_path / "main.cpp").write_text(src)
    exe = str(tmp_path / "prog")
    subprocess.run(["g++", "-O1", "-std=c++17", "-ffp-contract=off", "-I" + os.path.join(ROOT, "include"),
                    str(tmp_path / "main.cpp"), shim, "-L" + PKG, "-lfvgpu", "-Wl,-rpath," + PKG, "-o", exe],
                   check=True, timeout=300)
    meshgen.write_msh41(str(tmp_path / "square.msh"), _one_group(meshgen.rect_tri(8, 8, 1.0, 1.0), "wall"))
    return exe


@pytest.mark.parametrize("kw,message", [
    (dict(FLUX="for (int k = 0; k < 2; ++k) f[k] = 0.5 * (qi[k] + qj[k]) * n[0] - 0.01 * gx[k];"),
     "no device kind matches"),
    (dict(VARS="1", NAMES='{"T"}', ORDER2="false", FLUX="f[0] = -(gx[0] * n[0] + gy[0] * n[1]);",
          BC="b[0] = q[0];"), "smooth_residuals runs on the device with the Burgers-diffusion kind only"),
])
def test_unsupported_physics_is_refused(kw, message, tmp_path):
    """Refused in run() before any device work, as an uncaught
    std::invalid_argument naming what has no device kind."""
    exe = _build_program(tmp_path, **kw)
    r = subprocess.run([exe], cwd=str(tmp_path), capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "std::invalid_argument" in r.stderr and message in r.stderr, r.stderr


@pytest.mark.gpu
def test_smoothed_burgers_diffusion_program_runs(tmp_path, oracle):
    """A program with the physics of the reference's regression test
    (Burgers + diffusion, MUSCL with minmod, residual smoothing, tangential
    boundary state) runs through the shim as the Burgers-diffusion kind with
    smoothing; its VTU holds the oracle's state after 30 steps (6 decimals)."""
    import physics as P
    exe = _build_program(tmp_path)
    env = dict(os.environ, FVGPU_VTK_FORMAT="ascii", FVGPU_PRECISION="fp64_exact")
    r = subprocess.run([exe], cwd=str(tmp_path), env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    em = _one_group(meshgen.rect_tri(8, 8, 1.0, 1.0), "wall")
    g = oracle.build_mesh(em)
    p = oracle.physics(P.burgers_diffusion(), em.group_names)
    want = oracle.run_loop(g, p, np.zeros(g.n_total * 2), P.RK5_ALPHA, 30)["q"].reshape(-1, 2)[: g.n_real]
    got = np.stack([_read_ascii_cell_array(str(tmp_path / "square.vtu"), nm) for nm in ("u", "v")], 1)
    assert got.shape == want.shape and np.abs(want).max() > 1e-3
    assert np.abs(got - want).max() <= 5e-7 * max(1.0, np.abs(want).max())


def test_unknown_boundary_name_is_refused(tmp_path):
    em = _one_group(meshgen.rect_tri(6, 2, 1.0, 0.1), "inlet")  # shockTube defines only "wall"
    meshgen.write_msh41(str(tmp_path / "square.msh"), em)
    r = subprocess.run([_program("shockTube")], cwd=str(tmp_path), capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "Physical name inlet" in r.stderr and "not in mesh" in r.stderr, r.stderr


@pytest.mark.gpu
def test_naca_example_runs_from_the_reference_su2_mesh(tmp_path):
    """examples/naca/main.cpp, unchanged, on the SU2 mesh fvhyper ships for it
    (naca0012_129.su2 as naca.su2; the reference itself needs gmsh to convert
    it first): the run completes with falling residuals and writes naca.vtu."""
    src = os.path.join(EXAMPLES, "naca0012_129.su2")  # copied there by shim/examples.mk
    if not os.path.exists(src):
        pytest.skip("example programs and meshes are built from the fvhyper sources (shim/examples.mk)")
    shutil.copy(src, tmp_path / "naca.su2")
    out = _run_gpu("naca", str(tmp_path), vtk_format="binary")
    head, rows = _log(out)
    assert head.startswith("Step, Time, RealTime")
    first, last = rows[1], rows[-1]
    assert int(last[0]) <= 10000
    assert max(_num(x) for x in last[2]) < 0.1 * max(_num(x) for x in first[2]), (first, last)
    q = _read_binary_vtu(str(tmp_path / "naca.vtu"))
    assert q["rho"].size == 16384 and np.all(np.isfinite(q["rho"])) and np.all(q["rho"] > 0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["shockTube", "burgers", "naca", "nacaTransient"])
def test_extra_fields_evaluated_on_the_device_equal_the_host_callbacks(name, tmp_path):
    """The examples' post::extra_scalars / extra_vectors (pressure, Mach,
    velocity; Burgers' state vector) are identified with device output kinds
    and evaluated on the device by writeVtk: the binary VTU files (Float64
    values) are byte-identical to those written with every callback run on
    the host (FVGPU_POST=host)."""
    d_dev, d_host = str(tmp_path / "dev"), str(tmp_path / "host")
    _setup(d_dev, name)
    _setup(d_host, name)
    _run_gpu(name, d_dev, "binary")
    env = dict(os.environ, FVGPU_VTK_FORMAT="binary", FVGPU_PRECISION="fp64_exact", FVGPU_POST="host")
    r = subprocess.run([_program(name)], cwd=d_host, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    files = _outputs(d_host)
    assert files and _outputs(d_dev) == files
    for f in files:
        a = open(os.path.join(d_dev, f), "rb").read()
        b = open(os.path.join(d_host, f), "rb").read()
        assert a == b, f
