"""CPU tests of the native library: it loads, exports every C-ABI symbol the
headers declare, and its host-side mesh build (no GPU involved) reproduces
the reference geometry bit for bit."""
import ctypes
import os
import re

import numpy as np
import pytest

import fvgpu
import meshgen
from cases import CASES, random_euler_state

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(fv_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    L = fvgpu.lib()
    syms = declared_symbols()
    assert "fv_run" in syms and "fv_stage_update" in syms and len(syms) > 20
    for s in sorted(syms):
        assert hasattr(L, s), s


def bits_equal(a, b):
    a = np.ascontiguousarray(a); b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


@pytest.mark.parametrize("name", sorted(CASES))
def test_native_geometry_matches_oracle(name, oracle):
    em = CASES[name]["mesh"]()
    m = fvgpu.Mesh.from_elements(em)
    g = m.geometry()
    o = oracle.build_mesh(em)
    assert (m.n_real, m.n_total, m.n_edges, m.n_bound) == (o.n_real, o.n_total, o.n_edges, o.n_bound)
    for k in ("edge_cells", "edge_nodes", "enx", "eny", "elen", "ecx", "ecy", "area", "ccx", "ccy",
              "bound_edges", "bound_group"):
        assert bits_equal(g[k], getattr(o, k)), k
    order = m.device_order()
    assert sorted(order.tolist()) == list(range(m.n_total))
    assert np.all(order[: m.n_real] < m.n_real) and np.all(order[m.n_real:] >= m.n_real)


def test_msh_reader_matches_element_path(tmp_path):
    for em in (meshgen.forward_step(n=20), meshgen.naca_ogrid(ni=48, nj=12, r_far=10.0)):
        path = str(tmp_path / "m.msh")
        meshgen.write_msh41(path, em)
        a = fvgpu.Mesh.read_msh(path)
        b = fvgpu.Mesh.from_elements(em)
        assert a.group_names == em.group_names
        ga, gb = a.geometry(), b.geometry()
        for k in ga:
            assert bits_equal(ga[k], gb[k]), k


def test_mesh_errors(tmp_path):
    em = meshgen.sod_strip(8, 2)
    bad = meshgen.ElementMesh(em.nodes_x, em.nodes_y, em.cells, em.bnd_nodes.copy(), em.bnd_group, em.group_names)
    bad.bnd_nodes[0] = (0, em.nodes_x.size - 1)          # not an edge
    with pytest.raises(fvgpu.FvError) as e:
        fvgpu.Mesh.from_elements(bad)
    assert e.value.code == -3
    open_face = meshgen.ElementMesh(em.nodes_x, em.nodes_y, em.cells, em.bnd_nodes[1:], em.bnd_group[1:],
                                    em.group_names)   # one boundary segment missing
    with pytest.raises(fvgpu.FvError) as e:
        fvgpu.Mesh.from_elements(open_face)
    assert e.value.code == -3
    flat = meshgen.ElementMesh(em.nodes_x * 0.0, em.nodes_y, em.cells, em.bnd_nodes, em.bnd_group, em.group_names)
    with pytest.raises(fvgpu.FvError) as e:             # zero-area cells
        fvgpu.Mesh.from_elements(flat)
    assert e.value.code == -3
    with pytest.raises(fvgpu.FvError) as e:
        fvgpu.Mesh.read_msh(str(tmp_path / "missing.msh"))
    assert e.value.code == -7
    p = tmp_path / "trunc.msh"
    p.write_text("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n$Nodes\n1 2 1 2\n2 1 0 2\n1\n")
    with pytest.raises(fvgpu.FvError):
        fvgpu.Mesh.read_msh(str(p))


def test_face_lists_follow_reference_edge_order():
    """Per-cell faces are visited in increasing reference edge order (the
    accumulation order of the reference's edge loops)."""
    em = meshgen.forward_step(n=20)
    m = fvgpu.Mesh.from_elements(em)
    g = m.geometry()
    ec = g["edge_cells"].reshape(-1, 2)
    order = m.device_order()
    ref2new = np.empty_like(order); ref2new[order] = np.arange(order.size)
    # every real cell appears 3 times over both edge columns (triangles)
    cnt = np.bincount(ec[ec < m.n_real], minlength=m.n_real)
    assert np.all(cnt == 3)


def _build_adjoint_api(tmp_path):
    import subprocess
    pkg = os.path.join(ROOT, "finite-volume-2d-cpp_b200")
    exe = str(tmp_path / "adjoint_api")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "adjoint_api.cpp"), "-L" + pkg, "-lfvgpu",
                    "-Wl,-rpath," + pkg, "-o", exe], check=True)
    return exe


def test_cpp_adjoint_api_compiles_and_reports_errors(tmp_path):
    """The C++ reverse-mode header builds against the library; without a
    usable device its constructor throws with the library's message."""
    import subprocess
    exe = _build_adjoint_api(tmp_path)
    r = subprocess.run([exe, str(tmp_path / "missing.msh"), "5", "3.0"], capture_output=True, text=True)
    assert r.returncode == 3 and r.stdout.startswith("error:") and "missing.msh" in r.stdout


@pytest.mark.gpu
def test_cpp_adjoint_api_matches_python_binding(tmp_path):
    import subprocess
    import physics as P
    exe = _build_adjoint_api(tmp_path)
    em = meshgen.forward_step(n=20)
    path = str(tmp_path / "step.msh")
    meshgen.write_msh41(path, em)
    theta = [3.0, 0.004, -0.01, 0.002]
    r = subprocess.run([exe, path, "40"] + [repr(t) for t in theta], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    vals = [float(x) for x in r.stdout.split()]
    mesh = fvgpu.Mesh.read_msh(path)
    ph = P.forward_step(order2=True, limiter="venkat", K=5.0, cfl=0.8)
    ph.positivity_guard = True
    adj = fvgpu.Adjoint(mesh, ph, n_steps=40, checkpoint_every=10, n_bins=3)
    loss, g = adj.gradient(np.array(theta))
    assert vals[0] == loss and vals[1:] == g.tolist()
    adj.close()


def test_su2_reader_matches_element_path(tmp_path):
    """An SU2 file of a mesh gives the geometry of the same element mesh
    (which the MSH reader and fv_mesh_create build as the reference does)."""
    for em in (meshgen.forward_step(n=20), meshgen.naca_ogrid(ni=48, nj=12, r_far=10.0),
               meshgen.rect_tri(6, 3, 1.0, 0.5)):
        path = str(tmp_path / "m.su2")
        meshgen.write_su2(path, em)
        a = fvgpu.Mesh.read_su2(path)
        b = fvgpu.Mesh.from_elements(em)
        assert a.group_names == list(em.group_names)
        ga, gb = a.geometry(), b.geometry()
        for k in ga:
            assert bits_equal(ga[k], gb[k]), k


def test_su2_reader_reads_the_reference_naca_meshes():
    """The SU2 meshes fvhyper ships for its NACA example (to be converted with
    gmsh there) are read directly: quadrilateral O-grids, closed, with the
    airfoil and farfield markers."""
    from __graft_entry__ import REFERENCE
    base = os.path.join(REFERENCE, "examples", "naca")
    if not os.path.isdir(base):
        pytest.skip("fvhyper checkout not present")
    for fn, ncell in (("naca0012_129.su2", 16384), ("NACA_M.su2", 4096)):
        m = fvgpu.Mesh.read_su2(os.path.join(base, fn))
        assert m.n_real == ncell and sorted(m.group_names) == ["airfoil", "farfield"]
        g = m.geometry()
        assert np.all(g["area"] > 0)
        # every real cell's outward fluxes of a constant field cancel (closed cells)
        s = np.zeros((m.n_total, 2))
        ec = g["edge_cells"].reshape(-1, 2).astype(np.int64)
        for d, n in ((0, g["enx"]), (1, g["eny"])):
            np.add.at(s[:, d], ec[:, 0], n * g["elen"])
            np.add.at(s[:, d], ec[:, 1], -n * g["elen"])
        assert np.abs(s[: m.n_real]).max() < 1e-12 * max(1.0, g["elen"].max())


def test_su2_reader_errors(tmp_path):
    bad = tmp_path / "bad.su2"
    bad.write_text("NDIME= 3\nNELEM= 0\nNPOIN= 0\n")
    with pytest.raises(fvgpu.FvError, match="two-dimensional"):
        fvgpu.Mesh.read_su2(str(bad))
    with pytest.raises(fvgpu.FvError):
        fvgpu.Mesh.read_su2(str(tmp_path / "missing.su2"))


def test_host_diffusion_kind_matches_its_restatement():
    """fv_kind_face_gradient / fv_kind_flux_grad (the host copies of the
    device's diffusion kind, which the fvhyper shim matches calc_flux to)
    against numpy written in the order of gradient_for_diffusion
    (explicit.cpp:70-109) and examples/heatTransfer/main.cpp:63-73: IEEE
    float64 operations in the same order give the same bits."""
    import physics as P
    L = fvgpu.lib()
    dp = ctypes.POINTER(ctypes.c_double)
    rng = np.random.default_rng(5)
    heat = fvgpu.physics_struct(P.heat(), ["wall"])

    def p(a):
        return a.ctypes.data_as(dp)

    for V in (1, 2, 4):
        for _ in range(50):
            gxi, gyi, gxj, gyj, qi, qj = (rng.uniform(-3, 3, V) for _ in range(6))
            ci, cj = rng.uniform(-1, 1, 2), rng.uniform(-1, 1, 2)
            gxf, gyf = np.zeros(V), np.zeros(V)
            assert L.fv_kind_face_gradient(V, p(gxi), p(gyi), p(gxj), p(gyj), p(qi), p(qj), p(ci), p(cj),
                                           p(gxf), p(gyf)) == 0
            t = ci - cj
            lij = np.sqrt(t[0] * t[0] + t[1] * t[1])
            t = t / lij
            d = (qi - qj) / lij
            bx, by = (gxi + gxj) * 0.5, (gyi + gyj) * 0.5
            dot = bx * t[0] + by * t[1]
            assert bits_equal(gxf, bx - (dot - d) * t[0]) and bits_equal(gyf, by - (dot - d) * t[1])
            if V == 1:
                n = rng.normal(size=2)
                n /= np.hypot(*n)
                f = np.zeros(1)
                assert L.fv_kind_flux_grad(ctypes.byref(heat), p(qi), p(qj), p(gxf), p(gyf), p(n), p(f)) == 0
                assert bits_equal(f, -(gxf * n[0] + gyf * n[1]))
    # the diffusion kind needs its gradients; V = 3 is no device width
    z = np.zeros(4)
    assert L.fv_kind_flux(4, ctypes.c_double(0.0), p(z), p(z), p(z), p(z)) == -4
    assert L.fv_kind_face_gradient(3, p(z), p(z), p(z), p(z), p(z), p(z), p(z), p(z), p(z), p(z)) == -1
    # V = 1 boundaries: the copy kind
    q, b = np.array([0.75]), np.zeros(1)
    assert L.fv_kind_bc(0, 1, ctypes.c_double(1.4), None, p(q), p(np.array([1.0, 0.0])), p(b)) == 0
    assert b[0] == 0.75


def test_host_navier_stokes_kind_matches_oracle(oracle):
    """fv_kind_flux_grad for FV_FLUX_NS and fv_kind_bc for the no-slip wall
    and the b[0] far field (host copies of the device kinds the fvhyper shim
    matches the flatPlate / nacaTransient callbacks to) against the oracle,
    which is pinned to the reference build: bit for bit."""
    import physics as P
    from cases import random_euler_state
    L = fvgpu.lib()
    dp = ctypes.POINTER(ctypes.c_double)

    def p(a):
        return a.ctypes.data_as(dp)

    rng = np.random.default_rng(9)
    ph = P.flat_plate()
    names = ["top", "bot0", "bot1", "left", "right"]
    s = fvgpu.physics_struct(ph, names)
    o = oracle.physics(ph, names)
    for _ in range(100):
        qi, qj = random_euler_state(1, int(rng.integers(1 << 30))), random_euler_state(1, int(rng.integers(1 << 30)))
        gx, gy = rng.normal(size=4), rng.normal(size=4)
        t = rng.uniform(0, 2 * np.pi); n = np.array([np.cos(t), np.sin(t)])
        f = np.zeros(4)
        assert L.fv_kind_flux_grad(ctypes.byref(s), p(qi), p(qj), p(gx), p(gy), p(n), p(f)) == 0
        assert bits_equal(f, oracle.flux_grad(o, qi, qj, gx, gy, n))
        for g, kind in ((2, 4), (0, 5)):   # bot1 no-slip, top far field (b[0] form)
            b = np.zeros(4)
            bv = np.array(ph.bcs[names[g]][1] or [0.0] * 4, np.float64)
            assert L.fv_kind_bc(kind, 4, ctypes.c_double(ph.gamma), p(bv), p(qi), p(n), p(b)) == 0
            assert bits_equal(b, oracle.bc(o, g, qi, n))


def _tile_layout(m, T):
    import ctypes as C
    L = fvgpu.lib()
    sizes = np.zeros(5, np.int64)
    i64 = C.POINTER(C.c_int64)
    rc = L.fv_mesh_tile_layout(m._h, C.c_int32(T), sizes.ctypes.data_as(i64), None, None, None, None)
    assert rc == 0, L.fv_last_error()
    nt, _, _, nh, ne = (int(x) for x in sizes)
    info = np.zeros(4 * nt, np.int32)
    halo = np.zeros(max(nh, 1), np.int32)
    eij = np.zeros(max(ne, 1), np.uint32)
    face = np.zeros(4 * m.n_real, np.uint16)
    rc = L.fv_mesh_tile_layout(m._h, C.c_int32(T), sizes.ctypes.data_as(i64), info.ctypes.data_as(C.c_void_p),
                               halo.ctypes.data_as(C.c_void_p), eij.ctypes.data_as(C.c_void_p),
                               face.ctypes.data_as(C.c_void_p))
    assert rc == 0, L.fv_last_error()
    return sizes, info.reshape(nt, 4), halo[:nh], eij[:ne], face.reshape(4, m.n_real)


@pytest.mark.parametrize("T", [64, 128, 256])
def test_tile_layout_indices_stay_in_bounds(T):
    """Every index the tile kernels read through is inside the buffers they
    stage: edge endpoints inside the tile's owned + halo slots, face words
    naming one of the tile's edges with the cell on the stated side, halo
    lists holding exactly the neighbours outside the tile, and the sizes the
    shared-memory layout is built from bounding every tile (four meshes and a
    batch of three cases)."""
    meshes = [fvgpu.Mesh.from_elements(em) for em in
              (meshgen.forward_step(n=20), meshgen.naca_ogrid(ni=48, nj=12, r_far=10.0),
               meshgen.flat_plate(nx0=6, nx1=18, ny=20), meshgen.sod_strip(40, 4))]
    # a batch of strips of uneven sizes: tiles straddle case boundaries
    meshes.append(fvgpu.Mesh.batch([fvgpu.Mesh.from_elements(meshgen.riemann_strip(n)) for n in (150, 37, 260)]))
    for m in meshes:
        N, NT = m.n_real, m.n_total
        sizes, info, halo, eij, face = _tile_layout(m, T)
        nt, max_halo, max_edges = int(sizes[0]), int(sizes[1]), int(sizes[2])
        assert nt == (N + T - 1) // T
        assert max_halo + T <= 65535 and max_edges <= 0x3FFF
        assert np.all(np.diff(info[:, 0]) == info[:-1, 1]) and np.all(np.diff(info[:, 2]) == info[:-1, 3])
        assert info[:, 1].max() == max_edges and info[:, 3].max() == max_halo
        # neighbours of every device cell from the reference edges
        g = m.geometry()
        new2ref = m.device_order()
        ref2new = np.empty_like(new2ref); ref2new[new2ref] = np.arange(NT)
        ec = ref2new[g["edge_cells"].reshape(-1, 2).astype(np.int64)]
        nbrs = [set() for _ in range(N)]
        for a, b in ec:
            if a < N: nbrs[a].add(int(b))
            if b < N: nbrs[b].add(int(a))
        for t in range(nt):
            c0, nown = t * T, min(T, N - t * T)
            e0, ne_t, h0, nh_t = (int(x) for x in info[t])
            hl = halo[h0:h0 + nh_t]
            outside = set().union(*(nbrs[c] for c in range(c0, c0 + nown))) - set(range(c0, c0 + nown))
            assert set(hl.tolist()) == outside and len(hl) == len(outside)
            li, lj = eij[e0:e0 + ne_t] & 0xFFFF, eij[e0:e0 + ne_t] >> 16
            for x in (li, lj):
                assert np.all((x < nown) | ((x >= T) & (x < T + nh_t)))
            assert np.all((li < T) | (lj < T))  # every tile edge touches an owned cell
            for c in range(c0, c0 + nown):
                for f in range(4):
                    w = int(face[f, c])
                    if w == 0xFFFF:
                        continue
                    el, ghost, side = w & 0x3FFF, (w >> 14) & 1, w >> 15
                    assert el < ne_t
                    ij = int(eij[e0 + el])
                    me, other = (ij >> 16, ij & 0xFFFF) if side else (ij & 0xFFFF, ij >> 16)
                    assert me == c - c0
                    dev_other = c0 + other if other < T else int(hl[other - T])
                    assert dev_other in nbrs[c]
                    assert ghost == (dev_other >= N)


def _tile2_layout(m, T):
    import ctypes as C
    L = fvgpu.lib()
    sizes = np.zeros(8, np.int64)
    i64 = C.POINTER(C.c_int64)
    rc = L.fv_mesh_tile2_layout(m._h, C.c_int32(T), sizes.ctypes.data_as(i64), None, None, None, None)
    assert rc == 0, L.fv_last_error()
    nt, nh, ne, nf = int(sizes[0]), int(sizes[5]), int(sizes[6]), int(sizes[7])
    info = np.zeros(8 * nt, np.int32)
    halo = np.zeros(max(nh, 1), np.int32)
    eij = np.zeros(max(ne, 1), np.uint32)
    face = np.zeros(4 * max(nf, 1), np.uint16)
    rc = L.fv_mesh_tile2_layout(m._h, C.c_int32(T), sizes.ctypes.data_as(i64), info.ctypes.data_as(C.c_void_p),
                                halo.ctypes.data_as(C.c_void_p), eij.ctypes.data_as(C.c_void_p),
                                face.ctypes.data_as(C.c_void_p))
    assert rc == 0, L.fv_last_error()
    return sizes, info.reshape(nt, 8), halo[:nh], eij[:ne], face[: 4 * nf].reshape(-1, 4)


@pytest.mark.parametrize("T", [64, 128, 256])
def test_two_ring_tile_layout_indices_stay_in_bounds(T):
    """Every index the fused stage kernel reads through is inside what it
    stages: ring 1 is exactly the outside face neighbours of the owned cells,
    ring 2 exactly the further neighbours of the ring-1 real cells; flux edges
    (the first n_flux) join an owned cell to an owned or ring-1 slot; the other
    edges join a ring-1 real cell to a ring-1 or ring-2 slot; owned cells'
    face words name flux edges only; every gradient slot's face words name one
    of the tile's edges with the cell on the stated side, in increasing
    reference edge order; edge runs start on multiples of 4 and the sizes the
    shared-memory layout is built from bound every tile (four meshes and a
    batch of three cases)."""
    meshes = [fvgpu.Mesh.from_elements(em) for em in
              (meshgen.forward_step(n=20), meshgen.naca_ogrid(ni=48, nj=12, r_far=10.0),
               meshgen.flat_plate(nx0=6, nx1=18, ny=20), meshgen.sod_strip(40, 4))]
    meshes.append(fvgpu.Mesh.batch([fvgpu.Mesh.from_elements(meshgen.riemann_strip(n)) for n in (150, 37, 260)]))
    for m in meshes:
        N, NT = m.n_real, m.n_total
        sizes, info, halo, eij, face = _tile2_layout(m, T)
        nt, max_slots, max_grad, max_edges, max_flux = (int(x) for x in sizes[:5])
        assert nt == (N + T - 1) // T
        assert max_slots <= 65535 and max_edges <= 0x3FFF and max_edges % 4 == 0
        g = m.geometry()
        new2ref = m.device_order()
        ref2new = np.empty_like(new2ref); ref2new[new2ref] = np.arange(NT)
        ec_ref = g["edge_cells"].reshape(-1, 2).astype(np.int64)
        ec = ref2new[ec_ref]
        nbrs = [set() for _ in range(N)]
        edge_of = {}
        for e, (a, b) in enumerate(ec):
            if a < N: nbrs[a].add(int(b))
            if b < N: nbrs[b].add(int(a))
            edge_of[(int(a), int(b))] = e
        face_end = 0
        for t in range(nt):
            c0, nown = t * T, min(T, N - t * T)
            e0, ne_t, nfl, h0, n1, n2, f0, _ = (int(x) for x in info[t])
            assert e0 % 4 == 0 and nfl <= ne_t and (ne_t + 3) // 4 * 4 <= max_edges and nfl <= max_flux
            assert T + n1 + n2 <= max_slots and T + n1 <= max_grad
            assert f0 == face_end
            face_end += T + n1
            owned = set(range(c0, c0 + nown))
            r1, r2 = halo[h0:h0 + n1].tolist(), halo[h0 + n1:h0 + n1 + n2].tolist()
            ring1 = set().union(*(nbrs[c] for c in owned)) - owned
            assert set(r1) == ring1 and len(r1) == len(ring1)
            ring2 = set().union(*[nbrs[c] for c in r1 if c < N]) - owned - ring1 if r1 else set()
            assert set(r2) == ring2 and len(r2) == len(ring2)
            slots = list(range(c0, c0 + T)) + r1 + r2  # device cell of each local slot
            li, lj = (eij[e0:e0 + ne_t] & 0xFFFF).astype(np.int64), (eij[e0:e0 + ne_t] >> 16).astype(np.int64)
            for x in (li, lj):
                assert np.all((x < nown) | ((x >= T) & (x < T + n1 + n2)))
            # flux edges: an owned cell and an owned or ring-1 slot
            assert np.all((li[:nfl] < T) | (lj[:nfl] < T))
            assert np.all((li[:nfl] < T + n1) & (lj[:nfl] < T + n1))
            # the other edges: a ring-1 real cell and no owned cell
            assert np.all((li[nfl:] >= T) & (lj[nfl:] >= T))
            for e in range(ne_t):
                a, b = slots[li[e]], slots[lj[e]]
                assert (a, b) in edge_of  # reference orientation
            tf = face[f0:f0 + T + n1]
            for r in range(T + n1):
                if r < T and r >= nown:
                    assert np.all(tf[r] == 0xFFFF)
                    continue
                cell = slots[r]
                if cell >= N:  # ring-1 ghost: no faces
                    assert np.all(tf[r] == 0xFFFF)
                    continue
                prev_e = -1
                nf = 0
                for f in range(4):
                    w = int(tf[r, f])
                    if w == 0xFFFF:
                        continue
                    nf += 1
                    el, ghost, side = w & 0x3FFF, (w >> 14) & 1, w >> 15
                    assert el < ne_t
                    if r < T:
                        assert el < nfl
                    me, other = (lj[el], li[el]) if side else (li[el], lj[el])
                    assert me == r
                    dev_other = slots[other]
                    assert dev_other in nbrs[cell]
                    assert ghost == (dev_other >= N)
                    e_ref = edge_of[(slots[li[el]], slots[lj[el]])]
                    assert e_ref > prev_e  # reference edge order
                    prev_e = e_ref
                assert nf == len(nbrs[cell])
        assert face_end == len(face)


def test_output_kinds_follow_the_examples_arithmetic():
    """The host copies of the device output kinds are the examples' post::
    callbacks operation for operation (examples/forwardStep/main.cpp:37-39,
    283-299; burgers/main.cpp:133-137): pressure, Mach, velocity, q[0:2]."""
    import ctypes as C
    L = fvgpu.lib()
    p = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    g = 1.4
    for seed in range(200):
        q = random_euler_state(1, seed)
        pres = (g - 1) * (q[3] - 0.5 / q[0] * (q[1] * q[1] + q[2] * q[2]))
        want = {1: [pres], 2: [(np.sqrt(q[1] * q[1] + q[2] * q[2]) / q[0]) / np.sqrt(g * pres / q[0])],
                3: [q[1] / q[0], q[2] / q[0]], 4: [q[0], q[1]]}
        for k, w in want.items():
            out = np.zeros(2)
            assert L.fv_kind_output(k, C.c_double(g), p(q), p(out)) == len(w)
            assert out[: len(w)].tobytes() == np.array(w).tobytes(), (k, seed)
    assert L.fv_kind_output(9, C.c_double(g), p(q), p(out)) == -4
