"""Synthetic 2-D element meshes for the explicit FV step, and a Gmsh MSH 4.1
ASCII writer that the fvhyper reader accepts.

A mesh here is an *element* mesh (nodes, triangles/quads, boundary segments
with physical names), i.e. what ``fvhyper::mesh::read_file`` reads from an MSH
file (fvhyper/src/mesh.cpp:264-570) before it discovers edges and computes the
finite-volume geometry.  The geometry itself is built by the native library
(``fvgpu.build_mesh``), exactly as the reader would build it.

Workloads (gmsh is not available, so these stand in for the reference's
``.geo`` inputs; sizes follow the benchmark configurations):

* ``sod_strip``       [0,1]x[0,0.1], nx*ny quads split into 2 triangles.
* ``forward_step``    [0,3]x[0,1] minus the step x>=0.6, y<0.2; Delaunay
                      triangulation of a lattice whose interior nodes are
                      jittered by a fraction of the spacing (seeded).
* ``naca_ogrid``      NACA 0012 O-grid, ni around x nj radial quads split into
                      triangles, far field at 50 chords, seeded node jitter.
* ``riemann_strips``  many independent rectangular strips of uneven size.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class ElementMesh:
    """Nodes, cells and named boundary segments (file order is array order).

    cells: int32 [nc, 4], triangles padded with -1 in the 4th column.
    bnd_nodes: int32 [nb, 2] boundary segments as node pairs.
    bnd_group: int32 [nb] index into ``group_names``.
    """

    nodes_x: np.ndarray
    nodes_y: np.ndarray
    cells: np.ndarray
    bnd_nodes: np.ndarray
    bnd_group: np.ndarray
    group_names: list

    @property
    def n_cells(self) -> int:
        return int(self.cells.shape[0])

    @property
    def n_bound(self) -> int:
        return int(self.bnd_nodes.shape[0])

    def bc_name_per_segment(self):
        return [self.group_names[g] for g in self.bnd_group]


def _finish(nx_, ny_, cells, segs, groups, names) -> ElementMesh:
    cells = np.ascontiguousarray(cells, dtype=np.int32)
    segs = np.ascontiguousarray(segs, dtype=np.int32)
    groups = np.ascontiguousarray(groups, dtype=np.int32)
    order = np.argsort(groups, kind="stable")  # one MSH block per group
    return ElementMesh(np.ascontiguousarray(nx_, dtype=np.float64),
                       np.ascontiguousarray(ny_, dtype=np.float64),
                       cells, segs[order], groups[order], list(names))


# --------------------------------------------------------------------------
# Structured rectangle split into triangles (Sod, Riemann strips)
# --------------------------------------------------------------------------
def rect_tri(nx: int, ny: int, lx: float, ly: float, x0: float = 0.0, y0: float = 0.0,
             side_names=("wall", "ends")) -> ElementMesh:
    """nx*ny quads, each split on its lower-left/upper-right diagonal.

    Boundary groups: side_names[0] on bottom and top, side_names[1] on the
    left and right ends.
    """
    xs = x0 + lx * np.arange(nx + 1, dtype=np.float64) / nx
    ys = y0 + ly * np.arange(ny + 1, dtype=np.float64) / ny
    X, Y = np.meshgrid(xs, ys)  # [ny+1, nx+1]
    nid = np.arange((nx + 1) * (ny + 1), dtype=np.int64).reshape(ny + 1, nx + 1)
    n00 = nid[:-1, :-1].ravel(); n10 = nid[:-1, 1:].ravel()
    n11 = nid[1:, 1:].ravel(); n01 = nid[1:, :-1].ravel()
    t1 = np.stack([n00, n10, n11, -np.ones_like(n00)], 1)
    t2 = np.stack([n00, n11, n01, -np.ones_like(n00)], 1)
    cells = np.stack([t1, t2], 1).reshape(-1, 4)
    bottom = np.stack([nid[0, :-1], nid[0, 1:]], 1)
    top = np.stack([nid[-1, 1:], nid[-1, :-1]], 1)
    left = np.stack([nid[1:, 0], nid[:-1, 0]], 1)
    right = np.stack([nid[:-1, -1], nid[1:, -1]], 1)
    segs = np.concatenate([bottom, top, left, right])
    groups = np.concatenate([np.zeros(nx + nx, np.int32), np.ones(ny + ny, np.int32)])
    return _finish(X.ravel(), Y.ravel(), cells, segs, groups, side_names)


def _graded(n: int, ratio: float) -> np.ndarray:
    """n + 1 points on [0, 1], cell sizes growing by `ratio` from 0 to 1."""
    if n == 0:
        return np.zeros(1)
    w = ratio ** np.arange(n, dtype=np.float64)
    return np.concatenate([[0.0], np.cumsum(w) / w.sum()])


def flat_plate(nx0: int = 30, nx1: int = 90, ny: int = 110, x_lead: float = -0.1, lx: float = 1.0,
               ly: float = 0.2, r_up: float = 1.2, r_plate: float = 1.1, r_y: float = 1.1) -> ElementMesh:
    """Quadrilateral flat-plate mesh in the layout of examples/flatPlate/square.geo:
    x in [x_lead, lx], y in [0, ly]; nx0 columns upstream of the leading edge
    (x = 0) and nx1 along the plate, ny rows; cells shrink geometrically
    toward the leading edge (ratios r_up, r_plate) and the wall (r_y).
    Groups: top, bot0 (bottom, x < 0), bot1 (bottom, the plate), left, right."""
    xu = x_lead * _graded(nx0, r_up)[::-1]          # x_lead .. 0, fine at 0
    xp = lx * _graded(nx1, r_plate)                 # 0 .. lx, fine at 0
    xs = np.concatenate([xu, xp[1:]])
    ys = ly * _graded(ny, r_y)
    nx = nx0 + nx1
    X, Y = np.meshgrid(xs, ys)
    nid = np.arange((nx + 1) * (ny + 1), dtype=np.int64).reshape(ny + 1, nx + 1)
    cells = np.stack([nid[:-1, :-1].ravel(), nid[:-1, 1:].ravel(), nid[1:, 1:].ravel(),
                      nid[1:, :-1].ravel()], 1)
    bottom = np.stack([nid[0, :-1], nid[0, 1:]], 1)
    top = np.stack([nid[-1, 1:], nid[-1, :-1]], 1)
    left = np.stack([nid[1:, 0], nid[:-1, 0]], 1)
    right = np.stack([nid[:-1, -1], nid[1:, -1]], 1)
    segs = np.concatenate([top, bottom[:nx0], bottom[nx0:], left, right])
    groups = np.concatenate([np.zeros(nx, np.int32), np.ones(nx0, np.int32), np.full(nx1, 2, np.int32),
                             np.full(ny, 3, np.int32), np.full(ny, 4, np.int32)])
    m = _finish(X.ravel(), Y.ravel(), cells, segs, groups, ["top", "bot0", "bot1", "left", "right"])
    check_orientation(m)
    return m


def sod_strip(nx: int = 400, ny: int = 40, ly: float = 0.1) -> ElementMesh:
    """Sod shock tube domain [0,1]x[0,ly]: 'wall' top/bottom, 'ends' left/right."""
    return rect_tri(nx, ny, 1.0, ly)


# --------------------------------------------------------------------------
# Forward-facing step: jittered lattice + Delaunay
# --------------------------------------------------------------------------
def forward_step(n: int = 445, jitter: float = 0.2, seed: int = 2,
                 step_x: float = 0.6, step_h: float = 0.2) -> ElementMesh:
    """[0,3]x[0,1] with the step x>=step_x, y<step_h removed.

    Lattice spacing h = 1/n (n must make step_x/h and step_h/h integers);
    interior nodes are moved by U(-jitter*h, jitter*h) per coordinate, nodes
    on the boundary stay on it.  Groups: inlet (x=0), outlet (x=3),
    wall (top, bottom before the step, step top), step (the vertical face).
    """
    from scipy.spatial import Delaunay

    h = 1.0 / n
    ix_s, iy_s = round(step_x * n), round(step_h * n)
    if abs(ix_s * h - step_x) > 1e-12 or abs(iy_s * h - step_h) > 1e-12:
        raise ValueError("n must place lattice lines on the step")
    nxl, nyl = 3 * n, n
    I, J = np.meshgrid(np.arange(nxl + 1), np.arange(nyl + 1))
    I = I.ravel(); J = J.ravel()
    keep = ~((I > ix_s) & (J < iy_s))
    I = I[keep]; J = J[keep]
    x = I * h; y = J * h
    on_bnd = (I == 0) | (I == nxl) | (J == 0) | (J == nyl) | \
             ((I == ix_s) & (J <= iy_s)) | ((J == iy_s) & (I >= ix_s))
    rng = np.random.default_rng(seed)
    d = rng.uniform(-jitter * h, jitter * h, size=(x.size, 2))
    d[on_bnd] = 0.0
    x = x + d[:, 0]; y = y + d[:, 1]
    # exact lattice coordinates on the boundary
    x[on_bnd] = I[on_bnd] * h; y[on_bnd] = J[on_bnd] * h
    pts = np.stack([x, y], 1)
    tri = Delaunay(pts).simplices.astype(np.int64)
    cx = pts[tri, 0].mean(1); cy = pts[tri, 1].mean(1)
    area = 0.5 * np.abs((pts[tri[:, 1], 0] - pts[tri[:, 0], 0]) * (pts[tri[:, 2], 1] - pts[tri[:, 0], 1])
                        - (pts[tri[:, 2], 0] - pts[tri[:, 0], 0]) * (pts[tri[:, 1], 1] - pts[tri[:, 0], 1]))
    ok = ~((cx > step_x) & (cy < step_h)) & (area > 1e-6 * h * h)
    tri = tri[ok]; cx = cx[ok]; cy = cy[ok]
    # row-major cell order (strips of 8h), like a frontal mesher's output
    order = np.lexsort((cx, np.floor(cy / (8 * h))))
    tri = tri[order]
    # node index lookup by lattice coordinate for the boundary walk
    lut = -np.ones((nyl + 1, nxl + 1), dtype=np.int64)
    lut[J, I] = np.arange(I.size)

    def walk(pairs):
        return np.array([[lut[j0, i0], lut[j1, i1]] for (i0, j0), (i1, j1) in pairs], np.int64)

    segs, groups = [], []
    names = ["wall", "inlet", "outlet", "step"]

    def add(pairs, g):
        s = walk(pairs); segs.append(s); groups.append(np.full(len(s), g, np.int32))

    add([((i, 0), (i + 1, 0)) for i in range(ix_s)], 0)                      # bottom
    add([((ix_s, j), (ix_s, j + 1)) for j in range(iy_s)], 3)                # step face
    add([((i, iy_s), (i + 1, iy_s)) for i in range(ix_s, nxl)], 0)           # step top
    add([((nxl, j), (nxl, j + 1)) for j in range(iy_s, nyl)], 2)             # outlet
    add([((i + 1, nyl), (i, nyl)) for i in range(nxl)], 0)                   # top
    add([((0, j + 1), (0, j)) for j in range(nyl)], 1)                       # inlet
    segs = np.concatenate(segs); groups = np.concatenate(groups)
    cells = np.concatenate([tri, -np.ones((tri.shape[0], 1), np.int64)], 1)
    m = _finish(x, y, cells, segs, groups, names)
    check_closed(m)
    return m


# --------------------------------------------------------------------------
# NACA 0012 O-grid
# --------------------------------------------------------------------------
def naca0012_thickness(x):
    """Half thickness of the NACA 0012 section (4-digit formula, closed TE)."""
    t = 0.12
    return 5 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)


def naca_ogrid(ni: int = 1024, nj: int = 512, r_far: float = 50.0, first=None,
               jitter: float = 0.1, seed: int = 3) -> ElementMesh:
    """O-grid around NACA 0012 (chord 1, mid-chord at (0.5, 0)).

    ni nodes around the section at equal arc length, nj cell layers out to a
    circle of radius r_far with geometric growth from a first layer of
    ``first`` chords (default: the surface spacing, so wall cells are close to
    square); interior nodes are jittered by ``jitter`` times the local
    spacing.  Groups: airfoil (j=0), farfield (j=nj).
    """
    # dense cosine parametrisation of the closed section, resampled at equal
    # arc length; theta(s) also gives the direction of each radial line
    thd = np.linspace(0.0, 2 * np.pi, 200001)
    xd = 0.5 * (1 + np.cos(thd))
    yd = np.where(thd <= np.pi, 1.0, -1.0) * naca0012_thickness(xd)
    sd = np.concatenate([[0.0], np.cumsum(np.hypot(np.diff(xd), np.diff(yd)))])
    s_i = sd[-1] * np.arange(ni) / ni
    th = np.interp(s_i, sd, thd)
    xa = 0.5 * (1 + np.cos(th))
    ya = np.where(th <= np.pi, 1.0, -1.0) * naca0012_thickness(xa)
    ya[0] = 0.0
    if first is None:
        first = sd[-1] / ni
    # far-field node at the same parametric angle: rays leave the section at a
    # steep angle even near the thin trailing edge, so layers never fold
    xf = 0.5 + r_far * np.cos(th); yf = r_far * np.sin(th)
    # geometric growth ratio so that the first layer is `first` chords thick
    L = r_far - 0.5
    lo, hi = 1.0 + 1e-9, 1.5
    for _ in range(200):
        r = 0.5 * (lo + hi)
        if first * (r ** nj - 1) / (r - 1) > L:
            hi = r
        else:
            lo = r
    s = (r ** np.arange(nj + 1) - 1) / (r ** nj - 1)
    X = xa[None, :] + s[:, None] * (xf - xa)[None, :]   # [nj+1, ni]
    Y = ya[None, :] + s[:, None] * (yf - ya)[None, :]
    rng = np.random.default_rng(seed)
    dr = np.hypot(np.diff(X, axis=0), np.diff(Y, axis=0))          # [nj, ni]
    dt = np.hypot(np.roll(X, -1, 1) - X, np.roll(Y, -1, 1) - Y)   # [nj+1, ni]
    loc = np.minimum(np.minimum(dr[:-1], dr[1:]), np.minimum(dt[1:-1], np.roll(dt[1:-1], 1, 1)))
    d = rng.uniform(-1, 1, size=(nj - 1, ni, 2)) * (jitter * loc)[..., None]
    X[1:-1] += d[..., 0]; Y[1:-1] += d[..., 1]
    nid = np.arange((nj + 1) * ni, dtype=np.int64).reshape(nj + 1, ni)
    nid_ip = np.roll(nid, -1, 1)
    n00 = nid[:-1].ravel(); n10 = nid_ip[:-1].ravel()
    n11 = nid_ip[1:].ravel(); n01 = nid[1:].ravel()
    t1 = np.stack([n00, n10, n11, -np.ones_like(n00)], 1)
    t2 = np.stack([n00, n11, n01, -np.ones_like(n00)], 1)
    cells = np.stack([t1, t2], 1).reshape(-1, 4)
    air = np.stack([nid[0], nid_ip[0]], 1)
    far = np.stack([nid_ip[-1], nid[-1]], 1)
    segs = np.concatenate([air, far])
    groups = np.concatenate([np.zeros(ni, np.int32), np.ones(ni, np.int32)])
    m = _finish(X.ravel(), Y.ravel(), cells, segs, groups, ["airfoil", "farfield"])
    check_orientation(m)
    return m


# --------------------------------------------------------------------------
# Batched Riemann strips
# --------------------------------------------------------------------------
def riemann_strip_sizes(n_cases: int = 256, nmin: int = 2000, nmax: int = 200000, seed: int = 4,
                        ny: int = 8):
    """Cell counts log-uniform in [nmin, nmax]; each strip is nx x ny x 2 triangles."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(nmin), np.log(nmax), n_cases))
    nx = np.maximum(1, np.round(n / (2 * ny))).astype(np.int64)
    states = np.stack([rng.uniform(0.1, 1.0, n_cases), rng.uniform(-0.5, 0.5, n_cases),
                       rng.uniform(0.1, 1.0, n_cases), rng.uniform(0.1, 1.0, n_cases),
                       rng.uniform(-0.5, 0.5, n_cases), rng.uniform(0.1, 1.0, n_cases)], 1)
    return nx, states  # states: rhoL, uL, pL, rhoR, uR, pR


def riemann_strip(nx: int, ny: int = 8) -> ElementMesh:
    """One strip [0,1]x[0, ny/nx]: 'wall' top/bottom, 'ends' left/right."""
    return rect_tri(int(nx), ny, 1.0, ny / float(nx))


# --------------------------------------------------------------------------
# Checks and MSH 4.1 output
# --------------------------------------------------------------------------
def signed_areas(m: ElementMesh) -> np.ndarray:
    X, Y, c = m.nodes_x, m.nodes_y, m.cells
    return 0.5 * ((X[c[:, 1]] - X[c[:, 0]]) * (Y[c[:, 2]] - Y[c[:, 0]])
                  - (X[c[:, 2]] - X[c[:, 0]]) * (Y[c[:, 1]] - Y[c[:, 0]]))


def check_orientation(m: ElementMesh) -> None:
    """All triangles wound the same way (a folded mesh has mixed signs)."""
    sa = signed_areas(m)
    if not (np.all(sa > 0) or np.all(sa < 0)):
        raise ValueError(f"folded mesh: {int(np.sum(sa > 0))} positive / {int(np.sum(sa < 0))} negative cells")


def check_closed(m: ElementMesh) -> None:
    """Every edge used by one cell only must be a declared boundary segment."""
    c = m.cells
    ntri = c[:, 3] < 0
    e = []
    for k in range(4):
        a = c[:, k]; b = np.where((k == 2) & ntri, c[:, 0], c[:, (k + 1) % 4])
        valid = ~((k == 3) & ntri)
        e.append(np.stack([a[valid], b[valid]], 1))
    e = np.sort(np.concatenate(e), 1)
    key = e[:, 0].astype(np.int64) * (1 << 32) + e[:, 1]
    u, cnt = np.unique(key, return_counts=True)
    if np.any(cnt > 2):
        raise ValueError("non-manifold edge")
    once = set(u[cnt == 1].tolist())
    b = np.sort(m.bnd_nodes.astype(np.int64), 1)
    bkey = set((b[:, 0] * (1 << 32) + b[:, 1]).tolist())
    if once != bkey:
        raise ValueError(f"boundary mismatch: {len(once ^ bkey)} edges differ")


def write_msh41(path: str, m: ElementMesh) -> None:
    """Gmsh MSH 4.1 ASCII with one curve entity per boundary group.

    Coordinates use 17 significant digits so they read back bit-exact.  Cell
    and boundary-segment order in the file is array order (the reader keeps
    file order: mesh.cpp:487-570 for cells, 418-483 for boundary segments).
    """
    nn = m.nodes_x.size
    ng = len(m.group_names)
    surf_tag = ng + 1
    lines = ["$MeshFormat", "4.1 0 8", "$EndMeshFormat", "$PhysicalNames", str(ng + 1)]
    for g, name in enumerate(m.group_names):
        lines.append(f'1 {g + 1} "{name}"')
    lines.append(f'2 {surf_tag} "internal"')
    lines += ["$EndPhysicalNames", "$Entities", f"0 {ng} 1 0"]
    for g in range(ng):
        lines.append(f"{g + 1} 0 0 0 0 0 0 1 {g + 1} 0")
    lines.append("1 0 0 0 0 0 0 1 %d %d %s" % (surf_tag, ng, " ".join(str(g + 1) for g in range(ng))))
    lines += ["$EndEntities", "$Nodes", f"1 {nn} 1 {nn}", f"2 1 0 {nn}"]
    body = [("\n".join(map(str, range(1, nn + 1))))]
    xy = np.stack([m.nodes_x, m.nodes_y], 1)
    body.append("\n".join("%.17g %.17g 0" % (a, b) for a, b in xy))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
        f.write("\n".join(body) + "\n")
        f.write("$EndNodes\n$Elements\n")
        # element blocks: boundary runs per group, then runs of equal cell type
        blocks = []
        bg = m.bnd_group
        start = 0
        for i in range(1, bg.size + 1):
            if i == bg.size or bg[i] != bg[start]:
                blocks.append((1, int(bg[start]) + 1, 1, m.bnd_nodes[start:i]))
                start = i
        c = m.cells
        istri = c[:, 3] < 0
        start = 0
        for i in range(1, c.shape[0] + 1):
            if i == c.shape[0] or istri[i] != istri[start]:
                if istri[start]:
                    blocks.append((2, 1, 2, c[start:i, :3]))
                else:
                    blocks.append((2, 1, 3, c[start:i, :4]))
                start = i
        ne = sum(b[3].shape[0] for b in blocks)
        f.write(f"{len(blocks)} {ne} 1 {ne}\n")
        tag = 1
        for dim, ent, etype, conn in blocks:
            f.write(f"{dim} {ent} {etype} {conn.shape[0]}\n")
            tags = np.arange(tag, tag + conn.shape[0])[:, None]
            arr = np.concatenate([tags, conn.astype(np.int64) + 1], 1)
            f.write("\n".join(" ".join(map(str, r)) for r in arr.tolist()) + "\n")
            tag += conn.shape[0]
        f.write("$EndElements\n")


def write_su2(path: str, m: ElementMesh) -> None:
    """SU2 native ASCII mesh: triangles (VTK 5) / quadrilaterals (VTK 9), one
    marker per boundary group with its segments (VTK 3), in array order."""
    lines = ["NDIME= 2", f"NELEM= {m.cells.shape[0]}"]
    for e, c in enumerate(m.cells):
        if c[3] < 0:
            lines.append(f"5 {c[0]} {c[1]} {c[2]} {e}")
        else:
            lines.append(f"9 {c[0]} {c[1]} {c[2]} {c[3]} {e}")
    lines.append(f"NPOIN= {m.nodes_x.size}")
    for i in range(m.nodes_x.size):
        lines.append(f"{m.nodes_x[i]:.17g} {m.nodes_y[i]:.17g} {i}")
    lines.append(f"NMARK= {len(m.group_names)}")
    for g, name in enumerate(m.group_names):
        segs = m.bnd_nodes[m.bnd_group == g]
        lines.append(f"MARKER_TAG= {name}")
        lines.append(f"MARKER_ELEMS= {segs.shape[0]}")
        lines += [f"3 {a} {b}" for a, b in segs]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
