"""Pure-Python restatement of the reference mesh pipeline for SMALL meshes (test oracle only).

Follows, in order:
  * box_mesher.cpp:30-143   graded node positions, hex cells (k outer, i inner), patch tags;
  * cell_shapes.hpp:22-52   local faces of tets and hexes (outward right-hand normals);
  * mesh_builder.cpp:99-233 unique faces, internal faces sorted by (owner, neighbour),
                            boundary faces stable-sorted by (patch, owner), orientation flip;
  * mesh.cpp:100-186        face centres / area vectors, cell volumes / centres;
  * fv_geometry.cpp:17-69   over-relaxed delta coefficients, interpolation weights.
The 6-tet split of each box cell (all tets share the cube's main diagonal) and the jitter /
two-sided grading used for the synthetic pressure systems are this project's workload
definitions, implemented identically in the product generator (cfd_b200/csrc/synth.cpp).
Vector expressions are evaluated left to right (x, y, z) exactly as the C++ generator does.
"""
from __future__ import annotations

import math

import numpy as np

TET_FACES = [(0, 2, 1), (0, 1, 3), (0, 3, 2), (1, 2, 3)]
HEX_FACES = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)]
# Kuhn split: permutations of the axes; tet = (v000, v000+e_a, v000+e_a+e_b, v111).
KUHN_PERMS = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


def graded_positions(n: int, grading: float) -> list[float]:
    """box_mesher.cpp:36-46 (one-sided geometric grading)."""
    ratio = grading ** (1.0 / (n - 1)) if n > 1 else 1.0
    out = []
    for i in range(n + 1):
        if abs(ratio - 1.0) < 1e-12:
            out.append(i / n)
        else:
            out.append((ratio ** i - 1.0) / (ratio ** n - 1.0))
    return out


def two_sided_positions(n: int, ratio: float) -> list[float]:
    """Node positions in [0,1] with cell sizes growing by `ratio` from both ends to the centre
    (symmetric, smallest cells at both walls)."""
    sizes = []
    for i in range(n):
        k = min(i, n - 1 - i)
        sizes.append(ratio ** k)
    total = 0.0
    for s in sizes:
        total += s
    pos = [0.0]
    acc = 0.0
    for i in range(n):
        acc += sizes[i]
        pos.append(acc / total)
    pos[n] = 1.0
    return pos


def _sub(a, b):
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def _add(a, b):
    return (a[0] + b[0], a[1] + b[1], a[2] + b[2])


def _scale(a, s):
    return (a[0] * s, a[1] * s, a[2] * s)


def _div(a, s):
    return (a[0] / s, a[1] / s, a[2] / s)


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _norm(a):
    return math.sqrt(_dot(a, a))


class Mesh:
    def __init__(self, points, faces, owner, neighbour, n_cells, patches):
        self.points = points
        self.faces = faces          # list of node tuples (oriented owner -> neighbour / outward)
        self.owner = np.asarray(owner, np.int32)
        self.neighbour = np.asarray(neighbour, np.int32)
        self.n_cells = n_cells
        self.patches = patches      # list of (start, count)
        self._geometry()

    @property
    def n_internal_faces(self):
        return len(self.neighbour)

    def _geometry(self):
        """mesh.cpp:100-186."""
        nf = len(self.faces)
        pts = self.points
        fc, sf = [None] * nf, [None] * nf
        for f, nodes in enumerate(self.faces):
            if len(nodes) == 3:
                a, b, c = pts[nodes[0]], pts[nodes[1]], pts[nodes[2]]
                fc[f] = _div(_add(_add(a, b), c), 3.0)
                sf[f] = _scale(_cross(_sub(b, a), _sub(c, a)), 0.5)
                continue
            pc = (0.0, 0.0, 0.0)
            for p in nodes:
                pc = _add(pc, pts[p])
            pc = _div(pc, float(len(nodes)))
            sum_n, sum_ac, sum_a = (0.0, 0.0, 0.0), (0.0, 0.0, 0.0), 0.0
            for i in range(len(nodes)):
                p0, p1 = pts[nodes[i]], pts[nodes[(i + 1) % len(nodes)]]
                nvec = _cross(_sub(p1, p0), _sub(pc, p0))
                a = _norm(nvec)
                sum_n = _add(sum_n, nvec)
                sum_a += a
                sum_ac = _add(sum_ac, _scale(_add(_add(p0, p1), pc), a))
            fc[f] = _div(sum_ac, 3.0 * sum_a) if sum_a > 1e-300 else pc
            sf[f] = _scale(sum_n, 0.5)
        nc, nif = self.n_cells, self.n_internal_faces
        est = [(0.0, 0.0, 0.0)] * nc
        cnt = [0] * nc
        for f in range(nf):
            o = int(self.owner[f])
            est[o] = _add(est[o], fc[f])
            cnt[o] += 1
            if f < nif:
                n = int(self.neighbour[f])
                est[n] = _add(est[n], fc[f])
                cnt[n] += 1
        est = [_div(est[c], float(cnt[c])) if cnt[c] > 0 else est[c] for c in range(nc)]
        pyr = [0.0] * nc
        vc = [(0.0, 0.0, 0.0)] * nc
        for f in range(nf):
            o = int(self.owner[f])
            vo = _dot(sf[f], _sub(fc[f], est[o]))
            pyr[o] += vo
            vc[o] = _add(vc[o], _scale(_add(_scale(fc[f], 0.75), _scale(est[o], 0.25)), vo))
            if f < nif:
                n = int(self.neighbour[f])
                vn = _dot(sf[f], _sub(est[n], fc[f]))
                pyr[n] += vn
                vc[n] = _add(vc[n], _scale(_add(_scale(fc[f], 0.75), _scale(est[n], 0.25)), vn))
        self.face_centres = np.array(fc)
        self.face_areas = np.array(sf)
        self.cell_volumes = np.array([p / 3.0 for p in pyr])
        self.cell_centres = np.array([_div(vc[c], pyr[c]) if abs(pyr[c]) > 1e-300 else est[c]
                                      for c in range(nc)])

    def fv_geometry(self):
        """fv_geometry.cpp:17-69: returns (delta_coeffs, weights) of the internal faces."""
        nif = self.n_internal_faces
        delta = np.zeros(nif)
        w = np.zeros(nif)
        cc, cf, sfa = self.cell_centres, self.face_centres, self.face_areas
        for f in range(nif):
            s = tuple(sfa[f])
            area = _norm(s)
            cp = tuple(cc[self.owner[f]])
            cn = tuple(cc[self.neighbour[f]])
            d = _sub(cn, cp)
            s_dot_d = max(_dot(s, d), 0.05 * area * _norm(d))
            delta[f] = area * area / s_dot_d
            dp = _dot(s, _sub(tuple(cf[f]), cp))
            dn = _dot(s, _sub(cn, tuple(cf[f])))
            tot = dp + dn
            w[f] = min(max(dn / tot, 0.0), 1.0) if tot > 0.0 else 0.5
        return delta, w


def build_mesh(points, cells, tagged, n_patches):
    """MeshBuilder::build (mesh_builder.cpp:99-233). cells: list of (shape, nodes);
    tagged: list of (nodes, patch)."""
    faces = []          # [nodes(oriented from cell0), cell0, cell1]
    lookup = {}
    for c, (shape, nodes) in enumerate(cells):
        table = TET_FACES if shape == "tet" else HEX_FACES
        for lf in table:
            fn = tuple(nodes[i] for i in lf)
            key = tuple(sorted(fn))
            if key in lookup:
                rec = faces[lookup[key]]
                if rec[2] >= 0:
                    raise RuntimeError("face shared by more than two cells")
                rec[2] = c
            else:
                lookup[key] = len(faces)
                faces.append([fn, c, -1])
    face_patch = [-1] * len(faces)
    for nodes, patch in tagged:
        fi = lookup[tuple(sorted(nodes))]
        if faces[fi][2] < 0:
            face_patch[fi] = patch
    default = -1
    for f in range(len(faces)):
        if faces[f][2] < 0 and face_patch[f] < 0:
            if default < 0:
                default = n_patches
                n_patches += 1
            face_patch[f] = default

    def owner_of(f):
        r = faces[f]
        return min(r[1], r[2]) if r[2] >= 0 else r[1]

    def nb_of(f):
        r = faces[f]
        return max(r[1], r[2])

    internal = [f for f in range(len(faces)) if faces[f][2] >= 0]
    boundary = [f for f in range(len(faces)) if faces[f][2] < 0]
    internal.sort(key=lambda f: (owner_of(f), nb_of(f)))
    boundary.sort(key=lambda f: (face_patch[f], owner_of(f)))   # Python sort is stable
    out_faces, owner, neighbour = [], [], []
    for f in internal:
        nodes, c0 = faces[f][0], faces[f][1]
        o = owner_of(f)
        if c0 != o:
            nodes = (nodes[0],) + tuple(reversed(nodes[1:]))
        out_faces.append(nodes)
        owner.append(o)
        neighbour.append(nb_of(f))
    counts = [0] * n_patches
    for f in boundary:
        out_faces.append(faces[f][0])
        owner.append(faces[f][1])
        counts[face_patch[f]] += 1
    patches, start = [], len(internal)
    for p in range(n_patches):
        patches.append((start, counts[p]))
        start += counts[p]
    return Mesh(points, out_faces, owner, neighbour, len(cells), patches)


def lattice(nx, ny, nz, xs, ys, zs):
    pts = []
    for k in range(nz + 1):
        for j in range(ny + 1):
            for i in range(nx + 1):
                pts.append((xs[i], ys[j], zs[k]))
    return pts


def pid(nx, ny, i, j, k):
    return i + (nx + 1) * (j + (ny + 1) * k)


def box_tags(nx, ny, nz):
    """Patch tags of box_mesher.cpp:94-140: patch = 2*direction + side."""
    P = lambda i, j, k: pid(nx, ny, i, j, k)  # noqa: E731
    tags = []
    for i in (0, nx):
        patch = 0 if i == 0 else 1
        for k in range(nz):
            for j in range(ny):
                tags.append(((P(i, j, k), P(i, j + 1, k), P(i, j + 1, k + 1), P(i, j, k + 1)), patch))
    for j in (0, ny):
        patch = 2 if j == 0 else 3
        for k in range(nz):
            for i in range(nx):
                tags.append(((P(i, j, k), P(i + 1, j, k), P(i + 1, j, k + 1), P(i, j, k + 1)), patch))
    for k in (0, nz):
        patch = 4 if k == 0 else 5
        for j in range(ny):
            for i in range(nx):
                tags.append(((P(i, j, k), P(i + 1, j, k), P(i + 1, j + 1, k), P(i, j + 1, k)), patch))
    return tags


def hex_box(nx, ny, nz, xs, ys, zs):
    """Hex box mesh on the given node coordinates (make_box_mesh)."""
    pts = lattice(nx, ny, nz, xs, ys, zs)
    P = lambda i, j, k: pid(nx, ny, i, j, k)  # noqa: E731
    cells = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                cells.append(("hex", (P(i, j, k), P(i + 1, j, k), P(i + 1, j + 1, k), P(i, j + 1, k),
                                      P(i, j, k + 1), P(i + 1, j, k + 1), P(i + 1, j + 1, k + 1),
                                      P(i, j + 1, k + 1))))
    return build_mesh(pts, cells, box_tags(nx, ny, nz), 6)


def tet_box(nx, ny, nz, points):
    """6 tets per box cell sharing the main diagonal; boundary triangles tagged by side."""
    P = lambda i, j, k: pid(nx, ny, i, j, k)  # noqa: E731
    cells = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                for perm in KUHN_PERMS:
                    ijk = [i, j, k]
                    v = [P(*ijk)]
                    for ax in perm:
                        ijk[ax] += 1
                        v.append(P(*ijk))
                    # orientation on the undistorted lattice: sign of the permutation
                    if _perm_parity(perm) != 0:
                        v[1], v[2] = v[2], v[1]
                    cells.append(("tet", tuple(v)))
    tags = []
    for (quad, patch) in box_tags(nx, ny, nz):
        a, b, c, d = quad
        # each boundary quad is split by its diagonal through the lowest lattice corner a / c
        tags.append(((a, b, c), patch))
        tags.append(((a, c, d), patch))
    return build_mesh(points, cells, tags, 6)


def _perm_parity(perm):
    p = list(perm)
    par = 0
    for i in range(3):
        for j in range(i + 1, 3):
            if p[i] > p[j]:
                par ^= 1
    return par
