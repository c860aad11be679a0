"""Seeded synthetic fragment collections: the workloads the backend is measured on.

No reference data is needed or used. A wall (a pot of revolution, or a curved slab) is
partitioned into cells in its (u, v) parameter plane — for a pot by a seeded spherical
Voronoi partition of the directions from the pot's centre, for the slab by one cut — and every
cell becomes one closed triangle mesh:

  * the outer and inner shells (w = +1 and w = -1 through the wall) are meshed by rings
    between the cell centre and the cell boundary;
  * the boundary is found by bisection along rays from the centre on the partition's label
    function, so two neighbours share the same boundary curve;
  * the side wall joins the two shell boundaries in L layers; along a fracture (a boundary
    shared with another cell) it is displaced in the parameter plane by a seeded fBm field
    of the 3D position and of the depth in the wall, along the boundary normal oriented from
    the lower cell id to the higher one, so both neighbours carry the same fracture surface;
    along a rim (the end of the wall) it is left flat.

Samples follow R 3.5 (area-weighted faces, u+v folding): fracture samples `Pf` on the fracture
faces, surface samples `S` on every face, the breakline is the shell/fracture boundary of both
shells with the shell normal `brk_ns`, the margin is the surface samples on shell faces within
[0.15 t, 0.6 t] of the breakline, and the registration cloud is R 3.6's prefix split
(fragment/samples.rs:601-615). Each fragment is then placed by a seeded rigid pose; the
ground-truth relative pose of a pair is known exactly, and the ladder starts are drawn around
it (adjacent pairs) or at poses that bring the two fracture centroids together (the rest).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from scipy.spatial import cKDTree

# ---------------------------------------------------------------------------------------------
# walls
# ---------------------------------------------------------------------------------------------


class PotWall:
    """Surface of revolution r(z) = r0 + amp sin(z / wave), height h, wall t (normal offset)."""

    def __init__(self, t, r0=60.0, amp=15.0, wave=40.0, height=200.0):
        self.t, self.r0, self.amp, self.wave, self.height = t, r0, amp, wave, height
        self.rbar = r0
        self.period = 2 * np.pi * self.rbar
        self.centre = np.array([0.0, 0.0, height / 2])

    def r(self, v):
        return self.r0 + self.amp * np.sin(v / self.wave)

    def dr(self, v):
        return self.amp / self.wave * np.cos(v / self.wave)

    def point(self, u, v, w):
        th = u / self.rbar
        dr = self.dr(v)
        norm = np.sqrt(1.0 + dr * dr)
        nr, nz = 1.0 / norm, -dr / norm
        rad = self.r(v) + w * self.t / 2 * nr
        return np.stack([rad * np.cos(th), rad * np.sin(th), v + w * self.t / 2 * nz], axis=-1)

    def normal(self, u, v):
        th = u / self.rbar
        dr = self.dr(v)
        norm = np.sqrt(1.0 + dr * dr)
        return np.stack([np.cos(th) / norm, np.sin(th) / norm, -dr / norm], axis=-1)

    def inside_domain(self, u, v):
        return (v >= 0.0) & (v <= self.height)


class SlabWall:
    """A curved slab over [0, lu] x [0, lv] with an elliptic sag, wall t."""

    def __init__(self, t, lu=200.0, lv=100.0, sag=(20.0, 10.0)):
        self.t, self.lu, self.lv, self.sag = t, lu, lv, sag
        self.period = None

    def _z(self, u, v):
        a, b = self.sag
        return a * ((u - self.lu / 2) / self.lu) ** 2 + b * ((v - self.lv / 2) / self.lv) ** 2

    def normal(self, u, v):
        a, b = self.sag
        zu = 2 * a * (u - self.lu / 2) / self.lu ** 2
        zv = 2 * b * (v - self.lv / 2) / self.lv ** 2
        n = np.stack([-zu, -zv, np.ones_like(zu)], axis=-1)
        return n / np.linalg.norm(n, axis=-1, keepdims=True)

    def point(self, u, v, w):
        base = np.stack([u, v, self._z(u, v)], axis=-1)
        return base + (w * self.t / 2)[..., None] * self.normal(u, v) if np.ndim(w) else \
            base + w * self.t / 2 * self.normal(u, v)

    def inside_domain(self, u, v):
        return (u >= 0) & (u <= self.lu) & (v >= 0) & (v <= self.lv)


class SphereVoronoi:
    """Cells of the pot: the seed direction nearest the direction from the pot centre."""

    def __init__(self, wall: PotWall, seeds: np.ndarray):
        self.wall, self.seeds = wall, seeds

    def scores(self, u, v):
        p = self.wall.point(u, v, np.zeros_like(u)) - self.wall.centre
        p = p / np.linalg.norm(p, axis=-1, keepdims=True)
        return p @ self.seeds.T

    def label(self, u, v):
        lab = np.argmax(self.scores(u, v), axis=-1)
        return np.where(self.wall.inside_domain(u, v), lab, -1)


class SlabCut:
    """The slab's two cells, split at u = lu / 2 (the fracture's mean plane)."""

    def __init__(self, wall: SlabWall):
        self.wall = wall

    def scores(self, u, v):
        s = u - self.wall.lu / 2
        return np.stack([-s, s], axis=-1)

    def label(self, u, v):
        lab = (u > self.wall.lu / 2).astype(np.int64)
        return np.where(self.wall.inside_domain(u, v), lab, -1)


class Field:
    """fBm of a 3D point: a sum of octaves of random plane waves (plus optional sinusoids)."""

    def __init__(self, rng, wavelength, octaves=5, gain=0.5, extra_sines=0):
        self.k, self.phase, self.weight = [], [], []
        for o in range(octaves):
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            self.k.append(d * (2 * np.pi / wavelength) * 2.0 ** o)
            self.phase.append(rng.uniform(0, 2 * np.pi))
            self.weight.append(gain ** o)
        for _ in range(extra_sines):
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            self.k.append(d * (2 * np.pi / (wavelength * rng.uniform(2.0, 5.0))))
            self.phase.append(rng.uniform(0, 2 * np.pi))
            self.weight.append(1.0)
        self.k = np.array(self.k)
        self.phase = np.array(self.phase)
        self.weight = np.array(self.weight) / np.sum(self.weight)

    def __call__(self, x):
        return np.sin(x @ self.k.T + self.phase) @ self.weight


# ---------------------------------------------------------------------------------------------
# one cell -> one closed mesh
# ---------------------------------------------------------------------------------------------


@dataclass
class CellMesh:
    v: np.ndarray      # f64 (nv, 3), world frame
    f: np.ndarray      # u32 (nf, 3)
    frac: np.ndarray   # u8 (nf,) ground-truth fracture faces
    shell: np.ndarray  # u8 (nf,) outer/inner shell faces
    brk_p: np.ndarray  # f64 (nb, 3) shell/fracture boundary points
    brk_ns: np.ndarray  # f64 (nb, 3) shell normal there
    neighbours: set = field(default_factory=set)
    h: float = 0.0


def _march(part, cell, c, phi, rmax, step):
    """First exit radius of each ray from c (bisection to 1e-9 of rmax), and the label past it."""
    d = np.stack([np.cos(phi), np.sin(phi)], axis=-1)
    radii = np.arange(step, rmax + step, step)
    pts = c[None, None, :] + radii[None, :, None] * d[:, None, :]
    lab = part.label(pts[..., 0], pts[..., 1])
    out = lab != cell
    first = np.where(out.any(axis=1), out.argmax(axis=1), len(radii) - 1)
    hi = radii[first]
    lo = np.where(first > 0, radii[np.maximum(first - 1, 0)], 0.0)
    for _ in range(40):
        mid = 0.5 * (lo + hi)
        q = c + mid[:, None] * d
        inside = part.label(q[:, 0], q[:, 1]) == cell
        lo = np.where(inside, mid, lo)
        hi = np.where(inside, hi, mid)
    q = c + (hi + 1e-6)[:, None] * d
    nb = part.label(q[:, 0], q[:, 1])
    return lo, nb


def _edge_normal(part, i, j, u, v, eps=1e-3):
    """Unit gradient in the parameter plane of score_hi - score_lo, hi = max(i, j)."""
    lo_c, hi_c = np.minimum(i, j), np.maximum(i, j)

    def h(uu, vv):
        s = part.scores(uu, vv)
        idx = np.arange(len(uu))
        return s[idx, hi_c] - s[idx, lo_c]

    gu = (h(u + eps, v) - h(u - eps, v)) / (2 * eps)
    gv = (h(u, v + eps) - h(u, v - eps)) / (2 * eps)
    g = np.stack([gu, gv], axis=-1)
    return g / np.maximum(np.linalg.norm(g, axis=-1, keepdims=True), 1e-300)


def cell_mesh(wall, part, cell, centre, h, noise: Field, amp, rmax, rim_taper) -> CellMesh:
    """The closed mesh of one cell at target edge length h."""
    t = wall.t
    # Boundary rays: enough that the outermost spacing is about h.
    probe = np.linspace(0, 2 * np.pi, 64, endpoint=False)
    r0, _ = _march(part, cell, centre, probe, rmax, h)
    n_b = max(24, int(np.ceil(2 * np.pi * r0.max() / h)))
    phi = np.linspace(0, 2 * np.pi, n_b, endpoint=False)
    rho, nb = _march(part, cell, centre, phi, rmax, h / 2)
    b = centre + rho[:, None] * np.stack([np.cos(phi), np.sin(phi)], axis=-1)
    fracture = nb >= 0
    L = max(2, int(np.ceil(t / h)))
    w = np.linspace(-1.0, 1.0, L + 1)
    nu = np.zeros_like(b)
    if fracture.any():
        nu[fracture] = _edge_normal(part, np.full(fracture.sum(), cell), nb[fracture],
                                    b[fracture, 0], b[fracture, 1])
    mid3 = wall.point(b[:, 0], b[:, 1], np.zeros(n_b))
    taper = np.ones(n_b)
    if rim_taper is not None:
        taper = rim_taper(b[:, 0], b[:, 1])
    # Displaced boundary per wall layer: (n_b, L+1, 2).
    x = np.concatenate([np.repeat(mid3[:, None, :], L + 1, axis=1),
                        np.broadcast_to((w * t / 2)[None, :, None], (n_b, L + 1, 1))], axis=-1)
    delta = amp * noise(x.reshape(-1, 4)[:, :3] + x.reshape(-1, 4)[:, 3:4] * np.array([0.3, 0.5, 0.7]))
    delta = delta.reshape(n_b, L + 1) * (fracture * taper)[:, None]
    bd = b[:, None, :] + delta[..., None] * nu[:, None, :]
    # Vertices: side wall (n_b x (L+1)), then outer rings, then inner rings, then centres.
    M = max(2, int(np.ceil(rho.max() / h)))
    side = wall.point(bd[..., 0], bd[..., 1], np.broadcast_to(w[None, :], (n_b, L + 1)))
    verts = [side.reshape(-1, 3)]
    base_outer = 0
    n_side = n_b * (L + 1)

    def ring_vertices(level_b, wv):
        fr = (np.arange(1, M) / M)[:, None, None]
        pts = centre[None, None, :] + fr * (level_b[None, :, :] - centre[None, None, :])
        return wall.point(pts[..., 0], pts[..., 1], np.full(pts.shape[:2], wv)).reshape(-1, 3)

    outer = ring_vertices(bd[:, L, :], 1.0)
    inner = ring_vertices(bd[:, 0, :], -1.0)
    off_outer = n_side
    off_inner = off_outer + len(outer)
    c_outer = off_inner + len(inner)
    c_inner = c_outer + 1
    verts += [outer, inner, wall.point(centre[0:1], centre[1:2], np.array([1.0])),
              wall.point(centre[0:1], centre[1:2], np.array([-1.0]))]
    V = np.concatenate(verts)
    k = np.arange(n_b)
    k1 = (k + 1) % n_b

    def side_idx(kk, ll):
        return kk * (L + 1) + ll

    def ring_idx(off, m, kk, top_row):
        # ring m in 1..M; ring M is the side wall's row `top_row`
        if m == M:
            return side_idx(kk, top_row)
        return off + (m - 1) * n_b + kk

    faces = []
    labels = []
    shell = []
    # side wall
    for l in range(L):
        a = side_idx(k, l)
        bb = side_idx(k1, l)
        cc = side_idx(k1, l + 1)
        dd = side_idx(k, l + 1)
        fr = fracture & fracture[k1]
        faces += [np.stack([a, bb, cc], 1), np.stack([a, cc, dd], 1)]
        labels += [fr, fr]
        shell += [np.zeros(n_b, bool)] * 2
    # shells
    for off, top_row, centre_idx, flip in ((off_outer, L, c_outer, False),
                                           (off_inner, 0, c_inner, True)):
        tri = [np.stack([np.full(n_b, centre_idx), ring_idx(off, 1, k, top_row),
                         ring_idx(off, 1, k1, top_row)], 1)]
        for m in range(1, M):
            a = ring_idx(off, m, k, top_row)
            bb = ring_idx(off, m + 1, k, top_row)
            cc = ring_idx(off, m + 1, k1, top_row)
            dd = ring_idx(off, m, k1, top_row)
            tri += [np.stack([a, bb, cc], 1), np.stack([a, cc, dd], 1)]
        tri = np.concatenate(tri)
        if flip:
            tri = tri[:, ::-1]
        faces.append(tri)
        labels.append(np.zeros(len(tri), bool))
        shell.append(np.ones(len(tri), bool))
    F = np.concatenate(faces).astype(np.int64)
    frac = np.concatenate(labels)
    sh = np.concatenate(shell)
    # The whole mesh is oriented outward when its signed volume is positive.
    a, bq, cq = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    vol = np.einsum("ij,ij->i", a, np.cross(bq, cq)).sum() / 6.0
    if vol < 0:
        F = F[:, ::-1]
    # Breakline: both shells' boundary vertices along fractures, with the shell normal.
    bk = np.nonzero(fracture)[0]
    out_pts = side[bk, L]
    in_pts = side[bk, 0]
    n_out = wall.normal(bd[bk, L, 0], bd[bk, L, 1])
    n_in = -wall.normal(bd[bk, 0, 0], bd[bk, 0, 1])
    nbs = set(int(x) for x in np.unique(nb[fracture]))
    return CellMesh(v=V, f=F.astype(np.uint32), frac=frac.astype(np.uint8), shell=sh.astype(np.uint8),
                    brk_p=np.concatenate([out_pts, in_pts]), brk_ns=np.concatenate([n_out, n_in]),
                    neighbours=nbs, h=h)


# ---------------------------------------------------------------------------------------------
# samples (R 3.5 / R 3.6) and the fragment record
# ---------------------------------------------------------------------------------------------


def face_geometry(v, f):
    """mesh/geometry.rs:70-96 in numpy (the same element-wise operations)."""
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    e1, e2 = b - a, c - a
    n = np.stack([e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1],
                  e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2],
                  e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]], axis=1)
    length = np.sqrt((n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1]) + n[:, 2] * n[:, 2])
    den = np.maximum(length, 1e-12)
    return n / den[:, None], 0.5 * length, (a + b + c) / 3.0


def sample_on_faces(rng, v, f, areas, faces, n):
    """R 3.5's area-weighted sampling with u+v folding: (points, face ids)."""
    w = areas[faces]
    pick = faces[rng.choice(len(faces), size=n, p=w / w.sum())]
    uv = rng.uniform(size=(n, 2))
    fold = uv.sum(1) > 1
    uv[fold] = 1 - uv[fold]
    a, b, c = v[f[pick, 0]], v[f[pick, 1]], v[f[pick, 2]]
    return a + uv[:, :1] * (b - a) + uv[:, 1:] * (c - a), pick


def registration_split(n_frac, n_margin, reg_points):
    """fragment/samples.rs:601-615."""
    if reg_points == 0 or n_frac + n_margin <= reg_points:
        return n_frac, n_margin
    share = float(n_frac) * float(reg_points) / float(n_frac + n_margin)
    take_f = min(max(int(np.round(share)), 1), n_frac)
    return take_f, min(max(reg_points - take_f, 0), n_margin)


def random_rotation(rng, max_deg=None):
    """A rotation uniform over SO(3), or about a uniform axis by an angle uniform in [0, max]."""
    if max_deg is None:
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                         [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                         [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    axis = rng.normal(size=3)
    axis /= np.linalg.norm(axis)
    ang = np.radians(rng.uniform(0, max_deg))
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K


def rigid(R, tau):
    T = np.eye(4)
    T[:3, :3] = R
    T[:3, 3] = tau
    return T


@dataclass
class Fragment:
    """One fragment in its own frame, with every array the hot path reads."""
    name: str
    t: float
    res: float
    v: np.ndarray            # f32 (nv, 3)
    f: np.ndarray            # u32 (nf, 3)
    frac: np.ndarray         # u8 per face
    frac_area: float
    pf: np.ndarray
    pf_n: np.ndarray
    s: np.ndarray
    brk_p: np.ndarray
    brk_ns: np.ndarray
    margin_p: np.ndarray
    margin_n: np.ndarray
    reg_p: np.ndarray
    reg_n: np.ndarray
    pose: np.ndarray         # world -> fragment frame
    group: int = 0           # which wall it came from
    cell: int = 0
    neighbours: set = field(default_factory=set)

    @property
    def n_faces(self):
        return len(self.f)


def fragment_from_cell(rng, name, cm: CellMesh, t, frac_per_t2, frac_range, surface_points,
                       margin_points, reg_points, pose, group, cell) -> Fragment:
    v = cm.v.astype(np.float32).astype(np.float64)  # the mesh is f32, as RayScene is
    f = cm.f.astype(np.int64)
    fn, areas, _ = face_geometry(v, f)
    frac_faces = np.nonzero(cm.frac)[0]
    frac_area = float(areas[frac_faces].sum())
    n_pf = int(np.clip(round(frac_per_t2 * frac_area / (t * t)), *frac_range))
    pf, fp = sample_on_faces(rng, v, f, areas, frac_faces, n_pf)
    s, sp = sample_on_faces(rng, v, f, areas, np.arange(len(f)), surface_points)
    # The shell margin (R 3.5): shell-face samples between 0.15 t and 0.6 t from the
    # breakline, drawn from the shell faces near it so the band is fully populated.
    tree = cKDTree(cm.brk_p)
    _, _, cen = face_geometry(v, f)
    dc, _ = tree.query(cen)
    near = np.nonzero(cm.shell.astype(bool) & (dc <= 0.6 * t + 2 * cm.h))[0]
    margin_p = np.empty((0, 3))
    margin_n = np.empty((0, 3))
    if len(near):
        cand, cf = sample_on_faces(rng, v, f, areas, near, 3 * margin_points)
        d, _ = tree.query(cand)
        band = np.nonzero((d >= 0.15 * t) & (d <= 0.60 * t))[0][:margin_points]
        margin_p, margin_n = cand[band], fn[cf[band]]
    take_f, take_m = registration_split(len(pf), len(margin_p), reg_points)
    reg_p = np.concatenate([pf[:take_f], margin_p[:take_m]])
    reg_n = np.concatenate([fn[fp][:take_f], margin_n[:take_m]])
    R, tau = pose[:3, :3], pose[:3, 3]

    def mv(p):
        return p @ R.T + tau

    def rot(n):
        return n @ R.T

    edges = np.concatenate([v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 1]]])
    res = float(np.median(np.linalg.norm(edges, axis=1)))
    vf = mv(v).astype(np.float32)
    return Fragment(name=name, t=float(t), res=res, v=vf, f=cm.f, frac=cm.frac, frac_area=frac_area,
                    pf=mv(pf), pf_n=rot(fn[fp]), s=mv(s), brk_p=mv(cm.brk_p), brk_ns=rot(cm.brk_ns),
                    margin_p=mv(margin_p), margin_n=rot(margin_n), reg_p=mv(reg_p), reg_n=rot(reg_n),
                    pose=pose, group=group, cell=cell, neighbours={int(x) for x in cm.neighbours})


# ---------------------------------------------------------------------------------------------
# collections (the workloads)
# ---------------------------------------------------------------------------------------------


def _pot_seeds(rng, n, wall: PotWall):
    """n seed directions spread over the band of directions the wall covers."""
    top = np.arctan2(wall.height / 2, wall.r0)
    seeds = []
    tries = 0
    min_sep = np.sqrt(4.0 * np.pi * np.sin(top) / n) * 0.75
    while len(seeds) < n and tries < 100000:
        tries += 1
        z = rng.uniform(-np.sin(top) * 0.85, np.sin(top) * 0.85)
        th = rng.uniform(0, 2 * np.pi)
        d = np.array([np.sqrt(1 - z * z) * np.cos(th), np.sqrt(1 - z * z) * np.sin(th), z])
        if all(np.linalg.norm(d - s) > min_sep for s in seeds):
            seeds.append(d)
        elif tries % 2000 == 0:
            min_sep *= 0.9
    return np.array(seeds)


def _cell_centres(part, wall, n_cells, period):
    """A parameter point inside each cell: the label centroid on a coarse grid."""
    du = 1.0
    us = np.arange(0, period, du) if period else np.arange(0, wall.lu, du)
    vs = np.arange(0.5, wall.height if hasattr(wall, "height") else wall.lv, du)
    U, Vv = np.meshgrid(us, vs, indexing="ij")
    lab = part.label(U.ravel(), Vv.ravel())
    centres = []
    for c in range(n_cells):
        sel = lab == c
        if not sel.any():
            centres.append(None)
            continue
        u, v = U.ravel()[sel], Vv.ravel()[sel]
        if period:
            ang = u / period * 2 * np.pi
            mu = np.arctan2(np.sin(ang).mean(), np.cos(ang).mean()) % (2 * np.pi) * period / (2 * np.pi)
            u = (u - mu + period / 2) % period - period / 2 + mu
        cu, cv = u.mean(), v.mean()
        if part.label(np.array([cu]), np.array([cv]))[0] != c:
            k = np.argmin((u - cu) ** 2 + (v - cv) ** 2)
            cu, cv = u[k], v[k]
        centres.append(np.array([cu, cv]))
    return centres


@dataclass
class Pair:
    a: int
    b: int
    adjacent: bool
    truth: np.ndarray  # maps B's frame into A's frame


@dataclass
class Workload:
    name: str
    fragments: list
    pairs: list
    starts: list       # per pair: (n, 4, 4)
    seed: int

    @property
    def n_items(self):
        return int(sum(len(s) for s in self.starts))

    def describe(self):
        nf = [fr.n_faces for fr in self.fragments]
        npf = [len(fr.pf) for fr in self.fragments]
        return {"fragments": len(self.fragments), "pairs": len(self.pairs),
                "starts_per_pair": len(self.starts[0]) if self.starts else 0,
                "items": self.n_items, "faces_min": int(min(nf)), "faces_max": int(max(nf)),
                "faces_total": int(sum(nf)), "pf_min": int(min(npf)), "pf_max": int(max(npf)),
                "seed": self.seed}


def _scatter_pose(rng, extent=400.0):
    return rigid(random_rotation(rng), rng.uniform(-extent, extent, size=3))


def _pairs_and_starts(rng, frags, n_starts, all_pairs=True):
    pairs, starts = [], []
    n = len(frags)
    for i in range(n):
        for j in range(i + 1, n):
            A, B = frags[i], frags[j]
            adjacent = A.group == B.group and (B.cell in A.neighbours)
            if not all_pairs and not adjacent:
                continue
            truth = A.pose @ np.linalg.inv(B.pose)
            cA = A.pf.mean(0)
            cB = B.pf.mean(0)
            t_pair = min(A.t, B.t)
            inits = np.empty((n_starts, 4, 4))
            for k in range(n_starts):
                if adjacent:
                    inner = k < n_starts // 2
                    deg, dist = (5.0, 0.2 * t_pair) if inner else (30.0, 1.0 * t_pair)
                    R = random_rotation(rng, deg)
                    tau = rng.normal(size=3)
                    tau *= rng.uniform(0, dist) / np.linalg.norm(tau)
                    cB_in_A = truth[:3, :3] @ cB + truth[:3, 3]
                    D = rigid(R, cB_in_A - R @ cB_in_A + tau)
                    inits[k] = D @ truth
                else:
                    R = random_rotation(rng)
                    tau = cA - R @ cB + rng.normal(size=3) * 0.5 * t_pair
                    inits[k] = rigid(R, tau)
            pairs.append(Pair(i, j, adjacent, truth))
            starts.append(inits)
    return pairs, starts


def pot_collection(seed, walls, cells_per_wall, edges_per_t, n_starts, frac_per_t2=150.0,
                   frac_range=(5000, 12000), noise_amp=0.25, surface_points=20000,
                   margin_points=6000, reg_points=6000, all_pairs=True, name="pot"):
    """Fragments of pots broken by seeded spherical Voronoi partitions (the pot, collection,
    thin and scan workloads)."""
    rng = np.random.default_rng(seed)
    frags = []
    densities = frac_per_t2 if isinstance(frac_per_t2, tuple) else (frac_per_t2,) * len(walls)
    for g, (t, n_cells) in enumerate(zip(walls, cells_per_wall)):
        wall = PotWall(t)
        seeds = _pot_seeds(rng, n_cells, wall)
        part = SphereVoronoi(wall, seeds)
        noise = Field(rng, wavelength=4.0 * t)
        centres = _cell_centres(part, wall, len(seeds), wall.period)
        taper = lambda u, v, wall=wall: np.clip(np.minimum(v, wall.height - v) / (2 * wall.t), 0, 1)
        for c, centre in enumerate(centres):
            if centre is None:
                continue
            e = rng.uniform(*edges_per_t) if isinstance(edges_per_t, tuple) else edges_per_t
            cm = cell_mesh(wall, part, c, centre, t / e, noise, noise_amp * t, wall.height * 1.5,
                           taper)
            pose = _scatter_pose(rng)
            frags.append(fragment_from_cell(rng, f"{name}{g}_{c:02d}", cm, t, densities[g], frac_range,
                                            surface_points, margin_points, reg_points, pose, g, c))
    pairs, starts = _pairs_and_starts(rng, frags, n_starts, all_pairs)
    return Workload(name=name, fragments=frags, pairs=pairs, starts=starts, seed=seed)


def slab_collection(seed=0, t=10.0, edges_per_t=7.0, n_starts=16, noise_amp=0.3):
    """The slab pair: a 200 x 100 curved slab of wall t cut in two, B perturbed <= 30 deg,
    <= 2 t."""
    rng = np.random.default_rng(seed)
    wall = SlabWall(t)
    part = SlabCut(wall)
    noise = Field(rng, wavelength=4.0 * t, extra_sines=3)
    centres = [np.array([50.0, 50.0]), np.array([150.0, 50.0])]
    frags = []
    for c in range(2):
        cm = cell_mesh(wall, part, c, centres[c], t / edges_per_t, noise, noise_amp * t, 400.0, None)
        pose = np.eye(4) if c == 0 else rigid(random_rotation(rng, 30.0),
                                              rng.normal(size=3) / np.sqrt(3) * 2 * t * rng.uniform())
        frags.append(fragment_from_cell(rng, f"slab_{c}", cm, t, 150.0, (5000, 12000), 20000, 6000,
                                        6000, pose, 0, c))
    pairs, starts = _pairs_and_starts(rng, frags, n_starts, all_pairs=True)
    return Workload(name="slab", fragments=frags, pairs=pairs, starts=starts, seed=seed)


CONFIGS = {
    # The workloads: a slab pair; a pot (8 fragments, 28 pairs x 64 starts); a collection
    # (40 fragments of 3 pots, t = 5, 8, 12; 780 pairs x 128 starts; 1k-60k fracture points);
    # a thin pot (t = 2 at 4-6 edges per t, 6 fragments of about 1M faces, 500k surface
    # samples per fragment: 1M penetration samples per pair).
    # The ring meshing spends about twice the faces of an isotropic mesh at the same edge
    # length, so the edge lengths are set to land on each workload's face counts.
    "slab": lambda seed=0: slab_collection(seed, edges_per_t=7.0),
    "pot": lambda seed=0: pot_collection(seed, walls=(8.0,), cells_per_wall=(8,),
                                         edges_per_t=(5.5, 7.5), n_starts=64, name="pot"),
    "collection": lambda seed=0: pot_collection(
        seed, walls=(5.0, 8.0, 12.0), cells_per_wall=(14, 13, 13), edges_per_t=(6.5, 9.5),
        n_starts=128, frac_per_t2=(900.0, 300.0, 60.0), frac_range=(1000, 60000), name="coll"),
    "thin": lambda seed=0: pot_collection(seed, walls=(2.0,), cells_per_wall=(6,),
                                          edges_per_t=(4.0, 5.0), n_starts=128,
                                          surface_points=500_000, name="thin"),
    # R 9's input at full resolution: one pot of t = 24 in 8 fragments of 1.1M-2.2M faces (the
    # size of a 1.2M-face scan), 55k-90k fracture vertices each, 18 adjacent pairs.
    "scan": lambda seed=0: pot_collection(seed, walls=(24.0,), cells_per_wall=(8,),
                                          edges_per_t=(64.0, 66.0), n_starts=4, name="scan"),
}


def make(config: str, seed: int = 0) -> Workload:
    return CONFIGS[config](seed)
