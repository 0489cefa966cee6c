"""Half-sarcomere lattice: which filament faces which, once per size.

:meth:`SarcTopology.create` reproduces the reference builder
(``multifil_jax/core/sarc_geometry.py:379-645``) for both lattices:

* vertebrate: 1 thick : 2 thin, thin filaments at trigonal interstices with
  three faces, three heads per crown;
* invertebrate (insect flight muscle): 1 thick : 3 thin, thin filaments at the
  midpoints of thick-thick edges with two faces (sarc_geometry.py:915-1005),
  each thin filament's binding-site grid turned and shifted by its 3-fold
  registration class (:1134-1170, :1230-1262), optionally with the 3-class
  myosin superlattice of the thick filaments (:1118-1131) and any number of
  heads per crown (four in the insect presets, about half of them without a
  partner: ``xb_valid``);
* the legacy fixed crown-face table (:1357-1367, :1443-1447).

Every array it produces must be bit-identical to the reference's, so the
arithmetic below keeps the reference's float32/float64 dtype flow step by
step (numpy promotion rules included); the golden fixtures in
``tests/golden`` pin that.

Beyond the reference's arrays, :meth:`SarcTopology.device_arrays` derives the
compact layout the CUDA kernels read (per-XB target thin and face, per-face
candidate site lists, chain neighbours), see ``device_arrays``.
"""
from __future__ import annotations

from typing import List, Optional, Tuple

import numpy as np

from .params import StaticParams, DynamicParams

SQRT3 = np.float32(np.sqrt(3))
THICK_THIN_DISTANCE = np.float32(1.0 / np.sqrt(3))
# invertebrate: thin filaments half way along thick-thick edges, thick faces
# pointing along the edges (sarc_geometry.py:80, :101)
THICK_THIN_DISTANCE_INVERTEBRATE = np.float32(0.5)
THICK_FACE_ANGLES_INVERTEBRATE = np.array([0, 60, 120, 180, 240, 300], dtype=np.float32) * np.pi / 180
N_REGISTRATION_CLASSES = 3
# legacy crown levels 1..3 -> the three thick faces their heads use (sarc_geometry.py:1357)
LEGACY_FACE_TABLE = np.array([[0, 2, 4], [1, 3, 5], [0, 2, 4]])
# thin-face direction vectors, index = orientation code (sarc_geometry.py:88-95)
ORIENTATION_VECTORS = np.array([
    [0.866, -0.5], [0.0, -1.0], [-0.866, -0.5],
    [-0.866, 0.5], [0.0, 1.0], [0.866, 0.5]], dtype=np.float32)
# thick face k points at this angle (sarc_geometry.py:97)
THICK_FACE_ANGLES = np.array([150, 90, 30, 330, 270, 210], dtype=np.float32) * np.pi / 180
THIN_ORIENTATION_UPWARD = (4, 0, 2)
THIN_ORIENTATION_DOWNWARD = (3, 5, 1)


# --------------------------------------------------------------------------
# lattice placement (sarc_geometry.py:725-874)
# --------------------------------------------------------------------------

def _thick_positions(n_rows: int, n_cols: int) -> Tuple[np.ndarray, np.float32, np.float32]:
    a = np.float32(1.0)
    pts = []
    for row in range(n_rows):
        shift = np.float32(0.5) * a if row % 2 == 1 else np.float32(0.0)
        for col in range(n_cols):
            pts.append([col * a + shift, -row * SQRT3 / np.float32(2.0) * a])
    box_x = np.float32(n_cols) * a
    box_y = np.float32(n_rows) * SQRT3 / np.float32(2.0) * a
    return np.array(pts, dtype=np.float32), box_x, box_y


def _wrap_y(y, box_y):
    while y < -box_y / 2:
        y += box_y
    while y > box_y / 2:
        y -= box_y
    return np.float32(y)


def _wrap_x(x, box_x, tol=1e-6):
    x = x % box_x
    if abs(x - box_x) < tol or abs(x) < tol:
        x = 0.0
    return x


def _min_image_dist(p, q, box_x, box_y):
    dx = p[0] - q[0]
    dy = p[1] - q[1]
    dx = dx - box_x * np.round(dx / box_x)
    dy = dy - box_y * np.round(dy / box_y)
    return np.float32(np.sqrt(dx * dx + dy * dy))


def _face_point(thick_pos, face):
    ang = THICK_FACE_ANGLES[face]
    return (thick_pos[0] + THICK_THIN_DISTANCE * np.cos(ang),
            thick_pos[1] + THICK_THIN_DISTANCE * np.sin(ang))


def _thin_positions(thick_pos, box_x, box_y, periodic):
    """Thin filaments at trigonal interstices, ordered row by row (top first)."""
    tol = 0.05

    def key_of(face_xy):
        tx, ty = face_xy
        if periodic:
            tx = _wrap_x(tx, box_x)
            ty = _wrap_y(ty, box_y)
        return (round(tx / tol), round(ty / tol)), tx, ty

    # every interstice with the (thick, face) pairs that point at it
    spots = {}
    for t, p in enumerate(thick_pos):
        for f in range(6):
            k, tx, ty = key_of(_face_point(p, f))
            if k not in spots:
                spots[k] = [(np.float32(tx), np.float32(ty)), []]
            spots[k][1].append((t, f))

    rows = {}
    for t, p in enumerate(thick_pos):
        rows.setdefault(round(p[1] / 0.1), []).append((t, p))

    order = []
    seen = set()
    for rk in sorted(rows, reverse=True):
        in_row = sorted(rows[rk], key=lambda tp: tp[1][0])
        for faces in ((0, 1, 2), (5, 4, 3)):
            for _t, p in in_row:
                for f in faces:
                    k, _, _ = key_of(_face_point(p, f))
                    if k not in seen:
                        seen.add(k)
                        order.append(spots[k])

    positions, orientations = [], []
    for (tx, ty), faces in order:
        above = below = 0
        for t, _f in faces:
            ty_thick = thick_pos[t][1]
            if periodic:
                dy = ty_thick - ty
                dy = dy - box_y * np.round(dy / box_y)
                if dy > tol:
                    above += 1
                elif dy < -tol:
                    below += 1
            else:
                if ty_thick > ty + tol:
                    above += 1
                elif ty_thick < ty - tol:
                    below += 1
        positions.append([tx, ty])
        orientations.append(THIN_ORIENTATION_UPWARD if above <= below else THIN_ORIENTATION_DOWNWARD)
    return np.array(positions, dtype=np.float32), orientations


def _thin_positions_on_edges(thick_pos, box_x, box_y, periodic):
    """Invertebrate thin filaments at edge midpoints (sarc_geometry.py:915-1005).

    For every thick filament and each of its six neighbour directions with a
    thick filament one lattice unit away, one thin filament half way along
    the edge (each edge once); its two faces look back at the two thick
    filaments.  Returned sorted top row first, then by x, with the thick pair
    of every edge.
    """
    tol = 0.1
    dirs = np.array([0, 60, 120, 180, 240, 300], dtype=np.float32) * np.pi / 180
    face_dirs = np.array([np.arctan2(v[1], v[0]) for v in ORIENTATION_VECTORS])

    def nearest_code(a):
        d = np.abs(face_dirs - a)
        d = np.minimum(d, 2 * np.pi - d)
        return int(np.argmin(d))

    def thick_at(x, y):
        for idx, q in enumerate(thick_pos):
            if periodic:
                dx = x - q[0]
                dy = y - q[1]
                dx = dx - box_x * np.round(dx / box_x)
                dy = dy - box_y * np.round(dy / box_y)
                dist = np.sqrt(dx ** 2 + dy ** 2)
            else:
                dist = np.sqrt((x - q[0]) ** 2 + (y - q[1]) ** 2)
            if dist < tol:
                return idx
        return None

    edges, seen = [], set()
    for i, p in enumerate(thick_pos):
        for a in dirs:
            nx = p[0] + 1.0 * np.cos(a)
            ny = p[1] + 1.0 * np.sin(a)
            if periodic:
                nx = _wrap_x(nx, box_x)
                ny = _wrap_y(ny, box_y)
            j = thick_at(nx, ny)
            if j is None:
                continue
            mx = p[0] + 0.5 * 1.0 * np.cos(a)
            my = p[1] + 0.5 * 1.0 * np.sin(a)
            if periodic:
                mx = _wrap_x(mx, box_x)
                my = _wrap_y(my, box_y)
            k = (round(round(mx, 4) % box_x, 3), round(round(my, 4) % box_y, 3))
            if k in seen:
                continue
            seen.add(k)
            back = a + np.pi
            if back > np.pi:
                back -= 2 * np.pi
            oi, oj = nearest_code(back), nearest_code(a)
            if oi == oj:
                oj = (oi + 3) % 6
            edges.append((np.float32(mx), np.float32(my), (oi, oj), (i, j)))
    edges.sort(key=lambda e: (-e[1], e[0]))
    if not edges:
        return np.zeros((0, 2), dtype=np.float32), [], []
    return (np.array([[e[0], e[1]] for e in edges], dtype=np.float32), [e[2] for e in edges],
            [e[3] for e in edges])


def _edge_connectivity(thick_pos, thin_pos, pairs, box_x, box_y, periodic):
    """thick_to_thin / thin_to_thick of the edge lattice (sarc_geometry.py:1037-1055):
    thin face 0 faces the first thick filament of its edge, face 1 the second; on
    the thick side the face whose direction is closest to the thin filament."""
    n_thick, n_thin = len(thick_pos), len(thin_pos)
    t2n = [[None] * 6 for _ in range(n_thick)]
    n2t = [[None] * 2 for _ in range(n_thin)]
    for k in range(n_thin):
        q = thin_pos[k]
        for face, t in enumerate(pairs[k]):
            p = thick_pos[t]
            dx = q[0] - p[0]
            dy = q[1] - p[1]
            if periodic:
                dx = dx - box_x * np.round(dx / box_x)
                dy = dy - box_y * np.round(dy / box_y)
            ang = np.arctan2(dy, dx)
            best, best_d = 0, np.inf
            for f in range(6):
                d = abs((ang - THICK_FACE_ANGLES_INVERTEBRATE[f] + np.pi) % (2 * np.pi) - np.pi)
                if d < best_d:
                    best_d, best = d, f
            n2t[k][face] = (t, best)
            t2n[t][best] = (k, face)
    return t2n, n2t


def _registration_classes(thick_pos, pairs, box_x, box_y, periodic):
    """3-fold actin registration class of every edge thin filament: the edge's
    direction modulo 180 degrees in steps of 60 (sarc_geometry.py:1134-1170)."""
    cls = np.empty(len(pairs), dtype=np.int32)
    for k, (i, j) in enumerate(pairs):
        dx = thick_pos[j][0] - thick_pos[i][0]
        dy = thick_pos[j][1] - thick_pos[i][1]
        if periodic:
            dx = dx - box_x * np.round(dx / box_x)
            dy = dy - box_y * np.round(dy / box_y)
        deg = np.degrees(np.arctan2(dy, dx)) % 180.0
        cls[k] = int(np.round(deg / 60.0)) % N_REGISTRATION_CLASSES
    return cls


def _superlattice_classes(n_thick, ncols, n_classes):
    """Thick-filament class of the myosin superlattice: (q - r) mod n over the
    axial coordinates of the row-major grid (sarc_geometry.py:1118-1131)."""
    idx = np.arange(n_thick)
    row, col = idx // ncols, idx % ncols
    q = col - (row - (row & 1)) // 2
    return ((q - row) % n_classes).astype(np.int32)


def _thin_index_at(thin_pos, x, y, box_x, box_y, periodic, tol=0.01):
    for i, q in enumerate(thin_pos):
        d = (_min_image_dist([x, y], q, box_x, box_y) if periodic
             else np.sqrt((x - q[0]) ** 2 + (y - q[1]) ** 2))
        if d < tol:
            return i
    return None


def _facing_thin_face(thick_p, thin_p, orient, box_x, box_y, periodic):
    dx = thick_p[0] - thin_p[0]
    dy = thick_p[1] - thin_p[1]
    if periodic:
        dx = dx - box_x * np.round(dx / box_x)
        dy = dy - box_y * np.round(dy / box_y)
    target = np.arctan2(dy, dx)
    best, best_diff = 0, np.inf
    for face, code in enumerate(orient):
        v = ORIENTATION_VECTORS[code]
        diff = abs(target - np.arctan2(v[1], v[0]))
        if diff > np.pi:
            diff = 2 * np.pi - diff
        if diff < best_diff:
            best_diff, best = diff, face
    return best


def _connectivity(thick_pos, thin_pos, orients, box_x, box_y, periodic):
    """thick_to_thin[t][f] = (thin, thin_face) or None (sarc_geometry.py:1008-1082)."""
    n_thick, n_thin = len(thick_pos), len(thin_pos)
    t2n = [[None] * 6 for _ in range(n_thick)]
    n2t = [[None] * 3 for _ in range(n_thin)]
    for t in range(n_thick):
        p = thick_pos[t]
        for f in range(6):
            ex, ey = _face_point(p, f)
            if periodic:
                ex = ex % box_x
                ey = _wrap_y(ey, box_y)
            i = _thin_index_at(thin_pos, ex, ey, box_x, box_y, periodic, tol=0.1)
            if i is None:
                continue
            face = _facing_thin_face(p, thin_pos[i], orients[i], box_x, box_y, periodic)
            t2n[t][f] = (i, face)
            n2t[i][face] = (t, f)
    return t2n, n2t


# --------------------------------------------------------------------------
# axial offsets (sarc_geometry.py:1087-1367)
# --------------------------------------------------------------------------

def f32_linspace(lo: float, hi: float, num: int) -> np.ndarray:
    """float32 ``linspace`` computed the way ``jax.numpy.linspace`` does it.

    The reference bakes its bin edges with ``jnp.linspace(..., dtype=float32)``
    (``sarc_geometry.py:598-603``), which evaluates ``lo*(1-t) + hi*t`` with
    ``t = i/div`` entirely in float32 and appends ``hi`` -- not numpy's
    float64 ``lo + i*delta``.  The two differ by an ulp at some edges, and an
    edge ulp changes which bin a head lands in.
    """
    div = num - 1
    t = (np.arange(div, dtype=np.float32) / np.float32(div)).astype(np.float32)
    out = np.float32(lo) * (np.float32(1) - t) + np.float32(hi) * t
    return np.concatenate([out.astype(np.float32), np.array([hi], dtype=np.float32)])


def _spread_step(nv):
    target = max(1, round(nv / 1.6180339887))
    for d in range(nv):
        for s in (target - d, target + d):
            if 1 <= s < nv and np.gcd(s, nv) == 1:
                return s
    return 1


def _spread_starts(n, low, high):
    """Low-discrepancy deterministic starts on [low, high) (sarc_geometry.py:1102-1107)."""
    nv = high - low
    return (low + (np.arange(n) * _spread_step(nv)) % nv).astype(np.int32)


def _crown_offsets(n_crowns, bare_zone, spacing):
    bare_zone = np.asarray(bare_zone, dtype=np.float32)
    spacing = np.float32(spacing)
    offs = bare_zone[:, None] + np.arange(n_crowns, dtype=np.float32)[None, :] * spacing
    rests = np.full((bare_zone.shape[0], n_crowns), spacing, dtype=np.float32)
    rests[:, 0] = bare_zone
    return offs, rests


def _binding_sites(orients, thin_starts, n_thin, n_polymers, half_pitch, mono_per_poly,
                   base_turns, wiggle, reg_class=None):
    """Actin-helix binding sites per thin filament, sorted M-line-far first.

    Same monomer grid, azimuth test, site ordering, chain parity and chain
    neighbour rules as sarc_geometry.py:1194-1352.  A thin filament of
    registration class c has its helix start advanced by
    c * round(mono_per_poly / 3) monomers and its grid shifted by
    c * half_pitch / 3 towards the Z-line (class 0, every vertebrate filament:
    no change).
    """
    if reg_class is None:
        reg_class = np.zeros(n_thin, dtype=np.int32)
    ang_step = int(round(mono_per_poly / N_REGISTRATION_CLASSES))
    ax_step = np.float32(half_pitch / N_REGISTRATION_CLASSES)
    base_len = np.float32(2 * half_pitch)
    base_turns = np.float32(base_turns)
    rev = np.float32(2 * np.pi)
    pitch = base_turns * rev / mono_per_poly
    rise = base_len / mono_per_poly
    n_mono = mono_per_poly * n_polymers
    mono_off = (n_mono - np.arange(n_mono, dtype=np.float32)) * rise
    face_vecs = np.array([(0.866, -0.5), (0, -1.0), (-0.866, -0.5),
                          (-0.866, 0.5), (0, 1.0), (0.866, 0.5)], dtype=np.float32)
    out = dict(offsets=[], rests=[], faces=[], chains=[], prev=[], next=[])
    for i in range(n_thin):
        c = int(reg_class[i])
        start = thin_starts[i] + c * ang_step
        grid = mono_off + c * ax_step
        ang = np.array([((m + start + 1) % mono_per_poly) * pitch % rev for m in range(n_mono)],
                       dtype=np.float32)
        fv = face_vecs[list(orients[i])]
        fang = np.arctan2(fv[:, 1], fv[:, 0])
        fang = np.where(fang < 0, fang + rev, fang)
        w = np.float32(wiggle)
        hits = [np.where(np.abs(ang - a) < w)[0] for a in fang]
        by_face = [grid[h] for h in hits]
        if by_face and any(len(f) > 0 for f in by_face):
            flat = np.sort(np.hstack(by_face))[::-1]
        else:
            flat = grid[::-1]
        chain = []
        for o in flat:
            m = np.where(np.abs(grid - o) < 1e-6)[0]
            chain.append((m[0] if len(m) else 0) % 2)
        chain = np.array(chain, dtype=np.int32)
        n = len(flat)
        prv = np.arange(n, dtype=np.int32)
        nxt = np.arange(n, dtype=np.int32)
        for c in (0, 1):
            idx = np.where(chain == c)[0]
            prv[idx[1:]] = idx[:-1]
            nxt[idx[:-1]] = idx[1:]
        face_sites = []
        for f_off in by_face:
            s = []
            for o in f_off:
                j = np.where(np.abs(flat - o) < 1e-6)[0]
                if len(j):
                    s.append(j[0])
            face_sites.append(np.array(s, dtype=np.int32))
        if n > 1:
            r = np.append(flat[:-1] - flat[1:], flat[-1])
        else:
            r = np.array([flat[0] if n else rise], dtype=np.float32)
        out['offsets'].append(flat.astype(np.float32))
        out['rests'].append(r.astype(np.float32))
        out['faces'].append(face_sites)
        out['chains'].append(chain)
        out['prev'].append(prv)
        out['next'].append(nxt)
    return out


def _xb_maps(t2n, face_sites, n_per_face, thick_starts, n_thick, n_crowns, width,
             n_xb, rot_deg, wiggle_deg, legacy=False):
    """Fixed-width crossbridge -> candidate-site maps (sarc_geometry.py:1370-1492):
    a head's thick face from its azimuth (accepted within ``wiggle_deg`` of a
    hexagonal direction, else no partner), or from the legacy crown-level table."""
    total = n_thick * n_crowns * n_xb
    thin_id = np.zeros(total, dtype=np.int32)
    thin_face = np.zeros(total, dtype=np.int32)
    sites = np.zeros((total, width), dtype=np.int32)
    valid = np.ones(total, dtype=bool)
    for x in range(total):
        t = x // (n_crowns * n_xb)
        local = x % (n_crowns * n_xb)
        crown, k = local // n_xb, local % n_xb
        if legacy:
            face = LEGACY_FACE_TABLE[(crown + thick_starts[t] - 1) % 3, k]
            hit = True
        else:
            eff = crown + (thick_starts[t] - 1)
            az = (k * (360.0 / n_xb) + eff * rot_deg) % 360.0
            face = int(round(az / 60.0)) % 6
            res = abs(az - face * 60.0)
            res = min(res, 360.0 - res)
            hit = res < wiggle_deg
        if hit:
            ti, tf = t2n[t, face, 0], t2n[t, face, 1]
        else:
            ti, tf = -1, 0
        valid[x] = ti >= 0
        if ti < 0:
            ti, tf = 0, 0
        thin_id[x], thin_face[x] = ti, tf
        nv = n_per_face[ti, tf]
        row = face_sites[ti, tf, :]
        first = row[0] if nv > 0 else 0
        sites[x] = np.where(np.arange(width) < nv, row, first)
    return thin_id, thin_face, sites, valid


class SarcTopology:
    """Immutable lattice description shared by every condition of one size.

    Field names, shapes and dtypes follow the reference class
    (``core/sarc_geometry.py:112-176``).
    """

    INT_FIELDS = ('n_thick', 'n_crowns', 'n_thin', 'n_sites', 'n_titin', 'n_xb_per_crown',
                  'n_faces_per_thin', 'max_sites_per_face', 'total_xbs', 'n_xb_bins')
    ARRAY_FIELDS = ('xb_to_thin_id', 'xb_to_thin_face', 'xb_to_site_indices', 'xb_valid',
                    'thick_to_thin', 'thin_to_thick', 'face_to_sites', 'n_sites_per_face',
                    'titin_connections', 'crown_offsets', 'crown_rests', 'binding_offsets',
                    'binding_rests', 'tm_chains', 'thick_starts', 'thin_starts', 'eye_4', 'eye_6',
                    'xb_bin_edges', 'xb_bin_centers', 'tm_prev_neighbor', 'tm_next_neighbor')

    def __init__(self, **fields):
        for k in self.INT_FIELDS:
            setattr(self, k, int(fields.pop(k)))
        for k in self.ARRAY_FIELDS:
            setattr(self, k, np.asarray(fields.pop(k)))
        self.nrows = fields.pop('nrows', None)
        self.ncols = fields.pop('ncols', None)
        if fields:
            raise TypeError(f"unexpected fields {sorted(fields)}")
        self._device_cache = None

    # ------------------------------------------------------------------
    @classmethod
    def create(cls, nrows: int, ncols: int, static_params: Optional[StaticParams] = None,
               dynamic_params: Optional[DynamicParams] = None, periodic: bool = True,
               lattice_spacing: float = 14.0, thin_starts: Optional[List[int]] = None,
               thick_starts: Optional[List[int]] = None) -> 'SarcTopology':
        """Build the lattice on the CPU (reference ``sarc_geometry.py:379-645``)."""
        sp = static_params if static_params is not None else StaticParams()
        if nrows < 1 or ncols < 1:
            raise ValueError("nrows and ncols must be >= 1")
        vert = sp.actin_geometry == 'vertebrate'
        n_faces = 3 if vert else 2
        n_xb = sp.n_xb_per_crown
        thick_pos, box_x, box_y = _thick_positions(nrows, ncols)
        n_thick = len(thick_pos)
        if thick_starts is None:
            ts = _spread_starts(n_thick, 1, n_xb + 1)
        else:
            if len(thick_starts) != n_thick:
                raise ValueError(f"thick_starts must have length n_thick={n_thick}, got {len(thick_starts)}")
            ts = np.array(thick_starts, dtype=np.int32)
        if vert:
            thin_pos, orients = _thin_positions(thick_pos, box_x, box_y, periodic)
            pairs, reg = None, None
        else:
            thin_pos, orients, pairs = _thin_positions_on_edges(thick_pos, box_x, box_y, periodic)
            reg = _registration_classes(thick_pos, pairs, box_x, box_y, periodic)
        n_thin = len(thin_pos)
        if thin_starts is None:
            # invertebrate: the registration class is the only phase variation
            tn = _spread_starts(n_thin, 0, 26) if vert else np.zeros(n_thin, dtype=np.int32)
        else:
            if len(thin_starts) != n_thin:
                raise ValueError(f"thin_starts must have length n_thin={n_thin}, got {len(thin_starts)}")
            tn = np.array(thin_starts, dtype=np.int32)

        if vert:
            t2n_list, n2t_list = _connectivity(thick_pos, thin_pos, orients, box_x, box_y, periodic)
        else:
            t2n_list, n2t_list = _edge_connectivity(thick_pos, thin_pos, pairs, box_x, box_y, periodic)
        t2n = np.full((n_thick, 6, 2), -1, dtype=np.int32)
        for t, faces in enumerate(t2n_list):
            for f, c in enumerate(faces):
                if c is not None:
                    t2n[t, f] = [c[0], c[1]]
        n2t = np.full((n_thin, n_faces, 2), -1, dtype=np.int32)
        for i, faces in enumerate(n2t_list):
            for f, c in enumerate(faces):
                if c is not None:
                    n2t[i, f] = [c[0], c[1]]
        if periodic:
            missing = np.argwhere(t2n[:, :, 0] < 0)
            if len(missing):
                raise ValueError(f"thick_to_thin has {len(missing)} unconnected (thick, face) pair(s) "
                                 f"under periodic=True for nrows={nrows}, ncols={ncols}, "
                                 f"actin_geometry='{sp.actin_geometry}'; the invertebrate lattice needs "
                                 f"an even nrows")
        if periodic and sp.n_superlattice_classes == 3 and (nrows % 2 != 0 or ncols % 3 != 0):
            raise ValueError(f"n_superlattice_classes=3 requires nrows even and ncols a multiple of 3 "
                             f"under periodic=True (got nrows={nrows}, ncols={ncols})")
        titin = [(t, f, c[0], c[1]) for t in range(n_thick) for f in range(6)
                 if (c := t2n_list[t][f]) is not None]
        titin_arr = (np.array(titin, dtype=np.int32) if titin else np.zeros((0, 4), dtype=np.int32))

        sl = _superlattice_classes(n_thick, ncols, sp.n_superlattice_classes)
        bare = (sp.thick_bare_zone + sl.astype(np.float32) * (sp.thick_crown_spacing / sp.n_superlattice_classes))
        crown_off, crown_rests = _crown_offsets(sp.n_crowns, bare, sp.thick_crown_spacing)

        bs = _binding_sites(orients, tn, n_thin, sp.n_polymers_per_thin, sp.actin_half_pitch,
                            sp.mono_per_poly, sp.polymer_base_turns, sp.target_zone_wiggle, reg)
        max_sites = max(len(o) for o in bs['offsets'])
        b_off = np.zeros((n_thin, max_sites), dtype=np.float32)
        b_rest = np.full((n_thin, max_sites), 2.77, dtype=np.float32)
        chains = np.zeros((n_thin, max_sites), dtype=np.int32)
        prv = np.tile(np.arange(max_sites, dtype=np.int32), (n_thin, 1))
        nxt = np.tile(np.arange(max_sites, dtype=np.int32), (n_thin, 1))
        for i in range(n_thin):
            n = len(bs['offsets'][i])
            b_off[i, :n] = bs['offsets'][i]
            b_rest[i, :n] = bs['rests'][i]
            chains[i, :n] = bs['chains'][i]
            prv[i, :n] = bs['prev'][i]
            nxt[i, :n] = bs['next'][i]
        width = max((len(s) for faces in bs['faces'] for s in faces), default=0)
        f2s = np.full((n_thin, n_faces, width), -1, dtype=np.int32)
        npf = np.zeros((n_thin, n_faces), dtype=np.int32)
        for i in range(n_thin):
            for j, s in enumerate(bs['faces'][i]):
                f2s[i, j, :len(s)] = s
                npf[i, j] = len(s)

        thin_id, thin_face, sites, valid = _xb_maps(
            t2n, f2s, npf, ts, n_thick, sp.n_crowns, width, n_xb,
            sp.crown_rotation_deg, sp.crown_face_wiggle_deg, sp.legacy_crown_geometry)

        edges = f32_linspace(sp.xb_bin_lo, sp.xb_bin_hi, sp.n_xb_bins + 1)
        centers = (np.float32(0.5) * (edges[:-1] + edges[1:])).astype(np.float32)

        return cls(
            n_thick=n_thick, n_crowns=sp.n_crowns, n_thin=n_thin, n_sites=max_sites,
            n_titin=len(titin_arr), n_xb_per_crown=n_xb, n_faces_per_thin=n_faces,
            max_sites_per_face=width, total_xbs=n_thick * sp.n_crowns * n_xb,
            n_xb_bins=sp.n_xb_bins,
            xb_to_thin_id=thin_id, xb_to_thin_face=thin_face, xb_to_site_indices=sites,
            xb_valid=valid, thick_to_thin=t2n, thin_to_thick=n2t, face_to_sites=f2s,
            n_sites_per_face=npf, titin_connections=titin_arr, crown_offsets=crown_off,
            crown_rests=crown_rests, binding_offsets=b_off, binding_rests=b_rest,
            tm_chains=chains, thick_starts=ts, thin_starts=tn,
            eye_4=np.eye(4, dtype=np.float32), eye_6=np.eye(6, dtype=np.float32),
            xb_bin_edges=edges, xb_bin_centers=centers,
            tm_prev_neighbor=prv, tm_next_neighbor=nxt, nrows=nrows, ncols=ncols)

    # ------------------------------------------------------------------
    @property
    def n_dof(self) -> int:
        return self.n_thick * self.n_crowns + self.n_thin * self.n_sites

    @property
    def n_sites_total(self) -> int:
        return self.n_thin * self.n_sites

    def valid_xb_targets(self):
        """(xb_index, thin_id, thin_face) of heads that have a real partner."""
        idx = np.where(self.xb_valid)[0]
        return idx, self.xb_to_thin_id[idx], self.xb_to_thin_face[idx]

    def size_key(self) -> tuple:
        """Identity of the lattice for caching device copies (computed once: the
        lattice is immutable, and the key holds two array byte strings)."""
        key = self.__dict__.get('_size_key')
        if key is None:
            key = (self.n_thick, self.n_crowns, self.n_thin, self.n_sites, self.total_xbs,
                   self.max_sites_per_face, self.nrows, self.ncols,
                   self.binding_offsets.tobytes(), self.xb_to_site_indices.tobytes())
            self.__dict__['_size_key'] = key
        return key

    def __repr__(self) -> str:
        return (f"SarcTopology(n_thick={self.n_thick}, n_crowns={self.n_crowns}, "
                f"n_thin={self.n_thin}, n_sites={self.n_sites}, "
                f"total_xbs={self.total_xbs}, n_titin={self.n_titin})")


__all__ = ['SarcTopology']


def jax_cumsum_rows(a: np.ndarray) -> np.ndarray:
    """Row-wise prefix sum in the association order of ``jnp.cumsum``.

    ``jnp.cumsum`` lowers to ``lax.associative_scan`` on CPU and GPU, whose
    odd/even recursion adds in a different order than a running sum; the
    reference's thin-filament rest positions (``metrics_fn.py:256``) are that
    scan of ``binding_rests``.  float32 in, float32 out.
    """
    def rec(e):
        n = e.shape[1]
        if n < 2:
            return e
        odd = rec((e[:, 0:-1:2] + e[:, 1::2]).astype(np.float32))
        if n % 2 == 0:
            even = (odd[:, :-1] + e[:, 2::2]).astype(np.float32)
        else:
            even = (odd + e[:, 2::2]).astype(np.float32)
        even = np.concatenate([e[:, 0:1], even], axis=1)
        out = np.empty((e.shape[0], even.shape[1] + odd.shape[1]), dtype=np.float32)
        out[:, 0::2] = even
        out[:, 1::2] = odd
        return out
    return rec(np.asarray(a, dtype=np.float32))


def thin_rest_cumsum(topo: 'SarcTopology') -> np.ndarray:
    """cumsum(binding_rests, axis=1) in the reference's float32 association."""
    return jax_cumsum_rows(topo.binding_rests)
