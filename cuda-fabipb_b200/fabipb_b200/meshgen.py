"""Seeded synthetic surfaces and charge sets for the FABIPB hot path.

No public dataset is named for the reference's benchmarks, so every case is
generated here from a seed and written in the reference's own input formats
(MSMS ``.vert``/``.face`` + PQR, see ``meshio.py``):

* ``sphere``: icosphere of radius R (20*4^k flat triangles), outward normals
  = unit positions; charges uniform in a ball, q ~ N(0, s^2) shifted to a net
  charge.  The 20,480-triangle R=20 A sphere with 500 charges is the small
  Kirkwood case.
* ``star``: octahedral geodesic sphere of frequency f (8*f^2 triangles;
  f=160 gives 204,800), radially perturbed to r = R(1 + sum a_lm Y_lm),
  a_lm ~ N(0, 0.03^2), l = 2..6.  Charges uniform in the interior at least
  ``gap`` from the surface (radial test), q ~ N(0, 0.4^2) shifted to net -5.
* ``shell``: two closed geodesic spheres (inner radius Ri with faces and
  normals pointing into the cavity, outer radius Ro pointing outward), both
  perturbed by l <= 12 harmonics of relative amplitude 2%; charges uniform in
  the shell at least ``gap`` from both surfaces.

All faces are oriented counter-clockwise seen from the side the normal points
to, so that shared edges run in opposite directions in neighbouring faces (the
convention ``nrCommonVtx`` in ``src/numQuad.c:312-353`` relies on).
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
from scipy.special import sph_harm_y, spherical_kn, eval_legendre

from .meshio import ChargeSet, write_case


# ----------------------------------------------------------------------------
# base triangulations of the unit sphere
# ----------------------------------------------------------------------------

def _orient_outward(pos, faces):
    v = pos[faces]
    nrm = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
    ctr = v.mean(axis=1)
    flip = np.einsum("ij,ij->i", nrm, ctr) < 0
    faces = faces.copy()
    faces[flip] = faces[flip][:, [0, 2, 1]]
    return faces


def icosphere(nsub: int):
    """Unit icosphere with 20*4^nsub faces (midpoint subdivision)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    base = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
                     (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)],
                    dtype=np.float64)
    faces = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9),
                      (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2),
                      (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
                      (8, 6, 7), (9, 8, 1)], dtype=np.int64)
    verts = [v / np.linalg.norm(v) for v in base]
    for _ in range(nsub):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            j = cache.get(key)
            if j is None:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                j = cache[key] = len(verts) - 1
            return j

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = np.array(nf, dtype=np.int64)
    pos = np.array(verts)
    return pos, _orient_outward(pos, faces)


def octasphere(freq: int):
    """Unit octahedral geodesic sphere with 8*freq^2 faces.

    Points of each octahedron face are i*A + j*B + k*C (i+j+k = freq) with
    A,B,C signed unit axes, so integer coordinates identify shared vertices
    exactly before projection to the sphere.
    """
    axes = [np.array(a) for a in ((1, 0, 0), (0, 1, 0), (0, 0, 1))]
    key_to_idx = {}
    pts = []
    faces = []

    def vid(ic):
        k = (int(ic[0]), int(ic[1]), int(ic[2]))
        j = key_to_idx.get(k)
        if j is None:
            j = key_to_idx[k] = len(pts)
            pts.append(k)
        return j

    for sx in (1, -1):
        for sy in (1, -1):
            for sz in (1, -1):
                A, B, C = sx * axes[0], sy * axes[1], sz * axes[2]
                grid = {}
                for i in range(freq + 1):
                    for j in range(freq + 1 - i):
                        k = freq - i - j
                        grid[(i, j)] = vid(i * A + j * B + k * C)
                for i in range(freq):
                    for j in range(freq - i):
                        faces.append((grid[(i, j)], grid[(i + 1, j)], grid[(i, j + 1)]))
                        if i + j + 1 < freq:
                            faces.append((grid[(i + 1, j)], grid[(i + 1, j + 1)], grid[(i, j + 1)]))
    p = np.array(pts, dtype=np.float64)
    p /= np.linalg.norm(p, axis=1)[:, None]
    faces = np.array(faces, dtype=np.int64)
    return p, _orient_outward(p, faces)


# ----------------------------------------------------------------------------
# perturbations and normals
# ----------------------------------------------------------------------------

def real_sph_harm(l, m, theta, phi):
    """Real spherical harmonic Y_lm (theta polar, phi azimuth)."""
    if m == 0:
        return np.real(sph_harm_y(l, 0, theta, phi))
    y = sph_harm_y(l, abs(m), theta, phi)
    return np.sqrt(2.0) * ((-1) ** m) * (np.real(y) if m > 0 else np.imag(y))


def _harmonic_sum(coeffs, unit, chunk=32768):
    """1 + sum over coeffs (l, m, a) of a * Y_lm(unit), in the listed order.

    Each point's sum depends on that point alone, so the points are split into
    chunks summed on a thread pool (scipy's harmonics release the GIL); every
    chunk adds the terms in the same order, so the result does not depend on
    the split or the thread count.
    """
    n = unit.shape[0]

    def part(lo):
        u = unit[lo:lo + chunk]
        theta = np.arccos(np.clip(u[:, 2], -1.0, 1.0))
        phi = np.arctan2(u[:, 1], u[:, 0])
        f = np.ones(u.shape[0])
        for l, m, a in coeffs:
            f += a * real_sph_harm(l, m, theta, phi)
        return f

    starts = list(range(0, n, chunk))
    if len(starts) <= 1:
        return part(0) if n else np.ones(0)
    workers = min(len(starts), os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=workers) as ex:
        return np.concatenate(list(ex.map(part, starts)))


def radial_perturbation(unit, lmin, lmax, sigma, rng):
    """1 + sum_{l,m} a_lm Y_lm(unit) with a_lm ~ N(0, sigma^2)."""
    coeffs = []
    for l in range(lmin, lmax + 1):
        for m in range(-l, l + 1):
            coeffs.append((l, m, rng.normal(0.0, sigma)))
    return _harmonic_sum(coeffs, unit), coeffs


def eval_perturbation(coeffs, unit):
    return _harmonic_sum(coeffs, unit)


def vertex_normals(pos, faces):
    """Area-weighted average of incident face normals, normalised."""
    v = pos[faces]
    fn = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
    vn = np.zeros_like(pos)
    for k in range(3):
        np.add.at(vn, faces[:, k], fn)
    return vn / np.linalg.norm(vn, axis=1)[:, None]


def _charges(pos, rng, q_sigma, net, radius):
    q = rng.normal(0.0, q_sigma, pos.shape[0])
    q += (net - q.sum()) / pos.shape[0]
    if np.isscalar(radius):
        rad = np.full(pos.shape[0], float(radius))
    else:
        rad = radius
    return ChargeSet(pos, q, rad)


# ----------------------------------------------------------------------------
# the cases
# ----------------------------------------------------------------------------

def sphere_case(base, nsub=5, radius=20.0, n_charges=500, charge_radius=16.0,
                q_sigma=0.5, net=2.0, seed=0):
    """Kirkwood sphere: icosphere of ``radius`` with 20*4^nsub faces."""
    unit, faces = icosphere(nsub)
    pos = radius * unit
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n_charges, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    r = charge_radius * rng.random(n_charges) ** (1.0 / 3.0)
    ch = _charges(d * r[:, None], rng, q_sigma, net, 1.5)
    write_case(base, pos, unit, faces, ch)
    return {"kind": "sphere", "faces": int(len(faces)), "vertices": int(len(pos)),
            "charges": n_charges, "seed": seed, "radius": radius}


def star_case(base, freq=160, radius=25.0, n_charges=20000, gap=1.4, q_sigma=0.4,
              net=-5.0, seed=1):
    """Star-shaped globular surface on an octahedral geodesic (8*freq^2 faces)."""
    rng = np.random.default_rng(seed)
    unit, faces = octasphere(freq)
    f, coeffs = radial_perturbation(unit, 2, 6, 0.03, rng)
    pos = radius * f[:, None] * unit
    vn = vertex_normals(pos, faces)
    pts = []
    need = n_charges
    while need > 0:
        cand = rng.uniform(-1.0, 1.0, size=(4 * need, 3)) * radius * 1.5
        rr = np.linalg.norm(cand, axis=1)
        u = cand / np.maximum(rr, 1e-12)[:, None]
        rs = radius * eval_perturbation(coeffs, u)
        ok = rr <= rs - gap
        pts.append(cand[ok][:need])
        need -= int(min(ok.sum(), need))
    cpos = np.concatenate(pts)[:n_charges]
    rad = rng.uniform(1.2, 2.0, n_charges)
    ch = _charges(cpos, rng, q_sigma, net, rad)
    write_case(base, pos, vn, faces, ch)
    return {"kind": "star", "faces": int(len(faces)), "vertices": int(len(pos)),
            "charges": n_charges, "seed": seed, "radius": radius, "freq": freq}


def shell_case(base, freq=362, r_in=200.0, r_out=230.0, n_charges=500000, gap=1.4,
               q_sigma=0.4, net=0.0, amp=0.02, lmax=12, seed=2):
    """Spherical shell: inner surface faces the cavity, outer faces outward."""
    rng = np.random.default_rng(seed)
    unit, faces = octasphere(freq)
    sig = amp / np.sqrt((lmax + 1) ** 2)
    f_in, c_in = radial_perturbation(unit, 1, lmax, sig, rng)
    f_out, c_out = radial_perturbation(unit, 1, lmax, sig, rng)
    p_in = r_in * f_in[:, None] * unit
    p_out = r_out * f_out[:, None] * unit
    faces_in = faces[:, [0, 2, 1]]              # normals into the cavity
    n_in = vertex_normals(p_in, faces_in)
    n_out = vertex_normals(p_out, faces)
    nv = len(unit)
    pos = np.concatenate([p_in, p_out])
    vn = np.concatenate([n_in, n_out])
    allf = np.concatenate([faces_in, faces + nv])
    pts = []
    need = n_charges
    while need > 0:
        cand = rng.normal(size=(4 * need, 3))
        u = cand / np.linalg.norm(cand, axis=1)[:, None]
        rr = (rng.random(4 * need) * (r_out ** 3 - r_in ** 3) + r_in ** 3) ** (1.0 / 3.0)
        ri = r_in * eval_perturbation(c_in, u)
        ro = r_out * eval_perturbation(c_out, u)
        ok = (rr >= ri + gap) & (rr <= ro - gap)
        pts.append((u * rr[:, None])[ok][:need])
        need -= int(min(ok.sum(), need))
    cpos = np.concatenate(pts)[:n_charges]
    ch = _charges(cpos, rng, q_sigma, net, 1.5)
    write_case(base, pos, vn, allf, ch)
    return {"kind": "shell", "faces": int(len(allf)), "vertices": int(len(pos)),
            "charges": n_charges, "seed": seed, "r_in": r_in, "r_out": r_out, "freq": freq}


def kirkwood_energy(pos, q, a, eps_in, eps_out, kappa, lmax=60):
    """Analytic solvation energy (kcal/mol) of point charges in a dielectric sphere.

    Reaction-field series for a sphere of radius ``a`` with screening kappa
    outside: E = 1/2 * 332.0716/eps_in * sum_ij q_i q_j sum_n R_n
    (r_i r_j)^n / a^(2n+1) P_n(cos g_ij), R_n = (eps_out g_n + eps_in (n+1)) /
    (eps_in n - eps_out g_n), g_n = x k_n'(x)/k_n(x), x = kappa a.
    """
    r = np.linalg.norm(pos, axis=1)
    u = pos / r[:, None]
    cg = np.clip(u @ u.T, -1.0, 1.0)
    e = 0.0
    for n in range(lmax + 1):
        if kappa > 0:
            x = kappa * a
            g = x * spherical_kn(n, x, derivative=True) / spherical_kn(n, x)
        else:
            g = -(n + 1.0)
        rn = (eps_out * g + eps_in * (n + 1)) / (eps_in * n - eps_out * g)
        w = q * r ** n
        e += np.sum(np.outer(w, w) * eval_legendre(n, cg)) * rn / a ** (2 * n + 1)
    return 0.5 * e / eps_in * 332.0716


__all__ = ["icosphere", "octasphere", "sphere_case", "star_case", "shell_case",
           "kirkwood_energy", "vertex_normals"]
