"""Mesh and charge input for the FABIPB hot path.

Reads the MSMS-format ``.vert``/``.face`` pair and the PQR charge file the
reference solver consumes, and turns them into the panel arrays the CUDA
library takes.  Every step follows ``loadPanel`` in ``src/input.c`` so that the
panels (vertex coordinates, area, normal, and which faces survive the filter)
are bit-identical to the reference's:

* PQR: ATOM/HETATM records with at least 10 tokens; the last five are
  ``x y z q r`` (``input.c:38-95``).
* ``.vert``: two header lines, then ``nspt natm den prob``, then rows
  ``x y z nx ny nz ...`` (``input.c:547-613``).
* ``.face``: two header lines, then ``nface natm den prob``, then 1-based rows
  ``j1 j2 j3 ...`` (``input.c:615-677``).
* face filter: keep a face when its Heron area is >= 1e-5 and its centroid is
  not within squared distance 1e-5 of any of the previous 10 faces'
  centroids (``input.c:679-794``).
* panel normal: ``n0/2 + (n1+n2)/4`` normalised (``input.c:769-786``), or the
  geometric face normal aligned to it when ``FABIPB_PANEL_NORMAL=geometric``
  (``input.c:750-767``).
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np


@dataclass
class PanelSet:
    """Panels in input (mesh-face) order, as the reference's ``pnlOLst``."""

    vtx: np.ndarray      # (N, 3, 3) float64, vertex k of panel i is vtx[i, k]
    normal: np.ndarray   # (N, 3) float64 unit panel normals
    area: np.ndarray     # (N,) float64 Heron areas
    face_index: np.ndarray  # (N,) int32 index of the mesh face each panel came from

    @property
    def n(self) -> int:
        return int(self.area.shape[0])


@dataclass
class ChargeSet:
    pos: np.ndarray   # (M, 3) float64
    q: np.ndarray     # (M,) float64
    radius: np.ndarray  # (M,) float64


def read_pqr(path: str) -> ChargeSet:
    """Parse ATOM/HETATM records; the last five tokens are x y z q r."""
    pos, q, rad = [], [], []
    with open(path, "r") as fp:
        for line in fp:
            tok = line.split()
            if not tok or tok[0] not in ("ATOM", "HETATM"):
                continue
            if len(tok) < 10:
                continue
            try:
                x, y, z, c, r = (float(t) for t in tok[-5:])
            except ValueError:
                continue
            pos.append((x, y, z))
            q.append(c)
            rad.append(r)
    if not pos:
        raise ValueError(f"no ATOM/HETATM charge records parsed from {path}")
    return ChargeSet(np.asarray(pos, dtype=np.float64), np.asarray(q, dtype=np.float64),
                     np.asarray(rad, dtype=np.float64))


def _read_header_counts(fp, path):
    for _ in range(2):
        if not fp.readline():
            raise ValueError(f"{path} ended inside its 2-line header")
    parts = fp.readline().split()
    if len(parts) < 4:
        raise ValueError(f"malformed header in {path}")
    return int(parts[0])


def read_vert_face(base: str):
    """Return (positions (V,3), vertex normals (V,3), faces (F,3) 0-based)."""
    vpath, fpath = base + ".vert", base + ".face"
    with open(vpath, "r") as fp:
        nspt = _read_header_counts(fp, vpath)
        data = np.loadtxt(fp, dtype=np.float64, usecols=(0, 1, 2, 3, 4, 5), max_rows=nspt, ndmin=2)
    if data.shape[0] != nspt:
        raise ValueError(f"{vpath} truncated: {data.shape[0]} of {nspt} vertices")
    with open(fpath, "r") as fp:
        nface = _read_header_counts(fp, fpath)
        faces = np.loadtxt(fp, dtype=np.int64, usecols=(0, 1, 2), max_rows=nface, ndmin=2)
    if faces.shape[0] != nface:
        raise ValueError(f"{fpath} truncated: {faces.shape[0]} of {nface} faces")
    if faces.min() < 1 or faces.max() > nspt:
        raise ValueError(f"{fpath} references a vertex outside 1..{nspt}")
    return data[:, :3].copy(), data[:, 3:6].copy(), (faces - 1).astype(np.int64)


def _heron_area(v):
    """triangle_area() of input.c:114-127, same operation order."""
    a = v[:, 0] - v[:, 1]
    b = v[:, 0] - v[:, 2]
    c = v[:, 1] - v[:, 2]
    aa = np.sqrt((a[:, 0] * a[:, 0] + a[:, 1] * a[:, 1]) + a[:, 2] * a[:, 2])
    bb = np.sqrt((b[:, 0] * b[:, 0] + b[:, 1] * b[:, 1]) + b[:, 2] * b[:, 2])
    cc = np.sqrt((c[:, 0] * c[:, 0] + c[:, 1] * c[:, 1]) + c[:, 2] * c[:, 2])
    ss = 0.5 * ((aa + bb) + cc)
    with np.errstate(invalid="ignore"):
        return np.sqrt(((ss * (ss - aa)) * (ss - bb)) * (ss - cc))


def build_panels(pos, vnrm, faces, geometric_normals=None) -> PanelSet:
    """Apply the reference face filter and panel-normal rule to a mesh."""
    if geometric_normals is None:
        env = os.environ.get("FABIPB_PANEL_NORMAL", "")
        geometric_normals = env in ("geometric", "face")
    v = pos[faces]                      # (F,3,3)
    area = _heron_area(v)
    third = 1.0 / 3.0
    # centroid as xx[j] += 1/3*face[k][j] (input.c:694-699): left-to-right sum
    xx = ((0.0 + third * v[:, 0]) + third * v[:, 1]) + third * v[:, 2]
    nf = faces.shape[0]
    alert = np.zeros(nf, dtype=bool)
    for k in range(1, 11):          # face i against faces i-1 .. i-10
        if k >= nf:
            break
        d = xx[k:] - xx[:-k]
        dist = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        alert[k:] |= dist < 1.0e-5
    keep = (area >= 1.0e-5) & ~alert
    idx = np.nonzero(keep)[0]
    vk = v[idx]
    nv = vnrm[faces[idx]]
    nrm = nv[:, 0] / 2.0 + (nv[:, 1] + nv[:, 2]) / 4.0
    ln = np.sqrt((nrm[:, 0] * nrm[:, 0] + nrm[:, 1] * nrm[:, 1]) + nrm[:, 2] * nrm[:, 2])
    e1 = vk[:, 1] - vk[:, 0]
    e2 = vk[:, 2] - vk[:, 0]
    g = np.stack([e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1],
                  e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2],
                  e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]], axis=1)
    gl = np.sqrt((g[:, 0] * g[:, 0] + g[:, 1] * g[:, 1]) + g[:, 2] * g[:, 2])
    with np.errstate(invalid="ignore", divide="ignore"):
        if geometric_normals:
            vn = np.where(ln[:, None] > 0, nrm / ln[:, None], nrm)
            gn = np.where(gl[:, None] > 0, g / gl[:, None], vn)
            dot = (gn[:, 0] * vn[:, 0] + gn[:, 1] * vn[:, 1]) + gn[:, 2] * vn[:, 2]
            normal = np.where(dot[:, None] < 0, -gn, gn)
        else:
            geo = np.where(gl[:, None] > 0, g / gl[:, None], np.array([0.0, 0.0, 1.0]))
            normal = np.where(ln[:, None] > 0, nrm / ln[:, None], geo)
    return PanelSet(np.ascontiguousarray(vk), np.ascontiguousarray(normal),
                    np.ascontiguousarray(area[idx]), idx.astype(np.int32))


def load_case(base: str):
    """Read ``base.pqr``, ``base.vert``, ``base.face`` into (PanelSet, ChargeSet)."""
    charges = read_pqr(base + ".pqr")
    pos, vnrm, faces = read_vert_face(base)
    return build_panels(pos, vnrm, faces), charges


def write_case(base: str, pos, vnrm, faces, charges: ChargeSet) -> None:
    """Write an MSMS-format mesh (1-based faces) and a PQR file."""
    with open(base + ".vert", "w") as fp:
        fp.write("# synthetic surface\n# x y z nx ny nz\n%d 1 1.0 1.4\n" % len(pos))
        for p, n in zip(pos, vnrm):
            fp.write("%.9f %.9f %.9f %.9f %.9f %.9f 0 1 2\n" % (p[0], p[1], p[2], n[0], n[1], n[2]))
    with open(base + ".face", "w") as fp:
        fp.write("# synthetic surface\n# j1 j2 j3\n%d 1 1.0 1.4\n" % len(faces))
        for f in faces:
            fp.write("%d %d %d 1 1\n" % (f[0] + 1, f[1] + 1, f[2] + 1))
    with open(base + ".pqr", "w") as fp:
        for i, (p, c, r) in enumerate(zip(charges.pos, charges.q, charges.radius)):
            fp.write("ATOM %d C ALA A 1 %.4f %.4f %.4f %.4f %.4f\n" % (i + 1, p[0], p[1], p[2], c, r))


def centroid_tree_order(panels: PanelSet):
    """Panel centroid ``ONETHIRD*(v0+v1+v2)`` as loopPanels computes it (gkSetup.c:111-113)."""
    third = 0.33333333333333333333333333
    v = panels.vtx
    return third * ((v[:, 0] + v[:, 1]) + v[:, 2])


__all__ = ["PanelSet", "ChargeSet", "read_pqr", "read_vert_face", "build_panels",
           "load_case", "write_case", "centroid_tree_order"]

