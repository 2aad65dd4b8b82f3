"""Surface and molecule inputs of the solve path.

* ``read_pqr``    -- readin.f90:29-86 (atoms read as REAL*4).
* ``read_msms`` / ``write_msms`` -- the .vert/.face layout of readin.f90:204-246.
* ``face_filter`` -- readin.f90:264-333 (surface_area): drops faces of area
  below 1e-5 and faces whose centroid repeats one of the 10 faces before it.
* ``icosphere``   -- the Born-ion triangulation (icosahedron subdivided ``level``
  times: level 4 gives 5,120 faces / 2,562 vertices, exact unit normals).
* ``synthetic_molecule`` -- seeded globular molecules (uniform in a sphere,
  random sequential addition with a minimum separation, radii U(r0, r1),
  charges N(0, sigma) shifted to an integer net charge).
* ``gaussian_surface`` -- the project's MSMS-format surface generator
  (surfgen/surfgen.c), a Gaussian level set meshed by surface nets.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_SG_DIR = os.path.join(_PKG, "surfgen")
_SG_LIB = os.path.join(_SG_DIR, "_build", "libtabi_surfgen.so")
_sg = None


def read_pqr(path):
    """readin.f90:29-86: skip REMARK lines, read 'c1..c5 x y z q r' per line
    (list-directed), stop at END; values rounded through REAL*4.
    Returns (xyz (M,3) float64, charge (M,), radius (M,))."""
    xyz, q, r = [], [], []
    with open(path) as f:
        lines = f.readlines()
    i = 0
    while i < len(lines) and lines[i].split() and lines[i].split()[0][:6] == "REMARK":
        i += 1
    for line in lines[i:]:
        tok = line.split()
        if not tok:
            continue
        if tok[0][:3] in ("END", "TER"):
            if tok[0][:3] == "END":
                break
            continue
        if len(tok) < 10:
            continue
        v = np.array([float(t) for t in tok[5:10]], dtype=np.float32).astype(np.float64)
        xyz.append(v[:3])
        q.append(v[3])
        r.append(v[4])
    return np.array(xyz).reshape(-1, 3), np.array(q), np.array(r)


def write_pqr(path, xyz, q, r):
    with open(path, "w") as f:
        for i, (p, qq, rr) in enumerate(zip(xyz, q, r)):
            f.write("ATOM  %5d  C   MOL     1    %8.3f%8.3f%8.3f %7.4f %6.4f\n"
                    % (i + 1, p[0], p[1], p[2], qq, rr))
        f.write("END\n")


def write_xyzr(path, xyz, r):
    with open(path, "w") as f:
        for p, rr in zip(xyz, r):
            f.write("%.6f %.6f %.6f %.6f\n" % (p[0], p[1], p[2], rr))


def read_msms(prefix):
    """readin.f90:204-246: returns (sptpos (V,3), sptnrm (V,3), nvert (F,3) 1-based)."""
    with open(prefix + ".vert") as f:
        f.readline()
        f.readline()
        nspt = int(f.readline().split()[0])
        v = np.loadtxt(f, usecols=(0, 1, 2, 3, 4, 5), max_rows=nspt, ndmin=2)
    with open(prefix + ".face") as f:
        f.readline()
        f.readline()
        nface = int(f.readline().split()[0])
        fc = np.loadtxt(f, usecols=(0, 1, 2), max_rows=nface, dtype=np.int64, ndmin=2)
    return v[:, :3].copy(), v[:, 3:6].copy(), fc.astype(np.int32)


def write_msms(prefix, sptpos, sptnrm, nvert, natm=1, density=1.0, probe=1.4, fmt="%9.3f"):
    """MSMS layout; fmt '%9.3f' is MSMS's own precision, a wider format may be
    given since the reference reads list-directed."""
    sptpos = np.asarray(sptpos, np.float64)
    sptnrm = np.asarray(sptnrm, np.float64)
    nvert = np.asarray(nvert)
    row = " ".join([fmt] * 6) + " %7d %7d %2d\n"
    with open(prefix + ".vert", "w") as f:
        f.write("# MSMS solvent excluded surface vertices\n#vertex #sphere density probe_r\n")
        f.write("%7d %7d %6.2f %4.2f\n" % (len(sptpos), natm, density, probe))
        for p, n in zip(sptpos, sptnrm):
            f.write(row % (p[0], p[1], p[2], n[0], n[1], n[2], 0, 1, 1))
    with open(prefix + ".face", "w") as f:
        f.write("# MSMS solvent excluded surface faces\n#faces  #sphere density probe_r\n")
        f.write("%7d %7d %6.2f %4.2f\n" % (len(nvert), natm, density, probe))
        for t in nvert:
            f.write("%6d %6d %6d %2d %6d\n" % (t[0], t[1], t[2], 1, 1))


def icosphere(level=4, radius=2.0, center=(0.0, 0.0, 0.0)):
    """Icosahedron subdivided ``level`` times and projected to the sphere.
    Returns (sptpos, sptnrm, nvert 1-based); 20*4**level faces."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
         (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, float) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    nrm = np.array(verts)
    pos = nrm * radius + np.asarray(center, float)
    return pos, nrm.copy(), np.array(faces, dtype=np.int32) + 1


def synthetic_molecule(natm, radius, min_sep=2.0, rad_range=(1.5, 2.0), q_sigma=0.4, seed=0,
                       max_tries=200000):
    """Seeded globule: random sequential addition of ``natm`` atoms uniform in a
    sphere of ``radius`` with pairwise distance >= min_sep; radii U(rad_range);
    charges N(0, q_sigma) shifted to zero mean, then the total rounded to an
    integer with the remainder spread evenly.  Returns (xyz, q, r)."""
    rng = np.random.default_rng(seed)
    pts = np.zeros((natm, 3))
    # candidates are drawn in batches from a copy of the generator and the
    # placement (surfgen.c sg_rsa) runs over them in order; the generator then
    # advances by exactly the candidates consumed, so the stream -- and with it
    # the molecule, radii and charges -- is the one of drawing one candidate
    # (3 uniforms) at a time
    L = _sglib()
    placed = C.c_int(0)
    limit = max_tries * max(1, natm // 100)
    tries = 0
    batch = max(4096, 64 * natm)
    while placed.value < natm:
        if tries >= limit:
            raise RuntimeError(f"placed only {placed.value} of {natm} atoms at min_sep {min_sep}")
        tmp = np.random.Generator(np.random.PCG64())
        tmp.bit_generator.state = rng.bit_generator.state
        nb = min(batch, limit - tries)
        cand = np.ascontiguousarray(tmp.uniform(-radius, radius, (nb, 3)))
        used = L.sg_rsa(natm, float(radius), float(min_sep), cand.ctypes.data, nb, pts.ctypes.data,
                        C.byref(placed))
        if used < 0:
            raise RuntimeError("sg_rsa failed")
        rng.bit_generator.advance(3 * used)
        tries += used
    r = rng.uniform(rad_range[0], rad_range[1], natm)
    q = rng.normal(0.0, q_sigma, natm)
    q -= q.mean()
    net = np.round(q.sum() + rng.normal(0.0, 1.0))
    q += (net - q.sum()) / natm
    return pts, q, r


def _sglib():
    global _sg
    if _sg is None:
        src = [os.path.join(_SG_DIR, f) for f in ("surfgen.c", "surfgen.h")]
        if not os.path.exists(_SG_LIB) or os.path.getmtime(_SG_LIB) < max(map(os.path.getmtime, src)):
            build_surfgen()
        L = C.CDLL(_SG_LIB)
        L.sg_gaussian_surface.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                          C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_int),
                                          C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.c_int),
                                          C.POINTER(C.c_double)]
        L.sg_gaussian_surface.restype = C.c_int
        L.sg_free.argtypes = [C.c_void_p]
        L.sg_rsa.argtypes = [C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_int, C.c_void_p,
                             C.POINTER(C.c_int)]
        L.sg_rsa.restype = C.c_int
        _sg = L
    return _sg


def build_surfgen():
    out = os.path.join(_SG_DIR, "_build")
    os.makedirs(out, exist_ok=True)
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-O2", "-fPIC", "-shared", "-o", _SG_LIB,
                    os.path.join(_SG_DIR, "surfgen.c"), "-lm"], check=True)
    subprocess.run([cc, "-O2", "-o", os.path.join(out, "tabi_msms"),
                    os.path.join(_SG_DIR, "tabi_msms.c"), os.path.join(_SG_DIR, "surfgen.c"),
                    "-lm"], check=True)


def gaussian_surface(xyz, r, density=10.0, probe=1.4, blob=0.0, quantize=True):
    """Surface for atoms (xyz, r) at ``density`` vertices/A^2.  Returns
    (sptpos, sptnrm, nvert 1-based, grid spacing).  With quantize=True the
    vertices and normals are rounded to MSMS's %9.3f text precision, i.e. the
    values the reference would read back from the .vert file."""
    xyzr = np.ascontiguousarray(np.column_stack([xyz, r]), dtype=np.float64)
    L = _sglib()
    vp = C.POINTER(C.c_double)()
    fp = C.POINTER(C.c_int)()
    nv, nf, h = C.c_int(), C.c_int(), C.c_double()
    rc = L.sg_gaussian_surface(len(xyzr), xyzr.ctypes.data, probe, density, blob, C.byref(vp),
                               C.byref(nv), C.byref(fp), C.byref(nf), C.byref(h))
    if rc != 0:
        raise RuntimeError("surface generation failed")
    v = np.ctypeslib.as_array(vp, shape=(nv.value, 6)).copy()
    f = np.ctypeslib.as_array(fp, shape=(nf.value, 3)).copy().astype(np.int32)
    L.sg_free(C.cast(vp, C.c_void_p))
    L.sg_free(C.cast(fp, C.c_void_p))
    pos, nrm = v[:, :3], v[:, 3:]
    if quantize:
        pos = np.round(pos, 3)
        nrm = np.round(nrm, 3)
    return pos, nrm, f, h.value


def face_filter(sptpos, nvert):
    """readin.f90:264-333 (surface_area).  A face is dropped when its Heron area
    (readin.f90:336-340) is below 1e-5 or its centroid lies within
    sqrt(1e-5) of the centroid of any of the 10 faces before it in the
    ORIGINAL list (dropped ones included).  nvert: (nface, 3), 1-based.
    Returns (nvert of the kept faces, total area of all faces)."""
    sp = np.ascontiguousarray(sptpos, dtype=np.float64).reshape(-1, 3)
    nv = np.ascontiguousarray(nvert, dtype=np.int32).reshape(-1, 3)
    p0, p1, p2 = sp[nv[:, 0] - 1], sp[nv[:, 1] - 1], sp[nv[:, 2] - 1]
    third = 1.0 / 3.0
    cen = (third * p0 + third * p1) + third * p2  # accumulated in vertex order

    def dist(a, b):
        d = a - b
        return np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])

    aa, bb, cc = dist(p0, p1), dist(p0, p2), dist(p1, p2)
    s = 0.5 * ((aa + bb) + cc)
    area = np.sqrt(((s * (s - aa)) * (s - bb)) * (s - cc))
    alert = np.zeros(len(nv), bool)
    for k in range(1, 11):
        d = cen[k:] - cen[:-k]
        alert[k:] |= ((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]) < 1e-5
    keep = ~((area < 1e-5) | alert)
    return nv[keep].copy(), float(np.sum(area)) if len(area) else 0.0
