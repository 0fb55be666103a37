"""First-hit comparison of the CUDA path (FP32) with the oracle (FP64).

Buckets, per ray:
  exact     same primitive (flat id) and, when both hit, t within 1e-5
            relative, or within the FP32 rounding of the ray origin carried
            to the hit (origin_rounding below: rays leaving a surface
            have a short t, and at grazing incidence the rounding of their
            origin, ~6e-8 of its coordinates, moves the hit along the ray
            by that over the cosine of the incidence angle);
  tie       different primitives whose hits are within 1e-4 relative in t
            and 1e-3 apart: two surfaces at the same depth (a shared mesh
            edge, coincident surfaces), where either answer is the closest
            hit to within float precision;
  boundary  the ray passes within BOUNDARY world units of an edge of either
            side's triangle, or grazes either side's sphere (its closest
            approach to the centre within BOUNDARY of the radius): there the
            FP32 kernel's rounding of the ray (~1e-7 relative) can move the
            hit across the edge or the silhouette, so the two sides may
            legitimately hit different primitives or one of them nothing;
  other     everything else: a real disagreement.
Parity means no ray in `other`.
"""
from __future__ import annotations

import numpy as np

BOUNDARY = 1e-5


def flat_layout(scene) -> dict:
    ns = len(scene.spheres)
    nq = len(scene.cylinders) + len(scene.cones) + len(scene.hyperboloids)
    nt = scene.n_triangles
    return {"spheres": ns, "quadrics": nq, "tri_base": ns + nq, "triangles": nt}


def tri_edge_distance(o, d, tri):
    """Signed world distance of the ray's crossing of each triangle's plane
    to the triangle's nearest edge (negative: outside); +inf where the ray is
    parallel to the plane. o, d: (n,3); tri: (n,9) vertices."""
    v0, v1, v2 = tri[:, 0:3], tri[:, 3:6], tri[:, 6:9]
    e1, e2 = v1 - v0, v2 - v0
    h = np.cross(d, e2)
    det = np.einsum("ij,ij->i", e1, h)
    ok = np.abs(det) > 0
    f = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
    s = o - v0
    u = f * np.einsum("ij,ij->i", s, h)
    q = np.cross(s, e1)
    v = f * np.einsum("ij,ij->i", d, q)
    w = 1.0 - u - v
    area2 = np.linalg.norm(np.cross(e1, e2), axis=1)
    # distance to the edge opposite each vertex = barycentric x height
    dist = np.minimum.reduce([
        w * area2 / np.maximum(np.linalg.norm(v2 - v1, axis=1), 1e-300),
        u * area2 / np.maximum(np.linalg.norm(e2, axis=1), 1e-300),
        v * area2 / np.maximum(np.linalg.norm(e1, axis=1), 1e-300)])
    return np.where(ok, dist, np.inf)


def sphere_graze(o, d, centre, radius):
    """|closest approach of the ray's line to the centre - radius|."""
    dn = d / np.linalg.norm(d, axis=1, keepdims=True)
    oc = o - centre
    t = -np.einsum("ij,ij->i", oc, dn)
    closest = np.linalg.norm(oc + dn * t[:, None], axis=1)
    return np.abs(closest - radius)


def near_boundary(scene, tri_pos, o, d, prim):
    """True where `prim` (flat ids, -1 = none) is a triangle whose edge or a
    sphere whose silhouette the ray passes within BOUNDARY of."""
    lay = flat_layout(scene)
    out = np.zeros(len(prim), bool)
    k = np.nonzero((prim >= lay["tri_base"]) & (prim < lay["tri_base"] + lay["triangles"]))[0]
    if len(k):
        dist = tri_edge_distance(o[k], d[k], tri_pos[prim[k] - lay["tri_base"]])
        out[k] = np.abs(dist) < BOUNDARY
    k = np.nonzero((prim >= 0) & (prim < lay["spheres"]))[0]
    if len(k):
        cen = np.array([scene.spheres[p][0] for p in prim[k]], np.float64)
        rad = np.array([scene.spheres[p][1] for p in prim[k]], np.float64)
        out[k] = sphere_graze(o[k], d[k], cen, rad) < BOUNDARY
    return out


def origin_rounding(o, d, normal):
    """Bound on |t_fp32 - t_fp64| from rounding the ray origin to FP32:
    4 ulps of the largest origin coordinate per axis, over |cos| between the
    unit direction and the surface normal (floored at 1e-3)."""
    ulp = 2.0 ** -23 * np.max(np.abs(o), axis=1)
    dn = d / np.linalg.norm(d, axis=1, keepdims=True)
    nn = normal / np.maximum(np.linalg.norm(normal, axis=1, keepdims=True), 1e-300)
    cos = np.abs(np.einsum("ij,ij->i", dn, nn))
    return 4.0 * np.sqrt(3.0) * ulp / np.maximum(cos, 1e-3) / np.linalg.norm(d, axis=1)


def classify(scene, tri_pos, o, d, g, r):
    """Buckets of the GPU hits g against the oracle hits r (record arrays
    with prim, t, point)."""
    g_prim, r_prim = g["prim"].astype(np.int64), r["prim"].astype(np.int64)
    both = (g_prim >= 0) & (r_prim >= 0)
    same = g_prim == r_prim
    dt = np.abs(g["t"] - r["t"])
    t_rel = dt / np.maximum(np.abs(r["t"]), 1e-6)
    t_ok = (t_rel <= 1e-5) | (dt <= origin_rounding(o, d, r["normal"]))
    exact = same & ((~both) | t_ok)
    dist = np.linalg.norm(g["point"] - r["point"], axis=1)
    tie = (~same) & both & (t_rel <= 1e-4) & (dist <= 1e-3 * np.maximum(r["t"], 1.0))
    rest = ~(exact | tie)
    boundary = np.zeros(len(o), bool)
    if rest.any():
        k = np.nonzero(rest)[0]
        boundary[k] = (near_boundary(scene, tri_pos, o[k], d[k], g_prim[k])
                       | near_boundary(scene, tri_pos, o[k], d[k], r_prim[k]))
    other = rest & ~boundary
    return exact, tie, boundary, other
