"""Seeded synthetic scenes for the five workloads, built as flat mrt_scene_desc.

The reference publishes no benchmark scenes, so every workload is generated
here from a seed (numpy PCG64) with the shapes, sizes and value distributions
of the benchmark configurations:

  c0  320x240, 64 spp, depth 8: ground plane + 8 spheres (50% lambertian,
      30% metal, 20% dielectric) + one emissive sphere light, black sky.
  c1  1920x1080, 256 spp, depth 12: geodesic sphere of 1,310,720 triangles
      displaced by 4-octave value noise, 16 materials by noise band, RGBE sky
      2048x1024 (gradient + 1-degree Gaussian sun + log-normal noise).
  c2  1280x720, 128 spp, depth 10: glass sphere over a lambertian plane,
      512x512-vertex sinusoid heightfield slab (522,242 triangles), point
      light with colour*brightness = 1000, photon-mapped caustics.
  c3  64 scenes of uneven size (batched workload).
  c4  512x512, 64 spp, depth 8: c1 generator at 200,000 triangles with 32
      materials and a 512x256 sky (inverse rendering).
  q0  320x240, 64 spp, depth 8: two cylinders, two cones, two hyperboloids,
      two spheres and a ground plane (the reference's quadric objects).
  t0  320x240, 64 spp, depth 8: image, checker and fallback textures, normal,
      roughness, metallic, ao and emission maps (make_textured).

Values use the reference's own types: 8-bit colours, RGBE sky texels,
horizontal integer-degree field of view (viewport.c:57), so that the oracle and
the library read identical numbers.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

import mrt


def u8(c) -> tuple[int, int, int]:
    return tuple(int(max(0, min(255, round(float(x) * 255.0)))) for x in c)


def hfov_from_vfov(vfov_deg: float, aspect: float) -> int:
    """Integer horizontal fov whose vertical fov at `aspect` is closest to vfov."""
    return int(round(math.degrees(2 * math.atan(math.tan(math.radians(vfov_deg) / 2) * aspect))))


@dataclass
class MeshData:
    positions: np.ndarray          # (V,3) float64
    normals: np.ndarray            # (V,3) float64
    indices: np.ndarray            # (T,3) uint32
    tri_material: np.ndarray | None = None  # (T,) int32
    uvs: np.ndarray | None = None  # (V,2) float64
    material: int = -1
    color: tuple = (255, 255, 255)


@dataclass
class Scene:
    name: str
    width: int
    height: int
    spp: int
    max_bounces: int
    camera: dict
    materials: list = field(default_factory=list)
    spheres: list = field(default_factory=list)   # (center, radius, material, color)
    planes: list = field(default_factory=list)    # (point, normal, material, color)
    meshes: list = field(default_factory=list)    # MeshData
    lights: list = field(default_factory=list)    # dicts
    cylinders: list = field(default_factory=list)  # dicts: position, orientation, diameter, height, ...
    cones: list = field(default_factory=list)      # dicts: position (apex), orientation, diameter, height
    hyperboloids: list = field(default_factory=list)  # dicts: position, orientation, a, b, c, shape, height
    textures: list = field(default_factory=list)  # dicts: type, rgba (H,W,4) uint8 | checker_scale, c1, c2
    ambient_ratio: float = 0.0
    ambient_color: tuple = (0, 0, 0)
    hdr: np.ndarray | None = None                 # (H,W,4) uint8 RGBE
    hdr_exposure: float = 0.0
    hdr_gamma: float = 1.0
    ior_all: float = 1.0
    triangle_one_sided: int = 0
    caustic: dict | None = None
    seed: int = 0
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n_triangles(self) -> int:
        return int(sum(len(m.indices) for m in self.meshes))

    def n_prims_bvh(self) -> int:
        """Primitives the BVH holds: spheres, quadrics and triangles (not planes)."""
        return (len(self.spheres) + len(self.cylinders) + len(self.cones) + len(self.hyperboloids)
                + self.n_triangles)

    def desc(self) -> mrt.SceneDesc:
        """Build the C struct (keeps every array alive on self)."""
        keep = []
        d = mrt.SceneDesc()
        d.abi_version = mrt.MRT_ABI_VERSION
        d.render_width, d.render_height = self.width, self.height
        d.max_bounces = self.max_bounces
        d.triangle_one_sided = self.triangle_one_sided
        d.ior_all = self.ior_all
        cam = self.camera
        d.camera.position[:] = cam["position"]
        d.camera.orientation[:] = cam["orientation"]
        d.camera.focus_dist = cam.get("focus_dist", 0.0)
        d.camera.defocus_angle = cam.get("defocus_angle", 0.0)
        d.camera.fov = cam["fov"]
        d.ambient.ratio = self.ambient_ratio
        d.ambient.color[:] = self.ambient_color
        if self.hdr is not None:
            h = np.ascontiguousarray(self.hdr, np.uint8)
            keep.append(h)
            d.ambient.hdr_rgbe = h.ctypes.data_as(C.POINTER(C.c_uint8))
            d.ambient.hdr_height, d.ambient.hdr_width = h.shape[0], h.shape[1]
            d.ambient.hdr_exposure = self.hdr_exposure
            d.ambient.hdr_gamma = self.hdr_gamma
        if self.caustic:
            c = self.caustic
            d.caustic.enable = 1
            d.caustic.passes = c.get("passes", 1)
            d.caustic.photons_per_light = c["photons"]
            d.caustic.radius = c["radius"]
            d.caustic.norm_factor = c.get("norm", 1.0)
            d.caustic.shrink = c.get("shrink", 0.9)
            d.caustic.knn = c.get("k", 15)
            d.caustic.mode = c.get("mode", 0)
            d.caustic.spp_per_pass = c.get("spp_per_pass", 0)
        mats = (mrt.Material * max(1, len(self.materials)))()
        for i, m in enumerate(self.materials):
            mats[i].color[:] = m["color"]
            mats[i].emission_color[:] = m.get("emission_color", (255, 255, 255))
            mats[i].metallic = m.get("metallic", 0.0)
            mats[i].roughness = m.get("roughness", 0.0)
            mats[i].ior = m.get("ior", 0.0)
            mats[i].transmission = m.get("transmission", 0.0)
            mats[i].ao = m.get("ao", 1.0)
            mats[i].emission_strength = m.get("emission_strength", 0.0)
            mats[i].scale = m.get("scale", 1.0)
            for k in mrt.TEX_SLOTS:
                setattr(mats[i], k, int(m.get(k, 0)))
            mats[i].normal_intensity = m.get("normal_intensity", 1.0)
        keep.append(mats)
        tx = (mrt.Texture * max(1, len(self.textures)))()
        for i, t in enumerate(self.textures):
            tx[i].type = t["type"]
            if t.get("rgba") is not None:
                px = np.ascontiguousarray(t["rgba"], np.uint8)
                keep.append(px)
                tx[i].height, tx[i].width = px.shape[0], px.shape[1]
                tx[i].rgba = px.ctypes.data_as(C.POINTER(C.c_uint8))
            tx[i].checker_scale = t.get("checker_scale", 1.0)
            tx[i].c1[:] = t.get("c1", (0, 0, 0))
            tx[i].c2[:] = t.get("c2", (0, 0, 0))
        keep.append(tx)
        d.textures, d.n_textures = tx, len(self.textures)
        d.materials, d.n_materials = mats, len(self.materials)
        sph = (mrt.Sphere * max(1, len(self.spheres)))()
        for i, (c, r, mi, col) in enumerate(self.spheres):
            sph[i].center[:] = c
            sph[i].radius = r
            sph[i].material = mi
            sph[i].color[:] = col
        keep.append(sph)
        d.spheres, d.n_spheres = sph, len(self.spheres)
        pl = (mrt.Plane * max(1, len(self.planes)))()
        for i, (p, n, mi, col) in enumerate(self.planes):
            pl[i].point[:] = p
            pl[i].normal[:] = n
            pl[i].material = mi
            pl[i].color[:] = col
        keep.append(pl)
        d.planes, d.n_planes = pl, len(self.planes)
        ms = (mrt.Mesh * max(1, len(self.meshes)))()
        for i, m in enumerate(self.meshes):
            pos = np.ascontiguousarray(m.positions, np.float64)
            nrm = np.ascontiguousarray(m.normals, np.float64)
            idx = np.ascontiguousarray(m.indices, np.uint32)
            keep += [pos, nrm, idx]
            ms[i].n_vertices, ms[i].n_triangles = len(pos), len(idx)
            ms[i].positions = pos.ctypes.data_as(C.POINTER(C.c_double))
            ms[i].normals = nrm.ctypes.data_as(C.POINTER(C.c_double))
            ms[i].indices = idx.ctypes.data_as(C.POINTER(C.c_uint32))
            if m.uvs is not None:
                uv = np.ascontiguousarray(m.uvs, np.float64)
                keep.append(uv)
                ms[i].uvs = uv.ctypes.data_as(C.POINTER(C.c_double))
            if m.tri_material is not None:
                tm = np.ascontiguousarray(m.tri_material, np.int32)
                keep.append(tm)
                ms[i].tri_material = tm.ctypes.data_as(C.POINTER(C.c_int32))
            ms[i].material = m.material
            ms[i].color[:] = m.color
        keep.append(ms)
        d.meshes, d.n_meshes = ms, len(self.meshes)
        li = (mrt.Light * max(1, len(self.lights)))()
        for i, L in enumerate(self.lights):
            li[i].type = L.get("type", mrt.LIGHT_POINT)
            li[i].position[:] = L["position"]
            li[i].brightness = L["brightness"]
            li[i].color[:] = L["color"]
            li[i].radius = L.get("radius", 0.0)
            li[i].shadow_sample = L.get("shadow_sample", 0)
        keep.append(li)
        d.lights, d.n_lights = li, len(self.lights)
        cy = (mrt.Cylinder * max(1, len(self.cylinders)))()
        for i, q in enumerate(self.cylinders):
            cy[i].position[:] = q["position"]
            cy[i].orientation[:] = q["orientation"]
            cy[i].diameter, cy[i].height = q["diameter"], q["height"]
            cy[i].material = q.get("material", -1)
            cy[i].material_top = q.get("material_top", -1)
            cy[i].material_bot = q.get("material_bot", -1)
            cy[i].color[:] = q.get("color", (255, 255, 255))
        co = (mrt.Cone * max(1, len(self.cones)))()
        for i, q in enumerate(self.cones):
            co[i].position[:] = q["position"]
            co[i].orientation[:] = q["orientation"]
            co[i].diameter, co[i].height = q["diameter"], q["height"]
            co[i].material = q.get("material", -1)
            co[i].material_top = q.get("material_top", -1)
            co[i].color[:] = q.get("color", (255, 255, 255))
        hb = (mrt.Hyperboloid * max(1, len(self.hyperboloids)))()
        for i, q in enumerate(self.hyperboloids):
            hb[i].position[:] = q["position"]
            hb[i].orientation[:] = q["orientation"]
            hb[i].a, hb[i].b, hb[i].c = q["a"], q["b"], q["c"]
            hb[i].shape, hb[i].height = q["shape"], q["height"]
            hb[i].material = q.get("material", -1)
            hb[i].color[:] = q.get("color", (255, 255, 255))
        keep += [cy, co, hb]
        d.cylinders, d.n_cylinders = cy, len(self.cylinders)
        d.cones, d.n_cones = co, len(self.cones)
        d.hyperboloids, d.n_hyperboloids = hb, len(self.hyperboloids)
        self._keep = keep
        return d


# ----------------------------------------------------------------- helpers

def _material_mix(rng: np.random.Generator, kind: str) -> dict:
    if kind == "lambertian":
        return dict(color=u8(rng.uniform(0.1, 0.9, 3)), metallic=0.0, ior=0.0)
    if kind == "metal":
        return dict(color=u8(rng.uniform(0.1, 0.9, 3)), metallic=1.0,
                    roughness=float(rng.uniform(0.0, 0.3)))
    if kind == "dielectric":
        return dict(color=(255, 255, 255), metallic=0.0, ior=1.5, transmission=1.0)
    raise ValueError(kind)


def _kind(rng: np.random.Generator) -> str:
    x = rng.uniform()
    return "lambertian" if x < 0.5 else ("metal" if x < 0.8 else "dielectric")


def look_at(pos, target) -> tuple:
    d = np.asarray(target, float) - np.asarray(pos, float)
    return tuple(d / np.linalg.norm(d))


# ------------------------------------------------------------------ c0

def make_c0(seed: int = 0, width: int = 320, height: int = 240, spp: int = 64,
            depth: int = 8) -> Scene:
    rng = np.random.default_rng(seed)
    aspect = width / height
    sc = Scene("c0", width, height, spp, depth,
               camera=dict(position=(0.0, 2.0, 10.0), orientation=look_at((0, 2, 10), (0, 0, 0)),
                           fov=hfov_from_vfov(40.0, aspect)), seed=seed)
    sc.materials.append(dict(color=(204, 204, 204), metallic=0.0, ior=0.0))
    sc.planes.append(((0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 0, (204, 204, 204)))
    placed = []
    while len(placed) < 8:
        r = float(rng.uniform(0.3, 1.0))
        c = (float(rng.uniform(-4, 4)), r, float(rng.uniform(-4, 4)))
        if all(math.dist(c, c2) > r + r2 for c2, r2 in placed):
            placed.append((c, r))
    for c, r in placed:
        sc.materials.append(_material_mix(rng, _kind(rng)))
        sc.spheres.append((c, r, len(sc.materials) - 1, (255, 255, 255)))
    sc.materials.append(dict(color=(0, 0, 0), metallic=0.0, ior=0.0, emission_strength=10.0,
                             emission_color=(255, 255, 255)))
    sc.spheres.append(((0.0, 6.0, 0.0), 0.5, len(sc.materials) - 1, (0, 0, 0)))
    sc.ambient_ratio, sc.ambient_color = 0.0, (0, 0, 0)
    return sc


# ----------------------------------------------------- geodesic sphere mesh

_ICO_V = None


def _icosahedron():
    t = (1 + 5 ** 0.5) / 2
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], float)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9],
                  [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2],
                  [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
                  [8, 6, 7], [9, 8, 1]], np.int64)
    return v / np.linalg.norm(v, axis=1, keepdims=True), f


def geodesic_sphere(freq: int) -> tuple[np.ndarray, np.ndarray]:
    """Class-I geodesic sphere: each icosahedron face split into freq^2 triangles
    (20*freq^2 triangles). Returns unit vertices (V,3) and faces (T,3)."""
    v0, f0 = _icosahedron()
    n = freq
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    keep = ii + jj <= n
    ii, jj = ii[keep], jj[keep]                          # lattice points of one face
    lid = -np.ones((n + 1, n + 1), np.int64)
    lid[ii, jj] = np.arange(len(ii))
    # triangles in lattice coordinates
    a, b = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    up = a + b < n
    t_up = np.stack([lid[a[up], b[up]], lid[a[up] + 1, b[up]], lid[a[up], b[up] + 1]], 1)
    dn = a + b < n - 1
    t_dn = np.stack([lid[a[dn] + 1, b[dn]], lid[a[dn] + 1, b[dn] + 1], lid[a[dn], b[dn] + 1]], 1)
    tri_local = np.concatenate([t_up, t_dn])
    P, F = [], []
    for k, (ia, ib, ic) in enumerate(f0):
        A, B, Cc = v0[ia], v0[ib], v0[ic]
        pts = (A[None] * ((n - ii - jj) / n)[:, None] + B[None] * (ii / n)[:, None]
               + Cc[None] * (jj / n)[:, None])
        P.append(pts)
        F.append(tri_local + k * len(ii))
    P = np.concatenate(P)
    F = np.concatenate(F)
    P /= np.linalg.norm(P, axis=1, keepdims=True)
    q = np.round(P * 1e9).astype(np.int64)
    _, first, inv = np.unique(q, axis=0, return_index=True, return_inverse=True)
    inv = inv.reshape(-1)
    return P[first], inv[F].astype(np.uint32)


def _hash3(ix, iy, iz, seed):
    h = (ix.astype(np.uint64) * np.uint64(73856093)) ^ (iy.astype(np.uint64) * np.uint64(19349663)) \
        ^ (iz.astype(np.uint64) * np.uint64(83492791)) ^ np.uint64(seed * 2654435761 & 0xFFFFFFFF)
    h ^= h >> np.uint64(13)
    h *= np.uint64(0x5bd1e995)
    h ^= h >> np.uint64(15)
    return (h & np.uint64(0xFFFFFF)).astype(np.float64) / float(0xFFFFFF)


def value_noise(p: np.ndarray, octaves: int = 4, seed: int = 0, base_freq: float = 2.0) -> np.ndarray:
    """Sum of `octaves` octaves of trilinear value noise in [-1,1] (amplitude halves)."""
    out = np.zeros(len(p))
    amp, freq, norm = 1.0, base_freq, 0.0
    with np.errstate(over="ignore"):
        for o in range(octaves):
            q = p * freq + 17.0 * o
            i0 = np.floor(q).astype(np.int64)
            f = q - i0
            s = f * f * (3 - 2 * f)
            acc = np.zeros(len(p))
            for dx in (0, 1):
                for dy in (0, 1):
                    for dz in (0, 1):
                        w = (np.where(dx, s[:, 0], 1 - s[:, 0]) * np.where(dy, s[:, 1], 1 - s[:, 1])
                             * np.where(dz, s[:, 2], 1 - s[:, 2]))
                        acc += w * _hash3(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz, seed + o)
            out += amp * (2 * acc - 1)
            norm += amp
            amp *= 0.5
            freq *= 2.0
    return out / norm


def displaced_sphere(freq: int, seed: int, amplitude: float = 0.15, n_materials: int = 16):
    v, f = geodesic_sphere(freq)
    disp = value_noise(v, 4, seed)
    p = v * (1.0 + amplitude * disp)[:, None]
    p = p.astype(np.float32).astype(np.float64)          # float32 vertices, exact in double
    e1 = p[f[:, 1]] - p[f[:, 0]]
    e2 = p[f[:, 2]] - p[f[:, 0]]
    fn = np.cross(e1, e2)
    vn = np.zeros_like(p)
    for k in range(3):
        np.add.at(vn, f[:, k], fn)
    vn /= np.maximum(np.linalg.norm(vn, axis=1, keepdims=True), 1e-30)
    cen = (p[f[:, 0]] + p[f[:, 1]] + p[f[:, 2]]) / 3
    band = value_noise(cen, 2, seed + 101, base_freq=1.5)
    band = (band - band.min()) / max(1e-12, band.max() - band.min())
    tri_mat = np.minimum((band * n_materials).astype(np.int32), n_materials - 1)
    return p, vn, f, tri_mat


# ------------------------------------------------------------- HDRI sky

def rgbe_encode(rgb: np.ndarray) -> np.ndarray:
    """Float RGB (H,W,3) -> RGBE bytes decoded by the reference as
    c * 2^(e-128) / 255 (get_hdr_pixel, get_hdr_value.c:16-41)."""
    m = rgb.max(axis=2)
    out = np.zeros(rgb.shape[:2] + (4,), np.uint8)
    ok = m > 1e-32
    e = np.zeros_like(m, dtype=np.int64)
    e[ok] = np.floor(np.log2(m[ok])).astype(np.int64) + 1
    e = np.clip(e, -127, 127)
    scale = np.ldexp(1.0, (-e).astype(np.int64))          # 2^-e
    mant = np.clip(np.round(rgb * (scale * 255.0)[..., None]), 0, 255)
    out[..., :3] = np.where(ok[..., None], mant, 0).astype(np.uint8)
    out[..., 3] = np.where(ok, e + 128, 0).astype(np.uint8)
    return out


def make_sky(width: int, height: int, seed: int, sun_sigma_deg: float = 1.0,
             sun_peak: float = 5e4, noise_sigma: float = 0.5) -> np.ndarray:
    """Equirect sky in the reference's mapping (background.c:55-56):
    row v = 0.5 + asin(y)/pi, column u = 0.5 - atan2(z,x)/(2 pi)."""
    rng = np.random.default_rng(seed)
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    uu, vv = np.meshgrid(u, v)
    theta = (vv - 0.5) * np.pi                          # elevation
    phi = (0.5 - uu) * 2 * np.pi
    d = np.stack([np.cos(theta) * np.cos(phi), np.sin(theta), np.cos(theta) * np.sin(phi)], -1)
    grad = 0.2 + 0.8 * np.clip(vv, 0, 1)
    sun_el = rng.uniform(0.3, 1.0)
    sun_az = rng.uniform(0, 2 * np.pi)
    sd = np.array([np.cos(sun_el) * np.cos(sun_az), np.sin(sun_el), np.cos(sun_el) * np.sin(sun_az)])
    ang = np.arccos(np.clip(d @ sd, -1, 1))
    sun = sun_peak * np.exp(-0.5 * (ang / np.radians(sun_sigma_deg)) ** 2)
    noise = np.exp(noise_sigma * rng.standard_normal((height, width)))
    tint = np.array([1.0, 0.95, 0.85])
    rgb = ((grad + sun) * noise)[..., None] * tint[None, None]
    return rgbe_encode(rgb)


# ------------------------------------------------------------------ c1 / c4

def make_c1(seed: int = 1, width: int = 1920, height: int = 1080, spp: int = 256, depth: int = 12,
            freq: int = 256, n_materials: int = 16, sky=(2048, 1024)) -> Scene:
    rng = np.random.default_rng(seed)
    p, vn, f, tm = displaced_sphere(freq, seed, 0.15, n_materials)
    pos = (0.0, 0.6, 3.3)
    sc = Scene("c1", width, height, spp, depth,
               camera=dict(position=pos, orientation=look_at(pos, (0, 0, 0)), fov=50), seed=seed)
    for _ in range(n_materials):
        sc.materials.append(_material_mix(rng, _kind(rng)))
    sc.meshes.append(MeshData(p, vn, f, tm, None, 0, (255, 255, 255)))
    sc.ambient_ratio = 1.0
    sc.ambient_color = (255, 255, 255)
    sc.hdr = make_sky(sky[0], sky[1], seed + 7)
    return sc


def make_c4(seed: int = 4, width: int = 512, height: int = 512, spp: int = 64, depth: int = 8,
            freq: int = 100, n_materials: int = 32, sky=(512, 256)) -> Scene:
    """Inverse-rendering scene: the c1 generator at 20*freq^2 triangles
    (200,000 at freq 100) with 32 materials and a 512x256 sky. Roughness is
    drawn in [0.05, 1] for every material (metal and glass sample GGX
    directions with it), and one material in eight emits (white, strength
    0.5..2); the others carry a white emission colour at strength 0, so
    that emission has a gradient everywhere. Values are float32-exact."""
    sc = make_c1(seed, width, height, spp, depth, freq=freq, n_materials=n_materials, sky=sky)
    sc.name = "c4"
    rng = np.random.default_rng(seed + 1000)
    for i, m in enumerate(sc.materials):
        m["roughness"] = float(np.float32(rng.uniform(0.05, 1.0)))
        m["emission_color"] = (255, 255, 255)
        m["emission_strength"] = float(np.float32(rng.uniform(0.5, 2.0))) if i % 8 == 0 else 0.0
    return sc


def diff_theta(scene: Scene) -> np.ndarray:
    """theta of mrt_forward for a scene, computed on the host: colours / 255,
    roughness, emission strength and the linear sky radiance decoded from
    its RGBE texels (float32, as the renderer decodes them)."""
    mats = scene.materials
    alb = np.array([np.asarray(m.get("color", (0, 0, 0)), np.float64) / 255.0 for m in mats]).reshape(-1)
    rough = np.array([min(max(m.get("roughness", 0.0), 0.0), 1.0) for m in mats])
    emis = np.array([m.get("emission_strength", 0.0) for m in mats])
    parts = [alb.astype(np.float32), rough.astype(np.float32), emis.astype(np.float32)]
    if scene.hdr is not None:
        rgbe = np.asarray(scene.hdr, np.uint8).reshape(-1, 4)
        scale = np.ldexp(np.float32(1.0), rgbe[:, 3].astype(np.int32) - 128).astype(np.float32)
        sky = (rgbe[:, :3].astype(np.float32) * scale[:, None]) / np.float32(255.0)
        parts.append(sky.astype(np.float32).reshape(-1))
    return np.concatenate(parts).astype(np.float32)


# ------------------------------------------------------------------ c2

def heightfield(n: int, size: float, y0: float, seed: int, amplitude: float = 0.05):
    rng = np.random.default_rng(seed)
    xs = np.linspace(-size / 2, size / 2, n)
    X, Z = np.meshgrid(xs, xs, indexing="ij")
    H = np.zeros_like(X)
    dHx = np.zeros_like(X)
    dHz = np.zeros_like(X)
    for _ in range(8):
        k = rng.uniform(2.0, 9.0)
        th = rng.uniform(0, 2 * np.pi)
        ph = rng.uniform(0, 2 * np.pi)
        kx, kz = k * np.cos(th), k * np.sin(th)
        arg = kx * X + kz * Z + ph
        H += np.sin(arg) / 8
        dHx += kx * np.cos(arg) / 8
        dHz += kz * np.cos(arg) / 8
    Y = y0 + amplitude * H
    p = np.stack([X, Y, Z], -1).reshape(-1, 3).astype(np.float32).astype(np.float64)
    nrm = np.stack([-amplitude * dHx, np.ones_like(X), -amplitude * dHz], -1).reshape(-1, 3)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    i, j = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="ij")
    a = (i * n + j).reshape(-1)
    b = a + n
    f = np.concatenate([np.stack([a, b, a + 1], 1), np.stack([a + 1, b, b + 1], 1)]).astype(np.uint32)
    return p, nrm, f


def make_c2(seed: int = 2, width: int = 1280, height: int = 720, spp: int = 128, depth: int = 10,
            grid: int = 512, photons: int = 2_000_000, passes: int = 1, mode: int = 0,
            spp_per_pass: int = 0) -> Scene:
    pos = (0.0, 3.2, 6.5)
    sc = Scene("c2", width, height, spp, depth,
               camera=dict(position=pos, orientation=look_at(pos, (0, 0.6, 0)), fov=60), seed=seed)
    sc.materials.append(dict(color=(204, 204, 204), metallic=0.0, ior=0.0))          # floor
    sc.materials.append(dict(color=(255, 255, 255), metallic=0.0, ior=1.5, transmission=1.0))
    sc.materials.append(dict(color=(230, 242, 255), metallic=0.0, ior=1.33, transmission=1.0))
    sc.planes.append(((0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 0, (204, 204, 204)))
    sc.spheres.append(((0.0, 1.6, 0.0), 1.0, 1, (255, 255, 255)))
    p, n, f = heightfield(grid, 6.0, 0.35, seed)
    sc.meshes.append(MeshData(p, n, f, None, None, 2, (230, 242, 255)))
    sc.lights.append(dict(position=(2.0, 5.0, 1.0), brightness=1000.0 / 255.0,
                          color=(255, 255, 255)))
    sc.ambient_ratio, sc.ambient_color = 0.0, (0, 0, 0)
    sc.caustic = dict(photons=photons, radius=0.02, norm=1.0, k=15, passes=passes,
                      shrink=0.9, mode=mode, spp_per_pass=spp_per_pass)
    return sc


# ------------------------------------------------------------------ c3

def make_c3_specs(seed: int = 3, n: int = 64) -> list[dict]:
    """Per-scene sizes of the batched workload (log-uniform triangles, uniform
    resolution, spp from {16..256}, depth 8..16, half HDRI half area light)."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n):
        tris = float(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
        freq = max(4, int(round(math.sqrt(tris / 20))))
        side = int(rng.uniform(256, 1024))
        specs.append(dict(index=i, freq=freq, tris=20 * freq * freq, width=side, height=side,
                          spp=int(rng.choice([16, 32, 64, 128, 256])),
                          depth=int(rng.integers(8, 17)), hdri=(i % 2 == 0),
                          seed=int(rng.integers(1 << 30))))
    return specs


def make_c3_scene(spec: dict, sky_cache: dict | None = None) -> Scene:
    sc = make_c1(spec["seed"], spec["width"], spec["height"], spec["spp"], spec["depth"],
                 freq=spec["freq"], n_materials=16, sky=(1024, 512))
    sc.name = f"c3_{spec['index']}"
    if not spec["hdri"]:
        # area light: an emissive two-triangle quad above the object
        sc.hdr = None
        sc.ambient_ratio, sc.ambient_color = 0.0, (0, 0, 0)
        sc.materials.append(dict(color=(0, 0, 0), metallic=0.0, ior=0.0, emission_strength=8.0,
                                 emission_color=(255, 250, 240)))
        q = np.array([[-1, 3, -1], [1, 3, -1], [1, 3, 1], [-1, 3, 1]], float)
        nq = np.tile([[0.0, -1.0, 0.0]], (4, 1))
        fq = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
        sc.meshes.append(MeshData(q, nq, fq, None, None, len(sc.materials) - 1, (0, 0, 0)))
    return sc


def make_c2_progressive(**kw) -> Scene:
    """c2's extension mode: 16 photon passes of 2 M photons, 8 spp each
    (128 spp), fixed-radius gather shrinking by 0.9 per pass."""
    sc = make_c2(passes=16, mode=1, spp_per_pass=8, **kw)
    sc.name = "c2p"
    return sc


def _unit(v) -> tuple:
    v = np.asarray(v, float)
    return tuple(v / np.linalg.norm(v))


def make_quadrics(seed: int = 5, width: int = 320, height: int = 240, spp: int = 64,
                  depth: int = 8) -> Scene:
    """Cylinders, cones and hyperboloids (t_cylinder / t_cone / t_hyperboloid)
    over a ground plane: an upright cylinder with a metal top cap, a tilted
    glass cylinder with a lambertian bottom cap, an inverted cone with a metal
    cap, a tilted cone, a one-sheet and a two-sheet hyperboloid, an emissive
    sphere, a glass sphere and a point light under a blue-grey ambient sky.
    Orientations are unit vectors, as the reference's parser leaves them
    (parse_elements.c:28)."""
    rng = np.random.default_rng(seed)
    aspect = width / height
    sc = Scene("quadrics", width, height, spp, depth,
               camera=dict(position=(0.0, 3.0, 12.0), orientation=look_at((0, 3, 12), (0, 1, 0)),
                           fov=hfov_from_vfov(45.0, aspect)), seed=seed)

    def mat(**m):
        sc.materials.append(m)
        return len(sc.materials) - 1

    ground = mat(color=(200, 200, 190), metallic=0.0, ior=0.0)
    sc.planes.append(((0.0, 0.0, 0.0), (0.0, 1.0, 0.0), ground, (200, 200, 190)))
    lam = [mat(**_material_mix(rng, "lambertian")) for _ in range(4)]
    metal = [mat(**_material_mix(rng, "metal")) for _ in range(2)]
    glass = mat(**_material_mix(rng, "dielectric"))
    sc.cylinders.append(dict(position=(-3.0, 1.0, 0.0), orientation=(0.0, 1.0, 0.0), diameter=1.6,
                             height=2.0, material=lam[0], material_top=metal[0], color=(255, 255, 255)))
    sc.cylinders.append(dict(position=(2.5, 1.2, -1.0), orientation=_unit((1.0, 0.6, 0.3)), diameter=1.0,
                             height=2.5, material=glass, material_bot=lam[1], color=(255, 255, 255)))
    sc.cones.append(dict(position=(0.0, 2.5, -2.0), orientation=(0.0, -1.0, 0.0), diameter=2.0,
                         height=2.0, material=lam[2], material_top=metal[1], color=(255, 255, 255)))
    sc.cones.append(dict(position=(-1.2, 0.2, 2.5), orientation=_unit((0.3, 1.0, 0.2)), diameter=1.2,
                         height=1.5, material=lam[3], color=(255, 255, 255)))
    sc.hyperboloids.append(dict(position=(3.5, 1.5, 2.0), orientation=(0.0, 1.0, 0.0), a=0.5, b=0.7,
                                c=1.0, shape=1.0, height=3.0, material=lam[1], color=(255, 255, 255)))
    sc.hyperboloids.append(dict(position=(-4.0, 2.0, -3.0), orientation=_unit((0.2, 1.0, 0.1)), a=0.6,
                                b=0.6, c=0.8, shape=-1.0, height=3.0, material=metal[0],
                                color=(255, 255, 255)))
    light = mat(color=(0, 0, 0), metallic=0.0, ior=0.0, emission_strength=8.0,
                emission_color=(255, 240, 220))
    sc.spheres.append(((0.0, 7.0, 2.0), 0.8, light, (0, 0, 0)))
    sc.spheres.append(((1.0, 0.6, 3.0), 0.6, glass, (255, 255, 255)))
    sc.lights.append(dict(position=(2.0, 6.0, 6.0), brightness=0.6, color=(255, 255, 255)))
    sc.ambient_ratio, sc.ambient_color = 0.2, (120, 140, 200)
    return sc


def make_textured(seed: int = 6, width: int = 320, height: int = 240, spp: int = 64, depth: int = 8,
                  partial_alpha: bool = False) -> Scene:
    """Textures and maps (t_tex / apply_all_map): a ground plane with a 3-D
    checker, an image-textured sphere with cut-out (alpha 0) texels, a
    uv-checker sphere, a metal sphere with roughness and normal maps, a
    sphere with metallic and ao maps, an emissive sphere with emission
    strength and colour maps, an image-textured quad of two triangles with
    uvs, a cylinder with a uv checker, a sphere with an empty image (the
    reference's fallback checker) and one with an HDR-type texture (black in
    the reference). Every scalar-mapped material sits on one sphere only.
    partial_alpha adds texels of alpha 128 to the cut-out image."""
    rng = np.random.default_rng(seed)
    aspect = width / height
    sc = Scene("textured", width, height, spp, depth,
               camera=dict(position=(0.0, 2.5, 11.0), orientation=look_at((0, 2.5, 11), (0, 1, 0)),
                           fov=hfov_from_vfov(45.0, aspect)), seed=seed)

    def tex(**t):
        sc.textures.append(t)
        return len(sc.textures)            # 1-based, as the ABI names textures

    def mat(**m):
        sc.materials.append(m)
        return len(sc.materials) - 1

    img = rng.integers(0, 256, (16, 16, 4), dtype=np.uint8)
    img[..., 3] = 255
    img[rng.uniform(size=(16, 16)) < 0.25, 3] = 0
    if partial_alpha:
        img[rng.uniform(size=(16, 16)) < 0.2, 3] = 128
    t_img = tex(type=mrt.TEX_IMAGE, rgba=img)
    t_uvck = tex(type=mrt.TEX_CHECKER_LOCAL, checker_scale=8.0, c1=(230, 60, 40), c2=(30, 40, 200))
    t_glob = tex(type=mrt.TEX_CHECKER_GLOBAL, checker_scale=1.5, c1=(220, 220, 210), c2=(40, 40, 40))
    nrm = np.zeros((8, 8, 4), np.uint8)
    nrm[..., :2] = rng.integers(64, 192, (8, 8, 2))
    nrm[..., 2] = rng.integers(200, 256, (8, 8))
    nrm[..., 3] = 255
    t_nrm = tex(type=mrt.TEX_IMAGE, rgba=nrm)

    def grey(lo, hi, n=8):
        g = np.zeros((n, n, 4), np.uint8)
        g[..., :3] = rng.integers(lo, hi, (n, n))[..., None]
        g[..., 3] = 255
        return tex(type=mrt.TEX_IMAGE, rgba=g)

    t_rough, t_metal, t_ao, t_es = grey(10, 120), grey(0, 256), grey(100, 256), grey(0, 256)
    t_ec = tex(type=mrt.TEX_IMAGE, rgba=np.concatenate(
        [rng.integers(0, 256, (4, 4, 3), dtype=np.uint8), np.full((4, 4, 1), 255, np.uint8)], axis=2))
    t_empty = tex(type=mrt.TEX_IMAGE, rgba=None)
    t_hdr = tex(type=mrt.TEX_HDR)

    ground = mat(color=(200, 200, 200), metallic=0.0, ior=0.0, color_tex=t_glob, scale=1.0)
    sc.planes.append(((0.0, 0.0, 0.0), (0.0, 1.0, 0.0), ground, (200, 200, 200)))
    m_img = mat(color=(255, 255, 255), metallic=0.0, ior=0.0, color_tex=t_img)
    m_uv = mat(color=(255, 255, 255), metallic=0.0, ior=0.0, color_tex=t_uvck, scale=2.0)
    m_rough = mat(color=(210, 180, 120), metallic=1.0, roughness=0.3, roughness_tex=t_rough, normal_tex=t_nrm)
    m_metal = mat(color=(120, 200, 160), metallic=0.5, roughness=0.2, ior=1.5, metallic_tex=t_metal,
                  ao_tex=t_ao, normal_tex=t_nrm, normal_intensity=0.5)
    m_emit = mat(color=(0, 0, 0), metallic=0.0, ior=0.0, emission_strength=6.0, emission_color=(255, 255, 255),
                 emission_strength_tex=t_es, emission_color_tex=t_ec)
    m_quad = mat(color=(255, 255, 255), metallic=0.0, ior=0.0, color_tex=t_img, scale=1.0)
    m_cyl = mat(color=(255, 255, 255), metallic=0.0, ior=0.0, color_tex=t_uvck)
    m_empty = mat(color=(255, 255, 255), metallic=0.0, ior=0.0, color_tex=t_empty)
    m_hdr = mat(color=(255, 255, 255), metallic=0.0, ior=0.0, color_tex=t_hdr)
    sc.spheres += [((-3.0, 1.0, 0.0), 1.0, m_img, (255, 255, 255)),
                   ((-0.8, 0.8, 1.5), 0.8, m_uv, (255, 255, 255)),
                   ((1.3, 1.0, 0.2), 1.0, m_rough, (255, 255, 255)),
                   ((3.4, 0.7, 1.6), 0.7, m_metal, (255, 255, 255)),
                   ((0.5, 5.5, 1.0), 0.6, m_emit, (0, 0, 0)),
                   ((-1.9, 0.45, 3.2), 0.45, m_empty, (255, 255, 255)),
                   ((2.2, 0.45, 3.4), 0.45, m_hdr, (255, 255, 255))]
    pos = np.array([[-2.5, 0.0, -2.5], [2.5, 0.0, -2.5], [2.5, 3.5, -2.5], [-2.5, 3.5, -2.5]], np.float64)
    nrm_v = np.tile([0.0, 0.0, 1.0], (4, 1))
    uvs = np.array([[0.0, 1.0], [1.0, 1.0], [1.0, 0.0], [0.0, 0.0]], np.float64)
    sc.meshes.append(MeshData(pos, nrm_v, np.array([[0, 1, 2], [0, 2, 3]], np.uint32), None, uvs, m_quad,
                              (255, 255, 255)))
    sc.cylinders.append(dict(position=(4.3, 1.0, -1.0), orientation=(0.0, 1.0, 0.0), diameter=1.0, height=2.0,
                             material=m_cyl, color=(255, 255, 255)))
    sc.lights.append(dict(position=(-2.0, 6.0, 5.0), brightness=0.7, color=(255, 255, 255)))
    sc.ambient_ratio, sc.ambient_color = 0.25, (150, 170, 210)
    return sc


CONFIGS = {"c0": make_c0, "c1": make_c1, "c2": make_c2, "c2p": make_c2_progressive, "c4": make_c4,
           "q0": make_quadrics, "t0": make_textured}
