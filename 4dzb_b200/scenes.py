"""Seeded synthetic scenes for the FDZB soft-shadow path.

The reference's demo meshes (dragon_1.obj, plane.obj) are not in its repository,
so scenes are generated:

* receiver: height field z = 0.3 sin(x) cos(y) over [-8, 8]^2 sampled on a W x H
  grid with uniform +-0.5 cell jitter, analytic normals, positions pushed 1e-4
  along the normal; row-major float4 (w = 1) positions and normals, the layout
  of the reference's G-buffer textures (4DZB/Resources/shader/gatherData.shf);
* occluders: a triangle soup, centroids uniform in [-6, 6]^2 x [zlo, zhi],
  vertices = centroid + N(0, sigma^2) per axis, float4 vertices (stride 16 B),
  int3 indices (3t, 3t+1, 3t+2);
* light: square area light centred at (0, 0, 6) facing -z, up +y.

Random numbers: splitmix64 counter streams (one stream per purpose) mapped to
doubles in [0, 1); normal deviates by Box-Muller in double, cast to float32.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _splitmix(seed: int, stream: int, n: int) -> np.ndarray:
    """n uint64 outputs of the splitmix64 sequence for (seed, stream)."""
    with np.errstate(over="ignore"):
        base = np.uint64((seed * 0x100000001B3 + stream * 0x9E3779B1) & 0xFFFFFFFFFFFFFFFF)
        z = base + (np.arange(1, n + 1, dtype=np.uint64) * _GOLDEN)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, stream: int, n: int) -> np.ndarray:
    return (_splitmix(seed, stream, n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed: int, stream: int, n: int) -> np.ndarray:
    m = (n + 1) // 2
    u1 = uniform(seed, stream, m)
    u2 = uniform(seed, stream + 1000003, m)
    u1 = np.maximum(u1, 1e-300)
    r = np.sqrt(-2.0 * np.log(u1))
    z = np.concatenate([r * np.cos(2.0 * np.pi * u2), r * np.sin(2.0 * np.pi * u2)])
    return z[:n]


@dataclass
class Light:
    right_radius: float = 1.0
    top_radius: float = 1.0
    position: tuple = (0.0, 0.0, 6.0)
    view_dir: tuple = (0.0, 0.0, -1.0)
    up_dir: tuple = (0.0, 1.0, 0.0)
    n: int = 8               # lightResWidth: rows of a sample's mask, along x_delt
    nh: int = 0              # lightResHeight (0: square, = n): columns, along y_delt

    @property
    def rows(self) -> int:
        return self.n

    @property
    def cols(self) -> int:
        return self.nh if self.nh else self.n


@dataclass
class Scene:
    W: int
    H: int
    pos: np.ndarray          # float32 [H*W, 4]
    nrm: np.ndarray          # float32 [H*W, 4]
    vtx: np.ndarray          # float32 [V, 4]
    idx: np.ndarray          # int32 [T, 3]
    light: Light
    bins: int
    esp: float = 1e-3
    cull: bool = False
    name: str = ""
    depth_plane: bool = False   # also test each triangle's own plane (occluders not between)
    meta: dict = field(default_factory=dict)

    @property
    def S(self) -> int:
        return self.W * self.H

    @property
    def T(self) -> int:
        return int(self.idx.shape[0])

    @property
    def V(self) -> int:
        return int(self.vtx.shape[0])


def receiver(W: int, H: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    jx = uniform(seed, 1, W * H) - 0.5
    jy = uniform(seed, 2, W * H) - 0.5
    ii = np.tile(np.arange(W, dtype=np.float64), H)
    jj = np.repeat(np.arange(H, dtype=np.float64), W)
    x = -8.0 + (ii + 0.5 + jx) * (16.0 / W)
    y = -8.0 + (jj + 0.5 + jy) * (16.0 / H)
    z = 0.3 * np.sin(x) * np.cos(y)
    n = np.stack([-0.3 * np.cos(x) * np.cos(y), 0.3 * np.sin(x) * np.sin(y), np.ones_like(x)], axis=1)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    p = np.stack([x, y, z], axis=1) + 1e-4 * n
    pos = np.ones((W * H, 4), dtype=np.float32)
    nrm = np.zeros((W * H, 4), dtype=np.float32)
    pos[:, :3] = p.astype(np.float32)
    nrm[:, :3] = n.astype(np.float32)
    return pos, nrm


def occluders(T: int, seed: int, sigma: float, zlo: float, zhi: float) -> tuple[np.ndarray, np.ndarray]:
    cx = -6.0 + 12.0 * uniform(seed, 11, T)
    cy = -6.0 + 12.0 * uniform(seed, 12, T)
    cz = zlo + (zhi - zlo) * uniform(seed, 13, T)
    c = np.stack([cx, cy, cz], axis=1)
    d = normal(seed, 21, 9 * T).reshape(T, 3, 3) * sigma
    v = (c[:, None, :] + d).reshape(3 * T, 3)
    vtx = np.ones((3 * T, 4), dtype=np.float32)
    vtx[:, :3] = v.astype(np.float32)
    idx = np.arange(3 * T, dtype=np.int32).reshape(T, 3)
    return vtx, idx


def make_scene(W: int, H: int, T: int, n: int, bins: int, seed: int, sigma: float = 0.15,
               zlo: float = 0.5, zhi: float = 3.0, radius: float = 1.0, esp: float = 1e-3,
               cull: bool = False, name: str = "") -> Scene:
    pos, nrm = receiver(W, H, seed)
    vtx, idx = occluders(T, seed, sigma, zlo, zhi)
    light = Light(right_radius=radius, top_radius=radius, n=n)
    return Scene(W=W, H=H, pos=pos, nrm=nrm, vtx=vtx, idx=idx, light=light, bins=bins, esp=esp,
                 cull=cull, name=name,
                 meta=dict(seed=seed, sigma=sigma, zlo=zlo, zhi=zhi, radius=radius))


# The workloads: small (CPU-oracle scale), HD single frame, large single frame.
PRESETS = {
    "small": dict(W=256, H=256, T=1024, n=8, bins=32, seed=1, sigma=0.15, zlo=0.5, zhi=3.0, radius=1.0),
    "hd": dict(W=1920, H=1080, T=200_000, n=16, bins=128, seed=2, sigma=0.1, zlo=0.5, zhi=3.0, radius=1.0),
    "large": dict(W=3840, H=2160, T=2_000_000, n=32, bins=256, seed=3, sigma=0.05, zlo=0.2, zhi=4.0,
                  radius=2.0),
}


def preset(name: str, **over) -> Scene:
    kw = dict(PRESETS[name])
    kw.update(over)
    return make_scene(name=name, **kw)


def batch_frame(k: int, s_range=(256 * 256, 1920 * 1080), t_range=(10_000, 500_000), ns=(8, 16),
                light_side=(0.5, 4.0), seed_base: int = 1000) -> Scene:
    """Frame k of the batched workload: an independent scene (seed seed_base + k)
    whose sample count is log-uniform in s_range (aspect uniform in [1, 16/9]),
    triangle count log-uniform in t_range, light grid N drawn from ns and light
    side uniform in light_side; occluders as in the HD frame (sigma 0.1,
    heights in [0.5, 3]).  bins = 0: left to the autotuner."""
    seed = seed_base + k
    u = uniform(seed, 31, 5)
    S = float(np.exp(np.log(s_range[0]) + u[0] * (np.log(s_range[1]) - np.log(s_range[0]))))
    aspect = 1.0 + u[1] * (16.0 / 9.0 - 1.0)
    W = max(1, int(round(np.sqrt(S * aspect))))
    H = max(1, int(round(S / W)))
    T = int(round(np.exp(np.log(t_range[0]) + u[2] * (np.log(t_range[1]) - np.log(t_range[0])))))
    n = int(ns[min(int(u[3] * len(ns)), len(ns) - 1)])
    side = light_side[0] + u[4] * (light_side[1] - light_side[0])
    s = make_scene(W, H, T, n=n, bins=0, seed=seed, sigma=0.1, zlo=0.5, zhi=3.0, radius=side / 2.0,
                   name=f"batch{k}")
    return s


# ---- meshes for the G-buffer rasteriser ------------------------------------

def look_at(eye, center, up) -> np.ndarray:
    """gluLookAt view matrix (out = M @ v), float64."""
    e, c, u = (np.asarray(v, np.float64) for v in (eye, center, up))
    f = c - e
    f /= np.linalg.norm(f)
    s = np.cross(f, u)
    s /= np.linalg.norm(s)
    uu = np.cross(s, f)
    m = np.eye(4)
    m[0, :3], m[1, :3], m[2, :3] = s, uu, -f
    m[:3, 3] = -m[:3, :3] @ e
    return m


def perspective(fovy_deg: float, aspect: float, near: float, far: float) -> np.ndarray:
    """gluPerspective projection matrix (out = M @ v), float64."""
    f = 1.0 / np.tan(np.radians(fovy_deg) / 2.0)
    m = np.zeros((4, 4))
    m[0, 0], m[1, 1] = f / aspect, f
    m[2, 2], m[2, 3] = (far + near) / (near - far), 2.0 * far * near / (near - far)
    m[3, 2] = -1.0
    return m


@dataclass
class MeshScene:
    """Triangle meshes in the MeshManager vertex layout (8 floats: position,
    texcoord, normal) with per-triangle materials, a camera and an area light.
    Triangles [0, n_receiver) are the receiver surface (the app's mesh 0, which
    it leaves out of the shadow model, MeshManager.cpp:43); the rest occlude."""
    W: int
    H: int
    vtx: np.ndarray            # float32 [V, 8]
    idx: np.ndarray            # uint32 [T, 3]
    tri_material: np.ndarray   # int32 [T]
    materials: np.ndarray      # float32 [M, 10]: Ka, Kd, Ks, shininess
    model: np.ndarray          # 4x4
    view_proj: np.ndarray      # 4x4
    eye: tuple
    n_receiver: int
    light: Light

    @property
    def T(self) -> int:
        return int(self.idx.shape[0])


def mesh_scene(W: int, H: int, grid: int = 48, T: int = 1500, seed: int = 5, sigma: float = 0.15,
               eye=(0.0, -13.0, 11.0), center=(0.0, 0.0, 0.0), fovy: float = 50.0, near: float = 0.5,
               far: float = 100.0, n: int = 8) -> MeshScene:
    """A height-field receiver (z = 0.3 sin x cos y over [-8, 8]^2, grid x grid
    cells, analytic normals) and T occluder triangles (the soup of occluders()
    with face normals) seen by a perspective camera; light as make_scene's."""
    xs = np.linspace(-8.0, 8.0, grid + 1)
    X, Y = np.meshgrid(xs, xs)
    Z = 0.3 * np.sin(X) * np.cos(Y)
    N = np.stack([-0.3 * np.cos(X) * np.cos(Y), 0.3 * np.sin(X) * np.sin(Y), np.ones_like(X)], axis=-1)
    N /= np.linalg.norm(N, axis=-1, keepdims=True)
    rv = np.zeros(((grid + 1) ** 2, 8), np.float64)
    rv[:, 0], rv[:, 1], rv[:, 2] = X.ravel(), Y.ravel(), Z.ravel()
    rv[:, 5:8] = N.reshape(-1, 3)
    i = np.arange(grid)
    a = (i[:, None] * (grid + 1) + i[None, :]).ravel()
    quads = np.stack([a, a + 1, a + grid + 2, a + grid + 1], axis=1)
    ridx = np.concatenate([quads[:, [0, 1, 2]], quads[:, [0, 2, 3]]])
    ov, oi = occluders(T, seed, sigma, 0.5, 3.0)
    tri = ov[:, :3].astype(np.float64).reshape(-1, 3, 3)
    fn = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    fn /= np.maximum(np.linalg.norm(fn, axis=1, keepdims=True), 1e-30)
    sv = np.zeros((3 * T, 8), np.float64)
    sv[:, :3] = tri.reshape(-1, 3)
    sv[:, 5:8] = np.repeat(fn, 3, axis=0)
    vtx = np.concatenate([rv, sv]).astype(np.float32)
    idx = np.concatenate([ridx, oi.astype(np.int64) + rv.shape[0]]).astype(np.uint32)
    mat = np.concatenate([np.zeros(len(ridx), np.int32), np.ones(T, np.int32)])
    materials = np.array([[0.1, 0.1, 0.1, 0.6, 0.6, 0.55, 0.2, 0.2, 0.2, 16.0],
                          [0.1, 0.05, 0.05, 0.7, 0.2, 0.2, 0.5, 0.5, 0.5, 32.0]], np.float32)
    vp = perspective(fovy, W / H, near, far) @ look_at(eye, center, (0.0, 0.0, 1.0))
    return MeshScene(W=W, H=H, vtx=vtx, idx=idx, tri_material=mat, materials=materials, model=np.eye(4),
                     view_proj=vp, eye=tuple(eye), n_receiver=len(ridx), light=Light(n=n))


def shadow_scene(ms: MeshScene, g0: np.ndarray, g1: np.ndarray, bins: int = 32, cull: bool = False) -> Scene:
    """The shadow pipeline's input for a rasterised view: samples = the
    G-buffer's world positions and normals, occluders = the mesh triangles
    after the receiver, as xyz float4 vertices."""
    occ = ms.idx[ms.n_receiver:]
    used = ms.vtx[occ.reshape(-1), :3]
    vtx = np.ones((used.shape[0], 4), np.float32)
    vtx[:, :3] = used
    idx = np.arange(used.shape[0], dtype=np.int32).reshape(-1, 3)
    return Scene(W=ms.W, H=ms.H, pos=np.ascontiguousarray(g0, np.float32), nrm=np.ascontiguousarray(g1, np.float32),
                 vtx=vtx, idx=idx, light=ms.light, bins=bins, cull=cull, name="raster")
