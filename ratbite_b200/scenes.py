"""Seeded synthetic scenes in the renderer's upload format.

A scene here is the data ratbite's RenderingInterface would hand to the
drop-in: meshes of submeshes placed by instances, one material record per
submesh (MaterialData carries its submesh's index and attribute buffers,
src/core/rendering_interface.cpp:47-290), emissive triangles cut out of their
submesh into emissive subsets (src/core/scene.cpp:485-631), and the camera /
launch parameters (src/core/rendering_interface.cpp:623-668). Everything is
camera-relative with the camera at the origin.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi


class PCG32:
    """PCG-XSH-RR 32-bit generator (O'Neill 2014); the seed is recorded with
    each scene so the same scene can be regenerated anywhere."""

    MULT = 6364136223846793005
    MASK = (1 << 64) - 1

    def __init__(self, seed: int, stream: int = 54):
        self.state = 0
        self.inc = ((stream << 1) | 1) & self.MASK
        self.next_u32()
        self.state = (self.state + seed) & self.MASK
        self.next_u32()

    def next_u32(self) -> int:
        old = self.state
        self.state = (old * self.MULT + self.inc) & self.MASK
        xorshifted = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xorshifted >> rot) | (xorshifted << ((-rot) & 31))) & 0xFFFFFFFF

    def uniform(self, lo=0.0, hi=1.0) -> float:
        return lo + (hi - lo) * (self.next_u32() / 4294967296.0)


def oct_encode(n: np.ndarray) -> np.ndarray:
    """Octahedral encoding of unit vectors to float2, the encoding the
    reference uses for the NORMAL vertex attribute
    (src/core/rendering_interface.cpp:217-229). float32 throughout."""
    n = n.astype(np.float32)
    s = (np.abs(n[:, 0]) + np.abs(n[:, 1]) + np.abs(n[:, 2])).astype(np.float32)
    p = (n[:, :2] * (np.float32(1.0) / s)[:, None]).astype(np.float32)
    sign = np.where(p >= 0, np.float32(1.0), np.float32(-1.0)).astype(np.float32)
    folded = ((np.float32(1.0) - np.abs(p[:, ::-1])) * sign).astype(np.float32)
    return np.where((n[:, 2] <= 0)[:, None], folded, p).astype(np.float32)


def frame_encode(normals: np.ndarray, tangents: np.ndarray) -> np.ndarray:
    """Tangent frames as unit quaternions (x, y, z, w), the encoding the
    reference uses for the FRAME vertex attribute
    (src/core/rendering_interface.cpp:258-284): the rotation of the matrix
    with columns (tangent, normal x tangent, normal) by the largest-diagonal
    method (Shoemake's matrix-to-quaternion conversion, as glm::quat_cast
    evaluates it), then signed so that w carries the sign of the tangent's
    handedness (tangent.w); a w of zero becomes +0 or -0. float32 throughout."""
    F = np.float32
    n = np.asarray(normals, F)[:, :3]
    t4 = np.asarray(tangents, F)
    t = t4[:, :3]
    b = np.stack([n[:, 1] * t[:, 2] - t[:, 1] * n[:, 2],
                  n[:, 2] * t[:, 0] - t[:, 2] * n[:, 0],
                  n[:, 0] * t[:, 1] - t[:, 0] * n[:, 1]], 1).astype(F)
    m = np.stack([t, b, n], 1)                      # m[:, column, row]
    d0, d1, d2 = m[:, 0, 0], m[:, 1, 1], m[:, 2, 2]
    four = np.stack([(d0 + d1) + d2, (d0 - d1) - d2, (d1 - d0) - d2, (d2 - d0) - d1], 1).astype(F)
    big = np.zeros(len(n), np.int64)
    best = four[:, 0].copy()
    for k in (1, 2, 3):                             # strictly greater, in order, as the reference's glm
        take = four[:, k] > best
        best = np.where(take, four[:, k], best)
        big = np.where(take, k, big)
    val = (np.sqrt((best + F(1.0)).astype(F)) * F(0.5)).astype(F)
    mult = (F(0.25) / val).astype(F)
    a12, a21 = m[:, 1, 2], m[:, 2, 1]
    a20, a02 = m[:, 2, 0], m[:, 0, 2]
    a01, a10 = m[:, 0, 1], m[:, 1, 0]
    cand = {   # (w, x, y, z) per largest index
        0: (val, (a12 - a21) * mult, (a20 - a02) * mult, (a01 - a10) * mult),
        1: ((a12 - a21) * mult, val, (a01 + a10) * mult, (a20 + a02) * mult),
        2: ((a20 - a02) * mult, (a01 + a10) * mult, val, (a12 + a21) * mult),
        3: ((a01 - a10) * mult, (a20 + a02) * mult, (a12 + a21) * mult, val),
    }
    q = np.zeros((len(n), 4), F)                    # x, y, z, w
    for k, (w, x, y, z) in cand.items():
        sel = big == k
        q[sel] = np.stack([x, y, z, w], 1).astype(F)[sel]
    tw = t4[:, 3]
    zero = q[:, 3] == 0.0
    q[zero, 3] = np.where(tw[zero] > 0.0, F(0.0), F(-0.0))
    flip = ~zero & (q[:, 3] * tw < 0.0)
    q[flip] = -q[flip]
    return q


def icosphere(subdiv: int):
    """Unit icosphere: subdivision s gives 20*4^s triangles."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
             (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, dtype=np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}
        new_faces = []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            new_faces += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = new_faces
    return np.array(verts), np.array(faces, dtype=np.int64)


@dataclass
class Submesh:
    vertices: np.ndarray          # (V, 4) float32
    indices: np.ndarray           # (T, 3) uint16/uint32
    material: int
    normals: np.ndarray | None = None   # (V, 3) float32 shading normals
    discarded: list = field(default_factory=list)
    texcoords: np.ndarray | None = None   # (V, 2) float32, texture coordinate set 1
    texcoords2: np.ndarray | None = None  # (V, 2) float32, set 2
    tangents: np.ndarray | None = None    # (V, 4) float32, xyz and handedness w (with normals: FRAME)


@dataclass
class Texture:
    """An image with its sampler (rb_texture): (H, W, 4) or (H, W) uint8
    texels, row 0 first; `srgb` decodes r, g, b (r of a one-channel image)
    with the sRGB curve (the reference sets it for base-colour textures)."""
    data: np.ndarray
    srgb: bool = False
    address: tuple = (abi.RB_TEXADDR_WRAP, abi.RB_TEXADDR_WRAP)
    filter: int = abi.RB_TEXFILTER_LINEAR

    def texel(self, x: int, y: int) -> np.ndarray:
        """Raw 8-bit texel (4 channels; a one-channel image as (r, 0, 0, 0),
        as the texture unit reads it)."""
        d = self.data
        if d.ndim == 2:
            return np.array([d[y, x], 0, 0, 0], np.uint8)
        return d[y, x]


@dataclass
class Material:
    base_color: tuple = (1.0, 1.0, 1.0)
    metalness: float = 0.0
    roughness: float = 1.0
    transmission: float = 0.0
    ior: float = 1.5
    sheen_color: tuple | None = None
    sheen_roughness: float = 0.0
    emissive: tuple | None = None
    bxdf: int = abi.RB_BXDF_COMPLEX_SURFACE
    ior_spectrum: int = 0
    absorp_spectrum: int = 0
    mf_roughness: float = 0.0
    # explicit MaterialData factor bits (e.g. from a glTF descriptor); None:
    # base colour, metalness and roughness always present, the rest by value
    factors: int | None = None
    alpha: float = 1.0
    alpha_cutoff: float = 0.0
    double_sided: bool = False
    # texture slot (abi.RB_TEXTURE_*) -> (index into Scene.textures, coordinate set 1 or 2)
    textures: dict = field(default_factory=dict)


@dataclass
class Scene:
    """Upload-ready scene; keeps every numpy buffer alive for the ctypes
    records that point into them."""
    name: str
    seed: int
    meshes: list            # list[list[Submesh]]
    instances: list         # list[(mesh, transform (3,4))]
    materials: list         # list[Material]; index = submesh material
    emissive: list          # list[dict(transform, tris (n,9) object space, world (n,9), prim, flux, material)]
    width: int = 256
    height: int = 256
    spp: int = 64
    max_depth: int = 8
    fov_deg: float = 70.0
    cam_u: tuple = (1.0, 0.0, 0.0)
    cam_v: tuple = (0.0, 0.0, -1.0)
    cam_w: tuple = (0.0, 1.0, 0.0)
    textures: list = field(default_factory=list)   # list[Texture]
    _keep: list = field(default_factory=list)

    # ---- counts ---------------------------------------------------------
    def triangle_count(self) -> int:
        n = sum(len(e["prim"]) for e in self.emissive)
        for mesh_idx, _ in self.instances:
            n += sum(len(sm.indices) for sm in self.meshes[mesh_idx])
        return n

    # ---- ABI records ----------------------------------------------------
    def _attr_buffer(self, sm: Submesh):
        """Interleaved vertex attributes in the reference's order
        (src/core/rendering_interface.cpp:209-235): a tangent-frame
        quaternion (16 bytes) when both normals and tangents are present,
        else an octahedral normal (8 bytes), then texture coordinate sets 1
        and 2 (8 bytes each), as present. Returns the buffer, the stride, the
        RB_ATTR_* bits and the byte offsets of (normal or frame, set 1, set 2)."""
        parts, bits, offs, off = [], 0, [0, 0, 0], 0
        if sm.normals is not None and sm.tangents is not None:
            parts.append(frame_encode(sm.normals, sm.tangents))
            bits |= abi.RB_ATTR_FRAME
            off = 16
        elif sm.normals is not None:
            parts.append(oct_encode(sm.normals).astype(np.float32))
            bits |= abi.RB_ATTR_NORMAL
            off = 8
        for k, (arr, bit) in enumerate(((sm.texcoords, abi.RB_ATTR_TEX_COORD_1),
                                        (sm.texcoords2, abi.RB_ATTR_TEX_COORD_2)), start=1):
            if arr is None:
                continue
            parts.append(np.asarray(arr, np.float32).reshape(-1, 2))
            bits |= bit
            offs[k] = off
            off += 8
        if not parts:
            return None, 0, 0, offs
        return np.ascontiguousarray(np.concatenate(parts, axis=1), dtype=np.float32), off, bits, offs

    def texture_records(self):
        """One rb_texture per Scene.textures entry."""
        recs = (abi.rb_texture * max(len(self.textures), 1))()
        for i, t in enumerate(self.textures):
            d = np.ascontiguousarray(t.data, np.uint8)
            self._keep.append(d)
            r = recs[i]
            r.height, r.width = d.shape[0], d.shape[1]
            r.format = abi.RB_TEXFMT_R8 if d.ndim == 2 else abi.RB_TEXFMT_RGBA8
            if d.ndim == 3 and d.shape[2] != 4:
                raise ValueError("textures are (H, W) or (H, W, 4) uint8")
            r.srgb = 1 if t.srgb else 0
            r.address_u, r.address_v = t.address
            r.filter = t.filter
            r.data = d.ctypes.data
        self._keep.append(recs)
        # an empty table still passes a valid pointer; its length is len(self.textures)
        return recs if self.textures else (abi.rb_texture * 0)()

    def material_records(self):
        """One rb_material per submesh material slot."""
        owner = {}
        for mesh in self.meshes:
            for sm in mesh:
                owner.setdefault(sm.material, sm)
        recs = (abi.rb_material * len(self.materials))()
        for i, m in enumerate(self.materials):
            r = recs[i]
            sm = owner.get(i)
            r.bxdf = m.bxdf
            r.double_sided = 1 if m.double_sided else 0
            r.sheen_present = 1 if m.sheen_color is not None else 0
            r.ior = m.ior
            r.mf_roughness = m.mf_roughness
            r.ior_spectrum = m.ior_spectrum
            r.absorp_spectrum = m.absorp_spectrum
            factors = abi.RB_FACTOR_BASE_COLOR | abi.RB_FACTOR_METALNESS | abi.RB_FACTOR_ROUGHNESS
            r.base_color = abi.F4(*m.base_color, 1.0)
            r.metalness = m.metalness
            r.roughness = m.roughness
            if m.transmission != 0.0:
                factors |= abi.RB_FACTOR_TRANSMISSION
                r.transmission = m.transmission
            if m.sheen_color is not None:
                factors |= abi.RB_FACTOR_SHEEN_COLOR | abi.RB_FACTOR_SHEEN_ROUGH
                r.sheen_color = abi.F3(*m.sheen_color)
                r.sheen_roughness = m.sheen_roughness
            if m.emissive is not None:
                factors |= abi.RB_FACTOR_EMISSION
                r.emissive = abi.F3(*m.emissive)
            if m.factors is not None:
                factors = m.factors
                r.base_color = abi.F4(*m.base_color, m.alpha)
                r.alpha_cutoff = m.alpha_cutoff
            r.factors = factors
            for slot, (tex, coord_set) in m.textures.items():
                r.textures |= 1 << slot
                r.texture_index[slot] = tex
                if coord_set == 2:
                    r.texcoord_sets |= 1 << slot
            if sm is not None:
                idx = np.ascontiguousarray(sm.indices)
                self._keep.append(idx)
                r.index_type = abi.RB_INDEX_U16 if idx.dtype == np.uint16 else abi.RB_INDEX_U32
                r.triangle_count = len(idx)
                r.indices = idx.ctypes.data
                attr, stride, bits, offs = self._attr_buffer(sm)
                r.attributes = bits
                r.attribute_stride = stride
                r.normal_offset, r.texcoord1_offset, r.texcoord2_offset = offs
                r.frame_offset = offs[0]
                r.vertex_count = len(sm.vertices)
                if attr is not None:
                    self._keep.append(attr)
                    r.attribute_data = attr.ctypes.data
        self._keep.append(recs)
        return recs

    def geometry_record(self):
        mesh_recs = (abi.rb_mesh * len(self.meshes))()
        for mi, mesh in enumerate(self.meshes):
            subs = (abi.rb_submesh * len(mesh))()
            for si, sm in enumerate(mesh):
                v = np.ascontiguousarray(sm.vertices, dtype=np.float32)
                idx = np.ascontiguousarray(sm.indices)
                disc = np.ascontiguousarray(np.array(sm.discarded, dtype=np.uint32))
                self._keep += [v, idx, disc]
                s = subs[si]
                s.material = sm.material
                s.index_type = abi.RB_INDEX_U16 if idx.dtype == np.uint16 else abi.RB_INDEX_U32
                s.triangle_count = len(idx)
                s.indices = idx.ctypes.data
                s.vertex_count = len(v)
                s.vertices = v.ctypes.data
                s.discarded_count = len(disc)
                s.discarded = disc.ctypes.data if len(disc) else None
            self._keep.append(subs)
            mesh_recs[mi].submesh_count = len(mesh)
            mesh_recs[mi].submeshes = subs
        inst = (abi.rb_instance * len(self.instances))()
        for i, (m, xf) in enumerate(self.instances):
            inst[i].mesh = m
            inst[i].transform = abi.F12(*np.asarray(xf, dtype=np.float32).reshape(12))
        em = (abi.rb_emissive_subset * len(self.emissive))()
        for i, e in enumerate(self.emissive):
            tri = np.ascontiguousarray(e["tris"], dtype=np.float32)
            self._keep.append(tri)
            em[i].transform = abi.F12(*np.asarray(e["transform"], dtype=np.float32).reshape(12))
            em[i].triangle_count = len(tri)
            em[i].vertices = tri.ctypes.data
        g = abi.rb_geometry()
        g.mesh_count = len(self.meshes)
        g.meshes = mesh_recs
        g.instance_count = len(self.instances)
        g.instances = inst
        g.emissive_subset_count = len(self.emissive)
        g.emissive_subsets = em
        self._keep += [mesh_recs, inst, em, g]
        return g

    def emissive_arrays(self):
        """Flat emissive-triangle inputs of the light-tree builder, in the
        reference's enumeration order (src/core/rendering_interface.cpp:1084-1160):
        world-space vertices, flux, material index, primitive index."""
        if not self.emissive:
            z = np.zeros((0,), np.float32)
            return z.reshape(0, 9), z, np.zeros(0, np.uint32), np.zeros(0, np.uint32)
        world = np.concatenate([e["world"] for e in self.emissive]).astype(np.float32)
        flux = np.concatenate([e["flux"] for e in self.emissive]).astype(np.float32)
        mat = np.concatenate([np.full(len(e["prim"]), e["material"], np.uint32) for e in self.emissive])
        prim = np.concatenate([np.asarray(e["prim"], np.uint32) for e in self.emissive])
        return (np.ascontiguousarray(world), np.ascontiguousarray(flux),
                np.ascontiguousarray(mat), np.ascontiguousarray(prim))

    def emissive_uvs(self):
        """Texture coordinates of the emissive triangles' vertices, (N, 6),
        in the order of emissive_arrays (zero where an emitter has none): the
        `uvs` of EmissiveTriangleLightData (src/core/light_tree_types.h:40-46)."""
        if not self.emissive:
            return np.zeros((0, 6), np.float32)
        return np.ascontiguousarray(np.concatenate(
            [np.asarray(e["uv"], np.float32).reshape(-1, 6) if e.get("uv") is not None
             else np.zeros((len(e["prim"]), 6), np.float32) for e in self.emissive]))

    def launch_record(self, width=None, height=None, max_depth=None):
        w = width or self.width
        h = height or self.height
        d = max_depth or self.max_depth
        l = abi.rb_launch()
        l.width, l.height = w, h
        # RenderContext inverse sizes and prepareDataForRendering's scales
        # (src/core/render_context.h:35, src/core/rendering_interface.cpp:638-640).
        l.inv_width = float(np.float32(1.0) / np.float32(w))
        l.inv_height = float(np.float32(1.0) / np.float32(h))
        t = math.tan(math.radians(self.fov_deg) * 0.5)
        l.perspective_scale_w = float(np.float32(t) * (np.float32(w) / np.float32(h)))
        l.perspective_scale_h = float(np.float32(t))
        l.max_path_depth = d
        l.max_reflected_depth = d
        l.max_transmitted_depth = d
        l.cam_u = abi.F3(*self.cam_u)
        l.cam_v = abi.F3(*self.cam_v)
        l.cam_w = abi.F3(*self.cam_w)
        l.dof_enabled = 0
        l.aperture = 0.01
        l.focus_distance = 1.0
        return l


IDENTITY = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0]], dtype=np.float32)


# ------------------------------------------------------------ at-scale scene
def _smooth_noise(p: np.ndarray, rng: np.random.Generator, octaves: int = 4) -> np.ndarray:
    """Seeded smooth noise: a sum of random-direction sinusoids per octave."""
    out = np.zeros(len(p))
    amp, freq = 1.0, 2.0
    for _ in range(octaves):
        for _ in range(3):
            k = rng.normal(size=3)
            k /= np.linalg.norm(k)
            out += amp * np.sin(freq * (p @ k) + rng.uniform(0, 2 * np.pi))
        amp *= 0.5
        freq *= 2.0
    return out / 3.0


def _torus(major: float, minor: float, nu: int, nv: int):
    u = np.linspace(0, 2 * np.pi, nu, endpoint=False)
    v = np.linspace(0, 2 * np.pi, nv, endpoint=False)
    uu, vv = np.meshgrid(u, v, indexing="ij")
    pos = np.stack([(major + minor * np.cos(vv)) * np.cos(uu), minor * np.sin(vv),
                    (major + minor * np.cos(vv)) * np.sin(uu)], -1).reshape(-1, 3)
    nrm = np.stack([np.cos(vv) * np.cos(uu), np.sin(vv), np.cos(vv) * np.sin(uu)], -1).reshape(-1, 3)
    i, j = np.meshgrid(np.arange(nu), np.arange(nv), indexing="ij")
    a = i * nv + j
    b = ((i + 1) % nu) * nv + j
    c = ((i + 1) % nu) * nv + (j + 1) % nv
    d = i * nv + (j + 1) % nv
    faces = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3), np.stack([a, c, d], -1).reshape(-1, 3)])
    return pos, nrm, faces


def _box(n: int):
    """Unit box [-1,1]^3 with each face split into n x n quads."""
    verts, faces, normals = [], [], []
    t = np.linspace(-1, 1, n + 1)
    for axis in range(3):
        for sign in (-1.0, 1.0):
            a, b = [k for k in range(3) if k != axis]
            uu, vv = np.meshgrid(t, t, indexing="ij")
            p = np.zeros((n + 1, n + 1, 3))
            p[..., axis] = sign
            p[..., a] = uu
            p[..., b] = vv
            base = sum(len(x) for x in verts)
            verts.append(p.reshape(-1, 3))
            nn = np.zeros(3)
            nn[axis] = sign
            normals.append(np.repeat(nn[None], (n + 1) ** 2, 0))
            i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
            q0 = base + i * (n + 1) + j
            q1 = q0 + (n + 1)
            q2 = q1 + 1
            q3 = q0 + 1
            f = np.concatenate([np.stack([q0, q1, q2], -1).reshape(-1, 3), np.stack([q0, q2, q3], -1).reshape(-1, 3)])
            if sign < 0:
                f = f[:, ::-1]
            faces.append(f)
    return np.concatenate(verts), np.concatenate(normals), np.concatenate(faces)


def _vertex_normals(pos, faces):
    n = np.zeros_like(pos)
    fn = np.cross(pos[faces[:, 1]] - pos[faces[:, 0]], pos[faces[:, 2]] - pos[faces[:, 0]])
    for k in range(3):
        np.add.at(n, faces[:, k], fn)
    return n / np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-20)


def sky_envmap(width: int = 1024, height: int = 512, seed: int = 7, sun_deg: float = 0.5,
               dynamic_range: float = 1e4) -> np.ndarray:
    """Lat-long RGBA float32 map (theta = pi * v, phi = 2 pi u): a vertical
    sky gradient plus a Gaussian sun lobe of `sun_deg` angular size whose peak
    is `dynamic_range` times the darkest sky texel."""
    rng = np.random.default_rng(seed)
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    theta = np.pi * v[:, None]
    phi = 2 * np.pi * u[None, :]
    up = np.cos(theta)                                  # z-up lat-long
    horizon = np.array([0.9, 0.85, 0.8])
    zenith = np.array([0.25, 0.45, 0.9])
    ground = np.array([0.12, 0.1, 0.08])
    t = np.clip(up, 0, 1)[..., None]
    sky = np.where(up[..., None] > 0, horizon * (1 - t) + zenith * t, ground * np.ones_like(t))
    sky = sky * np.ones((height, width, 1))
    sun_t, sun_p = np.deg2rad(rng.uniform(25, 60)), rng.uniform(0, 2 * np.pi)
    d = np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta) * np.ones_like(phi)], -1)
    s = np.array([np.sin(sun_t) * np.cos(sun_p), np.sin(sun_t) * np.sin(sun_p), np.cos(sun_t)])
    ang = np.arccos(np.clip(d @ s, -1, 1))
    sigma = np.deg2rad(sun_deg) / 2.0
    lo = sky.mean(-1).min()
    sun = dynamic_range * lo * np.exp(-0.5 * (ang / sigma) ** 2)
    img = np.zeros((height, width, 4), np.float32)
    img[..., :3] = (sky + sun[..., None] * np.array([1.0, 0.95, 0.85])).astype(np.float32)
    img[..., 3] = 1.0
    return img


def scale_scene(seed: int = 3, target_tris: int = 2_000_000, n_emitters: int = 4096, width: int = 1920,
                height: int = 1080, spp: int = 256, max_depth: int = 12, envmap_size=(1024, 512)) -> Scene:
    """The plain-method workload at scale: ~target_tris triangles from seeded
    instanced procedural meshes (noise-displaced spheres, boxes, tori, 16
    submeshes each), n_emitters emissive triangles with lognormal(0, 1.5)
    grey radiance, 256 materials with OpenPBR-style parameters (base_weight
    U[0.5,1] scaling the base colour, metalness Bernoulli(0.3), roughness
    U[0.02,1], transmission Bernoulli(0.15), fuzz_weight U[0,0.5] as the sheen
    colour scale; coat Bernoulli(0.2) is drawn but has no counterpart in the
    reference BxDF), and a sky + sun environment map. Camera at the origin
    looking down -z."""
    rng = np.random.default_rng(seed)
    n_sub = 16
    materials: list[Material] = []

    def surface_material():
        base_weight = rng.uniform(0.5, 1.0)
        color = tuple(float(np.float32(c * base_weight)) for c in rng.uniform(0.05, 0.95, 3))
        metal = 1.0 if rng.random() < 0.3 else 0.0
        trans = 1.0 if rng.random() < 0.15 else 0.0
        fuzz = rng.uniform(0.0, 0.5)
        _coat = rng.random() < 0.2
        return Material(base_color=color, metalness=metal, roughness=float(np.float32(rng.uniform(0.02, 1.0))),
                        transmission=trans, ior=1.5,
                        sheen_color=tuple(float(np.float32(fuzz)) for _ in range(3)) if fuzz > 0.05 else None,
                        sheen_roughness=float(np.float32(rng.uniform(0.2, 0.8))))

    # Base meshes: 5 displaced spheres, 4 displaced tori, 3 boxes; 16
    # submeshes each. A material record belongs to one submesh (it carries
    # that submesh's index and attribute buffers), so 12 x 16 = 192 surface
    # materials, + 1 ground + 63 emitter groups = 256.
    bases = []
    sv, sf = icosphere(5)                                # 20,480 triangles
    for k in range(5):
        disp = 1.0 + 0.12 * _smooth_noise(sv, rng)
        pos = sv * disp[:, None]
        bases.append((pos, _vertex_normals(pos, sf), sf))
    for k in range(4):
        tp, tn, tf = _torus(1.0, 0.35, 128, 64)           # 16,384 triangles
        disp = 0.06 * _smooth_noise(tp, rng)
        pos = tp + tn * disp[:, None]
        bases.append((pos, _vertex_normals(pos, tf), tf))
    for k in range(3):
        bp, bn, bf = _box(24)                             # 6,912 triangles
        disp = 0.03 * _smooth_noise(bp, rng)
        pos = bp + bn * disp[:, None]
        bases.append((pos, bn, bf))
    meshes = []
    for mi, (pos, nrm, faces) in enumerate(bases):
        parts = np.array_split(np.arange(len(faces)), n_sub)
        subs = []
        for si, part in enumerate(parts):
            used, inv = np.unique(faces[part].reshape(-1), return_inverse=True)
            v4 = np.concatenate([pos[used], np.zeros((len(used), 1))], 1).astype(np.float32)
            idx = inv.reshape(-1, 3).astype(np.uint32 if len(used) > 65535 else np.uint16)
            materials.append(surface_material())
            subs.append(Submesh(v4, idx, len(materials) - 1, normals=nrm[used].astype(np.float32)))
        meshes.append(subs)
    tri_per_mesh = [len(f) for _, _, f in bases]
    instances = []
    total = 0
    k = 0
    while total < target_tris:
        m = k % len(bases)
        k += 1
        scale = rng.uniform(0.3, 1.2)
        ang = rng.uniform(0, 2 * np.pi, 3)
        cx, cy, cz = np.cos(ang)
        sx, sy, sz = np.sin(ang)
        rot = (np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]]) @ np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
               @ np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]]))
        pos = np.array([rng.uniform(-14, 14), rng.uniform(-3, 5), rng.uniform(-40, -6)])
        xf = np.concatenate([rot * scale, pos[:, None]], 1).astype(np.float32)
        instances.append((m, xf))
        total += tri_per_mesh[m]
    # Ground: a large subdivided box slab.
    gp, gn, gf = _box(32)
    gpos = gp * np.array([40.0, 0.5, 40.0]) + np.array([0.0, -4.5, -25.0])
    gmat = len(materials)
    materials.append(Material(base_color=(0.35, 0.33, 0.3), metalness=0.0, roughness=0.8))
    gv = np.concatenate([gpos, np.zeros((len(gpos), 1))], 1).astype(np.float32)
    meshes.append([Submesh(gv, gf.astype(np.uint16), gmat)])
    instances.append((len(meshes) - 1, IDENTITY))
    # Emitters: 63 emissive submeshes sharing n_emitters small triangles,
    # radiance ~ lognormal(0, 1.5) grey per submesh.
    groups = np.array_split(np.arange(n_emitters), 63)
    emissive = []
    em_subs = []
    for e, grp in enumerate(groups):
        per = len(grp)
        rad = float(np.exp(rng.normal(0.0, 1.5)))
        materials.append(Material(base_color=(0.8, 0.8, 0.8), emissive=(rad, rad, rad)))
        mat = len(materials) - 1
        c = np.stack([rng.uniform(-16, 16, per), rng.uniform(5.0, 9.0, per), rng.uniform(-42, -4, per)], 1)
        s = rng.uniform(0.1, 0.4, (per, 1))
        a = c
        b = c + s * np.array([1.0, 0.0, 0.0])
        d = c + s * np.array([0.3, 0.0, 1.0])
        tris = np.concatenate([a, d, b], 1).astype(np.float32)     # normal points down (-y)
        v4 = np.concatenate([tris.reshape(-1, 3), np.zeros((3 * per, 1))], 1).astype(np.float32)
        idx = np.arange(3 * per, dtype=np.uint16).reshape(per, 3)
        em_subs.append(Submesh(v4, idx, mat, discarded=list(range(per))))
        area = 0.5 * np.linalg.norm(np.cross(tris[:, 3:6] - tris[:, :3], tris[:, 6:9] - tris[:, :3]).astype(np.float32), axis=1)
        flux = (np.float32(rad) * area.astype(np.float32) * np.float32(math.pi)).astype(np.float32)
        emissive.append(dict(transform=IDENTITY, tris=tris, world=tris.copy(), prim=list(range(per)),
                             flux=flux, material=mat, submesh=e))
    meshes.append(em_subs)
    instances.append((len(meshes) - 1, IDENTITY))
    sc = Scene(name="scale_scene", seed=seed, meshes=meshes, instances=instances, materials=materials,
               emissive=emissive, width=width, height=height, spp=spp, max_depth=max_depth)
    sc.envmap = sky_envmap(*envmap_size, seed=seed)
    return sc


def _quad(p0, p1, p2, p3):
    """Two triangles (p0,p1,p2), (p0,p2,p3); normal = (p1-p0)x(p2-p0)."""
    v = np.array([p0, p1, p2, p3], dtype=np.float32)
    v4 = np.concatenate([v, np.zeros((4, 1), np.float32)], axis=1)
    return v4, np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint16)


def blackbody_rgb(temperature_k: float, cie_xyz: np.ndarray) -> np.ndarray:
    """Linear sRGB of a blackbody at `temperature_k`, normalised to max 1,
    from Planck's law and the given 471-bin CIE 1931 tables. Used as the
    emitter's RGB factor: the reference has only RGB emission
    (src/kernels/pathtrace.cu:1216-1231)."""
    lam = np.arange(360, 831, dtype=np.float64) * 1e-9
    h, c, k = 6.62607015e-34, 2.99792458e8, 1.380649e-23
    spd = 1.0 / (lam ** 5 * (np.exp(h * c / (lam * k * temperature_k)) - 1.0))
    xyz = cie_xyz.astype(np.float64) @ spd
    m = np.array([[3.2404542, -1.5371385, -0.4985314],
                  [-0.9692660, 1.8760108, 0.0415560],
                  [0.0556434, -0.2040259, 1.0572252]])
    rgb = np.maximum(m @ xyz, 0.0)
    return rgb / rgb.max()


def cornell_box(seed: int = 1, cie_xyz: np.ndarray | None = None, light_scale: float = 12.0,
                subdiv: int = 3, width: int = 256, height: int = 256, spp: int = 64,
                max_depth: int = 8) -> Scene:
    """The small plain-method workload: procedural Cornell box, 5 walls (10
    triangles, albedo U[0.2,0.8]^3 from PCG32(seed)), one 0.25 m^2 emissive
    quad (6500 K blackbody as RGB), a metal icosphere (roughness 0.3, F0 from
    PCG32) and a dielectric icosphere (IOR 1.5, roughness 0.05), 1280
    triangles each at subdivision 3. Camera at the origin looking down -z."""
    rng = PCG32(seed)
    cz = -3.2          # box centre depth
    x0, x1, y0, y1, z0, z1 = -1.0, 1.0, -1.0, 1.0, cz - 1.0, cz + 1.0
    materials: list[Material] = []
    walls: list[Submesh] = []
    quads = [
        ((x0, y0, z1), (x1, y0, z1), (x1, y0, z0), (x0, y0, z0)),   # floor, normal +y
        ((x0, y1, z0), (x1, y1, z0), (x1, y1, z1), (x0, y1, z1)),   # ceiling, normal -y
        ((x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0)),   # back, normal +z
        ((x0, y0, z1), (x0, y0, z0), (x0, y1, z0), (x0, y1, z1)),   # left, normal +x
        ((x1, y0, z0), (x1, y0, z1), (x1, y1, z1), (x1, y1, z0)),   # right, normal -x
    ]
    for q in quads:
        albedo = tuple(rng.uniform(0.2, 0.8) for _ in range(3))
        materials.append(Material(base_color=albedo, metalness=0.0, roughness=1.0))
        v, i = _quad(*q)
        walls.append(Submesh(v, i, len(materials) - 1))
    # Emissive quad, 0.5 m x 0.5 m just below the ceiling, facing down.
    if cie_xyz is None:
        rgb = np.array([1.0, 0.97, 0.93])
    else:
        rgb = blackbody_rgb(6500.0, cie_xyz)
    emissive_rgb = tuple(float(np.float32(c * light_scale)) for c in rgb)
    ly = y1 - 1e-3
    lq = ((-0.25, ly, cz - 0.25), (0.25, ly, cz - 0.25), (0.25, ly, cz + 0.25), (-0.25, ly, cz + 0.25))
    materials.append(Material(base_color=(0.78, 0.78, 0.78), metalness=0.0, roughness=1.0, emissive=emissive_rgb))
    lv, li = _quad(*lq)
    light_sub = Submesh(lv, li, len(materials) - 1, discarded=[0, 1])
    walls.append(light_sub)

    sv, sf = icosphere(subdiv)
    spheres = []
    for (cx, cy, czz, r), kind in (((-0.45, -0.6, cz - 0.3, 0.4), "metal"), ((0.45, -0.6, cz + 0.35, 0.4), "glass")):
        if kind == "metal":
            f0 = tuple(rng.uniform(0.5, 1.0) for _ in range(3))
            materials.append(Material(base_color=f0, metalness=1.0, roughness=0.3))
        else:
            materials.append(Material(base_color=(1.0, 1.0, 1.0), metalness=0.0, roughness=0.05,
                                      transmission=1.0, ior=1.5))
        pos = (sv * r + np.array([cx, cy, czz])).astype(np.float32)
        v4 = np.concatenate([pos, np.zeros((len(pos), 1), np.float32)], axis=1)
        spheres.append([Submesh(v4, sf.astype(np.uint16), len(materials) - 1,
                                normals=sv.astype(np.float32))])

    # Emissive subset: the light quad's triangles cut out of the wall mesh.
    tris_obj = np.stack([lv[li[k], :3].reshape(9) for k in range(2)]).astype(np.float32)
    flux = []
    for k in range(2):
        a, b, c = tris_obj[k, 0:3], tris_obj[k, 3:6], tris_obj[k, 6:9]
        area2 = np.linalg.norm(np.cross((b - a).astype(np.float32), (c - a).astype(np.float32)).astype(np.float32))
        # scene.cpp:518-523,607: average factor * area * pi, in float32.
        f = np.float32((np.float32(emissive_rgb[0]) + np.float32(emissive_rgb[1]) + np.float32(emissive_rgb[2])) / np.float32(3.0))
        f = np.float32(f * (np.float32(area2) * np.float32(0.5) * np.float32(math.pi)))
        flux.append(f)
    emissive = [dict(transform=IDENTITY, tris=tris_obj, world=tris_obj.copy(), prim=[0, 1],
                     flux=np.array(flux, np.float32), material=light_sub.material)]

    meshes = [walls, spheres[0], spheres[1]]
    instances = [(0, IDENTITY), (1, IDENTITY), (2, IDENTITY)]
    return Scene(name="cornell_box", seed=seed, meshes=meshes, instances=instances,
                 materials=materials, emissive=emissive, width=width, height=height,
                 spp=spp, max_depth=max_depth)


def _checker(n: int, cells: int, a, b, alpha_a: int = 255, alpha_b: int = 255) -> np.ndarray:
    """(n, n, 4) uint8 checkerboard of `cells` x `cells` squares."""
    y, x = np.mgrid[0:n, 0:n]
    on = ((x * cells // n) + (y * cells // n)) % 2 == 0
    img = np.zeros((n, n, 4), np.uint8)
    img[on] = (*a, alpha_a)
    img[~on] = (*b, alpha_b)
    return img


def textured_cornell(seed: int = 1, cie_xyz: np.ndarray | None = None, light_scale: float = 12.0,
                     width: int = 128, height: int = 128, spp: int = 16, max_depth: int = 8) -> Scene:
    """Cornell box with material textures on every surface kind the shading
    step samples (src/kernels/pathtrace.cu:1217-1228, 1437-1560, 1640-1650):
    base colour (sRGB, nearest and bilinear filtering, wrap / mirror / clamp
    addressing, coordinates beyond [0, 1]), alpha cutout from the base-colour
    alpha, a normal map, metal-roughness, transmission, sheen colour and
    roughness read from texture coordinate set 2, a one-channel texture, and
    an emissive texture on the light (its flux scaled by the texture's mean
    emission). Procedural textures from PCG32(seed)."""
    rng = PCG32(seed)
    cz = -3.2
    x0, x1, y0, y1, z0, z1 = -1.0, 1.0, -1.0, 1.0, cz - 1.0, cz + 1.0
    n = 32
    yy, xx = np.mgrid[0:n, 0:n]
    # textures
    tex: list[Texture] = []

    def add(t: Texture) -> int:
        tex.append(t)
        return len(tex) - 1

    col = lambda: tuple(int(rng.uniform(40, 230)) for _ in range(3))
    t_floor = add(Texture(_checker(n, 8, col(), col()), srgb=True, filter=abi.RB_TEXFILTER_NEAREST))
    mr = np.zeros((n, n, 4), np.uint8)
    mr[..., 1] = (60 + 190 * (xx / (n - 1))).astype(np.uint8)           # roughness
    mr[..., 2] = np.where((yy // 8) % 2 == 0, 0, 200).astype(np.uint8)  # metalness stripes
    mr[..., 3] = 255
    t_mr = add(Texture(mr))
    t_back = add(Texture(_checker(n, 4, col(), col()), srgb=True,
                         address=(abi.RB_TEXADDR_MIRROR, abi.RB_TEXADDR_MIRROR)))
    ph = 2.0 * math.pi * 3.0 * xx / n
    nm = np.zeros((n, n, 4), np.uint8)
    nm[..., 0] = np.clip(127.5 + 100.0 * np.sin(ph), 0, 255).astype(np.uint8)
    nm[..., 1] = 128
    nm[..., 2] = np.clip(127.5 + 127.0 * np.sqrt(np.clip(1.0 - (100.0 / 127.5 * np.sin(ph)) ** 2, 0.0, 1.0)),
                         0, 255).astype(np.uint8)
    nm[..., 3] = 255
    t_normal = add(Texture(nm))
    t_cut = add(Texture(_checker(n, 6, col(), col(), 255, 0), srgb=True,
                        address=(abi.RB_TEXADDR_CLAMP, abi.RB_TEXADDR_CLAMP)))
    t_gray = add(Texture(((xx + yy) * (255 // (2 * n - 2))).astype(np.uint8), srgb=True))   # one channel
    shc = _checker(n, 2, col(), col())
    t_shc = add(Texture(shc))
    shr = np.zeros((n, n, 4), np.uint8)
    shr[..., 3] = (50 + 200 * (yy / (n - 1))).astype(np.uint8)
    t_shr = add(Texture(shr))
    tr = ((xx // 4) % 2 * 255).astype(np.uint8)
    t_tr = add(Texture(tr, address=(abi.RB_TEXADDR_WRAP, abi.RB_TEXADDR_CLAMP)))
    em = np.zeros((n, n, 4), np.uint8)
    em[..., 0] = (128 + 127 * np.cos(2 * math.pi * xx / n)).astype(np.uint8)
    em[..., 1] = 200
    em[..., 2] = (128 + 127 * np.sin(2 * math.pi * yy / n)).astype(np.uint8)
    em[..., 3] = 255
    t_em = add(Texture(em))

    materials: list[Material] = []
    walls: list[Submesh] = []
    S = abi
    quads = [
        (((x0, y0, z1), (x1, y0, z1), (x1, y0, z0), (x0, y0, z0)), 3.0,     # floor: checker (nearest) + metal-rough
         Material(base_color=(1.0, 1.0, 1.0), metalness=1.0, roughness=0.8,
                  textures={S.RB_TEXTURE_BASE_COLOR: (t_floor, 1), S.RB_TEXTURE_MET_ROUGH: (t_mr, 1)})),
        (((x0, y1, z0), (x1, y1, z0), (x1, y1, z1), (x0, y1, z1)), 1.0,     # ceiling: sheen textures on set 2
         Material(base_color=(0.7, 0.7, 0.7), sheen_color=(1.0, 1.0, 1.0), sheen_roughness=0.6,
                  textures={S.RB_TEXTURE_SHEEN_COLOR: (t_shc, 2), S.RB_TEXTURE_SHEEN_ROUGH: (t_shr, 2)})),
        (((x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0)), 2.5,     # back: mirror-addressed colour + normal map
         Material(base_color=(0.9, 0.9, 0.9),
                  textures={S.RB_TEXTURE_BASE_COLOR: (t_back, 1), S.RB_TEXTURE_NORMAL: (t_normal, 1)})),
        (((x0, y0, z1), (x0, y0, z0), (x0, y1, z0), (x0, y1, z1)), 1.0,     # left: one-channel colour texture
         Material(textures={S.RB_TEXTURE_BASE_COLOR: (t_gray, 1)})),
        (((x1, y0, z0), (x1, y0, z1), (x1, y1, z1), (x1, y1, z0)), 1.2,     # right: alpha cutout (clamp)
         Material(base_color=(1.0, 1.0, 1.0), factors=S.RB_FACTOR_BASE_COLOR | S.RB_FACTOR_CUTOFF, alpha=1.0,
                  alpha_cutoff=0.5, textures={S.RB_TEXTURE_BASE_COLOR: (t_cut, 1)})),
    ]
    quad_uv = lambda s: np.array([[0.0, 0.0], [s, 0.0], [s, s], [0.0, s]], np.float32)
    for q, scale, mat in quads:
        materials.append(mat)
        v, i = _quad(*q)
        uv = quad_uv(scale)
        walls.append(Submesh(v, i, len(materials) - 1, texcoords=uv - 0.13 * scale,
                             texcoords2=(uv * 0.5 + 0.25).astype(np.float32)))
    rgb = np.array([1.0, 0.97, 0.93]) if cie_xyz is None else blackbody_rgb(6500.0, cie_xyz)
    emissive_rgb = tuple(float(np.float32(c * light_scale)) for c in rgb)
    ly = y1 - 1e-3
    lq = ((-0.25, ly, cz - 0.25), (0.25, ly, cz - 0.25), (0.25, ly, cz + 0.25), (-0.25, ly, cz + 0.25))
    materials.append(Material(base_color=(0.78, 0.78, 0.78), emissive=emissive_rgb,
                              textures={S.RB_TEXTURE_EMISSION: (t_em, 1)}))
    lv, li = _quad(*lq)
    luv = quad_uv(2.0)
    light_sub = Submesh(lv, li, len(materials) - 1, discarded=[0, 1], texcoords=luv)
    walls.append(light_sub)

    sv, sf = icosphere(3)
    sph_uv = np.stack([np.arctan2(sv[:, 0], sv[:, 2]) / (2 * math.pi) + 0.5,
                       np.arccos(np.clip(sv[:, 1], -1.0, 1.0)) / math.pi], axis=1).astype(np.float32)
    spheres = []
    for (cx, cy, czz, r), kind in (((-0.45, -0.6, cz - 0.3, 0.4), "metal"), ((0.45, -0.6, cz + 0.35, 0.4), "glass")):
        if kind == "metal":
            materials.append(Material(base_color=(0.9, 0.8, 0.6), metalness=1.0, roughness=0.5,
                                      textures={S.RB_TEXTURE_BASE_COLOR: (t_back, 1), S.RB_TEXTURE_MET_ROUGH: (t_mr, 1)}))
        else:
            materials.append(Material(base_color=(1.0, 1.0, 1.0), metalness=0.0, roughness=0.05,
                                      transmission=1.0, ior=1.5,
                                      textures={S.RB_TEXTURE_TRANSMISSION: (t_tr, 1)}))
        pos = (sv * r + np.array([cx, cy, czz])).astype(np.float32)
        v4 = np.concatenate([pos, np.zeros((len(pos), 1), np.float32)], axis=1)
        spheres.append([Submesh(v4, sf.astype(np.uint16), len(materials) - 1, normals=sv.astype(np.float32),
                                texcoords=sph_uv)])

    # emissive subset: the light quad's triangles, their texture coordinates,
    # and flux = mean factor x mean texture emission x area x pi
    tris_obj = np.stack([lv[li[k], :3].reshape(9) for k in range(2)]).astype(np.float32)
    tri_uv = np.stack([luv[li[k]].reshape(6) for k in range(2)]).astype(np.float32)
    e = em.astype(np.float64) / 255.0
    mean_em = float(np.mean((e[..., 0] + e[..., 1] + e[..., 2]) * e[..., 3] / 3.0))
    flux = []
    for k in range(2):
        a, b, c = tris_obj[k, 0:3], tris_obj[k, 3:6], tris_obj[k, 6:9]
        area2 = np.linalg.norm(np.cross((b - a).astype(np.float32), (c - a).astype(np.float32)).astype(np.float32))
        f = np.float32((np.float32(emissive_rgb[0]) + np.float32(emissive_rgb[1]) + np.float32(emissive_rgb[2])) / np.float32(3.0))
        f = np.float32(f * np.float32(mean_em))
        flux.append(np.float32(f * (np.float32(area2) * np.float32(0.5) * np.float32(math.pi))))
    emissive = [dict(transform=IDENTITY, tris=tris_obj, world=tris_obj.copy(), prim=[0, 1],
                     flux=np.array(flux, np.float32), material=light_sub.material, uv=tri_uv)]
    meshes = [walls, spheres[0], spheres[1]]
    instances = [(0, IDENTITY), (1, IDENTITY), (2, IDENTITY)]
    return Scene(name="textured_cornell", seed=seed, meshes=meshes, instances=instances, materials=materials,
                 emissive=emissive, width=width, height=height, spp=spp, max_depth=max_depth, textures=tex)
