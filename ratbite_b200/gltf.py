"""glTF 2.0 scene ingest (.gltf with external or embedded buffers, .glb).

Restates the reference's loader (SceneData::loadModel / loadGLTF and
processGLTFNode, src/core/scene.cpp:14-656, on cgltf) so a glTF file yields
the same meshes, material descriptors, instances and emissive subsets:

* positions and normals go from glTF's +Y-up to the reference's frame as
  (x, y, z) -> (-x, z, y), tangents likewise with w kept (:411-441);
* node transforms: cgltf's local matrix (the matrix, or T * R * S composed as
  cgltf_node_transform_local does), coordinate-corrected column by column and
  accumulated down the node graph with glm's mat4 product order (:21-34);
* material descriptors follow the reference field by field, including its
  defaults and quirks (alpha mode and alpha cutoff are read only when the
  material has pbrMetallicRoughness; IOR 1.5 without KHR_materials_ior;
  sheen only when its colour is not black) (:227-342);
* emissive primitives: every triangle of a submesh with an emissive factor
  gets flux = mean(emissive) * |cross(e1, e2)| / 2 * pi, is cut from the
  submesh (discarded) when the flux is positive, and is instanced per node
  with its world-space vertices and |det| of the instance transform as flux
  correction (:487-633, :44-63).

* images (PNG, from files or buffer views; the reference refuses data: URIs
  too) decoded to the channel layout stb_image gives the reference, textures
  with their sampler's filter and wrap modes (:114-202), base-colour textures
  flagged sRGB (:240), texture indices and texture-coordinate sets per slot,
  texture coordinates of sets 0 and 1 (8/16-bit normalized or float);
* emissive triangles with an emission texture: the flux scaled by the mean
  emission of the texels the triangle covers in texture space, found with
  the reference's scanline rasterizer (src/core/sw_rast.h, :524-606).

All arithmetic is float32 in the reference's operation order. `to_scene`
turns a loaded model into a ratbite_b200.scenes.Scene for upload.
"""
from __future__ import annotations

import base64
import json
import math
import struct
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import abi

F = np.float32
_COMP = {5120: np.int8, 5121: np.uint8, 5122: np.int16, 5123: np.uint16, 5125: np.uint32, 5126: np.float32}
_NCOMP = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4, "MAT2": 4, "MAT3": 9, "MAT4": 16}


@dataclass
class Descriptor:
    """SceneData::MaterialDescriptor (src/core/scene.h:33-97), factor fields."""
    double_sided: bool = False
    sheen_present: bool = False
    ior: float = 1.5
    bc_factor_present: bool = False
    base_color: tuple = (0.0, 0.0, 0.0, 0.0)
    alpha_mode: int = 0                  # 0 none, 1 cutoff, 2 blend
    alpha_cutoff: float = 0.0
    met_factor_present: bool = False
    metalness: float = 0.0
    rough_factor_present: bool = False
    roughness: float = 0.0
    transmit_factor_present: bool = False
    transmission: float = 0.0
    sheen_color_present: bool = False
    sheen_color: tuple = (0.0, 0.0, 0.0)
    sheen_rough_present: bool = False
    sheen_roughness: float = 0.0
    emissive_present: bool = False
    emissive: tuple = (0.0, 0.0, 0.0)
    textures: int = 0                    # bit per descriptor slot used: bc, mr, nm, tr, shc, shr, em
    tex_index: tuple = (-1,) * 7         # texture index per descriptor slot (-1: none)
    tex_coord: tuple = (0,) * 7          # texture-coordinate set per slot


@dataclass
class GltfSubmesh:
    material: int
    indices: np.ndarray                  # (T*3,) uint16 / uint32
    vertices: np.ndarray                 # (V, 4) float32, w = 0
    normals: np.ndarray | None = None    # (V, 4) float32
    tangents: np.ndarray | None = None   # (V, 4) float32
    texcoords0: np.ndarray | None = None  # (V, 2) float32
    discarded: list = field(default_factory=list)
    texcoords1: np.ndarray | None = None  # (V, 2) float32, TEXCOORD_1


@dataclass
class EmissiveSubset:
    instance: int
    submesh: int
    flux_correction: float
    world: np.ndarray                    # (n, 9) float32
    local: np.ndarray                    # (n, 9) float32, model space of the mesh
    prim: np.ndarray                     # (n,) uint32
    flux: np.ndarray                     # (n,) float32
    uv: np.ndarray | None = None         # (n, 6) float32: the emission texture's coordinates


@dataclass
class Model:
    meshes: list                         # list[list[GltfSubmesh]]
    descriptors: list                    # list[Descriptor], one per primitive
    instances: list                      # list[(mesh, (3, 4) float32 transform)]
    emissive: list                       # list[EmissiveSubset]
    triangle_count: int = 0              # the reference's count (vertices of attribute 0)
    images: list = field(default_factory=list)     # list[(H, W, C) uint8], C = 1 or 4
    textures: list = field(default_factory=list)   # list[dict(image, srgb, filter, address)]


# ------------------------------------------------------------------ files
def _load_json_and_buffers(path: Path):
    data = path.read_bytes()
    bin_chunk = None
    if data[:4] == b"glTF":
        _, _, length = struct.unpack("<III", data[:12])
        pos, doc = 12, None
        while pos < length:
            clen, ctype = struct.unpack("<II", data[pos:pos + 8])
            chunk = data[pos + 8:pos + 8 + clen]
            if ctype == 0x4E4F534A:
                doc = json.loads(chunk.decode("utf-8"))
            elif ctype == 0x004E4942:
                bin_chunk = chunk
            pos += 8 + clen
    else:
        doc = json.loads(data.decode("utf-8"))
    buffers = []
    for i, b in enumerate(doc.get("buffers", [])):
        uri = b.get("uri")
        if uri is None:
            buffers.append(bin_chunk)
        elif uri.startswith("data:"):
            buffers.append(base64.b64decode(uri.split(",", 1)[1]))
        else:
            buffers.append((path.parent / uri).read_bytes())
    return doc, buffers


def _accessor(doc, buffers, index):
    """(count, ncomp, dtype, base byte offset, stride, buffer bytes)."""
    a = doc["accessors"][index]
    view = doc["bufferViews"][a["bufferView"]]
    dt = np.dtype(_COMP[a["componentType"]])
    nc = _NCOMP[a["type"]]
    stride = view.get("byteStride") or dt.itemsize * nc
    base = view.get("byteOffset", 0) + a.get("byteOffset", 0)
    return a["count"], nc, dt, base, stride, buffers[view["buffer"]]


def _read(doc, buffers, index, ncomp=None):
    count, nc, dt, base, stride, buf = _accessor(doc, buffers, index)
    nc = ncomp or nc
    out = np.zeros((count, nc), dt)
    for i in range(count):
        out[i] = np.frombuffer(buf, dt, nc, base + i * stride)
    return out


# ------------------------------------------------------------------ images
def _png_decode(data: bytes):
    """PNG -> (H, W, C) uint8 with C = 1 for grey images and 4 otherwise, the
    channel layout stb_image returns for the reference's request (1 for a
    one-channel image, else 4: src/core/scene.cpp:137-139): grey+alpha as
    (g, g, g, a), RGB with alpha 255, palettes expanded (with tRNS alpha),
    16-bit samples reduced to their high byte, 1/2/4-bit grey scaled to
    0..255, a tRNS colour key (compared at the file's depth) as alpha 0 of a
    4-channel image. Interlaced images are not read."""
    import zlib
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("only PNG images are read")
    pos, idat, plte, trns = 8, [], None, None
    w = h = depth = ctype = None
    while pos < len(data):
        n, kind = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        if kind == b"IHDR":
            w, h, depth, ctype, _, _, interlace = struct.unpack(">IIBBBBB", body)
            if interlace:
                raise ValueError("interlaced PNG images are not read")
        elif kind == b"PLTE":
            plte = np.frombuffer(body, np.uint8).reshape(-1, 3)
        elif kind == b"tRNS":
            trns = body
        elif kind == b"IDAT":
            idat.append(body)
        elif kind == b"IEND":
            break
        pos += 12 + n
    chans = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
    bits = depth * chans
    stride = (w * bits + 7) // 8
    bpp = max(1, bits // 8)
    raw = np.frombuffer(zlib.decompress(b"".join(idat)), np.uint8)
    if len(raw) < h * (stride + 1):
        raise ValueError("truncated PNG image data")
    out = np.zeros((h, stride), np.uint8)
    prev = np.zeros(stride, np.int64)
    for y in range(h):
        row = raw[y * (stride + 1):(y + 1) * (stride + 1)]
        f, line = int(row[0]), row[1:].astype(np.int64)
        if f == 0:
            cur = line
        elif f == 1:                                         # Sub: a running sum per byte lane
            cur = np.zeros(stride, np.int64)
            for k in range(min(bpp, stride)):
                cur[k::bpp] = np.cumsum(line[k::bpp]) & 255
        elif f == 2:
            cur = (line + prev) & 255
        elif f in (3, 4):                                    # Average / Paeth: sequential along the row
            ln, up, cu = line.tolist(), prev.tolist(), [0] * stride
            for x in range(stride):
                a = cu[x - bpp] if x >= bpp else 0
                b = up[x]
                if f == 3:
                    p = (a + b) >> 1
                else:
                    c = up[x - bpp] if x >= bpp else 0
                    pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                    p = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
                cu[x] = (ln[x] + p) & 255
            cur = np.asarray(cu, np.int64)
        else:
            raise ValueError("bad PNG filter type")
        out[y] = cur
        prev = cur
    wide = None
    if depth == 16:
        wide = out.reshape(h, w * chans, 2).astype(np.uint16)
        wide = (wide[..., 0] << 8) | wide[..., 1]
        samples = (wide >> 8).astype(np.uint8)                # stb_image keeps the high byte
        wide = wide.reshape(h, w, chans)
    elif depth == 8:
        samples = out.reshape(h, w * chans)
    else:                                                    # 1, 2, 4 bits: grey or palette indices
        per = 8 // depth
        unpacked = np.zeros((h, stride * per), np.uint8)
        for k in range(per):
            unpacked[:, k::per] = (out >> (8 - depth * (k + 1))) & ((1 << depth) - 1)
        samples = unpacked[:, :w]
        if ctype == 0:
            samples = (samples.astype(np.uint32) * (255 // ((1 << depth) - 1))).astype(np.uint8)
    px = samples.reshape(h, w, chans)
    if ctype == 3:
        rgb = plte[px[..., 0]]
        if trns is not None:
            alpha = np.full(len(plte), 255, np.uint8)
            alpha[:len(trns)] = np.frombuffer(trns, np.uint8)
            return np.concatenate([rgb, alpha[px[..., 0]][..., None]], axis=2)
        return np.concatenate([rgb, np.full((h, w, 1), 255, np.uint8)], axis=2)
    if ctype == 0 and trns is None:
        return px
    if ctype == 0:                # grey with a colour key: grey + alpha, read as 4 channels
        key = struct.unpack(">H", trns[:2])[0]
        if depth == 16:
            a = np.where(wide[..., 0] == key, 0, 255)
        else:
            a = np.where(px[..., 0] == (key & 255) * (255 // ((1 << depth) - 1)), 0, 255)
        g = px[..., 0]
        return np.stack([g, g, g, a.astype(np.uint8)], axis=2)
    if ctype == 4:
        g, a = px[..., 0], px[..., 1]
        return np.stack([g, g, g, a], axis=2)
    if ctype == 2:
        a = np.full((h, w), 255, np.uint8)
        if trns is not None:                                 # the colour key, compared at full depth
            k = struct.unpack(">HHH", trns[:6])
            full = wide if depth == 16 else px.astype(np.uint16)
            if depth == 8:
                k = [v & 255 for v in k]
            a = np.where((full[..., 0] == k[0]) & (full[..., 1] == k[1]) & (full[..., 2] == k[2]), 0, 255)
            a = a.astype(np.uint8)
        return np.concatenate([px, a[..., None]], axis=2)
    return px


# --------------------------------------------------- emissive-texture flux
def _draw_triangle_2d(p0, p1, p2, visit):
    """The reference's scanline rasterizer (SoftwareRasterization::
    drawTriangle2D, src/core/sw_rast.h, sample point (0.5, 0.5)) in float32:
    visit(x, y) for every texel whose sample point the triangle covers."""
    half = F(0.5)
    vs = [p0, p1, p2]
    if vs[0][1] < vs[1][1]:
        vs[0], vs[1] = vs[1], vs[0]
    if vs[1][1] < vs[2][1]:
        vs[1], vs[2] = vs[2], vs[1]
    if vs[0][1] < vs[1][1]:
        vs[0], vs[1] = vs[1], vs[0]

    def scan(lx, rx, y):
        for x in range(lx, rx + 1):
            visit(x, y)

    def bottom_flat(v0, v1, v2):
        v0x, v0y = v0
        v1x, v1y = v1
        v2x, v2y = v2
        if v1x > v2x:
            v1x, v2x, v1y, v2y = v2x, v1x, v2y, v1y
        inv_l = F(F(v1x - v0x) / F(v0y - v1y))
        inv_r = F(F(v2x - v0x) / F(v0y - v2y))
        to_sample = F(v0y - F(F(np.floor(F(v0y - half))) + half))
        cl = F(v0x + F(inv_l * to_sample))
        cr = F(v0x + F(inv_r * to_sample))
        top = int(np.floor(F(v0y + F(F(1.0) - half))))
        bot = int(np.floor(F(v1y + F(F(1.0) - half))))
        for y in range(top - 1, bot - 1, -1):
            scan(int(np.floor(F(cl + F(F(1.0) - half)))), int(np.floor(F(cr + F(F(1.0) - half)))) - 1, y)
            cl = F(cl + inv_l)
            cr = F(cr + inv_r)

    def top_flat(v0, v1, v2):
        v2x, v2y = v2
        v0x, v0y = v0
        v1x, v1y = v1
        if v0x > v1x:
            v0x, v1x, v0y, v1y = v1x, v0x, v1y, v0y
        inv_l = F(F(v0x - v2x) / F(v0y - v2y))
        inv_r = F(F(v1x - v2x) / F(v1y - v2y))
        to_sample = F(F(F(np.ceil(F(v2y - half))) + half) - v2y)
        cl = F(v2x + F(inv_l * to_sample))
        cr = F(v2x + F(inv_r * to_sample))
        top = int(np.floor(F(v1y + F(F(1.0) - half))))
        bot = int(np.floor(F(v2y + F(F(1.0) - half))))
        for y in range(bot, top):
            scan(int(np.floor(F(cl + F(F(1.0) - half)))), int(np.floor(F(cr + F(F(1.0) - half)))) - 1, y)
            cl = F(cl + inv_l)
            cr = F(cr + inv_r)

    (v0x, v0y), (v1x, v1y), (v2x, v2y) = vs
    if v1y == v2y:
        bottom_flat(vs[0], vs[1], vs[2])
    elif v0y == v1y:
        top_flat(vs[0], vs[1], vs[2])
    else:
        v3 = (F(v0x + F(F(v2x - v0x) * F(F(v1y - v0y) / F(v2y - v0y)))), v1y)
        bottom_flat(vs[0], vs[1], v3)
        top_flat(vs[1], v3, vs[2])


def _emissive_texture_scale(image: np.ndarray, address: tuple, uvs) -> float:
    """Mean emission of an emissive texture over a triangle's texture
    footprint, as the reference computes it for the light tree's flux
    (src/core/scene.cpp:524-606): texels whose sample point the triangle
    covers (in texel units), each (r + g + b) * a / 3 of its raw 8-bit values
    (no sRGB decode), addressed by the texture's modes; when no texel centre
    is covered, the texels at the three vertices. A float64 mean."""
    h, w = image.shape[:2]
    if image.ndim != 3 or image.shape[2] != 4:
        raise ValueError("emissive textures must have 4 channels")
    tex = [(F(F(u) * F(w)), F(F(v) * F(h))) for u, v in uvs]
    acc = [0.0, 0]

    def axis(i, n, mode):
        if mode == abi.RB_TEXADDR_WRAP:
            i = i if i >= 0 else i + n * ((-i - 1) // n + 1)
            return i % n
        if mode == abi.RB_TEXADDR_CLAMP:
            return min(max(0, i), n - 1)
        if mode == abi.RB_TEXADDR_MIRROR:
            i = i if i >= 0 else i + n * ((-i - 1) // n + 2)
            even = (i // n) % 2 == 0
            i = i % n
            return n - 1 - i if even else i
        return 0

    def visit(x, y):
        x, y = axis(int(x), w, address[0]), axis(int(y), h, address[1])
        r, g, b, a = (F(F(image[y, x, k]) / F(255.0)) for k in range(4))
        acc[0] += float(F(F(F(F(r + g) + b) * a) / F(3.0)))
        acc[1] += 1

    with np.errstate(divide="ignore", invalid="ignore"):      # flat edges: slopes unused
        _draw_triangle_2d(tex[0], tex[1], tex[2], visit)
    if acc[1] == 0:
        for tx, ty in tex:
            visit(int(tx), int(ty))
    return acc[0] / acc[1]


# --------------------------------------------------------------- matrices
def _local_matrix(node) -> np.ndarray:
    """cgltf_node_transform_local: 16 floats, column-major."""
    if "matrix" in node:
        return np.asarray(node["matrix"], F)
    tx, ty, tz = (F(v) for v in node.get("translation", (0.0, 0.0, 0.0)))
    qx, qy, qz, qw = (F(v) for v in node.get("rotation", (0.0, 0.0, 0.0, 1.0)))
    sx, sy, sz = (F(v) for v in node.get("scale", (1.0, 1.0, 1.0)))
    one, two = F(1.0), F(2.0)
    m = np.zeros(16, F)
    m[0] = (one - two * qy * qy - two * qz * qz) * sx
    m[1] = (two * qx * qy + two * qz * qw) * sx
    m[2] = (two * qx * qz - two * qy * qw) * sx
    m[4] = (two * qx * qy - two * qz * qw) * sy
    m[5] = (one - two * qx * qx - two * qz * qz) * sy
    m[6] = (two * qy * qz + two * qx * qw) * sy
    m[8] = (two * qx * qz + two * qy * qw) * sz
    m[9] = (two * qy * qz - two * qx * qw) * sz
    m[10] = (one - two * qx * qx - two * qy * qy) * sz
    m[12], m[13], m[14], m[15] = tx, ty, tz, one
    return m


def _corrected(lm: np.ndarray) -> np.ndarray:
    """The coordinate-corrected local transform as 4 columns of 4 (:27-32)."""
    c0, c1, c2, c3 = lm[0:4], lm[4:8], lm[8:12], lm[12:16]
    return np.array([[c0[0], -c0[2], -c0[1], -c0[3]],
                     [-c2[0], c2[2], c2[1], c2[3]],
                     [-c1[0], c1[2], c1[1], c1[3]],
                     [-c3[0], c3[2], c3[1], c3[3]]], F)


def _mat4_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """glm mat4 * mat4 on column arrays: result[j] = ((a0*b[j][0] + a1*b[j][1]) + a2*b[j][2]) + a3*b[j][3]."""
    r = np.zeros((4, 4), F)
    for j in range(4):
        r[j] = ((a[0] * b[j][0] + a[1] * b[j][1]) + a[2] * b[j][2]) + a[3] * b[j][3]
    return r


def _mat4_vec4(m: np.ndarray, v: np.ndarray) -> np.ndarray:
    """glm mat4 * vec4: (m0*v0 + m1*v1) + (m2*v2 + m3*v3)."""
    return (m[0] * v[0] + m[1] * v[1]) + (m[2] * v[2] + m[3] * v[3])


def _det3(m: np.ndarray) -> np.float32:
    """glm::determinant of mat3(m) (columns)."""
    return F(+ m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2])
             - m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2])
             + m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]))


def _cross(a, b):
    return np.array([a[1] * b[2] - b[1] * a[2], a[2] * b[0] - b[2] * a[0], a[0] * b[1] - b[0] * a[1]], F)


def _length(v):
    t = v * v
    return F(math.sqrt(F(F(t[0] + t[1]) + t[2])))


# -------------------------------------------------------------- materials
def _descriptor(mat) -> Descriptor:
    d = Descriptor()
    if mat is None:
        return d
    ext = mat.get("extensions", {})
    d.double_sided = bool(mat.get("doubleSided", False))
    d.ior = float(F(ext["KHR_materials_ior"].get("ior", 1.5))) if "KHR_materials_ior" in ext else 1.5
    tex = 0
    idx, crd = [-1] * 7, [0] * 7

    def use(slot, info):
        idx[slot] = int(info["index"])
        crd[slot] = int(info.get("texCoord", 0))

    if "pbrMetallicRoughness" in mat:
        pbr = mat["pbrMetallicRoughness"]
        if "baseColorTexture" in pbr:
            tex |= 1 << 0
            use(0, pbr["baseColorTexture"])
        bc = [float(F(v)) for v in pbr.get("baseColorFactor", (1.0, 1.0, 1.0, 1.0))]
        if bc != [1.0, 1.0, 1.0, 1.0]:
            d.bc_factor_present = True
            d.base_color = tuple(bc)
        mode = mat.get("alphaMode", "OPAQUE")
        d.alpha_mode = 1 if mode == "MASK" else (2 if mode == "BLEND" else 0)
        d.alpha_cutoff = float(F(mat.get("alphaCutoff", 0.5)))
        met = float(F(pbr.get("metallicFactor", 1.0)))
        if met != 1.0:
            d.met_factor_present, d.metalness = True, met
        rough = float(F(pbr.get("roughnessFactor", 1.0)))
        if rough != 1.0:
            d.rough_factor_present, d.roughness = True, rough
        if "metallicRoughnessTexture" in pbr:
            tex |= 1 << 1
            use(1, pbr["metallicRoughnessTexture"])
    if "KHR_materials_transmission" in ext:
        tr = ext["KHR_materials_transmission"]
        if "transmissionTexture" in tr:
            tex |= 1 << 3
            use(3, tr["transmissionTexture"])
        f = float(F(tr.get("transmissionFactor", 0.0)))
        if f != 0.0:
            d.transmit_factor_present, d.transmission = True, f
    if "normalTexture" in mat:
        tex |= 1 << 2
        use(2, mat["normalTexture"])
    if "KHR_materials_sheen" in ext:
        sh = ext["KHR_materials_sheen"]
        col = [float(F(v)) for v in sh.get("sheenColorFactor", (0.0, 0.0, 0.0))]
        if col != [0.0, 0.0, 0.0]:
            d.sheen_present = True
            if col != [1.0, 1.0, 1.0]:
                d.sheen_color_present, d.sheen_color = True, tuple(col)
            d.sheen_rough_present = True
            d.sheen_roughness = float(F(sh.get("sheenRoughnessFactor", 0.0)))
            if "sheenColorTexture" in sh:
                tex |= 1 << 4
                use(4, sh["sheenColorTexture"])
            if "sheenRoughnessTexture" in sh:
                tex |= 1 << 5
                use(5, sh["sheenRoughnessTexture"])
    em = [F(v) for v in mat.get("emissiveFactor", (0.0, 0.0, 0.0))]
    if not (em[0] == 0.0 and em[1] == 0.0 and em[2] == 0.0):
        d.emissive_present = True
        if "KHR_materials_emissive_strength" in ext:
            s = F(ext["KHR_materials_emissive_strength"].get("emissiveStrength", 1.0))
            em = [e * s for e in em]
        d.emissive = tuple(float(e) for e in em)
        if "emissiveTexture" in mat:
            tex |= 1 << 6
            use(6, mat["emissiveTexture"])
    d.textures = tex
    d.tex_index, d.tex_coord = tuple(idx), tuple(crd)
    return d


# ---------------------------------------------------------------- loading
def load(path) -> Model:
    """Loads a .gltf / .glb file as the reference's loadModel does (identity
    model transform)."""
    path = Path(path)
    doc, buffers = _load_json_and_buffers(path)
    if not doc.get("meshes"):
        raise ValueError("model contains no meshes")
    images = []
    for im in doc.get("images", []):
        uri = im.get("uri")
        if uri is not None:
            if uri.startswith("data:"):
                raise ValueError("base64 image data is not supported (nor by the reference)")
            from urllib.parse import unquote
            blob = (path.parent / unquote(uri)).read_bytes()
        else:
            view = doc["bufferViews"][im["bufferView"]]
            off = view.get("byteOffset", 0)
            blob = buffers[view["buffer"]][off:off + view["byteLength"]]
        images.append(_png_decode(blob))
    wrap = {10497: abi.RB_TEXADDR_WRAP, 33071: abi.RB_TEXADDR_CLAMP, 33648: abi.RB_TEXADDR_MIRROR}
    textures = []
    for t in doc.get("textures", []):
        filt, ax, ay = abi.RB_TEXFILTER_LINEAR, abi.RB_TEXADDR_WRAP, abi.RB_TEXADDR_WRAP
        if "sampler" in t:
            smp = doc["samplers"][t["sampler"]]
            mag = smp.get("magFilter")
            filt = abi.RB_TEXFILTER_NEAREST if mag == 9728 else abi.RB_TEXFILTER_LINEAR
            ax = wrap.get(smp.get("wrapS", 10497), ax)
            ay = wrap.get(smp.get("wrapT", 10497), ay)
        textures.append(dict(image=int(t["source"]), srgb=False, filter=filt, address=(ax, ay)))
    descriptors, meshes, mesh_emissive = [], [], []
    for mesh in doc["meshes"]:
        subs, emis = [], []
        for j, prim in enumerate(mesh["primitives"]):
            if prim.get("mode", 4) != 4:
                continue                                   # only triangle lists
            mi = len(descriptors)
            mat = doc["materials"][prim["material"]] if "material" in prim else None
            d = _descriptor(mat)
            descriptors.append(d)
            if d.tex_index[0] >= 0:
                textures[d.tex_index[0]]["srgb"] = True           # base-colour textures are sRGB
            attrs = prim["attributes"]
            if "indices" not in prim:
                raise ValueError("non-indexed primitives are not supported")
            idx = _read(doc, buffers, prim["indices"], 1).reshape(-1)
            ct = doc["accessors"][prim["indices"]]["componentType"]
            if ct not in (5121, 5123, 5125):
                continue
            idx = idx.astype(np.uint32 if ct == 5125 else np.uint16)
            nv = doc["accessors"][next(iter(attrs.values()))]["count"]
            sm = GltfSubmesh(material=mi, indices=idx, vertices=np.zeros((nv, 4), F))
            for name, acc in attrs.items():
                if name == "POSITION":
                    p = _read(doc, buffers, acc).astype(F)
                    sm.vertices[:, 0], sm.vertices[:, 1], sm.vertices[:, 2] = -p[:, 0], p[:, 2], p[:, 1]
                elif name == "NORMAL":
                    n = _read(doc, buffers, acc).astype(F)
                    sm.normals = np.zeros((nv, 4), F)
                    sm.normals[:, 0], sm.normals[:, 1], sm.normals[:, 2] = -n[:, 0], n[:, 2], n[:, 1]
                elif name == "TANGENT":
                    t = _read(doc, buffers, acc).astype(F)
                    sm.tangents = np.stack([-t[:, 0], t[:, 2], t[:, 1], t[:, 3]], 1).astype(F)
                elif name in ("TEXCOORD_0", "TEXCOORD_1"):
                    _, _, dt, _, _, _ = _accessor(doc, buffers, acc)
                    raw = _read(doc, buffers, acc)
                    if dt == np.uint8:
                        tc = raw.astype(F) * F(1.0 / 255.0)
                    elif dt == np.uint16:
                        tc = raw.astype(F) * F(1.0 / 65535.0)
                    else:
                        tc = raw.astype(F)
                    if name == "TEXCOORD_0":
                        sm.texcoords0 = tc
                    else:
                        sm.texcoords1 = tc
            if d.emissive_present:
                e = d.emissive
                base = F(F(F(e[0]) + F(e[1])) + F(e[2])) / F(3.0)
                tri = sm.indices.reshape(-1, 3).astype(np.int64)
                em_tex = d.tex_index[6]
                coords = None
                if em_tex >= 0:
                    coords = sm.texcoords0 if d.tex_coord[6] == 0 else sm.texcoords1
                    if coords is None:
                        raise ValueError("emission texture reads a texture-coordinate set the primitive lacks")
                local, prims, flux, uvs = [], [], [], []
                for k, (a, b, c) in enumerate(tri):
                    v = [sm.vertices[a, :3], sm.vertices[b, :3], sm.vertices[c, :3]]
                    f = base
                    uv = np.zeros(6, F)
                    if em_tex >= 0:
                        t = textures[em_tex]
                        uv = np.concatenate([coords[a], coords[b], coords[c]]).astype(F)
                        scale = _emissive_texture_scale(images[t["image"]], t["address"],
                                                        [(uv[0], uv[1]), (uv[2], uv[3]), (uv[4], uv[5])])
                        f = F(float(f) * scale)
                    f = F(f * F(F(_length(_cross(v[1] - v[0], v[2] - v[0])) * F(0.5)) * F(math.pi)))
                    if f > 0.0:
                        sm.discarded.append(k)
                        local.append(np.concatenate(v).astype(F))
                        prims.append(k)
                        flux.append(f)
                        uvs.append(uv)
                if local:
                    emis.append((len(subs), np.stack(local), np.asarray(prims, np.uint32), np.asarray(flux, F),
                                 np.stack(uvs)))
            subs.append(sm)
        meshes.append(subs)
        mesh_emissive.append(emis)
    # node graph
    instances, emissive = [], []
    count = [0]
    identity = np.eye(4, dtype=F)

    def visit(ni, model_from_local):
        node = doc["nodes"][ni]
        mfl = _mat4_mul(model_from_local, _corrected(_local_matrix(node)))
        if "mesh" in node:
            m = node["mesh"]
            xf = np.ascontiguousarray(mfl[:, :3].T)        # (3, 4): rows of the 4x3 transform
            instances.append((m, xf))
            world_from_local = _mat4_mul(identity, mfl)
            for sub, local, prims, flux, uvs in mesh_emissive[m]:
                world = np.zeros_like(local)
                for r in range(len(local)):
                    for k in range(3):
                        v = np.array([local[r, 3 * k], local[r, 3 * k + 1], local[r, 3 * k + 2], 1.0], F)
                        world[r, 3 * k:3 * k + 3] = _mat4_vec4(world_from_local, v)[:3]
                emissive.append(EmissiveSubset(instance=len(instances) - 1, submesh=sub,
                                               flux_correction=float(abs(_det3(world_from_local))),
                                               world=world, local=local, prim=prims, flux=flux, uv=uvs))
            for p in doc["meshes"][m]["primitives"]:
                a = p.get("attributes")
                if a:
                    count[0] += doc["accessors"][next(iter(a.values()))]["count"]
        for child in node.get("children", []):
            visit(child, mfl)

    scene = doc["scenes"][doc.get("scene", 0)]
    for ni in scene.get("nodes", []):
        visit(ni, identity)
    return Model(meshes=meshes, descriptors=descriptors, instances=instances, emissive=emissive,
                 triangle_count=count[0], images=images, textures=textures)


# --------------------------------------------------------------- to Scene
def material_factors(d: Descriptor) -> int:
    """MaterialData::factors from a descriptor (fillModelMaterials,
    src/core/rendering_interface.cpp:94-188)."""
    f = 0
    if d.bc_factor_present:
        f |= abi.RB_FACTOR_BASE_COLOR
    if d.alpha_mode == 1:
        f |= abi.RB_FACTOR_CUTOFF
    elif d.alpha_mode == 2:
        f |= abi.RB_FACTOR_BLEND
    if d.met_factor_present:
        f |= abi.RB_FACTOR_METALNESS
    if d.rough_factor_present:
        f |= abi.RB_FACTOR_ROUGHNESS
    if d.transmit_factor_present:
        f |= abi.RB_FACTOR_TRANSMISSION
    if d.sheen_present and d.sheen_color_present:
        f |= abi.RB_FACTOR_SHEEN_COLOR
    if d.sheen_present and d.sheen_rough_present:
        f |= abi.RB_FACTOR_SHEEN_ROUGH
    if d.emissive_present:
        f |= abi.RB_FACTOR_EMISSION
    return f


def to_scene(model: Model, name: str = "gltf", width: int = 256, height: int = 256, spp: int = 16,
             max_depth: int = 8):
    """An upload-ready Scene: one material record per primitive (as the
    reference makes one MaterialData per submesh), instances with their 4x3
    transforms, emissive subsets with the flux corrected by the instance;
    one Texture per glTF texture (its image with the texture's sampler and
    sRGB flag, as fillModelMaterials makes one texture object per
    textureData: src/core/rendering_interface.cpp:47-66), each material
    slot's texture with set 2 where the slot reads TEXCOORD_1 (:89-186)."""
    from . import scenes
    textures = []
    for t in model.textures:
        img = model.images[t["image"]]
        data = img[..., 0] if img.shape[2] == 1 else img
        textures.append(scenes.Texture(np.ascontiguousarray(data), srgb=t["srgb"], address=tuple(t["address"]),
                                       filter=t["filter"]))
    # descriptor slot order (bc, mr, nm, tr, shc, shr, em) -> rb_material slots
    slot_of = (abi.RB_TEXTURE_BASE_COLOR, abi.RB_TEXTURE_MET_ROUGH, abi.RB_TEXTURE_NORMAL, abi.RB_TEXTURE_TRANSMISSION,
               abi.RB_TEXTURE_SHEEN_COLOR, abi.RB_TEXTURE_SHEEN_ROUGH, abi.RB_TEXTURE_EMISSION)
    mats = []
    for d in model.descriptors:
        m = scenes.Material(base_color=tuple(d.base_color[:3]) if d.bc_factor_present else (1.0, 1.0, 1.0),
                            metalness=d.metalness, roughness=d.roughness, transmission=d.transmission,
                            ior=d.ior, sheen_color=(tuple(d.sheen_color) if d.sheen_color_present else (1.0, 1.0, 1.0))
                            if d.sheen_present else None, sheen_roughness=d.sheen_roughness,
                            emissive=tuple(d.emissive) if d.emissive_present else None)
        m.factors = material_factors(d)
        m.alpha = d.base_color[3] if d.bc_factor_present else 0.0
        m.alpha_cutoff = d.alpha_cutoff
        m.double_sided = d.double_sided
        m.textures = {slot_of[k]: (d.tex_index[k], 2 if d.tex_coord[k] == 1 else 1)
                      for k in range(7) if (d.textures >> k) & 1}
        mats.append(m)
    meshes = []
    for subs in model.meshes:
        out = []
        for sm in subs:
            idx = sm.indices.reshape(-1, 3)
            out.append(scenes.Submesh(vertices=sm.vertices, indices=idx, material=sm.material,
                                      normals=None if sm.normals is None else sm.normals[:, :3].copy(),
                                      discarded=list(sm.discarded), texcoords=sm.texcoords0,
                                      texcoords2=sm.texcoords1, tangents=sm.tangents))
        meshes.append(out)
    emissive = []
    for e in model.emissive:
        mesh, xf = model.instances[e.instance]
        sub = model.meshes[mesh][e.submesh]
        emissive.append(dict(transform=xf, tris=e.local, world=e.world, prim=list(e.prim.tolist()),
                             flux=(e.flux * F(e.flux_correction)).astype(F), material=sub.material, uv=e.uv))
    return scenes.Scene(name=name, seed=0, meshes=meshes, instances=list(model.instances), materials=mats,
                        emissive=emissive, width=width, height=height, spp=spp, max_depth=max_depth,
                        textures=textures)
