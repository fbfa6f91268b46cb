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

All arithmetic is float32 in the reference's operation order. Textures are
not loaded (the product renders factor materials only); a material that uses
one is reported in `textures`. `to_scene` turns a loaded model into a
ratbite_b200.scenes.Scene for upload.
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
    textures: int = 0                    # bit per texture slot used (not loaded)


@dataclass
class GltfSubmesh:
    material: int
    indices: np.ndarray                  # (T*3,) uint16 / uint32
    vertices: np.ndarray                 # (V, 4) float32, w = 0
    normals: np.ndarray | None = None    # (V, 4) float32
    tangents: np.ndarray | None = None   # (V, 4) float32
    texcoords0: np.ndarray | None = None  # (V, 2) float32
    discarded: list = field(default_factory=list)


@dataclass
class EmissiveSubset:
    instance: int
    submesh: int
    flux_correction: float
    world: np.ndarray                    # (n, 9) float32
    local: np.ndarray                    # (n, 9) float32, model space of the mesh
    prim: np.ndarray                     # (n,) uint32
    flux: np.ndarray                     # (n,) float32


@dataclass
class Model:
    meshes: list                         # list[list[GltfSubmesh]]
    descriptors: list                    # list[Descriptor], one per primitive
    instances: list                      # list[(mesh, (3, 4) float32 transform)]
    emissive: list                       # list[EmissiveSubset]
    triangle_count: int = 0              # the reference's count (vertices of attribute 0)


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
    if "pbrMetallicRoughness" in mat:
        pbr = mat["pbrMetallicRoughness"]
        if "baseColorTexture" in pbr:
            tex |= 1 << 0
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
    if "KHR_materials_transmission" in ext:
        tr = ext["KHR_materials_transmission"]
        if "transmissionTexture" in tr:
            tex |= 1 << 3
        f = float(F(tr.get("transmissionFactor", 0.0)))
        if f != 0.0:
            d.transmit_factor_present, d.transmission = True, f
    if "normalTexture" in mat:
        tex |= 1 << 2
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
            if "sheenRoughnessTexture" in sh:
                tex |= 1 << 5
    em = [F(v) for v in mat.get("emissiveFactor", (0.0, 0.0, 0.0))]
    if not (em[0] == 0.0 and em[1] == 0.0 and em[2] == 0.0):
        d.emissive_present = True
        if "KHR_materials_emissive_strength" in ext:
            s = F(ext["KHR_materials_emissive_strength"].get("emissiveStrength", 1.0))
            em = [e * s for e in em]
        d.emissive = tuple(float(e) for e in em)
        if "emissiveTexture" in mat:
            tex |= 1 << 6
    d.textures = tex
    return d


# ---------------------------------------------------------------- loading
def load(path) -> Model:
    """Loads a .gltf / .glb file as the reference's loadModel does (identity
    model transform)."""
    path = Path(path)
    doc, buffers = _load_json_and_buffers(path)
    if not doc.get("meshes"):
        raise ValueError("model contains no meshes")
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
                elif name == "TEXCOORD_0":
                    _, _, dt, _, _, _ = _accessor(doc, buffers, acc)
                    raw = _read(doc, buffers, acc)
                    if dt == np.uint8:
                        sm.texcoords0 = raw.astype(F) * F(1.0 / 255.0)
                    elif dt == np.uint16:
                        sm.texcoords0 = raw.astype(F) * F(1.0 / 65535.0)
                    else:
                        sm.texcoords0 = raw.astype(F)
            if d.emissive_present:
                e = d.emissive
                base = F(F(F(e[0]) + F(e[1])) + F(e[2])) / F(3.0)
                tri = sm.indices.reshape(-1, 3).astype(np.int64)
                local, prims, flux = [], [], []
                for k, (a, b, c) in enumerate(tri):
                    v = [sm.vertices[a, :3], sm.vertices[b, :3], sm.vertices[c, :3]]
                    f = F(base * F(F(_length(_cross(v[1] - v[0], v[2] - v[0])) * F(0.5)) * F(math.pi)))
                    if f > 0.0:
                        sm.discarded.append(k)
                        local.append(np.concatenate(v).astype(F))
                        prims.append(k)
                        flux.append(f)
                if local:
                    emis.append((len(subs), np.stack(local), np.asarray(prims, np.uint32), np.asarray(flux, F)))
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
            for sub, local, prims, flux in mesh_emissive[m]:
                world = np.zeros_like(local)
                for r in range(len(local)):
                    for k in range(3):
                        v = np.array([local[r, 3 * k], local[r, 3 * k + 1], local[r, 3 * k + 2], 1.0], F)
                        world[r, 3 * k:3 * k + 3] = _mat4_vec4(world_from_local, v)[:3]
                emissive.append(EmissiveSubset(instance=len(instances) - 1, submesh=sub,
                                               flux_correction=float(abs(_det3(world_from_local))),
                                               world=world, local=local, prim=prims, flux=flux))
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
                 triangle_count=count[0])


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
    transforms, emissive subsets with the flux corrected by the instance."""
    from . import scenes
    if any(d.textures for d in model.descriptors):
        raise ValueError("materials with textures are not supported")
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
        mats.append(m)
    meshes = []
    for subs in model.meshes:
        out = []
        for sm in subs:
            idx = sm.indices.reshape(-1, 3)
            out.append(scenes.Submesh(vertices=sm.vertices, indices=idx, material=sm.material,
                                      normals=None if sm.normals is None else sm.normals[:, :3].copy(),
                                      discarded=list(sm.discarded)))
        meshes.append(out)
    emissive = []
    for e in model.emissive:
        mesh, xf = model.instances[e.instance]
        sub = model.meshes[mesh][e.submesh]
        emissive.append(dict(transform=xf, tris=e.local, world=e.world, prim=list(e.prim.tolist()),
                             flux=(e.flux * F(e.flux_correction)).astype(F), material=sub.material))
    return scenes.Scene(name=name, seed=0, meshes=meshes, instances=list(model.instances), materials=mats,
                        emissive=emissive, width=width, height=height, spp=spp, max_depth=max_depth)
