"""glTF ingest (ratbite_b200.gltf) against the reference's own loader
(SceneData::loadModel, src/core/scene.cpp, on its vendored cgltf), compiled
host-side in the oracle, on the same files.

The files are written here (JSON + .bin, and the same content as .glb):
two meshes, four primitives with u8 / u16 / u32 indices, normals, tangents
and u16-normalised texture coordinates; a node graph mixing TRS and matrix
transforms, a shared mesh instanced twice and a scaled instance; materials
without pbrMetallicRoughness, with factors, alpha mask / blend,
transmission + IOR, sheen, and an emissive factor with emissive strength.
Vertex data, indices, transforms and emissive fluxes must be bit-identical;
descriptors field-identical.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import struct

import numpy as np
import pytest

from oracle_lib import REF_DIR
from ratbite_b200 import gltf


# ---------------------------------------------------------------- fixtures
def _box(seed, n_rows=2):
    rng = np.random.default_rng(seed)
    pos, idx = [], []
    for r in range(n_rows):
        for c in range(3):
            base = len(pos)
            p0 = np.array([c * 1.1, r * 0.9, 0.0]) + rng.uniform(-0.05, 0.05, 3)
            pos += [p0, p0 + [1, 0, 0.1], p0 + [1, 1, -0.2], p0 + [0, 1, 0.05]]
            idx += [base, base + 1, base + 2, base, base + 2, base + 3]
    pos = np.asarray(pos, np.float32)
    nrm = rng.normal(size=pos.shape).astype(np.float32)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    tan = np.concatenate([rng.normal(size=pos.shape), np.sign(rng.normal(size=(len(pos), 1)))], 1).astype(np.float32)
    uv = rng.integers(0, 65535, (len(pos), 2)).astype(np.uint16)
    return pos, nrm, tan, uv, np.asarray(idx, np.uint32)


class _Writer:
    def __init__(self):
        self.bin = bytearray()
        self.views, self.accessors = [], []

    def add(self, arr, comp, typ, target=None):
        while len(self.bin) % 4:
            self.bin += b"\x00"
        off = len(self.bin)
        self.bin += arr.tobytes()
        v = {"buffer": 0, "byteOffset": off, "byteLength": arr.nbytes}
        if target:
            v["target"] = target
        self.views.append(v)
        a = {"bufferView": len(self.views) - 1, "componentType": comp, "count": len(arr), "type": typ}
        if comp == 5126 and typ == "VEC3":
            a["min"] = arr.min(0).tolist()
            a["max"] = arr.max(0).tolist()
        self.accessors.append(a)
        return len(self.accessors) - 1


def _document():
    w = _Writer()
    meshes = []
    prims0 = []
    for k, (itype, comp) in enumerate([(np.uint16, 5123), (np.uint32, 5125)]):
        pos, nrm, tan, uv, idx = _box(10 + k)
        attrs = {"POSITION": w.add(pos, 5126, "VEC3"), "NORMAL": w.add(nrm, 5126, "VEC3"),
                 "TANGENT": w.add(tan, 5126, "VEC4"), "TEXCOORD_0": w.add(uv, 5123, "VEC2")}
        prims0.append({"attributes": attrs, "indices": w.add(idx.astype(itype), comp, "SCALAR"), "material": k})
    meshes.append({"name": "boxes", "primitives": prims0})
    prims1 = []
    for k in range(2):
        pos, nrm, _, _, idx = _box(20 + k, 1)
        attrs = {"POSITION": w.add(pos, 5126, "VEC3"), "NORMAL": w.add(nrm, 5126, "VEC3")}
        prims1.append({"attributes": attrs, "indices": w.add(idx.astype(np.uint8), 5121, "SCALAR"),
                       "material": 2 + k})
    pos, _, _, _, idx = _box(30, 1)
    prims1.append({"attributes": {"POSITION": w.add(pos, 5126, "VEC3")},
                   "indices": w.add(idx.astype(np.uint16), 5123, "SCALAR"), "material": 4})
    pos, _, _, _, idx = _box(31, 1)
    prims1.append({"attributes": {"POSITION": w.add(pos, 5126, "VEC3")},
                   "indices": w.add(idx.astype(np.uint16), 5123, "SCALAR")})      # no material
    meshes.append({"name": "lights", "primitives": prims1})
    materials = [
        {"name": "plain"},
        {"pbrMetallicRoughness": {"baseColorFactor": [0.8, 0.3, 0.2, 0.7], "metallicFactor": 0.25,
                                  "roughnessFactor": 0.4}, "alphaMode": "MASK", "alphaCutoff": 0.3,
         "doubleSided": True},
        {"pbrMetallicRoughness": {"metallicFactor": 0.0}, "alphaMode": "BLEND", "emissiveFactor": [1.0, 0.5, 0.25],
         "extensions": {"KHR_materials_emissive_strength": {"emissiveStrength": 7.5}}},
        {"pbrMetallicRoughness": {"baseColorFactor": [1, 1, 1, 1]},
         "extensions": {"KHR_materials_transmission": {"transmissionFactor": 0.9},
                        "KHR_materials_ior": {"ior": 1.33},
                        "KHR_materials_sheen": {"sheenColorFactor": [0.5, 0.6, 0.7], "sheenRoughnessFactor": 0.3}}},
        {"emissiveFactor": [0.0, 2.0, 0.0],
         "extensions": {"KHR_materials_sheen": {"sheenColorFactor": [1, 1, 1]}}},
    ]
    q = [math.sin(0.35) * v for v in (0.3, 0.8, 0.5)] + [math.cos(0.35)]
    nq = math.sqrt(sum(v * v for v in q))
    q = [v / nq for v in q]
    nodes = [
        {"translation": [1.5, -0.25, 3.0], "rotation": q, "scale": [1.0, 2.0, 0.5], "children": [1, 2], "mesh": 0},
        {"matrix": [0.8, 0.0, -0.6, 0.0, 0.0, 1.0, 0.0, 0.0, 0.6, 0.0, 0.8, 0.0, -2.0, 0.5, 1.0, 1.0], "mesh": 1},
        {"translation": [0.0, 4.0, 0.0], "children": [3]},
        {"scale": [3.0, 3.0, 3.0], "rotation": [0.0, 0.7071068, 0.0, 0.7071068], "mesh": 1},
        {"translation": [-7.0, 0.0, 2.0], "mesh": 0},
    ]
    doc = {"asset": {"version": "2.0"}, "scene": 0, "scenes": [{"nodes": [0, 4]}], "nodes": nodes,
           "meshes": meshes, "materials": materials, "accessors": w.accessors, "bufferViews": w.views,
           "buffers": [{"byteLength": len(w.bin)}],
           "extensionsUsed": ["KHR_materials_emissive_strength", "KHR_materials_transmission",
                              "KHR_materials_ior", "KHR_materials_sheen"]}
    return doc, bytes(w.bin)


@pytest.fixture(scope="module", params=["gltf", "glb"])
def model_file(request, tmp_path_factory):
    d = tmp_path_factory.mktemp("gltf")
    doc, binary = _document()
    if request.param == "gltf":
        doc["buffers"][0]["uri"] = "scene_data.bin"
        (d / "scene_data.bin").write_bytes(binary)
        path = d / "model.gltf"
        path.write_text(json.dumps(doc))
    else:
        js = json.dumps(doc).encode()
        js += b" " * (-len(js) % 4)
        bn = binary + b"\x00" * (-len(binary) % 4)
        body = struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(bn), 0x004E4942) + bn
        path = d / "model.glb"
        path.write_bytes(struct.pack("<III", 0x46546C67, 2, 12 + len(body)) + body)
    return path


# ------------------------------------------------------------ the oracle
class _SubInfo(C.Structure):
    _fields_ = [("material", C.c_int32), ("index_type", C.c_int32), ("primitive_count", C.c_uint32),
                ("vertex_count", C.c_uint32), ("indices", C.c_void_p), ("vertices", C.c_void_p),
                ("normals", C.c_void_p), ("tangents", C.c_void_p), ("texcoords0", C.c_void_p),
                ("discarded_count", C.c_uint32), ("discarded", C.c_void_p), ("texcoords1", C.c_void_p)]


class _MatInfo(C.Structure):
    _fields_ = [("bxdf", C.c_int32), ("double_sided", C.c_int32), ("sheen_present", C.c_int32), ("ior", C.c_float),
                ("bc_factor_present", C.c_int32), ("base_color", C.c_float * 4), ("alpha_mode", C.c_int32),
                ("alpha_cutoff", C.c_float), ("met_factor_present", C.c_int32), ("metalness", C.c_float),
                ("rough_factor_present", C.c_int32), ("roughness", C.c_float),
                ("transmit_factor_present", C.c_int32), ("transmission", C.c_float),
                ("sheen_color_present", C.c_int32), ("sheen_color", C.c_float * 3),
                ("sheen_rough_present", C.c_int32), ("sheen_roughness", C.c_float),
                ("emissive_present", C.c_int32), ("emissive", C.c_float * 3), ("textures", C.c_int32),
                ("tex_index", C.c_int32 * 7), ("tex_coord", C.c_int32 * 7)]


def _arr(ptr, n, dtype):
    if not ptr or n == 0:
        return None
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dtype))), (n,)).copy()


@pytest.fixture(scope="module")
def ref():
    lib = C.CDLL(str(REF_DIR / "libratbite_ref_scene.so"))
    lib.rbref_scene_load.argtypes = [C.c_char_p]
    lib.rbref_scene_submesh.argtypes = [C.c_int, C.c_int, C.POINTER(_SubInfo)]
    lib.rbref_scene_material.argtypes = [C.c_int, C.POINTER(_MatInfo)]
    lib.rbref_scene_image.argtypes = [C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]
    return lib


def test_loader_matches_reference(ref, model_file):
    assert ref.rbref_scene_load(str(model_file).encode()) == 0
    counts = np.zeros(5, np.int64)
    ref.rbref_scene_counts(counts.ctypes.data)
    m = gltf.load(model_file)
    assert [len(m.meshes), len(m.instances), len(m.descriptors), len(m.emissive), m.triangle_count] == counts.tolist()
    # submeshes
    for mi, subs in enumerate(m.meshes):
        assert ref.rbref_scene_submesh_count(mi) == len(subs)
        for si, sm in enumerate(subs):
            info = _SubInfo()
            assert ref.rbref_scene_submesh(mi, si, C.byref(info)) == 0
            assert info.material == sm.material
            assert info.index_type == (1 if sm.indices.dtype == np.uint32 else 0)
            n = info.primitive_count * 3
            want_idx = _arr(info.indices, n, np.uint32 if info.index_type else np.uint16)
            assert np.array_equal(want_idx, sm.indices)
            nv = info.vertex_count
            assert np.array_equal(_arr(info.vertices, 4 * nv, np.float32).view(np.uint32),
                                  sm.vertices.reshape(-1).view(np.uint32))
            for ptr, ours, k in ((info.normals, sm.normals, 4), (info.tangents, sm.tangents, 4),
                                 (info.texcoords0, sm.texcoords0, 2)):
                want = _arr(ptr, k * nv, np.float32)
                if ours is None:
                    assert want is None
                else:
                    assert np.array_equal(want.view(np.uint32), ours.reshape(-1).view(np.uint32))
            want_disc = _arr(info.discarded, info.discarded_count, np.uint32)
            assert (want_disc.tolist() if want_disc is not None else []) == sm.discarded
    # material descriptors
    for i, d in enumerate(m.descriptors):
        info = _MatInfo()
        assert ref.rbref_scene_material(i, C.byref(info)) == 0
        assert info.bxdf == 2                                   # COMPLEX_SURFACE
        got = (d.double_sided, d.sheen_present, np.float32(d.ior), d.bc_factor_present,
               tuple(np.float32(v) for v in d.base_color) if d.bc_factor_present else None, d.alpha_mode,
               np.float32(d.alpha_cutoff), d.met_factor_present, np.float32(d.metalness), d.rough_factor_present,
               np.float32(d.roughness), d.transmit_factor_present, np.float32(d.transmission),
               d.sheen_color_present, tuple(np.float32(v) for v in d.sheen_color), d.sheen_rough_present,
               np.float32(d.sheen_roughness), d.emissive_present, tuple(np.float32(v) for v in d.emissive),
               d.textures)
        want = (bool(info.double_sided), bool(info.sheen_present), np.float32(info.ior), bool(info.bc_factor_present),
                tuple(np.float32(v) for v in info.base_color) if info.bc_factor_present else None, info.alpha_mode,
                np.float32(info.alpha_cutoff), bool(info.met_factor_present), np.float32(info.metalness),
                bool(info.rough_factor_present), np.float32(info.roughness), bool(info.transmit_factor_present),
                np.float32(info.transmission), bool(info.sheen_color_present),
                tuple(np.float32(v) for v in info.sheen_color), bool(info.sheen_rough_present),
                np.float32(info.sheen_roughness), bool(info.emissive_present),
                tuple(np.float32(v) for v in info.emissive), info.textures)
        assert got == want, (i, got, want)
    # instances: 4x3 transforms bit-identical
    for i, (mesh, xf) in enumerate(m.instances):
        wm = C.c_int32()
        wx = np.zeros(12, np.float32)
        assert ref.rbref_scene_instance(i, C.byref(wm), wx.ctypes.data) == 0
        assert wm.value == mesh
        assert np.array_equal(wx.reshape(4, 3).T.view(np.uint32), xf.view(np.uint32))
    # emissive subsets: world / local vertices, primitive indices, fluxes
    assert len(m.emissive) > 0
    for i, e in enumerate(m.emissive):
        inst, sub, nt = C.c_int32(), C.c_int32(), C.c_int32()
        corr = C.c_float()
        assert ref.rbref_scene_emissive(i, C.byref(inst), C.byref(sub), C.byref(corr), C.byref(nt)) == 0
        assert (inst.value, sub.value, nt.value) == (e.instance, e.submesh, len(e.prim))
        assert np.float32(corr.value).view(np.uint32) == np.float32(e.flux_correction).view(np.uint32)
        for k in range(nt.value):
            t = np.zeros(20, np.float32)
            assert ref.rbref_scene_emissive_triangle(i, k, t.ctypes.data) == 0
            assert np.array_equal(t[:9].view(np.uint32), e.world[k].view(np.uint32))
            assert np.array_equal(t[9:18].view(np.uint32), e.local[k].view(np.uint32))
            assert t[18:19].view(np.uint32)[0] == e.prim[k]
            assert t[19].view(np.uint32) == e.flux[k].view(np.uint32)


def test_scene_records(model_file):
    from ratbite_b200 import abi
    m = gltf.load(model_file)
    sc = gltf.to_scene(m, width=32, height=24, spp=2)
    recs = sc.material_records()
    assert len(recs) == len(m.descriptors)
    assert recs[1].factors & abi.RB_FACTOR_CUTOFF and abi.RB_FACTOR_BASE_COLOR & recs[1].factors
    assert abs(recs[1].base_color[3] - 0.7) < 1e-7 and abs(recs[1].alpha_cutoff - 0.3) < 1e-7
    assert recs[1].double_sided == 1
    assert recs[0].factors == 0
    assert recs[3].sheen_present == 1 and recs[3].factors & abi.RB_FACTOR_TRANSMISSION
    world, flux, mat, prim = sc.emissive_arrays()
    assert len(flux) == sum(len(e.prim) for e in m.emissive) and np.all(flux > 0)
    g = sc.geometry_record()
    assert g.instance_count == len(m.instances) and g.emissive_subset_count == len(m.emissive)


# ------------------------------------------------------------- textures
def _png(px, ctype, depth, palette=None, trns=None, filters=(0, 1, 2, 3, 4)):
    """A PNG of raw samples px (H, W, channels; palette indices for colour
    type 3), rows filtered with the given filter types in turn."""
    import zlib
    h, w = px.shape[:2]
    chans = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
    bits = depth * chans
    stride = (w * bits + 7) // 8
    bpp = max(1, bits // 8)
    rows = []
    for y in range(h):
        if depth == 16:
            row = px[y].reshape(-1).astype(">u2").tobytes()
        elif depth == 8:
            row = px[y].reshape(-1).astype(np.uint8).tobytes()
        else:
            vals = px[y].reshape(-1)
            acc = bytearray(stride)
            for i, v in enumerate(vals):
                bit = i * depth
                acc[bit // 8] |= int(v) << (8 - depth - bit % 8)
            row = bytes(acc)
        rows.append(np.frombuffer(row, np.uint8).astype(np.int64))
    out = bytearray()
    prev = np.zeros(stride, np.int64)
    for y, raw in enumerate(rows):
        f = filters[y % len(filters)]
        enc = np.zeros(stride, np.int64)
        for x in range(stride):
            a = raw[x - bpp] if x >= bpp else 0
            b = prev[x]
            c = prev[x - bpp] if x >= bpp else 0
            if f == 0:
                p = 0
            elif f == 1:
                p = a
            elif f == 2:
                p = b
            elif f == 3:
                p = (a + b) >> 1
            else:
                pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                p = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
            enc[x] = (raw[x] - p) & 255
        out += bytes([f]) + enc.astype(np.uint8).tobytes()
        prev = raw

    def chunk(kind, body):
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF)

    data = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, ctype, 0, 0, 0))
    if palette is not None:
        data += chunk(b"PLTE", np.asarray(palette, np.uint8).tobytes())
    if trns is not None:
        data += chunk(b"tRNS", trns)
    data += chunk(b"IDAT", zlib.compress(bytes(out)))
    return data + chunk(b"IEND", b"")


def _images():
    """PNG variants stb_image reads differently: every colour type, 1/2/4/8/16
    bits, palettes with and without tRNS, colour keys, all five filters."""
    rng = np.random.default_rng(77)
    r = lambda h, w, c, hi: rng.integers(0, hi + 1, (h, w, c))
    pal = rng.integers(0, 256, (16, 3))
    rgb_key = r(10, 9, 3, 255)
    rgb_key[2, 3] = rgb_key[5, 5] = (11, 22, 33)
    rgb16 = r(6, 7, 3, 65535)
    rgb16[1, 1] = (1000, 2000, 3000)
    rgb16[2, 2] = (1000, 2000, 3001)               # same high bytes, not the key
    grey16 = r(5, 4, 1, 65535)
    return [
        _png(r(16, 12, 4, 255), 6, 8),                                         # 0 RGBA8 (emission)
        _png(rgb_key, 2, 8, trns=struct.pack(">HHH", 11, 22, 33)),             # 1 RGB8 + colour key
        _png(r(7, 5, 1, 255), 0, 8),                                           # 2 grey8: one channel
        _png(r(6, 8, 2, 255), 4, 8),                                           # 3 grey + alpha
        _png(r(6, 9, 1, 15), 3, 4, palette=pal, trns=bytes([0, 128, 255, 7])),  # 4 palette 4-bit + tRNS
        _png(r(5, 6, 4, 65535), 6, 16),                                        # 5 RGBA16
        _png(r(4, 11, 1, 3), 0, 2),                                            # 6 grey 2-bit
        _png(rgb16, 2, 16, trns=struct.pack(">HHH", 1000, 2000, 3000)),        # 7 RGB16 + colour key
        _png(grey16, 0, 16, trns=struct.pack(">H", int(grey16[0, 0, 0]))),     # 8 grey16 + key: grey + alpha
        _png(r(5, 5, 1, 15), 3, 8, palette=pal),                               # 9 palette 8-bit
        _png(r(3, 13, 1, 1), 0, 1),                                            # 10 grey 1-bit
        _png(np.array([[[0], [1], [2], [3]], [[2], [2], [1], [0]]]), 0, 2, trns=struct.pack(">H", 2)),  # 11
        _png(np.array([[[7], [9]], [[9], [7]]]), 0, 8, trns=struct.pack(">H", 0x0109)),  # 12 key & 255 = 9
        _png(r(12, 10, 3, 255), 2, 8),                                         # 13 RGB8 (emission, via a buffer view)
    ]


def _textured_document(tmp_path, as_glb=False, edit=None):
    """_document plus images (files, and one in a buffer view), samplers
    with every filter / wrap mode, textures on every material slot (some on
    TEXCOORD_1), tangents, and emissive textures on the light mesh: one
    emitter with large triangles in texture space, one with triangles too
    small to cover a texel centre (the per-vertex fallback). `edit(doc)`
    may change the document before it is written."""
    doc, binary = _document()
    binary = bytearray(binary)
    pngs = _images()
    images = []
    for i, data in enumerate(pngs[:-1]):
        (tmp_path / f"img {i}.png").write_bytes(data)
        images.append({"uri": f"img%20{i}.png"})
    while len(binary) % 4:
        binary += b"\x00"
    doc["bufferViews"].append({"buffer": 0, "byteOffset": len(binary), "byteLength": len(pngs[-1])})
    binary += pngs[-1]
    images.append({"bufferView": len(doc["bufferViews"]) - 1, "mimeType": "image/png"})
    doc["images"] = images
    doc["samplers"] = [{"magFilter": 9728, "wrapS": 33648, "wrapT": 33071},
                       {"magFilter": 9729, "wrapS": 10497, "wrapT": 33648},
                       {"wrapS": 33071},
                       {"magFilter": 9728}]
    doc["textures"] = [{"source": 1, "sampler": 0}, {"source": 5, "sampler": 1}, {"source": 3},
                       {"source": 4, "sampler": 2}, {"source": 2, "sampler": 3}, {"source": 6, "sampler": 1},
                       {"source": 7}, {"source": 0, "sampler": 1}, {"source": 13, "sampler": 0},
                       {"source": 8}, {"source": 9, "sampler": 2}, {"source": 10}, {"source": 11},
                       {"source": 12}]
    doc["buffers"][0]["byteLength"] = len(binary)
    mats = doc["materials"]
    mats[1]["pbrMetallicRoughness"]["baseColorTexture"] = {"index": 0}
    mats[1]["pbrMetallicRoughness"]["metallicRoughnessTexture"] = {"index": 1, "texCoord": 1}
    mats[1]["normalTexture"] = {"index": 2}
    mats[3]["pbrMetallicRoughness"]["baseColorTexture"] = {"index": 4, "texCoord": 0}
    mats[3]["extensions"]["KHR_materials_transmission"]["transmissionTexture"] = {"index": 9}
    mats[3]["extensions"]["KHR_materials_sheen"]["sheenColorTexture"] = {"index": 3, "texCoord": 1}
    mats[3]["extensions"]["KHR_materials_sheen"]["sheenRoughnessTexture"] = {"index": 5}
    mats[2]["emissiveTexture"] = {"index": 7}
    mats[4]["emissiveTexture"] = {"index": 8, "texCoord": 1}
    mats[0]["pbrMetallicRoughness"] = {"baseColorTexture": {"index": 10}}
    mats[0]["normalTexture"] = {"index": 6, "texCoord": 1}
    mats[0]["emissiveTexture"] = {"index": 11}                       # no emissive factor: not read
    # TEXCOORD_1 (u8 normalized) on the first mesh, texture coordinates and
    # tangents on the light primitives
    w = _Writer()
    w.bin = binary
    w.views, w.accessors = doc["bufferViews"], doc["accessors"]
    rng = np.random.default_rng(5)
    for prim in doc["meshes"][0]["primitives"]:
        nv = doc["accessors"][prim["attributes"]["POSITION"]]["count"]
        prim["attributes"]["TEXCOORD_1"] = w.add(rng.integers(0, 255, (nv, 2)).astype(np.uint8), 5121, "VEC2")
    lights = doc["meshes"][1]["primitives"]
    for k, prim in enumerate(lights):
        nv = doc["accessors"][prim["attributes"]["POSITION"]]["count"]
        if k == 0:      # emitter 2: float coordinates well outside [0, 1] (wrap / mirror), large footprint
            uv = rng.uniform(-1.7, 2.4, (nv, 2)).astype(np.float32)
            prim["attributes"]["TEXCOORD_0"] = w.add(uv, 5126, "VEC2")
        if k == 1:      # transmissive + sheen material: texture sets 0 and 1, tangents
            prim["attributes"]["TEXCOORD_0"] = w.add(rng.uniform(0, 1, (nv, 2)).astype(np.float32), 5126, "VEC2")
            prim["attributes"]["TEXCOORD_1"] = w.add(rng.uniform(-1, 2, (nv, 2)).astype(np.float32), 5126, "VEC2")
            t = np.concatenate([rng.normal(size=(nv, 3)), np.where(rng.uniform(size=(nv, 1)) < 0.5, -1.0, 1.0)], 1)
            prim["attributes"]["TANGENT"] = w.add(t.astype(np.float32), 5126, "VEC4")
        if k == 2:      # emitter 4 on TEXCOORD_1: tiny triangles in texture space (the per-vertex fallback)
            base = rng.uniform(0.1, 0.9, (1, 2))
            prim["attributes"]["TEXCOORD_0"] = w.add(np.zeros((nv, 2), np.float32), 5126, "VEC2")
            prim["attributes"]["TEXCOORD_1"] = w.add((base + rng.uniform(0, 1e-3, (nv, 2))).astype(np.float32),
                                                     5126, "VEC2")
    binary = bytes(w.bin)
    doc["buffers"][0]["byteLength"] = len(binary)
    if edit is not None:
        edit(doc)
    if as_glb:
        js = json.dumps(doc).encode()
        js += b" " * (-len(js) % 4)
        bn = binary + b"\x00" * (-len(binary) % 4)
        body = struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(bn), 0x004E4942) + bn
        path = tmp_path / "textured.glb"
        path.write_bytes(struct.pack("<III", 0x46546C67, 2, 12 + len(body)) + body)
        return path
    doc["buffers"][0]["uri"] = "textured.bin"
    (tmp_path / "textured.bin").write_bytes(binary)
    path = tmp_path / "textured.gltf"
    path.write_text(json.dumps(doc))
    return path


@pytest.mark.parametrize("as_glb", [False, True])
def test_textured_loader_matches_reference(ref, tmp_path, as_glb):
    """Images (stb_image's decode of every PNG variant), textures with their
    samplers and sRGB flags, per-slot texture and coordinate-set indices,
    TEXCOORD_1, and the emissive fluxes scaled by the texels each triangle
    covers, with the emitters' texture coordinates: all identical to the
    reference loader's."""
    path = _textured_document(tmp_path, as_glb)
    assert ref.rbref_scene_load(str(path).encode()) == 0
    m = gltf.load(path)
    counts = np.zeros(2, np.int64)
    ref.rbref_scene_texture_counts(counts.ctypes.data)
    assert counts.tolist() == [len(m.images), len(m.textures)]
    for i, img in enumerate(m.images):
        dims = np.zeros(3, np.int32)
        ptr = C.c_void_p()
        assert ref.rbref_scene_image(i, dims.ctypes.data, C.byref(ptr)) == 0
        assert dims.tolist() == [img.shape[1], img.shape[0], img.shape[2]], i
        want = _arr(ptr.value, int(dims.prod()), np.uint8)
        assert np.array_equal(want, img.reshape(-1)), i
    for i, t in enumerate(m.textures):
        out = np.zeros(5, np.int32)
        assert ref.rbref_scene_texture(i, out.ctypes.data) == 0
        assert out.tolist() == [t["image"], int(t["srgb"]), t["filter"], *t["address"]], i
    for i, d in enumerate(m.descriptors):
        info = _MatInfo()
        assert ref.rbref_scene_material(i, C.byref(info)) == 0
        assert info.textures == d.textures
        assert list(info.tex_index) == list(d.tex_index), i
        got_crd = [c if d.tex_index[k] >= 0 else 0 for k, c in enumerate(d.tex_coord)]
        assert list(info.tex_coord) == got_crd, i
    for mi, subs in enumerate(m.meshes):
        for si, sm in enumerate(subs):
            info = _SubInfo()
            assert ref.rbref_scene_submesh(mi, si, C.byref(info)) == 0
            for ptr, ours in ((info.texcoords0, sm.texcoords0), (info.texcoords1, sm.texcoords1)):
                want = _arr(ptr, 2 * info.vertex_count, np.float32)
                if ours is None:
                    assert want is None
                else:
                    assert np.array_equal(want.view(np.uint32), ours.reshape(-1).view(np.uint32))
            want_disc = _arr(info.discarded, info.discarded_count, np.uint32)
            assert (want_disc.tolist() if want_disc is not None else []) == sm.discarded
    textured = 0
    for i, e in enumerate(m.emissive):
        inst, sub, nt = C.c_int32(), C.c_int32(), C.c_int32()
        corr = C.c_float()
        assert ref.rbref_scene_emissive(i, C.byref(inst), C.byref(sub), C.byref(corr), C.byref(nt)) == 0
        assert nt.value == len(e.prim)
        for k in range(nt.value):
            t = np.zeros(20, np.float32)
            uv = np.zeros(6, np.float32)
            assert ref.rbref_scene_emissive_triangle(i, k, t.ctypes.data) == 0
            assert ref.rbref_scene_emissive_uvs(i, k, uv.ctypes.data) == 0
            assert t[18:19].view(np.uint32)[0] == e.prim[k]
            assert t[19].view(np.uint32) == e.flux[k].view(np.uint32), (i, k, t[19], e.flux[k])
            assert np.array_equal(uv.view(np.uint32), e.uv[k].view(np.uint32))
            textured += bool(np.any(uv != 0))
    assert textured > 0


def test_png_variants_decode_as_stb_reads_them():
    """Spot checks of the decode rules on known pixels (the full comparison
    with stb_image is in the loader test): colour keys compare at full
    depth and make a 4-channel image, 16-bit keeps the high byte, low-depth
    grey is scaled."""
    imgs = [gltf._png_decode(d) for d in _images()]
    assert imgs[1].shape[2] == 4 and imgs[1][2, 3, 3] == 0 and imgs[1][5, 5, 3] == 0
    assert imgs[2].shape[2] == 1 and imgs[8].shape[2] == 4 and imgs[8][0, 0, 3] == 0
    assert imgs[7][1, 1, 3] == 0 and imgs[7][2, 2, 3] == 255 and imgs[7][2, 2, 2] == 3000 >> 8
    assert set(np.unique(imgs[6]).tolist()) <= {0, 85, 170, 255}
    assert set(np.unique(imgs[10]).tolist()) <= {0, 255}
    assert imgs[11][..., 3].tolist() == [[255, 255, 0, 255], [0, 0, 255, 255]]
    assert imgs[12][..., 3].tolist() == [[255, 0], [0, 255]]
    with pytest.raises(ValueError):
        gltf._png_decode(b"GIF89a")


def test_frame_packing_matches_reference(ref):
    """The FRAME attribute (tangent-frame quaternions) bit-identical to the
    reference's packing, including frames whose w is exactly zero (signed
    by the tangent's handedness) and each largest-diagonal case."""
    from ratbite_b200 import scenes
    rng = np.random.default_rng(9)
    n = rng.normal(size=(400, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    t = rng.normal(size=(400, 3))
    t -= (t * n).sum(1, keepdims=True) * n
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    t4 = np.concatenate([t, np.where(rng.uniform(size=(400, 1)) < 0.5, -1.0, 1.0)], 1)
    special = [((0, 0, -1), (1, 0, 0, 1)), ((0, 0, -1), (1, 0, 0, -1)), ((0, -1, 0), (0, 0, 1, 1)),
               ((0, 0, 1), (1, 0, 0, 1)), ((0, 0, 1), (-1, 0, 0, -1)), ((1, 0, 0), (0, 1, 0, 1))]
    n = np.concatenate([n, [s[0] for s in special]])
    t4 = np.concatenate([t4, [s[1] for s in special]])
    n4 = np.concatenate([n, np.zeros((len(n), 1))], 1).astype(np.float32)
    t4 = t4.astype(np.float32)
    want = np.zeros((len(n), 4), np.float32)
    ref.rbref_pack_frames(len(n), n4.ctypes.data, t4.ctypes.data, want.ctypes.data)
    got = scenes.frame_encode(n4, t4)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert np.any(want[:, 3] == 0.0)


def test_textured_scene_records(tmp_path):
    from ratbite_b200 import abi
    m = gltf.load(_textured_document(tmp_path))
    sc = gltf.to_scene(m, width=16, height=16, spp=1)
    assert len(sc.textures) == len(m.textures)
    recs = sc.material_records()
    texs = sc.texture_records()
    r1 = recs[1]
    assert r1.textures == (1 << abi.RB_TEXTURE_BASE_COLOR) | (1 << abi.RB_TEXTURE_MET_ROUGH) | (1 << abi.RB_TEXTURE_NORMAL)
    assert r1.texture_index[abi.RB_TEXTURE_MET_ROUGH] == 1 and r1.texcoord_sets == 1 << abi.RB_TEXTURE_MET_ROUGH
    assert r1.attributes & abi.RB_ATTR_TEX_COORD_1 and r1.attributes & abi.RB_ATTR_TEX_COORD_2
    assert texs[0].srgb == 1 and texs[4].srgb == 1 and texs[4].format == abi.RB_TEXFMT_R8
    assert texs[1].srgb == 0 and texs[0].filter == abi.RB_TEXFILTER_NEAREST
    assert (texs[0].address_u, texs[0].address_v) == (abi.RB_TEXADDR_MIRROR, abi.RB_TEXADDR_CLAMP)
    assert recs[0].textures == (1 << abi.RB_TEXTURE_BASE_COLOR) | (1 << abi.RB_TEXTURE_NORMAL)
    # the transmissive + sheen primitive has tangents: the FRAME attribute
    assert recs[3].attributes & abi.RB_ATTR_FRAME and recs[3].attribute_stride == 32
    assert recs[3].texture_index[abi.RB_TEXTURE_SHEEN_COLOR] == 3
    assert recs[3].texcoord_sets == 1 << abi.RB_TEXTURE_SHEEN_COLOR
    uvs = sc.emissive_uvs()
    assert uvs.shape == (len(sc.emissive_arrays()[1]), 6) and np.any(uvs != 0)


def test_images_in_data_uris_are_refused(tmp_path):
    doc, binary = _document()
    doc["images"] = [{"uri": "data:image/png;base64,AAAA"}]
    doc["buffers"][0]["uri"] = "b.bin"
    (tmp_path / "b.bin").write_bytes(binary)
    (tmp_path / "t.gltf").write_text(json.dumps(doc))
    with pytest.raises(ValueError):
        gltf.load(tmp_path / "t.gltf")
