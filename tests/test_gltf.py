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
                ("discarded_count", C.c_uint32), ("discarded", C.c_void_p)]


class _MatInfo(C.Structure):
    _fields_ = [("bxdf", C.c_int32), ("double_sided", C.c_int32), ("sheen_present", C.c_int32), ("ior", C.c_float),
                ("bc_factor_present", C.c_int32), ("base_color", C.c_float * 4), ("alpha_mode", C.c_int32),
                ("alpha_cutoff", C.c_float), ("met_factor_present", C.c_int32), ("metalness", C.c_float),
                ("rough_factor_present", C.c_int32), ("roughness", C.c_float),
                ("transmit_factor_present", C.c_int32), ("transmission", C.c_float),
                ("sheen_color_present", C.c_int32), ("sheen_color", C.c_float * 3),
                ("sheen_rough_present", C.c_int32), ("sheen_roughness", C.c_float),
                ("emissive_present", C.c_int32), ("emissive", C.c_float * 3), ("textures", C.c_int32)]


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


def test_textured_materials_are_rejected(tmp_path):
    doc, binary = _document()
    doc["materials"][1]["pbrMetallicRoughness"]["baseColorTexture"] = {"index": 0}
    doc["textures"] = [{"source": 0}]
    doc["images"] = [{"uri": "missing.png"}]
    doc["buffers"][0]["uri"] = "b.bin"
    (tmp_path / "b.bin").write_bytes(binary)
    (tmp_path / "t.gltf").write_text(json.dumps(doc))
    m = gltf.load(tmp_path / "t.gltf")
    assert m.descriptors[1].textures == 1
    with pytest.raises(ValueError):
        gltf.to_scene(m)
