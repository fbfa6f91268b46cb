"""A scene ingested from glTF (ratbite_b200.gltf) rendered on the GPU against
the oracle rendering the same records: the ingest path feeds the product and
the reference's per-sample code identically (factor materials with alpha
mask / blend, sheen, transmission and IOR, emissive primitives cut into light
subsets, instanced meshes under TRS and matrix transforms)."""
from __future__ import annotations

import json

import numpy as np
import pytest

from oracle_lib import RefLib, light_tree_record, load_scene_into_ref, ref_render, reference_luts
from ratbite_b200 import gltf
from ratbite_b200.rendering_interface import RenderingInterface
from test_gltf import _document, _textured_document

pytestmark = pytest.mark.gpu


def _in_front(doc):
    """In front of the camera: the renderer's -z is glTF's -y."""
    doc["nodes"].append({"translation": [1.0, -12.0, -3.5], "scale": [2.0, 2.0, 2.0],
                         "children": list(doc["scenes"][0]["nodes"])})
    doc["scenes"][0]["nodes"] = [len(doc["nodes"]) - 1]


def _render_both(sc, W, H, spp):
    ref = RefLib()
    tables = dict(cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())
    keep = load_scene_into_ref(ref, sc, tables["luts"], tables["cie"], tables["basis"])
    world, flux, mat, prim = sc.emissive_arrays()
    tris, nodes, ptrs, masks = ref.build_light_tree(world, flux, mat, prim)
    tris["uvs"] = sc.emissive_uvs()
    lt = light_tree_record(tris, nodes, ptrs, masks, keep)
    want = ref_render(ref, W, H, 0, spp)
    with RenderingInterface(device=0) as ri:
        ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lt)
        ri.render(0, spp)
        got = ri.read_accumulation()
        assert ri.status().flags == 0
    return got, want


def test_gltf_scene_renders_like_oracle(tmp_path):
    doc, binary = _document()
    _in_front(doc)
    doc["buffers"][0]["uri"] = "s.bin"
    (tmp_path / "s.bin").write_bytes(binary)
    (tmp_path / "s.gltf").write_text(json.dumps(doc))
    W, H, spp = 48, 32, 8
    sc = gltf.to_scene(gltf.load(tmp_path / "s.gltf"), width=W, height=H, spp=spp, max_depth=6)
    ref = RefLib()
    tables = dict(cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())
    keep = load_scene_into_ref(ref, sc, tables["luts"], tables["cie"], tables["basis"])
    world, flux, mat, prim = sc.emissive_arrays()
    tris, nodes, ptrs, masks = ref.build_light_tree(world, flux, mat, prim)
    lt = light_tree_record(tris, nodes, ptrs, masks, keep)
    want = ref_render(ref, W, H, 0, spp)
    with RenderingInterface(device=0) as ri:
        ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lt)
        ri.render(0, spp)
        got = ri.read_accumulation()
    g = got[..., :3] / np.maximum(got[..., 3:4], 1)
    w = want[..., :3] / np.maximum(want[..., 3:4], 1)
    lit = np.abs(w).sum()
    print(f"gltf scene: lit pixels {np.mean(np.abs(w).sum(-1) > 0):.1%}, image-mean rel diff "
          f"{abs(g.sum() - w.sum()) / lit:.3e}, per-pixel L1 {np.abs(g - w).sum() / lit:.3e}")
    assert np.mean(np.abs(w).sum(-1) > 0) > 0.05
    assert abs(g.sum() - w.sum()) / lit < 1e-3
    assert np.abs(g - w).sum() / lit < 2e-2


@pytest.mark.parametrize("as_glb", [False, True])
def test_textured_gltf_renders_like_oracle(tmp_path, as_glb):
    """The textured document (PNG images of every variant, all material
    texture slots, TEXCOORD_1, tangent frames, emissive textures with the
    texel-scaled fluxes) rendered by the product and by the oracle from the
    same records."""
    path = _textured_document(tmp_path, as_glb, edit=_in_front)
    W, H, spp = 48, 32, 8
    sc = gltf.to_scene(gltf.load(path), width=W, height=H, spp=spp, max_depth=6)
    assert sc.textures and any(m.textures for m in sc.materials)
    got, want = _render_both(sc, W, H, spp)
    g = got[..., :3] / np.maximum(got[..., 3:4], 1)
    w = want[..., :3] / np.maximum(want[..., 3:4], 1)
    lit = np.abs(w).sum()
    print(f"textured gltf scene: lit pixels {np.mean(np.abs(w).sum(-1) > 0):.1%}, image-mean rel diff "
          f"{abs(g.sum() - w.sum()) / lit:.3e}, per-pixel L1 {np.abs(g - w).sum() / lit:.3e}")
    assert np.mean(np.abs(w).sum(-1) > 0) > 0.05
    assert abs(g.sum() - w.sum()) / lit < 1e-3
    assert np.abs(g - w).sum() / lit < 2e-2
