"""Seeded inputs shared by the oracle and the GPU in the parity tests."""
from __future__ import annotations

import math

import numpy as np

from ratbite_b200 import abi, scenes

# SpectralDataType values (src/core/spectral.h:54-94) used by the conductor cases.
SPEC_AU_IOR = 10
SPEC_AU_AC = 17
SPEC_CU_IOR = 11
SPEC_CU_AC = 18


def unit_vectors(rng, n):
    v = rng.normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def frames(rng, n):
    """Random right-handed orthonormal frames (t, b, n) in float32."""
    nn = unit_vectors(rng, n)
    a = np.where(np.abs(nn[:, :1]) < 0.9, np.array([[1.0, 0, 0]]), np.array([[0, 1.0, 0]]))
    t = np.cross(a, nn)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    b = np.cross(nn, t)
    return t.astype(np.float32), b.astype(np.float32), nn


def sobol_inputs(seed=3, n=4096):
    rng = np.random.default_rng(seed)
    sample = rng.integers(0, 1 << 20, n, dtype=np.uint32)
    sample[:64] = np.arange(64, dtype=np.uint32)   # first samples of a pixel
    hashes = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    bounce = rng.integers(0, 12, n, dtype=np.uint32)
    dim = rng.integers(0, 9, n, dtype=np.uint32)
    return sample, hashes, bounce, dim


def material_table(ref_spectrum=None):
    """Materials used by the BxDF cases: the Cornell box table plus a sheen
    complex surface and two spectral conductors (PureConductor callable)."""
    mats = [
        scenes.Material(base_color=(0.7, 0.5, 0.3), metalness=0.0, roughness=1.0),
        scenes.Material(base_color=(0.9, 0.8, 0.6), metalness=1.0, roughness=0.3),
        scenes.Material(base_color=(1.0, 1.0, 1.0), metalness=0.0, roughness=0.05, transmission=1.0, ior=1.5),
        scenes.Material(base_color=(0.4, 0.6, 0.8), sheen_color=(0.9, 0.7, 0.5), sheen_roughness=0.4),
        scenes.Material(bxdf=abi.RB_BXDF_PURE_CONDUCTOR, ior_spectrum=0, absorp_spectrum=1, mf_roughness=0.35),
        scenes.Material(bxdf=abi.RB_BXDF_PURE_CONDUCTOR, ior_spectrum=2, absorp_spectrum=3, mf_roughness=0.0),
    ]
    return mats


def bxdf_cases(seed=5, n=6000):
    """BxDF calls across the material table with random frames, directions,
    surface parameters and path state; about half have an unoccluded light
    sample."""
    rng = np.random.default_rng(seed)
    cases = (abi.rb_bxdf_case * n)()
    t, b, nn = frames(rng, n)
    dirs = unit_vectors(rng, n)
    ldirs = unit_vectors(rng, n)
    for i in range(n):
        c = cases[i]
        kind = i % 6
        c.material = kind
        c.sample = int(rng.integers(0, 4096))
        c.hash = int(rng.integers(0, 1 << 32))
        c.bounce = int(rng.integers(0, 8))
        c.frame_t = abi.F3(*t[i]); c.frame_b = abi.F3(*b[i]); c.frame_n = abi.F3(*nn[i])
        # incoming ray mostly towards the surface
        d = dirs[i]
        if rng.random() < 0.8 and np.dot(d, nn[i]) > 0:
            d = -d
        c.dir = abi.F3(*d)
        c.layers = 3 if kind == 3 else 1
        c.base_color = abi.F3(*[float(np.float32(x)) for x in rng.uniform(0.05, 1.0, 3)])
        c.metalness = float(np.float32([0.0, 1.0, 0.0, rng.uniform(0, 1), 0.0, 0.0][kind]))
        c.ior = float(np.float32(rng.uniform(1.2, 2.0)))
        c.roughness = float(np.float32([1.0, rng.uniform(0.0, 1.0), rng.uniform(0.0, 0.3), rng.uniform(0.0005, 1.0), 0.3, 0.3][kind]))
        c.transmission = float(np.float32([0.0, 0.0, 1.0, rng.uniform(0, 1), 0.0, 0.0][kind]))
        c.sheen_color = abi.F3(*[float(np.float32(x)) for x in rng.uniform(0.0, 1.0, 3)])
        c.sheen_alpha = float(np.float32(rng.uniform(0.05, 1.0)))
        c.light_spectrum = abi.F4(*[float(np.float32(x)) for x in rng.uniform(0.0, 5.0, 4)])
        c.light_dir = abi.F3(*ldirs[i])
        c.light_pdf = float(np.float32(rng.uniform(0.05, 20.0)))
        c.occluded = int(rng.random() < 0.4)
        c.L = abi.F4(*[float(np.float32(x)) for x in rng.uniform(0.0, 1.0, 4)])
        lam = rng.uniform(380.0, 820.0, 4).astype(np.float32)
        c.lambda_ = abi.F4(*lam)
        c.lambda_pdf = abi.F4(*[float(np.float32(x)) for x in rng.uniform(0.001, 0.004, 4)])
        c.active_count = 4.0
        c.throughput = abi.F4(*[float(np.float32(x)) for x in rng.uniform(0.1, 1.0, 4)])
        c.bxdf_pdf = 1.0
        c.flags = int(rng.choice([0, abi.PS_REGULARIZED, abi.PS_PREVIOUS_HIT_SPECULAR]))
        c.refraction_scale = 1.0
    return cases


def bxdf_material_records(mats):
    """rb_material records for material_table() (no geometry attached)."""
    recs = (abi.rb_material * len(mats))()
    for i, m in enumerate(mats):
        r = recs[i]
        r.bxdf = m.bxdf
        r.ior = m.ior
        r.mf_roughness = m.mf_roughness
        r.ior_spectrum = m.ior_spectrum
        r.absorp_spectrum = m.absorp_spectrum
        r.sheen_present = 1 if m.sheen_color is not None else 0
        r.factors = abi.RB_FACTOR_BASE_COLOR | abi.RB_FACTOR_METALNESS | abi.RB_FACTOR_ROUGHNESS
        r.base_color = abi.F4(*m.base_color, 1.0)
        r.metalness = m.metalness
        r.roughness = m.roughness
    return recs


def many_lights_scene(seed=11, n_lights=96):
    """Cornell box whose ceiling carries n_lights small emissive triangles of
    lognormal radiance: a multi-level light tree."""
    sc = scenes.cornell_box(seed=seed, width=64, height=64, spp=8)
    rng = np.random.default_rng(seed)
    tris = []
    for k in range(n_lights):
        cx, cz = rng.uniform(-0.9, 0.9), rng.uniform(-4.1, -2.3)
        y = 0.998 - 0.001 * rng.random()
        s = rng.uniform(0.03, 0.12)
        a = (cx, y, cz); b = (cx + s, y, cz); c = (cx + s * 0.3, y, cz + s)
        tris.append(np.array([a, b, c], np.float32).reshape(9))
    tris = np.stack(tris).astype(np.float32)
    flux = []
    for k in range(n_lights):
        v = tris[k].reshape(3, 3)
        area = 0.5 * np.linalg.norm(np.cross(v[1] - v[0], v[2] - v[0]))
        rad = float(np.exp(rng.normal(0.0, 1.5)))
        flux.append(np.float32(rad * area * math.pi))
    # The lights are a submesh of the wall mesh, cut out as emissive (as
    # scene.cpp:485-631 does), with their own emissive material.
    sc.materials.append(scenes.Material(base_color=(0.7, 0.7, 0.7), emissive=(3.0, 2.8, 2.5)))
    mat = len(sc.materials) - 1
    v4 = np.concatenate([tris.reshape(-1, 3), np.zeros((3 * n_lights, 1), np.float32)], 1).astype(np.float32)
    idx = np.arange(3 * n_lights, dtype=np.uint16).reshape(n_lights, 3)
    sc.meshes[0].append(scenes.Submesh(v4, idx, mat, discarded=list(range(n_lights))))
    sc.emissive.append(dict(transform=scenes.IDENTITY, tris=tris, world=tris.copy(),
                            prim=list(range(n_lights)), flux=np.array(flux, np.float32), material=mat))
    return sc


def light_cases(seed=13, n=4096, box=None):
    rng = np.random.default_rng(seed)
    cases = (abi.rb_light_case * n)()
    pos = np.stack([rng.uniform(-0.95, 0.95, n), rng.uniform(-0.95, 0.9, n), rng.uniform(-4.1, -2.3, n)], 1).astype(np.float32)
    nrm = unit_vectors(rng, n)
    for i in range(n):
        c = cases[i]
        c.position = abi.F3(*pos[i])
        c.normal = abi.F3(*nrm[i])
        c.rand = float(np.float32(rng.random()))
        c.q_type = abi.LIGHT_TRIANGLE
        c.q_index = int(rng.integers(0, 98))
    return cases


def camera_rays(seed=17, n=2048, w=64, h=64):
    rng = np.random.default_rng(seed)
    pix = np.stack([rng.integers(0, w, n), rng.integers(0, h, n)], 1).astype(np.float32)
    fuv = rng.random((n, 2)).astype(np.float32)
    luv = rng.random((n, 2)).astype(np.float32)
    return pix, fuv, luv


def scene_rays(seed=19, n=8192):
    """Rays from the camera and from random points inside the box."""
    rng = np.random.default_rng(seed)
    o = np.stack([rng.uniform(-0.98, 0.98, n), rng.uniform(-0.98, 0.98, n), rng.uniform(-4.15, -2.25, n)], 1)
    o[: n // 4] = 0.0
    d = unit_vectors(rng, n)
    d[: n // 4, 2] = -np.abs(d[: n // 4, 2]) - 1.0
    d[: n // 4] /= np.linalg.norm(d[: n // 4], axis=1, keepdims=True)
    return np.concatenate([o, d], 1).astype(np.float32)
