"""Built-in spectral tables and look-up tables for callers that do not bring
their own.

ratbite loads its CIE curves, RGB basis and multiple-scattering LUTs from its
own data files; a caller of this library passes them through rb_set_spectra
and rb_set_luts. For standalone use (the benchmark, examples) this module
generates stand-ins from published formulas:

* CIE 1931 2-degree colour matching functions: the multi-lobe piecewise
  Gaussian fit of Wyman, Sloan and Shirley (JCGT 2013), sampled at 1 nm.
* RGB spectral basis: three smooth curves that sum to one at every
  wavelength (so white maps to a flat spectrum and albedos stay <= 1).
* GGX albedo tables: Monte-Carlo estimates of the directional albedo of the
  rough conductor / dielectric / glossy layer over (cos theta, roughness
  [, sqrt|f0|]) on the 32-point grids the renderer indexes, and a neutral
  sheen LTC table (A = 1, B = 0: a cosine lobe) with a small albedo.

They are approximations for workloads; parity tests always use the
reference's own tables.
"""
from __future__ import annotations

import numpy as np

BINS = 471
LAMBDA = np.arange(360, 831, dtype=np.float64)


def _g(lam, mu, s1, s2):
    s = np.where(lam < mu, s1, s2)
    return np.exp(-0.5 * ((lam - mu) / s) ** 2)


def cie_xyz() -> np.ndarray:
    lam = LAMBDA
    x = 1.056 * _g(lam, 599.8, 37.9, 31.0) + 0.362 * _g(lam, 442.0, 16.0, 26.7) - 0.065 * _g(lam, 501.1, 20.4, 26.2)
    y = 0.821 * _g(lam, 568.8, 46.9, 40.5) + 0.286 * _g(lam, 530.9, 16.3, 31.1)
    z = 1.217 * _g(lam, 437.0, 11.8, 36.0) + 0.681 * _g(lam, 459.0, 26.0, 13.8)
    return np.stack([x, y, z]).astype(np.float32)


def basis_rgb() -> np.ndarray:
    lam = LAMBDA
    b = 1.0 / (1.0 + np.exp((lam - 490.0) / 12.0))
    r = 1.0 / (1.0 + np.exp(-(lam - 590.0) / 12.0))
    g = np.clip(1.0 - r - b, 0.0, 1.0)
    s = r + g + b
    return np.stack([r / s, g / s, b / s]).astype(np.float32)


def _ggx_albedo(mu, rough, f0=None, n=512, seed=7):
    """Directional albedo of a GGX microfacet reflector (Smith G2 / G1
    estimator over visible-normal samples), with Schlick Fresnel if f0 given."""
    rng = np.random.default_rng(seed)
    a = max(rough * rough, 1e-4)
    wo = np.array([np.sqrt(max(1.0 - mu * mu, 0.0)), 0.0, mu])
    u1, u2 = rng.random(n), rng.random(n)
    # Heitz 2018 visible-normal sampling
    vh = np.array([a * wo[0], a * wo[1], wo[2]])
    vh /= np.linalg.norm(vh)
    lensq = vh[0] ** 2 + vh[1] ** 2
    t1 = np.array([-vh[1], vh[0], 0.0]) / np.sqrt(lensq) if lensq > 0 else np.array([1.0, 0.0, 0.0])
    t2 = np.cross(vh, t1)
    r = np.sqrt(u1)
    phi = 2 * np.pi * u2
    p1 = r * np.cos(phi)
    p2 = r * np.sin(phi)
    s = 0.5 * (1.0 + vh[2])
    p2 = (1.0 - s) * np.sqrt(np.maximum(1.0 - p1 * p1, 0)) + s * p2
    nh = p1[:, None] * t1 + p2[:, None] * t2 + np.sqrt(np.maximum(0, 1 - p1 * p1 - p2 * p2))[:, None] * vh
    m = np.stack([a * nh[:, 0], a * nh[:, 1], np.maximum(nh[:, 2], 1e-6)], 1)
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    wi = -wo + 2.0 * (m @ wo)[:, None] * m
    ok = wi[:, 2] > 0

    def lam_(w):
        t2_ = np.maximum(1 - w[..., 2] ** 2, 0) / np.maximum(w[..., 2] ** 2, 1e-12)
        return (np.sqrt(1 + a * a * t2_) - 1) / 2
    g1 = 1 / (1 + lam_(wo))
    g2 = 1 / (1 + lam_(wo) + lam_(wi))
    w = np.where(ok, g2 / g1, 0.0)
    if f0 is not None:
        c = np.clip(m @ wo, 0, 1)
        w = w * (f0 + (1 - f0) * (1 - c) ** 5)
    return float(w.mean())


def luts(n_mc: int = 256) -> dict:
    N = 32
    cond = np.zeros((N, N), np.float32)
    for j in range(N):           # roughness (y)
        for i in range(N):       # cos theta (x)
            mu = (i + 0.5) / N
            r = (j + 0.5) / N
            cond[j, i] = _ggx_albedo(mu, r, n=n_mc, seed=i * N + j)
    cond = np.clip(cond, 0.05, 1.0)
    # Dielectric albedo (3D, z = sqrt|f0|): energy of the specular layer plus
    # transmission, approximated by the conductor albedo; reflective part by
    # the Schlick-weighted albedo.
    diel = np.repeat(cond[None, :, :], N, axis=0).astype(np.float32)
    refl = np.zeros((N, N, N), np.float32)
    for k in range(N):
        f0 = ((k + 0.5) / N) ** 2
        mu = (np.arange(N) + 0.5) / N
        fres = f0 + (1 - f0) * (1 - mu) ** 5
        refl[k] = np.clip(cond * fres[None, :], 0.0, 0.99)
    sheen = np.zeros((N, N, 4), np.float32)
    sheen[..., 0] = 1.0
    sheen[..., 1] = 0.0
    alpha = (np.arange(N) + 0.5) / N
    mu = (np.arange(N) + 0.5) / N
    sheen[..., 2] = (0.15 * alpha[:, None] * (1.0 - 0.5 * mu[None, :])).astype(np.float32)
    return dict(conductor=cond.reshape(-1), dielectric_outer=diel.reshape(-1), dielectric_inner=diel.reshape(-1),
                reflective_outer=refl.reshape(-1), reflective_inner=refl.reshape(-1), sheen=sheen.reshape(-1))


def generated_luts(samples: int = 1 << 14, device: int = 0, sheen_paths: int = 1 << 18) -> dict:
    """The multiple-scattering tables regenerated on the GPU by Monte Carlo
    integration of the BxDF lobes (rb_k_generate_luts), and the sheen LTC
    table fitted to a simulated volumetric sheen layer
    (rb_k_generate_sheen_lut)."""
    import ctypes as C

    import torch

    from ._native import check, load
    lib = load()
    with torch.cuda.device(device):
        cond = torch.zeros(32 * 32, dtype=torch.float32, device="cuda")
        t3 = [torch.zeros(32 ** 3, dtype=torch.float32, device="cuda") for _ in range(4)]
        sheen = torch.zeros(32 * 32 * 4, dtype=torch.float32, device="cuda")
        check(lib.rb_k_generate_luts(samples, C.c_void_p(cond.data_ptr()), *[C.c_void_p(t.data_ptr()) for t in t3],
                                     None), None, "rb_k_generate_luts")
        check(lib.rb_k_generate_sheen_lut(sheen_paths, C.c_void_p(sheen.data_ptr()), None), None,
              "rb_k_generate_sheen_lut")
        torch.cuda.synchronize()
    out = luts(n_mc=1)
    out.update(conductor=cond.cpu().numpy(), dielectric_outer=t3[0].cpu().numpy(),
               dielectric_inner=t3[1].cpu().numpy(), reflective_outer=t3[2].cpu().numpy(),
               reflective_inner=t3[3].cpu().numpy(), sheen=sheen.cpu().numpy())
    return out
