/*
 * ratbite_b200 — batched per-function entry points.
 *
 * Each call evaluates one device function of the per-sample path for a batch
 * of independent inputs that already live in device memory, on `stream`
 * (a cudaStream_t, NULL = the context stream). They expose the exact code the
 * wavefront kernels run, one stage at a time, so every stage can be checked
 * against the reference on identical inputs. Functions that read scene data
 * (LUTs, spectra, materials, light tree, geometry) take the context those
 * were uploaded to.
 */
#ifndef RATBITE_B200_KERNELS_H
#define RATBITE_B200_KERNELS_H

#include "ratbite_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* QRNG::Sobol::sample1D/2D/3D (src/device/quasi_random.h:76-99) for a state
 * made of (sample index, pixel hash) advanced by `bounce` bounces
 * (State / advanceBounce, :38-64), at dimension offset `dim` (DimensionOffset,
 * :13-29). `dims` is 1, 2 or 3; out holds n*dims floats. */
int rb_k_sobol(uint32_t n, uint32_t dims, const uint32_t* sample, const uint32_t* hash,
               const uint32_t* bounce, const uint32_t* dim, float* out, void* stream);

/* QRNG::getPixelHash (src/device/quasi_random.h:30-37). */
int rb_k_pixel_hash(uint32_t n, const uint32_t* x, const uint32_t* y, uint32_t* out, void* stream);

/* SampledWavelengths::sampleVisible (src/device/spectral.h:227-241): four
 * hero wavelengths and their pdfs per input u. */
int rb_k_wavelengths(uint32_t n, const float* u, float* lambda, float* pdf, void* stream);

/* Camera ray of __raygen__main (src/kernels/pathtrace.cu:1136-1156) for
 * pixel (x, y): Gaussian filter jitter (src/device/filter.h:14) from
 * filter_uv, then pinhole (src/device/dir_gen.h:19) or thin-lens (:31) from
 * lens_uv, with the context's launch parameters. out: 6 floats (o, d). */
int rb_k_camera_ray(rb_ctx* ctx, uint32_t n, const float* pixel_xy, const float* filter_uv,
                    const float* lens_uv, float* out, void* stream);

/* Texture `texture` of the context's rb_set_textures table sampled at n
 * (u, v) pairs by the shading kernels' software sampler (soft, 4 floats
 * each) and by the texture unit through a CUDA texture object made from the
 * same texels and sampler settings, as the reference's CudaCombinedTexture
 * (src/core/texture.h:237-380) makes it (hw, 4 floats each): a check of the
 * sampler's semantics. Synchronizes. */
int rb_k_texture_sample(rb_ctx* ctx, uint32_t texture, uint32_t n, const float* uv, float* soft, float* hw,
                        void* stream);

/* One BxDF call as the raygen makes it (src/kernels/pathtrace.cu:1724-1733):
 * inputs and the in/out path state in one record. */
typedef struct rb_bxdf_case {
    /* inputs */
    uint32_t material;           /* material table index (selects the callable) */
    uint32_t sample, hash, bounce;  /* QRNG state */
    float frame_t[3], frame_b[3], frame_n[3];  /* shading frame columns (LocalTransform) */
    uint32_t layers;             /* microsurface::Layers: 1 base, 2 sheen */
    float base_color[3];
    float metalness;
    float ior;
    float roughness;
    float transmission;
    float sheen_color[3];
    float sheen_alpha;
    float light_spectrum[4];     /* DirectLightSampleData */
    float light_dir[3];
    float light_pdf;
    uint32_t occluded;
    /* in/out path state */
    float L[4];
    float lambda[4];
    float lambda_pdf[4];
    float active_count;
    float throughput[4];
    float bxdf_pdf;
    float dir[3];
    uint32_t flags;              /* PathStateBitfield */
    float refraction_scale;
} rb_bxdf_case;
int rb_k_bxdf(rb_ctx* ctx, uint32_t n, rb_bxdf_case* cases, void* stream);

/* Light tree (src/kernels/pathtrace.cu:974-1112): sampleLightTree for
 * (rand, position, normal) -> (type, index, pdf), and traverseLightTree for
 * the query light (q_type, q_index) -> q_pdf. */
typedef struct rb_light_case {
    float position[3];
    float normal[3];
    float rand;
    uint32_t type;               /* out: LightType (0 triangle, 1 sky, 2 none) */
    uint32_t index;              /* out */
    float pdf;                   /* out */
    uint32_t q_type;             /* in */
    uint32_t q_index;            /* in */
    float q_pdf;                 /* out */
} rb_light_case;
int rb_k_light_tree(rb_ctx* ctx, uint32_t n, rb_light_case* cases, void* stream);

/* utility::offsetPoint (src/device/util.h:15-30); in/out 3 floats each. */
int rb_k_offset_point(uint32_t n, const float* p, const float* normal, float* out, void* stream);

/* Octohedral::encodeU32 / decodeU32 (src/core/math_util.h:199-224). */
int rb_k_oct_encode(uint32_t n, const float* v, uint32_t* out, void* stream);
int rb_k_oct_decode(uint32_t n, const uint32_t* code, float* out, void* stream);

/* Closest-hit query against the context's BVH, returning the hit record in
 * the reference's 24-word payload layout (src/kernels/optix_programs_desc.h,
 * written by __closesthit__triangle / __miss__miss, pathtrace.cu:86-236) plus
 * the hit distance and the canonical triangle id (-1 on a miss). rays: 6
 * floats (o, d) each; tmin 0, tmax FLT_MAX as the raygen traces. */
int rb_k_trace(rb_ctx* ctx, uint32_t n, const float* rays, uint32_t* payload24,
               float* t, int32_t* tri, void* stream);
/* Any-hit occlusion on [0, tmax) (pathtrace.cu:1708-1719); out 1 = occluded. */
int rb_k_occluded(rb_ctx* ctx, uint32_t n, const float* rays, const float* tmax,
                  uint32_t* out, void* stream);

/* renderResolve + AgX tonemap (src/kernels/image.cu:16-121) over a caller
 * buffer: render_data is width*height double4 (sum X, Y, Z, count) in device
 * memory, out_rgba width*height RGBA8 in device memory (row-major), colorspace
 * 9 floats in host memory (column-major XYZ -> RGB). */
int rb_k_resolve(uint32_t width, uint32_t height, const float* colorspace, float exposure_scale,
                 const double* render_data, uint8_t* out_rgba, void* stream);

/* Environment-map 2D CDF (src/kernels/cdf.cu:332-535), in device memory:
 * rgba is w*h float4; outputs the inverted conditional (w*h) and marginal
 * (h) uint16 index tables and the integral divided by w*h, as
 * loadEnvironmentMap stores them (src/core/rendering_interface.cpp:1404-1431).
 * mode 0 = float32 sums in the reference's scan order (bit-exact indices),
 * mode 1 = float64 row/column sums. scratch must hold
 * rb_envmap_cdf_scratch_bytes(w, h) bytes of device memory; its contents on
 * entry do not matter (the call zeroes its completion counter on `stream`
 * before the build). */
size_t rb_envmap_cdf_scratch_bytes(uint32_t width, uint32_t height);
int rb_envmap_cdf(uint32_t width, uint32_t height, const float* rgba, int mode,
                  void* scratch, uint16_t* conditional_idx, uint16_t* marginal_idx,
                  float* integral, void* stream);

/* The same CDF build without any device allocation: it has no counterpart
 * in the reference. It is for callers that must not allocate device memory
 * once they are running, for example a host application or plugin host that
 * owns a fixed device-memory budget, or a per-frame loop that cannot afford
 * cudaMalloc / cudaFree (both may synchronise the whole device). The caller
 * still passes the image and the output tables; the scratch is a fixed
 * static device array inside this library, sized for images up to 8192
 * rows (about 100 KB), held by every GPU that loads the library until the
 * process exits. Taller images return RB_ERR_TOO_LARGE. Every call looks the
 * array's device address up in the current context (cudaGetSymbolAddress,
 * which allocates nothing); the first lookup on a device may load this
 * library's device code, so make the first call on a device before any
 * stream capture. All calls share the one array:
 * calls that overlap on the GPU (on different streams, or from different
 * threads) race, so serialise them. */
int rb_envmap_cdf_noalloc(uint32_t width, uint32_t height, const float* rgba, int mode,
                          uint16_t* conditional_idx, uint16_t* marginal_idx, float* integral,
                          void* stream);

/* The light tree built on the device (no reference counterpart as code: the
 * reference builds it on the host, LightTree::Builder,
 * src/core/light_tree.cpp:47-418, which rb_build_light_tree restates). Same
 * inputs and output layouts as rb_build_light_tree, all in device memory
 * except `camera` (host, 3 doubles): world (9 floats per emissive triangle),
 * flux, material and primitive per triangle, uvs (6 floats per triangle: the
 * emission texture's coordinates at its vertices, copied into the records;
 * NULL for zeros); outputs triangles (68-byte
 * EmissiveTriangleLightData, camera-relative), nodes (at most 2n - 1 32-byte
 * PackedNode), pointers (n), bitmasks (n) and *node_count (device). The tree
 * is a binned-SAOH tree in the reference's layouts, not a byte copy of the
 * host builder's. scratch: rb_k_build_light_tree_scratch_bytes(n) bytes of
 * device memory (contents on entry do not matter). Stream-ordered. */
size_t rb_k_build_light_tree_scratch_bytes(uint32_t n);
int rb_k_build_light_tree(uint32_t n, const float* world, const float* flux, const uint32_t* material,
                          const uint32_t* primitive, const float* uvs, const double* camera, void* scratch,
                          void* triangles,
                          void* nodes, uint32_t* pointers, uint64_t* bitmasks, uint32_t* node_count, void* stream);

/* Regenerates the multiple-scattering compensation tables (no counterpart in
 * the reference, which ships them as bin/*.bin without a generator) by Monte
 * Carlo integration of the BxDF lobes: `samples` visible-normal samples per
 * texel, on the reference's grids (i / 31 per axis). Outputs (device, 32x32
 * and 32^3 floats, the layouts rb_set_luts takes): conductor albedo;
 * dielectric albedo, eta > 1 and eta < 1; reflective share, eta > 1 and
 * eta < 1 (definitions in rb_lut.cu). */
int rb_k_generate_luts(uint32_t samples, float* conductor, float* dielectric_outer, float* dielectric_inner,
                       float* reflective_outer, float* reflective_inner, void* stream);

/* Regenerates the sheen LTC table (the reference's bin/sheenLUT.bin, no
 * generator shipped): per texel (x = cos theta_o = i / 31, at least 0.01;
 * y = sheen roughness alpha = j / 31) the LTC coefficients A, B and the
 * albedo R of a volumetric sheen layer simulated by random walks (`paths`
 * per texel; definitions in rb_lut.cu), A and B fitted by maximum
 * likelihood. Output: 32 x 32 float4 (A, B, R, 0) in device memory, the
 * layout rb_set_luts takes. Stream-ordered. */
int rb_k_generate_sheen_lut(uint32_t paths, float* sheen, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RATBITE_B200_KERNELS_H */
