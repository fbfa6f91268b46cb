/*
 * ratbite_b200 — C ABI of the B200-native per-sample rendering path.
 *
 * This library is a drop-in for what sits below ratbite's OptiX launch:
 * RenderingInterface keeps producing the same scene, material, light-tree,
 * spectral and LUT data (src/core/rendering_interface.cpp) and hands it to
 * these entry points instead of building OptiX acceleration structures and
 * calling optixLaunch. Everything below is plain C: pointers, sizes and
 * status codes. All functions return RB_OK (0) on success and a negative
 * status otherwise; rb_last_error() gives the message. No call aborts, and
 * device-side failures are reported through rb_status() (a status word the
 * kernels set instead of trapping).
 *
 * Coordinates follow the reference's camera-relative convention: instance
 * transforms, emissive triangles and light-tree node means are already offset
 * by -cameraPosition by the caller (src/core/rendering_interface.cpp:986,
 * 1449-1457, 1484-1486); camera rays start at the origin
 * (src/device/dir_gen.h:29).
 */
#ifndef RATBITE_B200_H
#define RATBITE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RB_ABI_VERSION 4

/* Status codes. */
#define RB_OK                  0
#define RB_ERR_INVALID        -1  /* bad argument or inconsistent data */
#define RB_ERR_CUDA           -2  /* a CUDA runtime call failed */
#define RB_ERR_UNSUPPORTED    -3  /* a feature outside this build's scope */
#define RB_ERR_NO_SCENE       -4  /* render called before geometry/launch set-up */
#define RB_ERR_DEVICE         -5  /* a kernel set the device status word */
#define RB_ERR_OOM            -6  /* device allocation failed */
#define RB_ERR_TOO_LARGE      -7  /* input larger than a fixed-size entry point supports */

/* Device status bits (rb_device_status.flags). */
#define RB_DEV_STACK_OVERFLOW   (1u << 0)  /* BVH traversal stack exhausted */
#define RB_DEV_QUEUE_OVERFLOW   (1u << 1)  /* a wavefront queue overflowed */
#define RB_DEV_NAN_RADIANCE     (1u << 2)  /* a path produced a non-finite sample */
#define RB_DEV_ITERATION_LIMIT  (1u << 3)  /* a bounded wait gave up */
#define RB_DEV_BAD_INDEX        (1u << 4)  /* an index read from scene data was out of range */
#define RB_DEV_BAD_GEOMETRY     (1u << 5)  /* a moved vertex is not finite (rb_update_instances) */

/* Index buffer element types (IndexType, src/core/material.h:9-15). */
#define RB_INDEX_U16 0
#define RB_INDEX_U32 1

/* BxDF callable indices (bxdfTypeToIndex, src/core/rendering_interface.cpp:1291-1309). */
#define RB_BXDF_PURE_CONDUCTOR   0
#define RB_BXDF_PURE_DIELECTRIC  1
#define RB_BXDF_COMPLEX_SURFACE  2

/* Bitfields of MaterialData (src/core/material.h:19-60), same bit values. */
#define RB_ATTR_NORMAL       (1u << 0)
#define RB_ATTR_FRAME        (1u << 1)
#define RB_ATTR_COLOR        (1u << 2)
#define RB_ATTR_TEX_COORD_1  (1u << 3)
#define RB_ATTR_TEX_COORD_2  (1u << 4)
#define RB_FACTOR_BASE_COLOR   (1u << 0)
#define RB_FACTOR_METALNESS    (1u << 1)
#define RB_FACTOR_ROUGHNESS    (1u << 2)
#define RB_FACTOR_TRANSMISSION (1u << 3)
#define RB_FACTOR_CUTOFF       (1u << 4)
#define RB_FACTOR_BLEND        (1u << 5)
#define RB_FACTOR_SHEEN_COLOR  (1u << 6)
#define RB_FACTOR_SHEEN_ROUGH  (1u << 7)
#define RB_FACTOR_EMISSION     (1u << 8)
/* rb_material.textures bits and texture slots (MaterialData::TextureTypeBitfield,
 * src/core/material.h:30-41): bit t set = texture_index[t] is used. */
#define RB_TEXTURE_BASE_COLOR   0u
#define RB_TEXTURE_NORMAL       1u
#define RB_TEXTURE_MET_ROUGH    2u
#define RB_TEXTURE_TRANSMISSION 3u
#define RB_TEXTURE_SHEEN_COLOR  4u
#define RB_TEXTURE_SHEEN_ROUGH  5u
#define RB_TEXTURE_EMISSION     6u
#define RB_TEXTURE_SLOTS        7u
/* rb_texture.format: 8-bit channels read as normalized floats (the
 * reference's R8_UNORM / R8G8B8A8_UNORM images, cudaReadModeNormalizedFloat),
 * with the sRGB curve applied per texel before filtering when `srgb` is set
 * (texDesc.sRGB, set for base-colour textures; src/core/texture.h:245-265). */
#define RB_TEXFMT_R8     0u
#define RB_TEXFMT_RGBA8  1u
/* rb_texture.address_u / address_v (TextureAddress, src/core/texture.h:33-38) */
#define RB_TEXADDR_WRAP   0u
#define RB_TEXADDR_CLAMP  1u
#define RB_TEXADDR_MIRROR 2u
/* rb_texture.filter (TextureFilter) */
#define RB_TEXFILTER_NEAREST 0u
#define RB_TEXFILTER_LINEAR  1u

#define RB_SPECTRUM_BINS 471   /* 360..830 nm, src/core/spectral_settings.h:5-9 */
#define RB_LUT_SIZE 32         /* LUT edge, src/core/rendering_interface.cpp:530-533 */

typedef struct rb_ctx rb_ctx;

typedef struct rb_config {
    int32_t device;              /* CUDA device ordinal */
    uint32_t max_paths_in_flight;/* wavefront capacity; 0 = default (16M paths) */
    uint32_t envmap_cdf_mode;    /* RB_CDF_FP64 (default, 0) or RB_CDF_REFERENCE */
    uint32_t failed_sample_mode; /* RB_FAILED_DROP (default, 0) or RB_FAILED_KEEP */
    /* Fault injection for tests (no reference counterpart), all 0 in normal use:
     * inject_queue_limit    wavefront queues accept at most this many entries
     *                       per bounce (the rest are dropped and
     *                       RB_DEV_QUEUE_OVERFLOW is set); 0 = their capacity;
     * inject_alloc_failure  the n-th device allocation of the context (1-based,
     *                       counted over all calls) fails once, as an
     *                       out-of-memory cudaMalloc would; 0 = none;
     * inject_stack_limit    BVH traversal stacks hold at most this many entries
     *                       (RB_DEV_STACK_OVERFLOW when one is full); 0 = the
     *                       full stack. */
    uint32_t inject_queue_limit;
    uint32_t inject_alloc_failure;
    uint32_t inject_stack_limit;
    uint32_t acceleration;       /* RB_ACCEL_FLAT (default, 0) or RB_ACCEL_INSTANCED */
} rb_config;
/* Ray-traversal structure built by rb_set_geometry. RB_ACCEL_FLAT: one BVH
 * over every instance's triangles in world space (memory and instance
 * updates scale with the instanced triangles). RB_ACCEL_INSTANCED: two
 * levels, as the reference's GAS per mesh and IAS over instances
 * (src/core/rendering_interface.cpp:733-848, 943-1064): one BVH per unique
 * mesh and per emissive subset in object space, and a top-level BVH over
 * the instances' world boxes that rb_update_instances rebuilds on the host
 * (memory scales with the unique triangles, an instance update with the
 * instance count). Both give bit-identical hits and images: rays enter
 * object space for the box tests, and triangles are intersected in world
 * space after the same transform the flat upload applies. The shared
 * wavefront (rb_render_jobs) takes flat contexts only. */
#define RB_ACCEL_FLAT       0u
#define RB_ACCEL_INSTANCED  1u
/* A BxDF sample that fails (a direction on the wrong side of the shading
 * hemisphere, a zero or infinite pdf) sets the path's terminated flag. The
 * reference then drops the whole sample, radiance gathered before included
 * (src/kernels/pathtrace.cu:1789-1812): RB_FAILED_DROP, the default. With
 * RB_FAILED_KEEP the path ends there and keeps what it gathered. */
#define RB_FAILED_DROP    0u
#define RB_FAILED_KEEP    1u
#define RB_CDF_FP64       0u     /* float64 row/column sums */
#define RB_CDF_REFERENCE  1u     /* float32 in the reference's scan order: bit-identical tables */

/*
 * One material record: MaterialData (src/core/material.h:17-107) field for
 * field, minus OptiX specifics; texture objects are indices into the table
 * of rb_set_textures. The index and attribute buffers are the per-submesh
 * vertex data the shading step reads (src/kernels/pathtrace.cu:1290-1431);
 * they are copied at upload.
 */
typedef struct rb_material {
    uint32_t bxdf;               /* RB_BXDF_* (bxdfIndexSBT) */
    uint32_t double_sided;
    uint32_t sheen_present;
    uint32_t index_type;         /* RB_INDEX_U16 / RB_INDEX_U32 */
    uint32_t attributes;         /* RB_ATTR_* bits */
    uint32_t attribute_stride;   /* bytes per vertex in attribute_data; it and the offsets of
                                  * the fields present are multiples of 8 (the reference's
                                  * packing: frame 16 B or normal 8 B, then 8 B per set) */
    uint32_t normal_offset, frame_offset, color_offset, texcoord1_offset, texcoord2_offset;
    uint32_t ior_spectrum;       /* index into the extra spectra (indexOfRefractSpectrumDataIndex) */
    uint32_t absorp_spectrum;    /* absorpCoefSpectrumDataIndex */
    uint32_t emission_spectrum;  /* emissionSpectrumDataIndex (not read on the device) */
    float mf_roughness;          /* mfRoughnessValue */
    float ior;
    float alpha_cutoff;
    uint32_t textures;           /* bit RB_TEXTURE_*: that slot of texture_index is sampled */
    uint32_t factors;            /* RB_FACTOR_* bits */
    float base_color[4];
    float metalness;
    float roughness;
    float transmission;
    float sheen_color[3];
    float sheen_roughness;
    float emissive[3];
    uint32_t triangle_count;     /* triangles in `indices` */
    const void* indices;         /* triangle_count * 3 indices of index_type */
    uint32_t vertex_count;       /* vertices in attribute_data */
    const void* attribute_data;  /* vertex_count * attribute_stride bytes, or NULL */
    uint32_t texcoord_sets;      /* bit RB_TEXTURE_*: that texture reads texture coordinate set 2
                                  * (the *TexCoordSetIndex flags) */
    uint32_t texture_index[RB_TEXTURE_SLOTS];  /* per slot, an index into the rb_set_textures table */
} rb_material;

/* One texture of the rb_set_textures table (an image with its sampler:
 * CudaCombinedTexture, src/core/texture.h:280-380). Texels are width x
 * height, row-major from the first row of the image, 1 (RB_TEXFMT_R8) or 4
 * bytes each; normalized coordinates, texel centres at (i + 0.5) / width. */
typedef struct rb_texture {
    uint32_t width, height;
    uint32_t format;             /* RB_TEXFMT_* */
    uint32_t srgb;               /* 1: the sRGB curve decodes r, g, b (r of an R8 texture) */
    uint32_t address_u, address_v;  /* RB_TEXADDR_* */
    uint32_t filter;             /* RB_TEXFILTER_* */
    uint32_t reserved;
    const void* data;            /* copied at upload */
} rb_texture;

/* Geometry: meshes of submeshes, placed by instances (SceneData::Mesh /
 * Submesh / Instance, src/core/scene.h:85-152). */
typedef struct rb_submesh {
    uint32_t material;           /* index into the rb_set_materials table (hit-group data) */
    uint32_t index_type;         /* RB_INDEX_U16 / RB_INDEX_U32 */
    uint32_t triangle_count;
    const void* indices;         /* triangle_count * 3 indices */
    uint32_t vertex_count;
    const float* vertices;       /* vertex_count * 4 floats: x, y, z, unused */
    uint32_t discarded_count;    /* primitives made degenerate (emissive ones, cut out) */
    const uint32_t* discarded;
} rb_submesh;

typedef struct rb_mesh {
    uint32_t submesh_count;
    const rb_submesh* submeshes;
} rb_mesh;

typedef struct rb_instance {
    uint32_t mesh;
    float transform[12];         /* object to camera-relative world, row-major 3x4 */
} rb_instance;

/* Emissive triangles are traced as their own instances, as the reference
 * builds one GAS per emissive subset (src/core/rendering_interface.cpp:849-942);
 * their primitive indices run over all subsets in order and index the
 * light-tree triangle table. */
typedef struct rb_emissive_subset {
    float transform[12];         /* object to camera-relative world, row-major 3x4 */
    uint32_t triangle_count;
    const float* vertices;       /* triangle_count * 9 floats, object space */
} rb_emissive_subset;

typedef struct rb_geometry {
    uint32_t mesh_count;
    const rb_mesh* meshes;
    uint32_t instance_count;
    const rb_instance* instances;
    uint32_t emissive_subset_count;
    const rb_emissive_subset* emissive_subsets;
} rb_geometry;

/* Light tree in the reference's byte layouts: EmissiveTriangleLightData
 * (68 B, src/core/light_tree_types.h:40-46), PackedNode (32 B, :119-163),
 * LightPointer (4 B, :191-207) and the per-triangle 64-bit path bitmasks
 * (src/core/light_tree.cpp:153-157). */
typedef struct rb_light_tree {
    uint32_t triangle_count;
    const void* triangles;
    uint32_t node_count;
    const void* nodes;
    uint32_t pointer_count;
    const uint32_t* pointers;
    const uint64_t* bitmasks;    /* triangle_count entries */
} rb_light_tree;

/* Launch parameters (LaunchParameters::ResolutionState / PathState /
 * CameraState, src/core/launch_parameters.h:18-50). */
typedef struct rb_launch {
    uint32_t width, height;
    float inv_width, inv_height;
    float perspective_scale_w, perspective_scale_h;
    uint32_t max_path_depth;
    uint32_t max_reflected_depth;
    uint32_t max_transmitted_depth;
    float cam_u[3], cam_v[3], cam_w[3];
    uint32_t dof_enabled;
    float aperture;
    float focus_distance;
} rb_launch;

typedef struct rb_device_status {
    uint32_t flags;              /* RB_DEV_* bits accumulated since the last reset */
    uint32_t first_code_detail;  /* implementation detail of the first failure */
    uint64_t paths_traced;       /* paths finished since rb_create */
    uint64_t rays_traced;        /* extension + shadow rays since rb_create */
} rb_device_status;

/* ---- context ---------------------------------------------------------- */
int rb_create(const rb_config* config, rb_ctx** out);
int rb_destroy(rb_ctx* ctx);
const char* rb_last_error(const rb_ctx* ctx);
int rb_abi_version(void);

/* ---- scene upload (RenderingInterface data producers) ------------------ */
/* Replaces loadLookUpTables' textures (src/core/rendering_interface.cpp:528-622):
 * conductor 32x32, four dielectric 32x32x32 and sheen-LTC 32x32 float4, the
 * layouts of bin/*.bin. */
int rb_set_luts(rb_ctx* ctx, const float* conductor_albedo,
                const float* dielectric_outer, const float* dielectric_inner,
                const float* reflective_outer, const float* reflective_inner,
                const float* sheen_ltc);
/* Replaces fillSpectralCurvesData (:518) and the spectra table (:1198-1258):
 * sensor curves X,Y,Z and RGB basis as 3 x 471 floats each, plus `extra`
 * dense spectra (n_extra x 471) indexed by rb_material spectrum indices. */
int rb_set_spectra(rb_ctx* ctx, const float* sensor_xyz, const float* basis_rgb,
                   const float* extra, uint32_t n_extra);
int rb_set_materials(rb_ctx* ctx, const rb_material* materials, uint32_t count);
/* The texture table materials index (replaces the images and textures of
 * fillModelMaterials, src/core/rendering_interface.cpp:46-66). Set it before
 * the materials that use it; materials are checked against it. */
int rb_set_textures(rb_ctx* ctx, const rb_texture* textures, uint32_t count);
/* Replaces buildGeometryAccelerationStructures (:733), buildLightAccelerationStructure
 * (:849) and updateInstanceAccelerationStructure (:943): builds the wide BVH. */
int rb_set_geometry(rb_ctx* ctx, const rb_geometry* geometry);
/* Replaces fillLightDataBuffer / fillLightTreeDataBuffers (:1433, :1470). */
/* Moves the instances of the last rb_set_geometry (replaces
 * updateInstanceAccelerationStructure, src/core/rendering_interface.cpp
 * :943-1063, run by the reference on every camera move): new camera-relative
 * 3x4 transforms, instance_transforms[12 * instance_count] in the order of
 * rb_geometry.instances and subset_transforms[12 * emissive_subset_count] in
 * the order of rb_geometry.emissive_subsets. World vertices, geometric normals
 * and the BVH boxes are recomputed on the device (the tree topology is kept),
 * stream-ordered on `stream`; the results equal those of rb_set_geometry with
 * the same transforms. The light data follows with rb_set_light_origin. */
int rb_update_instances(rb_ctx* ctx, const float* instance_transforms, const float* subset_transforms,
                        void* stream);
/* Light data: emissive triangles, light-tree nodes, light pointers, path
 * bitmasks. The triangle vertices and node means are taken relative to the
 * light origin (rb_set_light_origin; 0 until set, which uses them as given). */
int rb_set_lights(rb_ctx* ctx, const rb_light_tree* tree);
/* Builds the light tree on the device from emissive triangles in device
 * memory (world: 9 floats each, flux, material, primitive; the inputs
 * rb_build_light_tree takes, origin-independent; uvs: 6 floats each, the
 * emission texture's coordinates at the triangle's vertices, or NULL when no
 * emitter has an emission texture) and installs it as
 * rb_set_lights installs host-built records, the light origin of
 * rb_set_light_origin applied. No reference counterpart: the reference
 * rebuilds on the host (LightTree::Builder, src/core/light_tree.cpp:47-418)
 * on every light change. The tree is a binned-SAOH tree in the reference's
 * layouts (rb_k_build_light_tree). Synchronizes. */
int rb_build_lights(rb_ctx* ctx, uint32_t n, const float* world, const float* flux, const uint32_t* material,
                    const uint32_t* primitive, const float* uvs, void* stream);
/* The camera-move refresh of the light data on the device (the reference's
 * fillLightDataBuffer and fillLightTreeDataBuffers,
 * src/core/rendering_interface.cpp:1433-1510, run on CHANGE_CAMERA_POS
 * :1615-1622, 1810-1820): every emissive-triangle vertex and light-tree mean
 * becomes (value given to rb_set_lights) - origin, one float subtraction per
 * coordinate as the reference computes it on the host, and the tree is
 * unpacked again; stream-ordered on `stream`. */
int rb_set_light_origin(rb_ctx* ctx, const float origin[3], void* stream);
/* Host light-tree build (LightTree::Builder, src/core/light_tree.cpp:47-418,
 * driven as RenderingInterface::buildLightTree, src/core/rendering_interface.cpp:
 * 1065-1167): n emissive triangles with world-space vertices (9 floats each),
 * flux (already scaled by the instance's flux correction), material and
 * primitive indices, and the camera position. Writes the camera-relative
 * EmissiveTriangleLightData records (n x 68 B), the PackedNode array
 * (capacity 2n x 32 B), n light pointers and n path bitmasks, in the
 * reference's layouts and order; *out_node_count receives the node count.
 * Needs no device. */
int rb_build_light_tree(uint32_t n, const float* world_vertices, const float* flux,
                        const uint32_t* material, const uint32_t* primitive,
                        const double* camera_position, void* out_triangles, void* out_nodes,
                        uint32_t* out_pointers, uint64_t* out_bitmasks, uint32_t* out_node_count);
/* Replaces loadEnvironmentMap's CDF launches (:1339-1432): rgba is w*h float4
 * (w, h multiples of 4); the 2D CDF is built on the device. */
int rb_set_envmap(rb_ctx* ctx, const float* rgba, uint32_t width, uint32_t height);
/* Rebuilds the CDF of the resident map on `stream` (the per-frame rebuild of
 * the at-scale workload); stream-ordered, no host synchronisation. */
int rb_rebuild_envmap_cdf(rb_ctx* ctx, void* stream);
int rb_clear_envmap(rb_ctx* ctx);
int rb_set_launch(rb_ctx* ctx, const rb_launch* launch);

/* ---- render (replaces optixLaunch, :1873-1879) ------------------------- */
/* Renders samples [sample_offset, sample_offset + sample_count) of every pixel
 * into the FP64 accumulation buffer. sample_offset == 0 restarts the
 * accumulation (src/kernels/pathtrace.cu:1120). `stream` is a cudaStream_t or
 * NULL for the library stream; the call is asynchronous with respect to the
 * host. */
int rb_render(rb_ctx* ctx, uint32_t sample_offset, uint32_t sample_count, void* stream);
/* rb_render with the call's wave sequence captured once as a CUDA graph and
 * replayed (no reference counterpart: the reference launches one OptiX
 * pipeline per sub-launch): the same accumulation bit for bit, one kernel
 * launch plus one graph launch per call instead of ~8 launches per bounce.
 * A graph is kept per sample_count (up to 8) for the current scene state;
 * any setter, a new launch size or a new wave capacity captures anew. With a
 * radiance cache attached or statistics on, it is rb_render. */
int rb_render_graph(rb_ctx* ctx, uint32_t sample_offset, uint32_t sample_count, void* stream);

/* Several render jobs in one shared wavefront (no reference counterpart:
 * the reference renders one scene per launch). Job j is context jobs[j] with
 * its own scene, launch parameters and accumulation buffer; it renders
 * samples [offsets[j], offsets[j] + counts[j]) as rb_render(jobs[j], ...)
 * would (the same sample sequences and accumulation order, so the same
 * bits). Waves are filled with whole sample planes of the jobs in order and
 * mix jobs freely: every kernel of a wave serves all of its jobs' paths, each
 * path reading its job's scene. The wave buffers live in jobs[0]. Plain form
 * only (no attached radiance cache); films up to 65535 pixels a side. Jobs
 * must not render elsewhere while the call runs. Stream-ordered on `stream`
 * (0: jobs[0]'s stream) after the job and chunk tables are copied. */
typedef struct rb_jobs_options {
    uint32_t max_paths_in_flight; /* wave capacity (queue capacity) in paths; 0 = jobs[0]'s */
    uint32_t grid_percent;        /* blocks per kernel launch, % of the resident maximum; 0 = 100 */
    void* const* done_events;     /* per job a cudaEvent_t recorded on `stream` after the wave that
                                     finishes the job, or NULL */
} rb_jobs_options;
int rb_render_jobs(rb_ctx* const* jobs, uint32_t n, const uint32_t* offsets, const uint32_t* counts,
                   const rb_jobs_options* options, void* stream);
/* Copies the width*height*4 doubles (sum X, sum Y, sum Z, sample count) of
 * the accumulation buffer (renderData) to host memory; synchronizes. */
int rb_read_accum(rb_ctx* ctx, double* out);
/* Overwrites the accumulation buffer from host memory (width*height
 * double4, the layout rb_read_accum returns); synchronizes. With the next
 * sample offset, what a checkpoint needs to resume a progressive render
 * exactly: rb_render(ctx, offset, ...) with offset > 0 adds to it. No
 * reference counterpart (its accumulation lives only in the process). */
int rb_write_accum(rb_ctx* ctx, const double* in);
/* Device pointer of the accumulation buffer (width*height double4). */
int rb_accum_device_ptr(rb_ctx* ctx, void** out);
/* Stream-ordered copy of the accumulation buffer to `dst` (device or pinned
 * host memory, width*height*4 doubles), on `stream` (NULL: context stream). */
int rb_copy_accum_async(rb_ctx* ctx, void* dst, void* stream);
/* ---- progressive rendering (RenderingInterface::render,
 * updateSubLaunchData, updateSamplingState and the restart of
 * processCommands, src/core/rendering_interface.cpp:1830-1839, 1846-1872,
 * 1980-2013) ---------------------------------------------------------------- */
#define RB_MODE_IMMEDIATE 0   /* one sample per sub-launch (RenderContext::Mode) */
#define RB_MODE_GRADUAL   1   /* sub-launches grow as min(int(max(3, n)^1.5), 64) */
typedef struct rb_progress {
    uint32_t launched_offset;  /* first sample of the sub-launch this step started */
    uint32_t launched_count;   /* its sample count (0: nothing left to render) */
    uint32_t processed;        /* samples per pixel complete before it (m_processedSampleCount) */
    uint32_t total;            /* target samples per pixel */
    uint32_t finished;         /* 1 once every sample has been launched */
    uint32_t reserved;
} rb_progress;
/* Restarts the progressive render: the next step renders sample 0 alone and
 * restarts the accumulation, as a scene or camera change does. */
int rb_progressive_restart(rb_ctx* ctx, uint32_t total_samples, int mode);
/* Launches the current sub-launch (rb_render, asynchronous on `stream`) and
 * advances the schedule; a step after the last sample reports finished. */
int rb_progressive_step(rb_ctx* ctx, void* stream, rb_progress* out);
/* The schedule alone: writes up to `capacity` (offset, count) pairs of the
 * sub-launches of a render of total_samples in `mode`; returns their number
 * (negative on bad arguments). No device needed. */
int rb_progressive_plan(uint32_t total_samples, int mode, uint32_t* offsets, uint32_t* counts, uint32_t capacity);

/* ---- resolve (replaces resolveRender, src/core/rendering_interface.cpp
 * :1512-1532, and the GL image it writes) -------------------------------- */
/* Resolves the accumulation into the context's headless image: per pixel
 * sum/count, max(., 0) * exposure_scale, the XYZ -> RGB `colorspace` matrix
 * (9 floats, column-major as glm::mat3; Color::generateColorspaceConversionMatrix,
 * src/core/color.h:60-99), the AgX tonemap and 8-bit quantisation
 * (renderResolve + tonemap, src/kernels/image.cu:16-121). The reference passes
 * exposure_scale = 2^(exposure - 7). The image is width*height RGBA8, row-major,
 * owned by the context; stream-ordered on `stream` (NULL: context stream). */
int rb_resolve(rb_ctx* ctx, const float colorspace[9], float exposure_scale, void* stream);
/* Copies the width*height*4 bytes of the resolved image to host memory;
 * synchronizes. */
int rb_read_image(rb_ctx* ctx, uint8_t* out);
/* Device pointer of the resolved image (width*height RGBA8 words). */
int rb_image_device_ptr(rb_ctx* ctx, void** out);
/* Zeroes the accumulation buffer, stream-ordered. No reference counterpart
 * (the reference restarts only through sample_offset == 0): a rank that
 * renders its own sample range [offset, offset + count) of a frame with
 * offset > 0 starts its frame with this call. */
int rb_clear_accum(rb_ctx* ctx, void* stream);
int rb_status(rb_ctx* ctx, rb_device_status* out);
int rb_clear_status(rb_ctx* ctx);
int rb_synchronize(rb_ctx* ctx);

/* ---- per-stage instrumentation (no counterpart in the reference, which has
 * only -lineinfo; cudaEvent timers per stage) --------------------------- */
#define RB_STATS_COUNT 1u   /* count traversal work: nodes and triangles visited (slower kernels) */
#define RB_STATS_TIME  2u   /* time each kernel class with CUDA events on the render stream */
typedef struct rb_render_stats {
    uint64_t extend_rays, extend_nodes, extend_tris;
    uint64_t shadow_rays, shadow_nodes, shadow_tris;
    uint64_t waves;
    double ms_generate, ms_extend, ms_shade, ms_shadow, ms_resolve;
    uint32_t launches_generate, launches_extend, launches_shade, launches_shadow, launches_resolve;
    uint32_t reserved;
    /* the shading stage per kernel: ms_shade = ms_surface + ms_nee + ms_bsdf
     * (hit record, emission and frame; light sample; BxDF and next ray) */
    double ms_surface, ms_nee, ms_bsdf;
    uint32_t launches_nee, launches_bsdf;   /* launches_shade counts the surface and deferred-emission kernels */
    uint64_t surface_records;               /* path vertices shaded (RB_STATS_COUNT) */
} rb_render_stats;
int rb_set_stats(rb_ctx* ctx, uint32_t mode);
/* Synchronizes, returns what was gathered since the last call, then resets. */
int rb_get_stats(rb_ctx* ctx, rb_render_stats* out);

#ifdef __cplusplus
}
#endif
#endif /* RATBITE_B200_H */
