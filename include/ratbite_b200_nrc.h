/*
 * ratbite_b200 — neural radiance cache (a learned form on top of the plain
 * path; no counterpart in the reference).
 *
 * A multiresolution hash-grid encoding (16 levels x 2 features, 2^19 FP16
 * entries per level) and a 4 x 64 MLP (BF16 weights and activations on the
 * tensor cores, FP32 accumulation) map a path vertex to the radiance it
 * scatters toward the previous vertex at the four hero wavelengths. It is
 * trained online (relative L2 loss, Adam) on radiance estimates that the
 * renderer's own paths produce. All pointers passed to the calls below are
 * device pointers unless stated otherwise.
 */
#ifndef RATBITE_B200_NRC_H
#define RATBITE_B200_NRC_H

#include "ratbite_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Floats per query: position in [0,1]^3 (scene bounds), outgoing direction
 * (unit), shading normal (unit), hero wavelength mapped to [0,1]. */
#define kNrcInputs 10

typedef struct rb_nrc rb_nrc;
typedef struct rb_nrc_config {
    int32_t device;
    uint32_t seed;          /* parameter initialisation */
    float learning_rate;    /* Adam; 0: 1e-2 */
    float beta1, beta2;     /* 0: 0.9, 0.99 */
    float epsilon;          /* 0: 1e-15 */
    uint32_t reserved[2];
} rb_nrc_config;

int rb_nrc_create(const rb_nrc_config* config, rb_nrc** out);
int rb_nrc_destroy(rb_nrc* nrc);
/* Parameter counts: grid (16 * 2^19 * 2 floats) and MLP weights (5 matrices,
 * row-major [out][in]: 4 x 64 x 64, then the output layer as 16 x 64: rows
 * 0..3 radiance, row 4 the drop probability that only the cached form of
 * rb_render trains (see below; rb_nrc_train leaves it unchanged), rows 5..15
 * stay zero). */
size_t rb_nrc_grid_size(void);
size_t rb_nrc_weight_count(void);
/* Host copies of the FP32 master parameters (synchronizes). Setting them
 * also resets the optimiser (moments and step count). */
int rb_nrc_set_parameters(rb_nrc* nrc, const float* grid_host, const float* weights_host);
int rb_nrc_get_parameters(rb_nrc* nrc, float* grid_host, float* weights_host);
/* outputs[n][4] = network(inputs[n][kNrcInputs]), stream-ordered; outputs
 * 16-byte aligned. */
int rb_nrc_infer(rb_nrc* nrc, uint32_t n, const float* inputs, float* outputs, void* stream);
/* One optimisation step on n (input, target[4]) pairs, n <= 2^24; loss_out (host or
 * device, may be NULL) receives the batch's mean relative L2 loss before the
 * step, stream-ordered. */
int rb_nrc_train(rb_nrc* nrc, uint32_t n, const float* inputs, const float* targets, float* loss_out,
                 void* stream);

/* RB_DEV_* bits raised by the network's kernels since the handle was created
 * (RB_DEV_ITERATION_LIMIT: a tensor-core wait gave up and its tile was
 * skipped); synchronizes. No reference counterpart. */
int rb_nrc_status(rb_nrc* nrc, uint32_t* flags);

/* The gradients of the batch's mean loss with respect to the FP32 master
 * parameters (grid and weights, host buffers of the sizes above), without an
 * optimiser step; synchronizes. For checking the backward pass. */
int rb_nrc_gradients(rb_nrc* nrc, uint32_t n, const float* inputs, const float* targets, float* grid_grad_host,
                     float* weight_grad_host);

/* ---------------------------------------------------------------------
 * The cached form of rb_render (Mueller et al. 2021). With a cache
 * attached, a path that is not a training path stops at the first vertex
 * whose path spread exceeds the primary vertex's footprint, (sum over
 * vertices 2..n of sqrt(d^2 / (pdf |cos|)))^2 > c * d1^2 / (4 pi |cos1|), and
 * adds throughput x max(cache(vertex), 0) in place of its light sample and
 * further bounces; the emission found on arrival is still added. Paths do
 * not stop at metallic or transmissive surfaces smoother than
 * min_roughness. The plain path drops a whole sample (the radiance gathered
 * before as well) when a later BxDF sample fails (RB_FAILED_DROP, see
 * rb_config), so the cache also learns the probability q of that from the
 * vertex on, and a terminated path keeps (1 - q) of its radiance so far.
 * One path in train_one_in is traced like the plain path and records each
 * vertex; after the wave each record's targets -- (radiance gathered after
 * the vertex) / (throughput at the vertex), zero if the sample was dropped,
 * and 1 if it was dropped, else 0 -- feed the cache's optimiser
 * (targets_per_sample rows per sample plane, in steps of `batch` rows).
 * Queries, targets and steps stay on the device: no host synchronisation.
 * ------------------------------------------------------------------- */
typedef struct rb_cache_params {
    float spread_threshold;        /* c above; 0: 0.01 */
    uint32_t train_one_in;         /* 0: 16; 1: every path trains (none terminates) */
    uint32_t targets_per_sample;   /* 0: 65536 */
    uint32_t batch;                /* rows per optimisation step; 0: 131072 */
    uint32_t frozen;               /* 1: query only (no training paths, no optimisation steps) */
    uint32_t samples_per_wave;     /* sample planes per wave (the cache trains after each wave),
                                      bounded by the wavefront capacity; 0: 8 */
    float scene_min[3], scene_max[3];  /* position normalisation; an empty box: the geometry's bounds */
    float min_roughness;           /* see above; 0: 0.25, negative: no limit */
    uint32_t reserved[3];
} rb_cache_params;

/* cache NULL detaches (rb_render is the plain path again). The cache must
 * live on the context's device and outlive the attachment. */
int rb_attach_radiance_cache(rb_ctx* ctx, rb_nrc* cache, const rb_cache_params* params);

typedef struct rb_cache_stats {
    uint64_t queries;          /* paths terminated into the cache */
    uint64_t records;          /* training vertices recorded */
    uint64_t steps;            /* optimisation steps */
    float last_loss;           /* mean loss of the latest step */
    uint32_t launches;         /* this library's kernels launched for the cache */
    double ms_infer, ms_train; /* device time, with RB_STATS_TIME */
    float drop_bias;           /* correction added to the predicted drop probability of
                                  queries whose camera ray hit an emitter (current value) */
    float drop_bias_other;     /* the same for the other queries */
    float radiance_scale;      /* scale applied to the queries' radiance (current value) */
} rb_cache_stats;
/* Synchronizes, returns what was gathered since the last call, then resets. */
int rb_get_cache_stats(rb_ctx* ctx, rb_cache_stats* out);

#ifdef __cplusplus
}
#endif
#endif /* RATBITE_B200_NRC_H */
