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
 * row-major [out][in]: 4 x 64 x 64, then the output layer as 16 x 64 whose
 * rows 4..15 stay zero). */
size_t rb_nrc_grid_size(void);
size_t rb_nrc_weight_count(void);
/* Host copies of the FP32 master parameters (synchronizes). Setting them
 * also resets the optimiser's moments. */
int rb_nrc_set_parameters(rb_nrc* nrc, const float* grid_host, const float* weights_host);
int rb_nrc_get_parameters(rb_nrc* nrc, float* grid_host, float* weights_host);
/* outputs[n][4] = network(inputs[n][kNrcInputs]), stream-ordered. */
int rb_nrc_infer(rb_nrc* nrc, uint32_t n, const float* inputs, float* outputs, void* stream);
/* One optimisation step on n (input, target[4]) pairs; loss_out (host or
 * device, may be NULL) receives the batch's mean relative L2 loss before the
 * step, stream-ordered. */
int rb_nrc_train(rb_nrc* nrc, uint32_t n, const float* inputs, const float* targets, float* loss_out,
                 void* stream);

/* The gradients of the batch's mean loss with respect to the FP32 master
 * parameters (grid and weights, host buffers of the sizes above), without an
 * optimiser step; synchronizes. For checking the backward pass. */
int rb_nrc_gradients(rb_nrc* nrc, uint32_t n, const float* inputs, const float* targets, float* grid_grad_host,
                     float* weight_grad_host);

#ifdef __cplusplus
}
#endif
#endif /* RATBITE_B200_NRC_H */
