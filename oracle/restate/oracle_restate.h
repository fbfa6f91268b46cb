/* Oracle test infrastructure (not product code): C restatements of the
 * reference's integer / scan algorithms, used to pin the GPU kernels on the
 * CPU and validated against the reference compiled in oracle/_ref. */
#ifndef ORACLE_RESTATE_H
#define ORACLE_RESTATE_H
#include <stdint.h>
/* src/device/quasi_random.h:30-204 */
uint32_t orc_pixel_hash(uint32_t x, uint32_t y);
void orc_sobol(uint32_t n, uint32_t dims, const uint32_t* sample, const uint32_t* hash,
               const uint32_t* bounce, const uint32_t* dim, float* out);
/* src/kernels/cdf.cu:332-535 (mode 0) and the float64 variant (mode 1). */
int orc_envmap_cdf(uint32_t w, uint32_t h, const float* rgba, int mode,
                   uint16_t* cond, uint16_t* marg, float* integral);
#endif
