/* neon_b200_probe.h -- measurement utility, not part of the neon-facing drop-in interface.
 *
 * No counterpart in the reference: neon publishes no throughput numbers.  The element kernel's
 * compute roofline needs the device's FP64 / FP32 CUDA-core FMA rate, which the platform's
 * peak file does not carry, so it is measured with this probe next to every benchmark run. */
#ifndef NEON_B200_PROBE_H
#define NEON_B200_PROBE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Dense FMA-chain kernel on device 0; writes achieved FLOP/s (2 per FMA).  fp64 != 0 for FP64. */
int nb2_probe_fma_throughput(int32_t fp64, double* flops_per_second);

#ifdef __cplusplus
}
#endif

#endif
