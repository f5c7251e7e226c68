/*
 * qmcrt_bench.h - measurement helpers of the B200 ray tracer (no
 * counterpart in the reference): the roofline denominators of the tracing
 * kernel, measured on the current CUDA device.
 */
#ifndef QMCRT_BENCH_H
#define QMCRT_BENCH_H

#ifdef __cplusplus
extern "C" {
#endif

/* Non-tensor FP32 FMA throughput, TFLOP/s (an FMA counts as 2 flops). */
int qmcrt_microbench_fp32(double* tflops);
/* Float atomicAdd throughput into an n_pixels image at hashed addresses, 1e9/s. */
int qmcrt_microbench_atomics(int n_pixels, double* giga_per_s);

#ifdef __cplusplus
}
#endif

#endif
