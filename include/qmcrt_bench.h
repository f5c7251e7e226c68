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
/* Replays recorded deposits: device_codes holds n_codes per-ray outcome
 * codes in the tracer's lane order (pixel index >= 0 for a receiver hit, as
 * qmcrt_debug_hit_records writes them); one launch adds 1.0f at every pixel
 * code, `repeats` times over the list, 32 consecutive codes per warp.
 * ms_per_launch receives the launch's device time (after a warm-up launch):
 * hits x repeats / time is the L2 atomic rate of the tracer's own address
 * pattern. */
int qmcrt_microbench_atomics_replay(const int* device_codes, long long n_codes, int n_pixels, int repeats,
                                    double* ms_per_launch);

/* Checks the tracer's own correctly rounded float primitives against CUDA's
 * on every 32-bit input pattern: mismatches[0] = inputs where the device
 * qm_rn_rsqrt (series refinement of the hardware estimate) differs from
 * __frsqrt_rn, mismatches[1] = inputs in [2^-125, 2^125) where the series
 * without its range test (qm_rn_rsqrt_unit) does; over 12 receiver heights h
 * from 1 mm to 1 km and every pattern a, mismatches[2] = quotients
 * qm_div_by_rcp(a, h, RN(1/h)) that differ from __fdiv_rn(a, h) with a and
 * the quotient in [2^-90, 2^90],
 * mismatches[3] = u = quotient + 0.5 that differ while either lies in [0, 1];
 * mismatches[4] = x in [2^-100, 2^126) where the root from the reciprocal
 * root (qm_sqrt_by_rsqrt) differs from __fsqrt_rn, mismatches[5] = |x| in
 * [2^-100, 2^100] where the Newton reciprocal differs from __frcp_rn,
 * mismatches[6] = pairs (2^33 hashed, |a| in [2^-60, 2^70), |b| in
 * [2^-50, 2^64)) where Markstein's division with it differs from __fdiv_rn.
 * Entries past the checks are set to 0. */
int qmcrt_debug_check_primitives(unsigned long long* mismatches, int count);

#ifdef __cplusplus
}
#endif

#endif
