// Roofline denominators measured on the running GPU: non-tensor FP32 FMA
// throughput and L2 float-atomic throughput (include/qmcrt_bench.h).
#include <cuda_runtime.h>
#include <stdint.h>

#include "qmcrt_bench.h"
#include "vecmath.h"

namespace {

// Own correctly rounded primitives against CUDA's, one float bit pattern per
// thread (bits = begin + thread index): counts[0] = patterns where
// qm_rn_rsqrt differs from __frsqrt_rn (bit for bit; NaN results compare as
// NaN), counts[1] = patterns in [2^-125, 2^125) where qm_rn_rsqrt_unit (no
// range test) does.
__global__ void primitives_kernel(unsigned begin, unsigned long long* counts) {
  const unsigned bits = begin + blockIdx.x * blockDim.x + threadIdx.x;
  const float x = __uint_as_float(bits);
  const float a = qm_rn_rsqrt(x), b = __frsqrt_rn(x);
  if (__float_as_uint(a) != __float_as_uint(b) && !(a != a && b != b)) atomicAdd(counts + 0, 1ull);
  if (x >= 0x1p-125f && x < 0x1p125f && __float_as_uint(qm_rn_rsqrt_unit(x)) != __float_as_uint(b))
    atomicAdd(counts + 1, 1ull);
  // counts[4]: the root from the reciprocal root, x in [2^-100, 2^126);
  // counts[5]: the Newton reciprocal, |x| in [2^-100, 2^100]
  if (x >= 0x1p-100f && x < 0x1p126f && __float_as_uint(qm_sqrt_by_rsqrt(x, b)) != __float_as_uint(__fsqrt_rn(x)))
    atomicAdd(counts + 4, 1ull);
  const float ax = fabsf(x);
  if (ax >= 0x1p-100f && ax <= 0x1p100f && __float_as_uint(qm_rcp_newton(x)) != __float_as_uint(__frcp_rn(x)))
    atomicAdd(counts + 5, 1ull);
}

__device__ __forceinline__ unsigned mix32(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
// counts[6]: Markstein division with the Newton reciprocal against __fdiv_rn
// on hashed pairs, |a| in [2^-60, 2^70), |b| in [2^-50, 2^64) (random
// significands, signs and exponents), and on pairs whose quotient is close
// to a small integer plus a half (a = RN(b (k + 0.5))).
__global__ void division_pairs_kernel(unsigned seed, unsigned long long* counts) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned h1 = mix32(i * 2654435761u ^ seed), h2 = mix32(h1 ^ 0x9e3779b9u), h3 = mix32(h2 + i);
  const unsigned ea = 67u + h3 % 130u, eb = 77u + (h3 >> 8) % 114u;  // biased exponents
  const float a = __uint_as_float((h1 & 0x807fffffu) | (ea << 23));
  const float b = __uint_as_float((h2 & 0x807fffffu) | (eb << 23));
  if (__float_as_uint(qm_div_markstein(a, b, qm_rcp_newton(b))) != __float_as_uint(__fdiv_rn(a, b)))
    atomicAdd(counts + 6, 1ull);
  const float c = __fmul_rn(b, (float)(h3 >> 20) + 0.5f);
  const float ac = fabsf(c);
  if (ac >= 0x1p-60f && ac <= 0x1p70f &&
      __float_as_uint(qm_div_markstein(c, b, qm_rcp_newton(b))) != __float_as_uint(__fdiv_rn(c, b)))
    atomicAdd(counts + 6, 1ull);
}

// Division by a height h with the precomputed y = RN(1/h) (the cylinder's u):
// counts[2] = patterns a where the quotient differs from __fdiv_rn(a, h) while
// a and the quotient lie in [2^-90, 2^90] (Markstein's theorem needs the
// remainder a - h q, about 2^-24 a, to stay normal), counts[3] = patterns
// where u = q + 0.5 differs while either u lies in [0, 1] (where it decides a
// hit and a pixel row): none, since below that range u rounds to 0.5 either
// way.
__global__ void division_kernel(unsigned begin, float h, float y, unsigned long long* counts) {
  const unsigned bits = begin + blockIdx.x * blockDim.x + threadIdx.x;
  const float a = __uint_as_float(bits);
  const float q = qm_div_by_rcp(a, h, y), w = __fdiv_rn(a, h);
  const float aw = fabsf(w), aa = fabsf(a);
  if (aw >= 0x1p-90f && aw <= 0x1p90f && aa >= 0x1p-90f && aa <= 0x1p90f && __float_as_uint(q) != __float_as_uint(w))
    atomicAdd(counts + 2, 1ull);
  const float u = __fadd_rn(q, 0.5f), uw = __fadd_rn(w, 0.5f);
  const bool in = (u >= 0.0f && u <= 1.0f) || (uw >= 0.0f && uw <= 1.0f);
  if (in && __float_as_uint(u) != __float_as_uint(uw)) atomicAdd(counts + 3, 1ull);
}

__global__ void fma_kernel(float* out, int iters, float a, float b) {
  float x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
    x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
    x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
  }
  float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void atomic_kernel(float* img, int n_pix, int per_thread, uint32_t salt) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  for (int i = 0; i < per_thread; ++i) {
    uint32_t h = (t * 0x9e3779b1u) ^ (i * 0x85ebca6bu) ^ salt;
    h ^= h >> 15;
    h *= 0x2c1b3c6du;
    h ^= h >> 12;
    atomicAdd(img + (h % (uint32_t)n_pix), 1.0f);
  }
}

// Replays a recorded sequence of deposits: warp w of the grid takes groups
// of 32 consecutive codes (one per lane, in the tracer's lane order) in a
// grid-stride loop and adds 1 at every code >= 0 (a receiver pixel), as the
// tracer's flux deposit does for the same rays.
__global__ void replay_kernel(float* img, const int* __restrict__ codes, long long n_codes, int repeats) {
  const long long lane = threadIdx.x & 31;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
  const long long groups = (n_codes + 31) >> 5;
  for (int r = 0; r < repeats; ++r)
    for (long long g = warp; g < groups; g += warps) {
      const long long i = (g << 5) + lane;
      const int code = i < n_codes ? __ldg(codes + i) : -1;
      if (code >= 0) atomicAdd(img + code, 1.0f);
    }
}

float time_launch(void (*launch)(void*), void* ctx) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  launch(ctx);  // warm-up
  cudaEventRecord(a);
  launch(ctx);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms;
}

struct FmaCtx {
  float* out;
  int blocks, threads, iters;
};
void fma_launch(void* p) {
  auto* c = static_cast<FmaCtx*>(p);
  fma_kernel<<<c->blocks, c->threads>>>(c->out, c->iters, 0.999f, 0.001f);
}

struct AtomCtx {
  float* img;
  int n_pix, blocks, threads, per_thread;
};
void atom_launch(void* p) {
  auto* c = static_cast<AtomCtx*>(p);
  atomic_kernel<<<c->blocks, c->threads>>>(c->img, c->n_pix, c->per_thread, 17u);
}

struct ReplayCtx {
  float* img;
  const int* codes;
  long long n_codes;
  int blocks, threads, repeats;
};
void replay_launch(void* p) {
  auto* c = static_cast<ReplayCtx*>(p);
  replay_kernel<<<c->blocks, c->threads>>>(c->img, c->codes, c->n_codes, c->repeats);
}

}  // namespace

extern "C" int qmcrt_microbench_atomics_replay(const int* device_codes, long long n_codes, int n_pixels, int repeats,
                                               double* ms_per_launch) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (!device_codes || n_codes <= 0 || n_pixels <= 0 || repeats <= 0 || !ms_per_launch) return 1;
  ReplayCtx c{nullptr, device_codes, n_codes, sms * 16, 256, repeats};
  if (cudaMalloc(&c.img, sizeof(float) * n_pixels) != cudaSuccess) return 3;
  cudaMemset(c.img, 0, sizeof(float) * n_pixels);
  float ms = time_launch(replay_launch, &c);
  cudaFree(c.img);
  if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return 3;
  *ms_per_launch = (double)ms;
  return 0;
}

extern "C" int qmcrt_debug_check_primitives(unsigned long long* mismatches, int count) {
  constexpr int kChecks = 7;
  if (!mismatches || count < 1) return 1;
  unsigned long long* d = nullptr;
  if (cudaMalloc(&d, sizeof(unsigned long long) * kChecks) != cudaSuccess) return 3;
  cudaMemset(d, 0, sizeof(unsigned long long) * kChecks);
  // every 32-bit pattern: 16 launches of 2^28 threads
  for (unsigned long long begin = 0; begin < (1ull << 32); begin += (1ull << 28))
    primitives_kernel<<<(1u << 28) / 256, 256>>>((unsigned)begin, d);
  // receiver heights from a millimetre to a kilometre
  const float heights[] = {12.0f, 4.0f, 7.3f, 0.37f, 123.4f, 0.003f, 1000.0f, 1.0f, 3.0f, 0.1f, 6.0f, 17.77f};
  for (float h : heights)
    for (unsigned long long begin = 0; begin < (1ull << 32); begin += (1ull << 28))
      division_kernel<<<(1u << 28) / 256, 256>>>((unsigned)begin, h, 1.0f / h, d);
  for (unsigned seed = 0; seed < 16; ++seed) division_pairs_kernel<<<(1u << 28) / 256, 256>>>(0x5eed0000u + seed, d);
  unsigned long long host[kChecks] = {};
  const cudaError_t e = cudaMemcpy(host, d, sizeof host, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) return 3;
  for (int k = 0; k < count; ++k) mismatches[k] = k < kChecks ? host[k] : 0;
  return 0;
}

extern "C" int qmcrt_microbench_fp32(double* tflops) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  FmaCtx c{nullptr, sms * 16, 256, 1 << 14};
  if (cudaMalloc(&c.out, sizeof(float) * c.blocks * c.threads) != cudaSuccess) return 3;
  float ms = time_launch(fma_launch, &c);
  cudaFree(c.out);
  if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return 3;
  double flops = 2.0 * 8.0 * (double)c.iters * c.blocks * c.threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return 0;
}

extern "C" int qmcrt_microbench_atomics(int n_pixels, double* giga_per_s) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  AtomCtx c{nullptr, n_pixels, sms * 8, 256, 256};
  if (n_pixels <= 0 || cudaMalloc(&c.img, sizeof(float) * n_pixels) != cudaSuccess) return 3;
  cudaMemset(c.img, 0, sizeof(float) * n_pixels);
  float ms = time_launch(atom_launch, &c);
  cudaFree(c.img);
  if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return 3;
  *giga_per_s = (double)c.blocks * c.threads * c.per_thread / (ms * 1e-3) / 1e9;
  return 0;
}
