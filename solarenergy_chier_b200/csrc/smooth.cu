// Trimmed-mean smoother (Tool/Smoother/ImageSmoother.cu:13-113, heaps in
// Tool/Smoother/heap.cuh:16-225).
//
// Each output pixel is the mean of its (2r+1)^2 window clipped to the image,
// after dropping k = int(count * ratio) values at each end, where the k
// smallest and k largest are tracked by the reference's streaming max- and
// min-heaps in the reference's visiting order (row by row).  The heap
// updates and the summation order are kept, so the float result matches the
// reference's kernel, including the cases where its streaming selection
// differs from a sorted trim (k >= 2 with some value orders).
//
// The reference reads a texture copy of the image and writes in place; here
// the kernel reads an explicit copy (`src`) and writes `dst`.
#include "smooth.h"

namespace qm {
namespace {

// heap.cuh's array heap, 1-based, comparator `larger` (max-heap) or
// `smaller` (min-heap).
template <bool kMax>
struct ArrayHeap {
  float* e;
  int num;  // next free slot (1 when empty)
  int cap;  // size + 1
  __device__ __forceinline__ static bool cmp(float a, float b) { return kMax ? a > b : a < b; }
  __device__ __forceinline__ bool full() const { return num == cap; }
  __device__ __forceinline__ bool empty() const { return num == 1; }
  __device__ __forceinline__ float top() const { return empty() ? 0.0f : e[1]; }
  __device__ __forceinline__ void insert(float x) {
    if (full()) return;
    int i = num++;
    for (; i != 1 && cmp(x, e[i / 2]); i /= 2) e[i] = e[i / 2];
    e[i] = x;
  }
  __device__ __forceinline__ void replace_top(float x) {
    if (empty()) return;
    int i = 1;
    while (2 * i < num) {
      int c = (2 * i + 1 >= num || cmp(e[2 * i], e[2 * i + 1])) ? 2 * i : 2 * i + 1;
      if (cmp(e[c], x)) {
        e[i] = e[c];
        i = c;
      } else {
        break;
      }
    }
    e[i] = x;
  }
  __device__ __forceinline__ float sum() const {
    float s = 0.0f;
    for (int i = 1; i < num; ++i) s += e[i];
    return s;
  }
};

__global__ void trimmed_mean_kernel(const float* __restrict__ src, float* __restrict__ dst, int radius, float ratio,
                                    int width, int height, int heap_stride) {
  extern __shared__ float heaps[];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x > width - 1 || y > height - 1) return;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int x0 = (x - radius >= 0) ? x - radius : 0;
  const int y0 = (y - radius >= 0) ? y - radius : 0;
  const int x1 = (x + radius < width) ? x + radius : width - 1;
  const int y1 = (y + radius < height) ? y + radius : height - 1;
  const int cnt = (x1 - x0 + 1) * (y1 - y0 + 1);
  const int k = cnt * ratio;
  ArrayHeap<true> lo{heaps + (size_t)(2 * tid) * heap_stride, 1, k + 1};
  ArrayHeap<false> hi{heaps + (size_t)(2 * tid + 1) * heap_stride, 1, k + 1};
  float value = 0.0f;
  for (int r = y0; r <= y1; ++r) {
    for (int c = x0; c <= x1; ++c) {
      const float cur = __ldg(src + (size_t)r * width + c);
      value += cur;
      if (!lo.full()) {
        lo.insert(cur);
        hi.insert(cur);
      } else if (cur < lo.top()) {
        lo.replace_top(cur);
      } else if (cur > hi.top()) {
        hi.replace_top(cur);
      }
    }
  }
  dst[(size_t)y * width + x] = (value - lo.sum() - hi.sum()) / float(cnt - 2 * k);
}

}  // namespace

int smooth_heap_stride(int radius, float ratio) {
  return (2 * radius + 1) * (2 * radius + 1) * ratio + 1;
}

cudaError_t launch_trimmed_mean(const float* src, float* dst, int width, int height, int radius, float ratio,
                                cudaStream_t stream) {
  const dim3 block(16, 16);
  const dim3 grid((width + block.x - 1) / block.x, (height + block.y - 1) / block.y);
  const int stride = smooth_heap_stride(radius, ratio);
  const size_t smem = sizeof(float) * (size_t)stride * 2 * block.x * block.y;
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(trimmed_mean_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  trimmed_mean_kernel<<<grid, block, smem, stream>>>(src, dst, radius, ratio, width, height, stride);
  return cudaGetLastError();
}

}  // namespace qm
