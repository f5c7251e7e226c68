// CPU ORACLE - test infrastructure only.
//
// Host stand-ins for the CUDA runtime calls that the reference's *host* code
// makes while it loads and processes a scene (cudaMalloc/cudaMemcpy/cudaFree
// inside cpu2gpu, CGridHelioMatch, Receiver::Calloc_image, ...).  Linking the
// reference's host code against this file instead of libcudart lets that
// code run unchanged on a machine without a GPU: "device" buffers are plain
// host allocations, copies are memcpy.  Kernel launches are refused
// (cudaErrorNotSupported); the oracle never reaches one.
//
// The reference's cuRAND wrapper class (Tool/RandomNumberGenerator) is
// replaced by inert definitions: sample pools are always injected.
#include <cuda_runtime_api.h>
#include <curand.h>

#include <cstdlib>
#include <cstring>
#include <random>

#include "RandomNumberGenerator/RandomGenerator.cuh"

extern "C" {

cudaError_t cudaMalloc(void** p, size_t n) {
  *p = std::calloc(n ? n : 1, 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFree(void* p) {
  std::free(p);
  return cudaSuccess;
}
cudaError_t cudaMemcpy(void* dst, const void* src, size_t n, enum cudaMemcpyKind) {
  if (n) std::memmove(dst, src, n);
  return cudaSuccess;
}
cudaError_t cudaMemset(void* dst, int v, size_t n) {
  std::memset(dst, v, n);
  return cudaSuccess;
}
cudaError_t cudaDeviceSynchronize(void) { return cudaSuccess; }
cudaError_t cudaGetLastError(void) { return cudaSuccess; }
cudaError_t cudaPeekAtLastError(void) { return cudaSuccess; }
const char* cudaGetErrorString(cudaError_t e) { return e == cudaSuccess ? "no error" : "host stand-in: not supported"; }

cudaError_t cudaLaunchKernel(const void*, dim3, dim3, void**, size_t, cudaStream_t) { return cudaErrorNotSupported; }
unsigned __cudaPushCallConfiguration(dim3, dim3, size_t, struct CUstream_st*) { return 0; }
cudaError_t __cudaPopCallConfiguration(dim3*, dim3*, size_t*, void*) { return cudaErrorNotSupported; }

static void* g_fake_handle[4];
void** __cudaRegisterFatBinary(void*) { return g_fake_handle; }
void __cudaRegisterFatBinaryEnd(void**) {}
void __cudaUnregisterFatBinary(void**) {}
void __cudaRegisterFunction(void**, const char*, char*, const char*, int, uint3*, uint3*, dim3*, dim3*, int*) {}
void __cudaRegisterVar(void**, char*, char*, const char*, int, size_t, int, int) {}

}  // extern "C"

curandGenerator_t RandomGenerator::gen = nullptr;
std::default_random_engine RandomGenerator::generator;
void RandomGenerator::initSeed() {}
void RandomGenerator::initSeed(unsigned int) {}
void RandomGenerator::initCudaRandGenerator() {}
void RandomGenerator::destroyCudaRandGenerator() {}
bool RandomGenerator::cpu_Uniform(float*, int) { return false; }
bool RandomGenerator::gpu_Uniform(float*, int) { return false; }
bool RandomGenerator::cpu_Gaussian(float*, float, float, int) { return false; }
bool RandomGenerator::gpu_Gaussian(float*, float, float, int) { return false; }
bool RandomGenerator::cpu_Uniform(int*, int, int, int) { return false; }
bool RandomGenerator::gpu_Uniform(int*, int, int, int) { return false; }
