// context.cu -- context lifetime, twiddle tables and host helpers of the C ABI.
#include <cmath>
#include <vector>

#include "engine.cuh"

using namespace doe;

extern "C" int doe_abi_version(void) { return DOE_B200_ABI_VERSION; }

extern "C" int doe_ctx_create(int device, doe_ctx** out) {
  if (!out) return DOE_ERR_BAD_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    (void)cudaGetLastError();
    return DOE_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return DOE_ERR_BAD_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return DOE_ERR_CUDA;
  doe_ctx* c = new doe_ctx();
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return DOE_ERR_CUDA;
  }
  // Twiddle tables e^{-2 pi i m / N}, m < N, for every N <= kMaxN, rounded once
  // from FP64; the table for length N starts at element N.
  std::vector<float2> h(2 * (size_t)kMaxN);
  h[0] = make_float2(1.f, 0.f);
  for (int N = 1; N <= kMaxN; N <<= 1) {
    for (int m = 0; m < N; ++m) {
      const double a = -2.0 * M_PI * (double)m / (double)N;
      h[N + m] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
  }
  if (cudaMalloc(&c->tw, h.size() * sizeof(float2)) != cudaSuccess ||
      cudaMemcpy(c->tw, h.data(), h.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess) {
    (void)cudaGetLastError();
    doe_ctx_destroy(c);
    return DOE_ERR_CUDA;
  }
  *out = c;
  return DOE_OK;
}

extern "C" void doe_ctx_destroy(doe_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int s = 0; s < kSlotCount; ++s)
    if (c->slot[s]) cudaFree(c->slot[s]);
  if (c->tw) cudaFree(c->tw);
  if (c->pinned) cudaFreeHost(c->pinned);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" const char* doe_last_error(const doe_ctx* c) { return c ? c->err.c_str() : "no context"; }

extern "C" void* doe_ctx_stream(doe_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" int doe_ctx_synchronize(doe_ctx* c) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
}

extern "C" int doe_host_alloc(doe_ctx* c, void** ptr, unsigned long long bytes) {
  if (!c || !ptr) return DOE_ERR_BAD_ARG;
  DOE_CUDA(c, cudaMallocHost(ptr, bytes));
  return DOE_OK;
}

extern "C" int doe_host_free(doe_ctx* c, void* ptr) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_CUDA(c, cudaFreeHost(ptr));
  return DOE_OK;
}
