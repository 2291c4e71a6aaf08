// context.cu -- context lifetime, twiddle tables and host helpers of the C ABI.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <thread>
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
  // a quarter of the host's threads, at most 4, stage pageable caller planes (on a
  // 16-thread host 4 were fastest: more contend for the memory bus and the cores)
  c->host_copy_threads = (int)std::min<unsigned>(4u, std::max(1u, std::thread::hardware_concurrency() / 4));
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking) != cudaSuccess) {
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
  for (auto& r : c->prof) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  for (auto e : c->sync_ev) cudaEventDestroy(e);
  if (c->sweep_exec) cudaGraphExecDestroy(c->sweep_exec);
  if (c->aux) {
    cudaStreamSynchronize(c->aux);
    cudaStreamDestroy(c->aux);
  }
  if (c->pinned) cudaFreeHost(c->pinned);
  if (c->stream) cudaStreamSynchronize(c->stream);  // no DMA still reads a staging chunk
  for (int b = 0; b < 2; ++b) {
    if (c->stage[b]) cudaFreeHost(c->stage[b]);
    if (c->stage_ev[b]) cudaEventDestroy(c->stage_ev[b]);
  }
  destroy_copy_pool(c->copy_pool);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" const char* doe_last_error(const doe_ctx* c) { return c ? c->err.c_str() : "no context"; }

extern "C" void* doe_ctx_stream(doe_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" int doe_ctx_synchronize(doe_ctx* c) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  DOE_CUDA(c, cudaStreamSynchronize(c->aux));
  DOE_TRY(tc_check(c));  // a timed-out wait of an asynchronous tensor-core pass surfaces here
  return design_error_check(c);  // ... and one of the cluster-resident design loop
}

extern "C" unsigned long long doe_ctx_launch_count(doe_ctx* c) { return c ? c->launches : 0ull; }

extern "C" int doe_ctx_set_profiling(doe_ctx* c, int on) {
  if (!c) return DOE_ERR_BAD_ARG;
  c->prof_on = on ? 1 : 0;
  return DOE_OK;
}

// Fold pending launch events into per-label totals (synchronises the stream).
extern "C" int doe_ctx_profile_read(doe_ctx* c, int max_entries, char* names, int name_len, double* total_ms,
                                    unsigned long long* count) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  std::vector<std::string> labels;
  std::vector<double> ms;
  std::vector<unsigned long long> cnt;
  for (auto& r : c->prof) {
    float t = 0.f;
    cudaEventElapsedTime(&t, r.a, r.b);
    size_t k = 0;
    while (k < labels.size() && labels[k] != r.name) ++k;
    if (k == labels.size()) {
      labels.push_back(r.name);
      ms.push_back(0.0);
      cnt.push_back(0);
    }
    ms[k] += t;
    cnt[k] += 1;
    c->ev_pool.push_back(r.a);
    c->ev_pool.push_back(r.b);
  }
  c->prof.clear();
  const int n = (int)labels.size() < max_entries ? (int)labels.size() : max_entries;
  for (int k = 0; k < n; ++k) {
    if (names && name_len > 0) {
      snprintf(names + (size_t)k * name_len, name_len, "%s", labels[k].c_str());
    }
    if (total_ms) total_ms[k] = ms[k];
    if (count) count[k] = cnt[k];
  }
  return n;
}

extern "C" int doe_ctx_get_tuning(doe_ctx* c, const char* key, long long* value) {
  if (!c || !key || !value) return DOE_ERR_BAD_ARG;
  const std::string k(key);
  if (k == "sweep_group") {
    *value = c->tune_sweep_group;
  } else if (k == "sweep_fused") {
    *value = c->tune_sweep_fused;
  } else if (k == "sweep_graph") {
    *value = c->tune_sweep_graph;
  } else if (k == "sweep_tc") {
    *value = c->tune_sweep_tc;
  } else if (k == "sweep_hsym") {
    *value = c->tune_sweep_hsym;
  } else if (k == "sweep_res") {
    *value = c->tune_sweep_res;
  } else if (k == "host_copy_threads") {
    *value = c->host_copy_threads;
  } else if (k == "surrogate_tc") {
    *value = c->tune_surrogate_tc;
  } else if (k == "design_cluster") {
    *value = (long long)c->tune_design_cluster;  // bit log2(n) set: n^2 runs cluster-resident
  } else {
    return set_err(c, DOE_ERR_BAD_ARG, "unknown tuning key '%s'", key);
  }
  return DOE_OK;
}

extern "C" int doe_ctx_set_tuning(doe_ctx* c, const char* key, long long value) {
  if (!c || !key) return DOE_ERR_BAD_ARG;
  const std::string k(key);
  if (k == "sweep_fused") {
    c->tune_sweep_fused = value ? 1 : 0;
    return DOE_OK;
  }
  if (k == "sweep_graph") {
    c->tune_sweep_graph = value ? 1 : 0;
    return DOE_OK;
  }
  if (k == "sweep_tc") {
    c->tune_sweep_tc = value ? 1 : 0;
    return DOE_OK;
  }
  if (k == "host_copy_threads") {
    if (value < 0 || value > 64) return set_err(c, DOE_ERR_BAD_ARG, "host_copy_threads must be in [0, 64]");
    destroy_copy_pool(c->copy_pool);  // made again, with the new count, at the next staged copy
    c->copy_pool = nullptr;
    c->host_copy_threads = (int)value;
    return DOE_OK;
  }
  if (k == "sweep_res") {
    if (value < 1 || value > 64) return set_err(c, DOE_ERR_BAD_ARG, "sweep_res must be in [1, 64]");
    c->tune_sweep_res = (int)value;
    return DOE_OK;
  }
  if (k == "sweep_hsym") {
    if (value < 0 || value > 2) return set_err(c, DOE_ERR_BAD_ARG, "sweep_hsym must be 0, 1 or 2");
    c->tune_sweep_hsym = (int)value;
    return DOE_OK;
  }
  if (k == "surrogate_tc") {
    if (value < 0 || value > 3) return set_err(c, DOE_ERR_BAD_ARG, "surrogate_tc must be in [0, 3]");
    c->tune_surrogate_tc = (int)value;
    return DOE_OK;
  }
  if (k == "design_cluster") {
    // 0 / 1: every size it covers (64^2, 128^2, 256^2) off / on;
    // (log2(n) << 8) | on: that size alone
    if (value >= 256) {
      const int lg = (int)((value >> 8) & 0xff);
      if (lg > kMaxLog2) return set_err(c, DOE_ERR_BAD_ARG, "tuning: log2 length %d out of range", lg);
      const unsigned bit = 1u << lg;
      c->tune_design_cluster = (value & 1) ? (c->tune_design_cluster | bit) : (c->tune_design_cluster & ~bit);
    } else {
      c->tune_design_cluster = value ? ((1u << 6) | (1u << 7) | (1u << 8)) : 0u;
    }
    return DOE_OK;
  }
  if (k == "sweep_group") {
    if (value < 0 || value > 64) return set_err(c, DOE_ERR_BAD_ARG, "sweep_group must be in [0, 64]");
    c->tune_sweep_group = (long)value;
    return DOE_OK;
  }
  // "<kind>_row" / "<kind>_col" with value = (log2(n) << 8) | variant
  const char* kinds[] = {"fft", "sweep", "design"};
  for (int kind = 0; kind < 3; ++kind) {
    for (int rc = 0; rc < 2; ++rc) {
      if (k == std::string(kinds[kind]) + (rc ? "_col" : "_row")) {
        const int lg = (int)((value >> 8) & 0xff), var = (int)(value & 0xff);
        if (lg > kMaxLog2) return set_err(c, DOE_ERR_BAD_ARG, "tuning: log2 length %d out of range", lg);
        (rc ? c->tune_col : c->tune_row)[kind][lg] = (unsigned char)var;
        return DOE_OK;
      }
    }
  }
  return set_err(c, DOE_ERR_BAD_ARG, "unknown tuning key '%s'", key);
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

namespace doe {
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      (void)cudaGetLastError();
  });
  return fn;
}
}  // namespace doe
