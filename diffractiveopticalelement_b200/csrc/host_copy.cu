// host_copy.cu -- host <-> device copies of the caller's FP64 planes for the
// reference-facing entry points (no reference counterpart: the reference keeps
// its arrays in one address space).
//
// The reference's calls take and return ordinary JavaScript / NumPy arrays, so
// the planes arrive in pageable host memory. A copy from pageable memory is staged
// by the driver through its own pinned buffers at well below the link rate (~17
// GB/s measured on B200 hosts against ~57 GB/s for pinned memory). Here a plane
// of 1 MB or more from pageable memory goes through two pinned chunks of this
// context: host threads copy chunk k into one while the DMA engine moves chunk
// k - 1 out of the other (and the reverse for downloads), so the link and the
// host copy overlap. Pinned caller memory (doe_host_alloc, cudaHostAlloc,
// cudaHostRegister) is copied directly; "host_copy_threads" 0 turns the staging
// off.
#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "engine.cuh"

namespace doe {

// A fixed set of host threads that split one memcpy between them (the calling
// thread takes a share too).
struct CopyPool {
  std::vector<std::thread> th;
  std::mutex m;
  std::condition_variable go, done;
  unsigned long long gen = 0;
  int left = 0;
  bool stop = false;
  char* dst = nullptr;
  const char* src = nullptr;
  size_t bytes = 0;

  explicit CopyPool(int workers) {
    try {
      for (int i = 0; i < workers; ++i) th.emplace_back([this, i] { work(i + 1); });
    } catch (...) {  // a thread could not be started: stop the ones that were
      shutdown();
      throw;
    }
  }
  ~CopyPool() { shutdown(); }
  void shutdown() {
    {
      std::lock_guard<std::mutex> l(m);
      stop = true;
    }
    go.notify_all();
    for (auto& t : th)
      if (t.joinable()) t.join();
    th.clear();
  }
  void slice(int i) const {
    const size_t parts = th.size() + 1;
    size_t per = (bytes + parts - 1) / parts;
    per = (per + 4095) & ~(size_t)4095;  // whole pages per thread
    const size_t a = (size_t)i * per;
    if (a < bytes) memcpy(dst + a, src + a, std::min(per, bytes - a));
  }
  void work(int i) {
    unsigned long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> l(m);
        go.wait(l, [&] { return stop || gen != seen; });
        if (stop) return;
        seen = gen;
      }
      slice(i);
      std::lock_guard<std::mutex> l(m);
      if (--left == 0) done.notify_one();
    }
  }
  void copy(void* d, const void* s, size_t n) {
    {
      std::lock_guard<std::mutex> l(m);
      dst = static_cast<char*>(d);
      src = static_cast<const char*>(s);
      bytes = n;
      left = (int)th.size();
      ++gen;
    }
    go.notify_all();
    slice(0);
    std::unique_lock<std::mutex> l(m);
    done.wait(l, [&] { return left == 0; });
  }
};

void destroy_copy_pool(CopyPool* p) { delete p; }

namespace {

constexpr size_t kChunk = 4u << 20;     // bytes per staging chunk
constexpr size_t kStageMin = 1u << 20;  // smaller copies go straight through the driver

bool is_pinned(const void* h) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, h) != cudaSuccess) {
    cudaGetLastError();  // an unknown pointer is pageable memory; clear the status
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// The pinned chunks, their events and the host threads, made at the first staged
// copy. When any of them cannot be had (pinned memory or threads exhausted), the
// context stops staging and hands its planes to the driver from then on.
bool ensure_stage(doe_ctx* c) {
  if (!c->stage[0]) {
    for (int b = 0; b < 2; ++b) {
      if (cudaMallocHost(&c->stage[b], kChunk) != cudaSuccess ||
          cudaEventCreateWithFlags(&c->stage_ev[b], cudaEventDisableTiming) != cudaSuccess ||
          cudaEventRecord(c->stage_ev[b], c->stream) != cudaSuccess) {
        cudaGetLastError();
        c->host_copy_threads = 0;
        return false;
      }
    }
  }
  if (!c->copy_pool) {
    try {
      c->copy_pool = new CopyPool(c->host_copy_threads - 1);
    } catch (...) {
      c->host_copy_threads = 0;
      return false;
    }
  }
  return true;
}

bool staged(doe_ctx* c, const void* h, size_t bytes) {
  return c->host_copy_threads > 0 && bytes >= kStageMin && !is_pinned(h) && ensure_stage(c);
}

}  // namespace

int host_upload(doe_ctx* c, void* d, const void* h, size_t bytes) {
  if (!staged(c, h, bytes)) {
    DOE_CUDA(c, cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, c->stream));
    return DOE_OK;
  }
  for (size_t off = 0, k = 0; off < bytes; off += kChunk, ++k) {
    const int b = (int)(k & 1);  // chunk k's buffer was last read by the DMA of chunk k - 2
    const size_t len = std::min(kChunk, bytes - off);
    DOE_CUDA(c, cudaEventSynchronize(c->stage_ev[b]));  // the DMA that last read this chunk is done
    c->copy_pool->copy(c->stage[b], static_cast<const char*>(h) + off, len);
    DOE_CUDA(c, cudaMemcpyAsync(static_cast<char*>(d) + off, c->stage[b], len, cudaMemcpyHostToDevice, c->stream));
    DOE_CUDA(c, cudaEventRecord(c->stage_ev[b], c->stream));
  }
  return DOE_OK;
}

int host_download(doe_ctx* c, void* h, const void* d, size_t bytes) {
  if (!staged(c, h, bytes)) {
    DOE_CUDA(c, cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, c->stream));
    return DOE_OK;
  }
  // chunk k's DMA is queued before chunk k - 1 is copied out on the host; chunk
  // k's buffer was last read by the host copy of chunk k - 2, which has returned
  const size_t nch = (bytes + kChunk - 1) / kChunk;
  for (size_t k = 0; k <= nch; ++k) {
    if (k < nch) {
      const size_t off = k * kChunk;
      DOE_CUDA(c, cudaMemcpyAsync(c->stage[k & 1], static_cast<const char*>(d) + off, std::min(kChunk, bytes - off),
                                  cudaMemcpyDeviceToHost, c->stream));
      DOE_CUDA(c, cudaEventRecord(c->stage_ev[k & 1], c->stream));
    }
    if (k > 0) {
      const size_t pk = k - 1, off = pk * kChunk;
      DOE_CUDA(c, cudaEventSynchronize(c->stage_ev[pk & 1]));
      c->copy_pool->copy(static_cast<char*>(h) + off, c->stage[pk & 1], std::min(kChunk, bytes - off));
    }
  }
  return DOE_OK;
}

}  // namespace doe
