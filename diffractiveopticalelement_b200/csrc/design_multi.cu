// design_multi.cu -- designs of uneven sizes in one submission (no reference
// counterpart; the reference designs one element per call, src/doe.js:796-896).
//
// Each size class (one doe_design_dev_desc: B designs of one grid) runs on its own
// sub-context, so the classes' passes proceed concurrently on their own streams
// and scratch, forked from and joined back into the parent context's stream. The
// whole submission -- every pass of every iteration of every class -- can be
// captured once into a CUDA graph and relaunched as one graph launch per step.
#include <cstring>
#include <vector>

#include "design_ops.cuh"

using namespace doe;

struct doe_design_multi {
  doe_ctx* ctx = nullptr;
  std::vector<doe_ctx*> sub;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t exec = nullptr;
  unsigned long long graph_launches = 0;  // kernels inside the captured graph
  unsigned long long graph_gen = 0;       // sub-contexts' scratch generation at capture
};

namespace {

int ensure_classes(doe_design_multi* m, int k) {
  while ((int)m->sub.size() < k) {
    doe_ctx* s = nullptr;
    const int rc = doe_ctx_create(m->ctx->device, &s);
    if (rc) return set_err(m->ctx, rc, "design multi: sub-context creation failed (%d)", rc);
    m->sub.push_back(s);
    cudaEvent_t e;
    DOE_CUDA(m->ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    m->join.push_back(e);
  }
  return DOE_OK;
}

// Fork, run every class on its sub-context, join (on the parent stream).
int submit(doe_design_multi* m, int k, const doe_design_dev_desc* d, unsigned long long* launched) {
  doe_ctx* c = m->ctx;
  DOE_CUDA(c, cudaEventRecord(m->fork, c->stream));
  unsigned long long n0 = 0;
  for (int i = 0; i < k; ++i) n0 += m->sub[i]->launches;
  for (int i = 0; i < k; ++i) {
    doe_ctx* s = m->sub[i];
    // the classes run with the parent's design tuning (shape variants, cluster loop)
    memcpy(s->tune_row[kTuneDesign], c->tune_row[kTuneDesign], sizeof(c->tune_row[kTuneDesign]));
    memcpy(s->tune_col[kTuneDesign], c->tune_col[kTuneDesign], sizeof(c->tune_col[kTuneDesign]));
    s->tune_design_cluster = c->tune_design_cluster;
    DOE_CUDA(c, cudaStreamWaitEvent(s->stream, m->fork, 0));
    const int rc = doe_design_dev(s, &d[i]);
    if (rc) return set_err(c, rc, "design multi: class %d: %s", i, s->err.c_str());
    DOE_CUDA(c, cudaEventRecord(m->join[i], s->stream));
    DOE_CUDA(c, cudaStreamWaitEvent(c->stream, m->join[i], 0));
  }
  unsigned long long n1 = 0;
  for (int i = 0; i < k; ++i) n1 += m->sub[i]->launches;
  *launched = n1 - n0;
  return DOE_OK;
}

// Sum of the sub-contexts' scratch generations: it changes whenever one of them
// reallocates a slot, which leaves a captured graph pointing at freed memory.
unsigned long long scratch_gen(const doe_design_multi* m) {
  unsigned long long g = 0;
  for (auto s : m->sub) g += s->slot_gen;
  return g;
}

}  // namespace

extern "C" int doe_design_multi_create(doe_ctx* c, doe_design_multi** out) {
  if (!c || !out) return DOE_ERR_BAD_ARG;
  doe_design_multi* m = new doe_design_multi;
  m->ctx = c;
  if (cudaEventCreateWithFlags(&m->fork, cudaEventDisableTiming) != cudaSuccess) {
    delete m;
    return set_err(c, DOE_ERR_CUDA, "design multi: event creation failed");
  }
  *out = m;
  return DOE_OK;
}

extern "C" void doe_design_multi_destroy(doe_design_multi* m) {
  if (!m) return;
  if (m->ctx) cudaStreamSynchronize(m->ctx->stream);
  if (m->exec) cudaGraphExecDestroy(m->exec);
  for (auto e : m->join) cudaEventDestroy(e);
  if (m->fork) cudaEventDestroy(m->fork);
  for (auto s : m->sub) doe_ctx_destroy(s);
  delete m;
}

// mode 0: run directly; 1: capture the submission into a CUDA graph and launch it
// (a mode-0 call with the same shapes must come first, so that no scratch is
// allocated inside the capture); 2: relaunch the graph of the last mode-1 call
// (same descriptors; the device arrays are read and written again). A call in
// between that grew any scratch (a mode-0 call with larger shapes) makes the
// graph stale: mode 2 then fails with DOE_ERR_BAD_ARG instead of replaying it.
extern "C" int doe_design_multi_run(doe_design_multi* m, int nclasses, const doe_design_dev_desc* descs, int mode) {
  if (!m) return DOE_ERR_BAD_ARG;
  doe_ctx* c = m->ctx;
  if (mode == 2) {
    if (!m->exec) return set_err(c, DOE_ERR_BAD_ARG, "design multi: no captured graph to relaunch");
    if (scratch_gen(m) != m->graph_gen) {
      cudaGraphExecDestroy(m->exec);
      m->exec = nullptr;
      return set_err(c, DOE_ERR_BAD_ARG,
                     "design multi: the captured graph is stale (scratch was reallocated since capture); capture again");
    }
    DOE_CUDA(c, cudaGraphLaunch(m->exec, c->stream));
    c->launches += m->graph_launches;
    return DOE_OK;
  }
  if (nclasses < 1 || !descs) return set_err(c, DOE_ERR_BAD_ARG, "design multi: no size classes");
  DOE_TRY(ensure_classes(m, nclasses));
  unsigned long long launched = 0;
  if (mode == 0) {
    DOE_TRY(submit(m, nclasses, descs, &launched));
    c->launches += launched;
    return DOE_OK;
  }
  if (mode != 1) return set_err(c, DOE_ERR_BAD_ARG, "design multi: mode must be 0, 1 or 2");
  if (m->exec) {
    cudaGraphExecDestroy(m->exec);
    m->exec = nullptr;
  }
  DOE_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
  const int rc = submit(m, nclasses, descs, &launched);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return set_err(c, DOE_ERR_CUDA, "design multi: capture failed: %s", cudaGetErrorString(e));
  const cudaError_t e2 = cudaGraphInstantiate(&m->exec, g, 0);
  cudaGraphDestroy(g);
  if (e2 != cudaSuccess) {
    m->exec = nullptr;
    return set_err(c, DOE_ERR_CUDA, "design multi: graph instantiation failed: %s", cudaGetErrorString(e2));
  }
  m->graph_launches = launched;
  m->graph_gen = scratch_gen(m);
  DOE_CUDA(c, cudaGraphLaunch(m->exec, c->stream));
  c->launches += launched;
  return DOE_OK;
}
