// unet.cu -- the warm-start surrogate: a 4-level U-Net (32-256 channels by
// default) mapping a target irradiance (+ ROI) to a DOE phase, with its own BF16
// forward, backward and Adam kernels. No counterpart in the reference; the
// phase it predicts is only a starting point that WGS refines and scores.
//
// Graph (all 3x3 convolutions with bias + ReLU; C_l = base << l):
//   enc l < L-1 : a_l = conv(in_l, C_l); cat_l[:, 0:C_l] = conv(a_l, C_l); in_{l+1} = avgpool2(cat_l[:, 0:C_l])
//   bottleneck  : b1 = conv(in_{L-1}, C_{L-1}); b2 = conv(b1, C_{L-1})
//   dec l       : u_l = up2(prev); cat_l[:, C_l:2C_l] = conv(u_l, C_l);
//                 da_l = conv(cat_l, C_l); d_l = conv(da_l, C_l); prev = d_l
//   head        : (c, s) = 1x1 conv(d_0, 2); phase = atan2(s, c)
// in_0 has `base` channels: irradiance / max, ROI, ones, zeros.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "engine.cuh"
#include "unet_kernels.cuh"
#include "unet_tc.cuh"

using namespace doe;
using namespace doe::unet;
typedef __nv_bfloat16 bf16;

namespace {

// ------------------------------------------------------------------ elementwise kernels
__global__ void unet_input_kernel(const float* irr, const float* roi, const float* scale, int n, int base, long P,
                                  bf16* x0) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < P * base; i += (long)gridDim.x * blockDim.x) {
    const long p = i / base;
    const int c = (int)(i - p * base);
    float v = 0.f;
    if (c == 0) v = irr[p] * scale[p / n];
    else if (c == 1) v = roi ? roi[p] : 1.f;
    else if (c == 2) v = 1.f;  // constant plane: every pixel sees a non-zero input
    x0[i] = __float2bfloat16(v);
  }
}

// per-image 1 / max(irradiance) (0 when the image is empty)
__global__ void unet_scale_kernel(const float* irr, int n, float* scale) {
  __shared__ float red[256];
  const float* s = irr + (long)blockIdx.x * n;
  float m = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmaxf(m, s[i]);
  red[threadIdx.x] = m;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) scale[blockIdx.x] = red[0] > 0.f ? 1.f / red[0] : 0.f;
}

// 2x2 average pool: out[b][y][x][c] (H/2 x W/2) from in (H x W), C channels
__global__ void pool_fwd_kernel(const bf16* in, int in_cs, bf16* out, int out_cs, int B, int H, int W, int C) {
  const int H2 = H / 2, W2 = W / 2;
  const long total = (long)B * H2 * W2 * C;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long q = i / C;
    const int x = (int)(q % W2);
    const long r = q / W2;
    const int y = (int)(r % H2);
    const long b = r / H2;
    const long s = (b * H + 2 * y) * W + 2 * x;
    const float v = __bfloat162float(in[s * in_cs + c]) + __bfloat162float(in[(s + 1) * in_cs + c]) +
                    __bfloat162float(in[(s + W) * in_cs + c]) + __bfloat162float(in[(s + W + 1) * in_cs + c]);
    out[q * out_cs + c] = __float2bfloat16(0.25f * v);
  }
}

// g[p][c] = (g[p][c] + dpool[p/2][c] / 4) masked by act > 0 (skip + pool gradients of a ReLU output)
__global__ void pool_bwd_kernel(bf16* g, int g_cs, const bf16* dpool, int dp_cs, const bf16* act, int act_cs, int B,
                                int H, int W, int C) {
  const long total = (long)B * H * W * C;
  const int H2 = H / 2, W2 = W / 2;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long p = i / C;
    const int x = (int)(p % W);
    const long r = p / W;
    const int y = (int)(r % H);
    const long b = r / H;
    const long q = (b * H2 + y / 2) * W2 + x / 2;
    float v = __bfloat162float(g[p * g_cs + c]) + 0.25f * __bfloat162float(dpool[q * dp_cs + c]);
    if (!(__bfloat162float(act[p * act_cs + c]) > 0.f)) v = 0.f;
    g[p * g_cs + c] = __float2bfloat16(v);
  }
}

// nearest 2x upsample: out (2H x 2W) from in (H x W)
__global__ void up_fwd_kernel(const bf16* in, int in_cs, bf16* out, int out_cs, int B, int H, int W, int C) {
  const int H2 = 2 * H, W2 = 2 * W;
  const long total = (long)B * H2 * W2 * C;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long p = i / C;
    const int x = (int)(p % W2);
    const long r = p / W2;
    const int y = (int)(r % H2);
    const long b = r / H2;
    out[p * out_cs + c] = in[((b * H + y / 2) * W + x / 2) * in_cs + c];
  }
}

// g_in[q][c] = sum of the 4 upsampled gradients, masked by act > 0 (act = the ReLU output that was upsampled)
__global__ void up_bwd_kernel(const bf16* gout, int go_cs, bf16* gin, int gi_cs, const bf16* act, int act_cs, int B,
                              int H, int W, int C) {
  const long total = (long)B * H * W * C;
  const int W2 = 2 * W;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long q = i / C;
    const int x = (int)(q % W);
    const long r = q / W;
    const int y = (int)(r % H);
    const long b = r / H;
    const long s = (b * 2 * H + 2 * y) * W2 + 2 * x;
    float v = __bfloat162float(gout[s * go_cs + c]) + __bfloat162float(gout[(s + 1) * go_cs + c]) +
              __bfloat162float(gout[(s + W2) * go_cs + c]) + __bfloat162float(gout[(s + W2 + 1) * go_cs + c]);
    if (!(__bfloat162float(act[q * act_cs + c]) > 0.f)) v = 0.f;
    gin[q * gi_cs + c] = __float2bfloat16(v);
  }
}

// head: cs[p] = b + W d[p] (2 outputs), phase = atan2(s, c)
__global__ void head_fwd_kernel(const bf16* d, int C, const float* w, const float* b, long P, float2* cs,
                                float* phase) {
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < P; p += (long)gridDim.x * blockDim.x) {
    float c0 = b[0], c1 = b[1];
    for (int k = 0; k < C; ++k) {
      const float v = __bfloat162float(d[p * C + k]);
      c0 = fmaf(w[k], v, c0);
      c1 = fmaf(w[C + k], v, c1);
    }
    cs[p] = make_float2(c0, c1);
    phase[p] = atan2f(c1, c0);
  }
}

// head backward from dL/dphase: dd[p][k] (masked by d > 0), dW, db (block sums + atomics)
__global__ void head_bwd_kernel(const bf16* d, int C, const float* w, const float2* cs, const float* dphase, long P,
                                bf16* dd, float* dw, float* db) {
  __shared__ float sw[2 * 64 + 2];
  for (int i = threadIdx.x; i < 2 * C + 2; i += blockDim.x) sw[i] = 0.f;
  __syncthreads();
  float lw[2 * 64];
  for (int k = 0; k < 2 * C; ++k) lw[k] = 0.f;
  float lb0 = 0.f, lb1 = 0.f;
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < P; p += (long)gridDim.x * blockDim.x) {
    const float2 v = cs[p];
    const float r2 = v.x * v.x + v.y * v.y;
    // (c, s) within 1e-10 of the origin carries no usable direction: no gradient
    // (also keeps 1/r^2 finite, so a zero dL/dphase never meets an infinity)
    const float inv = r2 > 1e-20f ? 1.f / r2 : 0.f;
    const float g = dphase[p];
    const float gc = -v.y * inv * g, gs = v.x * inv * g;  // d atan2(s, c)
    lb0 += gc;
    lb1 += gs;
    for (int k = 0; k < C; ++k) {
      const float a = __bfloat162float(d[p * C + k]);
      lw[k] = fmaf(gc, a, lw[k]);
      lw[C + k] = fmaf(gs, a, lw[C + k]);
      const float gd = a > 0.f ? gc * w[k] + gs * w[C + k] : 0.f;
      dd[p * C + k] = __float2bfloat16(gd);
    }
  }
  for (int k = 0; k < 2 * C; ++k) atomicAdd(&sw[k], lw[k]);
  atomicAdd(&sw[2 * C], lb0);
  atomicAdd(&sw[2 * C + 1], lb1);
  __syncthreads();
  for (int i = threadIdx.x; i < 2 * C; i += blockDim.x) atomicAdd(&dw[i], sw[i]);
  if (threadIdx.x == 0) {
    atomicAdd(&db[0], sw[2 * C]);
    atomicAdd(&db[1], sw[2 * C + 1]);
  }
}

// bf16 copies of a conv layer: wb[co][t][ci] = W, wt[ci][8 - t][co] = W (flipped, transposed)
__global__ void weight_copy_kernel(const float* w, int cout, int cin, bf16* wb, bf16* wt) {
  const long total = (long)cout * 9 * cin;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int ci = (int)(i % cin);
    const long r = i / cin;
    const int t = (int)(r % 9);
    const int co = (int)(r / 9);
    const bf16 v = __float2bfloat16(w[i]);
    wb[i] = v;
    wt[((long)ci * 9 + (8 - t)) * cout + co] = v;
  }
}

// Adam (decoupled weight decay) on the FP32 master parameters.
__global__ void adam_kernel(float* w, const float* g, float* m, float* v, long n, float lr, float b1, float b2,
                            float eps, float wd, float bc1, float bc2, float gscale) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i] * gscale;
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * ((mi / bc1) / (sqrtf(vi / bc2) + eps) + wd * w[i]);
  }
}

// Seeded He-normal initialisation (xorshift + Box-Muller), biases zero.
__global__ void init_kernel(float* w, long n, float stddev, unsigned long long seed) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    unsigned long long s = seed ^ (0x9E3779B97F4A7C15ULL * (unsigned long long)(i + 1));
    s ^= s >> 33;
    s *= 0xff51afd7ed558ccdULL;
    s ^= s >> 33;
    s *= 0xc4ceb9fe1a85ec53ULL;
    s ^= s >> 33;
    const float u1 = ((float)((s >> 40) & 0xFFFFFF) + 0.5f) / 16777216.f;
    const float u2 = ((float)((s >> 16) & 0xFFFFFF) + 0.5f) / 16777216.f;
    w[i] = stddev * sqrtf(-2.f * logf(u1)) * cospif(2.f * u2);
  }
}

unsigned grid_for(long n) { return (unsigned)std::max<long>(1, std::min<long>((n + 255) / 256, 148L * 16)); }

}  // namespace

// ------------------------------------------------------------------ network object
struct Act {
  bf16* p = nullptr;  // activation
  bf16* g = nullptr;  // gradient
  int H = 0, W = 0, C = 0;  // C = channel stride
};

struct ConvLayer {
  int cin, cout;
  long off_w, off_b;   // into the FP32 parameter arrays
  bf16* wb = nullptr;  // [cout][9][cin]
  bf16* wt = nullptr;  // [cin][9][cout] flipped
};

struct doe_surrogate {
  doe_ctx* c = nullptr;
  int n = 0, base = 0, levels = 0, max_batch = 0;
  std::vector<ConvLayer> conv;
  long nparam = 0;
  long off_hw = 0, off_hb = 0;
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  long step = 0;
  std::vector<void*> allocs;
  // activations
  Act x0;
  std::vector<Act> a, cat, pin, u, da, d;  // per level
  Act b1, b2;
  float2* cs = nullptr;
  float* phase = nullptr;
  float* scale = nullptr;
  int batch = 0;  // batch of the last forward
};

namespace {

int dalloc(doe_surrogate* s, size_t bytes, void** out) {
  cudaError_t e = cudaMalloc(out, bytes);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return set_err(s->c, DOE_ERR_CUDA, "surrogate: device allocation of %zu bytes failed", bytes);
  }
  s->allocs.push_back(*out);
  return DOE_OK;
}

int make_act(doe_surrogate* s, Act& t, int H, int W, int C) {
  t.H = H;
  t.W = W;
  t.C = C;
  const size_t bytes = (size_t)s->max_batch * H * W * C * sizeof(bf16);
  void *p, *g;
  DOE_TRY(dalloc(s, bytes, &p));
  DOE_TRY(dalloc(s, bytes, &g));
  t.p = (bf16*)p;
  t.g = (bf16*)g;
  return DOE_OK;
}

int add_conv(doe_surrogate* s, int cin, int cout) {
  ConvLayer L;
  L.cin = cin;
  L.cout = cout;
  L.off_w = s->nparam;
  s->nparam += (long)cout * 9 * cin;
  L.off_b = s->nparam;
  s->nparam += cout;
  s->conv.push_back(L);
  return (int)s->conv.size() - 1;
}

// One 3x3 convolution launch: the tcgen05 kernel where its shape rules hold
// (kch input channels of the GEMM a multiple of 64, nout output channels a
// multiple of 32) and the context allows it ("surrogate_tc"), else mma.sync.
template <int BN, int S>
int launch_conv_tc_s(doe_ctx* c, const ConvArgs& a, long P, int nout) {
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device
  DOE_TRY(prepare_kernel(c, conv3x3_tc_kernel<BN, S>, ConvTc<BN, S>::SMEM, attr_set, false));
  int* err;
  DOE_TRY(design_error_word(c, &err));
  conv3x3_tc_kernel<BN, S>
      <<<dim3((unsigned)((P + 127) / 128), nout / BN), 128, ConvTc<BN, S>::SMEM, c->stream>>>(a, err);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}
// Three operand stages: deeper rings (4, 6) measured slower on B200 (2.36 ms
// against 2.63 and 3.29 ms for the tensor-core layers of a 16-design 256^2
// forward pass), the shared memory they take costing resident CTAs.
template <int BN>
int launch_conv_tc(doe_ctx* c, const ConvArgs& a, long P, int nout) {
  return launch_conv_tc_s<BN, 3>(c, a, P, nout);
}

// TMA-fed tcgen05 form; DOE_ERR_UNSUPPORTED when the layer's layout does not fit
// its boxes (the caller then takes the cp.async form).
template <int BN, int S>
int launch_conv_tma(doe_ctx* c, const ConvArgs& a, long P, int nout) {
  const auto enc = tmap_encoder();
  const int W = a.W, H = a.H, kch = a.cin;
  const int bw = W >= 128 ? 128 : W, bh = 128 / bw;
  const long hw = (long)H * W;
  if (!enc || (W & (W - 1)) || bh > H || hw % 128 || a.in_cs % 8 || (reinterpret_cast<uintptr_t>(a.in) & 15) ||
      (reinterpret_cast<uintptr_t>(a.w) & 15))
    return DOE_ERR_UNSUPPORTED;
  CUtensorMap ta, tb;
  const cuuint64_t da[4] = {(cuuint64_t)kch, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)a.B};
  const cuuint64_t sa[3] = {(cuuint64_t)a.in_cs * 2, (cuuint64_t)W * a.in_cs * 2, (cuuint64_t)hw * a.in_cs * 2};
  const cuuint32_t ba[4] = {64, (cuuint32_t)bw, (cuuint32_t)bh, 1}, ea[4] = {1, 1, 1, 1};
  if (enc(&ta, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(a.in), da, sa, ba, ea,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return DOE_ERR_UNSUPPORTED;
  const cuuint64_t db[2] = {(cuuint64_t)9 * kch, (cuuint64_t)nout};
  const cuuint64_t sb[1] = {(cuuint64_t)9 * kch * 2};
  const cuuint32_t bb[2] = {64, (cuuint32_t)BN}, eb[2] = {1, 1};
  if (enc(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(a.w), db, sb, bb, eb,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return DOE_ERR_UNSUPPORTED;
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device
  DOE_TRY(prepare_kernel(c, conv3x3_tma_kernel<BN, S>, ConvTma<BN, S>::SMEM, attr_set, false));
  int* err;
  DOE_TRY(design_error_word(c, &err));
  conv3x3_tma_kernel<BN, S><<<dim3((unsigned)(P / 128), nout / BN), 128, ConvTma<BN, S>::SMEM, c->stream>>>(
      ta, tb, a, bw, bh, err);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}

int conv_launch(doe_surrogate* s, const ConvArgs& a, int kch, int nout, const char* name, const char* tc_name) {
  const long P = (long)a.B * a.H * a.W;
  if (s->c->tune_surrogate_tc >= 2 && kch % 64 == 0 && nout % 32 == 0) {
    LaunchScope ls(s->c, tc_name);
    int rc = DOE_ERR_UNSUPPORTED;
    // 4-stage ring (measured best: 1.56 ms for the tensor-core layers of a 16-design
    // 256^2 forward pass, against 2.13 ms with 6 stages and 2.36 ms with cp.async)
    // or, with "surrogate_tc" 3, a 3-stage ring
    const bool s4 = s->c->tune_surrogate_tc == 2;
    if (nout % 128 == 0) rc = s4 ? launch_conv_tma<128, 4>(s->c, a, P, nout) : launch_conv_tma<128, 3>(s->c, a, P, nout);
    else if (nout % 64 == 0) rc = s4 ? launch_conv_tma<64, 4>(s->c, a, P, nout) : launch_conv_tma<64, 3>(s->c, a, P, nout);
    else rc = s4 ? launch_conv_tma<32, 4>(s->c, a, P, nout) : launch_conv_tma<32, 3>(s->c, a, P, nout);
    if (rc != DOE_ERR_UNSUPPORTED) return rc;
    if (nout % 128 == 0) return launch_conv_tc<128>(s->c, a, P, nout);
    if (nout % 64 == 0) return launch_conv_tc<64>(s->c, a, P, nout);
    return launch_conv_tc<32>(s->c, a, P, nout);
  }
  if (s->c->tune_surrogate_tc && kch % 64 == 0 && nout % 32 == 0) {
    LaunchScope ls(s->c, tc_name);
    if (nout % 128 == 0) return launch_conv_tc<128>(s->c, a, P, nout);
    if (nout % 64 == 0) return launch_conv_tc<64>(s->c, a, P, nout);
    return launch_conv_tc<32>(s->c, a, P, nout);
  }
  LaunchScope ls(s->c, name);
  if (nout % 64 == 0) {
    conv3x3_kernel<64><<<dim3((unsigned)((P + kBM - 1) / kBM), nout / 64), kConvThreads, 0, s->c->stream>>>(a);
  } else {
    conv3x3_kernel<32><<<dim3((unsigned)((P + kBM - 1) / kBM), nout / 32), kConvThreads, 0, s->c->stream>>>(a);
  }
  DOE_CUDA(s->c, cudaGetLastError());
  return DOE_OK;
}

// conv(in -> out) with bias + ReLU; layer index li
int conv_fwd(doe_surrogate* s, int li, int B, const bf16* in, int in_cs, bf16* out, int out_cs, int H, int W) {
  const ConvLayer& L = s->conv[li];
  ConvArgs a{in, in_cs, L.cin, L.wb, s->w + L.off_b, out, out_cs, L.cout, nullptr, 0, 1, B, H, W};
  return conv_launch(s, a, L.cin, L.cout, "unet_conv_fwd", "unet_conv_fwd_tc");
}

// input gradient: dIn = conv(dOut, flipped W^T), masked by `mask` (> 0) when given
int conv_dgrad(doe_surrogate* s, int li, int B, const bf16* dout, int dout_cs, bf16* din, int din_cs,
               const bf16* mask, int mask_cs, int H, int W) {
  const ConvLayer& L = s->conv[li];
  ConvArgs a{dout, dout_cs, L.cout, L.wt, nullptr, din, din_cs, L.cin, mask, mask_cs, 0, B, H, W};
  return conv_launch(s, a, L.cout, L.cin, "unet_conv_dgrad", "unet_conv_dgrad_tc");
}

int conv_wgrad(doe_surrogate* s, int li, int B, const bf16* in, int in_cs, const bf16* dout, int dout_cs, int H,
               int W) {
  const ConvLayer& L = s->conv[li];
  const long P = (long)B * H * W;
  // about 4 CTAs per SM across the (co, k) tiles
  const int tiles = (L.cout / (L.cout % 64 == 0 ? 64 : 32)) * (9 * L.cin / 32);
  long splits = std::max<long>(1, std::min<long>((148L * 4 + tiles - 1) / tiles, (P + kWP - 1) / kWP));
  long chunk = ((P + splits - 1) / splits + kWP - 1) / kWP * kWP;
  splits = (P + chunk - 1) / chunk;
  WgradArgs a{in, in_cs, L.cin, dout, dout_cs, L.cout, s->g + L.off_w, s->g + L.off_b, B, H, W, chunk};
  LaunchScope ls(s->c, "unet_conv_wgrad");
  if (L.cout % 64 == 0) {
    wgrad_kernel<64><<<dim3(L.cout / 64, 9 * L.cin / 32, (unsigned)splits), kConvThreads, 0, s->c->stream>>>(a);
  } else {
    wgrad_kernel<32><<<dim3(L.cout / 32, 9 * L.cin / 32, (unsigned)splits), kConvThreads, 0, s->c->stream>>>(a);
  }
  DOE_CUDA(s->c, cudaGetLastError());
  return DOE_OK;
}

int refresh_weights(doe_surrogate* s) {
  for (auto& L : s->conv) {
    LaunchScope ls(s->c, "unet_weight_copy");
    weight_copy_kernel<<<grid_for((long)L.cout * 9 * L.cin), 256, 0, s->c->stream>>>(s->w + L.off_w, L.cout, L.cin,
                                                                                    L.wb, L.wt);
    DOE_CUDA(s->c, cudaGetLastError());
  }
  return DOE_OK;
}

// layer indices in creation order
struct Idx {
  std::vector<int> enc_a, enc_b, dec_up, dec_a, dec_b;
  int bott_a, bott_b;
};

Idx layer_index(int L) {
  Idx x;
  int k = 0;
  for (int l = 0; l < L - 1; ++l) {
    x.enc_a.push_back(k++);
    x.enc_b.push_back(k++);
  }
  x.bott_a = k++;
  x.bott_b = k++;
  x.dec_up.resize(L - 1);
  x.dec_a.resize(L - 1);
  x.dec_b.resize(L - 1);
  for (int l = L - 2; l >= 0; --l) {
    x.dec_up[l] = k++;
    x.dec_a[l] = k++;
    x.dec_b[l] = k++;
  }
  return x;
}

}  // namespace

extern "C" int doe_surrogate_create(doe_ctx* c, int n, int base, int levels, int max_batch, unsigned long long seed,
                                    doe_surrogate** out) {
  if (!c || !out) return DOE_ERR_BAD_ARG;
  *out = nullptr;
  if (!is_pow2(n) || n < 16 || n > 4096) return set_err(c, DOE_ERR_BAD_ARG, "surrogate: n must be a power of two in [16, 4096]");
  if (levels < 2 || levels > 6 || (n >> (levels - 1)) < 2)
    return set_err(c, DOE_ERR_BAD_ARG, "surrogate: levels must be in [2, 6] with n / 2^(levels-1) >= 2");
  if (base != 32 && base != 64) return set_err(c, DOE_ERR_BAD_ARG, "surrogate: base channels must be 32 or 64");
  if ((base << (levels - 1)) > 512) return set_err(c, DOE_ERR_BAD_ARG, "surrogate: at most 512 channels");
  if (max_batch < 1) return set_err(c, DOE_ERR_BAD_ARG, "surrogate: max_batch must be >= 1");
  doe_surrogate* s = new doe_surrogate;
  s->c = c;
  s->n = n;
  s->base = base;
  s->levels = levels;
  s->max_batch = max_batch;
  const int L = levels;
  auto ch = [&](int l) { return base << l; };
  // parameters in creation order (matches layer_index)
  for (int l = 0; l < L - 1; ++l) {
    add_conv(s, l == 0 ? base : ch(l - 1), ch(l));
    add_conv(s, ch(l), ch(l));
  }
  add_conv(s, ch(L - 2), ch(L - 1));
  add_conv(s, ch(L - 1), ch(L - 1));
  for (int l = L - 2; l >= 0; --l) {
    add_conv(s, ch(l + 1), ch(l));
    add_conv(s, 2 * ch(l), ch(l));
    add_conv(s, ch(l), ch(l));
  }
  s->off_hw = s->nparam;
  s->nparam += 2 * base;
  s->off_hb = s->nparam;
  s->nparam += 2;
  int rc = DOE_OK;
  auto fail = [&](int r) {
    doe_surrogate_destroy(s);
    return r;
  };
  void* p;
  for (float** a : {&s->w, &s->g, &s->m, &s->v}) {
    if ((rc = dalloc(s, sizeof(float) * s->nparam, &p))) return fail(rc);
    *a = (float*)p;
  }
  for (auto& Ly : s->conv) {
    if ((rc = dalloc(s, sizeof(bf16) * Ly.cout * 9 * Ly.cin, &p))) return fail(rc);
    Ly.wb = (bf16*)p;
    if ((rc = dalloc(s, sizeof(bf16) * Ly.cout * 9 * Ly.cin, &p))) return fail(rc);
    Ly.wt = (bf16*)p;
  }
  // activations
  if ((rc = make_act(s, s->x0, n, n, base))) return fail(rc);
  s->a.resize(L);
  s->cat.resize(L);
  s->pin.resize(L);
  s->u.resize(L);
  s->da.resize(L);
  s->d.resize(L);
  for (int l = 0; l < L - 1; ++l) {
    const int hl = n >> l;
    if ((rc = make_act(s, s->a[l], hl, hl, ch(l)))) return fail(rc);
    if ((rc = make_act(s, s->cat[l], hl, hl, 2 * ch(l)))) return fail(rc);
    if ((rc = make_act(s, s->pin[l + 1], hl / 2, hl / 2, ch(l)))) return fail(rc);
    if ((rc = make_act(s, s->u[l], hl, hl, ch(l + 1)))) return fail(rc);
    if ((rc = make_act(s, s->da[l], hl, hl, ch(l)))) return fail(rc);
    if ((rc = make_act(s, s->d[l], hl, hl, ch(l)))) return fail(rc);
  }
  const int hb = n >> (L - 1);
  if ((rc = make_act(s, s->b1, hb, hb, ch(L - 1)))) return fail(rc);
  if ((rc = make_act(s, s->b2, hb, hb, ch(L - 1)))) return fail(rc);
  if ((rc = dalloc(s, sizeof(float2) * (size_t)max_batch * n * n, &p))) return fail(rc);
  s->cs = (float2*)p;
  if ((rc = dalloc(s, sizeof(float) * (size_t)max_batch * n * n, &p))) return fail(rc);
  s->phase = (float*)p;
  if ((rc = dalloc(s, sizeof(float) * max_batch, &p))) return fail(rc);
  s->scale = (float*)p;
  // He-normal weights, zero biases and head bias; Adam state zero
  DOE_CUDA(c, cudaMemsetAsync(s->w, 0, sizeof(float) * s->nparam, c->stream));
  DOE_CUDA(c, cudaMemsetAsync(s->m, 0, sizeof(float) * s->nparam, c->stream));
  DOE_CUDA(c, cudaMemsetAsync(s->v, 0, sizeof(float) * s->nparam, c->stream));
  DOE_CUDA(c, cudaMemsetAsync(s->g, 0, sizeof(float) * s->nparam, c->stream));
  unsigned long long k = seed;
  for (auto& Ly : s->conv) {
    const long cnt = (long)Ly.cout * 9 * Ly.cin;
    init_kernel<<<grid_for(cnt), 256, 0, c->stream>>>(s->w + Ly.off_w, cnt, sqrtf(2.f / (9.f * Ly.cin)), ++k);
  }
  init_kernel<<<1, 256, 0, c->stream>>>(s->w + s->off_hw, 2 * base, sqrtf(1.f / base), ++k);
  DOE_CUDA(c, cudaGetLastError());
  if ((rc = refresh_weights(s))) return fail(rc);
  *out = s;
  return DOE_OK;
}

extern "C" void doe_surrogate_destroy(doe_surrogate* s) {
  if (!s) return;
  if (s->c) cudaStreamSynchronize(s->c->stream);
  for (void* p : s->allocs) cudaFree(p);
  delete s;
}

extern "C" long long doe_surrogate_param_count(const doe_surrogate* s) { return s ? s->nparam : -1; }

extern "C" int doe_surrogate_params(doe_surrogate* s, float* host_out, int which) {
  if (!s || !host_out) return DOE_ERR_BAD_ARG;
  const float* src = which == 0 ? s->w : (which == 1 ? s->g : nullptr);
  if (!src) return set_err(s->c, DOE_ERR_BAD_ARG, "surrogate: which must be 0 (weights) or 1 (gradients)");
  DOE_CUDA(s->c, cudaMemcpyAsync(host_out, src, sizeof(float) * s->nparam, cudaMemcpyDeviceToHost, s->c->stream));
  DOE_CUDA(s->c, cudaStreamSynchronize(s->c->stream));
  return DOE_OK;
}

extern "C" int doe_surrogate_set_params(doe_surrogate* s, const float* host_in) {
  if (!s || !host_in) return DOE_ERR_BAD_ARG;
  DOE_CUDA(s->c, cudaMemcpyAsync(s->w, host_in, sizeof(float) * s->nparam, cudaMemcpyHostToDevice, s->c->stream));
  DOE_CUDA(s->c, cudaMemsetAsync(s->m, 0, sizeof(float) * s->nparam, s->c->stream));
  DOE_CUDA(s->c, cudaMemsetAsync(s->v, 0, sizeof(float) * s->nparam, s->c->stream));
  s->step = 0;
  return refresh_weights(s);
}

// Forward pass of B <= max_batch images: d_irr, d_roi (may be NULL) [B][n*n] FP32
// on the device; d_phase [B][n*n] receives atan2(s, c). Keeps the activations
// for doe_surrogate_backward.
extern "C" int doe_surrogate_forward(doe_surrogate* s, int B, const float* d_irr, const float* d_roi, float* d_phase) {
  if (!s || !d_irr || !d_phase) return DOE_ERR_BAD_ARG;
  if (B < 1 || B > s->max_batch) return set_err(s->c, DOE_ERR_BAD_ARG, "surrogate: batch %d outside [1, %d]", B, s->max_batch);
  doe_ctx* c = s->c;
  const int L = s->levels, n = s->n;
  const long nn = (long)n * n;
  const Idx I = layer_index(L);
  s->batch = B;
  {
    LaunchScope ls(c, "unet_input");
    unet_scale_kernel<<<B, 256, 0, c->stream>>>(d_irr, (int)nn, s->scale);
    unet_input_kernel<<<grid_for(B * nn * s->base), 256, 0, c->stream>>>(d_irr, d_roi, s->scale, (int)nn, s->base,
                                                                          B * nn, s->x0.p);
    DOE_CUDA(c, cudaGetLastError());
  }
  const bf16* in = s->x0.p;
  int in_cs = s->x0.C;
  for (int l = 0; l < L - 1; ++l) {
    const int h = n >> l, C = s->base << l;
    DOE_TRY(conv_fwd(s, I.enc_a[l], B, in, in_cs, s->a[l].p, s->a[l].C, h, h));
    DOE_TRY(conv_fwd(s, I.enc_b[l], B, s->a[l].p, s->a[l].C, s->cat[l].p, s->cat[l].C, h, h));
    LaunchScope ls(c, "unet_pool");
    pool_fwd_kernel<<<grid_for((long)B * h * h / 4 * C), 256, 0, c->stream>>>(s->cat[l].p, s->cat[l].C,
                                                                              s->pin[l + 1].p, s->pin[l + 1].C, B, h,
                                                                              h, C);
    DOE_CUDA(c, cudaGetLastError());
    in = s->pin[l + 1].p;
    in_cs = s->pin[l + 1].C;
  }
  const int hb = n >> (L - 1);
  DOE_TRY(conv_fwd(s, I.bott_a, B, in, in_cs, s->b1.p, s->b1.C, hb, hb));
  DOE_TRY(conv_fwd(s, I.bott_b, B, s->b1.p, s->b1.C, s->b2.p, s->b2.C, hb, hb));
  const bf16* prev = s->b2.p;
  int prev_cs = s->b2.C;
  for (int l = L - 2; l >= 0; --l) {
    const int h = n >> l, C = s->base << l, Cp = s->base << (l + 1);
    {
      LaunchScope ls(c, "unet_up");
      up_fwd_kernel<<<grid_for((long)B * h * h * Cp), 256, 0, c->stream>>>(prev, prev_cs, s->u[l].p, s->u[l].C, B,
                                                                          h / 2, h / 2, Cp);
      DOE_CUDA(c, cudaGetLastError());
    }
    DOE_TRY(conv_fwd(s, I.dec_up[l], B, s->u[l].p, s->u[l].C, s->cat[l].p + C, s->cat[l].C, h, h));
    DOE_TRY(conv_fwd(s, I.dec_a[l], B, s->cat[l].p, s->cat[l].C, s->da[l].p, s->da[l].C, h, h));
    DOE_TRY(conv_fwd(s, I.dec_b[l], B, s->da[l].p, s->da[l].C, s->d[l].p, s->d[l].C, h, h));
    prev = s->d[l].p;
    prev_cs = s->d[l].C;
  }
  {
    LaunchScope ls(c, "unet_head");
    head_fwd_kernel<<<grid_for(B * nn), 256, 0, c->stream>>>(s->d[0].p, s->base, s->w + s->off_hw, s->w + s->off_hb,
                                                             B * nn, s->cs, d_phase);
    DOE_CUDA(c, cudaGetLastError());
  }
  return DOE_OK;
}

// Backward pass of the last forward: d_dphase [B][n*n] = dL/dphase (device FP32).
// Gradients are accumulated into the FP32 gradient buffer (zeroed by
// doe_surrogate_zero_grad or by each Adam step).
extern "C" int doe_surrogate_backward(doe_surrogate* s, const float* d_dphase) {
  if (!s || !d_dphase) return DOE_ERR_BAD_ARG;
  if (s->batch < 1) return set_err(s->c, DOE_ERR_BAD_ARG, "surrogate: backward without a forward pass");
  doe_ctx* c = s->c;
  const int L = s->levels, n = s->n, B = s->batch;
  const long nn = (long)n * n;
  const Idx I = layer_index(L);
  {
    LaunchScope ls(c, "unet_head_bwd");
    head_bwd_kernel<<<grid_for(B * nn), 256, 0, c->stream>>>(s->d[0].p, s->base, s->w + s->off_hw, s->cs, d_dphase,
                                                             B * nn, s->d[0].g, s->g + s->off_hw, s->g + s->off_hb);
    DOE_CUDA(c, cudaGetLastError());
  }
  // decoder, from level 0 up; the gradient of `prev` (d_{l+1} or b2) comes out masked
  for (int l = 0; l <= L - 2; ++l) {
    const int h = n >> l, C = s->base << l, Cp = s->base << (l + 1);
    Act& dl = s->d[l];
    Act& dal = s->da[l];
    Act& cl = s->cat[l];
    Act& ul = s->u[l];
    DOE_TRY(conv_wgrad(s, I.dec_b[l], B, dal.p, dal.C, dl.g, dl.C, h, h));
    DOE_TRY(conv_dgrad(s, I.dec_b[l], B, dl.g, dl.C, dal.g, dal.C, dal.p, dal.C, h, h));
    DOE_TRY(conv_wgrad(s, I.dec_a[l], B, cl.p, cl.C, dal.g, dal.C, h, h));
    DOE_TRY(conv_dgrad(s, I.dec_a[l], B, dal.g, dal.C, cl.g, cl.C, cl.p, cl.C, h, h));
    DOE_TRY(conv_wgrad(s, I.dec_up[l], B, ul.p, ul.C, cl.g + C, cl.C, h, h));
    DOE_TRY(conv_dgrad(s, I.dec_up[l], B, cl.g + C, cl.C, ul.g, ul.C, nullptr, 0, h, h));
    // up-sample backward into the gradient of prev (masked by prev > 0)
    Act& pv = (l + 1 <= L - 2) ? s->d[l + 1] : s->b2;
    LaunchScope ls(c, "unet_up_bwd");
    up_bwd_kernel<<<grid_for((long)B * (h / 2) * (h / 2) * Cp), 256, 0, c->stream>>>(ul.g, ul.C, pv.g, pv.C, pv.p,
                                                                                      pv.C, B, h / 2, h / 2, Cp);
    DOE_CUDA(c, cudaGetLastError());
  }
  // bottleneck
  const int hb = n >> (L - 1);
  Act& pb = s->pin[L - 1];
  DOE_TRY(conv_wgrad(s, I.bott_b, B, s->b1.p, s->b1.C, s->b2.g, s->b2.C, hb, hb));
  DOE_TRY(conv_dgrad(s, I.bott_b, B, s->b2.g, s->b2.C, s->b1.g, s->b1.C, s->b1.p, s->b1.C, hb, hb));
  DOE_TRY(conv_wgrad(s, I.bott_a, B, pb.p, pb.C, s->b1.g, s->b1.C, hb, hb));
  DOE_TRY(conv_dgrad(s, I.bott_a, B, s->b1.g, s->b1.C, pb.g, pb.C, nullptr, 0, hb, hb));
  // encoder, from the deepest level down
  for (int l = L - 2; l >= 0; --l) {
    const int h = n >> l, C = s->base << l;
    Act& cl = s->cat[l];
    Act& al = s->a[l];
    {
      LaunchScope ls(c, "unet_pool_bwd");
      pool_bwd_kernel<<<grid_for((long)B * h * h * C), 256, 0, c->stream>>>(cl.g, cl.C, s->pin[l + 1].g,
                                                                            s->pin[l + 1].C, cl.p, cl.C, B, h, h, C);
      DOE_CUDA(c, cudaGetLastError());
    }
    DOE_TRY(conv_wgrad(s, I.enc_b[l], B, al.p, al.C, cl.g, cl.C, h, h));
    DOE_TRY(conv_dgrad(s, I.enc_b[l], B, cl.g, cl.C, al.g, al.C, al.p, al.C, h, h));
    const Act& in = l == 0 ? s->x0 : s->pin[l];
    DOE_TRY(conv_wgrad(s, I.enc_a[l], B, in.p, in.C, al.g, al.C, h, h));
    if (l > 0) DOE_TRY(conv_dgrad(s, I.enc_a[l], B, al.g, al.C, s->pin[l].g, s->pin[l].C, nullptr, 0, h, h));
  }
  return DOE_OK;
}

// Device copies of the FP32 gradient buffer, for data-parallel training
// (all-reduce between backward and Adam).
extern "C" int doe_surrogate_grads_dev(doe_surrogate* s, float* d_out) {
  if (!s || !d_out) return DOE_ERR_BAD_ARG;
  DOE_CUDA(s->c, cudaMemcpyAsync(d_out, s->g, sizeof(float) * s->nparam, cudaMemcpyDeviceToDevice, s->c->stream));
  return DOE_OK;
}
extern "C" int doe_surrogate_set_grads_dev(doe_surrogate* s, const float* d_in) {
  if (!s || !d_in) return DOE_ERR_BAD_ARG;
  DOE_CUDA(s->c, cudaMemcpyAsync(s->g, d_in, sizeof(float) * s->nparam, cudaMemcpyDeviceToDevice, s->c->stream));
  return DOE_OK;
}

extern "C" int doe_surrogate_zero_grad(doe_surrogate* s) {
  if (!s) return DOE_ERR_BAD_ARG;
  DOE_CUDA(s->c, cudaMemsetAsync(s->g, 0, sizeof(float) * s->nparam, s->c->stream));
  return DOE_OK;
}

// One Adam step on the accumulated gradients (scaled by grad_scale), then the
// gradients are zeroed and the BF16 weight copies refreshed.
extern "C" int doe_surrogate_adam(doe_surrogate* s, float lr, float beta1, float beta2, float eps, float weight_decay,
                                  float grad_scale) {
  if (!s) return DOE_ERR_BAD_ARG;
  s->step += 1;
  const float bc1 = 1.f - powf(beta1, (float)s->step), bc2 = 1.f - powf(beta2, (float)s->step);
  {
    LaunchScope ls(s->c, "unet_adam");
    adam_kernel<<<grid_for(s->nparam), 256, 0, s->c->stream>>>(s->w, s->g, s->m, s->v, s->nparam, lr, beta1, beta2,
                                                               eps, weight_decay, bc1, bc2, grad_scale);
    DOE_CUDA(s->c, cudaGetLastError());
  }
  DOE_TRY(doe_surrogate_zero_grad(s));
  return refresh_weights(s);
}

namespace {
// grad = sin(phase - target) / count; block sums of 1 - cos into one FP64 atomic
__global__ void supervised_kernel(long count, const float* ph, const float* tg, float* grad, double* loss) {
  __shared__ double red[256];
  double acc = 0.0;
  const float inv = 1.f / (float)count;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
    float sn, cs;
    sincosf(ph[i] - tg[i], &sn, &cs);
    grad[i] = sn * inv;
    acc += 1.0 - cs;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0 && loss) atomicAdd(loss, red[0] / (double)count);
}
}  // namespace

extern "C" int doe_phase_supervised_grad(doe_ctx* c, long long count, const float* d_phase, const float* d_target,
                                         float* d_grad, double* d_loss) {
  if (!c || !d_phase || !d_target || !d_grad || count <= 0) return DOE_ERR_BAD_ARG;
  if (d_loss) DOE_CUDA(c, cudaMemsetAsync(d_loss, 0, sizeof(double), c->stream));
  LaunchScope ls(c, "unet_supervised_loss");
  supervised_kernel<<<grid_for(count), 256, 0, c->stream>>>(count, d_phase, d_target, d_grad, d_loss);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}
