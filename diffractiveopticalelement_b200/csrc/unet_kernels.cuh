// unet_kernels.cuh -- BF16 kernels of the warm-start surrogate (a U-Net that maps
// a target irradiance to a DOE phase). No counterpart in the reference.
//
// Activations are NHWC bf16 with an explicit channel stride (a layer may read or
// write a channel slice of a wider concatenation buffer). Convolutions are 3x3,
// pad 1, stride 1, as implicit GEMMs on the tensor cores (mma.sync m16n8k16,
// BF16 operands, FP32 accumulation):
//   forward / input gradient : C[pixels][Cout] = A[pixels][9 Cin] * W^T,  A = im2col(in)
//   weight gradient          : dW[Cout][9 Cin] = dOut^T[Cout][pixels] * im2col(in)
// The input gradient is the forward convolution of dOut with the flipped,
// channel-transposed kernel. Operand tiles are staged in shared memory with
// cp.async (zero-filled halo) and fed to the MMAs with ldmatrix. Layers whose
// GEMM input has a multiple of 64 channels run the same GEMM on tcgen05 instead
// (unet_tc.cuh); these kernels serve the 32-channel layers and the weight gradient.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace doe {
namespace unet {

// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// 16-byte async copy global -> shared; src_bytes 0 fills zeros (src must still be valid).
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// ------------------------------------------------------------------ convolution
struct ConvArgs {
  const __nv_bfloat16* in;  // [P][in_cs], channels [0, cin)
  int in_cs, cin;
  const __nv_bfloat16* w;   // [cout][9][cin]
  const float* bias;        // [cout] or null
  __nv_bfloat16* out;       // [P][out_cs], channels [0, cout)
  int out_cs, cout;
  const __nv_bfloat16* mask;  // null, or [P][mask_cs]: zero the output where mask <= 0
  int mask_cs;
  int relu;
  int B, H, W;              // P = B H W pixels
};

constexpr int kBM = 128;     // pixels per CTA
constexpr int kBK = 32;      // reduction slice (channels of one tap)
constexpr int kSA = kBK + 8; // padded smem row (80 B): ldmatrix rows land in distinct banks
constexpr int kConvThreads = 128;

// Forward 3x3 convolution (also the input gradient with transformed weights).
// Grid: (ceil(P / 128), cout / BN). Requires cin % 32 == 0, cout % BN == 0.
template <int BN>
__global__ void __launch_bounds__(kConvThreads) conv3x3_kernel(ConvArgs a) {
  constexpr int WN = BN / 32;           // warps along N
  constexpr int WM = 4 / WN;            // warps along M
  constexpr int TM = kBM / WM;          // warp tile rows (64 or 32)
  constexpr int MF = TM / 16;
  constexpr int NF = 4;                 // 32 columns per warp
  __shared__ __align__(16) __nv_bfloat16 As[2][kBM * kSA];
  __shared__ __align__(16) __nv_bfloat16 Bs[2][BN * kSA];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % WM, wn = warp / WM;
  const long P = (long)a.B * a.H * a.W;
  const long p0 = (long)blockIdx.x * kBM;
  const int co0 = blockIdx.y * BN;
  const int K = 9 * a.cin;
  const int KT = K / kBK;

  // per-thread A rows: thread handles row r = tid (one pixel), 4 chunks of 8 channels
  const long p = p0 + tid;
  int py = 0, px = 0;
  long pbase = 0;  // pixel index of (n, 0, 0)
  const bool prow = p < P;
  if (prow) {
    const long hw = (long)a.H * a.W;
    const long n = p / hw;
    const long rem = p - n * hw;
    py = (int)(rem / a.W);
    px = (int)(rem - (long)py * a.W);
    pbase = n * hw;
  }

  auto load_tile = [&](int kt, int st) {
    const int k0 = kt * kBK;
    const int tap = k0 / a.cin, ci0 = k0 - tap * a.cin;
    const int ky = tap / 3, kx = tap - ky * 3;
    const int yy = py + ky - 1, xx = px + kx - 1;
    const bool ok = prow && yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
    const __nv_bfloat16* src = ok ? a.in + (pbase + (long)yy * a.W + xx) * a.in_cs + ci0 : a.in;
    __nv_bfloat16* dst = &As[st][tid * kSA];
#pragma unroll
    for (int c = 0; c < 4; ++c) cp_async16(dst + c * 8, ok ? src + c * 8 : a.in, ok ? 16 : 0);
    // B: BN rows x 4 chunks
#pragma unroll
    for (int i = tid; i < BN * 4; i += kConvThreads) {
      const int r = i >> 2, c = i & 3;
      cp_async16(&Bs[st][r * kSA + c * 8], a.w + (long)(co0 + r) * K + k0 + c * 8, 16);
    }
  };

  float acc[MF][NF][4];
#pragma unroll
  for (int i = 0; i < MF; ++i)
#pragma unroll
    for (int j = 0; j < NF; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;

  load_tile(0, 0);
  cp_async_commit();
  for (int kt = 0; kt < KT; ++kt) {
    const int st = kt & 1;
    if (kt + 1 < KT) {
      load_tile(kt + 1, st ^ 1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 16) {
      uint32_t af[MF][4];
#pragma unroll
      for (int i = 0; i < MF; ++i) {
        const int row = wm * TM + i * 16 + (lane & 15);
        ldsm_x4(af[i], &As[st][row * kSA + kk + (lane >> 4) * 8]);
      }
#pragma unroll
      for (int j = 0; j < NF; j += 2) {
        uint32_t bf[4];
        const int n = wn * 32 + j * 8 + (lane & 7) + ((lane >> 4) << 3);
        ldsm_x4(bf, &Bs[st][n * kSA + kk + ((lane >> 3) & 1) * 8]);
#pragma unroll
        for (int i = 0; i < MF; ++i) {
          mma_bf16(acc[i][j], af[i], bf[0], bf[1]);
          mma_bf16(acc[i][j + 1], af[i], bf[2], bf[3]);
        }
      }
    }
    __syncthreads();
  }

  // epilogue: bias, ReLU, mask, bf16 pairs
#pragma unroll
  for (int i = 0; i < MF; ++i) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long pr = p0 + wm * TM + i * 16 + (lane >> 2) + h * 8;
      if (pr >= P) continue;
#pragma unroll
      for (int j = 0; j < NF; ++j) {
        const int col = co0 + wn * 32 + j * 8 + 2 * (lane & 3);
        float v0 = acc[i][j][2 * h], v1 = acc[i][j][2 * h + 1];
        if (a.bias) {
          v0 += a.bias[col];
          v1 += a.bias[col + 1];
        }
        if (a.relu) {
          v0 = fmaxf(v0, 0.f);
          v1 = fmaxf(v1, 0.f);
        }
        if (a.mask) {
          const __nv_bfloat162 m = *reinterpret_cast<const __nv_bfloat162*>(a.mask + pr * a.mask_cs + col);
          if (!(__bfloat162float(m.x) > 0.f)) v0 = 0.f;
          if (!(__bfloat162float(m.y) > 0.f)) v1 = 0.f;
        }
        *reinterpret_cast<__nv_bfloat162*>(a.out + pr * a.out_cs + col) = __floats2bfloat162_rn(v0, v1);
      }
    }
  }
}

// Weight (and bias) gradient. dW32[co][tap][ci] += sum_p dOut[p][co] in[p + tap][ci].
// Grid: (cout / BMW, 9 cin / 32, splits); each CTA reduces pixels
// [z * chunk, (z+1) * chunk) in steps of 32 and adds its tile with FP32 atomics.
struct WgradArgs {
  const __nv_bfloat16* in;
  int in_cs, cin;
  const __nv_bfloat16* dout;
  int dout_cs, cout;
  float* dw;    // [cout][9 cin] FP32
  float* db;    // [cout] FP32 or null
  int B, H, W;
  long chunk;   // pixels per split (multiple of 32)
};

constexpr int kWP = 32;  // pixels per step
template <int BMW>
__global__ void __launch_bounds__(kConvThreads) wgrad_kernel(WgradArgs a) {
  constexpr int WM = BMW / 16;  // warps along M (co)
  constexpr int WN = 4 / WM;    // warps along N (k)
  constexpr int TN = 32 / WN;   // warp tile columns (32 or 16)
  constexpr int NF = TN / 8;
  constexpr int SD = BMW + 8;   // padded rows
  constexpr int SX = 32 + 8;
  __shared__ __align__(16) __nv_bfloat16 Ds[2][kWP * SD];
  __shared__ __align__(16) __nv_bfloat16 Xs[2][kWP * SX];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % WM, wn = warp / WM;
  const long P = (long)a.B * a.H * a.W;
  const long hw = (long)a.H * a.W;
  const int co0 = blockIdx.x * BMW;
  const int k0 = blockIdx.y * 32;
  const int tap = k0 / a.cin, ci0 = k0 - tap * a.cin;
  const int ky = tap / 3, kx = tap - ky * 3;
  const long pb = (long)blockIdx.z * a.chunk;
  const long pe = pb + a.chunk < P ? pb + a.chunk : P;
  const int steps = pe > pb ? (int)((pe - pb + kWP - 1) / kWP) : 0;

  auto load = [&](int s, int st) {
    const long ps = pb + (long)s * kWP;
    // dOut tile: 32 pixels x BMW channels (BMW / 8 chunks per pixel)
    for (int i = tid; i < kWP * (BMW / 8); i += kConvThreads) {
      const int r = i / (BMW / 8), c = i % (BMW / 8);
      const long p = ps + r;
      const bool ok = p < pe;
      cp_async16(&Ds[st][r * SD + c * 8], ok ? a.dout + p * a.dout_cs + co0 + c * 8 : a.dout, ok ? 16 : 0);
    }
    // im2col tile: 32 pixels x 32 channels of tap (ky, kx)
    {
      const int r = tid >> 2, c = tid & 3;
      const long p = ps + r;
      bool ok = p < pe;
      long src = 0;
      if (ok) {
        const long n = p / hw;
        const long rem = p - n * hw;
        const int y = (int)(rem / a.W), x = (int)(rem - (long)(rem / a.W) * a.W);
        const int yy = y + ky - 1, xx = x + kx - 1;
        ok = yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
        src = (n * hw + (long)yy * a.W + xx) * a.in_cs + ci0 + c * 8;
      }
      cp_async16(&Xs[st][r * SX + c * 8], ok ? a.in + src : a.in, ok ? 16 : 0);
    }
  };

  float acc[NF][4];
#pragma unroll
  for (int j = 0; j < NF; ++j)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[j][q] = 0.f;
  float bsum = 0.f;

  if (steps > 0) {
    load(0, 0);
    cp_async_commit();
  }
  for (int s = 0; s < steps; ++s) {
    const int st = s & 1;
    if (s + 1 < steps) {
      load(s + 1, st ^ 1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kWP; kk += 16) {
      // A = dOut^T (co x p): transposed loads from Ds[p][co]
      uint32_t af[4];
      {
        const int q = lane >> 3, i = lane & 7;
        const int pr = kk + i + ((q >> 1) << 3);
        const int cc = wm * 16 + ((q & 1) << 3);
        ldsm_x4_t(af, &Ds[st][pr * SD + cc]);
      }
#pragma unroll
      for (int j = 0; j < NF; j += 2) {
        uint32_t bf[4];
        const int q = lane >> 3, i = lane & 7;
        const int pr = kk + i + ((q & 1) << 3);
        const int nn = wn * TN + j * 8 + ((q >> 1) << 3);
        ldsm_x4_t(bf, &Xs[st][pr * SX + nn]);
        mma_bf16(acc[j], af, bf[0], bf[1]);
        mma_bf16(acc[j + 1], af, bf[2], bf[3]);
      }
    }
    // bias gradient: threads of the first k-tile sum their channel over the step
    if (a.db && blockIdx.y == 0 && tid < BMW) {
      for (int r = 0; r < kWP; ++r) bsum += __bfloat162float(Ds[st][r * SD + tid]);
    }
    __syncthreads();
  }
  // accumulate the tile
#pragma unroll
  for (int j = 0; j < NF; ++j) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int co = co0 + wm * 16 + (lane >> 2) + h * 8;
      const int kc = k0 + wn * TN + j * 8 + 2 * (lane & 3);
      float* d = a.dw + (long)co * 9 * a.cin + kc;
      atomicAdd(d, acc[j][2 * h]);
      atomicAdd(d + 1, acc[j][2 * h + 1]);
    }
  }
  if (a.db && blockIdx.y == 0 && tid < BMW && steps > 0) atomicAdd(a.db + co0 + tid, bsum);
}

}  // namespace unet
}  // namespace doe
