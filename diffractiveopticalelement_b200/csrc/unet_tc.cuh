// unet_tc.cuh -- the surrogate's 3x3 convolution (forward, and the input gradient
// with the flipped kernel) on the tcgen05 tensor cores. No counterpart in the
// reference.
//
// The same implicit GEMM as conv3x3_kernel, C[pixels][cout] = im2col(in) * W^T,
// with the accumulator in tensor memory: a CTA owns a tile of 128 consecutive
// pixels (TMEM lanes) x BN output channels (TMEM columns, FP32). The reduction
// runs over 9 taps x cin/64 chunks of 64 input channels; each chunk's operands are
// one 128-byte row per pixel (A, the tap's shifted pixel, zero outside the image)
// and per output channel (B, the weights), copied with cp.async into the K-major
// 128-byte-swizzled layout the MMA reads, through a ring of STAGES stages. One
// thread issues the four K = 16 BF16 MMAs of a chunk and commits them to the
// stage's mbarrier; the stage is refilled once that barrier reports the MMAs
// done with it. The epilogue reads each warp's 32 TMEM lanes, adds the bias,
// applies ReLU or the mask and stores BF16.
//
// Every mbarrier wait is bounded (1 s): on a timeout the CTA records code 3 in
// the context's error word, waits once more (bounded) for the MMAs it issued,
// frees its tensor memory and returns without storing.
#pragma once
#include <cuda.h>

#include "tcgen05.cuh"
#include "unet_kernels.cuh"

namespace doe {
namespace unet {

constexpr uint64_t kTcWaitNs = 1000000000ull;

template <int BN, int S_ = 3>
struct ConvTc {
  static constexpr int S = S_;  // stages of the operand ring
  static constexpr int A_BYTES = 128 * 128;  // 128 pixel rows x 64 bf16
  static constexpr int B_BYTES = BN * 128;   // BN weight rows x 64 bf16
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int BAR_OFF = S * STAGE;          // stage barriers, then the final one
  static constexpr int SLOT_OFF = BAR_OFF + 8 * (S + 1);
  static constexpr int SMEM = SLOT_OFF + 16 + 1024;          // + slack to align the base to 1024 B
  static constexpr uint32_t TMEM_COLS = BN < 32 ? 32 : BN;
  static_assert(STAGE % 1024 == 0, "swizzled tiles start on 1024-byte boundaries");
  // kind::f16 with BF16 A and B (formats 1 in bits [7,10) and [10,13)), FP32 accumulator
  static constexpr uint32_t IDESC = tc::idesc_f16_f32(128, BN) | (1u << 7) | (1u << 10);
};

// 32 consecutive FP32 TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Grid: (ceil(P / 128), cout / BN), 128 threads. Requires cin % 64 == 0, cout % BN == 0,
// channel strides multiples of 8 and 16-byte aligned planes (as conv3x3_kernel).
template <int BN, int STAGES>
__global__ void __launch_bounds__(128) conv3x3_tc_kernel(ConvArgs a, int* __restrict__ err) {
  using G = ConvTc<BN, STAGES>;
  constexpr int S = G::S;
  extern __shared__ unsigned char smraw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + G::BAR_OFF);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + G::SLOT_OFF);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long P = (long)a.B * a.H * a.W;
  const long p0 = (long)blockIdx.x * 128;
  const int co0 = blockIdx.y * BN;
  const int K = 9 * a.cin;  // length of a weight row
  const int CK = a.cin >> 6;
  const int KT = 9 * CK;

  // this thread's A row: pixel p0 + tid
  const long p = p0 + tid;
  const bool prow = p < P;
  int py = 0, px = 0;
  long pbase = 0;
  if (prow) {
    const long hw = (long)a.H * a.W;
    const long n = p / hw;
    const long rem = p - n * hw;
    py = (int)(rem / a.W);
    px = (int)(rem - (long)py * a.W);
    pbase = n * hw;
  }

  if (tid == 0) {
    for (int s = 0; s <= S; ++s) tc::mbar_init(&bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tc::tmem_alloc(tslot, G::TMEM_COLS);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tslot;

  auto load = [&](int kt, int st) {
    const int tap = kt / CK, ci0 = (kt - tap * CK) << 6;
    const int ky = tap / 3, kx = tap - ky * 3;
    const int yy = py + ky - 1, xx = px + kx - 1;
    const bool ok = prow && yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
    const __nv_bfloat16* src = ok ? a.in + (pbase + (long)yy * a.W + xx) * a.in_cs + ci0 : a.in;
    unsigned char* As = sm + st * G::STAGE;
#pragma unroll
    for (int c = 0; c < 8; ++c) cp_async16(As + tc::sw128_off(tid, c), ok ? src + c * 8 : a.in, ok ? 16 : 0);
    unsigned char* Bs = As + G::A_BYTES;
    const __nv_bfloat16* wrow = a.w + (long)co0 * K + tap * a.cin + ci0;
#pragma unroll
    for (int i = tid; i < BN * 8; i += 128) {
      const int r = i >> 3, c = i & 7;
      cp_async16(Bs + tc::sw128_off(r, c), wrow + (long)r * K + c * 8, 16);
    }
  };

  bool ok = true;
#pragma unroll
  for (int s = 0; s < S - 1; ++s) {
    if (s < KT) load(s, s);
    cp_async_commit();
  }
  for (int kt = 0; kt < KT; ++kt) {
    const int st = kt % S;
    cp_async_wait<S - 2>();  // this thread's copies of chunk kt have landed
    tc::fence_proxy_async();
    __syncthreads();         // ... and every other thread's
    if (tid == 0) {
      tc::fence_after();
      const uint32_t ab = tc::smem_u32(sm + st * G::STAGE), bb = ab + G::A_BYTES;
#pragma unroll
      for (int k = 0; k < 4; ++k)
        tc::mma_f16_ss(tmem, tc::desc_k_sw128(ab + 32 * k), tc::desc_k_sw128(bb + 32 * k), G::IDESC,
                       (kt | k) != 0 ? 1u : 0u);
      tc::commit(&bar[st]);
    }
    const int nk = kt + S - 1;  // refill the stage chunk kt - 1 used
    if (nk < KT) {
      const int ns = nk % S;
      if (kt >= 1 && !tc::mbar_wait_bounded(&bar[ns], (uint32_t)(((kt - 1) / S) & 1), kTcWaitNs)) ok = false;
      ok = __syncthreads_and(ok);
      if (!ok) break;
      load(nk, ns);
    }
    cp_async_commit();
  }
  cp_async_wait<0>();
  // every MMA this CTA issued is done once the final barrier completes
  if (tid == 0) {
    tc::fence_before();
    tc::commit(&bar[S]);
  }
  bool done = tc::mbar_wait_bounded(&bar[S], 0, kTcWaitNs);
  done = __syncthreads_and(done) && ok;
  tc::fence_after();
  if (done) {
    const int row = warp * 32 + lane;
    const long pr = p0 + row;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 32) {
      float v[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (pr < P) {
#pragma unroll
        for (int j = 0; j < 32; j += 2) {
          const int col = co0 + c0 + j;
          float v0 = v[j], v1 = v[j + 1];
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
  } else if (tid == 0) {
    atomicExch(err, 3);
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after();
    tc::tmem_dealloc(tmem, G::TMEM_COLS);
  }
}

// ------------------------------------------------------------------ TMA-fed form
// The same convolution with both operands brought in by the tensor memory
// accelerator (cp.async.bulk.tensor, no multicast): the A tile of a tap is one box
// of the NHWC activation tensor -- 64 channels x BW pixels x BH rows at the tap's
// shifted position, the halo outside the image filled with zeros by the copy
// itself -- and the B tile one box of the [nout][9 kch] weight matrix; both land
// in the 128-byte-swizzled K-major layout of the MMA. One thread drives the whole
// ring (each stage: expect the bytes, two bulk copies, wait full, four MMAs,
// commit; a stage is refilled once the MMAs that read it are done), so the loads
// need no warps of their own and the ring can be deep. A tile is 128 consecutive
// pixels of one image: a 128-pixel row segment (W >= 128) or 128 / W whole rows.
template <int BN, int S_>
struct ConvTma {
  static constexpr int S = S_;
  static constexpr int A_BYTES = 128 * 128;
  static constexpr int B_BYTES = BN * 128;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int BAR_OFF = S * STAGE;  // full[S], empty[S], done
  static constexpr int SLOT_OFF = BAR_OFF + 8 * (2 * S + 1);
  static constexpr int SMEM = SLOT_OFF + 16 + 1024;
  static constexpr uint32_t TMEM_COLS = BN < 32 ? 32 : BN;
  static constexpr uint32_t IDESC = tc::idesc_f16_f32(128, BN) | (1u << 7) | (1u << 10);
  static_assert(STAGE % 1024 == 0, "swizzled tiles start on 1024-byte boundaries");
};

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(tc::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(tc::smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          tc::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(tc::smem_u32(bar))
      : "memory");
}

// Grid: (P / 128, nout / BN), 128 threads. tmA: [B][H][W][kch] activations (channel
// stride a.in_cs), box {64, bw, bh, 1} with bw * bh = 128; tmB: [nout][9 kch]
// weights, box {64, BN}.
template <int BN, int STAGES>
__global__ void __launch_bounds__(128) conv3x3_tma_kernel(const __grid_constant__ CUtensorMap tmA,
                                                          const __grid_constant__ CUtensorMap tmB, ConvArgs a,
                                                          int bw, int bh, int* __restrict__ err) {
  using G = ConvTma<BN, STAGES>;
  constexpr int S = G::S;
  extern __shared__ unsigned char smraw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + G::BAR_OFF);
  uint64_t* empty = full + S;
  uint64_t* done_bar = full + 2 * S;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + G::SLOT_OFF);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long hw = (long)a.H * a.W;
  const long p0 = (long)blockIdx.x * 128;
  const int img = (int)(p0 / hw);
  const int rem = (int)(p0 - (long)img * hw);
  const int y0 = rem / a.W, x0 = rem - y0 * a.W;
  const int co0 = blockIdx.y * BN;
  const int CK = a.cin >> 6;
  const int KT = 9 * CK;

  if (tid == 0) {
    for (int s = 0; s < 2 * S + 1; ++s) tc::mbar_init(&full[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tc::tmem_alloc(tslot, G::TMEM_COLS);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tslot;

  bool ok = true;
  if (tid == 0) {
    int issued = 0, consumed = 0;  // chunks whose copies were issued / whose full barrier completed
    auto issue = [&](int kt, int st) {
      const int tap = kt / CK, ci0 = (kt - tap * CK) << 6;
      const int ky = tap / 3, kx = tap - ky * 3;
      unsigned char* As = sm + st * G::STAGE;
      mbar_expect_tx(&full[st], (uint32_t)G::STAGE);
      tma_load_4d(As, &tmA, ci0, x0 + kx - 1, y0 + ky - 1, img, &full[st]);
      tma_load_2d(As + G::A_BYTES, &tmB, tap * a.cin + ci0, co0, &full[st]);
      issued = kt + 1;
    };
    for (int k = 0; k < S && k < KT; ++k) issue(k, k);
    for (int kt = 0; kt < KT && ok; ++kt) {
      const int st = kt % S;
      if (!tc::mbar_wait_bounded(&full[st], (uint32_t)((kt / S) & 1), kTcWaitNs)) {
        ok = false;
        break;
      }
      consumed = kt + 1;
      tc::fence_after();
      const uint32_t ab = tc::smem_u32(sm + st * G::STAGE), bb = ab + G::A_BYTES;
#pragma unroll
      for (int k = 0; k < 4; ++k)
        tc::mma_f16_ss(tmem, tc::desc_k_sw128(ab + 32 * k), tc::desc_k_sw128(bb + 32 * k), G::IDESC,
                       (kt | k) != 0 ? 1u : 0u);
      tc::commit(&empty[st]);
      // refill the stage chunk kt - 1 read, once its MMAs are done
      if (kt >= 1 && kt - 1 + S < KT) {
        const int ps = (kt - 1) % S;
        if (!tc::mbar_wait_bounded(&empty[ps], (uint32_t)(((kt - 1) / S) & 1), kTcWaitNs)) {
          ok = false;
          break;
        }
        issue(kt - 1 + S, ps);
      }
    }
    // on a timeout, the copies still in flight land before the CTA leaves (bounded)
    for (int k = consumed; !ok && k < issued; ++k) (void)tc::mbar_wait_bounded(&full[k % S], (uint32_t)((k / S) & 1), kTcWaitNs);
    tc::fence_before();
    tc::commit(done_bar);  // arrives once every MMA issued above is done
  }
  ok = __syncthreads_and(ok);
  bool done = tc::mbar_wait_bounded(done_bar, 0, kTcWaitNs);
  done = __syncthreads_and(done) && ok;
  tc::fence_after();
  if (done) {
    const int row = warp * 32 + lane;
    const long pr = p0 + row;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 32) {
      float v[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
#pragma unroll
      for (int j = 0; j < 32; j += 2) {
        const int col = co0 + c0 + j;
        float v0 = v[j], v1 = v[j + 1];
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
  } else if (tid == 0) {
    atomicExch(err, 3);
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after();
    tc::tmem_dealloc(tmem, G::TMEM_COLS);
  }
}

}  // namespace unet
}  // namespace doe
