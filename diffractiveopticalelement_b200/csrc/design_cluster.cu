// design_cluster.cu -- image-plane weightedGerchbergSaxton (src/doe.js:455-546
// driving gerchbergSaxton, :327-437) with the whole iteration loop resident on
// chip: one thread-block cluster per design keeps the design's complex64 work
// plane in distributed shared memory for every pass of every iteration.
//
// Layout: the plane's N rows are split over the R CTAs of the cluster (rank r
// holds rows r*N/R .. +N/R in its shared memory; R = 4 for 256^2, 1 for 64^2 and
// 128^2, whose plane fits one CTA). Row passes work on the CTA's own rows; column
// passes take C columns at a time, reading and writing each column's elements in
// the CTAs that hold its rows (ld/st through cluster-mapped shared-memory
// addresses), so the field never leaves the chip. Only the per-pixel side planes
// (target, ROI, weights, illumination, phase, the tabulated transfer function)
// stream from L2 / HBM, and the FP64 per-design sums are exchanged between the
// CTAs through shared memory.
//
// The pass sequence, the pointwise arithmetic and the FFT plans are those of the
// multi-pass loop (design_wgs.cu with the operators of design_ops.cuh), so the
// results agree with it to FP32 rounding of the FP64 sums' grouping; the design
// state (weights, phase, best iterate, histories, stop iteration) is left in the
// same buffers, for the same epilogue kernels.
//
// Synchronisation between the passes is a cluster barrier made of mbarriers with
// bounded waits (1 s): a wait that runs out records an error code in the
// context's design error word, and the CTA skips to the end, where all CTAs of the
// cluster meet once more before exiting (no CTA leaves while another may still
// access its shared memory).
#include <cooperative_groups.h>

#include "design_ops.cuh"
#include "tcgen05.cuh"

namespace cg = cooperative_groups;

namespace doe {
namespace {

constexpr uint64_t kClusterWaitNs = 1000000000ull;

// 512 threads (16 warps) per CTA and one CTA per SM: a batch of a row pass
// transforms 512 / T rows, one of a column pass 512 / T columns (T threads per
// transform, the default plan of length N).
template <int N>
struct ClusterGeom {
  static constexpr int R = N >= 256 ? 4 : 1;  // CTAs per design
  static constexpr int ROWS = N / R;          // rows per CTA
  static constexpr int THREADS = 512;
  using P = typename DefaultPlan<N>::type;
  using RS = RowShape<P, THREADS / P::T>;
  using CS = ColShape<P, THREADS / P::T>;
  static_assert(RS::THREADS == THREADS && CS::THREADS == THREADS, "one CTA shape for both passes");
  static_assert(ROWS % RS::V == 0 && ROWS % CS::C == 0, "batches tile the CTA's rows and columns");
  static constexpr int SCRATCH = RS::SMEM > CS::SMEM ? RS::SMEM : CS::SMEM;
  static constexpr int PLANE_BYTES = ROWS * N * 8;
  static constexpr int RED_OFF = PLANE_BYTES + SCRATCH;  // [R][kRedKGoal] doubles, 8-byte aligned
  static constexpr int MBAR_OFF = RED_OFF + R * kRedKGoal * 8;
  static constexpr int SMEM = MBAR_OFF + 16;
  static_assert(SMEM <= 227 * 1024, "one CTA's share of the plane fits its shared memory");
};

// Cluster barrier with bounded waits: every CTA's thread 0 arrives (release,
// cluster scope) on the mbarrier of every CTA; each CTA waits (acquire) on its
// own. Returns false, uniformly over the CTA, when the wait ran out.
struct ClusterBar {
  uint64_t* mbar;
  uint32_t phase;
  int R;
  __device__ __forceinline__ bool sync() {
    if (R == 1) {
      __syncthreads();
      return true;
    }
    asm volatile("fence.acq_rel.cluster;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      const uint32_t local = tc::smem_u32(mbar);
      for (int q = 0; q < R; ++q) {
        uint32_t remote;
        asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(local), "r"(q));
        asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(remote) : "memory");
      }
    }
    bool ok = try_wait(phase);
    if (!ok) {
      const uint64_t t0 = tc::global_ns();
      while (!(ok = try_wait(phase)) && tc::global_ns() - t0 < kClusterWaitNs) {
      }
    }
    phase ^= 1u;
    return __syncthreads_and(ok);
  }
  __device__ __forceinline__ bool try_wait(uint32_t parity) const {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(tc::smem_u32(mbar)), "r"(parity)
        : "memory");
    return done != 0;
  }
};

template <int N, bool GOAL>
struct ClusterWgs {
  using G = ClusterGeom<N>;
  using P = typename G::P;
  using RS = typename G::RS;
  using CS = typename G::CS;
  static constexpr int K = GOAL ? kRedKGoal : kRedK;
  static constexpr int RMAX = P::RMAX;

  DesignBufs b;
  const float2* tw;  // FFT twiddles of length N
  float scale;       // 1 / (N N)
  int iters;
  int* err;

  // ---------------------------------------------------------------- plane access
  struct Plane {
    float2* local;  // this CTA's rows
    // element (y, x) of the plane, in the shared memory of the CTA holding row y
    __device__ __forceinline__ float2* at(int y, int x) const {
      float2* p = local + (y % G::ROWS) * N + x;
      if constexpr (G::R == 1) {
        return p;
      } else {
        uint64_t r;
        asm("mapa.u64 %0, %1, %2;" : "=l"(r) : "l"(p), "r"(y / G::ROWS));
        return reinterpret_cast<float2*>(r);
      }
    }
  };

  // Row pass over this CTA's rows: `load(y, x)` gives the input, `mid(y, x, v)`
  // acts between the two transforms (when STAGES == 2), `store(y, x, v, acc)`
  // consumes the output. All threads of the CTA take part (batches of V rows).
  // The side planes are read where they are used: an L1 prefetch of a whole
  // batch's lines ahead of the transform (as the multi-pass kernels do) measured
  // ~8 % slower here, the 32-row batch's lines exceeding what is left of L1 next
  // to the shared memory, and the extra load instructions throttling the LSU.
  template <bool INV1, bool INV2, int STAGES, class Load, class Mid, class Store>
  __device__ __forceinline__ void row_pass(const Plane& pl, float2* scratch, int row0, Load load, Mid mid,
                                           Store store, DAcc<K>& acc) const {
    constexpr int T = P::T, V = RS::V;
    const int lv = threadIdx.x / T, t = threadIdx.x % T;
    SmemVec<> s{scratch + lv * padded_len<N>(), 1, 0};
#pragma unroll 1
    for (int b0 = 0; b0 < G::ROWS; b0 += V) {
      const int yl = b0 + lv, y = row0 + yl;
      float2 v[RMAX];
#pragma unroll
      for (int q = 0; q < RMAX; ++q) v[q] = load(pl, yl, y, in_elem<P>(t, q));
      fft_run<P, INV1>(v, t, s, tw, BlockSync{});
      if constexpr (STAGES == 2) {
#pragma unroll
        for (int q = 0; q < RMAX; ++q) mid(yl, y, out_elem<P>(t, q), v[q]);
        relayout_out_to_in<P>(v, t, s, BlockSync{});
        fft_run<P, INV2>(v, t, s, tw, BlockSync{});
      }
#pragma unroll
      for (int q = 0; q < RMAX; ++q) store(pl, yl, y, out_elem<P>(t, q), v[q], acc);
      __syncthreads();  // the scratch is reused by the next batch
    }
  }

  // Column pass over this CTA's columns: forward column FFT, x H (or conj H),
  // inverse column FFT, in place in the distributed plane.
  template <bool CONJ>
  __device__ __forceinline__ void col_asm(const Plane& pl, float2* scratch, int col0, const float2* htab) const {
    constexpr int C = CS::C;
    const int c = threadIdx.x % C, t = threadIdx.x / C;
    SmemVec<P::PSHIFT> s{scratch, C, c};
#pragma unroll 1
    for (int b0 = 0; b0 < G::ROWS; b0 += C) {
      const int x = col0 + b0 + c;
#pragma unroll
      for (int q = 0; q < RMAX; ++q) prefetch_l1(&htab[(long)out_elem<P>(t, q) * N + x]);
      float2 v[RMAX];
#pragma unroll
      for (int q = 0; q < RMAX; ++q) v[q] = *pl.at(in_elem<P>(t, q), x);
      fft_run<P, false>(v, t, s, tw, BlockSync{});
#pragma unroll
      for (int q = 0; q < RMAX; ++q) {
        const float2 h = __ldg(&htab[(long)out_elem<P>(t, q) * N + x]);
        v[q] = CONJ ? cmulc(v[q], h) : cmul(v[q], h);
      }
      relayout_out_to_in<P>(v, t, s, BlockSync{});
      fft_run<P, true>(v, t, s, tw, BlockSync{});
#pragma unroll
      for (int q = 0; q < RMAX; ++q) *pl.at(out_elem<P>(t, q), x) = v[q];
      __syncthreads();
    }
  }

  // FP64 sums of this CTA -> every CTA's slot `rank` -> (after the barrier) the
  // design totals, folded in rank order (identical in every CTA).
  __device__ __forceinline__ bool cluster_sum(DAcc<K>& acc, double* red, int rank, ClusterBar& bar,
                                              double (&tot)[K]) const {
    block_sum<K>(acc);
    if (threadIdx.x == 0) {
      cg::cluster_group cl = cg::this_cluster();
      for (int q = 0; q < G::R; ++q) {
        double* dst = G::R > 1 ? cl.map_shared_rank(red, q) : red;
#pragma unroll
        for (int k = 0; k < K; ++k) dst[rank * kRedKGoal + k] = acc.v[k];
      }
    }
    if (!bar.sync()) return false;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double v = 0.0;
      for (int q = 0; q < G::R; ++q) v += red[q * kRedKGoal + k];
      tot[k] = v;
    }
    return true;
  }

  __device__ __forceinline__ void run() const {
    extern __shared__ __align__(16) unsigned char smraw[];
    float2* plane = reinterpret_cast<float2*>(smraw);
    float2* scratch = reinterpret_cast<float2*>(smraw + G::PLANE_BYTES);
    double* red = reinterpret_cast<double*>(smraw + G::RED_OFF);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smraw + G::MBAR_OFF);
    cg::cluster_group cl = cg::this_cluster();
    const int rank = G::R > 1 ? (int)cl.block_rank() : 0;
    const int d = blockIdx.x / G::R;  // design
    const int row0 = rank * G::ROWS;
    if (threadIdx.x == 0) {
      tc::mbar_init(mbar, G::R);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if constexpr (G::R > 1) {
      cl.sync();  // every mbarrier is initialised before the first remote arrive
    } else {
      __syncthreads();
    }
    const Plane pl{plane};
    ClusterBar bar{mbar, 0u, G::R};

    const long n = (long)N * N, o = (long)d * n;
    const float* A = b.illum + o;
    float* ph = b.phase + o;
    const float* tg = b.tgt + (long)d * b.tgt_stride;
    const float* m = b.roi ? b.roi + (long)d * b.tgt_stride : nullptr;
    float* wr = b.wraw + o;
    const float* sirr = (GOAL && b.screen_irr) ? b.screen_irr + o : nullptr;
    const float2* htab = b.htab + (long)d * b.htab_stride;
    DesignState S = b.st[d];  // identical copy in every CTA
    bool ok = true;
    DAcc<K> acc;
    auto clear = [&]() {
#pragma unroll
      for (int k = 0; k < K; ++k) acc.v[k] = 0.0;
    };
    double T[K];
    auto no_mid = [](int, int, int, float2&) {};
    auto keep = [](const Plane& p, int yl, int, int x, float2 v, DAcc<K>&) { p.local[yl * N + x] = v; };
    auto mine = [](const Plane& p, int yl, int, int x) { return p.local[yl * N + x]; };

    // ---- A exp(i phi), forward row FFT (RowDoeFwd)
    clear();
    row_pass<false, false, 1>(
        pl, scratch, row0,
        [=](const Plane&, int, int y, int x) {
          const float a = __ldg(&A[(long)y * N + x]);
          float sn, cs;
          sincosf(__ldg(&ph[(long)y * N + x]), &sn, &cs);
          return make_float2(a * cs, a * sn);
        },
        no_mid, keep, acc);
    ok = ok && bar.sync();
    if (ok) col_asm<false>(pl, scratch, row0, htab);
    ok = ok && bar.sync();
    // ---- forward field: inverse row FFT -> U (kept in the plane), efficiency (RowWgsTarget<true>)
    if (ok) {
      clear();
      row_pass<true, false, 1>(
          pl, scratch, row0, mine, no_mid,
          [=](const Plane& p, int yl, int y, int x, float2 v, DAcc<K>& a) {
            const long i = (long)y * N + x;
            const float mm = m ? __ldg(&m[i]) : 1.f;
            const float2 u = cscale(v, scale);
            p.local[yl * N + x] = u;
            const float am = sqrtf(u.x * u.x + u.y * u.y);
            const double ad = am, i2 = ad * ad;
            a.v[kTotal] += i2;
            if (mm > 0.f) a.v[kInRoi] += i2 * mm;
            if constexpr (GOAL) {
              const double Tv = sirr ? (double)__ldg(&sirr[i]) : (double)__ldg(&tg[i]) * __ldg(&tg[i]);
              a.v[kST] += Tv;
              if (mm > 0.f) a.v[kSTT] += Tv * Tv;
            }
          },
          acc);
      ok = cluster_sum(acc, red, rank, bar, T);
      if (ok) {
        S.eff_cur = T[kTotal] > 0 ? (T[kInRoi] * b.dx * b.dy) / (T[kTotal] * b.dx * b.dy) : 0.0;
        if constexpr (GOAL) {
          S.sT = T[kST];
          S.sTT = T[kSTT];
        }
      }
    }
    bool prev_improved = false;
    for (int it = 0; it < iters && ok; ++it) {
      // ---- constraint t w norm inside the ROI, snapshot of an improved previous
      // iterate, forward row FFT of the back-propagation (RowWgsConstrain)
      {
        const float wn = (float)S.norm;
        const bool snap = prev_improved;
        clear();
        row_pass<false, false, 1>(
            pl, scratch, row0,
            [=](const Plane& p, int yl, int y, int x) {
              const long i = (long)y * N + x;
              const float2 u = p.local[yl * N + x];
              const float mm = m ? __ldg(&m[i]) : 1.f;
              const float t = __ldg(&tg[i]);
              const float w = wr[i];
              const float am = sqrtf(u.x * u.x + u.y * u.y);
              if (snap) {
                b.best_phase[o + i] = ph[i];
                b.best_amp[o + i] = am;
              }
              if (mm > 0.f && am > 0.f) return cscale(u, (t * (w * wn)) / am);
              return u;
            },
            no_mid, keep, acc);
      }
      ok = bar.sync();
      if (!ok) break;
      col_asm<true>(pl, scratch, row0, htab);  // back-propagation (-z)
      ok = bar.sync();
      if (!ok) break;
      // ---- inverse row FFT, new phase, A exp(i phi), forward row FFT (RowDoeUpdate<true>)
      clear();
      row_pass<true, false, 2>(
          pl, scratch, row0, mine,
          [=](int, int y, int x, float2& v) {
            const long i = (long)y * N + x;
            const float a = __ldg(&A[i]);
            const float phv = atan2f(v.y, v.x);
            ph[i] = phv;
            const float2 u = unit_phasor(v);
            v = make_float2(a * u.x, a * u.y);
          },
          keep, acc);
      ok = bar.sync();
      if (!ok) break;
      col_asm<false>(pl, scratch, row0, htab);  // forward propagation (+z)
      ok = bar.sync();
      if (!ok) break;
      // ---- inverse row FFT -> U, RMSE, weight update, sums (RowWgsTarget<false>)
      {
        const float wn = (float)S.norm;
        clear();
        row_pass<true, false, 1>(
            pl, scratch, row0, mine, no_mid,
            [=](const Plane& p, int yl, int y, int x, float2 v, DAcc<K>& a) {
              const long i = (long)y * N + x;
              const float mm = m ? __ldg(&m[i]) : 1.f;
              const float t = __ldg(&tg[i]);
              const float wold = wr[i];
              const float2 u = cscale(v, scale);
              p.local[yl * N + x] = u;
              const float am = sqrtf(u.x * u.x + u.y * u.y);
              const double ad = am, i2 = ad * ad;
              a.v[kTotal] += i2;
              if (mm > 0.f) a.v[kInRoi] += i2 * mm;
              if (mm > 0.f) {
                const double dd = ad - (double)t;
                a.v[kRmseNum] += dd * dd;
                a.v[kRmseDen] += (double)t * t;
                const float ratio = am > 1e-30f ? t / am : 2.f;
                float w = wold * wn * powf(fminf(fmaxf(ratio, 0.25f), 4.f), b.beta);
                w = fminf(fmaxf(w, 1e-4f), 1e4f);
                wr[i] = w;
                a.v[kWsum] += (double)w * w * t * t;
                a.v[kTsum] += (double)t * t;
              }
              if constexpr (GOAL) {
                const double Tv = sirr ? (double)__ldg(&sirr[i]) : (double)t * t;
                a.v[kSIM] += i2 * mm;
                if (mm > 0.f) {
                  a.v[kSII] += i2 * i2;
                  a.v[kSIT] += i2 * Tv;
                }
              }
            },
            acc);
      }
      ok = cluster_sum(acc, red, rank, bar, T);
      if (!ok) break;
      const double eff = T[kTotal] > 0 ? (T[kInRoi] * b.dx * b.dy) / (T[kTotal] * b.dx * b.dy) : 0.0;
      const double rmse = T[kRmseDen] > 0 ? sqrt(T[kRmseNum] / T[kRmseDen]) : 0.0;
      bool imp = rmse < S.best;
      bool stop = false;
      if constexpr (GOAL) {
        // screen RMSE exactly as screen_metrics_kernel (the pitch cancels)
        const double sc = S.sT > 0 ? T[kSIM] / S.sT : 0.0;
        const double den = sc * sc * S.sTT;
        const double num = fmax(0.0, T[kSII] - 2.0 * sc * T[kSIT] + sc * sc * S.sTT);
        const double srm = den > 0 ? sqrt(num / den) : 0.0;
        if (srm <= b.rmse_goal) {
          S.stop = it;
          imp = true;  // return the iterate that met the goal
          stop = true;
        }
      }
      if (imp) S.best = rmse;
      const long h = (long)d * b.iters + it;
      if (rank == 0 && threadIdx.x == 0) {
        b.improved[h] = imp ? 1 : 0;
        b.err_hist[h] = S.best;
        b.eff_hist[h] = S.eff_cur;
      }
      S.eff_cur = eff;
      S.norm = T[kWsum] > 0 ? sqrt(T[kTsum] / T[kWsum]) : 1.0;
      prev_improved = imp;
      if (stop || it == iters - 1) {
        // the field that met the goal, or the last one, leaves the chip: the
        // snapshot of a stopped design is taken here, the last iteration's by the
        // epilogue kernel from U
        for (int k = threadIdx.x; k < G::ROWS * N; k += G::THREADS) {
          const long i = (long)row0 * N + k;
          const float2 u = pl.local[k];
          b.U[o + i] = u;
          if (stop) {
            b.best_phase[o + i] = ph[i];
            b.best_amp[o + i] = sqrtf(u.x * u.x + u.y * u.y);
          }
        }
        if (stop) break;
      }
    }
    if (!ok && threadIdx.x == 0) atomicExch(err, 2);
    if (rank == 0 && threadIdx.x == 0) b.st[d] = S;
    if constexpr (G::R > 1) cl.sync();  // no CTA exits while another may still use its shared memory
  }
};

template <int N, bool GOAL>
__global__ void __launch_bounds__(512, 1) wgs_cluster_kernel(ClusterWgs<N, GOAL> k) {
  k.run();
}

template <int N, bool GOAL>
int launch_cluster(doe_ctx* c, const DesignBufs& b, int B, int I) {
  using G = ClusterGeom<N>;
  int* err;
  DOE_TRY(design_error_word(c, &err));
  ClusterWgs<N, GOAL> k{b, c->tw + N, 1.f / (float)((long)N * N), I, err};
  auto kern = wgs_cluster_kernel<N, GOAL>;
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device
  if (!(attr_set.load() & (1ull << (c->device & 63)))) {
    DOE_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM));
    attr_set.fetch_or(1ull << (c->device & 63));
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(B * G::R));
  cfg.blockDim = dim3(G::THREADS);
  cfg.dynamicSmemBytes = G::SMEM;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = G::R;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  LaunchScope ls(c, "design_wgs_cluster");
  DOE_CUDA(c, cudaLaunchKernelEx(&cfg, kern, k));
  return DOE_OK;
}

}  // namespace

int design_error_word(doe_ctx* c, int** out) {
  const bool fresh = c->slot[kSlotErr] == nullptr;
  void* p;
  DOE_TRY(ensure_slot(c, kSlotErr, 64, &p));
  if (fresh) DOE_CUDA(c, cudaMemsetAsync(p, 0, 64, c->stream));
  *out = (int*)p;
  return DOE_OK;
}

int design_error_check(doe_ctx* c) {
  if (!c->slot[kSlotErr]) return DOE_OK;
  int h = 0;
  DOE_CUDA(c, cudaMemcpy(&h, c->slot[kSlotErr], sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    DOE_CUDA(c, cudaMemset(c->slot[kSlotErr], 0, sizeof(int)));
    return set_err(c, DOE_ERR_TIMEOUT,
                   "a bounded device wait gave up (code %d: 2 = a cluster barrier of the on-chip design loop, "
                   "3 = an MMA of the surrogate's tensor-core convolution, 4 = a TMA copy of the sweep column pass)",
                   h);
  }
  return DOE_OK;
}

// Cluster-resident image-plane WGS for square 64^2, 128^2 and 256^2 designs;
// returns DOE_ERR_UNSUPPORTED for other grids (the caller then runs the passes).
int design_run_wgs_cluster(doe_ctx* c, const DesignBufs& b, int B, int I) {
  if (b.nx != b.ny || !b.U || !b.wraw) return DOE_ERR_UNSUPPORTED;
  const bool goal = b.rmse_goal > 0;
  switch (b.nx) {
    case 64: return goal ? launch_cluster<64, true>(c, b, B, I) : launch_cluster<64, false>(c, b, B, I);
    case 128: return goal ? launch_cluster<128, true>(c, b, B, I) : launch_cluster<128, false>(c, b, B, I);
    case 256: return goal ? launch_cluster<256, true>(c, b, B, I) : launch_cluster<256, false>(c, b, B, I);
    default: return DOE_ERR_UNSUPPORTED;
  }
}

}  // namespace doe
