// stage_mixed.cu -- the mixed-precision low-storage RK stage.
//
// Same stage as lsrk_stage_kernel except for the interpolation. The
// per-element Vandermonde contraction that gives every particle its Lagrange
// values, l = W m(r) (push_monomial.hpp:155-210), is one GEMM for a whole
// CTA of 128 particles, L[128 x Np] = M[128 x Np] W^T with W shared by all
// elements, and runs on the 5th-generation tensor cores: the monomials
// (FP32) and W (rounded to FP32) are each split into three BF16 terms,
// x = x0 + x1 + x2, and the six products of total order < 3,
//   a0 b0 + a0 b1 + a1 b0 + a0 b2 + a1 b1 + a2 b0,
// accumulate in FP32 in tensor memory (tcgen05.mma kind::f16, M = 128, one
// thread issues, completion through an mbarrier). Each thread then reads its
// own row (tcgen05.ld, lane = particle), forms the six field components as
// FP32 sums over the element's nodes, and continues in FP64: force, RK
// update, relocation (stage_from_fields, shared with the FP64 stage).
//
// Shared-memory operands use the no-swizzle K-major canonical layout: for
// each chunk of 8 consecutive K elements, the R rows' 16-byte pieces are
// contiguous (offset (chunk * R + row) * 16): core matrices of 8 rows x 16
// bytes, 8-row groups 128 bytes apart (stride byte offset), K chunks
// R * 16 bytes apart (leading byte offset).
//
// A CTA walks tiles of 128 particles (the launch gives one tile per CTA);
// it allocates its tensor memory (32 columns, 64 for order 4), initialises its mbarrier and
// stages W once. The wait on the MMA's mbarrier is bounded; when it runs out the kernel
// records PRT_ERR_TIMEOUT, skips the update and the remaining tiles, waits
// again (bounded) and frees its tensor memory.

#include <cuda_bf16.h>

#include <cstring>
#include <mutex>
#include <vector>

#include "push.cuh"

namespace {

constexpr int MX_BLOCK = 128;  // particles per CTA = MMA M = tensor-memory lanes
constexpr unsigned MX_SPIN = 1u << 20;  // try_wait rounds before giving up


template <int ORDER>
struct MixedShape {
  static constexpr int NP = Lagrange<ORDER>::NP;
  static constexpr int KP = (NP + 15) / 16 * 16;    // monomials, padded to the K step (16)
  static constexpr int NPAD = (NP + 15) / 16 * 16;  // Lagrange values (N % 16 == 0 at M = 128)
  // tensor-memory columns: a power of two >= 32 and >= NPAD
  static constexpr int COLS = NPAD <= 32 ? 32 : 64;
  static constexpr int A_BYTES = MX_BLOCK * KP * 2; // one BF16 term of the monomials
  static constexpr int B_BYTES = NPAD * KP * 2;     // one BF16 term of W
  static constexpr int SMEM = 3 * A_BYTES + 3 * B_BYTES + 16;
  // Lagrange values read back per thread: 32 columns, plus 8 more for order 4
  static constexpr int LV = NP > 32 ? 40 : 32;
  static_assert(NPAD <= COLS && NP <= LV, "mixed stage: orders 1-4");
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// tcgen05 shared-memory matrix descriptor, no swizzle, K-major.
__device__ __forceinline__ uint64_t mma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of this architecture
  return d;                // base offset 0, layout type 0 (no swizzle)
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  for (unsigned k = 0; k < MX_SPIN; ++k)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// 8 FP32 values -> one 16-byte chunk of each of the three BF16 terms
__device__ __forceinline__ void split8(const float v[8], uint4 &t0, uint4 &t1, uint4 &t2) {
  uint32_t w0[4], w1[4], w2[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    __nv_bfloat16 h[2], m[2], l[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const float x = v[2 * k + e];
      h[e] = __float2bfloat16_rn(x);
      const float r1 = x - __bfloat162float(h[e]);
      m[e] = __float2bfloat16_rn(r1);
      l[e] = __float2bfloat16_rn(r1 - __bfloat162float(m[e]));
    }
    w0[k] = (uint32_t)__bfloat16_as_ushort(h[0]) | ((uint32_t)__bfloat16_as_ushort(h[1]) << 16);
    w1[k] = (uint32_t)__bfloat16_as_ushort(m[0]) | ((uint32_t)__bfloat16_as_ushort(m[1]) << 16);
    w2[k] = (uint32_t)__bfloat16_as_ushort(l[0]) | ((uint32_t)__bfloat16_as_ushort(l[1]) << 16);
  }
  t0 = make_uint4(w0[0], w0[1], w0[2], w0[3]);
  t1 = make_uint4(w1[0], w1[1], w1[2], w1[3]);
  t2 = make_uint4(w2[0], w2[1], w2[2], w2[3]);
}

template <int ORDER>
__global__ void __launch_bounds__(MX_BLOCK)
    lsrk_stage_mixed_kernel(DevMesh M, Fields6 F, const uint4 *__restrict__ wsplit, long long n,
                            double *__restrict__ x, double *__restrict__ p,
                            const double *__restrict__ q, const double *__restrict__ mass,
                            uint32_t *__restrict__ el, double *__restrict__ kx,
                            double *__restrict__ kp, double a, double b, double dt, double c,
                            DevStatus *st) {
  using SH = MixedShape<ORDER>;
  constexpr int NP = SH::NP, KP = SH::KP, NPAD = SH::NPAD;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *A = smem;                     // 3 terms x [KP/8 chunks][128 rows][16 B]
  unsigned char *Bm = smem + 3 * SH::A_BYTES;  // 3 terms x [KP/8 chunks][NPAD rows][16 B]
  uint64_t *bar = (uint64_t *)(Bm + 3 * SH::B_BYTES);
  uint32_t *tmem_slot = (uint32_t *)(bar + 1);

  const int tid = threadIdx.x, warp = tid >> 5;

  // once per CTA: tensor memory for the 128 x NPAD FP32 accumulator, the
  // mbarrier, the W terms (copied as laid out in global memory)
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"((uint32_t)SH::COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int k = tid; k < 3 * SH::B_BYTES / 16; k += MX_BLOCK)
    reinterpret_cast<uint4 *>(Bm)[k] = wsplit[k];
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t bar_a = smem_u32(bar);
  // kind::f16 instruction descriptor: D FP32, A and B BF16, both K-major,
  // N = NPAD, M = 128
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NPAD >> 3) << 17) |
                         ((uint32_t)(MX_BLOCK >> 4) << 24);

  bool ok = true;  // every wait so far completed
  uint32_t parity = 0;
  const long long tiles = (n + MX_BLOCK - 1) / MX_BLOCK;
  for (long long tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x, parity ^= 1u) {
    const long long i = tile * MX_BLOCK + tid;
    const uint32_t e = i < n ? el[i] : PRT_INVALID;
    bool live = e != PRT_INVALID;
    unsigned ctr[4] = {0, 0, 0, 0};

    // this particle's monomials (FP64 reference coordinates, FP32 values)
    double xx[3] = {0, 0, 0}, pp[3] = {0, 0, 0};
    float mono[KP];
#pragma unroll
    for (int j = 0; j < KP; ++j) mono[j] = 0.0f;
    if (live) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        xx[d] = x[d * n + i];
        pp[d] = p[d * n + i];
      }
      double r0, r1, r2;
      apply_map_exact(M.inv_maps + 12 * (size_t)e, xx[0], xx[1], xx[2], r0, r1, r2);
      double pw0[ORDER + 1], pw1[ORDER + 1], pw2[ORDER + 1];
      pw0[0] = pw1[0] = pw2[0] = 1.0;
#pragma unroll
      for (int k = 1; k <= ORDER; ++k) {
        pw0[k] = pw0[k - 1] * r0;
        pw1[k] = pw1[k - 1] * r1;
        pw2[k] = pw2[k - 1] * r2;
      }
      int idx = 0;
#pragma unroll
      for (int cc = 0; cc <= ORDER; ++cc)
#pragma unroll
        for (int bb = 0; bb <= ORDER - cc; ++bb)
#pragma unroll
          for (int aa = 0; aa <= ORDER - bb - cc; ++aa)
            mono[idx++] = (float)(pw0[aa] * pw1[bb] * pw2[cc]);
    }
    // the previous tile's tcgen05.ld of every thread is complete (waited
    // before its update): A may be overwritten and the accumulator reused
#pragma unroll
    for (int ch = 0; ch < KP / 8; ++ch) {
      uint4 t0, t1, t2;
      split8(mono + 8 * ch, t0, t1, t2);
      const size_t off = ((size_t)ch * MX_BLOCK + tid) * 16;
      *reinterpret_cast<uint4 *>(A + off) = t0;
      *reinterpret_cast<uint4 *>(A + SH::A_BYTES + off) = t1;
      *reinterpret_cast<uint4 *>(A + 2 * SH::A_BYTES + off) = t2;
    }
    // generic-proxy shared-memory writes -> visible to the tensor cores
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (tid == 0) {
      const uint32_t a0 = smem_u32(A), b0 = smem_u32(Bm);
      // (A term, W term) pairs of total order < 3
      const int ta[6] = {0, 0, 1, 0, 1, 2}, tb[6] = {0, 1, 0, 2, 1, 0};
      uint32_t acc = 0;
#pragma unroll
      for (int t = 0; t < 6; ++t)
#pragma unroll
        for (int kk = 0; kk < KP / 16; ++kk) {
          const uint64_t da = mma_desc(a0 + ta[t] * SH::A_BYTES + kk * 2 * MX_BLOCK * 16,
                                       MX_BLOCK * 16, 128);
          const uint64_t db =
              mma_desc(b0 + tb[t] * SH::B_BYTES + kk * 2 * NPAD * 16, NPAD * 16, 128);
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                  tmem),
              "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
              : "memory");
          acc = 1;
        }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              bar_a)
          : "memory");
    }

    const bool done = mbar_wait_bounded(bar_a, parity);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    ok = __syncthreads_and(done) != 0;  // CTA-uniform: every thread leaves together
    // this warp's 32 lanes, 32 (40) columns: row = particle
    uint32_t lv[SH::LV];
    if (ok) {
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
          "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
          "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
          "[%32];\n"
          : "=r"(lv[0]), "=r"(lv[1]), "=r"(lv[2]), "=r"(lv[3]), "=r"(lv[4]), "=r"(lv[5]),
            "=r"(lv[6]), "=r"(lv[7]), "=r"(lv[8]), "=r"(lv[9]), "=r"(lv[10]), "=r"(lv[11]),
            "=r"(lv[12]), "=r"(lv[13]), "=r"(lv[14]), "=r"(lv[15]), "=r"(lv[16]),
            "=r"(lv[17]), "=r"(lv[18]), "=r"(lv[19]), "=r"(lv[20]), "=r"(lv[21]),
            "=r"(lv[22]), "=r"(lv[23]), "=r"(lv[24]), "=r"(lv[25]), "=r"(lv[26]),
            "=r"(lv[27]), "=r"(lv[28]), "=r"(lv[29]), "=r"(lv[30]), "=r"(lv[31])
          : "r"(tmem + ((uint32_t)(warp * 32) << 16))
          : "memory");
      if constexpr (SH::LV > 32) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
            : "=r"(lv[32]), "=r"(lv[33]), "=r"(lv[34]), "=r"(lv[35]), "=r"(lv[36]),
              "=r"(lv[37]), "=r"(lv[38]), "=r"(lv[39])
            : "r"(tmem + ((uint32_t)(warp * 32) << 16) + 32u)
            : "memory");
      }
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    } else {
      if (live) record_error(st, PRT_ERR_TIMEOUT, i);
      live = false;
    }

    if (live) {
      // fields: FP32 sums over the element's nodes
      float ef32[6] = {0, 0, 0, 0, 0, 0};
      const size_t nb = (size_t)e * NP;
#pragma unroll
      for (int nd = 0; nd < NP; ++nd) {
        const float l = __uint_as_float(lv[nd]);
#pragma unroll
        for (int k = 0; k < 6; ++k)
          if (F.f[k]) ef32[k] = fmaf(l, (float)__ldg(F.f[k] + nb + nd), ef32[k]);
      }
      double ef[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) ef[k] = (double)ef32[k];
      int err = 0;
      const uint32_t ne = stage_from_fields(M, e, ef, xx, pp, q[i], mass[i], kx, kp, n, i, a,
                                            b, dt, c, ctr, &err);
      if (err) record_error(st, err, i);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        x[d * n + i] = xx[d];
        p[d * n + i] = pp[d];
      }
      if (!err) el[i] = ne;
    }
    flush_counters(st, ctr);
    if (!ok) mbar_wait_bounded(bar_a, parity);  // the MMA is complete before the exit
  }

  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"((uint32_t)SH::COLS)
                 : "memory");
  }
}

// host: round-to-nearest-even FP32 -> BF16 bits (finite inputs)
uint16_t bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

float bf16_value(uint16_t h) {
  const uint32_t u = (uint32_t)h << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

template <int ORDER>
int prepare(prt_pusher *P) {
  using SH = MixedShape<ORDER>;
  std::vector<uint16_t> h(3 * (size_t)SH::B_BYTES / 2, 0);
  for (int nd = 0; nd < SH::NP; ++nd)
    for (int j = 0; j < SH::NP; ++j) {
      const float w = (float)P->w[(size_t)nd * SH::NP + j];
      const uint16_t t0 = bf16_bits(w);
      const float r1 = w - bf16_value(t0);
      const uint16_t t1 = bf16_bits(r1);
      const uint16_t t2 = bf16_bits(r1 - bf16_value(t1));
      // row nd (N), column j (K): chunk j / 8, element j % 8
      const size_t off = ((size_t)(j / 8) * SH::NPAD + nd) * 8 + (j % 8);
      h[off] = t0;
      h[SH::B_BYTES / 2 + off] = t1;
      h[SH::B_BYTES + off] = t2;
    }
  PRT_CHECK_CUDA(cudaMalloc(&P->w_split, h.size() * 2));
  PRT_CHECK_CUDA(cudaMemcpy(P->w_split, h.data(), h.size() * 2, cudaMemcpyHostToDevice));
  return PRT_OK;
}

template <int ORDER>
int launch(const prt_pusher *P, prt_workspace *ws, long long n, double *x, double *p,
           const double *q, const double *m, uint32_t *el, double *kx, double *kp,
           const Fields6 &F, double a, double b, double dt, double c, cudaStream_t s) {
  using SH = MixedShape<ORDER>;
  static_assert(SH::SMEM <= 227 * 1024, "mixed stage shared memory within a CTA's limit");
  if constexpr (SH::SMEM > 48 * 1024) {
    // order 4: above the default dynamic shared-memory limit (once per process;
    // the attribute holds for every device the kernel runs on)
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
      attr = cudaFuncSetAttribute(lsrk_stage_mixed_kernel<ORDER>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, SH::SMEM);
    });
    PRT_CHECK_CUDA(attr);
  }
  ScopedTimer timer(ws, PRT_TIME_LSRK_STAGE, s);
  // one CTA per tile of 128 particles measured fastest (2.36 ms per 16M-particle
  // stage on B200, against 2.4-3.7 ms with 3-7 CTAs per SM walking the tiles):
  // resident CTAs at different phases hide each other's synchronisation
  const long long tiles = (n + MX_BLOCK - 1) / MX_BLOCK;
  const unsigned blocks = (unsigned)tiles;
  lsrk_stage_mixed_kernel<ORDER><<<blocks, MX_BLOCK, SH::SMEM, s>>>(
      P->mesh->dev, F, (const uint4 *)P->w_split, n, x, p, q, m, el, kx, kp, a, b, dt, c,
      ws->status);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

}  // namespace

int prt_pusher_prepare_mixed(prt_pusher *P) {
  switch (P->order) {
    case 1: return prepare<1>(P);
    case 2: return prepare<2>(P);
    case 3: return prepare<3>(P);
    case 4: return prepare<4>(P);
  }
  return PRT_OK;
}

int launch_stage_mixed(const prt_pusher *P, prt_workspace *ws, long long n, double *x,
                       double *p, const double *q, const double *m, uint32_t *el, double *kx,
                       double *kp, const Fields6 &F, double a, double b, double dt, double c,
                       cudaStream_t s) {
  switch (P->order) {
    case 1: return launch<1>(P, ws, n, x, p, q, m, el, kx, kp, F, a, b, dt, c, s);
    case 2: return launch<2>(P, ws, n, x, p, q, m, el, kx, kp, F, a, b, dt, c, s);
    case 3: return launch<3>(P, ws, n, x, p, q, m, el, kx, kp, F, a, b, dt, c, s);
    case 4: return launch<4>(P, ws, n, x, p, q, m, el, kx, kp, F, a, b, dt, c, s);
  }
  return PRT_ERR_INVALID_ARGUMENT;
}
