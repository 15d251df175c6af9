// deposit_tc.cu -- the chosen-form shape deposition on the tensor cores.
//
// The reference deposits q S(x_node - x_p) particle by particle over the
// elements its walk reaches (dep_shape.hpp:128-149), and the normalising
// depositor first integrates each particle's shape over the nodes it reaches,
// sum_e |J_e| sum_i w_i S_i, and deposits q / integral instead of q
// (dep_normshape.hpp:125-199). Both are sums over (particle, node position)
// pairs within the radius a of S(r) = N (a - r^2/a)^2 = N a^2 (1 - r^2/a^2)^2.
//
// Here the distinct node positions are cut into tiles of <= 128 (compact
// boxes at most two radii wide from recursive bisection, cut per shape
// radius; all but a few tiles hold exactly 128) and each CTA takes one tile:
//
//  1. candidates: the particles of the bin rows within the radius of the
//     tile's box (particles binned and packed in bin order, binning.cuh),
//     culled against the box grown by the radius, are staged 128 at a time
//     (a chunk) in a shared-memory ring by all eight warps;
//  2. score: one tcgen05.mma (kind::f16, M = 128 positions, N = 128
//     candidates, K = 16) gives s = SIGMA (1 - |u - w|^2 / a^2) for every
//     pair, with u and w the coordinates relative to the tile centre. The
//     operands are split into two FP16 terms (x = x_h + x_l) and laid out so
//     that one K = 16 product sums u_h v_h + u_h v_l + u_l v_h for the three
//     coordinates (v = 2 SIGMA w), the position term SIGMA (1 - |u|^2) and
//     the particle term -SIGMA |w|^2, each as two terms; the tensor cores
//     accumulate in FP32 into tensor memory;
//  3. weight: each thread reads its row (tcgen05.ld), forms
//     t = s + |s| = 2 max(s, 0) and the integer F = round(t^2) =
//     round(4 SIGMA^2 max(1 - r^2/a^2, 0)^2) < 2^23 with one FMA
//     (t t + 2^23 puts the rounded integer in the low mantissa bits), and
//     writes the word back in place (tcgen05.st): its bytes 0-2 are F's
//     base-256 digits, byte 3 a constant;
//  4. sums: tcgen05.mma kind::i8 with A in tensor memory (the weight words
//     as unsigned 8-bit K elements; int32 accumulation, exact) against digit
//     rows in shared memory laid out so that three views one row apart
//     multiply bytes 2, 1 and 0 by the digits and byte 3 by zero (N = 48):
//      - deposition: per candidate the charge c (q or q / integral) scaled
//        to a signed integer below 2^46 in six balanced signed digits and
//        c v (each component below 2^22, three digits), one 16-column
//        operand; rows =
//        positions, so tensor memory accumulates sum_p F c per position over
//        the whole tile (folded into FP64 every 256 chunks before int32
//        could overflow);
//      - normalisation: per position the weight sum_{nodes} |J_e| w_i (which
//        is negative at some nodes of order 2 and 4 elements) as a 47-bit
//        signed integer in six balanced signed digits; this pass scores with
//        rows = candidates (the same products, so bitwise the same F), so the
//        product is, per candidate, sum_u F W over the tile, which the CTA
//        adds to the particle's integral as two exact 64-bit integer atomics
//        (signed high part, low 40 bits): integer sums do not depend on the
//        order, so the result is deterministic.
//     The weights F of both passes are bitwise the same (same tiles, same
//     operands, same instructions), and every sum of F is exact, so the
//     deposited charge sum_u W_u rho_u equals sum_p q_p up to the 46-bit
//     representation of W and c and the final FP64 roundings (~1e-16).
//     The tiles are at most two radii wide, so every score operand stays
//     within FP16 range.
//
// Synchronisation per chunk k of a CTA: the score MMA of chunk k and the
// accumulation MMA of chunk k-1 run while the warps stage chunk k+1 (the
// ring of five chunks holds chunks k-1 .. k+1 and at most 255 slots more);
// the weights of chunk k are written over its scores once they are ready
// (mbarrier); one thread of a warp that stages nothing issues the
// accumulation MMA of chunk k and then the score MMA of chunk k+1 (the MMAs
// of one thread run in issue order, so the scores overwrite the weight words
// only after the accumulation has read them), and one commit signals the
// scores: it covers the accumulation issued before them too, so the sums of
// chunk k-1 are read (or the next window's tiles reuse its ring slots) once
// the scores of chunk k are ready; only the last chunk's sums have a commit
// of their own. Every
// mbarrier wait is bounded: a CTA whose wait runs out records PRT_ERR_TIMEOUT,
// stops, waits (bounded) for its issued MMAs and frees its tensor memory.

#include <cuda_fp16.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "binning.cuh"

namespace {

using namespace prt_dep;

constexpr int TM = 128;          // positions per tile: MMA M, tensor-memory lanes
constexpr int NC = 128;          // candidates per chunk: score MMA N
constexpr int RING = 5 * NC;     // candidate slots in shared memory: five chunks
constexpr int THREADS = 256;     // eight warps
constexpr int FILL_WARPS = 7;    // warps 0-6 stage candidates
constexpr int ISSUE_WARP = 7;    // warp 7 issues the tensor-core work
constexpr int MAXSEG = 512;      // bin-row segments per tile
constexpr uint32_t TMEM_COLS = 256;
constexpr uint32_t COL_ACC = 128;  // accumulators: weight byte 2 - j at +16 j (j = 0, 1, 2)
constexpr float SIGMA = 1448.0f;   // 4 SIGMA^2 < 2^23
constexpr int FLUSH_CHUNKS = 256;    // int32 accumulation window (256 * 128 * 255 * 128 < 2^31)
constexpr int CDIG = 6, JDIG = 3, WDIG = 6;


struct Smem {
  uint8_t apos[2 * TM * 16];     // position operand, K-major: [K chunk][row][16 B]
  uint8_t bcand[2 * RING * 16];  // candidate operands, K-major: [K chunk][slot][16 B]
  // The sums' B operand (MN-major rows of 16 digit bytes, one row per K): a
  // weight word holds the K elements 4 c .. 4 c + 3 (bytes 0-3 of F + 2^23),
  // so each candidate (deposition) or position (normalisation) c has four
  // rows, its digits in row 4 c + 3 and zeros in 4 c .. 4 c + 2; three views
  // one row apart (SBO 16 bytes) multiply bytes 2, 1, 0 by the digits
  union {
    uint8_t zdig[(4 * RING + 3) * 16];  // deposition: charge digits per slot
    struct {
      uint8_t zw[(4 * TM + 3) * 16];    // normalisation: position weight digits
      uint32_t slot_id[RING];           // bin-order particle of a slot
      uint32_t hits[2][2][NC];          // [chunk parity][column half][candidate]
    } n;
    double tsum[TM][16];                // deposition epilogue: digit sums per position
  };
  // per segment: the origin of its first bin relative to the tile centre
  // (periodic image included) and that bin's x index
  float4 seg_o[MAXSEG];
  uint2 seg_sl[MAXSEG];          // per segment: first bin-order particle, length
  unsigned long long bar_s, bar_a;
  uint32_t tmem;
  int tail, nseg, abort;
};
// 2 CTAs per SM at most (2 x 256 tensor-memory columns = all 512)
static_assert(sizeof(Smem) + 1024 > 228 * 1024 / 3, "shared memory keeps tensor memory within one SM");
static_assert(2 * (sizeof(Smem) + 1024) <= 228 * 1024, "two CTAs per SM");

struct TcArgs {
  BinGrid G;
  const double2 *__restrict__ pay;      // [n][4] bin-order payload (x, y | z, q | ...)
  const uint32_t *__restrict__ starts;  // [nbins + 1]
  const uint32_t *__restrict__ tile_starts;  // [tiles + 1] into tile_rows
  const uint32_t *__restrict__ tile_rows;    // position of each tile row
  const double *__restrict__ tile_boxes; // [tiles][6]: centre xyz, half extent xyz
  const uint4 *__restrict__ tile_ops;   // [tiles][256] position operands
  const uint4 *__restrict__ wdig;       // [tiles][128] weight digits
  const uint4 *__restrict__ cdig;       // [n] charge digits, bin order
  // [n] bin order: position relative to the particle's bin origin (FP32)
  // and the bin's x index (as a float: exact)
  const float4 *__restrict__ cpos;
  const uint32_t *__restrict__ order;   // launch order of the tiles (or NULL)
  double radius, inv_radius;
  unsigned long long *__restrict__ norm_hi, *__restrict__ norm_lo;  // [n], bin order
  uint32_t *__restrict__ hits;                                      // [n], bin order
  const double *__restrict__ out_scale;  // [4]: rho, jx, jy, jz factors
  double *__restrict__ vals;             // [4][npos]
  double *__restrict__ sums;             // [16][npos] digit sums instead of vals (or NULL)
  long long npos;
  unsigned long long *__restrict__ counters;  // [0]: candidates over all tiles
  DevStatus *st;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// tcgen05 shared-memory matrix descriptor, no swizzle
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of this architecture
  return d;
}

__device__ __forceinline__ void mma_f16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                        uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

// The sums of one chunk: 16 int8 MMAs (K = 32 each) with A in tensor memory
// (K-major: each 32-bit column holds four consecutive K elements) at columns
// a0, a0 + 8, ... and B described by desc0, desc0 + 32 (512 bytes
// further), ...; the first accumulates only if acc != 0, the rest always.
// One statement, so the 16 issue back to back.
__device__ __forceinline__ void mma_sums16(uint32_t d, uint32_t a0, uint64_t desc0,
                                           uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t.reg .b64 d;\n\t.reg .b32 a;\n\t"
      "setp.ne.b32 p, %3, 0;\n\tsetp.eq.b32 q, 0, 0;\n\t"
      "mov.b64 d, %1;\n\tmov.b32 a, %2;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, p;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "add.s64 d, d, 32;\n\tadd.u32 a, a, 8;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [a], d, %4, q;\n\t"
      "}\n"
      ::"r"(d), "l"(desc0), "r"(a0), "r"(acc), "r"(idesc)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
      : "memory");
}

// Bounded wait for the phase of `parity`. Each try_wait may suspend the
// thread until the phase completes, for at most WAIT_NS, so waiting warps
// take no issue slots; false after WAIT_TRIES tries (about one second).
constexpr unsigned WAIT_NS = 1000000;
constexpr unsigned WAIT_TRIES = 1024;
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (unsigned k = 0; k < WAIT_TRIES; ++k) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(WAIT_NS)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t addr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(addr)
      : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t addr, uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(addr)
      : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_st32(uint32_t addr, const uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
      "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, "
      "%17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};\n" ::"r"(
          addr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
      "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]),
      "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]),
      "r"(r[29]), "r"(r[30]), "r"(r[31])
      : "memory");
}

__device__ __forceinline__ void tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// FP32 -> (high, low) FP16 terms
__device__ __forceinline__ void split_half(float x, __half &h, __half &l) {
  h = __float2half_rn(x);
  l = __float2half_rn(x - __half2float(h));
}

__device__ __forceinline__ uint32_t pack2(__half a, __half b) {
  return (uint32_t)__half_as_ushort(a) | ((uint32_t)__half_as_ushort(b) << 16);
}

// The candidate operand of a particle at w (relative to the tile centre, in
// units of the radius), K = 16 halves:
//   [vx_h, vx_l, vx_h, vy_h, vy_l, vy_h, vz_h, vz_l, vz_h, 1, 1, g_h, g_l, 0, 0, 0]
// with v = 2 SIGMA w and g = -SIGMA |w|^2; the position operand is
//   [ux_h, ux_h, ux_l, uy_h, uy_h, uy_l, uz_h, uz_h, uz_l, b_h, b_l, 1, 1, 0, 0, 0]
// with b = SIGMA (1 - |u|^2), so the product is
//   u.v + b + g = SIGMA (1 - |u - w|^2) (up to the dropped low x low terms).
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
  return d;
}

__device__ __forceinline__ uint32_t h2bits(__half2 v) {
  uint32_t u;
  memcpy(&u, &v, sizeof(u));
  return u;
}

__device__ __forceinline__ void candidate_operand(float w0, float w1, float w2, uint4 &k0,
                                                  uint4 &k1) {
  const float v0 = 2.0f * SIGMA * w0, v1 = 2.0f * SIGMA * w1, v2 = 2.0f * SIGMA * w2;
  const float g = -SIGMA * fmaf(w0, w0, fmaf(w1, w1, w2 * w2));
  // high FP16 terms of (v0, v1) and (v2, g) in pairs, then the low terms of
  // the remainders (each value rounded to nearest, as one at a time)
  const __half2 h01 = __floats2half2_rn(v0, v1), h2g = __floats2half2_rn(v2, g);
  const float2 f01 = __half22float2(h01), f2g = __half22float2(h2g);
  const uint32_t H01 = h2bits(h01), H2G = h2bits(h2g);
  const uint32_t L01 = h2bits(__floats2half2_rn(v0 - f01.x, v1 - f01.y));
  const uint32_t L2G = h2bits(__floats2half2_rn(v2 - f2g.x, g - f2g.y));
  const uint32_t ONE = 0x3C00u;  // FP16 1.0
  // [h0 l0 | h0 h1 | l1 h1 | h2 l2], [h2 1 | 1 gh | gl 0 | 0 0]
  k0 = make_uint4(prmt(H01, L01, 0x5410), H01, prmt(L01, H01, 0x7632), prmt(H2G, L2G, 0x5410));
  k1 = make_uint4((H2G & 0xffffu) | (ONE << 16), ONE | (H2G & 0xffff0000u), L2G >> 16, 0u);
}

// Bin-row segments of a tile (warp 0): every run of bins along x, in the
// rows (bz, by) within the radius of the box [c - hf, c + hf], as ranges of
// bin-order particles with the origin of the run's first bin relative to the
// tile centre (periodic image included, FP64 rounded once to FP32: within
// 2.5 radii, so to ~2e-7 radii); the stream of candidates is the
// concatenation of the segments.
__device__ void build_segments(Smem &S, const TcArgs &A, const double c[3], const double hf[3],
                               int lane) {
  const BinGrid &G = A.G;
  const double rr = A.radius * (1 + 1e-5), rr2 = rr * rr;
  int ulo[3], uhi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    ulo[d] = bin_floor(G, d, c[d] - hf[d] - A.radius);
    uhi[d] = bin_floor(G, d, c[d] + hf[d] + A.radius);
    if (G.periodic[d]) {
      ulo[d] -= 1;
      uhi[d] += 1;
    } else {
      ulo[d] = max(ulo[d], 0);
      uhi[d] = min(uhi[d], G.dims[d] - 1);
    }
  }
  auto slab_gap = [&](int d, double blo) {
    const double e =
        fmax(0.0, fmax(blo - (c[d] + hf[d]), (c[d] - hf[d]) - (blo + G.w[d]))) - G.slack[d];
    return e > 0 ? e * e : 0.0;
  };
  const int ny = max(0, uhi[1] - ulo[1] + 1), nz = max(0, uhi[2] - ulo[2] + 1);
  const int nrows = ny * nz;
  int nseg = 0;
  bool overflow = false;
  for (int r0 = 0; r0 < nrows; r0 += 32) {
    const int r = r0 + lane;
    uint32_t s_start[3], s_len[3];
    float s_ox[3], s_bx[3], oy = 0, oz = 0;
    int cnt = 0;
    if (r < nrows) {
      const int bz = ulo[2] + r / ny, by = ulo[1] + r % ny;
      int wz = bz, qz = 0, wy = by, qy = 0;
      if (G.periodic[2]) {
        qz = floor_div(bz, G.dims[2]);
        wz = bz - qz * G.dims[2];
      }
      if (G.periodic[1]) {
        qy = floor_div(by, G.dims[1]);
        wy = by - qy * G.dims[1];
      }
      const double dyz2 = slab_gap(2, G.origin[2] + bz * G.w[2]) +
                          slab_gap(1, G.origin[1] + by * G.w[1]);
      if (dyz2 <= rr2) {
        const double rem = sqrt(rr2 - dyz2);
        int bx0 = bin_floor(G, 0, c[0] - hf[0] - rem);
        int bx1 = bin_floor(G, 0, c[0] + hf[0] + rem);
        if (G.periodic[0]) {
          bx0 -= 1;
          bx1 += 1;
        }
        bx0 = max(bx0, ulo[0]);
        bx1 = min(bx1, uhi[0]);
        const long long row = (long long)G.dims[0] * (wy + (long long)G.dims[1] * wz);
        oy = (float)(G.origin[1] + wy * G.w[1] + qy * G.period[1] - c[1]);
        oz = (float)(G.origin[2] + wz * G.w[2] + qz * G.period[2] - c[2]);
        int bx = bx0;
        while (bx <= bx1) {
          int wx = bx, qx = 0, seg_end = bx1;
          if (G.periodic[0]) {
            qx = floor_div(bx, G.dims[0]);
            wx = bx - qx * G.dims[0];
            seg_end = min(bx1, (qx + 1) * G.dims[0] - 1);
          }
          const uint32_t s0 = A.starts[row + wx];
          const uint32_t s1 = A.starts[row + wx + (seg_end - bx) + 1];
          bx = seg_end + 1;
          if (s1 > s0) {
            if (cnt < 3) {
              s_start[cnt] = s0;
              s_len[cnt] = s1 - s0;
              s_ox[cnt] = (float)(G.origin[0] + wx * G.w[0] + qx * G.period[0] - c[0]);
              s_bx[cnt] = (float)wx;
              ++cnt;
            } else {
              overflow = true;
            }
          }
        }
      }
    }
    // exclusive warp scan of the segment counts
    int cs = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int c2 = __shfl_up_sync(0xffffffffu, cs, o);
      if (lane >= o) cs += c2;
    }
    const int sbase = nseg + cs - cnt;
    for (int i = 0; i < cnt; ++i) {
      if (sbase + i < MAXSEG) {
        S.seg_sl[sbase + i] = make_uint2(s_start[i], s_len[i]);
        S.seg_o[sbase + i] = make_float4(s_ox[i], oy, oz, s_bx[i]);
      }
    }
    nseg += __shfl_sync(0xffffffffu, cs, 31);
  }
  overflow = __any_sync(0xffffffffu, overflow) || nseg > MAXSEG;
  if (lane == 0) {
    S.nseg = overflow ? 0 : nseg;
    if (overflow) {
      S.abort = 1;
      record_error(A.st, PRT_ERR_CAPACITY, -1);
    }
  }
}

// A warp's place in its tile's candidate stream: the warp stages the
// segments warp, warp + FILL_WARPS, ... of the tile, 32 particles (a batch) at a time,
// with three batches loaded ahead, each in its own registers (a batch's
// values are read only when it is processed, then the set is refilled).
struct Batch {
  int seg;       // seg < 0: none
  int n;         // particles of the batch (lanes 0 .. n-1)
  uint32_t k0;   // bin-order index of lane 0's particle
  float4 pos;    // the lane's particle: offset from its bin origin, bin x index
  uint4 dig;     // its charge digits (deposition pass)
};

struct Cursor {
  int cseg, coff;  // the next batch to load
  int nseg;        // segments of the tile
  int rot;         // the set that holds the oldest loaded batch
  Batch q0, q1, q2;
};

template <bool NORM>
__device__ __forceinline__ void next_batch(const Smem &S, const TcArgs &A, Cursor &C, Batch &B,
                                           int lane) {
  B.seg = C.cseg < C.nseg ? C.cseg : -1;
  if (B.seg < 0) return;
  const uint2 sl = S.seg_sl[B.seg];
  B.n = (int)sl.y - C.coff;
  B.k0 = sl.x + (uint32_t)C.coff;
  if (lane < B.n) {
    const size_t k = (size_t)B.k0 + lane;
    B.pos = A.cpos[k];
    if (!NORM) B.dig = A.cdig[k];
  }
  C.coff += 32;
  if (C.coff >= (int)sl.y) {
    C.coff = 0;
    C.cseg += FILL_WARPS;
  }
}

template <bool NORM>
__device__ __forceinline__ void cursor_init(const Smem &S, const TcArgs &A, Cursor &C, int warp,
                                            int lane) {
  C.cseg = warp;
  C.coff = 0;
  C.nseg = S.nseg;
  C.rot = 0;
  C.q0.pos = C.q1.pos = C.q2.pos = make_float4(0, 0, 0, 0);
  C.q0.dig = C.q1.dig = C.q2.dig = make_uint4(0, 0, 0, 0);
  next_batch<NORM>(S, A, C, C.q0, lane);
  next_batch<NORM>(S, A, C, C.q1, lane);
  next_batch<NORM>(S, A, C, C.q2, lane);
}

// Stages candidates into the ring until it holds `target` slots or every
// warp's segments are exhausted (every fill warp; at most 32 slots per warp
// past the target, so the ring holds at most target + 223).
// The fill's per-tile constants: the cull box's half extents and squared
// diameter (radius grown by 1e-5), 1/a and the bin width along x in FP32.
struct FillConst {
  float hf[3], rc4, inv_a, bw;
};

template <bool NORM>
__device__ __forceinline__ void fill(Smem &S, const TcArgs &A, const FillConst &F, int target,
                                     int lane, Cursor &C) {
  const float *hf = F.hf;
  const float rc4 = F.rc4, inv_a = F.inv_a, bw = F.bw;
  // culls batch B into the ring, then refills B with the warp's next batch
  auto process = [&](Batch &B) {
    const bool valid = lane < B.n;
    const uint32_t k = B.k0 + (uint32_t)lane;
    // the particle relative to the tile centre: its segment's first bin
    // origin, whole bins along x to its own bin, its offset in the bin
    const float4 o = S.seg_o[B.seg];
    bool in = false;
    float w0 = 0, w1 = 0, w2 = 0;
    if (valid) {
      w0 = fmaf(B.pos.w - o.w, bw, o.x) + B.pos.x;
      w1 = o.y + B.pos.y;
      w2 = o.z + B.pos.z;
      // rounded-box cull: per axis 2 max(|w| - half, 0) = d + |d|
      const float d0 = fabsf(w0) - hf[0], d1 = fabsf(w1) - hf[1], d2 = fabsf(w2) - hf[2];
      const float e0 = d0 + fabsf(d0), e1 = d1 + fabsf(d1), e2 = d2 + fabsf(d2);
      in = e0 * e0 + e1 * e1 + e2 * e2 <= rc4;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, in);
    int base = 0;
    if (lane == 0 && bal) base = atomicAdd(&S.tail, __popc(bal));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (in) {
      const int slot = (base + __popc(bal & ((1u << lane) - 1u))) % RING;
      uint4 k0, k1;
      candidate_operand(w0 * inv_a, w1 * inv_a, w2 * inv_a, k0, k1);
      *reinterpret_cast<uint4 *>(S.bcand + (size_t)slot * 16) = k0;
      *reinterpret_cast<uint4 *>(S.bcand + (size_t)(RING + slot) * 16) = k1;
      if (NORM)
        S.n.slot_id[slot] = k;
      else
        *reinterpret_cast<uint4 *>(S.zdig + (size_t)(4 * slot + 3) * 16) = B.dig;
    }
    next_batch<NORM>(S, A, C, B, lane);
  };
  for (;;) {
    const int tail = __shfl_sync(0xffffffffu, *(volatile int *)&S.tail, 0);
    const int bseg = C.rot == 0 ? C.q0.seg : C.rot == 1 ? C.q1.seg : C.q2.seg;
    if (tail >= target || bseg < 0) break;
    if (C.rot == 0)
      process(C.q0);
    else if (C.rot == 1)
      process(C.q1);
    else
      process(C.q2);
    C.rot = C.rot == 2 ? 0 : C.rot + 1;
  }
}

// Zeroes the candidate operands of slots [from, to) of a ring chunk (the
// tail of the last chunk): a zero operand gives score 0, weight 0, so the
// slots' digit rows (stale) are multiplied by zero.
__device__ __forceinline__ void pad_chunk(Smem &S, int from, int to, int tid) {
  for (int i = from + tid; i < to; i += THREADS) {
    const int slot = i % RING;
    *reinterpret_cast<uint4 *>(S.bcand + (size_t)slot * 16) = make_uint4(0, 0, 0, 0);
    *reinterpret_cast<uint4 *>(S.bcand + (size_t)(RING + slot) * 16) = make_uint4(0, 0, 0, 0);
  }
}

// The weights of one chunk, in place in tensor memory: thread (warp w, lane
// l) takes row 32 (w % 4) + l (a position in the deposition pass, a
// candidate in the normalisation pass) and columns 64 (w / 4) .. + 63, reads
// the scores s (tcgen05.ld), and writes back the words F + 2^23 with
// F = round(t^2), t = s + |s| (one FMA: t t + 2^23 puts the rounded integer
// in the low mantissa bits), so bytes 0-2 are F's base-256 digits and byte 3
// a constant the sums multiply by zero. Counts the words with F > 0 (hits).
template <bool HITS>
__device__ __forceinline__ uint32_t weights(uint32_t tmem, int warp, int lane) {
  const uint32_t base = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(64 * (warp >> 2));
  float hits = 0;  // below 65: exact
#pragma unroll 1
  for (int half = 0; half < 2; ++half) {
    uint32_t r[32];
    tmem_ld32(base + 32 * half, r);
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      const float sc = __uint_as_float(r[i]);
      const float t = sc + fabsf(sc);                        // 2 max(s, 0), exact
      const float f = fmaf(t, t, 8388608.0f);                // 2^23 + round(t^2)
      r[i] = __float_as_uint(f);
      if (HITS) hits += __saturatef(f - 8388608.0f);         // F > 0: 1, else 0
    }
    tmem_st32(base + 32 * half, r);
  }
  tmem_wait_st();
  return (uint32_t)hits;
}

// Instruction descriptors (M = 128):
//  score: D FP32, A/B FP16, both K-major, N = 128
constexpr uint32_t IDESC_SCORE =
    (1u << 4) | ((uint32_t)(NC >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
//  sums: D S32, A U8 K-major in tensor memory (the weight words, rows =
//  positions or candidates), B S8 MN-major (digit rows), N = 48 (three
//  views of the digit rows: weight bytes 2, 1, 0)
constexpr uint32_t IDESC_SUMS = (2u << 4) | (1u << 10) | (1u << 16) | (6u << 17) | (8u << 24);

// rho, j of a position from its digit sums T (T_i = sum_p F c_i over the
// particles, c_i the i-th digit column): charge = sum_i T_i 256^i over the
// six charge digits, each current component over its three, times the
// output scales. One formula for the fused epilogue and for the combination
// of summed partial results, so both give the same bits.
__device__ __forceinline__ void combine_position(const double T[16],
                                                 const double *__restrict__ scale,
                                                 double out[4]) {
  double r = T[CDIG - 1];
#pragma unroll
  for (int i = CDIG - 2; i >= 0; --i) r = fma(r, 256.0, T[i]);
  out[0] = r * scale[0];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int b = CDIG + JDIG * d;
    out[1 + d] = fma(fma(T[b + 2], 256.0, T[b + 1]), 256.0, T[b]) * scale[1 + d];
  }
}

template <bool NORM, bool IND>
__global__ void __launch_bounds__(THREADS, 2) tc_deposit_kernel(TcArgs A) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  Smem &S = *reinterpret_cast<Smem *>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long tile = A.order ? (long long)A.order[blockIdx.x] : (long long)blockIdx.x;
  const uint32_t p0 = A.tile_starts[tile];
  const int npt = (int)(A.tile_starts[tile + 1] - p0);
  double c[3], hfd[3];
  FillConst fc;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    c[d] = A.tile_boxes[6 * tile + d];
    hfd[d] = A.tile_boxes[6 * tile + 3 + d] + 1e-5 * A.radius;
    fc.hf[d] = (float)hfd[d];
  }
  {
    const float rcf = (float)(A.radius * (1 + 1e-5));
    fc.rc4 = 4.0f * rcf * rcf;
    fc.inv_a = (float)A.inv_radius;
    fc.bw = (float)A.G.w[0];
  }

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&S.tmem)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.bar_s)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.bar_a)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    S.tail = 0;
    S.abort = 0;
  }
  {
    const uint4 *src = A.tile_ops + (size_t)tile * 256;
    for (int i = tid; i < 256; i += THREADS) reinterpret_cast<uint4 *>(S.apos)[i] = src[i];
    // the digit rows: zeros, then (normalisation) each position's weight
    // digits in its row 4 u + 3
    uint4 *z = reinterpret_cast<uint4 *>(NORM ? S.n.zw : S.zdig);
    const int zrows = NORM ? 4 * TM + 3 : 4 * RING + 3;
    for (int i = tid; i < zrows; i += THREADS) z[i] = make_uint4(0, 0, 0, 0);
    if (NORM) {
      __syncthreads();
      const uint4 *ws = A.wdig + (size_t)tile * 128;
      for (int i = tid; i < 128; i += THREADS) z[4 * i + 3] = ws[i];
    }
  }
  __syncthreads();
  if (warp == 0) build_segments(S, A, c, hfd, lane);
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = S.tmem;
  const uint32_t bar_s = smem_u32(&S.bar_s), bar_a = smem_u32(&S.bar_a);
  const uint32_t a_pos = smem_u32(S.apos), b_cand = smem_u32(S.bcand);
  const uint32_t z_dig = smem_u32(NORM ? S.n.zw : S.zdig);
  // the scores of the chunk at ring slot `slot`: rows = positions
  // (deposition) or candidates (normalisation), the same products either way
  auto score_mma = [&](int slot) {
    const uint64_t dp = sdesc(a_pos, TM * 16, 128);
    const uint64_t dc = sdesc(b_cand + (uint32_t)(slot * 16), RING * 16, 128);
    mma_f16(tmem, NORM ? dc : dp, NORM ? dp : dc, IDESC_SCORE, 0);
  };

  // per thread: position row 32 (warp % 4) + lane, digit columns
  // 8 (warp / 4) .. + 7 of the deposition's sums over the weight digits
  // (FP64, exact integers, across int32 windows)
  double acc[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) acc[i] = 0;

  bool ok = S.abort == 0;
  int issued_s = 0, issued_a = 0, waited_s = 0, waited_a = 0;
  Cursor cur;
  if (warp < FILL_WARPS) {
    cursor_init<NORM>(S, A, cur, warp, lane);
  } else {
    cur.q0.seg = cur.q1.seg = cur.q2.seg = -1;
    cur.rot = 0;
  }
  int valid = 0;

  // readout of a normalisation chunk: per candidate its sum over the tile,
  // P = H 2^40 + L (0 <= L < 2^40), both parts added exactly to the
  // particle's integral (H modulo 2^64): warps 0-3 add H, warps 4-7 add L
  // and the hit count (a warp reads the tensor-memory lanes 32 (warp % 4) ..)
  auto norm_readout = [&](int chunk, int nvalid) {
    uint32_t d2[8], d1[8], d0[8];
    const uint32_t lane_addr = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    tmem_ld8(lane_addr + COL_ACC, d2);
    tmem_ld8(lane_addr + COL_ACC + 16, d1);
    tmem_ld8(lane_addr + COL_ACC + 32, d0);
    tmem_wait_ld();
    const int cr = 32 * (warp & 3) + lane;
    if (cr < nvalid) {
      // P = sum_kk 256^kk (65536 D2 + 256 D1 + D0) over the six W digits kk
      // = sum_j 256^j X_j with X_j = D0_j + D1_(j-1) + D2_(j-2) (|X| < 2^24,
      // int32) = Plo + 2^32 Phi (Plo, Phi: four X each, |.| < 2^48)
      int X[8];
#pragma unroll
      for (int j = 0; j < 8; ++j)
        X[j] = (j <= 5 ? (int)d0[j] : 0) + (j >= 1 && j <= 6 ? (int)d1[j - 1] : 0) +
               (j >= 2 ? (int)d2[j - 2] : 0);
      const long long plo =
          (long long)X[0] + 256ll * X[1] + 65536ll * X[2] + 16777216ll * X[3];
      const long long phi =
          (long long)X[4] + 256ll * X[5] + 65536ll * X[6] + 16777216ll * X[7];
      const long long M40 = (1ll << 40) - 1;
      const long long l1 = (plo & M40) + ((phi & 0xff) << 32);  // < 2^41
      const long long L = l1 & M40;
      const long long H = (plo >> 40) + (phi >> 8) + (l1 >> 40);
      const uint32_t id = S.n.slot_id[(chunk * NC + cr) % RING];
      if (warp < 4) {
        if (H != 0) atomicAdd(A.norm_hi + id, (unsigned long long)H);
      } else {
        if (L != 0) atomicAdd(A.norm_lo + id, (unsigned long long)L);
        if (IND) {
          const uint32_t h = S.n.hits[chunk & 1][0][cr] + S.n.hits[chunk & 1][1][cr];
          if (h) atomicAdd(A.hits + id, h);
        }
      }
    }
  };
  // deposition accumulators -> FP64: per digit column the exact integer
  // 65536 D2 + 256 D1 + D0 (below 2^53)
  auto dep_fold = [&]() {
    uint32_t d2[8], d1[8], d0[8];
    const uint32_t base = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + COL_ACC + 8 * (warp >> 2);
    tmem_ld8(base, d2);
    tmem_ld8(base + 16, d1);
    tmem_ld8(base + 32, d0);
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 8; ++i)
      acc[i] += (double)(65536ll * (int)d2[i] + 256ll * (int)d1[i] + (int)d0[i]);
  };
  auto wait_a = [&]() {
    const bool w = mbar_wait(bar_a, (uint32_t)(waited_a & 1));
    if (w) ++waited_a;
    return __syncthreads_and(w) != 0;
  };
  const bool issuer = warp == ISSUE_WARP && lane == 0;

  int window = 0;       // chunks in the current int32 deposition window
  int chunks = 0;       // chunks whose sums were issued
  int valid_prev = 0;   // valid slots of the chunk whose accumulation is in flight
  if (ok) {
    if (warp < FILL_WARPS) fill<NORM>(S, A, fc, NC, lane, cur);
    __syncthreads();
    valid = min(S.tail, NC);
    if (valid > 0 && valid < NC) pad_chunk(S, valid, NC, tid);
    fence_async_smem();
    fence_before();
    __syncthreads();
    if (valid > 0 && issuer) {
      fence_after();
      score_mma(0);
      mma_commit(bar_s);
    }
    if (valid > 0) ++issued_s;
  }
  // One CTA barrier per chunk: every thread waits for the tensor cores itself
  // (bounded), and the barrier after the weights joins the fill of chunk
  // k+1, the weights of chunk k and the waits' outcomes.
  for (int k = 0; ok && valid > 0; ++k) {
    // (1) the fill warps stage chunk k+1 while the tensor cores score chunk
    // k and sum chunk k-1: the fill writes slots of chunks k+1 .. k+3 (at
    // most 223 past chunk k+1), never those of chunk k-1 (ring of five)
    if (warp < FILL_WARPS) fill<NORM>(S, A, fc, (k + 2) * NC, lane, cur);
    // (2) the scores of chunk k are ready, and with them the sums of chunk
    // k-1 (the commit that signals the scores covers every MMA the issuing
    // thread issued before them): read the normalisation sums, or fold a
    // full window
    bool w = mbar_wait(bar_s, (uint32_t)(waited_s & 1));
    if (w) {
      ++waited_s;
      fence_after();
      if (k > 0) {
        if (NORM) {
          norm_readout(k - 1, valid_prev);
        } else if (window == FLUSH_CHUNKS) {
          dep_fold();
          window = 0;
        }
      }
      // (3) the weights of chunk k
      {
        const uint32_t h = weights<NORM && IND>(tmem, warp, lane);
        // the hits of this thread's candidate among its 64 positions, added
        // to the particle with the readout
        if (NORM && IND) S.n.hits[k & 1][warp >> 2][32 * (warp & 3) + lane] = h;
      }
    }
    fence_async_smem();
    fence_before();
    ok = __syncthreads_and(w) != 0;
    if (!ok) break;
    const int valid_next = min(max(S.tail - (k + 1) * NC, 0), NC);
    if (valid_next > 0 && valid_next < NC) {
      // the stream ends inside chunk k+1: zero its remaining slots
      pad_chunk(S, (k + 1) * NC + valid_next, (k + 2) * NC, tid);
      fence_async_smem();
      __syncthreads();
    }
    // (4) the sums of chunk k, then the scores of chunk k+1 (the issue warp;
    // the fill warps go on to chunk k+2). The sums read chunk k's weight
    // words from the tensor-memory columns the next scores overwrite: the
    // MMAs of one thread run in issue order.
    if (issuer) {
      fence_after();
      const int slot0 = (k * NC) % RING;
      const uint32_t zb = z_dig + (NORM ? 0u : (uint32_t)(64 * slot0));
      static_assert(NC / 8 == 16, "sixteen K steps per chunk");
      mma_sums16(tmem + COL_ACC, tmem, sdesc(zb + 16u, 128, 16), IDESC_SUMS,
                 (!NORM && window > 0) ? 1u : 0u);
      if (valid_next > 0) {
        const int slot1 = ((k + 1) * NC) % RING;
        score_mma(slot1);
        mma_commit(bar_s);
      } else {
        mma_commit(bar_a);  // the last chunk's sums
      }
    }
    if (valid_next > 0)
      ++issued_s;
    else
      ++issued_a;
    ++chunks;
    ++window;
    valid_prev = valid;
    valid = valid_next;
  }
  // the last chunk's sums
  if (ok && issued_a > waited_a) {
    ok = wait_a();
    if (ok) {
      fence_after();
      if (NORM)
        norm_readout(chunks - 1, valid_prev);
      else
        dep_fold();
    }
  }
  if (!ok) {
    // a wait ran out: record it, let the issued MMAs finish (bounded), stop
    if (tid == 0 && S.abort == 0) record_error(A.st, PRT_ERR_TIMEOUT, tile);
    while (waited_s < issued_s) {
      mbar_wait(bar_s, (uint32_t)(waited_s & 1));
      ++waited_s;
    }
    while (waited_a < issued_a) {
      mbar_wait(bar_a, (uint32_t)(waited_a & 1));
      ++waited_a;
    }
  } else {
    if (tid == 0) atomicAdd(A.counters, (unsigned long long)S.tail);
    if (!NORM) {
      // per position the 16 digit sums T_i (exact integers), then the charge
      // (six digits) and current (three digits per component)
      double(*tsum)[16] = S.tsum;
      const int row = 32 * (warp & 3) + lane;
#pragma unroll
      for (int i = 0; i < 8; ++i) tsum[row][8 * (warp >> 2) + i] = acc[i];
      __syncthreads();
      if (warp < 4 && row < npt) {
        double T[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) T[i] = tsum[row][i];
        const long long u = A.tile_rows[p0 + row];
        if (A.sums) {
#pragma unroll
          for (int i = 0; i < 16; ++i) A.sums[i * A.npos + u] = T[i];
        } else {
          double o[4];
          combine_position(T, A.out_scale, o);
#pragma unroll
          for (int d = 0; d < 4; ++d) A.vals[d * A.npos + u] = o[d];
        }
      }
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS)
                 : "memory");
  }
}

// ------------------------------------------------------------ preparation

// The candidates' compact positions (bin order): the offset from the
// particle's bin origin in FP32 (below a bin width: exact to ~1e-7 of it) and
// the bin's x index (a float, exact).
__global__ void candidate_positions_kernel(long long n, const uint32_t *__restrict__ perm,
                                           const double *__restrict__ x, BinGrid G,
                                           float4 *__restrict__ out) {
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t i = perm[s];
  float d[3];
  int b0 = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double xa = x[a * n + i];
    const int b = bin_coord(G, a, xa);
    d[a] = (float)(xa - (G.origin[a] + b * G.w[a]));
    if (a == 0) b0 = b;
  }
  out[s] = make_float4(d[0], d[1], d[2], (float)b0);
}

// Position operands of every tile, K-major: row u of tile t at
// [t][K chunk][u][16 B] (rows past the tile's positions are zero).
__global__ void tile_operands_kernel(long long tiles, const uint32_t *__restrict__ tile_starts,
                                     const uint32_t *__restrict__ tile_rows,
                                     const double *__restrict__ tile_boxes,
                                     const double *__restrict__ pos, double inv_radius,
                                     uint4 *__restrict__ out) {
  const long long t = blockIdx.x;
  const int u = threadIdx.x;
  if (t >= tiles) return;
  const uint32_t p0 = tile_starts[t];
  const int npt = (int)(tile_starts[t + 1] - p0);
  uint4 k0 = make_uint4(0, 0, 0, 0), k1 = make_uint4(0, 0, 0, 0);
  if (u < npt) {
    const long long p = tile_rows[p0 + u];
    const double ux = (pos[3 * p] - tile_boxes[6 * t]) * inv_radius;
    const double uy = (pos[3 * p + 1] - tile_boxes[6 * t + 1]) * inv_radius;
    const double uz = (pos[3 * p + 2] - tile_boxes[6 * t + 2]) * inv_radius;
    const double b = (double)SIGMA * (1.0 - (ux * ux + uy * uy + uz * uz));
    __half xh, xl, yh, yl, zh, zl, bh, bl;
    split_half((float)ux, xh, xl);
    split_half((float)uy, yh, yl);
    split_half((float)uz, zh, zl);
    split_half((float)b, bh, bl);
    const __half one = __float2half_rn(1.0f), zero = __float2half_rn(0.0f);
    k0 = make_uint4(pack2(xh, xh), pack2(xl, yh), pack2(yh, yl), pack2(zh, zh));
    k1 = make_uint4(pack2(zl, bh), pack2(bl, one), pack2(one, zero), pack2(zero, zero));
  }
  out[256 * t + u] = k0;
  out[256 * t + 128 + u] = k1;
}

__device__ __forceinline__ void atomic_max_abs(unsigned long long *m, double v) {
  atomicMax(m, (unsigned long long)__double_as_longlong(fabs(v)));
}

__global__ void max_abs_kernel(long long n, const double *__restrict__ v,
                               unsigned long long *__restrict__ m) {
  double a = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    a = fmax(a, fabs(v[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
  if ((threadIdx.x & 31) == 0 && a > 0) atomic_max_abs(m, a);
}

// exponent E with |v| 2^E < 2^bits for every |v| <= m
__device__ __forceinline__ int scale_exponent(unsigned long long mbits, int bits) {
  const double m = __longlong_as_double((long long)mbits);
  if (!(m > 0)) return 0;
  int e;
  frexp(m, &e);  // m < 2^e
  return bits - e;
}

// Scales of one call (device): out[0..3] the factors of rho, jx, jy, jz;
// integral the factor of the normalising sums; ex[0..4] the digit
// exponents of c, c vx, c vy, c vz, W.
struct TcScales {
  double out[4];
  double integral;
  int ex[5];
};

__global__ void weight_scale_kernel(const unsigned long long *__restrict__ mbits, double kappa,
                                    TcScales *sc) {
  const int e = scale_exponent(mbits[4], 46);
  sc->ex[4] = e;
  sc->integral = kappa * ldexp(1.0, -e);
}

// (the maxima are given as the bit patterns of non-negative doubles, which
// order like the doubles themselves)
__global__ void charge_scale_kernel(const unsigned long long *__restrict__ mbits, double kappa,
                                    TcScales *sc) {
  const int e0 = scale_exponent(mbits[0], 46);
  sc->ex[0] = e0;
  sc->out[0] = kappa * ldexp(1.0, -e0);
  for (int d = 1; d < 4; ++d) {
    const int e = scale_exponent(mbits[d], 22);
    sc->ex[d] = e;
    sc->out[d] = kappa * ldexp(1.0, -e);
  }
}

// Balanced signed base-256 digits (each in [-128, 127]) of X.
__device__ __forceinline__ void balanced_digits(long long X, int nd, uint8_t *out) {
  for (int i = 0; i < nd; ++i) {
    const int d = (int)(int8_t)(uint8_t)(X & 0xff);
    out[i] = (uint8_t)(int8_t)d;
    X = (X - d) >> 8;
  }
}

__device__ __forceinline__ uint4 pack16(const uint8_t b[16]) {
  uint32_t w[4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
    w[i] = (uint32_t)b[4 * i] | ((uint32_t)b[4 * i + 1] << 8) | ((uint32_t)b[4 * i + 2] << 16) |
           ((uint32_t)b[4 * i + 3] << 24);
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// Position weight digits: W 2^E (|W 2^E| < 2^46) in six balanced signed
// base-256 digits (columns 0-5), a one in column 6 (the indicator sum), per
// tile row.
__global__ void weight_digits_kernel(long long tiles, const uint32_t *__restrict__ tile_starts,
                                     const uint32_t *__restrict__ tile_rows,
                                     const double *__restrict__ W, const TcScales *sc,
                                     uint4 *__restrict__ out) {
  const long long t = blockIdx.x;
  const int u = threadIdx.x;
  if (t >= tiles) return;
  const uint32_t p0 = tile_starts[t];
  const int npt = (int)(tile_starts[t + 1] - p0);
  uint8_t b[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) b[i] = 0;
  if (u < npt) {
    balanced_digits(llrint(ldexp(W[tile_rows[p0 + u]], sc->ex[4])), WDIG, b);
    b[WDIG] = 1;
  }
  out[128 * t + u] = pack16(b);
}

// Per particle (bin order) the deposited charge c and c v: c = q (plain), or
// q / integral with the integral from the exact sums of the normalisation
// pass; the scale and hit count feed the statistics.
template <bool NORM>
__global__ void charges_kernel(long long n, const uint32_t *__restrict__ n_live,
                               const double2 *__restrict__ pay,
                               const unsigned long long *__restrict__ hi,
                               const unsigned long long *__restrict__ lo,
                               const uint32_t *__restrict__ hits, const TcScales *sc,
                               const uint32_t *__restrict__ perm, double *__restrict__ cv,
                               double *__restrict__ scale_out, double *__restrict__ hits_out,
                               unsigned long long *__restrict__ mbits, DevStatus *st) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double v[4] = {0, 0, 0, 0};
  if (k < n) {
    if (k < (long long)*n_live) {
      const double q = pay[4 * k + 1].y;
      const double2 j01 = pay[4 * k + 2], j2 = pay[4 * k + 3];
      if (NORM) {
        const double integral =
            fma((double)(long long)hi[k], 1099511627776.0, (double)lo[k]) * sc->integral;
        if (integral != 0) {
          const double f = 1.0 / integral;
          v[0] = q * f;
          v[1] = j01.x * f;
          v[2] = j01.y * f;
          v[3] = j2.x * f;
        } else {
          record_warning(st, PRT_WARN_ZERO_MASS, perm ? (long long)perm[k] : k);
        }
        scale_out[k] = v[0];
        hits_out[k] = hits ? (double)hits[k] : 0.0;
      } else {
        v[0] = q;
        v[1] = j01.x;
        v[2] = j01.y;
        v[3] = j2.x;
      }
    } else if (NORM) {
      scale_out[k] = 0;
      hits_out[k] = -1;
    }
#pragma unroll
    for (int d = 0; d < 4; ++d) cv[d * n + k] = v[d];
  }
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    double a = fabs(v[d]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
    if ((threadIdx.x & 31) == 0 && a > 0) atomic_max_abs(mbits + d, a);
  }
}

// Charge digits per particle (bin order): c 2^E0 in six balanced signed
// base-256 digits (columns 0-5), each c v component in three (6-8, 9-11,
// 12-14).
__global__ void charge_digits_kernel(long long n, const double *__restrict__ cv,
                                     const TcScales *sc, uint4 *__restrict__ out) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint8_t b[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) b[i] = 0;
  balanced_digits(llrint(ldexp(cv[k], sc->ex[0])), CDIG, b);
#pragma unroll
  for (int d = 1; d < 4; ++d)
    balanced_digits(llrint(ldexp(cv[d * n + k], sc->ex[d])), JDIG, b + CDIG + JDIG * (d - 1));
  out[k] = pack16(b);
}

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// rho, j of every position from summed digit sums (sharded form, step 3)
__global__ void combine_kernel(long long npos, const double *__restrict__ sums,
                               const TcScales *sc, double *__restrict__ vals) {
  const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (u >= npos) return;
  double T[16], o[4];
#pragma unroll
  for (int i = 0; i < 16; ++i) T[i] = sums[i * npos + u];
  combine_position(T, sc->out, o);
#pragma unroll
  for (int d = 0; d < 4; ++d) vals[d * npos + u] = o[d];
}

template <bool NORM, bool IND>
int launch_tc(const TcArgs &A, long long tiles, cudaStream_t s) {
  const int smem = (int)sizeof(Smem);
  PRT_CHECK_CUDA(cudaFuncSetAttribute(tc_deposit_kernel<NORM, IND>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  tc_deposit_kernel<NORM, IND><<<(unsigned)tiles, THREADS, smem, s>>>(A);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

// The workspace buffers of a call with n particles (the same sizes give the
// same buffers, so the steps of the sharded form find them again).
struct TcPtrs {
  unsigned long long *nhi, *nlo;
  uint32_t *hits;
  double *cv;
  uint4 *cdig;
  float4 *cpos;
  double *scale_bin, *hits_bin;
  unsigned long long *mbits, *counters;
  TcScales *sc;
  uint4 *tile_ops;
  const uint32_t *tile_starts, *tile_rows;
  const double *tile_boxes;
  double *vals;
  const uint32_t *perm;
};

// Recursive bisection of the positions idx[b, e) into compact parts:
// along the longest axis of the part's box, at a multiple of g rows (so that
// all parts but the last of a branch hold exactly g), until a part holds at
// most g positions and, when wmax > 0, is at most wmax wide along every axis.
// Appends each final part's start (depth first: neighbouring parts are
// neighbours in space) to `cuts` when given.
void bisect(const double *P, std::vector<uint32_t> &idx, uint32_t b, uint32_t e, uint32_t g,
            double wmax, std::vector<uint32_t> *cuts) {
  struct Part {
    uint32_t b, e;
  };
  std::vector<Part> stack{{b, e}};
  while (!stack.empty()) {
    const Part t = stack.back();
    stack.pop_back();
    const uint32_t n = t.e - t.b;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = t.b; i < t.e; ++i)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], P[3 * (size_t)idx[i] + a]);
        hi[a] = std::max(hi[a], P[3 * (size_t)idx[i] + a]);
      }
    int ax = 0;
    for (int a = 1; a < 3; ++a)
      if (hi[a] - lo[a] > hi[ax] - lo[ax]) ax = a;
    const bool wide = wmax > 0 && hi[ax] - lo[ax] > wmax;
    if (n <= 1 || (n <= g && !wide)) {
      if (cuts) cuts->push_back(t.b);
      continue;
    }
    uint32_t nl;
    if (n > g) {
      nl = g * std::max<uint32_t>(1, (uint32_t)std::lround((double)n / (2.0 * g)));
      if (nl >= n) nl = g * ((n - 1) / g);
    } else {
      nl = n / 2;
    }
    std::nth_element(idx.begin() + t.b, idx.begin() + t.b + nl, idx.begin() + t.e,
                     [&](uint32_t x, uint32_t y) {
                       const double px = P[3 * (size_t)x + ax], py = P[3 * (size_t)y + ax];
                       return px != py ? px < py : x < y;
                     });
    stack.push_back({t.b + nl, t.e});
    stack.push_back({t.b, t.b + nl});
  }
}

// The tiles of a target for a shape radius, kept in the workspace while
// target and radius stay the same: parts of <= 128 positions from recursive
// bisection, at most two radii wide along every axis (so that a candidate
// lies within 2 radii of the tile centre along every axis and the score
// operands stay in FP16 range); inside a tile the rows are bisected again
// into compact groups of 32 (one per weight warp's rows). With their
// bounding boxes and the position operands.
int tc_tiles(const TcTarget &T, prt_workspace *ws, double radius, cudaStream_t s) {
  if (ws->tc_mesh_uid == T.uid && ws->tc_radius == radius && ws->tc_tiles > 0)
    return PRT_OK;
  const long long npos = T.npos;
  const double *P = T.pos_host;
  std::vector<uint32_t> rows((size_t)npos), ts;
  for (long long u = 0; u < npos; ++u) rows[u] = (uint32_t)u;
  ts.reserve(npos / 64 + 2);
  bisect(P, rows, 0, (uint32_t)npos, TM, 2.0 * radius * (1 - 1e-9), &ts);
  ts.push_back((uint32_t)npos);
  const long long nt = (long long)ts.size() - 1;
  std::vector<double> tb(6 * (size_t)std::max<long long>(1, nt), 0.0);
  double hf_max = 0;
  for (long long t = 0; t < nt; ++t) {
    bisect(P, rows, ts[t], ts[t + 1], 32, 0.0, nullptr);
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = ts[t]; i < ts[t + 1]; ++i)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], P[3 * (size_t)rows[i] + a]);
        hi[a] = std::max(hi[a], P[3 * (size_t)rows[i] + a]);
      }
    for (int a = 0; a < 3; ++a) {
      tb[6 * t + a] = 0.5 * (lo[a] + hi[a]);
      tb[6 * t + 3 + a] = 0.5 * (hi[a] - lo[a]);
      hf_max = std::max(hf_max, tb[6 * t + 3 + a]);
    }
  }
  // particle bins a quarter radius wide (the bin rows that a tile stages hold
  // ~1.4 times the particles within the radius of its box; half-radius bins
  // ~1.9 times), wider where a tile's segments could exceed MAXSEG: per axis
  // at most (2 hf + 2 a) / w + 4 bin rows, a row in at most three pieces
  // along a periodic x
  const bool per_x = T.mesh->dev.pmin[0] != T.mesh->dev.pmax[0];
  double bw = 0.25 * radius;
  for (;;) {
    const double rows = (2 * hf_max + 2 * radius) / bw + 4;
    if (rows * rows * (per_x ? 3 : 1) <= MAXSEG) break;
    bw *= 1.125;
  }
  int rc;
  const size_t b_ts = align256(4 * (size_t)(nt + 1)), b_tb = align256(48 * (size_t)nt);
  char *set = (char *)ws_buffer(ws, PRT_WS_TC_TILESET, b_ts + b_tb + 4 * (size_t)npos, &rc);
  if (!set) return rc;
  uint4 *ops = (uint4 *)ws_buffer(ws, PRT_WS_TC_TILES, 4096 * (size_t)nt, &rc);
  if (!ops) return rc;
  // pageable sources: the copies are staged before the calls return
  PRT_CHECK_CUDA(cudaMemcpyAsync(set, ts.data(), 4 * (size_t)(nt + 1), cudaMemcpyHostToDevice, s));
  PRT_CHECK_CUDA(cudaMemcpyAsync(set + b_ts, tb.data(), 48 * (size_t)nt, cudaMemcpyHostToDevice, s));
  PRT_CHECK_CUDA(cudaMemcpyAsync(set + b_ts + b_tb, rows.data(), 4 * (size_t)npos,
                                 cudaMemcpyHostToDevice, s));
  tile_operands_kernel<<<(unsigned)nt, 128, 0, s>>>(
      nt, (const uint32_t *)set, (const uint32_t *)(set + b_ts + b_tb),
      (const double *)(set + b_ts), T.pos, 1.0 / radius, ops);
  PRT_CHECK_CUDA(cudaGetLastError());
  PRT_CHECK_CUDA(cudaStreamSynchronize(s));
  ws->tc_mesh_uid = T.uid;
  ws->tc_radius = radius;
  ws->tc_tiles = nt;
  ws->tc_bin_width = bw;
  return PRT_OK;
}

int tc_buffers(const TcTarget &T, prt_workspace *ws, long long n, TcPtrs &B) {
  const long long tiles = ws->tc_tiles;
  int rc;
  const size_t b_u64 = align256(8 * (size_t)n), b_u32 = align256(4 * (size_t)n);
  const size_t b_cv = align256(32 * (size_t)n), b_dig = align256(16 * (size_t)n);
  const size_t b_f64 = align256(8 * (size_t)n);
  char *part = (char *)ws_buffer(ws, PRT_WS_TC_PART,
                                 2 * b_u64 + b_u32 + b_cv + 2 * b_dig + 2 * b_f64, &rc);
  if (!part) return rc;
  B.nhi = (unsigned long long *)part;
  B.nlo = (unsigned long long *)(part + b_u64);
  B.hits = (uint32_t *)(part + 2 * b_u64);
  B.cv = (double *)(part + 2 * b_u64 + b_u32);
  B.cdig = (uint4 *)(part + 2 * b_u64 + b_u32 + b_cv);
  B.scale_bin = (double *)(part + 2 * b_u64 + b_u32 + b_cv + b_dig);
  B.hits_bin = (double *)(part + 2 * b_u64 + b_u32 + b_cv + b_dig + b_f64);
  B.cpos = (float4 *)(part + 2 * b_u64 + b_u32 + b_cv + b_dig + 2 * b_f64);
  // small: maxima of |c|, |c v|, W (bits), the candidate counter, the scales
  char *misc = (char *)ws_buffer(ws, PRT_WS_TC_MISC, 1024, &rc);
  if (!misc) return rc;
  B.mbits = (unsigned long long *)misc;  // [8]
  B.counters = B.mbits + 8;             // [4]
  B.sc = (TcScales *)(misc + 256);
  B.tile_ops = (uint4 *)ws_buffer(ws, PRT_WS_TC_TILES, 4096 * (size_t)tiles, &rc);
  if (!B.tile_ops) return rc;
  const size_t b_ts = align256(4 * (size_t)(tiles + 1)), b_tb = align256(48 * (size_t)tiles);
  char *set = (char *)ws_buffer(ws, PRT_WS_TC_TILESET, b_ts + b_tb + 4 * (size_t)T.npos, &rc);
  if (!set) return rc;
  B.tile_starts = (const uint32_t *)set;
  B.tile_boxes = (const double *)(set + b_ts);
  B.tile_rows = (const uint32_t *)(set + b_ts + b_tb);
  B.vals = (double *)ws_buffer(ws, PRT_WS_DEP_VALUES, 4 * sizeof(double) * T.npos, &rc);
  if (!B.vals) return rc;
  B.perm = (const uint32_t *)ws_buffer(ws, PRT_WS_DEP_VALS, 8 * (size_t)n, &rc);
  if (!B.perm) return rc;
  B.perm += n;  // the second half: bin order -> particle index
  return PRT_OK;
}

// The particle bins of the tensor-core deposition (after tc_tiles): the
// width the tiles chose.
int tc_bins(const TcTarget &T, const prt_workspace *ws, prt_shape_function shape,
            BinGrid &G) {
  int rc;
  if (!choose_bins(T.mesh, T.lo, T.hi, ws->tc_bin_width, shape.radius, G, &rc))
    return rc;
  return PRT_OK;
}

double tc_kappa(prt_shape_function shape) {
  return shape.normalizer * shape.radius * shape.radius / (4.0 * (double)SIGMA * (double)SIGMA);
}

void tc_args(const TcTarget &T, prt_workspace *ws, prt_shape_function shape,
             const BinGrid &G, const TcPtrs &B, TcArgs &A) {
  A.G = G;
  A.pay = reinterpret_cast<const double2 *>(ws->buf[PRT_WS_DEP_PARTICLES]);
  A.starts = reinterpret_cast<const uint32_t *>(ws->buf[PRT_WS_DEP_BINSTARTS]);
  A.tile_starts = B.tile_starts;
  A.tile_rows = B.tile_rows;
  A.tile_boxes = B.tile_boxes;
  A.tile_ops = B.tile_ops;
  A.wdig = nullptr;
  A.cdig = B.cdig;
  A.cpos = B.cpos;
  A.order = nullptr;  // bisection order: CTAs running together share candidates in L2
  A.radius = shape.radius;
  A.inv_radius = 1.0 / shape.radius;
  A.norm_hi = B.nhi;
  A.norm_lo = B.nlo;
  A.hits = B.hits;
  A.out_scale = B.sc->out;
  A.vals = B.vals;
  A.sums = nullptr;
  A.npos = T.npos;
  A.counters = B.counters;
  A.st = ws->status;
}

// Steps 1-2 of a call: tile operands, particles binned and packed, the
// tiles' launch order, the normalising pass (normalising mode), the
// deposited charge c and c v per particle and their maxima (B.mbits[0..3]).
int tc_charges(const TcTarget &T, prt_workspace *ws, int32_t mode, prt_shape_function shape,
               const double *iw, long long n, const double *x, const double *q, const double *v,
               const uint32_t *el, bool want_hits, cudaStream_t s, TcPtrs &B, BinGrid &G) {
  const bool norm = mode == PRT_DEPOSIT_NORMALIZED;
  int rc;
  if ((rc = tc_tiles(T, ws, shape.radius, s))) return rc;
  if ((rc = tc_bins(T, ws, shape, G))) return rc;
  const long long tiles = ws->tc_tiles;
  if ((rc = tc_buffers(T, ws, n, B))) return rc;
  const double kappa = tc_kappa(shape);
  // particles binned, sorted and packed (payload weight q, q v)
  DepParticles P;
  {
    ScopedTimer timer(ws, PRT_TIME_DEPOSIT_STAGE, s);
    if ((rc = stage_particles(ws, G, n, x, q, v, el, nullptr, 1.0, nullptr, P, s))) return rc;
  }
  // buffers may have moved while staging grew the workspace
  if ((rc = tc_buffers(T, ws, n, B))) return rc;
  candidate_positions_kernel<<<prt_grid_blocks(n, 256), 256, 0, s>>>(n, B.perm, x, G, B.cpos);
  PRT_CHECK_CUDA(cudaGetLastError());
  PRT_CHECK_CUDA(cudaMemsetAsync(B.mbits, 0, 256, s));
  TcArgs A;
  tc_args(T, ws, shape, G, B, A);
  const unsigned pblocks = (unsigned)((n + 255) / 256);
  const uint32_t *n_live = P.starts + G.nbins;
  if (norm) {
    // position weights -> digits; the normalisation pass
    char *wbuf = (char *)ws_buffer(ws, PRT_WS_TC_WDIG,
                                   2048 * (size_t)tiles + align256(8 * (size_t)T.npos), &rc);
    if (!wbuf) return rc;
    uint4 *wdig = (uint4 *)wbuf;
    double *W = (double *)(wbuf + 2048 * (size_t)tiles);
    if ((rc = prt_dep_position_weights(T.mesh, ws, iw, W, s))) return rc;
    max_abs_kernel<<<592, 256, 0, s>>>(T.npos, W, B.mbits + 4);
    PRT_CHECK_CUDA(cudaGetLastError());
    weight_scale_kernel<<<1, 1, 0, s>>>(B.mbits, kappa, B.sc);
    PRT_CHECK_CUDA(cudaGetLastError());
    weight_digits_kernel<<<(unsigned)tiles, 128, 0, s>>>(tiles, B.tile_starts, B.tile_rows, W,
                                                         B.sc, wdig);
    PRT_CHECK_CUDA(cudaGetLastError());
    PRT_CHECK_CUDA(cudaMemsetAsync(B.nhi, 0, 8 * (size_t)n, s));
    PRT_CHECK_CUDA(cudaMemsetAsync(B.nlo, 0, 8 * (size_t)n, s));
    PRT_CHECK_CUDA(cudaMemsetAsync(B.hits, 0, 4 * (size_t)n, s));
    A.wdig = wdig;
    {
      ScopedTimer timer(ws, PRT_TIME_DEPOSIT_NORMALIZE, s);
      rc = want_hits ? launch_tc<true, true>(A, tiles, s) : launch_tc<true, false>(A, tiles, s);
      if (rc) return rc;
    }
    charges_kernel<true><<<pblocks, 256, 0, s>>>(n, n_live, A.pay, B.nhi, B.nlo,
                                                 want_hits ? B.hits : nullptr, B.sc, B.perm, B.cv,
                                                 B.scale_bin, B.hits_bin, B.mbits, ws->status);
  } else {
    charges_kernel<false><<<pblocks, 256, 0, s>>>(n, n_live, A.pay, nullptr, nullptr, nullptr,
                                                  B.sc, B.perm, B.cv, nullptr, nullptr, B.mbits,
                                                  ws->status);
  }
  PRT_CHECK_CUDA(cudaGetLastError());
  ws->tc_n = n;
  return PRT_OK;
}

// Step 3: charge digits from the maxima (device, [4] doubles), the
// deposition pass into vals (sums == NULL) or into digit sums.
int tc_deposit(const TcTarget &T, prt_workspace *ws, prt_shape_function shape, long long n,
               const BinGrid &G, TcPtrs &B, const double *maxima, double *sums, cudaStream_t s) {
  TcArgs A;
  tc_args(T, ws, shape, G, B, A);
  A.sums = sums;
  charge_scale_kernel<<<1, 1, 0, s>>>(reinterpret_cast<const unsigned long long *>(maxima),
                                      tc_kappa(shape), B.sc);
  PRT_CHECK_CUDA(cudaGetLastError());
  charge_digits_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, B.cv, B.sc, B.cdig);
  PRT_CHECK_CUDA(cudaGetLastError());
  ScopedTimer timer(ws, PRT_TIME_DEPOSIT_GATHER, s);
  return launch_tc<false, false>(A, ws->tc_tiles, s);
}

int tc_stats(prt_workspace *ws, bool norm, long long n, const TcPtrs &B,
             prt_deposit_stats *stats, cudaStream_t s) {
  int rc;
  std::memset(stats, 0, sizeof(*stats));
  if (norm && (rc = prt_dep_norm_stats(ws, n, B.scale_bin, B.hits_bin, stats, s))) return rc;
  unsigned long long h[2] = {0, 0};
  PRT_CHECK_CUDA(cudaMemcpyAsync(h, B.counters, sizeof(h), cudaMemcpyDeviceToHost, s));
  PRT_CHECK_CUDA(cudaStreamSynchronize(s));
  // candidates of the deposition pass (the normalisation pass adds the same)
  stats->evaluated_pairs = (double)(h[0] / (norm ? 2 : 1)) * TM;
  return PRT_OK;
}

// A mesh's distinct node positions as a target.
TcTarget mesh_target(const prt_mesh *mesh) {
  TcTarget T;
  T.mesh = mesh;
  T.uid = mesh->uid;
  T.npos = mesh->positions.count;
  T.pos = mesh->positions.pos;
  T.pos_host = mesh->pos_host.data();
  for (int a = 0; a < 3; ++a) {
    T.lo[a] = mesh->box_lo[a];
    T.hi[a] = mesh->box_hi[a];
  }
  return T;
}

}  // namespace

int prt_deposit_points_tc(const TcTarget &T, prt_workspace *ws, prt_shape_function shape,
                          long long n, const double *x, const double *q, const double *v,
                          const uint32_t *el, double *rho, double *j, cudaStream_t s) {
  TcPtrs B;
  BinGrid G;
  int rc;
  if ((rc = tc_charges(T, ws, PRT_DEPOSIT_PLAIN, shape, nullptr, n, x, q, v, el, false, s, B, G)))
    return rc;
  if ((rc = tc_deposit(T, ws, shape, n, G, B, reinterpret_cast<const double *>(B.mbits), nullptr,
                       s)))
    return rc;
  if (rho)
    PRT_CHECK_CUDA(cudaMemcpyAsync(rho, B.vals, sizeof(double) * T.npos,
                                   cudaMemcpyDeviceToDevice, s));
  if (j)
    PRT_CHECK_CUDA(cudaMemcpyAsync(j, B.vals + T.npos, 3 * sizeof(double) * T.npos,
                                   cudaMemcpyDeviceToDevice, s));
  return PRT_OK;
}

int prt_deposit_shape_tc(const prt_mesh *mesh, prt_workspace *ws, int32_t mode,
                         prt_shape_function shape, const double *iw, long long n,
                         const double *x, const double *q, const double *v,
                         const uint32_t *el, double *rho, double *j,
                         prt_deposit_stats *stats, cudaStream_t s) {
  TcPtrs B;
  BinGrid G;
  int rc;
  const TcTarget T = mesh_target(mesh);
  if ((rc = tc_charges(T, ws, mode, shape, iw, n, x, q, v, el, stats != nullptr, s, B, G)))
    return rc;
  if ((rc = tc_deposit(T, ws, shape, n, G, B, reinterpret_cast<const double *>(B.mbits),
                       nullptr, s)))
    return rc;
  if ((rc = prt_dep_expand(mesh, B.vals, rho, j, s))) return rc;
  if (stats) return tc_stats(ws, mode == PRT_DEPOSIT_NORMALIZED, n, B, stats, s);
  return PRT_OK;
}

// ------------------------------------------------------ C ABI: sharded form

extern "C" int prt_mesh_position_count(const prt_mesh *mesh, int64_t *count) {
  if (!mesh || !count) return PRT_ERR_INVALID_ARGUMENT;
  *count = mesh->positions.count;
  return PRT_OK;
}

extern "C" int prt_deposit_shape_charges(const prt_mesh *mesh, prt_workspace *ws, int32_t mode,
                                         prt_shape_function shape, const double *iw, int64_t n,
                                         const double *x, const double *q, const double *v,
                                         const uint32_t *el, double *local_max,
                                         prt_deposit_stats *stats, void *stream) {
  if (!mesh || !ws || !local_max || n < 1 || n >= (1ll << 31)) return PRT_ERR_INVALID_ARGUMENT;
  if (shape.alpha != 2 || !(shape.radius > 0)) return PRT_ERR_INVALID_ARGUMENT;
  if (mode != PRT_DEPOSIT_PLAIN && mode != PRT_DEPOSIT_NORMALIZED) return PRT_ERR_INVALID_ARGUMENT;
  if ((mode == PRT_DEPOSIT_NORMALIZED && !iw) || !x || !q) return PRT_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  TcPtrs B;
  BinGrid G;
  int rc;
  if ((rc = tc_charges(mesh_target(mesh), ws, mode, shape, iw, n, x, q, v, el, stats != nullptr,
                       s, B, G)))
    return rc;
  PRT_CHECK_CUDA(cudaMemcpyAsync(local_max, B.mbits, 4 * sizeof(double),
                                 cudaMemcpyDeviceToDevice, s));
  if (stats) return tc_stats(ws, mode == PRT_DEPOSIT_NORMALIZED, n, B, stats, s);
  return PRT_OK;
}

extern "C" int prt_deposit_shape_sums(const prt_mesh *mesh, prt_workspace *ws,
                                      prt_shape_function shape, int64_t n,
                                      const double *global_max, double *sums, void *stream) {
  if (!mesh || !ws || !global_max || !sums || n < 1 || n != ws->tc_n)
    return PRT_ERR_INVALID_ARGUMENT;
  if (ws->tc_mesh_uid != mesh->uid || ws->tc_radius != shape.radius)
    return PRT_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  TcPtrs B;
  BinGrid G;
  int rc;
  const TcTarget T = mesh_target(mesh);
  if ((rc = tc_bins(T, ws, shape, G))) return rc;
  if ((rc = tc_buffers(T, ws, n, B))) return rc;
  return tc_deposit(T, ws, shape, n, G, B, global_max, sums, s);
}

extern "C" int prt_deposit_shape_combine(const prt_mesh *mesh, prt_workspace *ws,
                                         prt_shape_function shape, const double *global_max,
                                         const double *sums, double *rho, double *j,
                                         void *stream) {
  if (!mesh || !ws || !global_max || !sums || !(shape.radius > 0))
    return PRT_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  const PositionSet &PS = mesh->positions;
  int rc;
  char *misc = (char *)ws_buffer(ws, PRT_WS_TC_MISC, 1024, &rc);
  if (!misc) return rc;
  TcScales *sc = (TcScales *)(misc + 256);
  double *vals = (double *)ws_buffer(ws, PRT_WS_DEP_VALUES, 4 * sizeof(double) * PS.count, &rc);
  if (!vals) return rc;
  charge_scale_kernel<<<1, 1, 0, s>>>(reinterpret_cast<const unsigned long long *>(global_max),
                                      tc_kappa(shape), sc);
  PRT_CHECK_CUDA(cudaGetLastError());
  combine_kernel<<<prt_grid_blocks(PS.count, 256), 256, 0, s>>>(PS.count, sums, sc, vals);
  PRT_CHECK_CUDA(cudaGetLastError());
  return prt_dep_expand(mesh, vals, rho, j, s);
}
