// Learned warm start: the conv decoder that maps a body's geometry, Mach number and Reynolds number to a coarse
// flowfield, trained on converged solutions of this solver. No counterpart in the reference (its only warm start is the
// previous Mach point's field, crates/bowshock-core/src/engine/run.rs:54-63, analysis.rs:744-748).
//
// Every contraction (fully connected layers, 3x3 convolutions as im2col GEMMs, and their backward passes) runs on the
// 5th-generation tensor cores: k_gemm stages BF16 operand tiles with TMA (cp.async.bulk.tensor, 128-byte swizzle, no
// multicast) into a 4-stage shared-memory ring, one elected thread issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32)
// into a TMEM accumulator, and four warps read it back with tcgen05.ld for a fused epilogue (bias, leaky ReLU, BF16 store,
// or FP32 split-K accumulation). Weights are FP32 masters updated by Adam, with BF16 copies for the GEMMs; a training
// run keeps its dataset on the device and launches every step from the host without copies.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "../../include/bowshock_b200.h"
#include "stream_copy.cuh"
#include "tma.cuh"

namespace bknet {

typedef __nv_bfloat16 bf16;

// ------------------------------------------------------------------------------------------------ device primitives
using bktma::mbar_expect_tx;
using bktma::mbar_init;
using bktma::mbar_wait;
using bktma::tma_load_4d;
using bktma::smem_u32;
using bktma::tma_load_2d;
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_relinquish() { asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// D[tmem] (+)= A[smem] x B[smem]^T, BF16 operands, FP32 accumulation; accumulate = 0 overwrites D.
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
// arrive on `bar` once every tcgen05.mma issued so far by this thread has completed
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
        "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor of a K-major operand tile written by TMA with the 128-byte swizzle: rows of 64 BF16
// (128 B), 8-row swizzle atoms 1024 B apart (stride byte offset), descriptor version 1, layout type 2 (SWIZZLE_128B). The
// tile base must be 1024-byte aligned; stepping along K inside the atom adds the byte offset (32 B per 16 elements) to
// the start address field.
__device__ __forceinline__ uint64_t sw128_desc(const void* tile) {
  const uint64_t a = (uint64_t)((smem_u32(tile) & 0x3FFFFu) >> 4);
  return a | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}
// Instruction descriptor of kind::f16: FP32 D (bits 4-5 = 1), BF16 A and B (bits 7-9, 10-12 = 1), both K-major,
// N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// ------------------------------------------------------------------------------------------------ the GEMM
constexpr int BM = 128, BK = 64, STAGES = 4;
enum { EPI_F32 = 0, EPI_F32_ATOMIC = 1, EPI_BIAS_ACT_BF16 = 2, EPI_BIAS_F32 = 3 };

struct GemmArgs {
  int M, N, K;
  int kb_per_split;  // k blocks of BK per CTA along grid.z
  int mode;
  float* d;
  long long ldd;
  bf16* y;
  long long ldy;
  const float* bias;
  float slope;  // leaky ReLU slope of EPI_BIAS_ACT_BF16 (1 = identity)
  int* err;     // set to 1 when a wait gave up
  // implicit-GEMM convolution (k_gemm_conv): A is the im2col of the NHWC input cx [cB, cHin, cWin, cC] of a 3x3 'same'
  // convolution at (cHin << cup) x (cWin << cup), never stored; cC a multiple of 64
  const bf16* cx;
  int cB, cHin, cWin, cC, cup;
};

template <int BN>
__host__ __device__ constexpr int tmem_cols() {
  return BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
}
template <int BN>
__host__ __device__ constexpr int gemm_smem_bytes() {
  return STAGES * (BM * BK * 2 + BN * BK * 2) + 1024 + 256;
}

// Epilogue of 16 accumulator columns nb .. nb + 15 of output row `row` (r: their FP32 bits from TMEM): bias + leaky
// ReLU to BF16, FP32 with or without bias, or FP32 atomic adds (split-K). Whole 16-column chunks at 16-byte-aligned
// addresses go out as two (BF16) or four (FP32) 16-byte stores; the values are the same either way.
__device__ __forceinline__ void store16(const GemmArgs& g, int row, int nb, const uint32_t* r) {
  const bool whole = nb + 16 <= g.N;
  if (g.mode == EPI_BIAS_ACT_BF16) {
    bf16* yp = g.y + (long long)row * g.ldy + nb;
    if (whole && (reinterpret_cast<uintptr_t>(yp) & 15) == 0) {
      uint4 o[2];
      __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(o);
#pragma unroll
      for (int q = 0; q < 16; q += 2) {
        float v0 = __uint_as_float(r[q]) + g.bias[nb + q];
        v0 = v0 > 0.f ? v0 : g.slope * v0;
        float v1 = __uint_as_float(r[q + 1]) + g.bias[nb + q + 1];
        v1 = v1 > 0.f ? v1 : g.slope * v1;
        h[q / 2] = __floats2bfloat162_rn(v0, v1);
      }
      reinterpret_cast<uint4*>(yp)[0] = o[0];
      reinterpret_cast<uint4*>(yp)[1] = o[1];
      return;
    }
#pragma unroll
    for (int q = 0; q < 16; q += 2) {
      if (nb + q >= g.N) break;
      float v0 = __uint_as_float(r[q]) + g.bias[nb + q];
      v0 = v0 > 0.f ? v0 : g.slope * v0;
      if (nb + q + 1 < g.N) {
        float v1 = __uint_as_float(r[q + 1]) + g.bias[nb + q + 1];
        v1 = v1 > 0.f ? v1 : g.slope * v1;
        *reinterpret_cast<__nv_bfloat162*>(yp + q) = __floats2bfloat162_rn(v0, v1);
      } else {
        yp[q] = __float2bfloat16_rn(v0);
      }
    }
    return;
  }
  float* dp = g.d + (long long)row * g.ldd + nb;
  if (g.mode != EPI_F32_ATOMIC && whole && (reinterpret_cast<uintptr_t>(dp) & 15) == 0) {
#pragma unroll
    for (int q = 0; q < 16; q += 4) {
      float4 v = make_float4(__uint_as_float(r[q]), __uint_as_float(r[q + 1]), __uint_as_float(r[q + 2]), __uint_as_float(r[q + 3]));
      if (g.mode == EPI_BIAS_F32) v.x += g.bias[nb + q], v.y += g.bias[nb + q + 1], v.z += g.bias[nb + q + 2], v.w += g.bias[nb + q + 3];
      *reinterpret_cast<float4*>(dp + q) = v;
    }
    return;
  }
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    if (nb + q >= g.N) break;
    float v = __uint_as_float(r[q]);
    if (g.mode == EPI_F32_ATOMIC)
      atomicAdd(dp + q, v);
    else if (g.mode == EPI_BIAS_F32)
      dp[q] = v + g.bias[nb + q];
    else
      dp[q] = v;
  }
}

// D[M, N] = A[M, K] B[N, K]^T (A and B row-major BF16, K contiguous), one 128 x BN tile per CTA, the K blocks of
// blockIdx.z's split. Warp 0 lane 0 loads (TMA), warp 1 lane 0 issues the MMAs, all four warps run the epilogue (thread t
// owns accumulator row t: TMEM lane t).
// CONV: A is the implicit im2col of a 3x3 'same' convolution of the NHWC activations cx [cB, cHin, cWin, cC] (cC a
// multiple of 64, no upsampling), through a 4D tensor map over (C, W, H, B) whose box is 64 channels of 128 whole output
// pixels (cWin x R rows x NB images): K block kb is tap kb * 64 / cC, channels (kb * 64) % cC, and its A tile is that box
// loaded at the tile's first pixel shifted by the tap (dx, dy); the rows and columns the shift moves outside the image
// read zeros, which is the convolution's padding. A tile of 128 output pixels is 128 / cWin whole rows of one image (or
// whole images), so the box's smem rows are the tile's rows in order, in the 128-byte-swizzled layout the MMA reads.
// WGRAD: the weight gradient of such a convolution, D[cout, 9 cin] = sum over pixels of g[p, cout] x[p shifted by the
// tap, cin]: A is g transposed ([cout, pixels], 2D map), B a 4D map over xs [3 cin, B, H, W], the transposed
// activations in three copies shifted along x by dx = -1, 0, +1 (zeros past the row ends; W = 64, so a K block is one
// image row of 64 pixels and the box's x coordinate is always 0, aligned), whose box is 64 pixels x BN channels of copy
// dx, loaded at the image row shifted by the tap's dy (zeros above and below the image). The tap is that of the tile's
// columns (n0 / cin; BN divides cin).
enum { GEMM_PLAIN = 0, GEMM_CONV = 1, GEMM_WGRAD = 2 };
template <int BN, int KIND>
__global__ void __launch_bounds__(128, 1) k_gemm(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, GemmArgs g) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, TCOLS = tmem_cols<BN>();
  uint8_t* sa = smem;
  uint8_t* sb = smem + STAGES * A_BYTES;
  uint64_t* full = reinterpret_cast<uint64_t*>(sb + STAGES * B_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  __shared__ int s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int nkb_total = (g.K + BK - 1) / BK;
  const int kb0 = blockIdx.z * g.kb_per_split;
  const int nkb = min(g.kb_per_split, nkb_total - kb0);
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(full + s, 1), mbar_init(empty + s, 1);
    mbar_init(done, 1);
    bktma::mbar_init_fence();
    s_abort = 0;
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, TCOLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  constexpr uint32_t IDESC = idesc_bf16(BM, BN);
  if (nkb > 0 && warp == 0 && lane == 0) {  // producer: TMA loads into the stage ring
    for (int i = 0; i < nkb; ++i) {
      const int s = i % STAGES;
      const uint32_t ph = (uint32_t)((i / STAGES) & 1);
      if (i >= STAGES && !mbar_wait(empty + s, ph ^ 1u)) {
        s_abort = 1;
        break;
      }
      mbar_expect_tx(full + s, (uint32_t)(A_BYTES + B_BYTES));
      if constexpr (KIND == GEMM_CONV) {
        const int hw = g.cHin * g.cWin, k0 = (kb0 + i) * BK, tap = k0 / g.cC;
        tma_load_4d(sa + s * A_BYTES, &ta, full + s, k0 - tap * g.cC, tap % 3 - 1, (m0 % hw) / g.cWin + tap / 3 - 1, m0 / hw);
      } else {
        tma_load_2d(sa + s * A_BYTES, &ta, full + s, (kb0 + i) * BK, m0);
      }
      if constexpr (KIND == GEMM_WGRAD) {  // K block kb: image row kb % H of image kb / H
        const int kb = kb0 + i, tap = n0 / g.cC;
        tma_load_4d(sb + s * B_BYTES, &tb, full + s, 0, kb % g.cHin + tap / 3 - 1, kb / g.cHin, (tap % 3) * g.cC + n0 - tap * g.cC);
      } else {
        tma_load_2d(sb + s * B_BYTES, &tb, full + s, (kb0 + i) * BK, n0);
      }
    }
  } else if (nkb > 0 && warp == 1 && lane == 0) {  // MMA issuer
    for (int i = 0; i < nkb; ++i) {
      const int s = i % STAGES;
      const uint32_t ph = (uint32_t)((i / STAGES) & 1);
      if (!mbar_wait(full + s, ph)) {
        s_abort = 1;
        break;
      }
      tc_fence_after();
      const uint64_t ad = sw128_desc(sa + s * A_BYTES), bd = sw128_desc(sb + s * B_BYTES);
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) mma_bf16(tmem, ad + 2ull * kk, bd + 2ull * kk, IDESC, (i | kk) != 0);
      mma_commit(empty + s);  // the stage is free once these MMAs have read it
    }
    mma_commit(done);
  }
  __syncwarp();
  // epilogue: wait for the accumulator, TMEM -> registers -> global
  bool ok = nkb > 0 && mbar_wait(done, 0);
  if (!ok && nkb > 0) s_abort = 1;
  ok = __all_sync(0xffffffffu, ok);  // tcgen05.ld is warp-collective
  tc_fence_after();
  const int row = m0 + warp * 32 + lane;
  if (ok) {
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
      uint32_t r[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, r);
      tmem_ld_wait();
      if (row >= g.M) continue;
      const int nb = n0 + c;
      store16(g, row, nb, r);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (s_abort && threadIdx.x == 0) atomicExch(g.err, 1);
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, TCOLS);
  }
}

// The same GEMM with its A operand gathered on the fly (implicit-GEMM convolution): row m of A is output pixel m, and its
// K block kb holds the 64 input channels c0 .. c0 + 63 of tap (kb * 64) / C at the pixel shifted by the tap (zeros
// outside the image), 128 contiguous bytes of the NHWC input. The 64 threads of warps 2 and 3 copy each 128-row A tile
// with cp.async (16-byte chunks, zero fill outside), placed in the 128-byte-swizzle layout a TMA load would give (chunk
// q of row r at r * 128 + (q ^ (r & 7)) * 16); warp 0 lane 0 brings B (the weights) by TMA. A stage's barrier completes
// after that lane's expect-tx arrival (with the B bytes) and one arrival per copying thread, each made once the thread's
// copies of the stage have landed and been fenced for the tensor cores (the copies run LAG = 2 stages ahead of the
// arrivals). Warp 1 lane 0 issues the MMAs, all four warps run the epilogue.
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void cp_async16_zfill(uint32_t dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
template <int BN>
__global__ void __launch_bounds__(128, 1) k_gemm_conv(const __grid_constant__ CUtensorMap tb, GemmArgs g) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, TCOLS = tmem_cols<BN>(), LAG = 2;
  uint8_t* sa = smem;
  uint8_t* sb = smem + STAGES * A_BYTES;
  uint64_t* full = reinterpret_cast<uint64_t*>(sb + STAGES * B_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  __shared__ int s_abort;
  __shared__ int s_off[9][BM];  // element offset of tile row r's source pixel under tap t in cx (-1: outside the image, past M)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int nkb_total = (g.K + BK - 1) / BK;
  const int kb0 = blockIdx.z * g.kb_per_split;
  const int nkb = min(g.kb_per_split, nkb_total - kb0);
  const int H = g.cHin << g.cup, W = g.cWin << g.cup;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(full + s, 65), mbar_init(empty + s, 1);
    mbar_init(done, 1);
    bktma::mbar_init_fence();
    s_abort = 0;
  }
  {
    const int m = threadIdx.x, p = m0 + m;  // 128 threads, one row each
    int b = -1, y = 0, x = 0;
    if (p < g.M) x = p % W, y = (p / W) % H, b = p / (W * H);
#pragma unroll
    for (int t = 0; t < 9; ++t) {
      const int yy = y + t / 3 - 1, xx = x + t % 3 - 1;
      s_off[t][m] = (b >= 0 && yy >= 0 && yy < H && xx >= 0 && xx < W) ? ((b * g.cHin + (yy >> g.cup)) * g.cWin + (xx >> g.cup)) * g.cC : -1;
    }
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, TCOLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  constexpr uint32_t IDESC = idesc_bf16(BM, BN);
  if (nkb > 0 && warp == 0 && lane == 0) {  // B (the weights) by TMA
    for (int i = 0; i < nkb; ++i) {
      const int s = i % STAGES;
      const uint32_t ph = (uint32_t)((i / STAGES) & 1);
      if (i >= STAGES && !mbar_wait(empty + s, ph ^ 1u)) {
        s_abort = 1;
        break;
      }
      mbar_expect_tx(full + s, (uint32_t)B_BYTES);
      tma_load_2d(sb + s * B_BYTES, &tb, full + s, (kb0 + i) * BK, n0);
    }
  } else if (nkb > 0 && warp >= 2) {  // warps 2 and 3: A gathered by cp.async
    const int q = threadIdx.x - 64, part = q & 7, r0 = q >> 3;
    int issued = 0;
    bool aborted = false;
    for (int i = 0; i < nkb; ++i) {
      const int s = i % STAGES;
      const uint32_t ph = (uint32_t)((i / STAGES) & 1);
      int ok = 1;
      if (i >= STAGES && lane == 0) ok = mbar_wait(empty + s, ph ^ 1u) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) s_abort = 1;
        aborted = true;
        break;
      }
      const int k0 = (kb0 + i) * BK, tap = k0 / g.cC, c0 = k0 % g.cC;
      const int* offs = s_off[tap];
      // rows r0 + 8 t share r & 7, so this thread's chunk lands at the same swizzled position in each of its rows
      const uint32_t dst = smem_u32(sa + s * A_BYTES) + (uint32_t)(r0 * 128 + ((part ^ (r0 & 7)) << 4));
      const bf16* cxp = g.cx + c0 + part * 8;
#pragma unroll
      for (int t = 0; t < BM / 8; ++t) {
        const int o = offs[r0 + 8 * t];
        cp_async16_zfill(dst + (uint32_t)(t * 8 * 128), o >= 0 ? cxp + o : g.cx, o >= 0 ? 16u : 0u);
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
      ++issued;
      if (i >= LAG) {
        asm volatile("cp.async.wait_group 2;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(full + (i - LAG) % STAGES);
      }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (!aborted)
      for (int i = max(0, issued - LAG); i < issued; ++i) mbar_arrive(full + i % STAGES);
  } else if (nkb > 0 && warp == 1 && lane == 0) {  // MMA issuer (as k_gemm)
    for (int i = 0; i < nkb; ++i) {
      const int s = i % STAGES;
      const uint32_t ph = (uint32_t)((i / STAGES) & 1);
      if (!mbar_wait(full + s, ph)) {
        s_abort = 1;
        break;
      }
      tc_fence_after();
      const uint64_t ad = sw128_desc(sa + s * A_BYTES), bd = sw128_desc(sb + s * B_BYTES);
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) mma_bf16(tmem, ad + 2ull * kk, bd + 2ull * kk, IDESC, (i | kk) != 0);
      mma_commit(empty + s);
    }
    mma_commit(done);
  }
  __syncwarp();
  bool ok = nkb > 0 && mbar_wait(done, 0);
  if (!ok && nkb > 0) s_abort = 1;
  ok = __all_sync(0xffffffffu, ok);
  tc_fence_after();
  const int row = m0 + warp * 32 + lane;
  if (ok) {
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
      uint32_t r[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, r);
      tmem_ld_wait();
      if (row >= g.M) continue;
      const int nb = n0 + c;
      store16(g, row, nb, r);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (s_abort && threadIdx.x == 0) atomicExch(g.err, 1);
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, TCOLS);
  }
}

// ------------------------------------------------------------------------------------------------ elementwise kernels
// im2col of a 3x3 'same' convolution over NHWC input x [B, Hin, Win, C] (C a multiple of 8), optionally read through a
// nearest-neighbour 2x upsampling (up = 1: the convolution runs at 2Hin x 2Win): col [B*H*W, 9C], column (ky*3+kx)*C + c.
__global__ void k_im2col(const bf16* __restrict__ x, int B, int Hin, int Win, int C, int up, bf16* __restrict__ col) {
  const int H = Hin << up, W = Win << up, c8 = C >> 3;
  const long long total = (long long)B * H * W * 9 * c8;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int cc = (int)(t % c8);
    long long r = t / c8;
    const int tap = (int)(r % 9);
    const long long p = r / 9;
    const int xo = (int)(p % W), yo = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
    const int yy = yo + tap / 3 - 1, xx = xo + tap % 3 - 1;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (yy >= 0 && yy < H && xx >= 0 && xx < W) {
      const long long src = (((long long)b * Hin + (yy >> up)) * Win + (xx >> up)) * C + cc * 8;
      v = *reinterpret_cast<const uint4*>(x + src);
    }
    *reinterpret_cast<uint4*>(col + p * 9 * C + tap * C + cc * 8) = v;
  }
}

// out[c][r] = in[r][c] for an R x C BF16 matrix (ld_in, ld_out in elements), 32 x 32 tiles through shared memory
__global__ void k_transpose(const bf16* __restrict__ in, long long ld_in, int R, int C, bf16* __restrict__ out, long long ld_out) {
  __shared__ bf16 t[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    t[k][threadIdx.x] = (r < R && c < C) ? in[(long long)r * ld_in + c] : __float2bfloat16_rn(0.f);
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (c < C && r < R) out[(long long)c * ld_out + r] = t[threadIdx.x][k];
  }
}

// Weights of the input-gradient convolution: wt[ci][(ky', kx') * Cout + co] = w[co][((2-ky')*3 + (2-kx')) * Cin + ci]
__global__ void k_flip_weights(const bf16* __restrict__ w, int Cin, int Cout, bf16* __restrict__ wt) {
  const int total = Cin * 9 * Cout;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int co = t % Cout, tap = (t / Cout) % 9, ci = t / (9 * Cout);
    wt[t] = w[(long long)co * 9 * Cin + (8 - tap) * Cin + ci];
  }
}

// db[c] += sum over rows of g[r][c]: blocks of 32 columns x 8 row groups over a slice of the rows, reduced through
// shared memory, one atomic per column and block
__global__ void k_bias_grad(const bf16* __restrict__ g, long long rows, int C, float* __restrict__ db) {
  __shared__ float part[8][33];
  const int c = blockIdx.x * 32 + threadIdx.x;
  const long long per = (rows + gridDim.y - 1) / gridDim.y;
  const long long r0 = blockIdx.y * per, r1 = min(rows, r0 + per);
  float acc = 0.f;
  if (c < C)
    for (long long r = r0 + threadIdx.y; r < r1; r += 8) acc += __bfloat162float(g[r * C + c]);
  part[threadIdx.y][threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.y == 0 && c < C) {
    float t = 0.f;
    for (int k = 0; k < 8; ++k) t += part[k][threadIdx.x];
    atomicAdd(db + c, t);
  }
}

// The transposed im2col of a 3x3 'same' convolution's input (the dW operand): colT[(tap * C + c)][p], p over the
// B * H * W output pixels, written directly in 32 x 32 tiles through shared memory (reads along the channels, writes
// along the pixels); up = 1 reads the input through the nearest 2x upsampling.
__global__ void k_im2col_t(const bf16* __restrict__ x, int B, int Hin, int Win, int C, int up, bf16* __restrict__ colT, long long P) {
  __shared__ bf16 t[32][33];
  const int H = Hin << up, W = Win << up;
  const long long p0 = (long long)blockIdx.x * 32;
  const int cblocks = (C + 31) / 32;
  const int tap = blockIdx.y / cblocks, c0 = (blockIdx.y % cblocks) * 32;
  const int dy = tap / 3 - 1, dx = tap % 3 - 1;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const long long p = p0 + k;
    const int c = c0 + threadIdx.x;
    bf16 v = __float2bfloat16_rn(0.f);
    if (p < P && c < C) {
      const int xo = (int)(p % W), yo = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
      const int yy = yo + dy, xx = xo + dx;
      if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = x[(((long long)b * Hin + (yy >> up)) * Win + (xx >> up)) * C + c];
    }
    t[k][threadIdx.x] = v;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k;
    const long long p = p0 + threadIdx.x;
    if (c < C && p < P) colT[((long long)tap * C + c) * P + p] = t[threadIdx.x][k];
  }
}

// Gradient at the previous layer's output: g[b, y, x, c] = (sum of dx over the 2x2 children when the layer upsampled,
// else dx) x leaky-ReLU'(y_prev) (the sign of the output equals the sign of the pre-activation).
__global__ void k_grad_prev(const float* __restrict__ dx, int B, int Hin, int Win, int C, int up, const bf16* __restrict__ yprev, float slope,
                            bf16* __restrict__ g) {
  const long long total = (long long)B * Hin * Win * C;
  const int W = Win << up, H = Hin << up;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t % C);
    const long long p = t / C;
    float s;
    if (up) {
      const int x = (int)(p % Win), y = (int)((p / Win) % Hin), b = (int)(p / ((long long)Win * Hin));
      const long long q = ((long long)b * H + 2 * y) * W + 2 * x;
      s = dx[q * C + c] + dx[(q + 1) * C + c] + dx[(q + W) * C + c] + dx[(q + W + 1) * C + c];
    } else {
      s = dx[t];
    }
    const float yv = __bfloat162float(yprev[t]);
    g[t] = __float2bfloat16_rn(yv > 0.f ? s : slope * s);
  }
}

// Masked mean-squared error of the first `nout` channels of out [B*P, CO] against target [B, P, nout]; the gradient
// 2 (out - t) mask / count into g [B*P, CO] (BF16, zero in the padding channels); the loss summed into *loss.
// tstep (may be null): the loss goes to loss[*tstep] (a training step replayed from a CUDA graph reads its index here)
__global__ void k_loss(const float* __restrict__ out, int CO, const float* __restrict__ target, int nout, const uint8_t* __restrict__ mask, int P,
                       long long rows, float inv_count, bf16* __restrict__ g, float* __restrict__ loss, const int* __restrict__ tstep) {
  if (tstep) loss += *tstep;
  float acc = 0.f;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < rows * CO; t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t % CO);
    const long long r = t / CO;
    float gr = 0.f;
    if (c < nout && mask[r % P]) {
      const float e = out[t] - target[r * nout + c];
      acc += e * e;
      gr = 2.f * e * inv_count;
    }
    g[t] = __float2bfloat16_rn(gr);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc * inv_count);
}

// rows of the device dataset into a batch: x [B, nin] (BF16) and target [B, nt]
// tstep (may be null): the batch's rows are idx[*tstep * B ..] (a training step replayed from a CUDA graph)
__global__ void k_gather(const float* __restrict__ dsx, int nin, const float* __restrict__ dst, long long nt, const int* __restrict__ idx, int B,
                         bf16* __restrict__ x, float* __restrict__ t, const int* __restrict__ tstep) {
  if (tstep) idx += (long long)(*tstep) * B;
  const long long total = (long long)B * nt;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(q / nt);
    const long long k = q % nt;
    t[q] = dst[(long long)idx[b] * nt + k];
    if (k < nin) x[(long long)b * nin + k] = __float2bfloat16_rn(dsx[(long long)idx[b] * nin + k]);
  }
}

__global__ void k_to_bf16(const float* __restrict__ a, long long n, bf16* __restrict__ b) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) b[q] = __float2bfloat16_rn(a[q]);
}

// Adam step count and its bias-corrected learning rate, on the device so that a captured training step replays
// (and advances the training-step index tstep of a replayed step, when given)
__global__ void k_adam_prep(int* step, float* coef, float lr, float b1, float b2, int* tstep) {
  if (tstep) ++(*tstep);
  const int t = ++(*step);
  coef[0] = lr * sqrtf(1.f - powf(b2, (float)t)) / (1.f - powf(b1, (float)t));
}
// Adam (Kingma & Ba 2015) on the FP32 masters; the BF16 copies of the weight matrices refreshed (wb may be null)
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v, const float* __restrict__ g, long long n,
                       const float* __restrict__ coef, float b1, float b2, float eps, bf16* __restrict__ wb) {
  const float a = coef[0];
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.f - b1) * gq, vq = b2 * v[q] + (1.f - b2) * gq * gq;
    m[q] = mq, v[q] = vq;
    const float wq = w[q] - a * mq / (sqrtf(vq) + eps);
    w[q] = wq;
    if (wb) wb[q] = __float2bfloat16_rn(wq);
  }
}

// Persistent form of k_gemm for GEMMs without a K split: a grid of at most (SMs x resident CTAs) CTAs of 192 threads,
// each looping over the tiles t = blockIdx.x, blockIdx.x + gridDim.x, ... (tile t: rows (t % M tiles) x 128, columns
// (t / M tiles) x BN). Warp 0 lane 0 streams the A and B stages of all its tiles through the STAGES ring (TMA; A as in
// k_gemm<BN, KIND>), warp 1 lane 0 issues each tile's MMAs into one of two TMEM accumulators (alternating tiles), and
// warps 2-5 (each owning the TMEM lane quarter warp % 4) run the epilogue of one accumulator while the MMAs fill the
// other, so the loads, the MMAs and the epilogue of consecutive tiles overlap. Barriers: full / empty per stage,
// acc_full[2] (tcgen05.commit after a tile's last MMA), acc_empty[2] (one arrival per epilogue warp once its lanes are
// read). The MMAs and the K order of every tile are k_gemm's, so D is the same bit for bit. Every wait is bounded; a
// wait that gives up ends that role and sets the error flag.
template <int BN, int KIND>
__global__ void __launch_bounds__(192, 1) k_gemm_p(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, GemmArgs g) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, TC = tmem_cols<BN>();
  uint8_t* sa = smem;
  uint8_t* sb = smem + STAGES * A_BYTES;
  uint64_t* full = reinterpret_cast<uint64_t*>(sb + STAGES * B_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* acc_full = empty + STAGES;
  uint64_t* acc_empty = acc_full + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
  __shared__ int s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mtiles = (g.M + BM - 1) / BM, tiles = mtiles * ((g.N + BN - 1) / BN);
  const int nkb = (g.K + BK - 1) / BK;
  if (threadIdx.x == 0) {
    for (int q = 0; q < STAGES; ++q) mbar_init(full + q, 1), mbar_init(empty + q, 1);
    for (int q = 0; q < 2; ++q) mbar_init(acc_full + q, 1), mbar_init(acc_empty + q, 4);
    bktma::mbar_init_fence();
    s_abort = 0;
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 2 * TC);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  constexpr uint32_t IDESC = idesc_bf16(BM, BN);
  if (warp == 0 && lane == 0) {  // producer
    int it = 0;
    bool ok = true;
    for (int t = blockIdx.x; ok && t < tiles; t += gridDim.x) {
      const int m0 = (t % mtiles) * BM, n0 = (t / mtiles) * BN;
      for (int kb = 0; kb < nkb; ++kb, ++it) {
        const int q = it % STAGES;
        const uint32_t ph = (uint32_t)((it / STAGES) & 1);
        if (it >= STAGES && !mbar_wait(empty + q, ph ^ 1u)) {
          s_abort = 1;
          ok = false;
          break;
        }
        mbar_expect_tx(full + q, (uint32_t)(A_BYTES + B_BYTES));
        if constexpr (KIND == GEMM_CONV) {
          const int hw = g.cHin * g.cWin, k0 = kb * BK, tap = k0 / g.cC;
          tma_load_4d(sa + q * A_BYTES, &ta, full + q, k0 - tap * g.cC, tap % 3 - 1, (m0 % hw) / g.cWin + tap / 3 - 1, m0 / hw);
        } else {
          tma_load_2d(sa + q * A_BYTES, &ta, full + q, kb * BK, m0);
        }
        tma_load_2d(sb + q * B_BYTES, &tb, full + q, kb * BK, n0);
      }
    }
  } else if (warp == 1 && lane == 0) {  // MMA issuer
    int it = 0, tl = 0;
    bool ok = true;
    for (int t = blockIdx.x; ok && t < tiles; t += gridDim.x, ++tl) {
      const int buf = tl & 1;
      if (tl >= 2 && !mbar_wait(acc_empty + buf, (uint32_t)(((tl >> 1) & 1) ^ 1))) {
        s_abort = 1;
        break;
      }
      tc_fence_after();
      const uint32_t d = tmem + (uint32_t)(buf * TC);
      for (int kb = 0; kb < nkb; ++kb, ++it) {
        const int q = it % STAGES;
        const uint32_t ph = (uint32_t)((it / STAGES) & 1);
        if (!mbar_wait(full + q, ph)) {
          s_abort = 1;
          ok = false;
          break;
        }
        tc_fence_after();
        const uint64_t ad = sw128_desc(sa + q * A_BYTES), bd = sw128_desc(sb + q * B_BYTES);
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk) mma_bf16(d, ad + 2ull * kk, bd + 2ull * kk, IDESC, (kb | kk) != 0);
        mma_commit(empty + q);
      }
      if (ok) mma_commit(acc_full + buf);
    }
  } else if (warp >= 2) {  // epilogue
    const int quarter = warp & 3;
    int tl = 0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++tl) {
      const int buf = tl & 1;
      bool ok = mbar_wait(acc_full + buf, (uint32_t)((tl >> 1) & 1));
      ok = __all_sync(0xffffffffu, ok);  // tcgen05.ld is warp-collective
      if (!ok) {
        if (lane == 0) s_abort = 1;
        break;
      }
      tc_fence_after();
      const int m0 = (t % mtiles) * BM, n0 = (t / mtiles) * BN;
      const int row = m0 + quarter * 32 + lane;
#pragma unroll 1
      for (int c = 0; c < BN; c += 16) {
        uint32_t r[16];
        tmem_ld16(tmem + (uint32_t)(buf * TC) + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c, r);
        tmem_ld_wait();
        if (row < g.M) store16(g, row, n0 + c, r);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acc_empty + buf);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (s_abort && threadIdx.x == 0) atomicExch(g.err, 1);
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 2 * TC);
  }
}

// ------------------------------------------------------------------------------------------------ host side
static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
// GEMMs without a K split run the persistent kernel (k_gemm_p); false: one CTA per tile (k_gemm). Same results.
static bool persistent_gemm = true;
static bool get_encode(std::string& err) {
  if (!g_encode) g_encode = bktma::encoder(err);
  return g_encode != nullptr;
}

// Tensor map of a row-major BF16 matrix [rows, cols] with leading dimension ld (elements, a multiple of 8), boxes of
// 64 columns x box_rows rows, 128-byte swizzle, zero fill outside the matrix.
static bool make_map(CUtensorMap* m, const void* p, long long rows, long long cols, long long ld, int box_rows, std::string& err) {
  if (((uintptr_t)p & 15) || (ld % 8) || rows <= 0 || cols <= 0) {
    err = "GEMM operand not 16-byte aligned, or a leading dimension not a multiple of 8";
    return false;
  }
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(p), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
    return false;
  }
  return true;
}

template <int BN, int KIND = GEMM_PLAIN>
static cudaError_t launch_gemm_bn(const CUtensorMap& ta, const CUtensorMap& tb, const GemmArgs& g, dim3 grid, cudaStream_t st) {
  cudaError_t e;
  if constexpr (KIND != GEMM_WGRAD) {
    if (grid.z == 1 && persistent_gemm) {  // one K split: the persistent kernel over the grid.x x grid.y tiles
      if ((e = cudaFuncSetAttribute(k_gemm_p<BN, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, gemm_smem_bytes<BN>())) != cudaSuccess)
        return e;
      // SMs of the device x CTAs of k_gemm_p<BN, KIND> per SM, queried once (the grid only needs to be at most that; any
      // smaller grid gives the same results)
      static std::once_flag once;
      static long long slots = 148;
      std::call_once(once, [] {
        int dev = 0, sms = 0, resident = 0;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_gemm_p<BN, KIND>, 192, gemm_smem_bytes<BN>()) == cudaSuccess)
          slots = (long long)sms * std::max(resident, 1);
        (void)cudaGetLastError();
      });
      const long long tiles = (long long)grid.x * grid.y;
      const unsigned ctas = (unsigned)std::min<long long>(tiles, slots);
      k_gemm_p<BN, KIND><<<ctas, 192, gemm_smem_bytes<BN>(), st>>>(ta, tb, g);
      return cudaGetLastError();
    }
  }
  if ((e = cudaFuncSetAttribute(k_gemm<BN, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, gemm_smem_bytes<BN>())) != cudaSuccess) return e;
  k_gemm<BN, KIND><<<grid, 128, gemm_smem_bytes<BN>(), st>>>(ta, tb, g);
  return cudaGetLastError();
}

static int pick_bn(int N) { return N <= 16 ? 16 : N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256; }

// D = A B^T with A [M, K] (lda), B [N, K] (ldb), BF16 row-major; the epilogue as in g (M, N, K, kb_per_split set here).
// splits > 1 accumulates K slices atomically (mode EPI_F32_ATOMIC; D zeroed by the caller).
static int gemm(const bf16* A, long long lda, const bf16* B, long long ldb, int M, int N, int K, GemmArgs g, int splits, cudaStream_t st,
                std::string& err) {
  if (M <= 0 || N <= 0 || K <= 0) return 0;
  if (!get_encode(err)) return BOWSHOCK_CUDA_ERROR;
  const int bn = pick_bn(N);
  CUtensorMap ta, tb;
  if (!make_map(&ta, A, M, K, lda, BM, err) || !make_map(&tb, B, N, K, ldb, bn, err)) return BOWSHOCK_INVALID;
  const int nkb = (K + BK - 1) / BK;
  splits = std::max(1, std::min(splits, nkb));
  const int per = (nkb + splits - 1) / splits;
  splits = (nkb + per - 1) / per;
  if (splits > 1 && g.mode != EPI_F32_ATOMIC) {
    err = "split-K needs the atomic FP32 epilogue";
    return BOWSHOCK_INVALID;
  }
  g.M = M, g.N = N, g.K = K, g.kb_per_split = per;
  dim3 grid((M + BM - 1) / BM, (N + bn - 1) / bn, splits);
  cudaError_t e;
  switch (bn) {
    case 16: e = launch_gemm_bn<16>(ta, tb, g, grid, st); break;
    case 32: e = launch_gemm_bn<32>(ta, tb, g, grid, st); break;
    case 64: e = launch_gemm_bn<64>(ta, tb, g, grid, st); break;
    case 128: e = launch_gemm_bn<128>(ta, tb, g, grid, st); break;
    default: e = launch_gemm_bn<256>(ta, tb, g, grid, st); break;
  }
  if (e != cudaSuccess) {
    err = std::string("GEMM launch: ") + cudaGetErrorString(e);
    return BOWSHOCK_CUDA_ERROR;
  }
  return 0;
}

template <int BN>
static cudaError_t launch_conv_bn(const CUtensorMap& tb, const GemmArgs& g, dim3 grid, cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(k_gemm_conv<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, gemm_smem_bytes<BN>());
  if (e != cudaSuccess) return e;
  k_gemm_conv<BN><<<grid, 128, gemm_smem_bytes<BN>(), st>>>(tb, g);
  return cudaGetLastError();
}

// D[p, n] = sum over taps and channels of x[pixel p shifted by the tap][c] w[n][tap * C + c]: the 3x3 'same'
// convolution of the NHWC input x [B, Hin, Win, C] (C a multiple of 64, read through a 2x upsampling when up = 1) by the
// weights w [N, 9 C] (BF16, ldw elements per row) as an implicit GEMM (no im2col matrix); the epilogue as in g.
static int conv_gemm(const bf16* x, int B, int Hin, int Win, int C, int up, const bf16* w, long long ldw, int N, GemmArgs g, cudaStream_t st,
                     std::string& err) {
  if (C % 64) {
    err = "the implicit-GEMM convolution needs a multiple of 64 input channels";
    return BOWSHOCK_INVALID;
  }
  if (!get_encode(err)) return BOWSHOCK_CUDA_ERROR;
  const int bn = pick_bn(N);
  const long long M = (long long)B * (Hin << up) * (Win << up);
  CUtensorMap tb;
  if (!make_map(&tb, w, N, 9LL * C, ldw, bn, err)) return BOWSHOCK_INVALID;
  if (((uintptr_t)x & 15)) {
    err = "convolution input not 16-byte aligned";
    return BOWSHOCK_INVALID;
  }
  g.M = (int)M, g.N = N, g.K = 9 * C, g.kb_per_split = (9 * C) / BK;
  g.cx = x, g.cB = B, g.cHin = Hin, g.cWin = Win, g.cC = C, g.cup = up;
  dim3 grid((unsigned)((M + BM - 1) / BM), (unsigned)((N + bn - 1) / bn), 1);
  cudaError_t e;
  switch (bn) {
    case 16: e = launch_conv_bn<16>(tb, g, grid, st); break;
    case 32: e = launch_conv_bn<32>(tb, g, grid, st); break;
    case 64: e = launch_conv_bn<64>(tb, g, grid, st); break;
    case 128: e = launch_conv_bn<128>(tb, g, grid, st); break;
    default: e = launch_conv_bn<256>(tb, g, grid, st); break;
  }
  if (e != cudaSuccess) {
    err = std::string("convolution GEMM launch: ") + cudaGetErrorString(e);
    return BOWSHOCK_CUDA_ERROR;
  }
  return 0;
}

// Whether the TMA-fed convolution (k_gemm<BN, true>) takes an H x W image: its 128-pixel tiles must be whole rows of one
// image (H W a multiple of 128) or whole images (128 a multiple of H W), W dividing 128.
static bool conv_tma_fits(int H, int W) { return W >= 1 && W <= 128 && 128 % W == 0 && ((H * W) % 128 == 0 || 128 % (H * W) == 0); }

// The same convolution as conv_gemm (no upsampling) with both operands loaded by TMA: A through a 4D tensor map over the
// NHWC activations x [B, H, W, C] (box: 64 channels x W x R rows x NB images = 128 pixels, 128-byte swizzle, zeros
// outside), one box per K block at the tile's first pixel shifted by the tap.
static int conv_gemm_tma(const bf16* x, int B, int H, int W, int C, const bf16* w, long long ldw, int N, GemmArgs g, cudaStream_t st, std::string& err) {
  if (C % 64 || !conv_tma_fits(H, W)) {
    err = "the TMA convolution needs a multiple of 64 channels and 128-pixel tiles of whole rows or images";
    return BOWSHOCK_INVALID;
  }
  if (!get_encode(err)) return BOWSHOCK_CUDA_ERROR;
  if (((uintptr_t)x & 15)) {
    err = "convolution input not 16-byte aligned";
    return BOWSHOCK_INVALID;
  }
  const int bn = pick_bn(N);
  const int R = std::min(H, 128 / W), NB = 128 / (W * R);
  CUtensorMap ta, tb;
  cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
  cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
  cuuint32_t box[4] = {(cuuint32_t)BK, (cuuint32_t)W, (cuuint32_t)R, (cuuint32_t)NB};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = g_encode(&ta, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(x), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    err = "cuTensorMapEncodeTiled (4D activations) failed (" + std::to_string((int)r) + ")";
    return BOWSHOCK_INVALID;
  }
  if (!make_map(&tb, w, N, 9LL * C, ldw, bn, err)) return BOWSHOCK_INVALID;
  const long long M = (long long)B * H * W;
  g.M = (int)M, g.N = N, g.K = 9 * C, g.kb_per_split = (9 * C) / BK;
  g.cx = x, g.cB = B, g.cHin = H, g.cWin = W, g.cC = C, g.cup = 0;
  dim3 grid((unsigned)((M + BM - 1) / BM), (unsigned)((N + bn - 1) / bn), 1);
  cudaError_t e;
  switch (bn) {
    case 16: e = launch_gemm_bn<16, GEMM_CONV>(ta, tb, g, grid, st); break;
    case 32: e = launch_gemm_bn<32, GEMM_CONV>(ta, tb, g, grid, st); break;
    case 64: e = launch_gemm_bn<64, GEMM_CONV>(ta, tb, g, grid, st); break;
    case 128: e = launch_gemm_bn<128, GEMM_CONV>(ta, tb, g, grid, st); break;
    default: e = launch_gemm_bn<256, GEMM_CONV>(ta, tb, g, grid, st); break;
  }
  if (e != cudaSuccess) {
    err = std::string("convolution GEMM launch: ") + cudaGetErrorString(e);
    return BOWSHOCK_CUDA_ERROR;
  }
  return 0;
}

// The weight-gradient operands of a layer W <= 64 pixels wide (W dividing 64), on a row pitch of 64 pixels: x [rows W]
// [C] (rows = B H image rows) -> out [C][rows 64], out[c][row 64 + x] = x[row W + x][c] for x < W and 0 for the padding
// x >= W; with SHIFT3, three such planes shifted along x, out[s][c][row 64 + x] = x[row W + x + s - 1][c] where both x
// and x + s - 1 lie in [0, W), else 0. One image row (blockIdx.x) x 32 channels (blockIdx.y) per block through shared memory: coalesced reads of
// the pixels' channels, 128-byte rows written as BF16 pairs (the last channel block may be partial).
template <bool SHIFT3>
__global__ void __launch_bounds__(256) k_transpose_rows(const bf16* __restrict__ x, int C, int W, long long rows, bf16* __restrict__ out) {
  constexpr int P64 = 64, NS = SHIFT3 ? 3 : 1;
  __shared__ bf16 t[32][P64 + 2];
  const int c0 = blockIdx.y * 32, tx = threadIdx.x, ty = threadIdx.y;
  const long long row = blockIdx.x, pitch = rows * P64;
  const bf16 z = __float2bfloat16_rn(0.f);
#pragma unroll
  for (int q = ty; q < P64; q += 8) t[tx][q] = (q < W && c0 + tx < C) ? x[(row * W + q) * C + c0 + tx] : z;
  __syncthreads();
#pragma unroll 1
  for (int idx = ty; idx < NS * 32; idx += 8) {
    const int sft = SHIFT3 ? idx / 32 - 1 : 0, c = idx % 32, xa = 2 * tx, a = xa + sft, b = a + 1;
    if (c0 + c >= C) continue;
    __nv_bfloat162 v;
    v.x = (xa < W && a >= 0 && a < W) ? t[c][a] : z;
    v.y = (xa + 1 < W && b >= 0 && b < W) ? t[c][b] : z;
    reinterpret_cast<__nv_bfloat162*>(out + ((long long)(SHIFT3 ? sft + 1 : 0) * C + c0 + c) * pitch + row * P64)[tx] = v;
  }
}

// The weight gradient of a 3x3 'same' convolution: dw [cout, 9 cin] (FP32, accumulated atomically over split-K slices;
// zeroed by the caller) = sum over the pixels of gT[o][p] x[p shifted by the tap][c], gT the output gradient and xs
// the layer's input, both transposed onto a row pitch of 64 pixels (k_transpose_rows: gT [cout][B H 64], xs [3][cin]
// [B][H][64] with the shifted copies; the padding pixels are zeros on both sides, so they add nothing). cin a multiple
// of 64.
static int wgrad_gemm_tma(const bf16* gT, const bf16* xs, int B, int H, int cin, int cout, float* dw, int* err_flag, cudaStream_t st, std::string& err) {
  constexpr int W = 64;
  if (cin % 64) {
    err = "the TMA weight gradient needs a multiple of 64 input channels";
    return BOWSHOCK_INVALID;
  }
  if (!get_encode(err)) return BOWSHOCK_CUDA_ERROR;
  const int bn = cin % 128 == 0 ? 128 : 64;
  const long long r = (long long)B * H * W;
  CUtensorMap ta, tb;
  if (!make_map(&ta, gT, cout, r, r, BM, err)) return BOWSHOCK_INVALID;
  if (((uintptr_t)xs & 15)) {
    err = "transposed activations not 16-byte aligned";
    return BOWSHOCK_INVALID;
  }
  cuuint64_t dims[4] = {(cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B, 3ULL * cin};
  cuuint64_t strides[3] = {(cuuint64_t)W * 2, (cuuint64_t)H * W * 2, (cuuint64_t)r * 2};
  cuuint32_t box[4] = {(cuuint32_t)W, 1, 1, (cuuint32_t)bn};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult rr = g_encode(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(xs), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (rr != CUDA_SUCCESS) {
    err = "cuTensorMapEncodeTiled (4D transposed activations) failed (" + std::to_string((int)rr) + ")";
    return BOWSHOCK_INVALID;
  }
  GemmArgs g{};
  g.err = err_flag, g.mode = EPI_F32_ATOMIC, g.d = dw, g.ldd = 9LL * cin;
  const int nkb = (int)(r / BK);  // one image row per K block
  const int tiles = ((cout + BM - 1) / BM) * (9 * cin / bn);
  int splits = std::max(1, std::min(nkb, 2 * 148 / tiles));
  const int per = (nkb + splits - 1) / splits;
  splits = (nkb + per - 1) / per;
  g.M = cout, g.N = 9 * cin, g.K = (int)r, g.kb_per_split = per;
  g.cHin = H, g.cWin = W, g.cC = cin;
  dim3 grid((unsigned)((cout + BM - 1) / BM), (unsigned)(9 * cin / bn), (unsigned)splits);
  const cudaError_t e = bn == 128 ? launch_gemm_bn<128, GEMM_WGRAD>(ta, tb, g, grid, st) : launch_gemm_bn<64, GEMM_WGRAD>(ta, tb, g, grid, st);
  if (e != cudaSuccess) {
    err = std::string("weight-gradient GEMM launch: ") + cudaGetErrorString(e);
    return BOWSHOCK_CUDA_ERROR;
  }
  return 0;
}

static int grid_for(long long n, int threads = 256) { return (int)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148 * 16)); }

// y [B, 2 Hin, 2 Win, C] = x [B, Hin, Win, C] repeated 2 x 2 (nearest upsampling), 8 channels (16 bytes) per thread step
__global__ void k_upsample2x(const bf16* __restrict__ x, int B, int Hin, int Win, int C, bf16* __restrict__ y) {
  const int H = Hin * 2, W = Win * 2, c8 = C >> 3;
  const long long total = (long long)B * H * W * c8;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int cc = (int)(t % c8);
    const long long p = t / c8;
    const int xo = (int)(p % W), yo = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
    reinterpret_cast<uint4*>(y)[p * c8 + cc] = reinterpret_cast<const uint4*>(x)[(((long long)b * Hin + (yo >> 1)) * Win + (xo >> 1)) * c8 + cc];
  }
}

// ---------------------------------------------------------------------------------------------------- the network
struct Layer {
  int fc;         // fully connected (else 3x3 convolution)
  int cin, cout;  // channels (features of a fully connected layer)
  int H, W;       // output resolution (convolutions)
  int up;         // nearest 2x upsampling of the input before the convolution
  int act;        // leaky ReLU (else the linear output layer, FP32)
  long long kin;  // GEMM K: cin (fully connected) or 9 cin
  long long woff, boff;  // offsets of W [cout, kin] and b [cout] in the flat parameter vector
};

struct Net {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  std::vector<Layer> L;
  int maxB = 0;
  long long nparam = 0;
  float *w = nullptr, *gw = nullptr, *m1 = nullptr, *m2 = nullptr;  // FP32 masters, gradients, Adam moments
  bf16* wb = nullptr;                                                 // BF16 copies (same offsets)
  bf16* x = nullptr;                                                  // [maxB, NET_IN]
  std::vector<bf16*> act;                                             // per layer output [rows, cout] (the last layer: none)
  float* out = nullptr;                                               // last layer [rows, 16] FP32
  bf16 *col = nullptr, *colT = nullptr, *gT = nullptr, *wt = nullptr, *g0 = nullptr, *g1 = nullptr;
  float* dx = nullptr;
  float* loss = nullptr;   // per training step
  float* loss1 = nullptr;  // one gradient evaluation
  int* d_err = nullptr;
  int* d_step = nullptr;
  int* d_tstep = nullptr;  // index of the training step within a bowshock_net_train call (read by a replayed step)
  float* coef = nullptr;
  // dataset on the device
  float *dsx = nullptr, *dst = nullptr, *tb = nullptr;
  uint8_t* mask = nullptr;
  long long nds = 0;
  int* idx = nullptr;
  long long idx_cap = 0;
  double last_ms = 0.0;
  long long cap_col = 0, cap_rows = 0;  // elements of col / colT and of gT / g0 / g1
  int conv_mode = 2;  // 3x3 convolutions of 64k channels: 0 im2col + GEMM, 1 implicit GEMM (cp.async gather), 2 implicit GEMM (TMA boxes)

  ~Net() {
    for (void* p : {(void*)w, (void*)gw, (void*)m1, (void*)m2, (void*)wb, (void*)x, (void*)out, (void*)col, (void*)colT, (void*)gT, (void*)wt,
                    (void*)g0, (void*)g1, (void*)dx, (void*)loss, (void*)loss1, (void*)d_err, (void*)d_step, (void*)d_tstep, (void*)coef, (void*)dsx, (void*)dst, (void*)tb,
                    (void*)mask, (void*)idx})
      if (p) cudaFree(p);
    for (bf16* a : act)
      if (a) cudaFree(a);
    if (stream) cudaStreamDestroy(stream);
  }

  long long rows(const Layer& l, int B) const { return l.fc ? (long long)B : (long long)B * l.H * l.W; }

  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
#define NCK(x)                                                                \
  do {                                                                        \
    cudaError_t e_ = (x);                                                     \
    if (e_ != cudaSuccess) return fail(BOWSHOCK_CUDA_ERROR, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

  int create(int dev, int max_batch) {
    device = dev;
    maxB = max_batch;
    NCK(cudaSetDevice(device));
    NCK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    // the decoder: 16 inputs -> 256 -> 4 x 8 x 128 -> (conv 3x3, leaky ReLU) at 4 x 8, 8 x 16, 16 x 32, 32 x 64 -> 16 channels
    auto fc = [&](int cin, int cout) { L.push_back(Layer{1, cin, cout, 1, 1, 0, 1, cin, 0, 0}); };
    auto cv = [&](int cin, int cout, int H, int W, int up, int act) { L.push_back(Layer{0, cin, cout, H, W, up, act, 9LL * cin, 0, 0}); };
    fc(BOWSHOCK_NET_IN, 256);
    fc(256, 4 * 8 * 128);
    cv(128, 128, 4, 8, 0, 1);
    cv(128, 128, 4, 8, 0, 1);
    cv(128, 128, 8, 16, 1, 1);
    cv(128, 128, 8, 16, 0, 1);
    cv(128, 64, 16, 32, 1, 1);
    cv(64, 64, 16, 32, 0, 1);
    cv(64, 64, 32, 64, 1, 1);
    cv(64, 64, 32, 64, 0, 1);
    cv(64, BOWSHOCK_NET_OUT_PAD, 32, 64, 0, 0);
    long long off = 0;
    for (auto& l : L) {
      l.woff = off, off += (long long)l.cout * l.kin;
      l.boff = off, off += l.cout;
      off = (off + 7) & ~7LL;  // every W starts 16-byte aligned
    }
    nparam = off;
    NCK(cudaMalloc(&w, nparam * 4));
    NCK(cudaMalloc(&gw, nparam * 4));
    NCK(cudaMalloc(&m1, nparam * 4));
    NCK(cudaMalloc(&m2, nparam * 4));
    NCK(cudaMalloc(&wb, nparam * 2));
    NCK(cudaMemsetAsync(w, 0, nparam * 4, stream));
    NCK(cudaMemsetAsync(wb, 0, nparam * 2, stream));
    NCK(cudaMalloc(&x, (size_t)maxB * BOWSHOCK_NET_IN * 2));
    act.assign(L.size(), nullptr);
    long long max_col = 0, max_rows_c = 0;  // elements of the im2col buffers and of the gradient buffers
    for (size_t k = 0; k < L.size(); ++k) {
      const Layer& l = L[k];
      const long long r = rows(l, maxB);
      if (k + 1 < L.size()) NCK(cudaMalloc(&act[k], r * l.cout * 2));
      max_col = std::max(max_col, r * l.kin);
      if (!l.fc) max_col = std::max(max_col, r * 9LL * l.cout);  // im2col of the output gradient
      max_rows_c = std::max(max_rows_c, r * std::max<long long>(l.cout, l.cin));
    }
    const Layer& lo = L.back();
    NCK(cudaMalloc(&out, rows(lo, maxB) * lo.cout * 4));
    cap_col = max_col, cap_rows = max_rows_c;
    NCK(cudaMalloc(&col, max_col * 2));
    NCK(cudaMalloc(&colT, max_col * 2));
    NCK(cudaMalloc(&gT, max_rows_c * 2));
    NCK(cudaMalloc(&g0, max_rows_c * 2));
    NCK(cudaMalloc(&g1, max_rows_c * 2));
    NCK(cudaMalloc(&dx, max_rows_c * 4));
    long long maxw = 0;
    for (auto& l : L) maxw = std::max(maxw, (long long)l.cout * l.kin);
    NCK(cudaMalloc(&wt, maxw * 2));
    NCK(cudaMalloc(&d_err, sizeof(int)));
    NCK(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
    NCK(cudaMalloc(&d_step, sizeof(int)));
    NCK(cudaMalloc(&d_tstep, sizeof(int)));
    NCK(cudaMalloc(&coef, sizeof(float)));
    NCK(cudaMalloc(&loss1, sizeof(float)));
    NCK(cudaMalloc(&tb, (size_t)maxB * BOWSHOCK_NET_CELLS * BOWSHOCK_NET_OUT * 4));
    NCK(cudaMalloc(&mask, BOWSHOCK_NET_CELLS));
    NCK(cudaMemsetAsync(mask, 1, BOWSHOCK_NET_CELLS, stream));
    return reset_optimizer();
  }

  int reset_optimizer() {
    NCK(cudaMemsetAsync(m1, 0, nparam * 4, stream));
    NCK(cudaMemsetAsync(m2, 0, nparam * 4, stream));
    NCK(cudaMemsetAsync(d_step, 0, sizeof(int), stream));
    NCK(cudaStreamSynchronize(stream));
    return 0;
  }

  int set_params(const float* h) {
    NCK(copy_sync(stream, w, h, nparam * 4, cudaMemcpyHostToDevice));
    k_to_bf16<<<grid_for(nparam), 256, 0, stream>>>(w, nparam, wb);
    NCK(cudaGetLastError());
    NCK(cudaStreamSynchronize(stream));
    return 0;
  }

  int check_err() {
    int h = 0;
    NCK(copy_sync(stream, &h, d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
      cudaMemsetAsync(d_err, 0, sizeof(int), stream);
      cudaStreamSynchronize(stream);
      return fail(BOWSHOCK_TIMEOUT, "a tensor-core GEMM gave up waiting on its pipeline (bounded wait)");
    }
    return 0;
  }

  // forward pass of batch B from the BF16 input in x; every layer's output kept for the backward pass
  int forward(int B) {
    int rc;
    const bf16* in = x;
    for (size_t k = 0; k < L.size(); ++k) {
      const Layer& l = L[k];
      const long long r = rows(l, B);
      GemmArgs g{};
      g.err = d_err;
      g.bias = w + l.boff;
      const bf16* A;
      long long lda;
      if (l.act) {
        g.mode = EPI_BIAS_ACT_BF16, g.y = act[k], g.ldy = l.cout, g.slope = BOWSHOCK_NET_SLOPE;
      } else {
        g.mode = EPI_BIAS_F32, g.d = out, g.ldd = l.cout;
      }
      if (!l.fc && conv_mode == 2 && l.cin % 64 == 0 && conv_tma_fits(l.H, l.W)) {  // implicit GEMM, A tiles by TMA
        const bf16* src = in;
        if (l.up) {  // the TMA boxes read the upsampled activations (the im2col buffer holds them)
          k_upsample2x<<<grid_for((long long)B * l.H * l.W * (l.cin / 8)), 256, 0, stream>>>(in, B, l.H >> 1, l.W >> 1, l.cin, col);
          src = col;
        }
        if ((rc = conv_gemm_tma(src, B, l.H, l.W, l.cin, wb + l.woff, l.kin, l.cout, g, stream, err))) return rc;
        in = act[k];
        continue;
      }
      if (!l.fc && conv_mode >= 1 && l.cin % 64 == 0) {  // implicit GEMM, A tiles gathered by cp.async
        if ((rc = conv_gemm(in, B, l.H >> l.up, l.W >> l.up, l.cin, l.up, wb + l.woff, l.kin, l.cout, g, stream, err))) return rc;
        in = act[k];
        continue;
      }
      if (l.fc) {
        A = in, lda = l.cin;
      } else {
        const int Hin = l.H >> l.up, Win = l.W >> l.up;
        k_im2col<<<grid_for(r * 9 * (l.cin / 8)), 256, 0, stream>>>(in, B, Hin, Win, l.cin, l.up, col);
        A = col, lda = l.kin;
      }
      if ((rc = gemm(A, lda, wb + l.woff, l.kin, (int)r, l.cout, (int)l.kin, g, 1, stream, err))) return rc;
      in = act[k];
    }
    NCK(cudaGetLastError());
    return 0;
  }

  // gradients of the masked loss into gw (zeroed here), from the target batch in tb; loss summed into *loss_slot
  int backward(int B, float* loss_slot, const int* tstep = nullptr) {
    int rc;
    NCK(cudaMemsetAsync(gw, 0, nparam * 4, stream));
    const Layer& lo = L.back();
    const long long ro = rows(lo, B);
    const float inv = 1.f / (float)((long long)B * BOWSHOCK_NET_CELLS * BOWSHOCK_NET_OUT);  // mean over every entry (masked ones are 0)
    k_loss<<<grid_for(ro * lo.cout), 256, 0, stream>>>(out, lo.cout, tb, BOWSHOCK_NET_OUT, mask, BOWSHOCK_NET_CELLS, ro, inv, g0, loss_slot, tstep);
    bf16 *g = g0, *gnext = g1;
    for (int k = (int)L.size() - 1; k >= 0; --k) {
      const Layer& l = L[k];
      const long long r = rows(l, B);
      const bf16* xin = k > 0 ? act[k - 1] : x;
      // dW [cout, kin] = g^T X: K = rows. A convolution up to 64 pixels wide runs the TMA weight gradient: g and the
      // input transposed onto a row pitch of 64 pixels (zero padding), the input also in its three x-shifted copies
      const long long rows64 = (long long)B * l.H * 64;
      const bool wg = !l.fc && conv_mode == 2 && l.W <= 64 && 64 % l.W == 0 && l.cin % 64 == 0 && l.cout % 8 == 0 &&
                      (long long)l.cout * rows64 <= cap_rows && 3LL * l.cin * rows64 <= cap_col;
      if (wg) {
        k_transpose_rows<false><<<dim3((unsigned)(B * l.H), (unsigned)((l.cout + 31) / 32)), dim3(32, 8), 0, stream>>>(g, l.cout, l.W, (long long)B * l.H, gT);
      } else {
        dim3 tg((unsigned)((l.cout + 31) / 32), (unsigned)((r + 31) / 32));
        k_transpose<<<tg, dim3(32, 8), 0, stream>>>(g, l.cout, (int)r, l.cout, gT, r);
      }
      const bf16* XT;
      if (wg) {
        // the input (upsampled first where the layer upsamples) into one of the im2col buffers, its shifted copies
        // into the other, the taps' boxes loaded from those by TMA
        const bf16* src = xin;
        if (l.up) {
          k_upsample2x<<<grid_for(r * (l.cin / 8)), 256, 0, stream>>>(xin, B, l.H >> 1, l.W >> 1, l.cin, col);
          src = col;
        }
        bf16* xs = src == col ? colT : col;
        k_transpose_rows<true><<<dim3((unsigned)(B * l.H), (unsigned)(l.cin / 32)), dim3(32, 8), 0, stream>>>(src, l.cin, l.W, (long long)B * l.H, xs);
        if ((rc = wgrad_gemm_tma(gT, xs, B, l.H, l.cin, l.cout, gw + l.woff, d_err, stream, err))) return rc;
        XT = nullptr;
      } else if (l.fc) {
        dim3 tx((unsigned)((l.cin + 31) / 32), (unsigned)((r + 31) / 32));
        k_transpose<<<tx, dim3(32, 8), 0, stream>>>(xin, l.cin, (int)r, l.cin, colT, r);
        XT = colT;
      } else {
        const int Hin = l.H >> l.up, Win = l.W >> l.up;
        dim3 tx((unsigned)((r + 31) / 32), (unsigned)(9 * ((l.cin + 31) / 32)));
        k_im2col_t<<<tx, dim3(32, 8), 0, stream>>>(xin, B, Hin, Win, l.cin, l.up, colT, r);
        XT = colT;
      }
      GemmArgs gd{};
      gd.err = d_err, gd.mode = EPI_F32_ATOMIC, gd.d = gw + l.woff, gd.ldd = l.kin;
      const int tiles = ((l.cout + BM - 1) / BM) * (int)((l.kin + pick_bn((int)l.kin) - 1) / pick_bn((int)l.kin));
      const int splits = std::max(1, 2 * 148 / tiles);
      if (XT && (rc = gemm(gT, r, XT, r, l.cout, (int)l.kin, (int)r, gd, splits, stream, err))) return rc;
      k_bias_grad<<<dim3((unsigned)((l.cout + 31) / 32), (unsigned)std::min<long long>(1024, (r + 255) / 256)), dim3(32, 8), 0, stream>>>(
          g, r, l.cout, gw + l.boff);
      if (k == 0) break;
      // dX = g W (through the flipped convolution); then the previous layer's leaky ReLU derivative
      GemmArgs gx{};
      gx.err = d_err, gx.mode = EPI_F32, gx.d = dx, gx.ldd = l.cin;
      if (l.fc) {
        dim3 tw((unsigned)((l.kin + 31) / 32), (unsigned)((l.cout + 31) / 32));
        k_transpose<<<tw, dim3(32, 8), 0, stream>>>(wb + l.woff, l.kin, l.cout, (int)l.kin, wt, l.cout);
        if ((rc = gemm(g, l.cout, wt, l.cout, (int)r, l.cin, l.cout, gx, 1, stream, err))) return rc;
        k_grad_prev<<<grid_for(r * l.cin), 256, 0, stream>>>(dx, B, 1, 1, l.cin, 0, xin, BOWSHOCK_NET_SLOPE, gnext);
      } else {
        k_flip_weights<<<grid_for((long long)l.cin * 9 * l.cout), 256, 0, stream>>>(wb + l.woff, l.cin, l.cout, wt);
        if (conv_mode == 2 && l.cout % 64 == 0 && conv_tma_fits(l.H, l.W)) {
          if ((rc = conv_gemm_tma(g, B, l.H, l.W, l.cout, wt, 9LL * l.cout, l.cin, gx, stream, err))) return rc;
        } else if (conv_mode >= 1 && l.cout % 64 == 0) {
          if ((rc = conv_gemm(g, B, l.H, l.W, l.cout, 0, wt, 9LL * l.cout, l.cin, gx, stream, err))) return rc;
        } else {
          k_im2col<<<grid_for(r * 9 * (l.cout / 8)), 256, 0, stream>>>(g, B, l.H, l.W, l.cout, 0, col);
          if ((rc = gemm(col, 9LL * l.cout, wt, 9LL * l.cout, (int)r, l.cin, 9 * l.cout, gx, 1, stream, err))) return rc;
        }
        // the previous layer's output resolution (a fully connected layer's 4096 features are the 4 x 8 x 128 map)
        const int Hin = l.H >> l.up, Win = l.W >> l.up;
        k_grad_prev<<<grid_for((long long)B * Hin * Win * l.cin), 256, 0, stream>>>(dx, B, Hin, Win, l.cin, l.up, xin, BOWSHOCK_NET_SLOPE, gnext);
      }
      std::swap(g, gnext);
    }
    NCK(cudaGetLastError());
    return 0;
  }

  void adam(float lr, int* tstep = nullptr) {
    k_adam_prep<<<1, 1, 0, stream>>>(d_step, coef, lr, 0.9f, 0.999f, tstep);
    k_adam<<<grid_for(nparam), 256, 0, stream>>>(w, m1, m2, gw, nparam, coef, 0.9f, 0.999f, 1e-8f, wb);
  }

  // one training step of batch B on the dataset rows idx_dev[0..B): gather, forward, loss, backward, Adam
  // tstep (may be null): idx_dev and loss_slot are the bases of every step's indices and losses, offset on the device by
  // the step index *tstep, which the step advances (so that one captured step replays as every step)
  int train_step(int B, const int* idx_dev, float lr, float* loss_slot, int* tstep = nullptr) {
    k_gather<<<grid_for((long long)B * BOWSHOCK_NET_CELLS * BOWSHOCK_NET_OUT), 256, 0, stream>>>(
        dsx, BOWSHOCK_NET_IN, dst, (long long)BOWSHOCK_NET_CELLS * BOWSHOCK_NET_OUT, idx_dev, B, x, tb, tstep);
    int rc;
    if ((rc = forward(B))) return rc;
    if ((rc = backward(B, loss_slot, tstep))) return rc;
    adam(lr, tstep);
    NCK(cudaGetLastError());
    return 0;
  }
#undef NCK
};

}  // namespace bknet

// ================================================================================================ C ABI
using bknet::Net;
struct bowshock_net {
  Net n;
};

#define NET_CK(h, x)                                                                                  \
  do {                                                                                                \
    cudaError_t e_ = (x);                                                                             \
    if (e_ != cudaSuccess) {                                                                          \
      (h)->n.err = std::string(#x) + ": " + cudaGetErrorString(e_);                                  \
      return BOWSHOCK_CUDA_ERROR;                                                                     \
    }                                                                                                 \
  } while (0)

extern "C" {

int bowshock_net_create(int device, uint64_t max_batch, bowshock_net** out) {
  if (!out || max_batch == 0 || max_batch % 8 || max_batch > 4096) return BOWSHOCK_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return BOWSHOCK_CUDA_ERROR;
  auto* h = new bowshock_net();
  int rc = h->n.create(device, (int)max_batch);
  if (rc) {
    delete h;
    return rc;
  }
  *out = h;
  return BOWSHOCK_OK;
}

void bowshock_net_destroy(bowshock_net* h) {
  if (!h) return;
  cudaSetDevice(h->n.device);
  delete h;
}

const char* bowshock_net_last_error(const bowshock_net* h) { return h ? h->n.err.c_str() : "null handle"; }

int bowshock_net_num_params(const bowshock_net* h, uint64_t* n) {
  if (!h || !n) return BOWSHOCK_INVALID;
  *n = (uint64_t)h->n.nparam;
  return BOWSHOCK_OK;
}

int bowshock_net_layout(const bowshock_net* h, int64_t* out, uint64_t cap, uint64_t* nlayers) {
  if (!h || !nlayers) return BOWSHOCK_INVALID;
  *nlayers = h->n.L.size();
  if (!out) return BOWSHOCK_OK;
  for (size_t k = 0; k < h->n.L.size() && 9 * (k + 1) <= cap; ++k) {
    const bknet::Layer& l = h->n.L[k];
    int64_t* o = out + 9 * k;
    o[0] = l.fc, o[1] = l.cin, o[2] = l.cout, o[3] = l.H, o[4] = l.W, o[5] = l.up, o[6] = l.act, o[7] = l.woff, o[8] = l.boff;
  }
  return BOWSHOCK_OK;
}

int bowshock_net_set_params(bowshock_net* h, const float* p) {
  if (!h || !p) return BOWSHOCK_INVALID;
  NET_CK(h, cudaSetDevice(h->n.device));
  return h->n.set_params(p);
}

int bowshock_net_get_params(bowshock_net* h, float* p) {
  if (!h || !p) return BOWSHOCK_INVALID;
  NET_CK(h, cudaSetDevice(h->n.device));
  NET_CK(h, cudaStreamSynchronize(h->n.stream));
  NET_CK(h, copy_sync(h->n.stream, p, h->n.w, h->n.nparam * 4, cudaMemcpyDeviceToHost));
  return BOWSHOCK_OK;
}

int bowshock_net_set_mask(bowshock_net* h, const uint8_t* mask) {
  if (!h || !mask) return BOWSHOCK_INVALID;
  NET_CK(h, cudaSetDevice(h->n.device));
  NET_CK(h, copy_sync(h->n.stream, h->n.mask, mask, BOWSHOCK_NET_CELLS, cudaMemcpyHostToDevice));
  return BOWSHOCK_OK;
}

int bowshock_net_forward(bowshock_net* h, uint64_t batch, const float* x, float* y) {
  if (!h || !x || !y || batch == 0) return BOWSHOCK_INVALID;
  Net& n = h->n;
  NET_CK(h, cudaSetDevice(n.device));
  const int rc_err = n.check_err();
  if (rc_err) return rc_err;
  for (uint64_t b0 = 0; b0 < batch; b0 += (uint64_t)n.maxB) {
    const int B = (int)std::min<uint64_t>(batch - b0, (uint64_t)n.maxB);
    std::vector<bknet::bf16> xb((size_t)B * BOWSHOCK_NET_IN);
    for (size_t q = 0; q < xb.size(); ++q) xb[q] = __float2bfloat16_rn(x[b0 * BOWSHOCK_NET_IN + q]);
    NET_CK(h, cudaMemcpyAsync(n.x, xb.data(), xb.size() * 2, cudaMemcpyHostToDevice, n.stream));
    int rc = n.forward(B);
    if (rc) return rc;
    const bknet::Layer& lo = n.L.back();
    NET_CK(h, cudaMemcpy2DAsync(y + b0 * BOWSHOCK_NET_CELLS * BOWSHOCK_NET_OUT, BOWSHOCK_NET_OUT * 4, n.out, (size_t)lo.cout * 4,
                                BOWSHOCK_NET_OUT * 4, (size_t)B * BOWSHOCK_NET_CELLS, cudaMemcpyDeviceToHost, n.stream));
    NET_CK(h, cudaStreamSynchronize(n.stream));
  }
  return n.check_err();
}

int bowshock_net_gradients(bowshock_net* h, uint64_t batch, const float* x, const float* target, float* grad, double* loss) {
  if (!h || !x || !target || batch == 0 || batch % 8 || batch > (uint64_t)h->n.maxB) return BOWSHOCK_INVALID;
  Net& n = h->n;
  NET_CK(h, cudaSetDevice(n.device));
  const int B = (int)batch;
  std::vector<bknet::bf16> xb((size_t)B * BOWSHOCK_NET_IN);
  for (size_t q = 0; q < xb.size(); ++q) xb[q] = __float2bfloat16_rn(x[q]);
  NET_CK(h, cudaMemcpyAsync(n.x, xb.data(), xb.size() * 2, cudaMemcpyHostToDevice, n.stream));
  NET_CK(h, cudaMemcpyAsync(n.tb, target, (size_t)B * BOWSHOCK_NET_CELLS * BOWSHOCK_NET_OUT * 4, cudaMemcpyHostToDevice, n.stream));
  float* dl = n.loss1;
  NET_CK(h, cudaMemsetAsync(dl, 0, sizeof(float), n.stream));
  int rc = n.forward(B);
  if (!rc) rc = n.backward(B, dl);
  float hl = 0.f;
  if (!rc) {
    NET_CK(h, cudaMemcpyAsync(&hl, dl, sizeof(float), cudaMemcpyDeviceToHost, n.stream));
    if (grad) NET_CK(h, cudaMemcpyAsync(grad, n.gw, n.nparam * 4, cudaMemcpyDeviceToHost, n.stream));
  }
  NET_CK(h, cudaStreamSynchronize(n.stream));
  if (rc) return rc;
  if (loss) *loss = hl;
  return n.check_err();
}

int bowshock_net_set_dataset(bowshock_net* h, uint64_t n_samples, const float* x, const float* target) {
  if (!h || !x || !target || n_samples == 0) return BOWSHOCK_INVALID;
  Net& n = h->n;
  NET_CK(h, cudaSetDevice(n.device));
  if (n.dsx) cudaFree(n.dsx), n.dsx = nullptr;
  if (n.dst) cudaFree(n.dst), n.dst = nullptr;
  const size_t nt = (size_t)BOWSHOCK_NET_CELLS * BOWSHOCK_NET_OUT;
  NET_CK(h, cudaMalloc(&n.dsx, n_samples * BOWSHOCK_NET_IN * 4));
  NET_CK(h, cudaMalloc(&n.dst, n_samples * nt * 4));
  NET_CK(h, copy_sync(n.stream, n.dsx, x, n_samples * BOWSHOCK_NET_IN * 4, cudaMemcpyHostToDevice));
  NET_CK(h, copy_sync(n.stream, n.dst, target, n_samples * nt * 4, cudaMemcpyHostToDevice));
  n.nds = (long long)n_samples;
  return BOWSHOCK_OK;
}

int bowshock_net_reset_optimizer(bowshock_net* h) {
  if (!h) return BOWSHOCK_INVALID;
  NET_CK(h, cudaSetDevice(h->n.device));
  return h->n.reset_optimizer();
}

int bowshock_net_train(bowshock_net* h, uint64_t steps, uint64_t batch, double lr, uint64_t seed, double* loss) {
  if (!h || steps == 0 || batch == 0 || batch % 8 || batch > (uint64_t)h->n.maxB) return BOWSHOCK_INVALID;
  Net& n = h->n;
  if (!n.dsx || (uint64_t)n.nds < batch) {
    n.err = "no dataset of at least one batch (bowshock_net_set_dataset)";
    return BOWSHOCK_INVALID;
  }
  NET_CK(h, cudaSetDevice(n.device));
  const int B = (int)batch;
  // the batches of every step: epochs of a seeded shuffle of the dataset (each epoch drops its last partial batch)
  std::vector<int> order(n.nds);
  std::mt19937_64 rng(seed);
  const long long per_epoch = n.nds / B;
  std::vector<int> idx((size_t)steps * B);
  for (uint64_t s = 0; s < steps; ++s) {
    const long long e = (long long)s % per_epoch;
    if (e == 0) {
      for (long long q = 0; q < n.nds; ++q) order[q] = (int)q;
      std::shuffle(order.begin(), order.end(), rng);
    }
    for (int b = 0; b < B; ++b) idx[s * B + b] = order[e * B + b];
  }
  if ((long long)idx.size() > n.idx_cap) {
    if (n.idx) cudaFree(n.idx);
    NET_CK(h, cudaMalloc(&n.idx, idx.size() * sizeof(int)));
    n.idx_cap = (long long)idx.size();
  }
  if (n.loss) cudaFree(n.loss), n.loss = nullptr;
  NET_CK(h, cudaMalloc(&n.loss, steps * sizeof(float)));
  NET_CK(h, cudaMemsetAsync(n.loss, 0, steps * sizeof(float), n.stream));
  NET_CK(h, cudaMemcpyAsync(n.idx, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, n.stream));
  cudaEvent_t e0, e1;
  NET_CK(h, cudaEventCreate(&e0));
  NET_CK(h, cudaEventCreate(&e1));
  int rc = 0;
  // one step captured as a CUDA graph and replayed `steps` times (the step index, on the device, offsets each replay's
  // batch indices and loss slot); the steps launched one by one if the capture fails
  NET_CK(h, cudaMemsetAsync(n.d_tstep, 0, sizeof(int), n.stream));
  cudaGraphExec_t step_graph = nullptr;
  if (cudaStreamBeginCapture(n.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
    const int crc = n.train_step(B, n.idx, (float)lr, n.loss, n.d_tstep);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(n.stream, &g);
    if (!crc && ce == cudaSuccess && g && cudaGraphInstantiate(&step_graph, g, 0) != cudaSuccess) step_graph = nullptr;
    if (g) cudaGraphDestroy(g);
    (void)cudaGetLastError();  // a failed capture leaves the loop below to run (and report) the steps one by one
    n.err.clear();
  }
  NET_CK(h, cudaEventRecord(e0, n.stream));
  if (step_graph) {
    cudaError_t le = cudaSuccess;
    for (uint64_t s = 0; s < steps && le == cudaSuccess; ++s) le = cudaGraphLaunch(step_graph, n.stream);
    if (le != cudaSuccess) {
      cudaStreamSynchronize(n.stream);
      cudaGraphExecDestroy(step_graph);
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      n.err = std::string("cudaGraphLaunch: ") + cudaGetErrorString(le);
      return BOWSHOCK_CUDA_ERROR;
    }
  } else {
    for (uint64_t s = 0; s < steps && !rc; ++s) rc = n.train_step(B, n.idx + s * B, (float)lr, n.loss + s);
  }
  NET_CK(h, cudaEventRecord(e1, n.stream));
  NET_CK(h, cudaStreamSynchronize(n.stream));
  if (step_graph) cudaGraphExecDestroy(step_graph);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  n.last_ms = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (loss) {
    std::vector<float> hl(steps);
    NET_CK(h, copy_sync(n.stream, hl.data(), n.loss, steps * sizeof(float), cudaMemcpyDeviceToHost));
    for (uint64_t s = 0; s < steps; ++s) loss[s] = hl[s];
  }
  return n.check_err();
}

int bowshock_net_last_train_ms(const bowshock_net* h, double* ms) {
  if (!h || !ms) return BOWSHOCK_INVALID;
  *ms = h->n.last_ms;
  return BOWSHOCK_OK;
}

int bowshock_net_set_conv_mode(bowshock_net* h, int mode) {
  if (!h || mode < 0 || mode > 2) return BOWSHOCK_INVALID;
  h->n.conv_mode = mode;
  return BOWSHOCK_OK;
}

int bowshock_conv3x3_bf16(const void* x, int64_t batch, int64_t h_in, int64_t w_in, int64_t c, int64_t up, const void* w, int64_t n, float* d,
                          int32_t mode, void* stream, int* err_flag) {
  if (!x || !w || !d || !err_flag || batch <= 0 || h_in <= 0 || w_in <= 0 || c <= 0 || n <= 0 || (up != 0 && up != 1) || (mode != 1 && mode != 2) ||
      (mode == 2 && up))
    return BOWSHOCK_INVALID;
  std::string err;
  bknet::GemmArgs g{};
  g.mode = bknet::EPI_F32, g.d = d, g.ldd = n, g.err = err_flag;
  if (mode == 2)
    return bknet::conv_gemm_tma(reinterpret_cast<const bknet::bf16*>(x), (int)batch, (int)h_in, (int)w_in, (int)c,
                                reinterpret_cast<const bknet::bf16*>(w), 9 * c, (int)n, g, reinterpret_cast<cudaStream_t>(stream), err);
  return bknet::conv_gemm(reinterpret_cast<const bknet::bf16*>(x), (int)batch, (int)h_in, (int)w_in, (int)c, (int)up,
                          reinterpret_cast<const bknet::bf16*>(w), 9 * c, (int)n, g, reinterpret_cast<cudaStream_t>(stream), err);
}

int bowshock_gemm_set_persistent(int on) {
  const int was = bknet::persistent_gemm ? 1 : 0;
  bknet::persistent_gemm = on != 0;
  return was;
}

int bowshock_gemm_bf16(const void* a, int64_t lda, const void* b, int64_t ldb, float* d, int64_t ldd, int64_t m, int64_t n, int64_t k, int64_t splits,
                       void* stream, int* err_flag) {
  if (!a || !b || !d || !err_flag || m <= 0 || n <= 0 || k <= 0 || splits <= 0 || ldd < n) return BOWSHOCK_INVALID;
  std::string err;
  bknet::GemmArgs g{};
  g.mode = splits > 1 ? bknet::EPI_F32_ATOMIC : bknet::EPI_F32;
  g.d = d, g.ldd = ldd, g.err = err_flag;
  return bknet::gemm(reinterpret_cast<const bknet::bf16*>(a), lda, reinterpret_cast<const bknet::bf16*>(b), ldb, (int)m, (int)n, (int)k, g,
                     (int)splits, reinterpret_cast<cudaStream_t>(stream), err);
}

}  // extern "C"
