// A BF16 GEMM on the 5th-generation tensor cores of sm_100a, with the epilogues of the surrogate network.
//
// C[M, N] = A[M, K] B[N, K]^T, A and B row-major BF16 (both K-major), FP32 accumulation in tensor memory, in tiles of
// 128 x BN: TMA streams the K blocks of A and B into shared-memory stages (128-byte swizzle, tensor maps over this
// GPU's memory only), one thread issues the tcgen05.mma's (M 128, N BN, K 16 each, four per 64-wide K block) into a
// TMEM accumulator and hands each stage back with tcgen05.commit, and four warps read the accumulator (tcgen05.ld
// 32x32b) through the epilogue. Every wait on an mbarrier gives up after about a second of clock ticks: the CTA then
// sets *err, lets its issued copies finish (bounded waits), frees its tensor memory and returns.
//
// Epilogues: STORE (C in FP32), BIAS (C + bias in FP32), BIAS_SILU (z = C + bias, optionally kept in FP32; the BF16
// output silu(z) = z sigmoid(z)), DSILU (the backward of SiLU: BF16 C * silu'(z) with z read in FP32).
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace mxg {

constexpr int BM = 128, BK = 64;
enum Epilogue { STORE = 0, BIAS = 1, BIAS_SILU = 2, DSILU = 3 };

struct Epi {
  int mode;
  const float* bias;  // [N] (BIAS, BIAS_SILU)
  float* z;           // [M][ldz] FP32: written by BIAS_SILU when not null, read by DSILU
  int ldz;
  void* out;          // [M][ldo]: FP32 (STORE, BIAS) or BF16 (BIAS_SILU, DSILU)
  int ldo;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// The shared-memory matrix descriptor of a K-major operand tile in the 128-byte swizzle layout: rows of 64 BF16 (128
// bytes), 8-row groups 1024 bytes apart (stride byte offset), start address in 16-byte units, descriptor version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// The instruction descriptor of kind::f16 with BF16 A and B (K-major), FP32 accumulation, M 128, N n.
__host__ __device__ constexpr uint32_t bf16_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for the phase of the given parity; false (and *err set) after about 2^31 clock ticks (~1 s).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* err) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (clock64() - t0 > (1ll << 31)) {
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_load16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float sigmoid(float z) { return 1.0f / (1.0f + __expf(-z)); }

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Shared-memory bytes of one CTA: the stages (1024-aligned), the barriers and the TMEM address slot, plus the slack
// that aligns the dynamic base to 1024 bytes.
template <int BN, int STAGES>
__host__ __device__ constexpr int gemm_smem_bytes() {
  return STAGES * (BM + BN) * BK * 2 + 8 * (2 * STAGES + 4) + 16 + 1024;
}

// The epilogue of 16 accumulator columns of one row (a[16]): columns col .. col + 15 of row `row`.
__device__ __forceinline__ void epilogue16(const Epi& ep, float (&a)[16], int row, int col) {
  if (ep.mode == STORE || ep.mode == BIAS) {
    if (ep.mode == BIAS)
#pragma unroll
      for (int j = 0; j < 16; j++) a[j] += ep.bias[col + j];
    float4* o = (float4*)((float*)ep.out + (size_t)row * ep.ldo + col);
#pragma unroll
    for (int j = 0; j < 4; j++) o[j] = make_float4(a[4 * j], a[4 * j + 1], a[4 * j + 2], a[4 * j + 3]);
    return;
  }
  if (ep.mode == BIAS_SILU) {
#pragma unroll
    for (int j = 0; j < 16; j++) a[j] += ep.bias[col + j];
    if (ep.z) {
      float4* zo = (float4*)(ep.z + (size_t)row * ep.ldz + col);
#pragma unroll
      for (int j = 0; j < 4; j++) zo[j] = make_float4(a[4 * j], a[4 * j + 1], a[4 * j + 2], a[4 * j + 3]);
    }
#pragma unroll
    for (int j = 0; j < 16; j++) a[j] = a[j] * sigmoid(a[j]);
  } else {  // DSILU
    const float4* zi = (const float4*)(ep.z + (size_t)row * ep.ldz + col);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const float4 z4 = zi[j];
      const float zz[4] = {z4.x, z4.y, z4.z, z4.w};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float sg = sigmoid(zz[q]);
        a[4 * j + q] *= sg * (1.0f + zz[q] * (1.0f - sg));
      }
    }
  }
  uint32_t packed[8];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(a[2 * j], a[2 * j + 1]);
    packed[j] = *reinterpret_cast<const uint32_t*>(&p);
  }
  uint4* o = (uint4*)((__nv_bfloat16*)ep.out + (size_t)row * ep.ldo + col);
  o[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
  o[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
}

// Persistent and warp-specialised: one CTA of 6 warps per SM walks the output tiles (row tiles outer, column tiles
// inner, so neighbouring tiles share A's rows in L2). Warp 0 (one thread) streams the K blocks of A and B into a ring
// of STAGES shared-memory stages; warp 1 (one thread) issues the MMAs into one of two TMEM accumulators of BN columns
// each and commits; warps 2-5 drain the other accumulator (warp w the TMEM lanes 32 (w % 4) ..) through the epilogue
// and hand it back, so a tile's epilogue overlaps the next tile's MMAs.
template <int BN, int STAGES>
__global__ void __launch_bounds__(192, 1) gemm_kernel(const __grid_constant__ CUtensorMap ta,
                                                      const __grid_constant__ CUtensorMap tb, int M, int N, int K,
                                                      Epi ep, int* err) {
  extern __shared__ uint8_t gemm_smem_raw[];
  uint8_t* base = (uint8_t*)(((uintptr_t)gemm_smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sa = base;                                        // STAGES x [128][64] BF16
  uint8_t* sb = base + STAGES * BM * BK * 2;                 // STAGES x [BN][64] BF16
  uint64_t* bars = (uint64_t*)(sb + STAGES * BN * BK * 2);   // full[S], empty[S], acc_full[2], acc_empty[2]
  uint32_t* tslot = (uint32_t*)(bars + 2 * STAGES + 4);
  const int tid = (int)threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nk = K / BK, tiles_n = N / BN, tiles = ((M + BM - 1) / BM) * tiles_n;
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + STAGES);
  const uint32_t accf0 = smem_u32(bars + 2 * STAGES), acce0 = smem_u32(bars + 2 * STAGES + 2);
  if (tid == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(accf0 + 8 * b, 1);
      mbar_init(acce0 + 8 * b, 4);  // one arrival per epilogue warp
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {  // two accumulators of BN columns (2 BN a power of two >= 32, at most 512)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(2 * BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  const uint32_t tmem = *tslot;
  if (warp == 0 && lane == 0) {  // producer
    int issued_round[STAGES];
    for (int s = 0; s < STAGES; s++) issued_round[s] = -1;
    long long kc = 0;
    bool ok = true;
    for (int t = (int)blockIdx.x; t < tiles && ok; t += (int)gridDim.x) {
      const int m0 = (t / tiles_n) * BM, n0 = (t % tiles_n) * BN;
      for (int kb = 0; kb < nk; kb++, kc++) {
        const int s = (int)(kc % STAGES), r = (int)(kc / STAGES);
        if (r > 0 && !mbar_wait(empty0 + 8 * s, (uint32_t)((r - 1) & 1), err)) {
          ok = false;
          break;
        }
        mbar_expect_tx(full0 + 8 * s, (uint32_t)((BM + BN) * BK * 2));
        tma_load_2d(smem_u32(sa + s * BM * BK * 2), &ta, full0 + 8 * s, kb * BK, m0);
        tma_load_2d(smem_u32(sb + s * BN * BK * 2), &tb, full0 + 8 * s, kb * BK, n0);
        issued_round[s] = r;
      }
    }
    for (int s = 0; s < STAGES; s++)  // the copies this thread issued have landed before the CTA may exit
      if (issued_round[s] >= 0) mbar_wait(full0 + 8 * s, (uint32_t)(issued_round[s] & 1), err);
  } else if (warp == 1 && lane == 0) {  // MMA issuer
    constexpr uint32_t idesc = bf16_idesc(BN);
    long long kc = 0;
    bool ok = true;
    int i = 0;
    for (int t = (int)blockIdx.x; t < tiles && ok; t += (int)gridDim.x, i++) {
      const int acc = i & 1, use = i >> 1;
      if (use > 0 && !mbar_wait(acce0 + 8 * acc, (uint32_t)((use - 1) & 1), err)) break;
      tmem_fence_after();
      const uint32_t d = tmem + (uint32_t)(acc * BN);
      for (int kb = 0; kb < nk; kb++, kc++) {
        const int s = (int)(kc % STAGES), r = (int)(kc / STAGES);
        if (!mbar_wait(full0 + 8 * s, (uint32_t)(r & 1), err)) {
          ok = false;
          break;
        }
        tmem_fence_after();
        const uint64_t da = sw128_desc(smem_u32(sa + s * BM * BK * 2));
        const uint64_t db = sw128_desc(smem_u32(sb + s * BN * BK * 2));
#pragma unroll
        for (int k = 0; k < BK / 16; k++)  // +32 bytes along K within the swizzled 128-byte rows: +2 in 16-byte units
          umma_bf16(d, da + 2 * k, db + 2 * k, idesc, (kb > 0 || k > 0) ? 1u : 0u);
        umma_commit(empty0 + 8 * s);
      }
      umma_commit(accf0 + 8 * acc);  // fires when this tile's MMAs (and every earlier one) have completed
    }
  } else if (warp >= 2) {  // epilogue: warp w reads TMEM lanes 32 (w % 4) .. 32 (w % 4) + 31, one row per thread
    const int quarter = warp & 3;
    int i = 0;
    for (int t = (int)blockIdx.x; t < tiles; t += (int)gridDim.x, i++) {
      const int acc = i & 1, use = i >> 1;
      const int m0 = (t / tiles_n) * BM, n0 = (t % tiles_n) * BN;
      if (!mbar_wait(accf0 + 8 * acc, (uint32_t)(use & 1), err)) break;
      tmem_fence_after();
      const int row = m0 + 32 * quarter + lane;
#pragma unroll 1
      for (int c = 0; c < BN; c += 16) {
        uint32_t v[16];
        tmem_load16(tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(acc * BN + c), v);
        if (row < M) {
          float a[16];
#pragma unroll
          for (int j = 0; j < 16; j++) a[j] = __uint_as_float(v[j]);
          epilogue16(ep, a, row, n0 + c);
        }
      }
      tmem_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce0 + 8 * acc);
    }
  }
  tmem_fence_before();
  __syncthreads();
  if (warp == 1) {
    tmem_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN) : "memory");
  }
}

}  // namespace mxg
