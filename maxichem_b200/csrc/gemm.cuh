// A BF16 GEMM on the 5th-generation tensor cores of sm_100a, with the epilogues of the surrogate network.
//
// C[M, N] = A[M, K] B[N, K]^T, A and B row-major BF16 (both K-major), FP32 accumulation in tensor memory, in tiles of
// 128 x BN: TMA streams the K blocks of A and B into shared-memory stages (128-byte swizzle, tensor maps over this
// GPU's memory only), one thread issues the tcgen05.mma's (M 128, N BN, K 16 each, four per 64-wide K block) into a
// TMEM accumulator and hands each stage back with tcgen05.commit, and eight warps read the accumulator (tcgen05.ld
// 32x32b) through the epilogue, which stages each 32-row x 32-column piece of its outputs in shared memory (64- or
// 128-byte swizzle, conflict-free for the row-per-lane writes) and writes it with a TMA store. Every wait on an mbarrier
// gives up after about a second of clock ticks: the CTA then sets *err, lets its issued copies finish (bounded waits),
// frees its tensor memory and returns.
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
constexpr int EPI_WARPS = 8;                  // two per TMEM lane quarter, each over half the tile's columns
constexpr int THREADS = 64 + 32 * EPI_WARPS;  // producer warp, MMA warp, epilogue warps
constexpr int EPI_COLS = 32;                  // accumulator columns per epilogue step
enum Epilogue { STORE = 0, BIAS = 1, BIAS_SILU = 2, DSILU = 3 };
// The kernel is compiled per epilogue (its registers then hold only what that epilogue needs): BIAS_SILU splits into
// SILU (activation only, the inference pass) and SILU_Z (the pre-activation kept in FP32 too, the training pass).
enum Variant { V_STORE = 0, V_BIAS = 1, V_SILU = 2, V_SILU_Z = 3, V_DSILU = 4 };
__host__ __device__ constexpr int variant_of(int mode, bool keep_z) {
  return mode == STORE ? V_STORE : mode == BIAS ? V_BIAS : mode == BIAS_SILU ? (keep_z ? V_SILU_Z : V_SILU) : V_DSILU;
}

// Staging bytes per epilogue warp: the output piece at 0 (32 rows x 32 columns: 2 KB in BF16, 4 KB in FP32) and, for
// the epilogues with z, the z piece (FP32, 4 KB) at 2 KB. Less staging leaves room for a deeper ring of A and B stages.
__host__ __device__ constexpr int staging_bytes(int epi) {
  return epi == V_SILU ? 2048 : (epi == V_STORE || epi == V_BIAS) ? 4096 : 6144;
}

struct Epi {
  int mode;
  const float* bias;  // [N] (BIAS, BIAS_SILU)
  float* z;           // [M][ldz] FP32: written by BIAS_SILU when not null, read by DSILU
  int ldz;
  void* out;          // [M][ldo]: FP32 (STORE, BIAS) or BF16 (BIAS_SILU, DSILU)
  int ldo;
  int tma;            // 1: out (and z) through the output tensor maps; 0: plain stores (unaligned out or z)
  int splits;         // K split into this many consecutive ranges of 64-blocks (1: no split), each non-empty
  int split_rows;     // rows of out between two splits' partial products (splits > 1: out is [splits][split_rows][ldo])
};

// Output tile t of a launch: rows m0.., columns n0.., K blocks kb0 .. kb1 - 1, output rows offset by orow. With
// splits > 1 the tiles run split by split (consecutive CTAs share a split's K range of A and B in L2).
struct Tile {
  int m0, n0, kb0, kb1, orow;
};
template <int BN>
__device__ __forceinline__ Tile tile_at(int t, int tiles_mn, int tiles_n, int nks, int nk, const Epi& ep) {
  const int split = t / tiles_mn, tmn = t - split * tiles_mn;
  Tile r;
  r.m0 = (tmn / tiles_n) * BM;
  r.n0 = (tmn % tiles_n) * BN;
  r.kb0 = split * nks;
  r.kb1 = min(nk, r.kb0 + nks);
  r.orow = split * ep.split_rows;
  return r;
}

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

// A waiting thread may be suspended (it issues nothing) until the phase completes or this many nanoseconds pass, so the
// single-thread producer and MMA warps do not take issue slots from the epilogue warps on their SM sub-partitions.
constexpr uint32_t SUSPEND_NS = 100000;
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(SUSPEND_NS)
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

// A TMA store of one box from shared memory (rows past the tensor's end are not written), in the thread's bulk group.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, uint32_t src, int x, int y) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(src), "r"(x), "r"(y)
               : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the thread's committed stores have read their shared-memory sources (the staging may be written again)
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// the thread's committed stores are complete
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// this thread's shared-memory writes are visible to the TMA unit (the async proxy)
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

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

// 32 consecutive accumulator columns of the warp's 32 TMEM lanes (one row per thread), issued; tmem_wait waits for
// every load of the thread and ties v's registers to the wait, so that no use of them moves above it.
__device__ __forceinline__ void tmem_load(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait(uint32_t (&v)[32]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7]),
                 "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]), "+r"(v[14]), "+r"(v[15]),
                 "+r"(v[16]), "+r"(v[17]), "+r"(v[18]), "+r"(v[19]), "+r"(v[20]), "+r"(v[21]), "+r"(v[22]),
                 "+r"(v[23]), "+r"(v[24]), "+r"(v[25]), "+r"(v[26]), "+r"(v[27]), "+r"(v[28]), "+r"(v[29]),
                 "+r"(v[30]), "+r"(v[31])
               :
               : "memory");
}

// 1 / d for d in [1, 2^100] on the FMA pipe: a first estimate from the bit pattern (the exponent negated by an integer
// subtraction from a constant, relative error below 6 %), then two Newton-Raphson steps r <- r (2 - d r), which square
// the error twice (below 1e-5, ample for the BF16 outputs).
__device__ __forceinline__ float rcp_newton(float d) {
  float r = __int_as_float(0x7EF311C3 - __float_as_int(d));
  r = fmaf(r, fmaf(-d, r, 1.0f), r);
  return fmaf(r, fmaf(-d, r, 1.0f), r);
}

// 2^x and 1/x by the special-function unit's approximations (ex2.approx, rcp.approx: a few ulp, subnormals flushed).
__device__ __forceinline__ float ex2_sfu(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_sfu(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// sigmoid(z) = 1 / (1 + 2^(-z log2 e)), the reciprocal on the special-function unit (sigmoid_sfu) or on the FMA pipe
// (sigmoid_fma). The epilogue mixes the two across columns (column j on the special-function unit when
// j % SFU_EVERY == 0), so that neither unit alone limits it: one exponential and one reciprocal per element would ask
// the special-function unit (16 results per clock per SM) for as many cycles as the tensor core spends on a
// 512-deep tile.
constexpr float NEG_LOG2E = -1.4426950408889634f;
__device__ __forceinline__ float sigmoid_sfu(float z) { return rcp_sfu(1.0f + ex2_sfu(z * NEG_LOG2E)); }
__device__ __forceinline__ float sigmoid_fma(float z) { return rcp_newton(fminf(1.0f + ex2_sfu(z * NEG_LOG2E), 0x1p100f)); }
template <int SFU_EVERY>
__device__ __forceinline__ float sigmoid_at(float z, int j) {
  return j % SFU_EVERY == 0 ? sigmoid_sfu(z) : sigmoid_fma(z);
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// TMEM columns of the two accumulators: 2 BN rounded up to a power of two (an allocation's size), at most 512.
__host__ __device__ constexpr uint32_t tmem_columns(int bn) {
  uint32_t c = 32;
  while (c < 2u * (uint32_t)bn) c <<= 1;
  return c;
}

// Shared-memory bytes of one CTA: the stages (1024-aligned), the epilogue warps' staging, the barriers and the TMEM
// address slot, plus the slack that aligns the dynamic base to 1024 bytes.
__host__ __device__ constexpr int gemm_smem_bytes(int bn, int stages, int epi) {
  return stages * (BM + bn) * BK * 2 + EPI_WARPS * staging_bytes(epi) + 8 * (2 * stages + 4 + EPI_WARPS) + 16 + 1024;
}

// The deepest ring of stages (at most 8) that fits one CTA's 227 KB of shared memory beside the epilogue's staging:
// the bytes in flight between TMA and the tensor core are what hide the loads' latency.
__host__ __device__ constexpr int stages_for(int bn, int epi) {
  int s = 8;
  while (s > 2 && gemm_smem_bytes(bn, s, epi) > 232448) s--;
  return s;
}

// Byte offset of 16-byte chunk c of row r in a staging piece of RB-byte rows (32, 64 or 128) as the TMA unit lays out
// a box with the RB-byte swizzle: the chunk index XOR the address bits 7 and up. Eight consecutive lanes writing chunk
// c of their rows then hit eight different 16-byte bank groups.
template <int RB>
__device__ __forceinline__ uint32_t swz(int r, int c) {
  return (uint32_t)(r * RB + ((c ^ ((r * RB >> 7) & (RB / 16 - 1))) << 4));
}

// The epilogue's arithmetic on COLS accumulator columns (a, columns col ..) of one row; zz holds z for DSILU.
// BIAS_SILU leaves z = C + bias in zz and the activation in a.
template <int EPI, int SFU_EVERY>
__device__ __forceinline__ void epilogue_math(const Epi& ep, float (&a)[EPI_COLS], float (&zz)[EPI_COLS], int col) {
  if constexpr (EPI == V_BIAS || EPI == V_SILU || EPI == V_SILU_Z) {
    const float4* b4 = reinterpret_cast<const float4*>(ep.bias + col);
#pragma unroll
    for (int j = 0; j < EPI_COLS / 4; j++) {
      const float4 b = __ldg(b4 + j);
      a[4 * j] += b.x;
      a[4 * j + 1] += b.y;
      a[4 * j + 2] += b.z;
      a[4 * j + 3] += b.w;
    }
  }
  if constexpr (EPI == V_SILU || EPI == V_SILU_Z) {
#pragma unroll
    for (int j = 0; j < EPI_COLS; j++) {
      zz[j] = a[j];
      a[j] = a[j] * sigmoid_at<SFU_EVERY>(a[j], j);
    }
  } else if constexpr (EPI == V_DSILU) {
#pragma unroll
    for (int j = 0; j < EPI_COLS; j++) {
      const float sg = sigmoid_at<SFU_EVERY>(zz[j], j);
      a[j] *= sg * (1.0f + zz[j] * (1.0f - sg));
    }
  }
}

__device__ __forceinline__ void pack_bf16(const float (&a)[EPI_COLS], uint32_t (&p)[EPI_COLS / 2]) {
#pragma unroll
  for (int j = 0; j < EPI_COLS / 2; j++) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a[2 * j], a[2 * j + 1]);
    p[j] = *reinterpret_cast<const uint32_t*>(&h);
  }
}

// Persistent and warp-specialised: one CTA of 10 warps per SM walks the output tiles (row tiles outer, column tiles
// inner, so neighbouring tiles share A's rows in L2). Warp 0 (one thread) streams the K blocks of A and B into a ring
// of STAGES shared-memory stages; warp 1 (one thread) issues the MMAs into one of two TMEM accumulators of BN columns
// each and commits; warps 2-9 drain the other accumulator through the epilogue (warp w the TMEM lanes 32 (w % 4) ..
// 32 (w % 4) + 31, warps 2-5 the left half of the columns and 6-9 the right half) and hand it back, so a tile's
// epilogue overlaps the next tile's MMAs. With ep.tma, each epilogue warp stages its 32 x 32 output pieces in its own
// shared memory and stores them with TMA (one bulk group per warp, waited for before the staging is rewritten);
// DSILU's z pieces come in the same way by TMA loads, one ahead. EPI is the epilogue (Variant); SFU_EVERY the
// sigmoid's split between the special-function unit and the FMA pipe. (Sixteen epilogue warps in 16-column steps,
// four per SM sub-partition at 96 registers, were measured no faster.)
template <int BN, int STAGES, int EPI, int SFU_EVERY = 2>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb,
                const __grid_constant__ CUtensorMap to, const __grid_constant__ CUtensorMap tz, int M, int N, int K,
                Epi ep, int* err) {
  extern __shared__ uint8_t gemm_smem_raw[];
  uint8_t* base = (uint8_t*)(((uintptr_t)gemm_smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sa = base;                                       // STAGES x [128][64] BF16
  uint8_t* sb = base + STAGES * BM * BK * 2;                // STAGES x [BN][64] BF16
  constexpr int STAGING = staging_bytes(EPI);
  uint8_t* stg = sb + STAGES * BN * BK * 2;                 // EPI_WARPS x STAGING
  uint64_t* bars = (uint64_t*)(stg + EPI_WARPS * STAGING);  // full[S], empty[S], acc_full[2], acc_empty[2], z[8]
  uint32_t* tslot = (uint32_t*)(bars + 2 * STAGES + 4 + EPI_WARPS);
  const int tid = (int)threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nk = K / BK, tiles_n = N / BN, tiles_mn = ((M + BM - 1) / BM) * tiles_n;
  const int nks = (nk + ep.splits - 1) / ep.splits, tiles = tiles_mn * ep.splits;
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + STAGES);
  const uint32_t accf0 = smem_u32(bars + 2 * STAGES), acce0 = smem_u32(bars + 2 * STAGES + 2);
  const uint32_t zbar0 = smem_u32(bars + 2 * STAGES + 4);
  if (tid == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(accf0 + 8 * b, 1);
      mbar_init(acce0 + 8 * b, EPI_WARPS);  // one arrival per epilogue warp
    }
    for (int w = 0; w < EPI_WARPS; w++) mbar_init(zbar0 + 8 * w, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  constexpr uint32_t TMEM_COLS = tmem_columns(BN);
  if (warp == 1) {  // two accumulators of BN columns, in the power of two of columns at or above 2 BN
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(TMEM_COLS)
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
      const Tile tl = tile_at<BN>(t, tiles_mn, tiles_n, nks, nk, ep);
      const int m0 = tl.m0, n0 = tl.n0;
      for (int kb = tl.kb0; kb < tl.kb1; kb++, kc++) {
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
      const Tile tl = tile_at<BN>(t, tiles_mn, tiles_n, nks, nk, ep);
      for (int kb = tl.kb0; kb < tl.kb1; kb++, kc++) {
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
          umma_bf16(d, da + 2 * k, db + 2 * k, idesc, (kb > tl.kb0 || k > 0) ? 1u : 0u);
        umma_commit(empty0 + 8 * s);
      }
      umma_commit(accf0 + 8 * acc);  // fires when this tile's MMAs (and every earlier one) have completed
    }
  } else if (warp >= 2) {  // epilogue
    const int ew = warp - 2, quarter = warp & 3;
    constexpr int WCOLS = BN / 2;  // columns of the warp's half
    static_assert(WCOLS % EPI_COLS == 0, "the slice is whole steps");
    constexpr int RB16 = EPI_COLS * 2, RB32 = EPI_COLS * 4;  // staging row bytes: BF16 and FP32 pieces
    const int cbeg = (ew >> 2) * WCOLS, cend = cbeg + WCOLS;
    uint8_t* so = stg + ew * STAGING;  // output piece: 32 rows x RB16 (BF16) or RB32 (FP32)
    uint8_t* sz = so + 2048;           // z piece: 32 rows x RB32 (FP32)
    const uint32_t so_a = smem_u32(so), sz_a = smem_u32(sz), zbar = zbar0 + 8 * ew;
    constexpr bool f32_out = EPI == V_STORE || EPI == V_BIAS, zout = EPI == V_SILU_Z, zin = EPI == V_DSILU;
    const bool tma = ep.tma != 0;
    constexpr uint32_t ZBYTES = 32 * EPI_COLS * 4;
    uint32_t z_issued = 0, z_done = 0;  // TMA loads of z pieces issued and waited for (uniform across the warp)
    bool ok = true;
    int i = 0;
    for (int t = (int)blockIdx.x; t < tiles && ok; t += (int)gridDim.x, i++) {
      const int acc = i & 1, use = i >> 1;
      const Tile tl = tile_at<BN>(t, tiles_mn, tiles_n, nks, nk, ep);
      const int m0 = tl.m0, n0 = tl.n0, orow = tl.orow;  // orow: the split's rows in out (split-K partials)
      const int r0 = m0 + 32 * quarter, row = r0 + lane;
      if (zin && tma) {  // this tile's first z piece, while the MMAs run
        if (lane == 0) {
          mbar_expect_tx(zbar, ZBYTES);
          tma_load_2d(sz_a, &tz, zbar, n0 + cbeg, r0);
        }
        z_issued++;
      }
      if (!mbar_wait(accf0 + 8 * acc, (uint32_t)(use & 1), err)) break;
      tmem_fence_after();
      // one epilogue step: the 32 accumulator columns c .. c + 31 of the warp's rows, already read from TMEM into v
      auto step = [&](const uint32_t(&v)[EPI_COLS], int c) -> bool {
        float a[EPI_COLS], zz[EPI_COLS];
#pragma unroll
        for (int j = 0; j < EPI_COLS; j++) a[j] = __uint_as_float(v[j]);
        if (zin) {
          if (tma) {
            if (!mbar_wait(zbar, z_done & 1u, err)) return false;
            z_done++;
#pragma unroll
            for (int q = 0; q < EPI_COLS / 4; q++) {
              const float4 z4 = *reinterpret_cast<const float4*>(sz + swz<RB32>(lane, q));
              zz[4 * q] = z4.x;
              zz[4 * q + 1] = z4.y;
              zz[4 * q + 2] = z4.z;
              zz[4 * q + 3] = z4.w;
            }
          } else {
#pragma unroll
            for (int q = 0; q < EPI_COLS / 4; q++) {
              const float4 z4 = row < M ? *reinterpret_cast<const float4*>(ep.z + (size_t)row * ep.ldz + n0 + c + 4 * q)
                                        : make_float4(0.f, 0.f, 0.f, 0.f);
              zz[4 * q] = z4.x;
              zz[4 * q + 1] = z4.y;
              zz[4 * q + 2] = z4.z;
              zz[4 * q + 3] = z4.w;
            }
          }
        }
        epilogue_math<EPI, SFU_EVERY>(ep, a, zz, n0 + c);
        if (zin && tma) {  // the z piece is consumed: fetch the next one into the same staging
          __syncwarp();
          if (c + EPI_COLS < cend) {
            if (lane == 0) {
              mbar_expect_tx(zbar, ZBYTES);
              tma_load_2d(sz_a, &tz, zbar, n0 + c + EPI_COLS, r0);
            }
            z_issued++;
          }
        }
        if (tma) {
          if (lane == 0) bulk_wait_read();  // the previous piece has left the staging
          __syncwarp();
          if (f32_out) {
#pragma unroll
            for (int q = 0; q < EPI_COLS / 4; q++)
              *reinterpret_cast<float4*>(so + swz<RB32>(lane, q)) =
                  make_float4(a[4 * q], a[4 * q + 1], a[4 * q + 2], a[4 * q + 3]);
          } else {
            uint32_t p[EPI_COLS / 2];
            pack_bf16(a, p);
#pragma unroll
            for (int q = 0; q < EPI_COLS / 8; q++)
              *reinterpret_cast<uint4*>(so + swz<RB16>(lane, q)) =
                  make_uint4(p[4 * q], p[4 * q + 1], p[4 * q + 2], p[4 * q + 3]);
          }
          if (zout) {
#pragma unroll
            for (int q = 0; q < EPI_COLS / 4; q++)
              *reinterpret_cast<float4*>(sz + swz<RB32>(lane, q)) =
                  make_float4(zz[4 * q], zz[4 * q + 1], zz[4 * q + 2], zz[4 * q + 3]);
          }
          fence_async_shared();
          __syncwarp();
          if (lane == 0 && r0 < M) {  // a piece wholly below the last row has nothing to store
            tma_store_2d(&to, so_a, n0 + c, r0 + orow);
            if (zout) tma_store_2d(&tz, sz_a, n0 + c, r0);
            bulk_commit();
          }
        } else if (row < M) {
          if (f32_out) {
            float4* o = (float4*)((float*)ep.out + (size_t)(row + orow) * ep.ldo + n0 + c);
#pragma unroll
            for (int q = 0; q < EPI_COLS / 4; q++)
              o[q] = make_float4(a[4 * q], a[4 * q + 1], a[4 * q + 2], a[4 * q + 3]);
          } else {
            uint32_t p[EPI_COLS / 2];
            pack_bf16(a, p);
            uint4* o = (uint4*)((__nv_bfloat16*)ep.out + (size_t)row * ep.ldo + n0 + c);
#pragma unroll
            for (int q = 0; q < EPI_COLS / 8; q++) o[q] = make_uint4(p[4 * q], p[4 * q + 1], p[4 * q + 2], p[4 * q + 3]);
          }
          if (zout) {
            float4* zo = (float4*)(ep.z + (size_t)row * ep.ldz + n0 + c);
#pragma unroll
            for (int q = 0; q < EPI_COLS / 4; q++)
              zo[q] = make_float4(zz[4 * q], zz[4 * q + 1], zz[4 * q + 2], zz[4 * q + 3]);
          }
        }
        return true;
      };
      // the next step's columns are read from TMEM while this step's arithmetic runs (two register sets in turn)
      const uint32_t tbase = tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(acc * BN);
      // the accumulator goes back to the MMA warp as soon as its last columns are in registers
      bool released = false;
      auto release = [&]() {
        tmem_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acce0 + 8 * acc);
        released = true;
      };
      uint32_t va[EPI_COLS], vb[EPI_COLS];
      tmem_load(tbase + (uint32_t)cbeg, va);
      tmem_wait(va);
#pragma unroll 1
      for (int c = cbeg; c < cend && ok; c += 2 * EPI_COLS) {
        const bool more = c + EPI_COLS < cend, more2 = c + 2 * EPI_COLS < cend;
        if (more)
          tmem_load(tbase + (uint32_t)(c + EPI_COLS), vb);
        else
          release();
        ok = step(va, c);
        if (!more) break;
        tmem_wait(vb);
        if (!more2) release();
        if (!ok) break;
        if (more2) tmem_load(tbase + (uint32_t)(c + 2 * EPI_COLS), va);
        ok = step(vb, c + EPI_COLS);
        if (more2) tmem_wait(va);
      }
      if (!released && ok) release();
    }
    if (lane == 0) bulk_wait_all();  // every store of this warp is complete before its staging goes away
    if (z_issued > z_done) mbar_wait(zbar, z_done & 1u, err);  // a z piece still in flight (only after an error)
    __syncwarp();
  }
  tmem_fence_before();
  __syncthreads();
  if (warp == 1) {
    tmem_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

}  // namespace mxg
