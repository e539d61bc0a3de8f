// The learned part of the call: a BF16 MLP surrogate of the per-call solve, its training on the
// GPU, and the gated call that solves only the cells it cannot vouch for. No counterpart in the reference.
//
// Network: the features of a cell (log10 x per species floored at 1e-30, log10 T, P, dt and the carried h,
// log10(J + 1e-30) per branch, each standardised; zero padding to a multiple of 64) -> L hidden layers of width H with SiLU -> heads
// output blocks of (log10 x_out - log10 x_in per species, log10 h_out), standardised. Weights BF16 [out][in] (K-major
// for the tensor cores) with FP32 master copies, biases FP32. Every layer is one tcgen05 GEMM (gemm.cuh) with its
// bias and activation fused into the epilogue; training adds the backward GEMMs (dX with the SiLU derivative fused,
// dW from transposed operands), the bias sums and Adam.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "gemm.cuh"
#include "solver.cuh"

using namespace mxg;

namespace {

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::mutex g_encode_mutex;

cudaError_t encoder() {
  std::lock_guard<std::mutex> lock(g_encode_mutex);
  if (g_encode) return cudaSuccess;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
  const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
  if (e != cudaSuccess) return e;
  if (q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
  g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  return cudaSuccess;
}

// A tensor map over a row-major BF16 matrix [rows][ld] (its first `cols` columns), boxes of box_rows x 64 with the
// 128-byte swizzle; rows past the end read as zeros.
bool tensor_map(CUtensorMap* m, const void* p, uint64_t rows, uint64_t cols, uint64_t ld, uint32_t box_rows) {
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)BK, box_rows};
  const cuuint32_t es[2] = {1, 1};
  return g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(p), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// A tensor map for the epilogue's 32-row x cols-column pieces of an output (or of z) [rows][ld], BF16 or FP32, with
// the swizzle of the piece's row bytes (32, 64 or 128), the layouts the epilogue writes its staging in. False when the pointer or
// the row pitch is not a multiple of 16 bytes or the encoding fails (the epilogue then stores directly, 16 bytes at a
// time, which asks for the same alignment: the launcher refuses anything less).
bool piece_map(CUtensorMap* m, const void* p, uint64_t rows, uint64_t cols, uint64_t ld, bool f32, int piece_cols) {
  const uint64_t es = f32 ? 4 : 2;
  if (((uintptr_t)p & 15) || (ld * es) % 16) return false;
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {ld * es};
  const cuuint32_t box[2] = {(cuuint32_t)piece_cols, 32};
  const uint64_t row_bytes = (uint64_t)piece_cols * es;
  const CUtensorMapSwizzle sw = row_bytes == 128  ? CU_TENSOR_MAP_SWIZZLE_128B
                                : row_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                                                  : CU_TENSOR_MAP_SWIZZLE_32B;
  const cuuint32_t step[2] = {1, 1};
  return g_encode(m, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                  const_cast<void*>(p), dims, strides, box, step, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  sw, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int g_sms = 0;

// the column tile of a product with N columns: the widest of 256, 192, 128, 64 that divides N
int tile_width(int N) { return N % 256 == 0 ? 256 : N % 192 == 0 ? 192 : N % 128 == 0 ? 128 : 64; }

template <int BN, int EPI>
cudaError_t launch_tile(const CUtensorMap& ta, const CUtensorMap& tb, const CUtensorMap& to, const CUtensorMap& tz,
                        int64_t M, int N, int K, const Epi& ep, int* err, cudaStream_t st) {
  // the opt-in shared memory, set once per instance and device (a bit per device; devices past 63 set it every time)
  static std::atomic<unsigned long long> configured{0};
  constexpr int STAGES = stages_for(BN, EPI), smem = gemm_smem_bytes(BN, STAGES, EPI);
  static_assert(smem <= 232448, "more shared memory than a CTA of sm_100a may opt into");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return cudaErrorInvalidDevice;
  const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
  if (!bit || !(configured.load() & bit)) {
    const cudaError_t e = cudaFuncSetAttribute((const void*)gemm_kernel<BN, STAGES, EPI>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    configured.fetch_or(bit);
  }
  if (!g_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
  }
  const long long tiles = ((M + BM - 1) / BM) * (long long)(N / BN) * ep.splits;
  const int grid = (int)std::min<long long>(tiles, std::max(g_sms, 1));  // persistent: one CTA per SM
  gemm_kernel<BN, STAGES, EPI><<<grid, THREADS, smem, st>>>(ta, tb, to, tz, (int)M, N, K, ep, err);
  return cudaGetLastError();
}

// the kernel for a column tile width and an epilogue
template <int BN>
cudaError_t launch_epi(int epi, const CUtensorMap& ta, const CUtensorMap& tb, const CUtensorMap& to,
                       const CUtensorMap& tz, int64_t M, int N, int K, const Epi& ep, int* err, cudaStream_t st) {
  switch (epi) {
    case V_STORE: return launch_tile<BN, V_STORE>(ta, tb, to, tz, M, N, K, ep, err, st);
    case V_BIAS: return launch_tile<BN, V_BIAS>(ta, tb, to, tz, M, N, K, ep, err, st);
    case V_SILU: return launch_tile<BN, V_SILU>(ta, tb, to, tz, M, N, K, ep, err, st);
    case V_SILU_Z: return launch_tile<BN, V_SILU_Z>(ta, tb, to, tz, M, N, K, ep, err, st);
    default: return launch_tile<BN, V_DSILU>(ta, tb, to, tz, M, N, K, ep, err, st);
  }
}

}  // namespace

// C[M, N] = A[M, K] B[N, K]^T with the epilogue ep (gemm.cuh). Returns MX_ERR_ARGUMENT for shapes the kernel does not
// take: K a multiple of 64, N of 64, 16-byte aligned pointers (A, B, out, bias, z) and row pitches (lda, ldb, ldo,
// ldz in bytes). ep.splits > 1 (STORE only): K in that many consecutive non-empty ranges, split s's partial product
// in out's rows s * ep.split_rows .. (split_rows at least M rounded up to 128).
int mx_gemm_launch(const void* A, int lda, const void* B, int ldb, int64_t M, int N, int K, const Epi& ep, int* err,
                   cudaStream_t st) {
  const bool f32_out = ep.mode == STORE || ep.mode == BIAS;
  const bool has_bias = ep.mode == BIAS || ep.mode == BIAS_SILU, uses_z = (ep.mode == BIAS_SILU && ep.z) ||
                                                                          ep.mode == DSILU;
  if (M < 1 || M > 0x7fffffff || N < 64 || N % 64 || K < 64 || K % 64 || lda < K || ldb < K || lda % 8 || ldb % 8 ||
      ((uintptr_t)A & 15) || ((uintptr_t)B & 15) || !err || !ep.out || ((uintptr_t)ep.out & 15) || ep.ldo < N ||
      ep.ldo % (f32_out ? 4 : 8) || (has_bias && (!ep.bias || ((uintptr_t)ep.bias & 15))) ||
      (uses_z && (!ep.z || ((uintptr_t)ep.z & 15) || ep.ldz < N || ep.ldz % 4)))
    return MX_ERR_ARGUMENT;
  const int splits = std::max(ep.splits, 1), nk = K / BK, nks = (nk + splits - 1) / splits;
  if (splits > 1 && (ep.mode != STORE || (splits - 1) * nks >= nk || ep.split_rows < (M + BM - 1) / BM * BM))
    return MX_ERR_ARGUMENT;
  if (encoder() != cudaSuccess) return MX_ERR_CUDA;
  const int bn = tile_width(N);
  CUtensorMap ta, tb, to, tz;
  if (!tensor_map(&ta, A, (uint64_t)M, (uint64_t)K, (uint64_t)lda, BM) ||
      !tensor_map(&tb, B, (uint64_t)N, (uint64_t)K, (uint64_t)ldb, (uint32_t)bn))
    return MX_ERR_ARGUMENT;
  // the epilogue's outputs go through TMA stores when their maps can be made, else through plain stores
  Epi e2 = ep;
  e2.splits = splits;
  e2.split_rows = splits > 1 ? ep.split_rows : 0;
  memset(&to, 0, sizeof(to));
  memset(&tz, 0, sizeof(tz));
  const uint64_t out_rows = splits > 1 ? (uint64_t)splits * (uint64_t)ep.split_rows : (uint64_t)M;
  const int epi = variant_of(ep.mode, ep.mode == BIAS_SILU && ep.z != nullptr);
  const int pcols = EPI_COLS;
  e2.tma = piece_map(&to, ep.out, out_rows, (uint64_t)N, (uint64_t)ep.ldo, f32_out, pcols) &&
           (!uses_z || piece_map(&tz, ep.z, (uint64_t)M, (uint64_t)N, (uint64_t)ep.ldz, true, pcols));
  const cudaError_t e = bn == 256   ? launch_epi<256>(epi, ta, tb, to, tz, M, N, K, e2, err, st)
                        : bn == 192 ? launch_epi<192>(epi, ta, tb, to, tz, M, N, K, e2, err, st)
                        : bn == 128 ? launch_epi<128>(epi, ta, tb, to, tz, M, N, K, e2, err, st)
                                    : launch_epi<64>(epi, ta, tb, to, tz, M, N, K, e2, err, st);
  return e == cudaSuccess ? MX_OK : MX_ERR_CUDA;
}

namespace {

// out[m][n] (pitch ldo) = the sum over s = 0 .. splits - 1, in that order, of ws[s * split_rows + m][n] (pitch n)
__global__ void split_sum_kernel(const float* __restrict__ ws, int splits, int split_rows, int M, int N, float* out,
                                 int ldo) {
  const long long total = (long long)M * N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int m = (int)(i / N), n = (int)(i % N);
    float acc = 0.0f;
    for (int q = 0; q < splits; q++) acc += ws[((size_t)q * split_rows + m) * N + n];
    out[(size_t)m * ldo + n] = acc;
  }
}

// K split so that the launch has about one output tile per SM: 1 when the output alone fills the SMs
int splits_for(int64_t M, int N, int K) {
  if (!g_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
  }
  const int bn = tile_width(N), nk = K / BK;
  const long long tiles = ((M + BM - 1) / BM) * (long long)(N / bn);
  const long long want = std::max<long long>(1, std::max(g_sms, 1) / std::max<long long>(tiles, 1));
  if (want < 2 || nk < 2) return 1;
  const int nks = (int)((nk + want - 1) / want);
  return (nk + nks - 1) / nks;  // every split non-empty
}

}  // namespace

// Floats of workspace a split-K product of this shape uses (0: it is not split).
size_t mx_split_workspace(int64_t M, int N, int K) {
  const int splits = splits_for(M, N, K);
  return splits > 1 ? (size_t)splits * (size_t)((M + BM - 1) / BM * BM) * (size_t)N : 0;
}

// out[M][N] (FP32, pitch ldo) = A B^T with K split across the SMs when the output has fewer tiles than SMs: the
// partial products go to ws (mx_split_workspace floats) and are added in split order by a second kernel, so the
// result is the same bits run to run. The weight gradients' products (M, N the layer's sizes, K the batch) are this
// shape: a few tiles, a long K.
int mx_gemm_store_split(const void* A, int lda, const void* B, int ldb, int64_t M, int N, int K, float* ws,
                        float* out, int ldo, int* err, cudaStream_t st) {
  const int splits = splits_for(M, N, K);
  if (splits == 1) {
    Epi ep{STORE, nullptr, nullptr, 0, out, ldo, 0, 1, 0};
    return mx_gemm_launch(A, lda, B, ldb, M, N, K, ep, err, st);
  }
  if (!ws || !out || ldo < N || ldo % 4 || ((uintptr_t)out & 15)) return MX_ERR_ARGUMENT;
  const int rows = (int)((M + BM - 1) / BM * BM);
  Epi ep{STORE, nullptr, nullptr, 0, ws, N, 0, splits, rows};
  const int rc = mx_gemm_launch(A, lda, B, ldb, M, N, K, ep, err, st);
  if (rc) return rc;
  const int grid = (int)std::min<long long>((M * (long long)N + 255) / 256, 148LL * 64);
  split_sum_kernel<<<grid, 256, 0, st>>>(ws, splits, rows, (int)M, N, out, ldo);
  return cudaGetLastError() == cudaSuccess ? MX_OK : MX_ERR_CUDA;
}

extern "C" int mx_gemm_bf16_split(const void* A, int32_t lda, const void* B, int32_t ldb, int64_t M, int32_t N,
                                  int32_t K, float* workspace, float* out, int32_t ldo, int32_t* err_flag,
                                  void* stream) {
  return mx_gemm_store_split(A, lda, B, ldb, M, N, K, workspace, out, ldo, err_flag, (cudaStream_t)stream);
}

extern "C" int64_t mx_gemm_split_workspace(int64_t M, int32_t N, int32_t K) {
  return (int64_t)mx_split_workspace(M, N, K);
}

extern "C" int mx_gemm_bf16(const void* A, int32_t lda, const void* B, int32_t ldb, int64_t M, int32_t N, int32_t K,
                            int32_t mode, const float* bias, float* z, int32_t ldz, void* out, int32_t ldo,
                            int32_t* err_flag, void* stream) {
  if (mode < STORE || mode > DSILU) return MX_ERR_ARGUMENT;
  Epi ep{mode, bias, z, ldz, out, ldo, 0, 1, 0};
  return mx_gemm_launch(A, lda, B, ldb, M, N, K, ep, err_flag, (cudaStream_t)stream);
}

namespace {

constexpr int MAX_LAYERS = 8;
constexpr double X_FLOOR = 1e-30;  // log10 x and log10(J + floor) of the features and targets
constexpr double AUDIT_FLOOR = 1e-20;  // species the audit and the spread gate judge: mole fraction above this

// ---- features: one warp per cell ----
// f = log10 x (ns, floored), log10 T, log10 P, log10 dt, log10 h (the carried step: how stiff and how settled the
// cell is), log10(J + floor) (nj), zeros to kin; standardised, BF16. in_range: every feature within the training
// set's [lo, hi] (and finite).
__global__ void features_kernel(const double* x, const double* T, const double* P, const double* dt, const double* h,
                                const double* J, int B, int ns, int nj, int kin, const float* mean,
                                const float* inv_std, const float* lo, const float* hi, __nv_bfloat16* feat,
                                int* in_range) {
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = (int)(threadIdx.x & 31);
  if (warp >= B) return;
  const size_t cell = (size_t)warp;
  const int nf = ns + 4 + nj;
  bool inside = true;
  for (int f = lane; f < kin; f += 32) {
    double v = 0.0;
    if (f < ns)
      v = log10(fmax(x[cell * ns + f], X_FLOOR));
    else if (f == ns)
      v = log10(T[cell]);
    else if (f == ns + 1)
      v = log10(P[cell]);
    else if (f == ns + 2)
      v = log10(fmax(dt[cell], X_FLOOR));
    else if (f == ns + 3)
      v = log10(fmax(h[cell], X_FLOOR));
    else if (f < nf)
      v = log10(J[cell * nj + (f - ns - 4)] + X_FLOOR);
    float q = 0.0f;
    if (f < nf) {
      const float vf = (float)v;
      inside = inside && (vf >= lo[f]) && (vf <= hi[f]);
      q = (vf - mean[f]) * inv_std[f];
    }
    feat[cell * kin + f] = __float2bfloat16_rn(q);
  }
  inside = __all_sync(0xffffffffu, inside);
  if (in_range && lane == 0) in_range[cell] = inside ? 1 : 0;
}

// ---- training: the loss's gradient at the heads, transposes, bias sums, Adam ----

// The gradient of the weighted loss at the heads, BF16, zero in the padding columns (standardised targets, per-sample
// bootstrap weight w of each head): for delta 0 the mean square error, dpred = 2 w (pred - tgt) / (M heads nt); for
// delta > 0 the Huber loss of width delta (quadratic within delta, linear beyond, so the few large misses of far
// from settled cells do not outweigh the many small ones the gate must get right): dpred = 2 w clamp(pred - tgt,
// -delta, delta) / (M heads nt). *loss += the weighted loss (for reports).
__global__ void loss_grad_kernel(const float* pred, int ldp, const float* tgt, const float* wts, int M, int nt,
                                 int heads, int kout, float delta, __nv_bfloat16* dpred, float* loss) {
  __shared__ float part[256];
  const float scale = 1.0f / ((float)M * (float)heads * (float)nt);
  float acc = 0.0f;
  const long long total = (long long)M * kout;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(idx / kout), col = (int)(idx % kout), head = col / nt, i = col - head * nt;
    float g = 0.0f;
    if (head < heads) {
      const float d = pred[(size_t)row * ldp + col] - tgt[(size_t)row * nt + i];
      const float w = wts[(size_t)row * heads + head];
      if (delta > 0.0f && fabsf(d) > delta) {
        g = 2.0f * w * copysignf(delta, d) * scale;
        acc += w * delta * (2.0f * fabsf(d) - delta);
      } else {
        g = 2.0f * w * d * scale;
        acc += w * d * d;
      }
    }
    dpred[(size_t)row * kout + col] = __float2bfloat16_rn(g);
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0 && loss) atomicAdd(loss, part[0] * scale);
}

// out [C][R] = in [R][C] (BF16; R and C even, rows 4-byte aligned), 64 x 64 tiles through shared memory: each warp
// reads and writes 128 contiguous bytes of a row as 32 pairs; the tile's odd row stride (65 elements) keeps the
// column reads free of bank conflicts.
__global__ void transpose_kernel(const __nv_bfloat16* in, int R, int C, __nv_bfloat16* out) {
  __shared__ __nv_bfloat16 tile[64][65];
  const int c0 = (int)blockIdx.x * 64, r0 = (int)blockIdx.y * 64, tx = (int)threadIdx.x, ty = (int)threadIdx.y;
  const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
  for (int k = ty; k < 64; k += 8) {
    const int r = r0 + k, c = c0 + 2 * tx;
    __nv_bfloat162 v = __halves2bfloat162(zero, zero);
    if (r < R && c < C) v = *reinterpret_cast<const __nv_bfloat162*>(in + (size_t)r * C + c);  // c + 1 < C: C even
    tile[k][2 * tx] = v.x;
    tile[k][2 * tx + 1] = v.y;
  }
  __syncthreads();
  for (int k = ty; k < 64; k += 8) {
    const int c = c0 + k, r = r0 + 2 * tx;
    if (c < C && r < R)  // r + 1 < R: R even
      *reinterpret_cast<__nv_bfloat162*>(out + (size_t)c * R + r) = __halves2bfloat162(tile[2 * tx][k], tile[2 * tx + 1][k]);
  }
}

// part[chunk][n] = sum over the chunk's rows of g[m][n] (BF16), rows in ascending order per thread, then the 8
// threads' sums in order: a fixed order, so the bias gradients do not depend on the launch.
__global__ void colsum_part_kernel(const __nv_bfloat16* g, int M, int N, int rows_per_chunk, float* part) {
  __shared__ float s[8][33];
  const int n = (int)blockIdx.x * 32 + (int)threadIdx.x, ty = (int)threadIdx.y;
  const int m0 = (int)blockIdx.y * rows_per_chunk, m1 = min(M, m0 + rows_per_chunk);
  float acc = 0.0f;
  if (n < N)
    for (int m = m0 + ty; m < m1; m += 8) acc += __bfloat162float(g[(size_t)m * N + n]);
  s[ty][threadIdx.x] = acc;
  __syncthreads();
  if (ty == 0 && n < N) {
    float t = 0.0f;
    for (int k = 0; k < 8; k++) t += s[k][threadIdx.x];
    part[(size_t)blockIdx.y * N + n] = t;
  }
}

__global__ void colsum_final_kernel(const float* part, int chunks, int N, float* out) {
  const int n = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (n >= N) return;
  float t = 0.0f;
  for (int k = 0; k < chunks; k++) t += part[(size_t)k * N + n];
  out[n] = t;
}

struct Layers {
  int n;                      // layers with weights (hidden + output)
  long long w_off[MAX_LAYERS], b_off[MAX_LAYERS];  // offsets into the FP32 parameters (and gradients, moments)
  long long wb_off[MAX_LAYERS];                    // offsets into the BF16 weight copies (W and W^T)
  int rows[MAX_LAYERS], cols[MAX_LAYERS];          // W_l is [rows][cols] = [out][in]
};

// Adam on every parameter (FP32 master copies), then the BF16 weights in both layouts: W [out][in] for the forward
// GEMMs and W^T [in][out] for the backward dX GEMMs.
__global__ void adam_kernel(float* p, const float* g, float* m1, float* m2, long long P, float lr, float b1, float b2,
                            float eps, float c1, float c2, Layers L, __nv_bfloat16* wb, __nv_bfloat16* wtb) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi, b = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float v = p[i] - lr * (a * c1) / (sqrtf(b * c2) + eps);
    p[i] = v;
    for (int l = 0; l < L.n; l++) {
      const long long k = i - L.w_off[l];
      if (k >= 0 && k < (long long)L.rows[l] * L.cols[l]) {
        const int r = (int)(k / L.cols[l]), c = (int)(k % L.cols[l]);
        const __nv_bfloat16 q = __float2bfloat16_rn(v);
        wb[L.wb_off[l] + k] = q;
        wtb[L.wb_off[l] + (long long)c * L.rows[l] + r] = q;
      }
    }
  }
}

// The BF16 copies of the master weights (after they were set from the host).
__global__ void weights_bf16_kernel(const float* p, long long P, Layers L, __nv_bfloat16* wb, __nv_bfloat16* wtb) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P; i += (long long)gridDim.x * blockDim.x) {
    for (int l = 0; l < L.n; l++) {
      const long long k = i - L.w_off[l];
      if (k >= 0 && k < (long long)L.rows[l] * L.cols[l]) {
        const int r = (int)(k / L.cols[l]), c = (int)(k % L.cols[l]);
        const __nv_bfloat16 q = __float2bfloat16_rn(p[i]);
        wb[L.wb_off[l] + k] = q;
        wtb[L.wb_off[l] + (long long)c * L.rows[l] + r] = q;
      }
    }
  }
}

// ---- the gated call ----

struct GateArgs {
  const double *x, *T, *dt, *h;
  int B, ns, nel, nt, heads, ldp;
  const float *pred, *tmean, *tstd;
  const int* in_range;
  const double* atoms;  // [ns][nel], network order
  double spread_max, proj_max, drift, atol, etot;
  int audit_every;
  unsigned seed;
  double *x_out, *h_out, *steps;
  int *done, *flag, *status, *count;
  int* list;        // cells the Rodas3 fallback steps: rejected and audited
  int* list_count;  // [0] listed, [1] the fallback kernel's queue
  int* audit_cells;
  double* audit_x;  // [audit_cap][ns] the audited cells' proposals
  int audit_cap;
  int* audit_count;
  unsigned long long* stats;  // accepted, audited, out of range, spread, projection, refused or non-finite
  double* diag;  // propose mode: per cell the spread, the projection's size, 1 if usable and in range, the h proposal
};

__device__ __forceinline__ unsigned mix32(unsigned v) {  // an integer hash (xorshift-multiply) for the audit draw
  v ^= v >> 16;
  v *= 0x7feb352du;
  v ^= v >> 15;
  v *= 0x846ca68bu;
  v ^= v >> 16;
  return v;
}

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double wmax(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// One warp per cell: the heads' mean proposal of log10 x and log10 h, the ensemble's spread, the element-share
// projection, and the decision. Accepted cells get their outputs here; rejected and audited cells are listed for the
// Rodas3 fallback. Shared memory per warp: the proposal [ns] and the element system.
__global__ void gate_kernel(GateArgs g) {
  extern __shared__ double gate_smem[];
  constexpr int ME = MX_MAX_ELEMENTS;
  const int wib = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
  const int cell = (int)(blockIdx.x * (blockDim.x >> 5)) + wib;
  if (cell >= g.B) return;
  const int ns = g.ns, nel = g.nel, nt = g.nt;
  double* p = gate_smem + (size_t)wib * (ns + ME * ME + 4 * ME + 4);
  double* mat = p + ns;        // [ME][ME]
  double* rhs = mat + ME * ME;  // [ME]
  double* lam = rhs + ME;       // [ME]
  double* e0 = lam + ME;        // [ME]
  double* e1 = e0 + ME;         // [ME]
  const double* xin = g.x + (size_t)cell * ns;
  const float* pr = g.pred + (size_t)cell * g.ldp;
  const double Tc = g.T[cell], dtc = g.dt[cell];
  bool usable = isfinite(Tc) && Tc >= MX_T_MIN && Tc <= MX_T_MAX && dtc > 0.0 && isfinite(dtc);
  // proposal (mean over heads) and spread (the heads' sample deviation), in dex, per species
  double spread = 0.0;
  for (int i = lane; i < nt; i += 32) {
    double mu = 0.0;
    double d[8];
    for (int k = 0; k < g.heads; k++) {
      d[k] = (double)pr[k * nt + i] * (double)g.tstd[i] + (double)g.tmean[i];
      mu += d[k];
    }
    mu /= g.heads;
    double var = 0.0;
    for (int k = 0; k < g.heads; k++) var += (d[k] - mu) * (d[k] - mu);
    const double sd = sqrt(var / fmax(1.0, (double)(g.heads - 1)));
    if (i < ns) {
      const double xi = xin[i];
      const double q = exp10(log10(fmax(xi, X_FLOOR)) + mu);
      p[i] = q;
      if (fmax(xi, q) > AUDIT_FLOOR) spread = fmax(spread, sd);
      usable = usable && isfinite(q) && isfinite(xi) && xi >= 0.0;
    } else {
      lam[0] = mu;  // log10 h, read after the next warp sync
    }
  }
  __syncwarp();
  const double log_h = lam[0];
  spread = wmax(spread);
  usable = __all_sync(0xffffffffu, usable);
  const bool in_range = g.in_range[cell] != 0;
  // normalise, then the projection onto the input's element shares: twice x <- x (1 + sum_e lambda_e a_ie), lambda
  // from (A X A^T) lambda = e0 s1 / s0 - e1 (the guard's correction, guard.cuh:24-57, without its clamp)
  double s = 0.0;
  for (int i = lane; i < ns; i += 32) s += p[i];
  s = wsum(s);
  for (int i = lane; i < ns; i += 32) p[i] /= s;
  __syncwarp();
  double proj = 0.0;
  for (int e = 0; e < nel; e++) {
    double a0 = 0.0;
    for (int i = lane; i < ns; i += 32) a0 = fma(g.atoms[i * nel + e], xin[i], a0);
    a0 = wsum(a0);
    if (lane == 0) e0[e] = a0;
  }
  for (int it = 0; it < 2; it++) {
    for (int e = 0; e < nel; e++) {
      double a1 = 0.0;
      for (int i = lane; i < ns; i += 32) a1 = fma(g.atoms[i * nel + e], p[i], a1);
      a1 = wsum(a1);
      if (lane == 0) e1[e] = a1;
      for (int f = e; f < nel; f++) {
        double m = 0.0;
        for (int i = lane; i < ns; i += 32) m = fma(g.atoms[i * nel + e] * g.atoms[i * nel + f], p[i], m);
        m = wsum(m);
        if (lane == 0) mat[e * ME + f] = m;
      }
    }
    __syncwarp();
    if (lane == 0) {  // LDL^T of the small system, elements whose pivot vanishes left out
      double s0 = 0.0, s1 = 0.0, m0[ME];
      for (int e = 0; e < nel; e++) {
        s0 += e0[e];
        s1 += e1[e];
      }
      for (int e = 0; e < nel; e++) {
        m0[e] = mat[e * ME + e];
        rhs[e] = fma(e0[e], s1 / s0, -e1[e]);
      }
      for (int k = 0; k < nel; k++) {
        if (!(mat[k * ME + k] > MX_ELEMENT_PIVOT_MIN * m0[k])) continue;
        for (int j = k + 1; j < nel; j++) {
          const double l = mat[k * ME + j] / mat[k * ME + k];
          for (int f = j; f < nel; f++) mat[j * ME + f] = fma(-l, mat[k * ME + f], mat[j * ME + f]);
          rhs[j] = fma(-l, rhs[k], rhs[j]);
        }
      }
      for (int k = nel - 1; k >= 0; k--) {
        lam[k] = 0.0;
        if (!(mat[k * ME + k] > MX_ELEMENT_PIVOT_MIN * m0[k])) continue;
        double b = rhs[k];
        for (int f = k + 1; f < nel; f++) b = fma(-mat[k * ME + f], lam[f], b);
        lam[k] = b / mat[k * ME + k];
      }
    }
    __syncwarp();
    double gmax = 0.0, sum = 0.0;
    for (int i = lane; i < ns; i += 32) {
      double gi = 0.0;
      for (int e = 0; e < nel; e++) gi = fma(lam[e], g.atoms[i * nel + e], gi);
      gmax = fmax(gmax, fabs(gi));
      const double q = p[i] * (1.0 + gi);
      p[i] = q;
      sum += q;
      usable = usable && q >= 0.0 && isfinite(q);
    }
    gmax = wmax(gmax);
    if (it == 0) proj = gmax;
    sum = wsum(sum);
    __syncwarp();
    for (int i = lane; i < ns; i += 32) p[i] /= sum;
    __syncwarp();
  }
  usable = __all_sync(0xffffffffu, usable);
  // the guard's drift test on the projected proposal (guard.cuh:13-21), one accepted step's atol allowance
  bool drift = false;
  {
    double s0 = 0.0, s1 = 0.0;
    double a1s[ME];
    for (int e = 0; e < nel; e++) {
      double a1 = 0.0;
      for (int i = lane; i < ns; i += 32) a1 = fma(g.atoms[i * nel + e], p[i], a1);
      a1s[e] = wsum(a1);
      s0 += e0[e];
      s1 += a1s[e];
    }
    for (int e = 0; e < nel; e++)
      drift = drift || fabs(a1s[e] / s1 - e0[e] / s0) > g.drift * e0[e] / s0 + 2.0 * g.atol * g.etot / s0;
  }
  const double hprop = exp10(log_h);
  if (g.diag) {  // propose mode: the projected proposal of every cell and the gate's measures, nothing decided
    double* xo = g.x_out + (size_t)cell * ns;
    for (int i = lane; i < ns; i += 32) xo[i] = p[i];
    if (lane == 0) {
      double* d = g.diag + (size_t)cell * 4;
      d[0] = spread;
      d[1] = drift ? INFINITY : proj;
      d[2] = (usable && in_range && isfinite(hprop)) ? 1.0 : 0.0;
      d[3] = hprop;
    }
    return;
  }
  const bool spread_ok = spread <= g.spread_max, proj_ok = proj <= g.proj_max && !drift;
  const bool accept = usable && in_range && spread_ok && proj_ok && isfinite(hprop);
  const bool audit = accept && g.audit_every > 0 && (mix32((unsigned)cell * 2654435761u ^ g.seed) % (unsigned)g.audit_every) == 0;
  if (accept) {
    double* xo = g.x_out + (size_t)cell * ns;
    for (int i = lane; i < ns; i += 32) xo[i] = p[i];
  }
  int slot = -1;
  if (lane == 0) {
    atomicAdd(g.count + MX_COUNT_QUEUE, 1);
    if (accept) {
      g.h_out[cell] = fmin(fmax(hprop, MX_H_MIN), dtc);
      g.done[cell] = 1;
      g.steps[cell] = 0.0;
      g.flag[cell] = 0;
      g.status[cell] = 0;
      atomicAdd(g.stats + 0, 1ull);
    } else {
      atomicAdd(g.stats + (!usable ? 5 : !in_range ? 2 : !spread_ok ? 3 : 4), 1ull);
    }
    if (!accept || audit) g.list[atomicAdd(g.list_count, 1)] = cell;
    if (audit) {
      atomicAdd(g.stats + 1, 1ull);
      slot = atomicAdd(g.audit_count, 1);
      if (slot < g.audit_cap) g.audit_cells[slot] = cell;
    }
  }
  slot = __shfl_sync(0xffffffffu, slot, 0);
  if (slot >= 0 && slot < g.audit_cap)
    for (int i = lane; i < ns; i += 32) g.audit_x[(size_t)slot * ns + i] = p[i];
}

// The audit: per audited cell (one warp each) and species, |proposal - Rodas3| / Rodas3 for species above the floor
// in the Rodas3 result (else 0), into err [audit_cap][ns] (FP32).
__global__ void audit_kernel(const int* cells, const int* count, int cap, const double* audit_x, const double* x_out,
                             int ns, float* err) {
  const int k = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = (int)(threadIdx.x & 31);
  if (k >= min(*count, cap)) return;
  const double* ref = x_out + (size_t)cells[k] * ns;
  for (int i = lane; i < ns; i += 32) {
    const double r = ref[i];
    err[(size_t)k * ns + i] = r > AUDIT_FLOOR ? (float)(fabs(audit_x[(size_t)k * ns + i] - r) / r) : 0.0f;
  }
}

int round64(int v) { return (v + 63) / 64 * 64; }

// The heads' padded width: the first multiple of 64 at or above v that a 128-, 192- or 256-column tile divides, so
// that their GEMM runs in wide tiles (A, the 65,536-row activations, is read once per column tile).
int heads_width(int v) {
  for (int w = round64(v);; w += 64)
    if (w % 128 == 0 || w % 192 == 0) return w;
}

}  // namespace

struct mx_surrogate {
  int device = 0, ns = 0, nj = 0, nel = 0, hidden = 0, layers = 0, heads = 0;
  std::vector<void*> persist;  // parameters, moments, weight copies, scaling, atoms: freed by mx_sur_destroy
  int nf = 0, kin = 0, nt = 0, kout = 0;
  long long P = 0, PW = 0;  // FP32 parameters; BF16 weight entries
  Layers L{};
  float *param = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
  __nv_bfloat16 *wb = nullptr, *wtb = nullptr;
  float *fmean = nullptr, *finv = nullptr, *flo = nullptr, *fhi = nullptr, *tmean = nullptr, *tstd = nullptr;
  double* atoms = nullptr;
  double etot = 0.0;
  int* err = nullptr;
  int step = 0;
  // training workspace for a batch of up to `rows` rows
  int64_t rows = 0;
  std::vector<void*> work;
  __nv_bfloat16* act[MAX_LAYERS] = {};  // a_0 (the features are the caller's) .. a_L
  float* z[MAX_LAYERS] = {};
  float* pred = nullptr;
  __nv_bfloat16 *dz = nullptr, *dz2 = nullptr, *dzt = nullptr, *at = nullptr;
  float* colpart = nullptr;
  float* ws = nullptr;  // split-K partial products of the weight gradients
  // the gated call's workspace for up to `call_rows` cells
  int64_t call_rows = 0;
  std::vector<void*> call_work;
  __nv_bfloat16 *cfeat = nullptr, *cbuf[2] = {nullptr, nullptr};
  float* cpred = nullptr;
  int *in_range = nullptr, *list = nullptr, *list_count = nullptr;
};

namespace {

constexpr int CHUNK = 65536;  // rows of one inference pass: two BF16 activation buffers of 64 MB, about L2's size

template <typename T>
cudaError_t alloc(std::vector<void*>& keep, T** p, size_t n) {
  void* q = nullptr;
  const cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
  if (e == cudaSuccess) {
    keep.push_back(q);
    *p = (T*)q;
  }
  return e;
}

void free_all(std::vector<void*>& keep) {
  for (void* q : keep) cudaFree(q);
  keep.clear();
}

// the forward pass of `M` rows of features feat [M][kin]: hidden layers into act (training: z kept) or the two
// chunk buffers (inference), the heads into pred [M][kout]
int forward(mx_surrogate* s, const __nv_bfloat16* feat, int64_t M, float* pred, bool keep, cudaStream_t st) {
  const __nv_bfloat16* a = feat;
  int K = s->kin;
  for (int l = 0; l < s->layers; l++) {
    __nv_bfloat16* out = keep ? s->act[l + 1] : s->cbuf[l & 1];
    Epi ep{BIAS_SILU, s->param + s->L.b_off[l], keep ? s->z[l] : nullptr, s->hidden, out, s->hidden};
    const int rc = mx_gemm_launch(a, K, s->wb + s->L.wb_off[l], K, M, s->hidden, K, ep, s->err, st);
    if (rc) return rc;
    a = out;
    K = s->hidden;
  }
  const int l = s->layers;
  Epi ep{BIAS, s->param + s->L.b_off[l], nullptr, 0, pred, s->kout};
  return mx_gemm_launch(a, K, s->wb + s->L.wb_off[l], K, M, s->kout, K, ep, s->err, st);
}

cudaError_t grow_train(mx_surrogate* s, int64_t M) {
  if (M <= s->rows) return cudaSuccess;
  free_all(s->work);
  s->rows = 0;
  cudaError_t e = cudaSuccess;
  for (int l = 1; l <= s->layers && e == cudaSuccess; l++) e = alloc(s->work, &s->act[l], (size_t)M * s->hidden);
  for (int l = 0; l < s->layers && e == cudaSuccess; l++) e = alloc(s->work, &s->z[l], (size_t)M * s->hidden);
  const int wide = std::max(std::max(s->hidden, s->kout), s->kin);
  if (e == cudaSuccess) e = alloc(s->work, &s->pred, (size_t)M * s->kout);
  if (e == cudaSuccess) e = alloc(s->work, &s->dz, (size_t)M * wide);
  if (e == cudaSuccess) e = alloc(s->work, &s->dz2, (size_t)M * wide);
  if (e == cudaSuccess) e = alloc(s->work, &s->dzt, (size_t)M * wide);
  if (e == cudaSuccess) e = alloc(s->work, &s->at, (size_t)M * wide);
  if (e == cudaSuccess) e = alloc(s->work, &s->colpart, (size_t)64 * wide);
  size_t ws = 0;
  for (int l = 0; l <= s->layers; l++) ws = std::max(ws, mx_split_workspace(s->L.rows[l], s->L.cols[l], (int)M));
  if (e == cudaSuccess && ws) e = alloc(s->work, &s->ws, ws);
  if (e == cudaSuccess) s->rows = M;
  return e;
}

cudaError_t grow_call(mx_surrogate* s, int64_t B) {
  if (B <= s->call_rows) return cudaSuccess;
  free_all(s->call_work);
  s->call_rows = 0;
  const int64_t chunk = std::min<int64_t>(B, CHUNK);
  cudaError_t e = alloc(s->call_work, &s->cfeat, (size_t)B * s->kin);
  if (e == cudaSuccess) e = alloc(s->call_work, &s->cbuf[0], (size_t)chunk * s->hidden);
  if (e == cudaSuccess) e = alloc(s->call_work, &s->cbuf[1], (size_t)chunk * s->hidden);
  if (e == cudaSuccess) e = alloc(s->call_work, &s->cpred, (size_t)B * s->kout);
  if (e == cudaSuccess) e = alloc(s->call_work, &s->in_range, (size_t)B);
  if (e == cudaSuccess) e = alloc(s->call_work, &s->list, (size_t)B);
  if (e == cudaSuccess) e = alloc(s->call_work, &s->list_count, 2);
  if (e == cudaSuccess) s->call_rows = B;
  return e;
}

int blocks_for(long long n, int threads) { return (int)std::min<long long>((n + threads - 1) / threads, 148LL * 64); }

}  // namespace

extern "C" int mx_sur_create(int32_t ns, int32_t nj, int32_t nel, const double* atoms, int32_t hidden, int32_t layers,
                             int32_t heads, int32_t device, mx_surrogate** out, char* err, size_t errlen) {
  if (!out || !atoms || ns < 1 || ns > MX_MAX_SPECIES || nj < 0 || nel < 1 || nel > MX_MAX_ELEMENTS || hidden < 64 ||
      hidden % 64 || layers < 1 || layers + 1 > MAX_LAYERS || heads < 1 || heads > 8) {
    set_error(err, errlen, "mx_sur_create: sizes out of range (ns %d, nj %d, nel %d, hidden %d, layers %d, heads %d)",
              ns, nj, nel, hidden, layers, heads);
    return MX_ERR_ARGUMENT;
  }
  *out = nullptr;
  DeviceScope scope(device);
  if (scope.status != cudaSuccess) {
    set_error(err, errlen, "mx_sur_create: device %d: %s", device, cudaGetErrorString(scope.status));
    return MX_ERR_CUDA;
  }
  mx_surrogate* s = new (std::nothrow) mx_surrogate();
  if (!s) return MX_ERR_CUDA;
  s->device = device;
  s->ns = ns;
  s->nj = nj;
  s->nel = nel;
  s->hidden = hidden;
  s->layers = layers;
  s->heads = heads;
  s->nf = ns + 4 + nj;
  s->kin = round64(s->nf);
  s->nt = ns + 1;
  s->kout = heads_width(heads * s->nt);
  Layers& L = s->L;
  L.n = layers + 1;
  long long off = 0, woff = 0;
  for (int l = 0; l <= layers; l++) {
    L.rows[l] = l < layers ? hidden : s->kout;
    L.cols[l] = l == 0 ? s->kin : hidden;
    L.w_off[l] = off;
    off += (long long)L.rows[l] * L.cols[l];
    L.b_off[l] = off;
    off += L.rows[l];
    L.wb_off[l] = woff;
    woff += (long long)L.rows[l] * L.cols[l];
  }
  s->P = off;
  s->PW = woff;
  double etot = 0.0;
  for (int i = 0; i < ns * nel; i++) etot += atoms[i];
  s->etot = etot;
  std::vector<void*>& base = s->persist;
  cudaError_t e = alloc(base, &s->param, (size_t)s->P);
  if (e == cudaSuccess) e = alloc(base, &s->grad, (size_t)s->P);
  if (e == cudaSuccess) e = alloc(base, &s->m1, (size_t)s->P);
  if (e == cudaSuccess) e = alloc(base, &s->m2, (size_t)s->P);
  if (e == cudaSuccess) e = alloc(base, &s->wb, (size_t)s->PW);
  if (e == cudaSuccess) e = alloc(base, &s->wtb, (size_t)s->PW);
  if (e == cudaSuccess) e = alloc(base, &s->fmean, (size_t)s->kin);
  if (e == cudaSuccess) e = alloc(base, &s->finv, (size_t)s->kin);
  if (e == cudaSuccess) e = alloc(base, &s->flo, (size_t)s->kin);
  if (e == cudaSuccess) e = alloc(base, &s->fhi, (size_t)s->kin);
  if (e == cudaSuccess) e = alloc(base, &s->tmean, (size_t)s->nt);
  if (e == cudaSuccess) e = alloc(base, &s->tstd, (size_t)s->nt);
  if (e == cudaSuccess) e = alloc(base, &s->atoms, (size_t)ns * nel);
  if (e == cudaSuccess) e = alloc(base, &s->err, 1);
  if (e == cudaSuccess) e = cudaMemcpy(s->atoms, atoms, sizeof(double) * ns * nel, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(s->param, 0, sizeof(float) * s->P);
  if (e == cudaSuccess) e = cudaMemset(s->m1, 0, sizeof(float) * s->P);
  if (e == cudaSuccess) e = cudaMemset(s->m2, 0, sizeof(float) * s->P);
  if (e == cudaSuccess) e = cudaMemset(s->wb, 0, sizeof(__nv_bfloat16) * s->PW);
  if (e == cudaSuccess) e = cudaMemset(s->wtb, 0, sizeof(__nv_bfloat16) * s->PW);
  if (e == cudaSuccess) e = cudaMemset(s->err, 0, sizeof(int));
  if (e == cudaSuccess) {  // unit scaling and the widest range until mx_sur_set_scaling
    const int n = std::max(s->kin, s->nt);
    std::vector<float> zero(n, 0.0f), one(n, 1.0f), lo(n, -3e38f), hi(n, 3e38f);
    e = cudaMemcpy(s->fmean, zero.data(), sizeof(float) * s->kin, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->finv, one.data(), sizeof(float) * s->kin, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->flo, lo.data(), sizeof(float) * s->kin, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->fhi, hi.data(), sizeof(float) * s->kin, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->tmean, zero.data(), sizeof(float) * s->nt, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->tstd, one.data(), sizeof(float) * s->nt, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    free_all(s->persist);
    set_error(err, errlen, "mx_sur_create: %s", cudaGetErrorString(e));
    delete s;
    return MX_ERR_CUDA;
  }
  *out = s;
  return MX_OK;
}

extern "C" int mx_sur_info(const mx_surrogate* s, int64_t* values, int32_t n) {
  if (!s || !values) return MX_ERR_ARGUMENT;
  const int64_t v[] = {s->nf, s->kin, s->nt, s->kout, s->P, s->layers, s->hidden, s->heads, s->step};
  for (int i = 0; i < n && i < (int)(sizeof v / sizeof v[0]); i++) values[i] = v[i];
  return MX_OK;
}

extern "C" int mx_sur_set_scaling(mx_surrogate* s, const float* feat_mean, const float* feat_std, const float* feat_lo,
                                  const float* feat_hi, const float* tgt_mean, const float* tgt_std) {
  if (!s || !feat_mean || !feat_std || !feat_lo || !feat_hi || !tgt_mean || !tgt_std) return MX_ERR_ARGUMENT;
  DeviceScope scope(s->device);
  std::vector<float> mean(s->kin, 0.0f), inv(s->kin, 0.0f), lo(s->kin, -3e38f), hi(s->kin, 3e38f);
  for (int f = 0; f < s->nf; f++) {
    if (!(feat_std[f] >= 0.0f) || !std::isfinite(feat_mean[f])) return MX_ERR_ARGUMENT;
    mean[f] = feat_mean[f];
    inv[f] = feat_std[f] > 0.0f ? 1.0f / feat_std[f] : 1.0f;
    lo[f] = feat_lo[f];
    hi[f] = feat_hi[f];
  }
  std::vector<float> tm(tgt_mean, tgt_mean + s->nt), ts(tgt_std, tgt_std + s->nt);
  for (int i = 0; i < s->nt; i++)
    if (!(ts[i] > 0.0f) || !std::isfinite(tm[i])) return MX_ERR_ARGUMENT;
  cudaError_t e = cudaMemcpy(s->fmean, mean.data(), sizeof(float) * s->kin, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(s->finv, inv.data(), sizeof(float) * s->kin, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(s->flo, lo.data(), sizeof(float) * s->kin, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(s->fhi, hi.data(), sizeof(float) * s->kin, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(s->tmean, tm.data(), sizeof(float) * s->nt, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(s->tstd, ts.data(), sizeof(float) * s->nt, cudaMemcpyHostToDevice);
  return e == cudaSuccess ? MX_OK : MX_ERR_CUDA;
}

extern "C" int mx_sur_features(mx_surrogate* s, const double* x, const double* T, const double* P, const double* dt,
                               const double* h, const double* J, int64_t B, void* feat, int32_t* in_range,
                               void* stream) {
  if (!s || B < 0 || B > 0x7fffffff || (B > 0 && (!x || !T || !P || !dt || !h || !feat || (s->nj > 0 && !J))))
    return MX_ERR_ARGUMENT;
  if (B == 0) return MX_OK;
  DeviceScope scope(s->device);
  const int threads = 256, blocks = (int)((B * 32 + threads - 1) / threads);
  features_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(x, T, P, dt, h, J, (int)B, s->ns, s->nj, s->kin,
                                                                s->fmean, s->finv, s->flo, s->fhi,
                                                                (__nv_bfloat16*)feat, in_range);
  return cudaGetLastError() == cudaSuccess ? MX_OK : MX_ERR_CUDA;
}

extern "C" int mx_sur_forward(mx_surrogate* s, const void* feat, int64_t B, float* pred, void* stream) {
  if (!s || B < 0 || B > 0x7fffffff || (B > 0 && (!feat || !pred))) return MX_ERR_ARGUMENT;
  if (B == 0) return MX_OK;
  DeviceScope scope(s->device);
  if (grow_call(s, std::min<int64_t>(B, CHUNK)) != cudaSuccess) return MX_ERR_CUDA;
  const __nv_bfloat16* f = (const __nv_bfloat16*)feat;
  for (int64_t r = 0; r < B; r += CHUNK) {
    const int64_t rows = std::min<int64_t>(CHUNK, B - r);
    const int rc = forward(s, f + r * s->kin, rows, pred + r * s->kout, false, (cudaStream_t)stream);
    if (rc) return rc;
  }
  return MX_OK;
}

extern "C" int mx_sur_train_step(mx_surrogate* s, const void* feat, const float* tgt, const float* wts, int64_t M,
                                 float lr, float delta, float* loss, void* stream) {
  if (!s || !feat || !tgt || !wts || M < 64 || M % 64 || M > 0x7fffffff || !(lr >= 0.0f) || !(delta >= 0.0f))
    return MX_ERR_ARGUMENT;
  DeviceScope scope(s->device);
  cudaStream_t st = (cudaStream_t)stream;
  if (grow_train(s, M) != cudaSuccess) return MX_ERR_CUDA;
  const __nv_bfloat16* f = (const __nv_bfloat16*)feat;
  int rc = forward(s, f, M, s->pred, true, st);
  if (rc) return rc;
  loss_grad_kernel<<<blocks_for(M * s->kout, 256), 256, 0, st>>>(s->pred, s->kout, tgt, wts, (int)M, s->nt, s->heads,
                                                                  s->kout, delta, s->dz, loss);
  __nv_bfloat16 *dZ = s->dz, *dZ2 = s->dz2;
  int N = s->kout;
  for (int l = s->layers; l >= 0; l--) {
    const __nv_bfloat16* a = l == 0 ? f : s->act[l];
    const int K = s->L.cols[l];
    const dim3 tb(32, 8);
    transpose_kernel<<<dim3((N + 63) / 64, (unsigned)((M + 63) / 64)), tb, 0, st>>>(dZ, (int)M, N, s->dzt);
    transpose_kernel<<<dim3((K + 63) / 64, (unsigned)((M + 63) / 64)), tb, 0, st>>>(a, (int)M, K, s->at);
    rc = mx_gemm_store_split(s->dzt, (int)M, s->at, (int)M, N, K, (int)M, s->ws, s->grad + s->L.w_off[l], K, s->err,
                             st);
    if (rc) return rc;
    const int chunks = (int)std::min<int64_t>(64, (M + 127) / 128), per = (int)((M + chunks - 1) / chunks);
    colsum_part_kernel<<<dim3((N + 31) / 32, chunks), tb, 0, st>>>(dZ, (int)M, N, per, s->colpart);
    colsum_final_kernel<<<(N + 127) / 128, 128, 0, st>>>(s->colpart, chunks, N, s->grad + s->L.b_off[l]);
    if (l > 0) {
      Epi dx{DSILU, nullptr, s->z[l - 1], s->hidden, dZ2, K};
      rc = mx_gemm_launch(dZ, N, s->wtb + s->L.wb_off[l], N, M, K, N, dx, s->err, st);
      if (rc) return rc;
      std::swap(dZ, dZ2);
      N = K;
    }
  }
  s->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f / (1.0f - powf(b1, (float)s->step)), c2 = 1.0f / (1.0f - powf(b2, (float)s->step));
  adam_kernel<<<blocks_for(s->P, 256), 256, 0, st>>>(s->param, s->grad, s->m1, s->m2, s->P, lr, b1, b2, 1e-8f, c1, c2,
                                                     s->L, s->wb, s->wtb);
  return cudaGetLastError() == cudaSuccess ? MX_OK : MX_ERR_CUDA;
}

// which: 0 the FP32 parameters, 1 their gradients of the last training step. Synchronises the device.
extern "C" int mx_sur_params(mx_surrogate* s, int32_t which, float* host, int64_t n) {
  if (!s || !host || n != s->P || which < 0 || which > 1) return MX_ERR_ARGUMENT;
  DeviceScope scope(s->device);
  return cudaMemcpy(host, which ? s->grad : s->param, sizeof(float) * s->P, cudaMemcpyDeviceToHost) == cudaSuccess
             ? MX_OK
             : MX_ERR_CUDA;
}

// The FP32 parameters from the host (their BF16 copies follow); Adam's moments and step count restart.
extern "C" int mx_sur_set_params(mx_surrogate* s, const float* host, int64_t n) {
  if (!s || !host || n != s->P) return MX_ERR_ARGUMENT;
  DeviceScope scope(s->device);
  cudaError_t e = cudaMemcpy(s->param, host, sizeof(float) * s->P, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(s->m1, 0, sizeof(float) * s->P);
  if (e == cudaSuccess) e = cudaMemset(s->m2, 0, sizeof(float) * s->P);
  if (e != cudaSuccess) return MX_ERR_CUDA;
  s->step = 0;
  weights_bf16_kernel<<<blocks_for(s->P, 256), 256>>>(s->param, s->P, s->L, s->wb, s->wtb);
  return cudaDeviceSynchronize() == cudaSuccess ? MX_OK : MX_ERR_CUDA;
}

// The GEMMs' error flag (1 after a wait gave up), read and cleared. Synchronises the device.
extern "C" int mx_sur_error(mx_surrogate* s, int32_t* flag) {
  if (!s || !flag) return MX_ERR_ARGUMENT;
  DeviceScope scope(s->device);
  int v = 0;
  cudaError_t e = cudaMemcpy(&v, s->err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemset(s->err, 0, sizeof(int));
  *flag = v;
  return e == cudaSuccess ? MX_OK : MX_ERR_CUDA;
}

extern "C" int mx_sur_call(mx_surrogate* s, mx_solver* solver, const double* x, const double* T, const double* P,
                           const double* dt, const double* h_in, const double* J, int64_t B, double rtol, double atol,
                           int32_t max_steps, double spread_max, double proj_max, int32_t audit_every, uint32_t seed,
                           double* x_out, double* h_out, int32_t* done, double* steps, int32_t* flag,
                           int32_t* status, int32_t* count, int64_t* total, uint64_t* stats, int32_t* audit_cells,
                           double* audit_x, float* audit_err, int32_t* audit_count, int32_t audit_cap, void* stream,
                           char* err, size_t errlen) {
  if (!s || !solver) {
    set_error(err, errlen, "mx_sur_call: a closed surrogate or solver");
    return MX_ERR_CLOSED;
  }
  if (solver->net.ns != s->ns || solver->net.nj != s->nj || solver->device != s->device) {
    set_error(err, errlen, "mx_sur_call: the surrogate (%d species, %d branches, device %d) does not match the solver "
              "(%d, %d, %d)", s->ns, s->nj, s->device, solver->net.ns, solver->net.nj, solver->device);
    return MX_ERR_ARGUMENT;
  }
  if (B < 0 || B > 0x7fffffff || !(rtol > 0.0 && rtol < 1e300 && atol > 0.0 && atol < 1e300) || max_steps < 1 ||
      (int64_t)MX_REC_STEPS * max_steps > 0x7fffffff || !(spread_max >= 0.0) || !(proj_max >= 0.0) ||
      audit_every < 0 || audit_cap < 0 || !count || !total || !stats || !audit_count ||
      (audit_cap > 0 && (!audit_cells || !audit_x || !audit_err)) ||
      (B > 0 && (!x || !T || !P || !dt || !h_in || !x_out || !h_out || !done || !steps || !flag || !status ||
                 (s->nj > 0 && !J)))) {
    set_error(err, errlen, "mx_sur_call: bad arguments");
    return MX_ERR_ARGUMENT;
  }
  DeviceScope scope(s->device);
  if (scope.status != cudaSuccess) {
    set_error(err, errlen, "mx_sur_call: device %d: %s", s->device, cudaGetErrorString(scope.status));
    return MX_ERR_CUDA;
  }
  cudaStream_t st = (cudaStream_t)stream;
  int rc = grow_list(solver, std::max<int64_t>(B, 1), err, errlen);
  if (rc) return rc;
  const bool mixed = solver->precision == MX_PRECISION_MIXED;
  cudaError_t e = grow_call(s, std::max<int64_t>(B, 1));
  if (e == cudaSuccess && mixed && (!solver->sel_count || solver->sel_capacity < B)) {
    if (!solver->sel_count) e = cudaMalloc(&solver->sel_count, 2 * sizeof(int));
    if (e == cudaSuccess && solver->sel_capacity < B) {
      if (solver->sel) cudaFree(solver->sel);
      solver->sel = nullptr;
      solver->sel_capacity = 0;
      e = cudaMalloc(&solver->sel, (size_t)std::max<int64_t>(B, 1) * sizeof(int));
      if (e == cudaSuccess) solver->sel_capacity = std::max<int64_t>(B, 1);
    }
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(count, 0, MX_COUNT_SLOTS * sizeof(int32_t), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->list_count, 0, 2 * sizeof(int), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(audit_count, 0, sizeof(int), st);
  if (e == cudaSuccess && mixed) e = cudaMemsetAsync(solver->sel_count, 0, 2 * sizeof(int), st);
  if (e != cudaSuccess) {
    set_error(err, errlen, "mx_sur_call: %s", cudaGetErrorString(e));
    return MX_ERR_CUDA;
  }
  if (B > 0) {
    rc = mx_sur_features(s, x, T, P, dt, h_in, J, B, s->cfeat, s->in_range, stream);
    if (!rc) rc = mx_sur_forward(s, s->cfeat, B, s->cpred, stream);
    if (rc) {
      set_error(err, errlen, "mx_sur_call: the network's forward pass failed (%d)", rc);
      return rc;
    }
    GateArgs g{x, T, dt, h_in, (int)B, s->ns, s->nel, s->nt, s->heads, s->kout, s->cpred, s->tmean, s->tstd,
               s->in_range, s->atoms, spread_max, proj_max, solver->net.drift, atol, s->etot, audit_every, seed,
               x_out, h_out, steps, done, flag, status, count, s->list, s->list_count, audit_cells, audit_x,
               audit_cap, audit_count, (unsigned long long*)stats, nullptr};
    const int warps = 4, gsmem = warps * (s->ns + MX_MAX_ELEMENTS * MX_MAX_ELEMENTS + 4 * MX_MAX_ELEMENTS + 4) * 8;
    gate_kernel<<<(int)((B + warps - 1) / warps), 32 * warps, gsmem, st>>>(g);
    // the Rodas3 fallback on the listed cells, then the recovery of what its guard listed
    mx::CallArgs a{x, T, P, dt, h_in, J, (int)B, rtol, atol, max_steps, x_out, h_out, done, steps, flag, status, count,
                   solver->list, solver->tries, s->list, s->list_count, solver->sel, solver->sel_count};
    const int grid = call_grid(solver, B);
    if (mixed) {
      e = mx_mixed_launch(solver, a, B, true, st);
      mx::CallArgs back = a;
      back.in_list = solver->sel;
      back.in_count = solver->sel_count;
      if (e == cudaSuccess) solver->call_list<<<grid, 32 * solver->warps, solver->smem, st>>>(solver->net, back, nullptr);
    } else {
      solver->call_list<<<grid, 32 * solver->warps, solver->smem, st>>>(solver->net, a, nullptr);
    }
    const int rgrid = (int)std::min<int64_t>(B, (int64_t)solver->recover_ctas * solver->sms);
    if (e == cudaSuccess)
      solver->recover<<<rgrid, 32 * solver->warps, solver->smem, st>>>(solver->net, a, MX_REC_STEPS * max_steps);
    if (e == cudaSuccess && audit_cap > 0)
      audit_kernel<<<(audit_cap + 3) / 4, 128, 0, st>>>(audit_cells, audit_count, audit_cap, audit_x, x_out, s->ns,
                                                        audit_err);
    if (e == cudaSuccess) e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    add_counts_kernel<<<1, 32, 0, st>>>(count, (long long*)total);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_error(err, errlen, "mx_sur_call: %s", cudaGetErrorString(e));
    return MX_ERR_CUDA;
  }
  return MX_OK;
}

extern "C" int mx_sur_propose(mx_surrogate* s, const double* x, const double* T, const double* P, const double* dt,
                              const double* h_in, const double* J, int64_t B, double drift, double atol,
                              double* x_prop, double* diag, void* stream) {
  if (!s || B < 0 || B > 0x7fffffff || !(drift >= 0.0) || !(atol > 0.0) ||
      (B > 0 && (!x || !T || !P || !dt || !h_in || !x_prop || !diag || (s->nj > 0 && !J))))
    return MX_ERR_ARGUMENT;
  if (B == 0) return MX_OK;
  DeviceScope scope(s->device);
  if (grow_call(s, B) != cudaSuccess) return MX_ERR_CUDA;
  int rc = mx_sur_features(s, x, T, P, dt, h_in, J, B, s->cfeat, s->in_range, stream);
  if (!rc) rc = mx_sur_forward(s, s->cfeat, B, s->cpred, stream);
  if (rc) return rc;
  GateArgs g{x, T, dt, h_in, (int)B, s->ns, s->nel, s->nt, s->heads, s->kout, s->cpred, s->tmean, s->tstd,
             s->in_range, s->atoms, 0.0, 0.0, drift, atol, s->etot, 0, 0u, x_prop, nullptr, nullptr, nullptr,
             nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0, nullptr, nullptr, diag};
  const int warps = 4, gsmem = warps * (s->ns + MX_MAX_ELEMENTS * MX_MAX_ELEMENTS + 4 * MX_MAX_ELEMENTS + 4) * 8;
  gate_kernel<<<(int)((B + warps - 1) / warps), 32 * warps, gsmem, (cudaStream_t)stream>>>(g);
  return cudaGetLastError() == cudaSuccess ? MX_OK : MX_ERR_CUDA;
}

extern "C" int mx_sur_destroy(mx_surrogate* s) {
  if (!s) return MX_OK;
  {
    DeviceScope scope(s->device);
    cudaDeviceSynchronize();
    free_all(s->work);
    free_all(s->call_work);
    free_all(s->persist);
  }
  delete s;
  return MX_OK;
}
