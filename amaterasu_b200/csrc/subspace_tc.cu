// Davidson subspace products of the complex64 engine on the tensor cores (tcgen05,
// split-TF32), for the per-k packed operands of ama_kbatch_zgemm:
//
//   form NC  C (m x n, small) = alpha * A (m x npw) . B (n x npw)^H + beta * C
//            Gram, Rayleigh-Ritz and projection matrices: the reduction runs over the
//            plane waves. Real form over interleaved (re, im) storage:
//              Re C = A' . B'      A' = A as stored           (2 npw reals per row)
//              Im C = As . B'      As = (Ai, -Ar) per pair    ("swapped" A)
//            The GEMM's M rows are [A' rows ; As rows], so one CTA row tile holds either
//            real or imaginary parts; FP32 partial tiles are reduced in FP64 afterwards.
//   form NN  C (m x npw, long) = alpha * A (m x k, small) . B (k x npw) + beta * C
//            rotations and projections of basis blocks. Real form with the plane-wave
//            index as GEMM rows: D[g][2r+p] = sum_{i,c} BT[g][2i+c] R[2r+p][2i+c]
//              BT[g][2i+c] = B[i][g] (re, im)  (the transposed basis)
//              R[2r][.]  = (Ar, -Ai)  -> Re C[r][g];   R[2r+1][.] = (Ai, Ar) -> Im C[r][g]
//            so each thread of the epilogue holds whole complex outputs and writes them
//            coalesced along g.
//
// Operands are staged once per call into padded FP32 arrays split into a TF32-exact "hi"
// and a TF32 "lo" remainder; the GEMM (tc_chain.cuh) adds hi.hi + hi.lo + lo.hi with its
// accumulator drained into registers every 2 k-blocks; long reductions are additionally
// split across CTAs and the splits summed in FP64. Timeouts of the kernel's bounded waits
// are reported by ama_subspace_tc_status.
#include "common.cuh"
#include "tc_chain.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <string>

using namespace ama;
using namespace ama::tc;

namespace {

constexpr int kMaxChainsPerCta = 96;

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

using KOpDev = ChainOp;

KOpDev to_dev(const AmaKOperand* o) {
  return KOpDev{(const float*)o->base, o->rows_per_k, o->row0, o->ld, o->kstride, o->ragged};
}

__device__ __forceinline__ const float* op_rows(const KOpDev& o, int z, int np, int64_t po, int64_t& ld) {
  return chain_rows(o, z, np, po, ld);
}

// ------------------------------------------------------------------ staging kernels
// NC, A operand: rows [0, mpad) = A', rows [mpad, 2 mpad) = As; zero outside (m, 2 npw_k).
__global__ void stage_nc_a_kernel(KOpDev a, const int* __restrict__ npw, const int64_t* __restrict__ pw_off, int m,
                                  int mpad, int kp, float* __restrict__ hi, float* __restrict__ lo) {
  const int z = blockIdx.z, r = blockIdx.y;
  const int np = npw[z];
  const bool sw = r >= mpad;
  const int i = sw ? r - mpad : r;
  int64_t ld;
  const float* rows = op_rows(a, z, np, pw_off[z], ld);
  const float* src = rows + 2 * (int64_t)i * ld;
  float* h = hi + ((int64_t)z * 2 * mpad + r) * kp;
  float* l = lo + ((int64_t)z * 2 * mpad + r) * kp;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < kp; c += gridDim.x * blockDim.x) {
    float v = 0.f;
    if (i < m && c < 2 * np) {
      if (!sw) v = src[c];
      else v = (c & 1) ? -src[c - 1] : src[c + 1];
    }
    float x, y;
    tf32_split(v, x, y);
    h[c] = x;
    l[c] = y;
  }
}

// NC, B operand: rows [0, npad) = B'; zero outside (n, 2 npw_k).
__global__ void stage_nc_b_kernel(KOpDev b, const int* __restrict__ npw, const int64_t* __restrict__ pw_off, int n,
                                  int npad, int kp, float* __restrict__ hi, float* __restrict__ lo) {
  const int z = blockIdx.z, r = blockIdx.y;
  const int np = npw[z];
  int64_t ld;
  const float* rows = op_rows(b, z, np, pw_off[z], ld);
  const float* src = rows + 2 * (int64_t)r * ld;
  float* h = hi + ((int64_t)z * npad + r) * kp;
  float* l = lo + ((int64_t)z * npad + r) * kp;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < kp; c += gridDim.x * blockDim.x) {
    const float v = (r < n && c < 2 * np) ? src[c] : 0.f;
    float x, y;
    tf32_split(v, x, y);
    h[c] = x;
    l[c] = y;
  }
}

// NN, basis operand transposed: BT[z][g][2i + c] = B[i][g].c for g < npw_k, i < kdim; zero
// elsewhere in [gpad][kp]. 32 x 32 complex tiles through shared memory.
__global__ void stage_nn_bt_kernel(KOpDev b, const int* __restrict__ npw, const int64_t* __restrict__ pw_off,
                                   int kdim, int gpad, int kp, float* __restrict__ hi, float* __restrict__ lo) {
  __shared__ float2 tile[32][33];
  const int z = blockIdx.z;
  const int np = npw[z];
  const int g0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
  int64_t ld;
  const float2* src = reinterpret_cast<const float2*>(op_rows(b, z, np, pw_off[z], ld));
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int i = i0 + j, g = g0 + threadIdx.x;
    tile[j][threadIdx.x] = (i < kdim && g < np) ? src[(int64_t)i * ld + g] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int g = g0 + j, i = i0 + threadIdx.x;
    if (g >= gpad || 2 * i >= kp) continue;
    const float2 v = tile[threadIdx.x][j];
    float2 h, l;
    tf32_split(v.x, h.x, l.x);
    tf32_split(v.y, h.y, l.y);
    const int64_t off = ((int64_t)z * gpad + g) * kp + 2 * i;
    *reinterpret_cast<float2*>(hi + off) = h;
    *reinterpret_cast<float2*>(lo + off) = l;
  }
}

// NN, small operand expanded: R[z][2r + p][2i + c] from A[r][i] (see the header).
__global__ void stage_nn_r_kernel(KOpDev a, const int* __restrict__ npw, const int64_t* __restrict__ pw_off, int m,
                                  int kdim, int rpad, int kp, float* __restrict__ hi, float* __restrict__ lo) {
  const int z = blockIdx.z, row = blockIdx.y;
  const int r = row >> 1, p = row & 1;
  int64_t ld;
  const float2* rows = reinterpret_cast<const float2*>(op_rows(a, z, npw[z], pw_off[z], ld));
  const float2* src = rows + (int64_t)r * ld;
  float* h = hi + ((int64_t)z * rpad + row) * kp;
  float* l = lo + ((int64_t)z * rpad + row) * kp;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < kp; c += gridDim.x * blockDim.x) {
    const int i = c >> 1, ci = c & 1;
    float v = 0.f;
    if (r < m && i < kdim) {
      const float2 x = src[i];
      v = p == 0 ? (ci == 0 ? x.x : -x.y) : (ci == 0 ? x.y : x.x);
    }
    float s, t;
    tf32_split(v, s, t);
    h[c] = s;
    l[c] = t;
  }
}

// NC: C[z][i][j] = alpha (sum_s part[z,s][j][i] + i sum_s part[z,s][j][mpad + i]) + beta C, FP64 sums.
__global__ void finalize_nc_kernel(const float* __restrict__ part, int splits, int nrows, int ncols, int mpad, int m,
                                   int n, KOpDev c, const int* __restrict__ npw, const int64_t* __restrict__ pw_off,
                                   double2 alpha, double2 beta) {
  const int z = blockIdx.y;
  int64_t ld;
  float2* out = const_cast<float2*>(reinterpret_cast<const float2*>(op_rows(c, z, npw[z], pw_off[z], ld)));
  const bool use_beta = beta.x != 0.0 || beta.y != 0.0;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m * n; e += gridDim.x * blockDim.x) {
    const int i = e % m, j = e / m;
    double re = 0.0, im = 0.0;
    for (int s = 0; s < splits; ++s) {
      const float* ps = part + ((int64_t)z * splits + s) * ncols * nrows + (int64_t)j * nrows;
      re += ps[i];
      im += ps[mpad + i];
    }
    double ore = alpha.x * re - alpha.y * im, oim = alpha.x * im + alpha.y * re;
    float2* d = out + (int64_t)i * ld + j;
    if (use_beta) {
      const float2 old = *d;
      ore += beta.x * old.x - beta.y * old.y;
      oim += beta.x * old.y + beta.y * old.x;
    }
    *d = make_float2((float)ore, (float)oim);
  }
}

// ------------------------------------------------------------------ host
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* ptr = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  }
  return fn;
}

// 3D FP32 map over [z][y][x] (x contiguous), box {32, box_y, 1}, 128-byte swizzle.
int make_map(CUtensorMap* map, const float* base, int x, int y, int z, int box_y) {
  auto fn = encode_fn();
  AMA_REQUIRE(fn, AMA_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  cuuint64_t dims[3] = {(cuuint64_t)x, (cuuint64_t)y, (cuuint64_t)z};
  cuuint64_t strides[2] = {(cuuint64_t)x * 4, (cuuint64_t)x * y * 4};
  cuuint32_t box[3] = {(cuuint32_t)kBK, (cuuint32_t)box_y, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  AMA_REQUIRE(r == CUDA_SUCCESS, AMA_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return AMA_OK;
}

struct Buf {
  float* p = nullptr;
  size_t bytes = 0;
  int grow(size_t need) {
    if (bytes >= need) return AMA_OK;
    bump_memory_epoch();
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    AMA_CUDA_TRY(cudaMalloc((void**)&p, need));
    bytes = need;
    return AMA_OK;
  }
};

struct TcScratch {
  Buf a, b, part;
  int* err = nullptr;
};
thread_local PerDevice<TcScratch> g_tc_dev;  // per host thread and device
PerDevice<std::atomic<int>> g_tc_attrs;       // kernel attributes set on this device

int tile_n(int cols) { return cols >= kChainBN ? kChainBN : std::max(16, round_up(cols, 16)); }

int ensure_err() {
  TcScratch* gt = g_tc_dev.here();
  AMA_REQUIRE(gt, AMA_ERR_CUDA, "tensor-core subspace GEMM: no usable current CUDA device");
  TcScratch& g_tc = *gt;
  if (!g_tc.err) {
    bump_memory_epoch();
    AMA_CUDA_TRY(cudaMalloc((void**)&g_tc.err, sizeof(int)));
    AMA_CUDA_TRY(cudaMemset(g_tc.err, 0, sizeof(int)));
  }
  std::atomic<int>& attrs = *g_tc_attrs.here();
  if (!attrs.load()) {
    AMA_CUDA_TRY(cudaFuncSetAttribute(tc_chain_kernel<kChainPartial>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      kChainSmemCap));
    AMA_CUDA_TRY(cudaFuncSetAttribute(tc_chain_kernel<kChainComplexNN>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, kChainSmemCap));
    attrs.store(1);
  }
  return AMA_OK;
}

int run_nc(int nk, int m, int n, const int32_t* npw, const int64_t* pw_off, const AmaKOperand* a,
           const AmaKOperand* b, const AmaKOperand* c, const double* alpha, const double* beta, int max_npw,
           cudaStream_t s) {
  if (int rc = ensure_err()) return rc;
  TcScratch& g_tc = *g_tc_dev.here();
  const int mpad = round_up(m, 64);
  const int rows_a = 2 * mpad;
  const int bn = tile_n(n);
  const int npad = round_up(n, bn);
  const int kp = round_up(2 * max_npw, kBK);
  const int kblocks = kp / kBK;
  const int tiles = (rows_a / kBM) * (npad / bn) * nk;
  const int chains = (kblocks + kChain - 1) / kChain;
  int splits = std::max((chains + kMaxChainsPerCta - 1) / kMaxChainsPerCta, (2 * 148 + tiles - 1) / tiles);
  splits = std::max(1, std::min(splits, kblocks));
  const size_t a_half = (size_t)nk * rows_a * kp, b_half = (size_t)nk * npad * kp;
  int rc = g_tc.a.grow(2 * a_half * sizeof(float));
  if (!rc) rc = g_tc.b.grow(2 * b_half * sizeof(float));
  if (!rc) rc = g_tc.part.grow((size_t)nk * splits * npad * rows_a * sizeof(float));
  if (!rc) rc = ensure_err();
  if (rc) return rc;
  float *ahi = g_tc.a.p, *alo = g_tc.a.p + a_half, *bhi = g_tc.b.p, *blo = g_tc.b.p + b_half;
  const KOpDev ad = to_dev(a), bd = to_dev(b), cd = to_dev(c);
  stage_nc_a_kernel<<<dim3((kp + 255) / 256, rows_a, nk), 256, 0, s>>>(ad, npw, pw_off, m, mpad, kp, ahi, alo);
  AMA_CHECK_LAUNCH();
  stage_nc_b_kernel<<<dim3((kp + 255) / 256, npad, nk), 256, 0, s>>>(bd, npw, pw_off, n, npad, kp, bhi, blo);
  AMA_CHECK_LAUNCH();
  CUtensorMap mah, mal, mbh, mbl;
  rc = make_map(&mah, ahi, kp, rows_a, nk, kBM);
  if (!rc) rc = make_map(&mal, alo, kp, rows_a, nk, kBM);
  if (!rc) rc = make_map(&mbh, bhi, kp, npad, nk, bn);
  if (!rc) rc = make_map(&mbl, blo, kp, npad, nk, bn);
  if (rc) return rc;
  ChainArgs args{};
  args.kblocks = kblocks;
  args.splits = splits;
  args.bn = bn;
  args.stages = chain_stages(bn);
  args.part = g_tc.part.p;
  args.nrows = rows_a;
  args.ncols = npad;
  args.err = g_tc.err;
  tc_chain_kernel<kChainPartial><<<dim3(npad / bn, rows_a / kBM, nk * splits), kChainThreads,
                                   chain_smem(bn, args.stages), s>>>(mah, mal, mbh, mbl, args);
  AMA_CHECK_LAUNCH();
  const int fin_blocks = std::max(1, std::min(1024, (m * n + 255) / 256));
  finalize_nc_kernel<<<dim3(fin_blocks, nk), 256, 0, s>>>(g_tc.part.p, splits, rows_a, npad, mpad, m, n, cd, npw,
                                                          pw_off, make_double2(alpha[0], alpha[1]),
                                                          make_double2(beta[0], beta[1]));
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

int run_nn(int nk, int m, int kdim, const int32_t* npw, const int64_t* pw_off, const AmaKOperand* a,
           const AmaKOperand* b, const AmaKOperand* c, const double* alpha, const double* beta, int max_npw,
           cudaStream_t s) {
  if (int rc = ensure_err()) return rc;
  TcScratch& g_tc = *g_tc_dev.here();
  const int gpad = round_up(max_npw, kBM);
  const int kp = round_up(2 * kdim, kBK);
  const int bn = tile_n(2 * m);
  const int rpad = round_up(2 * m, bn);
  const size_t a_half = (size_t)nk * gpad * kp, b_half = (size_t)nk * rpad * kp;
  int rc = g_tc.a.grow(2 * a_half * sizeof(float));
  if (!rc) rc = g_tc.b.grow(2 * b_half * sizeof(float));
  if (!rc) rc = ensure_err();
  if (rc) return rc;
  float *ahi = g_tc.a.p, *alo = g_tc.a.p + a_half, *bhi = g_tc.b.p, *blo = g_tc.b.p + b_half;
  const KOpDev ad = to_dev(a), bd = to_dev(b), cd = to_dev(c);
  stage_nn_bt_kernel<<<dim3(gpad / 32, kp / 64 + 1, nk), dim3(32, 8), 0, s>>>(bd, npw, pw_off, kdim, gpad, kp, ahi,
                                                                              alo);
  AMA_CHECK_LAUNCH();
  stage_nn_r_kernel<<<dim3((kp + 255) / 256, rpad, nk), 256, 0, s>>>(ad, npw, pw_off, m, kdim, rpad, kp, bhi, blo);
  AMA_CHECK_LAUNCH();
  CUtensorMap mah, mal, mbh, mbl;
  rc = make_map(&mah, ahi, kp, gpad, nk, kBM);
  if (!rc) rc = make_map(&mal, alo, kp, gpad, nk, kBM);
  if (!rc) rc = make_map(&mbh, bhi, kp, rpad, nk, bn);
  if (!rc) rc = make_map(&mbl, blo, kp, rpad, nk, bn);
  if (rc) return rc;
  ChainArgs args{};
  args.kblocks = kp / kBK;
  args.splits = 1;
  args.bn = bn;
  args.stages = chain_stages(bn);
  args.c = cd;
  args.npw = npw;
  args.pw_off = pw_off;
  args.m = m;
  args.alpha = make_float2((float)alpha[0], (float)alpha[1]);
  args.beta = make_float2((float)beta[0], (float)beta[1]);
  args.err = g_tc.err;
  tc_chain_kernel<kChainComplexNN><<<dim3(rpad / bn, gpad / kBM, nk), kChainThreads, chain_smem(bn, args.stages),
                                     s>>>(mah, mal, mbh, mbl, args);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

}  // namespace

extern "C" int ama_kbatch_zgemm_tc(int32_t form, int32_t nk, int32_t m, int32_t n, int32_t k, const int32_t* npw,
                                   const int64_t* pw_off, const AmaKOperand* a, const AmaKOperand* b,
                                   const AmaKOperand* c, const double* alpha, const double* beta, int32_t max_npw,
                                   void* stream) {
  AMA_REQUIRE(a && b && c && npw && pw_off && alpha && beta, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(nk >= 1 && max_npw >= 1, AMA_ERR_SHAPE, "bad sizes");
  cudaStream_t s = (cudaStream_t)stream;
  if (form == 1) {
    AMA_REQUIRE(k == -1 && m >= 1 && n >= 1, AMA_ERR_SHAPE,
                "tensor-core NC form: the reduction must run over the plane waves (k = -1)");
    AMA_REQUIRE(a->ragged && b->ragged && !c->ragged, AMA_ERR_SHAPE,
                "tensor-core NC form: A and B must be per-k blocks and C a small matrix");
    return run_nc(nk, m, n, npw, pw_off, a, b, c, alpha, beta, max_npw, s);
  }
  if (form == 0) {
    AMA_REQUIRE(n == -1 && m >= 1 && k >= 1, AMA_ERR_SHAPE,
                "tensor-core NN form: the output columns must be the plane waves (n = -1)");
    AMA_REQUIRE(!a->ragged && b->ragged && c->ragged, AMA_ERR_SHAPE,
                "tensor-core NN form: A must be a small matrix and B, C per-k blocks");
    return run_nn(nk, m, k, npw, pw_off, a, b, c, alpha, beta, max_npw, s);
  }
  ama::set_error("tensor-core subspace GEMM: forms 0 (NN) and 1 (NC) only");
  return AMA_ERR_UNSUPPORTED;
}

extern "C" int ama_subspace_tc_status(int32_t* code) {
  AMA_REQUIRE(code, AMA_ERR_ARG, "null argument");
  *code = 0;
  TcScratch* gt = g_tc_dev.here();
  if (gt && gt->err) AMA_CUDA_TRY(cudaMemcpy(code, gt->err, sizeof(int), cudaMemcpyDeviceToHost));
  return AMA_OK;
}
