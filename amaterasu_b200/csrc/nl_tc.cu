// Nonlocal (Kleinman-Bylander) products of the complex64 engine on the tensor cores.
//
// Both complex products are rewritten as real GEMMs over the interleaved (re, im) storage,
// so psi and H.psi are used in place, and the per-k projector matrices are expanded once:
//
//   project   P = psi B^H          D1[j][m] = sum_k' Bx[j][k'] psi_r[m][k']     (k' = 2G + re/im)
//             Bx = [B as stored; B "swapped" (-Bi, Br)]  -> rows j < nproj give Re P, the
//             rest Im P. Long reduction (2 npw): split over K, partial sums reduced after.
//   apply     hpsi += P (D B)       D2[g'][m] = sum_j DxT[g'][j] Q_r[m][j]   (g' = 2G + re/im)
//             Q_r = P stored interleaved, DxT the real expansion of D.B; written straight
//             into the interleaved hpsi rows (accumulating onto the FFT result).
//
// The operands carry a split-TF32 (hi, lo) pair; the tensor-core kernel (tc_chain.cuh) adds
// hi.hi + hi.lo + lo.hi with its FP32 accumulator drained into registers every 2 k-blocks;
// the projection's reduction splits are summed in FP64. Layouts in HBM (FP32, zero padded):
//   Bx  [nk][p2][kp]   DxT [nk][mp][k2]   psi [k_count][nbp][kp]   Q [k_count][nbp][k2]
#include "common.cuh"
#include "engine_impl.cuh"
#include "tc_chain.cuh"

#include <cudaTypedefs.h>

#include <algorithm>

using namespace ama;
using namespace ama::tc;

namespace {

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

// --------------------------------------------------------------- set-up kernels
__global__ void build_bx_kernel(const float2* __restrict__ proj, const int64_t* __restrict__ pw_off,
                                const int* __restrict__ npw, int nproj, int p2, int kp, float* hi, float* lo) {
  const int k = blockIdx.z;
  const int row = blockIdx.y;
  const int np = npw[k];
  const float2* src = proj + pw_off[k] * nproj;
  float* h = hi + ((int64_t)k * p2 + row) * kp;
  float* l = lo + ((int64_t)k * p2 + row) * kp;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < kp; c += gridDim.x * blockDim.x) {
    float v = 0.f;
    const int g = c >> 1, ri = c & 1;
    if (g < np && row < 2 * nproj) {
      const int j = row % nproj;
      const float2 b = src[(int64_t)j * np + g];
      if (row < nproj) v = ri ? b.y : b.x;          // Re P row: (Br, Bi)
      else v = ri ? b.x : -b.y;                     // Im P row: (-Bi, Br)
    }
    float a, r;
    tf32_split(v, a, r);
    h[c] = a;
    l[c] = r;
  }
}

__global__ void build_dxt_kernel(const float2* __restrict__ dproj, const int64_t* __restrict__ pw_off,
                                 const int* __restrict__ npw, int nproj, int mp, int k2, float* hi, float* lo) {
  const int k = blockIdx.z;
  const int np = npw[k];
  const float2* src = dproj + pw_off[k] * nproj;
  const int64_t total = (int64_t)mp * k2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int gp = (int)(e / k2), j = (int)(e % k2);
    float v = 0.f;
    const int g = gp >> 1, gi = gp & 1, p = j >> 1, d = j & 1;
    if (g < np && p < nproj) {
      const float2 b = src[(int64_t)p * np + g];
      // re row: (DBr, -DBi); im row: (DBi, DBr)
      v = gi == 0 ? (d == 0 ? b.x : -b.y) : (d == 0 ? b.y : b.x);
    }
    float a, r;
    tf32_split(v, a, r);
    hi[(int64_t)k * total + e] = a;
    lo[(int64_t)k * total + e] = r;
  }
}

// ------------------------------------------------------------------ per-call
// psi (interleaved, back to back per k) -> padded split copies [k][nbp][kp].
__global__ void split_psi_kernel(const float* __restrict__ psi, const int64_t* __restrict__ pw_off,
                                 const int* __restrict__ npw, int k_first, int nbands, int nbp, int kp,
                                 float* hi, float* lo) {
  const int kl = blockIdx.z, m = blockIdx.y;
  const int k = k_first + kl;
  const int np2 = 2 * npw[k];
  const float* src = psi + 2 * ((pw_off[k] - pw_off[k_first]) * nbands + (int64_t)m * npw[k]);
  float* h = hi + ((int64_t)kl * nbp + m) * kp;
  float* l = lo + ((int64_t)kl * nbp + m) * kp;
  // four consecutive values per thread (kp is a multiple of 32, rows are 16-byte aligned)
  for (int c = 4 * (blockIdx.x * blockDim.x + threadIdx.x); c < kp; c += 4 * gridDim.x * blockDim.x) {
    float v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = (m < nbands && c + u < np2) ? src[c + u] : 0.f;
    float4 a, r;
    tf32_split(v[0], a.x, r.x);
    tf32_split(v[1], a.y, r.y);
    tf32_split(v[2], a.z, r.z);
    tf32_split(v[3], a.w, r.w);
    *reinterpret_cast<float4*>(h + c) = a;
    *reinterpret_cast<float4*>(l + c) = r;
  }
}

// partial [kl][split][nbp][p2] -> Q split copies [kl][nbp][k2]; Q[m][2p+d] = D1[d*nproj+p][m]
// (splits summed in FP64).
__global__ void reduce_q_kernel(const float* __restrict__ part, int splits, int nbp, int p2, int k2, int nproj,
                                float* hi, float* lo) {
  const int kl = blockIdx.z;
  const int m = blockIdx.y;
  for (int j = threadIdx.x; j < k2; j += blockDim.x) {
    double acc = 0.0;
    if (j < 2 * nproj) {
      const int p = j >> 1, d = j & 1;
      const int row = d * nproj + p;
      for (int s = 0; s < splits; ++s) acc += part[(((int64_t)kl * splits + s) * nbp + m) * p2 + row];
    }
    const float v = (float)acc;
    float a, r;
    tf32_split(v, a, r);
    hi[((int64_t)kl * nbp + m) * k2 + j] = a;
    lo[((int64_t)kl * nbp + m) * k2 + j] = r;
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

int grow(float** p, size_t* have, size_t need) {
  if (*have >= need) return AMA_OK;
  ama::bump_memory_epoch();
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  AMA_CUDA_TRY(cudaMalloc((void**)p, need));
  *have = need;
  return AMA_OK;
}

}  // namespace

namespace ama {

int nl_tc_setup(AmaEngine* e) {
  NlTcState& t = e->tc;
  if (t.ready || e->nproj <= 0 || !(e->precisions & (1u << AMA_C64))) return AMA_OK;
  t.kp = round_up(2 * e->max_npw, kBK);
  t.p2 = round_up(2 * e->nproj, kBM);
  t.k2 = round_up(2 * e->nproj, kBK);
  t.mp = round_up(2 * e->max_npw, kBM);
  const size_t bx = (size_t)e->nk * t.p2 * t.kp * sizeof(float);
  const size_t dx = (size_t)e->nk * t.mp * t.k2 * sizeof(float);
  ama::bump_memory_epoch();
  for (int h = 0; h < 2; ++h) {
    AMA_CUDA_TRY(cudaMalloc((void**)&t.bx[h], bx));
    AMA_CUDA_TRY(cudaMalloc((void**)&t.dxt[h], dx));
  }
  AMA_CUDA_TRY(cudaMalloc((void**)&t.err, sizeof(int)));
  AMA_CUDA_TRY(cudaMemset(t.err, 0, sizeof(int)));
  dim3 g1((t.kp + 255) / 256, t.p2, e->nk);
  build_bx_kernel<<<g1, 256>>>((const float2*)e->d.proj[AMA_C64], e->d.pw_off, e->d.npw, e->nproj, t.p2, t.kp,
                               t.bx[0], t.bx[1]);
  AMA_CHECK_LAUNCH();
  dim3 g2(256, 1, e->nk);
  build_dxt_kernel<<<g2, 256>>>((const float2*)e->d.dproj[AMA_C64], e->d.pw_off, e->d.npw, e->nproj, t.mp, t.k2,
                                t.dxt[0], t.dxt[1]);
  AMA_CHECK_LAUNCH();
  AMA_CUDA_TRY(cudaDeviceSynchronize());
  for (int h = 0; h < 2; ++h) {
    int rc = make_map(&t.map_bx[h], t.bx[h], t.kp, t.p2, e->nk, kBM);
    if (!rc) rc = make_map(&t.map_dxt[h], t.dxt[h], t.k2, t.mp, e->nk, kBM);
    if (rc) return rc;
  }
  AMA_CUDA_TRY(cudaFuncSetAttribute(tc_chain_kernel<kChainPartial>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    kChainSmemCap));
  AMA_CUDA_TRY(cudaFuncSetAttribute(tc_chain_kernel<kChainAddRows>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    kChainSmemCap));
  t.ready = true;
  return AMA_OK;
}

int nl_tc_run(AmaEngine* e, int k_first, int k_count, int nbands, const float2* psi, float2* hpsi,
              cudaStream_t s, int phase) {
  NlTcState& t = e->tc;
  const int ntile = (nbands + 255) / 256;
  const int bn = round_up((nbands + ntile - 1) / ntile, 16);
  const int nbp = bn * ntile;
  if (phase == 1) return nl_tc_apply(e, k_first, k_count, nbands, hpsi, s, ntile, bn);
  // hi and lo halves live in one allocation each; maps are rebuilt whenever a buffer moves
  const size_t psi_half = (size_t)k_count * nbp * t.kp;
  const size_t q_half = (size_t)k_count * nbp * t.k2;
  float* old_psi = t.psi[0];
  float* old_q = t.q[0];
  int rc = grow(&t.psi[0], &t.psi_bytes, 2 * psi_half * sizeof(float));
  if (rc) return rc;
  rc = grow(&t.q[0], &t.q_bytes, 2 * q_half * sizeof(float));
  if (rc) return rc;
  t.psi[1] = t.psi[0] + psi_half;
  t.q[1] = t.q[0] + q_half;
  const int kblocks = t.kp / kBK;
  const int mtiles1 = t.p2 / kBM;
  // enough splits to fill the GPU twice, and at most 96 drained chains summed in FP32
  // registers per CTA
  constexpr int kMaxChainsPerCta = 96;
  const int chains = (kblocks + kChain - 1) / kChain;
  int splits = std::max(1, (2 * 148 + mtiles1 * ntile * k_count - 1) / (mtiles1 * ntile * k_count));
  splits = std::max(splits, (chains + kMaxChainsPerCta - 1) / kMaxChainsPerCta);
  splits = std::min(splits, kblocks);
  rc = grow(&t.part, &t.part_bytes, (size_t)k_count * splits * nbp * t.p2 * sizeof(float));
  if (rc) return rc;
  if (t.cached_kcount != k_count || t.cached_nbp != nbp || old_psi != t.psi[0] || old_q != t.q[0]) {
    for (int h = 0; h < 2; ++h) {
      rc = make_map(&t.map_psi[h], t.psi[h], t.kp, nbp, k_count, bn);
      if (!rc) rc = make_map(&t.map_q[h], t.q[h], t.k2, nbp, k_count, bn);
      if (rc) return rc;
    }
    t.cached_kcount = k_count;
    t.cached_nbp = nbp;
  }

  dim3 gs((t.kp / 4 + 255) / 256, nbp, k_count);
  split_psi_kernel<<<gs, 256, 0, s>>>((const float*)psi, e->d.pw_off, e->d.npw, k_first, nbands, nbp, t.kp,
                                      t.psi[0], t.psi[1]);
  AMA_CHECK_LAUNCH();

  ChainArgs a{};
  a.kblocks = kblocks;
  a.splits = splits;
  a.bn = bn;
  a.stages = chain_stages(bn);
  a.a_z0 = k_first;
  a.part = t.part;
  a.nrows = t.p2;
  a.ncols = nbp;
  a.err = t.err;
  dim3 g1(ntile, mtiles1, k_count * splits);
  tc_chain_kernel<kChainPartial><<<g1, kChainThreads, chain_smem(bn, a.stages), s>>>(t.map_bx[0], t.map_bx[1],
                                                                                     t.map_psi[0], t.map_psi[1], a);
  AMA_CHECK_LAUNCH();

  dim3 gr(1, nbp, k_count);
  reduce_q_kernel<<<gr, 256, 0, s>>>(t.part, splits, nbp, t.p2, t.k2, e->nproj, t.q[0], t.q[1]);
  AMA_CHECK_LAUNCH();
  if (phase == 0) return AMA_OK;
  return nl_tc_apply(e, k_first, k_count, nbands, hpsi, s, ntile, bn);
}

// hpsi += P (D B) from the split Q of the projection phase
int nl_tc_apply(AmaEngine* e, int k_first, int k_count, int nbands, float2* hpsi, cudaStream_t s, int ntile,
                int bn) {
  NlTcState& t = e->tc;
  ChainArgs b{};
  b.kblocks = t.k2 / kBK;
  b.splits = 1;
  b.bn = bn;
  b.stages = chain_stages(bn);
  b.a_z0 = k_first;
  b.out = (float*)hpsi;
  b.pw_off = e->d.pw_off;
  b.npw = e->d.npw;
  b.k_first = k_first;
  b.nbands = nbands;
  b.n_valid = nbands;
  b.err = t.err;
  dim3 g2(ntile, t.mp / kBM, k_count);
  tc_chain_kernel<kChainAddRows><<<g2, kChainThreads, chain_smem(bn, b.stages), s>>>(t.map_dxt[0], t.map_dxt[1],
                                                                                     t.map_q[0], t.map_q[1], b);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

void nl_tc_free(AmaEngine* e) {
  NlTcState& t = e->tc;
  ama::bump_memory_epoch();
  auto f = [](void* p) { if (p) cudaFree(p); };
  for (int h = 0; h < 2; ++h) { f(t.bx[h]); f(t.dxt[h]); }
  f(t.psi[0]);
  f(t.q[0]);
  f(t.part);
  f(t.err);
  t = NlTcState();
}

}  // namespace ama

extern "C" int ama_tc_status(AmaEngine* e, int32_t* code) {
  AMA_REQUIRE(e && code, AMA_ERR_ARG, "null argument");
  *code = 0;
  if (e->tc.err) AMA_CUDA_TRY(cudaMemcpy(code, e->tc.err, sizeof(int), cudaMemcpyDeviceToHost));
  return AMA_OK;
}
