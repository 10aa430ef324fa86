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
// The operands carry a split-TF32 (hi, lo) pair; the tensor-core kernel adds
// hi.hi + hi.lo + lo.hi in FP32 (tc_gemm.cuh). Layouts in HBM (FP32, zero padded):
//   Bx  [nk][p2][kp]   DxT [nk][mp][k2]   psi [k_count][nbp][kp]   Q [k_count][nbp][k2]
#include "common.cuh"
#include "engine_impl.cuh"
#include "tc_gemm.cuh"

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
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < kp; c += gridDim.x * blockDim.x) {
    const float v = (m < nbands && c < np2) ? src[c] : 0.f;
    float a, r;
    tf32_split(v, a, r);
    h[c] = a;
    l[c] = r;
  }
}

// partial [kl][split][nbp][p2] -> Q split copies [kl][nbp][k2]; Q[m][2p+d] = D1[d*nproj+p][m].
__global__ void reduce_q_kernel(const float* __restrict__ part, int splits, int nbp, int p2, int k2, int nproj,
                                float* hi, float* lo) {
  const int kl = blockIdx.z;
  const int m = blockIdx.y;
  for (int j = threadIdx.x; j < k2; j += blockDim.x) {
    float v = 0.f;
    if (j < 2 * nproj) {
      const int p = j >> 1, d = j & 1;
      const int row = d * nproj + p;
      for (int s = 0; s < splits; ++s) v += part[(((int64_t)kl * splits + s) * nbp + m) * p2 + row];
    }
    float a, r;
    tf32_split(v, a, r);
    hi[((int64_t)kl * nbp + m) * k2 + j] = a;
    lo[((int64_t)kl * nbp + m) * k2 + j] = r;
  }
}

// ------------------------------------------------------------------ GEMM
struct TcArgs {
  int kblocks;     // K / 32 of the whole reduction
  int splits;      // K splits (project) or 1 (apply)
  int bn;          // N tile (multiple of 16, <= 256)
  int n_valid;     // valid N (bands)
  int stages;
  int k_first;     // engine k of z = 0 (for the A operand maps that span all k)
  // mode 0: partial[kl][split][nbp][p2] (column-major tile store)
  float* part;
  int nbp, p2;
  // mode 1: hpsi interleaved accumulate
  float* out;
  const int64_t* pw_off;
  const int* npw;
  int nbands;
  int* err;
};

template <int MODE>
__global__ void __launch_bounds__(kThreads, 1)
tc_gemm_kernel(const __grid_constant__ CUtensorMap a_hi, const __grid_constant__ CUtensorMap a_lo,
               const __grid_constant__ CUtensorMap b_hi, const __grid_constant__ CUtensorMap b_lo, TcArgs p) {
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  __shared__ __align__(8) uint64_t full_bar[kMaxStages], empty_bar[kMaxStages], done_bar;
  __shared__ uint32_t tmem_slot;

  // 1024-byte aligned operand ring
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_dyn) + 1023) & ~static_cast<uintptr_t>(1023));
  const int a_bytes = kBM * kBK * 4;
  const int b_bytes = p.bn * kBK * 4;
  const int stage_bytes = 2 * a_bytes + 2 * b_bytes;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mt = blockIdx.x, nt = blockIdx.y;
  const int kl = blockIdx.z / p.splits, split = blockIdx.z % p.splits;
  const int per = (p.kblocks + p.splits - 1) / p.splits;
  const int kb0 = split * per;
  const int nkb = max(0, min(p.kblocks, kb0 + per) - kb0);
  uint32_t ncols = 32;
  while ((int)ncols < p.bn) ncols <<= 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < p.stages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&done_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    asm volatile("tcgen05.fence::before_thread_sync;");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_slot;
  bool ok = true;

  if (warp == 0 && lane == 0 && nkb > 0) {
    // ---------------- TMA producer
    const int zA = p.k_first + kl;
    for (int i = 0; i < nkb && ok; ++i) {
      const int s = i % p.stages;
      if (i >= p.stages && !mbar_wait(&empty_bar[s], ((i / p.stages) & 1) ^ 1)) {
        ok = false;
        atomicExch(p.err, 1);
        break;
      }
      unsigned char* st = base + s * stage_bytes;
      mbar_expect_tx(&full_bar[s], stage_bytes);
      const int x = (kb0 + i) * kBK;
      tma_load_3d(st, &a_hi, &full_bar[s], x, mt * kBM, zA);
      tma_load_3d(st + a_bytes, &a_lo, &full_bar[s], x, mt * kBM, zA);
      tma_load_3d(st + 2 * a_bytes, &b_hi, &full_bar[s], x, nt * p.bn, kl);
      tma_load_3d(st + 2 * a_bytes + b_bytes, &b_lo, &full_bar[s], x, nt * p.bn, kl);
    }
  } else if (warp == 1 && lane == 0 && nkb > 0) {
    // ---------------- MMA issuer
    const uint32_t idesc = idesc_tf32(p.bn);
    for (int i = 0; i < nkb; ++i) {
      const int s = i % p.stages;
      if (!mbar_wait(&full_bar[s], (i / p.stages) & 1)) {
        atomicExch(p.err, 2);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      unsigned char* st = base + s * stage_bytes;
      const uint64_t ah = smem_desc(st), al = smem_desc(st + a_bytes);
      const uint64_t bh = smem_desc(st + 2 * a_bytes), bl = smem_desc(st + 2 * a_bytes + b_bytes);
#pragma unroll
      for (int kk = 0; kk < kBK / 8; ++kk) {
        const uint64_t off = (uint64_t)(kk * 32) >> 4;  // 8 TF32 = 32 bytes along K
        mma_tf32(tmem, ah + off, bh + off, idesc, (i | kk) != 0);
        mma_tf32(tmem, ah + off, bl + off, idesc, 1);
        mma_tf32(tmem, al + off, bh + off, idesc, 1);
      }
      mma_commit(&empty_bar[s]);
    }
    mma_commit(&done_bar);
  }
  __syncwarp();

  // ---------------- epilogue: TMEM -> registers -> global
  bool have = nkb > 0;
  if (have) {
    if (!mbar_wait(&done_bar, 0)) {
      atomicExch(p.err, 3);
      have = false;
    }
  }
  asm volatile("tcgen05.fence::after_thread_sync;");
  const int row = mt * kBM + warp * 32 + lane;
  const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
  if (MODE == 0) {
    float* dst = p.part + ((int64_t)kl * p.splits + split) * (int64_t)p.nbp * p.p2;
    for (int c0 = 0; c0 < p.bn; c0 += 8) {
      float v[8];
      if (have) {
        tmem_ld8(trow + c0, v);
      } else {
#pragma unroll
        for (int t = 0; t < 8; ++t) v[t] = 0.f;
      }
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const int col = nt * p.bn + c0 + t;
        if (col < p.nbp && row < p.p2) dst[(int64_t)col * p.p2 + row] = v[t];
      }
    }
  } else if (have) {
    // hpsi[m][row] += D[row][m]: 32 columns per round so that 32 independent loads of the
    // FFT result are in flight per thread before the adds and stores.
    const int k = p.k_first + kl;
    const int ld = 2 * p.npw[k];
    float* __restrict__ outk = p.out + 2 * (p.pw_off[k] - p.pw_off[p.k_first]) * p.nbands;
    const bool row_ok = row < ld;
    for (int c0 = 0; c0 < p.bn; c0 += 32) {
      float v[32];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float w[8];
        if (c0 + 8 * q < p.bn) {
          tmem_ld8(trow + c0 + 8 * q, w);
        } else {
#pragma unroll
          for (int t = 0; t < 8; ++t) w[t] = 0.f;
        }
#pragma unroll
        for (int t = 0; t < 8; ++t) v[8 * q + t] = w[t];
      }
      float old[32];
#pragma unroll
      for (int t = 0; t < 32; ++t) {
        const int m = nt * p.bn + c0 + t;
        old[t] = (row_ok && c0 + t < p.bn && m < p.n_valid) ? outk[(int64_t)m * ld + row] : 0.f;
      }
#pragma unroll
      for (int t = 0; t < 32; ++t) {
        const int m = nt * p.bn + c0 + t;
        if (row_ok && c0 + t < p.bn && m < p.n_valid) outk[(int64_t)m * ld + row] = old[t] + v[t];
      }
    }
  }
  __syncthreads();
  if (warp == 2) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
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
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  AMA_CUDA_TRY(cudaMalloc((void**)p, need));
  *have = need;
  return AMA_OK;
}

// dynamic shared memory: the operand ring plus 1 KB of alignment slack, under the 227 KB
// per-CTA limit minus the kernel's static barriers
constexpr int kSmemCap = 227 * 1024 - 1024;

size_t smem_bytes(int bn, int stages) { return (size_t)stages * (2 * kBM * kBK * 4 + 2 * bn * kBK * 4) + 1024; }

int pick_stages(int bn) {
  int s = kMaxStages;
  while (s > 2 && smem_bytes(bn, s) > (size_t)kSmemCap) --s;
  return s;
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
  AMA_CUDA_TRY(cudaFuncSetAttribute(tc_gemm_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemCap));
  AMA_CUDA_TRY(cudaFuncSetAttribute(tc_gemm_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemCap));
  t.ready = true;
  return AMA_OK;
}

int nl_tc_run(AmaEngine* e, int k_first, int k_count, int nbands, const float2* psi, float2* hpsi,
              cudaStream_t s) {
  NlTcState& t = e->tc;
  const int ntile = (nbands + 255) / 256;
  const int bn = round_up((nbands + ntile - 1) / ntile, 16);
  const int nbp = bn * ntile;
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
  // Each CTA accumulates at most kChainBlocks k-blocks in tensor memory: the tensor cores
  // add into the FP32 accumulator with truncation, whose error grows with the chain length;
  // the split partial sums are then added in FP32 with round-to-nearest by the reduction.
  constexpr int kChainBlocks = 16;
  int splits = std::max(1, (2 * 148 + mtiles1 * ntile * k_count - 1) / (mtiles1 * ntile * k_count));
  splits = std::max(splits, (kblocks + kChainBlocks - 1) / kChainBlocks);
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

  dim3 gs((t.kp + 255) / 256, nbp, k_count);
  split_psi_kernel<<<gs, 256, 0, s>>>((const float*)psi, e->d.pw_off, e->d.npw, k_first, nbands, nbp, t.kp,
                                      t.psi[0], t.psi[1]);
  AMA_CHECK_LAUNCH();

  TcArgs a{};
  a.kblocks = kblocks;
  a.splits = splits;
  a.bn = bn;
  a.n_valid = nbands;
  a.stages = pick_stages(bn);
  a.k_first = k_first;
  a.part = t.part;
  a.nbp = nbp;
  a.p2 = t.p2;
  a.err = t.err;
  dim3 g1(mtiles1, ntile, k_count * splits);
  tc_gemm_kernel<0><<<g1, kThreads, smem_bytes(bn, a.stages), s>>>(t.map_bx[0], t.map_bx[1], t.map_psi[0],
                                                                   t.map_psi[1], a);
  AMA_CHECK_LAUNCH();

  dim3 gr(1, nbp, k_count);
  reduce_q_kernel<<<gr, 256, 0, s>>>(t.part, splits, nbp, t.p2, t.k2, e->nproj, t.q[0], t.q[1]);
  AMA_CHECK_LAUNCH();

  TcArgs b{};
  b.kblocks = t.k2 / kBK;
  b.splits = 1;
  b.bn = bn;
  b.n_valid = nbands;
  b.stages = pick_stages(bn);
  b.k_first = k_first;
  b.out = (float*)hpsi;
  b.pw_off = e->d.pw_off;
  b.npw = e->d.npw;
  b.nbands = nbands;
  b.err = t.err;
  dim3 g2(t.mp / kBM, ntile, k_count);
  tc_gemm_kernel<1><<<g2, kThreads, smem_bytes(bn, b.stages), s>>>(t.map_dxt[0], t.map_dxt[1], t.map_q[0],
                                                                   t.map_q[1], b);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

void nl_tc_free(AmaEngine* e) {
  NlTcState& t = e->tc;
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
