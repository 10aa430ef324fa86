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
// and a TF32 "lo" remainder; the MMA adds hi.hi + hi.lo + lo.hi. Accuracy: the tensor
// cores accumulate in FP32 with truncation, so the accumulator is restarted every kChain
// k-blocks (24 products per element) and drained into FP32 registers by the epilogue warps
// (round to nearest) while the MMAs continue into the other of two TMEM buffers; long
// reductions are additionally split across CTAs and the splits summed in FP64.
//
// CTA roles (192 threads): warp 0 lane 0 issues TMA loads (no multicast), warp 1 allocates
// tensor memory and lane 0 issues the MMAs, warps 2-5 drain and write (warp w reads TMEM
// lanes 32 (w % 4) .. +31). Every mbarrier wait is bounded; on timeout the CTA records an
// error code in a device flag (read by ama_subspace_tc_status) and skips ahead to teardown.
#include "common.cuh"
#include "tc_gemm.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <string>

using namespace ama;
using namespace ama::tc;

namespace {

constexpr int kStThreads = 192;
constexpr int kStStages = 3;
constexpr int kStBN = 128;   // N tile (columns of D) at most
constexpr int kChain = 2;    // k-blocks per tensor-memory accumulation chain
constexpr int kMaxChainsPerCta = 96;

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

struct KOpDev {
  const float* base;  // interleaved complex64 storage viewed as floats
  int64_t rows_per_k, row0, ld, kstride;
  int ragged;
};

KOpDev to_dev(const AmaKOperand* o) {
  return KOpDev{(const float*)o->base, o->rows_per_k, o->row0, o->ld, o->kstride, o->ragged};
}

// first row of operand `o` at k-point z, and its row length in complex elements
__device__ __forceinline__ const float* op_rows(const KOpDev& o, int z, int np, int64_t po, int64_t& ld) {
  if (o.ragged) {
    ld = np;
    return o.base + 2 * (o.rows_per_k * po + o.row0 * np);
  }
  ld = o.ld;
  return o.base + 2 * (z * o.kstride + o.row0 * o.ld);
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

// ------------------------------------------------------------------ GEMM
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

struct StArgs {
  int kblocks;  // k-blocks of the whole reduction
  int splits;   // reduction splits (grid z = k-point * splits + split)
  int bn;       // N tile, multiple of 16, <= kStBN
  // NC: FP32 partial tiles, column-major [z][ncols][nrows]
  float* part;
  int nrows, ncols;
  // NN: complex64 output
  KOpDev c;
  const int* npw;
  const int64_t* pw_off;
  int m;
  float2 alpha, beta;
  int* err;
};

template <int MODE>  // 0 = NC partials, 1 = NN output
__global__ void __launch_bounds__(kStThreads, 1)
subspace_tc_kernel(const __grid_constant__ CUtensorMap a_hi, const __grid_constant__ CUtensorMap a_lo,
                   const __grid_constant__ CUtensorMap b_hi, const __grid_constant__ CUtensorMap b_lo, StArgs p) {
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  __shared__ __align__(8) uint64_t full_bar[kStStages], empty_bar[kStStages], tfull[2], tempty[2];
  __shared__ uint32_t tmem_slot;

  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_dyn) + 1023) & ~static_cast<uintptr_t>(1023));
  const int a_bytes = kBM * kBK * 4;
  const int b_bytes = p.bn * kBK * 4;
  const int stage_bytes = 2 * a_bytes + 2 * b_bytes;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nt = blockIdx.x, mt = blockIdx.y;
  const int kz = blockIdx.z / p.splits, split = blockIdx.z % p.splits;
  const int per = (p.kblocks + p.splits - 1) / p.splits;
  const int kb0 = split * per;
  const int nkb = max(0, min(p.kblocks, kb0 + per) - kb0);
  const int nchains = (nkb + kChain - 1) / kChain;
  uint32_t ncols = 32;
  while ((int)ncols < 2 * p.bn) ncols <<= 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStStages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    asm volatile("tcgen05.fence::before_thread_sync;");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      for (int i = 0; i < nkb; ++i) {
        const int s = i % kStStages;
        if (i >= kStStages && !mbar_wait(&empty_bar[s], ((i / kStStages) & 1) ^ 1)) {
          atomicExch(p.err, 11);
          break;
        }
        unsigned char* st = base + s * stage_bytes;
        mbar_expect_tx(&full_bar[s], stage_bytes);
        const int x = (kb0 + i) * kBK;
        tma_load_3d(st, &a_hi, &full_bar[s], x, mt * kBM, kz);
        tma_load_3d(st + a_bytes, &a_lo, &full_bar[s], x, mt * kBM, kz);
        tma_load_3d(st + 2 * a_bytes, &b_hi, &full_bar[s], x, nt * p.bn, kz);
        tma_load_3d(st + 2 * a_bytes + b_bytes, &b_lo, &full_bar[s], x, nt * p.bn, kz);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_tf32(p.bn);
      for (int i = 0; i < nkb; ++i) {
        const int c = i / kChain, buf = c & 1;
        const bool first = (i % kChain) == 0;
        if (first && c >= 2 && !mbar_wait(&tempty[buf], ((c >> 1) - 1) & 1)) {
          atomicExch(p.err, 12);
          break;
        }
        const int s = i % kStStages;
        if (!mbar_wait(&full_bar[s], (i / kStStages) & 1)) {
          atomicExch(p.err, 13);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        unsigned char* st = base + s * stage_bytes;
        const uint64_t ah = smem_desc(st), al = smem_desc(st + a_bytes);
        const uint64_t bh = smem_desc(st + 2 * a_bytes), bl = smem_desc(st + 2 * a_bytes + b_bytes);
        const uint32_t td = tmem + (uint32_t)(buf * p.bn);
#pragma unroll
        for (int kk = 0; kk < kBK / 8; ++kk) {
          const uint64_t off = (uint64_t)(kk * 32) >> 4;
          mma_tf32(td, ah + off, bh + off, idesc, (first && kk == 0) ? 0u : 1u);
          mma_tf32(td, ah + off, bl + off, idesc, 1);
          mma_tf32(td, al + off, bh + off, idesc, 1);
        }
        mma_commit(&empty_bar[s]);
        if ((i % kChain) == kChain - 1 || i == nkb - 1) mma_commit(&tfull[buf]);
      }
    }
  } else {
    // ---------------- epilogue warps: drain chains into registers, then write
    const int q = warp & 3;
    const int row = mt * kBM + q * 32 + lane;
    const uint32_t tlane = tmem + ((uint32_t)(q * 32) << 16);
    float acc[kStBN];
#pragma unroll
    for (int t = 0; t < kStBN; ++t) acc[t] = 0.f;
    for (int c = 0; c < nchains; ++c) {
      const int buf = c & 1;
      if (!mbar_wait(&tfull[buf], (c >> 1) & 1)) {
        atomicExch(p.err, 14);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
      for (int c0 = 0; c0 < kStBN; c0 += 32) {
        if (c0 < p.bn) {
          float v[32];
          tmem_ld32(tlane + (uint32_t)(buf * p.bn + c0), v);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int t = 0; t < 32; ++t) acc[c0 + t] += v[t];
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[buf]);
    }
    if (MODE == 0) {
      float* dst = p.part + (int64_t)blockIdx.z * p.ncols * p.nrows;
#pragma unroll
      for (int t = 0; t < kStBN; ++t) {
        const int col = nt * p.bn + t;
        if (t < p.bn && col < p.ncols && row < p.nrows) dst[(int64_t)col * p.nrows + row] = acc[t];
      }
    } else {
      const int np = p.npw[kz];
      if (row < np) {
        int64_t ld;
        float2* outk = const_cast<float2*>(
            reinterpret_cast<const float2*>(op_rows(p.c, kz, np, p.pw_off[kz], ld)));
        const bool use_beta = p.beta.x != 0.f || p.beta.y != 0.f;
#pragma unroll
        for (int t = 0; t < kStBN; t += 2) {
          const int r = (nt * p.bn + t) >> 1;
          if (t < p.bn && r < p.m) {
            const float re = acc[t], im = acc[t + 1];
            float2 o = make_float2(p.alpha.x * re - p.alpha.y * im, p.alpha.x * im + p.alpha.y * re);
            float2* d = outk + (int64_t)r * ld + row;
            if (use_beta) {
              const float2 old = *d;
              o.x += p.beta.x * old.x - p.beta.y * old.y;
              o.y += p.beta.x * old.y + p.beta.y * old.x;
            }
            *d = o;
          }
        }
      }
    }
  }
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
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
thread_local TcScratch g_tc;

size_t st_smem(int bn) { return (size_t)kStStages * (2 * kBM * kBK * 4 + 2 * bn * kBK * 4) + 1024; }

int tile_n(int cols) { return cols >= kStBN ? kStBN : std::max(16, round_up(cols, 16)); }

int ensure_err() {
  if (!g_tc.err) {
    AMA_CUDA_TRY(cudaMalloc((void**)&g_tc.err, sizeof(int)));
    AMA_CUDA_TRY(cudaMemset(g_tc.err, 0, sizeof(int)));
  }
  static bool attrs = false;
  if (!attrs) {
    AMA_CUDA_TRY(cudaFuncSetAttribute(subspace_tc_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)st_smem(kStBN)));
    AMA_CUDA_TRY(cudaFuncSetAttribute(subspace_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)st_smem(kStBN)));
    attrs = true;
  }
  return AMA_OK;
}

int run_nc(int nk, int m, int n, const int32_t* npw, const int64_t* pw_off, const AmaKOperand* a,
           const AmaKOperand* b, const AmaKOperand* c, const double* alpha, const double* beta, int max_npw,
           cudaStream_t s) {
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
  StArgs args{};
  args.kblocks = kblocks;
  args.splits = splits;
  args.bn = bn;
  args.part = g_tc.part.p;
  args.nrows = rows_a;
  args.ncols = npad;
  args.err = g_tc.err;
  subspace_tc_kernel<0><<<dim3(npad / bn, rows_a / kBM, nk * splits), kStThreads, st_smem(bn), s>>>(mah, mal, mbh,
                                                                                                  mbl, args);
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
  StArgs args{};
  args.kblocks = kp / kBK;
  args.splits = 1;
  args.bn = bn;
  args.c = cd;
  args.npw = npw;
  args.pw_off = pw_off;
  args.m = m;
  args.alpha = make_float2((float)alpha[0], (float)alpha[1]);
  args.beta = make_float2((float)beta[0], (float)beta[1]);
  args.err = g_tc.err;
  subspace_tc_kernel<1><<<dim3(rpad / bn, gpad / kBM, nk), kStThreads, st_smem(bn), s>>>(mah, mal, mbh, mbl, args);
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
  if (g_tc.err) AMA_CUDA_TRY(cudaMemcpy(code, g_tc.err, sizeof(int), cudaMemcpyDeviceToHost));
  return AMA_OK;
}
