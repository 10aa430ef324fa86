// Split-TF32 tensor-core GEMM with drained accumulation chains (tcgen05, sm_100a):
//
//   D (128 x bn tile) = sum over the CTA's k-blocks of  A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T
//
// A and B are K-major FP32 arrays pre-split into a TF32-exact "hi" and a TF32 "lo" part
// (tc_gemm.cuh), read through 3D tensor maps [z][rows][K] by TMA (no multicast). The tensor
// cores accumulate in FP32 with truncation, so a long accumulation loses accuracy with its
// length. Here the accumulator is restarted every kChain k-blocks (24 products per output):
// the MMA issuer alternates between two TMEM buffers, and eight epilogue warps drain each
// finished buffer into FP32 registers (round to nearest) while the next chain runs.
//
// CTA roles (320 threads): warp 0 lane 0 = TMA producer; warp 1 allocates TMEM and lane 0
// issues the MMAs; warps 2..9 drain and write (warp w reads TMEM lanes 32 (w % 4) .. +31,
// columns 128 ((w - 2) / 4) .. +127 of the tile). Every mbarrier wait is bounded; on timeout
// the CTA stores an error code in a device flag and skips ahead to teardown.
//
// Epilogues:
//   kChainPartial   FP32 tile, column-major, to part[z][col][row] (z = blockIdx.z)
//   kChainComplexNN complex output from column pairs (2r, 2r+1) = (Re, Im) of row r,
//                   C[r][g] = alpha * D + beta * C with g = tile row (a plane wave)
//   kChainAddRows   out[m][row] += D[row][m] on interleaved per-k rows (nonlocal apply)
#pragma once
#include "common.cuh"
#include "tc_gemm.cuh"

namespace ama {
namespace tc {

constexpr int kChainThreads = 320;
constexpr int kChainBN = 256;       // widest N tile
constexpr int kChain = 2;           // k-blocks per accumulation chain
constexpr int kChainSmemCap = 227 * 1024 - 1024;

enum ChainMode { kChainPartial = 0, kChainComplexNN = 1, kChainAddRows = 2 };

struct ChainOp {  // a per-k operand: ragged (row length npw_k, packed per k) or a small dense matrix
  const float* base;  // complex64 storage viewed as floats
  int64_t rows_per_k, row0, ld, kstride;
  int ragged;
};

// first row of operand `o` at k-point z, and its row length in complex elements
__device__ __forceinline__ const float* chain_rows(const ChainOp& o, int z, int np, int64_t po, int64_t& ld) {
  if (o.ragged) {
    ld = np;
    return o.base + 2 * (o.rows_per_k * po + o.row0 * np);
  }
  ld = o.ld;
  return o.base + 2 * (z * o.kstride + o.row0 * o.ld);
}

struct ChainArgs {
  int kblocks;   // k-blocks of the whole reduction
  int splits;    // reduction splits: grid z = kz * splits + split
  int bn;        // N tile, multiple of 16, <= kChainBN
  int stages;    // operand ring depth, <= kMaxStages
  int a_z0;      // z offset of the A map (A spanning more k-points than the call)
  // kChainPartial
  float* part;
  int nrows, ncols;
  // kChainComplexNN
  ChainOp c;
  int m;
  float2 alpha, beta;
  // kChainComplexNN and kChainAddRows
  const int* npw;
  const int64_t* pw_off;
  // kChainAddRows
  float* out;
  int k_first, nbands, n_valid;
  int* err;
};

inline size_t chain_stage_bytes(int bn) { return (size_t)2 * kBM * kBK * 4 + (size_t)2 * bn * kBK * 4; }
inline int chain_stages(int bn) {
  int s = kMaxStages;
  while (s > 2 && (size_t)s * chain_stage_bytes(bn) + 1024 > (size_t)kChainSmemCap) --s;
  return s;
}
inline size_t chain_smem(int bn, int stages) { return (size_t)stages * chain_stage_bytes(bn) + 1024; }

__device__ __forceinline__ void chain_arrive(uint64_t* bar) {
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

template <int MODE>
__global__ void __launch_bounds__(kChainThreads, 1)
tc_chain_kernel(const __grid_constant__ CUtensorMap a_hi, const __grid_constant__ CUtensorMap a_lo,
                const __grid_constant__ CUtensorMap b_hi, const __grid_constant__ CUtensorMap b_lo, ChainArgs p) {
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  __shared__ __align__(8) uint64_t full_bar[kMaxStages], empty_bar[kMaxStages], tfull[2], tempty[2];
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
    for (int s = 0; s < p.stages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 8);
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
      const int za = p.a_z0 + kz;
      for (int i = 0; i < nkb; ++i) {
        const int s = i % p.stages;
        if (i >= p.stages && !mbar_wait(&empty_bar[s], ((i / p.stages) & 1) ^ 1)) {
          atomicExch(p.err, 11);
          break;
        }
        unsigned char* st = base + s * stage_bytes;
        mbar_expect_tx(&full_bar[s], stage_bytes);
        const int x = (kb0 + i) * kBK;
        tma_load_3d(st, &a_hi, &full_bar[s], x, mt * kBM, za);
        tma_load_3d(st + a_bytes, &a_lo, &full_bar[s], x, mt * kBM, za);
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
        const int s = i % p.stages;
        if (!mbar_wait(&full_bar[s], (i / p.stages) & 1)) {
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
    // ---------------- epilogue warps
    const int q = warp & 3;
    const int col0 = ((warp - 2) >> 2) * 128;  // first tile column of this warp
    const int row = mt * kBM + q * 32 + lane;
    const uint32_t tlane = tmem + ((uint32_t)(q * 32) << 16);
    float acc[128];
#pragma unroll
    for (int t = 0; t < 128; ++t) acc[t] = 0.f;
    for (int c = 0; c < nchains; ++c) {
      const int buf = c & 1;
      if (!mbar_wait(&tfull[buf], (c >> 1) & 1)) {
        atomicExch(p.err, 14);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
      for (int c0 = 0; c0 < 128; c0 += 32) {
        if (col0 + c0 < p.bn) {
          float v[32];
          tmem_ld32(tlane + (uint32_t)(buf * p.bn + col0 + c0), v);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int t = 0; t < 32; ++t) acc[c0 + t] += v[t];
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) chain_arrive(&tempty[buf]);
    }
    if (MODE == kChainPartial) {
      float* dst = p.part + (int64_t)blockIdx.z * p.ncols * p.nrows;
#pragma unroll
      for (int t = 0; t < 128; ++t) {
        const int lc = col0 + t, col = nt * p.bn + lc;
        if (lc < p.bn && col < p.ncols && row < p.nrows) dst[(int64_t)col * p.nrows + row] = acc[t];
      }
    } else if (MODE == kChainComplexNN) {
      const int np = p.npw[kz];
      if (row < np) {
        int64_t ld;
        const float* rows = chain_rows(p.c, kz, np, p.pw_off[kz], ld);
        float2* outk = const_cast<float2*>(reinterpret_cast<const float2*>(rows));
        const bool use_beta = p.beta.x != 0.f || p.beta.y != 0.f;
#pragma unroll
        for (int t = 0; t < 128; t += 2) {
          const int lc = col0 + t;
          const int r = (nt * p.bn + lc) >> 1;
          if (lc < p.bn && r < p.m) {
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
    } else {
      // out[m][row] += D[row][m]: 16 loads of the existing rows in flight before the stores
      const int k = p.k_first + kz;
      const int ld = 2 * p.npw[k];
      float* __restrict__ outk = p.out + 2 * (p.pw_off[k] - p.pw_off[p.k_first]) * p.nbands;
      if (row < ld) {
#pragma unroll
        for (int c0 = 0; c0 < 128; c0 += 16) {
          float old[16];
#pragma unroll
          for (int t = 0; t < 16; ++t) {
            const int lc = col0 + c0 + t, m = nt * p.bn + lc;
            old[t] = (lc < p.bn && m < p.n_valid) ? outk[(int64_t)m * ld + row] : 0.f;
          }
#pragma unroll
          for (int t = 0; t < 16; ++t) {
            const int lc = col0 + c0 + t, m = nt * p.bn + lc;
            if (lc < p.bn && m < p.n_valid) outk[(int64_t)m * ld + row] = old[t] + acc[c0 + t];
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

}  // namespace tc
}  // namespace ama
