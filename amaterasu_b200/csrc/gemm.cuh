// Complex GEMM on the SIMT pipes (FP32 or FP64), tiled 64x64 per CTA with a 4x4
// complex micro-tile per thread, split-K over a partial-sum buffer for long reductions.
// The FP32 form adds its running sums into FP64 registers every kFlushTiles k-tiles
// (128 products), so a long reduction (plane-wave count ~1e5) carries the rounding of a
// 128-term FP32 sum, not of the whole sum; split-K partials are FP64 for both precisions.
//
// Forms (all row-major):
//   NN : C = alpha * A(m x k) * B(k x n)        + beta * C
//   NC : C = alpha * A(m x k) * conj(B(n x k))^T + beta * C
//   CN : C = alpha * conj(A(k x m))^T * B(k x n) + beta * C
// Batches are described by a functor giving the matrix pointers and sizes of batch z,
// which lets the engine run ragged per-k products (different npw per k) in one launch.
#pragma once
#include "common.cuh"

#include <type_traits>

namespace ama {

enum GemmForm { kNN = 0, kNC = 1, kCN = 2 };

template <typename C> struct GemmProblem {
  const C* a; const C* b; C* c;
  int m, n, k;
  int64_t lda, ldb, ldc;
};

constexpr int kBM = 64, kBN = 64, kGemmThreads = 256;
template <typename T> struct GemmBK { static constexpr int value = 16; };
template <> struct GemmBK<double> { static constexpr int value = 8; };
constexpr int kFlushTiles = 8;  // FP32: 8 k-tiles of 16 = 128 products per FP32 partial sum

// One CTA computes a kBM x kBN tile of batch blockIdx.z / splits, reduction slice
// blockIdx.z % splits. If `partial` is non-null the raw tile sum goes to
// partial[(z_split * M*N ...)] (see engine), else the alpha/beta epilogue is applied.
template <typename T, int FORM, class Batch>
__global__ void __launch_bounds__(kGemmThreads)
cgemm_tile_kernel(Batch batch, int splits, cx_t<T> alpha, cx_t<T> beta, double2* partial,
                  int64_t partial_stride) {
  using C = cx_t<T>;
  constexpr int BK = GemmBK<T>::value;
  constexpr int LA = BK * kBM / kGemmThreads;  // tile elements each thread stages
  constexpr int LB = BK * kBN / kGemmThreads;
  // two shared-memory buffers: the next k-tile is loaded into registers while the current
  // one is multiplied, then stored into the other buffer (one barrier per k-tile)
  __shared__ C As[2][BK][kBM + 1];
  __shared__ C Bs[2][BK][kBN + 1];

  const int z = blockIdx.z;
  const int bz = z / splits, sz = z % splits;
  const GemmProblem<C> p = batch(bz);
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  if (m0 >= p.m || n0 >= p.n) return;
  const int kchunk = ((p.k + splits - 1) / splits + BK - 1) / BK * BK;
  const int kbeg = sz * kchunk;
  const int kend = min(p.k, kbeg + kchunk);

  const int tid = threadIdx.x;
  const int tx = tid % 16, ty = tid / 16;
  constexpr bool kFlush = std::is_same<T, float>::value;
  C acc[4][4];
  double2 dacc[kFlush ? 4 : 1][kFlush ? 4 : 1];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = mk<C>(0, 0);
  if constexpr (kFlush) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) dacc[i][j] = make_double2(0.0, 0.0);
  }

  C ra[LA], rb[LB];
  auto load_tile = [&](int k0) {
#pragma unroll
    for (int l = 0; l < LA; ++l) {
      const int e = tid + l * kGemmThreads;
      int mm, kk;
      if (FORM == kCN) { mm = e % kBM; kk = e / kBM; }   // A is (k x m): m contiguous
      else { kk = e % BK; mm = e / BK; }                  // A is (m x k): k contiguous
      const int gm = m0 + mm, gk = k0 + kk;
      C v = mk<C>(0, 0);
      if (gm < p.m && gk < kend) {
        if (FORM == kCN) { v = p.a[(int64_t)gk * p.lda + gm]; v.y = -v.y; }
        else v = p.a[(int64_t)gm * p.lda + gk];
      }
      ra[l] = v;
    }
#pragma unroll
    for (int l = 0; l < LB; ++l) {
      const int e = tid + l * kGemmThreads;
      int nn, kk;
      if (FORM == kNC) { kk = e % BK; nn = e / BK; }      // B is (n x k): k contiguous
      else { nn = e % kBN; kk = e / kBN; }                // B is (k x n): n contiguous
      const int gn = n0 + nn, gk = k0 + kk;
      C v = mk<C>(0, 0);
      if (gn < p.n && gk < kend) {
        if (FORM == kNC) { v = p.b[(int64_t)gn * p.ldb + gk]; v.y = -v.y; }
        else v = p.b[(int64_t)gk * p.ldb + gn];
      }
      rb[l] = v;
    }
  };
  auto store_tile = [&](int buf) {
#pragma unroll
    for (int l = 0; l < LA; ++l) {
      const int e = tid + l * kGemmThreads;
      if (FORM == kCN) As[buf][e / kBM][e % kBM] = ra[l];
      else As[buf][e % BK][e / BK] = ra[l];
    }
#pragma unroll
    for (int l = 0; l < LB; ++l) {
      const int e = tid + l * kGemmThreads;
      if (FORM == kNC) Bs[buf][e % BK][e / BK] = rb[l];
      else Bs[buf][e / kBN][e % kBN] = rb[l];
    }
  };

  int tile_count = 0, buf = 0;
  if (kbeg < kend) {
    load_tile(kbeg);
    store_tile(0);
  }
  __syncthreads();
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    const bool more = k0 + BK < kend;
    if (more) load_tile(k0 + BK);  // global loads in flight during the products below
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      C a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[buf][kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[buf][kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x += a[i].x * b[j].x - a[i].y * b[j].y;
          acc[i][j].y += a[i].x * b[j].y + a[i].y * b[j].x;
        }
    }
    if (more) store_tile(buf ^ 1);
    __syncthreads();
    buf ^= 1;
    if constexpr (kFlush) {
      if (++tile_count == kFlushTiles) {
        tile_count = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            dacc[i][j].x += (double)acc[i][j].x;
            dacc[i][j].y += (double)acc[i][j].y;
            acc[i][j] = mk<C>(0, 0);
          }
      }
    }
  }
  // the tile's sums in FP64
  double2 sum[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if constexpr (kFlush)
        sum[i][j] = make_double2(dacc[i][j].x + (double)acc[i][j].x, dacc[i][j].y + (double)acc[i][j].y);
      else
        sum[i][j] = make_double2((double)acc[i][j].x, (double)acc[i][j].y);
    }

#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gm = m0 + ty + 16 * i;
    if (gm >= p.m) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gn = n0 + tx + 16 * j;
      if (gn >= p.n) continue;
      if (partial) {
        partial[(int64_t)z * partial_stride + (int64_t)gm * p.n + gn] = sum[i][j];
      } else {
        C* dst = p.c + (int64_t)gm * p.ldc + gn;
        C r = cmul(alpha, mk<C>(sum[i][j].x, sum[i][j].y));
        if (beta.x != T(0) || beta.y != T(0)) r = cadd(r, cmul(beta, *dst));
        *dst = r;
      }
    }
  }
}

// FP64 complex GEMM on the FP64 tensor cores (mma.sync m8n8k4, DMMA): same forms, batches,
// split-K and epilogue as cgemm_tile_kernel<double>. A CTA computes a BM x BN complex tile
// with 8 warps (WMW along M x 8/WMW along N); the 64 x 64 tile has 2 x 4 warps of 32 x 16
// complex = 4 x 2 blocks of 8 x 8 each. The k-tile (8) is staged as separate real and
// imaginary planes, k-major with a row pitch of BM + 8 (BN + 8) doubles, 8 modulo 16 (the
// fragment loads of a warp then take the minimum two wavefronts), double buffered with a
// register prefetch of the next tile. Per 8 x 8 block and k-step of 4:
//   Re C += Ar Br + (-Ai) Bi,   Im C += Ar Bi + Ai Br   (four DMMAs).
// The tensor cores compute the whole padded tile, so short operands (the Davidson's block
// of at most 32 new directions, its small Gram and projection matrices) take a 32-row tile:
// 32 x 128 (warps 1 x 8, the same 32 x 16 warp tile) or 32 x 32 (warps 2 x 4 of 16 x 8).
constexpr int kDmmaBK = 8;

__device__ __forceinline__ void dmma_884(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// The CTA tile of the FP64 kernel for a problem of at most max_m x max_n.
struct DmmaTile {
  int bm, bn;
};
inline DmmaTile dmma_tile(int max_m, int max_n) {
  if (max_m <= 32 && max_n <= 64) return {32, 32};
  if (max_m <= 32) return {32, 128};
  return {64, 64};
}

// The CTA tile launch_cgemm<T> uses: the FP64 tensor-core kernel's choice for complex128,
// and for complex64 too when at most 32 rows (complex64 operands staged in FP64; longer
// ones take the 64 x 64 SIMT FP32 tile).
template <typename T> inline DmmaTile gemm_tile(int max_m, int max_n) {
  if (std::is_same<T, double>::value || max_m <= 32) return dmma_tile(max_m, max_n);
  return {kBM, kBN};
}

// Tiles the launch of launch_cgemm<T> covers (split-K counts are sized from it).
template <typename T> inline int64_t gemm_tile_count(int max_m, int max_n, int nbatch) {
  const DmmaTile t = gemm_tile<T>(max_m, max_n);
  return (int64_t)((max_m + t.bm - 1) / t.bm) * ((max_n + t.bn - 1) / t.bn) * nbatch;
}

template <typename T, int FORM, int BM, int BN, int WMW, class Batch>
__global__ void __launch_bounds__(kGemmThreads, 2)
zgemm_dmma_kernel(Batch batch, int splits, double2 alpha, double2 beta, double2* partial, int64_t partial_stride) {
  using C = cx_t<T>;  // operands and result; staged, multiplied and summed in FP64
  constexpr int BK = kDmmaBK, PA = BM + 8, PB = BN + 8;
  constexpr int WNW = kGemmThreads / 32 / WMW;
  constexpr int WTM = BM / WMW, WTN = BN / WNW;  // warp tile
  constexpr int IM = WTM / 8, JN = WTN / 8;      // 8 x 8 blocks per warp
  constexpr int LA = BK * BM / kGemmThreads, LB = BK * BN / kGemmThreads;
  static_assert(WTM % 8 == 0 && WTN % 8 == 0 && LA >= 1 && LB >= 1 && BK * BM % kGemmThreads == 0 &&
                    BK * BN % kGemmThreads == 0 && PA % 16 == 8 && PB % 16 == 8,
                "DMMA tile shape");
  __shared__ double Ar[2][BK][PA], Ai[2][BK][PA], Br[2][BK][PB], Bi[2][BK][PB];

  const int z = blockIdx.z;
  const int bz = z / splits, sz = z % splits;
  const GemmProblem<C> p = batch(bz);
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  if (m0 >= p.m || n0 >= p.n) return;
  const int kchunk = ((p.k + splits - 1) / splits + BK - 1) / BK * BK;
  const int kbeg = sz * kchunk;
  const int kend = min(p.k, kbeg + kchunk);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp % WMW) * WTM, wn = (warp / WMW) * WTN;
  const int fr = lane >> 2, fk = lane & 3;  // fragment row (m or n) and k of this lane

  double cre[IM][JN][2], cim[IM][JN][2];
#pragma unroll
  for (int i = 0; i < IM; ++i)
#pragma unroll
    for (int j = 0; j < JN; ++j) cre[i][j][0] = cre[i][j][1] = cim[i][j][0] = cim[i][j][1] = 0.0;

  double2 ra[LA], rb[LB];
  auto load_tile = [&](int k0) {
#pragma unroll
    for (int l = 0; l < LA; ++l) {
      const int e = tid + l * kGemmThreads;
      int mm, kk;
      if (FORM == kCN) { mm = e % BM; kk = e / BM; }
      else { kk = e % BK; mm = e / BK; }
      const int gm = m0 + mm, gk = k0 + kk;
      double2 v = make_double2(0.0, 0.0);
      if (gm < p.m && gk < kend) {
        const C x = FORM == kCN ? p.a[(int64_t)gk * p.lda + gm] : p.a[(int64_t)gm * p.lda + gk];
        v = make_double2((double)x.x, FORM == kCN ? -(double)x.y : (double)x.y);
      }
      ra[l] = v;
    }
#pragma unroll
    for (int l = 0; l < LB; ++l) {
      const int e = tid + l * kGemmThreads;
      int nn, kk;
      if (FORM == kNC) { kk = e % BK; nn = e / BK; }
      else { nn = e % BN; kk = e / BN; }
      const int gn = n0 + nn, gk = k0 + kk;
      double2 v = make_double2(0.0, 0.0);
      if (gn < p.n && gk < kend) {
        const C x = FORM == kNC ? p.b[(int64_t)gn * p.ldb + gk] : p.b[(int64_t)gk * p.ldb + gn];
        v = make_double2((double)x.x, FORM == kNC ? -(double)x.y : (double)x.y);
      }
      rb[l] = v;
    }
  };
  auto store_tile = [&](int buf) {
#pragma unroll
    for (int l = 0; l < LA; ++l) {
      const int e = tid + l * kGemmThreads;
      int mm, kk;
      if (FORM == kCN) { mm = e % BM; kk = e / BM; }
      else { kk = e % BK; mm = e / BK; }
      Ar[buf][kk][mm] = ra[l].x;
      Ai[buf][kk][mm] = ra[l].y;
    }
#pragma unroll
    for (int l = 0; l < LB; ++l) {
      const int e = tid + l * kGemmThreads;
      int nn, kk;
      if (FORM == kNC) { kk = e % BK; nn = e / BK; }
      else { nn = e % BN; kk = e / BN; }
      Br[buf][kk][nn] = rb[l].x;
      Bi[buf][kk][nn] = rb[l].y;
    }
  };

  int buf = 0;
  if (kbeg < kend) {
    load_tile(kbeg);
    store_tile(0);
  }
  __syncthreads();
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    const bool more = k0 + BK < kend;
    if (more) load_tile(k0 + BK);
#pragma unroll
    for (int ks = 0; ks < BK; ks += 4) {
      double ar[IM], ai[IM], nai[IM], br[JN], bi[JN];
#pragma unroll
      for (int i = 0; i < IM; ++i) {
        ar[i] = Ar[buf][ks + fk][wm + 8 * i + fr];
        ai[i] = Ai[buf][ks + fk][wm + 8 * i + fr];
        nai[i] = -ai[i];
      }
#pragma unroll
      for (int j = 0; j < JN; ++j) {
        br[j] = Br[buf][ks + fk][wn + 8 * j + fr];
        bi[j] = Bi[buf][ks + fk][wn + 8 * j + fr];
      }
#pragma unroll
      for (int i = 0; i < IM; ++i)
#pragma unroll
        for (int j = 0; j < JN; ++j) {
          dmma_884(cre[i][j], ar[i], br[j]);
          dmma_884(cre[i][j], nai[i], bi[j]);
          dmma_884(cim[i][j], ar[i], bi[j]);
          dmma_884(cim[i][j], ai[i], br[j]);
        }
    }
    if (more) store_tile(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }

  // lane holds C[wm + 8 i + fr][wn + 8 j + 2 fk + t]
#pragma unroll
  for (int i = 0; i < IM; ++i) {
    const int gm = m0 + wm + 8 * i + fr;
    if (gm >= p.m) continue;
#pragma unroll
    for (int j = 0; j < JN; ++j)
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int gn = n0 + wn + 8 * j + 2 * fk + t;
        if (gn >= p.n) continue;
        const double2 sum = make_double2(cre[i][j][t], cim[i][j][t]);
        if (partial) {
          partial[(int64_t)z * partial_stride + (int64_t)gm * p.n + gn] = sum;
        } else {
          C* dst = p.c + (int64_t)gm * p.ldc + gn;
          double2 r = cmul(alpha, sum);
          if (beta.x != 0.0 || beta.y != 0.0) {
            const C d = *dst;
            r = cadd(r, cmul(beta, make_double2((double)d.x, (double)d.y)));
          }
          *dst = mk<C>(r.x, r.y);
        }
      }
  }
}

// Sum the split-K partials of each batch and apply the epilogue.
template <typename T, class Batch>
__global__ void cgemm_reduce_kernel(Batch batch, int splits, cx_t<T> alpha, cx_t<T> beta,
                                    const double2* partial, int64_t partial_stride) {
  using C = cx_t<T>;
  const int bz = blockIdx.y;
  const GemmProblem<C> p = batch(bz);
  const int64_t total = (int64_t)p.m * p.n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    double2 s = make_double2(0.0, 0.0);
    for (int sidx = 0; sidx < splits; ++sidx) {
      const double2 v = partial[(int64_t)(bz * splits + sidx) * partial_stride + e];
      s.x += v.x;
      s.y += v.y;
    }
    const int gm = (int)(e / p.n), gn = (int)(e % p.n);
    C* dst = p.c + (int64_t)gm * p.ldc + gn;
    C r = cmul(alpha, mk<C>(s.x, s.y));
    if (beta.x != T(0) || beta.y != T(0)) r = cadd(r, cmul(beta, *dst));
    *dst = r;
  }
}

// Launch helper. `max_m/max_n/max_k` bound the batch's sizes (grid shape); `splits` > 1
// needs `partial` sized batch*splits*partial_stride FP64 complex elements with
// partial_stride >= m*n.
template <typename T, int FORM, class Batch>
cudaError_t launch_cgemm(Batch batch, int nbatch, int max_m, int max_n, int splits,
                         cx_t<T> alpha, cx_t<T> beta, double2* partial, int64_t partial_stride,
                         cudaStream_t stream) {
  dim3 grid((max_n + kBN - 1) / kBN, (max_m + kBM - 1) / kBM, nbatch * splits);
  const DmmaTile t = gemm_tile<T>(max_m, max_n);
  if (std::is_same<T, double>::value || t.bm == 32) {  // the FP64 tensor cores
    grid = dim3((max_n + t.bn - 1) / t.bn, (max_m + t.bm - 1) / t.bm, nbatch * splits);
    const int sp = splits <= 1 ? 1 : splits;
    double2* part = splits <= 1 ? nullptr : partial;
    const double2 al = make_double2((double)alpha.x, (double)alpha.y);
    const double2 be = make_double2((double)beta.x, (double)beta.y);
    if (t.bm == 32 && t.bn == 32)
      zgemm_dmma_kernel<T, FORM, 32, 32, 2><<<grid, kGemmThreads, 0, stream>>>(batch, sp, al, be, part,
                                                                             partial_stride);
    else if (t.bm == 32)
      zgemm_dmma_kernel<T, FORM, 32, 128, 1><<<grid, kGemmThreads, 0, stream>>>(batch, sp, al, be, part,
                                                                              partial_stride);
    else if constexpr (std::is_same<T, double>::value)
      zgemm_dmma_kernel<T, FORM, 64, 64, 2><<<grid, kGemmThreads, 0, stream>>>(batch, sp, al, be, part,
                                                                             partial_stride);
    if (splits <= 1) return cudaGetLastError();
  } else {
    if (splits <= 1) {
      cgemm_tile_kernel<T, FORM><<<grid, kGemmThreads, 0, stream>>>(batch, 1, alpha, beta, nullptr, 0);
      return cudaGetLastError();
    }
    cgemm_tile_kernel<T, FORM><<<grid, kGemmThreads, 0, stream>>>(batch, splits, alpha, beta, partial,
                                                                  partial_stride);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  dim3 rgrid(64, nbatch);
  cgemm_reduce_kernel<T><<<rgrid, 256, 0, stream>>>(batch, splits, alpha, beta, partial, partial_stride);
  return cudaGetLastError();
}

}  // namespace ama
