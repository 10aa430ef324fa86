// ama_zgemm: strided-batched complex GEMM for the Davidson subspace products.
#include "common.cuh"
#include "gemm.cuh"

#include <algorithm>

using namespace ama;

namespace {

template <typename C> struct StridedBatch {
  const C* a; const C* b; C* c;
  int m, n, k;
  int64_t lda, ldb, ldc, sa, sb, sc;
  __device__ GemmProblem<C> operator()(int z) const {
    GemmProblem<C> p;
    p.a = a + z * sa; p.b = b + z * sb; p.c = c + z * sc;
    p.m = m; p.n = n; p.k = k; p.lda = lda; p.ldb = ldb; p.ldc = ldc;
    return p;
  }
};

struct Scratch { void* ptr = nullptr; size_t bytes = 0; };
thread_local PerDevice<Scratch> g_partial_dev;  // per host thread and device

template <typename T>
int zgemm_impl(int form, int m, int n, int k, const double* alpha, const void* a, int64_t lda,
               int64_t sa, const void* b, int64_t ldb, int64_t sb, const double* beta, void* c,
               int64_t ldc, int64_t sc, int batch, cudaStream_t s) {
  using C = cx_t<T>;
  StridedBatch<C> sbch{(const C*)a, (const C*)b, (C*)c, m, n, k, lda, ldb, ldc, sa, sb, sc};
  const C al = mk<C>(alpha[0], alpha[1]), be = mk<C>(beta[0], beta[1]);
  const int tiles = (int)std::min<int64_t>(gemm_tile_count<T>(m, n, batch), 1 << 30);
  int splits = std::max(1, std::min(32, (2 * 148 + tiles - 1) / tiles));
  splits = std::min(splits, std::max(1, k / 512));
  const int64_t pstride = (int64_t)m * n;
  Scratch* gpd = g_partial_dev.here();
  AMA_REQUIRE(gpd, AMA_ERR_CUDA, "complex GEMM: no usable current CUDA device");
  Scratch& g_partial = *gpd;
  if (splits > 1) {
    const size_t need = (size_t)batch * splits * pstride * sizeof(double2);
    if (g_partial.bytes < need) {
      bump_memory_epoch();
      if (g_partial.ptr) cudaFree(g_partial.ptr);
      g_partial.ptr = nullptr; g_partial.bytes = 0;
      AMA_CUDA_TRY(cudaMalloc(&g_partial.ptr, need));
      g_partial.bytes = need;
    }
  }
  cudaError_t err;
  if (form == 0) err = launch_cgemm<T, kNN>(sbch, batch, m, n, splits, al, be, (double2*)g_partial.ptr, pstride, s);
  else if (form == 1) err = launch_cgemm<T, kNC>(sbch, batch, m, n, splits, al, be, (double2*)g_partial.ptr, pstride, s);
  else err = launch_cgemm<T, kCN>(sbch, batch, m, n, splits, al, be, (double2*)g_partial.ptr, pstride, s);
  AMA_CUDA_TRY(err);
  return AMA_OK;
}

}  // namespace

extern "C" int ama_zgemm(int32_t precision, int32_t trans_b, int32_t m, int32_t n, int32_t k,
                         const double* alpha, const void* a, int64_t lda, int64_t stride_a,
                         const void* b, int64_t ldb, int64_t stride_b, const double* beta, void* c,
                         int64_t ldc, int64_t stride_c, int32_t batch, void* stream) {
  AMA_REQUIRE(precision == AMA_C64 || precision == AMA_C128, AMA_ERR_ARG, "bad precision");
  AMA_REQUIRE(trans_b >= 0 && trans_b <= 2, AMA_ERR_ARG, "trans_b must be 0, 1 or 2");
  AMA_REQUIRE(alpha && beta && a && b && c, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(m >= 0 && n >= 0 && k >= 0 && batch >= 1, AMA_ERR_SHAPE, "negative size");
  if (m == 0 || n == 0) return AMA_OK;
  cudaStream_t s = (cudaStream_t)stream;
  return precision == AMA_C64
             ? zgemm_impl<float>(trans_b, m, n, k, alpha, a, lda, stride_a, b, ldb, stride_b, beta, c, ldc, stride_c, batch, s)
             : zgemm_impl<double>(trans_b, m, n, k, alpha, a, lda, stride_a, b, ldb, stride_b, beta, c, ldc, stride_c, batch, s);
}

// ------------------------------------------------------------ per-k ragged batches
// One GEMM per k-point in one launch; any of m, n, k may be the k-point's plane-wave
// count (passed as -1). Operands live in packed per-k blocks (see AmaKOperand in ama.h).
namespace {

struct KOp {
  char* base;
  int64_t rows_per_k, row0, ld, kstride;
  int32_t ragged;
};

template <typename C> struct KBatch {
  KOp a, b, c;
  int m, n, k;
  const int* npw;
  const int64_t* pw_off;
  __device__ const C* at(const KOp& o, int z, int np, int64_t po) const {
    int64_t off;
    if (o.ragged) off = o.rows_per_k * po + o.row0 * np;
    else off = z * o.kstride + o.row0 * o.ld;
    return reinterpret_cast<const C*>(o.base) + off;
  }
  __device__ GemmProblem<C> operator()(int z) const {
    const int np = npw[z];
    const int64_t po = pw_off[z];
    GemmProblem<C> p;
    p.a = at(a, z, np, po);
    p.b = at(b, z, np, po);
    p.c = const_cast<C*>(at(c, z, np, po));
    p.m = m < 0 ? np : m;
    p.n = n < 0 ? np : n;
    p.k = k < 0 ? np : k;
    p.lda = a.ragged ? np : a.ld;
    p.ldb = b.ragged ? np : b.ld;
    p.ldc = c.ragged ? np : c.ld;
    return p;
  }
};

KOp to_kop(const AmaKOperand* o) {
  KOp r;
  r.base = (char*)o->base;
  r.rows_per_k = o->rows_per_k;
  r.row0 = o->row0;
  r.ld = o->ld;
  r.kstride = o->kstride;
  r.ragged = o->ragged;
  return r;
}

template <typename T>
int kbatch_impl(int form, int nk, int m, int n, int k, const int32_t* npw, const int64_t* pw_off,
                const AmaKOperand* a, const AmaKOperand* b, const AmaKOperand* c, const double* alpha,
                const double* beta, int max_m, int max_n, cudaStream_t s) {
  using C = cx_t<T>;
  KBatch<C> kb{to_kop(a), to_kop(b), to_kop(c), m, n, k, npw, pw_off};
  const C al = mk<C>(alpha[0], alpha[1]), be = mk<C>(beta[0], beta[1]);
  // split a long (plane-wave) reduction when the tile grid alone does not fill the GPU
  int splits = 1;
  if (k < 0) {  // a slice shorter than one k-tile (few plane waves) just writes zeros
    const int tiles = (int)std::min<int64_t>(gemm_tile_count<T>(max_m, max_n, nk), 1 << 30);
    splits = std::max(1, std::min(32, (2 * 148 + tiles - 1) / tiles));
  }
  const int64_t pstride = (int64_t)max_m * max_n;
  Scratch* gpd = g_partial_dev.here();
  AMA_REQUIRE(gpd, AMA_ERR_CUDA, "complex GEMM: no usable current CUDA device");
  Scratch& g_partial = *gpd;
  if (splits > 1) {
    const size_t need = (size_t)nk * splits * pstride * sizeof(double2);
    if (g_partial.bytes < need) {
      bump_memory_epoch();
      if (g_partial.ptr) cudaFree(g_partial.ptr);
      g_partial.ptr = nullptr; g_partial.bytes = 0;
      AMA_CUDA_TRY(cudaMalloc(&g_partial.ptr, need));
      g_partial.bytes = need;
    }
  }
  double2* part = (double2*)g_partial.ptr;
  cudaError_t err;
  if (form == 0) err = launch_cgemm<T, kNN>(kb, nk, max_m, max_n, splits, al, be, part, pstride, s);
  else if (form == 1) err = launch_cgemm<T, kNC>(kb, nk, max_m, max_n, splits, al, be, part, pstride, s);
  else err = launch_cgemm<T, kCN>(kb, nk, max_m, max_n, splits, al, be, part, pstride, s);
  AMA_CUDA_TRY(err);
  return AMA_OK;
}

}  // namespace

extern "C" int ama_kbatch_zgemm(int32_t precision, int32_t form, int32_t nk, int32_t m, int32_t n, int32_t k,
                                const int32_t* npw, const int64_t* pw_off, const AmaKOperand* a,
                                const AmaKOperand* b, const AmaKOperand* c, const double* alpha,
                                const double* beta, int32_t max_m, int32_t max_n, void* stream) {
  AMA_REQUIRE(precision == AMA_C64 || precision == AMA_C128, AMA_ERR_ARG, "bad precision");
  AMA_REQUIRE(form >= 0 && form <= 2, AMA_ERR_ARG, "form must be 0, 1 or 2");
  AMA_REQUIRE(a && b && c && npw && pw_off && alpha && beta, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(nk >= 1 && max_m >= 1 && max_n >= 1, AMA_ERR_SHAPE, "bad sizes");
  cudaStream_t s = (cudaStream_t)stream;
  return precision == AMA_C64 ? kbatch_impl<float>(form, nk, m, n, k, npw, pw_off, a, b, c, alpha, beta, max_m, max_n, s)
                              : kbatch_impl<double>(form, nk, m, n, k, npw, pw_off, a, b, c, alpha, beta, max_m, max_n, s);
}
