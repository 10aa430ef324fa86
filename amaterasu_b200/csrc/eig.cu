// Dense FP64 Hermitian eigensolver for the Rayleigh-Ritz subspace matrices (cuSOLVER
// zheevd, the LAPACK routine the reference reaches through scipy.linalg.eigh).
#include "common.cuh"

#include <cusolverDn.h>

#include <algorithm>
#include <vector>

using namespace ama;

namespace {

struct SolverState {
  cusolverDnHandle_t handle = nullptr;
  void* work = nullptr;
  size_t work_bytes = 0;
  int* info = nullptr;
};
thread_local SolverState g_solver;

// Row-major Hermitian A read as column-major is conj(A); zheevd then returns conj(v_j)
// in column j, i.e. row j of the row-major array. Transpose-conjugate in place so that
// the row-major result holds v_j in column j (numpy's eigh convention).
__global__ void conj_transpose_kernel(double2* m, int n) {
  double2* a = m + (int64_t)blockIdx.y * n * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = e / n, j = e % n;
    if (j < i) continue;
    double2 x = a[(int64_t)i * n + j], y = a[(int64_t)j * n + i];
    a[(int64_t)i * n + j] = make_double2(y.x, -y.y);
    a[(int64_t)j * n + i] = make_double2(x.x, -x.y);
  }
}

__global__ void check_info_kernel(const int* info, int* flag) {
  if (threadIdx.x == 0 && *info != 0) *flag = *info;
}

}  // namespace

extern "C" int ama_heev(int32_t n, void* matrices, double* eigenvalues, int32_t batch, void* stream) {
  AMA_REQUIRE(matrices && eigenvalues, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(n >= 1 && batch >= 1, AMA_ERR_SHAPE, "bad sizes");
  cudaStream_t s = (cudaStream_t)stream;
  if (!g_solver.handle) {
    if (cusolverDnCreate(&g_solver.handle) != CUSOLVER_STATUS_SUCCESS) {
      set_error("cusolverDnCreate failed");
      return AMA_ERR_CUDA;
    }
    AMA_CUDA_TRY(cudaMalloc((void**)&g_solver.info, 2 * sizeof(int)));
  }
  cusolverDnSetStream(g_solver.handle, s);
  int lwork = 0;
  if (cusolverDnZheevd_bufferSize(g_solver.handle, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n,
                                  (cuDoubleComplex*)matrices, n, eigenvalues, &lwork) != CUSOLVER_STATUS_SUCCESS) {
    set_error("cusolverDnZheevd_bufferSize failed");
    return AMA_ERR_CUDA;
  }
  const size_t need = (size_t)lwork * sizeof(cuDoubleComplex);
  if (g_solver.work_bytes < need) {
    if (g_solver.work) cudaFree(g_solver.work);
    g_solver.work = nullptr; g_solver.work_bytes = 0;
    AMA_CUDA_TRY(cudaMalloc(&g_solver.work, need));
    g_solver.work_bytes = need;
  }
  AMA_CUDA_TRY(cudaMemsetAsync(g_solver.info + 1, 0, sizeof(int), s));
  for (int b = 0; b < batch; ++b) {
    cuDoubleComplex* a = (cuDoubleComplex*)matrices + (int64_t)b * n * n;
    if (cusolverDnZheevd(g_solver.handle, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, a, n,
                         eigenvalues + (int64_t)b * n, (cuDoubleComplex*)g_solver.work, lwork,
                         g_solver.info) != CUSOLVER_STATUS_SUCCESS) {
      set_error("cusolverDnZheevd failed");
      return AMA_ERR_CUDA;
    }
    check_info_kernel<<<1, 32, 0, s>>>(g_solver.info, g_solver.info + 1);
  }
  dim3 grid(std::max(1, std::min(64, (n * n + 255) / 256)), batch);
  conj_transpose_kernel<<<grid, 256, 0, s>>>((double2*)matrices, n);
  AMA_CHECK_LAUNCH();
  int flag = 0;
  AMA_CUDA_TRY(cudaMemcpyAsync(&flag, g_solver.info + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  AMA_CUDA_TRY(cudaStreamSynchronize(s));
  AMA_REQUIRE(flag == 0, AMA_ERR_NOT_CONVERGED, "zheevd did not converge");
  return AMA_OK;
}

// The lowest nvec eigenpairs only (zheevdx, index range 1..nvec): the tridiagonal reduction
// is the same, but bisection and inverse iteration replace divide and conquer and only nvec
// vectors are back-transformed. Eigenvalues [0, nvec) ascending; eigenvectors in columns
// [0, nvec) (row-major, as ama_heev); the other entries are undefined.
extern "C" int ama_heev_lowest(int32_t n, int32_t nvec, void* matrices, double* eigenvalues, int32_t batch,
                               void* stream) {
  AMA_REQUIRE(matrices && eigenvalues, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(n >= 1 && batch >= 1 && nvec >= 1 && nvec <= n, AMA_ERR_SHAPE, "bad sizes");
  cudaStream_t s = (cudaStream_t)stream;
  if (!g_solver.handle) {
    if (cusolverDnCreate(&g_solver.handle) != CUSOLVER_STATUS_SUCCESS) {
      set_error("cusolverDnCreate failed");
      return AMA_ERR_CUDA;
    }
    AMA_CUDA_TRY(cudaMalloc((void**)&g_solver.info, 2 * sizeof(int)));
  }
  cusolverDnSetStream(g_solver.handle, s);
  int lwork = 0, meig = 0;
  if (cusolverDnZheevdx_bufferSize(g_solver.handle, CUSOLVER_EIG_MODE_VECTOR, CUSOLVER_EIG_RANGE_I,
                                   CUBLAS_FILL_MODE_LOWER, n, (cuDoubleComplex*)matrices, n, 0.0, 0.0, 1, nvec,
                                   &meig, eigenvalues, &lwork) != CUSOLVER_STATUS_SUCCESS) {
    set_error("cusolverDnZheevdx_bufferSize failed");
    return AMA_ERR_CUDA;
  }
  const size_t need = (size_t)lwork * sizeof(cuDoubleComplex);
  if (g_solver.work_bytes < need) {
    if (g_solver.work) cudaFree(g_solver.work);
    g_solver.work = nullptr; g_solver.work_bytes = 0;
    AMA_CUDA_TRY(cudaMalloc(&g_solver.work, need));
    g_solver.work_bytes = need;
  }
  AMA_CUDA_TRY(cudaMemsetAsync(g_solver.info + 1, 0, sizeof(int), s));
  for (int b = 0; b < batch; ++b) {
    cuDoubleComplex* a = (cuDoubleComplex*)matrices + (int64_t)b * n * n;
    if (cusolverDnZheevdx(g_solver.handle, CUSOLVER_EIG_MODE_VECTOR, CUSOLVER_EIG_RANGE_I, CUBLAS_FILL_MODE_LOWER,
                          n, a, n, 0.0, 0.0, 1, nvec, &meig, eigenvalues + (int64_t)b * n,
                          (cuDoubleComplex*)g_solver.work, lwork, g_solver.info) != CUSOLVER_STATUS_SUCCESS) {
      set_error("cusolverDnZheevdx failed");
      return AMA_ERR_CUDA;
    }
    check_info_kernel<<<1, 32, 0, s>>>(g_solver.info, g_solver.info + 1);
  }
  dim3 grid(std::max(1, std::min(64, (n * n + 255) / 256)), batch);
  conj_transpose_kernel<<<grid, 256, 0, s>>>((double2*)matrices, n);
  AMA_CHECK_LAUNCH();
  int flag = 0;
  AMA_CUDA_TRY(cudaMemcpyAsync(&flag, g_solver.info + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  AMA_CUDA_TRY(cudaStreamSynchronize(s));
  AMA_REQUIRE(flag == 0, AMA_ERR_NOT_CONVERGED, "zheevdx did not converge");
  AMA_REQUIRE(meig == nvec, AMA_ERR_NOT_CONVERGED, "zheevdx returned fewer eigenpairs than asked for");
  return AMA_OK;
}

namespace {
// Keep only the row-major upper triangle (where the column-major lower result lands),
// then conjugate-transpose so the row-major lower triangle holds the result.
__global__ void keep_upper_conj_transpose_kernel(double2* m, int n) {
  double2* a = m + (int64_t)blockIdx.y * n * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = e / n, j = e % n;
    if (j < i) continue;
    const double2 up = a[(int64_t)i * n + j];
    a[(int64_t)j * n + i] = make_double2(up.x, -up.y);
    if (j != i) a[(int64_t)i * n + j] = make_double2(0.0, 0.0);
  }
}
}  // namespace

extern "C" int ama_potrf_inv(int32_t n, void* matrices, int32_t batch, void* stream) {
  AMA_REQUIRE(matrices, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(n >= 1 && batch >= 1, AMA_ERR_SHAPE, "bad sizes");
  cudaStream_t s = (cudaStream_t)stream;
  if (!g_solver.handle) {
    if (cusolverDnCreate(&g_solver.handle) != CUSOLVER_STATUS_SUCCESS) {
      set_error("cusolverDnCreate failed");
      return AMA_ERR_CUDA;
    }
    AMA_CUDA_TRY(cudaMalloc((void**)&g_solver.info, 2 * sizeof(int)));
  }
  cusolverDnSetStream(g_solver.handle, s);
  int lwork = 0;
  if (cusolverDnZpotrf_bufferSize(g_solver.handle, CUBLAS_FILL_MODE_LOWER, n, (cuDoubleComplex*)matrices, n,
                                  &lwork) != CUSOLVER_STATUS_SUCCESS) {
    set_error("cusolverDnZpotrf_bufferSize failed");
    return AMA_ERR_CUDA;
  }
  size_t dev_bytes = 0, host_bytes = 0;
  cusolverDnParams_t params;
  cusolverDnCreateParams(&params);
  if (cusolverDnXtrtri_bufferSize(g_solver.handle, CUBLAS_FILL_MODE_LOWER, CUBLAS_DIAG_NON_UNIT, n, CUDA_C_64F,
                                  matrices, n, &dev_bytes, &host_bytes) != CUSOLVER_STATUS_SUCCESS) {
    cusolverDnDestroyParams(params);
    set_error("cusolverDnXtrtri_bufferSize failed");
    return AMA_ERR_CUDA;
  }
  cusolverDnDestroyParams(params);
  const size_t need = std::max((size_t)lwork * sizeof(cuDoubleComplex), dev_bytes) + 256;
  if (g_solver.work_bytes < need) {
    if (g_solver.work) cudaFree(g_solver.work);
    g_solver.work = nullptr; g_solver.work_bytes = 0;
    AMA_CUDA_TRY(cudaMalloc(&g_solver.work, need));
    g_solver.work_bytes = need;
  }
  std::vector<char> host_work(std::max<size_t>(host_bytes, 1));
  AMA_CUDA_TRY(cudaMemsetAsync(g_solver.info + 1, 0, sizeof(int), s));
  for (int b = 0; b < batch; ++b) {
    cuDoubleComplex* a = (cuDoubleComplex*)matrices + (int64_t)b * n * n;
    if (cusolverDnZpotrf(g_solver.handle, CUBLAS_FILL_MODE_LOWER, n, a, n, (cuDoubleComplex*)g_solver.work,
                         lwork, g_solver.info) != CUSOLVER_STATUS_SUCCESS) {
      set_error("cusolverDnZpotrf failed");
      return AMA_ERR_CUDA;
    }
    check_info_kernel<<<1, 32, 0, s>>>(g_solver.info, g_solver.info + 1);
    if (cusolverDnXtrtri(g_solver.handle, CUBLAS_FILL_MODE_LOWER, CUBLAS_DIAG_NON_UNIT, n, CUDA_C_64F, a, n,
                         g_solver.work, dev_bytes, host_work.data(), host_bytes,
                         g_solver.info) != CUSOLVER_STATUS_SUCCESS) {
      set_error("cusolverDnXtrtri failed");
      return AMA_ERR_CUDA;
    }
    check_info_kernel<<<1, 32, 0, s>>>(g_solver.info, g_solver.info + 1);
  }
  dim3 grid(std::max(1, std::min(64, (n * n + 255) / 256)), batch);
  keep_upper_conj_transpose_kernel<<<grid, 256, 0, s>>>((double2*)matrices, n);
  AMA_CHECK_LAUNCH();
  int flag = 0;
  AMA_CUDA_TRY(cudaMemcpyAsync(&flag, g_solver.info + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  AMA_CUDA_TRY(cudaStreamSynchronize(s));
  AMA_REQUIRE(flag == 0, AMA_ERR_NOT_SPD, "Cholesky factorisation met a non-positive pivot");
  return AMA_OK;
}

// ============================================ batched small Hermitian eigensolver
// One CTA per matrix: cyclic Jacobi with the round-robin (circle) ordering, n/2 disjoint
// rotations per round, all of A and V in shared memory (n <= kJacobiMaxN). Each rotation
// is the phase rotation diag(1, e^{-i phi}) that makes A_pq real, followed by the real
// Jacobi rotation that zeroes it. Sweeps stop when the off-diagonal Frobenius norm falls
// below 1e-15 of the total (at most kJacobiMaxSweeps). Eigenvalues are returned ascending,
// eigenvectors as columns (row-major), matching ama_heev.
namespace {
constexpr int kJacobiMaxN = 80;
constexpr int kJacobiMaxSweeps = 40;
constexpr int kJacobiThreads = 256;

__device__ __forceinline__ double2 cmuld(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__global__ void __launch_bounds__(kJacobiThreads) jacobi_heev_kernel(double2* mats, double* evals, int n) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int np = n + (n & 1);  // padded to even; the dummy index never rotates
  double2* A = reinterpret_cast<double2*>(smem_raw);  // [n][n]
  double2* V = A + n * n;                             // [n][n]
  double* rc = reinterpret_cast<double*>(V + n * n);  // [np/2] cos
  double* rs = rc + np / 2;                           // [np/2] sin
  double2* ph = reinterpret_cast<double2*>(rs + np / 2);  // [np/2] e^{i phi}
  int* pp = reinterpret_cast<int*>(ph + np / 2);          // [np/2]
  int* qq = pp + np / 2;                                  // [np/2]
  __shared__ double red[32];
  __shared__ int done_flag;
  double2* M = mats + (int64_t)blockIdx.x * n * n;
  for (int e = threadIdx.x; e < n * n; e += kJacobiThreads) {
    A[e] = M[e];
    V[e] = make_double2((e / n) == (e % n) ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  const int half = np / 2;
  for (int sweep = 0; sweep < kJacobiMaxSweeps; ++sweep) {
    // convergence: off-diagonal vs total Frobenius norm
    double off = 0.0, tot = 0.0;
    for (int e = threadIdx.x; e < n * n; e += kJacobiThreads) {
      const double2 a = A[e];
      const double m2 = a.x * a.x + a.y * a.y;
      tot += m2;
      if (e / n != e % n) off += m2;
    }
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      tot += __shfl_xor_sync(0xffffffffu, tot, o);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = off;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < kJacobiThreads / 32; ++w) s += red[w];
      red[31] = s;
    }
    __syncthreads();
    const double off_sum = red[31];
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = tot;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < kJacobiThreads / 32; ++w) s += red[w];
      done_flag = off_sum <= 1e-30 * s || s == 0.0;
    }
    __syncthreads();
    if (done_flag) break;
    for (int round = 0; round < np - 1; ++round) {
      // circle method: index np-1 fixed, the others rotate
      for (int t = threadIdx.x; t < half; t += kJacobiThreads) {
        int a, b;
        if (t == 0) {
          a = np - 1;
          b = round;
        } else {
          a = (round + t) % (np - 1);
          b = (round - t + (np - 1)) % (np - 1);
        }
        const int p = min(a, b), q = max(a, b);
        pp[t] = p;
        qq[t] = q;
        double c = 1.0, s = 0.0;
        double2 e = make_double2(1.0, 0.0);
        if (q < n) {
          const double2 apq = A[p * n + q];
          const double mag = sqrt(apq.x * apq.x + apq.y * apq.y);
          if (mag > 0.0) {
            e = make_double2(apq.x / mag, apq.y / mag);
            const double zeta = (A[q * n + q].x - A[p * n + p].x) / (2.0 * mag);
            const double tt = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            c = 1.0 / sqrt(1.0 + tt * tt);
            s = tt * c;
          }
        }
        rc[t] = c;
        rs[t] = s;
        ph[t] = e;
      }
      __syncthreads();
      // rows: A[p][:] <- c A[p][:] - s e A[q][:],  A[q][:] <- s A[p][:] + c e A[q][:]
      for (int w = threadIdx.x; w < half * n; w += kJacobiThreads) {
        const int t = w / n, j = w % n;
        const int p = pp[t], q = qq[t];
        if (q >= n || rs[t] == 0.0) continue;
        const double c = rc[t], s = rs[t];
        const double2 e = ph[t];
        const double2 ap = A[p * n + j], aq = cmuld(e, A[q * n + j]);
        A[p * n + j] = make_double2(c * ap.x - s * aq.x, c * ap.y - s * aq.y);
        A[q * n + j] = make_double2(s * ap.x + c * aq.x, s * ap.y + c * aq.y);
      }
      __syncthreads();
      // columns of A and V: X[:][p] <- c X[:][p] - s e* X[:][q],  X[:][q] <- s X[:][p] + c e* X[:][q]
      for (int w = threadIdx.x; w < half * n; w += kJacobiThreads) {
        const int t = w / n, i = w % n;
        const int p = pp[t], q = qq[t];
        if (q >= n || rs[t] == 0.0) continue;
        const double c = rc[t], s = rs[t];
        const double2 ec = make_double2(ph[t].x, -ph[t].y);
        double2 xp = A[i * n + p], xq = cmuld(ec, A[i * n + q]);
        A[i * n + p] = make_double2(c * xp.x - s * xq.x, c * xp.y - s * xq.y);
        A[i * n + q] = make_double2(s * xp.x + c * xq.x, s * xp.y + c * xq.y);
        xp = V[i * n + p];
        xq = cmuld(ec, V[i * n + q]);
        V[i * n + p] = make_double2(c * xp.x - s * xq.x, c * xp.y - s * xq.y);
        V[i * n + q] = make_double2(s * xp.x + c * xq.x, s * xp.y + c * xq.y);
      }
      __syncthreads();
    }
  }
  // sort eigenvalues ascending (rank by counting; ties broken by index) and write out
  double* w = evals + (int64_t)blockIdx.x * n;
  for (int j = threadIdx.x; j < n; j += kJacobiThreads) {
    const double dj = A[j * n + j].x;
    int rank = 0;
    for (int k = 0; k < n; ++k) {
      const double dk = A[k * n + k].x;
      rank += (dk < dj) || (dk == dj && k < j);
    }
    w[rank] = dj;
    for (int i = 0; i < n; ++i) M[(int64_t)i * n + rank] = V[i * n + j];
  }
}
}  // namespace

extern "C" int ama_heev_small(int32_t n, void* matrices, double* eigenvalues, int32_t batch, void* stream) {
  AMA_REQUIRE(matrices && eigenvalues, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(n >= 1 && n <= kJacobiMaxN && batch >= 1, AMA_ERR_SHAPE,
              "ama_heev_small: order must be 1.." + std::to_string(kJacobiMaxN));
  const int np = n + (n & 1);
  const size_t smem = (size_t)2 * n * n * sizeof(double2) + (size_t)(np / 2) * (2 * sizeof(double) + sizeof(double2) +
                                                                          2 * sizeof(int));
  AMA_CUDA_TRY(cudaFuncSetAttribute(jacobi_heev_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  jacobi_heev_kernel<<<batch, kJacobiThreads, smem, (cudaStream_t)stream>>>((double2*)matrices, eigenvalues, n);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}
