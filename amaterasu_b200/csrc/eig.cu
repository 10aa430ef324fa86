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
