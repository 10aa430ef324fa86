// Batched small Hermitian eigensolver (cyclic Jacobi in shared memory) for the per-k-point
// Rayleigh-Ritz problems of the batched Davidson. The dense solver for large orders and the
// inverse Cholesky factor are in hermitian.cu.
#include "common.cuh"

#include <algorithm>

using namespace ama;

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
