// Dense FP64 Hermitian eigensolver and inverse Cholesky factor for the Davidson subspace
// problems, written for sm_100a with no vendor solver library.
//
// Eigensolver (ama_heev, ama_heev_lowest), the classical tridiagonal route, restated for a
// GPU whose subspace matrices (n <= 2400, 92 MB at most; usually n <= 1760, 50 MB) stay
// resident in the 126 MB L2:
//   1. tridiag_kernel: Householder similarity transforms A <- H A H, H = I - tau u u^H, in ONE
//      cooperative launch (all CTAs resident). Each column costs one grid barrier: after the
//      barrier every CTA rebuilds the next reflector itself from the updated pivot row (same
//      thread layout, same reduction order, so all CTAs hold bit-identical copies in shared
//      memory), then updates its own rows of the trailing matrix and, in the same pass, forms
//      its rows of the next product p = tau A u. The reflectors are kept in the rows they
//      annihilated (upper part), the subdiagonal comes out complex.
//   2. tri_prep_kernel: the diagonal phase similarity D = diag(delta), delta_{j+1} =
//      delta_j e_j/|e_j| (a parallel prefix product of unit complex numbers), turns the
//      tridiagonal real symmetric; Gershgorin bounds.
//   3. bisect_kernel: eigenvalue k by Sturm counts (Givens' bisection, generalised to
//      65-section: the 32 lanes of a warp test 2 interior points each per step), the
//      tridiagonal staged in shared memory.
//   4. invit_kernel: eigenvectors of the real tridiagonal by inverse iteration (Wilkinson):
//      Gaussian elimination with partial pivoting of T - lambda I, a fixed pseudo-random start
//      vector, two solves, every eigenvalue on its own warp; only (near-)degenerate
//      eigenvalues, closer than 1e-12 ||T||, form a cluster handled by one warp, which
//      orthogonalises each new vector against the cluster's earlier ones after every solve.
//      Valence spectra are dense but rarely degenerate, so the work stays parallel.
//   5. backtransform_kernel: z = Q D y with Q = H_0 H_1 ..., the reflectors applied in blocks
//      of 32 in compact WY form (wy_factor_kernel builds the triangular factors) to a few
//      columns per CTA held in shared memory.
//   6. Two Newton-Schulz steps Z <- (3I - Z Z^H) Z / 2 on the FP64 tensor-core GEMM
//      restore orthonormality to working precision: inverse-iteration vectors of eigenvalues
//      a gap g apart overlap by ~1e-16 ||T|| / g, and removing that overlap mixes them by as
//      much, which moves their residuals by only ~1e-16 ||T||. A tiled transpose writes the
//      columns out.
// Nothing synchronises with the host: a barrier wait that runs out (it never should, every
// CTA of a cooperative launch is resident) is recorded in a per-device status word that
// ama_solver_status reads.
//
// Inverse Cholesky factor (ama_potrf_inv): one CTA per matrix, right-looking column
// Cholesky in place, then the columns of L^{-1} from the right, every row in parallel.
#include "common.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cfloat>
#include <vector>

using namespace ama;

namespace {

constexpr int kTriT = 512;
constexpr int kTriW = kTriT / 32;
constexpr int kTriChunk = 8;                    // columns per lane per pass (x 2 rows in flight)
constexpr long long kBarrierSpin = 1ll << 24;  // polls (each an L2 round trip): ~1-2 s
constexpr int kMaxOrder = 2400;                 // shared memory: 4 n complex (tridiagonal and back)
// Eigenvalues closer than kClusterTol ||T|| are treated as one cluster (vectors orthogonalised
// in sequence); every other vector is computed on its own and the whole set is polished by
// Newton-Schulz afterwards. Bisection fixes each eigenvalue to ~4e-16 ||T||, so two inverse
// iterations separate eigenvalues 1e-12 ||T|| apart by a factor (1e-12/4e-16)^2 ~ 1e7.
constexpr double kClusterTol = 1e-12;
constexpr int kPts = 2;                         // Sturm points per lane in a multisection step
constexpr int kSections = 32 * kPts + 1;        // 64 interior points per step
constexpr int kBackCols = 4;                    // columns per CTA in the back-transformation
constexpr int kBackT = 512;

struct SolverCtl {
  unsigned count;
  unsigned gen;
  int err;   // 1: a grid-barrier wait ran out
  int pad;
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_acquire_s32(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Barrier over all CTAs of a cooperative launch; false when the kernel must stop (a wait ran
// out here or in another CTA). Every wait is bounded.
__device__ bool grid_barrier(SolverCtl* ctl, int* s_flag) {
  __syncthreads();  // the CTA's writes happen before thread 0's fence (fences are cumulative)
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned g = ld_acquire_u32(&ctl->gen);
    const unsigned arrived = atomicAdd(&ctl->count, 1u);
    int ok = 1;
    if (arrived == gridDim.x - 1) {
      atomicExch(&ctl->count, 0u);
      __threadfence();
      atomicAdd(&ctl->gen, 1u);
    } else {
      long long spin = 0;
      while (ld_acquire_u32(&ctl->gen) == g) {
        if (ld_acquire_s32(&ctl->err) != 0) { ok = 0; break; }
        if (++spin > kBarrierSpin) { atomicExch(&ctl->err, 1); ok = 0; break; }
      }
    }
    if (ld_acquire_s32(&ctl->err) != 0) ok = 0;
    *s_flag = ok;
  }
  __syncthreads();
  return *s_flag != 0;
}

__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cfma(double2 acc, double2 a, double2 b) {  // acc + a b
  acc.x = fma(a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y); acc.y = fma(a.y, b.x, acc.y);
  return acc;
}
__device__ __forceinline__ double2 cfma_conj(double2 acc, double2 a, double2 b) {  // acc + conj(a) b
  acc.x = fma(a.x, b.x, acc.x); acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y); acc.y = fma(-a.y, b.x, acc.y);
  return acc;
}
// a - x conj(y) - z conj(v): one entry of the rank-2 update A - u w^H - w u^H
__device__ __forceinline__ double2 rank2(double2 a, double2 x, double2 y, double2 z, double2 v) {
  a.x -= x.x * y.x + x.y * y.y; a.y -= x.y * y.x - x.x * y.y;
  a.x -= z.x * v.x + z.y * v.y; a.y -= z.y * v.x - z.x * v.y;
  return a;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum (fixed order); red needs NT/32 + 1 doubles.
template <int NT>
__device__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < NT / 32; ++w) t += red[w];
    red[NT / 32] = t;
  }
  __syncthreads();
  const double t = red[NT / 32];
  __syncthreads();
  return t;
}

// From x[0..len) (already in shared memory as u) and |x|^2: turn u into the Householder
// vector u = x + e^{i arg x0} |x| e_0 with tau = 1/(|x| (|x| + |x0|)), so that
// (I - tau u u^H) x = -e^{i arg x0} |x| e_0. Returns tau; *sub = -e^{i arg x0} |x|.
__device__ double finish_reflector(double2* u, double xnorm2, double2* sub) {
  const double xn = sqrt(xnorm2);
  const double2 x0 = u[0];
  const double a0 = hypot(x0.x, x0.y);
  if (xn == 0.0) {
    *sub = make_double2(0.0, 0.0);
    return 0.0;
  }
  const double2 ph = a0 > 0.0 ? make_double2(x0.x / a0, x0.y / a0) : make_double2(1.0, 0.0);
  *sub = make_double2(-ph.x * xn, -ph.y * xn);
  __syncthreads();  // every thread has read u[0]
  if (threadIdx.x == 0) u[0] = make_double2(x0.x + ph.x * xn, x0.y + ph.y * xn);
  __syncthreads();
  return 1.0 / (xn * (xn + a0));
}

// ---------------------------------------------------------------- 1. tridiagonalisation
__global__ void __launch_bounds__(kTriT, 1)
tridiag_kernel(int n, double2* __restrict__ A, double* __restrict__ dg, double2* __restrict__ sub,
               double* __restrict__ taus, double2* __restrict__ pbuf, SolverCtl* ctl) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* u = reinterpret_cast<double2*>(smem_raw);  // reflector of this step (length s)
  double2* w = u + n;                                   // w = p - K u
  double2* un = w + n;                                  // next reflector
  double2* rw = un + n;                                 // pivot row o as read
  __shared__ double red[kTriW + 1];
  __shared__ double2 seg_part[kTriW][2];  // per-segment partial sums of the next p (two rows)
  __shared__ int s_flag;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gwarp = blockIdx.x * kTriW + warp, nwarps = gridDim.x * kTriW;
  const bool lead = blockIdx.x == 0 && tid == 0;

  if (n <= 2) {
    if (lead) {
      dg[0] = __ldcg(A).x;
      if (n == 2) {
        dg[1] = __ldcg(A + 3).x;
        sub[0] = __ldcg(A + 2);  // T[1][0] = A[1][0]
      }
    }
    return;
  }

  // reflector 0 from row 0: x = conj(A[0][1..n))
  double part = 0.0;
  for (int c = tid; c < n - 1; c += kTriT) {
    const double2 a = __ldcg(A + 1 + c);
    u[c] = cconj(a);
    part += a.x * a.x + a.y * a.y;
  }
  __syncthreads();
  double2 e;
  double tau = finish_reflector(u, block_sum<kTriT>(part, red), &e);
  if (lead) {
    dg[0] = __ldcg(A).x;
    sub[0] = e;
    taus[0] = tau;
  }
  // p_0 = tau A_t u_0 over the trailing rows 1..n-1 (buffer 0)
  for (int r = gwarp; r < n - 1; r += nwarps) {
    const double2* row = A + (int64_t)(1 + r) * n + 1;
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll 8
    for (int c = lane; c < n - 1; c += 32) acc = cfma(acc, __ldcg(row + c), u[c]);
    acc.x = warp_sum(acc.x);
    acc.y = warp_sum(acc.y);
    if (lane == 0) __stcg(pbuf + r, make_double2(tau * acc.x, tau * acc.y));
  }
  if (!grid_barrier(ctl, &s_flag)) return;

  for (int j = 0; j <= n - 3; ++j) {
    const int o = j + 1, s = n - o;
    const double2* p = pbuf + (j & 1) * n;
    double2* pn = pbuf + ((j + 1) & 1) * n;
    // (a) keep reflector j in row j (deferred until every CTA has finished reading row j)
    if (blockIdx.x == 0)
      for (int c = tid; c < s; c += kTriT) __stcg(A + (int64_t)j * n + o + c, u[c]);
    // (a') K = (tau/2) Re(u^H p), w = p - K u; the pivot row o is fetched in the same pass
    const double2* ro = A + (int64_t)o * n + o;
    part = 0.0;
#pragma unroll 4
    for (int i = tid; i < s; i += kTriT) {
      const double2 pi = __ldcg(p + i), ri = __ldcg(ro + i), ui = u[i];
      part += ui.x * pi.x + ui.y * pi.y;
      w[i] = pi;
      rw[i] = ri;
    }
    const double K = 0.5 * tau * block_sum<kTriT>(part, red);
    for (int i = tid; i < s; i += kTriT) {
      const double2 ui = u[i];
      w[i] = make_double2(w[i].x - K * ui.x, w[i].y - K * ui.y);
    }
    __syncthreads();
    // (b) the updated pivot row o gives the next reflector (or the last 2x2 block)
    const bool more = o <= n - 3;
    const double2 u0 = u[0], w0 = w[0];
    part = 0.0;
    for (int c = 1 + tid; c < s; c += kTriT) {
      const double2 a = rank2(rw[c], u0, w[c], w0, u[c]);
      un[c - 1] = cconj(a);
      part += a.x * a.x + a.y * a.y;
    }
    if (lead) dg[o] = rank2(rw[0], u0, w0, w0, u0).x;
    const double nrm2 = block_sum<kTriT>(part, red);
    double taun = 0.0;
    if (more) {
      taun = finish_reflector(un, nrm2, &e);
      if (lead) {
        sub[o] = e;
        taus[o] = taun;
      }
    } else if (lead) {
      sub[o] = un[0];  // T[n-1][n-2] = conj(A[n-2][n-1])
    }
    // (c) own rows o+1..n-1: rank-2 update, and their entries of the next p. Rows go in
    // pairs (the shared-memory vectors are read once for both) to CTAs round-robin; inside a
    // CTA the columns of a pair are split over several warps when the CTA has fewer pairs
    // than warps (partial sums combined in a fixed order), and every lane keeps
    // 2 x kTriChunk loads in flight: the pass is bound by L2 bandwidth, not latency.
    if (!more) {
      if (blockIdx.x == 0 && tid == 0)  // o = n-2: only the last diagonal entry is left
        dg[n - 1] = rank2(__ldcg(A + (int64_t)(n - 1) * n + (n - 1)), u[1], w[1], w[1], u[1]).x;
    } else {
      const double2 zero = make_double2(0.0, 0.0);
      const int pairs = s / 2;  // rows 1..s-1 -> pairs (1,2), (3,4), ...; the last may be single
      const int my_pairs = pairs > (int)blockIdx.x ? (pairs - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
      const int wpp = my_pairs >= kTriW ? 1 : kTriW / max(my_pairs, 1);  // warps per pair
      const int seg = ((s - 1 + wpp - 1) / wpp + 31) & ~31;                // columns per warp
      for (int item = warp; item < my_pairs * wpp; item += kTriW) {
        const int lp = item / wpp, sg = item % wpp;
        const int r0 = 1 + 2 * ((int)blockIdx.x + lp * (int)gridDim.x), r1 = r0 + 1;
        const bool two = r1 < s;
        double2* row0 = A + (int64_t)(o + r0) * n + o;
        double2* row1 = A + (int64_t)(o + (two ? r1 : r0)) * n + o;
        const double2 u0r = u[r0], w0r = w[r0];
        const double2 u1r = two ? u[r1] : zero, w1r = two ? w[r1] : zero;
        double2 acc0 = zero, acc1 = zero;
        const int c_end = min(s, 1 + (sg + 1) * seg);
        for (int cb = 1 + sg * seg; cb < c_end; cb += 32 * kTriChunk) {
          double2 a0[kTriChunk], a1[kTriChunk];
#pragma unroll
          for (int q = 0; q < kTriChunk; ++q) {
            const int c = cb + lane + 32 * q;
            a0[q] = c < c_end ? __ldcg(row0 + c) : zero;
            a1[q] = (two && c < c_end) ? __ldcg(row1 + c) : zero;
          }
#pragma unroll
          for (int q = 0; q < kTriChunk; ++q) {
            const int c = cb + lane + 32 * q;
            if (c < c_end) {
              const double2 wc = w[c], uc = u[c], vc = un[c - 1];
              const double2 b0 = rank2(a0[q], u0r, wc, w0r, uc);
              __stcg(row0 + c, b0);
              acc0 = cfma(acc0, b0, vc);
              if (two) {
                const double2 b1 = rank2(a1[q], u1r, wc, w1r, uc);
                __stcg(row1 + c, b1);
                acc1 = cfma(acc1, b1, vc);
              }
            }
          }
        }
        acc0.x = warp_sum(acc0.x);
        acc0.y = warp_sum(acc0.y);
        acc1.x = warp_sum(acc1.x);
        acc1.y = warp_sum(acc1.y);
        if (lane == 0) {
          if (wpp == 1) {
            __stcg(pn + (r0 - 1), make_double2(taun * acc0.x, taun * acc0.y));
            if (two) __stcg(pn + (r1 - 1), make_double2(taun * acc1.x, taun * acc1.y));
          } else {
            seg_part[item][0] = acc0;
            seg_part[item][1] = acc1;
          }
        }
      }
      if (wpp > 1) {  // combine the column segments of each pair in a fixed order
        __syncthreads();
        if (tid < 2 * my_pairs) {
          const int lp = tid >> 1, h = tid & 1;
          const int r = 1 + 2 * ((int)blockIdx.x + lp * (int)gridDim.x) + h;
          if (r < s) {
            double2 acc = zero;
            for (int sg = 0; sg < wpp; ++sg) {
              acc.x += seg_part[lp * wpp + sg][h].x;
              acc.y += seg_part[lp * wpp + sg][h].y;
            }
            __stcg(pn + (r - 1), make_double2(taun * acc.x, taun * acc.y));
          }
        }
      }
    }
    if (!grid_barrier(ctl, &s_flag)) return;
    double2* t = u; u = un; un = t;
    tau = taun;
  }
}

// ---------------------------------------------------------------- 2. phases and bounds
// misc[0] = lower Gershgorin bound, misc[1] = upper, misc[2] = ||T||_inf, misc[3] = pivmin
constexpr int kPrepT = 1024;

__global__ void __launch_bounds__(kPrepT)
tri_prep_kernel(int n, const double* __restrict__ dg, const double2* __restrict__ sub, double* __restrict__ f2,
                double* __restrict__ fabs_e, double2* __restrict__ delta, double* __restrict__ misc) {
  __shared__ double2 scan[kPrepT];
  const int tid = threadIdx.x;
  // unit phases of the subdiagonal, then a chunked prefix product
  const int chunk = (n + kPrepT - 1) / kPrepT;
  const int i0 = tid * chunk, i1 = min(n, i0 + chunk);
  double2 prod = make_double2(1.0, 0.0);
  for (int i = i0; i < i1; ++i) {
    delta[i] = prod;  // exclusive within the chunk
    if (i < n - 1) {
      const double2 e = sub[i];
      const double a = hypot(e.x, e.y);
      if (a > 0.0) prod = cmul(prod, make_double2(e.x / a, e.y / a));
    }
  }
  scan[tid] = prod;
  __syncthreads();
  for (int off = 1; off < kPrepT; off <<= 1) {  // inclusive Hillis-Steele scan of chunk products
    double2 v = scan[tid];
    if (tid >= off) v = cmul(scan[tid - off], v);
    __syncthreads();
    scan[tid] = v;
    __syncthreads();
  }
  const double2 before = tid > 0 ? scan[tid - 1] : make_double2(1.0, 0.0);
  for (int i = i0; i < i1; ++i) {
    double2 v = cmul(before, delta[i]);
    const double m = hypot(v.x, v.y);
    delta[i] = make_double2(v.x / m, v.y / m);
  }
  // |e|^2, Gershgorin interval, norm
  double lo = DBL_MAX, hi = -DBL_MAX, nrm = 0.0, fmax2 = 0.0;
  for (int i = tid; i < n; i += kPrepT) {
    const double fl = i > 0 ? hypot(sub[i - 1].x, sub[i - 1].y) : 0.0;
    const double fr = i < n - 1 ? hypot(sub[i].x, sub[i].y) : 0.0;
    if (i < n - 1) {
      f2[i] = fr * fr;
      fabs_e[i] = fr;
      fmax2 = fmax(fmax2, fr * fr);
    } else {
      fabs_e[i] = 0.0;
    }
    lo = fmin(lo, dg[i] - fl - fr);
    hi = fmax(hi, dg[i] + fl + fr);
    nrm = fmax(nrm, fabs(dg[i]) + fl + fr);
  }
  // max/min reductions (order-independent)
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    nrm = fmax(nrm, __shfl_xor_sync(0xffffffffu, nrm, o));
    fmax2 = fmax(fmax2, __shfl_xor_sync(0xffffffffu, fmax2, o));
  }
  __shared__ double r4[4][kPrepT / 32];
  if ((tid & 31) == 0) {
    r4[0][tid >> 5] = lo; r4[1][tid >> 5] = hi; r4[2][tid >> 5] = nrm; r4[3][tid >> 5] = fmax2;
  }
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < kPrepT / 32; ++w) {
      lo = fmin(lo, r4[0][w]); hi = fmax(hi, r4[1][w]); nrm = fmax(nrm, r4[2][w]); fmax2 = fmax(fmax2, r4[3][w]);
    }
    const double pad = 2.0 * DBL_EPSILON * fmax(nrm, DBL_MIN) * n;
    misc[0] = lo - pad;
    misc[1] = hi + pad;
    misc[2] = nrm;
    misc[3] = DBL_MIN * fmax(1.0, fmax2);
  }
}

// ---------------------------------------------------------------- 3. bisection
// Numbers of eigenvalues of T below each x[p] (Sturm sequences of the LDL^T pivots of
// T - x I), kPts interleaved recurrences so that their division latencies overlap.
__device__ __forceinline__ void sturm_counts(int n, const double* __restrict__ dg, const double* __restrict__ f2,
                                             const double (&x)[kPts], double pivmin, int (&cnt)[kPts]) {
  double q[kPts];
  const double d0 = dg[0];
#pragma unroll
  for (int p = 0; p < kPts; ++p) {
    q[p] = d0 - x[p];
    if (fabs(q[p]) < pivmin) q[p] = -pivmin;
    cnt[p] = q[p] < 0.0;
  }
  for (int i = 1; i < n; ++i) {
    const double d = dg[i], f = f2[i - 1];
#pragma unroll
    for (int p = 0; p < kPts; ++p) {
      q[p] = d - x[p] - f / q[p];
      if (fabs(q[p]) < pivmin) q[p] = -pivmin;
      cnt[p] += q[p] < 0.0;
    }
  }
}

constexpr int kBisT = 64;

// One warp per eigenvalue: each step tests 32 kPts interior points of the bracket [a, b]
// (count(a) <= k < count(b)) and keeps the sub-interval where the count passes k.
__global__ void __launch_bounds__(kBisT)
bisect_kernel(int n, int nvec, const double* __restrict__ dg_g, const double* __restrict__ f2_g,
              const double* __restrict__ misc, double* __restrict__ lam) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* dg = reinterpret_cast<double*>(smem_raw);  // [n]
  double* f2 = dg + n;                                // [n]
  for (int i = threadIdx.x; i < n; i += kBisT) {
    dg[i] = dg_g[i];
    f2[i] = i < n - 1 ? f2_g[i] : 0.0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int k = (blockIdx.x * kBisT + threadIdx.x) >> 5;
  if (k >= nvec) return;
  double a = misc[0], b = misc[1];
  const double tnorm = misc[2], pivmin = misc[3];
  for (int it = 0; it < 64; ++it) {
    const double width = b - a;
    if (width <= 2.0 * DBL_EPSILON * fmax(fmax(fabs(a), fabs(b)), 1e-3 * tnorm) + pivmin) break;
    double x[kPts];
    int c[kPts];
#pragma unroll
    for (int p = 0; p < kPts; ++p) x[p] = a + width * (double)(lane * kPts + p + 1) / (double)kSections;
    sturm_counts(n, dg, f2, x, pivmin, c);
    // counts grow with x: the first lane whose last point is above k holds the crossing
    const unsigned above = __ballot_sync(0xffffffffu, c[kPts - 1] > k);
    const double last = x[kPts - 1];
    const double prev_last = __shfl_up_sync(0xffffffffu, last, 1);
    double lo_here = lane == 0 ? a : prev_last, hi_here = last;
#pragma unroll
    for (int p = kPts - 1; p >= 0; --p)
      if (c[p] > k) {
        hi_here = x[p];
        lo_here = p > 0 ? x[p - 1] : (lane == 0 ? a : prev_last);
      }
    double na, nb;
    if (above == 0u) {
      na = __shfl_sync(0xffffffffu, last, 31);
      nb = b;
    } else {
      const int f = __ffs(above) - 1;
      na = __shfl_sync(0xffffffffu, lo_here, f);
      nb = __shfl_sync(0xffffffffu, hi_here, f);
    }
    if (!(na > a || nb < b)) break;  // no representable progress left
    a = na;
    b = nb;
  }
  if (lane == 0) lam[k] = 0.5 * (a + b);
}

// ---------------------------------------------------------------- 4. inverse iteration

__device__ __forceinline__ double start_entry(int m, int i) {
  // fixed pseudo-random start in [-1, 1): a 64-bit integer hash (splitmix64 finaliser)
  unsigned long long z = 0x9E3779B97F4A7C15ull * (unsigned long long)(m + 1) + (unsigned long long)i * 0xD1B54A32D192ED03ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// LU with partial pivoting of the tridiagonal T - lam I (rows: sub f, diag d - lam, super f),
// keeping the reciprocals of the pivots so that the solves need no division.
__device__ void tri_factor(int n, const double* __restrict__ dg, const double* __restrict__ fv, double lam,
                           double tiny, double* u1r, double* u2, double* u3, double* l, unsigned char* piv) {
  double ca = dg[0] - lam, cb = n > 1 ? fv[0] : 0.0;
  for (int i = 0; i < n - 1; ++i) {
    const double ci = fv[i], na = dg[i + 1] - lam, nbv = i + 1 < n - 1 ? fv[i + 1] : 0.0;
    if (fabs(ci) > fabs(ca)) {
      piv[i] = 1;
      const double r = 1.0 / ci;
      u1r[i] = r; u2[i] = na; u3[i] = nbv;
      const double m = ca * r;
      l[i] = m;
      ca = cb - m * na;
      cb = -m * nbv;
    } else {
      piv[i] = 0;
      if (fabs(ca) < tiny) ca = ca < 0.0 ? -tiny : tiny;
      const double r = 1.0 / ca;
      u1r[i] = r; u2[i] = cb; u3[i] = 0.0;
      const double m = ci * r;
      l[i] = m;
      ca = na - m * cb;
      cb = nbv;
    }
  }
  if (fabs(ca) < tiny) ca = ca < 0.0 ? -tiny : tiny;
  u1r[n - 1] = 1.0 / ca;
  u2[n - 1] = 0.0;  // the back substitution reads these (times zero): never leave them unset
  u3[n - 1] = 0.0;
  l[n - 1] = 0.0;
  piv[n - 1] = 0;
}

__device__ void tri_solve(int n, const double* u1r, const double* u2, const double* u3, const double* l,
                          const unsigned char* piv, double* y) {
  for (int i = 0; i < n - 1; ++i) {
    if (piv[i]) {
      const double t = y[i];
      y[i] = y[i + 1];
      y[i + 1] = t - l[i] * y[i + 1];
    } else {
      y[i + 1] -= l[i] * y[i];
    }
  }
  double z1 = 0.0, z2 = 0.0;  // y[i+1], y[i+2] of the back substitution
  for (int i = n - 1; i >= 0; --i) {
    const double zi = (y[i] - u2[i] * z1 - u3[i] * z2) * u1r[i];
    y[i] = zi;
    z2 = z1;
    z1 = zi;
  }
}

// One warp (one CTA) per eigenvalue index; the first index of each cluster does the whole
// cluster. The factorisation and the iterate live in shared memory (41 n bytes, so that
// three CTAs fit an SM): the recurrences are serial, every step must be a short-latency
// access.
// Y: column-contiguous eigenvectors of the real tridiagonal, Y[m * n + i].
__global__ void __launch_bounds__(32)
invit_kernel(int n, int nvec, const double* __restrict__ dg, const double* __restrict__ f2,
             const double* __restrict__ misc, const double* __restrict__ lam, double* __restrict__ fv,
             double* __restrict__ Y) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x;
  const int k = blockIdx.x;
  const double tnorm = misc[2];
  const double ortol = kClusterTol * tnorm;
  if (k > 0 && lam[k] - lam[k - 1] < ortol) return;  // not the first of its cluster
  int k1 = k + 1;
  while (k1 < nvec && lam[k1] - lam[k1 - 1] < ortol) ++k1;
  double* wk = reinterpret_cast<double*>(smem_raw);
  double *u1r = wk, *u2 = wk + n, *u3 = wk + 2 * n, *l = wk + 3 * n, *y = wk + 4 * n;
  unsigned char* piv = reinterpret_cast<unsigned char*>(wk + 5 * n);
  const double tiny = DBL_EPSILON * fmax(tnorm, DBL_MIN);
  const int solves = k1 - k > 1 ? 3 : 2;
  for (int m = k; m < k1; ++m) {
    if (lane == 0) tri_factor(n, dg, fv, lam[m], tiny, u1r, u2, u3, l, piv);
    for (int i = lane; i < n; i += 32) y[i] = start_entry(m, i);
    __syncwarp();
    for (int it = 0; it < solves; ++it) {
      double ss = 0.0;
      for (int i = lane; i < n; i += 32) ss += y[i] * y[i];
      ss = warp_sum(ss);
      const double inv = ss > 0.0 ? 1.0 / sqrt(ss) : 0.0;
      for (int i = lane; i < n; i += 32) y[i] *= inv;
      __syncwarp();
      if (lane == 0) tri_solve(n, u1r, u2, u3, l, piv, y);
      __syncwarp();
      for (int q = k; q < m; ++q) {  // Gram-Schmidt against the cluster's earlier vectors
        const double* yq = Y + (int64_t)q * n;
        double dot = 0.0;
        for (int i = lane; i < n; i += 32) dot += yq[i] * y[i];
        dot = warp_sum(dot);
        for (int i = lane; i < n; i += 32) y[i] -= dot * yq[i];
        __syncwarp();
      }
    }
    double ss = 0.0;
    for (int i = lane; i < n; i += 32) ss += y[i] * y[i];
    ss = warp_sum(ss);
    const double inv = ss > 0.0 ? 1.0 / sqrt(ss) : 0.0;
    double* ym = Y + (int64_t)m * n;
    for (int i = lane; i < n; i += 32) ym[i] = y[i] * inv;
    __syncwarp();
  }
  (void)f2;
}

__host__ __device__ constexpr size_t invit_smem(int n) { return (size_t)n * (5 * sizeof(double) + 1); }

// ---------------------------------------------------------------- 5. back-transformation
// Reflectors are applied in blocks of kWY in the compact WY form of Schreiber and Van Loan:
// H_{j0} ... H_{j0+b-1} = I - V T V^H, V = [v_j0 .. v_j0+b-1] (v_j zero above row j+1, u_j
// below, read from row j of A), T upper triangular.
constexpr int kWY = 32;

__global__ void __launch_bounds__(kBackT)
wy_factor_kernel(int n, const double2* __restrict__ A, const double* __restrict__ taus, double2* __restrict__ Tbuf) {
  __shared__ double2 G[kWY][kWY + 1];  // G[i][l] = v_i^H v_l, i < l
  __shared__ double2 T[kWY][kWY + 1];
  const int j0 = blockIdx.x * kWY;
  const int b = min(kWY, n - 2 - j0);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int pr = warp; pr < b * b; pr += kBackT / 32) {
    const int i = pr / b, l = pr % b;
    if (i >= l) continue;  // warp-uniform
    const double2* vi = A + (int64_t)(j0 + i) * n;
    const double2* vl = A + (int64_t)(j0 + l) * n;
    double2 acc = make_double2(0.0, 0.0);
    for (int row = j0 + l + 1 + lane; row < n; row += 32) acc = cfma_conj(acc, vi[row], vl[row]);
    acc.x = warp_sum(acc.x);
    acc.y = warp_sum(acc.y);
    if (lane == 0) G[i][l] = acc;
  }
  __syncthreads();
  if (warp == 0) {
    // T[i][i] = tau_i ; T[0:i, i] = -tau_i T[0:i, 0:i] G[0:i, i]  (lane k owns row k of T)
    for (int i = 0; i < b; ++i) {
      const double ti = taus[j0 + i];
      if (lane < i) {
        double2 acc = make_double2(0.0, 0.0);
        for (int m = lane; m < i; ++m) acc = cfma(acc, T[lane][m], G[m][i]);
        T[lane][i] = make_double2(-ti * acc.x, -ti * acc.y);
      } else if (lane == i) {
        T[i][i] = make_double2(ti, 0.0);
      }
      __syncwarp();
    }
  }
  __syncthreads();
  double2* out = Tbuf + (int64_t)blockIdx.x * kWY * kWY;
  for (int e = threadIdx.x; e < kWY * kWY; e += kBackT) {
    const int i = e / kWY, l = e % kWY;
    out[e] = (i < b && l < b && l >= i) ? T[i][l] : make_double2(0.0, 0.0);
  }
}

// Z[k][i] = (Q D y_k)_i for kBackCols columns per CTA held in shared memory; the reflector
// blocks are applied last to first, z <- z - V (T (V^H z)). V is streamed through shared
// memory kVRows rows at a time (coalesced loads, 8 per thread in flight), twice per block.
constexpr int kVRows = 128;

__host__ __device__ constexpr size_t back_smem(int n) {
  return (size_t)kBackCols * n * sizeof(double2) + (size_t)kWY * kVRows * sizeof(double2);
}

__device__ __forceinline__ void stage_v(int n, const double2* __restrict__ A, int j0, int b, int rc,
                                        double2* __restrict__ vs) {
  // vs[i][t] = v_{j0+i}[rc + t] (zero above the reflector's first row and past the end)
  for (int e = threadIdx.x; e < kWY * kVRows; e += kBackT) {
    const int i = e / kVRows, t = e % kVRows, row = rc + t;
    vs[e] = (i < b && row < n && row > j0 + i) ? __ldg(A + (int64_t)(j0 + i) * n + row) : make_double2(0.0, 0.0);
  }
}

__global__ void __launch_bounds__(kBackT)
backtransform_kernel(int n, int nvec, const double2* __restrict__ A, const double2* __restrict__ Tbuf,
                     const double2* __restrict__ delta, const double* __restrict__ Y, double2* __restrict__ Z) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* zc = reinterpret_cast<double2*>(smem_raw);  // [kBackCols][n]
  double2* vs = zc + (size_t)kBackCols * n;            // [kWY][kVRows]
  __shared__ double2 W[kWY][kBackCols];
  __shared__ double2 W2[kWY][kBackCols];
  __shared__ double2 Wp[kBackT / (kWY * kBackCols)][kWY][kBackCols];
  constexpr int kSplit = kBackT / (kWY * kBackCols);  // threads per W entry
  const int tid = threadIdx.x;
  const int k0 = blockIdx.x * kBackCols;
  for (int e = tid; e < kBackCols * n; e += kBackT) {
    const int c = e / n, i = e % n;
    const double yv = k0 + c < nvec ? Y[(int64_t)(k0 + c) * n + i] : 0.0;
    const double2 dl = delta[i];
    zc[e] = make_double2(dl.x * yv, dl.y * yv);
  }
  __syncthreads();
  // fixed roles: thread -> (reflector i, column c, slice h) for W; (row t, column c) for the update
  const int wi = tid / (kBackCols * kSplit), wc = (tid / kSplit) % kBackCols, wh = tid % kSplit;
  const int ut = tid / kBackCols, uc = tid % kBackCols;
  const int nref = n - 2;
  for (int J = (nref + kWY - 1) / kWY - 1; J >= 0; --J) {
    const int j0 = J * kWY, b = min(kWY, nref - j0);
    // W = V^H z, in row chunks
    double2 acc = make_double2(0.0, 0.0);
    for (int rc = j0 + 1; rc < n; rc += kVRows) {
      stage_v(n, A, j0, b, rc, vs);
      __syncthreads();
      for (int t = wh; t < kVRows; t += kSplit) {
        const int row = rc + t;
        if (row < n) acc = cfma_conj(acc, vs[wi * kVRows + t], zc[wc * n + row]);
      }
      __syncthreads();
    }
    Wp[wh][wi][wc] = acc;
    __syncthreads();
    if (tid < kWY * kBackCols) {
      const int i = tid / kBackCols, c = tid % kBackCols;
      double2 sum = make_double2(0.0, 0.0);
      for (int h = 0; h < kSplit; ++h) {
        sum.x += Wp[h][i][c].x;
        sum.y += Wp[h][i][c].y;
      }
      W[i][c] = sum;
    }
    __syncthreads();
    // W2 = T W
    const double2* Tj = Tbuf + (int64_t)J * kWY * kWY;
    if (tid < kWY * kBackCols) {
      const int i = tid / kBackCols, c = tid % kBackCols;
      double2 sum = make_double2(0.0, 0.0);
      for (int m = i; m < b; ++m) sum = cfma(sum, Tj[i * kWY + m], W[m][c]);
      W2[i][c] = sum;
    }
    __syncthreads();
    // z -= V W2, in row chunks
    for (int rc = j0 + 1; rc < n; rc += kVRows) {
      stage_v(n, A, j0, b, rc, vs);
      __syncthreads();
      for (int t = ut; t < kVRows; t += kBackT / kBackCols) {
        const int row = rc + t;
        if (row < n) {
          double2 sum = make_double2(0.0, 0.0);
          for (int i = 0; i < b; ++i) sum = cfma(sum, vs[i * kVRows + t], W2[i][uc]);
          double2 z = zc[uc * n + row];
          z.x -= sum.x;
          z.y -= sum.y;
          zc[uc * n + row] = z;
        }
      }
      __syncthreads();
    }
  }
  for (int e = tid; e < kBackCols * n; e += kBackT) {
    const int c = e / n;
    if (k0 + c < nvec) Z[(int64_t)(k0 + c) * n + (e % n)] = zc[e];
  }
}

// out[i][k] = Z[k][i] for k < nvec (row-major n x n output, columns 0..nvec-1)
__global__ void transpose_out_kernel(int n, int nvec, const double2* __restrict__ Z, double2* __restrict__ out) {
  __shared__ double2 tile[32][33];
  const int k0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int k = k0 + r, i = i0 + threadIdx.x;
    if (k < nvec && i < n) tile[r][threadIdx.x] = Z[(int64_t)k * n + i];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, k = k0 + threadIdx.x;
    if (k < nvec && i < n) out[(int64_t)i * n + k] = tile[threadIdx.x][r];
  }
}

// G <- (3 I - G) / 2
__global__ void ns_factor_kernel(int m, double2* __restrict__ G) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)m * m; e += (int64_t)gridDim.x * blockDim.x) {
    const double2 g = G[e];
    const bool diag = e / m == e % m;
    G[e] = make_double2((diag ? 3.0 : 0.0) * 0.5 - 0.5 * g.x, -0.5 * g.y);
  }
}

__global__ void copy_eigenvalues_kernel(int nvec, const double* __restrict__ lam, double* __restrict__ w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nvec; i += gridDim.x * blockDim.x) w[i] = lam[i];
}

__global__ void fold_status_kernel(const SolverCtl* ctl, int* status) {
  if (threadIdx.x == 0 && ctl->err != 0 && *status == 0) *status = ctl->err;
}

// ---------------------------------------------------------------- scratch (per device)
struct EigScratch {
  char* base = nullptr;
  size_t bytes = 0;
  int* status = nullptr;  // sticky device status word (0 fine, 1 a barrier wait ran out)
  int coop_blocks = 0;    // co-resident CTAs of tridiag_kernel at the largest shared memory
  int sms = 0;
};
thread_local PerDevice<EigScratch> g_eig;

struct EigLayout {
  SolverCtl* ctl;
  double *dg, *taus, *f2, *fv, *lam, *misc, *Y;
  double2 *sub, *delta, *pbuf, *Z, *Z2, *G, *Tbuf;
  size_t total;
};

EigLayout layout(char* base, int n, int nvec) {
  EigLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p = base + off;
    off += (bytes + 255) & ~size_t(255);
    return p;
  };
  L.ctl = (SolverCtl*)take(sizeof(SolverCtl));
  L.dg = (double*)take(sizeof(double) * n);
  L.taus = (double*)take(sizeof(double) * n);
  L.f2 = (double*)take(sizeof(double) * n);
  L.fv = (double*)take(sizeof(double) * n);
  L.lam = (double*)take(sizeof(double) * n);
  L.misc = (double*)take(sizeof(double) * 8);
  L.sub = (double2*)take(sizeof(double2) * n);
  L.delta = (double2*)take(sizeof(double2) * n);
  L.pbuf = (double2*)take(sizeof(double2) * 2 * n);
  L.Y = (double*)take(sizeof(double) * (size_t)n * nvec);
  L.Z = (double2*)take(sizeof(double2) * (size_t)n * nvec);
  L.Z2 = (double2*)take(sizeof(double2) * (size_t)n * nvec);
  L.G = (double2*)take(sizeof(double2) * (size_t)nvec * nvec);
  L.Tbuf = (double2*)take(sizeof(double2) * (size_t)((n + kWY - 1) / kWY) * kWY * kWY);
  L.total = off;
  return L;
}

int eig_scratch(int n, int nvec, EigScratch** out, EigLayout* L) {
  EigScratch* sc = g_eig.here();
  AMA_REQUIRE(sc, AMA_ERR_CUDA, "eigensolver: no usable current CUDA device");
  const size_t need = layout(nullptr, n, nvec).total;
  if (sc->bytes < need) {
    bump_memory_epoch();
    if (sc->base) cudaFree(sc->base);
    sc->base = nullptr;
    sc->bytes = 0;
    AMA_CUDA_TRY(cudaMalloc((void**)&sc->base, need));
    sc->bytes = need;
  }
  if (!sc->status) {
    bump_memory_epoch();
    AMA_CUDA_TRY(cudaMalloc((void**)&sc->status, sizeof(int)));
    AMA_CUDA_TRY(cudaMemset(sc->status, 0, sizeof(int)));
    int dev = 0;
    AMA_CUDA_TRY(cudaGetDevice(&dev));
    AMA_CUDA_TRY(cudaDeviceGetAttribute(&sc->sms, cudaDevAttrMultiProcessorCount, dev));
    const int smem = 4 * kMaxOrder * (int)sizeof(double2);
    AMA_CUDA_TRY(cudaFuncSetAttribute(tridiag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    AMA_CUDA_TRY(cudaFuncSetAttribute(backtransform_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)back_smem(kMaxOrder)));
    AMA_CUDA_TRY(cudaFuncSetAttribute(invit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)invit_smem(kMaxOrder)));
    int per_sm = 0;
    AMA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tridiag_kernel, kTriT, smem));
    sc->coop_blocks = per_sm * sc->sms;
  }
  *out = sc;
  *L = layout(sc->base, n, nvec);
  return AMA_OK;
}

int tridiag_ctas(int n, const EigScratch* sc) {
  const char* env = getenv("AMA_HEEV_CTAS");  // tuning override (may exceed one CTA per SM)
  int g = env ? atoi(env) : (n + 11) / 12;
  int cap = std::min(sc->coop_blocks, sc->sms);
  if (env) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tridiag_kernel, kTriT, 4 * n * sizeof(double2)) ==
        cudaSuccess)
      cap = std::max(cap, per_sm * sc->sms);
  }
  return std::max(1, std::min(g, cap));
}

int polish_orthonormal(int n, int nvec, double2* Z, double2* Z2, double2* G, cudaStream_t s);

int solve_one(int n, int nvec, double2* a, double* w, EigScratch* sc, const EigLayout& L, cudaStream_t s) {
  AMA_CUDA_TRY(cudaMemsetAsync(L.ctl, 0, sizeof(SolverCtl), s));
  int nn = n;
  int g = tridiag_ctas(n, sc);
  void* args[] = {&nn, &a, (void*)&L.dg, (void*)&L.sub, (void*)&L.taus, (void*)&L.pbuf, (void*)&L.ctl};
  const size_t smem = (size_t)4 * n * sizeof(double2);
  AMA_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)tridiag_kernel, dim3(g), dim3(kTriT), args, smem, s));
  tri_prep_kernel<<<1, kPrepT, 0, s>>>(n, L.dg, L.sub, L.f2, L.fv, L.delta, L.misc);
  bisect_kernel<<<(nvec * 32 + kBisT - 1) / kBisT, kBisT, 2 * n * sizeof(double), s>>>(n, nvec, L.dg, L.f2, L.misc,
                                                                                      L.lam);
  invit_kernel<<<nvec, 32, invit_smem(n), s>>>(n, nvec, L.dg, L.f2, L.misc, L.lam, L.fv, L.Y);
  if (n > 2) wy_factor_kernel<<<(n - 2 + kWY - 1) / kWY, kBackT, 0, s>>>(n, a, L.taus, L.Tbuf);
  backtransform_kernel<<<(nvec + kBackCols - 1) / kBackCols, kBackT, back_smem(n), s>>>(
      n, nvec, a, L.Tbuf, L.delta, L.Y, L.Z);
  AMA_CHECK_LAUNCH();
  if (int rc = polish_orthonormal(n, nvec, L.Z, L.Z2, L.G, s)) return rc;
  transpose_out_kernel<<<dim3((nvec + 31) / 32, (n + 31) / 32), dim3(32, 8), 0, s>>>(n, nvec, L.Z, a);
  copy_eigenvalues_kernel<<<(nvec + 255) / 256, 256, 0, s>>>(nvec, L.lam, w);
  fold_status_kernel<<<1, 32, 0, s>>>(L.ctl, sc->status);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

// Two Newton-Schulz steps on the rows of Z (nvec x n, row-major): G = Z Z^H, Z <- ((3I - G)/2) Z.
int polish_orthonormal(int n, int nvec, double2* Z, double2* Z2, double2* G, cudaStream_t s) {
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  for (int step = 0; step < 2; ++step) {
    double2* src = step == 0 ? Z : Z2;
    double2* dst = step == 0 ? Z2 : Z;
    if (int rc = ama_zgemm(AMA_C128, 1, nvec, nvec, n, one, src, n, 0, src, n, 0, zero, G, nvec, 0, 1, s)) return rc;
    ns_factor_kernel<<<std::max(1, std::min(1184, (nvec * nvec + 255) / 256)), 256, 0, s>>>(nvec, G);
    AMA_CHECK_LAUNCH();
    if (int rc = ama_zgemm(AMA_C128, 0, nvec, n, nvec, one, G, nvec, 0, src, n, 0, zero, dst, n, 0, 1, s)) return rc;
  }
  return AMA_OK;
}

int heev_impl(int32_t n, int32_t nvec, void* matrices, double* eigenvalues, int32_t batch, void* stream) {
  AMA_REQUIRE(matrices && eigenvalues, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(n >= 1 && batch >= 1 && nvec >= 1 && nvec <= n, AMA_ERR_SHAPE, "bad sizes");
  AMA_REQUIRE(n <= kMaxOrder, AMA_ERR_SHAPE,
              "Hermitian eigensolver: order " + std::to_string(n) + " above " + std::to_string(kMaxOrder));
  EigScratch* sc = nullptr;
  EigLayout L{};
  if (int rc = eig_scratch(n, nvec, &sc, &L)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  for (int b = 0; b < batch; ++b) {
    double2* a = (double2*)matrices + (int64_t)b * n * n;
    if (int rc = solve_one(n, nvec, a, eigenvalues + (int64_t)b * n, sc, L, s)) return rc;
  }
  return AMA_OK;
}

// ---------------------------------------------------------------- inverse Cholesky
// One CTA per matrix. Right-looking Cholesky A = L L^H (one warp per trailing row), then
// X = L^{-1} column by column from the right: X L = I gives, for i > j,
// X[i][j] = -(sum_{k=j+1..i} X[i][k] L[k][j]) / L[j][j], every row i independent (one warp
// per row); column j of X is staged in shared memory before it overwrites column j of L.
constexpr int kCholT = 1024;

__global__ void __launch_bounds__(kCholT) potrf_inv_kernel(int n, double2* __restrict__ mats, int* __restrict__ flag) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* col = reinterpret_cast<double2*>(smem_raw);  // [n]
  double2* A = mats + (int64_t)blockIdx.x * n * n;
  __shared__ double s_piv;
  __shared__ int s_bad;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int kWarps = kCholT / 32;
  if (tid == 0) s_bad = 0;
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    if (tid == 0) {
      const double a = A[(int64_t)j * n + j].x;
      if (!(a > 0.0)) s_bad = 1;
      s_piv = a > 0.0 ? sqrt(a) : 1.0;
    }
    __syncthreads();
    if (s_bad) break;
    const double ljj = s_piv, inv = 1.0 / ljj;
    for (int i = j + 1 + tid; i < n; i += kCholT) {
      const double2 v = A[(int64_t)i * n + j];
      A[(int64_t)i * n + j] = make_double2(v.x * inv, v.y * inv);
    }
    if (tid == 0) A[(int64_t)j * n + j] = make_double2(ljj, 0.0);
    __syncthreads();
    for (int i = j + 1 + warp; i < n; i += kWarps) {  // A[i][c] -= L[i][j] conj(L[c][j]), j < c <= i
      const double2 li = A[(int64_t)i * n + j];
      for (int c = j + 1 + lane; c <= i; c += 32) {
        const double2 lc = A[(int64_t)c * n + j];
        double2 v = A[(int64_t)i * n + c];
        v.x -= li.x * lc.x + li.y * lc.y;
        v.y -= li.y * lc.x - li.x * lc.y;
        A[(int64_t)i * n + c] = v;
      }
    }
    __syncthreads();
  }
  if (s_bad) {
    if (tid == 0) atomicExch(flag, 1);
    return;
  }
  for (int j = n - 1; j >= 0; --j) {
    const double xjj = 1.0 / A[(int64_t)j * n + j].x;
    for (int i = j + 1 + warp; i < n; i += kWarps) {
      double2 acc = make_double2(0.0, 0.0);
      for (int k = j + 1 + lane; k <= i; k += 32) acc = cfma(acc, A[(int64_t)i * n + k], A[(int64_t)k * n + j]);
      acc.x = warp_sum(acc.x);
      acc.y = warp_sum(acc.y);
      if (lane == 0) col[i] = make_double2(-acc.x * xjj, -acc.y * xjj);
    }
    __syncthreads();
    for (int i = j + 1 + tid; i < n; i += kCholT) A[(int64_t)i * n + j] = col[i];
    if (tid == 0) A[(int64_t)j * n + j] = make_double2(xjj, 0.0);
    __syncthreads();
  }
  for (int64_t e = tid; e < (int64_t)n * n; e += kCholT)
    if ((int)(e % n) > (int)(e / n)) A[e] = make_double2(0.0, 0.0);
}

struct CholScratch {
  int* flag = nullptr;
};
thread_local PerDevice<CholScratch> g_chol;

}  // namespace

extern "C" int ama_heev(int32_t n, void* matrices, double* eigenvalues, int32_t batch, void* stream) {
  return heev_impl(n, n, matrices, eigenvalues, batch, stream);
}

extern "C" int ama_heev_lowest(int32_t n, int32_t nvec, void* matrices, double* eigenvalues, int32_t batch,
                               void* stream) {
  return heev_impl(n, nvec, matrices, eigenvalues, batch, stream);
}

extern "C" int ama_solver_status(int32_t* code) {
  AMA_REQUIRE(code, AMA_ERR_ARG, "null argument");
  *code = 0;
  EigScratch* sc = g_eig.here();
  if (sc && sc->status) {
    AMA_CUDA_TRY(cudaMemcpy(code, sc->status, sizeof(int), cudaMemcpyDeviceToHost));
    AMA_CUDA_TRY(cudaMemset(sc->status, 0, sizeof(int)));
  }
  return AMA_OK;
}

extern "C" int ama_potrf_inv(int32_t n, void* matrices, int32_t batch, void* stream) {
  AMA_REQUIRE(matrices, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(n >= 1 && batch >= 1, AMA_ERR_SHAPE, "bad sizes");
  CholScratch* cs = g_chol.here();
  AMA_REQUIRE(cs, AMA_ERR_CUDA, "inverse Cholesky: no usable current CUDA device");
  if (!cs->flag) bump_memory_epoch();
  if (!cs->flag) AMA_CUDA_TRY(cudaMalloc((void**)&cs->flag, sizeof(int)));
  cudaStream_t s = (cudaStream_t)stream;
  AMA_CUDA_TRY(cudaMemsetAsync(cs->flag, 0, sizeof(int), s));
  const size_t smem = (size_t)n * sizeof(double2);
  AMA_REQUIRE(smem <= 200 * 1024, AMA_ERR_SHAPE, "inverse Cholesky: order above 12800");
  AMA_CUDA_TRY(cudaFuncSetAttribute(potrf_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  potrf_inv_kernel<<<batch, kCholT, smem, s>>>(n, (double2*)matrices, cs->flag);
  AMA_CHECK_LAUNCH();
  int flag = 0;
  AMA_CUDA_TRY(cudaMemcpyAsync(&flag, cs->flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  AMA_CUDA_TRY(cudaStreamSynchronize(s));
  AMA_REQUIRE(flag == 0, AMA_ERR_NOT_SPD, "Cholesky factorisation met a non-positive pivot");
  return AMA_OK;
}
