// Small in-register DFT codelets and the two shared-memory passes that build a
// length-n transform (n = A*B) out of them.
//
// A length-n transform is split "four-step" style and done in place in shared memory:
//
//   natural input -> position p = c*B + d holds X[c + A*d]   (either sign):
//     strided pass: for each b < B, DFT_A over x[a*B + b], times w_n^{S b c}, stored back
//     contiguous pass: for each c < A, DFT_B over the B contiguous values at c*B
//   input in that permuted order -> natural output            (either sign):
//     contiguous pass: for each c < A, DFT_B over c*B + d, times w_n^{S c e}, stored back
//     strided pass: for each e < B, DFT_A over c*B + e, stored back (natural order)
// The H.psi path uses the first form backward (G -> r) and the second forward (r -> G);
// the grid filters (Hartree, Kerker) use the first form forward and the second backward.
//
// Every task reads its elements and writes results to exactly the same positions, so no
// second buffer is needed. The real-space grid is therefore kept in a permuted order on
// each axis; the engine permutes V(r) the same way once per potential.
#pragma once
#include "common.cuh"
#include "twiddles.h"

namespace ama {

// Every FFT-stage kernel runs with this many threads per CTA; the passes stride by it.
constexpr int kFftThreads = 256;

// ---------------------------------------------------------------- codelets
// In-register DFT of length R with sign S (+1 backward, -1 forward), natural order in
// and out. Odd lengths use the symmetric pair form; even lengths split radix-2.
template <int R, int S, typename C>
__device__ __forceinline__ void dft_reg(C (&v)[R]);

template <int R, int S, typename C>
__device__ __forceinline__ void dft_odd(C (&v)[R]) {
  using T = decltype(v[0].x);
  constexpr int H = (R - 1) / 2;
  C a[H + 1], b[H + 1];
  static_for<H>([&](auto jj) {
    constexpr int j = decltype(jj)::value + 1;
    a[j] = cadd(v[j], v[R - j]);
    b[j] = csub(v[j], v[R - j]);
  });
  C x0 = v[0];
  C sum = x0;
  static_for<H>([&](auto jj) { constexpr int j = decltype(jj)::value + 1; sum = cadd(sum, a[j]); });
  v[0] = sum;
  static_for<H>([&](auto kk) {
    constexpr int k = decltype(kk)::value + 1;
    T ar = x0.x, ai = x0.y, br = T(0), bi = T(0);
    static_for<H>([&](auto jj) {
      constexpr int j = decltype(jj)::value + 1;
      constexpr int idx = (j * k) % R;
      constexpr T c = (T)kCos[R][idx];
      constexpr T s = (T)kSin[R][idx];
      ar += a[j].x * c;
      ai += a[j].y * c;
      br += b[j].y * s;
      bi += b[j].x * s;
    });
    if constexpr (S > 0) {
      v[k].x = ar - br; v[k].y = ai + bi;
      v[R - k].x = ar + br; v[R - k].y = ai - bi;
    } else {
      v[k].x = ar + br; v[k].y = ai - bi;
      v[R - k].x = ar - br; v[R - k].y = ai + bi;
    }
  });
}

template <int R, int S, typename C>
__device__ __forceinline__ void dft_even(C (&v)[R]) {
  using T = decltype(v[0].x);
  constexpr int M = R / 2;
  C e[M], o[M];
  static_for<M>([&](auto ii) {
    constexpr int i = decltype(ii)::value;
    e[i] = v[2 * i];
    o[i] = v[2 * i + 1];
  });
  dft_reg<M, S>(e);
  dft_reg<M, S>(o);
  static_for<M>([&](auto kk) {
    constexpr int k = decltype(kk)::value;
    C t;
    if constexpr (k == 0) {
      t = o[k];
    } else if constexpr (4 * k == R) {  // w = (0, S)
      t.x = -T(S) * o[k].y;
      t.y = T(S) * o[k].x;
    } else {
      constexpr T c = (T)kCos[R][k];
      constexpr T s = (T)(S * kSin[R][k]);
      t.x = o[k].x * c - o[k].y * s;
      t.y = o[k].x * s + o[k].y * c;
    }
    v[k] = cadd(e[k], t);
    v[k + M] = csub(e[k], t);
  });
}

template <int R, int S, typename C>
__device__ __forceinline__ void dft_reg(C (&v)[R]) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R % 2 == 0) {
    dft_even<R, S>(v);
  } else {
    dft_odd<R, S>(v);
  }
}

// ------------------------------------------------------ sparse-input codelets
// DFT of length R (sign S, natural order) whose inputs outside MASK (bit j set: v[j] may be
// nonzero) are zero: the arithmetic on the zero inputs is skipped; the zero entries of v are
// not read. Same transform as dft_reg, with the additions in the same order minus the zero
// terms.
template <int R, int S, uint32_t MASK, typename C>
__device__ __forceinline__ void dft_reg_sparse(C (&v)[R]);

template <int R, int S, uint32_t MASK, typename C>
__device__ __forceinline__ void dft_odd_sparse(C (&v)[R]) {
  using T = decltype(v[0].x);
  constexpr int H = (R - 1) / 2;
  constexpr bool in0 = (MASK & 1u) != 0;
  C a[H + 1], b[H + 1];
  static_for<H>([&](auto jj) {
    constexpr int j = decltype(jj)::value + 1;
    constexpr bool p = (MASK >> j) & 1u, q = (MASK >> (R - j)) & 1u;
    if constexpr (p && q) {
      a[j] = cadd(v[j], v[R - j]);
      b[j] = csub(v[j], v[R - j]);
    } else if constexpr (p) {
      a[j] = v[j];
      b[j] = v[j];
    } else if constexpr (q) {
      a[j] = v[R - j];
      b[j] = mk<C>(-v[R - j].x, -v[R - j].y);
    }
  });
  const C x0 = in0 ? v[0] : mk<C>(0, 0);
  C sum = x0;
  static_for<H>([&](auto jj) {
    constexpr int j = decltype(jj)::value + 1;
    if constexpr (((MASK >> j) & 1u) || ((MASK >> (R - j)) & 1u)) sum = cadd(sum, a[j]);
  });
  v[0] = sum;
  static_for<H>([&](auto kk) {
    constexpr int k = decltype(kk)::value + 1;
    T ar = x0.x, ai = x0.y, br = T(0), bi = T(0);
    static_for<H>([&](auto jj) {
      constexpr int j = decltype(jj)::value + 1;
      if constexpr (((MASK >> j) & 1u) || ((MASK >> (R - j)) & 1u)) {
        constexpr int idx = (j * k) % R;
        constexpr T c = (T)kCos[R][idx];
        constexpr T s = (T)kSin[R][idx];
        ar += a[j].x * c;
        ai += a[j].y * c;
        br += b[j].y * s;
        bi += b[j].x * s;
      }
    });
    if constexpr (S > 0) {
      v[k].x = ar - br; v[k].y = ai + bi;
      v[R - k].x = ar + br; v[R - k].y = ai - bi;
    } else {
      v[k].x = ar + br; v[k].y = ai - bi;
      v[R - k].x = ar - br; v[R - k].y = ai + bi;
    }
  });
}

template <int M>
constexpr uint32_t sparse_half_mask(uint32_t mask, int parity) {
  uint32_t out = 0;
  for (int i = 0; i < M; ++i)
    if ((mask >> (2 * i + parity)) & 1u) out |= 1u << i;
  return out;
}

template <int R, int S, uint32_t MASK, typename C>
__device__ __forceinline__ void dft_even_sparse(C (&v)[R]) {
  using T = decltype(v[0].x);
  constexpr int M = R / 2;
  constexpr uint32_t EM = sparse_half_mask<M>(MASK, 0), OM = sparse_half_mask<M>(MASK, 1);
  C e[M], o[M];
  static_for<M>([&](auto ii) {
    constexpr int i = decltype(ii)::value;
    if constexpr ((EM >> i) & 1u) e[i] = v[2 * i];
    if constexpr ((OM >> i) & 1u) o[i] = v[2 * i + 1];
  });
  if constexpr (EM != 0) dft_reg_sparse<M, S, EM>(e);
  if constexpr (OM != 0) dft_reg_sparse<M, S, OM>(o);
  static_for<M>([&](auto kk) {
    constexpr int k = decltype(kk)::value;
    if constexpr (OM == 0) {
      v[k] = e[k];
      v[k + M] = e[k];
    } else {
      C t;
      if constexpr (k == 0) {
        t = o[k];
      } else if constexpr (4 * k == R) {
        t.x = -T(S) * o[k].y;
        t.y = T(S) * o[k].x;
      } else {
        constexpr T c = (T)kCos[R][k];
        constexpr T s = (T)(S * kSin[R][k]);
        t.x = o[k].x * c - o[k].y * s;
        t.y = o[k].x * s + o[k].y * c;
      }
      if constexpr (EM == 0) {
        v[k] = t;
        v[k + M] = mk<C>(-t.x, -t.y);
      } else {
        v[k] = cadd(e[k], t);
        v[k + M] = csub(e[k], t);
      }
    }
  });
}

template <int R, int S, uint32_t MASK, typename C>
__device__ __forceinline__ void dft_reg_sparse(C (&v)[R]) {
  constexpr uint32_t full = (R >= 32) ? 0xffffffffu : ((1u << R) - 1u);
  if constexpr ((MASK & full) == full) {
    dft_reg<R, S>(v);
  } else if constexpr ((MASK & full) == 0) {
    static_for<R>([&](auto kk) { v[decltype(kk)::value] = mk<C>(0, 0); });
  } else if constexpr (R == 2) {
    if constexpr (MASK & 1u) {
      v[1] = v[0];
    } else {
      v[0] = v[1];
      v[1] = mk<C>(-v[1].x, -v[1].y);
    }
  } else if constexpr (R % 2 == 0) {
    dft_even_sparse<R, S, MASK>(v);
  } else {
    dft_odd_sparse<R, S, MASK>(v);
  }
}

// ------------------------------------------------------------- smem passes
// A "line" is n = A*B elements spaced `es` apart starting at `base`.
//
// Row mode: lines are rows of a [rows x n] smem array (es = 1), line list given.
// Column mode: lines are the `ncols` columns of a [n x ncols] array (es = ncols).
//
// strided pass (DFT of length RA over a*B + b for fixed b, B = n/RA):
//   twiddle (if TW) multiplies output index c by tw[(b*c) % n]  (tw already carries the
//   sign of the transform).
// contiguous pass (DFT of length RB over c*RB + d for fixed c):
//   twiddle (if TW) multiplies output index e by tw[(c*e) % n].

template <int RA, int S, bool TW, typename C>
__device__ __forceinline__ void strided_task(C* __restrict__ base, int es, int n, int b,
                                             const C* __restrict__ tw) {
  if constexpr (RA > 1) {
  const int B = n / RA;
  C v[RA];
#pragma unroll
  for (int a = 0; a < RA; ++a) v[a] = base[(a * B + b) * es];
  dft_reg<RA, S>(v);
  if constexpr (TW) {
    int idx = 0;  // (b * c) mod n, advanced without a division (b < n)
#pragma unroll
    for (int c = 1; c < RA; ++c) {
      idx += b;
      if (idx >= n) idx -= n;
      v[c] = cmul(v[c], tw[idx]);
    }
  }
#pragma unroll
  for (int c = 0; c < RA; ++c) base[(c * B + b) * es] = v[c];
  }
}

template <int RB, int S, bool TW, typename C>
__device__ __forceinline__ void contig_task(C* __restrict__ base, int es, int n, int c,
                                            const C* __restrict__ tw) {
  if constexpr (RB > 1) {
  C v[RB];
#pragma unroll
  for (int d = 0; d < RB; ++d) v[d] = base[(c * RB + d) * es];
  dft_reg<RB, S>(v);
  if constexpr (TW) {
    int idx = 0;  // (c * e) mod n
#pragma unroll
    for (int e = 1; e < RB; ++e) {
      idx += c;
      if (idx >= n) idx -= n;
      v[e] = cmul(v[e], tw[idx]);
    }
  }
#pragma unroll
  for (int d = 0; d < RB; ++d) base[(c * RB + d) * es] = v[d];
  }
}

// Column mode: consecutive threads take consecutive columns (conflict-free smem).
template <int RA, int S, bool TW, int NT = kFftThreads, typename C>
__device__ void strided_cols(C* sm, int n, int ncols, const C* tw) {
  const int B = n / RA;
  const int tasks = B * ncols;
  for (int t = threadIdx.x; t < tasks; t += NT) {
    const int col = t % ncols, b = t / ncols;
    strided_task<RA, S, TW>(sm + col, ncols, n, b, tw);
  }
}
template <int RB, int S, bool TW, int NT = kFftThreads, typename C>
__device__ void contig_cols(C* sm, int n, int ncols, const C* tw) {
  const int A = n / RB;
  const int tasks = A * ncols;
  for (int t = threadIdx.x; t < tasks; t += NT) {
    const int col = t % ncols, c = t / ncols;
    contig_task<RB, S, TW>(sm + col, ncols, n, c, tw);
  }
}
// Row mode over a list of row indices (rows have stride `ld`).
template <int RA, int S, bool TW, int NT = kFftThreads, typename C>
__device__ void strided_rows(C* sm, int n, int ld, const int* rows, int nrows, const C* tw) {
  const int B = n / RA;
  const int tasks = B * nrows;
  for (int t = threadIdx.x; t < tasks; t += NT) {
    const int b = t % B, r = rows[t / B];
    strided_task<RA, S, TW>(sm + r * ld, 1, n, b, tw);
  }
}
template <int RB, int S, bool TW, int NT = kFftThreads, typename C>
__device__ void contig_rows(C* sm, int n, int ld, const int* rows, int nrows, const C* tw) {
  const int A = n / RB;
  const int tasks = A * nrows;
  for (int t = threadIdx.x; t < tasks; t += NT) {
    const int c = t % A, r = rows[t / A];
    contig_task<RB, S, TW>(sm + r * ld, 1, n, c, tw);
  }
}

// The contiguous column pass writing its output to a global array with the same
// (n x ncols) layout instead of back to shared memory: the last pass of a natural-in
// transform stores straight to HBM, and the plane copy from shared memory disappears.
template <int RB, int S, int NT = kFftThreads, typename C>
__device__ void contig_cols_to(const C* sm, C* __restrict__ g, int n, int ncols) {
  const int A = n / RB;
  const int tasks = A * ncols;
  for (int t = threadIdx.x; t < tasks; t += NT) {
    const int col = t % ncols, c = t / ncols;
    C v[RB];
#pragma unroll
    for (int d = 0; d < RB; ++d) v[d] = sm[(c * RB + d) * ncols + col];
    dft_reg<RB, S>(v);
#pragma unroll
    for (int d = 0; d < RB; ++d) g[(int64_t)(c * RB + d) * ncols + col] = v[d];
  }
}

// Supported codelet lengths (1..16 except 13); dispatch a runtime length to a template.
#define AMA_RADIX_CASES(X) \
  X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(14) X(15) X(16)

// Full 1D transform along columns or rows; A/B are the runtime split of n (n = A*B).
// NAT_IN (natural input, permuted output): strided(A, twiddle) then contiguous(B).
// Permuted input, natural output: contiguous(B, twiddle) then strided(A). The sign S
// only selects the codelet direction; `tw` must hold w_n^(S t). Each pass ends with a
// block barrier.
template <int S, bool NAT_IN = (S > 0), int NT = kFftThreads, typename C>
__device__ void dft_cols(C* sm, int n, int A, int B, int ncols, const C* tw) {
  if constexpr (NAT_IN) {
    switch (A) {
#define CASE(R) case R: strided_cols<R, S, true, NT>(sm, n, ncols, tw); break;
      AMA_RADIX_CASES(CASE)
#undef CASE
    }
    __syncthreads();
    switch (B) {
#define CASE(R) case R: contig_cols<R, S, false, NT>(sm, n, ncols, tw); break;
      AMA_RADIX_CASES(CASE)
#undef CASE
    }
    __syncthreads();
  } else {
    switch (B) {
#define CASE(R) case R: contig_cols<R, S, true, NT>(sm, n, ncols, tw); break;
      AMA_RADIX_CASES(CASE)
#undef CASE
    }
    __syncthreads();
    switch (A) {
#define CASE(R) case R: strided_cols<R, S, false, NT>(sm, n, ncols, tw); break;
      AMA_RADIX_CASES(CASE)
#undef CASE
    }
    __syncthreads();
  }
}

// dft_cols (natural in, permuted out) with the contiguous pass writing to the global
// plane `g` (same layout) instead of back to shared memory.
template <int S, int NT = kFftThreads, typename C>
__device__ void dft_cols_store(C* sm, C* __restrict__ g, int n, int A, int B, int ncols, const C* tw) {
  switch (A) {
#define CASE(R) case R: strided_cols<R, S, true, NT>(sm, n, ncols, tw); break;
    AMA_RADIX_CASES(CASE)
#undef CASE
  }
  __syncthreads();
  switch (B) {
#define CASE(R) case R: contig_cols_to<R, S, NT>(sm, g, n, ncols); break;
    AMA_RADIX_CASES(CASE)
#undef CASE
  }
}

template <int S, bool NAT_IN = (S > 0), int NT = kFftThreads, typename C>
__device__ void dft_rows(C* sm, int n, int A, int B, int ld, const int* rows, int nrows,
                         const C* tw) {
  if constexpr (NAT_IN) {
    switch (A) {
#define CASE(R) case R: strided_rows<R, S, true, NT>(sm, n, ld, rows, nrows, tw); break;
      AMA_RADIX_CASES(CASE)
#undef CASE
    }
    __syncthreads();
    switch (B) {
#define CASE(R) case R: contig_rows<R, S, false, NT>(sm, n, ld, rows, nrows, tw); break;
      AMA_RADIX_CASES(CASE)
#undef CASE
    }
    __syncthreads();
  } else {
    switch (B) {
#define CASE(R) case R: contig_rows<R, S, true, NT>(sm, n, ld, rows, nrows, tw); break;
      AMA_RADIX_CASES(CASE)
#undef CASE
    }
    __syncthreads();
    switch (A) {
#define CASE(R) case R: strided_rows<R, S, false, NT>(sm, n, ld, rows, nrows, tw); break;
      AMA_RADIX_CASES(CASE)
#undef CASE
    }
    __syncthreads();
  }
}

}  // namespace ama
