// The H.psi engine: sphere<->grid maps, the three fused FFT stages, the nonlocal
// projector products and the density accumulation.
//
// Layout in HBM
//   psi, hpsi      per k-point a row-major (nbands, npw_k) block, blocks back to back.
//   work           per band the x-planes that can hold sphere coefficients ("slots",
//                  2*h_max+1 of the n1 planes), each a full (n2, n3) plane:
//                  work[band][slot][y][z]. After stage A the plane is in real space along
//                  y and z, after stage B also along x and already multiplied by V.
//   V              per spin, real, in the permuted real-space order the in-place DFTs
//                  produce (see dft.cuh), pre-scaled by 1/N (the forward-transform norm).
//
// Stage A  (grid: slot x band)   scatter the slot's sphere points into a zeroed smem plane,
//                                backward DFT along z (only rows holding points), then y.
// Stage B  (grid: y x band)      gather the slots' rows at one y into an (n1, n3) smem slab,
//                                backward DFT along x, multiply by V, forward DFT along x,
//                                write the slot rows back.
// Stage C  (grid: slot x band)   forward DFT along y, then z (rows holding points), gather
//                                the sphere points and write T*psi + that into hpsi.
// The nonlocal term is added by two GEMMs: P = psi B^H (split-K), hpsi += P (D B).
#include "common.cuh"
#include "dft.cuh"
#include "gemm.cuh"
#include "engine_impl.cuh"
#include "twiddles_line.h"

#include <algorithm>
#include <cmath>
#include <atomic>
#include <map>
#include <numeric>
#include <vector>

namespace ama {

static bool split_length(int n, AxisPlan* out) {
  // n = A*B with A, B in the codelet set; minimise max(A, B), prefer A >= B.
  auto ok = [](int r) { return r >= 1 && r <= 16 && r != 13; };
  int best_a = -1, best_b = -1;
  for (int b = 1; b <= 16; ++b) {
    if (n % b) continue;
    int a = n / b;
    if (!ok(a) || !ok(b) || a < b) continue;
    if (best_a < 0 || std::max(a, b) < std::max(best_a, best_b)) { best_a = a; best_b = b; }
  }
  if (best_a < 0) return false;
  *out = {n, best_a, best_b};
  return true;
}


}  // namespace ama

namespace {

template <typename T> cudaError_t grow(void** ptr, size_t* have, size_t need) {
  if (*have >= need) return cudaSuccess;
  ama::bump_memory_epoch();
  if (*ptr) cudaFree(*ptr);
  *ptr = nullptr;
  *have = 0;
  cudaError_t e = cudaMalloc(ptr, need);
  if (e == cudaSuccess) *have = need;
  return e;
}

template <typename T> int upload(T** dst, const T* src, size_t count) {
  ama::bump_memory_epoch();
  AMA_CUDA_TRY(cudaMalloc((void**)dst, std::max<size_t>(count, 1) * sizeof(T)));
  if (count) AMA_CUDA_TRY(cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice));
  return AMA_OK;
}

// ------------------------------------------------------------------ kernels
struct HpsiView {
  int n1, n2, n3;
  int A1, B1, A2, B2, A3, B3;
  int nslots;
  const int* plane_x;
  const int* slot_of_x;
  const int2* entries;
  const int* entry_start;
  const int* rows;
  const int* row_start;
  const int64_t* pw_off;
  const int* npw;
  int k_first, nbands;
  int64_t plane_elems, band_elems;  // n2*n3, nslots*n2*n3
};

template <typename C>
__device__ __forceinline__ void load_twiddles(C* dst, const C* src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// Grid sizes: compile-time for the engine's common grids (all index arithmetic folds to
// constants), read from the view otherwise.
struct DynDims {
  static constexpr int zsplit = 1;
  template <class V> __device__ static __forceinline__ int n1(const V& v) { return v.n1; }
  template <class V> __device__ static __forceinline__ int a1(const V& v) { return v.A1; }
  template <class V> __device__ static __forceinline__ int n2(const V& v) { return v.n2; }
  template <class V> __device__ static __forceinline__ int a2(const V& v) { return v.A2; }
  template <class V> __device__ static __forceinline__ int n3(const V& v) { return v.n3; }
  template <class V> __device__ static __forceinline__ int a3(const V& v) { return v.A3; }
};
template <int N1, int A1, int N2, int A2, int N3, int A3, int ZS = 1> struct FixDims {
  static constexpr int n3c() { return N3; }
  // stage B may split each (x, z) slab into ZS parts along z (less shared memory per CTA,
  // more CTAs per SM); one part by default, the split is an autotuned variant
  static constexpr int zsplit = ZS;
  template <class V> __device__ static constexpr int n1(const V&) { return N1; }
  template <class V> __device__ static constexpr int a1(const V&) { return A1; }
  template <class V> __device__ static constexpr int n2(const V&) { return N2; }
  template <class V> __device__ static constexpr int a2(const V&) { return A2; }
  template <class V> __device__ static constexpr int n3(const V&) { return N3; }
  template <class V> __device__ static constexpr int a3(const V&) { return A3; }
};

#define AMA_DIMS(D, v)                                                    \
  const int n1 = D::n1(v), A1 = D::a1(v), B1 = n1 / A1;                   \
  const int n2 = D::n2(v), A2 = D::a2(v), B2 = n2 / A2;                   \
  const int n3 = D::n3(v), A3 = D::a3(v), B3 = n3 / A3;                   \
  const int plane = n2 * n3;                                              \
  (void)B1; (void)B2; (void)B3; (void)A1; (void)A2; (void)A3; (void)plane;

template <typename C>
__device__ __forceinline__ void load_tw(C* dst, const C* src, int n) {
  for (int i = threadIdx.x; i < n; i += kFftThreads) dst[i] = src[i];
}

// Asynchronous global -> shared copy of n contiguous complex elements (cp.async): every
// thread issues all of its copies before any completes, so a whole plane is in flight at
// once. 16-byte copies when both ends are 16-byte aligned and the size is a multiple of 16,
// else one copy per element. Completed by async_copy_wait().
template <typename C>
__device__ __forceinline__ void async_copy(C* dst, const C* src, int n) {
  const uint32_t sdst = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  const size_t bytes = (size_t)n * sizeof(C);
  if (((reinterpret_cast<uintptr_t>(src) | sdst) & 15) == 0 && (bytes & 15) == 0) {
    const char* g = reinterpret_cast<const char*>(src);
    for (int i = threadIdx.x; i < (int)(bytes >> 4); i += kFftThreads)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sdst + 16 * i), "l"(g + 16 * i) : "memory");
  } else {
    for (int i = threadIdx.x; i < n; i += kFftThreads) {
      if constexpr (sizeof(C) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sdst + 16 * i), "l"(src + i) : "memory");
      else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sdst + 8 * i), "l"(src + i) : "memory");
    }
  }
}

__device__ __forceinline__ void async_copy_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Zero the (n2, n3) slot plane, load the list of its rows that hold sphere points, and
// scatter the band's coefficients into it (four entries per thread in flight: the psi load
// depends on the entry load). NT threads; ends with a barrier. Returns the row count.
template <int NT, typename C>
__device__ __forceinline__ int plane_scatter(const HpsiView& v, int plane, int k, int slot,
                                             const C* __restrict__ src, C* pl, int* rows) {
  for (int i = threadIdx.x; i < plane; i += NT) pl[i] = mk<C>(0, 0);
  const int rs = v.row_start[k * (v.nslots + 1) + slot];
  const int nrows = v.row_start[k * (v.nslots + 1) + slot + 1] - rs;
  for (int i = threadIdx.x; i < nrows; i += NT) rows[i] = v.rows[rs + i];
  __syncthreads();
  const int es = v.entry_start[k * (v.nslots + 1) + slot];
  const int ee = v.entry_start[k * (v.nslots + 1) + slot + 1];
  int t = es + threadIdx.x;
  for (; t + 3 * NT < ee; t += 4 * NT) {
    int2 en[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) en[u] = v.entries[t + u * NT];
    C val[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) val[u] = src[en[u].x];
#pragma unroll
    for (int u = 0; u < 4; ++u) pl[en[u].y] = val[u];
  }
  for (; t < ee; t += NT) {
    const int2 en = v.entries[t];
    pl[en.y] = src[en.x];
  }
  __syncthreads();
  return nrows;
}

// Gather the band's sphere points out of the transformed plane and add the kinetic term:
// hpsi = plane value + T_G psi (four entries per thread in flight). NT threads.
template <int NT, typename T>
__device__ __forceinline__ void plane_gather(const HpsiView& v, int k, int slot, const cx_t<T>* pl,
                                             const T* __restrict__ kk, const cx_t<T>* __restrict__ psi,
                                             cx_t<T>* __restrict__ hpsi, int64_t boff) {
  using C = cx_t<T>;
  const int es = v.entry_start[k * (v.nslots + 1) + slot];
  const int ee = v.entry_start[k * (v.nslots + 1) + slot + 1];
  int t = es + threadIdx.x;
  for (; t + 3 * NT < ee; t += 4 * NT) {
    int2 en[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) en[u] = v.entries[t + u * NT];
    C p[4];
    T tg[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      p[u] = psi[boff + en[u].x];
      tg[u] = kk[en[u].x];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      C r = pl[en[u].y];
      r.x += tg[u] * p[u].x;
      r.y += tg[u] * p[u].y;
      hpsi[boff + en[u].x] = r;
    }
  }
  for (; t < ee; t += NT) {
    const int2 en = v.entries[t];
    const C p = psi[boff + en.x];
    C r = pl[en.y];
    const T tg = kk[en.x];
    r.x += tg * p.x;
    r.y += tg * p.y;
    hpsi[boff + en.x] = r;
  }
}

template <typename T, class D>
__global__ void __launch_bounds__(kFftThreads)
stage_a_kernel(HpsiView v, const cx_t<T>* __restrict__ tw_y, const cx_t<T>* __restrict__ tw_z,
               const cx_t<T>* __restrict__ psi, cx_t<T>* __restrict__ work) {
  using C = cx_t<T>;
  AMA_DIMS(D, v)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* pl = reinterpret_cast<C*>(smem_raw);
  C* sty = pl + plane;
  C* stz = sty + n2;
  int* rows = reinterpret_cast<int*>(stz + n3);

  const int slot = blockIdx.x;
  const int gb = blockIdx.y;
  const int kl = gb / v.nbands, band = gb - kl * v.nbands;
  const int k = v.k_first + kl;
  const int npw = v.npw[k];
  const C* src = psi + (v.pw_off[k] - v.pw_off[v.k_first]) * v.nbands + (int64_t)band * npw;

  load_tw(sty, tw_y, n2);
  load_tw(stz, tw_z, n3);
  const int nrows = plane_scatter<kFftThreads>(v, plane, k, slot, src, pl, rows);
  dft_rows<+1>(pl, n3, A3, B3, n3, rows, nrows, stz);
  // y transform; its last pass writes the slot plane straight to HBM
  dft_cols_store<+1>(pl, work + (int64_t)gb * v.band_elems + (int64_t)slot * plane, n2, A2, B2, n3, sty);
}

// Load the slot rows at one y (columns z0 .. z0+nz-1) into an (n1, nz) slab, zero
// elsewhere, backward x transform.
template <typename T, class D>
__device__ __forceinline__ void slab_load_backward(const HpsiView& v, const cx_t<T>* wb, cx_t<T>* slab,
                                                   const cx_t<T>* twb, int nz) {
  using C = cx_t<T>;
  AMA_DIMS(D, v)
  for (int e = threadIdx.x; e < n1 * nz; e += kFftThreads) {
    const int x = e / nz, z = e - x * nz;
    const int slot = v.slot_of_x[x];
    slab[e] = slot >= 0 ? wb[(int64_t)slot * plane + z] : mk<C>(0, 0);
  }
  __syncthreads();
  dft_cols<+1>(slab, n1, A1, B1, nz, twb);
}

template <typename T, class D>
__global__ void __launch_bounds__(kFftThreads)
stage_b_kernel(HpsiView v, const cx_t<T>* __restrict__ tw_xb, const cx_t<T>* __restrict__ tw_xf,
               const T* __restrict__ vpot, cx_t<T>* __restrict__ work) {
  using C = cx_t<T>;
  AMA_DIMS(D, v)
  constexpr int ZS = D::zsplit;
  const int nz = n3 / ZS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* slab = reinterpret_cast<C*>(smem_raw);  // [n1][nz]
  C* twb = slab + n1 * nz;
  C* twf = twb + n1;
  const int y = blockIdx.x / ZS, z0 = (blockIdx.x - y * ZS) * nz;
  const int gb = blockIdx.y;
  load_tw(twb, tw_xb, n1);
  load_tw(twf, tw_xf, n1);
  C* wb = work + (int64_t)gb * v.band_elems + (int64_t)y * n3 + z0;
  slab_load_backward<T, D>(v, wb, slab, twb, nz);
  const T* vy = vpot + (int64_t)y * n3 + z0;
  for (int e = threadIdx.x; e < n1 * nz; e += kFftThreads) {
    const int x = e / nz, z = e - x * nz;
    slab[e] = cscale(slab[e], vy[(int64_t)x * plane + z]);
  }
  __syncthreads();
  dft_cols<-1>(slab, n1, A1, B1, nz, twf);
  for (int e = threadIdx.x; e < v.nslots * nz; e += kFftThreads) {
    const int slot = e / nz, z = e - slot * nz;
    wb[(int64_t)slot * plane + z] = slab[v.plane_x[slot] * nz + z];
  }
}

// Stage B with each x column held in registers (complex64, compile-time n1): one thread
// per (y, z) column of a band, no shared memory. The backward transform (natural x in,
// permuted out), the V multiply and the forward transform (permuted in, natural out) are
// the same four-step DFTs as the shared-memory passes, done on a register array.
constexpr int kRegBThreads = 128;

// a * w^M with w = exp(S 2 pi i / N): an immediate twiddle when the line length has a
// compile-time table, else a load from the uploaded table (which carries the sign)
template <int N, int S, int M>
__device__ __forceinline__ float2 line_twiddle(float2 a, const float2* __restrict__ tw) {
  if constexpr (LineTwiddles<N>::kHave) {
    constexpr float c = (float)LineTwiddles<N>::cos[M];
    constexpr float s = (float)(S * LineTwiddles<N>::sin[M]);
    return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
  } else {
    return cmul(a, __ldg(tw + M));
  }
}

template <int N, int A, int S, bool NAT_IN>
__device__ __forceinline__ void dft_line_reg(float2 (&v)[N], const float2* __restrict__ tw) {
  constexpr int B = N / A;
  if constexpr (NAT_IN) {
    static_for<B>([&](auto bb) {
      constexpr int b = decltype(bb)::value;
      float2 t[A];
      static_for<A>([&](auto aa) { t[decltype(aa)::value] = v[decltype(aa)::value * B + b]; });
      dft_reg<A, S>(t);
      static_for<A>([&](auto cc) {
        constexpr int c = decltype(cc)::value;
        if constexpr (b * c % N != 0) t[c] = line_twiddle<N, S, (b * c) % N>(t[c], tw);
        v[c * B + b] = t[c];
      });
    });
    static_for<A>([&](auto cc) {
      constexpr int c = decltype(cc)::value;
      float2 t[B];
      static_for<B>([&](auto dd) { t[decltype(dd)::value] = v[c * B + decltype(dd)::value]; });
      dft_reg<B, S>(t);
      static_for<B>([&](auto dd) { v[c * B + decltype(dd)::value] = t[decltype(dd)::value]; });
    });
  } else {
    static_for<A>([&](auto cc) {
      constexpr int c = decltype(cc)::value;
      float2 t[B];
      static_for<B>([&](auto dd) { t[decltype(dd)::value] = v[c * B + decltype(dd)::value]; });
      dft_reg<B, S>(t);
      static_for<B>([&](auto ee) {
        constexpr int e = decltype(ee)::value;
        if constexpr (c * e % N != 0) t[e] = line_twiddle<N, S, (c * e) % N>(t[e], tw);
        v[c * B + e] = t[e];
      });
    });
    static_for<B>([&](auto ee) {
      constexpr int e = decltype(ee)::value;
      float2 t[A];
      static_for<A>([&](auto cc) { t[decltype(cc)::value] = v[decltype(cc)::value * B + e]; });
      dft_reg<A, S>(t);
      static_for<A>([&](auto gg) { v[decltype(gg)::value * B + e] = t[decltype(gg)::value]; });
    });
  }
}

template <int NX, int AX, class D>
__global__ void __launch_bounds__(kRegBThreads)
stage_b_reg_kernel(HpsiView v, const float2* __restrict__ tw_xb, const float2* __restrict__ tw_xf,
                   const float* __restrict__ vpot, float2* __restrict__ work) {
  AMA_DIMS(D, v)
  const int col = blockIdx.x * kRegBThreads + threadIdx.x;  // y * n3 + z
  if (col >= plane) return;
  float2* wb = work + (int64_t)blockIdx.y * v.band_elems + col;
  float2 r[NX];
  static_for<NX>([&](auto xx) {
    constexpr int x = decltype(xx)::value;
    const int slot = __ldg(v.slot_of_x + x);
    r[x] = slot >= 0 ? wb[(int64_t)slot * plane] : make_float2(0.f, 0.f);
  });
  dft_line_reg<NX, AX, +1, true>(r, tw_xb);
  static_for<NX>([&](auto pp) {
    constexpr int p = decltype(pp)::value;
    const float s = __ldg(vpot + (int64_t)p * plane + col);
    r[p].x *= s;
    r[p].y *= s;
  });
  dft_line_reg<NX, AX, -1, false>(r, tw_xf);
  static_for<NX>([&](auto xx) {
    constexpr int x = decltype(xx)::value;
    const int slot = __ldg(v.slot_of_x + x);
    if (slot >= 0) wb[(int64_t)slot * plane] = r[x];
  });
}

// x-planes used by the spheres when they are the set x <= HP, x >= N - HN (Miller indices
// -HN .. HP), numbered in increasing x
template <int N, int HP, int HN>
struct SlotSet {
  static constexpr bool used(int x) { return x <= HP || x >= N - HN; }
  static constexpr int slot(int x) { return x <= HP ? x : x - (N - HN - HP - 1); }
  // inputs of the strided DFT-A at offset b (x = a B + b) that can be nonzero
  static constexpr uint32_t line_mask(int A, int b) {
    uint32_t m = 0;
    for (int a = 0; a < A; ++a)
      if (used(a * (N / A) + b)) m |= 1u << a;
    return m;
  }
};

// Stage B for a compile-time slot set: the x transform's zero inputs (x-planes without
// sphere points) are skipped in the backward transform's first pass, and only the used
// outputs of the forward transform are computed (the stores, and with them everything that
// feeds only unused outputs, are resolved at compile time).
template <int NX, int AX, int HP, int HN, class D>
__global__ void __launch_bounds__(kRegBThreads)
stage_b_sparse_kernel(HpsiView v, const float2* __restrict__ tw_xb, const float2* __restrict__ tw_xf,
                      const float* __restrict__ vpot, float2* __restrict__ work) {
  using SS = SlotSet<NX, HP, HN>;
  constexpr int BX = NX / AX;
  AMA_DIMS(D, v)
  const int col = blockIdx.x * kRegBThreads + threadIdx.x;  // y * n3 + z
  if (col >= plane) return;
  float2* wb = work + (int64_t)blockIdx.y * v.band_elems + col;
  float2 r[NX];
  static_for<NX>([&](auto xx) {
    constexpr int x = decltype(xx)::value;
    if constexpr (SS::used(x)) r[x] = wb[(int64_t)SS::slot(x) * plane];
  });
  // backward x transform, natural in: strided DFT-A on the sparse inputs, twiddle, DFT-B
  static_for<BX>([&](auto bb) {
    constexpr int b = decltype(bb)::value;
    constexpr uint32_t mask = SS::line_mask(AX, b);
    float2 t[AX];
    static_for<AX>([&](auto aa) {
      constexpr int a = decltype(aa)::value;
      if constexpr ((mask >> a) & 1u) t[a] = r[a * BX + b];
    });
    dft_reg_sparse<AX, +1, mask>(t);
    static_for<AX>([&](auto cc) {
      constexpr int c = decltype(cc)::value;
      if constexpr (b * c % NX != 0) t[c] = line_twiddle<NX, +1, (b * c) % NX>(t[c], tw_xb);
      r[c * BX + b] = t[c];
    });
  });
  static_for<AX>([&](auto cc) {
    constexpr int c = decltype(cc)::value;
    float2 t[BX];
    static_for<BX>([&](auto dd) { t[decltype(dd)::value] = r[c * BX + decltype(dd)::value]; });
    dft_reg<BX, +1>(t);
    static_for<BX>([&](auto dd) { r[c * BX + decltype(dd)::value] = t[decltype(dd)::value]; });
  });
  static_for<NX>([&](auto pp) {
    constexpr int p = decltype(pp)::value;
    const float s = __ldg(vpot + (int64_t)p * plane + col);
    r[p].x *= s;
    r[p].y *= s;
  });
  dft_line_reg<NX, AX, -1, false>(r, tw_xf);
  static_for<NX>([&](auto xx) {
    constexpr int x = decltype(xx)::value;
    if constexpr (SS::used(x)) wb[(int64_t)SS::slot(x) * plane] = r[x];
  });
}

// Stage B with two threads per (y, z) column (complex64, even compile-time n1 = 2 M): each
// lane of an adjacent pair holds M of the n1 values, so the line never spills out of
// registers. Backward transform by decimation in frequency index: lane h takes the inputs
// G = 2m + h and transforms them with a length-M register DFT; the radix-2 combination
// X[k + M j] = Y_0[k] + (-1)^j w^k Y_1[k] (w = e^{2 pi i / n1}) is done across the pair with
// warp shuffles, lane h keeping the half j = h. The potential multiplies the natural x
// index i = k + M h at the engine's permuted x position. The forward transform mirrors it:
// Z_h[k] = (X[k] + (-1)^h X[k + M]) w^{-h k} across the pair, then a length-M DFT gives the
// outputs G = 2m + h. Slots are looked up at run time; unused x-planes are neither read
// nor written.
template <int M, int AH>
__host__ __device__ constexpr int half_index(int p) {  // index held at register p after the natural-in DFT
  return p / (M / AH) + AH * (p % (M / AH));
}

template <int NX, int AH, class D>
__global__ void __launch_bounds__(kRegBThreads)
stage_b_pair_kernel(HpsiView v, const float2* __restrict__ tw_xb, const float2* __restrict__ tw_xf,
                    const float* __restrict__ vpot, float2* __restrict__ work) {
  constexpr int M = NX / 2;
  AMA_DIMS(D, v)
  const int gt = blockIdx.x * kRegBThreads + threadIdx.x;
  const int col_raw = gt >> 1, h = gt & 1;
  const bool live = col_raw < plane;  // both lanes of a pair agree
  const int col = live ? col_raw : 0;  // dead pairs still take part in the shuffles
  float2* wb = work + (int64_t)blockIdx.y * v.band_elems + col;
  float2 r[M];
  static_for<M>([&](auto mm) {
    constexpr int m = decltype(mm)::value;
    const int slot = live ? __ldg(v.slot_of_x + 2 * m + h) : -1;
    r[m] = slot >= 0 ? wb[(int64_t)slot * plane] : make_float2(0.f, 0.f);
  });
  dft_line_reg<M, AH, +1, true>(r, tw_xb);
  static_for<M>([&](auto pp) {
    constexpr int p = decltype(pp)::value;
    constexpr int k = half_index<M, AH>(p);
    const float2 mine = r[p];
    const float2 other = make_float2(__shfl_xor_sync(0xffffffffu, mine.x, 1), __shfl_xor_sync(0xffffffffu, mine.y, 1));
    const float2 y0 = h ? other : mine;
    const float2 t = line_twiddle<NX, +1, k>(h ? mine : other, tw_xb);
    r[p] = h ? csub(y0, t) : cadd(y0, t);
    const int i = k + M * h;                       // natural x index of the real-space value
    const int pos = (i % A1) * B1 + i / A1;        // its position in the engine's permuted x order
    const float sv = __ldg(vpot + (int64_t)pos * plane + col);
    r[p].x *= sv;
    r[p].y *= sv;
  });
  static_for<M>([&](auto pp) {
    constexpr int p = decltype(pp)::value;
    constexpr int k = half_index<M, AH>(p);
    const float2 mine = r[p];
    const float2 other = make_float2(__shfl_xor_sync(0xffffffffu, mine.x, 1), __shfl_xor_sync(0xffffffffu, mine.y, 1));
    const float2 lo = h ? other : mine, hi = h ? mine : other;  // X[k], X[k + M]
    const float2 z = h ? csub(lo, hi) : cadd(lo, hi);
    const float2 zt = line_twiddle<NX, -1, k>(z, tw_xf);
    r[p] = h ? zt : z;
  });
  dft_line_reg<M, AH, -1, false>(r, tw_xf);
  if (!live) return;
  static_for<M>([&](auto mm) {
    constexpr int m = decltype(mm)::value;
    const int slot = __ldg(v.slot_of_x + 2 * m + h);
    if (slot >= 0) wb[(int64_t)slot * plane] = r[m];
  });
}

template <typename T, class D>
__global__ void __launch_bounds__(kFftThreads)
stage_c_kernel(HpsiView v, const cx_t<T>* __restrict__ tw_y, const cx_t<T>* __restrict__ tw_z,
               const T* __restrict__ kin, const cx_t<T>* __restrict__ psi,
               const cx_t<T>* __restrict__ work, cx_t<T>* __restrict__ hpsi) {
  using C = cx_t<T>;
  AMA_DIMS(D, v)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* pl = reinterpret_cast<C*>(smem_raw);
  C* sty = pl + plane;
  C* stz = sty + n2;
  int* rows = reinterpret_cast<int*>(stz + n3);

  const int slot = blockIdx.x;
  const int gb = blockIdx.y;
  const int kl = gb / v.nbands, band = gb - kl * v.nbands;
  const int k = v.k_first + kl;
  const int npw = v.npw[k];
  const int64_t boff = (v.pw_off[k] - v.pw_off[v.k_first]) * v.nbands + (int64_t)band * npw;

  const C* srcw = work + (int64_t)gb * v.band_elems + (int64_t)slot * plane;
  // the whole slot plane in flight while the tables load (measured faster than reading it
  // inside the first y pass, whose seven loads per task keep fewer requests in flight)
  async_copy(pl, srcw, plane);
  load_tw(sty, tw_y, n2);
  load_tw(stz, tw_z, n3);
  const int rs = v.row_start[k * (v.nslots + 1) + slot];
  const int nrows = v.row_start[k * (v.nslots + 1) + slot + 1] - rs;
  for (int i = threadIdx.x; i < nrows; i += kFftThreads) rows[i] = v.rows[rs + i];
  async_copy_wait();
  __syncthreads();
  dft_cols<-1>(pl, n2, A2, B2, n3, sty);
  dft_rows<-1>(pl, n3, A3, B3, n3, rows, nrows, stz);
  plane_gather<kFftThreads, T>(v, k, slot, pl, kin + v.pw_off[k], psi, hpsi, boff);
}

// ------------------------------------------- y transforms in registers, four lanes per column
// Stages A and C of complex64 H.psi with the y transform of each (slot, band) plane done in
// registers instead of two shared-memory passes over the whole plane: four adjacent lanes
// share a z column, lane h holding the M = n2 / 4 values of y index 4 m + h. Backward, each
// lane transforms its values with a length-M register DFT (Y_h[k] = sum_m u[4m+h] w_M^{mk})
// and the lanes combine them by
//   X[k + M j] = sum_h (w^{hk} Y_h[k]) i^{hj}          (w = e^{2 pi i / n2})
// as a 4-point DFT across the lanes in two butterfly steps (shuffles with lane distance 2,
// then 1), after which lane h = h0 + 2 h1 holds X[k + M (h1 + 2 h0)]. The forward transform
// is the adjoint of the same steps in reverse order, ending with length-M register DFTs
// whose outputs are y = 4 m + h. Stage A writes its registers straight to the slot plane in
// HBM (the engine's permuted y order), stage C loads them straight from it, so besides
// the y passes the plane copy through shared memory is gone too. The z transforms (rows
// with sphere points only) stay in shared memory.
template <int N3>
constexpr int quad_threads() { return (4 * N3 + 31) / 32 * 32; }

template <int N, int M, int AH>
__host__ __device__ constexpr int quad_index(int p) { return half_index<M, AH>(p); }

// a * w^{S h K} for the lane's h in 0..3 (w = e^{2 pi i / N}), twiddles as immediates
template <int N, int S, int K>
__device__ __forceinline__ float2 quad_twiddle(float2 a, int h) {
  if constexpr (K == 0) {
    return a;
  } else {
    constexpr float c1 = (float)LineTwiddles<N>::cos[K % N], s1 = (float)(S * LineTwiddles<N>::sin[K % N]);
    constexpr float c2 = (float)LineTwiddles<N>::cos[2 * K % N], s2 = (float)(S * LineTwiddles<N>::sin[2 * K % N]);
    constexpr float c3 = (float)LineTwiddles<N>::cos[3 * K % N], s3 = (float)(S * LineTwiddles<N>::sin[3 * K % N]);
    const float c = h == 0 ? 1.f : (h == 1 ? c1 : (h == 2 ? c2 : c3));
    const float sn = h == 0 ? 0.f : (h == 1 ? s1 : (h == 2 ? s2 : s3));
    return make_float2(a.x * c - a.y * sn, a.x * sn + a.y * c);
  }
}

__device__ __forceinline__ float2 shfl_xor_c(float2 a, int d) {
  return make_float2(__shfl_xor_sync(0xffffffffu, a.x, d), __shfl_xor_sync(0xffffffffu, a.y, d));
}

// backward: r[p] = Y_h[k] (k = quad_index(p)) -> X[k + M (h1 + 2 h0)]
template <int N, int M, int AH>
__device__ __forceinline__ void quad_combine_backward(float2 (&r)[M], int h) {
  const int h0 = h & 1, h1 = h >> 1;
  static_for<M>([&](auto pp) {
    constexpr int p = decltype(pp)::value;
    constexpr int k = quad_index<N, M, AH>(p);
    const float2 t = quad_twiddle<N, +1, k>(r[p], h);
    const float2 o = shfl_xor_c(t, 2);
    const float2 u = h1 ? csub(o, t) : cadd(t, o);  // U_{h0}(j parity h1)
    const float2 q = shfl_xor_c(u, 1);
    const float2 u0 = h0 ? q : u, u1 = h0 ? u : q;
    const float2 v = h1 ? make_float2(-u1.y, u1.x) : u1;  // i^{h1} U_1
    r[p] = h0 ? csub(u0, v) : cadd(u0, v);
  });
}

// forward, the adjoint: r[p] = X[k + M (h1 + 2 h0)] -> Z_h[k] = w^{-hk} sum_j X[k + M j] (-i)^{hj}
template <int N, int M, int AH>
__device__ __forceinline__ void quad_combine_forward(float2 (&r)[M], int h) {
  const int h0 = h & 1, h1 = h >> 1;
  static_for<M>([&](auto pp) {
    constexpr int p = decltype(pp)::value;
    constexpr int k = quad_index<N, M, AH>(p);
    const float2 a = r[p];
    const float2 q = shfl_xor_c(a, 1);
    const float2 d = csub(q, a);                              // (lane h0=0) - (lane h0=1), seen from h0=1
    const float2 u1 = h1 ? make_float2(d.y, -d.x) : d;        // conj(i^{h1}) (a - b)
    const float2 u = h0 ? u1 : cadd(a, q);
    const float2 o = shfl_xor_c(u, 2);
    const float2 t = h1 ? csub(o, u) : cadd(u, o);
    r[p] = quad_twiddle<N, -1, k>(t, h);
  });
}

template <int NY, int AQ, class D>
__global__ void __launch_bounds__(quad_threads<D::n3c()>())
stage_a_quad_kernel(HpsiView v, const float2* __restrict__ tw_y, const float2* __restrict__ tw_z,
                    const float2* __restrict__ psi, float2* __restrict__ work) {
  using C = float2;
  constexpr int NT = quad_threads<D::n3c()>();
  constexpr int M = NY / 4;
  AMA_DIMS(D, v)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* pl = reinterpret_cast<C*>(smem_raw);
  C* stz = pl + plane + n2;  // the shared layout of stage A (no y twiddles needed)
  int* rows = reinterpret_cast<int*>(stz + n3);

  const int slot = blockIdx.x;
  const int gb = blockIdx.y;
  const int kl = gb / v.nbands, band = gb - kl * v.nbands;
  const int k = v.k_first + kl;
  const int npw = v.npw[k];
  const C* src = psi + (v.pw_off[k] - v.pw_off[v.k_first]) * v.nbands + (int64_t)band * npw;
  for (int i = threadIdx.x; i < n3; i += NT) stz[i] = tw_z[i];
  const int nrows = plane_scatter<NT>(v, plane, k, slot, src, pl, rows);
  dft_rows<+1, true, NT>(pl, n3, A3, B3, n3, rows, nrows, stz);
  // y columns: lanes 4c .. 4c+3 take column c; lanes past the last column shuffle along
  const int col_raw = threadIdx.x >> 2, h = threadIdx.x & 3;
  if ((int)(threadIdx.x & ~31u) >= 4 * n3) return;  // the whole warp is past the last column
  const bool live = col_raw < n3;
  const int col = live ? col_raw : 0;
  float2 r[M];
  static_for<M>([&](auto mm) {
    constexpr int m = decltype(mm)::value;
    r[m] = pl[(4 * m + h) * n3 + col];
  });
  dft_line_reg<M, AQ, +1, true>(r, tw_y);
  quad_combine_backward<NY, M, AQ>(r, h);
  if (!live) return;
  C* dst = work + (int64_t)gb * v.band_elems + (int64_t)slot * plane + col;
  const int j = (h >> 1) + 2 * (h & 1);
  static_for<M>([&](auto pp) {
    constexpr int p = decltype(pp)::value;
    const int i = quad_index<NY, M, AQ>(p) + M * j;  // natural y index held in r[p]
    dst[(int64_t)((i % A2) * B2 + i / A2) * n3] = r[p];
  });
}

template <int NY, int AQ, class D>
__global__ void __launch_bounds__(quad_threads<D::n3c()>())
stage_c_quad_kernel(HpsiView v, const float2* __restrict__ tw_y, const float2* __restrict__ tw_z,
                    const float* __restrict__ kin, const float2* __restrict__ psi,
                    const float2* __restrict__ work, float2* __restrict__ hpsi) {
  using C = float2;
  constexpr int NT = quad_threads<D::n3c()>();
  constexpr int M = NY / 4;
  AMA_DIMS(D, v)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* pl = reinterpret_cast<C*>(smem_raw);
  C* stz = pl + plane + n2;
  int* rows = reinterpret_cast<int*>(stz + n3);

  const int slot = blockIdx.x;
  const int gb = blockIdx.y;
  const int kl = gb / v.nbands, band = gb - kl * v.nbands;
  const int k = v.k_first + kl;
  const int npw = v.npw[k];
  const int64_t boff = (v.pw_off[k] - v.pw_off[v.k_first]) * v.nbands + (int64_t)band * npw;
  for (int i = threadIdx.x; i < n3; i += NT) stz[i] = tw_z[i];
  const int rs = v.row_start[k * (v.nslots + 1) + slot];
  const int nrows = v.row_start[k * (v.nslots + 1) + slot + 1] - rs;
  for (int i = threadIdx.x; i < nrows; i += NT) rows[i] = v.rows[rs + i];
  const int col_raw = threadIdx.x >> 2, h = threadIdx.x & 3;
  if ((int)(threadIdx.x & ~31u) < 4 * n3) {  // warps with at least one live column
    const bool live = col_raw < n3;
    const int col = live ? col_raw : 0;
    const C* srcw = work + (int64_t)gb * v.band_elems + (int64_t)slot * plane + col;
    const int j = (h >> 1) + 2 * (h & 1);
    float2 r[M];
    static_for<M>([&](auto pp) {
      constexpr int p = decltype(pp)::value;
      const int i = quad_index<NY, M, AQ>(p) + M * j;
      r[p] = __ldg(srcw + (int64_t)((i % A2) * B2 + i / A2) * n3);
    });
    quad_combine_forward<NY, M, AQ>(r, h);
    dft_line_reg<M, AQ, -1, false>(r, tw_y);
    if (live) {
      static_for<M>([&](auto mm) {
        constexpr int m = decltype(mm)::value;
        pl[(4 * m + h) * n3 + col] = r[m];
      });
    }
  }
  __syncthreads();
  dft_rows<-1, false, NT>(pl, n3, A3, B3, n3, rows, nrows, stz);
  plane_gather<NT, float>(v, k, slot, pl, kin + v.pw_off[k], psi, hpsi, boff);
}

// density: stage A output -> backward x, then weighted |u|^2 into a permuted FP64 grid.
template <typename T, class D>
__global__ void __launch_bounds__(kFftThreads)
density_b_kernel(HpsiView v, const cx_t<T>* __restrict__ tw_xb, const cx_t<T>* __restrict__ work,
                 const double* __restrict__ w, double* __restrict__ acc) {
  using C = cx_t<T>;
  AMA_DIMS(D, v)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* slab = reinterpret_cast<C*>(smem_raw);
  C* twb = slab + n1 * n3;
  const int y = blockIdx.x;
  const int gb = blockIdx.y;
  const double weight = w[gb];
  if (weight == 0.0) return;
  load_tw(twb, tw_xb, n1);
  const C* wb = work + (int64_t)gb * v.band_elems + (int64_t)y * n3;
  slab_load_backward<T, D>(v, wb, slab, twb, n3);
  for (int e = threadIdx.x; e < n1 * n3; e += kFftThreads) {
    const int x = e / n3, z = e - x * n3;
    const C u = slab[e];
    atomicAdd(acc + (int64_t)x * plane + (int64_t)y * n3 + z,
              weight * ((double)u.x * (double)u.x + (double)u.y * (double)u.y));
  }
}

// The stage B variants compiled for a grid: [0] shared-memory slab, [1] register-resident
// x columns, [2] register-resident with the compile-time slot set, [3] register-resident
// with two threads per column, [4] shared-memory slab split in two along z (null when
// absent), with the z split of each.
// The stage A/C pairs: [0] shared-memory y passes, [1] y transforms in registers with four
// lanes per column (null when absent), with their threads per CTA.
struct StageInfo {
  int zsplit;
  bool regb;
  const void* b_variant[5];
  int b_zsplit[5] = {1, 1, 1, 1, 2};
  const void* ac_variant[2][2] = {};
  int ac_threads[2] = {kFftThreads, kFftThreads};
};

template <typename T, class D>
StageInfo fill_stage_table(const void** fn) {
  fn[0] = (const void*)stage_a_kernel<T, D>;
  fn[1] = (const void*)stage_b_kernel<T, D>;
  fn[2] = (const void*)stage_c_kernel<T, D>;
  fn[3] = (const void*)density_b_kernel<T, D>;
  StageInfo info{D::zsplit, false, {fn[1], nullptr, nullptr, nullptr, nullptr}};
  info.ac_variant[0][0] = fn[0];
  info.ac_variant[0][1] = fn[2];
  return info;
}

// the four-lanes-per-column stages A and C, when n2 = 4 M with a nontrivial split of M and
// both y lengths have immediate twiddles
template <int N2, class D>
void add_quad_variant(StageInfo& info) {
  if constexpr (N2 % 4 == 0 && N2 >= 80) {  // short y lines stay with the shared-memory passes
    constexpr int M = N2 / 4;
    constexpr int AQ = M % 3 == 0 && M > 3 ? 3 : (M % 2 == 0 && M > 2 ? 2 : 0);
    if constexpr (AQ > 0 && LineTwiddles<M>::kHave && LineTwiddles<N2>::kHave) {
      info.ac_variant[1][0] = (const void*)stage_a_quad_kernel<N2, AQ, D>;
      info.ac_variant[1][1] = (const void*)stage_c_quad_kernel<N2, AQ, D>;
      info.ac_threads[1] = quad_threads<D::n3c()>();
    }
  }
}

// the two-lanes-per-column stage B, when n1 is even and both line lengths have immediate
// twiddles (the half-length DFT cannot take its twiddles from the n1 table)
template <int N1, class D>
void add_pair_variant(StageInfo& info) {
  if constexpr (N1 % 2 == 0 && N1 >= 40) {  // shorter lines fit one thread's registers
    constexpr int M = N1 / 2;
    if constexpr (LineTwiddles<M>::kHave && LineTwiddles<N1>::kHave) {
      constexpr int AH = M % 6 == 0 && M / 6 > 1 ? 6 : (M % 3 == 0 ? 3 : (M % 2 == 0 ? 2 : M));
      info.b_variant[3] = (const void*)stage_b_pair_kernel<N1, AH, D>;
    }
  }
}

// the shared-memory stage B with each (x, z) slab split in two along z, where the whole
// slab is large: complex64 lines of 100 or more, complex128 lines of 40 or more (the
// whole-slab CTA of a 108^3 grid holds 93 KB in complex64, 186 KB in complex128; of an 84^3
// grid 113 KB in complex128, which leaves one or two CTAs per SM)
template <typename T, int N1, int A1, int N2, int A2, int N3, int A3>
void add_zsplit_variant(StageInfo& info) {
  constexpr int kMinLine = std::is_same<T, double>::value ? 40 : 100;
  if constexpr (N3 % 2 == 0 && N1 >= kMinLine)
    info.b_variant[4] = (const void*)stage_b_kernel<T, FixDims<N1, A1, N2, A2, N3, A3, 2>>;
}

// complex64 on a compile-time grid with short x columns: register-resident stage B
// (register-resident y columns for stages A and C were measured slower than the
// shared-memory passes at 84^3 and are not used)
template <int N1, int A1, int N2, int A2, int N3, class D>
StageInfo fill_stage_table_reg(const void** fn, int hp, int hn) {
  StageInfo info = fill_stage_table<float, D>(fn);
  fn[1] = (const void*)stage_b_reg_kernel<N1, A1, D>;
  info.regb = true;
  info.b_variant[1] = fn[1];
  add_pair_variant<N1, D>(info);
  add_quad_variant<N2, D>(info);
  if constexpr (N1 == 84) {  // the Si64 benchmark grid: sparse-x variants for its slot sets
#define AMA_SPARSE(P, Q) \
    if (hp == P && hn == Q) fn[1] = info.b_variant[2] = (const void*)stage_b_sparse_kernel<84, 12, P, Q, D>;
    AMA_SPARSE(20, 20) AMA_SPARSE(20, 21) AMA_SPARSE(21, 20) AMA_SPARSE(21, 21)
#undef AMA_SPARSE
  }
  return info;
}

// Grids with compile-time kernels (cubic cells of the benchmark workloads); any other grid
// runs the same kernels with sizes read at run time.
template <typename T>
StageInfo select_stage_table(const AxisPlan* ax, const void** fn, int hp, int hn) {
#define AMA_FIX(N1, A1, N2, A2, N3, A3)                                                         \
  if (ax[0].n == N1 && ax[0].A == A1 && ax[1].n == N2 && ax[1].A == A2 && ax[2].n == N3 &&      \
      ax[2].A == A3) {                                                                           \
    using D = FixDims<N1, A1, N2, A2, N3, A3>;                                                   \
    if constexpr (std::is_same<T, float>::value && N1 <= 96) {                                   \
      return fill_stage_table_reg<N1, A1, N2, A2, N3, D>(fn, hp, hn);                            \
    } else if constexpr (std::is_same<T, float>::value) { /* longer x lines: only two lanes */   \
      StageInfo info = fill_stage_table<T, D>(fn);                                               \
      add_pair_variant<N1, D>(info);                                                             \
      add_quad_variant<N2, D>(info);                                                             \
      add_zsplit_variant<T, N1, A1, N2, A2, N3, A3>(info);                                       \
      return info;                                                                               \
    } else {                                                                                     \
      StageInfo info = fill_stage_table<T, D>(fn);                                               \
      add_zsplit_variant<T, N1, A1, N2, A2, N3, A3>(info);                                       \
      return info;                                                                               \
    }                                                                                            \
  }
  AMA_FIX(20, 5, 20, 5, 20, 5)
  AMA_FIX(25, 5, 25, 5, 25, 5)
  AMA_FIX(35, 7, 35, 7, 35, 7)
  AMA_FIX(36, 6, 36, 6, 36, 6)
  AMA_FIX(42, 7, 42, 7, 42, 7)
  AMA_FIX(84, 12, 84, 12, 84, 12)
  AMA_FIX(108, 12, 108, 12, 108, 12)
#undef AMA_FIX
  return fill_stage_table<T, DynDims>(fn);
}

template <typename T>
using StageAFn = void (*)(HpsiView, const cx_t<T>*, const cx_t<T>*, const cx_t<T>*, cx_t<T>*);
template <typename T>
using StageBFn = void (*)(HpsiView, const cx_t<T>*, const cx_t<T>*, const T*, cx_t<T>*);
template <typename T>
using StageCFn = void (*)(HpsiView, const cx_t<T>*, const cx_t<T>*, const T*, const cx_t<T>*,
                          const cx_t<T>*, cx_t<T>*);
template <typename T>
using DensFn = void (*)(HpsiView, const cx_t<T>*, const cx_t<T>*, const double*, double*);


template <typename T>
__global__ void permute_potential_kernel(const double* __restrict__ v, T* __restrict__ out,
                                         int n1, int n2, int n3, int A1, int B1, int A2, int B2,
                                         int A3, int B3, double scale) {
  const int64_t N = (int64_t)n1 * n2 * n3;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < N;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int p3 = e % n3, p2 = (e / n3) % n2, p1 = e / ((int64_t)n2 * n3);
    const int x = p1 / B1 + A1 * (p1 % B1);
    const int y = p2 / B2 + A2 * (p2 % B2);
    const int z = p3 / B3 + A3 * (p3 % B3);
    out[e] = (T)(v[((int64_t)x * n2 + y) * n3 + z] * scale);
  }
}

__global__ void unpermute_add_kernel(const double* __restrict__ acc, double* __restrict__ rho,
                                     int n1, int n2, int n3, int A1, int B1, int A2, int B2,
                                     int A3, int B3) {
  const int64_t N = (int64_t)n1 * n2 * n3;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < N;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int p3 = e % n3, p2 = (e / n3) % n2, p1 = e / ((int64_t)n2 * n3);
    const int x = p1 / B1 + A1 * (p1 % B1);
    const int y = p2 / B2 + A2 * (p2 % B2);
    const int z = p3 / B3 + A3 * (p3 % B3);
    rho[((int64_t)x * n2 + y) * n3 + z] += acc[e];
  }
}

// Batch functors for the nonlocal products over k-points of one call.
template <typename C> struct ProjectBatch {  // P_k = psi_k B_k^H  (nbands x nproj)
  const C* psi; const C* proj; C* out; const int64_t* pw_off; const int* npw;
  int k_first, nbands, nproj;
  __device__ GemmProblem<C> operator()(int z) const {
    const int k = k_first + z;
    const int64_t off = pw_off[k] - pw_off[k_first];
    GemmProblem<C> p;
    p.a = psi + off * nbands; p.b = proj + pw_off[k] * nproj; p.c = out + (int64_t)z * nbands * nproj;
    p.m = nbands; p.n = nproj; p.k = npw[k];
    p.lda = npw[k]; p.ldb = npw[k]; p.ldc = nproj;
    return p;
  }
};
template <typename C> struct ApplyBatch {    // hpsi_k += P_k (D B_k)  (nbands x npw_k)
  const C* pmat; const C* dproj; C* out; const int64_t* pw_off; const int* npw;
  int k_first, nbands, nproj;
  __device__ GemmProblem<C> operator()(int z) const {
    const int k = k_first + z;
    const int64_t off = pw_off[k] - pw_off[k_first];
    GemmProblem<C> p;
    p.a = pmat + (int64_t)z * nbands * nproj; p.b = dproj + pw_off[k] * nproj; p.c = out + off * nbands;
    p.m = nbands; p.n = npw[k]; p.k = nproj;
    p.lda = nproj; p.ldb = npw[k]; p.ldc = npw[k];
    return p;
  }
};

HpsiView make_view(const AmaEngine* e, int k_first, int nbands) {
  HpsiView v;
  v.n1 = e->ax[0].n; v.n2 = e->ax[1].n; v.n3 = e->ax[2].n;
  v.A1 = e->ax[0].A; v.B1 = e->ax[0].B; v.A2 = e->ax[1].A; v.B2 = e->ax[1].B;
  v.A3 = e->ax[2].A; v.B3 = e->ax[2].B;
  v.nslots = e->nslots;
  v.plane_x = e->d.plane_x; v.slot_of_x = e->d.slot_of_x; v.entries = e->d.entries;
  v.entry_start = e->d.entry_start; v.rows = e->d.rows; v.row_start = e->d.row_start;
  v.pw_off = e->d.pw_off; v.npw = e->d.npw;
  v.k_first = k_first; v.nbands = nbands;
  v.plane_elems = (int64_t)v.n2 * v.n3;
  v.band_elems = v.plane_elems * v.nslots;
  return v;
}


template <typename T>
size_t plane_smem(const AmaEngine* e) {
  return (size_t)(e->ax[1].n * e->ax[2].n + e->ax[1].n + e->ax[2].n) * sizeof(cx_t<T>) +
         (size_t)e->ax[1].n * sizeof(int);
}
template <typename T>
size_t slab_smem(const AmaEngine* e) {
  return (size_t)(e->ax[0].n * e->ax[2].n + 2 * e->ax[0].n) * sizeof(cx_t<T>);
}
template <typename T>
size_t slab_b_smem(const AmaEngine* e) {
  const int p = std::is_same<T, float>::value ? AMA_C64 : AMA_C128;
  return (size_t)(e->ax[0].n * (e->ax[2].n / e->zsplit[p]) + 2 * e->ax[0].n) * sizeof(cx_t<T>);
}

template <typename T>
int set_smem_limits(const AmaEngine* e) {
  const size_t ps = plane_smem<T>(e), ss = slab_smem<T>(e);
  int dev = 0, optin = 0;
  AMA_CUDA_TRY(cudaGetDevice(&dev));
  AMA_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  AMA_REQUIRE(ps <= (size_t)optin && ss <= (size_t)optin, AMA_ERR_UNSUPPORTED,
              "grid plane does not fit in shared memory at this precision");
  const int p = std::is_same<T, float>::value ? AMA_C64 : AMA_C128;
  const void** fn = const_cast<AmaEngine*>(e)->stage_fn[p];
  const StageInfo info = select_stage_table<T>(e->ax, fn, e->slot_hp, e->slot_hn);
  const_cast<AmaEngine*>(e)->zsplit[p] = info.zsplit;
  const_cast<AmaEngine*>(e)->regb[p] = info.regb;
  const_cast<AmaEngine*>(e)->bthreads[p] = 1;
  for (int i = 0; i < 5; ++i) {
    const_cast<AmaEngine*>(e)->b_variant[p][i] = info.b_variant[i];
    const_cast<AmaEngine*>(e)->b_zsplit[p][i] = info.b_zsplit[i];
  }
  if (info.b_variant[4]) {
    const size_t zs2 = (size_t)(e->ax[0].n * (e->ax[2].n / 2) + 2 * e->ax[0].n) * sizeof(cx_t<T>);
    AMA_CUDA_TRY(cudaFuncSetAttribute(info.b_variant[4], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zs2));
  }
  for (int i = 0; i < 2; ++i) {
    const_cast<AmaEngine*>(e)->ac_variant[p][i][0] = info.ac_variant[i][0];
    const_cast<AmaEngine*>(e)->ac_variant[p][i][1] = info.ac_variant[i][1];
    const_cast<AmaEngine*>(e)->ac_threads_of[p][i] = info.ac_threads[i];
    if (info.ac_variant[i][0]) {
      AMA_CUDA_TRY(cudaFuncSetAttribute(info.ac_variant[i][0], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps));
      AMA_CUDA_TRY(cudaFuncSetAttribute(info.ac_variant[i][1], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps));
    }
  }
  const_cast<AmaEngine*>(e)->ac_threads[p] = kFftThreads;

  AMA_CUDA_TRY(cudaFuncSetAttribute(fn[0], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps));
  AMA_CUDA_TRY(cudaFuncSetAttribute(fn[2], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps));
  AMA_CUDA_TRY(cudaFuncSetAttribute(info.b_variant[0], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)slab_b_smem<T>(e)));
  AMA_CUDA_TRY(cudaFuncSetAttribute(fn[3], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ss));
  return AMA_OK;
}

int prec_ok(const AmaEngine* e, int precision) {
  AMA_REQUIRE(precision == AMA_C64 || precision == AMA_C128, AMA_ERR_ARG, "precision must be AMA_C64 or AMA_C128");
  AMA_REQUIRE(e->precisions & (1u << precision), AMA_ERR_ARG,
              "the engine was created without this precision");
  return AMA_OK;
}

int ensure_work(AmaEngine* e, int precision, int64_t bands) {
  const size_t el = precision == AMA_C64 ? sizeof(float2) : sizeof(double2);
  const size_t need = (size_t)bands * e->nslots * e->ax[1].n * e->ax[2].n * el;
  AMA_CUDA_TRY(grow<char>(&e->work[precision], &e->work_bytes[precision], need));
  return AMA_OK;
}

template <typename T>
int run_fft_stages_a(AmaEngine* e, const HpsiView& v, int nb_total, const void* psi, cudaStream_t s) {
  using C = cx_t<T>;
  const int p = std::is_same<T, float>::value ? AMA_C64 : AMA_C128;
  dim3 ga(e->nslots, nb_total);
  ((StageAFn<T>)e->stage_fn[p][0])<<<ga, e->ac_threads[p], plane_smem<T>(e), s>>>(
      v, (const C*)e->d.tw[p][1][0], (const C*)e->d.tw[p][2][0], (const C*)psi, (C*)e->work[p]);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

template <typename T>
int hpsi_impl(AmaEngine* e, int k_first, int k_count, int nbands, int spin, const void* psi,
              void* hpsi, cudaStream_t s) {
  using C = cx_t<T>;
  const int p = std::is_same<T, float>::value ? AMA_C64 : AMA_C128;
  const int64_t nb_total = (int64_t)k_count * nbands;
  AMA_REQUIRE(nb_total <= 65535, AMA_ERR_UNSUPPORTED, "more than 65535 bands in one H.psi call");
  int rc = ensure_work(e, p, nb_total);
  if (rc) return rc;
  HpsiView v = make_view(e, k_first, nbands);
  const T* vpot = (p == AMA_C64 ? (const T*)e->d.v32 : (const T*)e->d.v64) + (int64_t)spin * e->N;
  const T* kin = p == AMA_C64 ? (const T*)e->d.kin32 : (const T*)e->d.kin64;

  // complex64 tensor-core nonlocal path. Running its projection on a second stream next to
  // the FFT stages was measured: ~1% faster on average, but with the projection's
  // 222 KB-shared-memory CTAs waiting for whole SMs to drain, some runs were 50% slower, so
  // the products run in stream order after stage C.
  const bool tc_nl = e->nproj > 0 && std::is_same<T, float>::value && e->use_tc && e->tc.ready;

  rc = run_fft_stages_a<T>(e, v, (int)nb_total, psi, s);
  if (rc) return rc;
  if (e->regb[p]) {
    dim3 gr((e->ax[1].n * e->ax[2].n * e->bthreads[p] + kRegBThreads - 1) / kRegBThreads, nb_total);
    ((StageBFn<T>)e->stage_fn[p][1])<<<gr, kRegBThreads, 0, s>>>(
        v, (const C*)e->d.tw[p][0][0], (const C*)e->d.tw[p][0][1], vpot, (C*)e->work[p]);
  } else {
    dim3 gb(e->ax[1].n * e->zsplit[p], nb_total);
    ((StageBFn<T>)e->stage_fn[p][1])<<<gb, kFftThreads, slab_b_smem<T>(e), s>>>(
      v, (const C*)e->d.tw[p][0][0], (const C*)e->d.tw[p][0][1], vpot, (C*)e->work[p]);
  }
  AMA_CHECK_LAUNCH();
  dim3 gc(e->nslots, nb_total);
  ((StageCFn<T>)e->stage_fn[p][2])<<<gc, e->ac_threads[p], plane_smem<T>(e), s>>>(
      v, (const C*)e->d.tw[p][1][1], (const C*)e->d.tw[p][2][1], kin, (const C*)psi,
      (const C*)e->work[p], (C*)hpsi);
  AMA_CHECK_LAUNCH();

  if (tc_nl) {
    rc = nl_tc_run(e, k_first, k_count, nbands, (const float2*)psi, (float2*)hpsi, s);
    if (rc) return rc;
  } else if (e->nproj > 0) {
    const size_t el = sizeof(C);
    const size_t pbytes = (size_t)nb_total * e->nproj * el;
    AMA_CUDA_TRY(grow<char>(&e->ws_proj[p], &e->ws_proj_bytes[p], pbytes));
    int maxnpw = 0;
    for (int k = k_first; k < k_first + k_count; ++k) maxnpw = std::max(maxnpw, e->npw[k]);
    // split the long npw reduction so that the tile grid covers the GPU several times
    const int tiles = (int)std::min<int64_t>(gemm_tile_count<T>(nbands, e->nproj, k_count), 1 << 30);
    int splits = std::max(1, std::min(64, (4 * 148 + tiles - 1) / tiles));
    splits = std::min(splits, std::max(1, maxnpw / 256));
    const int64_t pstride = (int64_t)nbands * e->nproj;
    if (splits > 1)
      AMA_CUDA_TRY(grow<char>(&e->ws_part[p], &e->ws_part_bytes[p], (size_t)k_count * splits * pstride * sizeof(double2)));
    ProjectBatch<C> pb{(const C*)psi, (const C*)e->d.proj[p], (C*)e->ws_proj[p], e->d.pw_off, e->d.npw,
                       k_first, nbands, e->nproj};
    AMA_CUDA_TRY((launch_cgemm<T, kNC>(pb, k_count, nbands, e->nproj, splits, mk<C>(1, 0), mk<C>(0, 0),
                                       (double2*)e->ws_part[p], pstride, s)));
    ApplyBatch<C> ab{(const C*)e->ws_proj[p], (const C*)e->d.dproj[p], (C*)hpsi, e->d.pw_off, e->d.npw,
                     k_first, nbands, e->nproj};
    AMA_CUDA_TRY((launch_cgemm<T, kNN>(ab, k_count, nbands, maxnpw, 1, mk<C>(1, 0), mk<C>(1, 0),
                                       nullptr, 0, s)));
  }
  return AMA_OK;
}

template <typename T>
int density_impl(AmaEngine* e, int k_first, int k_count, int nbands, const void* psi,
                 const double* weights, double* rho, cudaStream_t s) {
  using C = cx_t<T>;
  const int p = std::is_same<T, float>::value ? AMA_C64 : AMA_C128;
  const int64_t nb_total = (int64_t)k_count * nbands;
  AMA_REQUIRE(nb_total <= 65535, AMA_ERR_UNSUPPORTED, "more than 65535 bands in one density call");
  int rc = ensure_work(e, p, nb_total);
  if (rc) return rc;
  AMA_CUDA_TRY(grow<char>((void**)&e->ws_dens, &e->ws_dens_bytes, (size_t)e->N * sizeof(double)));
  AMA_CUDA_TRY(cudaMemsetAsync(e->ws_dens, 0, (size_t)e->N * sizeof(double), s));
  HpsiView v = make_view(e, k_first, nbands);
  rc = run_fft_stages_a<T>(e, v, (int)nb_total, psi, s);
  if (rc) return rc;
  dim3 gb(e->ax[1].n, nb_total);
  ((DensFn<T>)e->stage_fn[p][3])<<<gb, kFftThreads, slab_smem<T>(e), s>>>(v, (const C*)e->d.tw[p][0][0],
                                                                  (const C*)e->work[p], weights, e->ws_dens);
  AMA_CHECK_LAUNCH();
  unpermute_add_kernel<<<592, 256, 0, s>>>(e->ws_dens, rho, e->ax[0].n, e->ax[1].n, e->ax[2].n,
                                           e->ax[0].A, e->ax[0].B, e->ax[1].A, e->ax[1].B, e->ax[2].A,
                                           e->ax[2].B);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

template <typename T>
int upload_twiddles(AmaEngine* e, int prec) {
  using C = cx_t<T>;
  for (int a = 0; a < 3; ++a) {
    const int n = e->ax[a].n;
    for (int dir = 0; dir < 2; ++dir) {
      const double sign = dir == 0 ? 1.0 : -1.0;
      std::vector<C> h(n);
      for (int t = 0; t < n; ++t) {
        const double ang = 2.0 * M_PI * (double)t / (double)n;
        h[t] = mk<C>(std::cos(ang), sign * std::sin(ang));
      }
      C* dptr = nullptr;
      int rc = upload(&dptr, h.data(), h.size());
      if (rc) return rc;
      e->d.tw[prec][a][dir] = dptr;
    }
  }
  return AMA_OK;
}

void free_grid_filters(AmaEngine* e);

void free_engine(AmaEngine* e) {
  ama::bump_memory_epoch();
  free_grid_filters(e);
  nl_tc_free(e);
  auto f = [](void* p) { if (p) cudaFree(p); };
  f(e->d.plane_x); f(e->d.slot_of_x); f(e->d.entries); f(e->d.entry_start); f(e->d.rows);
  f(e->d.row_start); f(e->d.pw_off); f(e->d.npw); f(e->d.kin64); f(e->d.kin32); f(e->d.v64); f(e->d.v32);
  for (int p = 0; p < 2; ++p) {
    for (int a = 0; a < 3; ++a) for (int d = 0; d < 2; ++d) f(e->d.tw[p][a][d]);
    f(e->d.proj[p]); f(e->d.dproj[p]); f(e->work[p]); f(e->ws_proj[p]); f(e->ws_part[p]);
  }
  f(e->ws_dens);
  delete e;
}

}  // namespace

// ===================================================================== C-ABI
extern "C" int ama_engine_create(const AmaSystemDesc* desc, AmaEngine** out) {
  AMA_REQUIRE(desc && out, AMA_ERR_ARG, "null argument");
  *out = nullptr;
  AMA_REQUIRE(desc->nk >= 1 && desc->npw && desc->miller && desc->kinetic, AMA_ERR_ARG,
              "desc needs nk >= 1, npw, miller and kinetic");
  AMA_REQUIRE(desc->nspin == 1 || desc->nspin == 2, AMA_ERR_ARG, "nspin must be 1 or 2");
  AMA_REQUIRE(desc->nproj >= 0 && (desc->nproj == 0 || (desc->projectors && desc->dij)), AMA_ERR_ARG,
              "projectors and dij are required when nproj > 0");
  AMA_REQUIRE((desc->precisions & 3u) != 0, AMA_ERR_ARG, "no precision requested");
  AmaEngine* e = new AmaEngine();
  if (cudaGetDevice(&e->device) != cudaSuccess) {
    delete e;
    ama::set_error("ama_engine_create: no current CUDA device");
    return AMA_ERR_CUDA;
  }
  const int dims[3] = {desc->n1, desc->n2, desc->n3};
  for (int a = 0; a < 3; ++a) {
    if (dims[a] < 1 || !split_length(dims[a], &e->ax[a])) {
      delete e;
      ama::set_error("grid length " + std::to_string(dims[a]) +
                     " is not a product of two codelet lengths (1..16, no 13)");
      return AMA_ERR_UNSUPPORTED;
    }
  }
  const int n1 = dims[0], n2 = dims[1], n3 = dims[2];
  e->N = (int64_t)n1 * n2 * n3;
  e->nk = desc->nk;
  e->nspin = desc->nspin;
  e->nproj = desc->nproj;
  e->precisions = desc->precisions & 3u;
  e->npw.assign(desc->npw, desc->npw + desc->nk);
  e->pw_off.assign(e->nk + 1, 0);
  for (int k = 0; k < e->nk; ++k) {
    if (e->npw[k] < 1) { delete e; ama::set_error("npw must be positive"); return AMA_ERR_SHAPE; }
    e->pw_off[k + 1] = e->pw_off[k] + e->npw[k];
    e->max_npw = std::max(e->max_npw, e->npw[k]);
  }
  const int64_t total_pw = e->pw_off[e->nk];

  // x-plane slots: every natural x index that any k-point's sphere touches
  std::vector<int> x_used(n1, 0);
  for (int64_t g = 0; g < total_pw; ++g) {
    const int h = desc->miller[3 * g], kk = desc->miller[3 * g + 1], l = desc->miller[3 * g + 2];
    if (2 * std::abs(h) + 1 > n1 || 2 * std::abs(kk) + 1 > n2 || 2 * std::abs(l) + 1 > n3) {
      delete e;
      ama::set_error("grid is too small for the Miller indices of the spheres");
      return AMA_ERR_SHAPE;
    }
    x_used[((h % n1) + n1) % n1] = 1;
  }
  std::vector<int> plane_x, slot_of_x(n1, -1);
  for (int x = 0; x < n1; ++x)
    if (x_used[x]) { slot_of_x[x] = (int)plane_x.size(); plane_x.push_back(x); }
  e->nslots = (int)plane_x.size();
  const int ns = e->nslots;
  {  // is the slot set x <= hp, x >= n1 - hn (contiguous Miller range -hn .. hp)?
    int hp = -1, hn = 0;
    while (hp + 1 < n1 && x_used[hp + 1]) ++hp;
    while (hn + 1 < n1 - hp - 1 && x_used[n1 - 1 - hn]) ++hn;
    bool ok = hp >= 0;
    for (int x = 0; x < n1 && ok; ++x) ok = (x_used[x] != 0) == (x <= hp || x >= n1 - hn);
    if (ok) { e->slot_hp = hp; e->slot_hn = hn; }
  }

  // per (k, slot): sphere entries and the y rows they occupy
  std::vector<int2> entries(total_pw);
  std::vector<int> entry_start((size_t)e->nk * (ns + 1));
  std::vector<int> rows, row_start((size_t)e->nk * (ns + 1));
  for (int k = 0; k < e->nk; ++k) {
    const int64_t base = e->pw_off[k];
    const int np = e->npw[k];
    std::vector<int> count(ns, 0);
    std::vector<int> slot_g(np), pos_g(np);
    for (int g = 0; g < np; ++g) {
      const int32_t* m = desc->miller + 3 * (base + g);
      const int x = ((m[0] % n1) + n1) % n1, y = ((m[1] % n2) + n2) % n2, z = ((m[2] % n3) + n3) % n3;
      slot_g[g] = slot_of_x[x];
      pos_g[g] = y * n3 + z;
      count[slot_g[g]]++;
    }
    std::vector<int> start(ns + 1, 0);
    for (int s = 0; s < ns; ++s) start[s + 1] = start[s] + count[s];
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int g = 0; g < np; ++g) {
      const int s = slot_g[g];
      entries[base + fill[s]++] = make_int2(g, pos_g[g]);
    }
    for (int s = 0; s <= ns; ++s) entry_start[(size_t)k * (ns + 1) + s] = (int)(base + start[s]);
    for (int s = 0; s < ns; ++s) {
      row_start[(size_t)k * (ns + 1) + s] = (int)rows.size();
      std::vector<char> used(n2, 0);
      for (int t = start[s]; t < start[s + 1]; ++t) used[entries[base + t].y / n3] = 1;
      int cnt = 0;
      for (int y = 0; y < n2; ++y) if (used[y]) { rows.push_back(y); ++cnt; }
      e->max_rows = std::max(e->max_rows, cnt);
    }
    row_start[(size_t)k * (ns + 1) + ns] = (int)rows.size();
  }

  int rc = AMA_OK;
  std::vector<float> kin32(desc->kinetic, desc->kinetic + total_pw);
  std::vector<int64_t> pw_off(e->pw_off);
  if ((rc = upload(&e->d.plane_x, plane_x.data(), plane_x.size())) ||
      (rc = upload(&e->d.slot_of_x, slot_of_x.data(), slot_of_x.size())) ||
      (rc = upload(&e->d.entries, entries.data(), entries.size())) ||
      (rc = upload(&e->d.entry_start, entry_start.data(), entry_start.size())) ||
      (rc = upload(&e->d.rows, rows.data(), rows.size())) ||
      (rc = upload(&e->d.row_start, row_start.data(), row_start.size())) ||
      (rc = upload(&e->d.pw_off, pw_off.data(), pw_off.size())) ||
      (rc = upload(&e->d.npw, e->npw.data(), e->npw.size())) ||
      (rc = upload(&e->d.kin64, desc->kinetic, (size_t)total_pw)) ||
      (rc = upload(&e->d.kin32, kin32.data(), kin32.size()))) {
    free_engine(e);
    return rc;
  }
  for (int p = 0; p < 2; ++p) {
    if (!(e->precisions & (1u << p))) continue;
    rc = p == AMA_C64 ? upload_twiddles<float>(e, p) : upload_twiddles<double>(e, p);
    if (!rc) rc = p == AMA_C64 ? set_smem_limits<float>(e) : set_smem_limits<double>(e);
    if (rc) { free_engine(e); return rc; }
  }
  if (e->nproj > 0) {
    // D.B per k on the host: D is block-diagonal, so loop over its nonzeros only.
    const int np = e->nproj;
    std::vector<std::vector<std::pair<int, double>>> dnz(np);
    for (int i = 0; i < np; ++i)
      for (int j = 0; j < np; ++j)
        if (desc->dij[(size_t)i * np + j] != 0.0) dnz[i].push_back({j, desc->dij[(size_t)i * np + j]});
    const size_t nel = (size_t)total_pw * np;
    std::vector<double> db(2 * nel, 0.0);
    for (int k = 0; k < e->nk; ++k) {
      const size_t kb = (size_t)e->pw_off[k] * np;
      const int npk = e->npw[k];
      for (int i = 0; i < np; ++i) {
        double* dst = db.data() + 2 * (kb + (size_t)i * npk);
        for (auto& jd : dnz[i]) {
          const double* src = desc->projectors + 2 * (kb + (size_t)jd.first * npk);
          for (int g = 0; g < 2 * npk; ++g) dst[g] += jd.second * src[g];
        }
      }
    }
    for (int p = 0; p < 2 && !rc; ++p) {
      if (!(e->precisions & (1u << p))) continue;
      if (p == AMA_C128) {
        double2* b = nullptr; double2* d = nullptr;
        rc = upload(&b, (const double2*)desc->projectors, nel);
        if (!rc) rc = upload(&d, (const double2*)db.data(), nel);
        e->d.proj[p] = b; e->d.dproj[p] = d;
      } else {
        std::vector<float2> bf(nel), df(nel);
        for (size_t i = 0; i < nel; ++i) {
          bf[i] = make_float2((float)desc->projectors[2 * i], (float)desc->projectors[2 * i + 1]);
          df[i] = make_float2((float)db[2 * i], (float)db[2 * i + 1]);
        }
        float2* b = nullptr; float2* d = nullptr;
        rc = upload(&b, bf.data(), nel);
        if (!rc) rc = upload(&d, df.data(), nel);
        e->d.proj[p] = b; e->d.dproj[p] = d;
      }
    }
    if (rc) { free_engine(e); return rc; }
  }
  if (e->nproj > 0 && (e->precisions & (1u << AMA_C64))) {
    rc = nl_tc_setup(e);
    if (rc) { free_engine(e); return rc; }
  }
  if (int rc = ama::noalloc_prepare()) {  // the fixed grid array's address, before any capture
    free_engine(e);
    return rc;
  }
  *out = e;
  return AMA_OK;
}

extern "C" int ama_engine_destroy(AmaEngine* e) {
  if (!e) return AMA_OK;
  cudaDeviceSynchronize();
  free_engine(e);
  return AMA_OK;
}

extern "C" int ama_set_potential(AmaEngine* e, const double* v, int32_t nspin, void* stream) {
  AMA_REQUIRE(e && v, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(nspin == e->nspin, AMA_ERR_SHAPE, "potential spin channels do not match the engine");
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t N = e->N;
  if ((!e->d.v64 && (e->precisions & (1u << AMA_C128))) || (!e->d.v32 && (e->precisions & (1u << AMA_C64))))
    ama::bump_memory_epoch();
  if (!e->d.v64 && (e->precisions & (1u << AMA_C128)))
    AMA_CUDA_TRY(cudaMalloc((void**)&e->d.v64, (size_t)nspin * N * sizeof(double)));
  if (!e->d.v32 && (e->precisions & (1u << AMA_C64)))
    AMA_CUDA_TRY(cudaMalloc((void**)&e->d.v32, (size_t)nspin * N * sizeof(float)));
  const double scale = 1.0 / (double)N;
  for (int sp = 0; sp < nspin; ++sp) {
    if (e->d.v64)
      permute_potential_kernel<double><<<592, 256, 0, s>>>(v + sp * N, e->d.v64 + sp * N, e->ax[0].n, e->ax[1].n,
                                                           e->ax[2].n, e->ax[0].A, e->ax[0].B, e->ax[1].A,
                                                           e->ax[1].B, e->ax[2].A, e->ax[2].B, scale);
    if (e->d.v32)
      permute_potential_kernel<float><<<592, 256, 0, s>>>(v + sp * N, e->d.v32 + sp * N, e->ax[0].n, e->ax[1].n,
                                                          e->ax[2].n, e->ax[0].A, e->ax[0].B, e->ax[1].A,
                                                          e->ax[1].B, e->ax[2].A, e->ax[2].B, scale);
  }
  AMA_CHECK_LAUNCH();
  e->has_potential = true;
  return AMA_OK;
}

extern "C" int ama_reserve(AmaEngine* e, int32_t precision, int64_t max_bands) {
  AMA_REQUIRE(e, AMA_ERR_ARG, "null engine");
  int rc = prec_ok(e, precision);
  if (rc) return rc;
  return ensure_work(e, precision, max_bands);
}

static int check_call(AmaEngine* e, int precision, int k_first, int k_count, int nbands) {
  AMA_REQUIRE(e, AMA_ERR_ARG, "null engine");
  int rc = prec_ok(e, precision);
  if (rc) return rc;
  AMA_REQUIRE(k_first >= 0 && k_count >= 1 && k_first + k_count <= e->nk, AMA_ERR_SHAPE,
              "k-point range outside the engine's k-points");
  AMA_REQUIRE(nbands >= 1, AMA_ERR_SHAPE, "nbands must be positive");
  return AMA_OK;
}

extern "C" int ama_hpsi(AmaEngine* e, int32_t precision, int32_t k_first, int32_t k_count,
                        int32_t nbands, int32_t spin, const void* psi, void* hpsi, void* stream) {
  int rc = check_call(e, precision, k_first, k_count, nbands);
  if (rc) return rc;
  AMA_REQUIRE(psi && hpsi, AMA_ERR_ARG, "null psi/hpsi");
  AMA_REQUIRE(psi != hpsi, AMA_ERR_ARG, "hpsi must not alias psi");
  AMA_REQUIRE(spin >= 0 && spin < e->nspin, AMA_ERR_ARG, "spin out of range");
  AMA_REQUIRE(e->has_potential, AMA_ERR_ARG, "ama_set_potential has not been called");
  cudaStream_t s = (cudaStream_t)stream;
  return precision == AMA_C64 ? hpsi_impl<float>(e, k_first, k_count, nbands, spin, psi, hpsi, s)
                              : hpsi_impl<double>(e, k_first, k_count, nbands, spin, psi, hpsi, s);
}

extern "C" int ama_density_accumulate(AmaEngine* e, int32_t precision, int32_t k_first,
                                      int32_t k_count, int32_t nbands, const void* psi,
                                      const double* weights, double* rho, void* stream) {
  int rc = check_call(e, precision, k_first, k_count, nbands);
  if (rc) return rc;
  AMA_REQUIRE(psi && weights && rho, AMA_ERR_ARG, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  return precision == AMA_C64 ? density_impl<float>(e, k_first, k_count, nbands, psi, weights, rho, s)
                              : density_impl<double>(e, k_first, k_count, nbands, psi, weights, rho, s);
}

template <typename T>
static int project_impl(AmaEngine* e, int k, int nbands, const void* psi, void* out, cudaStream_t s) {
  using C = cx_t<T>;
  const int p = std::is_same<T, float>::value ? AMA_C64 : AMA_C128;
  const int tiles = (int)std::min<int64_t>(gemm_tile_count<T>(nbands, e->nproj, 1), 1 << 30);
  int splits = std::max(1, std::min(64, (4 * 148 + tiles - 1) / tiles));
  splits = std::min(splits, std::max(1, e->npw[k] / 256));
  const int64_t pstride = (int64_t)nbands * e->nproj;
  if (splits > 1)
    AMA_CUDA_TRY(grow<char>(&e->ws_part[p], &e->ws_part_bytes[p], (size_t)splits * pstride * sizeof(double2)));
  ProjectBatch<C> pb{(const C*)psi, (const C*)e->d.proj[p], (C*)out, e->d.pw_off, e->d.npw, k, nbands, e->nproj};
  AMA_CUDA_TRY((launch_cgemm<T, kNC>(pb, 1, nbands, e->nproj, splits, mk<C>(1, 0), mk<C>(0, 0),
                                     (double2*)e->ws_part[p], pstride, s)));
  return AMA_OK;
}

extern "C" int ama_project(AmaEngine* e, int32_t precision, int32_t k, int32_t nbands,
                           const void* psi, void* proj, void* stream) {
  int rc = check_call(e, precision, k, 1, nbands);
  if (rc) return rc;
  AMA_REQUIRE(psi && proj, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(e->nproj > 0, AMA_ERR_SHAPE, "the engine has no projectors");
  cudaStream_t s = (cudaStream_t)stream;
  return precision == AMA_C64 ? project_impl<float>(e, k, nbands, psi, proj, s)
                              : project_impl<double>(e, k, nbands, psi, proj, s);
}

// ============================================================ grid filters
// out(r) = Re sum_G f(G) rho(G) e^{iGr},  rho(G) = (1/N) sum_r rho(r) e^{-iGr},
// energy += sum_G f_e(G) |rho(G)|^2. Three stages like H.psi but over every plane:
// G1 forward z,y per x-plane; G2 forward x, filter, backward x per y; G3 backward y,z.
// The filter is stored in the storage order of the forward transform's output.
namespace {

struct GridView {
  int n1, n2, n3, A1, B1, A2, B2, A3, B3;
  int64_t plane_elems;
};

GridView grid_view(const AmaEngine* e) {
  GridView g;
  g.n1 = e->ax[0].n; g.n2 = e->ax[1].n; g.n3 = e->ax[2].n;
  g.A1 = e->ax[0].A; g.B1 = e->ax[0].B; g.A2 = e->ax[1].A; g.B2 = e->ax[1].B;
  g.A3 = e->ax[2].A; g.B3 = e->ax[2].B;
  g.plane_elems = (int64_t)g.n2 * g.n3;
  return g;
}

__global__ void __launch_bounds__(kFftThreads) grid_g1_kernel(GridView g, const double2* tw_y, const double2* tw_z,
                               const double* __restrict__ in, double2* __restrict__ work) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* plane = reinterpret_cast<double2*>(smem_raw);
  double2* sty = plane + g.plane_elems;
  double2* stz = sty + g.n2;
  int* rows = reinterpret_cast<int*>(stz + g.n3);
  const int x = blockIdx.x;
  load_twiddles(sty, tw_y, g.n2);
  load_twiddles(stz, tw_z, g.n3);
  for (int i = threadIdx.x; i < g.n2; i += blockDim.x) rows[i] = i;
  const double* src = in + (int64_t)x * g.plane_elems;
  for (int64_t i = threadIdx.x; i < g.plane_elems; i += blockDim.x) plane[i] = make_double2(src[i], 0.0);
  __syncthreads();
  dft_rows<-1, true>(plane, g.n3, g.A3, g.B3, g.n3, rows, g.n2, stz);
  dft_cols<-1, true>(plane, g.n2, g.A2, g.B2, g.n3, sty);
  double2* dst = work + (int64_t)x * g.plane_elems;
  for (int64_t i = threadIdx.x; i < g.plane_elems; i += blockDim.x) dst[i] = plane[i];
}

__global__ void __launch_bounds__(kFftThreads) grid_g2_kernel(GridView g, const double2* tw_f, const double2* tw_b,
                               const double* __restrict__ filt, const double* __restrict__ efilt,
                               double scale, double escale, double2* __restrict__ work,
                               double* __restrict__ energy) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* slab = reinterpret_cast<double2*>(smem_raw);
  double2* twf = slab + (int64_t)g.n1 * g.n3;
  double2* twb = twf + g.n1;
  __shared__ double red[32];
  const int y = blockIdx.x;
  load_twiddles(twf, tw_f, g.n1);
  load_twiddles(twb, tw_b, g.n1);
  double2* wb = work + (int64_t)y * g.n3;
  const int total = g.n1 * g.n3;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int x = e / g.n3, z = e % g.n3;
    slab[e] = wb[(int64_t)x * g.plane_elems + z];
  }
  __syncthreads();
  dft_cols<-1, true>(slab, g.n1, g.A1, g.B1, g.n3, twf);
  const int64_t xstride = g.plane_elems;
  double acc = 0.0;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int x = e / g.n3, z = e % g.n3;
    const int64_t gi = x * xstride + (int64_t)y * g.n3 + z;
    const double2 c = slab[e];
    if (efilt) acc += efilt[gi] * (c.x * c.x + c.y * c.y);
    const double f = filt[gi] * scale;
    slab[e] = make_double2(c.x * f, c.y * f);
  }
  if (energy) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  }
  __syncthreads();
  if (energy && threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    atomicAdd(energy, t * escale);
  }
  dft_cols<+1, false>(slab, g.n1, g.A1, g.B1, g.n3, twb);
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int x = e / g.n3, z = e % g.n3;
    wb[(int64_t)x * g.plane_elems + z] = slab[e];
  }
}

__global__ void __launch_bounds__(kFftThreads) grid_g3_kernel(GridView g, const double2* tw_y, const double2* tw_z,
                               const double2* __restrict__ work, double* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* plane = reinterpret_cast<double2*>(smem_raw);
  double2* sty = plane + g.plane_elems;
  double2* stz = sty + g.n2;
  int* rows = reinterpret_cast<int*>(stz + g.n3);
  const int x = blockIdx.x;
  load_twiddles(sty, tw_y, g.n2);
  load_twiddles(stz, tw_z, g.n3);
  for (int i = threadIdx.x; i < g.n2; i += blockDim.x) rows[i] = i;
  const double2* src = work + (int64_t)x * g.plane_elems;
  for (int64_t i = threadIdx.x; i < g.plane_elems; i += blockDim.x) plane[i] = src[i];
  __syncthreads();
  dft_cols<+1, false>(plane, g.n2, g.A2, g.B2, g.n3, sty);
  dft_rows<+1, false>(plane, g.n3, g.A3, g.B3, g.n3, rows, g.n2, stz);
  double* dst = out + (int64_t)x * g.plane_elems;
  for (int64_t i = threadIdx.x; i < g.plane_elems; i += blockDim.x) dst[i] = plane[i].x;
}

}  // namespace

namespace {
// Forward x transform of the G1 output and scatter to natural (x, y, z) order with 1/N:
// out[G] = (1/N) sum_r in(r) e^{-iG.r}.
__global__ void __launch_bounds__(kFftThreads) grid_g2f_kernel(GridView g, const double2* tw_f, const double2* __restrict__ work,
                                double2* __restrict__ out, double scale) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* slab = reinterpret_cast<double2*>(smem_raw);
  double2* twf = slab + (int64_t)g.n1 * g.n3;
  const int p2 = blockIdx.x;
  load_twiddles(twf, tw_f, g.n1);
  const double2* wb = work + (int64_t)p2 * g.n3;
  const int total = g.n1 * g.n3;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int x = e / g.n3, z = e % g.n3;
    slab[e] = wb[(int64_t)x * g.plane_elems + z];
  }
  __syncthreads();
  dft_cols<-1, true>(slab, g.n1, g.A1, g.B1, g.n3, twf);
  const int y = p2 / g.B2 + g.A2 * (p2 % g.B2);
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int p1 = e / g.n3, p3 = e % g.n3;
    const int x = p1 / g.B1 + g.A1 * (p1 % g.B1);
    const int z = p3 / g.B3 + g.A3 * (p3 % g.B3);
    const double2 c = slab[e];
    out[((int64_t)x * g.n2 + y) * g.n3 + z] = make_double2(c.x * scale, c.y * scale);
  }
}
}  // namespace

namespace {
// i G_a / N (times a caller scale) at the forward transform's storage position (p1, p2, p3):
// G = sum_i m_i b_i with m the signed frequency of each axis, zero at the Nyquist frequency
// of an even axis (the spectral derivative of a real field stays real).
struct Recip {
  double b[3][3];  // rows: reciprocal lattice vectors b_1, b_2, b_3 (Cartesian, 1/Bohr)
};

__device__ __forceinline__ int signed_freq(int p, int n, int A, int B) {
  const int f = p / B + A * (p % B);  // natural frequency index held at storage position p
  if (2 * f == n) return 0;           // Nyquist of an even axis
  return 2 * f > n ? f - n : f;
}

// G2 of the spectral gradient: slab y of the G1 output, forward x, times i G_a scale / N,
// backward x, into work_out + a N (a = blockIdx.y).
__global__ void __launch_bounds__(kFftThreads) grid_g2_grad_kernel(GridView g, const double2* tw_f, const double2* tw_b,
                                    Recip rc, double scale, const double2* __restrict__ work_in,
                                    double2* __restrict__ work_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* slab = reinterpret_cast<double2*>(smem_raw);
  double2* twf = slab + (int64_t)g.n1 * g.n3;
  double2* twb = twf + g.n1;
  const int p2 = blockIdx.x, axis = blockIdx.y;
  load_twiddles(twf, tw_f, g.n1);
  load_twiddles(twb, tw_b, g.n1);
  const double2* wb = work_in + (int64_t)p2 * g.n3;
  const int total = g.n1 * g.n3;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int x = e / g.n3, z = e % g.n3;
    slab[e] = wb[(int64_t)x * g.plane_elems + z];
  }
  __syncthreads();
  dft_cols<-1, true>(slab, g.n1, g.A1, g.B1, g.n3, twf);
  const int m2 = signed_freq(p2, g.n2, g.A2, g.B2);
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int p1 = e / g.n3, p3 = e % g.n3;
    const int m1 = signed_freq(p1, g.n1, g.A1, g.B1), m3 = signed_freq(p3, g.n3, g.A3, g.B3);
    const double ga = (m1 * rc.b[0][axis] + m2 * rc.b[1][axis] + m3 * rc.b[2][axis]) * scale;
    const double2 c = slab[e];
    slab[e] = make_double2(-ga * c.y, ga * c.x);  // i G_a c
  }
  __syncthreads();
  dft_cols<+1, false>(slab, g.n1, g.A1, g.B1, g.n3, twb);
  double2* ob = work_out + (int64_t)axis * g.n1 * g.plane_elems + (int64_t)p2 * g.n3;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int x = e / g.n3, z = e % g.n3;
    ob[(int64_t)x * g.plane_elems + z] = slab[e];
  }
}

// G2 of the spectral divergence: for each component a, slab y of its G1 output (work + a N),
// forward x, times i G_a scale / N, summed over a (the running sum kept in component 0's
// slab, which only this CTA touches), then backward x into component 0.
__global__ void __launch_bounds__(kFftThreads) grid_g2_div_kernel(GridView g, const double2* tw_f, const double2* tw_b,
                                   Recip rc, double scale, double2* __restrict__ work) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* slab = reinterpret_cast<double2*>(smem_raw);
  double2* twf = slab + (int64_t)g.n1 * g.n3;
  double2* twb = twf + g.n1;
  const int p2 = blockIdx.x;
  load_twiddles(twf, tw_f, g.n1);
  load_twiddles(twb, tw_b, g.n1);
  const int total = g.n1 * g.n3;
  const int64_t field = (int64_t)g.n1 * g.plane_elems;
  double2* acc = work + (int64_t)p2 * g.n3;
  const int m2 = signed_freq(p2, g.n2, g.A2, g.B2);
  for (int axis = 0; axis < 3; ++axis) {
    const double2* wb = work + axis * field + (int64_t)p2 * g.n3;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int x = e / g.n3, z = e % g.n3;
      slab[e] = wb[(int64_t)x * g.plane_elems + z];
    }
    __syncthreads();
    dft_cols<-1, true>(slab, g.n1, g.A1, g.B1, g.n3, twf);
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int p1 = e / g.n3, p3 = e % g.n3;
      const int m1 = signed_freq(p1, g.n1, g.A1, g.B1), m3 = signed_freq(p3, g.n3, g.A3, g.B3);
      const double ga = (m1 * rc.b[0][axis] + m2 * rc.b[1][axis] + m3 * rc.b[2][axis]) * scale;
      const double2 c = slab[e];
      double2 t = make_double2(-ga * c.y, ga * c.x);
      const int64_t gi = (int64_t)p1 * g.plane_elems + p3;  // this thread's own element
      if (axis > 0) {
        const double2 prev = acc[gi];
        t.x += prev.x;
        t.y += prev.y;
      }
      if (axis < 2) acc[gi] = t;
      else slab[e] = t;
    }
    __syncthreads();
  }
  dft_cols<+1, false>(slab, g.n1, g.A1, g.B1, g.n3, twb);
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int x = e / g.n3, z = e % g.n3;
    acc[(int64_t)x * g.plane_elems + z] = slab[e];
  }
}

// G3 that adds: out = beta out + alpha Re(backward y, z of the plane).
__global__ void __launch_bounds__(kFftThreads) grid_g3_axpy_kernel(GridView g, const double2* tw_y, const double2* tw_z,
                                    const double2* __restrict__ work, double alpha, double beta,
                                    double* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* plane = reinterpret_cast<double2*>(smem_raw);
  double2* sty = plane + g.plane_elems;
  double2* stz = sty + g.n2;
  int* rows = reinterpret_cast<int*>(stz + g.n3);
  const int x = blockIdx.x;
  load_twiddles(sty, tw_y, g.n2);
  load_twiddles(stz, tw_z, g.n3);
  for (int i = threadIdx.x; i < g.n2; i += blockDim.x) rows[i] = i;
  const double2* src = work + (int64_t)x * g.plane_elems;
  for (int64_t i = threadIdx.x; i < g.plane_elems; i += blockDim.x) plane[i] = src[i];
  __syncthreads();
  dft_cols<+1, false>(plane, g.n2, g.A2, g.B2, g.n3, sty);
  dft_rows<+1, false>(plane, g.n3, g.A3, g.B3, g.n3, rows, g.n2, stz);
  double* dst = out + (int64_t)x * g.plane_elems;
  for (int64_t i = threadIdx.x; i < g.plane_elems; i += blockDim.x)
    dst[i] = (beta == 0.0 ? 0.0 : beta * dst[i]) + alpha * plane[i].x;
}
}  // namespace

namespace {
void free_grid_filters(AmaEngine* e) {
  ama::bump_memory_epoch();
  for (double*& p : e->grid_filt) {
    if (p) cudaFree(p);
    p = nullptr;
  }
  if (e->grid_work) cudaFree(e->grid_work);
  e->grid_work = nullptr;
  e->grid_work_bytes = 0;
}

int ensure_grid_work(AmaEngine* e, int fields = 1) {
  const size_t need = (size_t)fields * e->N * sizeof(double2);
  if (e->grid_work_bytes >= need) return AMA_OK;
  ama::bump_memory_epoch();
  if (e->grid_work) cudaFree(e->grid_work);
  e->grid_work = nullptr;
  e->grid_work_bytes = 0;
  AMA_CUDA_TRY(cudaMalloc((void**)&e->grid_work, need));
  e->grid_work_bytes = need;
  return AMA_OK;
}

// The engine's tables live on the device that was current at ama_engine_create.
int require_engine_device(const AmaEngine* e) {
  int dev = 0;
  AMA_CUDA_TRY(cudaGetDevice(&dev));
  AMA_REQUIRE(dev == e->device, AMA_ERR_ARG,
              "the engine was created on device " + std::to_string(e->device) + " but device " +
                  std::to_string(dev) + " is current");
  return AMA_OK;
}
}  // namespace

extern "C" int ama_set_grid_filter(AmaEngine* e, int32_t slot, const double* filter) {
  AMA_REQUIRE(e && filter, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(slot >= 0 && slot < 4, AMA_ERR_ARG, "filter slot must be 0..3");
  AMA_REQUIRE(e->precisions & (1u << AMA_C128), AMA_ERR_ARG, "grid filters need the complex128 tables");
  const int n1 = e->ax[0].n, n2 = e->ax[1].n, n3 = e->ax[2].n;
  std::vector<double> perm((size_t)e->N);
  for (int p1 = 0; p1 < n1; ++p1) {
    const int x = p1 / e->ax[0].B + e->ax[0].A * (p1 % e->ax[0].B);
    for (int p2 = 0; p2 < n2; ++p2) {
      const int y = p2 / e->ax[1].B + e->ax[1].A * (p2 % e->ax[1].B);
      for (int p3 = 0; p3 < n3; ++p3) {
        const int z = p3 / e->ax[2].B + e->ax[2].A * (p3 % e->ax[2].B);
        perm[((size_t)p1 * n2 + p2) * n3 + p3] = filter[((size_t)x * n2 + y) * n3 + z];
      }
    }
  }
  if (int rc = require_engine_device(e)) return rc;
  if (!e->grid_filt[slot]) ama::bump_memory_epoch();
  if (!e->grid_filt[slot]) AMA_CUDA_TRY(cudaMalloc((void**)&e->grid_filt[slot], (size_t)e->N * sizeof(double)));
  AMA_CUDA_TRY(cudaMemcpy(e->grid_filt[slot], perm.data(), (size_t)e->N * sizeof(double), cudaMemcpyHostToDevice));
  return AMA_OK;
}

extern "C" int ama_grid_filter(AmaEngine* e, int32_t slot, int32_t energy_slot, const double* in,
                               double* out, double* energy, void* stream) {
  AMA_REQUIRE(e && in && out, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(slot >= 0 && slot < 4 && energy_slot >= -1 && energy_slot < 4, AMA_ERR_ARG, "bad slot");
  AMA_REQUIRE(e->grid_filt[slot], AMA_ERR_ARG, "filter slot not set");
  const double* ef = nullptr;
  if (energy_slot >= 0) {
    ef = e->grid_filt[energy_slot];
    AMA_REQUIRE(ef && energy, AMA_ERR_ARG, "energy filter slot not set or energy is null");
  }
  if (int rc = require_engine_device(e)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (int rc = ensure_grid_work(e)) return rc;
  GridView g = grid_view(e);
  const size_t ps = plane_smem<double>(e), ss = slab_smem<double>(e);
  AMA_CUDA_TRY(cudaFuncSetAttribute(grid_g1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps));
  AMA_CUDA_TRY(cudaFuncSetAttribute(grid_g3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps));
  AMA_CUDA_TRY(cudaFuncSetAttribute(grid_g2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ss));
  auto T = [&](int axis, int dir) { return (const double2*)e->d.tw[AMA_C128][axis][dir]; };
  const double invN = 1.0 / (double)e->N;
  grid_g1_kernel<<<g.n1, kFftThreads, ps, s>>>(g, T(1, 1), T(2, 1), in, e->grid_work);
  AMA_CHECK_LAUNCH();
  grid_g2_kernel<<<g.n2, kFftThreads, ss, s>>>(g, T(0, 1), T(0, 0), e->grid_filt[slot], ef, invN,
                                                  invN * invN, e->grid_work, energy);
  AMA_CHECK_LAUNCH();
  grid_g3_kernel<<<g.n1, kFftThreads, ps, s>>>(g, T(1, 0), T(2, 0), e->grid_work, out);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_grid_fft_forward(AmaEngine* e, const double* in, void* out, void* stream) {
  AMA_REQUIRE(e && in && out, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(e->precisions & (1u << AMA_C128), AMA_ERR_ARG, "grid transforms need the complex128 tables");
  if (int rc = require_engine_device(e)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (int rc = ensure_grid_work(e)) return rc;
  GridView g = grid_view(e);
  const size_t ps = plane_smem<double>(e), ss = slab_smem<double>(e);
  AMA_CUDA_TRY(cudaFuncSetAttribute(grid_g1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps));
  AMA_CUDA_TRY(cudaFuncSetAttribute(grid_g2f_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ss));
  auto T = [&](int axis, int dir) { return (const double2*)e->d.tw[AMA_C128][axis][dir]; };
  grid_g1_kernel<<<g.n1, kFftThreads, ps, s>>>(g, T(1, 1), T(2, 1), in, e->grid_work);
  AMA_CHECK_LAUNCH();
  grid_g2f_kernel<<<g.n2, kFftThreads, ss, s>>>(g, T(0, 1), e->grid_work, (double2*)out, 1.0 / (double)e->N);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

namespace {
Recip recip_of(const double* cell) {
  // b_i = 2 pi (inverse of the cell matrix whose rows are a_1, a_2, a_3), transposed
  const double* a = cell;
  const double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                     a[2] * (a[3] * a[7] - a[4] * a[6]);
  const double f = 2.0 * M_PI / det;
  Recip r;
  // b_1 = 2 pi (a_2 x a_3) / det, and cyclically
  const int nx[3][2] = {{1, 2}, {2, 0}, {0, 1}};
  for (int i = 0; i < 3; ++i) {
    const double* u = a + 3 * nx[i][0];
    const double* v = a + 3 * nx[i][1];
    r.b[i][0] = f * (u[1] * v[2] - u[2] * v[1]);
    r.b[i][1] = f * (u[2] * v[0] - u[0] * v[2]);
    r.b[i][2] = f * (u[0] * v[1] - u[1] * v[0]);
  }
  return r;
}

int grid_prepare(AmaEngine* e, int fields) {
  AMA_REQUIRE(e->precisions & (1u << AMA_C128), AMA_ERR_ARG, "grid transforms need the complex128 tables");
  if (int rc = require_engine_device(e)) return rc;
  if (int rc = ensure_grid_work(e, fields)) return rc;
  const size_t ps = plane_smem<double>(e), ss = slab_smem<double>(e);
  AMA_CUDA_TRY(cudaFuncSetAttribute(grid_g1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps));
  AMA_CUDA_TRY(cudaFuncSetAttribute(grid_g3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps));
  AMA_CUDA_TRY(cudaFuncSetAttribute(grid_g3_axpy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps));
  AMA_CUDA_TRY(cudaFuncSetAttribute(grid_g2_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ss));
  AMA_CUDA_TRY(cudaFuncSetAttribute(grid_g2_div_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ss));
  return AMA_OK;
}
}  // namespace

extern "C" int ama_grid_gradient(AmaEngine* e, const double* cell, const double* in, double scale, double* out,
                                 void* stream) {
  AMA_REQUIRE(e && cell && in && out, AMA_ERR_ARG, "null argument");
  if (int rc = grid_prepare(e, 4)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  GridView g = grid_view(e);
  const size_t ps = plane_smem<double>(e), ss = slab_smem<double>(e);
  auto T = [&](int axis, int dir) { return (const double2*)e->d.tw[AMA_C128][axis][dir]; };
  double2* w0 = e->grid_work;
  double2* w1 = w0 + e->N;  // three outputs follow the G1 field
  grid_g1_kernel<<<g.n1, kFftThreads, ps, s>>>(g, T(1, 1), T(2, 1), in, w0);
  AMA_CHECK_LAUNCH();
  grid_g2_grad_kernel<<<dim3(g.n2, 3), kFftThreads, ss, s>>>(g, T(0, 1), T(0, 0), recip_of(cell),
                                                              scale / (double)e->N, w0, w1);
  AMA_CHECK_LAUNCH();
  for (int a = 0; a < 3; ++a) {
    grid_g3_kernel<<<g.n1, kFftThreads, ps, s>>>(g, T(1, 0), T(2, 0), w1 + a * e->N, out + a * e->N);
    AMA_CHECK_LAUNCH();
  }
  return AMA_OK;
}

extern "C" int ama_grid_divergence(AmaEngine* e, const double* cell, const double* in, double alpha, double beta,
                                   double* out, void* stream) {
  AMA_REQUIRE(e && cell && in && out, AMA_ERR_ARG, "null argument");
  if (int rc = grid_prepare(e, 3)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  GridView g = grid_view(e);
  const size_t ps = plane_smem<double>(e), ss = slab_smem<double>(e);
  auto T = [&](int axis, int dir) { return (const double2*)e->d.tw[AMA_C128][axis][dir]; };
  double2* w = e->grid_work;
  for (int a = 0; a < 3; ++a) {
    grid_g1_kernel<<<g.n1, kFftThreads, ps, s>>>(g, T(1, 1), T(2, 1), in + a * e->N, w + a * e->N);
    AMA_CHECK_LAUNCH();
  }
  grid_g2_div_kernel<<<g.n2, kFftThreads, ss, s>>>(g, T(0, 1), T(0, 0), recip_of(cell), 1.0 / (double)e->N, w);
  AMA_CHECK_LAUNCH();
  grid_g3_axpy_kernel<<<g.n1, kFftThreads, ps, s>>>(g, T(1, 0), T(2, 0), w, alpha, beta, out);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_engine_option(AmaEngine* e, int32_t option, int32_t value) {
  AMA_REQUIRE(e, AMA_ERR_ARG, "null engine");
  if (option != 4) ama::bump_memory_epoch();  // captured graphs hold the previous kernels and shapes
  switch (option) {
    case 0:  // nonlocal products of the complex64 path on the tensor cores (1) or SIMT (0)
      e->use_tc = value != 0;
      return AMA_OK;
    case 1:  // complex64 stage B variant: 0 shared memory, 1 register, 2 register + slot set,
             // 3 register, two threads per column, 4 shared memory split along z
    case 2: {  // complex128 stage B variant (0 and, on long lines, 4)
      const int p = option == 1 ? AMA_C64 : AMA_C128;
      AMA_REQUIRE(e->precisions & (1u << p), AMA_ERR_ARG, "the engine was created without this precision");
      AMA_REQUIRE(value >= 0 && value < 5, AMA_ERR_ARG, "stage B variant must be 0 .. 4");
      AMA_REQUIRE(e->b_variant[p][value] != nullptr, AMA_ERR_UNSUPPORTED,
                  "this stage B variant is not compiled for the engine's grid");
      e->stage_fn[p][1] = e->b_variant[p][value];
      e->regb[p] = value >= 1 && value <= 3;
      e->bthreads[p] = value == 3 ? 2 : 1;
      e->zsplit[p] = e->b_zsplit[p][value];
      return AMA_OK;
    }
    case 3: {  // complex64 stages A and C: 0 shared-memory y passes, 1 y in registers (4 lanes)
      AMA_REQUIRE(e->precisions & (1u << AMA_C64), AMA_ERR_ARG, "the engine was created without complex64");
      AMA_REQUIRE(value == 0 || value == 1, AMA_ERR_ARG, "stage A/C variant must be 0 or 1");
      AMA_REQUIRE(e->ac_variant[AMA_C64][value][0] != nullptr, AMA_ERR_UNSUPPORTED,
                  "this stage A/C variant is not compiled for the engine's grid");
      e->stage_fn[AMA_C64][0] = e->ac_variant[AMA_C64][value][0];
      e->stage_fn[AMA_C64][2] = e->ac_variant[AMA_C64][value][1];
      e->ac_threads[AMA_C64] = e->ac_threads_of[AMA_C64][value];
      return AMA_OK;
    }
    case 4:  // ama_davidson: iteration segments replayed as CUDA graphs (1, default) or launched (0)
      e->dav_graphs = value != 0;
      return AMA_OK;
    default:
      ama::set_error("unknown engine option");
      return AMA_ERR_ARG;
  }
}

// ============================================= grid filter without allocation
// Some callers cannot let a library call cudaMalloc: applications whose device memory is
// owned by a framework allocator that has already reserved most of the GPU (a cudaMalloc
// from inside the library then fails or fragments that pool), and latency-sensitive loops
// in which the implicit device-wide synchronisation of cudaMalloc/cudaFree is not
// acceptable. For them, ama_grid_filter_noalloc runs the same three-stage filter as
// ama_grid_filter with its complex work grid in a fixed file-scope device array instead
// of the lazily grown allocation. The array holds kNoAllocGridPoints complex FP64 values
// (128^3 points, 32 MiB) and lives on every GPU that loads the library until the process
// exits. Its device address is looked up (cudaGetSymbolAddress, with the device current)
// when an engine is created on that device, which also loads the library's device code
// there under lazy module loading, so the array is in place before a framework allocator
// reserves the rest of the GPU; a call on a device without an engine looks it up on its
// first use, which should then come before any stream capture. The library does not
// survive a cudaDeviceReset of a device it has used. Every call shares the array and
// overwrites it completely before reading it, so nothing needs clearing between calls;
// calls that overlap on the GPU (different streams, no ordering between them) race on the
// array.
namespace {
constexpr int64_t kNoAllocGridPoints = 128 * 128 * 128;
__device__ __align__(256) double2 g_noalloc_grid[kNoAllocGridPoints];
std::atomic<void*> g_noalloc_addr[kMaxDevices];

// The array's device address on the current device (looked up once per device).
int noalloc_address(double2** out) {
  const int dev = current_device();
  AMA_REQUIRE(dev >= 0, AMA_ERR_UNSUPPORTED, "device index out of range");
  void* addr = g_noalloc_addr[dev].load(std::memory_order_acquire);
  if (!addr) {
    AMA_CUDA_TRY(cudaGetSymbolAddress(&addr, g_noalloc_grid));
    g_noalloc_addr[dev].store(addr, std::memory_order_release);  // every thread finds the same address
  }
  *out = static_cast<double2*>(addr);
  return AMA_OK;
}
}  // namespace

namespace ama {
int noalloc_prepare() {
  double2* unused = nullptr;
  return noalloc_address(&unused);
}
}  // namespace ama

extern "C" int ama_grid_filter_noalloc(AmaEngine* e, int32_t slot, int32_t energy_slot, const double* in,
                                       double* out, double* energy, void* stream) {
  AMA_REQUIRE(e && in && out, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(slot >= 0 && slot < 4 && energy_slot >= -1 && energy_slot < 4, AMA_ERR_ARG, "bad slot");
  AMA_REQUIRE(e->N <= kNoAllocGridPoints, AMA_ERR_SHAPE,
              "ama_grid_filter_noalloc: grid of " + std::to_string(e->N) + " points exceeds the fixed work array of " +
                  std::to_string(kNoAllocGridPoints) + " points (use ama_grid_filter)");
  AMA_REQUIRE(e->grid_filt[slot], AMA_ERR_ARG, "filter slot not set");
  const double* ef = nullptr;
  if (energy_slot >= 0) {
    ef = e->grid_filt[energy_slot];
    AMA_REQUIRE(ef && energy, AMA_ERR_ARG, "energy filter slot not set or energy is null");
  }
  if (int rc = require_engine_device(e)) return rc;
  double2* work = nullptr;
  if (int rc = noalloc_address(&work)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  GridView g = grid_view(e);
  const size_t ps = plane_smem<double>(e), ss = slab_smem<double>(e);
  AMA_CUDA_TRY(cudaFuncSetAttribute(grid_g1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps));
  AMA_CUDA_TRY(cudaFuncSetAttribute(grid_g3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps));
  AMA_CUDA_TRY(cudaFuncSetAttribute(grid_g2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ss));
  auto T = [&](int axis, int dir) { return (const double2*)e->d.tw[AMA_C128][axis][dir]; };
  const double invN = 1.0 / (double)e->N;
  grid_g1_kernel<<<g.n1, kFftThreads, ps, s>>>(g, T(1, 1), T(2, 1), in, work);
  AMA_CHECK_LAUNCH();
  grid_g2_kernel<<<g.n2, kFftThreads, ss, s>>>(g, T(0, 1), T(0, 0), e->grid_filt[slot], ef, invN, invN * invN,
                                                work, energy);
  AMA_CHECK_LAUNCH();
  grid_g3_kernel<<<g.n1, kFftThreads, ps, s>>>(g, T(1, 0), T(2, 0), work, out);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}
