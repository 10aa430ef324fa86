// Block Davidson for the lowest eigenpairs at every k-point of an engine, all k-points in
// lockstep, orchestrated from C++ (ama_davidson): no interpreter between the launches.
//
// Per k-point this is the reference's algorithm (amaterasu scf/eigen/davidson.py:48-111):
// Rayleigh-Ritz over the basis, residuals of the Ritz pairs, Teter-Payne-Allan corrections
// of the bands whose residual norm is above the tolerance, two projections off the basis,
// directions below 1e-7 of the largest dropped, orthonormalisation, H applied to the new
// block, the basis extended, and collapsed onto the Ritz vectors when one more block would
// not fit under 4 nbands. Batched over k, every step is one launch over all k-points (ragged
// plane-wave counts). A k-point with fewer new directions than the others carries zero
// rows marked invalid; their Rayleigh-Ritz diagonal is set just above that k-point's
// Gershgorin bound, which decouples them without inflating the matrix norm.
//
// The host synchronises twice per iteration for all k-points together, and every shape
// decision is made there: (1) after the residual norms (how many bands are active: the
// block width nn), (2) after the rank test of the new directions and their overlap's
// distance from the identity (whether any direction survived; whether the Newton-Schulz
// orthonormalisation is admissible, the overlap within 0.5 of the identity in Frobenius
// norm, and how many of its steps are needed; otherwise the overlap is decomposed). Which
// bands are active, which rows are valid and the eigenvalues stay on the device. The work
// between two synchronisations is a segment whose launches depend only on (basis size,
// block width, Newton-Schulz steps); a segment seen before is captured once as a CUDA graph
// and replayed from then on (every buffer it touches is owned by the library and the
// library's allocation generation tells when a pointer in a graph went stale). Segments
// whose eigensolves are above the batched Jacobi order run launch by launch: their kernels
// are long and the tridiagonal reduction is a cooperative launch.
//
// Orthonormalisation: the rank-revealing pass uses the overlap's eigendecomposition (which
// spans the same space as the reference's SVD); the second pass (the reference's Cholesky)
// is the Newton-Schulz iteration for S^{-1/2} on FP64 GEMMs, a symmetric orthonormalisation
// of rows that are already orthonormal to rounding there. The Ritz pairs agree.
#include "common.cuh"
#include "engine_impl.cuh"

#include <algorithm>
#include <array>
#include <cmath>
#include <vector>

using namespace ama;

namespace {

constexpr int kSmT = 256;
constexpr int kJacobiMax = 80;
constexpr double kGap = 1.0;  // Ha above the Gershgorin bound for invalid rows
constexpr int kGraphCacheMax = 48;  // executable graphs kept per device and host thread

// out[k][i][j] = v_i v_j (a'_ij + conj(a'_ji)) / 2 + (1 - v_i) delta_ij inval_diag,
// a' = conj(a) when conj_in, a the k-th (n x n) block (row-major, leading dimension n) of
// `in`; v = valid[k * vstride + i] (all valid when null).
template <typename T>
__global__ void __launch_bounds__(kSmT) small_hermitise_kernel(const cx_t<T>* __restrict__ in, double2* __restrict__ out,
                                                               int nk, int n, int conj_in, const uint8_t* __restrict__ valid,
                                                               int vstride, double inval_diag) {
  const int64_t per = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)kSmT + threadIdx.x; t < per * nk; t += (int64_t)gridDim.x * kSmT) {
    const int k = (int)(t / per);
    const int64_t r = t - k * per;
    const int i = (int)(r / n), j = (int)(r - (int64_t)i * n);
    const cx_t<T> a = in[k * per + (int64_t)i * n + j], b = in[k * per + (int64_t)j * n + i];
    double ax = a.x, ay = conj_in ? -(double)a.y : (double)a.y;
    double bx = b.x, by = conj_in ? -(double)b.y : (double)b.y;
    double2 h = make_double2(0.5 * (ax + bx), 0.5 * (ay - by));
    const bool vi = valid ? valid[k * vstride + i] != 0 : true;
    const bool vj = valid ? valid[k * vstride + j] != 0 : true;
    if (!(vi && vj)) h = make_double2(0.0, 0.0);
    if (i == j && !vi) h.x = inval_diag;
    out[t] = h;
  }
}

// p_ii += bound for the invalid rows i of each k, bound = max_i sum_j |p_ij| + gap.
__global__ void __launch_bounds__(kSmT) gershgorin_shift_kernel(double2* __restrict__ p, int n, const uint8_t* __restrict__ valid,
                                                                int vstride, double gap) {
  __shared__ double red[kSmT / 32];
  __shared__ double bound;
  const int k = blockIdx.x;
  double2* pk = p + (int64_t)k * n * n;
  double mx = 0.0;
  for (int i = threadIdx.x; i < n; i += kSmT) {
    double s = 0.0;
    for (int j = 0; j < n; ++j) {
      const double2 v = pk[(int64_t)i * n + j];
      s += sqrt(v.x * v.x + v.y * v.y);
    }
    mx = fmax(mx, s);
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < kSmT / 32; ++w) m = fmax(m, red[w]);
    bound = m + gap;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += kSmT)
    if (!valid[k * vstride + i]) pk[(int64_t)i * n + i].x += bound;
}

// rot[k][b][i] = v[k][i][b] for b < nb (eigenvectors as rows), in the working precision.
template <typename T>
__global__ void __launch_bounds__(kSmT) ritz_rotation_kernel(const double2* __restrict__ v, cx_t<T>* __restrict__ rot, int nk,
                                                             int m, int nb) {
  const int64_t per = (int64_t)nb * m;
  for (int64_t t = blockIdx.x * (int64_t)kSmT + threadIdx.x; t < per * nk; t += (int64_t)gridDim.x * kSmT) {
    const int k = (int)(t / per);
    const int64_t r = t - k * per;
    const int b = (int)(r / m), i = (int)(r - (int64_t)b * m);
    const double2 x = v[(int64_t)k * m * m + (int64_t)i * m + b];
    rot[t] = mk<cx_t<T>>(x.x, x.y);
  }
}

// Rows and columns whose diagonal is at most thr2 set to zero (directions too short to keep).
__global__ void __launch_bounds__(kSmT) drop_small_kernel(double2* __restrict__ g, int nk, int n, double thr2) {
  const int64_t per = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)kSmT + threadIdx.x; t < per * nk; t += (int64_t)gridDim.x * kSmT) {
    const int k = (int)(t / per);
    const int64_t r = t - k * per;
    const int i = (int)(r / n), j = (int)(r - (int64_t)i * n);
    const double2* gk = g + k * per;
    // a zeroed diagonal stays at most thr2, so the decision does not depend on the order
    if (gk[(int64_t)i * n + i].x <= thr2 || gk[(int64_t)j * n + j].x <= thr2)
      g[t] = make_double2(0.0, 0.0);
  }
}

// From the overlap's eigenpairs (u columns, w ascending): s_j = sqrt(max(w_j, 0)); keep_j =
// s_j > thr max_j s_j; rot[k][j][i] = keep_j conj(u_ij) / s_j (the rows u_j^H / s_j).
template <typename T>
__global__ void __launch_bounds__(kSmT) inv_sqrt_rotation_kernel(const double2* __restrict__ u, const double* __restrict__ w,
                                                                 cx_t<T>* __restrict__ rot, uint8_t* __restrict__ keep,
                                                                 int n, double thr) {
  __shared__ double red[kSmT / 32];
  __shared__ double smax;
  const int k = blockIdx.x;
  double mx = 0.0;
  for (int j = threadIdx.x; j < n; j += kSmT) mx = fmax(mx, sqrt(fmax(w[(int64_t)k * n + j], 0.0)));
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int q = 0; q < kSmT / 32; ++q) m = fmax(m, red[q]);
    smax = fmax(m, 1e-300);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += kSmT) keep[(int64_t)k * n + j] = sqrt(fmax(w[(int64_t)k * n + j], 0.0)) > thr * smax;
  __syncthreads();
  const double2* uk = u + (int64_t)k * n * n;
  for (int64_t t = threadIdx.x; t < (int64_t)n * n; t += kSmT) {
    const int j = (int)(t / n), i = (int)(t - (int64_t)j * n);
    const double s = sqrt(fmax(w[(int64_t)k * n + j], 0.0));
    const double2 x = uk[(int64_t)i * n + j];
    const bool kp = keep[(int64_t)k * n + j] != 0;
    rot[(int64_t)k * n * n + t] = kp ? mk<cx_t<T>>(x.x / s, -x.y / s) : mk<cx_t<T>>(0.0, 0.0);
  }
}

// dev[k] = || g_k - I ||_F
__global__ void __launch_bounds__(kSmT) frobenius_deviation_kernel(const double2* __restrict__ g, int n, double* __restrict__ dev) {
  __shared__ double red[kSmT / 32];
  const int k = blockIdx.x;
  double s = 0.0;
  for (int64_t t = threadIdx.x; t < (int64_t)n * n; t += kSmT) {
    const int i = (int)(t / n), j = (int)(t - (int64_t)i * n);
    double2 v = g[(int64_t)k * n * n + t];
    if (i == j) v.x -= 1.0;
    s += v.x * v.x + v.y * v.y;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < kSmT / 32; ++q) t += red[q];
    dev[k] = sqrt(t);
  }
}

// t = 1.5 I - 0.5 t; when ident is set, out = I instead (the Newton-Schulz start Z = I).
__global__ void __launch_bounds__(kSmT) ns_affine_kernel(double2* __restrict__ t, int nk, int n, int ident) {
  const int64_t per = (int64_t)n * n;
  for (int64_t q = blockIdx.x * (int64_t)kSmT + threadIdx.x; q < per * nk; q += (int64_t)gridDim.x * kSmT) {
    const int64_t r = q % per;
    const bool diag = (r / n) == (r % n);
    if (ident) {
      t[q] = make_double2(diag ? 1.0 : 0.0, 0.0);
    } else {
      const double2 v = t[q];
      t[q] = make_double2((diag ? 1.5 : 0.0) - 0.5 * v.x, -0.5 * v.y);
    }
  }
}

// double2 -> working precision copy
template <typename T>
__global__ void __launch_bounds__(kSmT) to_precision_kernel(const double2* __restrict__ in, cx_t<T>* __restrict__ out, int64_t count) {
  for (int64_t q = blockIdx.x * (int64_t)kSmT + threadIdx.x; q < count; q += (int64_t)gridDim.x * kSmT)
    out[q] = mk<cx_t<T>>(in[q].x, in[q].y);
}

// rows[k][b] = rank of band b among k's bands whose residual norm is above *tol, or -1
// (converged); one thread per k-point, bands in order.
__global__ void __launch_bounds__(kSmT) active_rows_kernel(const double* __restrict__ nrm, const double* __restrict__ tol,
                                                           int nk, int nb, int32_t* __restrict__ rows) {
  const int k = blockIdx.x * kSmT + threadIdx.x;
  if (k >= nk) return;
  const double t = *tol;
  int c = 0;
  for (int b = 0; b < nb; ++b) rows[(int64_t)k * nb + b] = nrm[(int64_t)k * nb + b] > t ? c++ : -1;
}

// valid[k][i] = (i < count) for i < cap: the basis holds `count` valid rows per k-point.
__global__ void __launch_bounds__(kSmT) valid_prefix_kernel(uint8_t* __restrict__ valid, int nk, int cap, int count) {
  for (int64_t t = blockIdx.x * (int64_t)kSmT + threadIdx.x; t < (int64_t)nk * cap; t += (int64_t)gridDim.x * kSmT)
    valid[t] = (t % cap) < count;
}

// valid[k][m + i] = keep[k][i] for i < nn: the rank test's decision on the appended rows.
__global__ void __launch_bounds__(kSmT) valid_append_kernel(uint8_t* __restrict__ valid, const uint8_t* __restrict__ keep,
                                                            int nk, int cap, int m, int nn) {
  for (int64_t t = blockIdx.x * (int64_t)kSmT + threadIdx.x; t < (int64_t)nk * nn; t += (int64_t)gridDim.x * kSmT) {
    const int64_t k = t / nn, i = t - k * nn;
    valid[k * cap + m + i] = keep[t];
  }
}

int blocks_for(int64_t count) { return (int)std::max<int64_t>(1, std::min<int64_t>((count + kSmT - 1) / kSmT, 4 * 148)); }

// A device (or pinned host) buffer that only grows.
template <bool Host>
struct GrowBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int need(size_t b) {
    if (bytes >= b) return AMA_OK;
    bump_memory_epoch();
    if (p) AMA_CUDA_TRY(Host ? cudaFreeHost(p) : cudaFree(p));
    p = nullptr;
    bytes = 0;
    const size_t sz = std::max<size_t>(b, 256);
    AMA_CUDA_TRY(Host ? cudaMallocHost(&p, sz) : cudaMalloc(&p, sz));
    bytes = sz;
    return AMA_OK;
  }
  template <typename X> X* as() const { return static_cast<X*>(p); }
};
using Buf = GrowBuf<false>;
using HostBuf = GrowBuf<true>;

// Executable graphs of iteration segments, keyed by everything their launches depend on.
using SegKey = std::array<int64_t, 10>;
struct GraphCache {
  uint64_t epoch = 0;
  std::vector<std::pair<SegKey, cudaGraphExec_t>> execs;
  std::vector<SegKey> seen, refused;
  int64_t captured = 0, replayed = 0, launched = 0;
  // only called with the segment stream idle (right after a host synchronisation)
  void drop() {
    for (auto& x : execs) cudaGraphExecDestroy(x.second);
    execs.clear();
    seen.clear();
    refused.clear();
  }
};

struct DavWork {
  Buf B, HB, X, HX, O1, O2, C, HN, X0;          // packed per-k blocks
  Buf p, t, rot;                                // small, working precision
  Buf g, y, z, tt, tmp;                         // small, FP64 complex
  Buf w, dev, keep, valid, rows, nrm, eps, tol; // per-k vectors
  HostBuf h_norms, h_keep, h_dev, h_tol;        // pinned: what the host decides on
  cudaStream_t stream = nullptr;                // the library's own (capturable) stream
  cudaEvent_t ready = nullptr;
  GraphCache graphs;
};
thread_local PerDevice<DavWork> g_dav;

template <typename T>
struct Davidson {
  using C = cx_t<T>;
  AmaEngine* e;
  int prec, spin, nb, nk, cap, max_sub, max_npw;
  int64_t total_pw;
  bool tc, graphs;
  cudaStream_t s;
  DavWork& wk;

  Davidson(AmaEngine* e_, int prec_, int spin_, int nb_, bool tc_, bool graphs_, cudaStream_t s_, DavWork& wk_)
      : e(e_), prec(prec_), spin(spin_), nb(nb_), nk(e_->nk), tc(tc_), graphs(graphs_), s(s_), wk(wk_) {
    max_npw = e->max_npw;
    total_pw = e->pw_off[nk];
    int min_npw = *std::min_element(e->npw.begin(), e->npw.end());
    max_sub = std::min(4 * nb, min_npw);
    cap = max_sub + nb;
  }

  SegKey key(int seg, int m, int nn, int ns_steps, int tail) const {
    return {(int64_t)(intptr_t)e, prec, spin, nb, nk, tc ? 1 : 0, seg, m, nn, (int64_t)ns_steps * 2 + tail};
  }

  // Runs `body` (launches on s only, no host synchronisation, no host state changed) as a
  // CUDA graph when this segment was seen before in the current allocation generation:
  // the first occurrence launches directly (and grows every buffer the segment needs), the
  // second is captured, later ones replay. A capture that fails (or that saw an allocation)
  // is discarded and the segment is launched directly instead, then and from then on.
  template <class F>
  int segment(const SegKey& k, bool capturable, F&& body) {
    GraphCache& gc = wk.graphs;
    if (!graphs || !capturable) {
      ++gc.launched;
      return body();
    }
    const uint64_t ep = memory_epoch();
    if (gc.epoch != ep) {
      gc.drop();
      gc.epoch = ep;
    }
    for (auto& x : gc.execs)
      if (x.first == k) {
        AMA_CUDA_TRY(cudaGraphLaunch(x.second, s));
        ++gc.replayed;
        return AMA_OK;
      }
    auto has = [&k](const std::vector<SegKey>& v) { return std::find(v.begin(), v.end(), k) != v.end(); };
    if (!has(gc.seen) || has(gc.refused)) {
      if (gc.seen.size() > 1024) gc.seen.clear();
      if (!has(gc.seen)) gc.seen.push_back(k);
      ++gc.launched;
      return body();
    }
    if ((int)gc.execs.size() >= kGraphCacheMax) {
      cudaGraphExecDestroy(gc.execs.front().second);
      gc.execs.erase(gc.execs.begin());
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool good = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (good) {
      const int rc = body();
      const cudaError_t ce = cudaStreamEndCapture(s, &graph);
      good = rc == AMA_OK && ce == cudaSuccess && graph != nullptr && memory_epoch() == ep &&
             cudaGraphInstantiate(&exec, graph, 0ULL) == cudaSuccess;
      if (graph) cudaGraphDestroy(graph);
    }
    if (!good) {
      (void)cudaGetLastError();
      if (exec) cudaGraphExecDestroy(exec);
      gc.refused.push_back(k);
      ++gc.launched;
      return body();
    }
    gc.execs.emplace_back(k, exec);
    ++gc.captured;
    AMA_CUDA_TRY(cudaGraphLaunch(exec, s));
    return AMA_OK;
  }

  size_t esz() const { return sizeof(C); }

  static AmaKOperand op(void* base, int64_t rows_per_k, int64_t row0, int ragged, int64_t ld = 0, int64_t kstride = 0) {
    AmaKOperand o;
    o.base = base; o.rows_per_k = rows_per_k; o.row0 = row0; o.ragged = ragged; o.ld = ld; o.kstride = kstride;
    return o;
  }

  int gemm(int form, int m, int n, int k, const AmaKOperand& a, const AmaKOperand& b, const AmaKOperand& c,
           double alpha = 1.0, double beta = 0.0) {
    const double al[2] = {alpha, 0.0}, be[2] = {beta, 0.0};
    if (tc && ((form == 1 && k < 0 && m > 0 && n > 0) || (form == 0 && n < 0 && m > 0 && k > 0)))
      return ama_kbatch_zgemm_tc(form, nk, m, n, k, e->d.npw, e->d.pw_off, &a, &b, &c, al, be, max_npw, s);
    const int mm = m < 0 ? max_npw : m, nn = n < 0 ? max_npw : n;
    return ama_kbatch_zgemm(prec, form, nk, m, n, k, e->d.npw, e->d.pw_off, &a, &b, &c, al, be, mm, nn, s);
  }

  // g = hermitised FP64 overlap of `rows` rows of a packed block (valid mask optional)
  int gram(void* blk, int rows, const uint8_t* vmask, int vstride, double inval_diag) {
    if (int rc = wk.p.need((size_t)nk * rows * rows * esz())) return rc;
    if (int rc = wk.g.need((size_t)nk * rows * rows * sizeof(double2))) return rc;
    if (int rc = gemm(1, rows, rows, -1, op(blk, rows, 0, 1), op(blk, rows, 0, 1),
                      op(wk.p.p, 0, 0, 0, rows, (int64_t)rows * rows)))
      return rc;
    small_hermitise_kernel<T><<<blocks_for((int64_t)nk * rows * rows), kSmT, 0, s>>>(
        wk.p.as<C>(), wk.g.as<double2>(), nk, rows, 0, vmask, vstride, inval_diag);
    AMA_CHECK_LAUNCH();
    return AMA_OK;
  }

  // eigenpairs of the nk (n x n) FP64 matrices in g (in place: vectors as columns)
  int heev(double2* mats, int n, int lowest) {
    if (int rc = wk.w.need((size_t)nk * n * sizeof(double))) return rc;
    if (n <= kJacobiMax) return ama_heev_small(n, mats, wk.w.as<double>(), nk, s);
    if (lowest > 0 && lowest < n) return ama_heev_lowest(n, lowest, mats, wk.w.as<double>(), nk, s);
    return ama_heev(n, mats, wk.w.as<double>(), nk, s);
  }

  // out (out_rows per k) = rot[k] (out_rows x k_rows, working precision) . src[k][:k_rows]
  int rotate(const void* rot, const void* src, int src_rows_per_k, int k_rows, int out_rows, void* out) {
    return gemm(0, out_rows, -1, k_rows, op(const_cast<void*>(rot), 0, 0, 0, k_rows, (int64_t)out_rows * k_rows),
                op(const_cast<void*>(src), src_rows_per_k, 0, 1), op(out, out_rows, 0, 1));
  }

  int copy_rows(const void* src, int src_rpk, int src_r0, void* dst, int dst_rpk, int dst_r0, int nrows) {
    return ama_kbatch_copy_rows(prec, nk, nrows, e->d.npw, e->d.pw_off, src, src_rpk, src_r0, dst, dst_rpk, dst_r0,
                                s);
  }

  int apply(const void* blk, int rows, void* out) { return ama_hpsi(e, prec, 0, nk, rows, spin, blk, out, s); }

  // Orthonormal rows spanning the dominant part of each k's block -> out; which of them are
  // kept -> wk.keep [nk][rows] (device)
  int orthonormal_rows(void* blk, int rows, double threshold, bool drop_small, void* out) {
    if (int rc = gram(blk, rows, nullptr, 0, 0.0)) return rc;
    double2* g = wk.g.as<double2>();
    if (drop_small) {
      drop_small_kernel<<<blocks_for((int64_t)nk * rows * rows), kSmT, 0, s>>>(g, nk, rows, threshold * threshold);
      AMA_CHECK_LAUNCH();
    }
    if (int rc = heev(g, rows, 0)) return rc;
    if (int rc = wk.rot.need((size_t)nk * rows * rows * esz())) return rc;
    if (int rc = wk.keep.need((size_t)nk * rows)) return rc;
    inv_sqrt_rotation_kernel<T><<<nk, kSmT, 0, s>>>(g, wk.w.as<double>(), wk.rot.as<C>(), wk.keep.as<uint8_t>(), rows,
                                                    threshold);
    AMA_CHECK_LAUNCH();
    return rotate(wk.rot.p, blk, rows, rows, rows, out);
  }

  // The FP64 overlap of the rows of blk that wk.keep marks (others set to the identity) ->
  // wk.g, and its Frobenius distance from the identity -> wk.dev [nk] (device).
  int lowdin_measure(void* blk, int rows) {
    if (int rc = gram(blk, rows, wk.keep.as<uint8_t>(), rows, 1.0)) return rc;
    frobenius_deviation_kernel<<<nk, kSmT, 0, s>>>(wk.g.as<double2>(), rows, wk.dev.as<double>());
    AMA_CHECK_LAUNCH();
    return AMA_OK;
  }

  // Newton-Schulz steps for the measured distance (host copy in wk.h_dev), or -1 when the
  // overlap is too far from the identity: every step squares the error, stop at 1e-18.
  int newton_schulz_steps() const {
    double dmax = 0.0;
    for (int k = 0; k < nk; ++k) {
      const double d = wk.h_dev.as<double>()[k];
      dmax = std::isnan(d) ? INFINITY : std::max(dmax, d);
    }
    if (!(dmax < 0.5)) return -1;
    int iters = 0;
    double err = std::max(dmax, 1e-300);
    while (err > 1e-18 && iters < 6) {
      err *= err;
      ++iters;
    }
    return iters;
  }

  // Newton-Schulz (coupled Y <- Y T, Z <- T Z, T = (3I - Z Y)/2) for S^{-1/2} of the overlap
  // in wk.g (rows orthonormal to rounding), applied to blk -> out.
  int lowdin_apply(void* blk, int rows, int iters, void* out) {
    const size_t sb = (size_t)nk * rows * rows * sizeof(double2);
    if (int rc = wk.y.need(sb)) return rc;
    if (int rc = wk.z.need(sb)) return rc;
    if (int rc = wk.tt.need(sb)) return rc;
    if (int rc = wk.tmp.need(sb)) return rc;
    double2 *y = wk.y.as<double2>(), *z = wk.z.as<double2>(), *t = wk.tt.as<double2>(), *tmp = wk.tmp.as<double2>();
    AMA_CUDA_TRY(cudaMemcpyAsync(y, wk.g.p, sb, cudaMemcpyDeviceToDevice, s));
    const int nb_ = blocks_for((int64_t)nk * rows * rows);
    ns_affine_kernel<<<nb_, kSmT, 0, s>>>(z, nk, rows, 1);
    AMA_CHECK_LAUNCH();
    const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
    const int64_t st = (int64_t)rows * rows;
    for (int q = 0; q < iters; ++q) {
      if (int rc = ama_zgemm(AMA_C128, 0, rows, rows, rows, one, z, rows, st, y, rows, st, zero, t, rows, st, nk, s))
        return rc;
      ns_affine_kernel<<<nb_, kSmT, 0, s>>>(t, nk, rows, 0);
      AMA_CHECK_LAUNCH();
      if (int rc = ama_zgemm(AMA_C128, 0, rows, rows, rows, one, y, rows, st, t, rows, st, zero, tmp, rows, st, nk, s))
        return rc;
      std::swap(y, tmp);
      if (int rc = ama_zgemm(AMA_C128, 0, rows, rows, rows, one, t, rows, st, z, rows, st, zero, tmp, rows, st, nk, s))
        return rc;
      std::swap(z, tmp);
    }
    if (int rc = wk.rot.need((size_t)nk * rows * rows * esz())) return rc;
    to_precision_kernel<T><<<nb_, kSmT, 0, s>>>(z, wk.rot.as<C>(), (int64_t)nk * rows * rows);
    AMA_CHECK_LAUNCH();
    return rotate(wk.rot.p, blk, rows, rows, rows, out);
  }

  // Rayleigh-Ritz over the first m rows of B / HB (validity wk.valid): eigenvalues -> wk.eps
  // [nk][nb], Ritz vectors -> X, HX
  int rayleigh_ritz(int m) {
    if (int rc = wk.p.need((size_t)nk * m * m * esz())) return rc;
    if (int rc = wk.g.need((size_t)nk * m * m * sizeof(double2))) return rc;
    if (int rc = gemm(1, m, m, -1, op(wk.B.p, cap, 0, 1), op(wk.HB.p, cap, 0, 1),
                      op(wk.p.p, 0, 0, 0, m, (int64_t)m * m)))
      return rc;
    double2* g = wk.g.as<double2>();
    small_hermitise_kernel<T><<<blocks_for((int64_t)nk * m * m), kSmT, 0, s>>>(wk.p.as<C>(), g, nk, m, 1,
                                                                              wk.valid.as<uint8_t>(), cap, 0.0);
    AMA_CHECK_LAUNCH();
    gershgorin_shift_kernel<<<nk, kSmT, 0, s>>>(g, m, wk.valid.as<uint8_t>(), cap, kGap);
    AMA_CHECK_LAUNCH();
    if (int rc = heev(g, m, nb)) return rc;
    if (int rc = wk.rot.need((size_t)nk * nb * m * esz())) return rc;
    ritz_rotation_kernel<T><<<blocks_for((int64_t)nk * nb * m), kSmT, 0, s>>>(g, wk.rot.as<C>(), nk, m, nb);
    AMA_CHECK_LAUNCH();
    if (int rc = rotate(wk.rot.p, wk.B.p, cap, m, nb, wk.X.p)) return rc;
    if (int rc = rotate(wk.rot.p, wk.HB.p, cap, m, nb, wk.HX.p)) return rc;
    AMA_CUDA_TRY(cudaMemcpy2DAsync(wk.eps.p, nb * sizeof(double), wk.w.p, m * sizeof(double), nb * sizeof(double),
                                   nk, cudaMemcpyDeviceToDevice, s));
    return AMA_OK;
  }

  int valid_prefix(int count) {
    valid_prefix_kernel<<<blocks_for((int64_t)nk * cap), kSmT, 0, s>>>(wk.valid.as<uint8_t>(), nk, cap, count);
    AMA_CHECK_LAUNCH();
    return AMA_OK;
  }

  // residual norms of the Ritz pairs -> wk.nrm and (once the stream gets there) wk.h_norms
  int residual_norms() {
    if (int rc = ama_kbatch_residual(prec, nk, nb, e->d.npw, e->d.pw_off, wk.X.p, wk.HX.p, wk.eps.as<double>(),
                                     e->d.kin64, wk.nrm.as<double>(), nullptr, 0, nullptr, s))
      return rc;
    AMA_CUDA_TRY(cudaMemcpyAsync(wk.h_norms.p, wk.nrm.p, (size_t)nk * nb * sizeof(double), cudaMemcpyDeviceToHost, s));
    return AMA_OK;
  }

  int run(const void* guess, double tol, int maxit, double* eps_out, void* x_out, double* norms_out, int* iterations) {
    const size_t blk = (size_t)total_pw * esz();
    const size_t nkb = (size_t)nk * nb;
    for (Buf* b : {&wk.B, &wk.HB})
      if (int rc = b->need(blk * cap)) return rc;
    for (Buf* b : {&wk.X, &wk.HX, &wk.O1, &wk.O2, &wk.C, &wk.HN, &wk.X0})
      if (int rc = b->need(blk * nb)) return rc;
    for (Buf* b : {&wk.nrm, &wk.eps})
      if (int rc = b->need(nkb * sizeof(double))) return rc;
    if (int rc = wk.rows.need(nkb * sizeof(int32_t))) return rc;
    if (int rc = wk.tol.need(sizeof(double))) return rc;
    if (int rc = wk.dev.need((size_t)nk * sizeof(double))) return rc;
    for (Buf* b : {&wk.keep, &wk.valid})
      if (int rc = b->need((size_t)nk * cap)) return rc;
    if (int rc = wk.h_norms.need(nkb * sizeof(double))) return rc;
    if (int rc = wk.h_keep.need(nkb)) return rc;
    if (int rc = wk.h_dev.need((size_t)nk * sizeof(double))) return rc;
    if (int rc = wk.h_tol.need(sizeof(double))) return rc;
    double* h_norms = wk.h_norms.as<double>();
    const uint8_t* h_keep = wk.h_keep.as<uint8_t>();
    *wk.h_tol.as<double>() = tol;
    AMA_CUDA_TRY(cudaMemcpyAsync(wk.tol.p, wk.h_tol.p, sizeof(double), cudaMemcpyHostToDevice, s));

    // the guess is usually the previous step's orthonormal orbitals: polish them without a
    // decomposition, else decompose the overlap (and reject a rank-deficient start)
    void* start = const_cast<void*>(guess);
    AMA_CUDA_TRY(cudaMemsetAsync(wk.keep.p, 1, nkb, s));
    if (int rc = lowdin_measure(start, nb)) return rc;
    AMA_CUDA_TRY(cudaMemcpyAsync(wk.h_dev.p, wk.dev.p, (size_t)nk * sizeof(double), cudaMemcpyDeviceToHost, s));
    AMA_CUDA_TRY(cudaStreamSynchronize(s));
    const int steps0 = newton_schulz_steps();
    if (steps0 >= 0) {
      if (int rc = lowdin_apply(start, nb, steps0, wk.X0.p)) return rc;
    } else {
      if (int rc = orthonormal_rows(start, nb, 1e-10, false, wk.X0.p)) return rc;
      AMA_CUDA_TRY(cudaMemcpyAsync(wk.h_keep.p, wk.keep.p, nkb, cudaMemcpyDeviceToHost, s));
      AMA_CUDA_TRY(cudaStreamSynchronize(s));
      for (size_t q = 0; q < nkb; ++q)
        AMA_REQUIRE(h_keep[q], AMA_ERR_ARG, "the starting block of some k-point is rank deficient");
    }
    if (int rc = apply(wk.X0.p, nb, wk.HN.p)) return rc;
    if (int rc = copy_rows(wk.X0.p, nb, 0, wk.B.p, cap, 0, nb)) return rc;
    if (int rc = copy_rows(wk.HN.p, nb, 0, wk.HB.p, cap, 0, nb)) return rc;
    if (int rc = valid_prefix(nb)) return rc;
    int m = nb;
    if (int rc = rayleigh_ritz(m)) return rc;
    std::fill(h_norms, h_norms + nkb, INFINITY);
    if (maxit >= 1)
      if (int rc = residual_norms()) return rc;
    AMA_CUDA_TRY(cudaStreamSynchronize(s));

    int it = 0;
    for (it = 1; it <= maxit; ++it) {
      // h_norms: the residual norms of the current Ritz pairs
      int nn = 0;
      for (int k = 0; k < nk; ++k) {
        int c = 0;
        for (int b = 0; b < nb; ++b) c += h_norms[(size_t)k * nb + b] > tol;
        nn = std::max(nn, c);
      }
      if (nn == 0) break;
      const int m0 = m, m1 = m + nn;
      // segment 1: corrections of the active bands, two projections off the basis, the rank
      // test (-> O1, wk.keep) and the survivors' overlap (-> wk.g, wk.dev); rows of k-points
      // with fewer active bands stay zero and are dropped by the rank test
      int rc = segment(key(1, m0, nn, 0, 0), nn <= kJacobiMax, [&]() -> int {
        active_rows_kernel<<<(nk + kSmT - 1) / kSmT, kSmT, 0, s>>>(wk.nrm.as<double>(), wk.tol.as<double>(), nk, nb,
                                                                  wk.rows.as<int32_t>());
        AMA_CHECK_LAUNCH();
        AMA_CUDA_TRY(cudaMemsetAsync(wk.C.p, 0, blk * nn, s));
        if (int r = ama_kbatch_residual(prec, nk, nb, e->d.npw, e->d.pw_off, wk.X.p, wk.HX.p, wk.eps.as<double>(),
                                        e->d.kin64, wk.nrm.as<double>(), wk.rows.as<int32_t>(), nn, wk.C.p, s))
          return r;
        if (int r = wk.t.need((size_t)nk * nn * m0 * esz())) return r;
        for (int pass = 0; pass < 2; ++pass) {
          const AmaKOperand top = op(wk.t.p, 0, 0, 0, m0, (int64_t)nn * m0);
          if (int r = gemm(1, nn, m0, -1, op(wk.C.p, nn, 0, 1), op(wk.B.p, cap, 0, 1), top)) return r;
          if (int r = gemm(0, nn, -1, m0, top, op(wk.B.p, cap, 0, 1), op(wk.C.p, nn, 0, 1), -1.0, 1.0)) return r;
        }
        if (int r = orthonormal_rows(wk.C.p, nn, 1e-7, true, wk.O1.p)) return r;
        if (int r = lowdin_measure(wk.O1.p, nn)) return r;
        AMA_CUDA_TRY(cudaMemcpyAsync(wk.h_keep.p, wk.keep.p, (size_t)nk * nn, cudaMemcpyDeviceToHost, s));
        AMA_CUDA_TRY(cudaMemcpyAsync(wk.h_dev.p, wk.dev.p, (size_t)nk * sizeof(double), cudaMemcpyDeviceToHost, s));
        return AMA_OK;
      });
      if (rc) return rc;
      AMA_CUDA_TRY(cudaStreamSynchronize(s));
      if (std::none_of(h_keep, h_keep + (size_t)nk * nn, [](uint8_t v) { return v != 0; })) break;  // all dependent
      const int steps = newton_schulz_steps();
      const bool collapse = m1 + nb > max_sub, tail = it < maxit;
      // segment 2: second orthonormalisation (-> O2, wk.keep), H on the new block, the basis
      // extended, Rayleigh-Ritz, the collapse onto the Ritz vectors when one more block would
      // not fit, and the next iteration's residual norms
      rc = segment(key(2, m0, nn, steps, tail), m1 <= kJacobiMax, [&]() -> int {
        if (steps >= 0) {
          if (int r = lowdin_apply(wk.O1.p, nn, steps, wk.O2.p)) return r;
        } else {
          if (int r = orthonormal_rows(wk.O1.p, nn, 0.5, false, wk.O2.p)) return r;
        }
        if (int r = apply(wk.O2.p, nn, wk.HN.p)) return r;
        if (int r = copy_rows(wk.O2.p, nn, 0, wk.B.p, cap, m0, nn)) return r;
        if (int r = copy_rows(wk.HN.p, nn, 0, wk.HB.p, cap, m0, nn)) return r;
        valid_append_kernel<<<blocks_for((int64_t)nk * nn), kSmT, 0, s>>>(wk.valid.as<uint8_t>(), wk.keep.as<uint8_t>(),
                                                                          nk, cap, m0, nn);
        AMA_CHECK_LAUNCH();
        if (int r = rayleigh_ritz(m1)) return r;
        if (collapse) {
          if (int r = copy_rows(wk.X.p, nb, 0, wk.B.p, cap, 0, nb)) return r;
          if (int r = copy_rows(wk.HX.p, nb, 0, wk.HB.p, cap, 0, nb)) return r;
          if (int r = valid_prefix(nb)) return r;
        }
        return tail ? residual_norms() : AMA_OK;
      });
      if (rc) return rc;
      m = collapse ? nb : m1;
      AMA_CUDA_TRY(cudaStreamSynchronize(s));
    }
    if (it > maxit) it = maxit;
    AMA_CUDA_TRY(cudaMemcpyAsync(eps_out, wk.eps.p, nkb * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (x_out != wk.X.p) AMA_CUDA_TRY(cudaMemcpyAsync(x_out, wk.X.p, blk * nb, cudaMemcpyDeviceToDevice, s));
    if (norms_out) AMA_CUDA_TRY(cudaMemcpyAsync(norms_out, h_norms, nkb * sizeof(double), cudaMemcpyHostToDevice, s));
    AMA_CUDA_TRY(cudaStreamSynchronize(s));
    *iterations = it;
    return AMA_OK;
  }
};

}  // namespace

extern "C" int ama_davidson(AmaEngine* e, int32_t precision, int32_t spin, int32_t nbands, const void* guess,
                            double tolerance, int32_t max_iterations, int32_t tc_min_npw, double* eigenvalues,
                            void* x, double* norms, int32_t* iterations, void* stream) {
  AMA_REQUIRE(e && guess && eigenvalues && x && iterations, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(precision == AMA_C64 || precision == AMA_C128, AMA_ERR_ARG, "precision must be AMA_C64 or AMA_C128");
  AMA_REQUIRE(e->precisions & (1u << precision), AMA_ERR_ARG, "the engine was created without this precision");
  AMA_REQUIRE(e->has_potential, AMA_ERR_ARG, "set the effective potential first");
  AMA_REQUIRE(spin >= 0 && spin < e->nspin, AMA_ERR_ARG, "spin out of range");
  AMA_REQUIRE(nbands >= 1 && max_iterations >= 0, AMA_ERR_ARG, "bad band count or iteration limit");
  const int min_npw = *std::min_element(e->npw.begin(), e->npw.end());
  AMA_REQUIRE(nbands <= min_npw, AMA_ERR_SHAPE, "more bands than plane waves at some k-point");
  DavWork* wk = g_dav.here();
  AMA_REQUIRE(wk, AMA_ERR_UNSUPPORTED, "device index out of range");
  // the iterations run on the library's own stream (the caller's may be the legacy default
  // stream, which cannot be captured), after the work already queued on the caller's
  if (!wk->stream) {
    AMA_CUDA_TRY(cudaStreamCreateWithFlags(&wk->stream, cudaStreamNonBlocking));
    AMA_CUDA_TRY(cudaEventCreateWithFlags(&wk->ready, cudaEventDisableTiming));
  }
  cudaStream_t s = wk->stream;
  AMA_CUDA_TRY(cudaEventRecord(wk->ready, (cudaStream_t)stream));
  AMA_CUDA_TRY(cudaStreamWaitEvent(s, wk->ready, 0));
  int it = 0, rc;
  if (precision == AMA_C64) {
    Davidson<float> d(e, precision, spin, nbands, tc_min_npw > 0 && e->max_npw >= tc_min_npw, e->dav_graphs, s, *wk);
    rc = d.run(guess, tolerance, max_iterations, eigenvalues, x, norms, &it);
  } else {
    Davidson<double> d(e, precision, spin, nbands, false, e->dav_graphs, s, *wk);
    rc = d.run(guess, tolerance, max_iterations, eigenvalues, x, norms, &it);
  }
  if (rc) (void)cudaStreamSynchronize(s);  // nothing of this call is left running on an error
  *iterations = it;
  return rc;
}

extern "C" int ama_davidson_graph_stats(int64_t* captured, int64_t* replayed, int64_t* launched, int32_t reset) {
  AMA_REQUIRE(captured && replayed && launched, AMA_ERR_ARG, "null argument");
  DavWork* wk = g_dav.here();
  AMA_REQUIRE(wk, AMA_ERR_UNSUPPORTED, "device index out of range");
  GraphCache& gc = wk->graphs;
  *captured = gc.captured;
  *replayed = gc.replayed;
  *launched = gc.launched;
  if (reset) gc.captured = gc.replayed = gc.launched = 0;
  return AMA_OK;
}
