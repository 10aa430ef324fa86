// FP64 grid-vector kernels of the SCF loop: the density mixers' overlap matrices and linear
// combinations, the floor-and-rescale of a new density, and the reductions behind the
// energy terms. All HBM-bound single passes; every reduction is two-stage (per-CTA partial
// sums, then one CTA adding them in a fixed order), so results are reproducible bit for bit.
#include "common.cuh"

#include <algorithm>

using namespace ama;

namespace {

constexpr int kVecT = 256;
constexpr int kMaxVecs = 16;     // history vectors per call
constexpr int kMaxOut = kMaxVecs + 1;
constexpr int kMaxPairs = kMaxOut * (kMaxOut + 1) / 2;
constexpr int kPartialCtas = 592;  // 4 per SM

struct GramArgs {
  const double* v[kMaxVecs];
  double coef[kMaxVecs * kMaxVecs];  // [a][j]: u_a = sum_j coef[a][j] v_j
  const double* w;                   // optional extra vector (u_ncomb = w)
  int nvec, ncomb;
  int64_t n;
};

struct CombArgs {
  const double* v[kMaxVecs];
  double coef[kMaxVecs];
  int nvec;
  int64_t n;
};

// Partial Gram of the combinations over a grid-stride set of kVecT-point tiles.
__global__ void __launch_bounds__(kVecT) gram_partial_kernel(GramArgs g, double* __restrict__ partial) {
  __shared__ double us[kMaxOut][kVecT + 1];
  const int nout = g.ncomb + (g.w ? 1 : 0);
  const int npairs = nout * (nout + 1) / 2;
  int pa = 0, pb = 0;  // this thread's pair (a <= b)
  if (threadIdx.x < npairs) {
    int t = threadIdx.x;
    while (t >= nout - pa) { t -= nout - pa; ++pa; }
    pb = pa + t;
  }
  double acc = 0.0;
  for (int64_t base = (int64_t)blockIdx.x * kVecT; base < g.n; base += (int64_t)gridDim.x * kVecT) {
    const int64_t x = base + threadIdx.x;
    double vals[kMaxVecs];
    for (int j = 0; j < g.nvec; ++j) vals[j] = x < g.n ? g.v[j][x] : 0.0;
    for (int a = 0; a < g.ncomb; ++a) {
      double u = 0.0;
      for (int j = 0; j < g.nvec; ++j) u += g.coef[a * kMaxVecs + j] * vals[j];
      us[a][threadIdx.x] = u;
    }
    if (g.w) us[g.ncomb][threadIdx.x] = x < g.n ? g.w[x] : 0.0;
    __syncthreads();
    if (threadIdx.x < npairs)
      for (int t = 0; t < kVecT; ++t) acc += us[pa][t] * us[pb][t];
    __syncthreads();
  }
  if (threadIdx.x < npairs) partial[(int64_t)blockIdx.x * kMaxPairs + threadIdx.x] = acc;
}

__global__ void __launch_bounds__(kVecT)
gram_final_kernel(int nout, int nblocks, const double* __restrict__ partial, double* __restrict__ gram) {
  __shared__ double red[kVecT];
  const int p = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += kVecT) s += partial[(int64_t)b * kMaxPairs + p];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = kVecT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int a = 0, t = p;
    while (t >= nout - a) { t -= nout - a; ++a; }
    const int b = a + t;
    gram[a * nout + b] = red[0];
    gram[b * nout + a] = red[0];
  }
}

__global__ void __launch_bounds__(kVecT) lincomb_kernel(CombArgs c, double* __restrict__ out) {
  for (int64_t x = blockIdx.x * (int64_t)kVecT + threadIdx.x; x < c.n; x += (int64_t)gridDim.x * kVecT) {
    double s = 0.0;
    for (int j = 0; j < c.nvec; ++j) s += c.coef[j] * c.v[j][x];
    out[x] = s;
  }
}

// op 0: sum a*b; op 1: sum |a - b|; op 2: sum a; op 3: sum max(a, 0)
__device__ __forceinline__ double reduce_term(int op, double a, double b) {
  switch (op) {
    case 0: return a * b;
    case 1: return fabs(a - b);
    case 2: return a;
    default: return fmax(a, 0.0);
  }
}

__global__ void __launch_bounds__(kVecT)
reduce_partial_kernel(int op, int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                      double* __restrict__ partial) {
  __shared__ double red[kVecT];
  double s = 0.0;
  for (int64_t x = blockIdx.x * (int64_t)kVecT + threadIdx.x; x < n; x += (int64_t)gridDim.x * kVecT)
    s += reduce_term(op, a[x], b ? b[x] : 0.0);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = kVecT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// out[slot] (+)= scale * sum of the partials
__global__ void __launch_bounds__(kVecT)
reduce_final_kernel(int nblocks, const double* __restrict__ partial, double scale, int accumulate,
                    double* __restrict__ out) {
  __shared__ double red[kVecT];
  double s = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += kVecT) s += partial[b];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = kVecT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = (accumulate ? *out : 0.0) + scale * red[0];
}

// rho <- max(rho / volume, 0) * before / after per channel (before/after: sums of rho/volume
// and of its positive part), the charge-preserving floor of a new density.
__global__ void __launch_bounds__(kVecT)
floor_rescale_kernel(int64_t n, double inv_volume, const double* __restrict__ sums, double* __restrict__ rho) {
  const int ch = blockIdx.y;
  const double before = sums[2 * ch], after = sums[2 * ch + 1];
  const double scale = after > 0.0 ? before / after : 1.0;
  double* r = rho + (int64_t)ch * n;
  for (int64_t x = blockIdx.x * (int64_t)kVecT + threadIdx.x; x < n; x += (int64_t)gridDim.x * kVecT)
    r[x] = fmax(r[x] * inv_volume, 0.0) * scale;
}

// Per band (row) of the packed per-k blocks: sum_G |psi|^2 T_G (kinetic) into rows[k*nb+n].
template <typename T>
__global__ void __launch_bounds__(kVecT)
band_kinetic_kernel(int nbands, const int* __restrict__ npw, const int64_t* __restrict__ pw_off,
                    const cx_t<T>* __restrict__ psi, const double* __restrict__ kin, double* __restrict__ rows) {
  __shared__ double red[kVecT];
  const int k = blockIdx.y, nb = blockIdx.x;
  const int n = npw[k];
  const cx_t<T>* row = psi + pw_off[k] * nbands + (int64_t)nb * n;
  const double* t = kin + pw_off[k];
  double s = 0.0;
  for (int g = threadIdx.x; g < n; g += kVecT) {
    const cx_t<T> v = row[g];
    s += ((double)v.x * v.x + (double)v.y * v.y) * t[g];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = kVecT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) rows[(int64_t)k * nbands + nb] = red[0];
}

// rows[i] = Re sum_j conj(a[i][j]) b[i][j] (complex128)
__global__ void __launch_bounds__(kVecT)
rowdot_kernel(int ncols, const double2* __restrict__ a, const double2* __restrict__ b, double* __restrict__ rows) {
  __shared__ double red[kVecT];
  const int i = blockIdx.x;
  double s = 0.0;
  for (int j = threadIdx.x; j < ncols; j += kVecT) {
    const double2 x = a[(int64_t)i * ncols + j], y = b[(int64_t)i * ncols + j];
    s += x.x * y.x + x.y * y.y;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = kVecT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) rows[i] = red[0];
}

struct VecScratch {
  double* partial = nullptr;
  double* sums = nullptr;
};
thread_local PerDevice<VecScratch> g_vec;

int vec_scratch(VecScratch** out) {
  VecScratch* v = g_vec.here();
  AMA_REQUIRE(v, AMA_ERR_CUDA, "grid vectors: no usable current CUDA device");
  if (!v->partial || !v->sums) bump_memory_epoch();
  if (!v->partial) AMA_CUDA_TRY(cudaMalloc((void**)&v->partial, sizeof(double) * kPartialCtas * kMaxPairs));
  if (!v->sums) AMA_CUDA_TRY(cudaMalloc((void**)&v->sums, sizeof(double) * 8));
  *out = v;
  return AMA_OK;
}

int ctas_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>(kPartialCtas, (n + kVecT - 1) / kVecT)); }

}  // namespace

extern "C" int ama_vec_gram(int32_t nvec, const double* const* vectors, int32_t ncomb, const double* coef,
                            const double* extra, int64_t n, double* gram, void* stream) {
  AMA_REQUIRE(vectors && coef && gram, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(nvec >= 1 && nvec <= kMaxVecs && ncomb >= 0 && ncomb <= kMaxVecs && ncomb + (extra ? 1 : 0) >= 1 &&
                  n >= 1,
              AMA_ERR_SHAPE, "ama_vec_gram: 1..16 vectors and combinations");
  VecScratch* sc = nullptr;
  if (int rc = vec_scratch(&sc)) return rc;
  GramArgs g{};
  for (int j = 0; j < nvec; ++j) g.v[j] = vectors[j];
  for (int a = 0; a < ncomb; ++a)
    for (int j = 0; j < nvec; ++j) g.coef[a * kMaxVecs + j] = coef[a * nvec + j];
  g.w = extra;
  g.nvec = nvec;
  g.ncomb = ncomb;
  g.n = n;
  const int nout = ncomb + (extra ? 1 : 0);
  const int blocks = ctas_for(n);
  cudaStream_t s = (cudaStream_t)stream;
  gram_partial_kernel<<<blocks, kVecT, 0, s>>>(g, sc->partial);
  gram_final_kernel<<<nout * (nout + 1) / 2, kVecT, 0, s>>>(nout, blocks, sc->partial, gram);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_vec_lincomb(int32_t nvec, const double* const* vectors, const double* coef, int64_t n,
                               double* out, void* stream) {
  AMA_REQUIRE(vectors && coef && out, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(nvec >= 1 && nvec <= kMaxVecs && n >= 1, AMA_ERR_SHAPE, "ama_vec_lincomb: 1..16 vectors");
  CombArgs c{};
  for (int j = 0; j < nvec; ++j) {
    c.v[j] = vectors[j];
    c.coef[j] = coef[j];
  }
  c.nvec = nvec;
  c.n = n;
  lincomb_kernel<<<ctas_for(n), kVecT, 0, (cudaStream_t)stream>>>(c, out);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_vec_reduce(int32_t op, int64_t n, const double* a, const double* b, double scale,
                              int32_t accumulate, double* out, void* stream) {
  AMA_REQUIRE(a && out && (op == 2 || op == 3 || b), AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(op >= 0 && op <= 3 && n >= 1, AMA_ERR_ARG, "ama_vec_reduce: op 0..3");
  VecScratch* sc = nullptr;
  if (int rc = vec_scratch(&sc)) return rc;
  const int blocks = ctas_for(n);
  cudaStream_t s = (cudaStream_t)stream;
  reduce_partial_kernel<<<blocks, kVecT, 0, s>>>(op, n, a, b, sc->partial);
  reduce_final_kernel<<<1, kVecT, 0, s>>>(blocks, sc->partial, scale, accumulate, out);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_density_floor(int32_t nchannels, int64_t n, double volume, double* rho, void* stream) {
  AMA_REQUIRE(rho, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(nchannels >= 1 && nchannels <= 4 && n >= 1 && volume > 0.0, AMA_ERR_SHAPE, "bad sizes");
  VecScratch* sc = nullptr;
  if (int rc = vec_scratch(&sc)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = ctas_for(n);
  const double inv = 1.0 / volume;
  for (int ch = 0; ch < nchannels; ++ch) {
    const double* r = rho + (int64_t)ch * n;
    reduce_partial_kernel<<<blocks, kVecT, 0, s>>>(2, n, r, nullptr, sc->partial);
    reduce_final_kernel<<<1, kVecT, 0, s>>>(blocks, sc->partial, inv, 0, sc->sums + 2 * ch);
    reduce_partial_kernel<<<blocks, kVecT, 0, s>>>(3, n, r, nullptr, sc->partial);
    reduce_final_kernel<<<1, kVecT, 0, s>>>(blocks, sc->partial, inv, 0, sc->sums + 2 * ch + 1);
  }
  floor_rescale_kernel<<<dim3(blocks, nchannels), kVecT, 0, s>>>(n, inv, sc->sums, rho);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_band_kinetic(int32_t precision, int32_t nk, int32_t nbands, const int32_t* npw,
                                const int64_t* pw_off, const void* psi, const double* kinetic, double* rows,
                                void* stream) {
  AMA_REQUIRE(npw && pw_off && psi && kinetic && rows, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(nk >= 1 && nbands >= 1 && nk <= 65535, AMA_ERR_SHAPE, "bad sizes");
  const dim3 grid(nbands, nk);
  cudaStream_t s = (cudaStream_t)stream;
  if (precision == AMA_C64)
    band_kinetic_kernel<float><<<grid, kVecT, 0, s>>>(nbands, npw, pw_off, (const float2*)psi, kinetic, rows);
  else if (precision == AMA_C128)
    band_kinetic_kernel<double><<<grid, kVecT, 0, s>>>(nbands, npw, pw_off, (const double2*)psi, kinetic, rows);
  else {
    ama::set_error("bad precision");
    return AMA_ERR_ARG;
  }
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_rowdot(int32_t nrows, int32_t ncols, const void* a, const void* b, double* rows, void* stream) {
  AMA_REQUIRE(a && b && rows, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(nrows >= 1 && ncols >= 1, AMA_ERR_SHAPE, "bad sizes");
  rowdot_kernel<<<nrows, kVecT, 0, (cudaStream_t)stream>>>(ncols, (const double2*)a, (const double2*)b, rows);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}
