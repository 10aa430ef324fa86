// Band-wise kernels of the Davidson iteration and pointwise grid functionals.
#include "common.cuh"

#include <cmath>

using namespace ama;

namespace {

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < NT / 32) t = sh[threadIdx.x];
  if (wid == 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) sh[0] = t;
  }
  __syncthreads();
  return sh[0];
}

constexpr int kRowThreads = 256;

// One CTA per band: residual norm; for listed rows also the preconditioned, normalised
// correction (Teter-Payne-Allan, PRB 40, 12255 (1989)).
template <typename T>
__global__ void __launch_bounds__(kRowThreads)
residual_precondition_kernel(int nbands, int npw, const cx_t<T>* __restrict__ x,
                             const cx_t<T>* __restrict__ hx, const double* __restrict__ eps,
                             const double* __restrict__ kin, double* __restrict__ norms,
                             const int* __restrict__ row_of_band, cx_t<T>* __restrict__ out) {
  using C = cx_t<T>;
  __shared__ double sh[32];
  const int n = blockIdx.x;
  const C* xr = x + (int64_t)n * npw;
  const C* hr = hx + (int64_t)n * npw;
  const double e = eps[n];
  double rr = 0.0, tk = 0.0;
  for (int g = threadIdx.x; g < npw; g += kRowThreads) {
    const C xv = xr[g], hv = hr[g];
    const double re = (double)hv.x - e * (double)xv.x, im = (double)hv.y - e * (double)xv.y;
    rr += re * re + im * im;
    tk += ((double)xv.x * xv.x + (double)xv.y * xv.y) * kin[g];
  }
  rr = block_sum<kRowThreads>(rr, sh);
  tk = block_sum<kRowThreads>(tk, sh);
  if (threadIdx.x == 0) norms[n] = sqrt(rr);
  const int row = row_of_band ? row_of_band[n] : -1;
  if (row < 0) return;
  const double ref = fmax(tk, 1e-8);
  C* orow = out + (int64_t)row * npw;
  double cc = 0.0;
  for (int g = threadIdx.x; g < npw; g += kRowThreads) {
    const C xv = xr[g], hv = hr[g];
    const double re = (double)hv.x - e * (double)xv.x, im = (double)hv.y - e * (double)xv.y;
    const double q = kin[g] / ref;
    const double poly = 27.0 + q * (18.0 + q * (12.0 + 8.0 * q));
    const double k = poly / (poly + 16.0 * q * q * q * q);
    cc += k * k * (re * re + im * im);
    orow[g] = mk<C>(k * re, k * im);
  }
  cc = block_sum<kRowThreads>(cc, sh);
  const double inv = 1.0 / fmax(sqrt(cc), 1e-300);
  for (int g = threadIdx.x; g < npw; g += kRowThreads) {
    C v = orow[g];
    orow[g] = mk<C>((double)v.x * inv, (double)v.y * inv);
  }
}

__global__ void rows_to_map_kernel(const int* rows, int nrows, int* map, int nbands) {
  for (int i = threadIdx.x; i < nbands; i += blockDim.x) map[i] = -1;
  __syncthreads();
  for (int i = threadIdx.x; i < nrows; i += blockDim.x) {
    const int b = rows[i];
    if (b >= 0 && b < nbands) map[b] = i;
  }
}

// ---------------------------------------------------------------- LDA-PZ
// Parameters of Perdew & Zunger, PRB 23, 5048 (1981), index 0 unpolarised, 1 polarised;
// exchange and spin-interpolation constants as in libxc (X_FACTOR_C, RS_FACTOR).
__constant__ double kPZ_gamma[2] = {-0.1423, -0.0843};
__constant__ double kPZ_beta1[2] = {1.0529, 1.3981};
__constant__ double kPZ_beta2[2] = {0.3334, 0.2611};
__constant__ double kPZ_a[2] = {0.0311, 0.01555};
__constant__ double kPZ_b[2] = {-0.048, -0.0269};
__constant__ double kPZ_c[2] = {0.0020, 0.0007};
__constant__ double kPZ_d[2] = {-0.0116, -0.0048};
constexpr double kXFactorC = 0.9305257363491000250020102180716672510262;
constexpr double kRsFactor = 0.6203504908994000166680068120477781673508;
constexpr double kDensityThreshold = 1e-24;

__global__ void lda_pz_kernel(const double* __restrict__ rho, int64_t npts, double* __restrict__ eps_out,
                              double* __restrict__ vrho) {
  const double fz_den = pow(2.0, 4.0 / 3.0) - 2.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npts;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double ru = rho[i], rd = rho[npts + i];
    const double total = ru + rd;
    const bool active = total > kDensityThreshold;
    if (!active) {
      eps_out[i] = 0.0; vrho[i] = 0.0; vrho[npts + i] = 0.0;
      continue;
    }
    // exchange: e_x = -X sum_s n_s^(4/3)
    const double su = fmax(ru, 0.0), sd = fmax(rd, 0.0);
    const double cu = cbrt(su), cd = cbrt(sd);
    const double eps_x = -kXFactorC * (cu * su + cd * sd) / total;
    const double vxu = -(4.0 / 3.0) * kXFactorC * cu;
    const double vxd = -(4.0 / 3.0) * kXFactorC * cd;
    // correlation
    const double safe = fmax(total, kDensityThreshold);
    const double rs = kRsFactor / cbrt(safe);
    const double zeta = fmin(fmax((ru - rd) / safe, -1.0), 1.0);
    double ec[2], dec[2];
    const double sq = sqrt(rs);
    const double lrs = log(fmax(rs, 1e-300));
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if (rs < 1.0) {
        ec[j] = kPZ_a[j] * lrs + kPZ_b[j] + kPZ_c[j] * rs * lrs + kPZ_d[j] * rs;
        dec[j] = kPZ_a[j] / rs + kPZ_c[j] * (lrs + 1.0) + kPZ_d[j];
      } else {
        const double den = 1.0 + kPZ_beta1[j] * sq + kPZ_beta2[j] * rs;
        ec[j] = kPZ_gamma[j] / den;
        dec[j] = -kPZ_gamma[j] * (0.5 * kPZ_beta1[j] / sq + kPZ_beta2[j]) / (den * den);
      }
    }
    const double opz = fmax(1.0 + zeta, 0.0), omz = fmax(1.0 - zeta, 0.0);
    const double fz = (pow(opz, 4.0 / 3.0) + pow(omz, 4.0 / 3.0) - 2.0) / fz_den;
    const double dfz = (4.0 / 3.0) * (cbrt(opz) - cbrt(omz)) / fz_den;
    const double eps_c = ec[0] + fz * (ec[1] - ec[0]);
    const double d_drs = dec[0] + fz * (dec[1] - dec[0]);
    const double d_dz = dfz * (ec[1] - ec[0]);
    const double common = eps_c - (rs / 3.0) * d_drs;
    eps_out[i] = eps_x + eps_c;
    vrho[i] = vxu + common + (1.0 - zeta) * d_dz;
    vrho[npts + i] = vxd + common - (1.0 + zeta) * d_dz;
  }
}

struct MapScratch { int* ptr = nullptr; int n = 0; };
thread_local PerDevice<MapScratch> g_map_dev;  // per host thread and device

}  // namespace

extern "C" int ama_residual_precondition(int32_t precision, int32_t nbands, int32_t npw,
                                         const void* x, const void* hx, const double* eps,
                                         const double* kinetic, double* norms, const int32_t* rows,
                                         int32_t nrows, void* out, void* stream) {
  AMA_REQUIRE(precision == AMA_C64 || precision == AMA_C128, AMA_ERR_ARG, "bad precision");
  AMA_REQUIRE(x && hx && eps && kinetic && norms, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(nbands >= 1 && npw >= 1 && nrows >= 0 && nrows <= nbands, AMA_ERR_SHAPE, "bad sizes");
  AMA_REQUIRE(nrows == 0 || (rows && out), AMA_ERR_ARG, "rows/out required when nrows > 0");
  cudaStream_t s = (cudaStream_t)stream;
  int* map = nullptr;
  if (nrows > 0) {
    MapScratch* gm = g_map_dev.here();
    AMA_REQUIRE(gm, AMA_ERR_CUDA, "no usable current CUDA device");
    MapScratch& g_map = *gm;
    if (g_map.n < nbands) {
      bump_memory_epoch();
      if (g_map.ptr) cudaFree(g_map.ptr);
      g_map.ptr = nullptr; g_map.n = 0;
      AMA_CUDA_TRY(cudaMalloc((void**)&g_map.ptr, sizeof(int) * nbands));
      g_map.n = nbands;
    }
    map = g_map.ptr;
    rows_to_map_kernel<<<1, 256, 0, s>>>(rows, nrows, map, nbands);
    AMA_CHECK_LAUNCH();
  }
  if (precision == AMA_C64)
    residual_precondition_kernel<float><<<nbands, kRowThreads, 0, s>>>(
        nbands, npw, (const float2*)x, (const float2*)hx, eps, kinetic, norms, map, (float2*)out);
  else
    residual_precondition_kernel<double><<<nbands, kRowThreads, 0, s>>>(
        nbands, npw, (const double2*)x, (const double2*)hx, eps, kinetic, norms, map, (double2*)out);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_lda_pz(const double* rho, int64_t npoints, double* eps, double* vrho, void* stream) {
  AMA_REQUIRE(rho && eps && vrho, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(npoints >= 0, AMA_ERR_SHAPE, "negative size");
  if (npoints == 0) return AMA_OK;
  const int blocks = (int)std::min<int64_t>((npoints + 255) / 256, 148 * 16);
  lda_pz_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(rho, npoints, eps, vrho);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

// ------------------------------------------------------------ per-k ragged variants
namespace {

template <typename T>
__global__ void __launch_bounds__(kRowThreads)
kbatch_residual_kernel(int nb, const int* __restrict__ npw, const int64_t* __restrict__ pw_off,
                       const cx_t<T>* __restrict__ x, const cx_t<T>* __restrict__ hx, const double* __restrict__ eps,
                       const double* __restrict__ kin, double* __restrict__ norms, const int* __restrict__ rows,
                       int nrows, cx_t<T>* __restrict__ out) {
  using C = cx_t<T>;
  __shared__ double sh[32];
  const int k = blockIdx.x / nb, n = blockIdx.x % nb;
  const int np = npw[k];
  const int64_t po = pw_off[k];
  const C* xr = x + po * nb + (int64_t)n * np;
  const C* hr = hx + po * nb + (int64_t)n * np;
  const double* kk = kin + po;
  const double e = eps[blockIdx.x];
  double rr = 0.0, tk = 0.0;
  for (int g = threadIdx.x; g < np; g += kRowThreads) {
    const C xv = xr[g], hv = hr[g];
    const double re = (double)hv.x - e * (double)xv.x, im = (double)hv.y - e * (double)xv.y;
    rr += re * re + im * im;
    tk += ((double)xv.x * xv.x + (double)xv.y * xv.y) * kk[g];
  }
  rr = block_sum<kRowThreads>(rr, sh);
  tk = block_sum<kRowThreads>(tk, sh);
  if (threadIdx.x == 0) norms[blockIdx.x] = sqrt(rr);
  const int row = rows ? rows[blockIdx.x] : -1;
  if (row < 0) return;
  const double ref = fmax(tk, 1e-8);
  C* orow = out + po * nrows + (int64_t)row * np;
  double cc = 0.0;
  for (int g = threadIdx.x; g < np; g += kRowThreads) {
    const C xv = xr[g], hv = hr[g];
    const double re = (double)hv.x - e * (double)xv.x, im = (double)hv.y - e * (double)xv.y;
    const double q = kk[g] / ref;
    const double poly = 27.0 + q * (18.0 + q * (12.0 + 8.0 * q));
    const double kf = poly / (poly + 16.0 * q * q * q * q);
    cc += kf * kf * (re * re + im * im);
    orow[g] = mk<C>(kf * re, kf * im);
  }
  cc = block_sum<kRowThreads>(cc, sh);
  const double inv = 1.0 / fmax(sqrt(cc), 1e-300);
  for (int g = threadIdx.x; g < np; g += kRowThreads) {
    C v = orow[g];
    orow[g] = mk<C>((double)v.x * inv, (double)v.y * inv);
  }
}

template <typename C>
__global__ void kbatch_copy_kernel(int nrows, const int* __restrict__ npw, const int64_t* __restrict__ pw_off,
                                   const C* __restrict__ src, int64_t src_rows_per_k, int64_t src_row0,
                                   C* __restrict__ dst, int64_t dst_rows_per_k, int64_t dst_row0) {
  const int k = blockIdx.y;
  const int np = npw[k];
  const int64_t po = pw_off[k];
  const C* s = src + src_rows_per_k * po + src_row0 * np;
  C* d = dst + dst_rows_per_k * po + dst_row0 * np;
  const int64_t total = (int64_t)nrows * np;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    d[e] = s[e];
}

}  // namespace

extern "C" int ama_kbatch_residual(int32_t precision, int32_t nk, int32_t nbands, const int32_t* npw,
                                   const int64_t* pw_off, const void* x, const void* hx, const double* eps,
                                   const double* kinetic, double* norms, const int32_t* rows, int32_t nrows,
                                   void* out, void* stream) {
  AMA_REQUIRE(precision == AMA_C64 || precision == AMA_C128, AMA_ERR_ARG, "bad precision");
  AMA_REQUIRE(npw && pw_off && x && hx && eps && kinetic && norms, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(nk >= 1 && nbands >= 1, AMA_ERR_SHAPE, "bad sizes");
  AMA_REQUIRE(!rows || (out && nrows >= 1), AMA_ERR_ARG, "out required with rows");
  cudaStream_t s = (cudaStream_t)stream;
  if (precision == AMA_C64)
    kbatch_residual_kernel<float><<<nk * nbands, kRowThreads, 0, s>>>(
        nbands, npw, pw_off, (const float2*)x, (const float2*)hx, eps, kinetic, norms, rows, nrows, (float2*)out);
  else
    kbatch_residual_kernel<double><<<nk * nbands, kRowThreads, 0, s>>>(
        nbands, npw, pw_off, (const double2*)x, (const double2*)hx, eps, kinetic, norms, rows, nrows, (double2*)out);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_kbatch_copy_rows(int32_t precision, int32_t nk, int32_t nrows, const int32_t* npw,
                                    const int64_t* pw_off, const void* src, int64_t src_rows_per_k,
                                    int64_t src_row0, void* dst, int64_t dst_rows_per_k, int64_t dst_row0,
                                    void* stream) {
  AMA_REQUIRE(precision == AMA_C64 || precision == AMA_C128, AMA_ERR_ARG, "bad precision");
  AMA_REQUIRE(npw && pw_off && src && dst, AMA_ERR_ARG, "null argument");
  if (nrows <= 0) return AMA_OK;
  dim3 grid(32, nk);
  cudaStream_t s = (cudaStream_t)stream;
  if (precision == AMA_C64)
    kbatch_copy_kernel<float2><<<grid, 256, 0, s>>>(nrows, npw, pw_off, (const float2*)src, src_rows_per_k, src_row0,
                                                    (float2*)dst, dst_rows_per_k, dst_row0);
  else
    kbatch_copy_kernel<double2><<<grid, 256, 0, s>>>(nrows, npw, pw_off, (const double2*)src, src_rows_per_k,
                                                     src_row0, (double2*)dst, dst_rows_per_k, dst_row0);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

// ---------------------------------------------------------------- structure sums
// out[g] = scale * sum_a radial[species[a]][g] * exp(-i G_g . tau_a): the superposition of
// per-species radial form factors with the atoms' phases (reference hamiltonian/local.py:
// 37-74, structure factors and per-species sums). One thread per G vector, looping over
// the atoms in FP64 (sincos of G.tau).
namespace {
__global__ void structure_sum_kernel(const double* __restrict__ gcart, int ng, const double* __restrict__ pos,
                                     const int* __restrict__ species, int natoms, const double* __restrict__ radial,
                                     double scale, double2* __restrict__ out) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
    const double gx = gcart[3 * g], gy = gcart[3 * g + 1], gz = gcart[3 * g + 2];
    double re = 0.0, im = 0.0;
    for (int a = 0; a < natoms; ++a) {
      const double th = gx * __ldg(pos + 3 * a) + gy * __ldg(pos + 3 * a + 1) + gz * __ldg(pos + 3 * a + 2);
      double s, c;
      sincos(th, &s, &c);
      const double f = __ldg(radial + (int64_t)__ldg(species + a) * ng + g);
      re += f * c;
      im -= f * s;
    }
    out[g] = make_double2(scale * re, scale * im);
  }
}
}  // namespace

extern "C" int ama_structure_sum(const double* gcart, int32_t ng, const double* positions, const int32_t* species,
                                 int32_t natoms, const double* radial, double scale, double* out, void* stream) {
  AMA_REQUIRE(gcart && positions && species && radial && out, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(ng >= 0 && natoms >= 0, AMA_ERR_SHAPE, "negative size");
  if (ng == 0) return AMA_OK;
  const int blocks = std::max(1, std::min(4 * 148, (ng + 255) / 256));
  structure_sum_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(gcart, ng, positions, species, natoms, radial,
                                                                 scale, (double2*)out);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}
