// Ion-ion Ewald energy, forces and stress in FP64 on the GPU.
//
// E = 1/2 sum'_{a,b,R} Z_a Z_b erfc(eta r)/r            (r = |tau_a - tau_b + R|, real space)
//   + (2 pi / Omega) sum_{G != 0} |S(G)|^2 f(G^2)       (f(x) = exp(-x / 4 eta^2) / x,
//                                                         S(G) = sum_a Z_a exp(i G.tau_a))
//   - eta / sqrt(pi) sum_a Z_a^2 - pi Q^2 / (2 Omega eta^2)
// Forces F_a = -dE/dtau_a; stress sigma = (1/Omega) dE/d eps (eps the strain).
//
// Work decomposition: one CTA per atom for the real-space sum (its threads stride over the
// (partner, translation) pairs; terms beyond the cutoff radius are skipped), one CTA per
// atom for the reciprocal-space force, and G-parallel CTAs for the structure factors and
// the reciprocal energy and stress. Every CTA writes its partial sums to its own slot and
// a final single-CTA pass adds the slots in a fixed order, so results are reproducible bit
// for bit. The lattice translations and G vectors come from the host (they depend only on
// the cell and the cutoffs).
#include "common.cuh"

#include <cmath>

using namespace ama;

namespace {

constexpr int kEwT = 256;
constexpr int kOut = 10;  // energy, 3 force components, 6 stress components (xx yy zz yz xz xy)

__device__ __forceinline__ double block_sum_ew(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kEwT / 32; ++w) t += red[w];
  return t;  // valid in thread 0
}

// Real space: CTA a sums over partners b and translations R.
__global__ void __launch_bounds__(kEwT)
ewald_real_kernel(int natoms, const double* __restrict__ pos, const double* __restrict__ z,
                  const double* __restrict__ shifts, int nshift, double eta, double rcut, double inv_volume,
                  double* __restrict__ part) {
  __shared__ double red[kEwT / 32];
  const int a = blockIdx.x;
  const double ax = pos[3 * a], ay = pos[3 * a + 1], az = pos[3 * a + 2], za = z[a];
  const double c2 = 2.0 * eta / sqrt(M_PI);
  double acc[kOut] = {};
  const int64_t total = (int64_t)natoms * nshift;
  for (int64_t q = threadIdx.x; q < total; q += kEwT) {
    const int b = (int)(q / nshift), t = (int)(q % nshift);
    const double dx = ax - pos[3 * b] + shifts[3 * t];
    const double dy = ay - pos[3 * b + 1] + shifts[3 * t + 1];
    const double dz = az - pos[3 * b + 2] + shifts[3 * t + 2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 == 0.0 || r2 > rcut * rcut) continue;  // the atom itself, or beyond the cutoff
    const double r = sqrt(r2);
    const double zz = za * z[b];
    const double er = erfc(eta * r) / r;
    const double g = zz * (er + c2 * exp(-eta * eta * r2)) / r2;  // -zz phi'(r) / r
    acc[0] += 0.5 * zz * er;
    acc[1] += g * dx;
    acc[2] += g * dy;
    acc[3] += g * dz;
    const double s = -0.5 * g * inv_volume;
    acc[4] += s * dx * dx;
    acc[5] += s * dy * dy;
    acc[6] += s * dz * dz;
    acc[7] += s * dy * dz;
    acc[8] += s * dx * dz;
    acc[9] += s * dx * dy;
  }
  for (int c = 0; c < kOut; ++c) {
    const double t = block_sum_ew(acc[c], red);
    if (threadIdx.x == 0) part[(int64_t)a * kOut + c] = t;
  }
}

// Structure factors S(G) and the per-G reciprocal energy and stress terms.
__global__ void __launch_bounds__(kEwT)
ewald_sfac_kernel(int natoms, const double* __restrict__ pos, const double* __restrict__ z,
                  const double* __restrict__ gv, int ng, double eta, double volume, double2* __restrict__ sfac,
                  double* __restrict__ gpart) {
  const int g = blockIdx.x * kEwT + threadIdx.x;
  if (g >= ng) return;
  const double gx = gv[3 * g], gy = gv[3 * g + 1], gz = gv[3 * g + 2];
  double re = 0.0, im = 0.0;
  for (int a = 0; a < natoms; ++a) {
    double sn, cs;
    sincos(gx * pos[3 * a] + gy * pos[3 * a + 1] + gz * pos[3 * a + 2], &sn, &cs);
    re += z[a] * cs;
    im += z[a] * sn;
  }
  sfac[g] = make_double2(re, im);
  const double g2 = gx * gx + gy * gy + gz * gz;
  const double w = 2.0 * M_PI / volume * exp(-g2 / (4.0 * eta * eta)) / g2 * (re * re + im * im);
  const double h = 2.0 * (1.0 / (4.0 * eta * eta) + 1.0 / g2) / volume;
  double* o = gpart + (int64_t)g * 7;
  o[0] = w;
  o[1] = w * (h * gx * gx - 1.0 / volume);
  o[2] = w * (h * gy * gy - 1.0 / volume);
  o[3] = w * (h * gz * gz - 1.0 / volume);
  o[4] = w * h * gy * gz;
  o[5] = w * h * gx * gz;
  o[6] = w * h * gx * gy;
}

// Reciprocal force on atom a: (4 pi / Omega) Z_a sum_G f(G^2) G Im(e^{i G.tau_a} conj S(G)).
__global__ void __launch_bounds__(kEwT)
ewald_recip_force_kernel(const double* __restrict__ pos, const double* __restrict__ z,
                         const double* __restrict__ gv, int ng, const double2* __restrict__ sfac, double eta,
                         double volume, double* __restrict__ fpart) {
  __shared__ double red[kEwT / 32];
  const int a = blockIdx.x;
  const double ax = pos[3 * a], ay = pos[3 * a + 1], az = pos[3 * a + 2];
  double f[3] = {};
  for (int g = threadIdx.x; g < ng; g += kEwT) {
    const double gx = gv[3 * g], gy = gv[3 * g + 1], gz = gv[3 * g + 2];
    const double g2 = gx * gx + gy * gy + gz * gz;
    double sn, cs;
    sincos(gx * ax + gy * ay + gz * az, &sn, &cs);
    const double2 s = sfac[g];
    const double m = exp(-g2 / (4.0 * eta * eta)) / g2 * (sn * s.x - cs * s.y);  // f(G^2) Im(e^{i G.tau} conj S)
    f[0] += m * gx;
    f[1] += m * gy;
    f[2] += m * gz;
  }
  const double pref = 4.0 * M_PI / volume * z[a];
  for (int c = 0; c < 3; ++c) {
    const double t = block_sum_ew(f[c], red);
    if (threadIdx.x == 0) fpart[(int64_t)a * 3 + c] = pref * t;
  }
}

// out[0] energy; out[1 + 3a + c] force; out[1 + 3 natoms + 0..8] stress (row-major 3x3).
__global__ void __launch_bounds__(kEwT)
ewald_finish_kernel(int natoms, int ng, const double* __restrict__ z, const double* __restrict__ part,
                    const double* __restrict__ gpart, const double* __restrict__ fpart, double eta, double volume,
                    double* __restrict__ out) {
  __shared__ double red[kEwT / 32];
  // real-space energy and stress plus reciprocal energy and stress, each summed in a fixed order
  double e = 0.0, s[6] = {}, q = 0.0, z2 = 0.0;
  for (int a = threadIdx.x; a < natoms; a += kEwT) {
    e += part[(int64_t)a * kOut];
    for (int c = 0; c < 6; ++c) s[c] += part[(int64_t)a * kOut + 4 + c];
    q += z[a];
    z2 += z[a] * z[a];
  }
  double er = 0.0, sr[6] = {};
  for (int g = threadIdx.x; g < ng; g += kEwT) {
    er += gpart[(int64_t)g * 7];
    for (int c = 0; c < 6; ++c) sr[c] += gpart[(int64_t)g * 7 + 1 + c];
  }
  const double E = block_sum_ew(e, red), ER = block_sum_ew(er, red);
  const double Q = block_sum_ew(q, red), Z2 = block_sum_ew(z2, red);
  double S[6], SR[6];
  for (int c = 0; c < 6; ++c) {
    S[c] = block_sum_ew(s[c], red);
    SR[c] = block_sum_ew(sr[c], red);
  }
  if (threadIdx.x == 0) {
    const double background = M_PI * Q * Q / (2.0 * volume * eta * eta);
    out[0] = E + ER - eta / sqrt(M_PI) * Z2 - background;
    const double diag = background / volume;
    const double st[6] = {S[0] + SR[0] + diag, S[1] + SR[1] + diag, S[2] + SR[2] + diag,
                          S[3] + SR[3], S[4] + SR[4], S[5] + SR[5]};
    double* o = out + 1 + 3 * natoms;
    o[0] = st[0]; o[4] = st[1]; o[8] = st[2];
    o[5] = o[7] = st[3];
    o[2] = o[6] = st[4];
    o[1] = o[3] = st[5];
  }
  for (int a = threadIdx.x; a < natoms; a += kEwT)
    for (int c = 0; c < 3; ++c) out[1 + 3 * a + c] = part[(int64_t)a * kOut + 1 + c] + fpart[(int64_t)a * 3 + c];
}

}  // namespace

extern "C" int ama_ewald(int32_t natoms, const double* positions, const double* charges, const double* shifts,
                         int32_t nshift, const double* gvectors, int32_t ng, double eta, double rcut, double volume,
                         double* work, double* out, void* stream) {
  AMA_REQUIRE(positions && charges && shifts && out && work && (ng == 0 || gvectors), AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(natoms >= 1 && nshift >= 1 && ng >= 0, AMA_ERR_SHAPE, "bad sizes");
  AMA_REQUIRE(eta > 0.0 && rcut > 0.0 && volume > 0.0, AMA_ERR_ARG, "eta, rcut and volume must be positive");
  cudaStream_t s = (cudaStream_t)stream;
  // the double2 array first: work is 16-byte aligned, the double arrays need only 8
  AMA_REQUIRE(((uintptr_t)work & 15u) == 0, AMA_ERR_ARG, "ama_ewald: work must be 16-byte aligned");
  double2* sfac = (double2*)work;                        // [ng]
  double* part = work + 2 * (int64_t)ng;                 // [natoms][10]
  double* fpart = part + (int64_t)natoms * kOut;         // [natoms][3]
  double* gpart = fpart + (int64_t)natoms * 3;           // [ng][7]
  ewald_real_kernel<<<natoms, kEwT, 0, s>>>(natoms, positions, charges, shifts, nshift, eta, rcut, 1.0 / volume,
                                            part);
  if (ng > 0) {
    ewald_sfac_kernel<<<(ng + kEwT - 1) / kEwT, kEwT, 0, s>>>(natoms, positions, charges, gvectors, ng, eta, volume,
                                                              sfac, gpart);
    ewald_recip_force_kernel<<<natoms, kEwT, 0, s>>>(positions, charges, gvectors, ng, sfac, eta, volume, fpart);
  } else {
    AMA_CUDA_TRY(cudaMemsetAsync(fpart, 0, sizeof(double) * 3 * (size_t)natoms, s));
  }
  ewald_finish_kernel<<<1, kEwT, 0, s>>>(natoms, ng, charges, part, gpart, fpart, eta, volume, out);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}
