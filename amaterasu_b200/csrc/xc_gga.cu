// PBE and PBEsol exchange-correlation on the grid, FP64 on the GPU.
//
// v_s(r) = d(n eps)/dn_s - div( 2 vsigma_ss grad n_s + vsigma_ud grad n_s' ),
// E_xc = sum_r n eps dV, with the gradients and the divergence taken spectrally (i G, the
// Nyquist frequency zeroed) by ama_grid_gradient / ama_grid_divergence. The pointwise
// kernel evaluates, per grid point,
//
//   exchange (exact spin scaling, per channel):
//     e_x = -C_X n_s^{4/3} F(s^2),  F = 1 + kappa mu s^2 / (kappa + mu s^2),
//     s^2 = X2S^2 sigma_ss / n_s^{8/3};
//     d e_x/dn_s = -(4/3) C_X n_s^{1/3} (F - 2 kappa^2 mu s^2 / D^2),  D = kappa + mu s^2,
//     d e_x/dsigma_ss = -C_X kappa^2 mu X2S^2 / (n_s^{4/3} D^2);
//   correlation (PBE's H on the modified PW92 local part):
//     eps_c = eps_lda(rs, zeta) + H,  H = gamma phi^3 ln(1 + w),
//     w = (beta/gamma) u / (1 + A u),  u = t^2 + A t^4,  A = (beta/gamma) / (e^y - 1),
//     y = -eps_lda / (gamma phi^3),  t^2 = sigma_tot / (16 2^{2/3} phi^2 rs n^{8/3}),
//   with the derivatives by the chain rule through (rs, zeta, phi, A, t^2):
//     dH/dt^2 = phi^3 beta (1 + 2 A t^2) / ((1 + w) (1 + A u)^2),
//     dH/dA   = phi^3 beta (t^4 - u^2) / ((1 + w) (1 + A u)^2),
//     dH/dphi = 3 gamma phi^2 ln(1 + w)  (explicit),
//     dA/deps = beta e^y / (gamma^2 phi^3 (e^y - 1)^2),  dA/dphi = -3 eps_lda dA/deps / phi,
//     n d eps_c/dn |zeta = -(rs/3) eps_lda,rs (1 + H_A A_eps) - (7/3) t^2 H_t2,
//     v_c^{u,d} = eps_c + n d eps_c/dn |zeta +/- (1 -/+ zeta) d eps_c/dzeta |n,
//     vsigma_c = n H_t2 t^2 / sigma_tot (formed without dividing by sigma_tot).
// Thresholds as in the reference (amaterasu xc/gga.py:112-254, xc/lda.py:97-103): points
// with n <= 1e-24 give zero, a channel with n_s <= 1e-24 has no exchange, zeta is clipped to
// [-1, 1] and 1 +/- zeta floored at 1e-24 inside phi.
//
// The kernel also forms the gradient part of the stress, sum_r [2 vsigma_uu g_u g_u +
// vsigma_ud (g_u g_d + g_d g_u) + 2 vsigma_dd g_d g_d] dV, and reduces the energy and those
// six components deterministically (per-CTA partials, then one CTA in a fixed order).
#include "common.cuh"
#include "engine_impl.cuh"

#include <cmath>

using namespace ama;

extern "C" int ama_grid_gradient(AmaEngine* e, const double* cell, const double* in, double scale, double* out,
                                 void* stream);
extern "C" int ama_grid_divergence(AmaEngine* e, const double* cell, const double* in, double alpha, double beta,
                                   double* out, void* stream);

namespace {

constexpr int kXcT = 256;
constexpr int kXcOut = 7;  // energy, stress xx yy zz yz xz xy
constexpr double kThr = 1e-24;
constexpr double kCx = 0.9305257363491000250020102180716672510262;
constexpr double kRs = 0.6203504908994000166680068120477781673508;
constexpr double kX2S = 0.1282782438530421943003109254455883701296;
constexpr double kGamma = 0.031090690869654895034;
constexpr double kKappa = 0.804;
constexpr double kFz20 = 1.709920934161365617563962776245;

struct GgaParams {
  double mu, beta;
};

struct Pw92 {
  double a, a1, b1, b2, b3, b4;
};
__constant__ Pw92 kPw92[3] = {{0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294},
                              {0.01554535, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517},
                              {0.0168869, 0.11125, 10.357, 3.6231, 0.88026, 0.49671}};

// G(rs) of PW92 and dG/drs
__device__ __forceinline__ void pw92_g(double rs, const Pw92& c, double& g, double& dg) {
  const double srs = sqrt(rs);
  const double q = srs * (c.b1 + srs * (c.b2 + srs * (c.b3 + srs * c.b4)));
  const double dq = 0.5 * c.b1 / srs + c.b2 + 1.5 * c.b3 * srs + 2.0 * c.b4 * rs;
  const double lg = log1p(1.0 / (2.0 * c.a * q));
  g = -2.0 * c.a * (1.0 + c.a1 * rs) * lg;
  dg = -2.0 * c.a * c.a1 * lg + 2.0 * c.a * (1.0 + c.a1 * rs) * dq / (2.0 * c.a * q * q + q);
}

// one exchange channel: energy density, d/dn_s, d/dsigma_ss
__device__ __forceinline__ void exchange_channel(double ns, double sig, double mu, double& e, double& vn, double& vs) {
  const double n13 = cbrt(ns), n43 = ns * n13;
  const double s2 = kX2S * kX2S * sig / (n43 * n43);
  const double D = kKappa + mu * s2;
  const double F = 1.0 + kKappa * mu * s2 / D;
  e = -kCx * n43 * F;
  vn = -(4.0 / 3.0) * kCx * n13 * (F - 2.0 * kKappa * kKappa * mu * s2 / (D * D));
  vs = -kCx * kKappa * kKappa * mu * kX2S * kX2S / (n43 * D * D);
}

// correlation: n eps_c, v_c^u, v_c^d, vsigma_tot
__device__ __forceinline__ void correlation(double nu, double nd, double sig_tot, double beta, double& e, double& vu,
                                            double& vd, double& vsig) {
  const double n = nu + nd;
  const double n13 = cbrt(n);
  const double rs = kRs / n13;
  const double z = fmin(1.0, fmax(-1.0, (nu - nd) / n));
  const double opz = fmax(1.0 + z, 0.0), omz = fmax(1.0 - z, 0.0);
  const double den = 2.0 * cbrt(2.0) - 2.0;  // 2^{4/3} - 2
  const double co = cbrt(opz), cm = cbrt(omz);
  const double fz = (opz * co + omz * cm - 2.0) / den;
  const double dfz = (4.0 / 3.0) * (co - cm) / den;
  double g0, dg0, g1, dg1, g2, dg2;
  pw92_g(rs, kPw92[0], g0, dg0);
  pw92_g(rs, kPw92[1], g1, dg1);
  pw92_g(rs, kPw92[2], g2, dg2);
  const double z3 = z * z * z, z4 = z3 * z;
  const double br = g1 - g0 + g2 / kFz20;
  const double el = g0 + z4 * fz * br - fz * g2 / kFz20;
  const double el_rs = dg0 + z4 * fz * (dg1 - dg0 + dg2 / kFz20) - fz * dg2 / kFz20;
  const double el_z = (4.0 * z3 * fz + z4 * dfz) * br - dfz * g2 / kFz20;
  // spin scaling phi
  const double op = fmax(1.0 + z, kThr), om = fmax(1.0 - z, kThr);
  const double cop = cbrt(op), com = cbrt(om);
  const double phi = 0.5 * (cop * cop + com * com);
  const double dphi = (1.0 / 3.0) * (1.0 / cop - 1.0 / com);
  const double phi2 = phi * phi, phi3 = phi2 * phi;
  // t^2 = K sigma_tot
  const double n83 = (n * n13) * (n * n13);
  const double c16 = 16.0 * cbrt(4.0);  // (4 2^{1/3})^2
  const double K = 1.0 / (c16 * phi2 * rs * n83);
  const double t2 = K * sig_tot;
  const double y = -el / (kGamma * phi3);
  const double E = expm1(y);
  const double Es = fabs(E) < 1e-300 ? 1e-300 : E;
  const double A = beta / (kGamma * Es);
  const double u = t2 + A * t2 * t2;
  const double Dd = 1.0 + A * u;
  const double w = beta * u / (kGamma * Dd);
  const double lw = log1p(w);
  const double H = kGamma * phi3 * lw;
  const double pre = phi3 * beta / ((1.0 + w) * Dd * Dd);
  const double H_t2 = pre * (1.0 + 2.0 * A * t2);
  const double H_A = pre * (t2 * t2 - u * u);
  const double H_phi = 3.0 * kGamma * phi2 * lw;
  const double A_eps = beta * (E + 1.0) / (kGamma * kGamma * phi3 * Es * Es);
  const double A_phi = -3.0 * el * A_eps / phi;
  const double ec = el + H;
  const double n_dn = -(rs / 3.0) * el_rs * (1.0 + H_A * A_eps) - (7.0 / 3.0) * t2 * H_t2;
  const double d_z = el_z + H_phi * dphi + H_A * (A_eps * el_z + A_phi * dphi) - 2.0 * t2 / phi * H_t2 * dphi;
  const double common = ec + n_dn;
  e = n * ec;
  vu = common + (1.0 - z) * d_z;
  vd = common - (1.0 + z) * d_z;
  vsig = n * H_t2 * K;
}

// Per point: rho (nspin N), gradients g_u = gscale * grad[0..3N), g_d = gscale * grad[3N..6N)
// (nspin 1: the same buffer for both channels, n_s = rho / 2). Writes v (nspin N, the local
// part), flux (nspin x 3N: 2 vsigma_ss g_s + vsigma_ud g_s') and per-CTA partials.
__global__ void __launch_bounds__(kXcT) gga_point_kernel(int64_t N, int nspin, GgaParams prm, const double* __restrict__ rho,
                                                         const double* __restrict__ grad, double gscale,
                                                         double* __restrict__ v, double* __restrict__ flux,
                                                         double* __restrict__ part) {
  __shared__ double red[kXcT / 32][kXcOut];
  double acc[kXcOut] = {};
  for (int64_t i = blockIdx.x * (int64_t)kXcT + threadIdx.x; i < N; i += (int64_t)gridDim.x * kXcT) {
    const double ru = nspin == 1 ? 0.5 * rho[i] : rho[i];
    const double rd = nspin == 1 ? ru : rho[N + i];
    const double* gdp = nspin == 1 ? grad : grad + 3 * N;
    const double gu[3] = {gscale * grad[i], gscale * grad[N + i], gscale * grad[2 * N + i]};
    const double gd[3] = {gscale * gdp[i], gscale * gdp[N + i], gscale * gdp[2 * N + i]};
    const double suu = gu[0] * gu[0] + gu[1] * gu[1] + gu[2] * gu[2];
    const double sud = gu[0] * gd[0] + gu[1] * gd[1] + gu[2] * gd[2];
    const double sdd = gd[0] * gd[0] + gd[1] * gd[1] + gd[2] * gd[2];
    const double n = ru + rd;
    double vu = 0.0, vd = 0.0, vsu = 0.0, vsd = 0.0, vsc = 0.0, en = 0.0;
    if (n > kThr) {
      double e, a, b;
      if (ru > kThr) {
        exchange_channel(ru, fmax(suu, 0.0), prm.mu, e, a, b);
        en += e; vu += a; vsu += b;
      }
      if (rd > kThr) {
        exchange_channel(rd, fmax(sdd, 0.0), prm.mu, e, a, b);
        en += e; vd += a; vsd += b;
      }
      double ce, cu, cd, cs;
      correlation(ru, rd, fmax(suu + 2.0 * sud + sdd, 0.0), prm.beta, ce, cu, cd, cs);
      en += ce; vu += cu; vd += cd; vsc = cs;
    }
    // vsigma_uu = vsu + vsc, vsigma_ud = 2 vsc, vsigma_dd = vsd + vsc
    const double wuu = vsu + vsc, wud = 2.0 * vsc, wdd = vsd + vsc;
    v[i] = vu;
    if (nspin == 2) v[N + i] = vd;
    for (int c = 0; c < 3; ++c) {
      flux[c * N + i] = 2.0 * wuu * gu[c] + wud * gd[c];
      if (nspin == 2) flux[(3 + c) * N + i] = 2.0 * wdd * gd[c] + wud * gu[c];
    }
    acc[0] += en;
    const int pa[6][2] = {{0, 0}, {1, 1}, {2, 2}, {1, 2}, {0, 2}, {0, 1}};
    for (int c = 0; c < 6; ++c) {
      const int a = pa[c][0], b = pa[c][1];
      acc[1 + c] += 2.0 * wuu * gu[a] * gu[b] + wud * (gu[a] * gd[b] + gd[a] * gu[b]) + 2.0 * wdd * gd[a] * gd[b];
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = 0; c < kXcOut; ++c) {
    double t = acc[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) red[warp][c] = t;
  }
  __syncthreads();
  if (threadIdx.x < kXcOut) {
    double t = 0.0;
    for (int w = 0; w < kXcT / 32; ++w) t += red[w][threadIdx.x];
    part[(int64_t)blockIdx.x * kXcOut + threadIdx.x] = t;
  }
}

__global__ void __launch_bounds__(kXcT) gga_finish_kernel(int nblocks, double dv, const double* __restrict__ part,
                                                          double* __restrict__ out) {
  if (threadIdx.x < kXcOut) {
    double t = 0.0;
    for (int b = 0; b < nblocks; ++b) t += part[(int64_t)b * kXcOut + threadIdx.x];
    out[threadIdx.x] = t * dv;
  }
}

struct XcScratch {
  double* buf = nullptr;
  size_t bytes = 0;
};
thread_local PerDevice<XcScratch> g_xc_scratch;

}  // namespace

extern "C" int ama_xc_gga(AmaEngine* e, int32_t functional, int32_t nspin, const double* cell, const double* rho,
                          double* vxc, double* result, void* stream) {
  AMA_REQUIRE(e && cell && rho && vxc && result, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(functional == 0 || functional == 1, AMA_ERR_ARG, "functional must be 0 (PBE) or 1 (PBEsol)");
  AMA_REQUIRE(nspin == 1 || nspin == 2, AMA_ERR_ARG, "nspin must be 1 or 2");
  const GgaParams prm = functional == 0 ? GgaParams{0.2195149727645171, 0.06672455060314922}
                                        : GgaParams{10.0 / 81.0, 0.046};
  const int64_t N = e->N;
  const int nblocks = (int)std::min<int64_t>((N + kXcT - 1) / kXcT, 8 * 148);
  // scratch: gradients (nspin x 3N), fluxes (nspin x 3N), partials
  const size_t need = sizeof(double) * ((size_t)12 * N + (size_t)nblocks * kXcOut);
  XcScratch* scp = g_xc_scratch.here();
  AMA_REQUIRE(scp, AMA_ERR_UNSUPPORTED, "device index out of range");
  XcScratch& sc = *scp;
  if (sc.bytes < need) {
    bump_memory_epoch();
    if (sc.buf) AMA_CUDA_TRY(cudaFree(sc.buf));
    sc.buf = nullptr;
    sc.bytes = 0;
    AMA_CUDA_TRY(cudaMalloc((void**)&sc.buf, need));
    sc.bytes = need;
  }
  double* grad = sc.buf;
  double* flux = grad + 6 * N;
  double* part = flux + 6 * N;
  cudaStream_t s = (cudaStream_t)stream;
  // nspin 1: one gradient of the total density, each channel's gradient being half of it
  for (int sp = 0; sp < nspin; ++sp)
    if (int rc = ama_grid_gradient(e, cell, rho + sp * N, 1.0, grad + 3 * sp * N, stream)) return rc;
  gga_point_kernel<<<nblocks, kXcT, 0, s>>>(N, nspin, prm, rho, grad, nspin == 1 ? 0.5 : 1.0, vxc, flux, part);
  AMA_CHECK_LAUNCH();
  for (int sp = 0; sp < nspin; ++sp)
    if (int rc = ama_grid_divergence(e, cell, flux + 3 * sp * N, -1.0, 1.0, vxc + sp * N, stream)) return rc;
  double det = cell[0] * (cell[4] * cell[8] - cell[5] * cell[7]) - cell[1] * (cell[3] * cell[8] - cell[5] * cell[6]) +
               cell[2] * (cell[3] * cell[7] - cell[4] * cell[6]);
  gga_finish_kernel<<<1, kXcT, 0, s>>>(nblocks, fabs(det) / (double)N, part, result);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}
