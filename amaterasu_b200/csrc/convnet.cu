// Periodic 3D convolution kernels of the learned start-density network (BF16 operands,
// FP32 accumulation), forward and backward, plus the elementwise pieces of the network.
//
// Tensors are [batch][channels][D][D][D] (cubic grids), row-major. A convolution has a
// 3x3x3 kernel w[co][ci][kz][ky][kx], stride 1 or 2 and circular padding of 1:
//   y[b][co][o] = bias[co] + sum_ci sum_k w[co][ci][k] x[b][ci][(s*o + k - 1) mod Din]
// with Dout = Din / s. Activations are BF16, the convolution outputs and all gradients
// FP32, weights BF16 (the trainer keeps FP32 master copies).
#include "common.cuh"

#include <cuda_bf16.h>

namespace {

constexpr int kConvThreads = 256;
constexpr int kCoTile = 8;  // output channels per thread

__device__ __forceinline__ int wrap(int i, int n) {
  i %= n;
  return i < 0 ? i + n : i;
}

// One thread: one output voxel x kCoTile output channels. Weights of the CTA's channel
// tile are staged in shared memory.
__global__ void __launch_bounds__(kConvThreads)
conv3d_fwd_kernel(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ w,
                  const float* __restrict__ bias, float* __restrict__ y, int ci_n, int co_n, int din, int stride) {
  extern __shared__ float wsm[];  // [kCoTile][ci_n][27]
  const int dout = din / stride;
  const int64_t vout = (int64_t)dout * dout * dout;
  const int co0 = blockIdx.y * kCoTile;
  const int b = blockIdx.z;
  for (int e = threadIdx.x; e < kCoTile * ci_n * 27; e += kConvThreads) {
    const int t = e / (ci_n * 27), r = e % (ci_n * 27);
    wsm[e] = (co0 + t < co_n) ? __bfloat162float(w[(int64_t)(co0 + t) * ci_n * 27 + r]) : 0.f;
  }
  __syncthreads();
  const int64_t o = blockIdx.x * (int64_t)kConvThreads + threadIdx.x;
  if (o >= vout) return;
  const int oz = o / (dout * dout), oy = (o / dout) % dout, ox = o % dout;
  float acc[kCoTile];
#pragma unroll
  for (int t = 0; t < kCoTile; ++t) acc[t] = (co0 + t < co_n) ? bias[co0 + t] : 0.f;
  const int64_t vin = (int64_t)din * din * din;
  const __nv_bfloat16* xb = x + (int64_t)b * ci_n * vin;
  int iz[3], iy[3], ix[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    iz[k] = wrap(stride * oz + k - 1, din);
    iy[k] = wrap(stride * oy + k - 1, din);
    ix[k] = wrap(stride * ox + k - 1, din);
  }
  for (int ci = 0; ci < ci_n; ++ci) {
    const __nv_bfloat16* xc = xb + (int64_t)ci * vin;
    const float* wc = wsm + ci * 27;
#pragma unroll
    for (int kz = 0; kz < 3; ++kz)
#pragma unroll
      for (int ky = 0; ky < 3; ++ky)
#pragma unroll
        for (int kx = 0; kx < 3; ++kx) {
          const float v = __bfloat162float(xc[((int64_t)iz[kz] * din + iy[ky]) * din + ix[kx]]);
          const int k = (kz * 3 + ky) * 3 + kx;
#pragma unroll
          for (int t = 0; t < kCoTile; ++t) acc[t] += wc[t * ci_n * 27 + k] * v;
        }
  }
  float* yb = y + ((int64_t)b * co_n) * vout + o;
#pragma unroll
  for (int t = 0; t < kCoTile; ++t)
    if (co0 + t < co_n) yb[(int64_t)(co0 + t) * vout] = acc[t];
}

// dx[b][ci][i] = sum_co sum_k w[co][ci][k] dy[b][co][o] over o with s*o + k - 1 == i (mod Din).
__global__ void __launch_bounds__(kConvThreads)
conv3d_bwd_data_kernel(const float* __restrict__ dy, const __nv_bfloat16* __restrict__ w, float* __restrict__ dx,
                       int ci_n, int co_n, int din, int stride) {
  extern __shared__ float wsm[];  // [kCoTile (ci)][co_n][27]
  const int dout = din / stride;
  const int64_t vin = (int64_t)din * din * din, vout = (int64_t)dout * dout * dout;
  const int ci0 = blockIdx.y * kCoTile;
  const int b = blockIdx.z;
  for (int e = threadIdx.x; e < kCoTile * co_n * 27; e += kConvThreads) {
    const int t = e / (co_n * 27), r = e % (co_n * 27);
    const int co = r / 27, k = r % 27;
    wsm[e] = (ci0 + t < ci_n) ? __bfloat162float(w[((int64_t)co * ci_n + ci0 + t) * 27 + k]) : 0.f;
  }
  __syncthreads();
  const int64_t i = blockIdx.x * (int64_t)kConvThreads + threadIdx.x;
  if (i >= vin) return;
  const int iz = i / (din * din), iy = (i / din) % din, ix = i % din;
  float acc[kCoTile];
#pragma unroll
  for (int t = 0; t < kCoTile; ++t) acc[t] = 0.f;
  const float* dyb = dy + (int64_t)b * co_n * vout;
  for (int kz = 0; kz < 3; ++kz) {
    const int pz = wrap(iz - kz + 1, din);
    if (pz % stride) continue;
    const int oz = pz / stride;
    for (int ky = 0; ky < 3; ++ky) {
      const int py = wrap(iy - ky + 1, din);
      if (py % stride) continue;
      const int oy = py / stride;
      for (int kx = 0; kx < 3; ++kx) {
        const int px = wrap(ix - kx + 1, din);
        if (px % stride) continue;
        const int ox = px / stride;
        const int k = (kz * 3 + ky) * 3 + kx;
        const int64_t oo = ((int64_t)oz * dout + oy) * dout + ox;
        for (int co = 0; co < co_n; ++co) {
          const float g = dyb[(int64_t)co * vout + oo];
#pragma unroll
          for (int t = 0; t < kCoTile; ++t) acc[t] += wsm[(t * co_n + co) * 27 + k] * g;
        }
      }
    }
  }
  float* dxb = dx + (int64_t)b * ci_n * vin + i;
#pragma unroll
  for (int t = 0; t < kCoTile; ++t)
    if (ci0 + t < ci_n) dxb[(int64_t)(ci0 + t) * vin] = acc[t];
}

// dw[co][ci][k] = sum_b sum_o dy[b][co][o] x[b][ci][s*o + k - 1]; one CTA per (co, ci),
// 27 register accumulators per thread, block reduction. dbias[co] from the ci == 0 CTA.
__global__ void __launch_bounds__(kConvThreads)
conv3d_bwd_weight_kernel(const float* __restrict__ dy, const __nv_bfloat16* __restrict__ x, float* __restrict__ dw,
                         float* __restrict__ dbias, int batch, int ci_n, int co_n, int din, int stride) {
  __shared__ float red[kConvThreads / 32][28];
  const int co = blockIdx.x / ci_n, ci = blockIdx.x % ci_n;
  const int dout = din / stride;
  const int64_t vin = (int64_t)din * din * din, vout = (int64_t)dout * dout * dout;
  float acc[28];
#pragma unroll
  for (int k = 0; k < 28; ++k) acc[k] = 0.f;
  for (int b = 0; b < batch; ++b) {
    const float* g = dy + ((int64_t)b * co_n + co) * vout;
    const __nv_bfloat16* xc = x + ((int64_t)b * ci_n + ci) * vin;
    for (int64_t o = threadIdx.x; o < vout; o += kConvThreads) {
      const float gv = g[o];
      const int oz = o / (dout * dout), oy = (o / dout) % dout, ox = o % dout;
      acc[27] += gv;
#pragma unroll
      for (int kz = 0; kz < 3; ++kz) {
        const int iz = wrap(stride * oz + kz - 1, din);
#pragma unroll
        for (int ky = 0; ky < 3; ++ky) {
          const int iy = wrap(stride * oy + ky - 1, din);
#pragma unroll
          for (int kx = 0; kx < 3; ++kx) {
            const int ix = wrap(stride * ox + kx - 1, din);
            acc[(kz * 3 + ky) * 3 + kx] += gv * __bfloat162float(xc[((int64_t)iz * din + iy) * din + ix]);
          }
        }
      }
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 28; ++k) {
    float v = acc[k];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if (lane == 0) red[wid][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < 28) {
    float s = 0.f;
    for (int w2 = 0; w2 < kConvThreads / 32; ++w2) s += red[w2][threadIdx.x];
    if (threadIdx.x < 27) dw[((int64_t)co * ci_n + ci) * 27 + threadIdx.x] = s;
    else if (ci == 0) dbias[co] = s;
  }
}

// y = silu(x) as BF16 (keeps nothing: the backward recomputes from the FP32 input)
__global__ void silu_fwd_kernel(const float* __restrict__ x, __nv_bfloat16* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float v = x[i];
    y[i] = __float2bfloat16(v / (1.f + __expf(-v)));
  }
}

// dx = dy * silu'(x)
__global__ void silu_bwd_kernel(const float* __restrict__ x, const float* __restrict__ dy, float* __restrict__ dx,
                                int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float v = x[i];
    const float s = 1.f / (1.f + __expf(-v));
    dx[i] = dy[i] * s * (1.f + v * (1.f - s));
  }
}

// nearest-neighbour x2 upsampling of [bc][d][d][d] BF16 -> [bc][2d][2d][2d] (fwd) and
// the sum over the 8 children (bwd, FP32).
__global__ void upsample2_fwd_kernel(const __nv_bfloat16* __restrict__ x, __nv_bfloat16* __restrict__ y, int64_t bc,
                                     int d) {
  const int D = 2 * d;
  const int64_t n = bc * (int64_t)D * D * D;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = i / ((int64_t)D * D * D);
    const int64_t r = i % ((int64_t)D * D * D);
    const int z = r / (D * D), yy = (r / D) % D, xx = r % D;
    y[i] = x[c * d * d * d + ((int64_t)(z >> 1) * d + (yy >> 1)) * d + (xx >> 1)];
  }
}

__global__ void upsample2_bwd_kernel(const float* __restrict__ dy, float* __restrict__ dx, int64_t bc, int d) {
  const int D = 2 * d;
  const int64_t n = bc * (int64_t)d * d * d;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = i / ((int64_t)d * d * d);
    const int64_t r = i % ((int64_t)d * d * d);
    const int z = r / (d * d), yy = (r / d) % d, xx = r % d;
    const float* src = dy + c * (int64_t)D * D * D;
    float s = 0.f;
    for (int a = 0; a < 2; ++a)
      for (int bb = 0; bb < 2; ++bb)
        for (int cc = 0; cc < 2; ++cc) s += src[((int64_t)(2 * z + a) * D + (2 * yy + bb)) * D + (2 * xx + cc)];
    dx[i] = s;
  }
}

int blocks_for(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 32); }

}  // namespace

extern "C" int ama_conv3d_fwd_bf16(const void* x, const void* w, const float* bias, float* y, int32_t batch,
                                   int32_t ci, int32_t co, int32_t din, int32_t stride, void* stream) {
  AMA_REQUIRE(x && w && bias && y, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(batch >= 1 && ci >= 1 && co >= 1 && din >= 1 && (stride == 1 || stride == 2) && din % stride == 0,
              AMA_ERR_SHAPE, "bad convolution sizes");
  const int dout = din / stride;
  const int64_t vout = (int64_t)dout * dout * dout;
  const size_t smem = (size_t)kCoTile * ci * 27 * sizeof(float);
  AMA_REQUIRE(smem <= 200 * 1024, AMA_ERR_UNSUPPORTED, "too many input channels");
  AMA_CUDA_TRY(cudaFuncSetAttribute(conv3d_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((vout + kConvThreads - 1) / kConvThreads, (co + kCoTile - 1) / kCoTile, batch);
  conv3d_fwd_kernel<<<grid, kConvThreads, smem, (cudaStream_t)stream>>>((const __nv_bfloat16*)x, (const __nv_bfloat16*)w,
                                                                         bias, y, ci, co, din, stride);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_conv3d_bwd_data_bf16(const float* dy, const void* w, float* dx, int32_t batch, int32_t ci,
                                        int32_t co, int32_t din, int32_t stride, void* stream) {
  AMA_REQUIRE(dy && w && dx, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(batch >= 1 && ci >= 1 && co >= 1 && din >= 1 && (stride == 1 || stride == 2) && din % stride == 0,
              AMA_ERR_SHAPE, "bad convolution sizes");
  const int64_t vin = (int64_t)din * din * din;
  const size_t smem = (size_t)kCoTile * co * 27 * sizeof(float);
  AMA_REQUIRE(smem <= 200 * 1024, AMA_ERR_UNSUPPORTED, "too many output channels");
  AMA_CUDA_TRY(cudaFuncSetAttribute(conv3d_bwd_data_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((vin + kConvThreads - 1) / kConvThreads, (ci + kCoTile - 1) / kCoTile, batch);
  conv3d_bwd_data_kernel<<<grid, kConvThreads, smem, (cudaStream_t)stream>>>(dy, (const __nv_bfloat16*)w, dx, ci, co,
                                                                             din, stride);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_conv3d_bwd_weight_bf16(const float* dy, const void* x, float* dw, float* dbias, int32_t batch,
                                          int32_t ci, int32_t co, int32_t din, int32_t stride, void* stream) {
  AMA_REQUIRE(dy && x && dw && dbias, AMA_ERR_ARG, "null argument");
  AMA_REQUIRE(batch >= 1 && ci >= 1 && co >= 1 && din >= 1 && (stride == 1 || stride == 2) && din % stride == 0,
              AMA_ERR_SHAPE, "bad convolution sizes");
  conv3d_bwd_weight_kernel<<<co * ci, kConvThreads, 0, (cudaStream_t)stream>>>(dy, (const __nv_bfloat16*)x, dw, dbias,
                                                                               batch, ci, co, din, stride);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_silu_fwd_bf16(const float* x, void* y, int64_t n, void* stream) {
  AMA_REQUIRE(x && y && n >= 0, AMA_ERR_ARG, "bad argument");
  if (n == 0) return AMA_OK;
  silu_fwd_kernel<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(x, (__nv_bfloat16*)y, n);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_silu_bwd(const float* x, const float* dy, float* dx, int64_t n, void* stream) {
  AMA_REQUIRE(x && dy && dx && n >= 0, AMA_ERR_ARG, "bad argument");
  if (n == 0) return AMA_OK;
  silu_bwd_kernel<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(x, dy, dx, n);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_upsample2_fwd_bf16(const void* x, void* y, int64_t bc, int32_t d, void* stream) {
  AMA_REQUIRE(x && y && bc >= 1 && d >= 1, AMA_ERR_ARG, "bad argument");
  upsample2_fwd_kernel<<<blocks_for(bc * 8LL * d * d * d), 256, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)x, (__nv_bfloat16*)y, bc, d);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}

extern "C" int ama_upsample2_bwd(const float* dy, float* dx, int64_t bc, int32_t d, void* stream) {
  AMA_REQUIRE(dy && dx && bc >= 1 && d >= 1, AMA_ERR_ARG, "bad argument");
  upsample2_bwd_kernel<<<blocks_for(bc * (int64_t)d * d * d), 256, 0, (cudaStream_t)stream>>>(dy, dx, bc, d);
  AMA_CHECK_LAUNCH();
  return AMA_OK;
}
