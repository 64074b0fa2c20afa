// surrogate.cu - kernels of the learned conduction surrogate
// (include/lare_surrogate.h): bf16 tensor-core convolutions for training and
// inference, the loss, the optimiser, and the glue between the network and
// the resident MHD state (feature extraction, window gather, update, plain
// RKL2 re-check of sampled patches).
//
// Convolutions are implicit GEMMs on mma.sync m16n8k16 (bf16 in, FP32
// accumulate): rows = output voxels, columns = output channels, reduction =
// 27 taps x input channels.  A CTA of 4 warps keeps the layer's weights in
// shared memory (rows padded by 8 bf16 so that the B-fragment loads of a
// warp hit 32 different banks) and walks tiles of 128 output voxels, 32 per
// warp.  The weight gradient is the transposed GEMM (rows = output channels,
// columns = input channels, reduction = voxels) with per-chunk partials
// summed in a fixed order, so training is deterministic.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdint>

#include "../../include/lare_gpu.h"
#include "../../include/lare_surrogate.h"

namespace {

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ void mma_16816(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t ld32(const bf16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ uint32_t pack2f(float lo, float hi) {
  return pack2(__float2bfloat16(lo), __float2bfloat16(hi));
}

}  // namespace

#include "conv_tc.cuh"

namespace {

int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

// ---------------------------------------------------------------------
// Convolution (forward, and backward-data with pad = 2).
constexpr int kConvThreads = 128;
constexpr int kWarpRows = 32;                             // output voxels per warp
constexpr int kTileRows = kWarpRows * kConvThreads / 32;  // per CTA tile

template <int CIN>
struct WRow {
  static constexpr int stride = CIN + 8;  // bf16 per smem weight row
};

template <int CIN, int COUT>
constexpr size_t conv_smem() {
  return (size_t)27 * COUT * WRow<CIN>::stride * sizeof(bf16);
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) k_conv(const bf16* __restrict__ x, int din, int pad,
                                                       const bf16* __restrict__ w, const float* __restrict__ bias,
                                                       void* __restrict__ y, int dout, int nb,
                                                       const bf16* __restrict__ mask, int relu, int out_f32) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  bf16* ws = reinterpret_cast<bf16*>(smem_raw);
  constexpr int RS = WRow<CIN>::stride;
  constexpr int NJ = COUT / 8;
  // stage [27][COUT][CIN] -> [27][COUT][RS] in 4-byte words
  for (int i = threadIdx.x; i < 27 * COUT * CIN / 2; i += blockDim.x) {
    const int row = i / (CIN / 2), col = i - row * (CIN / 2);
    reinterpret_cast<uint32_t*>(ws + row * RS)[col] = reinterpret_cast<const uint32_t*>(w)[i];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const long long vox = (long long)dout * dout * dout;
  const long long M = vox * nb;
  const long long ntiles = (M + kTileRows - 1) / kTileRows;
  const long long dd = (long long)din * din;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long m0 = tile * kTileRows + warp * kWarpRows;
    // four rows per thread: g, g+8, g+16, g+24 of the warp's 32
    long long row[4], base[4];
    int oz[4], oy[4], ox[4];
    bool valid[4];
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      long long r = m0 + g + 8 * h;
      valid[h] = r < M;
      if (!valid[h]) r = M - 1;
      row[h] = r;
      const long long b = r / vox;
      const long long v = r - b * vox;
      ox[h] = (int)(v % dout);
      oy[h] = (int)((v / dout) % dout);
      oz[h] = (int)(v / ((long long)dout * dout));
      base[h] = b * dd * din;
    }
    float acc[2][NJ][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[mt][j][q] = 0.f;
    for (int tap = 0; tap < 27; ++tap) {
      const int dz = tap / 9 - pad, dy = (tap / 3) % 3 - pad, dx = tap % 3 - pad;
      const bf16* src[4];
      bool ok[4];
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const int iz = oz[h] + dz, iy = oy[h] + dy, ix = ox[h] + dx;
        ok[h] = (unsigned)iz < (unsigned)din && (unsigned)iy < (unsigned)din && (unsigned)ix < (unsigned)din;
        src[h] = x + (ok[h] ? (base[h] + (iz * dd + (long long)iy * din + ix)) * CIN : 0);
      }
      const bf16* wt = ws + tap * COUT * RS;
#pragma unroll
      for (int kc = 0; kc < CIN / 16; ++kc) {
        uint32_t a[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
          const int h0 = 2 * mt, h1 = 2 * mt + 1;  // rows g + 16 mt and g + 16 mt + 8
          a[mt][0] = ok[h0] ? ld32(src[h0] + kc * 16 + 2 * t) : 0u;
          a[mt][1] = ok[h1] ? ld32(src[h1] + kc * 16 + 2 * t) : 0u;
          a[mt][2] = ok[h0] ? ld32(src[h0] + kc * 16 + 8 + 2 * t) : 0u;
          a[mt][3] = ok[h1] ? ld32(src[h1] + kc * 16 + 8 + 2 * t) : 0u;
        }
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          const bf16* wr = wt + (j * 8 + g) * RS + kc * 16;
          const uint32_t b[2] = {ld32(wr + 2 * t), ld32(wr + 8 + 2 * t)};
          mma_16816(acc[0][j], a[0], b);
          mma_16816(acc[1][j], a[1], b);
        }
      }
    }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int co = j * 8 + 2 * t;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          const int h = 2 * mt + hh;
          if (!valid[h]) continue;
          float v0 = acc[mt][j][2 * hh], v1 = acc[mt][j][2 * hh + 1];
          if (bias) {
            v0 += bias[co];
            v1 += bias[co + 1];
          }
          if (relu) {
            v0 = fmaxf(v0, 0.f);
            v1 = fmaxf(v1, 0.f);
          }
          const long long o = row[h] * COUT + co;
          if (mask) {
            const uint32_t mk = ld32(mask + o);
            if (!(__bfloat162float(__ushort_as_bfloat16((unsigned short)(mk & 0xffffu))) > 0.f)) v0 = 0.f;
            if (!(__bfloat162float(__ushort_as_bfloat16((unsigned short)(mk >> 16))) > 0.f)) v1 = 0.f;
          }
          if (out_f32) {
            *reinterpret_cast<float2*>(reinterpret_cast<float*>(y) + o) = make_float2(v0, v1);
          } else {
            *reinterpret_cast<uint32_t*>(reinterpret_cast<bf16*>(y) + o) = pack2f(v0, v1);
          }
        }
      }
  }
}

bool g_use_tc = true;  // tcgen05 convolution (else the mma.sync one)

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

template <int CIN, int NTC, int COUT>
int launch_conv_tc(const void* x, int din, int pad, const void* w, const float* bias, void* y, int nb,
                   const void* mask, int relu, int out_f32, cudaStream_t s) {
  const TcGeom g = tc_geom(din, pad, nb);
  const size_t smem = tc_smem_bytes<CIN, NTC>(g.SS);
  if (smem > 220 * 1024 || g.D > 256 || g.nyb > 256 || g.NY < 1) return LARE_ETOOLARGE;
  if (((uintptr_t)x & 15u) != 0) return LARE_EINVAL;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return LARE_ECUDA;
  // activations [nb][din][din][din][CIN] bf16 as a 5-D tensor, channels innermost
  CUtensorMap xmap;
  const cuuint64_t e = 2ull * CIN;
  const cuuint64_t dims[5] = {(cuuint64_t)CIN, (cuuint64_t)din, (cuuint64_t)din, (cuuint64_t)din, (cuuint64_t)nb};
  const cuuint64_t strides[4] = {e, e * din, e * din * din, e * din * din * din};
  const cuuint32_t box[5] = {8u, (cuuint32_t)g.D, (cuuint32_t)g.nyb, 1u, 1u};
  const cuuint32_t estr[5] = {1u, 1u, 1u, 1u, 1u};
  if (enc(&xmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(x), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return LARE_ECUDA;
  static int attr[64] = {};
  const int dev = current_device();
  if (dev < 0 || dev >= 64) return LARE_ECUDA;
  if (attr[dev] < (int)smem) {
    if (cudaFuncSetAttribute(k_conv_tc<CIN, NTC, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return LARE_ECUDA;
    attr[dev] = (int)smem;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long items = (long long)nb * g.E * g.ntg;
  const unsigned blocks = (unsigned)(items < sms ? items : sms);
  k_conv_tc<CIN, NTC, COUT><<<blocks, kTcEpiThreads, smem, s>>>(xmap, (const bf16*)w, bias, y, (const bf16*)mask, g,
                                                             relu, out_f32);
  return cudaGetLastError() == cudaSuccess ? LARE_OK : LARE_ECUDA;
}

// Single-output-channel convolution (the network's last layer).
template <int CIN>
int launch_conv_tc_c1(const void* x, int din, int pad, const void* w, const float* bias, float* y, int nb, int relu,
                      cudaStream_t s) {
  TcGeom g = tc_geom(din, pad, nb);
  const int nu = g.NY * g.D + 2 * g.D + 2, nut = (nu + 127) / 128;
  if (g.D > 76 || nut > (kTcT * 128 + 2 * 76 + 2 + 127) / 128 + 1) return LARE_ETOOLARGE;
  if (g.SS < nut * 128) g.SS = nut * 128;  // every MMA row stays inside the staged slabs
  const size_t smem = 128 + (size_t)3 * (CIN / 8) * 16 * 16 + (size_t)3 * (CIN / 8) * g.SS * 16 +
                      (size_t)nut * 128 * 16 * sizeof(float);
  if (smem > 220 * 1024 || g.nyb > 256 || g.NY < 1) return LARE_ETOOLARGE;
  if (((uintptr_t)x & 15u) != 0) return LARE_EINVAL;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return LARE_ECUDA;
  CUtensorMap xmap;
  const cuuint64_t e = 2ull * CIN;
  const cuuint64_t dims[5] = {(cuuint64_t)CIN, (cuuint64_t)din, (cuuint64_t)din, (cuuint64_t)din, (cuuint64_t)nb};
  const cuuint64_t strides[4] = {e, e * din, e * din * din, e * din * din * din};
  const cuuint32_t box[5] = {8u, (cuuint32_t)g.D, (cuuint32_t)g.nyb, 1u, 1u};
  const cuuint32_t estr[5] = {1u, 1u, 1u, 1u, 1u};
  if (enc(&xmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(x), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return LARE_ECUDA;
  static int attr[64] = {};
  const int dev = current_device();
  if (dev < 0 || dev >= 64) return LARE_ECUDA;
  if (attr[dev] < (int)smem) {
    if (cudaFuncSetAttribute(k_conv_tc_c1<CIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return LARE_ECUDA;
    attr[dev] = (int)smem;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long items = (long long)nb * g.E * g.ntg;
  const unsigned blocks = (unsigned)(items < sms ? items : sms);
  k_conv_tc_c1<CIN><<<blocks, kTcThreads, smem, s>>>(xmap, (const bf16*)w, bias, y, g, relu);
  return cudaGetLastError() == cudaSuccess ? LARE_OK : LARE_ECUDA;
}

// Single output channel on the CUDA cores (the alternative engine): one
// thread per output voxel, taps and channels in the forward conv's order.
template <int CIN>
__global__ void k_conv_c1(const bf16* __restrict__ x, int din, int pad, const bf16* __restrict__ w,
                          const float* __restrict__ bias, float* __restrict__ y, int dout, int nb, int relu) {
  const long long n = (long long)dout * dout * dout * nb;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long vox = (long long)dout * dout * dout;
  const int b = (int)(i / vox);
  const long long v = i - (long long)b * vox;
  const int ox = (int)(v % dout), oy = (int)((v / dout) % dout), oz = (int)(v / ((long long)dout * dout));
  float a = 0.f;
  for (int tap = 0; tap < 27; ++tap) {
    const int iz = oz + tap / 9 - pad, iy = oy + (tap / 3) % 3 - pad, ix = ox + tap % 3 - pad;
    if ((unsigned)iz >= (unsigned)din || (unsigned)iy >= (unsigned)din || (unsigned)ix >= (unsigned)din) continue;
    const bf16* xp = x + ((((long long)b * din + iz) * din + iy) * din + ix) * CIN;
    const bf16* wp = w + (long long)tap * CIN;
#pragma unroll
    for (int c = 0; c < CIN; ++c) a += __bfloat162float(xp[c]) * __bfloat162float(wp[c]);
  }
  a += bias ? bias[0] : 0.f;
  if (relu) a = fmaxf(a, 0.f);
  y[i] = a;
}

template <int CIN, int COUT>
int launch_conv(const void* x, int din, int pad, const void* w, const float* bias, void* y, int dout, int nb,
                const void* mask, int relu, int out_f32, cudaStream_t s) {
  if (g_use_tc) {
    (void)dout;
    return launch_conv_tc<CIN, (COUT < 16 ? 16 : COUT), COUT>(x, din, pad, w, bias, y, nb, mask, relu, out_f32, s);
  }
  constexpr size_t smem = conv_smem<CIN, COUT>();
  static bool attr[64] = {};
  const int dev = current_device();
  if (dev < 0 || dev >= 64) return LARE_ECUDA;
  if (!attr[dev]) {
    if (cudaFuncSetAttribute(k_conv<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return LARE_ECUDA;
    attr[dev] = true;
  }
  int sms = 148, per_sm = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_conv<CIN, COUT>, kConvThreads, smem);
  if (per_sm < 1) per_sm = 1;
  const long long M = (long long)dout * dout * dout * nb;
  const long long ntiles = (M + kTileRows - 1) / kTileRows;
  const long long cap = (long long)sms * per_sm;
  const unsigned blocks = (unsigned)(ntiles < cap ? ntiles : cap);
  k_conv<CIN, COUT><<<blocks, kConvThreads, smem, s>>>((const bf16*)x, din, pad, (const bf16*)w, bias, y, dout, nb,
                                                       (const bf16*)mask, relu, out_f32);
  return cudaGetLastError() == cudaSuccess ? LARE_OK : LARE_ECUDA;
}

// ---------------------------------------------------------------------
// Weight gradient: CTA (chunk, tap) accumulates dW[tap][co][ci] over its
// voxel chunk; the four warps are summed in a fixed order.
constexpr int kWChunk = 2048;  // voxels per CTA (multiple of 64)

template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_wgrad(const bf16* __restrict__ dy, const bf16* __restrict__ x, int din,
                                               int dout, long long nvox, float* __restrict__ partial) {
  __shared__ float red[4][COUT * CIN];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int tap = blockIdx.y;
  const int dz = tap / 9, dyy = (tap / 3) % 3, dx = tap % 3;
  const long long vox = (long long)dout * dout * dout;
  float acc[COUT / 16][CIN / 8][4];
#pragma unroll
  for (int i = 0; i < COUT / 16; ++i)
#pragma unroll
    for (int j = 0; j < CIN / 8; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;
  const long long base = (long long)blockIdx.x * kWChunk + warp * (kWChunk / 4);
  const bf16 zero = __float2bfloat16(0.f);
  for (int s = 0; s < kWChunk / 4; s += 16) {
    // the reduction (voxel) indices this thread supplies: 2t, 2t+1, 2t+8, 2t+9
    const bf16* dyp[4];
    const bf16* xp[4];
    bool ok[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const long long v = base + s + 2 * t + (q & 1) + (q >> 1) * 8;
      ok[q] = v < nvox;
      const long long vv = ok[q] ? v : 0;
      const long long b = vv / vox;
      const long long r = vv - b * vox;
      const int ox = (int)(r % dout), oy = (int)((r / dout) % dout), oz = (int)(r / ((long long)dout * dout));
      dyp[q] = dy + vv * COUT;
      xp[q] = x + (((b * din + oz + dz) * din + oy + dyy) * (long long)din + ox + dx) * CIN;
    }
#pragma unroll
    for (int mi = 0; mi < COUT / 16; ++mi) {
      const int c0 = mi * 16 + g, c1 = c0 + 8;
      uint32_t a[4];
      a[0] = pack2(ok[0] ? dyp[0][c0] : zero, ok[1] ? dyp[1][c0] : zero);
      a[1] = pack2(ok[0] ? dyp[0][c1] : zero, ok[1] ? dyp[1][c1] : zero);
      a[2] = pack2(ok[2] ? dyp[2][c0] : zero, ok[3] ? dyp[3][c0] : zero);
      a[3] = pack2(ok[2] ? dyp[2][c1] : zero, ok[3] ? dyp[3][c1] : zero);
#pragma unroll
      for (int nj = 0; nj < CIN / 8; ++nj) {
        const int ci = nj * 8 + g;
        uint32_t b[2];
        b[0] = pack2(ok[0] ? xp[0][ci] : zero, ok[1] ? xp[1][ci] : zero);
        b[1] = pack2(ok[2] ? xp[2][ci] : zero, ok[3] ? xp[3][ci] : zero);
        mma_16816(acc[mi][nj], a, b);
      }
    }
  }
#pragma unroll
  for (int mi = 0; mi < COUT / 16; ++mi)
#pragma unroll
    for (int nj = 0; nj < CIN / 8; ++nj)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int co = mi * 16 + g + (q >= 2 ? 8 : 0);
        const int ci = nj * 8 + 2 * t + (q & 1);
        red[warp][co * CIN + ci] = acc[mi][nj][q];
      }
  __syncthreads();
  float* out = partial + ((long long)blockIdx.x * 27 + tap) * (COUT * CIN);
  for (int i = threadIdx.x; i < COUT * CIN; i += blockDim.x)
    out[i] = ((red[0][i] + red[1][i]) + red[2][i]) + red[3][i];
}

// Sum chunk partials in order into dw[tap][co][ci].
__global__ void k_wgrad_reduce(const float* __restrict__ partial, int nchunks, int per, float* __restrict__ dw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= per) return;
  float s = 0.f;
  for (int c = 0; c < nchunks; ++c) s += partial[(long long)c * per + i];
  dw[i] = s;
}

// Bias gradient: one block per output channel, fixed-order tree.
__global__ void k_bgrad(const bf16* __restrict__ dy, long long nvox, int cout, float* __restrict__ db) {
  __shared__ float sh[256];
  const int co = blockIdx.x;
  float s = 0.f;
  for (long long v = threadIdx.x; v < nvox; v += blockDim.x) s += __bfloat162float(dy[v * cout + co]);
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[co] = sh[0];
}

template <int CIN, int COUT>
int launch_wgrad(const void* dy, const void* x, int din, int dout, int nb, float* work, float* dw, float* db,
                 cudaStream_t s) {
  const long long nvox = (long long)dout * dout * dout * nb;
  const int nchunks = (int)((nvox + kWChunk - 1) / kWChunk);
  dim3 grid(nchunks, 27);
  k_wgrad<CIN, COUT><<<grid, 128, 0, s>>>((const bf16*)dy, (const bf16*)x, din, dout, nvox, work);
  const int per = 27 * COUT * CIN;
  k_wgrad_reduce<<<(per + 255) / 256, 256, 0, s>>>(work, nchunks, per, dw);
  if (db) k_bgrad<<<COUT, 256, 0, s>>>((const bf16*)dy, nvox, COUT, db);
  return cudaGetLastError() == cudaSuccess ? LARE_OK : LARE_ECUDA;
}

// ---------------------------------------------------------------------
__global__ void k_mse(const float* __restrict__ pred, int pc, const float* __restrict__ tgt, long long n, int cpad,
                      float scale, bf16* __restrict__ dy, float* __restrict__ part) {
  __shared__ float sh[256];
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float d2 = 0.f;
  if (i < n) {
    const float d = pred[i * pc] - tgt[i];
    d2 = d * d;
    bf16* o = dy + i * cpad;
    o[0] = __float2bfloat16(scale * d);
    for (int c = 1; c < cpad; ++c) o[c] = __float2bfloat16(0.f);
  }
  sh[threadIdx.x] = d2;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_mse_finish(const float* __restrict__ part, int nparts, float inv_n, float* __restrict__ loss) {
  __shared__ float sh[256];
  float s = 0.f;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += part[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss[0] = sh[0] * inv_n;
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / c1, vh = vi / c2;
  p[i] -= lr * mh / (sqrtf(vh) + eps);
}

// wm [27][cout][cin] FP32 -> wf [27][cout_f][cin], wb [27][cin][cout] (taps flipped)
__global__ void k_pack(const float* __restrict__ wm, int cin, int cout, int cout_f, bf16* __restrict__ wf,
                       bf16* __restrict__ wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nf = 27 * cout_f * cin;
  if (i < nf) {
    const int ci = i % cin, co = (i / cin) % cout_f, tap = i / (cin * cout_f);
    wf[i] = __float2bfloat16(wm[(tap * cout + co) * cin + ci]);
  }
  const int nbk = 27 * cin * cout;
  if (wb && i < nbk) {
    const int co = i % cout, ci = (i / cout) % cin, tapb = i / (cout * cin);
    wb[i] = __float2bfloat16(wm[((26 - tapb) * cout + co) * cin + ci]);
  }
}

// ---------------------------------------------------------------------
// Engine-array glue.
template <class R>
struct Box {
  const R* p;
  int sx, sxy;
  __device__ __forceinline__ R operator()(int i, int j, int k) const { return p[i + sx * j + (long long)sxy * k]; }
};

template <class R>
__global__ void k_extract(Box<R> energy, Box<R> rho, Box<R> bx, Box<R> by, Box<R> bz, int nx, int ny, int nz,
                          double gamma, double xi_n, double ip, float s0, float s1, float* __restrict__ feat,
                          float* __restrict__ tout, int tmode) {
  const long long n = (long long)nx * ny * nz;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((long long)nx * ny));
  const int i = x + 1, j = y + 1, k = z + 1;
  const double e = (double)energy(i, j, k);
  const float T = (float)((gamma - 1.0) / (2.0 - xi_n) * (e - (1.0 - xi_n) * ip));
  const float bcx = 0.5f * ((float)bx(i - 1, j, k) + (float)bx(i, j, k));
  const float bcy = 0.5f * ((float)by(i, j - 1, k) + (float)by(i, j, k));
  const float bcz = 0.5f * ((float)bz(i, j, k - 1) + (float)bz(i, j, k));
  const float inv = rsqrtf(bcx * bcx + bcy * bcy + bcz * bcz + 1.0e-30f);
  if (feat) {
    feat[c] = T * s0;
    feat[n + c] = (float)rho(i, j, k) * s1;
    feat[2 * n + c] = bcx * inv;
    feat[3 * n + c] = bcy * inv;
    feat[4 * n + c] = bcz * inv;
  }
  if (tout) tout[c] = tmode ? T - tout[c] : T;
}

__global__ void k_gather(const float* __restrict__ store, int nx, int ny, int nz, const int* __restrict__ org, int nb,
                         int win, int halo, bf16* __restrict__ x, const float* __restrict__ tstore, float tscale,
                         float* __restrict__ tgt) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long w3 = (long long)win * win * win;
  if (i >= w3 * nb) return;
  const int b = (int)(i / w3);
  const long long r = i - (long long)b * w3;
  const int lx = (int)(r % win), ly = (int)((r / win) % win), lz = (int)(r / ((long long)win * win));
  const int s = org[4 * b];
  int gx = org[4 * b + 1] + lx, gy = org[4 * b + 2] + ly, gz = org[4 * b + 3] + lz;
  gx = ((gx % nx) + nx) % nx;
  gy = ((gy % ny) + ny) % ny;
  gz = gz < 0 ? 0 : (gz >= nz ? nz - 1 : gz);
  const long long nc = (long long)nx * ny * nz;
  const long long cell = ((long long)gz * ny + gy) * nx + gx;
  const float* f = store + (long long)s * 5 * nc;
  // T and rho as a bf16 pair each (value, 256 x remainder): bf16 alone
  // resolves only 2^-8 of T, too coarse for the cell-to-cell differences
  // that drive conduction.
  const float tv = f[cell], rv = f[nc + cell];
  const bf16 th = __float2bfloat16(tv), rh = __float2bfloat16(rv);
  const float tl = (tv - __bfloat162float(th)) * 256.f, rl = (rv - __bfloat162float(rh)) * 256.f;
  uint4 lo, hi;
  lo.x = pack2(th, rh);
  lo.y = pack2f(f[2 * nc + cell], f[3 * nc + cell]);
  lo.z = pack2f(f[4 * nc + cell], tl);
  lo.w = pack2f(rl, 0.f);
  hi.x = hi.y = hi.z = hi.w = 0u;
  uint4* dst = reinterpret_cast<uint4*>(x + i * 16);
  dst[0] = lo;
  dst[1] = hi;
  if (tstore && tgt && lx >= halo && lx < win - halo && ly >= halo && ly < win - halo && lz >= halo &&
      lz < win - halo) {
    const int pw = win - 2 * halo;
    const long long ti =
        (long long)b * pw * pw * pw + ((long long)(lz - halo) * pw + (ly - halo)) * pw + (lx - halo);
    tgt[ti] = tstore[(long long)s * nc + cell] * tscale;
  }
}

template <class R>
__global__ void k_apply(R* __restrict__ energy, int sx, int sxy, int nx, int ny, int nz,
                        const float* __restrict__ pred, int pc, const int* __restrict__ org, int nb, int pw, int halo,
                        double out_scale) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long p3 = (long long)pw * pw * pw;
  if (i >= p3 * nb) return;
  const int b = (int)(i / p3);
  const long long r = i - (long long)b * p3;
  const int lx = (int)(r % pw), ly = (int)((r / pw) % pw), lz = (int)(r / ((long long)pw * pw));
  int gx = org[4 * b + 1] + halo + lx, gy = org[4 * b + 2] + halo + ly;
  const int gz = org[4 * b + 3] + halo + lz;
  if (gz < 0 || gz >= nz) return;
  gx = ((gx % nx) + nx) % nx;
  gy = ((gy % ny) + ny) % ny;
  R* e = energy + (gx + 1) + (long long)sx * (gy + 1) + (long long)sxy * (gz + 1);
  *e = (R)((double)*e + out_scale * (double)pred[i * pc]);
}

struct Ptrs8 {
  const void* src[8];
  void* dst[8];
};

template <class R>
__global__ void k_copy_column(Ptrs8 P, int n, int sx, int sxy, int nx, int ny, int wsx, int wsxy, int wnx, int wny,
                              int nz, int x0, int y0) {
  const long long ex = wnx + 5, ey = wny + 5, ez = nz + 5;
  const long long tot = ex * ey * ez;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= tot) return;
  const int i = (int)(t % ex) - 2, j = (int)((t / ex) % ey) - 2, k = (int)(t / (ex * ey)) - 2;
  const int si = (((x0 + i - 1) % nx) + nx) % nx + 1;
  const int sj = (((y0 + j - 1) % ny) + ny) % ny + 1;
  const long long so = si + (long long)sx * sj + (long long)sxy * k;
  const long long dofs = i + (long long)wsx * j + (long long)wsxy * k;
  for (int a = 0; a < n; ++a) reinterpret_cast<R*>(P.dst[a])[dofs] = reinterpret_cast<const R*>(P.src[a])[so];
}

template <class R>
__global__ void k_recheck(R* __restrict__ energy, int sx, int sxy, int nx, int ny, const R* __restrict__ ew, int wsx,
                          int wsxy, int x0, int y0, int px0, int py0, int pz0, int npx, int npy, int patch,
                          double gamma, double xi_n, double ip, double bound, float* __restrict__ err,
                          int* __restrict__ n_rejected) {
  __shared__ float sh[256];
  __shared__ int reject;
  const int p = blockIdx.x;
  const int a = p % npx, b = (p / npx) % npy, c = p / (npx * npy);
  const int p3 = patch * patch * patch;
  const double cT = (gamma - 1.0) / (2.0 - xi_n), e0 = (1.0 - xi_n) * ip;
  float m = 0.f;
  for (int l = threadIdx.x; l < p3; l += blockDim.x) {
    const int lx = l % patch, ly = (l / patch) % patch, lz = l / (patch * patch);
    const int ux = px0 + a * patch + lx, uy = py0 + b * patch + ly, gz = pz0 + c * patch + lz;
    const int gx = ux % nx, gy = uy % ny;
    const int wi = ux - x0 + 1, wj = uy - y0 + 1;
    const double t = cT * ((double)energy[(gx + 1) + (long long)sx * (gy + 1) + (long long)sxy * (gz + 1)] - e0);
    const double tw = cT * ((double)ew[wi + (long long)wsx * wj + (long long)wsxy * (gz + 1)] - e0);
    const float rel = (float)(fabs(t - tw) / fmax(fabs(tw), 1e-300));
    m = fmaxf(m, rel);
  }
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = fmaxf(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    err[p] = sh[0];
    reject = !(sh[0] <= (float)bound);
    if (reject) atomicAdd(n_rejected, 1);
  }
  __syncthreads();
  if (!reject) return;
  for (int l = threadIdx.x; l < p3; l += blockDim.x) {
    const int lx = l % patch, ly = (l / patch) % patch, lz = l / (patch * patch);
    const int ux = px0 + a * patch + lx, uy = py0 + b * patch + ly, gz = pz0 + c * patch + lz;
    const int gx = ux % nx, gy = uy % ny;
    const int wi = ux - x0 + 1, wj = uy - y0 + 1;
    energy[(gx + 1) + (long long)sx * (gy + 1) + (long long)sxy * (gz + 1)] =
        ew[wi + (long long)wsx * wj + (long long)wsxy * (gz + 1)];
  }
}

int done() { return cudaGetLastError() == cudaSuccess ? LARE_OK : LARE_ECUDA; }

}  // namespace

extern "C" {

int lare_sur_conv(int cin, int cout, int relu, int out_f32, const void* x, int din, int pad, const void* w,
                  const float* bias, void* y, int dout, int nb, const void* mask, void* stream) {
  if (!x || !w || !y || din < 1 || dout < 1 || nb < 1 || (pad != 0 && pad != 2)) return LARE_EINVAL;
  if (din - 2 + 2 * pad != dout) return LARE_EINVAL;
  if (out_f32 && mask) return LARE_EINVAL;
  if ((long long)dout * dout * dout * nb * (cout > cin ? cout : cin) >= (1LL << 40)) return LARE_ETOOLARGE;
  cudaStream_t s = (cudaStream_t)stream;
  if (cin == 16 && cout == 32) return launch_conv<16, 32>(x, din, pad, w, bias, y, dout, nb, mask, relu, out_f32, s);
  if (cin == 32 && cout == 32) return launch_conv<32, 32>(x, din, pad, w, bias, y, dout, nb, mask, relu, out_f32, s);
  if (cin == 32 && cout == 8) return launch_conv<32, 8>(x, din, pad, w, bias, y, dout, nb, mask, relu, out_f32, s);
  if (cin == 32 && cout == 1) {
    if (!out_f32 || mask) return LARE_EINVAL;
    if (g_use_tc) return launch_conv_tc_c1<32>(x, din, pad, w, bias, (float*)y, nb, relu, s);
    const long long n = (long long)dout * dout * dout * nb;
    k_conv_c1<32><<<(unsigned)((n + 255) / 256), 256, 0, s>>>((const bf16*)x, din, pad, (const bf16*)w, bias,
                                                             (float*)y, dout, nb, relu);
    return cudaGetLastError() == cudaSuccess ? LARE_OK : LARE_ECUDA;
  }
  return LARE_EINVAL;
}

int lare_sur_set_engine(int tensor_cores) {
  g_use_tc = tensor_cores != 0;
  return LARE_OK;
}

int lare_sur_status(int clear) {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_sur_status, sizeof(int)) != cudaSuccess) return LARE_ECUDA;
  if (clear) {
    const int z = 0;
    if (cudaMemcpyToSymbol(g_sur_status, &z, sizeof(int)) != cudaSuccess) return LARE_ECUDA;
  }
  return v;
}

long long lare_sur_conv_wgrad_work(int cin, int cout, int dout, int nb) {
  if (cin < 1 || cout < 1 || dout < 1 || nb < 1) return -1;
  const long long nvox = (long long)dout * dout * dout * nb;
  const long long nchunks = (nvox + kWChunk - 1) / kWChunk;
  return nchunks * 27 * cin * cout;
}

int lare_sur_conv_wgrad(int cin, int cout, const void* dy, const void* x, int din, int dout, int nb, float* work,
                        float* dw, float* db, void* stream) {
  if (!dy || !x || !work || !dw || dout < 1 || din != dout + 2 || nb < 1) return LARE_EINVAL;
  if ((long long)dout * dout * dout * nb >= (1LL << 31) * (long long)kWChunk) return LARE_ETOOLARGE;
  cudaStream_t s = (cudaStream_t)stream;
  if (cin == 16 && cout == 32) return launch_wgrad<16, 32>(dy, x, din, dout, nb, work, dw, db, s);
  if (cin == 32 && cout == 32) return launch_wgrad<32, 32>(dy, x, din, dout, nb, work, dw, db, s);
  if (cin == 32 && cout == 16) return launch_wgrad<32, 16>(dy, x, din, dout, nb, work, dw, db, s);
  return LARE_EINVAL;
}

int lare_sur_mse(const float* pred, int pc, const float* target, long long count, int cpad, float* loss, void* dy,
                 float* work, void* stream) {
  if (!pred || !target || !loss || !dy || !work || pc < 1 || count < 1 || cpad < 1) return LARE_EINVAL;
  const long long blocks = (count + 255) / 256;
  if (blocks >= (1LL << 31)) return LARE_ETOOLARGE;
  cudaStream_t s = (cudaStream_t)stream;
  k_mse<<<(unsigned)blocks, 256, 0, s>>>(pred, pc, target, count, cpad, (float)(2.0 / (double)count), (bf16*)dy,
                                         work);
  k_mse_finish<<<1, 256, 0, s>>>(work, (int)blocks, (float)(1.0 / (double)count), loss);
  return done();
}

int lare_sur_adam(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps, int t,
                  void* stream) {
  if (!p || !g || !m || !v || n < 1 || t < 1) return LARE_EINVAL;
  const float c1 = (float)(1.0 - std::pow((double)b1, (double)t));
  const float c2 = (float)(1.0 - std::pow((double)b2, (double)t));
  k_adam<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2);
  return done();
}

int lare_sur_pack(const float* wm, int cin, int cout, int cout_f, void* wf, void* wb, void* stream) {
  if (!wm || !wf || cin < 1 || cout < 1 || cout_f < 1 || cout_f > cout) return LARE_EINVAL;
  const int n = 27 * cout * cin;
  k_pack<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(wm, cin, cout, cout_f, (bf16*)wf, (bf16*)wb);
  return done();
}

int lare_sur_extract(int elem_bytes, const void* energy, const void* rho, const void* bx, const void* by,
                     const void* bz, int sx, int sxy, int nx, int ny, int nz, double gamma, double xi_n,
                     double ionise_pot, float t_scale, float rho_scale, float* feat, float* tout, int tmode,
                     void* stream) {
  if (!energy || !rho || !bx || !by || !bz || (!feat && !tout) || nx < 1 || ny < 1 || nz < 1)
    return LARE_EINVAL;
  if (sx < nx + 5 || sxy < sx * (ny + 5) || (elem_bytes != 4 && elem_bytes != 8)) return LARE_EINVAL;
  const long long n = (long long)nx * ny * nz;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  cudaStream_t s = (cudaStream_t)stream;
  if (elem_bytes == 8) {
    typedef double R;
    k_extract<R><<<blocks, 256, 0, s>>>(Box<R>{(const R*)energy, sx, sxy}, Box<R>{(const R*)rho, sx, sxy},
                                        Box<R>{(const R*)bx, sx, sxy}, Box<R>{(const R*)by, sx, sxy},
                                        Box<R>{(const R*)bz, sx, sxy}, nx, ny, nz, gamma, xi_n, ionise_pot, t_scale,
                                        rho_scale, feat, tout, tmode);
  } else {
    typedef float R;
    k_extract<R><<<blocks, 256, 0, s>>>(Box<R>{(const R*)energy, sx, sxy}, Box<R>{(const R*)rho, sx, sxy},
                                        Box<R>{(const R*)bx, sx, sxy}, Box<R>{(const R*)by, sx, sxy},
                                        Box<R>{(const R*)bz, sx, sxy}, nx, ny, nz, gamma, xi_n, ionise_pot, t_scale,
                                        rho_scale, feat, tout, tmode);
  }
  return done();
}

int lare_sur_gather(const float* store, int nx, int ny, int nz, const int* org, int nb, int win, int halo, void* x,
                    const float* tstore, float tscale, float* tgt, void* stream) {
  if (!store || !org || !x || nx < 1 || ny < 1 || nz < 1 || nb < 1 || win < 1 || halo < 0 || 2 * halo >= win)
    return LARE_EINVAL;
  const long long tot = (long long)win * win * win * nb;
  k_gather<<<(unsigned)((tot + 255) / 256), 256, 0, (cudaStream_t)stream>>>(store, nx, ny, nz, org, nb, win, halo,
                                                                           (bf16*)x, tstore, tscale, tgt);
  return done();
}

int lare_sur_apply(int elem_bytes, void* energy, int sx, int sxy, int nx, int ny, int nz, const float* pred, int pc,
                   const int* org, int nb, int pw, int halo, double out_scale, void* stream) {
  if (!energy || !pred || !org || pc < 1 || nb < 1 || pw < 1 || halo < 0 || nx < 1 || ny < 1 || nz < 1)
    return LARE_EINVAL;
  if (elem_bytes != 4 && elem_bytes != 8) return LARE_EINVAL;
  const long long tot = (long long)pw * pw * pw * nb;
  const unsigned blocks = (unsigned)((tot + 255) / 256);
  cudaStream_t s = (cudaStream_t)stream;
  if (elem_bytes == 8)
    k_apply<double><<<blocks, 256, 0, s>>>((double*)energy, sx, sxy, nx, ny, nz, pred, pc, org, nb, pw, halo,
                                           out_scale);
  else
    k_apply<float><<<blocks, 256, 0, s>>>((float*)energy, sx, sxy, nx, ny, nz, pred, pc, org, nb, pw, halo,
                                          out_scale);
  return done();
}

int lare_sur_copy_column(int elem_bytes, const void* const* src, int sx, int sxy, int nx, int ny, void* const* dst,
                         int wsx, int wsxy, int wnx, int wny, int nz, int x0, int y0, int n, void* stream) {
  if (!src || !dst || n < 1 || n > 8 || nx < 1 || ny < 1 || nz < 1 || wnx < 1 || wny < 1) return LARE_EINVAL;
  if (wsx < wnx + 5 || wsxy < wsx * (wny + 5) || (elem_bytes != 4 && elem_bytes != 8)) return LARE_EINVAL;
  Ptrs8 P = {};
  for (int a = 0; a < n; ++a) {
    if (!src[a] || !dst[a]) return LARE_EINVAL;
    P.src[a] = src[a];
    P.dst[a] = dst[a];
  }
  const long long tot = (long long)(wnx + 5) * (wny + 5) * (nz + 5);
  const unsigned blocks = (unsigned)((tot + 255) / 256);
  cudaStream_t s = (cudaStream_t)stream;
  if (elem_bytes == 8)
    k_copy_column<double><<<blocks, 256, 0, s>>>(P, n, sx, sxy, nx, ny, wsx, wsxy, wnx, wny, nz, x0, y0);
  else
    k_copy_column<float><<<blocks, 256, 0, s>>>(P, n, sx, sxy, nx, ny, wsx, wsxy, wnx, wny, nz, x0, y0);
  return done();
}

int lare_sur_recheck(int elem_bytes, void* energy, int sx, int sxy, int nx, int ny, const void* energy_w, int wsx,
                     int wsxy, int wnx, int wny, int x0, int y0, int px0, int py0, int pz0, int npx, int npy, int npz,
                     int patch, double gamma, double xi_n, double ionise_pot, double bound, float* err,
                     int* n_rejected, void* stream) {
  if (!energy || !energy_w || !err || !n_rejected || npx < 1 || npy < 1 || npz < 1 || patch < 1) return LARE_EINVAL;
  if (px0 < 0 || py0 < 0 || pz0 < 0 || px0 < x0 || py0 < y0 || px0 - x0 + npx * patch > wnx ||
      py0 - y0 + npy * patch > wny || wsx < wnx + 5 || wsxy < wsx * (wny + 5))
    return LARE_EINVAL;
  if (elem_bytes != 4 && elem_bytes != 8) return LARE_EINVAL;
  const int np = npx * npy * npz;
  cudaStream_t s = (cudaStream_t)stream;
  if (elem_bytes == 8)
    k_recheck<double><<<np, 256, 0, s>>>((double*)energy, sx, sxy, nx, ny, (const double*)energy_w, wsx, wsxy, x0,
                                         y0, px0, py0, pz0, npx, npy, patch, gamma, xi_n, ionise_pot, bound, err,
                                         n_rejected);
  else
    k_recheck<float><<<np, 256, 0, s>>>((float*)energy, sx, sxy, nx, ny, (const float*)energy_w, wsx, wsxy, x0, y0,
                                        px0, py0, pz0, npx, npy, patch, gamma, xi_n, ionise_pot, bound, err,
                                        n_rejected);
  return done();
}

}  // extern "C"
