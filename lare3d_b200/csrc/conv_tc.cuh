// conv_tc.cuh - the surrogate's 3-D convolution on the 5th-generation
// tensor cores (tcgen05.mma, accumulators in tensor memory).
//
// Implicit GEMM with shifted operands.  For an output z-plane oz, output
// voxels are numbered r = oy*D + ox with the INPUT row length D (columns
// ox >= E = D - 2 are computed and dropped), so that for tap (dz, dy, dx)
// the input voxel of row r is row r + dy*D + dx of input plane oz + dz: one
// constant shift per tap.  A work item is NY whole output rows of one plane;
// the tensor memory accelerator (cp.async.bulk.tensor, one 5-D box per input
// plane and channel group, zero fill outside the input, which also provides
// the padding of the backward-data convolution) stages the three input
// planes' rows in shared memory as [plane][channel group of 8][row][8 bf16]
// -- the no-swizzle K-major operand layout, in which 8 consecutive rows of
// 16 bytes form one core matrix -- so the A operand of every tap is the same
// buffer with a different start address.  The weights stay resident as
// [tap][channel group][cout][8].  One elected thread issues
// T x 27 x (CIN/16) MMAs of 128 x N x 16 (N = output channels) into T
// accumulator tiles in tensor memory, commits them to an mbarrier, and
// eight warps (two per 32-lane quadrant of tensor memory, each for half of
// the output channels) read the accumulators back (tcgen05.ld), add the
// bias (held in registers), apply the
// ReLU or the mask and store bf16 or FP32.  Padding (pad = 2, the
// backward-data convolution) comes from the zero fill of the staging.
//
// Every wait is bounded; a wait that runs out records kErrWait in the
// device status word and the CTA frees its tensor memory and returns.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace {

constexpr int kTcT = 4;           // accumulator tiles (128 rows each) per work item
constexpr int kTcThreads = 128;   // k_conv_tc_c1
constexpr int kTcEpiThreads = 256; // k_conv_tc: two warps per tensor-memory lane quadrant in the epilogue
constexpr int kErrWait = 1;

__device__ int g_sur_status = 0;  // sticky error word of the tensor-core kernels

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 16-byte asynchronous global -> shared copy; src_bytes = 0 writes zeros.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Shared-memory matrix descriptor, K-major, no swizzle: start, leading
// (K-direction core-matrix) byte offset, stride (M/N-direction core-matrix)
// byte offset, descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::f16: FP32 accumulate, bf16 A and B, both
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t umma_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

template <int N>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float (&v)[N]);

template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <>
__device__ __forceinline__ void tmem_ld<8>(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

template <>
__device__ __forceinline__ void tmem_ld<32>(uint32_t taddr, float (&v)[32]) {
  float a[16], b[16];
  tmem_ld<16>(taddr, a);
  tmem_ld<16>(taddr + 16, b);
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    v[i] = a[i];
    v[16 + i] = b[i];
  }
}

struct TcGeom {
  int D;      // virtual (padded) input edge
  int E;      // output edge = D - 2
  int din;    // real input edge
  int pad;    // 0 or 2
  int nb;
  int NY;     // output rows per work item (NY * D <= 128 * kTcT)
  int nyb;    // input rows staged per plane (covers every MMA row's taps)
  int RS;     // staged voxels per plane and channel group = nyb * D
  int SS;     // slab stride in voxels: RS rounded up to 8 (128-byte TMA destinations)
  int ntg;    // work items per output plane
};

__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            int c4, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
      "[%7];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(mbar)
      : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// CIN input channels, NTC = MMA N (output channels computed), COUT = output
// channels stored.
template <int CIN, int NTC, int COUT>
__global__ void __launch_bounds__(kTcEpiThreads, 1)
    k_conv_tc(const __grid_constant__ CUtensorMap xmap, const __nv_bfloat16* __restrict__ w,
              const float* __restrict__ bias, void* __restrict__ y, const __nv_bfloat16* __restrict__ mask,
              TcGeom g, int relu, int out_f32) {
  constexpr int KG = CIN / 8;
  constexpr int WBYTES = 27 * KG * NTC * 16;
  constexpr int TCOLS = kTcT * NTC <= 32 ? 32 : (kTcT * NTC <= 64 ? 64 : 128);
  extern __shared__ __align__(128) unsigned char sm_raw[];
  // 128-byte aligned base: TMA destinations must be 128-byte aligned
  unsigned char* sm = sm_raw + ((128u - (smem_u32(sm_raw) & 127u)) & 127u);
  unsigned char* sw = sm;                        // weights
  unsigned char* sx = sm + WBYTES;               // staged input
  __shared__ __align__(8) uint64_t mbar;   // MMA completion
  __shared__ __align__(8) uint64_t tbar;   // staging (TMA) completion
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int SS = g.SS, D = g.D;
  constexpr int HALF = NTC / 2;                 // output channels per epilogue warp
  const int quad = warp & 3;                    // tensor-memory lane quadrant of this warp
  const int HC0 = (warp >> 2) * HALF;           // its first output channel
  float bv[HALF];
#pragma unroll
  for (int c = 0; c < HALF; ++c) bv[c] = (bias && HC0 + c < COUT) ? bias[HC0 + c] : 0.f;

  // weights: global [27][COUT][CIN] -> shared [27][KG][NTC][8] (rows >= COUT zero)
  for (int q = tid; q < 27 * KG * NTC; q += kTcEpiThreads) {
    const int co = q % NTC, kg = (q / NTC) % KG, tap = q / (NTC * KG);
    const __nv_bfloat16* src = w + ((long long)tap * COUT + (co < COUT ? co : 0)) * CIN + kg * 8;
    cp_async16(smem_u32(sw + (size_t)q * 16), src, co < COUT ? 16u : 0u);
  }
  cp_async_wait_all();
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&tbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tbase = tmem_slot;
  const uint32_t mb = smem_u32(&mbar);
  const uint32_t sw_a = smem_u32(sw), sx_a = smem_u32(sx);
  const uint32_t tb = smem_u32(&tbar);
  const uint32_t idesc = umma_idesc(NTC);
  uint32_t phase = 0, tphase = 0;
  bool failed = false;
  auto wait_bar = [&](uint32_t bar, uint32_t& ph) -> bool {
    long long spins = 0;
    bool timed_out = false;
    while (!mbar_try(bar, ph)) {
      if (++spins > (1LL << 22)) {
        timed_out = true;
        break;
      }
      __nanosleep(32);  // leave the issue slots to the thread that issues the MMAs
    }
    ph ^= 1u;
    return __syncthreads_or(timed_out) != 0;
  };

  const long long items = (long long)g.nb * g.E * g.ntg;
  // stage item `it` (three input planes, every channel group) with the TMA
  auto stage = [&](long long it) {
    const int tg = (int)(it % g.ntg);
    const int oz = (int)((it / g.ntg) % g.E);
    const int b = (int)(it / ((long long)g.ntg * g.E));
    const int y0 = tg * g.NY;
    mbar_expect_tx(tb, (uint32_t)(3 * KG * g.RS * 16));
    for (int p = 0; p < 3; ++p)
      for (int kg = 0; kg < KG; ++kg)
        tma_load_5d(sx_a + (uint32_t)((p * KG + kg) * SS * 16), &xmap, kg * 8, -g.pad, y0 - g.pad, oz + p - g.pad, b,
                    tb);
  };
  // descriptors advance by the operand offset in 16-byte units (the start
  // address field holds address >> 4 and shared memory is < 256 KB)
  const uint64_t ad0 = umma_desc(sx_a, (uint32_t)SS * 16u, 128u);
  const uint64_t bd0 = umma_desc(sw_a, (uint32_t)NTC * 16u, 128u);
  if (tid == 0 && (long long)blockIdx.x < items) stage(blockIdx.x);
  for (long long it = blockIdx.x; it < items && !failed; it += gridDim.x) {
    const int tg = (int)(it % g.ntg);
    const int oz = (int)((it / g.ntg) % g.E);
    const int b = (int)(it / ((long long)g.ntg * g.E));
    const int y0 = tg * g.NY;
    const int r0 = y0 * D;
    if ((failed = wait_bar(tb, tphase))) break;  // this item's planes have landed
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      // the kTcT accumulator tiles are independent: interleave them so that
      // consecutive MMAs do not wait on the same accumulator
      for (int tap = 0; tap < 27; ++tap) {
        const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
#pragma unroll
        for (int kc = 0; kc < KG / 2; ++kc) {
          const uint64_t bd = bd0 + (uint64_t)((tap * KG + 2 * kc) * NTC);
          const uint32_t acc = (tap > 0 || kc > 0) ? 1u : 0u;
          const uint64_t adk = ad0 + (uint64_t)((dz * KG + 2 * kc) * SS + dy * D + dx);
#pragma unroll
          for (int t = 0; t < kTcT; ++t) umma_f16(tbase + (uint32_t)(t * NTC), adk + (uint64_t)(t * 128), bd, idesc, acc);
        }
      }
      umma_commit(mb);
    }
    // wait for the accumulators (bounded; uniform over the CTA)
    if ((failed = wait_bar(mb, phase))) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // the staged planes are free again: fetch the next item while this
    // item's accumulators drain
    const long long nxt = it + gridDim.x;
    if (tid == 0 && nxt < items) stage(nxt);
    // epilogue: warps w and w+4 own accumulator rows 32(w%4)..32(w%4)+31 of
    // every tile, each for half of the output channels
#pragma unroll 1
    for (int t = 0; t < kTcT; ++t) {
      if (HC0 >= COUT) break;
      float v[HALF];
      tmem_ld<HALF>(tbase + ((uint32_t)(32 * quad) << 16) + (uint32_t)(t * NTC + HC0), v);
      const int r = r0 + t * 128 + 32 * quad + lane;
      const int oy = r / D, ox = r - (r / D) * D;
      if (oy < g.E && oy < y0 + g.NY && ox < g.E) {
        const long long o = (((long long)b * g.E + oz) * g.E + oy) * g.E + ox;
        if (out_f32) {
          float* yo = reinterpret_cast<float*>(y) + o * COUT + HC0;
#pragma unroll
          for (int c = 0; c < HALF; ++c) {
            if (HC0 + c >= COUT) break;
            float a = v[c] + bv[c];
            if (relu) a = fmaxf(a, 0.f);
            yo[c] = a;
          }
        } else {
          __nv_bfloat16* yo = reinterpret_cast<__nv_bfloat16*>(y) + o * COUT + HC0;
#pragma unroll
          for (int c = 0; c < HALF; c += 8) {
            if (HC0 + c >= COUT) break;
            float a[8];
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
              a[jj] = v[c + jj] + bv[c + jj];
              if (relu) a[jj] = fmaxf(a[jj], 0.f);
            }
            if (mask) {
              const uint4 mk = *reinterpret_cast<const uint4*>(mask + o * COUT + HC0 + c);
              const uint32_t mw[4] = {mk.x, mk.y, mk.z, mk.w};
#pragma unroll
              for (int jj = 0; jj < 8; ++jj) {
                const unsigned short h = (unsigned short)((mw[jj >> 1] >> (16 * (jj & 1))) & 0xffffu);
                if (!(__bfloat162float(__ushort_as_bfloat16(h)) > 0.f)) a[jj] = 0.f;
              }
            }
            uint4 o4;
            o4.x = pack2f(a[0], a[1]);
            o4.y = pack2f(a[2], a[3]);
            o4.z = pack2f(a[4], a[5]);
            o4.w = pack2f(a[6], a[7]);
            *reinterpret_cast<uint4*>(yo + c) = o4;
          }
        }
      }
    }
    // every warp has read the accumulators before the next item's MMAs
    // overwrite them
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (failed && tid == 0) atomicOr(&g_sur_status, kErrWait);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TCOLS) : "memory");
  }
}

// Single output channel (the network's last layer, dT): the nine (dy, dx)
// taps of a plane share one shift-free operand, so the MMA's N dimension
// holds the taps instead of output channels:
//   P[u][j] = sum_{dz, ci} X[plane oz+dz][row u][ci] W[dz*9 + j][ci]   (j = dy*3 + dx)
// accumulated over the three planes and both channel halves in tensor
// memory (N = 16, taps 9..15 zero), and out[v] = bias + sum_j P[v + dy*D + dx][j]
// is formed in the epilogue from a shared-memory copy of P.  36 MMAs per
// work item instead of 216.
template <int CIN>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_conv_tc_c1(const __grid_constant__ CUtensorMap xmap, const __nv_bfloat16* __restrict__ w,
                 const float* __restrict__ bias, float* __restrict__ y, TcGeom g, int relu) {
  constexpr int KG = CIN / 8;
  constexpr int NJ = 16;                         // taps per plane (9) padded to the MMA's N
  constexpr int WBYTES = 3 * KG * NJ * 16;       // weights [plane][kg][j][8]
  constexpr int NUT = (kTcT * 128 + 2 * 76 + 2 + 127) / 128 + 1;  // u tiles (bounded by D <= 76)
  constexpr int TCOLS = NUT * NJ <= 32 ? 32 : (NUT * NJ <= 64 ? 64 : 128);
  extern __shared__ __align__(128) unsigned char sm_raw[];
  unsigned char* sm = sm_raw + ((128u - (smem_u32(sm_raw) & 127u)) & 127u);
  unsigned char* sw = sm;
  unsigned char* sx = sm + WBYTES;
  __shared__ __align__(8) uint64_t mbar;
  __shared__ __align__(8) uint64_t tbar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int SS = g.SS, D = g.D;
  float* Psm = reinterpret_cast<float*>(sx + (size_t)3 * KG * SS * 16);  // [u][NJ]
  // weights: global [27][1][CIN] -> shared [3][KG][NJ][8], j >= 9 zero
  for (int q = tid; q < 3 * KG * NJ; q += kTcThreads) {
    const int j = q % NJ, kg = (q / NJ) % KG, p = q / (NJ * KG);
    const __nv_bfloat16* src = w + ((long long)(p * 9 + (j < 9 ? j : 0))) * CIN + kg * 8;
    cp_async16(smem_u32(sw + (size_t)q * 16), src, j < 9 ? 16u : 0u);
  }
  cp_async_wait_all();
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&tbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tbase = tmem_slot;
  const uint32_t mb = smem_u32(&mbar), tb = smem_u32(&tbar);
  const uint32_t sw_a = smem_u32(sw), sx_a = smem_u32(sx);
  const uint32_t idesc = umma_idesc(NJ);
  uint32_t phase = 0, tphase = 0;
  bool failed = false;
  auto wait_bar = [&](uint32_t bar, uint32_t& ph) -> bool {
    long long spins = 0;
    bool timed_out = false;
    while (!mbar_try(bar, ph)) {
      if (++spins > (1LL << 22)) {
        timed_out = true;
        break;
      }
    }
    ph ^= 1u;
    return __syncthreads_or(timed_out) != 0;
  };
  const int nrow = g.NY * D;                       // output rows of an item (padded numbering)
  const int nu = nrow + 2 * D + 2;                 // P rows an item needs
  const int nut = (nu + 127) / 128;
  const long long items = (long long)g.nb * g.E * g.ntg;
  auto stage = [&](long long it) {
    const int tg = (int)(it % g.ntg);
    const int oz = (int)((it / g.ntg) % g.E);
    const int b = (int)(it / ((long long)g.ntg * g.E));
    mbar_expect_tx(tb, (uint32_t)(3 * KG * g.RS * 16));
    for (int p = 0; p < 3; ++p)
      for (int kg = 0; kg < KG; ++kg)
        tma_load_5d(sx_a + (uint32_t)((p * KG + kg) * SS * 16), &xmap, kg * 8, -g.pad, tg * g.NY - g.pad,
                    oz + p - g.pad, b, tb);
  };
  const uint64_t ad0 = umma_desc(sx_a, (uint32_t)SS * 16u, 128u);
  const uint64_t bd0 = umma_desc(sw_a, (uint32_t)NJ * 16u, 128u);
  const float b0 = bias ? bias[0] : 0.f;
  if (tid == 0 && (long long)blockIdx.x < items) stage(blockIdx.x);
  for (long long it = blockIdx.x; it < items && !failed; it += gridDim.x) {
    const int tg = (int)(it % g.ntg);
    const int oz = (int)((it / g.ntg) % g.E);
    const int b = (int)(it / ((long long)g.ntg * g.E));
    const int y0 = tg * g.NY;
    if ((failed = wait_bar(tb, tphase))) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      for (int p = 0; p < 3; ++p) {
#pragma unroll
        for (int kc = 0; kc < KG / 2; ++kc) {
          const uint64_t bd = bd0 + (uint64_t)((p * KG + 2 * kc) * NJ);
          const uint64_t adk = ad0 + (uint64_t)((p * KG + 2 * kc) * SS);
          const uint32_t acc = (p > 0 || kc > 0) ? 1u : 0u;
          for (int ut = 0; ut < nut; ++ut)
            umma_f16(tbase + (uint32_t)(ut * NJ), adk + (uint64_t)(ut * 128), bd, idesc, acc);
        }
      }
      umma_commit(mb);
    }
    if ((failed = wait_bar(mb, phase))) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const long long nxt = it + gridDim.x;
    if (tid == 0 && nxt < items) stage(nxt);
    // P to shared memory: warp w writes rows ut*128 + 32w + lane
    for (int ut = 0; ut < nut; ++ut) {
      float v[NJ];
      tmem_ld<NJ>(tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)(ut * NJ), v);
      const int u = ut * 128 + 32 * warp + lane;
      float4* dst = reinterpret_cast<float4*>(Psm + (size_t)u * NJ);
#pragma unroll
      for (int q = 0; q < NJ / 4; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    for (int r = tid; r < nrow; r += kTcThreads) {
      const int oy = y0 + r / D, ox = r - (r / D) * D;
      if (oy >= g.E || ox >= g.E) continue;
      float a = 0.f;
#pragma unroll
      for (int j = 0; j < 9; ++j) a += Psm[(size_t)(r + (j / 3) * D + (j % 3)) * NJ + j];
      a += b0;
      if (relu) a = fmaxf(a, 0.f);
      y[(((long long)b * g.E + oz) * g.E + oy) * g.E + ox] = a;
    }
    __syncthreads();
  }
  if (failed && tid == 0) atomicOr(&g_sur_status, kErrWait);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TCOLS) : "memory");
  }
}

// Geometry of one convolution call (see the file comment).
inline TcGeom tc_geom(int din, int pad, int nb) {
  TcGeom g;
  g.din = din;
  g.pad = pad;
  g.D = din + 2 * pad;
  g.E = g.D - 2;
  g.nb = nb;
  g.NY = (kTcT * 128) / g.D;
  if (g.NY > g.E) g.NY = g.E;
  // the last MMA row of the last tile reads row index kTcT*128 - 1 + 2D + 2
  g.nyb = (kTcT * 128 + 2 * g.D + 2 + g.D - 1) / g.D;
  g.RS = g.nyb * g.D;
  g.SS = (g.RS + 7) / 8 * 8;
  g.ntg = (g.E + g.NY - 1) / g.NY;
  return g;
}

template <int CIN, int NTC>
constexpr size_t tc_smem_bytes(int ss) {
  // 128 bytes of alignment slack + weights + 3 planes x channel groups of slabs
  return 128 + (size_t)27 * (CIN / 8) * NTC * 16 + (size_t)3 * (CIN / 8) * ss * 16;
}

}  // namespace
