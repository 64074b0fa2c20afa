// common.cuh - device layout, launch helpers and deterministic reductions.
//
// Layout: every 3-D array lives in one common padded box covering Fortran
// indices -2..n+2 in each dimension (the union of the cell, node and face
// bounds of mpi_routines.F90:295-327), x fastest, row pitch sx >= nx+5
// rounded up to 4 elements.  One index formula then serves every
// staggering, and element (i,j,k) of any array is  p0[i + sx*j + sxy*k]
// with p0 pointing at Fortran (0,0,0).
#pragma once

#include <cuda_runtime.h>

#include <cfloat>
#include <climits>
#include <cstdint>

#include "variant.h"

LARE_BEGIN

template <class R>
struct A3 {
  R* p;  // element (0,0,0)
  int sx, sxy;
  __device__ __forceinline__ R& operator()(int i, int j, int k) const { return p[i + sx * j + sxy * k]; }
};

template <class R>
struct A1 {
  const R* p;  // element 0 (Fortran lower bound may be -1 or -2)
  __device__ __forceinline__ R operator()(int i) const { return p[i]; }
};

template <class R>
struct Num;
template <>
struct Num<double> {
  static __host__ __device__ constexpr double tiny() { return DBL_MIN; }  // TINY(1.0_num)
  static __host__ __device__ constexpr double huge() { return DBL_MAX; }  // HUGE(1.0_num)
};
template <>
struct Num<float> {
  static __host__ __device__ constexpr float tiny() { return FLT_MIN; }
  static __host__ __device__ constexpr float huge() { return FLT_MAX; }
};

// a / b given rb = RN(1/b), bitwise equal to the IEEE quotient, for divisors
// with a precomputed reciprocal (the 1-D grid metrics).  q0 = RN(a*rb) is
// within 1.5 ulp of a/b; one correction q + (a - b*q)*rb makes it faithful,
// and a second is correctly rounded by Markstein's theorem (P. Markstein,
// IBM J. Res. Dev. 34(1), 1990: with y = RN(1/b) and q within one ulp of
// a/b, RN(q + (a - b*q)*y) = RN(a/b); the FMA remainder is exact).  The
// theorem needs exact remainders, so non-finite values and |a| or |b|
// outside [2^-500, 2^500] take the plain division, except a zero a over such
// a b, whose quotient a*rb is exact (a signed zero).  FP32 keeps the build's
// division.
__device__ __forceinline__ double div_rcp(double a, double b, double rb) {
#if LARE_FAST
  // product build: the product with the reciprocal (within 1.5 ulp)
  (void)b;
  return a * rb;
#endif
  const unsigned ea = ((unsigned)__double2hiint(a) >> 20) & 0x7ffu;
  const unsigned eb = ((unsigned)__double2hiint(b) >> 20) & 0x7ffu;
  if (ea - 523u > 1000u || eb - 523u > 1000u) return (a == 0.0 && eb - 523u <= 1000u) ? a * rb : a / b;
  double q = a * rb;
  double r = fma(-b, q, a);
  q = fma(r, rb, q);
  r = fma(-b, q, a);
  return fma(r, rb, q);
}
__device__ __forceinline__ float div_rcp(float a, float b, float) { return a / b; }

// Reciprocal of the product build: the hardware's approximate FP64
// reciprocal (PTX rcp.approx.ftz.f64, measured on the B200 within 2^-20
// relative over 2^22 operands spread across 120 binades) refined by one step
// of the third-order Newton-Raphson iteration for 1/x: with e = 1 - x*y,
// y <- y + y*(e + e^2) cubes the relative error, 2^-60 before rounding, so
// the result is within one ulp of 1/x (checked on the GPU against numpy by
// tests/test_division_gpu.py).  For finite, normal x with |x| in
// [2^-1000, 2^1000]; the product build divides only by cell widths,
// volumes, densities and similar positive quantities in that range.  No
// branch, no slow path.
__device__ __forceinline__ double fast_rcp(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x, y, 1.0);
  return fma(fma(e, e, e), y, y);
}
__device__ __forceinline__ float fast_rcp(float x) { return 1.0f / x; }

// A quotient in the engine variant's arithmetic: IEEE a / b in the exact
// builds, a times the reciprocal above in the product build (LARE_FAST),
// within about two ulps of a / b.
template <class R>
__device__ __forceinline__ R qdiv(R a, R b) {
#if LARE_FAST
  return a * fast_rcp(b);
#else
  return a / b;
#endif
}
// A divisor in the form a kernel carries between neighbouring points: the
// value in the exact builds, its reciprocal in the product build; dv_div
// divides by it.
template <class R>
__device__ __forceinline__ R dv_of(R x) {
#if LARE_FAST
  return fast_rcp(x);
#else
  return x;
#endif
}
template <class R>
__device__ __forceinline__ R dv_div(R a, R dv) {
#if LARE_FAST
  return a * dv;
#else
  return a / dv;
#endif
}

// Asynchronous copy of one element from global to shared memory (PTX
// cp.async, 4 or 8 bytes, cached in L1), in commit groups that complete in
// order: a plane of a tile is copied without passing through registers.
template <class R>
__device__ __forceinline__ void cp_async_elem(R* smem, const R* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(s), "l"(gmem), "n"((int)sizeof(R)) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Wait until at most N of this thread's most recent groups are in flight.
template <int N>
__device__ __forceinline__ void cp_async_wait_prior() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Scalar slots kept in device memory so that a whole step can run (and be
// captured in a CUDA graph) without the host knowing dt.
enum Slot {
  SC_DT = 0,       // dt (shared_data)
  SC_DT2,          // dt2 = dt/2 (lagran.F90:132), also the predictor remap dt
  SC_DTR,          // dtr
  SC_TIME,         // time
  SC_DTSUB,        // resistive sub-cycle dt (lagran.F90:143)
  SC_DTCOND,       // dt used by an isolated conduct_heat call
  SC_VISC2N,       // visc2_norm (lagran.F90:545)
  SC_VISC_TOT,     // total_visc_heating
  SC_OHM_TOT,      // total_ohmic_heating
  SC_SUBSTEPS,     // resistive sub-cycles (integer value)
  SC_STAGES,       // RKL2 stages (integer value)
  SC_DTPARAB,      // explicit conduction limit
  SC_EN_B, SC_EN_KE, SC_EN_INT,
  SC_ERROR,        // LARE_E* code raised on the device (0 = none)
  SC_LOOP,         // remaining resistive sub-cycles of a captured step
  SC_NSLOTS = 24
};
// Integer min-reduction targets (bit patterns of positive doubles order
// like unsigned integers).
enum USlot { U_DTMIN = 0, U_DTRMIN, U_DTPARAB, U_NSLOTS = 4 };

struct Box {
  int lo[3], hi[3];
};

template <class Fn>
__global__ void __launch_bounds__(256) k_box(int i0, int j0, int k0, int ni, int nj, Fn fn) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= ni || j >= nj) return;
  fn(i0 + i, j0 + j, k0 + (int)blockIdx.z);
}
// The same with an occupancy hint: MINB blocks of 256 threads must fit on
// one SM, which caps the registers per thread.
template <int MINB, class Fn>
__global__ void __launch_bounds__(256, MINB) k_box_mb(int i0, int j0, int k0, int ni, int nj, Fn fn) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= ni || j >= nj) return;
  fn(i0 + i, j0 + j, k0 + (int)blockIdx.z);
}

// Block shape bx x by (bx * by <= 256), chosen per context (the ensemble
// autotuner sets it per grid size); every point runs the same arithmetic
// whatever the shape.
// ZP > 1: each thread takes ZP consecutive planes (more independent loads
// per thread; helps some FP32 kernels, whose 4-byte words leave few bytes
// in flight).  The order in which points are computed does not matter: a
// point kernel writes only its own point.
template <int ZP, class Fn>
__global__ void __launch_bounds__(256) k_box_z(int i0, int j0, int k0, int ni, int nj, int nk, Fn fn) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= ni || j >= nj) return;
#pragma unroll
  for (int p = 0; p < ZP; ++p) {
    const int k = (int)blockIdx.z * ZP + p;
    if (k < nk) fn(i0 + i, j0 + j, k0 + k);
  }
}

template <int MINB = 0, int ZP = 1, class Fn>
inline void launch_box(cudaStream_t s, long long& count, int i0, int i1, int j0, int j1, int k0, int k1, Fn fn,
                       int bx = 64, int by = 4) {
  int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
  if (ni <= 0 || nj <= 0 || nk <= 0) return;
  dim3 blk(bx, by, 1);
  dim3 grd((ni + bx - 1) / bx, (nj + by - 1) / by, nk);
  if constexpr (MINB > 0) {
    k_box_mb<MINB><<<grd, blk, 0, s>>>(i0, j0, k0, ni, nj, fn);
  } else if constexpr (ZP > 1) {
    grd.z = (nk + ZP - 1) / ZP;
    k_box_z<ZP><<<grd, blk, 0, s>>>(i0, j0, k0, ni, nj, nk, fn);
  } else {
    k_box<<<grd, blk, 0, s>>>(i0, j0, k0, ni, nj, fn);
  }
  ++count;
}

// Single-thread kernel for scalar bookkeeping on the device.
template <class Fn>
__global__ void k_scalar(Fn fn) {
  fn();
}
template <class Fn>
inline void launch_scalar(cudaStream_t s, long long& count, Fn fn) {
  k_scalar<<<1, 1, 0, s>>>(fn);
  ++count;
}

// ---------------------------------------------------------------------
// Deterministic sums: each block reduces NV values per thread in a fixed
// tree and writes its partials; one block then adds the partials in a
// fixed order.  Results are run-to-run reproducible (not equal to a
// serial left-to-right sum, which no parallel order can reproduce).
template <int NV>
__device__ __forceinline__ void block_sum_write(double (&v)[NV], double* partial, int bid) {
  __shared__ double sh[NV][8];
  for (int q = 0; q < NV; ++q) {
    double x = v[q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    v[q] = x;
  }
  int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
  int warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
  if (lane == 0)
    for (int q = 0; q < NV; ++q) sh[q][warp] = v[q];
  __syncthreads();
  if (warp == 0) {
    int nw = (blockDim.x * blockDim.y) >> 5;
    for (int q = 0; q < NV; ++q) {
      double x = lane < nw ? sh[q][lane] : 0.0;
      for (int o = 4; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) partial[(size_t)bid * NV + q] = x;
    }
  }
}

// Each block covers `planes` consecutive planes (kSumPlanes by default:
// fewer partials for the final pass; 1 for heavy point functions, whose
// planes would otherwise run one after another); a thread adds its points
// plane by plane, so the order of every sum is fixed.
constexpr int kSumPlanes = 4;

template <int NV, class Fn>
__global__ void __launch_bounds__(256) k_box_sum(int i0, int j0, int k0, int ni, int nj, int nk, int planes, Fn fn,
                                                 double* partial) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  double v[NV];
  for (int q = 0; q < NV; ++q) v[q] = 0.0;
  if (i < ni && j < nj) {
    const int kb = (int)blockIdx.z * planes;
    for (int kk = kb; kk < kb + planes && kk < nk; ++kk) {
      double w[NV];
      for (int q = 0; q < NV; ++q) w[q] = 0.0;
      fn(i0 + i, j0 + j, k0 + kk, w);
      for (int q = 0; q < NV; ++q) v[q] += w[q];
    }
  }
  int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  block_sum_write<NV>(v, partial, bid);
}

template <int NV>
__global__ void __launch_bounds__(1024) k_sum_partials(const double* partial, int nb, double* out, int accumulate) {
  __shared__ double sh[NV][32];
  int t = threadIdx.x;
  for (int q = 0; q < NV; ++q) {
    double x = 0.0;
    for (int b = t; b < nb; b += blockDim.x) x += partial[(size_t)b * NV + q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((t & 31) == 0) sh[q][t >> 5] = x;
  }
  __syncthreads();
  if (t < 32) {
    for (int q = 0; q < NV; ++q) {
      double x = sh[q][t];
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (t == 0) out[q] = accumulate ? out[q] + x : x;
    }
  }
}

// Min of positive doubles through their bit patterns.
__device__ __forceinline__ void atomic_min_pos(unsigned long long* u, double v) {
  atomicMin(u, (unsigned long long)__double_as_longlong(v));
}

template <int NV, class Fn>
__global__ void __launch_bounds__(256) k_box_min(int i0, int j0, int k0, int ni, int nj, int nk, int planes, Fn fn,
                                                 unsigned long long* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  double v[NV];
  for (int q = 0; q < NV; ++q) v[q] = DBL_MAX;
  // `planes` consecutive planes per block (the min does not depend on the
  // order), so that few blocks contend for the atomic on the result
  if (i < ni && j < nj) {
    const int kb = (int)blockIdx.z * planes;
    for (int kk = kb; kk < kb + planes && kk < nk; ++kk) {
      double w[NV];
      for (int q = 0; q < NV; ++q) w[q] = DBL_MAX;
      fn(i0 + i, j0 + j, k0 + kk, w);
      for (int q = 0; q < NV; ++q) v[q] = fmin(v[q], w[q]);
    }
  }
  __shared__ double sh[NV][8];
  for (int q = 0; q < NV; ++q) {
    double x = v[q];
    for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_down_sync(0xffffffffu, x, o));
    v[q] = x;
  }
  int tid = threadIdx.y * blockDim.x + threadIdx.x;
  int lane = tid & 31, warp = tid >> 5;
  if (lane == 0)
    for (int q = 0; q < NV; ++q) sh[q][warp] = v[q];
  __syncthreads();
  if (warp == 0) {
    int nw = (blockDim.x * blockDim.y) >> 5;
    for (int q = 0; q < NV; ++q) {
      double x = lane < nw ? sh[q][lane] : DBL_MAX;
      for (int o = 4; o > 0; o >>= 1) x = fmin(x, __shfl_down_sync(0xffffffffu, x, o));
      if (lane == 0) atomic_min_pos(out + q, x);
    }
  }
}

// ---------------------------------------------------------------------
// Ghost fills.  Every fill of boundary.f90 / mpiboundary.f90 on one rank is
// a sequence of whole-plane copies (periodic self-exchange, BC_USER mirror)
// or zeroings, applied dimension after dimension over the full extent of
// the other dimensions.  Such a sequence equals the composite map
//   out(i,j,k) = in(m_x(i), m_y(j), m_z(k))  (or 0 if any m_d says zero)
// applied to every point that some step writes, where m_d maps a written
// index to its source and leaves others alone.  All sources lie in the
// never-written range, so one kernel can apply the map in place.
struct GDim {
  int lo, hi;      // array extent in this dimension
  int a, b;        // contiguous never-written range
  int nw;          // number of written indices
  int widx[6];     // written indices
  int wsrc[6];     // source index, or INT_MIN for "set to zero"
};
struct GSpec {
  GDim d[3];
  long long c0, c1, c2;  // points in the three disjoint regions
};

__device__ __forceinline__ int gmap(const GDim& g, int i, bool& zero) {
  for (int q = 0; q < g.nw; ++q)
    if (g.widx[q] == i) {
      if (g.wsrc[q] == INT_MIN) { zero = true; return i; }
      return g.wsrc[q];
    }
  return i;
}

// Up to kMaxGhostJobs fills in one launch: blockIdx.y selects the job; a job
// applies one GSpec to up to three arrays.
constexpr int kMaxGhostJobs = 6;
template <class R>
struct GJobs {
  GSpec s[kMaxGhostJobs];
  R* p[kMaxGhostJobs][3];
  int n;
};

template <class R>
__device__ __forceinline__ void ghost_point(const GSpec& s, R* p0, R* p1, R* p2, int sx, int sxy, long long t);

template <class R>
__global__ void __launch_bounds__(256) k_ghost_multi(GJobs<R> J, int sx, int sxy) {
  const int j = blockIdx.y;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  ghost_point<R>(J.s[j], J.p[j][0], J.p[j][1], J.p[j][2], sx, sxy, t);
}

template <class R>
__global__ void __launch_bounds__(256) k_ghost(GSpec s, R* p0, R* p1, R* p2, int sx, int sxy) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  ghost_point<R>(s, p0, p1, p2, sx, sxy, t);
}

template <class R>
__device__ __forceinline__ void ghost_point(const GSpec& s, R* p0, R* p1, R* p2, int sx, int sxy, long long t64) {
  const GDim &X = s.d[0], &Y = s.d[1], &Z = s.d[2];
  // 32-bit index arithmetic (the host keeps c0 + c1 + c2 below 2^31): a
  // 64-bit division costs several times a 32-bit one, and these kernels
  // are dominated by it
  const unsigned c0 = (unsigned)s.c0, c1 = (unsigned)s.c1, c2 = (unsigned)s.c2;
  unsigned t = (unsigned)t64;
  if (t64 >= (long long)c0 + c1 + c2) return;
  int i, j, k;
  if (t < c0) {
    const unsigned nw = (unsigned)X.nw, ey = (unsigned)(Y.hi - Y.lo + 1);
    const unsigned r = t / nw;
    i = X.widx[t - r * nw];
    const unsigned rk = r / ey;
    j = Y.lo + (int)(r - rk * ey);
    k = Z.lo + (int)rk;
  } else if (t < c0 + c1) {
    t -= c0;
    const unsigned ex = (unsigned)(X.b - X.a + 1), nw = (unsigned)Y.nw;
    const unsigned r = t / ex;
    i = X.a + (int)(t - r * ex);
    const unsigned rk = r / nw;
    j = Y.widx[r - rk * nw];
    k = Z.lo + (int)rk;
  } else {
    t -= c0 + c1;
    const unsigned ex = (unsigned)(X.b - X.a + 1), ey = (unsigned)(Y.b - Y.a + 1);
    const unsigned r = t / ex;
    i = X.a + (int)(t - r * ex);
    const unsigned rk = r / ey;
    j = Y.a + (int)(r - rk * ey);
    k = Z.widx[rk];
  }
  bool zero = false;
  int si = gmap(X, i, zero), sj = gmap(Y, j, zero), sk = gmap(Z, k, zero);
  long long dst = i + (long long)sx * j + (long long)sxy * k;
  long long src = si + (long long)sx * sj + (long long)sxy * sk;
  R* ps[3] = {p0, p1, p2};
  for (int q = 0; q < 3; ++q) {
    R* p = ps[q];
    if (!p) continue;
    p[dst] = zero ? R(0) : p[src];
  }
}

LARE_END  // namespace lare
