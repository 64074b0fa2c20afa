// lare_noalloc.cu - energy budget of caller-owned device arrays, with no
// device allocation.
//
// Who needs this: a caller that keeps Lare3d's state in its own device
// memory and may not, or cannot, let a library call cudaMalloc - e.g. a
// driver whose device memory comes from a fixed pool it manages itself, one
// that must not grow the device footprint between its own allocations, or
// one that issues this call between stream-ordered steps where an
// allocation would synchronise the device.  lare_gpu_energy() needs a
// context, which allocates the full state; this entry point needs nothing
// but the caller's arrays.
//
// Its scratch (one FP64 partial sum per block and quantity) is the
// file-scope array below, sized for LARE_NOALLOC_MAX_POINTS points.  It is
// part of the library image: every GPU that loads the library holds it
// until the process exits.  All calls share it, so two calls that overlap on
// the GPU (different streams, or different host threads without ordering)
// race on it; calls on one stream are ordered and safe.  Each call writes
// every slot it later reads before reading it, so no slot has to start at
// zero and nothing is cleared.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/lare_gpu.h"

namespace {

constexpr int kThreads = 256;
constexpr long long kPointsPerBlock = 8192;
// One slot triple per block; a launch uses ceil(points / kPointsPerBlock)
// blocks, so the array is sized by the same rounding.
constexpr int kMaxBlocks = (int)((LARE_NOALLOC_MAX_POINTS + kPointsPerBlock - 1) / kPointsPerBlock);
static_assert((long long)kMaxBlocks * kPointsPerBlock >= (long long)LARE_NOALLOC_MAX_POINTS,
              "the scratch must hold one partial per block of the largest accepted grid");
constexpr int kMaxDevices = 64;

// Block partials: [block][0] en_b, [block][1] en_ke, [block][2] en_int.
static __device__ __align__(256) double g_energy_scratch[3 * kMaxBlocks];

// The scratch address is looked up once per CUDA context and cached with
// that context's unique id (cuCtxGetId ids are never reused in a process).
// After cudaDeviceReset, or when the primary context is released and made
// again, the library image is loaded anew, possibly at another address; the
// id then differs and the address is looked up again instead of reusing a
// stale one.
struct ScratchSlot {
  unsigned long long ctx_id;
  double* ptr;
};
std::mutex g_mu;
ScratchSlot g_slot[kMaxDevices] = {};

using PfnCtxGetCurrent = CUresult (*)(CUcontext*);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long*);

// The current context's id through the driver entry points the runtime
// hands out (no link-time dependency on libcuda); 0 when unavailable, in
// which case the address is looked up on every call.
unsigned long long current_context_id() {
  static PfnCtxGetCurrent get_current = nullptr;
  static PfnCtxGetId get_id = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (PfnCtxGetCurrent)f;
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (PfnCtxGetId)f;
  }
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// The device address of g_energy_scratch in the current context
// (cudaGetSymbolAddress with the caller's device current).  In host code
// the symbol name is only a stand-in and must not be passed to a kernel.
int scratch_for_current_device(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return LARE_ECUDA;
  std::lock_guard<std::mutex> lock(g_mu);
  // With no context current yet (id 0), the lookup below makes the device's
  // primary context current, and its id is read after it.
  const unsigned long long id = current_context_id();
  ScratchSlot& s = g_slot[dev];
  if (id == 0 || s.ctx_id != id || !s.ptr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_energy_scratch);
    if (e != cudaSuccess || !p) return LARE_ECUDA;
    s.ptr = (double*)p;
    s.ctx_id = id != 0 ? id : current_context_id();
  }
  *out = s.ptr;
  return LARE_OK;
}

struct Dims {
  int nx, ny, nz;
};

__device__ __forceinline__ double block_reduce(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = lane < (kThreads / 32) ? sh[lane] : 0.0;
    for (int o = 4; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;
}

// diagnostics.F90:517-609 (do_sum = .FALSE.): block b sums cells and
// vertices [b*P, (b+1)*P) of the two loops, each thread in a fixed order.
__global__ void __launch_bounds__(kThreads)
k_energy_partials(Dims d, const double* __restrict__ rho, const double* __restrict__ energy,
                  const double* __restrict__ vx, const double* __restrict__ vy, const double* __restrict__ vz,
                  const double* __restrict__ bx, const double* __restrict__ by, const double* __restrict__ bz,
                  const double* __restrict__ dxb, const double* __restrict__ dyb, const double* __restrict__ dzb,
                  double* __restrict__ partial) {
  __shared__ double sh[kThreads / 32];
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  // Fortran-bounded strides: cell (-1:n+2), node (-2:n+2), bx (-2:,-1:,-1:),
  // by (-1:,-2:,-1:), bz (-1:,-1:,-2:); metrics dxb(-1:n+2).
  const long long cx = nx + 4, cxy = cx * (ny + 4);
  const long long nxs = nx + 5, nxys = nxs * (ny + 5);
  const long long bxx = nx + 5, bxxy = bxx * (ny + 4);
  const long long byx = nx + 4, byxy = byx * (ny + 5);
  const long long bzx = nx + 4, bzxy = bzx * (ny + 4);
  auto C = [&](const double* a, int i, int j, int k) { return a[(i + 1) + cx * (j + 1) + cxy * (k + 1)]; };
  auto N = [&](const double* a, int i, int j, int k) { return a[(i + 2) + nxs * (j + 2) + nxys * (k + 2)]; };
  auto BX = [&](int i, int j, int k) { return bx[(i + 2) + bxx * (j + 1) + bxxy * (k + 1)]; };
  auto BY = [&](int i, int j, int k) { return by[(i + 1) + byx * (j + 2) + byxy * (k + 1)]; };
  auto BZ = [&](int i, int j, int k) { return bz[(i + 1) + bzx * (j + 1) + bzxy * (k + 2)]; };
  auto cv = [&](int i, int j, int k) { return dxb[i + 1] * dyb[j + 1] * dzb[k + 1]; };

  const long long base = (long long)blockIdx.x * kPointsPerBlock;
  double eb = 0.0, ei = 0.0, eke = 0.0;
  const long long ncell = (long long)nx * ny * nz;
  for (long long t = base + threadIdx.x; t < base + kPointsPerBlock && t < ncell; t += kThreads) {
    int ix = 1 + (int)(t % nx);
    long long r = t / nx;
    int iy = 1 + (int)(r % ny);
    int iz = 1 + (int)(r / ny);
    int ixm = ix - 1, iym = iy - 1, izm = iz - 1;
    double b0 = BX(ix, iy, iz), b1 = BX(ixm, iy, iz), c0 = BY(ix, iy, iz), c1 = BY(ix, iym, iz);
    double e0 = BZ(ix, iy, iz), e1 = BZ(ix, iy, izm);
    double w1 = (b0 * b0 + b1 * b1) * 0.5;
    double w2 = (c0 * c0 + c1 * c1) * 0.5;
    double w3 = (e0 * e0 + e1 * e1) * 0.5;
    w1 = (w1 + w2 + w3) * 0.5;
    double v = cv(ix, iy, iz);
    eb += w1 * v;
    ei += C(energy, ix, iy, iz) * C(rho, ix, iy, iz) * v;
  }
  const long long nvert = (long long)(nx + 1) * (ny + 1) * (nz + 1);
  for (long long t = base + threadIdx.x; t < base + kPointsPerBlock && t < nvert; t += kThreads) {
    int ix = (int)(t % (nx + 1));
    long long r = t / (nx + 1);
    int iy = (int)(r % (ny + 1));
    int iz = (int)(r / (ny + 1));
    int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
    double rv = C(rho, ix, iy, iz) * cv(ix, iy, iz) + C(rho, ixp, iy, iz) * cv(ixp, iy, iz) +
                C(rho, ix, iyp, iz) * cv(ix, iyp, iz) + C(rho, ixp, iyp, iz) * cv(ixp, iyp, iz) +
                C(rho, ix, iy, izp) * cv(ix, iy, izp) + C(rho, ixp, iy, izp) * cv(ixp, iy, izp) +
                C(rho, ix, iyp, izp) * cv(ix, iyp, izp) + C(rho, ixp, iyp, izp) * cv(ixp, iyp, izp);
    double cvv = cv(ix, iy, iz) + cv(ixp, iy, iz) + cv(ix, iyp, iz) + cv(ixp, iyp, iz) + cv(ix, iy, izp) +
                 cv(ixp, iy, izp) + cv(ix, iyp, izp) + cv(ixp, iyp, izp);
    rv = rv / cvv;
    cvv = cvv * 0.125;
    double ux = N(vx, ix, iy, iz), uy = N(vy, ix, iy, iz), uz = N(vz, ix, iy, iz);
    double w1 = rv * cvv * (ux * ux + uy * uy + uz * uz);
    if (ix == 0 || ix == nx) w1 = w1 * 0.5;
    if (iy == 0 || iy == ny) w1 = w1 * 0.5;
    if (iz == 0 || iz == nz) w1 = w1 * 0.5;
    eke += w1 * 0.5;
  }
  eb = block_reduce(eb, sh);
  eke = block_reduce(eke, sh);
  ei = block_reduce(ei, sh);
  if (threadIdx.x == 0) {
    partial[3 * blockIdx.x + 0] = eb;
    partial[3 * blockIdx.x + 1] = eke;
    partial[3 * blockIdx.x + 2] = ei;
  }
}

// Sum the nb block partials in a fixed order into out[0..2].
__global__ void __launch_bounds__(1024) k_energy_finish(const double* __restrict__ partial, int nb,
                                                        double* __restrict__ out) {
  __shared__ double sh[32];
  for (int q = 0; q < 3; ++q) {
    double v = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) v += partial[3 * b + q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
      double r = sh[threadIdx.x];
      for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
      if (threadIdx.x == 0) out[q] = r;
    }
    __syncthreads();
  }
}

}  // namespace

extern "C" int lare_gpu_energy_noalloc(int nx, int ny, int nz, const double* rho, const double* energy,
                                       const double* vx, const double* vy, const double* vz, const double* bx,
                                       const double* by, const double* bz, const double* dxb, const double* dyb,
                                       const double* dzb, double* out3, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1) return LARE_EINVAL;
  const long long nvert = (long long)(nx + 1) * (ny + 1) * (nz + 1);
  if (nvert > (long long)LARE_NOALLOC_MAX_POINTS) return LARE_ETOOLARGE;
  if (!rho || !energy || !vx || !vy || !vz || !bx || !by || !bz || !dxb || !dyb || !dzb || !out3)
    return LARE_EINVAL;
  double* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc != LARE_OK) return rc;
  const int nb = (int)((nvert + kPointsPerBlock - 1) / kPointsPerBlock);
  cudaStream_t s = (cudaStream_t)stream;
  Dims d{nx, ny, nz};
  k_energy_partials<<<nb, kThreads, 0, s>>>(d, rho, energy, vx, vy, vz, bx, by, bz, dxb, dyb, dzb, scratch);
  k_energy_finish<<<1, 1024, 0, s>>>(scratch, nb, out3);
  return cudaGetLastError() == cudaSuccess ? LARE_OK : LARE_ECUDA;
}
