// conduct.cuh - the RKL2 stage of conduct.f90:299-416 as one tiled kernel.
//
// The reference's heat_flux (conduct.f90:152-291) forms every face flux
// once and scatters it into the two cells that share the face.  A gather
// over cells computes each face twice; this kernel computes each once per
// stage: a CTA owns a 32 x 8 column of cells and walks up a chunk of z,
// holding the temperature of planes z-1, z, z+1 (with a one-cell x/y halo)
// in shared memory, the x and y face fluxes of the current plane in shared
// memory, and the z face flux below each cell in a register carried to the
// next plane.  The divergence adds the six scaled face fluxes of a cell in
// the order in which the reference's scatter delivers them to that cell:
//   +Fz(c-ez), +Fy(c-ey), +Fx(c-ex), -Fx(c), -Fy(c), -Fz(c)
// (iteration (i,j,k-1) precedes (i,j-1,k) precedes (i-1,j,k) precedes
// (i,j,k)).
#pragma once

namespace lare {

constexpr int kCTX = 32, kCTY = 8, kCZ = 16;  // CTA tile (x, y) and z chunk
constexpr int kCPlane = (kCTX + 2) * (kCTY + 2);

// Temperature of planes iz-1, iz, iz+1 of a CTA tile in shared memory.
template <class R>
struct PlaneT {
  const R* pm;
  const R* p0;
  const R* pp;
  int ix0, iy0, iz;
  __device__ __forceinline__ R operator()(int i, int j, int k) const {
    const R* p = k < iz ? pm : (k > iz ? pp : p0);
    return p[(j - iy0 + 1) * (kCTX + 2) + (i - ix0 + 1)];
  }
};

// FIRST: stage 1 (y_in = energy = Y0): Lc_Y0 = flux / rho and
//        out = Y0 + mt * dt * Lc_Y0.
// else:  stage j: out = mu Y2 + nu Y1 + (1 - mu - nu) Y0 + mt dt Lc + gt dt Lc_Y0
//        with Lc the flux of T(Y2) / rho.
template <class R, bool FIRST>
__global__ void __launch_bounds__(kCTX* kCTY) k_rkl2_stage(HeatFluxArgs<R> h, A3<R> y2, A3<R> y1, A3<R> y0,
                                                          A3<R> lc0, A3<R> rho, A3<R> out,
                                                          const double* __restrict__ sc, int dt_slot, R mt, R mu,
                                                          R nu, R omn, R gt, int nx, int ny, int nz) {
  __shared__ R Ts[3][kCPlane];
  __shared__ R fx[kCTY][kCTX + 1];
  __shared__ R fy[kCTY + 1][kCTX];
  const int tid = threadIdx.x;
  const int tx = tid % kCTX, ty = tid / kCTX;
  const int ix0 = 1 + blockIdx.x * kCTX, iy0 = 1 + blockIdx.y * kCTY;
  const int iz0 = 1 + blockIdx.z * kCZ;
  const int iz1 = min(nz, iz0 + kCZ - 1);
  const int ix = ix0 + tx, iy = iy0 + ty;
  const bool active = ix <= nx && iy <= ny;
  const R dt = (R)sc[dt_slot];
  auto slot = [](int k) { return (k + 3) % 3; };
  auto load_plane = [&](int k) {
    R* d = Ts[slot(k)];
    for (int e = tid; e < kCPlane; e += kCTX * kCTY) {
      const int jj = e / (kCTX + 2), ii = e - jj * (kCTX + 2);
      const int i = min(ix0 - 1 + ii, nx + 2), j = min(iy0 - 1 + jj, ny + 2);
      d[e] = h.T(i, j, k);
    }
  };
  load_plane(iz0 - 1);
  load_plane(iz0);
  R fz_m = R(0);
  for (int iz = iz0; iz <= iz1; ++iz) {
    load_plane(iz + 1);
    __syncthreads();
    const PlaneT<R> P{Ts[slot(iz - 1)], Ts[slot(iz)], Ts[slot(iz + 1)], ix0, iy0, iz};
    if (iz == iz0 && active) {
      const PlaneT<R> Pm{nullptr, Ts[slot(iz - 1)], Ts[slot(iz)], ix0, iy0, iz - 1};
      fz_m = face_flux(h, Pm, 2, ix, iy, iz - 1);
    }
    for (int f = tid; f < kCTY * (kCTX + 1); f += kCTX * kCTY) {
      const int r = f / (kCTX + 1), c = f - r * (kCTX + 1);
      const int fi = ix0 - 1 + c, fj = iy0 + r;
      if (fi <= nx && fj <= ny) fx[r][c] = face_flux(h, P, 0, fi, fj, iz);
    }
    for (int f = tid; f < (kCTY + 1) * kCTX; f += kCTX * kCTY) {
      const int r = f / kCTX, c = f - r * kCTX;
      const int fi = ix0 + c, fj = iy0 - 1 + r;
      if (fi <= nx && fj <= ny) fy[r][c] = face_flux(h, P, 1, fi, fj, iz);
    }
    R fz_p = R(0);
    if (active) fz_p = face_flux(h, P, 2, ix, iy, iz);
    __syncthreads();
    if (active) {
      R f = R(0);
      f = f + fz_m;
      f = f + fy[ty][tx];
      f = f + fx[ty][tx];
      f = f - fx[ty][tx + 1];
      f = f - fy[ty + 1][tx];
      f = f - fz_p;
      if (FIRST) {
        const R lc = (R(1) / rho(ix, iy, iz)) * f;
        lc0(ix, iy, iz) = lc;
        out(ix, iy, iz) = y0(ix, iy, iz) + mt * dt * lc;
      } else {
        const R c0 = gt * dt * lc0(ix, iy, iz);
        const R Lc = (R(1) / rho(ix, iy, iz)) * f;
        const R c1 = mt * dt * Lc;
        const R v = mu * y2(ix, iy, iz) + nu * y1(ix, iy, iz) + omn * y0(ix, iy, iz);
        out(ix, iy, iz) = v + c1 + c0;
      }
    }
    fz_m = fz_p;
  }
}

template <class R, bool FIRST>
void rkl2_stage(Run<R>& run, int line, const HeatFluxArgs<R>& h, A3<R> y2, A3<R> y1, A3<R> y0, A3<R> out,
                int dt_slot, R mt, R mu, R nu, R omn, R gt) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  dim3 grid((nx + kCTX - 1) / kCTX, (ny + kCTY - 1) / kCTY, (nz + kCZ - 1) / kCZ);
  const int k = run.prof_begin("rkl2_stage", line, FIRST ? 9 : 10, (double)nx * ny * nz);
  k_rkl2_stage<R, FIRST><<<grid, kCTX * kCTY, 0, run.s>>>(h, y2, y1, y0, run.a.Lc_Y0, run.a.rho, out, run.sc,
                                                          dt_slot, mt, mu, nu, omn, gt, nx, ny, nz);
  run.prof_end(k);
  ++run.launches;
}

}  // namespace lare
