// lp4_tile.cuh - p_visc, the viscous heating and the viscous vertex forces
// of shock_viscosity (lagran.F90:680-789) as a tiled z-march.
//
// Per cell c (0:n+1) the kernel needs the velocity differences along the
// twelve edges of the cell, whose corners are the vertices (x-1..x,
// y-1..y, z-1..z), the edge viscosities alpha1..3 of the cell and of its
// neighbours, and per vertex (0:n) the velocity at the vertex and its six
// neighbours.  A CTA of 32 x 8 threads owns a 32 x 8 column and walks a
// 16-plane chunk of z with the planes of vx, vy, vz, alpha1, alpha2 and
// alpha3 (a one-point x/y halo on each side) in a ring of four
// shared-memory slots; plane z+2 is copied into the fourth by cp.async
// while plane z is computed, so no register holds a plane in flight.  Every
// stencil operand comes from shared memory; cv and cv_v are read per point.
// At 256^3: 0.65 ms in FP64 against 0.70 ms for the point kernel (one thread
// a point, about 60 loads with run-time strides), 0.69 ms with only the
// velocities in the ring and 0.77 ms with them staged in registers
// (127 registers, two CTAs an SM); in FP32 0.36 against 0.42 ms with only
// the velocities in the ring.  The same expressions over the same operands
// as the point form, so the exact build stays bit for bit.
#pragma once

LARE_BEGIN

constexpr int kL4X = 32, kL4Y = 8, kL4Z = 16;
constexpr int kL4W = kL4X + 2;           // plane row with a one-vertex halo each side
constexpr int kL4P = kL4W * (kL4Y + 2);  // plane size

template <class R>
struct LP4Args {
  const R* vx;
  const R* vy;
  const R* vz;
  const R* alpha1;
  const R* alpha2;
  const R* alpha3;
  const R* cv;
  const R* cv_v;
  R* p_visc;
  R* visc_heat;
  R* fx;
  R* fy;
  R* fz;
  A1<R> dxb, dyb, dzb, dxc, dyc, dzc;
  int nx, ny, nz, sx, sxy;
};

// Dynamic shared memory of k_lp4_tile: four slots of six planes.
template <class R>
constexpr size_t lp4_smem_bytes() {
  return (size_t)4 * 6 * kL4P * sizeof(R);
}

template <class R>
__global__ void __launch_bounds__(kL4X * kL4Y, sizeof(R) == 8 ? 3 : 4) k_lp4_tile(LP4Args<R> g) {
  extern __shared__ __align__(16) unsigned char l4_smem[];
  R* const buf = reinterpret_cast<R*>(l4_smem);  // [slot][array][element]
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kL4X + tx;
  const int ix0 = blockIdx.x * kL4X, iy0 = blockIdx.y * kL4Y;
  const int ix = ix0 + tx, iy = iy0 + ty;
  const int iz0 = blockIdx.z * kL4Z;
  const int iz1 = min(iz0 + kL4Z - 1, g.nz + 1);
  const int sx = g.sx, sxy = g.sxy;
  const bool cell = ix <= g.nx + 1 && iy <= g.ny + 1;
  const bool vert = ix <= g.nx && iy <= g.ny;
  int off[2];
  bool has[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int e = tid + q * kL4X * kL4Y;
    has[q] = e < kL4P;
    const int jj = has[q] ? e / kL4W : 0, ii = has[q] ? e - jj * kL4W : 0;
    off[q] = min(ix0 - 1 + ii, g.nx + 2) + sx * min(iy0 - 1 + jj, g.ny + 2);
  }
  const R* const V[6] = {g.vx, g.vy, g.vz, g.alpha1, g.alpha2, g.alpha3};
  auto P = [&](int slot, int m) { return buf + (slot * 6 + m) * kL4P; };
  auto issue = [&](int k) {
    const int slot = (k + 4) & 3;
#pragma unroll
    for (int m = 0; m < 6; ++m)
#pragma unroll
      for (int q = 0; q < 2; ++q)
        if (has[q]) cp_async_elem(P(slot, m) + tid + q * kL4X * kL4Y, V[m] + off[q] + sxy * k);
    cp_async_commit();
  };
  const int e = (ty + 1) * kL4W + tx + 1;
  const int X = 1, Y = kL4W;
  issue(iz0 - 1);
  issue(iz0);
  issue(iz0 + 1);
  const R ddx = g.dxb(min(ix, g.nx + 1)), ddy = g.dyb(min(iy, g.ny + 1));
  const R dcx = g.dxc(min(ix, g.nx)), dcy = g.dyc(min(iy, g.ny));
  for (int iz = iz0; iz <= iz1; ++iz) {
    if (iz < iz1) {
      issue(iz + 2);
    } else {
      cp_async_commit();
    }
    cp_async_wait_prior<1>();
    __syncthreads();
    const int sm = (iz + 3) & 3, s0 = iz & 3, sp = (iz + 1) & 3;
    const int c = ix + sx * iy + sxy * iz;
    if (cell) {
      auto d2 = [&](int s1, int o1, int s2, int o2) {
        const R ux = P(s1, 0)[e + o1] - P(s2, 0)[e + o2];
        const R uy = P(s1, 1)[e + o1] - P(s2, 1)[e + o2];
        const R uz = P(s1, 2)[e + o1] - P(s2, 2)[e + o2];
        return ux * ux + uy * uy + uz * uz;
      };
      const R* const a1 = P(s0, 3);
      const R* const a2 = P(s0, 4);
      const R* const a3 = P(s0, 5);
      const R* const a1p = P(sp, 3);
      const R* const a2p = P(sp, 4);
      const R* const a3p = P(sp, 5);
      const R e1 = d2(sm, -X - Y, sm, -Y);
      const R e2 = d2(sm, -Y, sm, 0);
      const R e3 = d2(sm, 0, sm, -X);
      const R e4 = d2(sm, -X, sm, -X - Y);
      const R e5 = d2(s0, -X - Y, s0, -Y);
      const R e6 = d2(s0, -Y, s0, 0);
      const R e7 = d2(s0, 0, s0, -X);
      const R e8 = d2(s0, -X, s0, -X - Y);
      const R e9 = d2(sm, 0, s0, 0);
      const R e10 = d2(sm, -X, s0, -X);
      const R e11 = d2(sm, -X - Y, s0, -X - Y);
      const R e12 = d2(sm, -Y, s0, -Y);
      R pv = R(0);
      pv = fmax(pv, -a1[e] * sqrt(e1));
      pv = fmax(pv, -a2[e] * sqrt(e2));
      pv = fmax(pv, -a3[e] * sqrt(e9));
      g.p_visc[c] = pv;
      const R ddz = g.dzb(iz);
      const R vh = -R(0.25) * ddy * ddz * a1[e] * e1 - R(0.25) * ddx * ddz * a2[e] * e2 -
                   R(0.25) * ddy * ddz * a1[e + Y] * e3 - R(0.25) * ddx * ddz * a2[e - X] * e4 -
                   R(0.25) * ddy * ddz * a1p[e] * e5 - R(0.25) * ddx * ddz * a2p[e] * e6 -
                   R(0.25) * ddy * ddz * a1p[e + Y] * e7 - R(0.25) * ddx * ddz * a2p[e - X] * e8 -
                   R(0.25) * ddx * ddy * a3[e] * e9 - R(0.25) * ddx * ddy * a3[e - X] * e10 -
                   R(0.25) * ddx * ddy * a3[e - X - Y] * e11 - R(0.25) * ddx * ddy * a3[e - Y] * e12;
      g.visc_heat[c] = qdiv(vh, g.cv[c]);
      if (vert && iz <= g.nz) {
        const R dcz = g.dzc(iz);
        const R b1 = a1p[e + Y] * dcy * dcz;
        const R b2 = a1p[e + X + Y] * dcy * dcz;
        const R b3 = a2p[e] * dcx * dcz;
        const R b4 = a2p[e + Y] * dcx * dcz;
        const R b5 = a3[e] * dcx * dcy;
        const R b6 = a3p[e] * dcx * dcy;
        const R cvv = dv_of(g.cv_v[c]);
        auto f = [&](int m) {
          const R* const v0p = P(s0, m);
          const R v0 = v0p[e];
          return dv_div(b1 * (v0 - v0p[e - X]) + b2 * (v0 - v0p[e + X]) + b3 * (v0 - v0p[e - Y]) +
                            b4 * (v0 - v0p[e + Y]) + b5 * (v0 - P(sm, m)[e]) + b6 * (v0 - P(sp, m)[e]),
                        cvv);
        };
        g.fx[c] = f(0);
        g.fy[c] = f(1);
        g.fz[c] = f(2);
      }
    }
    __syncthreads();
  }
  cp_async_wait_prior<0>();
}

LARE_END  // namespace lare
