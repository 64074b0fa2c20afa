// lp4_tile.cuh - p_visc, the viscous heating and the viscous vertex forces
// of shock_viscosity (lagran.F90:680-789) as a tiled z-march.
//
// Per cell c (0:n+1) the kernel needs the velocity differences along the
// twelve edges of the cell, whose corners are the vertices (x-1..x,
// y-1..y, z-1..z), and per vertex (0:n) the velocity at the vertex and its
// six neighbours.  A CTA of 32 x 8 threads owns a 32 x 8 column and walks a
// 16-plane chunk of z with the velocity planes z-1, z and z+1 (a one-vertex
// x/y halo on each side) in a ring of four shared-memory slots; plane z+2
// is copied into the fourth by cp.async while plane z is computed, so no
// register holds a plane in flight.  Each velocity is read from memory about
// once per CTA instead of through 33 cached loads per point with run-time
// strides; the edge viscosities and metrics are read per point.  At 256^3:
// 0.67 ms in FP64 against 0.70 ms for the point kernel (one thread a point,
// every operand from memory) and 0.77 ms for the same tile with the next
// plane staged in registers (127 registers, two CTAs an SM); 0.42 against
// 0.43 ms in FP32.  The same expressions over the same operands as the point
// form, so the exact build stays bit for bit.
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

template <class R>
__global__ void __launch_bounds__(kL4X * kL4Y, sizeof(R) == 8 ? 3 : 4) k_lp4_tile(LP4Args<R> g) {
  __shared__ R Vs[4][3][kL4P];  // [plane slot][component][element]
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kL4X + tx;
  const int ix0 = blockIdx.x * kL4X, iy0 = blockIdx.y * kL4Y;
  const int ix = ix0 + tx, iy = iy0 + ty;
  const int iz0 = blockIdx.z * kL4Z;
  const int iz1 = min(iz0 + kL4Z - 1, g.nz + 1);
  const int sx = g.sx, sxy = g.sxy;
  const bool cell = ix <= g.nx + 1 && iy <= g.ny + 1;  // p_visc, visc_heat
  const bool vert = ix <= g.nx && iy <= g.ny;          // the forces
  // the plane elements this thread copies: halo box x in ix0-1..ix0+32,
  // y in iy0-1..iy0+8 (clamped to the array; clamped values are never used)
  int off[2];
  bool has[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int e = tid + q * kL4X * kL4Y;
    has[q] = e < kL4P;
    const int jj = has[q] ? e / kL4W : 0, ii = has[q] ? e - jj * kL4W : 0;
    off[q] = min(ix0 - 1 + ii, g.nx + 2) + sx * min(iy0 - 1 + jj, g.ny + 2);
  }
  const R* const V[3] = {g.vx, g.vy, g.vz};
  // plane k (-1 <= k <= nz + 2) into slot (k + 4) % 4, as one commit group
  auto issue = [&](int k) {
    const int slot = (k + 4) & 3;
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
      for (int q = 0; q < 2; ++q)
        if (has[q]) cp_async_elem(&Vs[slot][m][tid + q * kL4X * kL4Y], V[m] + off[q] + sxy * k);
    cp_async_commit();
  };
  const int e = (ty + 1) * kL4W + tx + 1;  // this thread's vertex (x, y) in a plane slot
  const int X = 1, Y = kL4W;               // neighbours within a plane slot
  issue(iz0 - 1);
  issue(iz0);
  issue(iz0 + 1);
  const R ddx = g.dxb(min(ix, g.nx + 1)), ddy = g.dyb(min(iy, g.ny + 1));
  const R dcx = g.dxc(min(ix, g.nx)), dcy = g.dyc(min(iy, g.ny));
  for (int iz = iz0; iz <= iz1; ++iz) {
    // plane iz + 2 goes to the slot of plane iz - 2, last read before the
    // previous barrier (an empty group at the end keeps the count)
    if (iz < iz1) {
      issue(iz + 2);
    } else {
      cp_async_commit();
    }
    cp_async_wait_prior<1>();  // planes up to iz + 1 have landed
    __syncthreads();
    const int sm = (iz + 3) & 3, s0 = iz & 3, sp = (iz + 1) & 3;
    const int c = ix + sx * iy + sxy * iz;
    if (cell) {
      // |dv|^2 between two vertices given as (slot, offset)
      auto d2 = [&](int s1, int o1, int s2, int o2) {
        const R ux = Vs[s1][0][e + o1] - Vs[s2][0][e + o2];
        const R uy = Vs[s1][1][e + o1] - Vs[s2][1][e + o2];
        const R uz = Vs[s1][2][e + o1] - Vs[s2][2][e + o2];
        return ux * ux + uy * uy + uz * uz;
      };
      // the vertices c - X - Y - Z ... c of the point form, as (plane, offset)
      const R a1 = d2(sm, -X - Y, sm, -Y);
      const R a2 = d2(sm, -Y, sm, 0);
      const R a3 = d2(sm, 0, sm, -X);
      const R a4 = d2(sm, -X, sm, -X - Y);
      const R a5 = d2(s0, -X - Y, s0, -Y);
      const R a6 = d2(s0, -Y, s0, 0);
      const R a7 = d2(s0, 0, s0, -X);
      const R a8 = d2(s0, -X, s0, -X - Y);
      const R a9 = d2(sm, 0, s0, 0);
      const R a10 = d2(sm, -X, s0, -X);
      const R a11 = d2(sm, -X - Y, s0, -X - Y);
      const R a12 = d2(sm, -Y, s0, -Y);
      const int GY = sx, GZ = sxy, GX = 1;
      R pv = R(0);
      pv = fmax(pv, -g.alpha1[c] * sqrt(a1));
      pv = fmax(pv, -g.alpha2[c] * sqrt(a2));
      pv = fmax(pv, -g.alpha3[c] * sqrt(a9));
      g.p_visc[c] = pv;
      const R ddz = g.dzb(iz);
      const R vh = -R(0.25) * ddy * ddz * g.alpha1[c] * a1 - R(0.25) * ddx * ddz * g.alpha2[c] * a2 -
                   R(0.25) * ddy * ddz * g.alpha1[c + GY] * a3 - R(0.25) * ddx * ddz * g.alpha2[c - GX] * a4 -
                   R(0.25) * ddy * ddz * g.alpha1[c + GZ] * a5 - R(0.25) * ddx * ddz * g.alpha2[c + GZ] * a6 -
                   R(0.25) * ddy * ddz * g.alpha1[c + GY + GZ] * a7 -
                   R(0.25) * ddx * ddz * g.alpha2[c - GX + GZ] * a8 - R(0.25) * ddx * ddy * g.alpha3[c] * a9 -
                   R(0.25) * ddx * ddy * g.alpha3[c - GX] * a10 - R(0.25) * ddx * ddy * g.alpha3[c - GX - GY] * a11 -
                   R(0.25) * ddx * ddy * g.alpha3[c - GY] * a12;
      g.visc_heat[c] = qdiv(vh, g.cv[c]);
      if (vert && iz <= g.nz) {
        const R dcz = g.dzc(iz);
        const R b1 = g.alpha1[c + GY + GZ] * dcy * dcz;
        const R b2 = g.alpha1[c + GX + GY + GZ] * dcy * dcz;
        const R b3 = g.alpha2[c + GZ] * dcx * dcz;
        const R b4 = g.alpha2[c + GY + GZ] * dcx * dcz;
        const R b5 = g.alpha3[c] * dcx * dcy;
        const R b6 = g.alpha3[c + GZ] * dcx * dcy;
        const R cvv = dv_of(g.cv_v[c]);
        auto f = [&](int m) {
          const R v0 = Vs[s0][m][e];
          return dv_div(b1 * (v0 - Vs[s0][m][e - X]) + b2 * (v0 - Vs[s0][m][e + X]) +
                            b3 * (v0 - Vs[s0][m][e - Y]) + b4 * (v0 - Vs[s0][m][e + Y]) +
                            b5 * (v0 - Vs[sm][m][e]) + b6 * (v0 - Vs[sp][m][e]),
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
