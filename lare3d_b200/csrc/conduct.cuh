// conduct.cuh - the heat flux of conduct.f90:152-291 and the RKL2 stage of
// conduct.f90:299-416 as tiled kernels.
//
// Face flux (conduct.f90:170-275), x face between cells ix and ix+1:
//   q = -L k0 T_f^{5/2} (b0 (b0 g_x + by_f g_y + bz_f g_z) + min_b g_x) / |B|^2
// with T_f the face-mean temperature, g the temperature gradient at the
// face (the transverse parts from the face-mean temperatures of the two
// neighbouring rows), L the Larsen factor of cell ix and |B|^2 = b0^2 +
// by_f^2 + bz_f^2 + min_b.  heat_flux scatters q / dxb(ix) into the two
// cells.  Everything but T is fixed during a conduction step, so
// face_coefficients forms, once per step, three coefficients per face
//   k_n = L (b0^2 + min_b) / |B|^2 / dxc(ix) / dxb(ix)
//   k_1 = L b0 by_f / |B|^2 / (2 (dyc(iy) + dyc(iy-1))) / dxb(ix)
//   k_2 = L b0 bz_f / |B|^2 / (2 (dzc(iz) + dzc(iz-1))) / dxb(ix)
// and the stage kernel evaluates q / dxb = -k0 T_f^{5/2} (k_n dT_n + k_1 dS_1
// + k_2 dS_2) with dT_n = T(ix+1) - T(ix) and dS the differences of the
// two-point temperature sums of the neighbouring rows.  The same algebra,
// regrouped (and T^{5/2} = T^2 sqrt(T)), agrees with the reference to
// rounding (relative 1e-12 in FP64).
//
// Stage kernel: a CTA owns a 32 x 8 column of cells and walks up a chunk of
// z, holding the temperature of planes z-1, z, z+1 (one-cell x/y halo) in
// shared memory, the x and y face fluxes of the current plane in shared
// memory and the z face flux below each cell in a register carried to the
// next plane, so each face flux is formed once.  A cell adds its six scaled
// face fluxes in the order in which the reference's scatter delivers them:
//   +Fz(c-ez), +Fy(c-ey), +Fx(c-ex), -Fx(c), -Fy(c), -Fz(c).
#pragma once

LARE_BEGIN

constexpr int kCTX = 32, kCTY = 8, kCZ = 16;  // CTA tile (x, y) and z chunk
constexpr int kCW = kCTX + 2;                 // plane row length with halo
constexpr int kCPlane = kCW * (kCTY + 2);

// Coefficients of every face of cells 0..n (conduct.f90:170-275 regrouped).
template <class R>
void face_coefficients(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  Arrays<R>& A = run.a;
  auto bx = A.bx, by = A.by, bz = A.bz, larsen = A.larsen;
  const A1<R> rdb0 = A.rdb[0], rdb1 = A.rdb[1], rdb2 = A.rdb[2];
  const A1<R> rdc0 = A.rdc[0], rdc1 = A.rdc[1], rdc2 = A.rdc[2];
  const A1<R> rs0 = A.rdc2[0], rs1 = A.rdc2[1], rs2 = A.rdc2[2];
  A3<R> k[9];
  for (int q = 0; q < 9; ++q) k[q] = A.kf[q];
  const A3<R> k0 = k[0], k1 = k[1], k2 = k[2], k3 = k[3], k4 = k[4], k5 = k[5], k6 = k[6], k7 = k[7], k8 = k[8];
  // Extension, not in the reference: kappa_perp = rp kappa_par adds
  // rp (g_n - b_n (b . g) / |B|^2) to the bracket, i.e. rp (|B|^2 - b0^2)
  // to the normal coefficient's numerator and a factor (1 - rp) to the
  // transverse ones; rp = 0 is the reference's flux.
  const R rp = (R)run.p.kappa_perp_ratio, orp = R(1) - rp;
  LARE_BOXW(run, 13, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz) {
    const R min_b = R(1.0e-10);  // conduct.f90:28
    const R half = R(0.5), q4 = R(0.25);
    const int ixp = ix + 1, ixm = ix - 1, iyp = iy + 1, iym = iy - 1, izp = iz + 1, izm = iz - 1;
    const R lf = larsen(ix, iy, iz);
    {  // x face
      const R byf = q4 * (by(ix, iy, iz) + by(ixp, iy, iz) + by(ix, iym, iz) + by(ixp, iym, iz));
      const R bzf = q4 * (bz(ix, iy, iz) + bz(ixp, iy, iz) + bz(ix, iy, izm) + bz(ixp, iy, izm));
      const R b0 = bx(ix, iy, iz);
      const R modb = b0 * b0 + byf * byf + bzf * bzf + min_b;
      const R w = lf / modb * rdb0(ix);
      k0(ix, iy, iz) = w * ((b0 * b0 + min_b) + rp * (modb - b0 * b0)) * rdc0(ix);
      k1(ix, iy, iz) = w * b0 * byf * orp * half * rs1(iy);
      k2(ix, iy, iz) = w * b0 * bzf * orp * half * rs2(iz);
    }
    {  // y face
      const R bxf = q4 * (bx(ix, iy, iz) + bx(ix, iyp, iz) + bx(ixm, iy, iz) + bx(ixm, iyp, iz));
      const R bzf = q4 * (bz(ix, iy, iz) + bz(ix, iyp, iz) + bz(ix, iy, izm) + bz(ix, iyp, izm));
      const R b0 = by(ix, iy, iz);
      const R modb = bxf * bxf + b0 * b0 + bzf * bzf + min_b;
      const R w = lf / modb * rdb1(iy);
      k3(ix, iy, iz) = w * ((b0 * b0 + min_b) + rp * (modb - b0 * b0)) * rdc1(iy);
      k4(ix, iy, iz) = w * b0 * bxf * orp * half * rs0(ix);
      k5(ix, iy, iz) = w * b0 * bzf * orp * half * rs2(iz);
    }
    {  // z face
      const R bxf = q4 * (bx(ix, iy, iz) + bx(ix, iy, izp) + bx(ixm, iy, iz) + bx(ixm, iy, izp));
      const R byf = q4 * (by(ix, iy, iz) + by(ix, iy, izp) + by(ix, iym, iz) + by(ix, iym, izp));
      const R b0 = bz(ix, iy, iz);
      const R modb = bxf * bxf + byf * byf + b0 * b0 + min_b;
      const R w = lf / modb * rdb2(iz);
      k6(ix, iy, iz) = w * ((b0 * b0 + min_b) + rp * (modb - b0 * b0)) * rdc2(iz);
      k7(ix, iy, iz) = w * b0 * bxf * orp * half * rs0(ix);
      k8(ix, iy, iz) = w * b0 * byf * orp * half * rs1(iy);
    }
  });
}

template <class R>
struct StageArgs {
  TempOf<R> T;                      // temperature of the stage input
  A3<R> k[9];                       // face coefficients
  A3<R> y2, y1, y0, lc0, rho, out;  // stage arrays
  R k0, mt, mu, nu, omn, gt;
  int dt_slot, nx, ny, nz;
};

template <class R>
__device__ __forceinline__ R face_q(R k0, R T0, R T1, R kn, R k1, R s1, R k2, R s2) {
  R tb = (T1 + T0) * R(0.5);
  tb = tb > R(0) ? tb : R(0);
  return -k0 * pow25(tb) * (kn * (T1 - T0) + k1 * s1 + k2 * s2);
}

// Stage kernel.  A CTA of 32 x 8 threads owns a tile of 31 x 8 cells and
// walks a chunk of z.  Each thread forms the x face flux on the low side of
// its cell; lane 31's cell belongs to the next tile and only hands its low
// face to lane 30 (the high face of every cell comes from the lane above by
// a shuffle, so no lane forms a face twice).  Each thread also forms the y
// face flux on the low side of its cell into shared memory, where the row
// above reads it as its high face; the top row forms its high face itself.
// The z face flux on the high side is carried to the next plane.  The
// temperature of planes z-1, z, z+1 with a one-cell x/y halo sits in shared
// memory, loaded a plane ahead.
constexpr int kSTX = 31;  // cells per tile along x (a warp of 32 lanes)
constexpr int kSW = kSTX + 2;
constexpr int kSPlane = kSW * (kCTY + 2);

template <class R>
struct StagePre {
  R kx[3], ky[3], ky2[3], kz[3];
  R rho, y0, y1, y2, lc;
};

// FIRST: stage 1 (y2 = energy = Y0): Lc_Y0 = flux / rho and
//        out = Y0 + mt * dt * Lc_Y0.
// else:  stage j: out = mu Y2 + nu Y1 + (1 - mu - nu) Y0 + mt dt Lc + gt dt Lc_Y0
//        with Lc the flux of T(Y2) / rho.
template <class R, bool FIRST>
__global__ void __launch_bounds__(32 * kCTY, sizeof(R) == 4 ? 4 : 2)
    k_rkl2_stage(StageArgs<R> a, const double* __restrict__ sc) {
  __shared__ R Ts[3][kSPlane];
  __shared__ R fy[kCTY + 1][32];
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int lane = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * 32 + lane;
  const int ix0 = 1 + blockIdx.x * kSTX, iy0 = 1 + blockIdx.y * kCTY;
  const int iz0 = 1 + blockIdx.z * kCZ;
  const int iz1 = min(nz, iz0 + kCZ - 1);
  const int ix = ix0 + lane, iy = iy0 + ty;
  // lane 31 only forms the x face below its cell (the high x face of lane 30)
  const bool own = lane < kSTX;
  const bool active = own && ix <= nx && iy <= ny;            // cells this tile updates
  const bool hx = ix - 1 <= nx && iy <= ny;                   // x face at ix - 1 (low side)
  const bool hy = own && ix <= nx && iy - 1 <= ny;            // y face at iy - 1 (low side)
  const bool top = ty == kCTY - 1;                            // the top row also forms its high y face
  const bool hy2 = own && top && ix <= nx && iy <= ny;
  const bool cell = active;                                   // z faces of the cells updated here
  const int sx = a.T.y.sx, sxy = a.T.y.sxy;
  const int cxy = min(ix, nx + 2) + sx * min(iy, ny + 2);     // this thread's column (clamped)
  // the (up to two) plane elements this thread loads, as column offsets
  int off[2];
  bool has[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int e = tid + q * 32 * kCTY;
    has[q] = e < kSPlane;
    const int jj = has[q] ? e / kSW : 0, ii = has[q] ? e - jj * kSW : 0;
    off[q] = min(ix0 - 1 + ii, nx + 2) + sx * min(iy0 - 1 + jj, ny + 2);
  }
  const R tc = a.T.c, te0 = a.T.e0;
  const R* __restrict__ ysrc = a.T.y.p;
  const R dt = (R)sc[a.dt_slot];
  auto load_plane = [&](int k) {
    R* d = Ts[(k + 3) % 3];
#pragma unroll
    for (int q = 0; q < 2; ++q)
      if (has[q]) d[tid + q * 32 * kCTY] = tc * (ysrc[off[q] + sxy * k] - te0);
  };
  auto fetch = [&](int k) {
    StagePre<R> q;
    const int c = cxy + sxy * k;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      q.kx[m] = hx ? a.k[m].p[c - 1] : R(0);
      q.ky[m] = hy ? a.k[3 + m].p[c - sx] : R(0);
      q.ky2[m] = hy2 ? a.k[3 + m].p[c] : R(0);
      q.kz[m] = cell ? a.k[6 + m].p[c] : R(0);
    }
    q.rho = active ? a.rho.p[c] : R(1);
    q.y0 = active ? a.y0.p[c] : R(0);
    q.y1 = (active && !FIRST) ? a.y1.p[c] : R(0);
    q.y2 = (active && !FIRST) ? a.y2.p[c] : R(0);
    q.lc = (active && !FIRST) ? a.lc0.p[c] : R(0);
    return q;
  };
  // z face above cell e of plane slots pm (lower) and pp (upper)
  auto zface = [&](const R* pm, const R* pp, int e, R k6, R k7, R k8) {
    return face_q(a.k0, pm[e], pp[e], k6, k7, (pp[e + 1] + pm[e + 1]) - (pp[e - 1] + pm[e - 1]), k8,
                  (pp[e + kSW] + pm[e + kSW]) - (pp[e - kSW] + pm[e - kSW]));
  };
  // y face between cell e - kSW and cell e of plane slots Pm, P0, Pp
  auto yface = [&](const R* Pm, const R* P0, const R* Pp, int e, const R (&k)[3]) {
    const int b = e - kSW;
    return face_q(a.k0, P0[b], P0[e], k[0], k[1], (P0[b + 1] + P0[e + 1]) - (P0[b - 1] + P0[e - 1]), k[2],
                  (Pp[b] + Pp[e]) - (Pm[b] + Pm[e]));
  };
  const int ec = (ty + 1) * kSW + lane + 1;  // this thread's cell in a plane slot
  load_plane(iz0 - 1);
  load_plane(iz0);
  R fz_m = R(0);
  R b6 = R(0), b7 = R(0), b8 = R(0);
  if (cell) {
    const int c = cxy + sxy * (iz0 - 1);
    b6 = a.k[6].p[c];
    b7 = a.k[7].p[c];
    b8 = a.k[8].p[c];
  }
  __syncthreads();
  if (cell) fz_m = zface(Ts[(iz0 + 2) % 3], Ts[iz0 % 3], ec, b6, b7, b8);
  StagePre<R> nxt = fetch(iz0);
  for (int iz = iz0; iz <= iz1; ++iz) {
    const StagePre<R> cur = nxt;
    load_plane(iz + 1);
    if (iz < iz1) nxt = fetch(iz + 1);
    __syncthreads();
    const R* Pm = Ts[(iz + 2) % 3];
    const R* P0 = Ts[iz % 3];
    const R* Pp = Ts[(iz + 1) % 3];
    R fx_lo = R(0);
    if (hx) {
      const int e = ec - 1;  // face between cells ix - 1 and ix
      fx_lo = face_q(a.k0, P0[e], P0[e + 1], cur.kx[0], cur.kx[1],
                     (P0[e + kSW + 1] + P0[e + kSW]) - (P0[e - kSW + 1] + P0[e - kSW]), cur.kx[2],
                     (Pp[e + 1] + Pp[e]) - (Pm[e + 1] + Pm[e]));
    }
    const R fx_hi = __shfl_down_sync(0xffffffffu, fx_lo, 1);
    if (hy) fy[ty][lane] = yface(Pm, P0, Pp, ec, cur.ky);
    if (hy2) fy[kCTY][lane] = yface(Pm, P0, Pp, ec + kSW, cur.ky2);
    R fz_p = R(0);
    if (cell) fz_p = zface(P0, Pp, ec, cur.kz[0], cur.kz[1], cur.kz[2]);
    __syncthreads();
    if (active) {
      R f = R(0);
      f = f + fz_m;
      f = f + fy[ty][lane];
      f = f + fx_lo;
      f = f - fx_hi;
      f = f - fy[ty + 1][lane];
      f = f - fz_p;
      const int c = cxy + sxy * iz;
      if (FIRST) {
        const R lc = (R(1) / cur.rho) * f;
        a.lc0.p[c] = lc;
        a.out.p[c] = cur.y0 + a.mt * dt * lc;
      } else {
        const R c0 = a.gt * dt * cur.lc;
        const R Lc = (R(1) / cur.rho) * f;
        const R c1 = a.mt * dt * Lc;
        const R v = a.mu * cur.y2 + a.nu * cur.y1 + a.omn * cur.y0;
        a.out.p[c] = v + c1 + c0;
      }
    }
    fz_m = fz_p;
  }
}

template <class R, bool FIRST>
void rkl2_stage(Run<R>& run, int line, const TempOf<R>& T, A3<R> y2, A3<R> y1, A3<R> y0, A3<R> out, int dt_slot,
                R mt, R mu, R nu, R omn, R gt) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  StageArgs<R> a;
  a.T = T;
  for (int q = 0; q < 9; ++q) a.k[q] = run.a.kf[q];
  a.y2 = y2;
  a.y1 = y1;
  a.y0 = y0;
  a.lc0 = run.a.Lc_Y0;
  a.rho = run.a.rho;
  a.out = out;
  a.k0 = (R)run.p.kappa_0;
  a.mt = mt;
  a.mu = mu;
  a.nu = nu;
  a.omn = omn;
  a.gt = gt;
  a.dt_slot = dt_slot;
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  dim3 grid((nx + kSTX - 1) / kSTX, (ny + kCTY - 1) / kCTY, (nz + kCZ - 1) / kCZ);
  // words per point: T stencil input, 9 coefficients, rho, Lc_Y0, output (+ Y1, Y0 after stage 1)
  const int k = run.prof_begin("rkl2_stage", line, FIRST ? 13 : 15, (double)nx * ny * nz);
  k_rkl2_stage<R, FIRST><<<grid, dim3(32, kCTY, 1), 0, run.s>>>(a, run.sc);
  run.prof_end(k);
  ++run.launches;
}

LARE_END  // namespace lare
