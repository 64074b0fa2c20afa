// lagran.cuh - lagrangian_step (lagran.F90:50-200) with its callees, fused.
//
// Kernels (each element computed by the reference's own expression over
// the reference's own inputs, so results are bit-identical; only where
// intermediates live changes):
//   LP1 prologue   face->cell B, pressure, sound speed cs, vertex rho_v and
//                  cv_v (:83-125, shock_viscosity :551-559); the cell B
//                  averages stay in registers
//   LP2 cs_v       (:561-581)
//   LP3 alphas     the three edge-viscosity loops (:583-678)
//   LP4 p_visc, visc_heat and the viscous forces (:680-789)
//   RS1 eta_calc + rkstep: one current evaluation serves both (:1182-1225,
//                  :1470-1503, identical expressions)
//   RS2 bstep      the three face updates (:1582-1631) into a second B
//                  buffer; bfield_bcs then writes every element outside
//                  the update ranges, so the buffers swap instead of the
//                  bx1 = bx copy (:1259-1261)
//   RS3 ohmic heating, energy = MAX(energy, 0) and total_ohmic_heating
//   PR  the predictor's half-dt B remap on a converted copy of B, so the
//                  saved bx0 and the restore (:223-225, :389-393) become a
//                  pointer swap, and v is read in place of the vx1 = vx copy
//   PC1 energy = MAX(energy0 + delta, 0) (:180-181) and the predictor
//                  pressure (:234-249)
//   PC2 vertex forces and the half-step velocity (:251-387)
//   PC3 shock_heating (:861-937) and v = 2 v1 - v (:399-407) into a second
//                  v buffer
//   PC4 final cv1, energy, rho and total_visc_heating (:415-462)
// The repeated velocity_bcs at the end of lagrangian_step (:198) follows an
// identical one with no velocity change in between, so it is skipped.
#pragma once

#include <utility>

#include "lp4_tile.cuh"

LARE_BEGIN

// Vertex current of eta_calc (lagran.F90:1190-1216), rkstep (:1479-1494)
// and the predictor force (:358-373): the three places use the same
// expressions (eta_calc and rkstep evaluate them in k_eta_march, which
// carries operands between vertices).  With RCP the divisions by the cell
// widths go through their reciprocals (rx, ry, rz) and div_rcp, which
// returns the same quotients; the predictor force measured faster that way.
template <class R, bool RCP>
__device__ __forceinline__ void vertex_current(const R* bx, const R* by, const R* bz, int c, int sx, int sxy,
                                               R dxc, R dyc, R dzc, R rx, R ry, R rz, R& jx, R& jy, R& jz) {
  auto div_rcp = [](R a, R b, R r) { return RCP ? lare::div_rcp(a, b, r) : a / b; };
  R jx1 = div_rcp(bz[c + sx] - bz[c], dyc, ry) - div_rcp(by[c + sxy] - by[c], dzc, rz);
  R jx2 = div_rcp(bz[c + 1 + sx] - bz[c + 1], dyc, ry) - div_rcp(by[c + 1 + sxy] - by[c + 1], dzc, rz);
  R jy1 = div_rcp(bx[c + sxy] - bx[c], dzc, rz) - div_rcp(bz[c + 1] - bz[c], dxc, rx);
  R jy2 = div_rcp(bx[c + sx + sxy] - bx[c + sx], dzc, rz) - div_rcp(bz[c + 1 + sx] - bz[c + sx], dxc, rx);
  R jz1 = div_rcp(by[c + 1] - by[c], dxc, rx) - div_rcp(bx[c + sx] - bx[c], dyc, ry);
  R jz2 = div_rcp(by[c + 1 + sxy] - by[c + sxy], dxc, rx) - div_rcp(bx[c + sx + sxy] - bx[c + sxy], dyc, ry);
  jx = (jx1 + jx2) * R(0.5);
  jy = (jy1 + jy2) * R(0.5);
  jz = (jz1 + jz2) * R(0.5);
}

// eta_calc (+ rkstep) as a z-marching kernel: a thread owns an (x, y)
// column of vertices and walks a chunk of z.  Of the vertex current's
// operands, bx and by at z+1 (c+Z, c+X+Z, c+Y+Z) are the next vertex's c,
// c+X, c+Y, and the two quotients of jz2, (by(c+X+Z)-by(c+Z))/dxc and
// (bx(c+Y+Z)-bx(c+Z))/dyc, are the next vertex's jz1 terms; a step loads
// 8 values and divides 10 times instead of 12 and 12.  Same expressions,
// same operands, same results bit for bit.
constexpr int kEtaZ = 32;

template <class R>
struct EtaArgs {
  const R* bx;
  const R* by;
  const R* bz;
  R* eta;
  R* fx;
  R* fy;
  R* fz;
  R* curlb;
  const R* eta_perp;  // Cowling branch only
  A1<R> dxc, dyc, dzc;
  R jmax, eb, e0;
  int nx, ny, nz, sx, sxy;
  bool rkstep;
};

// COW: rkstep's partially ionised branch (lagran.F90:1506-1575), which
// splits the current into its parts along and across the vertex field and
// adds eta_perp to the cross-field part.  The vertex field averages use the
// same bx, by and bz values the current does.
template <class R, bool COW>
__global__ void __launch_bounds__(128) k_eta_march(EtaArgs<R> g) {
  // distinct arrays (no output is an input): restrict lets the compiler
  // hoist the next plane's loads above this plane's stores
  const R* __restrict__ bx_r = g.bx;
  const R* __restrict__ by_r = g.by;
  const R* __restrict__ bz_r = g.bz;
  R* __restrict__ eta_r = g.eta;
  R* __restrict__ fx_r = g.fx;
  R* __restrict__ fy_r = g.fy;
  R* __restrict__ fz_r = g.fz;
  R* __restrict__ curlb_r = g.curlb;
  const int ix = -1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int iy = -1 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  if (ix > g.nx + 1 || iy > g.ny + 1) return;
  const int z0 = -1 + (int)blockIdx.z * kEtaZ;
  const int z1 = min(z0 + kEtaZ - 1, g.nz + 1);
  const int sx = g.sx, sxy = g.sxy;
  const R dxc = g.dxc(ix), dyc = g.dyc(iy);
  const R vxc = dv_of(dxc), vyc = dv_of(dyc);  // divisors in the variant's form
  int c = ix + sx * iy + sxy * z0;
  // plane z0 values of bx (c, c+Y) and by (c, c+X), and the jz1 quotients
  R bx0 = bx_r[c], bxy = bx_r[c + sx], by0 = by_r[c], byx = by_r[c + 1];
  R qa = dv_div(byx - by0, vxc), qb = dv_div(bxy - bx0, vyc);
  const bool inxy = ix >= 0 && ix <= g.nx && iy >= 0 && iy <= g.ny;
  for (int iz = z0; iz <= z1; ++iz, c += sxy) {
    const R dzc = g.dzc(iz);
    const R vzc = dv_of(dzc);
    const R bz0 = bz_r[c], bzx = bz_r[c + 1], bzy = bz_r[c + sx], bzxy = bz_r[c + 1 + sx];
    const R bxz = bx_r[c + sxy], bxyz = bx_r[c + sx + sxy], byz = by_r[c + sxy], byxz = by_r[c + 1 + sxy];
    const R jx1 = dv_div(bzy - bz0, vyc) - dv_div(byz - by0, vzc);
    const R jx2 = dv_div(bzxy - bzx, vyc) - dv_div(byxz - byx, vzc);
    const R jy1 = dv_div(bxz - bx0, vzc) - dv_div(bzx - bz0, vxc);
    const R jy2 = dv_div(bxyz - bxy, vzc) - dv_div(bzxy - bzy, vxc);
    const R qa2 = dv_div(byxz - byz, vxc), qb2 = dv_div(bxyz - bxz, vyc);
    const R jz1 = qa - qb;
    const R jz2 = qa2 - qb2;
    const R jx = (jx1 + jx2) * R(0.5);
    const R jy = (jy1 + jy2) * R(0.5);
    const R jz = (jz1 + jz2) * R(0.5);
    const R j2 = jx * jx + jy * jy + jz * jz;
    const R e = sqrt(j2) > g.jmax ? g.eb + g.e0 : g.eb;
    eta_r[c] = e;
    if (g.rkstep && inxy && iz >= 0 && iz <= g.nz) {
      if constexpr (COW) {
        const R bxv = (bx0 + bxy + bxz + bxyz) * R(0.25);
        const R byv = (by0 + byx + byz + byxz) * R(0.25);
        const R bzv = (bz0 + bzx + bzy + bzxy) * R(0.25);
        const R magn_b = bxv * bxv + byv * byv + bzv * bzv;
        R jpx = R(0), jpy = R(0), jpz = R(0);
        if (magn_b > Num<R>::tiny()) {
          const R vmb = dv_of(magn_b);
          jpx = dv_div((jx * bxv + jy * byv + jz * bzv) * bxv, vmb);
          jpy = dv_div((jx * bxv + jy * byv + jz * bzv) * byv, vmb);
          jpz = dv_div((jx * bxv + jy * byv + jz * bzv) * bzv, vmb);
        }
        const R jqx = jx - jpx, jqy = jy - jpy, jqz = jz - jpz;
        const R mpar = sqrt(jpx * jpx + jpy * jpy + jpz * jpz);
        const R mperp = sqrt(jqx * jqx + jqy * jqy + jqz * jqz);
        const R ep = g.eta_perp[c];
        curlb_r[c] = e * (mpar * mpar) + (ep + e) * (mperp * mperp);
        fx_r[c] = -((jpx + jqx) * e + jqx * ep) * dxc * R(0.5);
        fy_r[c] = -((jpy + jqy) * e + jqy * ep) * dyc * R(0.5);
        fz_r[c] = -((jpz + jqz) * e + jqz * ep) * dzc * R(0.5);
      } else {
        fx_r[c] = -jx * e * dxc * R(0.5);
        fy_r[c] = -jy * e * dyc * R(0.5);
        fz_r[c] = -jz * e * dzc * R(0.5);
        curlb_r[c] = e * j2;
      }
    }
    bx0 = bxz;
    bxy = bxyz;
    by0 = byz;
    byx = byxz;
    qa = qa2;
    qb = qb2;
  }
}

// ---------------------------------------------------------------------
// eta_calc (lagran.F90:1176-1230), optionally fused with rkstep (:1470-1503)
// whose fluxes need eta at the same vertex.
template <class R>
void eta_and_rkstep(Run<R>& run, bool with_rkstep) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  const int sx = run.sx, sxy = run.sxy;
  R* const eta = run.a.eta.p;
  if (!run.p.resistive_mhd) {
    whole(run, [=] __device__(int i, int j, int k) { eta[i + sx * j + sxy * k] = R(0); });
    return;
  }
  const R* bx = run.a.bx.p;
  const R* by = run.a.by.p;
  const R* bz = run.a.bz.p;
  R* const fxp = run.a.flux_x.p;
  R* const fyp = run.a.flux_y.p;
  R* const fzp = run.a.flux_z.p;
  R* const curlb = run.a.curlb.p;
  auto dxc = run.a.dxc, dyc = run.a.dyc, dzc = run.a.dzc;
  const R jmax = (R)run.p.j_max, eb = (R)run.p.eta_background, e0 = (R)run.p.eta0;
  EtaArgs<R> ga;
  ga.bx = bx;
  ga.by = by;
  ga.bz = bz;
  ga.eta = eta;
  ga.fx = fxp;
  ga.fy = fyp;
  ga.fz = fzp;
  ga.curlb = curlb;
  ga.eta_perp = run.a.eta_perp.p;
  ga.dxc = dxc;
  ga.dyc = dyc;
  ga.dzc = dzc;
  ga.jmax = jmax;
  ga.eb = eb;
  ga.e0 = e0;
  ga.nx = nx;
  ga.ny = ny;
  ga.nz = nz;
  ga.sx = sx;
  ga.sxy = sxy;
  ga.rkstep = with_rkstep;
  dim3 grd((nx + 3 + 31) / 32, (ny + 3 + 3) / 4, (nz + 3 + kEtaZ - 1) / kEtaZ);
  const int k = run.prof_begin("eta_and_rkstep", 0, with_rkstep ? 8 : 4, (double)(nx + 3) * (ny + 3) * (nz + 3));
  if (with_rkstep && run.cowling)
    k_eta_march<R, true><<<grd, dim3(32, 4, 1), 0, run.s>>>(ga);
  else
    k_eta_march<R, false><<<grd, dim3(32, 4, 1), 0, run.s>>>(ga);
  run.prof_end(k);
  ++run.launches;
}

template <class R>
void eta_calc(Run<R>& run) {
  eta_and_rkstep(run, false);
}

// ---------------------------------------------------------------------
// lagran.F90:1239-1452 resistive_effects (first order, no cooling term),
// after eta_and_rkstep.
template <class R>
void resistive_update(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  const int sx = run.sx, sxy = run.sxy;
  Arrays<R>& A = run.a;
  const R* bxo = A.bx.p;
  const R* byo = A.by.p;
  const R* bzo = A.bz.p;
  R* const bxn = A.bx1.p;
  R* const byn = A.by1.p;
  R* const bzn = A.bz1.p;
  const R* kx = A.flux_x.p;
  const R* ky = A.flux_y.p;
  const R* kz = A.flux_z.p;
  auto dxb = A.dxb, dyb = A.dyb, dzb = A.dzb, dxc = A.dxc, dyc = A.dyc, dzc = A.dzc;
  const double* sc = run.sc;
  // RS2: bstep (:1588-1631) into the second buffers
  LARE_BOXWH(run, 4, 4, 9, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz) {
    const R dt = (R)sc[SC_DTSUB];
    const int c = ix + sx * iy + sxy * iz;
    if (iy >= 1 && iz >= 1) {
      R area = dyb(iy) * dzb(iz);
      bxn[c] = bxo[c] + qdiv((kz[c] - kz[c - sx] + kz[c - sxy] - kz[c - sx - sxy] - ky[c] + ky[c - sxy] - ky[c - sx] +
                              ky[c - sx - sxy]) * dt,
                             area);
    }
    if (ix >= 1 && iz >= 1) {
      R area = dxb(ix) * dzb(iz);
      byn[c] = byo[c] + qdiv((kx[c] - kx[c - sxy] + kx[c - 1] - kx[c - 1 - sxy] - kz[c] + kz[c - 1] - kz[c - sxy] +
                              kz[c - 1 - sxy]) * dt,
                             area);
    }
    if (ix >= 1 && iy >= 1) {
      R area = dxb(ix) * dyb(iy);
      bzn[c] = bzo[c] + qdiv((ky[c] - ky[c - 1] + ky[c - sx] - ky[c - 1 - sx] - kx[c] + kx[c - sx] - kx[c - 1] +
                              kx[c - 1 - sx]) * dt,
                             area);
    }
  });
  std::swap(A.bx.p, A.bx1.p);
  std::swap(A.by.p, A.by1.p);
  std::swap(A.bz.p, A.bz1.p);
  {
    // bstep updates bx over 0:n x 1:n x 1:n, by over 1:n x 0:n x 1:n, bz
    // over 1:n x 1:n x 0:n (lagran.F90:1588-1631)
    R* const nb[3] = {A.bx.p, A.by.p, A.bz.p};
    R* const ob[3] = {A.bx1.p, A.by1.p, A.bz1.p};
    for (int q = 0; q < 3; ++q) {
      int lo[3] = {-1, -1, -1}, hi[3] = {nx + 2, ny + 2, nz + 2}, a[3] = {1, 1, 1}, b[3] = {nx, ny, nz};
      lo[q] = -2;
      a[q] = 0;
      carry_outside(run, nb[q], ob[q], lo, hi, a, b);
    }
  }
  bfield_bcs(run);
  // RS3: ohmic heating (1:n), MAX(energy, 0) (-1:n+2) and the
  // total_ohmic_heating sum over vertices 0:n (:1270-1328)
  R* const energy = A.energy.p;
  R* const ohmic = A.ohmic_dep.p;
  const R* curlb = A.curlb.p;
  const R* rho = A.rho.p;
  R* const ctb = run.p.cooling_term ? A.cool_term_b.p : nullptr;  // :1290-1302
  const R alpha = (R)run.p.alpha_av;
  box_sum<1>(run, "ohmic_heating_sum", -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz, double* v) {
    const R dt = (R)sc[SC_DTSUB];
    const int c = ix + sx * iy + sxy * iz;
    R e = energy[c];
    if (ix >= 1 && ix <= nx && iy >= 1 && iy <= ny && iz >= 1 && iz <= nz) {
      R lh = qdiv(+(curlb[c] + curlb[c - 1] + curlb[c - sx] + curlb[c - 1 - sx] + curlb[c - sxy] + curlb[c - 1 - sxy] +
                    curlb[c - sx - sxy] + curlb[c - 1 - sx - sxy]) * dt,
                  R(8) * rho[c]);
      ohmic[c] = ohmic[c] + lh;
      e = e + lh;
      if (ctb) {
        // the moving average of the heating of the iz plane's four
        // vertices only, as the reference writes it
        const R lh4 = qdiv((curlb[c] + curlb[c - 1] + curlb[c - sx] + curlb[c - 1 - sx]) * dt, R(4) * rho[c]);
        const R t = alpha * lh4 + (R(1) - alpha) * ctb[c];
        ctb[c] = t;
        e = e - t;
      }
    }
    energy[c] = e > R(0) ? e : R(0);
    if (ix >= 0 && ix <= nx && iy >= 0 && iy <= ny && iz >= 0 && iz <= nz) {
      R w1 = dt * dxc(ix) * dyc(iy) * dzc(iz) * curlb[c];
      if (ix == 0 || ix == nx) w1 = w1 * R(0.5);
      if (iy == 0 || iy == ny) w1 = w1 * R(0.5);
      if (iz == 0 || iz == nz) w1 = w1 * R(0.5);
      v[0] = (double)w1;
    }
  }, SC_OHM_TOT, true, ctb ? 8 : 6);
  energy_bcs(run);
}

// ---------------------------------------------------------------------
// LP1-LP4: prologue and shock_viscosity (lagran.F90:83-125, 532-857)
template <class R>
void prologue_and_shock_viscosity(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  const int sx = run.sx, sxy = run.sxy;
  Arrays<R>& A = run.a;
  if (!run.visc2_norm_set) {
    run.visc2_norm_set = true;
    double v2n = 0.25 * (run.p.gamma + 1.0) * run.p.visc2;
    if (sizeof(R) == 4) v2n = (double)(R(0.25) * (R(run.p.gamma) + R(1)) * R(run.p.visc2));
    cudaMemcpyAsync(run.sc + SC_VISC2N, &v2n, sizeof(double), cudaMemcpyHostToDevice, run.s);
    cudaStreamSynchronize(run.s);
  }
  const R* bx = A.bx.p;
  const R* by = A.by.p;
  const R* bz = A.bz.p;
  const R* rho = A.rho.p;
  const R* energy = A.energy.p;
  const R* cv = A.cv.p;
  const R* gamma_boris = A.gamma_boris.p;
  R* const pressure = A.pressure.p;
  R* const cs = A.cs.p;
  R* const rho_v = A.rho_v.p;
  R* const cv_v = A.cv_v.p;
  R* const p_visc = A.p_visc.p;
  const R g = (R)run.p.gamma, xi = (R)run.p.xi_n, ip = (R)run.p.ionise_pot;
  const R* xin = run.pip ? A.xi.p : nullptr;  // per-cell xi_n (neutral.f90) or the constant
  // LP1
  LARE_BOXWH(run, 0, 4, 11, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
    const int c = ix + sx * iy + sxy * iz;
    R bx1 = (bx[c] + bx[c - 1]) * R(0.5);
    R by1 = (by[c] + by[c - sx]) * R(0.5);
    R bz1 = (bz[c] + bz[c - sxy]) * R(0.5);
    R r = rho[c];
    const R x = xin ? xin[c] : xi;
    R pr = (g - R(1)) * r * (energy[c] - (R(1) - x) * ip);
    pressure[c] = pr;
    R rmin = fmax(r, Num<R>::tiny());
    R b2 = bx1 * bx1 + by1 * by1 + bz1 * bz1;
    cs[c] = sqrt(qdiv(g * pr + gamma_boris[c] * b2, rmin));
    if (ix == -1 || ix == nx + 2 || iy == -1 || iy == ny + 2 || iz == -1 || iz == nz + 2)
      p_visc[c] = R(0);  // p_visc = 0 (:548) outside the 0:n+1 MAX loop
    if (ix <= nx + 1 && iy <= ny + 1 && iz <= nz + 1) {
      // the eight cells around vertex c, in the reference's order
      const int o1 = 1, o2 = sx, o3 = 1 + sx, o4 = sxy, o5 = 1 + sxy, o6 = sx + sxy, o7 = 1 + sx + sxy;
      R rv = rho[c] * cv[c] + rho[c + o1] * cv[c + o1] + rho[c + o2] * cv[c + o2] + rho[c + o3] * cv[c + o3] +
             rho[c + o4] * cv[c + o4] + rho[c + o5] * cv[c + o5] + rho[c + o6] * cv[c + o6] +
             rho[c + o7] * cv[c + o7];
      R cvv = cv[c] + cv[c + o1] + cv[c + o2] + cv[c + o3] + cv[c + o4] + cv[c + o5] + cv[c + o6] + cv[c + o7];
      rho_v[c] = qdiv(rv, cvv);
      cv_v[c] = R(0.125) * cvv;
    }
  });
  if (run.p.coronal_heating) {
    // lagran.F90:127 user_defined_heating (radiative.f90:88-91): after the
    // pressure, before the viscosity; dt is still the previous set_dt's
    R* const en = A.energy.p;
    const R* hin = A.heat_in.p;
    const double* scp = run.sc;
    LARE_BOXW(run, 3, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
      const int c = ix + sx * iy + sxy * iz;
      en[c] = en[c] + hin[c] * (R)scp[SC_DT] / rho[c];
    });
    energy_bcs(run);
  }
  if (run.p.use_viscous_damping) viscous_damping(run);
  // LP2: cs_v (:561-581)
  R* const cs_v = A.cs_v.p;
  LARE_BOXWH(run, 0, 4, 4, -1, nx + 1, -1, ny + 1, -1, nz + 1, [=] __device__(int ix, int iy, int iz) {
    const int c = ix + sx * iy + sxy * iz;
    const int o1 = 1, o2 = sx, o3 = 1 + sx, o4 = sxy, o5 = 1 + sxy, o6 = sx + sxy, o7 = 1 + sx + sxy;
    R s = cs[c] * cv[c] + cs[c + o1] * cv[c + o1] + cs[c + o2] * cv[c + o2] + cs[c + o3] * cv[c + o3] +
          cs[c + o4] * cv[c + o4] + cs[c + o5] * cv[c + o5] + cs[c + o6] * cv[c + o6] + cs[c + o7] * cv[c + o7];
    cs_v[c] = qdiv(R(0.125) * s, cv_v[c]);
  });
  // LP3: alpha1 (0:n+1, 0:n+2, 0:n+2), alpha2 (-1:n+1, 0:n+1, 0:n+2),
  // alpha3 (-1:n+1, -1:n+1, 0:n+1)
  const R* vx = A.vx.p;
  const R* vy = A.vy.p;
  const R* vz = A.vz.p;
  R* const alpha1 = A.alpha1.p;
  R* const alpha2 = A.alpha2.p;
  R* const alpha3 = A.alpha3.p;
  auto dxb = A.dxb, dyb = A.dyb, dzb = A.dzb, dxc = A.dxc, dyc = A.dyc, dzc = A.dzc;
  const R visc1 = (R)run.p.visc1;
  const double* sc = run.sc;
  LARE_BOXWH(run, 4, 2, 8, -1, nx + 1, -1, ny + 2, 0, nz + 2, [=] __device__(int ix, int iy, int iz) {
    const R dt = (R)sc[SC_DT], v2n = (R)sc[SC_VISC2N];
    const int c = ix + sx * iy + sxy * iz;
    auto edge = [&](const R* vcomp, int i1, int i2, R dx) {
      R dvdots = -(vcomp[i1] - vcomp[i2]);
      return edge_viscosity<R>(dvdots, rho_v[i1], rho_v[i2], cs_v[i1], cs_v[i2], vx[i1] - vx[i2], vy[i1] - vy[i2],
                               vz[i1] - vz[i2], dx, dt, visc1, v2n);
    };
    if (ix >= 0 && iy >= 0) alpha1[c] = edge(vx, c - 1 - sx - sxy, c - sx - sxy, dxb(ix));
    if (iy >= 0 && iy <= ny + 1) alpha2[c] = edge(vy, c - sx - sxy, c - sxy, dyb(iy));
    if (iy <= ny + 1 && iz <= nz + 1) alpha3[c] = edge(vz, c - sxy, c, dzb(iz));
  });
  // LP4: p_visc and visc_heat (0:n+1), viscous forces (0:n)
  R* const visc_heat = A.visc_heat.p;
  R* const fxv = A.fx_visc.p;
  R* const fyv = A.fy_visc.p;
  R* const fzv = A.fz_visc.p;
  {
    LP4Args<R> l4;
    l4.vx = vx;
    l4.vy = vy;
    l4.vz = vz;
    l4.alpha1 = alpha1;
    l4.alpha2 = alpha2;
    l4.alpha3 = alpha3;
    l4.cv = cv;
    l4.cv_v = cv_v;
    l4.p_visc = p_visc;
    l4.visc_heat = visc_heat;
    l4.fx = fxv;
    l4.fy = fyv;
    l4.fz = fzv;
    l4.dxb = dxb;
    l4.dyb = dyb;
    l4.dzb = dzb;
    l4.dxc = dxc;
    l4.dyc = dyc;
    l4.dzc = dzc;
    l4.nx = nx;
    l4.ny = ny;
    l4.nz = nz;
    l4.sx = sx;
    l4.sxy = sxy;
    const dim3 blk(kL4X, kL4Y, 1);
    const dim3 grd((nx + 2 + kL4X - 1) / kL4X, (ny + 2 + kL4Y - 1) / kL4Y, (nz + 2 + kL4Z - 1) / kL4Z);
    const int k = run.prof_begin("shock_viscosity_lp4_tile", 0, 13, (double)(nx + 2) * (ny + 2) * (nz + 2));
    k_lp4_tile<R><<<grd, blk, lp4_smem_bytes<R>(), run.s>>>(l4);
    run.prof_end(k);
    ++run.launches;
  }
}

// ---------------------------------------------------------------------
// lagran.F90:1070-1166 set_dt, on the device.
template <class R>
void set_dt(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  const int sx = run.sx, sxy = run.sxy;
  double* sc = run.sc;
  unsigned long long* us = run.us;
  if (run.set_dt_first) {
    run.set_dt_first = false;
    if (run.p.restart) {
      const double d = run.p.dt_from_restart;
      launch_scalar(run.s, run.launches, [=] __device__() {
        sc[SC_DT] = d;
        sc[SC_DT2] = 0.5 * d;
      });
      return;
    }
  }
  Arrays<R>& A = run.a;
  const R* bx = A.bx.p;
  const R* by = A.by.p;
  const R* bz = A.bz.p;
  const R* rho = A.rho.p;
  const R* pressure = A.pressure.p;
  const R* p_visc = A.p_visc.p;
  const R* vx = A.vx.p;
  const R* vy = A.vy.p;
  const R* vz = A.vz.p;
  const R* eta = A.eta.p;
  const R* eta_perp = A.eta_perp.p;
  R* const gamma_boris = A.gamma_boris.p;
  auto dxb = A.dxb, dyb = A.dyb, dzb = A.dzb;
  const bool boris = run.p.boris != 0, resistive = run.p.resistive_mhd != 0, cowling = run.cowling;
  const R g = (R)run.p.gamma;
  const R va_max2 = (R)run.p.va_max * (R)run.p.va_max;
  if (!run.gamma_boris_one || boris) {
    whole(run, [=] __device__(int i, int j, int k) {
      if (i >= -1 && j >= -1 && k >= -1) gamma_boris[i + sx * j + sxy * k] = R(1);
    });
    run.gamma_boris_one = !boris;
  }
  launch_scalar(run.s, run.launches, [=] __device__() {
    us[U_DTMIN] = (unsigned long long)__double_as_longlong(DBL_MAX);
    us[U_DTRMIN] = (unsigned long long)__double_as_longlong(DBL_MAX);
  });
  box_min<2>(run, "set_dt_min", 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz, double* v) {
    const int c = ix + sx * iy + sxy * iz;
    R w1 = bx[c] * bx[c] + by[c] * by[c] + bz[c] * bz[c];
    R rho0 = fmax(rho[c], Num<R>::tiny());
    const R dr = dv_of(rho0);
    R w2 = dv_div(w1, dr);
    R gb = gamma_boris[c];
    if (boris && (w2 >= va_max2)) {
      gb = qdiv(R(1), R(1) + qdiv(w2, va_max2));
      gamma_boris[c] = gb;
    }
    R cs2 = dv_div(g * pressure[c] + gb * w1, dr);
    R c_visc2 = dv_div(p_visc[c], dr);
    R length = fmin(fmin(dxb(ix), dyb(iy)), dzb(iz));
    R dt1 = qdiv(length, sqrt(c_visc2) + sqrt(cs2 + c_visc2));
    R dt_local = fmin(Num<R>::huge(), dt1);
    R dt2 = fmin(fmin(qdiv(dxb(ix), fmax(fabs(vx[c]), Num<R>::tiny())), qdiv(dyb(iy), fmax(fabs(vy[c]), Num<R>::tiny()))),
                 qdiv(dzb(iz), fmax(fabs(vz[c]), Num<R>::tiny())));
    dt_local = fmin(dt_local, dt2);
    R dt3 = Num<R>::huge();
    if (cowling || resistive) {  // lagran.F90:1132-1134 (Cowling), :1136-1138
      const R dxlocal =
          qdiv(R(1), qdiv(R(1), dxb(ix) * dxb(ix)) + qdiv(R(1), dyb(iy) * dyb(iy)) + qdiv(R(1), dzb(iz) * dzb(iz)));
      const R e = cowling ? fmax(eta[c], eta_perp[c]) : eta[c];
      dt3 = qdiv(R(0.2) * dxlocal, fmax(e, Num<R>::tiny()));
    }
    v[0] = (double)dt_local;
    v[1] = (double)dt3;
  }, U_DTMIN, cowling ? 11 : (resistive ? 10 : 9));
  const double mult = run.p.dt_multiplier;
  const bool f32 = sizeof(R) == 4;
  launch_scalar(run.s, run.launches, [=] __device__() {
    double dtm = __longlong_as_double((long long)us[U_DTMIN]);
    double dtrm = __longlong_as_double((long long)us[U_DTRMIN]);
    if (f32) {
      dtm = fmin(dtm, (double)FLT_MAX);
      dtrm = fmin(dtrm, (double)FLT_MAX);
    }
    sc[SC_DT] = mult * dtm;
    sc[SC_DTR] = mult * dtrm;
  });
  if (run.p.conduction) {
    calc_s_stages(run, SC_DT);
    launch_scalar(run.s, run.launches, [=] __device__() {
      const double ss_limit = 60;
      int ns = (int)sc[SC_STAGES];
      if (ns >= ss_limit) {
        double f1 = 2.0 * ss_limit * ss_limit - 9.0;
        double f2 = (double)(2 * ns * ns - 9);
        sc[SC_DT] = sc[SC_DT] * f1 / f2;
        sc[SC_DTR] = sc[SC_DTR] * f1 / f2;
      }
    });
  }
  launch_scalar(run.s, run.launches, [=] __device__() {
    sc[SC_TIME] = sc[SC_TIME] + sc[SC_DT];
    sc[SC_DT2] = 0.5 * sc[SC_DT];
  });
}

// ---------------------------------------------------------------------
// The predictor's B-only remap (b_field_and_cv1_update, lagran.F90:1050-
// 1060): B * area is written to the bx0 buffers, which then serve as B for
// the three half-dt sweeps, the back-conversion and bfield_bcs.  On return
// run.a.bx holds the predicted B and run.a.bx0 the untouched B of the step.
template <class R>
void predictor_remap(Run<R>& run, int step) {
  Arrays<R>& A = run.a;
  // B -> flux form (remap.f90:43-69, into the B0 buffers, which are then
  // swapped in so that B itself is kept as B0) and back (:101-127) are done
  // by the first and last sweeps' B kernels on the way (remap_sweep's bmode).
  // vx1 = vx (lagran.F90:1051-1053): the sweeps read v itself.  vx1's own
  // nodes 0:n are rewritten by the predictor force and its ghosts by
  // remap_v_bcs, except on an open side: there the copy's ghost values are
  // carried into the vx1 buffer.
  R* const keep[3] = {A.vx1.p, A.vy1.p, A.vz1.p};
  {
    R* const ov[3] = {A.vx.p, A.vy.p, A.vz.p};
    carry_velocity(run, keep, ov);
  }
  A.vx1.p = A.vx.p;
  A.vy1.p = A.vy.p;
  A.vz1.p = A.vz.p;
  static const int order[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {0, 2, 1}, {2, 1, 0}, {1, 0, 2}};
  int cse = ((step % 6) + 6) % 6;
  int pass[3] = {1, 1, 1};
  for (int s = 0; s < 3; ++s) {
    const int bmode = s == 0 ? 1 : (s == 2 ? 2 : 0);
    switch (order[cse][s]) {
      case 0: remap_sweep<0>(run, true, SC_DT2, pass, bmode); break;
      case 1: remap_sweep<1>(run, true, SC_DT2, pass, bmode); break;
      default: remap_sweep<2>(run, true, SC_DT2, pass, bmode); break;
    }
  }
  A.vx1.p = keep[0];
  A.vy1.p = keep[1];
  A.vz1.p = keep[2];
  bfield_bcs(run);
}

// PC3 (shock_heating, lagran.F90:396-458, and v = 2 v1 - v) as a tiled
// z-march: a CTA of 32 x 8 threads owns 32 x 8 cells and walks a chunk of z
// with the corner planes z-1 and z of the six velocity arrays (v and v1,
// with a one-vertex halo below in x and y) in shared memory; plane z+1 is
// loaded into registers while plane z is computed.  The twelve edge terms of
// cell (x, y, z) join the four corners of plane z-1 (c-Z, c-X-Z, c-Y-Z,
// c-X-Y-Z) and of plane z (c, c-X, c-Y, c-X-Y); the four plane z-1 edges are
// the previous cell's plane z edges and are carried, and alpha1 and alpha2
// at c+Z, c+Y+Z, c-X+Z are the next cell's c, c+Y, c-X.  Each velocity is
// read from memory about once per CTA, and no thread holds a window of
// corner values (a register-window march needed 130 registers and ran
// 0.59-0.64 ms against 0.55 ms at 256^3 in FP64, 0.33 against 0.30 ms in
// FP32).  Same expressions, same operands, same results bit for bit.
constexpr int kShockZ = 32;

template <class R>
struct ShockArgs {
  const R* v[6];  // vx, vy, vz, vx1, vy1, vz1
  const R* alpha1;
  const R* alpha2;
  const R* alpha3;
  const R* cv;
  R* vhp;
  R* nv[3];
  A1<R> dxb, dyb, dzb;
  int nx, ny, nz, sx, sxy;
};

constexpr int kShX = 32, kShY = 8;
constexpr int kShW = kShX + 1, kShP = kShW * (kShY + 1);  // plane row and size

template <class R>
__global__ void __launch_bounds__(kShX * kShY, sizeof(R) == 8 ? 2 : 4) k_shock_tile(ShockArgs<R> g) {
  __shared__ R Vs[2][6][kShP];  // [plane slot][array][element]
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kShX + tx;
  const int ix0 = blockIdx.x * kShX, iy0 = blockIdx.y * kShY;
  const int ix = ix0 + tx, iy = iy0 + ty;
  const int z0 = (int)blockIdx.z * kShockZ;
  const int z1 = min(z0 + kShockZ - 1, g.nz + 1);
  const int sx = g.sx, sxy = g.sxy;
  const bool cell = ix <= g.nx + 1 && iy <= g.ny + 1;
  // the plane elements this thread loads (vertex x in ix0-1..ix0+31, y in
  // iy0-1..iy0+7, clamped to the array: clamped values are never used)
  int off[2];
  bool has[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int e = tid + q * kShX * kShY;
    has[q] = e < kShP;
    const int jj = has[q] ? e / kShW : 0, ii = has[q] ? e - jj * kShW : 0;
    off[q] = min(ix0 - 1 + ii, g.nx + 2) + sx * min(iy0 - 1 + jj, g.ny + 2);
  }
  R nxt[6][2];  // plane k's elements, in flight
  auto fetch = [&](int k) {
#pragma unroll
    for (int m = 0; m < 6; ++m)
#pragma unroll
      for (int q = 0; q < 2; ++q)
        if (has[q]) nxt[m][q] = __ldg(g.v[m] + off[q] + sxy * k);
  };
  auto stash = [&](int k) {
#pragma unroll
    for (int m = 0; m < 6; ++m)
#pragma unroll
      for (int q = 0; q < 2; ++q)
        if (has[q]) Vs[k & 1][m][tid + q * kShX * kShY] = nxt[m][q];
  };
  const int e = (ty + 1) * kShW + tx + 1;  // corner c of this thread's cell in a plane slot
  const int oc[4] = {0, -1, -kShW, -1 - kShW};  // corners c, c-X, c-Y, c-X-Y
  // dd of two corners (slot, corner): the components' dv * dv1 summed in order
  auto dd = [&](int s1, int i, int s2, int j) {
    const int p = e + oc[i], r = e + oc[j];
    return (Vs[s1][0][p] - Vs[s2][0][r]) * (Vs[s1][3][p] - Vs[s2][3][r]) +
           (Vs[s1][1][p] - Vs[s2][1][r]) * (Vs[s1][4][p] - Vs[s2][4][r]) +
           (Vs[s1][2][p] - Vs[s2][2][r]) * (Vs[s1][5][p] - Vs[s2][5][r]);
  };
  fetch(z0 - 1);
  stash(z0 - 1);
  fetch(z0);
  __syncthreads();
  const int sl0 = (z0 - 1) & 1;
  // plane z0-1 edges: a1 = (c-X-Y-Z, c-Y-Z), a2 = (c-Y-Z, c-Z), a3 = (c-Z, c-X-Z), a4 = (c-X-Z, c-X-Y-Z)
  R a1 = dd(sl0, 3, sl0, 2), a2 = dd(sl0, 2, sl0, 0), a3 = dd(sl0, 0, sl0, 1), a4 = dd(sl0, 1, sl0, 3);
  int c = min(ix, g.nx + 1) + sx * min(iy, g.ny + 1) + sxy * z0;
  R al1 = g.alpha1[c], al1y = g.alpha1[c + sx], al2 = g.alpha2[c], al2x = g.alpha2[c - 1];
  const R ddx = g.dxb(min(ix, g.nx + 1)), ddy = g.dyb(min(iy, g.ny + 1));
  for (int iz = z0; iz <= z1; ++iz, c += sxy) {
    stash(iz);  // its slot held plane iz - 2, last read before the previous barrier
    if (iz < z1) fetch(iz + 1);
    __syncthreads();
    const int su = iz & 1, sl = su ^ 1;
    const R a5 = dd(su, 3, su, 2);   // (c-X-Y, c-Y)
    const R a6 = dd(su, 2, su, 0);   // (c-Y, c)
    const R a7 = dd(su, 0, su, 1);   // (c, c-X)
    const R a8 = dd(su, 1, su, 3);   // (c-X, c-X-Y)
    const R a9 = dd(sl, 0, su, 0);   // (c-Z, c)
    const R a10 = dd(sl, 1, su, 1);  // (c-X-Z, c-X)
    const R a11 = dd(sl, 3, su, 3);  // (c-X-Y-Z, c-X-Y)
    const R a12 = dd(sl, 2, su, 2);  // (c-Y-Z, c-Y)
    const R al1z = g.alpha1[c + sxy], al1yz = g.alpha1[c + sx + sxy];
    const R al2z = g.alpha2[c + sxy], al2xz = g.alpha2[c - 1 + sxy];
    if (cell) {
      const R ddz = g.dzb(iz);
      const R vh = -R(0.25) * ddy * ddz * al1 * a1 - R(0.25) * ddx * ddz * al2 * a2 -
                   R(0.25) * ddy * ddz * al1y * a3 - R(0.25) * ddx * ddz * al2x * a4 -
                   R(0.25) * ddy * ddz * al1z * a5 - R(0.25) * ddx * ddz * al2z * a6 -
                   R(0.25) * ddy * ddz * al1yz * a7 - R(0.25) * ddx * ddz * al2xz * a8 -
                   R(0.25) * ddx * ddy * g.alpha3[c] * a9 - R(0.25) * ddx * ddy * g.alpha3[c - 1] * a10 -
                   R(0.25) * ddx * ddy * g.alpha3[c - 1 - sx] * a11 - R(0.25) * ddx * ddy * g.alpha3[c - sx] * a12;
      const R v = qdiv(vh, g.cv[c]);
      g.vhp[c] = v > R(0) ? v : R(0);
      if (ix <= g.nx && iy <= g.ny && iz <= g.nz) {
#pragma unroll
        for (int k = 0; k < 3; ++k) g.nv[k][c] = R(2) * Vs[su][k + 3][e] - Vs[su][k][e];
      }
    }
    a1 = a5;
    a2 = a6;
    a3 = a7;
    a4 = a8;
    al1 = al1z;
    al1y = al1yz;
    al2 = al2z;
    al2x = al2xz;
    __syncthreads();
  }
}

// ---------------------------------------------------------------------
// lagran.F90:208-478 predictor_corrector_step (non-CAUCHY, no cooling),
// including the energy0 + delta_energy / MAX(energy, 0) of :180-181.
template <class R>
void predictor_corrector_step(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  const int sx = run.sx, sxy = run.sxy;
  Arrays<R>& A = run.a;
  predictor_remap(run, run.cur_step);
  // PC1 (-1:n+2): energy = MAX(energy0 + delta, 0); predictor pressure (0:n+1)
  R* const energy = A.energy.p;
  const R* energy0 = A.energy0.p;
  R* const pressure = A.pressure.p;
  const R* cv1 = A.cv1.p;
  const R* cv = A.cv.p;
  const R* rho = A.rho.p;
  const R* visc_heat = A.visc_heat.p;
  const bool cond = run.p.conduction != 0;
  const R* erad = run.p.radiation ? A.erad.p : nullptr;  // the energy after rad_losses
  const R g = (R)run.p.gamma, xi = (R)run.p.xi_n, ip = (R)run.p.ionise_pot;
  const R* xin = run.pip ? A.xi.p : nullptr;
  const double* sc = run.sc;
  LARE_BOXWH(run, 0, 4, 8, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
    const int c = ix + sx * iy + sxy * iz;
    R e;
    if (cond) {
      R e0 = energy0[c];
      R d = energy[c] - e0;
      if (erad) d = d + (erad[c] - e0);
      e = e0 + d;
    } else if (erad) {
      R e0 = energy[c];
      R d = R(0) + (erad[c] - e0);
      e = e0 + d;
    } else {
      e = energy[c] + R(0);
    }
    e = e > R(0) ? e : R(0);
    energy[c] = e;
    if (ix >= 0 && ix <= nx + 1 && iy >= 0 && iy <= ny + 1 && iz >= 0 && iz <= nz + 1) {
      const R dt2 = (R)sc[SC_DT2];
      const R rr = dv_of(rho[c]);
      R dv = qdiv(cv1[c], cv[c]) - R(1);
      R e1 = e - dv_div(pressure[c] * dv, rr);
      e1 = e1 + dv_div(visc_heat[c] * dt2, rr);
      const R x = xin ? xin[c] : xi;
      pressure[c] = qdiv((e1 - (R(1) - x) * ip) * (g - R(1)) * rho[c] * cv[c], cv1[c]);
    }
  });
  // PC2 (0:n): vertex forces with the predicted B; half-step velocity
  const R* bx = A.bx.p;  // predicted B
  const R* by = A.by.p;
  const R* bz = A.bz.p;
  const R* gamma_boris = A.gamma_boris.p;
  const R* rho_v = A.rho_v.p;
  R* const vx = A.vx.p;
  R* const vy = A.vy.p;
  R* const vz = A.vz.p;
  R* const vx1 = A.vx1.p;
  R* const vy1 = A.vy1.p;
  R* const vz1 = A.vz1.p;
  const R* fxv = A.fx_visc.p;
  const R* fyv = A.fy_visc.p;
  const R* fzv = A.fz_visc.p;
  auto dxc = A.dxc, dyc = A.dyc, dzc = A.dzc, grav = A.grav;
  auto rdcx = A.rdc[0], rdcy = A.rdc[1], rdcz = A.rdc[2];
  LARE_BOXWH(run, 5, 4, 17, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz) {
    const R dt2 = (R)sc[SC_DT2];
    const int c = ix + sx * iy + sxy * iz;
    const int X = 1, Y = sx, Z = sxy;
    R pp = pressure[c], ppx = pressure[c + X], ppy = pressure[c + Y];
    R ppz = pressure[c + Z], ppxy = pressure[c + X + Y], ppxz = pressure[c + X + Z];
    R ppyz = pressure[c + Y + Z], ppxyz = pressure[c + X + Y + Z];
    R w1 = (pp + ppy + ppz + ppyz) * R(0.25);
    R w2 = (ppx + ppxy + ppxz + ppxyz) * R(0.25);
    R fx = -div_rcp(w2 - w1, dxc(ix), rdcx(ix));
    w1 = (pp + ppx + ppz + ppxz) * R(0.25);
    w2 = (ppy + ppxy + ppyz + ppxyz) * R(0.25);
    R fy = -div_rcp(w2 - w1, dyc(iy), rdcy(iy));
    w1 = (pp + ppx + ppy + ppxy) * R(0.25);
    w2 = (ppz + ppxz + ppyz + ppxyz) * R(0.25);
    R fz = -div_rcp(w2 - w1, dzc(iz), rdcz(iz));
    R bxv = R(0.25) * (bx[c] + bx[c + Y] + bx[c + Z] + bx[c + Y + Z]);
    R byv = R(0.25) * (by[c] + by[c + X] + by[c + Z] + by[c + X + Z]);
    R bzv = R(0.25) * (bz[c] + bz[c + Y] + bz[c + X] + bz[c + X + Y]);
    R jx, jy, jz;
    vertex_current<R, true>(bx, by, bz, c, sx, sxy, dxc(ix), dyc(iy), dzc(iz), rdcx(ix), rdcy(iy), rdcz(iz), jx,
                            jy, jz);
    R gb = gamma_boris[c];
    fx = fx + gb * (jy * bzv - jz * byv);
    fy = fy + gb * (jz * bxv - jx * bzv);
    fz = fz + gb * (jx * byv - jy * bxv);
    R rv = rho_v[c];
    fz = fz - rv * grav(iz);
    const R drv = dv_of(rv);
    vx1[c] = vx[c] + dv_div(dt2 * (fxv[c] + fx), drv);
    vy1[c] = vy[c] + dv_div(dt2 * (fyv[c] + fy), drv);
    vz1[c] = vz[c] + dv_div(dt2 * (fzv[c] + fz), drv);
  });
  // B = B0 (:389-393)
  std::swap(A.bx.p, A.bx0.p);
  std::swap(A.by.p, A.by0.p);
  std::swap(A.bz.p, A.bz0.p);
  remap_v_bcs(run);
  // PC3: shock_heating (0:n+1) and v = 2 v1 - v (0:n) into the q buffers
  const R* alpha1 = A.alpha1.p;
  const R* alpha2 = A.alpha2.p;
  const R* alpha3 = A.alpha3.p;
  R* const vhp = A.visc_heat.p;
  R* const nvx = A.qx.p;
  R* const nvy = A.qy.p;
  R* const nvz = A.qz.p;
  auto dxb = A.dxb, dyb = A.dyb, dzb = A.dzb;
  {
    ShockArgs<R> ga;
    const R* vs[6] = {vx, vy, vz, vx1, vy1, vz1};
    for (int k = 0; k < 6; ++k) ga.v[k] = vs[k];
    ga.alpha1 = alpha1;
    ga.alpha2 = alpha2;
    ga.alpha3 = alpha3;
    ga.cv = cv;
    ga.vhp = vhp;
    ga.nv[0] = nvx;
    ga.nv[1] = nvy;
    ga.nv[2] = nvz;
    ga.dxb = dxb;
    ga.dyb = dyb;
    ga.dzb = dzb;
    ga.nx = nx;
    ga.ny = ny;
    ga.nz = nz;
    ga.sx = sx;
    ga.sxy = sxy;
    dim3 blk(kShX, kShY, 1);
    dim3 grd((nx + 2 + kShX - 1) / kShX, (ny + 2 + kShY - 1) / kShY, (nz + 2 + kShockZ - 1) / kShockZ);
    const int k = run.prof_begin("shock_heating", 0, 14, (double)(nx + 2) * (ny + 2) * (nz + 2));
    k_shock_tile<R><<<grd, blk, 0, run.s>>>(ga);
    run.prof_end(k);
    ++run.launches;
  }
  std::swap(A.vx.p, A.qx.p);
  std::swap(A.vy.p, A.qy.p);
  std::swap(A.vz.p, A.qz.p);
  {
    R* const nv[3] = {A.vx.p, A.vy.p, A.vz.p};
    R* const ov[3] = {A.qx.p, A.qy.p, A.qz.p};
    carry_velocity(run, nv, ov);
  }
  velocity_bcs(run);
  open_bcs(run);  // lagran.F90:410-412 (no launch unless a side is open)
  // PC4 (1:n): final cv1, energy, visc_dep, rho; total_visc_heating
  R* const cv1w = A.cv1.p;
  R* const rhow = A.rho.p;
  R* const visc_dep = A.visc_dep.p;
  const A1<R> rbx = A.rdb[0], rby = A.rdb[1], rbz = A.rdb[2];
  box_sum<1>(run, "corrector_visc_heating_sum", 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz, double* v) {
    const R dt = (R)sc[SC_DT];
    const int c = ix + sx * iy + sxy * iz;
    const int X = 1, Y = sx, Z = sxy;
    R vxb = (vx1[c] + vx1[c - Y] + vx1[c - Z] + vx1[c - Y - Z]) * R(0.25);
    R vxbm = (vx1[c - X] + vx1[c - X - Y] + vx1[c - X - Z] + vx1[c - X - Y - Z]) * R(0.25);
    R vyb = (vy1[c] + vy1[c - X] + vy1[c - Z] + vy1[c - X - Z]) * R(0.25);
    R vybm = (vy1[c - Y] + vy1[c - X - Y] + vy1[c - Y - Z] + vy1[c - X - Y - Z]) * R(0.25);
    R vzb = (vz1[c] + vz1[c - X] + vz1[c - Y] + vz1[c - X - Y]) * R(0.25);
    R vzbm = (vz1[c - Z] + vz1[c - X - Z] + vz1[c - Y - Z] + vz1[c - X - Y - Z]) * R(0.25);
#if LARE_FAST
    R dv = ((vxb - vxbm) * rbx(ix) + (vyb - vybm) * rby(iy) + (vzb - vzbm) * rbz(iz)) * dt;
#else
    R dv = ((vxb - vxbm) / dxb(ix) + (vyb - vybm) / dyb(iy) + (vzb - vzbm) / dzb(iz)) * dt;
#endif
    cv1w[c] = cv[c] * (R(1) + dv);
    R vh = vhp[c];
    R r = rhow[c];
    energy[c] = energy[c] + qdiv(dt * vh - dv * pressure[c], r);
    visc_dep[c] = visc_dep[c] + dt * vh;
    rhow[c] = qdiv(r, R(1) + dv);
    v[0] = (double)(dt * vh * cv[c]);
  }, SC_VISC_TOT, true, 13);
  if (run.p.cooling_term) {
    // :464-475: an exponential moving average of the viscous heating
    // (weight alpha_av) is taken off the energy of cells 1:n, then
    // energy = MAX(energy, 0) over the whole array
    R* const ctv = A.cool_term_v.p;
    const R* vhp2 = A.visc_heat.p;
    const R* rho2 = A.rho.p;
    R* const en = A.energy.p;
    const R alpha = (R)run.p.alpha_av;
    LARE_BOXW(run, 5, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
      const int c = ix + sx * iy + sxy * iz;
      R e = en[c];
      if (ix >= 1 && ix <= nx && iy >= 1 && iy <= ny && iz >= 1 && iz <= nz) {
        const R dt = (R)sc[SC_DT];
        const R t = alpha * dt * vhp2[c] / rho2[c] + (R(1) - alpha) * ctv[c];
        ctv[c] = t;
        e = e - t;
      }
      en[c] = e > R(0) ? e : R(0);
    });
  }
}

// ---------------------------------------------------------------------
// lagran.F90:147-148 in each resistive sub-cycle, after eta_calc (which
// reads neither result, so it may follow them here, fused with rkstep).
template <class R>
void neutral_models(Run<R>& run) {
  if (run.pip) neutral_fraction(run, run.a.energy);
  if (run.cowling) perpendicular_resistivity(run);
}

// ---------------------------------------------------------------------
// lagran.F90:135-150, the resistive sub-cycles, recorded into a CUDA graph:
// the count is known only on the device, so the loop is a conditional WHILE
// node whose body (eta + rkstep, bstep, ohmic heating) ends with a kernel
// that counts down and sets the loop condition.  A bad dt sets sc[SC_ERROR]
// and skips the loop; the host reads the flag after the graph has run.
template <class R>
int resistive_subcycles_captured(Run<R>& run) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  if (cudaStreamGetCaptureInfo(run.s, &st, nullptr, &g, &deps, &nd) != cudaSuccess ||
      st != cudaStreamCaptureStatusActive)
    return LARE_ECUDA;
  cudaGraphConditionalHandle h;
  if (cudaGraphConditionalHandleCreate(&h, g, 0, 0) != cudaSuccess) return LARE_ECUDA;
  double* sc = run.sc;
  launch_scalar(run.s, run.launches, [=] __device__() {
    const double dt = sc[SC_DT];
    const double q = dt / sc[SC_DTR];
    int substeps = 0;
    if (dt > 0.0 && isfinite(dt) && q >= 0.0 && q < 99999.0) {  // at most 1e5 device-side cycles
      substeps = (int)q + 1;
      sc[SC_DTSUB] = dt / (double)substeps;
    } else {
      sc[SC_ERROR] = (double)LARE_EDT;
    }
    sc[SC_SUBSTEPS] = (double)substeps;
    sc[SC_LOOP] = (double)substeps;
    cudaGraphSetConditional(h, substeps > 0 ? 1u : 0u);
  });
  if (cudaStreamGetCaptureInfo(run.s, &st, nullptr, &g, &deps, &nd) != cudaSuccess) return LARE_ECUDA;
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if (cudaGraphAddNode(&node, g, deps, nd, &cp) != cudaSuccess) return LARE_ECUDA;
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  if (cudaStreamBeginCaptureToGraph(run.s_body, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
      cudaSuccess)
    return LARE_ECUDA;
  cudaStream_t outer = run.s;
  run.s = run.s_body;
  neutral_models(run);
  eta_and_rkstep(run, true);
  resistive_update(run);
  {
    // bstep swapped the B buffers on the host, but the body replays with
    // the pointers it was recorded with: copy the new B back into the
    // buffers the body reads and restore the pointers, so every pass starts
    // from the previous pass's field.
    Arrays<R>& A = run.a;
    for (A3<R>* b : {&A.bx, &A.by, &A.bz}) {
      A3<R>& o = b == &A.bx ? A.bx1 : (b == &A.by ? A.by1 : A.bz1);
      copy_whole(run, o, *b);
      std::swap(b->p, o.p);
    }
  }
  launch_scalar(run.s, run.launches, [=] __device__() {
    const double left = sc[SC_LOOP] - 1.0;
    sc[SC_LOOP] = left;
    cudaGraphSetConditional(h, left > 0.5 ? 1u : 0u);
  });
  run.s = outer;
  cudaGraph_t captured = nullptr;
  if (cudaStreamEndCapture(run.s_body, &captured) != cudaSuccess) return LARE_ECUDA;
  if (cudaStreamUpdateCaptureDependencies(run.s, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
    return LARE_ECUDA;
  return LARE_OK;
}

// ---------------------------------------------------------------------
// lagran.F90:50-200 lagrangian_step
template <class R>
int lagrangian_step(Run<R>& run, int step) {
  run.cur_step = step;
  prologue_and_shock_viscosity(run);
  set_dt(run);
  double* sc = run.sc;
  run.last_substeps = 0;
  if (run.p.resistive_mhd && run.capturing) {
    int rc = resistive_subcycles_captured(run);
    if (rc) return rc;
  } else if (run.p.resistive_mhd) {
    launch_scalar(run.s, run.launches, [=] __device__() {
      double dt = sc[SC_DT];
      int substeps = (int)(dt / sc[SC_DTR]) + 1;
      sc[SC_SUBSTEPS] = (double)substeps;
      sc[SC_DTSUB] = dt / (double)substeps;
    });
    if (pull_scalars(run) != cudaSuccess) return LARE_ECUDA;
    int substeps = (int)run.host_sc[SC_SUBSTEPS];
    double dtv = run.host_sc[SC_DT];
    if (!(dtv > 0.0) || !std::isfinite(dtv)) return LARE_EDT;
    if (substeps < 1 || substeps > 1000000) return LARE_EDT;
    if (substeps > run.peak_substeps) run.peak_substeps = substeps;
    run.last_substeps = substeps;
    for (int i = 1; i <= substeps; ++i) {
      neutral_models(run);
      eta_and_rkstep(run, true);
      resistive_update(run);
    }
    // The cell B averages recomputed at :152-163 only feed the CAUCHY branch.
  }
  if (run.p.conduction) {
    if (run.capturing) return LARE_EINVAL;  // the stage count and coefficients are host-side
    copy_whole(run, run.a.energy0, run.a.energy);
    calc_s_stages(run, SC_DT);
    if (pull_scalars(run) != cudaSuccess) return LARE_ECUDA;
    int ns = (int)run.host_sc[SC_STAGES];
    if (ns < 1 || ns > 100000) return LARE_ESTAGES;
    run.n_s_stages = ns;
    heat_conduct_sts2(run, SC_DT);
  }
  // lagran.F90:174-178: rad_losses on the energy before conduction (energy0
  // when conduction ran, else the energy itself); PC1 adds the two deltas
  if (run.p.radiation) rad_losses(run, run.a.erad, run.p.conduction ? run.a.energy0 : run.a.energy, SC_DT);
  predictor_corrector_step(run);
  end_of_step_bcs(run);
  ++run.steps_taken;
  return LARE_OK;
}

LARE_END  // namespace lare
