// engine.cuh - the Lagrangian-remap timestep on the device.
//
// Each routine below corresponds to a routine of the reference (file:line
// cited) and launches one kernel per reference loop nest over exactly the
// same index box, with the same left-to-right expression order.  Compiled
// with --fmad=false for FP64 (engine_f64.cu) the arithmetic is then
// bit-for-bit that of a gfortran -O3 x86-64 build of the reference, which
// emits no FMA; pow() (conduction only) is the one call whose last bit may
// differ.  engine_f32.cu instantiates the same code in FP32 (the FP32 form).
//
// All routines are free functions over Run<R>&; kernels capture only local
// copies of array handles and scalars (a capture of `run` itself fails to
// compile under -Werror cross-execution-space-call because Run owns a
// std::string).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/lare_gpu.h"
#include "common.cuh"

namespace lare {

struct Par {
  double gamma, visc1, visc2, eta_background, eta0, j_max, kappa_0, flux_limiter;
  double ionise_pot, xi_n, va_max, dt_multiplier, dt_from_restart, kappa_perp_ratio;
  int resistive_mhd, conduction, heat_flux_limiter, use_viscous_damping, boris, restart;
  int bc[3][2];   // [dim][0=min,1=max]
  bool per[3];    // periodic communicator in this dimension (mpi_routines.F90:195-210)
};

template <class R>
struct Arrays {
  // persistent
  A3<R> rho, energy, temperature, eta, cv, cv1, p_visc, visc_dep, ohmic_dep, gamma_boris;
  A3<R> vx, vy, vz, vx1, vy1, vz1, visc3, bx, by, bz;
  // lagran.F90 temporaries
  A3<R> bx0, by0, bz0, bx1, by1, bz1, alpha1, alpha2, alpha3, visc_heat, pressure, rho_v, cv_v;
  A3<R> flux_x, flux_y, flux_z, curlb, fx_visc, fy_visc, fz_visc, qx, qy, qz, energy0, cs, cs_v;
  // [xyz]remap.f90 temporaries (f1, f2: the two B fluxes; rho_alt: second
  // density buffer; cv1v, cv2v, dmv: vertex averages; mf?: momentum fluxes)
  A3<R> db1, dc1, r_rho_v, r_rho_v1, rho1, dm, cv2, flux;
  A3<R> f1, f2, rho_alt, cv1v, cv2v, dmv, mfx, mfy, mfz;
  // conduct.f90 temporaries
  A3<R> larsen, c_flux, Y0, Y1, Y2, Y3, Lc_Y0;
  // 1-D metrics (pointers at Fortran index 0)
  A1<R> dxb, dxc, dyb, dyc, dzb, dzc, grav;
};

enum Stag { ST_C = 0, ST_N = 1, ST_F = 2 };

// Per-launch-site timing (instrumentation, off by default).  A site is a
// launch statement (function, line); `words` is the number of distinct 3-D
// arrays it reads plus writes, so bytes = words * points * sizeof(R).
struct ProfSite {
  const char* func;
  int line;
  int words;
  long long count = 0;
  double ms = 0.0, bytes = 0.0;
};
struct Prof {
  bool on = false;
  std::vector<cudaEvent_t> ev;
  size_t used = 0;
  std::vector<int> ev_site;          // per event pair
  std::vector<double> ev_bytes;
  std::map<std::pair<const char*, int>, int> index;
  std::vector<ProfSite> sites;
};

template <class R>
struct Run {
  Par p;
  int n[3];
  int sx, sxy, ntot;    // padded box
  size_t elems;         // elements per array
  Arrays<R> a;
  double* sc = nullptr;             // device scalar slots (Slot)
  unsigned long long* us = nullptr; // device min-reduction slots (USlot)
  double* partial = nullptr;        // block partial sums
  size_t partial_cap = 0;
  double* host_sc = nullptr;        // pinned mirror of sc
  cudaStream_t s = nullptr;
  long long launches = 0;
  std::vector<void*> allocations;
  bool visc2_norm_set = false;      // lagran.F90:539 first_call (SAVE)
  bool set_dt_first = true;         // lagran.F90:1078 first (SAVE)
  bool gamma_boris_one = true;      // gamma_boris holds 1 everywhere
  int cur_step = 0;
  int peak_substeps = 0, last_substeps = 0, steps_taken = 0, n_s_stages = 0;
  GSpec g_cell, g_node, g_bx, g_by, g_bz, g_cell_mpi, g_cell_user, g_dm[3];
  Prof prof;
  std::string err;

  // Bracket one launch with events when profiling.
  int prof_begin(const char* func, int line, int words, double points) {
    if (!prof.on) return -1;
    auto key = std::make_pair(func, line);
    auto it = prof.index.find(key);
    int site;
    if (it == prof.index.end()) {
      site = (int)prof.sites.size();
      prof.index[key] = site;
      ProfSite ps;
      ps.func = func;
      ps.line = line;
      ps.words = words;
      prof.sites.push_back(ps);
    } else {
      site = it->second;
    }
    size_t k = prof.used;
    while (prof.ev.size() < 2 * (k + 1)) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      prof.ev.push_back(e);
    }
    prof.ev_site.resize(k + 1);
    prof.ev_bytes.resize(k + 1);
    prof.ev_site[k] = site;
    prof.ev_bytes[k] = (double)words * points * (double)sizeof(R);
    cudaEventRecord(prof.ev[2 * k], s);
    return (int)k;
  }
  void prof_end(int k) {
    if (k < 0) return;
    cudaEventRecord(prof.ev[2 * k + 1], s);
    prof.used = k + 1;
  }
  // Fold recorded events into the per-site totals.
  void prof_collect() {
    cudaStreamSynchronize(s);
    for (size_t k = 0; k < prof.used; ++k) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, prof.ev[2 * k], prof.ev[2 * k + 1]);
      ProfSite& ps = prof.sites[prof.ev_site[k]];
      ps.ms += ms;
      ps.count += 1;
      ps.bytes += prof.ev_bytes[k];
    }
    prof.used = 0;
  }
};

// ---------------------------------------------------------------------
// Launch shorthands
template <class R, class Fn>
inline void rbox(Run<R>& run, const char* func, int line, int words, int i0, int i1, int j0, int j1, int k0, int k1,
                 Fn fn) {
  double pts = (double)(i1 - i0 + 1) * (double)(j1 - j0 + 1) * (double)(k1 - k0 + 1);
  int k = run.prof_begin(func, line, words, pts);
  launch_box(run.s, run.launches, i0, i1, j0, j1, k0, k1, fn);
  run.prof_end(k);
}
// LARE_BOX: one kernel over an inclusive Fortran index box.  LARE_BOXW also
// states the kernel's algorithmic word count per point (arrays read +
// written), used for the roofline of profiled launches.
#define LARE_BOX(run, i0, i1, j0, j1, k0, k1, ...) \
  rbox((run), __func__, __LINE__, 0, (i0), (i1), (j0), (j1), (k0), (k1), __VA_ARGS__)
#define LARE_BOXW(run, words, i0, i1, j0, j1, k0, k1, ...) \
  rbox((run), __func__, __LINE__, (words), (i0), (i1), (j0), (j1), (k0), (k1), __VA_ARGS__)

template <class R>
inline void ghost(Run<R>& run, const GSpec& g, A3<R> a, A3<R>* b = nullptr, A3<R>* c = nullptr) {
  long long tot = g.c0 + g.c1 + g.c2;
  if (tot <= 0) return;
  int blocks = (int)((tot + 255) / 256);
  int narr = 1 + (b ? 1 : 0) + (c ? 1 : 0);
  int k = run.prof_begin("ghost", 0, 2 * narr, (double)tot);
  k_ghost<R><<<blocks, 256, 0, run.s>>>(g, a.p, b ? b->p : nullptr, c ? c->p : nullptr, run.sx, run.sxy);
  run.prof_end(k);
  ++run.launches;
}

// Deterministic sum of NV values over a box, into sc[slot..] (+=).
template <int NV, class R, class Fn>
inline void box_sum(Run<R>& run, int i0, int i1, int j0, int j1, int k0, int k1, Fn fn, int slot, bool acc) {
  int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
  dim3 blk(64, 4, 1);
  dim3 grd((ni + 63) / 64, (nj + 3) / 4, nk);
  int nb = grd.x * grd.y * grd.z;
  int k = run.prof_begin("box_sum", 0, 0, (double)ni * nj * nk);
  k_box_sum<NV><<<grd, blk, 0, run.s>>>(i0, j0, k0, ni, nj, fn, run.partial);
  k_sum_partials<NV><<<1, 1024, 0, run.s>>>(run.partial, nb, run.sc + slot, acc ? 1 : 0);
  run.prof_end(k);
  run.launches += 2;
}

template <int NV, class R, class Fn>
inline void box_min(Run<R>& run, int i0, int i1, int j0, int j1, int k0, int k1, Fn fn, int uslot) {
  int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
  dim3 blk(64, 4, 1);
  dim3 grd((ni + 63) / 64, (nj + 3) / 4, nk);
  int k = run.prof_begin("box_min", 0, 0, (double)ni * nj * nk);
  k_box_min<NV><<<grd, blk, 0, run.s>>>(i0, j0, k0, ni, nj, fn, run.us + uslot);
  run.prof_end(k);
  ++run.launches;
}

// ---------------------------------------------------------------------
// boundary.f90
template <class R> inline void energy_bcs(Run<R>& r) { ghost(r, r.g_cell, r.a.energy); }
template <class R> inline void density_bcs(Run<R>& r) { ghost(r, r.g_cell, r.a.rho); }
template <class R> inline void velocity_bcs(Run<R>& r) { ghost(r, r.g_node, r.a.vx, &r.a.vy, &r.a.vz); }
template <class R> inline void remap_v_bcs(Run<R>& r) { ghost(r, r.g_node, r.a.vx1, &r.a.vy1, &r.a.vz1); }
template <class R> inline void bfield_bcs(Run<R>& r) {
  ghost(r, r.g_bx, r.a.bx);
  ghost(r, r.g_by, r.a.by);
  ghost(r, r.g_bz, r.a.bz);
}
// boundary.f90:212 temperature_bcs exchanges rho (:214), then mirrors T.
template <class R> inline void temperature_bcs(Run<R>& r) {
  ghost(r, r.g_cell_mpi, r.a.rho);
  ghost(r, r.g_cell_user, r.a.temperature);
}
template <class R> inline void boundary_conditions(Run<R>& r) {
  bfield_bcs(r);
  energy_bcs(r);
  density_bcs(r);
  velocity_bcs(r);
}

// Full-array elementwise helpers (Fortran whole-array statements).
template <class R, class Fn>
inline void whole(Run<R>& r, Fn fn) {
  LARE_BOX(r, -2, r.n[0] + 2, -2, r.n[1] + 2, -2, r.n[2] + 2, fn);
}

// ---------------------------------------------------------------------
// lagran.F90:1176-1230 eta_calc
template <class R>
void eta_calc(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  auto eta = run.a.eta;
  if (!run.p.resistive_mhd) {
    whole(run, [=] __device__(int i, int j, int k) { eta(i, j, k) = R(0); });
    return;
  }
  auto bx = run.a.bx, by = run.a.by, bz = run.a.bz;
  auto dxc = run.a.dxc, dyc = run.a.dyc, dzc = run.a.dzc;
  const R jmax = (R)run.p.j_max, eb = (R)run.p.eta_background, e0 = (R)run.p.eta0;
  LARE_BOXW(run, 4, -1, nx + 1, -1, ny + 1, -1, nz + 1, [=] __device__(int ix, int iy, int iz) {
    int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
    R jx = (bz(ix, iyp, iz) - bz(ix, iy, iz)) / dyc(iy) - (by(ix, iy, izp) - by(ix, iy, iz)) / dzc(iz);
    R jxp = (bz(ixp, iyp, iz) - bz(ixp, iy, iz)) / dyc(iy) - (by(ixp, iy, izp) - by(ixp, iy, iz)) / dzc(iz);
    R jy = (bx(ix, iy, izp) - bx(ix, iy, iz)) / dzc(iz) - (bz(ixp, iy, iz) - bz(ix, iy, iz)) / dxc(ix);
    R jyp = (bx(ix, iyp, izp) - bx(ix, iyp, iz)) / dzc(iz) - (bz(ixp, iyp, iz) - bz(ix, iyp, iz)) / dxc(ix);
    R jz = (by(ixp, iy, iz) - by(ix, iy, iz)) / dxc(ix) - (bx(ix, iyp, iz) - bx(ix, iy, iz)) / dyc(iy);
    R jzp = (by(ixp, iy, izp) - by(ix, iy, izp)) / dxc(ix) - (bx(ix, iyp, izp) - bx(ix, iy, izp)) / dyc(iy);
    jx = (jx + jxp) * R(0.5);
    jy = (jy + jyp) * R(0.5);
    jz = (jz + jzp) * R(0.5);
    if (sqrt(jx * jx + jy * jy + jz * jz) > jmax) eta(ix, iy, iz) = eb + e0;
    else eta(ix, iy, iz) = eb;
  });
}

// ---------------------------------------------------------------------
// lagran.F90:483-524 viscous_damping
template <class R>
void viscous_damping(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  auto vx = run.a.vx, vy = run.a.vy, vz = run.a.vz, visc3 = run.a.visc3;
  auto qx = run.a.qx, qy = run.a.qy, qz = run.a.qz;
  auto dxb = run.a.dxb, dyb = run.a.dyb, dzb = run.a.dzb, dxc = run.a.dxc, dyc = run.a.dyc, dzc = run.a.dzc;
  const double* sc = run.sc;
  LARE_BOXW(run, 7, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz) {
    int ixp = ix + 1, ixm = ix - 1, iyp = iy + 1, iym = iy - 1, izp = iz + 1, izm = iz - 1;
    A3<R> vv[3] = {vx, vy, vz};
    A3<R> qq[3] = {qx, qy, qz};
    for (int c = 0; c < 3; ++c) {
      A3<R> v = vv[c];
      qq[c](ix, iy, iz) = visc3(ix, iy, iz) *
          (((v(ixp, iy, iz) - v(ix, iy, iz)) / dxb(ixp) - (v(ix, iy, iz) - v(ixm, iy, iz)) / dxb(ix)) / dxc(ix) +
           ((v(ix, iyp, iz) - v(ix, iy, iz)) / dyb(iyp) - (v(ix, iy, iz) - v(ix, iym, iz)) / dyb(iy)) / dyc(iy) +
           ((v(ix, iy, izp) - v(ix, iy, iz)) / dzb(izp) - (v(ix, iy, iz) - v(ix, iy, izm)) / dzb(iz)) / dzc(iz));
    }
  });
  LARE_BOXW(run, 9, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz) {
    const R dt = (R)sc[SC_DT];
    vx(ix, iy, iz) = vx(ix, iy, iz) + dt * qx(ix, iy, iz);
    vy(ix, iy, iz) = vy(ix, iy, iz) + dt * qy(ix, iy, iz);
    vz(ix, iy, iz) = vz(ix, iy, iz) + dt * qz(ix, iy, iz);
  });
}

// ---------------------------------------------------------------------
// lagran.F90:795-855 edge_viscosity with the default DEFINES (psi = 0).
template <class R>
__device__ __forceinline__ R edge_viscosity(R dvdots, R r1, R r2, R c1, R c2, R dvx, R dvy, R dvz, R dx, R dt,
                                            R visc1, R visc2_norm) {
  dvdots = -fabs(dvdots);
  R rho_edge = R(2) * r1 * r2 / (r1 + r2);
  R cs_edge = fmin(c1, c2);
  R dv2 = dvx * dvx + dvy * dvy + dvz * dvz;
  R dv = sqrt(dv2);
  R psi = R(0);
  if (dv * dt / dx < R(1.e-14)) dvdots = R(0);
  else dvdots = dvdots / dv;
  R vc = visc1 * cs_edge;
  R q_k_bar = rho_edge * (visc2_norm * dv + sqrt(visc2_norm * visc2_norm * dv2 + vc * vc));
  return q_k_bar * (R(1) - psi) * dvdots;
}

// lagran.F90:532-857 shock_viscosity
template <class R>
void shock_viscosity(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  if (!run.visc2_norm_set) {
    run.visc2_norm_set = true;
    double v2n = 0.25 * (run.p.gamma + 1.0) * run.p.visc2;
    if (sizeof(R) == 4) v2n = (double)(R(0.25) * (R(run.p.gamma) + R(1)) * R(run.p.visc2));
    cudaMemcpyAsync(run.sc + SC_VISC2N, &v2n, sizeof(double), cudaMemcpyHostToDevice, run.s);
    cudaStreamSynchronize(run.s);
  }
  auto rho = run.a.rho, pressure = run.a.pressure, gamma_boris = run.a.gamma_boris, cs = run.a.cs;
  auto bx1 = run.a.bx1, by1 = run.a.by1, bz1 = run.a.bz1, cv = run.a.cv, cv_v = run.a.cv_v, cs_v = run.a.cs_v;
  auto p_visc = run.a.p_visc, visc_heat = run.a.visc_heat;
  auto vx = run.a.vx, vy = run.a.vy, vz = run.a.vz, rho_v = run.a.rho_v;
  auto alpha1 = run.a.alpha1, alpha2 = run.a.alpha2, alpha3 = run.a.alpha3;
  auto dxb = run.a.dxb, dyb = run.a.dyb, dzb = run.a.dzb, dxc = run.a.dxc, dyc = run.a.dyc, dzc = run.a.dzc;
  auto fx_visc = run.a.fx_visc, fy_visc = run.a.fy_visc, fz_visc = run.a.fz_visc;
  const R g = (R)run.p.gamma, visc1 = (R)run.p.visc1;
  const double* sc = run.sc;

  // p_visc = 0 and visc_heat = 0 (:548-549) are folded into the writes
  // below: p_visc(0:n+1) is written by the MAX loop from 0, and the
  // remaining p_visc elements are zeroed here.
  whole(run, [=] __device__(int i, int j, int k) {
    if (i < 0 || i > nx + 1 || j < 0 || j > ny + 1 || k < 0 || k > nz + 1) p_visc(i, j, k) = R(0);
  });
  LARE_BOXW(run, 7, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
    R rmin = fmax(rho(ix, iy, iz), Num<R>::tiny());
    R b2 = bx1(ix, iy, iz) * bx1(ix, iy, iz) + by1(ix, iy, iz) * by1(ix, iy, iz) + bz1(ix, iy, iz) * bz1(ix, iy, iz);
    cs(ix, iy, iz) = sqrt((g * pressure(ix, iy, iz) + gamma_boris(ix, iy, iz) * b2) / rmin);
  });
  LARE_BOXW(run, 4, -1, nx + 1, -1, ny + 1, -1, nz + 1, [=] __device__(int ix, int iy, int iz) {
    int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
    R s = cs(ix, iy, iz) * cv(ix, iy, iz) + cs(ixp, iy, iz) * cv(ixp, iy, iz) + cs(ix, iyp, iz) * cv(ix, iyp, iz) +
          cs(ixp, iyp, iz) * cv(ixp, iyp, iz) + cs(ix, iy, izp) * cv(ix, iy, izp) + cs(ixp, iy, izp) * cv(ixp, iy, izp) +
          cs(ix, iyp, izp) * cv(ix, iyp, izp) + cs(ixp, iyp, izp) * cv(ixp, iyp, izp);
    cs_v(ix, iy, iz) = R(0.125) * s / cv_v(ix, iy, iz);
  });
  LARE_BOXW(run, 6, 0, nx + 1, 0, ny + 2, 0, nz + 2, [=] __device__(int ix, int iy, int iz) {
    const R dt = (R)sc[SC_DT], v2n = (R)sc[SC_VISC2N];
    int i1 = ix - 1, j1 = iy - 1, k1 = iz - 1, i2 = ix, j2 = iy - 1, k2 = iz - 1;
    R dvdots = -(vx(i1, j1, k1) - vx(i2, j2, k2));
    alpha1(ix, iy, iz) = edge_viscosity<R>(dvdots, rho_v(i1, j1, k1), rho_v(i2, j2, k2), cs_v(i1, j1, k1),
                                           cs_v(i2, j2, k2), vx(i1, j1, k1) - vx(i2, j2, k2),
                                           vy(i1, j1, k1) - vy(i2, j2, k2), vz(i1, j1, k1) - vz(i2, j2, k2),
                                           dxb(ix), dt, visc1, v2n);
  });
  LARE_BOXW(run, 6, -1, nx + 1, 0, ny + 1, 0, nz + 2, [=] __device__(int ix, int iy, int iz) {
    const R dt = (R)sc[SC_DT], v2n = (R)sc[SC_VISC2N];
    int i1 = ix, j1 = iy - 1, k1 = iz - 1, i2 = ix, j2 = iy, k2 = iz - 1;
    R dvdots = -(vy(i1, j1, k1) - vy(i2, j2, k2));
    alpha2(ix, iy, iz) = edge_viscosity<R>(dvdots, rho_v(i1, j1, k1), rho_v(i2, j2, k2), cs_v(i1, j1, k1),
                                           cs_v(i2, j2, k2), vx(i1, j1, k1) - vx(i2, j2, k2),
                                           vy(i1, j1, k1) - vy(i2, j2, k2), vz(i1, j1, k1) - vz(i2, j2, k2),
                                           dyb(iy), dt, visc1, v2n);
  });
  LARE_BOXW(run, 6, -1, nx + 1, -1, ny + 1, 0, nz + 1, [=] __device__(int ix, int iy, int iz) {
    const R dt = (R)sc[SC_DT], v2n = (R)sc[SC_VISC2N];
    int i1 = ix, j1 = iy, k1 = iz - 1, i2 = ix, j2 = iy, k2 = iz;
    R dvdots = -(vz(i1, j1, k1) - vz(i2, j2, k2));
    alpha3(ix, iy, iz) = edge_viscosity<R>(dvdots, rho_v(i1, j1, k1), rho_v(i2, j2, k2), cs_v(i1, j1, k1),
                                           cs_v(i2, j2, k2), vx(i1, j1, k1) - vx(i2, j2, k2),
                                           vy(i1, j1, k1) - vy(i2, j2, k2), vz(i1, j1, k1) - vz(i2, j2, k2),
                                           dzb(iz), dt, visc1, v2n);
  });
  LARE_BOXW(run, 9, 0, nx + 1, 0, ny + 1, 0, nz + 1, [=] __device__(int ix, int iy, int iz) {
    int ixm = ix - 1, iym = iy - 1, izm = iz - 1, iyp = iy + 1, izp = iz + 1;
    auto d2 = [&](int a0, int b0, int c0, int a1, int b1, int c1) {
      R ux = vx(a0, b0, c0) - vx(a1, b1, c1);
      R uy = vy(a0, b0, c0) - vy(a1, b1, c1);
      R uz = vz(a0, b0, c0) - vz(a1, b1, c1);
      return ux * ux + uy * uy + uz * uz;
    };
    R a1 = d2(ixm, iym, izm, ix, iym, izm);
    R a2 = d2(ix, iym, izm, ix, iy, izm);
    R a3 = d2(ix, iy, izm, ixm, iy, izm);
    R a4 = d2(ixm, iy, izm, ixm, iym, izm);
    R a5 = d2(ixm, iym, iz, ix, iym, iz);
    R a6 = d2(ix, iym, iz, ix, iy, iz);
    R a7 = d2(ix, iy, iz, ixm, iy, iz);
    R a8 = d2(ixm, iy, iz, ixm, iym, iz);
    R a9 = d2(ix, iy, izm, ix, iy, iz);
    R a10 = d2(ixm, iy, izm, ixm, iy, iz);
    R a11 = d2(ixm, iym, izm, ixm, iym, iz);
    R a12 = d2(ix, iym, izm, ix, iym, iz);
    R pv = R(0);
    pv = fmax(pv, -alpha1(ix, iy, iz) * sqrt(a1));
    pv = fmax(pv, -alpha2(ix, iy, iz) * sqrt(a2));
    pv = fmax(pv, -alpha3(ix, iy, iz) * sqrt(a9));
    p_visc(ix, iy, iz) = pv;
    R ddx = dxb(ix), ddy = dyb(iy), ddz = dzb(iz);
    R vh = -R(0.25) * ddy * ddz * alpha1(ix, iy, iz) * a1 - R(0.25) * ddx * ddz * alpha2(ix, iy, iz) * a2 -
           R(0.25) * ddy * ddz * alpha1(ix, iyp, iz) * a3 - R(0.25) * ddx * ddz * alpha2(ixm, iy, iz) * a4 -
           R(0.25) * ddy * ddz * alpha1(ix, iy, izp) * a5 - R(0.25) * ddx * ddz * alpha2(ix, iy, izp) * a6 -
           R(0.25) * ddy * ddz * alpha1(ix, iyp, izp) * a7 - R(0.25) * ddx * ddz * alpha2(ixm, iy, izp) * a8 -
           R(0.25) * ddx * ddy * alpha3(ix, iy, iz) * a9 - R(0.25) * ddx * ddy * alpha3(ixm, iy, iz) * a10 -
           R(0.25) * ddx * ddy * alpha3(ixm, iym, iz) * a11 - R(0.25) * ddx * ddy * alpha3(ix, iym, iz) * a12;
    visc_heat(ix, iy, iz) = vh / cv(ix, iy, iz);
  });
  LARE_BOXW(run, 10, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz) {
    int ixm = ix - 1, ixp = ix + 1, iym = iy - 1, iyp = iy + 1, izm = iz - 1, izp = iz + 1;
    R a1 = alpha1(ix, iyp, izp) * dyc(iy) * dzc(iz);
    R a2 = alpha1(ixp, iyp, izp) * dyc(iy) * dzc(iz);
    R a3 = alpha2(ix, iy, izp) * dxc(ix) * dzc(iz);
    R a4 = alpha2(ix, iyp, izp) * dxc(ix) * dzc(iz);
    R a5 = alpha3(ix, iy, iz) * dxc(ix) * dyc(iy);
    R a6 = alpha3(ix, iy, izp) * dxc(ix) * dyc(iy);
    A3<R> vv[3] = {vx, vy, vz};
    A3<R> ff[3] = {fx_visc, fy_visc, fz_visc};
    R cvv = cv_v(ix, iy, iz);
    for (int c = 0; c < 3; ++c) {
      A3<R> v = vv[c];
      R v0 = v(ix, iy, iz);
      ff[c](ix, iy, iz) = (a1 * (v0 - v(ixm, iy, iz)) + a2 * (v0 - v(ixp, iy, iz)) + a3 * (v0 - v(ix, iym, iz)) +
                           a4 * (v0 - v(ix, iyp, iz)) + a5 * (v0 - v(ix, iy, izm)) + a6 * (v0 - v(ix, iy, izp))) /
                          cvv;
    }
  });
}

// lagran.F90:861-937 shock_heating (visc_heat = MAX(visc_heat, 0) folded in)
template <class R>
void shock_heating(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  auto vx = run.a.vx, vy = run.a.vy, vz = run.a.vz, vx1 = run.a.vx1, vy1 = run.a.vy1, vz1 = run.a.vz1;
  auto alpha1 = run.a.alpha1, alpha2 = run.a.alpha2, alpha3 = run.a.alpha3, cv = run.a.cv, visc_heat = run.a.visc_heat;
  auto dxb = run.a.dxb, dyb = run.a.dyb, dzb = run.a.dzb;
  LARE_BOXW(run, 11, 0, nx + 1, 0, ny + 1, 0, nz + 1, [=] __device__(int ix, int iy, int iz) {
    int ixm = ix - 1, iym = iy - 1, izm = iz - 1, iyp = iy + 1, izp = iz + 1;
    auto dd = [&](int a0, int b0, int c0, int a1, int b1, int c1) {
      return (vx(a0, b0, c0) - vx(a1, b1, c1)) * (vx1(a0, b0, c0) - vx1(a1, b1, c1)) +
             (vy(a0, b0, c0) - vy(a1, b1, c1)) * (vy1(a0, b0, c0) - vy1(a1, b1, c1)) +
             (vz(a0, b0, c0) - vz(a1, b1, c1)) * (vz1(a0, b0, c0) - vz1(a1, b1, c1));
    };
    R a1 = dd(ixm, iym, izm, ix, iym, izm);
    R a2 = dd(ix, iym, izm, ix, iy, izm);
    R a3 = dd(ix, iy, izm, ixm, iy, izm);
    R a4 = dd(ixm, iy, izm, ixm, iym, izm);
    R a5 = dd(ixm, iym, iz, ix, iym, iz);
    R a6 = dd(ix, iym, iz, ix, iy, iz);
    R a7 = dd(ix, iy, iz, ixm, iy, iz);
    R a8 = dd(ixm, iy, iz, ixm, iym, iz);
    R a9 = dd(ix, iy, izm, ix, iy, iz);
    R a10 = dd(ixm, iy, izm, ixm, iy, iz);
    R a11 = dd(ixm, iym, izm, ixm, iym, iz);
    R a12 = dd(ix, iym, izm, ix, iym, iz);
    R ddx = dxb(ix), ddy = dyb(iy), ddz = dzb(iz);
    R vh = -R(0.25) * ddy * ddz * alpha1(ix, iy, iz) * a1 - R(0.25) * ddx * ddz * alpha2(ix, iy, iz) * a2 -
           R(0.25) * ddy * ddz * alpha1(ix, iyp, iz) * a3 - R(0.25) * ddx * ddz * alpha2(ixm, iy, iz) * a4 -
           R(0.25) * ddy * ddz * alpha1(ix, iy, izp) * a5 - R(0.25) * ddx * ddz * alpha2(ix, iy, izp) * a6 -
           R(0.25) * ddy * ddz * alpha1(ix, iyp, izp) * a7 - R(0.25) * ddx * ddz * alpha2(ixm, iy, izp) * a8 -
           R(0.25) * ddx * ddy * alpha3(ix, iy, iz) * a9 - R(0.25) * ddx * ddy * alpha3(ixm, iy, iz) * a10 -
           R(0.25) * ddx * ddy * alpha3(ixm, iym, iz) * a11 - R(0.25) * ddx * ddy * alpha3(ix, iym, iz) * a12;
    R v = vh / cv(ix, iy, iz);
    visc_heat(ix, iy, iz) = v > R(0) ? v : R(0);
  });
}

// ---------------------------------------------------------------------
// conduct.f90:56-143 calc_s_stages.  Produces larsen_factor and the stage
// count in sc[SC_STAGES] from the dt in sc[dt_slot].
template <class R>
void calc_s_stages(Run<R>& run, int dt_slot) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  auto temperature = run.a.temperature, energy = run.a.energy, rho = run.a.rho, larsen = run.a.larsen;
  auto dxb = run.a.dxb, dyb = run.a.dyb, dzb = run.a.dzb;
  const R g = (R)run.p.gamma, xi = (R)run.p.xi_n, ip = (R)run.p.ionise_pot, k0 = (R)run.p.kappa_0;
  const R fl = (R)run.p.flux_limiter;
  const bool limiter = run.p.heat_flux_limiter != 0;
  LARE_BOXW(run, 2, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
    temperature(ix, iy, iz) = (g - R(1)) / (R(2) - xi) * (energy(ix, iy, iz) - (R(1) - xi) * ip);
  });
  LARE_BOXW(run, 3, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz) {
    if (!limiter) { larsen(ix, iy, iz) = R(1); return; }
    int ixm = ix - 1, ixp = ix + 1, iym = iy - 1, iyp = iy + 1, izm = iz - 1, izp = iz + 1;
    R T = temperature(ix, iy, iz);
    R temp = pow(T, R(2.5));
    R q_fs = fl * R(42.85) * rho(ix, iy, iz) * pow(T, R(1.5));
    R q_fs2 = q_fs * q_fs;
    R q_spx = -k0 * temp * (temperature(ixp, iy, iz) - temperature(ixm, iy, iz)) * R(0.5) / dxb(ix);
    R q_spy = -k0 * temp * (temperature(ix, iyp, iz) - temperature(ix, iym, iz)) * R(0.5) / dyb(iy);
    R q_spz = -k0 * temp * (temperature(ix, iy, izp) - temperature(ix, iy, izm)) * R(0.5) / dzb(iz);
    R q_sp2 = q_spx * q_spx + q_spy * q_spy + q_spz * q_spz;
    larsen(ix, iy, iz) = q_fs / sqrt(q_fs2 + q_sp2);
  });
  unsigned long long* us = run.us;
  launch_scalar(run.s, run.launches, [=] __device__() { us[U_DTPARAB] = (unsigned long long)__double_as_longlong(1.e10); });
  box_min<1>(run, 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz, double* v) {
    R kappa1 = k0 * larsen(ix, iy, iz);
    R temp = (g - R(1)) / (R(2) - xi) * (energy(ix, iy, iz) - (R(1) - xi) * ip);
    R tp = pow(temp, R(2.5));
    R r = rho(ix, iy, iz);
    R dt1 = r * (dxb(ix) * dxb(ix)) / (R(2) * kappa1 * tp);
    R dt2 = r * (dyb(iy) * dyb(iy)) / (R(2) * kappa1 * tp);
    R dt3 = r * (dzb(iz) * dzb(iz)) / (R(2) * kappa1 * tp);
    v[0] = (double)fmin(fmin(dt1, dt2), dt3);
  }, U_DTPARAB);
  double* sc = run.sc;
  const double mult = run.p.dt_multiplier;
  const bool f32 = sizeof(R) == 4;
  launch_scalar(run.s, run.launches, [=] __device__() {
    double dtp_min = __longlong_as_double((long long)us[U_DTPARAB]);
    double dt = sc[dt_slot];
    double stages, dt_parab;
    if (f32) {
      // The FP32 form keeps this recurrence in FP64 but starts from the
      // FP32 minimum, as the field arithmetic produced it.
      dt_parab = mult * fmin(dtp_min, 1.e10) / sqrt(3.0);
    } else {
      dt_parab = mult * fmin(dtp_min, 1.e10) / sqrt(3.0);
    }
    stages = 0.5 * (sqrt(9.0 + 16.0 * (dt / dt_parab)) - 1.0);
    int ns = (int)ceil(stages);
    if (ns % 2 == 0) ns = ns + 1;
    sc[SC_STAGES] = (double)ns;
    sc[SC_DTPARAB] = dt_parab;
  });
}

// conduct.f90:152-291 heat_flux as a gather.  The reference scatters each
// cell's three face fluxes into flux(c) and flux(c+e); for cell c the
// contributions therefore arrive in loop order as
//   +Fz(c-ez), +Fy(c-ey), +Fx(c-ex), -Fx(c), -Fy(c), -Fz(c)
// (iteration (i,j,k-1) precedes (i,j-1,k) precedes (i-1,j,k) precedes
// (i,j,k)), which this kernel reproduces term for term, with no atomics.
template <class R>
struct HeatFluxArgs {
  A3<R> T, bx, by, bz, larsen;
  A1<R> dxb, dyb, dzb, dxc, dyc, dzc;
  R k0;
};

template <class R>
__device__ __forceinline__ R face_flux(const HeatFluxArgs<R>& h, int axis, int ix, int iy, int iz) {
  const R min_b = R(1.0e-10);  // conduct.f90:28
  const A3<R>& T = h.T;
  int ixp = ix + 1, ixm = ix - 1, iyp = iy + 1, iym = iy - 1, izp = iz + 1, izm = iz - 1;
  R lf = h.larsen(ix, iy, iz);
  if (axis == 0) {
    R byf = R(0.25) * (h.by(ix, iy, iz) + h.by(ixp, iy, iz) + h.by(ix, iym, iz) + h.by(ixp, iym, iz));
    R bzf = R(0.25) * (h.bz(ix, iy, iz) + h.bz(ixp, iy, iz) + h.bz(ix, iy, izm) + h.bz(ixp, iy, izm));
    R b0 = h.bx(ix, iy, iz);
    R modb = b0 * b0 + byf * byf + bzf * bzf + min_b;
    R tb = (T(ixp, iy, iz) + T(ix, iy, iz)) / R(2);
    R tb_p = (T(ixp, iyp, iz) + T(ix, iyp, iz)) / R(2);
    R tb_m = (T(ixp, iym, iz) + T(ix, iym, iz)) / R(2);
    R tg_a1 = (tb_p - tb_m) / (h.dyc(iy) + h.dyc(iym));
    tb_p = (T(ixp, iy, izp) + T(ix, iy, izp)) / R(2);
    tb_m = (T(ixp, iy, izm) + T(ix, iy, izm)) / R(2);
    R tg_a2 = (tb_p - tb_m) / (h.dzc(iz) + h.dzc(izm));
    R tg = (T(ixp, iy, iz) - T(ix, iy, iz)) / h.dxc(ix);
    tb = tb > R(0) ? tb : R(0);
    return -lf * h.k0 * pow(tb, R(2.5)) * (b0 * (tg * b0 + tg_a1 * byf + tg_a2 * bzf) + tg * min_b) / modb;
  } else if (axis == 1) {
    R bxf = R(0.25) * (h.bx(ix, iy, iz) + h.bx(ix, iyp, iz) + h.bx(ixm, iy, iz) + h.bx(ixm, iyp, iz));
    R bzf = R(0.25) * (h.bz(ix, iy, iz) + h.bz(ix, iyp, iz) + h.bz(ix, iy, izm) + h.bz(ix, iyp, izm));
    R b0 = h.by(ix, iy, iz);
    R modb = bxf * bxf + b0 * b0 + bzf * bzf + min_b;
    R tb = (T(ix, iyp, iz) + T(ix, iy, iz)) / R(2);
    R tb_p = (T(ixp, iy, iz) + T(ixp, iyp, iz)) / R(2);
    R tb_m = (T(ixm, iyp, iz) + T(ixm, iy, iz)) / R(2);
    R tg_a1 = (tb_p - tb_m) / (h.dxc(ix) + h.dxc(ixm));
    tb_p = (T(ix, iyp, izp) + T(ix, iy, izp)) / R(2);
    tb_m = (T(ix, iyp, izm) + T(ix, iy, izm)) / R(2);
    R tg_a2 = (tb_p - tb_m) / (h.dzc(iz) + h.dzc(izm));
    R tg = (T(ix, iyp, iz) - T(ix, iy, iz)) / h.dyc(iy);
    tb = tb > R(0) ? tb : R(0);
    return -lf * h.k0 * pow(tb, R(2.5)) * (b0 * (tg * b0 + tg_a1 * bxf + tg_a2 * bzf) + tg * min_b) / modb;
  } else {
    R bxf = R(0.25) * (h.bx(ix, iy, iz) + h.bx(ix, iy, izp) + h.bx(ixm, iy, iz) + h.bx(ixm, iy, izp));
    R byf = R(0.25) * (h.by(ix, iy, iz) + h.by(ix, iy, izp) + h.by(ix, iym, iz) + h.by(ix, iym, izp));
    R b0 = h.bz(ix, iy, iz);
    R modb = bxf * bxf + byf * byf + b0 * b0 + min_b;
    R tb = (T(ix, iy, izp) + T(ix, iy, iz)) / R(2);
    R tb_p = (T(ixp, iy, izp) + T(ixp, iy, iz)) / R(2);
    R tb_m = (T(ixm, iy, izp) + T(ixm, iy, iz)) / R(2);
    R tg_a1 = (tb_p - tb_m) / (h.dxc(ix) + h.dxc(ixm));
    tb_p = (T(ix, iyp, izp) + T(ix, iyp, iz)) / R(2);
    tb_m = (T(ix, iym, izp) + T(ix, iym, iz)) / R(2);
    R tg_a2 = (tb_p - tb_m) / (h.dyc(iy) + h.dyc(iym));
    R tg = (T(ix, iy, izp) - T(ix, iy, iz)) / h.dzc(iz);
    tb = tb > R(0) ? tb : R(0);
    return -lf * h.k0 * pow(tb, R(2.5)) * (b0 * (tg * b0 + tg_a1 * bxf + tg_a2 * byf) + tg * min_b) / modb;
  }
}

template <class R>
__device__ __forceinline__ R heat_flux_gather(const HeatFluxArgs<R>& h, int ix, int iy, int iz) {
  R f = R(0);
  f = f + face_flux(h, 2, ix, iy, iz - 1) / h.dzb(iz - 1);
  f = f + face_flux(h, 1, ix, iy - 1, iz) / h.dyb(iy - 1);
  f = f + face_flux(h, 0, ix - 1, iy, iz) / h.dxb(ix - 1);
  f = f - face_flux(h, 0, ix, iy, iz) / h.dxb(ix);
  f = f - face_flux(h, 1, ix, iy, iz) / h.dyb(iy);
  f = f - face_flux(h, 2, ix, iy, iz) / h.dzb(iz);
  return f;
}

template <class R>
void temperature_from(Run<R>& run, A3<R> e) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  auto temperature = run.a.temperature;
  const R g = (R)run.p.gamma, xi = (R)run.p.xi_n, ip = (R)run.p.ionise_pot;
  LARE_BOXW(run, 2, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
    temperature(ix, iy, iz) = (g - R(1)) / (R(2) - xi) * (e(ix, iy, iz) - (R(1) - xi) * ip);
  });
}

// Copy between whole arrays (Fortran whole-array assignment).
template <class R>
void copy_whole(Run<R>& run, A3<R> dst, A3<R> src) {
  int k = run.prof_begin("copy_whole", 0, 2, (double)run.elems);
  cudaMemcpyAsync(dst.p - (2 + 2 * run.sx + 2 * run.sxy), src.p - (2 + 2 * run.sx + 2 * run.sxy),
                  run.elems * sizeof(R), cudaMemcpyDeviceToDevice, run.s);
  run.prof_end(k);
}

// conduct.f90:299-416 heat_conduct_sts2, dt from sc[dt_slot]; the stage
// count s must already be known on the host (run.n_s_stages).
template <class R>
void heat_conduct_sts2(Run<R>& run, int dt_slot) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  const int s = run.n_s_stages;
  std::vector<double> a(s + 1), b(s + 1), mu_tilde(s + 1), mu(s + 1), nu(s + 1), gamma_tilde(s + 1);
  double ds = (double)s;
  double omega_1 = 4.0 / (ds * ds + ds - 2.0);
  for (int j = 0; j <= (s < 2 ? s : 2); ++j) b[j] = 1.0 / 3.0;
  for (int j = 3; j <= s; ++j) {
    double dj = (double)j;
    b[j] = (dj * dj + dj - 2.0) / (2.0 * dj * (dj + 1.0));
  }
  for (int j = 0; j <= s; ++j) a[j] = 1.0 - b[j];
  mu_tilde[1] = omega_1 / 3.0;
  for (int j = 2; j <= s; ++j) {
    double dj = (double)j;
    mu_tilde[j] = ((2.0 * dj - 1.0) / dj) * omega_1 * (b[j] / b[j - 1]);
    mu[j] = ((2.0 * dj - 1.0) / dj) * (b[j] / b[j - 1]);
    nu[j] = -1.0 * ((dj - 1.0) / dj) * (b[j] / b[j - 2]);
    gamma_tilde[j] = -1.0 * a[j - 1] * mu_tilde[j];
  }
  Arrays<R>& A = run.a;
  auto Y0 = A.Y0, Y1 = A.Y1, Y2 = A.Y2, Y3 = A.Y3, Lc_Y0 = A.Lc_Y0, rho = A.rho, energy = A.energy;
  HeatFluxArgs<R> h{A.temperature, A.bx, A.by, A.bz, A.larsen, A.dxb, A.dyb, A.dzb, A.dxc, A.dyc, A.dzc,
                    (R)run.p.kappa_0};
  const double* sc = run.sc;
  copy_whole(run, Y0, energy);
  copy_whole(run, Y1, energy);
  copy_whole(run, Y2, energy);
  copy_whole(run, Y3, energy);
  temperature_from(run, Y0);
  const R mt1 = (R)mu_tilde[1];
  LARE_BOXW(run, 10, 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz) {
    const R dt = (R)sc[dt_slot];
    R f = heat_flux_gather<R>(h, ix, iy, iz);
    R lc = (R(1) / rho(ix, iy, iz)) * f;
    Lc_Y0(ix, iy, iz) = lc;
    R c0 = mt1 * dt * lc;
    R y1 = Y0(ix, iy, iz) + c0;
    // Y(2) = Y(1); Y(1) = Y(0) on 1:n (conduct.f90:366-367)
    Y2(ix, iy, iz) = y1;
    Y1(ix, iy, iz) = Y0(ix, iy, iz);
  });
  for (int j = 2; j <= s; ++j) {
    temperature_from(run, Y2);
    temperature_bcs(run);
    const R gt = (R)gamma_tilde[j], mtj = (R)mu_tilde[j], mj = (R)mu[j], nj = (R)nu[j];
    const R omn = (R)(1.0 - mu[j] - nu[j]);
    const R omn_r = R(1) - mj - nj;
    LARE_BOXW(run, 11, 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz) {
      const R dt = (R)sc[dt_slot];
      (void)omn;
      R f = heat_flux_gather<R>(h, ix, iy, iz);
      R c0 = gt * dt * Lc_Y0(ix, iy, iz);
      R Lc = (R(1) / rho(ix, iy, iz)) * f;
      R c1 = mtj * dt * Lc;
      R y3 = mj * Y2(ix, iy, iz) + nj * Y1(ix, iy, iz) + omn_r * Y0(ix, iy, iz);
      Y3(ix, iy, iz) = y3 + c1 + c0;
    });
    if (j < s) {
      copy_whole(run, Y1, Y2);
      copy_whole(run, energy, Y3);
      energy_bcs(run);
      copy_whole(run, Y2, energy);
      // Y(3)(1:n) = 0 (conduct.f90:406): every later read of Y3 on 1:n is
      // preceded by the next stage's write, so the zeroing is not needed.
    }
  }
  if (s >= 2) {
    LARE_BOXW(run, 3, 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz) { energy(ix, iy, iz) = Y3(ix, iy, iz); });
  }
  energy_bcs(run);
}

// ---------------------------------------------------------------------
// lagran.F90:1239-1452 resistive_effects, first order in time, no cooling.
template <class R>
void resistive_effects(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  Arrays<R>& A = run.a;
  auto bx = A.bx, by = A.by, bz = A.bz, bx1 = A.bx1, by1 = A.by1, bz1 = A.bz1, eta = A.eta;
  auto flux_x = A.flux_x, flux_y = A.flux_y, flux_z = A.flux_z, curlb = A.curlb;
  auto rho = A.rho, energy = A.energy, ohmic_dep = A.ohmic_dep;
  auto dxb = A.dxb, dyb = A.dyb, dzb = A.dzb, dxc = A.dxc, dyc = A.dyc, dzc = A.dzc;
  const double* sc = run.sc;
  // bx1 = bx(-1:nx+2, ...) etc. (:1259-1261)
  LARE_BOXW(run, 6, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
    bx1(ix, iy, iz) = bx(ix, iy, iz);
    by1(ix, iy, iz) = by(ix, iy, iz);
    bz1(ix, iy, iz) = bz(ix, iy, iz);
  });
  // rkstep (:1470-1503)
  LARE_BOXW(run, 8, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz) {
    int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
    R jx1 = (bz(ix, iyp, iz) - bz(ix, iy, iz)) / dyc(iy) - (by(ix, iy, izp) - by(ix, iy, iz)) / dzc(iz);
    R jx2 = (bz(ixp, iyp, iz) - bz(ixp, iy, iz)) / dyc(iy) - (by(ixp, iy, izp) - by(ixp, iy, iz)) / dzc(iz);
    R jy1 = (bx(ix, iy, izp) - bx(ix, iy, iz)) / dzc(iz) - (bz(ixp, iy, iz) - bz(ix, iy, iz)) / dxc(ix);
    R jy2 = (bx(ix, iyp, izp) - bx(ix, iyp, iz)) / dzc(iz) - (bz(ixp, iyp, iz) - bz(ix, iyp, iz)) / dxc(ix);
    R jz1 = (by(ixp, iy, iz) - by(ix, iy, iz)) / dxc(ix) - (bx(ix, iyp, iz) - bx(ix, iy, iz)) / dyc(iy);
    R jz2 = (by(ixp, iy, izp) - by(ix, iy, izp)) / dxc(ix) - (bx(ix, iyp, izp) - bx(ix, iy, izp)) / dyc(iy);
    R jx = (jx1 + jx2) * R(0.5), jy = (jy1 + jy2) * R(0.5), jz = (jz1 + jz2) * R(0.5);
    R e = eta(ix, iy, iz);
    flux_x(ix, iy, iz) = -jx * e * dxc(ix) * R(0.5);
    flux_y(ix, iy, iz) = -jy * e * dyc(iy) * R(0.5);
    flux_z(ix, iy, iz) = -jz * e * dzc(iz) * R(0.5);
    curlb(ix, iy, iz) = e * (jx * jx + jy * jy + jz * jz);
  });
  // bstep (:1582-1635)
  auto kx = flux_x, ky = flux_y, kz = flux_z;
  LARE_BOXW(run, 4, 0, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz) {
    const R dt = (R)sc[SC_DTSUB];
    int iym = iy - 1, izm = iz - 1;
    R area = dyb(iy) * dzb(iz);
    bx(ix, iy, iz) = bx1(ix, iy, iz) + (kz(ix, iy, iz) - kz(ix, iym, iz) + kz(ix, iy, izm) - kz(ix, iym, izm) -
                                        ky(ix, iy, iz) + ky(ix, iy, izm) - ky(ix, iym, iz) + ky(ix, iym, izm)) *
                                           dt / area;
  });
  LARE_BOXW(run, 4, 1, nx, 0, ny, 1, nz, [=] __device__(int ix, int iy, int iz) {
    const R dt = (R)sc[SC_DTSUB];
    int ixm = ix - 1, izm = iz - 1;
    R area = dxb(ix) * dzb(iz);
    by(ix, iy, iz) = by1(ix, iy, iz) + (kx(ix, iy, iz) - kx(ix, iy, izm) + kx(ixm, iy, iz) - kx(ixm, iy, izm) -
                                        kz(ix, iy, iz) + kz(ixm, iy, iz) - kz(ix, iy, izm) + kz(ixm, iy, izm)) *
                                           dt / area;
  });
  LARE_BOXW(run, 4, 1, nx, 1, ny, 0, nz, [=] __device__(int ix, int iy, int iz) {
    const R dt = (R)sc[SC_DTSUB];
    int ixm = ix - 1, iym = iy - 1;
    R area = dxb(ix) * dyb(iy);
    bz(ix, iy, iz) = bz1(ix, iy, iz) + (ky(ix, iy, iz) - ky(ixm, iy, iz) + ky(ix, iym, iz) - ky(ixm, iym, iz) -
                                        kx(ix, iy, iz) + kx(ix, iym, iz) - kx(ixm, iy, iz) + kx(ixm, iym, iz)) *
                                           dt / area;
  });
  bfield_bcs(run);
  // ohmic heating (:1270-1288) and energy = MAX(energy, 0) (:1305) over the
  // whole array; the interior write and the clamp of the ghosts are fused.
  whole(run, [=] __device__(int ix, int iy, int iz) {
    R e = energy(ix, iy, iz);
    if (ix >= 1 && ix <= nx && iy >= 1 && iy <= ny && iz >= 1 && iz <= nz) {
      const R dt = (R)sc[SC_DTSUB];
      int ixm = ix - 1, iym = iy - 1, izm = iz - 1;
      R lh = +(curlb(ix, iy, iz) + curlb(ixm, iy, iz) + curlb(ix, iym, iz) + curlb(ixm, iym, iz) +
               curlb(ix, iy, izm) + curlb(ixm, iy, izm) + curlb(ix, iym, izm) + curlb(ixm, iym, izm)) *
             dt / (R(8) * rho(ix, iy, iz));
      ohmic_dep(ix, iy, iz) = ohmic_dep(ix, iy, iz) + lh;
      e = e + lh;
    }
    if (ix >= -1 && iy >= -1 && iz >= -1) energy(ix, iy, iz) = e > R(0) ? e : R(0);
  });
  energy_bcs(run);
  // total_ohmic_heating (:1309-1328)
  box_sum<1>(run, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz, double* v) {
    const R dt = (R)sc[SC_DTSUB];
    R w1 = dt * dxc(ix) * dyc(iy) * dzc(iz) * curlb(ix, iy, iz);
    if (ix == 0 || ix == nx) w1 = w1 * R(0.5);
    if (iy == 0 || iy == ny) w1 = w1 * R(0.5);
    if (iz == 0 || iz == nz) w1 = w1 * R(0.5);
    v[0] = (double)w1;
  }, SC_OHM_TOT, true);
}

// ---------------------------------------------------------------------
// Limited Van Leer flux shared by the *_flux routines of [xyz]remap.f90.
template <class R>
struct LimOut {
  R sign_v, vad_p, vad_m, fu, Di, dxbu, phi;
};
template <class R>
__device__ __forceinline__ LimOut<R> limiter(R v_advect, R fm, R fi, R fp, R fp2, R dxci, R dxcm, R dxcp, R dxbi,
                                             R dxbp, R dxu_p, R dxu_m, R dt, bool phi_from_dxu) {
  LimOut<R> L;
  R dfm = fi - fm, dfi = fp - fi, dfp = fp2 - fp;
  L.sign_v = copysign(R(1), v_advect);
  L.vad_p = (L.sign_v + R(1)) * R(0.5);
  L.vad_m = R(1) - L.vad_p;
  L.fu = fi * L.vad_p + fp * L.vad_m;
  R dfu = dfm * L.vad_p + dfp * L.vad_m;
  R dxcu = dxcm * L.vad_p + dxcp * L.vad_m;
  L.dxbu = dxbi * L.vad_p + dxbp * L.vad_m;
  if (phi_from_dxu) {
    R dxu = dxu_p * L.vad_p + dxu_m * L.vad_m;
    L.phi = fabs(v_advect) * dt / dxu;
  } else {
    L.phi = fabs(v_advect) * dt / L.dxbu;
  }
  R Da = (R(2) - L.phi) * fabs(dfi) / dxci + (R(1) + L.phi) * fabs(dfu) / dxcu;
  Da = Da * (R(1) / R(6));
  R ss = R(0.5) * (copysign(R(1), dfi) + copysign(R(1), dfu));
  L.Di = L.sign_v * ss * fmin(fmin(fabs(Da) * L.dxbu, fabs(dfi)), fabs(dfu));
  return L;
}

}  // namespace lare

#include "remap.cuh"

namespace lare {

// remap.f90:33-131 eulerian_remap
template <class R>
void eulerian_remap(Run<R>& run, int step, bool predictor) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  auto bx = run.a.bx, by = run.a.by, bz = run.a.bz;
  auto dxb = run.a.dxb, dyb = run.a.dyb, dzb = run.a.dzb;
  int pass[3] = {1, 1, 1};
  // B -> flux (remap.f90:43-69), including the -2 layers.
  LARE_BOXW(run, 6, -2, nx + 2, -2, ny + 2, -2, nz + 2, [=] __device__(int ix, int iy, int iz) {
    if (iy >= -1 && iz >= -1) bx(ix, iy, iz) = bx(ix, iy, iz) * dyb(iy) * dzb(iz);
    if (ix >= -1 && iz >= -1) by(ix, iy, iz) = by(ix, iy, iz) * dxb(ix) * dzb(iz);
    if (ix >= -1 && iy >= -1) bz(ix, iy, iz) = bz(ix, iy, iz) * dxb(ix) * dyb(iy);
  });
  static const int order[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {0, 2, 1}, {2, 1, 0}, {1, 0, 2}};
  int c = ((step % 6) + 6) % 6;
  const int dt_slot = predictor ? SC_DT2 : SC_DT;
  for (int s = 0; s < 3; ++s) {
    switch (order[c][s]) {
      case 0: remap_sweep<0>(run, predictor, dt_slot, pass); break;
      case 1: remap_sweep<1>(run, predictor, dt_slot, pass); break;
      default: remap_sweep<2>(run, predictor, dt_slot, pass); break;
    }
  }
  // flux -> B (remap.f90:101-127)
  LARE_BOXW(run, 6, -2, nx + 2, -2, ny + 2, -2, nz + 2, [=] __device__(int ix, int iy, int iz) {
    if (iy >= -1 && iz >= -1) bx(ix, iy, iz) = bx(ix, iy, iz) / dyb(iy) / dzb(iz);
    if (ix >= -1 && iz >= -1) by(ix, iy, iz) = by(ix, iy, iz) / dxb(ix) / dzb(iz);
    if (ix >= -1 && iy >= -1) bz(ix, iy, iz) = bz(ix, iy, iz) / dxb(ix) / dyb(iy);
  });
  bfield_bcs(run);
}

// ---------------------------------------------------------------------
// lagran.F90:1070-1166 set_dt.  Everything stays on the device; the host
// later reads dt/dtr/stages only to size its launch loops.
template <class R>
void set_dt(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  double* sc = run.sc;
  unsigned long long* us = run.us;
  if (run.set_dt_first) {
    run.set_dt_first = false;
    if (run.p.restart) {
      const double d = run.p.dt_from_restart;
      launch_scalar(run.s, run.launches, [=] __device__() { sc[SC_DT] = d; });
      return;
    }
  }
  Arrays<R>& A = run.a;
  auto bx = A.bx, by = A.by, bz = A.bz, rho = A.rho, pressure = A.pressure, p_visc = A.p_visc;
  auto vx = A.vx, vy = A.vy, vz = A.vz, eta = A.eta, gamma_boris = A.gamma_boris;
  auto dxb = A.dxb, dyb = A.dyb, dzb = A.dzb;
  const bool boris = run.p.boris != 0, resistive = run.p.resistive_mhd != 0;
  const R g = (R)run.p.gamma;
  const R va_max2 = (R)run.p.va_max * (R)run.p.va_max;
  if (!run.gamma_boris_one || boris) {
    whole(run, [=] __device__(int i, int j, int k) {
      if (i >= -1 && j >= -1 && k >= -1) gamma_boris(i, j, k) = R(1);
    });
    run.gamma_boris_one = !boris;
  }
  launch_scalar(run.s, run.launches, [=] __device__() {
    us[U_DTMIN] = (unsigned long long)__double_as_longlong(DBL_MAX);
    us[U_DTRMIN] = (unsigned long long)__double_as_longlong(DBL_MAX);
  });
  box_min<2>(run, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz, double* v) {
    R w1 = bx(ix, iy, iz) * bx(ix, iy, iz) + by(ix, iy, iz) * by(ix, iy, iz) + bz(ix, iy, iz) * bz(ix, iy, iz);
    R rho0 = fmax(rho(ix, iy, iz), Num<R>::tiny());
    R w2 = w1 / rho0;
    R gb = gamma_boris(ix, iy, iz);
    if (boris && (w2 >= va_max2)) {
      gb = R(1) / (R(1) + w2 / va_max2);
      gamma_boris(ix, iy, iz) = gb;
    }
    R cs2 = (g * pressure(ix, iy, iz) + gb * w1) / rho0;
    R c_visc2 = p_visc(ix, iy, iz) / rho0;
    R length = fmin(fmin(dxb(ix), dyb(iy)), dzb(iz));
    R dt1 = length / (sqrt(c_visc2) + sqrt(cs2 + c_visc2));
    R dt_local = Num<R>::huge();
    dt_local = fmin(dt_local, dt1);
    R dt2 = fmin(fmin(dxb(ix) / fmax(fabs(vx(ix, iy, iz)), Num<R>::tiny()),
                      dyb(iy) / fmax(fabs(vy(ix, iy, iz)), Num<R>::tiny())),
                 dzb(iz) / fmax(fabs(vz(ix, iy, iz)), Num<R>::tiny()));
    dt_local = fmin(dt_local, dt2);
    R dxlocal = R(1) / (R(1) / (dxb(ix) * dxb(ix)) + R(1) / (dyb(iy) * dyb(iy)) + R(1) / (dzb(iz) * dzb(iz)));
    R dt3 = Num<R>::huge();
    if (resistive) dt3 = R(0.2) * dxlocal / fmax(eta(ix, iy, iz), Num<R>::tiny());
    v[0] = (double)dt_local;
    v[1] = (double)dt3;
  }, U_DTMIN);
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

// Pull the scalar slots to the host (one sync).
template <class R>
cudaError_t pull_scalars(Run<R>& run) {
  cudaMemcpyAsync(run.host_sc, run.sc, SC_NSLOTS * sizeof(double), cudaMemcpyDeviceToHost, run.s);
  return cudaStreamSynchronize(run.s);
}

// ---------------------------------------------------------------------
// lagran.F90:208-478 predictor_corrector_step (non-CAUCHY, no cooling).
template <class R>
void predictor_corrector_step(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  Arrays<R>& A = run.a;
  copy_whole(run, A.bx0, A.bx);
  copy_whole(run, A.by0, A.by);
  copy_whole(run, A.bz0, A.bz);
  // b_field_and_cv1_update (:945-1062): the cv1 it forms (:952-983) is
  // overwritten by the first predictor sweep before any read.
  copy_whole(run, A.vx1, A.vx);
  copy_whole(run, A.vy1, A.vy);
  copy_whole(run, A.vz1, A.vz);
  eulerian_remap(run, run.cur_step, true);
  // bx1 = bx1 * cv1 (:230-232) only feeds the CAUCHY branch.
  auto cv1 = A.cv1, cv = A.cv, energy = A.energy, pressure = A.pressure, rho = A.rho, visc_heat = A.visc_heat;
  const R g = (R)run.p.gamma, xi = (R)run.p.xi_n, ip = (R)run.p.ionise_pot;
  const double* sc = run.sc;
  LARE_BOXW(run, 7, 0, nx + 1, 0, ny + 1, 0, nz + 1, [=] __device__(int ix, int iy, int iz) {
    const R dt2 = (R)sc[SC_DT2];
    R dv = cv1(ix, iy, iz) / cv(ix, iy, iz) - R(1);
    R e1 = energy(ix, iy, iz) - pressure(ix, iy, iz) * dv / rho(ix, iy, iz);
    e1 = e1 + visc_heat(ix, iy, iz) * dt2 / rho(ix, iy, iz);
    pressure(ix, iy, iz) = (e1 - (R(1) - xi) * ip) * (g - R(1)) * rho(ix, iy, iz) * cv(ix, iy, iz) / cv1(ix, iy, iz);
  });
  auto bx = A.bx, by = A.by, bz = A.bz, gamma_boris = A.gamma_boris, rho_v = A.rho_v;
  auto vx = A.vx, vy = A.vy, vz = A.vz, vx1 = A.vx1, vy1 = A.vy1, vz1 = A.vz1;
  auto fx_visc = A.fx_visc, fy_visc = A.fy_visc, fz_visc = A.fz_visc;
  auto dxc = A.dxc, dyc = A.dyc, dzc = A.dzc, grav = A.grav;
  LARE_BOXW(run, 16, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz) {
    const R dt2 = (R)sc[SC_DT2];
    int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
    R pp = pressure(ix, iy, iz), ppx = pressure(ixp, iy, iz), ppy = pressure(ix, iyp, iz);
    R ppz = pressure(ix, iy, izp), ppxy = pressure(ixp, iyp, iz), ppxz = pressure(ixp, iy, izp);
    R ppyz = pressure(ix, iyp, izp), ppxyz = pressure(ixp, iyp, izp);
    R w1 = (pp + ppy + ppz + ppyz) * R(0.25);
    R w2 = (ppx + ppxy + ppxz + ppxyz) * R(0.25);
    R fx = -(w2 - w1) / dxc(ix);
    w1 = (pp + ppx + ppz + ppxz) * R(0.25);
    w2 = (ppy + ppxy + ppyz + ppxyz) * R(0.25);
    R fy = -(w2 - w1) / dyc(iy);
    w1 = (pp + ppx + ppy + ppxy) * R(0.25);
    w2 = (ppz + ppxz + ppyz + ppxyz) * R(0.25);
    R fz = -(w2 - w1) / dzc(iz);
    R bxv = R(0.25) * (bx(ix, iy, iz) + bx(ix, iyp, iz) + bx(ix, iy, izp) + bx(ix, iyp, izp));
    R byv = R(0.25) * (by(ix, iy, iz) + by(ixp, iy, iz) + by(ix, iy, izp) + by(ixp, iy, izp));
    R bzv = R(0.25) * (bz(ix, iy, iz) + bz(ix, iyp, iz) + bz(ixp, iy, iz) + bz(ixp, iyp, iz));
    R jx1 = (bz(ix, iyp, iz) - bz(ix, iy, iz)) / dyc(iy) - (by(ix, iy, izp) - by(ix, iy, iz)) / dzc(iz);
    R jx2 = (bz(ixp, iyp, iz) - bz(ixp, iy, iz)) / dyc(iy) - (by(ixp, iy, izp) - by(ixp, iy, iz)) / dzc(iz);
    R jy1 = (bx(ix, iy, izp) - bx(ix, iy, iz)) / dzc(iz) - (bz(ixp, iy, iz) - bz(ix, iy, iz)) / dxc(ix);
    R jy2 = (bx(ix, iyp, izp) - bx(ix, iyp, iz)) / dzc(iz) - (bz(ixp, iyp, iz) - bz(ix, iyp, iz)) / dxc(ix);
    R jz1 = (by(ixp, iy, iz) - by(ix, iy, iz)) / dxc(ix) - (bx(ix, iyp, iz) - bx(ix, iy, iz)) / dyc(iy);
    R jz2 = (by(ixp, iy, izp) - by(ix, iy, izp)) / dxc(ix) - (bx(ix, iyp, izp) - bx(ix, iy, izp)) / dyc(iy);
    R jx = (jx1 + jx2) * R(0.5), jy = (jy1 + jy2) * R(0.5), jz = (jz1 + jz2) * R(0.5);
    R gb = gamma_boris(ix, iy, iz);
    fx = fx + gb * (jy * bzv - jz * byv);
    fy = fy + gb * (jz * bxv - jx * bzv);
    fz = fz + gb * (jx * byv - jy * bxv);
    fz = fz - rho_v(ix, iy, iz) * grav(iz);
    R rv = rho_v(ix, iy, iz);
    vx1(ix, iy, iz) = vx(ix, iy, iz) + dt2 * (fx_visc(ix, iy, iz) + fx) / rv;
    vy1(ix, iy, iz) = vy(ix, iy, iz) + dt2 * (fy_visc(ix, iy, iz) + fy) / rv;
    vz1(ix, iy, iz) = vz(ix, iy, iz) + dt2 * (fz_visc(ix, iy, iz) + fz) / rv;
  });
  copy_whole(run, A.bx, A.bx0);
  copy_whole(run, A.by, A.by0);
  copy_whole(run, A.bz, A.bz0);
  remap_v_bcs(run);
  shock_heating(run);
  LARE_BOXW(run, 9, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz) {
    vx(ix, iy, iz) = R(2) * vx1(ix, iy, iz) - vx(ix, iy, iz);
    vy(ix, iy, iz) = R(2) * vy1(ix, iy, iz) - vy(ix, iy, iz);
    vz(ix, iy, iz) = R(2) * vz1(ix, iy, iz) - vz(ix, iy, iz);
  });
  velocity_bcs(run);
  // Final density and energy (:415-462) with the total_visc_heating sum.
  auto visc_dep = A.visc_dep;
  auto dxb = A.dxb, dyb = A.dyb, dzb = A.dzb;
  box_sum<1>(run, 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz, double* v) {
    const R dt = (R)sc[SC_DT];
    int ixm = ix - 1, iym = iy - 1, izm = iz - 1;
    R vxb = (vx1(ix, iy, iz) + vx1(ix, iym, iz) + vx1(ix, iy, izm) + vx1(ix, iym, izm)) * R(0.25);
    R vxbm = (vx1(ixm, iy, iz) + vx1(ixm, iym, iz) + vx1(ixm, iy, izm) + vx1(ixm, iym, izm)) * R(0.25);
    R vyb = (vy1(ix, iy, iz) + vy1(ixm, iy, iz) + vy1(ix, iy, izm) + vy1(ixm, iy, izm)) * R(0.25);
    R vybm = (vy1(ix, iym, iz) + vy1(ixm, iym, iz) + vy1(ix, iym, izm) + vy1(ixm, iym, izm)) * R(0.25);
    R vzb = (vz1(ix, iy, iz) + vz1(ixm, iy, iz) + vz1(ix, iym, iz) + vz1(ixm, iym, iz)) * R(0.25);
    R vzbm = (vz1(ix, iy, izm) + vz1(ixm, iy, izm) + vz1(ix, iym, izm) + vz1(ixm, iym, izm)) * R(0.25);
    R dv = ((vxb - vxbm) / dxb(ix) + (vyb - vybm) / dyb(iy) + (vzb - vzbm) / dzb(iz)) * dt;
    cv1(ix, iy, iz) = cv(ix, iy, iz) * (R(1) + dv);
    R vh = visc_heat(ix, iy, iz);
    energy(ix, iy, iz) = energy(ix, iy, iz) + (dt * vh - dv * pressure(ix, iy, iz)) / rho(ix, iy, iz);
    visc_dep(ix, iy, iz) = visc_dep(ix, iy, iz) + dt * vh;
    rho(ix, iy, iz) = rho(ix, iy, iz) / (R(1) + dv);
    v[0] = (double)(dt * vh * cv(ix, iy, iz));
  }, SC_VISC_TOT, true);
}

// ---------------------------------------------------------------------
// lagran.F90:50-200 lagrangian_step
template <class R>
int lagrangian_step(Run<R>& run, int step) {
  run.cur_step = step;
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  Arrays<R>& A = run.a;
  auto bx = A.bx, by = A.by, bz = A.bz, bx1 = A.bx1, by1 = A.by1, bz1 = A.bz1;
  auto rho = A.rho, energy = A.energy, pressure = A.pressure, cv = A.cv, rho_v = A.rho_v, cv_v = A.cv_v;
  const R g = (R)run.p.gamma, xi = (R)run.p.xi_n, ip = (R)run.p.ionise_pot;
  LARE_BOXW(run, 9, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
    int ixm = ix - 1, iym = iy - 1, izm = iz - 1;
    bx1(ix, iy, iz) = (bx(ix, iy, iz) + bx(ixm, iy, iz)) * R(0.5);
    by1(ix, iy, iz) = (by(ix, iy, iz) + by(ix, iym, iz)) * R(0.5);
    bz1(ix, iy, iz) = (bz(ix, iy, iz) + bz(ix, iy, izm)) * R(0.5);
    pressure(ix, iy, iz) = (g - R(1)) * rho(ix, iy, iz) * (energy(ix, iy, iz) - (R(1) - xi) * ip);
  });
  LARE_BOXW(run, 4, -1, nx + 1, -1, ny + 1, -1, nz + 1, [=] __device__(int ix, int iy, int iz) {
    int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
    R rv = rho(ix, iy, iz) * cv(ix, iy, iz) + rho(ixp, iy, iz) * cv(ixp, iy, iz) + rho(ix, iyp, iz) * cv(ix, iyp, iz) +
           rho(ixp, iyp, iz) * cv(ixp, iyp, iz) + rho(ix, iy, izp) * cv(ix, iy, izp) +
           rho(ixp, iy, izp) * cv(ixp, iy, izp) + rho(ix, iyp, izp) * cv(ix, iyp, izp) +
           rho(ixp, iyp, izp) * cv(ixp, iyp, izp);
    R cvv = cv(ix, iy, iz) + cv(ixp, iy, iz) + cv(ix, iyp, iz) + cv(ixp, iyp, iz) + cv(ix, iy, izp) +
            cv(ixp, iy, izp) + cv(ix, iyp, izp) + cv(ixp, iyp, izp);
    rho_v(ix, iy, iz) = rv / cvv;
    cv_v(ix, iy, iz) = R(0.125) * cvv;
  });
  if (run.p.use_viscous_damping) viscous_damping(run);
  shock_viscosity(run);
  set_dt(run);

  double* sc = run.sc;
  run.last_substeps = 0;
  if (run.p.resistive_mhd) {
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
    for (int sc_i = 1; sc_i <= substeps; ++sc_i) {
      eta_calc(run);
      resistive_effects(run);
    }
    LARE_BOXW(run, 6, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
      int ixm = ix - 1, iym = iy - 1, izm = iz - 1;
      bx1(ix, iy, iz) = (bx(ix, iy, iz) + bx(ixm, iy, iz)) * R(0.5);
      by1(ix, iy, iz) = (by(ix, iy, iz) + by(ix, iym, iz)) * R(0.5);
      bz1(ix, iy, iz) = (bz(ix, iy, iz) + bz(ix, iy, izm)) * R(0.5);
    });
  }
  // :168-181 energy0 / delta_energy
  auto energy0 = A.energy0;
  if (run.p.conduction) {
    copy_whole(run, energy0, energy);
    calc_s_stages(run, SC_DT);
    if (pull_scalars(run) != cudaSuccess) return LARE_ECUDA;
    int ns = (int)run.host_sc[SC_STAGES];
    if (ns < 1 || ns > 100000) return LARE_ESTAGES;
    run.n_s_stages = ns;
    heat_conduct_sts2(run, SC_DT);
    // energy = energy0 + (energy - energy0), then MAX(energy, 0)
    whole(run, [=] __device__(int i, int j, int k) {
      if (i >= -1 && j >= -1 && k >= -1) {
        R e0 = energy0(i, j, k);
        R d = energy(i, j, k) - e0;
        R e = e0 + d;
        energy(i, j, k) = e > R(0) ? e : R(0);
      }
    });
  } else {
    whole(run, [=] __device__(int i, int j, int k) {
      if (i >= -1 && j >= -1 && k >= -1) {
        R e = energy(i, j, k) + R(0);
        energy(i, j, k) = e > R(0) ? e : R(0);
      }
    });
  }
  predictor_corrector_step(run);
  energy_bcs(run);
  density_bcs(run);
  velocity_bcs(run);
  ++run.steps_taken;
  return LARE_OK;
}

// ---------------------------------------------------------------------
// diagnostics.F90:517-609 energy_account into sc[SC_EN_B..SC_EN_INT].
template <class R>
void energy_account(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  Arrays<R>& A = run.a;
  auto bx = A.bx, by = A.by, bz = A.bz, cv = A.cv, energy = A.energy, rho = A.rho;
  auto vx = A.vx, vy = A.vy, vz = A.vz;
  box_sum<2>(run, 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz, double* v) {
    int ixm = ix - 1, iym = iy - 1, izm = iz - 1;
    double b0 = bx(ix, iy, iz), b1 = bx(ixm, iy, iz), c0 = by(ix, iy, iz), c1 = by(ix, iym, iz);
    double d0 = bz(ix, iy, iz), d1 = bz(ix, iy, izm);
    double w1 = (b0 * b0 + b1 * b1) * 0.5;
    double w2 = (c0 * c0 + c1 * c1) * 0.5;
    double w3 = (d0 * d0 + d1 * d1) * 0.5;
    w1 = (w1 + w2 + w3) * 0.5;
    v[0] = w1 * (double)cv(ix, iy, iz);
    v[1] = (double)energy(ix, iy, iz) * (double)rho(ix, iy, iz) * (double)cv(ix, iy, iz);
  }, SC_EN_B, false);
  // SC_EN_B and SC_EN_B+1 hold en_b and en_int; move en_int to its slot.
  double* sc = run.sc;
  launch_scalar(run.s, run.launches, [=] __device__() { sc[SC_EN_INT] = sc[SC_EN_B + 1]; });
  box_sum<1>(run, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz, double* v) {
    int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
    auto r = [&](int a, int b, int c) { return (double)rho(a, b, c) * (double)cv(a, b, c); };
    auto w = [&](int a, int b, int c) { return (double)cv(a, b, c); };
    double rv = r(ix, iy, iz) + r(ixp, iy, iz) + r(ix, iyp, iz) + r(ixp, iyp, iz) + r(ix, iy, izp) + r(ixp, iy, izp) +
                r(ix, iyp, izp) + r(ixp, iyp, izp);
    double cvv = w(ix, iy, iz) + w(ixp, iy, iz) + w(ix, iyp, iz) + w(ixp, iyp, iz) + w(ix, iy, izp) + w(ixp, iy, izp) +
                 w(ix, iyp, izp) + w(ixp, iyp, izp);
    rv = rv / cvv;
    cvv = cvv * 0.125;
    double ux = vx(ix, iy, iz), uy = vy(ix, iy, iz), uz = vz(ix, iy, iz);
    double w1 = rv * cvv * (ux * ux + uy * uy + uz * uz);
    if (ix == 0 || ix == nx) w1 = w1 * 0.5;
    if (iy == 0 || iy == ny) w1 = w1 * 0.5;
    if (iz == 0 || iz == nz) w1 = w1 * 0.5;
    v[0] = w1 * 0.5;
  }, SC_EN_KE, false);
}

}  // namespace lare
