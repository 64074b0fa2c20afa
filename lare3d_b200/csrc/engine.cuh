// engine.cuh - the Lagrangian-remap timestep on the device.
//
// Each routine below corresponds to a routine of the reference (file:line
// cited) and launches one kernel per reference loop nest over exactly the
// same index box, with the same left-to-right expression order.  Compiled
// with --fmad=false for FP64 (engine_f64.cu) the arithmetic is then
// bit-for-bit that of a gfortran -O3 x86-64 build of the reference, which
// emits no FMA.  Conduction is the exception: it forms T^2.5 and T^1.5 as
// T*T*sqrt(T) and T*sqrt(T) where the reference calls pow(), so its results
// differ in the last bits.  engine_f32.cu instantiates the same code in FP32
// (the FP32 form).
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

LARE_BEGIN

struct Par {
  double gamma, visc1, visc2, eta_background, eta0, j_max, kappa_0, flux_limiter;
  double ionise_pot, xi_n, va_max, dt_multiplier, dt_from_restart, kappa_perp_ratio;
  int resistive_mhd, conduction, heat_flux_limiter, use_viscous_damping, boris, restart;
  int eos_number, cowling_resistivity;                 // neutral.f90 (eos_number 0 read as EOS_IDEAL)
  double f_bar, t_bar, r_bar, tr, eta_bar;
  int radiation;                                       // radiative.f90
  int rke;                                             // the remap's kinetic-energy correction
  int cooling_term;                                    // lagran.F90:464, :1290
  double alpha_av;
  int coronal_heating;                                 // lagran.F90:127
  double temp_norm, time_norm, rho_norm, mf;
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
  A3<R> larsen, Y1, Y2, Y3, Lc_Y0;  // RKL2 (Y0 is read from energy itself)
  A3<R> kf[9];                        // stage-invariant face coefficients, 3 per face direction
  // neutral.f90 (allocated only for a partially ionised run)
  A3<R> xi, eta_perp;
  // the energy after rad_losses (radiative.f90), allocated with radiation on
  A3<R> erad;
  // rke: the remap's kinetic-energy defect (shared_data.F90:108) and the
  // three momentum fluxes before their product with dm
  A3<R> delta_ke, rke_f[3], rke_dk[3];
  // cooling_term: moving averages of the viscous and ohmic heating
  // (shared_data.F90:109), persistent across steps
  A3<R> cool_term_v, cool_term_b;
  // coronal_heating: the user's heating rate (user_defined_heating's heat_in)
  A3<R> heat_in;
  // 1-D metrics (pointers at Fortran index 0)
  A1<R> dxb, dxc, dyb, dyc, dzb, dzc, grav;
  // reciprocals for conduction: 1/dxb, 1/dxc, 1/(dxc(i) + dxc(i-1)), per axis
  A1<R> rdb[3], rdc[3], rdc2[3];
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
  std::map<std::pair<std::string, int>, int> index;  // by name and line (the same name in several template instances is one site)
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
  bool any_open = false;            // some side has BC_OPEN (boundary.f90:35-38)
  bool pip = false;                 // eos_number /= EOS_IDEAL: xi_n is the per-cell array a.xi
  bool cowling = false;             // cowling_resistivity: eta_perp in set_dt and rkstep
  int cur_step = 0;
  int peak_substeps = 0, last_substeps = 0, steps_taken = 0, n_s_stages = 0;
  int blk_x = 32, blk_y = 4;            // block shape of the point kernels (measured best at 256^3)
  bool capturing = false;               // recording a CUDA graph of whole steps
  cudaStream_t s_body = nullptr;        // captures the body of the resistive sub-cycle loop
  GSpec g_cell, g_node, g_bx, g_by, g_bz, g_cell_mpi, g_cell_user, g_dm[3];
  Prof prof;
  std::string err;

  // Bracket one launch with events when profiling.
  int prof_begin(const char* func, int line, int words, double points) {
    if (!prof.on) return -1;
    auto key = std::make_pair(std::string(func), line);
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
template <int MINB64 = 0, int ZP32 = 1, class R, class Fn>
inline void rbox(Run<R>& run, const char* func, int line, int words, int i0, int i1, int j0, int j1, int k0, int k1,
                 Fn fn) {
  double pts = (double)(i1 - i0 + 1) * (double)(j1 - j0 + 1) * (double)(k1 - k0 + 1);
  int k = run.prof_begin(func, line, words, pts);
  launch_box<sizeof(R) == 8 ? MINB64 : 0, sizeof(R) == 4 ? ZP32 : 1>(run.s, run.launches, i0, i1, j0, j1, k0, k1, fn, run.blk_x, run.blk_y);
  run.prof_end(k);
}
// LARE_BOX: one kernel over an inclusive Fortran index box.  LARE_BOXW also
// states the kernel's algorithmic word count per point (arrays read +
// written), used for the roofline of profiled launches.  LARE_BOXWB adds an
// occupancy hint for the FP64 build (k_box_mb's MINB): latency-bound stencils
// with many live values run faster with a register cap that lets more
// blocks share an SM (measured per kernel at 256^3; FP32 keeps the default).
#define LARE_BOX(run, i0, i1, j0, j1, k0, k1, ...) \
  rbox((run), __func__, __LINE__, 0, (i0), (i1), (j0), (j1), (k0), (k1), __VA_ARGS__)
#define LARE_BOXW(run, words, i0, i1, j0, j1, k0, k1, ...) \
  rbox((run), __func__, __LINE__, (words), (i0), (i1), (j0), (j1), (k0), (k1), __VA_ARGS__)
#define LARE_BOXWB(run, minb, words, i0, i1, j0, j1, k0, k1, ...) \
  rbox<minb>((run), __func__, __LINE__, (words), (i0), (i1), (j0), (j1), (k0), (k1), __VA_ARGS__)
// LARE_BOXWH: both hints, the FP64 occupancy hint and the FP32 planes per
// thread (k_box_z's ZP), each measured per kernel at 256^3.
#define LARE_BOXWH(run, minb64, zp32, words, i0, i1, j0, j1, k0, k1, ...) \
  rbox<minb64, zp32>((run), __func__, __LINE__, (words), (i0), (i1), (j0), (j1), (k0), (k1), __VA_ARGS__)

// Some kernels write an array's new values into a second buffer that is
// then swapped in, covering only the points the reference updates (which it
// does in place, so every other point keeps its old value).  Periodic and
// BC_USER ghost fills rewrite every ghost right after; an open side is never
// refilled, so with an open side every point of the array's bounds [lo, hi]
// outside the updated box [a, b] is carried from the old buffer.
// The shell [lo, hi] minus [a, b] as six disjoint slabs (x below and above
// over the whole y, z range, then y below and above within a's x range,
// then z below and above within a's x and y ranges), walked by one flat
// index; up to three arrays share the walk.
template <class R>
struct CarryArgs {
  R* dst[3];
  const R* src[3];
  int narr, sx, sxy;
  int box[6][6];         // i0, i1, j0, j1, k0, k1 per slab
  long long start[7];    // first flat index of each slab; start[6] = total
};

template <class R>
__global__ void __launch_bounds__(256) k_carry(CarryArgs<R> g) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.start[6]) return;
  int s = 0;
  while (t >= g.start[s + 1]) ++s;  // at most five steps
  const int* q = g.box[s];
  const long long r = t - g.start[s];
  const long long e0 = q[1] - q[0] + 1, e1 = q[3] - q[2] + 1;
  const int i = q[0] + (int)(r % e0);
  const int j = q[2] + (int)((r / e0) % e1);
  const int k = q[4] + (int)(r / (e0 * e1));
  const int c = i + g.sx * j + g.sxy * k;
  for (int m = 0; m < g.narr; ++m) g.dst[m][c] = g.src[m][c];
}

template <class R>
inline void carry_outside_n(Run<R>& run, int narr, R* const* dst, const R* const* src, const int lo[3],
                            const int hi[3], const int a[3], const int b[3]) {
  if (!run.any_open) return;
  CarryArgs<R> g;
  g.narr = narr;
  g.sx = run.sx;
  g.sxy = run.sxy;
  for (int m = 0; m < 3; ++m) {
    g.dst[m] = m < narr ? dst[m] : nullptr;
    g.src[m] = m < narr ? src[m] : nullptr;
  }
  const int slab[6][6] = {
      {lo[0], a[0] - 1, lo[1], hi[1], lo[2], hi[2]}, {b[0] + 1, hi[0], lo[1], hi[1], lo[2], hi[2]},
      {a[0], b[0], lo[1], a[1] - 1, lo[2], hi[2]},   {a[0], b[0], b[1] + 1, hi[1], lo[2], hi[2]},
      {a[0], b[0], a[1], b[1], lo[2], a[2] - 1},     {a[0], b[0], a[1], b[1], b[2] + 1, hi[2]}};
  long long tot = 0;
  for (int s = 0; s < 6; ++s) {
    for (int d = 0; d < 6; ++d) g.box[s][d] = slab[s][d];
    g.start[s] = tot;
    const long long n0 = slab[s][1] - slab[s][0] + 1, n1 = slab[s][3] - slab[s][2] + 1,
                    n2 = slab[s][5] - slab[s][4] + 1;
    if (n0 > 0 && n1 > 0 && n2 > 0) tot += n0 * n1 * n2;
  }
  g.start[6] = tot;
  if (tot == 0) return;
  const int k = run.prof_begin("carry_outside", 0, 2 * narr, (double)tot);
  k_carry<R><<<(unsigned)((tot + 255) / 256), 256, 0, run.s>>>(g);
  run.prof_end(k);
  ++run.launches;
}

template <class R>
inline void carry_outside(Run<R>& run, R* dst, const R* src, const int lo[3], const int hi[3], const int a[3],
                          const int b[3]) {
  R* const d[1] = {dst};
  const R* const s[1] = {src};
  carry_outside_n(run, 1, d, s, lo, hi, a, b);
}

// the three velocity components after an update of the nodes 0:n
template <class R>
inline void carry_velocity(Run<R>& run, R* const nv[3], R* const ov[3]) {
  const int lo[3] = {-2, -2, -2}, hi[3] = {run.n[0] + 2, run.n[1] + 2, run.n[2] + 2};
  const int a[3] = {0, 0, 0}, b[3] = {run.n[0], run.n[1], run.n[2]};
  const R* const src[3] = {ov[0], ov[1], ov[2]};
  carry_outside_n(run, 3, nv, src, lo, hi, a, b);
}

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
// site names the launch in the profile; words: the algorithmic words per
// point the kernel moves.
template <int NV, class R, class Fn>
inline void box_sum(Run<R>& run, const char* site, int i0, int i1, int j0, int j1, int k0, int k1, Fn fn, int slot,
                    bool acc, int words = 0, int planes = kSumPlanes) {
  int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
  dim3 blk(64, 4, 1);
  dim3 grd((ni + 63) / 64, (nj + 3) / 4, (nk + planes - 1) / planes);
  int nb = grd.x * grd.y * grd.z;
  int k = run.prof_begin(site, 0, words, (double)ni * nj * nk);
  k_box_sum<NV><<<grd, blk, 0, run.s>>>(i0, j0, k0, ni, nj, nk, planes, fn, run.partial);
  k_sum_partials<NV><<<1, 1024, 0, run.s>>>(run.partial, nb, run.sc + slot, acc ? 1 : 0);
  run.prof_end(k);
  run.launches += 2;
}

template <int NV, class R, class Fn>
inline void box_min(Run<R>& run, const char* site, int i0, int i1, int j0, int j1, int k0, int k1, Fn fn, int uslot,
                    int words = 0) {
  int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
  // planes per block: fewer blocks contend for the atomic, at the cost of
  // resident warps; measured at 256^3: 8 in FP32 (0.23 -> 0.18 ms for set_dt),
  // 1 in FP64 (8 took 0.38 -> 0.42 ms)
  constexpr int kMinPlanes = sizeof(R) == 4 ? 8 : 1;
  dim3 blk(64, 4, 1);
  dim3 grd((ni + 63) / 64, (nj + 3) / 4, (nk + kMinPlanes - 1) / kMinPlanes);
  int k = run.prof_begin(site, 0, words, (double)ni * nj * nk);
  k_box_min<NV><<<grd, blk, 0, run.s>>>(i0, j0, k0, ni, nj, nk, kMinPlanes, fn, run.us + uslot);
  run.prof_end(k);
  ++run.launches;
}

// ---------------------------------------------------------------------
// boundary.f90 fills, batched: every group of fills the reference performs
// back to back goes out as one launch (one job per array kind).
template <class R>
struct GhostBatch {
  GJobs<R> J;
  long long maxtot = 0;
  GhostBatch() { J.n = 0; }
  void add(const GSpec& g, R* p0, R* p1 = nullptr, R* p2 = nullptr) {
    J.s[J.n] = g;
    J.p[J.n][0] = p0;
    J.p[J.n][1] = p1;
    J.p[J.n][2] = p2;
    long long t = g.c0 + g.c1 + g.c2;
    if (t > maxtot) maxtot = t;
    ++J.n;
  }
};
template <class R>
inline void ghost_flush(Run<R>& run, GhostBatch<R>& b) {
  if (b.J.n == 0 || b.maxtot == 0) return;
  dim3 grd((unsigned)((b.maxtot + 255) / 256), (unsigned)b.J.n);
  int k = run.prof_begin("ghost", 0, 0, (double)b.maxtot * b.J.n);
  k_ghost_multi<R><<<grd, 256, 0, run.s>>>(b.J, run.sx, run.sxy);
  run.prof_end(k);
  ++run.launches;
}
template <class R> inline void energy_bcs(Run<R>& r) { GhostBatch<R> b; b.add(r.g_cell, r.a.energy.p); ghost_flush(r, b); }
template <class R> inline void density_bcs(Run<R>& r) { GhostBatch<R> b; b.add(r.g_cell, r.a.rho.p); ghost_flush(r, b); }
template <class R> inline void velocity_bcs(Run<R>& r) {
  GhostBatch<R> b;
  b.add(r.g_node, r.a.vx.p, r.a.vy.p, r.a.vz.p);
  ghost_flush(r, b);
}
template <class R> inline void remap_v_bcs(Run<R>& r) {
  GhostBatch<R> b;
  b.add(r.g_node, r.a.vx1.p, r.a.vy1.p, r.a.vz1.p);
  ghost_flush(r, b);
}
template <class R> inline void bfield_bcs(Run<R>& r) {
  GhostBatch<R> b;
  b.add(r.g_bx, r.a.bx.p);
  b.add(r.g_by, r.a.by.p);
  b.add(r.g_bz, r.a.bz.p);
  ghost_flush(r, b);
}
// boundary.f90:212 temperature_bcs exchanges rho (:214), then mirrors T.
template <class R> inline void temperature_bcs(Run<R>& r) {
  GhostBatch<R> b;
  b.add(r.g_cell_mpi, r.a.rho.p);
  b.add(r.g_cell_user, r.a.temperature.p);
  ghost_flush(r, b);
}
// boundary.f90:48-55 boundary_conditions
template <class R> inline void boundary_conditions(Run<R>& r) {
  GhostBatch<R> b;
  b.add(r.g_bx, r.a.bx.p);
  b.add(r.g_by, r.a.by.p);
  b.add(r.g_bz, r.a.bz.p);
  b.add(r.g_cell, r.a.energy.p, r.a.rho.p);
  b.add(r.g_node, r.a.vx.p, r.a.vy.p, r.a.vz.p);
  ghost_flush(r, b);
}
// energy_bcs + density_bcs at the end of lagrangian_step (lagran.F90:196-197)
template <class R> inline void end_of_step_bcs(Run<R>& r) {
  GhostBatch<R> b;
  b.add(r.g_cell, r.a.energy.p, r.a.rho.p);
  ghost_flush(r, b);
}

// Full-array elementwise helpers (Fortran whole-array statements).
template <class R, class Fn>
inline void whole(Run<R>& r, Fn fn) {
  LARE_BOX(r, -2, r.n[0] + 2, -2, r.n[1] + 2, -2, r.n[2] + 2, fn);
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
  R rho_edge = qdiv(R(2) * r1 * r2, r1 + r2);
  R cs_edge = fmin(c1, c2);
  R dv2 = dvx * dvx + dvy * dvy + dvz * dvz;
  R dv = sqrt(dv2);
  R psi = R(0);
  if (qdiv(dv * dt, dx) < R(1.e-14)) dvdots = R(0);
  else dvdots = qdiv(dvdots, dv);
  R vc = visc1 * cs_edge;
  R q_k_bar = rho_edge * (visc2_norm * dv + sqrt(visc2_norm * visc2_norm * dv2 + vc * vc));
  return q_k_bar * (R(1) - psi) * dvdots;
}

// ---------------------------------------------------------------------
// x^2.5 and x^1.5 as x*x*sqrt(x) and x*sqrt(x): within an ulp or two of
// pow() and several times cheaper (the reference calls pow, so conduction is
// compared with the oracle at a 1e-12 relative tolerance, not bitwise).
template <class R>
__device__ __forceinline__ R pow25(R x) { return x * x * sqrt(x); }
template <class R>
__device__ __forceinline__ R pow15(R x) { return x * sqrt(x); }

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
  const bool pip = run.pip;
  auto xia = run.a.xi;  // per-cell xi_n when partially ionised
  LARE_BOXW(run, 2, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
    const R x = pip ? xia(ix, iy, iz) : xi;
    temperature(ix, iy, iz) = (g - R(1)) / (R(2) - x) * (energy(ix, iy, iz) - (R(1) - x) * ip);
  });
  LARE_BOXW(run, 3, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz) {
    if (!limiter) { larsen(ix, iy, iz) = R(1); return; }
    int ixm = ix - 1, ixp = ix + 1, iym = iy - 1, iyp = iy + 1, izm = iz - 1, izp = iz + 1;
    R T = temperature(ix, iy, iz);
    R temp = pow25(T);
    R q_fs = fl * R(42.85) * rho(ix, iy, iz) * pow15(T);
    R q_fs2 = q_fs * q_fs;
    R q_spx = -k0 * temp * (temperature(ixp, iy, iz) - temperature(ixm, iy, iz)) * R(0.5) / dxb(ix);
    R q_spy = -k0 * temp * (temperature(ix, iyp, iz) - temperature(ix, iym, iz)) * R(0.5) / dyb(iy);
    R q_spz = -k0 * temp * (temperature(ix, iy, izp) - temperature(ix, iy, izm)) * R(0.5) / dzb(iz);
    R q_sp2 = q_spx * q_spx + q_spy * q_spy + q_spz * q_spz;
    larsen(ix, iy, iz) = q_fs / sqrt(q_fs2 + q_sp2);
  });
  unsigned long long* us = run.us;
  launch_scalar(run.s, run.launches, [=] __device__() { us[U_DTPARAB] = (unsigned long long)__double_as_longlong(1.e10); });
  box_min<1>(run, "parabolic_dt_min", 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz, double* v) {
    R kappa1 = k0 * larsen(ix, iy, iz);
    const R x = pip ? xia(ix, iy, iz) : xi;
    R temp = (g - R(1)) / (R(2) - x) * (energy(ix, iy, iz) - (R(1) - x) * ip);
    R tp = pow25(temp);
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

// Temperature of an energy-like array, conduct.f90:68 and :371-374,
// evaluated where it is needed instead of stored.
template <class R>
struct TempOf {
  A3<R> y;
  R c, e0;  // (gamma - 1)/(2 - xi_n), (1 - xi_n)*ionise_pot
  __device__ __forceinline__ R operator()(int i, int j, int k) const { return c * (y(i, j, k) - e0); }
};

template <class R>
void temperature_from(Run<R>& run, A3<R> e) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  auto temperature = run.a.temperature;
  const R g = (R)run.p.gamma, xi = (R)run.p.xi_n, ip = (R)run.p.ionise_pot;
  const bool pip = run.pip;
  auto xia = run.a.xi;
  LARE_BOXW(run, 2, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
    const R x = pip ? xia(ix, iy, iz) : xi;
    temperature(ix, iy, iz) = (g - R(1)) / (R(2) - x) * (e(ix, iy, iz) - (R(1) - x) * ip);
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

LARE_END  // namespace lare

#include "neutral.cuh"
#include "radiative.cuh"
#include "conduct.cuh"

LARE_BEGIN

// conduct.f90:299-416 heat_conduct_sts2, dt from sc[dt_slot]; the stage
// count s must already be known on the host (run.n_s_stages).
//
// The reference keeps Y(0:3) and copies whole arrays between stages
// (Y1 = Y2; energy = Y3; energy_bcs; Y2 = energy).  Here the stages rotate
// three buffers instead, with Y0 read straight from `energy` (untouched
// until the end), and the temperature of Y2 is formed where the flux needs
// it.  The values are the same as the reference's, including its boundary
// detail: the temperature ghosts of stage 2 in MPI/periodic directions come
// from Y2's ghost cells, which still hold the energy's (temperature_bcs
// refreshes only BC_USER faces), so Y2 starts as a whole copy of energy and
// gets only the BC_USER fill before stage 2; from stage 3 on, Y2 is the
// previous Y3 after the full energy boundary fill.
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
  auto energy = A.energy;
  const R g = (R)run.p.gamma, xi = (R)run.p.xi_n, ip = (R)run.p.ionise_pot;
  const R tc = (g - R(1)) / (R(2) - xi), te0 = (R(1) - xi) * ip;
  // With a per-cell xi_n (partially ionised) the temperature changes with
  // xi_n between stages, so each stage forms it into the temperature array
  // exactly as conduct.f90:346-376 does, and the stage reads it back
  // through 1 * (T - 0) = T.
  const bool pip = run.pip;
  auto temp = [&](A3<R> y) { return pip ? TempOf<R>{A.temperature, R(1), R(0)} : TempOf<R>{y, tc, te0}; };
  if (s < 2) {
    // The stage loop is empty and energy(1:n) = Y(3)(1:n) = energy: the
    // reference leaves the energy unchanged (conduct.f90:409).
    energy_bcs(run);
    return;
  }
  // rotating buffers: Y0 = energy (read only), Y1 = energy for stage 2
  A3<R> bufs[3] = {A.Y1, A.Y2, A.Y3};
  A3<R> Y1 = energy, Y2 = bufs[0], Y3 = bufs[1];
  int next_free = 2;
  copy_whole(run, Y2, energy);
  if (run.any_open) {
    // The reference's Y(3) keeps the energy's ghosts throughout (only
    // 1:n is written), and energy_bcs leaves an open side's ghosts alone:
    // every stage buffer starts as the energy so that those ghosts match.
    copy_whole(run, bufs[1], energy);
    copy_whole(run, bufs[2], energy);
  }
  face_coefficients(run);
  if (pip) temperature_from(run, energy);
  rkl2_stage<R, true>(run, __LINE__, temp(energy), energy, energy, energy, Y2, dt_slot, (R)mu_tilde[1], R(0), R(0),
                      R(0), R(0));
  ghost(run, run.g_cell_user, Y2);
  {
    GhostBatch<R> bb;
    bb.add(run.g_cell_mpi, A.rho.p);  // density_mpi of temperature_bcs (a no-op on a consistent rho)
    ghost_flush(run, bb);
  }
  for (int j = 2; j <= s; ++j) {
    const R gt = (R)gamma_tilde[j], mtj = (R)mu_tilde[j], mj = (R)mu[j], nj = (R)nu[j];
    const R omn_r = R(1) - mj - nj;
    if (pip) {
      temperature_from(run, Y2);
      temperature_bcs(run);
    }
    rkl2_stage<R, false>(run, __LINE__, temp(Y2), Y2, Y1, energy, Y3, dt_slot, mtj, mj, nj, omn_r, gt);
    if (j < s) {
      GhostBatch<R> bb;
      bb.add(run.g_cell, Y3.p);  // energy_bcs on the copy of Y3
      ghost_flush(run, bb);
      if (pip) neutral_fraction(run, Y3);  // conduct.f90:404
      A3<R> freed = Y1;
      Y1 = Y2;
      Y2 = Y3;
      if (freed.p == energy.p) {
        Y3 = bufs[next_free];
      } else {
        Y3 = freed;
      }
    }
  }
  // The reference leaves temperature = T(Y2 of the last stage) after
  // temperature_bcs; keep that, then energy(1:n) = Y3(1:n) and energy_bcs.
  {
    auto temperature = A.temperature;
    A3<R> y2 = Y2, y3 = Y3;
    if (!pip) {  // (a partially ionised run formed it for the last stage)
      LARE_BOXW(run, 2, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
        temperature(ix, iy, iz) = tc * (y2(ix, iy, iz) - te0);
      });
      GhostBatch<R> bb;
      bb.add(run.g_cell_user, temperature.p);
      ghost_flush(run, bb);
    }
    LARE_BOXW(run, 2, 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz) { energy(ix, iy, iz) = y3(ix, iy, iz); });
  }
  energy_bcs(run);
}

// ---------------------------------------------------------------------
// Limited Van Leer flux shared by the *_flux routines of [xyz]remap.f90.
//
// Divisors arrive in carried form (dv_of): the value itself in the exact
// builds, its reciprocal in the product build, so a kernel that moves along
// a line forms each reciprocal once per point.  The exact builds evaluate
// the reference's expressions unchanged; the product build takes the upwind
// divisors by selection (vad_p is exactly 0 or 1, so the reference's
// weighted sums dxcm*vad_p + dxcp*vad_m equal one of the two) and multiplies.
template <class R>
struct LimOut {
  R sign_v, vad_p, vad_m, fu, Di, dxbu, phi;
};
template <class R>
__device__ __forceinline__ LimOut<R> limiter_dv(R v_advect, R fm, R fi, R fp, R fp2, R dvci, R dvcm, R dvcp,
                                                R dxbi, R dxbp, R dvu_p, R dvu_m, R dt, bool phi_from_dxu) {
  LimOut<R> L;
  R dfm = fi - fm, dfi = fp - fi, dfp = fp2 - fp;
  L.sign_v = copysign(R(1), v_advect);
  L.vad_p = (L.sign_v + R(1)) * R(0.5);
  L.vad_m = R(1) - L.vad_p;
  L.fu = fi * L.vad_p + fp * L.vad_m;
  R dfu = dfm * L.vad_p + dfp * L.vad_m;
  L.dxbu = dxbi * L.vad_p + dxbp * L.vad_m;
#if LARE_FAST
  const bool up = !signbit(v_advect);
  const R dvcu = up ? dvcm : dvcp;
  if (phi_from_dxu) {
    L.phi = fabs(v_advect) * dt * (up ? dvu_p : dvu_m);
  } else {
    L.phi = fabs(v_advect) * dt * fast_rcp(L.dxbu);
  }
#else
  R dvcu = dvcm * L.vad_p + dvcp * L.vad_m;
  if (phi_from_dxu) {
    R dxu = dvu_p * L.vad_p + dvu_m * L.vad_m;
    L.phi = fabs(v_advect) * dt / dxu;
  } else {
    L.phi = fabs(v_advect) * dt / L.dxbu;
  }
#endif
  R Da = dv_div((R(2) - L.phi) * fabs(dfi), dvci) + dv_div((R(1) + L.phi) * fabs(dfu), dvcu);
  Da = Da * (R(1) / R(6));
  R ss = R(0.5) * (copysign(R(1), dfi) + copysign(R(1), dfu));
  L.Di = L.sign_v * ss * fmin(fmin(fabs(Da) * L.dxbu, fabs(dfi)), fabs(dfu));
  return L;
}
// The same with plain divisors.
template <class R>
__device__ __forceinline__ LimOut<R> limiter(R v_advect, R fm, R fi, R fp, R fp2, R dxci, R dxcm, R dxcp, R dxbi,
                                             R dxbp, R dxu_p, R dxu_m, R dt, bool phi_from_dxu) {
  return limiter_dv(v_advect, fm, fi, fp, fp2, dv_of(dxci), dv_of(dxcm), dv_of(dxcp), dxbi, dxbp,
                    phi_from_dxu ? dv_of(dxu_p) : dxu_p, phi_from_dxu ? dv_of(dxu_m) : dxu_m, dt, phi_from_dxu);
}

LARE_END  // namespace lare

#include "remap.cuh"

LARE_BEGIN

// remap.f90:33-131 eulerian_remap (the corrector's full remap; the
// predictor's B-only remap is predictor_remap in lagran.cuh).
template <class R>
void eulerian_remap(Run<R>& run, int step) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  const int sx = run.sx, sxy = run.sxy;
  int pass[3] = {1, 1, 1};
  if (run.p.rke) {  // remap.f90:38
    R* const dke = run.a.delta_ke.p;
    LARE_BOXW(run, 1, 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz) { dke[ix + sx * iy + sxy * iz] = R(0); });
  }
  // B -> flux form (remap.f90:43-69) and back (:101-127) are done by the
  // first and last sweeps' B kernels on the way (remap_sweep's bmode).
  static const int order[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {0, 2, 1}, {2, 1, 0}, {1, 0, 2}};
  int cse = ((step % 6) + 6) % 6;
  for (int s = 0; s < 3; ++s) {
    const int bmode = s == 0 ? 1 : (s == 2 ? 2 : 0);
    switch (order[cse][s]) {
      case 0: remap_sweep<0>(run, false, SC_DT, pass, bmode); break;
      case 1: remap_sweep<1>(run, false, SC_DT, pass, bmode); break;
      default: remap_sweep<2>(run, false, SC_DT, pass, bmode); break;
    }
  }
  bfield_bcs(run);
}

// Pull the scalar slots to the host (one sync).
template <class R>
cudaError_t pull_scalars(Run<R>& run) {
  cudaMemcpyAsync(run.host_sc, run.sc, SC_NSLOTS * sizeof(double), cudaMemcpyDeviceToHost, run.s);
  return cudaStreamSynchronize(run.s);
}

// ---------------------------------------------------------------------
// diagnostics.F90:517-609 energy_account into sc[SC_EN_B..SC_EN_INT].
template <class R>
void energy_account(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  Arrays<R>& A = run.a;
  auto bx = A.bx, by = A.by, bz = A.bz, cv = A.cv, energy = A.energy, rho = A.rho;
  auto vx = A.vx, vy = A.vy, vz = A.vz;
  box_sum<2>(run, "energy_account_cells", 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz, double* v) {
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
  box_sum<1>(run, "energy_account_vertices", 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz, double* v) {
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

LARE_END  // namespace lare

LARE_BEGIN

// diagnostics.F90:613-629 energy_correction, after eulerian_remap when rke
// is on (lare3d.f90:86): the kinetic energy the remap lost, where it lost
// some, goes into the internal energy of cells 1:n; then energy_bcs.
template <class R>
void energy_correction(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  auto dke = run.a.delta_ke, rho = run.a.rho, cv = run.a.cv, energy = run.a.energy;
  LARE_BOXW(run, 5, 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz) {
    R d = -dke(ix, iy, iz);
    if (d < R(0)) d = R(0);
    d = d / (rho(ix, iy, iz) * cv(ix, iy, iz));
    dke(ix, iy, iz) = d;
    energy(ix, iy, iz) = energy(ix, iy, iz) + d;
  });
  energy_bcs(run);
}

LARE_END  // namespace lare

#include "openbc.cuh"

LARE_BEGIN

template <int F, class R>
inline void open_face(Run<R>& run, const OpenArgs<R>& g) {
  if (run.p.bc[F / 2][F & 1] != LARE_BC_OPEN) return;
  const int nu = F / 2 == 0 ? run.n[1] : run.n[0], nw = F / 2 == 2 ? run.n[1] : run.n[2];
  dim3 blk(32, 4, 1);
  dim3 grd((nu + 2 + 31) / 32, (nw + 2 + 3) / 4, 1);
  const int k = run.prof_begin("open_bcs", F, 0, (double)(nu + 2) * (nw + 2));
  k_open_face<F, R><<<grd, blk, 0, run.s>>>(g);
  run.prof_end(k);
  ++run.launches;
}

// openboundary.f90:30-324 open_bcs: the open faces in the reference's order.
template <class R>
void open_bcs(Run<R>& run) {
  OpenArgs<R> g;
  g.vx = run.a.vx.p;
  g.vy = run.a.vy.p;
  g.vz = run.a.vz.p;
  g.bx = run.a.bx.p;
  g.by = run.a.by.p;
  g.bz = run.a.bz.p;
  g.rho = run.a.rho.p;
  g.energy = run.a.energy.p;
  g.g = (R)run.p.gamma;
  g.nx = run.n[0];
  g.ny = run.n[1];
  g.nz = run.n[2];
  g.sx = run.sx;
  g.sxy = run.sxy;
  open_face<0>(run, g);
  open_face<1>(run, g);
  open_face<2>(run, g);
  open_face<3>(run, g);
  open_face<4>(run, g);
  open_face<5>(run, g);
}

LARE_END  // namespace lare

#include "lagran.cuh"
