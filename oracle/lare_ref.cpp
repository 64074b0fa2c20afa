// lare_ref.cpp - CPU oracle for the Lare3d Lagrangian-remap timestep.
//
// TEST INFRASTRUCTURE ONLY.  This file restates the reference's Fortran hot
// path in C++ so that the CUDA implementation can be checked against it.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// it; the product library never does.
//
// Parity status: the reference ships no tests, golden files or fixtures for
// this path and no Fortran compiler exists where this was written, so this
// restatement is pinned by the reference's source text only (every routine
// cites the file:line it follows) plus the invariants the tests check
// (conservation, div B, symmetry, uniform-state preservation).  "Parity
// unpinned" in the sense that no output of the reference itself was
// compared.
//
// Rules followed so that results are reproducible bit for bit:
//   * every loop nest keeps the reference's index ranges and its
//     left-to-right expression order; compile with -ffp-contract=off
//     (gfortran -O3 on x86-64 emits no FMA);
//   * Fortran SIGN(1,x) -> copysign, x**2 -> x*x, x**2.5 -> pow;
//   * reductions that are order-sensitive (energy budgets, heating totals)
//     run serially in the reference's loop order; min reductions may run in
//     parallel (min is order-independent).
// Default compile-time DEFINES of the reference only (no CAUCHY,
// SHOCKLIMITER, SHOCKCOMPRESSION, FOURTHORDER, SINGLE).

#include "lare_ref.h"

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Array with Fortran bounds, column-major.
struct F3 {
  int lo[3] = {0, 0, 0}, hi[3] = {-1, -1, -1};
  long s1 = 0, s2 = 0;
  std::vector<double> d;
  void alloc(int l0, int h0, int l1, int h1, int l2, int h2, double v = 0.0) {
    lo[0] = l0; hi[0] = h0; lo[1] = l1; hi[1] = h1; lo[2] = l2; hi[2] = h2;
    s1 = h0 - l0 + 1;
    s2 = s1 * (h1 - l1 + 1);
    d.assign((size_t)s2 * (h2 - l2 + 1), v);
  }
  inline double& operator()(int i, int j, int k) {
#ifdef LARE_REF_BOUNDS
    if (i < lo[0] || i > hi[0] || j < lo[1] || j > hi[1] || k < lo[2] || k > hi[2]) {
      std::fprintf(stderr, "oracle bounds violation (%d,%d,%d) in [%d:%d,%d:%d,%d:%d]\n",
                   i, j, k, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]);
      std::abort();
    }
#endif
    return d[(size_t)((i - lo[0]) + s1 * (j - lo[1]) + s2 * (k - lo[2]))];
  }
  void fill(double v) { std::fill(d.begin(), d.end(), v); }
  size_t size() const { return d.size(); }
};

struct F1 {
  int lo = 0, hi = -1;
  std::vector<double> d;
  void alloc(int l, int h, double v = 0.0) { lo = l; hi = h; d.assign(h - l + 1, v); }
  inline double operator()(int i) const {
#ifdef LARE_REF_BOUNDS
    if (i < lo || i > hi) { std::fprintf(stderr, "oracle 1d bounds %d [%d:%d]\n", i, lo, hi); std::abort(); }
#endif
    return d[(size_t)(i - lo)];
  }
  inline double& at(int i) { return d[(size_t)(i - lo)]; }
};

// Parallel map over an inclusive index box.  Every loop nest of the hot path
// writes each element from values it does not write in the same nest, so the
// iteration order does not change any result.
template <class Fn>
inline void box(int i0, int i1, int j0, int j1, int k0, int k1, Fn fn) {
#pragma omp parallel for schedule(static)
  for (int iz = k0; iz <= k1; ++iz)
    for (int iy = j0; iy <= j1; ++iy)
      for (int ix = i0; ix <= i1; ++ix) fn(ix, iy, iz);
}

inline double fmin3(double a, double b, double c) { return std::fmin(std::fmin(a, b), c); }
inline double fmax0(double a) { return a > 0.0 ? a : 0.0; }

const double none_zero = DBL_MIN;         // TINY(1.0_num), shared_data.F90:62
const double largest_number = DBL_MAX;    // HUGE(1.0_num), shared_data.F90:63
const double sixth = 1.0 / 6.0;           // shared_data.F90:64
const double pow_c = 5.0 / 2.0;           // conduct.f90:27

// The exponential of the ionisation model: Cody and Waite's reduction
// x = k ln2 + r (ln 2 as a 33-bit head plus its tail), a Taylor polynomial
// through r^13 by Horner's rule and a scaling by 2^k.  The reference calls
// the Fortran EXP (the C library's exp); this one is within about 1 ulp of
// the exact value and is used so that the checked library, which evaluates
// the same operations, gives identical bits through the bisection.
double cw_exp(double x) {
  if (!(x == x)) return x;
  if (x > 709.782712893384) return HUGE_VAL;
  if (x < -745.1332191019412) return 0.0;
  const double ln2_hi = 0x1.62e42fee00000p-1, ln2_lo = 0x1.a39ef35793c76p-33;
  const double k = std::rint(x * 0x1.71547652b82fep+0);
  const double r = (x - k * ln2_hi) - k * ln2_lo;
  static const double c[] = {0x1.1eed8eff8d898p-29, 0x1.ae64567f544e4p-26, 0x1.27e4fb7789f5cp-22,
                             0x1.71de3a556c734p-19, 0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-13,
                             0x1.6c16c16c16c17p-10, 0x1.1111111111111p-7,  0x1.5555555555555p-5,
                             0x1.5555555555555p-3,  0.5,                   1.0,
                             1.0};
  double q = 0x1.6124613a86d09p-33;  // 1/13!, then 1/12! ... 1/2!, 1, 1
  for (double ci : c) q = q * r + ci;
  return std::ldexp(q, (int)k);
}
const double min_b = 1.0e-10;             // conduct.f90:28

}  // namespace

struct lare_ref {
  lare_params p;
  int nx, ny, nz;
  int n[3];
  std::string err;

  // 1-D grid metrics (setup.F90:162-180).
  F1 dxb, dxc, dyb, dyc, dzb, dzc, grav;
  F1* db[3];
  F1* dc[3];

  // Persistent state (mpi_routines.F90:295-334, neutral.f90:37).
  F3 rho, energy, temperature, eta, cv, cv1, p_visc, visc_dep, ohmic_dep, gamma_boris;
  F3 vx, vy, vz, vx1, vy1, vz1, visc3;
  F3 bx, by, bz;
  F3* V[3];
  F3* V1[3];
  F3* B[3];

  // lagran.F90 module temporaries (:36-42, allocated :56-81).
  F3 bx0, by0, bz0, bx1, by1, bz1, alpha1, alpha2, alpha3;
  F3 visc_heat, pressure, rho_v, cv_v, flux_x, flux_y, flux_z, curlb;
  F3 fx_visc, fy_visc, fz_visc, qx, qy, qz, energy0, delta_energy;
  F3 cs, cs_v;
  // [xyz]remap.f90 module temporaries (:30-31).
  F3 r_db1, r_dc1, r_rho_v, r_rho_v1, r_rho1, r_dm, r_cv2, r_flux[3];
  // conduct.f90 temporaries.
  F3 larsen_factor, c_flux, Y[4], Lc_Y0;
  // neutral.f90:37-44 (xi_n always exists in the reference; eta_perp with
  // cowling_resistivity)
  F3 xi_n, eta_perp;
  bool eos_error = false;  // neutral.f90:171-174 'Temperature bounds problem'
  F3 delta_ke;             // rke (shared_data.F90:108, allocated mpi_routines.F90:313)
  F3 cool_term_v, cool_term_b;  // cooling_term (shared_data.F90:109, mpi_routines.F90:315-319)
  F3 heat_in;                   // coronal_heating: user_defined_heating's rate (radiative.f90:73)

  // shared_data scalars.
  double time = 0.0, dt = 0.0, dt2 = 0.0, dtr = 0.0;
  double visc2_norm = 0.0;
  double total_visc_heating = 0.0, total_ohmic_heating = 0.0;
  int xpass = 1, ypass = 1, zpass = 1;
  int n_s_stages = 0, peak_substeps = 0, last_substeps = 0, steps_taken = 0, cur_step = 0;
  bool predictor_step = false;
  bool shock_first_call = true;   // lagran.F90:539 (SAVE)
  bool set_dt_first = true;       // lagran.F90:1078 (SAVE)

  std::map<std::string, F3*> fields;

  // ------------------------------------------------------------------
  void allocate() {
    const int N = nx, M = ny, L = nz;
    auto cell = [&](F3& a) { a.alloc(-1, N + 2, -1, M + 2, -1, L + 2); };
    auto node = [&](F3& a) { a.alloc(-2, N + 2, -2, M + 2, -2, L + 2); };
    cell(rho); cell(energy); cell(temperature); cell(eta); cell(cv); cell(cv1);
    cell(p_visc); cell(visc_dep); cell(ohmic_dep); cell(gamma_boris);
    node(vx); node(vy); node(vz); node(vx1); node(vy1); node(vz1); node(visc3);
    bx.alloc(-2, N + 2, -1, M + 2, -1, L + 2);
    by.alloc(-1, N + 2, -2, M + 2, -1, L + 2);
    bz.alloc(-1, N + 2, -1, M + 2, -2, L + 2);
    bx0.alloc(-2, N + 2, -1, M + 2, -1, L + 2);
    by0.alloc(-1, N + 2, -2, M + 2, -1, L + 2);
    bz0.alloc(-1, N + 2, -1, M + 2, -2, L + 2);
    cell(bx1); cell(by1); cell(bz1);
    alpha1.alloc(0, N + 1, 0, M + 2, 0, L + 2);
    alpha2.alloc(-1, N + 1, 0, M + 1, 0, L + 2);
    alpha3.alloc(-1, N + 1, -1, M + 1, 0, L + 1);
    visc_heat.alloc(0, N + 1, 0, M + 1, 0, L + 1);
    cell(pressure);
    rho_v.alloc(-1, N + 1, -1, M + 1, -1, L + 1);
    cv_v.alloc(-1, N + 1, -1, M + 1, -1, L + 1);
    for (F3* a : {&fx_visc, &fy_visc, &fz_visc, &flux_x, &flux_y, &flux_z, &curlb})
      a->alloc(0, N, 0, M, 0, L);
    for (F3* a : {&qx, &qy, &qz}) a->alloc(0, N + 1, 0, M + 1, 0, L + 1);
    cell(energy0); cell(delta_energy);
    cell(cs);
    cs_v.alloc(-1, N + 1, -1, M + 1, -1, L + 1);
    for (F3* a : {&r_db1, &r_dc1, &r_rho_v, &r_rho_v1, &r_rho1, &r_dm, &r_cv2}) cell(*a);
    r_flux[0].alloc(-2, N + 2, -1, M + 2, -1, L + 2);
    r_flux[1].alloc(-1, N + 2, -2, M + 2, -1, L + 2);
    r_flux[2].alloc(-1, N + 2, -1, M + 2, -2, L + 2);
    larsen_factor.alloc(0, N, 0, M, 0, L);
    cell(c_flux);
    for (int j = 0; j < 4; ++j) cell(Y[j]);
    Lc_Y0.alloc(1, N, 1, M, 1, L);
    gamma_boris.fill(1.0);
    // xi_n = 0 (neutral.f90:38), or 1 for a neutral gas under EOS_IDEAL
    // (lare3d.f90:72): the constant p.xi_n until neutral_fraction runs
    cell(xi_n);
    xi_n.fill(p.xi_n);
    if (p.cowling_resistivity) cell(eta_perp);
    if (p.rke) cell(delta_ke);
    if (p.coronal_heating) cell(heat_in);
    if (p.cooling_term) {
      cool_term_v.alloc(1, N, 1, M, 1, L);
      cool_term_b.alloc(1, N, 1, M, 1, L);
    }

    V[0] = &vx; V[1] = &vy; V[2] = &vz;
    V1[0] = &vx1; V1[1] = &vy1; V1[2] = &vz1;
    B[0] = &bx; B[1] = &by; B[2] = &bz;
    db[0] = &dxb; db[1] = &dyb; db[2] = &dzb;
    dc[0] = &dxc; dc[1] = &dyc; dc[2] = &dzc;

    fields = {{"rho", &rho}, {"energy", &energy}, {"temperature", &temperature},
              {"eta", &eta}, {"cv", &cv}, {"cv1", &cv1}, {"p_visc", &p_visc},
              {"visc_dep", &visc_dep}, {"ohmic_dep", &ohmic_dep},
              {"gamma_boris", &gamma_boris}, {"vx", &vx}, {"vy", &vy}, {"vz", &vz},
              {"vx1", &vx1}, {"vy1", &vy1}, {"vz1", &vz1}, {"visc3", &visc3},
              {"bx", &bx}, {"by", &by}, {"bz", &bz}, {"bx1", &bx1}, {"by1", &by1},
              {"bz1", &bz1}, {"alpha1", &alpha1}, {"alpha2", &alpha2},
              {"alpha3", &alpha3}, {"visc_heat", &visc_heat}, {"pressure", &pressure},
              {"rho_v", &rho_v}, {"cv_v", &cv_v}, {"fx_visc", &fx_visc},
              {"fy_visc", &fy_visc}, {"fz_visc", &fz_visc}, {"larsen_factor", &larsen_factor},
              {"xi_n", &xi_n}};
    if (p.cowling_resistivity) fields["eta_perp"] = &eta_perp;
    if (p.rke) fields["delta_ke"] = &delta_ke;
    if (p.coronal_heating) fields["heat_in"] = &heat_in;
    if (p.cooling_term) {
      fields["cool_term_v"] = &cool_term_v;
      fields["cool_term_b"] = &cool_term_b;
    }
  }

  // ------------------------------------------------------------------
  // Ghost fills: boundary.f90 + mpiboundary.f90 on one rank.  With a
  // periodic Cartesian communicator of one rank every MPI_SENDRECV sends to
  // itself; with BC_USER the neighbour is MPI_PROC_NULL and the mirror rules
  // of boundary.f90 apply.  Each helper reproduces the exact slab copies.
  bool per(int d, bool maxside) const {
    (void)maxside;
    // The communicator is periodic in a direction unless either side is
    // BC_USER/BC_OPEN (mpi_routines.F90:195-210).
    int a = d == 0 ? p.xbc_min : d == 1 ? p.ybc_min : p.zbc_min;
    int b = d == 0 ? p.xbc_max : d == 1 ? p.ybc_max : p.zbc_max;
    return a == LARE_BC_PERIODIC && b == LARE_BC_PERIODIC;
  }
  bool user(int d, bool maxside) const {
    int c = d == 0 ? (maxside ? p.xbc_max : p.xbc_min)
          : d == 1 ? (maxside ? p.ybc_max : p.ybc_min) : (maxside ? p.zbc_max : p.zbc_min);
    return !per(d, maxside) && c == LARE_BC_USER;
  }

  // Copy plane src -> plane dst along dimension d over the full extent of
  // the other two dimensions.
  static void copy_plane(F3& a, int d, int dst, int src) {
    int lo0 = a.lo[0], hi0 = a.hi[0], lo1 = a.lo[1], hi1 = a.hi[1], lo2 = a.lo[2], hi2 = a.hi[2];
    if (d == 0) { for (int k = lo2; k <= hi2; ++k) for (int j = lo1; j <= hi1; ++j) a(dst, j, k) = a(src, j, k); }
    else if (d == 1) { for (int k = lo2; k <= hi2; ++k) for (int i = lo0; i <= hi0; ++i) a(i, dst, k) = a(i, src, k); }
    else { for (int j = lo1; j <= hi1; ++j) for (int i = lo0; i <= hi0; ++i) a(i, j, dst) = a(i, j, src); }
  }
  static void zero_plane(F3& a, int d, int pl) {
    int lo0 = a.lo[0], hi0 = a.hi[0], lo1 = a.lo[1], hi1 = a.hi[1], lo2 = a.lo[2], hi2 = a.hi[2];
    if (d == 0) { for (int k = lo2; k <= hi2; ++k) for (int j = lo1; j <= hi1; ++j) a(pl, j, k) = 0.0; }
    else if (d == 1) { for (int k = lo2; k <= hi2; ++k) for (int i = lo0; i <= hi0; ++i) a(i, pl, k) = 0.0; }
    else { for (int j = lo1; j <= hi1; ++j) for (int i = lo0; i <= hi0; ++i) a(i, j, pl) = 0.0; }
  }

  // Cell-centred exchange (cell_[xyz]face, ng = 2): energy_mpi /
  // density_mpi (mpiboundary.f90:122-187).  Sends 1:2 -> n+1:n+2, then
  // n-1:n -> -1:0.
  void cell_mpi(F3& a) {
    for (int d = 0; d < 3; ++d) {
      if (!per(d, false)) continue;
      int N = n[d];
      copy_plane(a, d, N + 1, 1); copy_plane(a, d, N + 2, 2);
      copy_plane(a, d, -1, N - 1); copy_plane(a, d, 0, N);
    }
  }
  // BC_USER mirror for cell arrays (boundary.f90:133-161).
  void cell_user(F3& a) {
    for (int d = 0; d < 3; ++d) {
      int N = n[d];
      if (user(d, false)) { copy_plane(a, d, 0, 1); copy_plane(a, d, -1, 2); }
      if (user(d, true)) { copy_plane(a, d, N + 1, N); copy_plane(a, d, N + 2, N - 1); }
    }
  }
  void energy_bcs() { cell_mpi(energy); cell_user(energy); }        // boundary.f90:129
  void density_bcs() { cell_mpi(rho); cell_user(rho); }             // boundary.f90:171
  void temperature_bcs() { cell_mpi(rho); cell_user(temperature); } // boundary.f90:212 (exchanges rho, :214)

  // Node exchange: node_[xyz]face1 (3 layers) 0:2 -> n:n+2, then
  // node_[xyz]face (2 layers) n-2:n-1 -> -2:-1 (mpiboundary.f90:195-278).
  void node_mpi(F3& a) {
    for (int d = 0; d < 3; ++d) {
      if (!per(d, false)) continue;
      int N = n[d];
      copy_plane(a, d, N, 0); copy_plane(a, d, N + 1, 1); copy_plane(a, d, N + 2, 2);
      copy_plane(a, d, -2, N - 2); copy_plane(a, d, -1, N - 1);
    }
  }
  // v = 0 in BC_USER ghosts and on the boundary node (boundary.f90:259-293).
  void node_user(F3& a) {
    for (int d = 0; d < 3; ++d) {
      int N = n[d];
      if (user(d, false)) for (int q = -2; q <= 0; ++q) zero_plane(a, d, q);
      if (user(d, true)) for (int q = N; q <= N + 2; ++q) zero_plane(a, d, q);
    }
  }
  // ------------------------------------------------------------------
  // Open (characteristic) boundaries, openboundary.f90.  A side with
  // BC_OPEN gets no ghost fill from boundary.f90 (the direction is not
  // periodic and the mirror rules are BC_USER only), so its second ghost
  // layer keeps the uploaded far-field state; once per step (after
  // velocity_bcs in predictor_corrector_step, lagran.F90:409-412) the first
  // ghost layer of B, rho and energy is set from the Riemann invariants
  // carried out of the domain and in from the far field.
  struct OpenIn {
    double vn, vx1, vy1, vz1, bx1, by1, bz1, r1, e1, pbc, pfar, uxf, uyf, uzf, bxf, byf, bzf, rf;
  };
  struct OpenOut {
    double bx0, by0, bz0, r0, e0;
  };
  // openboundary.f90:326-378, open_bcs_fast (transverse field present)
  static OpenOut open_fast(const OpenIn& a, double g) {
    OpenOut o;
    const double c0far = std::sqrt(g * a.pfar / a.rf);
    const double ctfar = std::sqrt((a.byf * a.byf + a.bzf * a.bzf) / a.rf);
    const double cffar = std::sqrt(c0far * c0far + ctfar * ctfar);
    const double c0 = std::sqrt(g * (g - 1.0) * a.e1);
    const double ct = std::sqrt((a.by1 * a.by1 + a.bz1 * a.bz1) / a.r1);
    const double cf = std::sqrt(c0 * c0 + ct * ct);
    const double vtest[3] = {a.vn + cf, a.vn - cf, a.vn};
    double pstar[3], pmag[3], vstar[3], rstar[3], bys[3], bzs[3];
    for (int i = 0; i < 3; ++i) {
      if (vtest[i] >= 0.0) {
        pstar[i] = a.pbc + 0.5 * (a.by1 * a.by1 + a.bz1 * a.bz1);
        pmag[i] = 0.5 * (a.by1 * a.by1 + a.bz1 * a.bz1);
        vstar[i] = a.vx1;
        rstar[i] = a.r1;
        bys[i] = a.by1;
        bzs[i] = a.bz1;
      } else {
        pstar[i] = a.pfar + 0.5 * (a.byf * a.byf + a.bzf * a.bzf);
        pmag[i] = 0.5 * (a.byf * a.byf + a.bzf * a.bzf);
        vstar[i] = a.uxf;
        rstar[i] = a.rf;
        bys[i] = a.byf;
        bzs[i] = a.bzf;
      }
    }
    o.bx0 = 0.5 * (a.bx1 + a.bxf);
    o.by0 = 0.5 * (bys[0] + bys[1]);
    o.bz0 = 0.5 * (bzs[0] + bzs[1]);
    double pg = 0.5 * (pstar[0] + pstar[1] + a.rf * cffar * (vstar[0] - vstar[1])) - 0.5 * (pmag[0] + pmag[1]);
    pg = std::fmax(pg, 0.0);
    const double rhog = rstar[2] + (pg - (pstar[2] - pmag[2])) / (c0far * c0far);
    o.r0 = std::fmax(rhog, none_zero);
    o.e0 = pg / (g - 1.0) / o.r0;
    return o;
  }
  // openboundary.f90:382-455, open_bcs_alfven (no transverse far field)
  static OpenOut open_alfven(const OpenIn& a, double g) {
    OpenOut o;
    const double lyfar = -(a.bxf * a.byf), lzfar = -(a.bxf * a.bzf);
    const double c0far = std::sqrt(g * a.pfar / a.rf);
    const double cxfar = std::sqrt(a.bxf * a.bxf / a.rf);
    const double c0 = std::sqrt(g * (g - 1.0) * a.e1);
    const double cx = std::sqrt(a.bx1 * a.bx1 / a.r1);
    const double vtest[5] = {a.vn + c0, a.vn - c0, a.vn + cx, a.vn - cx, a.vn};
    double pstar[5], pmag[5], ly[5], lz[5], ux[5], uy[5], uz[5], rstar[5];
    for (int i = 0; i < 5; ++i) {
      if (vtest[i] >= 0.0) {
        pstar[i] = a.pbc + 0.5 * (a.by1 * a.by1 + a.bz1 * a.bz1 - a.bx1 * a.bx1);
        pmag[i] = 0.5 * (a.by1 * a.by1 + a.bz1 * a.bz1 - a.bx1 * a.bx1);
        ly[i] = -(a.by1 * a.bx1);
        lz[i] = -(a.bz1 * a.bx1);
        ux[i] = a.vx1;
        uy[i] = a.vy1;
        uz[i] = a.vz1;
        rstar[i] = a.r1;
      } else {
        pstar[i] = a.pfar + 0.5 * (a.byf * a.byf + a.bzf * a.bzf - a.bxf * a.bxf);
        pmag[i] = 0.5 * (a.byf * a.byf + a.bzf * a.bzf - a.bxf * a.bxf);
        ly[i] = lyfar;
        lz[i] = lzfar;
        ux[i] = a.uxf;
        uy[i] = a.uyf;
        uz[i] = a.uzf;
        rstar[i] = a.rf;
      }
    }
    o.bx0 = 0.5 * (a.bx1 + a.bxf);
    if (std::fabs(o.bx0) <= none_zero) o.bx0 = none_zero;
    double lg = 0.5 * (ly[2] + ly[3] + a.rf * cxfar * (uy[2] - uy[3]));
    o.by0 = -(lg / o.bx0);
    lg = 0.5 * (lz[2] + lz[3] + a.rf * cxfar * (uz[2] - uz[3]));
    o.bz0 = -(lg / o.bx0);
    double pg = 0.5 * (pstar[0] + pstar[1] + a.rf * c0far * (ux[0] - ux[1])) -
                0.5 * (o.by0 * o.by0 + o.bz0 * o.bz0 - o.bx0 * o.bx0);
    pg = std::fmax(pg, none_zero);
    const double rhog = rstar[4] + (pg - (pstar[4] - pmag[4])) / (c0far * c0far);
    o.r0 = std::fmax(rhog, none_zero);
    o.e0 = pg / (g - 1.0) / o.r0;
    return o;
  }
  static OpenOut open_solve(const OpenIn& a, double g) {
    // solver choice on the far-field transverse field (openboundary.f90:63-71)
    const double bperp = std::sqrt(a.byf * a.byf + a.bzf * a.bzf);
    return bperp <= none_zero ? open_alfven(a, g) : open_fast(a, g);
  }
  bool any_open() const {
    const int c[6] = {p.xbc_min, p.xbc_max, p.ybc_min, p.ybc_max, p.zbc_min, p.zbc_max};
    for (int q = 0; q < 6; ++q)
      if (c[q] == LARE_BC_OPEN) return true;
    return false;
  }
  // openboundary.f90:30-324, faces in the reference's order; a later face
  // reads edge values an earlier one wrote.  In each face the normal
  // velocity and field are sign-flipped on the min side, and the far field
  // is the second ghost layer.
  void open_bcs() {
    const double g = p.gamma;
    auto pres = [&](int i, int j, int k) { return (g - 1.0) * energy(i, j, k) * rho(i, j, k); };
    if (p.xbc_min == LARE_BC_OPEN) {  // :35-80
      for (int iz = 0; iz <= nz + 1; ++iz)
        for (int iy = 0; iy <= ny + 1; ++iy) {
          OpenIn a{-vx(0, iy, iz), -vx(0, iy, iz), vy(0, iy, iz), vz(0, iy, iz), -bx(0, iy, iz), by(1, iy, iz),
                   bz(1, iy, iz), rho(1, iy, iz), energy(1, iy, iz), pres(1, iy, iz), pres(-1, iy, iz),
                   -vx(-2, iy, iz), vy(-2, iy, iz), vz(-2, iy, iz), -bx(-2, iy, iz), by(-1, iy, iz),
                   bz(-1, iy, iz), rho(-1, iy, iz)};
          OpenOut o = open_solve(a, g);
          bx(-1, iy, iz) = -o.bx0;
          by(0, iy, iz) = o.by0;
          bz(0, iy, iz) = o.bz0;
          rho(0, iy, iz) = o.r0;
          energy(0, iy, iz) = o.e0;
        }
    }
    if (p.xbc_max == LARE_BC_OPEN) {  // :83-128
      for (int iz = 0; iz <= nz + 1; ++iz)
        for (int iy = 0; iy <= ny + 1; ++iy) {
          OpenIn a{vx(nx, iy, iz), vx(nx, iy, iz), vy(nx, iy, iz), vz(nx, iy, iz), bx(nx, iy, iz), by(nx, iy, iz),
                   bz(nx, iy, iz), rho(nx, iy, iz), energy(nx, iy, iz), pres(nx, iy, iz), pres(nx + 2, iy, iz),
                   vx(nx + 2, iy, iz), vy(nx + 2, iy, iz), vz(nx + 2, iy, iz), bx(nx + 2, iy, iz),
                   by(nx + 2, iy, iz), bz(nx + 2, iy, iz), rho(nx + 2, iy, iz)};
          OpenOut o = open_solve(a, g);
          bx(nx + 1, iy, iz) = o.bx0;
          by(nx + 1, iy, iz) = o.by0;
          bz(nx + 1, iy, iz) = o.bz0;
          rho(nx + 1, iy, iz) = o.r0;
          energy(nx + 1, iy, iz) = o.e0;
        }
    }
    if (p.ybc_min == LARE_BC_OPEN) {  // :131-176
      for (int iz = 0; iz <= nz + 1; ++iz)
        for (int ix = 0; ix <= nx + 1; ++ix) {
          OpenIn a{-vy(ix, 0, iz), -vy(ix, 0, iz), vx(ix, 0, iz), vz(ix, 0, iz), -by(ix, 0, iz), bx(ix, 1, iz),
                   bz(ix, 1, iz), rho(ix, 1, iz), energy(ix, 1, iz), pres(ix, 1, iz), pres(ix, -1, iz),
                   -vy(ix, -2, iz), vx(ix, -2, iz), vz(ix, -2, iz), -by(ix, -2, iz), bx(ix, -1, iz),
                   bz(ix, -1, iz), rho(ix, -1, iz)};
          OpenOut o = open_solve(a, g);
          bx(ix, 0, iz) = o.by0;
          by(ix, -1, iz) = -o.bx0;
          bz(ix, 0, iz) = o.bz0;
          rho(ix, 0, iz) = o.r0;
          energy(ix, 0, iz) = o.e0;
        }
    }
    if (p.ybc_max == LARE_BC_OPEN) {  // :179-224
      for (int iz = 0; iz <= nz + 1; ++iz)
        for (int ix = 0; ix <= nx + 1; ++ix) {
          OpenIn a{vy(ix, ny, iz), vy(ix, ny, iz), vx(ix, ny, iz), vz(ix, ny, iz), by(ix, ny, iz), bx(ix, ny, iz),
                   bz(ix, ny, iz), rho(ix, ny, iz), energy(ix, ny, iz), pres(ix, ny, iz), pres(ix, ny + 2, iz),
                   vy(ix, ny + 2, iz), vx(ix, ny + 2, iz), vz(ix, ny + 2, iz), by(ix, ny + 2, iz),
                   bx(ix, ny + 2, iz), bz(ix, ny + 2, iz), rho(ix, ny + 2, iz)};
          OpenOut o = open_solve(a, g);
          bx(ix, ny + 1, iz) = o.by0;
          by(ix, ny + 1, iz) = o.bx0;
          bz(ix, ny + 1, iz) = o.bz0;
          rho(ix, ny + 1, iz) = o.r0;
          energy(ix, ny + 1, iz) = o.e0;
        }
    }
    if (p.zbc_min == LARE_BC_OPEN) {  // :227-273
      for (int iy = 0; iy <= ny + 1; ++iy)
        for (int ix = 0; ix <= nx + 1; ++ix) {
          OpenIn a{-vz(ix, iy, 0), -vz(ix, iy, 0), vy(ix, iy, 0), vx(ix, iy, 0), -bz(ix, iy, 0), by(ix, iy, 1),
                   bx(ix, iy, 1), rho(ix, iy, 1), energy(ix, iy, 1), pres(ix, iy, 1), pres(ix, iy, -1),
                   -vz(ix, iy, -2), vy(ix, iy, -2), vx(ix, iy, -2), -bz(ix, iy, -2), by(ix, iy, -1),
                   bx(ix, iy, -1), rho(ix, iy, -1)};
          OpenOut o = open_solve(a, g);
          bx(ix, iy, 0) = o.bz0;
          by(ix, iy, 0) = o.by0;
          bz(ix, iy, -1) = -o.bx0;
          rho(ix, iy, 0) = o.r0;
          energy(ix, iy, 0) = o.e0;
        }
    }
    if (p.zbc_max == LARE_BC_OPEN) {  // :276-320
      for (int iy = 0; iy <= ny + 1; ++iy)
        for (int ix = 0; ix <= nx + 1; ++ix) {
          OpenIn a{vz(ix, iy, nz), vz(ix, iy, nz), vy(ix, iy, nz), vx(ix, iy, nz), bz(ix, iy, nz), by(ix, iy, nz),
                   bx(ix, iy, nz), rho(ix, iy, nz), energy(ix, iy, nz), pres(ix, iy, nz), pres(ix, iy, nz + 2),
                   vz(ix, iy, nz + 2), vy(ix, iy, nz + 2), vx(ix, iy, nz + 2), bz(ix, iy, nz + 2),
                   by(ix, iy, nz + 2), bx(ix, iy, nz + 2), rho(ix, iy, nz + 2)};
          OpenOut o = open_solve(a, g);
          bx(ix, iy, nz + 1) = o.bz0;
          by(ix, iy, nz + 1) = o.by0;
          bz(ix, iy, nz + 1) = o.bx0;
          rho(ix, iy, nz + 1) = o.r0;
          energy(ix, iy, nz + 1) = o.e0;
        }
    }
  }

  void velocity_bcs() {  // boundary.f90:255
    node_mpi(vx); node_mpi(vy); node_mpi(vz);
    node_user(vx); node_user(vy); node_user(vz);
  }
  void remap_v_bcs() {  // boundary.f90:303
    node_mpi(vx1); node_mpi(vy1); node_mpi(vz1);
    node_user(vx1); node_user(vy1); node_user(vz1);
  }

  // Face field exchange, bfield_mpi (mpiboundary.f90:31-114): along its own
  // direction a component sends 1:2 -> n+1:n+2 and n-2:n -> -2:0 (3 layers,
  // b?_?face1); along the other directions it behaves as a cell array.
  void face_mpi(F3& a, int comp) {
    for (int d = 0; d < 3; ++d) {
      if (!per(d, false)) continue;
      int N = n[d];
      copy_plane(a, d, N + 1, 1); copy_plane(a, d, N + 2, 2);
      if (d == comp) {
        copy_plane(a, d, -2, N - 2); copy_plane(a, d, -1, N - 1); copy_plane(a, d, 0, N);
      } else {
        copy_plane(a, d, -1, N - 1); copy_plane(a, d, 0, N);
      }
    }
  }
  void bfield_bcs() {  // boundary.f90:63-121
    face_mpi(bx, 0); face_mpi(by, 1); face_mpi(bz, 2);
    for (int d = 0; d < 3; ++d) {
      int N = n[d];
      if (user(d, false)) {
        for (int c = 0; c < 3; ++c) {
          F3& a = *B[c];
          if (c == d) { copy_plane(a, d, -1, 1); copy_plane(a, d, -2, 2); }
          else { copy_plane(a, d, 0, 1); copy_plane(a, d, -1, 2); }
        }
      }
      if (user(d, true)) {
        for (int c = 0; c < 3; ++c) {
          F3& a = *B[c];
          if (c == d) { copy_plane(a, d, N + 1, N - 1); copy_plane(a, d, N + 2, N - 2); }
          else { copy_plane(a, d, N + 1, N); copy_plane(a, d, N + 2, N - 1); }
        }
      }
    }
  }
  void boundary_conditions() {  // boundary.f90:48-55
    bfield_bcs(); energy_bcs(); density_bcs(); velocity_bcs();
  }

  // dm_[xyz]_bcs (xremap.f90:899-917 and mirrors): one cell-face exchange
  // along the sweep axis, or linear extrapolation at a non-periodic edge.
  void dm_bcs(int a) {
    F3& dm = r_dm;
    int N = n[a];
    if (per(a, false)) {
      copy_plane(dm, a, N + 1, 1); copy_plane(dm, a, N + 2, 2);
    } else {
      // dm(n+1, 0:ny+1, 0:nz+1) = dm(n, ...)
      int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
      for (int k = 0; k <= n[t2] + 1; ++k)
        for (int j = 0; j <= n[t1] + 1; ++j) {
          int s[3], q[3];
          s[a] = N; s[t1] = j; s[t2] = k;
          q[a] = N + 1; q[t1] = j; q[t2] = k;
          dm(q[0], q[1], q[2]) = dm(s[0], s[1], s[2]);
        }
    }
    if (per(a, false)) {
      copy_plane(dm, a, -1, N - 1); copy_plane(dm, a, 0, N);
    } else {
      int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
      for (int k = 0; k <= n[t2] + 1; ++k)
        for (int j = 0; j <= n[t1] + 1; ++j) {
          int s[3], q[3];
          s[a] = 0; s[t1] = j; s[t2] = k;
          q[a] = -1; q[t1] = j; q[t2] = k;
          dm(q[0], q[1], q[2]) = dm(s[0], s[1], s[2]);
        }
    }
  }

  // ------------------------------------------------------------------
  // lagran.F90:50-200 lagrangian_step
  void lagrangian_step(int step) {
    cur_step = step;
    const double g = p.gamma;
    const double ip = p.ionise_pot;
    box(-1, nx + 2, -1, ny + 2, -1, nz + 2, [&](int ix, int iy, int iz) {
      int ixm = ix - 1, iym = iy - 1, izm = iz - 1;
      bx1(ix, iy, iz) = (bx(ix, iy, iz) + bx(ixm, iy, iz)) * 0.5;
      by1(ix, iy, iz) = (by(ix, iy, iz) + by(ix, iym, iz)) * 0.5;
      bz1(ix, iy, iz) = (bz(ix, iy, iz) + bz(ix, iy, izm)) * 0.5;
      pressure(ix, iy, iz) = (g - 1.0) * rho(ix, iy, iz) * (energy(ix, iy, iz) - (1.0 - xi_n(ix, iy, iz)) * ip);
    });
    box(-1, nx + 1, -1, ny + 1, -1, nz + 1, [&](int ix, int iy, int iz) {
      int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
      double rv = rho(ix, iy, iz) * cv(ix, iy, iz) + rho(ixp, iy, iz) * cv(ixp, iy, iz)
                + rho(ix, iyp, iz) * cv(ix, iyp, iz) + rho(ixp, iyp, iz) * cv(ixp, iyp, iz)
                + rho(ix, iy, izp) * cv(ix, iy, izp) + rho(ixp, iy, izp) * cv(ixp, iy, izp)
                + rho(ix, iyp, izp) * cv(ix, iyp, izp) + rho(ixp, iyp, izp) * cv(ixp, iyp, izp);
      double cvv = cv(ix, iy, iz) + cv(ixp, iy, iz) + cv(ix, iyp, iz) + cv(ixp, iyp, iz)
                 + cv(ix, iy, izp) + cv(ixp, iy, izp) + cv(ix, iyp, izp) + cv(ixp, iyp, izp);
      rho_v(ix, iy, iz) = rv / cvv;
      cv_v(ix, iy, iz) = 0.125 * cvv;
    });

    if (p.coronal_heating) {  // :127 user_defined_heating (radiative.f90:88-91)
      for (size_t q = 0; q < energy.size(); ++q)
        energy.d[q] = energy.d[q] + heat_in.d[q] * dt / rho.d[q];
      energy_bcs();
    }
    if (p.use_viscous_damping) viscous_damping();
    shock_viscosity();
    set_dt();
    dt2 = 0.5 * dt;

    last_substeps = 0;
    if (p.resistive_mhd) {
      double dt_sub = dtr;
      int substeps = (int)(dt / dt_sub) + 1;  // INT() truncates, :139
      if (substeps > peak_substeps) peak_substeps = substeps;
      last_substeps = substeps;
      double actual_dt = dt;
      dt = dt / (double)substeps;
      for (int sc = 1; sc <= substeps; ++sc) {
        eta_calc();
        if (eos_number() != LARE_EOS_IDEAL) neutral_fraction(energy);  // :147
        if (p.cowling_resistivity) perpendicular_resistivity();        // :148
        resistive_effects();
      }
      box(-1, nx + 2, -1, ny + 2, -1, nz + 2, [&](int ix, int iy, int iz) {
        int ixm = ix - 1, iym = iy - 1, izm = iz - 1;
        bx1(ix, iy, iz) = (bx(ix, iy, iz) + bx(ixm, iy, iz)) * 0.5;
        by1(ix, iy, iz) = (by(ix, iy, iz) + by(ix, iym, iz)) * 0.5;
        bz1(ix, iy, iz) = (bz(ix, iy, iz) + bz(ix, iy, izm)) * 0.5;
      });
      dt = actual_dt;
    }

    // :168-181 (radiation is not part of this path)
    delta_energy.fill(0.0);
    energy0.d = energy.d;
    if (p.conduction) {
      conduct_heat();
      for (size_t q = 0; q < energy.size(); ++q) delta_energy.d[q] = energy.d[q] - energy0.d[q];
      energy.d = energy0.d;
    }
    if (p.radiation) {
      rad_losses();
      for (size_t q = 0; q < energy.size(); ++q) delta_energy.d[q] = delta_energy.d[q] + (energy.d[q] - energy0.d[q]);
      energy.d = energy0.d;
    }
    for (size_t q = 0; q < energy.size(); ++q) energy.d[q] = energy0.d[q] + delta_energy.d[q];
    for (size_t q = 0; q < energy.size(); ++q) energy.d[q] = fmax0(energy.d[q]);

    predictor_corrector_step();

    energy_bcs();
    density_bcs();
    velocity_bcs();
    ++steps_taken;
  }

  // lagran.F90:208-478
  void predictor_corrector_step() {
    const double g = p.gamma, ip = p.ionise_pot;
    bx0.d = bx.d; by0.d = by.d; bz0.d = bz.d;

    b_field_and_cv1_update();
    // :230-232 (bx1 = bx1 * cv1) only feeds the CAUCHY branch; not built.

    box(0, nx + 1, 0, ny + 1, 0, nz + 1, [&](int ix, int iy, int iz) {
      double dv = cv1(ix, iy, iz) / cv(ix, iy, iz) - 1.0;
      double e1 = energy(ix, iy, iz) - pressure(ix, iy, iz) * dv / rho(ix, iy, iz);
      e1 = e1 + visc_heat(ix, iy, iz) * dt2 / rho(ix, iy, iz);
      pressure(ix, iy, iz) = (e1 - (1.0 - xi_n(ix, iy, iz)) * ip) * (g - 1.0) * rho(ix, iy, iz) * cv(ix, iy, iz)
                           / cv1(ix, iy, iz);
    });

    box(0, nx, 0, ny, 0, nz, [&](int ix, int iy, int iz) {
      int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
      double pp = pressure(ix, iy, iz), ppx = pressure(ixp, iy, iz), ppy = pressure(ix, iyp, iz);
      double ppz = pressure(ix, iy, izp), ppxy = pressure(ixp, iyp, iz), ppxz = pressure(ixp, iy, izp);
      double ppyz = pressure(ix, iyp, izp), ppxyz = pressure(ixp, iyp, izp);
      double w1 = (pp + ppy + ppz + ppyz) * 0.25;
      double w2 = (ppx + ppxy + ppxz + ppxyz) * 0.25;
      double fx = -(w2 - w1) / dxc(ix);
      w1 = (pp + ppx + ppz + ppxz) * 0.25;
      w2 = (ppy + ppxy + ppyz + ppxyz) * 0.25;
      double fy = -(w2 - w1) / dyc(iy);
      w1 = (pp + ppx + ppy + ppxy) * 0.25;
      w2 = (ppz + ppxz + ppyz + ppxyz) * 0.25;
      double fz = -(w2 - w1) / dzc(iz);

      double bxv = 0.25 * (bx(ix, iy, iz) + bx(ix, iyp, iz) + bx(ix, iy, izp) + bx(ix, iyp, izp));
      double byv = 0.25 * (by(ix, iy, iz) + by(ixp, iy, iz) + by(ix, iy, izp) + by(ixp, iy, izp));
      double bzv = 0.25 * (bz(ix, iy, iz) + bz(ix, iyp, iz) + bz(ixp, iy, iz) + bz(ixp, iyp, iz));

      double jx1 = (bz(ix, iyp, iz) - bz(ix, iy, iz)) / dyc(iy) - (by(ix, iy, izp) - by(ix, iy, iz)) / dzc(iz);
      double jx2 = (bz(ixp, iyp, iz) - bz(ixp, iy, iz)) / dyc(iy) - (by(ixp, iy, izp) - by(ixp, iy, iz)) / dzc(iz);
      double jy1 = (bx(ix, iy, izp) - bx(ix, iy, iz)) / dzc(iz) - (bz(ixp, iy, iz) - bz(ix, iy, iz)) / dxc(ix);
      double jy2 = (bx(ix, iyp, izp) - bx(ix, iyp, iz)) / dzc(iz) - (bz(ixp, iyp, iz) - bz(ix, iyp, iz)) / dxc(ix);
      double jz1 = (by(ixp, iy, iz) - by(ix, iy, iz)) / dxc(ix) - (bx(ix, iyp, iz) - bx(ix, iy, iz)) / dyc(iy);
      double jz2 = (by(ixp, iy, izp) - by(ix, iy, izp)) / dxc(ix) - (bx(ix, iyp, izp) - bx(ix, iy, izp)) / dyc(iy);
      double jx = (jx1 + jx2) * 0.5, jy = (jy1 + jy2) * 0.5, jz = (jz1 + jz2) * 0.5;

      double gb = gamma_boris(ix, iy, iz);
      fx = fx + gb * (jy * bzv - jz * byv);
      fy = fy + gb * (jz * bxv - jx * bzv);
      fz = fz + gb * (jx * byv - jy * bxv);
      fz = fz - rho_v(ix, iy, iz) * grav(iz);

      vx1(ix, iy, iz) = vx(ix, iy, iz) + dt2 * (fx_visc(ix, iy, iz) + fx) / rho_v(ix, iy, iz);
      vy1(ix, iy, iz) = vy(ix, iy, iz) + dt2 * (fy_visc(ix, iy, iz) + fy) / rho_v(ix, iy, iz);
      vz1(ix, iy, iz) = vz(ix, iy, iz) + dt2 * (fz_visc(ix, iy, iz) + fz) / rho_v(ix, iy, iz);
    });

    bx.d = bx0.d; by.d = by0.d; bz.d = bz0.d;
    remap_v_bcs();
    shock_heating();

    box(0, nx, 0, ny, 0, nz, [&](int ix, int iy, int iz) {
      vx(ix, iy, iz) = 2.0 * vx1(ix, iy, iz) - vx(ix, iy, iz);
      vy(ix, iy, iz) = 2.0 * vy1(ix, iy, iz) - vy(ix, iy, iz);
      vz(ix, iy, iz) = 2.0 * vz1(ix, iy, iz) - vz(ix, iy, iz);
    });
    velocity_bcs();
    if (any_open()) open_bcs();  // :409-412

    // :415-462, serial because of the total_visc_heating sum.
    for (int iz = 1; iz <= nz; ++iz) {
      int izm = iz - 1;
      for (int iy = 1; iy <= ny; ++iy) {
        int iym = iy - 1;
        for (int ix = 1; ix <= nx; ++ix) {
          int ixm = ix - 1;
          double vxb = (vx1(ix, iy, iz) + vx1(ix, iym, iz) + vx1(ix, iy, izm) + vx1(ix, iym, izm)) * 0.25;
          double vxbm = (vx1(ixm, iy, iz) + vx1(ixm, iym, iz) + vx1(ixm, iy, izm) + vx1(ixm, iym, izm)) * 0.25;
          double vyb = (vy1(ix, iy, iz) + vy1(ixm, iy, iz) + vy1(ix, iy, izm) + vy1(ixm, iy, izm)) * 0.25;
          double vybm = (vy1(ix, iym, iz) + vy1(ixm, iym, iz) + vy1(ix, iym, izm) + vy1(ixm, iym, izm)) * 0.25;
          double vzb = (vz1(ix, iy, iz) + vz1(ixm, iy, iz) + vz1(ix, iym, iz) + vz1(ixm, iym, iz)) * 0.25;
          double vzbm = (vz1(ix, iy, izm) + vz1(ixm, iy, izm) + vz1(ix, iym, izm) + vz1(ixm, iym, izm)) * 0.25;
          double dv = ((vxb - vxbm) / dxb(ix) + (vyb - vybm) / dyb(iy) + (vzb - vzbm) / dzb(iz)) * dt;
          cv1(ix, iy, iz) = cv(ix, iy, iz) * (1.0 + dv);
          energy(ix, iy, iz) = energy(ix, iy, iz)
              + (dt * visc_heat(ix, iy, iz) - dv * pressure(ix, iy, iz)) / rho(ix, iy, iz);
          visc_dep(ix, iy, iz) = visc_dep(ix, iy, iz) + dt * visc_heat(ix, iy, iz);
          rho(ix, iy, iz) = rho(ix, iy, iz) / (1.0 + dv);
          total_visc_heating = total_visc_heating + dt * visc_heat(ix, iy, iz) * cv(ix, iy, iz);
        }
      }
    }
    if (p.cooling_term) {  // :464-475
      const double al = p.alpha_av;
      box(1, nx, 1, ny, 1, nz, [&](int ix, int iy, int iz) {
        cool_term_v(ix, iy, iz) = al * dt * visc_heat(ix, iy, iz) / rho(ix, iy, iz)
                                + (1.0 - al) * cool_term_v(ix, iy, iz);
        energy(ix, iy, iz) = energy(ix, iy, iz) - cool_term_v(ix, iy, iz);
      });
      for (size_t q = 0; q < energy.size(); ++q) energy.d[q] = fmax0(energy.d[q]);
    }
  }

  // lagran.F90:483-524
  void viscous_damping() {
    qx.fill(0.0); qy.fill(0.0); qz.fill(0.0);
    box(0, nx, 0, ny, 0, nz, [&](int ix, int iy, int iz) {
      int ixp = ix + 1, ixm = ix - 1, iyp = iy + 1, iym = iy - 1, izp = iz + 1, izm = iz - 1;
      F3* vv[3] = {&vx, &vy, &vz};
      F3* qq[3] = {&qx, &qy, &qz};
      for (int c = 0; c < 3; ++c) {
        F3& v = *vv[c];
        (*qq[c])(ix, iy, iz) = visc3(ix, iy, iz)
            * (((v(ixp, iy, iz) - v(ix, iy, iz)) / dxb(ixp) - (v(ix, iy, iz) - v(ixm, iy, iz)) / dxb(ix)) / dxc(ix)
             + ((v(ix, iyp, iz) - v(ix, iy, iz)) / dyb(iyp) - (v(ix, iy, iz) - v(ix, iym, iz)) / dyb(iy)) / dyc(iy)
             + ((v(ix, iy, izp) - v(ix, iy, iz)) / dzb(izp) - (v(ix, iy, iz) - v(ix, iy, izm)) / dzb(iz)) / dzc(iz));
      }
    });
    box(0, nx, 0, ny, 0, nz, [&](int ix, int iy, int iz) {
      vx(ix, iy, iz) = vx(ix, iy, iz) + dt * qx(ix, iy, iz);
      vy(ix, iy, iz) = vy(ix, iy, iz) + dt * qy(ix, iy, iz);
      vz(ix, iy, iz) = vz(ix, iy, iz) + dt * qz(ix, iy, iz);
    });
  }

  // lagran.F90:795-855 edge_viscosity (default DEFINES: psi = 0).
  inline double edge_viscosity(double dvdots, int i1, int j1, int k1, int i2, int j2, int k2,
                               double dx) {
    dvdots = -std::fabs(dvdots);
    double r1 = rho_v(i1, j1, k1), r2 = rho_v(i2, j2, k2);
    double rho_edge = 2.0 * r1 * r2 / (r1 + r2);
    double cs_edge = std::fmin(cs_v(i1, j1, k1), cs_v(i2, j2, k2));
    double dvx = vx(i1, j1, k1) - vx(i2, j2, k2);
    double dvy = vy(i1, j1, k1) - vy(i2, j2, k2);
    double dvz = vz(i1, j1, k1) - vz(i2, j2, k2);
    double dv2 = dvx * dvx + dvy * dvy + dvz * dvz;
    double dv = std::sqrt(dv2);
    double psi = 0.0;
    if (dv * dt / dx < 1.e-14) dvdots = 0.0;
    else dvdots = dvdots / dv;
    double vc = p.visc1 * cs_edge;
    double q_k_bar = rho_edge * (visc2_norm * dv + std::sqrt(visc2_norm * visc2_norm * dv2 + vc * vc));
    return q_k_bar * (1.0 - psi) * dvdots;
  }

  // lagran.F90:532-857
  void shock_viscosity() {
    const double g = p.gamma;
    if (shock_first_call) {
      shock_first_call = false;
      visc2_norm = 0.25 * (g + 1.0) * p.visc2;
    }
    p_visc.fill(0.0);
    visc_heat.fill(0.0);
    box(-1, nx + 2, -1, ny + 2, -1, nz + 2, [&](int ix, int iy, int iz) {
      double rmin = std::fmax(rho(ix, iy, iz), none_zero);
      double b2 = bx1(ix, iy, iz) * bx1(ix, iy, iz) + by1(ix, iy, iz) * by1(ix, iy, iz)
                + bz1(ix, iy, iz) * bz1(ix, iy, iz);
      cs(ix, iy, iz) = std::sqrt((g * pressure(ix, iy, iz) + gamma_boris(ix, iy, iz) * b2) / rmin);
    });
    box(-1, nx + 1, -1, ny + 1, -1, nz + 1, [&](int ix, int iy, int iz) {
      int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
      double s = cs(ix, iy, iz) * cv(ix, iy, iz) + cs(ixp, iy, iz) * cv(ixp, iy, iz)
               + cs(ix, iyp, iz) * cv(ix, iyp, iz) + cs(ixp, iyp, iz) * cv(ixp, iyp, iz)
               + cs(ix, iy, izp) * cv(ix, iy, izp) + cs(ixp, iy, izp) * cv(ixp, iy, izp)
               + cs(ix, iyp, izp) * cv(ix, iyp, izp) + cs(ixp, iyp, izp) * cv(ixp, iyp, izp);
      cs_v(ix, iy, iz) = 0.125 * s / cv_v(ix, iy, iz);
    });
    box(0, nx + 1, 0, ny + 2, 0, nz + 2, [&](int ix, int iy, int iz) {
      int i1 = ix - 1, j1 = iy - 1, k1 = iz - 1, i2 = ix, j2 = iy - 1, k2 = iz - 1;
      double dvdots = -(vx(i1, j1, k1) - vx(i2, j2, k2));
      alpha1(ix, iy, iz) = edge_viscosity(dvdots, i1, j1, k1, i2, j2, k2, dxb(ix));
    });
    box(-1, nx + 1, 0, ny + 1, 0, nz + 2, [&](int ix, int iy, int iz) {
      int i1 = ix, j1 = iy - 1, k1 = iz - 1, i2 = ix, j2 = iy, k2 = iz - 1;
      double dvdots = -(vy(i1, j1, k1) - vy(i2, j2, k2));
      alpha2(ix, iy, iz) = edge_viscosity(dvdots, i1, j1, k1, i2, j2, k2, dyb(iy));
    });
    box(-1, nx + 1, -1, ny + 1, 0, nz + 1, [&](int ix, int iy, int iz) {
      int i1 = ix, j1 = iy, k1 = iz - 1, i2 = ix, j2 = iy, k2 = iz;
      double dvdots = -(vz(i1, j1, k1) - vz(i2, j2, k2));
      alpha3(ix, iy, iz) = edge_viscosity(dvdots, i1, j1, k1, i2, j2, k2, dzb(iz));
    });
    box(0, nx + 1, 0, ny + 1, 0, nz + 1, [&](int ix, int iy, int iz) {
      int ixm = ix - 1, iym = iy - 1, izm = iz - 1, iyp = iy + 1, izp = iz + 1;
      auto d2 = [&](int a0, int b0, int c0, int a1, int b1, int c1) {
        double ux = vx(a0, b0, c0) - vx(a1, b1, c1);
        double uy = vy(a0, b0, c0) - vy(a1, b1, c1);
        double uz = vz(a0, b0, c0) - vz(a1, b1, c1);
        return ux * ux + uy * uy + uz * uz;
      };
      double a1 = d2(ixm, iym, izm, ix, iym, izm);
      double a2 = d2(ix, iym, izm, ix, iy, izm);
      double a3 = d2(ix, iy, izm, ixm, iy, izm);
      double a4 = d2(ixm, iy, izm, ixm, iym, izm);
      double a5 = d2(ixm, iym, iz, ix, iym, iz);
      double a6 = d2(ix, iym, iz, ix, iy, iz);
      double a7 = d2(ix, iy, iz, ixm, iy, iz);
      double a8 = d2(ixm, iy, iz, ixm, iym, iz);
      double a9 = d2(ix, iy, izm, ix, iy, iz);
      double a10 = d2(ixm, iy, izm, ixm, iy, iz);
      double a11 = d2(ixm, iym, izm, ixm, iym, iz);
      double a12 = d2(ix, iym, izm, ix, iym, iz);
      double pv = p_visc(ix, iy, iz);
      pv = std::fmax(pv, -alpha1(ix, iy, iz) * std::sqrt(a1));
      pv = std::fmax(pv, -alpha2(ix, iy, iz) * std::sqrt(a2));
      pv = std::fmax(pv, -alpha3(ix, iy, iz) * std::sqrt(a9));
      p_visc(ix, iy, iz) = pv;
      double ddx = dxb(ix), ddy = dyb(iy), ddz = dzb(iz);
      double vh = -0.25 * ddy * ddz * alpha1(ix, iy, iz) * a1
                - 0.25 * ddx * ddz * alpha2(ix, iy, iz) * a2
                - 0.25 * ddy * ddz * alpha1(ix, iyp, iz) * a3
                - 0.25 * ddx * ddz * alpha2(ixm, iy, iz) * a4
                - 0.25 * ddy * ddz * alpha1(ix, iy, izp) * a5
                - 0.25 * ddx * ddz * alpha2(ix, iy, izp) * a6
                - 0.25 * ddy * ddz * alpha1(ix, iyp, izp) * a7
                - 0.25 * ddx * ddz * alpha2(ixm, iy, izp) * a8
                - 0.25 * ddx * ddy * alpha3(ix, iy, iz) * a9
                - 0.25 * ddx * ddy * alpha3(ixm, iy, iz) * a10
                - 0.25 * ddx * ddy * alpha3(ixm, iym, iz) * a11
                - 0.25 * ddx * ddy * alpha3(ix, iym, iz) * a12;
      visc_heat(ix, iy, iz) = vh / cv(ix, iy, iz);
    });
    fx_visc.fill(0.0); fy_visc.fill(0.0); fz_visc.fill(0.0);
    box(0, nx, 0, ny, 0, nz, [&](int ix, int iy, int iz) {
      int ixm = ix - 1, ixp = ix + 1, iym = iy - 1, iyp = iy + 1, izm = iz - 1, izp = iz + 1;
      double a1 = alpha1(ix, iyp, izp) * dyc(iy) * dzc(iz);
      double a2 = alpha1(ixp, iyp, izp) * dyc(iy) * dzc(iz);
      double a3 = alpha2(ix, iy, izp) * dxc(ix) * dzc(iz);
      double a4 = alpha2(ix, iyp, izp) * dxc(ix) * dzc(iz);
      double a5 = alpha3(ix, iy, iz) * dxc(ix) * dyc(iy);
      double a6 = alpha3(ix, iy, izp) * dxc(ix) * dyc(iy);
      F3* vv[3] = {&vx, &vy, &vz};
      F3* ff[3] = {&fx_visc, &fy_visc, &fz_visc};
      for (int c = 0; c < 3; ++c) {
        F3& v = *vv[c];
        double v0 = v(ix, iy, iz);
        (*ff[c])(ix, iy, iz) = (a1 * (v0 - v(ixm, iy, iz)) + a2 * (v0 - v(ixp, iy, iz))
                              + a3 * (v0 - v(ix, iym, iz)) + a4 * (v0 - v(ix, iyp, iz))
                              + a5 * (v0 - v(ix, iy, izm)) + a6 * (v0 - v(ix, iy, izp)))
                              / cv_v(ix, iy, iz);
      }
    });
  }

  // lagran.F90:861-937
  void shock_heating() {
    visc_heat.fill(0.0);
    box(0, nx + 1, 0, ny + 1, 0, nz + 1, [&](int ix, int iy, int iz) {
      int ixm = ix - 1, iym = iy - 1, izm = iz - 1, iyp = iy + 1, izp = iz + 1;
      auto dd = [&](int a0, int b0, int c0, int a1, int b1, int c1) {
        return (vx(a0, b0, c0) - vx(a1, b1, c1)) * (vx1(a0, b0, c0) - vx1(a1, b1, c1))
             + (vy(a0, b0, c0) - vy(a1, b1, c1)) * (vy1(a0, b0, c0) - vy1(a1, b1, c1))
             + (vz(a0, b0, c0) - vz(a1, b1, c1)) * (vz1(a0, b0, c0) - vz1(a1, b1, c1));
      };
      double a1 = dd(ixm, iym, izm, ix, iym, izm);
      double a2 = dd(ix, iym, izm, ix, iy, izm);
      double a3 = dd(ix, iy, izm, ixm, iy, izm);
      double a4 = dd(ixm, iy, izm, ixm, iym, izm);
      double a5 = dd(ixm, iym, iz, ix, iym, iz);
      double a6 = dd(ix, iym, iz, ix, iy, iz);
      double a7 = dd(ix, iy, iz, ixm, iy, iz);
      double a8 = dd(ixm, iy, iz, ixm, iym, iz);
      double a9 = dd(ix, iy, izm, ix, iy, iz);
      double a10 = dd(ixm, iy, izm, ixm, iy, iz);
      double a11 = dd(ixm, iym, izm, ixm, iym, iz);
      double a12 = dd(ix, iym, izm, ix, iym, iz);
      double ddx = dxb(ix), ddy = dyb(iy), ddz = dzb(iz);
      double vh = -0.25 * ddy * ddz * alpha1(ix, iy, iz) * a1
                - 0.25 * ddx * ddz * alpha2(ix, iy, iz) * a2
                - 0.25 * ddy * ddz * alpha1(ix, iyp, iz) * a3
                - 0.25 * ddx * ddz * alpha2(ixm, iy, iz) * a4
                - 0.25 * ddy * ddz * alpha1(ix, iy, izp) * a5
                - 0.25 * ddx * ddz * alpha2(ix, iy, izp) * a6
                - 0.25 * ddy * ddz * alpha1(ix, iyp, izp) * a7
                - 0.25 * ddx * ddz * alpha2(ixm, iy, izp) * a8
                - 0.25 * ddx * ddy * alpha3(ix, iy, iz) * a9
                - 0.25 * ddx * ddy * alpha3(ixm, iy, iz) * a10
                - 0.25 * ddx * ddy * alpha3(ixm, iym, iz) * a11
                - 0.25 * ddx * ddy * alpha3(ix, iym, iz) * a12;
      visc_heat(ix, iy, iz) = fmax0(vh / cv(ix, iy, iz));
    });
  }

  // lagran.F90:945-1062 (non-CAUCHY).  The cv1 computed at :952-983 is
  // overwritten by the first sweep of the predictor remap before any read,
  // so only the vx1 copy and the half-dt B-only remap matter.
  void b_field_and_cv1_update() {
    vx1.d = vx.d; vy1.d = vy.d; vz1.d = vz.d;
    predictor_step = true;
    dt = 0.5 * dt;
    eulerian_remap(cur_step);
    dt = 2.0 * dt;
    predictor_step = false;
  }

  // lagran.F90:1070-1166
  void set_dt() {
    if (set_dt_first) {
      set_dt_first = false;
      if (p.restart) { dt = p.dt_from_restart; return; }
    }
    double dt_local = largest_number, dtr_local = largest_number;
    gamma_boris.fill(1.0);
    const double g = p.gamma, va_max2 = p.va_max * p.va_max;
#pragma omp parallel for reduction(min : dt_local, dtr_local) schedule(static)
    for (int iz = 0; iz <= nz; ++iz)
      for (int iy = 0; iy <= ny; ++iy)
        for (int ix = 0; ix <= nx; ++ix) {
          double w1 = bx(ix, iy, iz) * bx(ix, iy, iz) + by(ix, iy, iz) * by(ix, iy, iz)
                    + bz(ix, iy, iz) * bz(ix, iy, iz);
          double rho0 = std::fmax(rho(ix, iy, iz), none_zero);
          double w2 = w1 / rho0;
          if (p.boris && (w2 >= va_max2)) gamma_boris(ix, iy, iz) = 1.0 / (1.0 + w2 / va_max2);
          double cs2 = (g * pressure(ix, iy, iz) + gamma_boris(ix, iy, iz) * w1) / rho0;
          double c_visc2 = p_visc(ix, iy, iz) / rho0;
          double length = fmin3(dxb(ix), dyb(iy), dzb(iz));
          double dt1 = length / (std::sqrt(c_visc2) + std::sqrt(cs2 + c_visc2));
          dt_local = std::fmin(dt_local, dt1);
          double dt2l = fmin3(dxb(ix) / std::fmax(std::fabs(vx(ix, iy, iz)), none_zero),
                              dyb(iy) / std::fmax(std::fabs(vy(ix, iy, iz)), none_zero),
                              dzb(iz) / std::fmax(std::fabs(vz(ix, iy, iz)), none_zero));
          dt_local = std::fmin(dt_local, dt2l);
          double dxlocal = 1.0 / (1.0 / (dxb(ix) * dxb(ix)) + 1.0 / (dyb(iy) * dyb(iy))
                                  + 1.0 / (dzb(iz) * dzb(iz)));
          double dt3 = largest_number;
          if (p.cowling_resistivity)  // :1132-1134
            dt3 = 0.2 * dxlocal / std::fmax(std::fmax(eta(ix, iy, iz), eta_perp(ix, iy, iz)), none_zero);
          else if (p.resistive_mhd)
            dt3 = 0.2 * dxlocal / std::fmax(eta(ix, iy, iz), none_zero);
          dtr_local = std::fmin(dtr_local, dt3);
        }
    dt = p.dt_multiplier * dt_local;
    dtr = p.dt_multiplier * dtr_local;
    if (p.conduction) {
      calc_s_stages(true);
      double ss_limit = 60;
      if (n_s_stages >= ss_limit) {
        dt = dt * (double)(2.0 * ss_limit * ss_limit - 9.0) / (double)(2 * n_s_stages * n_s_stages - 9);
        dtr = dtr * (double)(2.0 * ss_limit * ss_limit - 9.0) / (double)(2 * n_s_stages * n_s_stages - 9);
      }
    }
    time = time + dt;
  }

  // lagran.F90:1176-1230
  void eta_calc() {
    if (!p.resistive_mhd) { eta.fill(0.0); return; }
    box(-1, nx + 1, -1, ny + 1, -1, nz + 1, [&](int ix, int iy, int iz) {
      int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
      double jx = (bz(ix, iyp, iz) - bz(ix, iy, iz)) / dyc(iy) - (by(ix, iy, izp) - by(ix, iy, iz)) / dzc(iz);
      double jxp = (bz(ixp, iyp, iz) - bz(ixp, iy, iz)) / dyc(iy) - (by(ixp, iy, izp) - by(ixp, iy, iz)) / dzc(iz);
      double jy = (bx(ix, iy, izp) - bx(ix, iy, iz)) / dzc(iz) - (bz(ixp, iy, iz) - bz(ix, iy, iz)) / dxc(ix);
      double jyp = (bx(ix, iyp, izp) - bx(ix, iyp, iz)) / dzc(iz) - (bz(ixp, iyp, iz) - bz(ix, iyp, iz)) / dxc(ix);
      double jz = (by(ixp, iy, iz) - by(ix, iy, iz)) / dxc(ix) - (bx(ix, iyp, iz) - bx(ix, iy, iz)) / dyc(iy);
      double jzp = (by(ixp, iy, izp) - by(ix, iy, izp)) / dxc(ix) - (bx(ix, iyp, izp) - bx(ix, iy, izp)) / dyc(iy);
      jx = (jx + jxp) * 0.5; jy = (jy + jyp) * 0.5; jz = (jz + jzp) * 0.5;
      if (std::sqrt(jx * jx + jy * jy + jz * jz) > p.j_max) eta(ix, iy, iz) = p.eta_background + p.eta0;
      else eta(ix, iy, iz) = p.eta_background;
    });
  }

  // lagran.F90:1239-1452 (first order in time, no cooling term).  The
  // trailing rkstep (:1445) only refreshes temporaries that the next call
  // recomputes before use, and jx_r (:1417-1442) is an output-only
  // diagnostic; neither changes the state.
  void resistive_effects() {
    box(-1, nx + 2, -1, ny + 2, -1, nz + 2, [&](int ix, int iy, int iz) {
      bx1(ix, iy, iz) = bx(ix, iy, iz);
      by1(ix, iy, iz) = by(ix, iy, iz);
      bz1(ix, iy, iz) = bz(ix, iy, iz);
    });
    rkstep();
    bstep(dt);
    // :1270-1288 ohmic heating, 1:n
    box(1, nx, 1, ny, 1, nz, [&](int ix, int iy, int iz) {
      int ixm = ix - 1, iym = iy - 1, izm = iz - 1;
      double lh = +(curlb(ix, iy, iz) + curlb(ixm, iy, iz) + curlb(ix, iym, iz) + curlb(ixm, iym, iz)
                   + curlb(ix, iy, izm) + curlb(ixm, iy, izm) + curlb(ix, iym, izm) + curlb(ixm, iym, izm))
                  * dt / (8.0 * rho(ix, iy, iz));
      ohmic_dep(ix, iy, iz) = ohmic_dep(ix, iy, iz) + lh;
      energy(ix, iy, iz) = energy(ix, iy, iz) + lh;
    });
    if (p.cooling_term) {  // :1290-1302 (four curlb terms, the iz plane only)
      const double al = p.alpha_av;
      box(1, nx, 1, ny, 1, nz, [&](int ix, int iy, int iz) {
        int ixm = ix - 1, iym = iy - 1;
        double local_heating = (curlb(ix, iy, iz) + curlb(ixm, iy, iz) + curlb(ix, iym, iz) + curlb(ixm, iym, iz))
                             * dt / (4.0 * rho(ix, iy, iz));
        cool_term_b(ix, iy, iz) = al * local_heating + (1.0 - al) * cool_term_b(ix, iy, iz);
        energy(ix, iy, iz) = energy(ix, iy, iz) - cool_term_b(ix, iy, iz);
      });
    }
    for (size_t q = 0; q < energy.size(); ++q) energy.d[q] = fmax0(energy.d[q]);
    energy_bcs();
    for (int iz = 0; iz <= nz; ++iz)
      for (int iy = 0; iy <= ny; ++iy)
        for (int ix = 0; ix <= nx; ++ix) {
          double w1 = dt * dxc(ix) * dyc(iy) * dzc(iz) * curlb(ix, iy, iz);
          if (ix == 0 || ix == nx) w1 = w1 * 0.5;
          if (iy == 0 || iy == ny) w1 = w1 * 0.5;
          if (iz == 0 || iz == nz) w1 = w1 * 0.5;
          total_ohmic_heating = total_ohmic_heating + w1;
        }
  }

  // lagran.F90:1460-1503 (no Cowling resistivity)
  void rkstep() {
    box(0, nx, 0, ny, 0, nz, [&](int ix, int iy, int iz) {
      int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
      double jx1 = (bz(ix, iyp, iz) - bz(ix, iy, iz)) / dyc(iy) - (by(ix, iy, izp) - by(ix, iy, iz)) / dzc(iz);
      double jx2 = (bz(ixp, iyp, iz) - bz(ixp, iy, iz)) / dyc(iy) - (by(ixp, iy, izp) - by(ixp, iy, iz)) / dzc(iz);
      double jy1 = (bx(ix, iy, izp) - bx(ix, iy, iz)) / dzc(iz) - (bz(ixp, iy, iz) - bz(ix, iy, iz)) / dxc(ix);
      double jy2 = (bx(ix, iyp, izp) - bx(ix, iyp, iz)) / dzc(iz) - (bz(ixp, iyp, iz) - bz(ix, iyp, iz)) / dxc(ix);
      double jz1 = (by(ixp, iy, iz) - by(ix, iy, iz)) / dxc(ix) - (bx(ix, iyp, iz) - bx(ix, iy, iz)) / dyc(iy);
      double jz2 = (by(ixp, iy, izp) - by(ix, iy, izp)) / dxc(ix) - (bx(ix, iyp, izp) - bx(ix, iy, izp)) / dyc(iy);
      double jx = (jx1 + jx2) * 0.5, jy = (jy1 + jy2) * 0.5, jz = (jz1 + jz2) * 0.5;
      double e = eta(ix, iy, iz);
      if (!p.cowling_resistivity) {
        flux_x(ix, iy, iz) = -jx * e * dxc(ix) * 0.5;
        flux_y(ix, iy, iz) = -jy * e * dyc(iy) * 0.5;
        flux_z(ix, iy, iz) = -jz * e * dzc(iz) * 0.5;
        curlb(ix, iy, iz) = e * (jx * jx + jy * jy + jz * jz);
        return;
      }
      // :1527-1572, the partially ionised branch
      double bxv = (bx(ix, iy, iz) + bx(ix, iyp, iz) + bx(ix, iy, izp) + bx(ix, iyp, izp)) * 0.25;
      double byv = (by(ix, iy, iz) + by(ixp, iy, iz) + by(ix, iy, izp) + by(ixp, iy, izp)) * 0.25;
      double bzv = (bz(ix, iy, iz) + bz(ixp, iy, iz) + bz(ix, iyp, iz) + bz(ixp, iyp, iz)) * 0.25;
      double magn_b = bxv * bxv + byv * byv + bzv * bzv;
      double j_par_x = 0.0, j_par_y = 0.0, j_par_z = 0.0;
      if (magn_b > none_zero) {
        j_par_x = (jx * bxv + jy * byv + jz * bzv) * bxv / magn_b;
        j_par_y = (jx * bxv + jy * byv + jz * bzv) * byv / magn_b;
        j_par_z = (jx * bxv + jy * byv + jz * bzv) * bzv / magn_b;
      }
      double j_perp_x = jx - j_par_x, j_perp_y = jy - j_par_y, j_perp_z = jz - j_par_z;
      double magn_j_par = std::sqrt(j_par_x * j_par_x + j_par_y * j_par_y + j_par_z * j_par_z);
      double magn_j_perp = std::sqrt(j_perp_x * j_perp_x + j_perp_y * j_perp_y + j_perp_z * j_perp_z);
      double ep = eta_perp(ix, iy, iz);
      curlb(ix, iy, iz) = e * (magn_j_par * magn_j_par) + (ep + e) * (magn_j_perp * magn_j_perp);
      flux_x(ix, iy, iz) = -((j_par_x + j_perp_x) * e + j_perp_x * ep) * dxc(ix) * 0.5;
      flux_y(ix, iy, iz) = -((j_par_y + j_perp_y) * e + j_perp_y * ep) * dyc(iy) * 0.5;
      flux_z(ix, iy, iz) = -((j_par_z + j_perp_z) * e + j_perp_z * ep) * dzc(iz) * 0.5;
    });
  }

  int eos_number() const { return p.eos_number == 0 ? LARE_EOS_IDEAL : p.eos_number; }

  // diagnostics.F90:613-629
  void energy_correction() {
    for (size_t q = 0; q < delta_ke.d.size(); ++q) delta_ke.d[q] = -delta_ke.d[q];
    for (size_t q = 0; q < delta_ke.d.size(); ++q)
      if (delta_ke.d[q] < 0.0) delta_ke.d[q] = 0.0;
    for (size_t q = 0; q < delta_ke.d.size(); ++q) delta_ke.d[q] = delta_ke.d[q] / (rho.d[q] * cv.d[q]);
    box(1, nx, 1, ny, 1, nz, [&](int ix, int iy, int iz) {
      energy(ix, iy, iz) = energy(ix, iy, iz) + delta_ke(ix, iy, iz);
    });
    energy_bcs();
  }

  // radiative.f90:38-62 setup_loss_function and :180-208
  // set_exact_integration_arrays (n = 7 boundaries, kmax = 6 bands)
  struct Rad {
    double t_boundary[8], pow[7], psi[7], yk[8], qk[8], ratios[8];
    int alpha[7];
    double cool, ratio;
  };
  Rad rad;
  bool rad_first_call = true;
  void setup_radiation() {
    const int n = 7, kmax = 6;
    const double tb[] = {0.02, 0.0398, 0.0794, 0.251, 0.562, 1.995, 10.0};
    for (int i = 1; i <= n; ++i) rad.t_boundary[i] = tb[i - 1] * 1e6;
    const double frac = -2.0 / 3.0;
    const int al[] = {0, 2, 0, -2, 0, 0};
    const double ex[] = {0.0, 0.0, 0.0, 0.0, 0.0, frac};
    const double ps[] = {-21.85, -31.0, -21.2, -10.4, -21.94, -17.73};
    for (int k = 1; k <= kmax; ++k) {
      rad.alpha[k] = al[k - 1];
      rad.pow[k] = (double)al[k - 1] + ex[k - 1];
      rad.psi[k] = 1.e-13 * std::pow(10.0, ps[k - 1]);
    }
    for (int k = 1; k <= kmax; ++k) rad.qk[k] = rad.psi[k] * std::pow(rad.t_boundary[k], rad.pow[k]);
    rad.qk[n] = rad.qk[n - 1] * std::pow(rad.t_boundary[n] / rad.t_boundary[n - 1], rad.pow[n - 1]);
    rad.ratio = rad.qk[n] / rad.t_boundary[n];
    const double kb_si = 1.3806488e-23, mh_si = 1.672621777e-27;
    rad.cool = 0.5 * rad.ratio * (p.gamma - 1.0) * p.rho_norm / (kb_si * p.mf * mh_si);
    for (int k = 1; k <= n; ++k) rad.ratios[k] = rad.ratio * (rad.t_boundary[k] / rad.qk[k]);
    rad.yk[n] = 0.0;
    for (int k = kmax; k >= 1; --k) {
      if (rad.alpha[k] != 1) {
        double fac = 1.0 / (1.0 - rad.pow[k]);
        rad.yk[k] = rad.yk[k + 1]
                  - fac * rad.ratios[k] * (1.0 - std::pow(rad.t_boundary[k] / rad.t_boundary[k + 1], rad.pow[k] - 1.0));
      } else {
        rad.yk[k] = rad.yk[k + 1] - rad.ratios[k] * std::log(rad.t_boundary[k] / rad.t_boundary[k + 1]);
      }
    }
  }

  // radiative.f90:98-176 rad_losses / exact_intergation_method
  void rad_losses() {
    if (rad_first_call) { rad_first_call = false; setup_radiation(); }
    const int kmax = 6;
    const double g = p.gamma;
    box(1, nx, 1, ny, 1, nz, [&](int ix, int iy, int iz) {
      double temp_si = 0.5 * p.temp_norm * energy(ix, iy, iz) * (g - 1.0);
      int k = -1;
      for (int i = 1; i <= kmax; ++i)
        if (temp_si > rad.t_boundary[i] && temp_si <= rad.t_boundary[i + 1]) { k = i; break; }
      if (k < 0) return;
      double yt;
      if (rad.alpha[k] != 1) {
        double fac = 1.0 / (1.0 - rad.pow[k]);
        yt = rad.yk[k] + fac * rad.ratios[k] * (1.0 - std::pow(rad.t_boundary[k] / temp_si, rad.pow[k] - 1.0));
      } else {
        yt = rad.yk[k] + rad.ratios[k] * std::log(rad.t_boundary[k] / temp_si);
      }
      double inverse_t_cool = rad.cool * rho(ix, iy, iz);
      yt = yt + dt * inverse_t_cool * p.time_norm;
      k = -1;
      for (int i = 1; i <= kmax; ++i)
        if ((yt > rad.yk[i] && yt <= rad.yk[i + 1]) || (yt < rad.yk[i] && yt >= rad.yk[i + 1])) { k = i; break; }
      if (k < 0) {
        temp_si = rad.t_boundary[1];
        energy(ix, iy, iz) = temp_si * 2.0 / (g - 1.0) / p.temp_norm;
        return;
      }
      if (rad.alpha[k] != 1) {
        double fac = 1.0 / (1.0 - rad.pow[k]);
        temp_si = rad.t_boundary[k] * std::pow(1.0 - (1.0 - rad.pow[k]) / rad.ratios[k] * (yt - rad.yk[k]), fac);
      } else {
        temp_si = rad.t_boundary[k] * std::exp((yt - rad.yk[k]) / rad.ratios[k]);
      }
      energy(ix, iy, iz) = temp_si * 2.0 / (g - 1.0) / p.temp_norm;
    });
    energy_bcs();
  }

  // neutral.f90:140-153
  double get_neutral(double t_v, double rho_v) const {
    double t_rad = p.tr, dilution = 0.5;
    double bof = 1.0 / (dilution * p.f_bar * t_rad * std::sqrt(t_v))
               * cw_exp((0.25 * (t_v / t_rad - 1.0) + 1.0) * p.t_bar / t_v);
    double r = 0.5 * (-1.0 + std::sqrt(1.0 + p.r_bar * rho_v * bof));
    return r / (1.0 + r);
  }

  // neutral.f90:158-195, on the energy-like array e
  void neutral_fraction(F3& e) {
    const double g = p.gamma, ip = p.ionise_pot;
    box(-1, nx + 2, -1, ny + 2, -1, nz + 2, [&](int ix, int iy, int iz) {
      double rho0 = rho(ix, iy, iz), e0 = e(ix, iy, iz);
      double ta1 = (g - 1.0) * std::fmax((e0 - ip) / 2.0, none_zero), ta2 = (g - 1.0) * e0;
      if (ta1 > ta2) {
        eos_error = true;  // the reference prints and STOPs
        return;
      }
      double dx = ta2 - ta1, t = ta1, x = ta1;
      for (int loop = 1; loop <= 100; ++loop) {
        dx = dx / 2.0;
        x = t + dx;
        double xi_a = get_neutral(x, rho0);
        double fa = x - (g - 1.0) * (e0 - (1.0 - xi_a) * ip) / (2.0 - xi_a);
        if (fa <= 0.0) t = x;
        if (std::fabs(dx) < 1.e-8 || std::fabs(fa) < 1.e-8) break;
      }
      xi_n(ix, iy, iz) = get_neutral(x, rho0);
    });
  }

  // neutral.f90:68-124 (bxv and byv take their z terms from bz, as written)
  void perpendicular_resistivity() {
    const double g = p.gamma, ip = p.ionise_pot;
    box(0, nx, 0, ny, 0, nz, [&](int ix, int iy, int iz) {
      int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
      double rho_v = rho(ix, iy, iz) * cv(ix, iy, iz) + rho(ixp, iy, iz) * cv(ixp, iy, iz)
                   + rho(ix, iyp, iz) * cv(ix, iyp, iz) + rho(ixp, iyp, iz) * cv(ixp, iyp, iz)
                   + rho(ix, iy, izp) * cv(ix, iy, izp) + rho(ixp, iy, izp) * cv(ixp, iy, izp)
                   + rho(ix, iyp, izp) * cv(ix, iyp, izp) + rho(ixp, iyp, izp) * cv(ixp, iyp, izp);
      rho_v = rho_v / (cv(ix, iy, iz) + cv(ixp, iy, iz) + cv(ix, iyp, iz) + cv(ixp, iyp, iz)
                       + cv(ix, iy, izp) + cv(ixp, iy, izp) + cv(ix, iyp, izp) + cv(ixp, iyp, izp));
      double bxv = bx(ix, iy, iz) + bx(ix, iyp, iz) + bz(ix, iy, izp) + bz(ix, iyp, izp);
      double byv = by(ix, iy, iz) + by(ixp, iy, iz) + bz(ix, iy, izp) + bz(ixp, iy, izp);
      double bzv = bz(ix, iy, iz) + bz(ixp, iy, iz) + bz(ix, iyp, iz) + bz(ixp, iyp, iz);
      bxv = 0.25 * bxv;
      byv = 0.25 * byv;
      bzv = 0.25 * bzv;
      double bfieldsq = bxv * bxv + byv * byv + bzv * bzv;
      double t_v = 0.0;
      for (int iz2 = iz; iz2 <= iz + 1; ++iz2)
        for (int iy2 = iy; iy2 <= iy + 1; ++iy2)
          for (int ix2 = ix; ix2 <= ix + 1; ++ix2)
            t_v = t_v + (energy(ix2, iy2, iz2) - (1.0 - xi_n(ix2, iy2, iz2)) * ip) / (2.0 - xi_n(ix2, iy2, iz2));
      t_v = t_v * (g - 1.0) / 8.0;
      double xi_v = get_neutral(t_v, rho_v);
      double f = std::fmax(1.0 - xi_v, none_zero);
      if (f > 0) eta_perp(ix, iy, iz) = p.eta_bar * xi_v / f * bfieldsq / (rho_v * rho_v) / std::sqrt(t_v);
      else eta_perp(ix, iy, iz) = 0.0;
    });
    for (double& v : eta_perp.d) v = std::fmin(v, 100.0);  // :122
  }

  // lagran.F90:1582-1635
  void bstep(double dtl) {
    F3 &kx = flux_x, &ky = flux_y, &kz = flux_z;
    box(0, nx, 1, ny, 1, nz, [&](int ix, int iy, int iz) {
      int iym = iy - 1, izm = iz - 1;
      double area = dyb(iy) * dzb(iz);
      bx(ix, iy, iz) = bx1(ix, iy, iz)
          + (kz(ix, iy, iz) - kz(ix, iym, iz) + kz(ix, iy, izm) - kz(ix, iym, izm)
             - ky(ix, iy, iz) + ky(ix, iy, izm) - ky(ix, iym, iz) + ky(ix, iym, izm)) * dtl / area;
    });
    box(1, nx, 0, ny, 1, nz, [&](int ix, int iy, int iz) {
      int ixm = ix - 1, izm = iz - 1;
      double area = dxb(ix) * dzb(iz);
      by(ix, iy, iz) = by1(ix, iy, iz)
          + (kx(ix, iy, iz) - kx(ix, iy, izm) + kx(ixm, iy, iz) - kx(ixm, iy, izm)
             - kz(ix, iy, iz) + kz(ixm, iy, iz) - kz(ix, iy, izm) + kz(ixm, iy, izm)) * dtl / area;
    });
    box(1, nx, 1, ny, 0, nz, [&](int ix, int iy, int iz) {
      int ixm = ix - 1, iym = iy - 1;
      double area = dxb(ix) * dyb(iy);
      bz(ix, iy, iz) = bz1(ix, iy, iz)
          + (ky(ix, iy, iz) - ky(ixm, iy, iz) + ky(ix, iym, iz) - ky(ixm, iym, iz)
             - kx(ix, iy, iz) + kx(ix, iym, iz) - kx(ixm, iy, iz) + kx(ixm, iym, iz)) * dtl / area;
    });
    bfield_bcs();
  }

  // ------------------------------------------------------------------
  // remap.f90:33-131
  void eulerian_remap(int step) {
    if (p.rke) delta_ke.fill(0.0);  // remap.f90:38
    xpass = ypass = zpass = 1;
    box(-1, nx + 2, -1, ny + 2, -1, nz + 2, [&](int ix, int iy, int iz) {
      bx(ix, iy, iz) = bx(ix, iy, iz) * dyb(iy) * dzb(iz);
      by(ix, iy, iz) = by(ix, iy, iz) * dxb(ix) * dzb(iz);
      bz(ix, iy, iz) = bz(ix, iy, iz) * dxb(ix) * dyb(iy);
    });
    for (int iz = -1; iz <= nz + 2; ++iz)
      for (int iy = -1; iy <= ny + 2; ++iy) bx(-2, iy, iz) = bx(-2, iy, iz) * dyb(iy) * dzb(iz);
    for (int iz = -1; iz <= nz + 2; ++iz)
      for (int ix = -1; ix <= nx + 2; ++ix) by(ix, -2, iz) = by(ix, -2, iz) * dxb(ix) * dzb(iz);
    for (int iy = -1; iy <= ny + 2; ++iy)
      for (int ix = -1; ix <= nx + 2; ++ix) bz(ix, iy, -2) = bz(ix, iy, -2) * dxb(ix) * dyb(iy);

    static const int order[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {0, 2, 1}, {2, 1, 0}, {1, 0, 2}};
    int c = ((step % 6) + 6) % 6;  // MODULO
    for (int s = 0; s < 3; ++s) remap_axis(order[c][s]);

    box(-1, nx + 2, -1, ny + 2, -1, nz + 2, [&](int ix, int iy, int iz) {
      bx(ix, iy, iz) = bx(ix, iy, iz) / dyb(iy) / dzb(iz);
      by(ix, iy, iz) = by(ix, iy, iz) / dxb(ix) / dzb(iz);
      bz(ix, iy, iz) = bz(ix, iy, iz) / dxb(ix) / dyb(iy);
    });
    for (int iz = -1; iz <= nz + 2; ++iz)
      for (int iy = -1; iy <= ny + 2; ++iy) bx(-2, iy, iz) = bx(-2, iy, iz) / dyb(iy) / dzb(iz);
    for (int iz = -1; iz <= nz + 2; ++iz)
      for (int ix = -1; ix <= nx + 2; ++ix) by(ix, -2, iz) = by(ix, -2, iz) / dxb(ix) / dzb(iz);
    for (int iy = -1; iy <= ny + 2; ++iy)
      for (int ix = -1; ix <= nx + 2; ++ix) bz(ix, iy, -2) = bz(ix, iy, -2) / dxb(ix) / dyb(iy);
    bfield_bcs();
  }

  // Limited Van Leer flux shared by every *_flux routine of [xyz]remap.f90:
  // returns (fu + Di*(1 - w)) where w = phi or dmu is supplied by the caller
  // through `wfun` after vad_p/vad_m and dxbu are known.
  struct Lim {
    double sign_v, vad_p, vad_m, fu, Di, dxbu;
  };
  static inline Lim limiter(double v_advect, double fm, double fi, double fp, double fp2,
                            double dxci, double dxcm, double dxcp, double dxbi, double dxbp,
                            double phi_den_p, double phi_den_m, double dtl, double& phi,
                            bool phi_from_dxu) {
    Lim L;
    double dfm = fi - fm, dfi = fp - fi, dfp = fp2 - fp;
    L.sign_v = std::copysign(1.0, v_advect);
    L.vad_p = (L.sign_v + 1.0) * 0.5;
    L.vad_m = 1.0 - L.vad_p;
    L.fu = fi * L.vad_p + fp * L.vad_m;
    double dfu = dfm * L.vad_p + dfp * L.vad_m;
    double dxcu = dxcm * L.vad_p + dxcp * L.vad_m;
    L.dxbu = dxbi * L.vad_p + dxbp * L.vad_m;
    if (phi_from_dxu) {
      double dxu = phi_den_p * L.vad_p + phi_den_m * L.vad_m;
      phi = std::fabs(v_advect) * dtl / dxu;
    } else {
      phi = std::fabs(v_advect) * dtl / L.dxbu;
    }
    double Da = (2.0 - phi) * std::fabs(dfi) / dxci + (1.0 + phi) * std::fabs(dfu) / dxcu;
    Da = Da * sixth;
    double ss = 0.5 * (std::copysign(1.0, dfi) + std::copysign(1.0, dfu));
    L.Di = L.sign_v * ss * fmin3(std::fabs(Da) * L.dxbu, std::fabs(dfi), std::fabs(dfu));
    return L;
  }

  // Index helpers for an axis-generic sweep.  Unit offset along axis d.
  static inline void sh(const int* p, int d, int s, int* q) { q[0] = p[0]; q[1] = p[1]; q[2] = p[2]; q[d] += s; }

  // xremap.f90:37-336 remap_x and its mirrors yremap.f90:37-337,
  // zremap.f90:37-336.  The three files differ only by the axis
  // permutation, except for the loop ranges of the constrained-transport
  // updates, which are tabulated below exactly as written in each file.
  void remap_axis(int a) {
    const int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;  // transverse axes, t1 < t2
    F3& va = *V1[a];
    F3& db1 = r_db1;
    F3& dc1 = r_dc1;
    const F1& dba = *db[a];
    const int na = n[a];
    const double pass_t1 = (double)(t1 == 0 ? xpass : t1 == 1 ? ypass : zpass);
    const double pass_t2 = (double)(t2 == 0 ? xpass : t2 == 1 ? ypass : zpass);
    F3* vt[3] = {&vx1, &vy1, &vz1};
    const F1* dbb[3] = {&dxb, &dyb, &dzb};

    // First loop (xremap.f90:57-105): cv1, cv2, dxb1 over -1:n+2.
    box(-1, nx + 2, -1, ny + 2, -1, nz + 2, [&](int ix, int iy, int iz) {
      int ixm = ix - 1, iym = iy - 1, izm = iz - 1;
      double vxb = (vx1(ix, iy, iz) + vx1(ix, iym, iz) + vx1(ix, iy, izm) + vx1(ix, iym, izm)) * 0.25;
      double vxbm = (vx1(ixm, iy, iz) + vx1(ixm, iym, iz) + vx1(ixm, iy, izm) + vx1(ixm, iym, izm)) * 0.25;
      double vyb = (vy1(ix, iy, iz) + vy1(ixm, iy, iz) + vy1(ix, iy, izm) + vy1(ixm, iy, izm)) * 0.25;
      double vybm = (vy1(ix, iym, iz) + vy1(ixm, iym, iz) + vy1(ix, iym, izm) + vy1(ixm, iym, izm)) * 0.25;
      double vzb = (vz1(ix, iy, iz) + vz1(ixm, iy, iz) + vz1(ix, iym, iz) + vz1(ixm, iym, iz)) * 0.25;
      double vzbm = (vz1(ix, iy, izm) + vz1(ixm, iy, izm) + vz1(ix, iym, izm) + vz1(ixm, iym, izm)) * 0.25;
      double dvv[3] = {vxb - vxbm, vyb - vybm, vzb - vzbm};
      int pp[3] = {ix, iy, iz};
      double term_t1 = pass_t1 * dvv[t1] / (*dbb[t1])(pp[t1]);
      double term_t2 = pass_t2 * dvv[t2] / (*dbb[t2])(pp[t2]);
      double term_a = dvv[a] / (*dbb[a])(pp[a]);
      double dv = (term_t1 + term_t2 + term_a) * dt;
      cv1(ix, iy, iz) = cv(ix, iy, iz) * (1.0 + dv);
      dv = (term_t1 + term_t2) * dt;
      r_cv2(ix, iy, iz) = cv(ix, iy, iz) * (1.0 + dv);
      db1(ix, iy, iz) = dba(pp[a]) + dvv[a] * dt;
    });
    // dxc1 (xremap.f90:107-115)
    box(-1, nx + 2, -1, ny + 2, -1, nz + 2, [&](int ix, int iy, int iz) {
      int pp[3] = {ix, iy, iz}, q[3];
      sh(pp, a, 0, q);
      q[a] = std::min(pp[a] + 1, na + 2);
      dc1(ix, iy, iz) = 0.5 * (db1(ix, iy, iz) + db1(q[0], q[1], q[2]));
    });

    // Constrained-transport B flux remap.  For the sweep along a the two
    // transported components are b (first) and then the other one.
    const int bfirst = a == 0 ? 1 : 0;
    const int bsecond = a == 2 ? 1 : 2;
    // Ranges [lo..hi] per dimension of the two updates after each flux
    // routine, as written in each file (xremap.f90:121-157,
    // yremap.f90:122-158, zremap.f90:121-157).
    struct R { int l[3], h[3]; };
    auto full = [&]() { R r; for (int d = 0; d < 3; ++d) { r.l[d] = 0; r.h[d] = n[d] + 1; } return r; };
    R r1a = full(), r1b = full(), r2a = full(), r2b = full();
    if (a == 0) {
      // bz update: iz 0:nz, iy 1:ny, ix 1:nx ; bx update: iz 0:nz+1, iy 0:ny+1, ix 0:nx
      r2a.l[0] = 1; r2a.h[0] = nx; r2a.l[1] = 1; r2a.h[1] = ny; r2a.l[2] = 0; r2a.h[2] = nz;
      r2b.l[0] = 0; r2b.h[0] = nx;
    } else if (a == 1) {
      // second by update: iz 1:nz, iy 0:ny, ix 1:nx
      r2b.l[0] = 1; r2b.h[0] = nx; r2b.l[1] = 0; r2b.h[1] = ny; r2b.l[2] = 1; r2b.h[2] = nz;
    }
    for (int pass = 0; pass < 2; ++pass) {
      const int b = pass == 0 ? bfirst : bsecond;
      const int o = 3 - a - b;
      F3& Bb = *B[b];
      F3& Ba = *B[a];
      F3& flux = r_flux[a];
      // v[ab]_b?_flux (xremap.f90:340-403, 407-470 and mirrors)
      box(-1, nx + 1, -1, ny + 1, -1, nz + 1, [&](int ix, int iy, int iz) {
        int pp[3] = {ix, iy, iz}, pm[3], pq[3], pp2[3], po[3], t[3];
        sh(pp, a, 0, pm); pm[a] = std::max(pp[a] - 1, -1);
        sh(pp, a, 1, pq);
        sh(pp, a, 0, pp2); pp2[a] = std::min(pp[a] + 2, na + 2);
        sh(pp, o, -1, po);
        double v_advect = (va(pp[0], pp[1], pp[2]) + va(po[0], po[1], po[2])) * 0.5;
        auto dbv = [&](const int* q) { sh(q, b, 1, t); return (db1(q[0], q[1], q[2]) + db1(t[0], t[1], t[2])) * 0.5; };
        double dbx = dbv(pp), dbxp = dbv(pq), dbxp2 = dbv(pp2), dbxm = dbv(pm);
        double fm = Bb(pm[0], pm[1], pm[2]) / dbxm;
        double fi = Bb(pp[0], pp[1], pp[2]) / dbx;
        double fp = Bb(pq[0], pq[1], pq[2]) / dbxp;
        double fp2 = Bb(pp2[0], pp2[1], pp2[2]) / dbxp2;
        double phi;
        Lim L = limiter(v_advect, fm, fi, fp, fp2, dc1(pp[0], pp[1], pp[2]), dc1(pm[0], pm[1], pm[2]),
                        dc1(pq[0], pq[1], pq[2]), db1(pp[0], pp[1], pp[2]), db1(pq[0], pq[1], pq[2]),
                        dbx, dbxp, dt, phi, true);
        flux(ix, iy, iz) = (L.fu + L.Di * (1.0 - phi)) * v_advect * dt;
      });
      const R& ra = pass == 0 ? r1a : r2a;
      const R& rb = pass == 0 ? r1b : r2b;
      box(ra.l[0], ra.h[0], ra.l[1], ra.h[1], ra.l[2], ra.h[2], [&](int ix, int iy, int iz) {
        int pp[3] = {ix, iy, iz}, q[3];
        sh(pp, a, -1, q);
        Bb(ix, iy, iz) = Bb(ix, iy, iz) - flux(ix, iy, iz) + flux(q[0], q[1], q[2]);
      });
      box(rb.l[0], rb.h[0], rb.l[1], rb.h[1], rb.l[2], rb.h[2], [&](int ix, int iy, int iz) {
        int pp[3] = {ix, iy, iz}, q[3];
        sh(pp, b, -1, q);
        Ba(ix, iy, iz) = Ba(ix, iy, iz) + flux(ix, iy, iz) - flux(q[0], q[1], q[2]);
      });
    }

    if (predictor_step) return;  // xremap.f90:159-162 (pass flag not reset)

    F3& dm = r_dm;
    F3& rho1 = r_rho1;
    F3& cv2 = r_cv2;
    F3& flux = r_flux[a];
    dm.fill(0.0);
    rho1.d = rho.d;
    // x_mass_flux (xremap.f90:474-533): a 0:n, transverse 0:n+1
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) { lo[d] = 0; hi[d] = n[d] + 1; }
    hi[a] = na;
    auto vadv4 = [&](const int* pp) {
      int q1[3], q2[3], q12[3];
      sh(pp, t1, -1, q1); sh(pp, t2, -1, q2); sh(q1, t2, -1, q12);
      return (va(pp[0], pp[1], pp[2]) + va(q1[0], q1[1], q1[2]) + va(q2[0], q2[1], q2[2])
              + va(q12[0], q12[1], q12[2])) * 0.25;
    };
    auto area_b = [&](const int* pp) { return (*dbb[t1])(pp[t1]) * (*dbb[t2])(pp[t2]); };
    box(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], [&](int ix, int iy, int iz) {
      int pp[3] = {ix, iy, iz}, pm[3], pq[3], pp2[3];
      sh(pp, a, -1, pm); sh(pp, a, 1, pq); sh(pp, a, 2, pp2);
      double area = area_b(pp);
      double v_advect = vadv4(pp);
      double phi;
      Lim L = limiter(v_advect, rho(pm[0], pm[1], pm[2]), rho(ix, iy, iz), rho(pq[0], pq[1], pq[2]),
                      rho(pp2[0], pp2[1], pp2[2]), dc1(ix, iy, iz), dc1(pm[0], pm[1], pm[2]),
                      dc1(pq[0], pq[1], pq[2]), db1(ix, iy, iz), db1(pq[0], pq[1], pq[2]), 0, 0, dt, phi,
                      false);
      dm(ix, iy, iz) = (L.fu + L.Di * (1.0 - phi)) * v_advect * dt * area;
    });
    dm_bcs(a);
    box(1, nx, 1, ny, 1, nz, [&](int ix, int iy, int iz) {
      int pp[3] = {ix, iy, iz}, q[3];
      sh(pp, a, -1, q);
      rho(ix, iy, iz) = (rho1(ix, iy, iz) * cv1(ix, iy, iz) + dm(q[0], q[1], q[2]) - dm(ix, iy, iz))
                      / cv2(ix, iy, iz);
    });
    // x_energy_flux (xremap.f90:539-601): all 0:n
    box(0, nx, 0, ny, 0, nz, [&](int ix, int iy, int iz) {
      int pp[3] = {ix, iy, iz}, pm[3], pq[3], pp2[3];
      sh(pp, a, -1, pm); sh(pp, a, 1, pq); sh(pp, a, 2, pp2);
      double area = area_b(pp);
      double v_advect = vadv4(pp);
      double phi;
      Lim L = limiter(v_advect, energy(pm[0], pm[1], pm[2]), energy(ix, iy, iz),
                      energy(pq[0], pq[1], pq[2]), energy(pp2[0], pp2[1], pp2[2]), dc1(ix, iy, iz),
                      dc1(pm[0], pm[1], pm[2]), dc1(pq[0], pq[1], pq[2]), db1(ix, iy, iz),
                      db1(pq[0], pq[1], pq[2]), 0, 0, dt, phi, false);
      double rhou = rho1(ix, iy, iz) * L.vad_p + rho1(pq[0], pq[1], pq[2]) * L.vad_m;
      double dmu = std::fabs(dm(ix, iy, iz)) / area / L.dxbu / rhou;
      flux(ix, iy, iz) = (L.fu + L.Di * (1.0 - dmu)) * dm(ix, iy, iz);
    });
    box(1, nx, 1, ny, 1, nz, [&](int ix, int iy, int iz) {
      int pp[3] = {ix, iy, iz}, q[3];
      sh(pp, a, -1, q);
      energy(ix, iy, iz) = (energy(ix, iy, iz) * cv1(ix, iy, iz) * rho1(ix, iy, iz)
                            + flux(q[0], q[1], q[2]) - flux(ix, iy, iz))
                         / (cv2(ix, iy, iz) * rho(ix, iy, iz));
    });

    // Vertex quantities (xremap.f90:201-290).
    F3& rv = r_rho_v;
    F3& rv1 = r_rho_v1;
    for (int d = 0; d < 3; ++d) { lo[d] = 0; hi[d] = n[d]; }
    lo[a] = -1; hi[a] = na + 1;
    box(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], [&](int ix, int iy, int iz) {
      int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
      double s = rho1(ix, iy, iz) * cv1(ix, iy, iz) + rho1(ixp, iy, iz) * cv1(ixp, iy, iz)
               + rho1(ix, iyp, iz) * cv1(ix, iyp, iz) + rho1(ixp, iyp, iz) * cv1(ixp, iyp, iz)
               + rho1(ix, iy, izp) * cv1(ix, iy, izp) + rho1(ixp, iy, izp) * cv1(ixp, iy, izp)
               + rho1(ix, iyp, izp) * cv1(ix, iyp, izp) + rho1(ixp, iyp, izp) * cv1(ixp, iyp, izp);
      rv(ix, iy, iz) = s / (cv1(ix, iy, iz) + cv1(ixp, iy, iz) + cv1(ix, iyp, iz) + cv1(ixp, iyp, iz)
                            + cv1(ix, iy, izp) + cv1(ixp, iy, izp) + cv1(ix, iyp, izp) + cv1(ixp, iyp, izp));
    });
    auto avg8 = [&](F3& src, F3& dst, int i0, int i1, int j0, int j1, int k0, int k1) {
      box(i0, i1, j0, j1, k0, k1, [&](int ix, int iy, int iz) {
        int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
        flux(ix, iy, iz) = src(ix, iy, iz) + src(ixp, iy, iz) + src(ix, iyp, iz) + src(ixp, iyp, iz)
                         + src(ix, iy, izp) + src(ixp, iy, izp) + src(ix, iyp, izp) + src(ixp, iyp, izp);
      });
      box(i0, i1, j0, j1, k0, k1, [&](int ix, int iy, int iz) {
        dst(ix, iy, iz) = flux(ix, iy, iz) * 0.125;
      });
    };
    avg8(cv1, cv1, 0, nx, 0, ny, 0, nz);
    avg8(cv2, cv2, 0, nx, 0, ny, 0, nz);
    // v1 along a at faces of the vertex cell: a -2:n+1, transverse 0:n
    for (int d = 0; d < 3; ++d) { lo[d] = 0; hi[d] = n[d]; }
    lo[a] = -2; hi[a] = na + 1;
    box(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], [&](int ix, int iy, int iz) {
      int pp[3] = {ix, iy, iz}, q[3];
      sh(pp, a, 1, q);
      flux(ix, iy, iz) = (va(ix, iy, iz) + va(q[0], q[1], q[2])) * 0.5;
    });
    box(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], [&](int ix, int iy, int iz) { va(ix, iy, iz) = flux(ix, iy, iz); });
    // dm at vertex faces: a -1:n, transverse 0:n
    lo[a] = -1; hi[a] = na;
    {
      int l0 = lo[0], h0 = hi[0], l1 = lo[1], h1 = hi[1], l2 = lo[2], h2 = hi[2];
      avg8(dm, dm, l0, h0, l1, h1, l2, h2);
    }
    box(0, nx, 0, ny, 0, nz, [&](int ix, int iy, int iz) {
      int pp[3] = {ix, iy, iz}, q[3];
      sh(pp, a, -1, q);
      rv1(ix, iy, iz) = (rv(ix, iy, iz) * cv1(ix, iy, iz) + dm(q[0], q[1], q[2]) - dm(ix, iy, iz))
                      / cv2(ix, iy, iz);
    });
    // x_mom{x,y,z}_flux (xremap.f90:605-895) and the v updates (:292-329)
    const F1* dcc[3] = {&dxc, &dyc, &dzc};
    for (int comp = 0; comp < 3; ++comp) {
      F3& vc = *V[comp];
      for (int d = 0; d < 3; ++d) { lo[d] = 0; hi[d] = n[d]; }
      lo[a] = -1; hi[a] = na;
      box(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], [&](int ix, int iy, int iz) {
        int pp[3] = {ix, iy, iz}, pm[3], pq[3], pp2[3];
        sh(pp, a, -1, pm); sh(pp, a, 1, pq); sh(pp, a, 2, pp2);
        double area = (*dcc[t1])(pp[t1]) * (*dcc[t2])(pp[t2]);
        double v_advect = va(ix, iy, iz);
        double phi;
        Lim L = limiter(v_advect, vc(pm[0], pm[1], pm[2]), vc(ix, iy, iz), vc(pq[0], pq[1], pq[2]),
                        vc(pp2[0], pp2[1], pp2[2]), db1(pq[0], pq[1], pq[2]), db1(ix, iy, iz),
                        db1(pp2[0], pp2[1], pp2[2]), dc1(ix, iy, iz), dc1(pq[0], pq[1], pq[2]), 0, 0, dt,
                        phi, false);
        double rhou = rv(ix, iy, iz) * L.vad_p + rv(pq[0], pq[1], pq[2]) * L.vad_m;
        double dmu = std::fabs(dm(ix, iy, iz)) / area / L.dxbu / rhou;
        flux(ix, iy, iz) = L.fu + L.Di * (1.0 - dmu);
      });
      if (p.rke) {
        // xremap.f90:664-695 (and the eight siblings): serial, in the
        // reference's loop order, because the scatter adds into shared cells
        int rlo[3] = {0, 0, 0}, rhi[3] = {nx, ny, nz};
        rhi[a] = na - 1;
        const int u = a == 0 ? 1 : 0, w = a == 2 ? 1 : 2;  // transverse axes, u < w
        for (int iz = rlo[2]; iz <= rhi[2]; ++iz)
          for (int iy = rlo[1]; iy <= rhi[1]; ++iy)
            for (int ix = rlo[0]; ix <= rhi[0]; ++ix) {
              int pp[3] = {ix, iy, iz}, pm[3], pq[3];
              sh(pp, a, -1, pm);
              sh(pp, a, 1, pq);
              double m = rv1(ix, iy, iz) * cv2(ix, iy, iz);
              double mp = rv1(pq[0], pq[1], pq[2]) * cv2(pq[0], pq[1], pq[2]);
              double v0 = vc(ix, iy, iz), v1 = vc(pq[0], pq[1], pq[2]);
              double fm = flux(pm[0], pm[1], pm[2]), f0 = flux(ix, iy, iz), fp = flux(pq[0], pq[1], pq[2]);
              double dmm = dm(pm[0], pm[1], pm[2]), dm0 = dm(ix, iy, iz), dmp = dm(pq[0], pq[1], pq[2]);
              double ai = (v0 - fm) * dmm / m - (v0 - f0) * dm0 / m;
              double aip = (v1 - f0) * dm0 / mp - (v1 - fp) * dmp / mp;
              double dk = (v1 - v0) * (f0 - 0.5 * (v1 + v0)) - 0.5 * ai * (v0 - f0) + 0.5 * aip * (v1 - f0);
              dk = dk * dm0 * 0.5;
              int t[3] = {pq[0], pq[1], pq[2]};
              delta_ke(t[0], t[1], t[2]) = delta_ke(t[0], t[1], t[2]) + dk;
              t[u] += 1;
              delta_ke(t[0], t[1], t[2]) = delta_ke(t[0], t[1], t[2]) + dk;
              t[u] -= 1;
              t[w] += 1;
              delta_ke(t[0], t[1], t[2]) = delta_ke(t[0], t[1], t[2]) + dk;
              t[u] += 1;
              delta_ke(t[0], t[1], t[2]) = delta_ke(t[0], t[1], t[2]) + dk;
            }
      }
      box(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], [&](int ix, int iy, int iz) {
        flux(ix, iy, iz) = flux(ix, iy, iz) * dm(ix, iy, iz);
      });
      box(0, nx, 0, ny, 0, nz, [&](int ix, int iy, int iz) {
        int pp[3] = {ix, iy, iz}, q[3];
        sh(pp, a, -1, q);
        vc(ix, iy, iz) = (rv(ix, iy, iz) * vc(ix, iy, iz) * cv1(ix, iy, iz) + flux(q[0], q[1], q[2])
                          - flux(ix, iy, iz))
                       / (cv2(ix, iy, iz) * rv1(ix, iy, iz));
      });
    }
    boundary_conditions();
    if (a == 0) xpass = 0;
    else if (a == 1) ypass = 0;
    else zpass = 0;
    (void)vt;
  }

  // ------------------------------------------------------------------
  // conduct.f90:39-48
  void conduct_heat() {
    calc_s_stages(false);
    heat_conduct_sts2();
  }

  void temperature_from(F3& e) {
    const double g = p.gamma, ip = p.ionise_pot;
    box(-1, nx + 2, -1, ny + 2, -1, nz + 2, [&](int ix, int iy, int iz) {
      const double xi = xi_n(ix, iy, iz);
      temperature(ix, iy, iz) = (g - 1.0) / (2.0 - xi) * (e(ix, iy, iz) - (1.0 - xi) * ip);
    });
  }

  // conduct.f90:56-143
  void calc_s_stages(bool lagrangian_call) {
    (void)lagrangian_call;
    const double g = p.gamma, xi = p.xi_n, ip = p.ionise_pot, k0 = p.kappa_0;
    temperature_from(energy);
    box(0, nx, 0, ny, 0, nz, [&](int ix, int iy, int iz) {
      int ixm = ix - 1, ixp = ix + 1, iym = iy - 1, iyp = iy + 1, izm = iz - 1, izp = iz + 1;
      double T = temperature(ix, iy, iz);
      double temp = std::pow(T, pow_c);
      double q_fs = p.flux_limiter * 42.85 * rho(ix, iy, iz) * std::pow(T, 1.5);
      double q_fs2 = q_fs * q_fs;
      double q_spx = -k0 * temp * (temperature(ixp, iy, iz) - temperature(ixm, iy, iz)) * 0.5 / dxb(ix);
      double q_spy = -k0 * temp * (temperature(ix, iyp, iz) - temperature(ix, iym, iz)) * 0.5 / dyb(iy);
      double q_spz = -k0 * temp * (temperature(ix, iy, izp) - temperature(ix, iy, izm)) * 0.5 / dzb(iz);
      double q_sp2 = q_spx * q_spx + q_spy * q_spy + q_spz * q_spz;
      larsen_factor(ix, iy, iz) = q_fs / std::sqrt(q_fs2 + q_sp2);
    });
    if (!p.heat_flux_limiter) larsen_factor.fill(1.0);
    double dt_parab = 1.e10;
#pragma omp parallel for reduction(min : dt_parab) schedule(static)
    for (int iz = 1; iz <= nz; ++iz)
      for (int iy = 1; iy <= ny; ++iy)
        for (int ix = 1; ix <= nx; ++ix) {
          double kappa1 = k0 * larsen_factor(ix, iy, iz);
          double temp = (g - 1.0) / (2.0 - xi_n(ix, iy, iz)) * (energy(ix, iy, iz) - (1.0 - xi_n(ix, iy, iz)) * ip);
          double tp = std::pow(temp, pow_c);
          double r = rho(ix, iy, iz);
          double dt1 = r * (dxb(ix) * dxb(ix)) / (2.0 * kappa1 * tp);
          double dt2l = r * (dyb(iy) * dyb(iy)) / (2.0 * kappa1 * tp);
          double dt3 = r * (dzb(iz) * dzb(iz)) / (2.0 * kappa1 * tp);
          dt_parab = std::fmin(dt_parab, std::fmin(std::fmin(dt1, dt2l), dt3));
        }
    dt_parab = p.dt_multiplier * dt_parab / std::sqrt(3.0);
    double stages = 0.5 * (std::sqrt(9.0 + 16.0 * (dt / dt_parab)) - 1.0);
    int ns = (int)std::ceil(stages);
    if (ns % 2 == 0) ns = ns + 1;
    n_s_stages = ns;
  }

  // conduct.f90:152-291 as a gather: each cell sums its six face fluxes in
  // the order the reference's scatter loop delivers them (see kernel docs).
  inline double face_flux(int axis, int ix, int iy, int iz) {
    F3& T = temperature;
    const double k0 = p.kappa_0;
    // Extension, not in the reference: a cross-field conductivity
    // kappa_perp = rp kappa_par adds rp (g_n - b_n (b . g) / |b|^2) to the
    // bracket; rp = 0 leaves the reference's expression untouched.
    const double rp = p.kappa_perp_ratio;
    int ixp = ix + 1, ixm = ix - 1, iyp = iy + 1, iym = iy - 1, izp = iz + 1, izm = iz - 1;
    double lf = larsen_factor(ix, iy, iz);
    if (axis == 0) {
      double byf = 0.25 * (by(ix, iy, iz) + by(ixp, iy, iz) + by(ix, iym, iz) + by(ixp, iym, iz));
      double bzf = 0.25 * (bz(ix, iy, iz) + bz(ixp, iy, iz) + bz(ix, iy, izm) + bz(ixp, iy, izm));
      double b0 = bx(ix, iy, iz);
      double modb = b0 * b0 + byf * byf + bzf * bzf + min_b;
      double tb = (T(ixp, iy, iz) + T(ix, iy, iz)) / 2.0;
      double tb_p = (T(ixp, iyp, iz) + T(ix, iyp, iz)) / 2.0;
      double tb_m = (T(ixp, iym, iz) + T(ix, iym, iz)) / 2.0;
      double tg_a1 = (tb_p - tb_m) / (dyc(iy) + dyc(iym));
      tb_p = (T(ixp, iy, izp) + T(ix, iy, izp)) / 2.0;
      tb_m = (T(ixp, iy, izm) + T(ix, iy, izm)) / 2.0;
      double tg_a2 = (tb_p - tb_m) / (dzc(iz) + dzc(izm));
      double tg = (T(ixp, iy, iz) - T(ix, iy, iz)) / dxc(ix);
      tb = fmax0(tb);
      if (rp != 0.0) {
        double bg = b0 * (tg * b0 + tg_a1 * byf + tg_a2 * bzf);
        return -lf * k0 * std::pow(tb, pow_c) * ((bg + tg * min_b) / modb + rp * (tg - bg / modb));
      }
      return -lf * k0 * std::pow(tb, pow_c) * (b0 * (tg * b0 + tg_a1 * byf + tg_a2 * bzf) + tg * min_b) / modb;
    } else if (axis == 1) {
      double bxf = 0.25 * (bx(ix, iy, iz) + bx(ix, iyp, iz) + bx(ixm, iy, iz) + bx(ixm, iyp, iz));
      double bzf = 0.25 * (bz(ix, iy, iz) + bz(ix, iyp, iz) + bz(ix, iy, izm) + bz(ix, iyp, izm));
      double b0 = by(ix, iy, iz);
      double modb = bxf * bxf + b0 * b0 + bzf * bzf + min_b;
      double tb = (T(ix, iyp, iz) + T(ix, iy, iz)) / 2.0;
      double tb_p = (T(ixp, iy, iz) + T(ixp, iyp, iz)) / 2.0;
      double tb_m = (T(ixm, iyp, iz) + T(ixm, iy, iz)) / 2.0;
      double tg_a1 = (tb_p - tb_m) / (dxc(ix) + dxc(ixm));
      tb_p = (T(ix, iyp, izp) + T(ix, iy, izp)) / 2.0;
      tb_m = (T(ix, iyp, izm) + T(ix, iy, izm)) / 2.0;
      double tg_a2 = (tb_p - tb_m) / (dzc(iz) + dzc(izm));
      double tg = (T(ix, iyp, iz) - T(ix, iy, iz)) / dyc(iy);
      tb = fmax0(tb);
      if (rp != 0.0) {
        double bg = b0 * (tg * b0 + tg_a1 * bxf + tg_a2 * bzf);
        return -lf * k0 * std::pow(tb, pow_c) * ((bg + tg * min_b) / modb + rp * (tg - bg / modb));
      }
      return -lf * k0 * std::pow(tb, pow_c) * (b0 * (tg * b0 + tg_a1 * bxf + tg_a2 * bzf) + tg * min_b) / modb;
    } else {
      double bxf = 0.25 * (bx(ix, iy, iz) + bx(ix, iy, izp) + bx(ixm, iy, iz) + bx(ixm, iy, izp));
      double byf = 0.25 * (by(ix, iy, iz) + by(ix, iy, izp) + by(ix, iym, iz) + by(ix, iym, izp));
      double b0 = bz(ix, iy, iz);
      double modb = bxf * bxf + byf * byf + b0 * b0 + min_b;
      double tb = (T(ix, iy, izp) + T(ix, iy, iz)) / 2.0;
      double tb_p = (T(ixp, iy, izp) + T(ixp, iy, iz)) / 2.0;
      double tb_m = (T(ixm, iy, izp) + T(ixm, iy, iz)) / 2.0;
      double tg_a1 = (tb_p - tb_m) / (dxc(ix) + dxc(ixm));
      tb_p = (T(ix, iyp, izp) + T(ix, iyp, iz)) / 2.0;
      tb_m = (T(ix, iym, izp) + T(ix, iym, iz)) / 2.0;
      double tg_a2 = (tb_p - tb_m) / (dyc(iy) + dyc(iym));
      double tg = (T(ix, iy, izp) - T(ix, iy, iz)) / dzc(iz);
      tb = fmax0(tb);
      if (rp != 0.0) {
        double bg = b0 * (tg * b0 + tg_a1 * bxf + tg_a2 * byf);
        return -lf * k0 * std::pow(tb, pow_c) * ((bg + tg * min_b) / modb + rp * (tg - bg / modb));
      }
      return -lf * k0 * std::pow(tb, pow_c) * (b0 * (tg * b0 + tg_a1 * bxf + tg_a2 * byf) + tg * min_b) / modb;
    }
  }

  void heat_flux() {
    F3& flux = c_flux;
    flux.fill(0.0);
    box(1, nx, 1, ny, 1, nz, [&](int ix, int iy, int iz) {
      double f = 0.0;
      f = f + face_flux(2, ix, iy, iz - 1) / dzb(iz - 1);
      f = f + face_flux(1, ix, iy - 1, iz) / dyb(iy - 1);
      f = f + face_flux(0, ix - 1, iy, iz) / dxb(ix - 1);
      f = f - face_flux(0, ix, iy, iz) / dxb(ix);
      f = f - face_flux(1, ix, iy, iz) / dyb(iy);
      f = f - face_flux(2, ix, iy, iz) / dzb(iz);
      flux(ix, iy, iz) = f;
    });
  }

  // conduct.f90:299-416
  void heat_conduct_sts2() {
    const int s = n_s_stages;
    std::vector<double> a(s + 1), b(s + 1), mu_tilde(s + 1), mu(s + 1), nu(s + 1), gamma_tilde(s + 1);
    double ds = (double)s;
    double omega_1 = 4.0 / (ds * ds + ds - 2.0);
    for (int j = 0; j <= std::min(2, s); ++j) b[j] = 1.0 / 3.0;
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
    for (int j = 0; j < 4; ++j) Y[j].d = energy.d;
    temperature_from(Y[0]);
    heat_flux();
    box(1, nx, 1, ny, 1, nz, [&](int ix, int iy, int iz) {
      Lc_Y0(ix, iy, iz) = (1.0 / rho(ix, iy, iz)) * c_flux(ix, iy, iz);
      double c0 = mu_tilde[1] * dt * Lc_Y0(ix, iy, iz);
      Y[1](ix, iy, iz) = Y[0](ix, iy, iz) + c0;
    });
    box(1, nx, 1, ny, 1, nz, [&](int ix, int iy, int iz) {
      Y[2](ix, iy, iz) = Y[1](ix, iy, iz);
      Y[1](ix, iy, iz) = Y[0](ix, iy, iz);
    });
    for (int j = 2; j <= s; ++j) {
      temperature_from(Y[2]);
      temperature_bcs();
      heat_flux();
      const double gt = gamma_tilde[j], mt = mu_tilde[j], mj = mu[j], nj = nu[j];
      box(1, nx, 1, ny, 1, nz, [&](int ix, int iy, int iz) {
        double c0 = gt * dt * Lc_Y0(ix, iy, iz);
        double Lc = (1.0 / rho(ix, iy, iz)) * c_flux(ix, iy, iz);
        double c1 = mt * dt * Lc;
        double y3 = mj * Y[2](ix, iy, iz) + nj * Y[1](ix, iy, iz) + (1.0 - mj - nj) * Y[0](ix, iy, iz);
        Y[3](ix, iy, iz) = y3 + c1 + c0;
      });
      if (j < s) {
        Y[1].d = Y[2].d;
        energy.d = Y[3].d;
        energy_bcs();
        if (eos_number() != LARE_EOS_IDEAL) neutral_fraction(energy);  // conduct.f90:404
        Y[2].d = energy.d;
        box(1, nx, 1, ny, 1, nz, [&](int ix, int iy, int iz) { Y[3](ix, iy, iz) = 0.0; });
      }
    }
    box(1, nx, 1, ny, 1, nz, [&](int ix, int iy, int iz) { energy(ix, iy, iz) = Y[3](ix, iy, iz); });
    energy_bcs();
  }

  // ------------------------------------------------------------------
  // diagnostics.F90:517-609 (do_sum = .FALSE.), serial sums.
  void energy_account(double& en_b, double& en_ke, double& en_int) {
    double eb = 0.0, eke = 0.0, ei = 0.0;
    for (int iz = 1; iz <= nz; ++iz)
      for (int iy = 1; iy <= ny; ++iy)
        for (int ix = 1; ix <= nx; ++ix) {
          int ixm = ix - 1, iym = iy - 1, izm = iz - 1;
          double w1 = (bx(ix, iy, iz) * bx(ix, iy, iz) + bx(ixm, iy, iz) * bx(ixm, iy, iz)) * 0.5;
          double w2 = (by(ix, iy, iz) * by(ix, iy, iz) + by(ix, iym, iz) * by(ix, iym, iz)) * 0.5;
          double w3 = (bz(ix, iy, iz) * bz(ix, iy, iz) + bz(ix, iy, izm) * bz(ix, iy, izm)) * 0.5;
          w1 = (w1 + w2 + w3) * 0.5;
          eb = eb + w1 * cv(ix, iy, iz);
          ei = ei + energy(ix, iy, iz) * rho(ix, iy, iz) * cv(ix, iy, iz);
        }
    for (int iz = 0; iz <= nz; ++iz)
      for (int iy = 0; iy <= ny; ++iy)
        for (int ix = 0; ix <= nx; ++ix) {
          int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
          double rv = rho(ix, iy, iz) * cv(ix, iy, iz) + rho(ixp, iy, iz) * cv(ixp, iy, iz)
                    + rho(ix, iyp, iz) * cv(ix, iyp, iz) + rho(ixp, iyp, iz) * cv(ixp, iyp, iz)
                    + rho(ix, iy, izp) * cv(ix, iy, izp) + rho(ixp, iy, izp) * cv(ixp, iy, izp)
                    + rho(ix, iyp, izp) * cv(ix, iyp, izp) + rho(ixp, iyp, izp) * cv(ixp, iyp, izp);
          double cvv = cv(ix, iy, iz) + cv(ixp, iy, iz) + cv(ix, iyp, iz) + cv(ixp, iyp, iz)
                     + cv(ix, iy, izp) + cv(ixp, iy, izp) + cv(ix, iyp, izp) + cv(ixp, iyp, izp);
          rv = rv / cvv;
          cvv = cvv * 0.125;
          double w1 = rv * cvv * (vx(ix, iy, iz) * vx(ix, iy, iz) + vy(ix, iy, iz) * vy(ix, iy, iz)
                                  + vz(ix, iy, iz) * vz(ix, iy, iz));
          if (ix == 0 || ix == nx) w1 = w1 * 0.5;
          if (iy == 0 || iy == ny) w1 = w1 * 0.5;
          if (iz == 0 || iz == nz) w1 = w1 * 0.5;
          eke = eke + w1 * 0.5;
        }
    en_b = eb; en_ke = eke; en_int = ei;
  }
};

// ----------------------------------------------------------------------
// C ABI
namespace {
int fail(lare_ref* r, int code, const char* msg) {
  if (r) r->err = msg;
  return code;
}
bool bc_ok(int c) { return c == LARE_BC_PERIODIC || c == LARE_BC_USER || c == LARE_BC_OPEN; }

void copy_in(F3& a, const double* h) { std::memcpy(a.d.data(), h, a.d.size() * sizeof(double)); }
void copy_out(F3& a, double* h) { std::memcpy(h, a.d.data(), a.d.size() * sizeof(double)); }
}  // namespace

extern "C" {

int lare_ref_init(const lare_params* params, int nx, int ny, int nz, const double* dxb,
                  const double* dxc, const double* dyb, const double* dyc, const double* dzb,
                  const double* dzc, lare_ref** out) {
  if (!params || !out || !dxb || !dxc || !dyb || !dyc || !dzb || !dzc) return LARE_EINVAL;
  if (nx < 4 || ny < 4 || nz < 4) return LARE_EINVAL;
  const lare_params& p = *params;
  if (!bc_ok(p.xbc_min) || !bc_ok(p.xbc_max) || !bc_ok(p.ybc_min) || !bc_ok(p.ybc_max) ||
      !bc_ok(p.zbc_min) || !bc_ok(p.zbc_max))
    return LARE_EINVAL;
  if (p.eos_number < 0 || p.eos_number > LARE_EOS_PI) return LARE_EINVAL;
  lare_ref* r = new lare_ref();
  r->p = p;
  r->nx = nx; r->ny = ny; r->nz = nz;
  r->n[0] = nx; r->n[1] = ny; r->n[2] = nz;
  r->dxb.alloc(-1, nx + 2); r->dxc.alloc(-1, nx + 1);
  r->dyb.alloc(-1, ny + 2); r->dyc.alloc(-1, ny + 1);
  r->dzb.alloc(-1, nz + 2); r->dzc.alloc(-1, nz + 1);
  r->grav.alloc(-1, nz + 2, 0.0);
  std::memcpy(r->dxb.d.data(), dxb, sizeof(double) * (nx + 4));
  std::memcpy(r->dxc.d.data(), dxc, sizeof(double) * (nx + 3));
  std::memcpy(r->dyb.d.data(), dyb, sizeof(double) * (ny + 4));
  std::memcpy(r->dyc.d.data(), dyc, sizeof(double) * (ny + 3));
  std::memcpy(r->dzb.d.data(), dzb, sizeof(double) * (nz + 4));
  std::memcpy(r->dzc.d.data(), dzc, sizeof(double) * (nz + 3));
  r->allocate();
  // setup.F90:239-245
  box(-1, nx + 2, -1, ny + 2, -1, nz + 2, [&](int ix, int iy, int iz) {
    r->cv(ix, iy, iz) = r->dxb(ix) * r->dyb(iy) * r->dzb(iz);
  });
  *out = r;
  return LARE_OK;
}

int lare_ref_upload(lare_ref* r, const double* rho, const double* energy, const double* vx,
                    const double* vy, const double* vz, const double* bx, const double* by,
                    const double* bz) {
  if (!r) return LARE_EINVAL;
  if (rho) copy_in(r->rho, rho);
  if (energy) copy_in(r->energy, energy);
  if (vx) copy_in(r->vx, vx);
  if (vy) copy_in(r->vy, vy);
  if (vz) copy_in(r->vz, vz);
  if (bx) copy_in(r->bx, bx);
  if (by) copy_in(r->by, by);
  if (bz) copy_in(r->bz, bz);
  return LARE_OK;
}

int lare_ref_upload_aux(lare_ref* r, const double* eta, const double* visc3, const double* grav,
                        const double* gamma_boris) {
  if (!r) return LARE_EINVAL;
  if (eta) copy_in(r->eta, eta);
  if (visc3) copy_in(r->visc3, visc3);
  if (grav) std::memcpy(r->grav.d.data(), grav, sizeof(double) * r->grav.d.size());
  if (gamma_boris) copy_in(r->gamma_boris, gamma_boris);
  return LARE_OK;
}

int lare_ref_set_time(lare_ref* r, double time, double dt) {
  if (!r) return LARE_EINVAL;
  r->time = time; r->dt = dt;
  return LARE_OK;
}

int lare_ref_lagrangian_step(lare_ref* r, int step) {
  if (!r) return LARE_EINVAL;
  r->lagrangian_step(step);
  if (r->eos_error) return fail(r, LARE_EEOS, "Temperature bounds problem");
  if (!(r->dt > 0.0) || !std::isfinite(r->dt)) return fail(r, LARE_EDT, "dt underflow or non-finite");
  return LARE_OK;
}
int lare_ref_neutral_fraction(lare_ref* r) {
  if (!r) return LARE_EINVAL;
  if (r->eos_number() == LARE_EOS_IDEAL) return LARE_OK;
  r->neutral_fraction(r->energy);
  if (r->eos_error) return fail(r, LARE_EEOS, "Temperature bounds problem");
  return LARE_OK;
}
double lare_ref_exp(double x) { return cw_exp(x); }
int lare_ref_energy_correction(lare_ref* r) {
  if (!r) return LARE_EINVAL;
  if (!r->p.rke) return fail(r, LARE_EINVAL, "rke is off");
  r->energy_correction();
  return LARE_OK;
}
int lare_ref_perpendicular_resistivity(lare_ref* r) {
  if (!r) return LARE_EINVAL;
  if (!r->p.cowling_resistivity) return fail(r, LARE_EINVAL, "cowling_resistivity is off");
  r->perpendicular_resistivity();
  return LARE_OK;
}
int lare_ref_eulerian_remap(lare_ref* r, int step) {
  if (!r) return LARE_EINVAL;
  r->eulerian_remap(step);
  return LARE_OK;
}
int lare_ref_eta_calc(lare_ref* r) {
  if (!r) return LARE_EINVAL;
  r->eta_calc();
  return LARE_OK;
}
int lare_ref_boundary_conditions(lare_ref* r) {
  if (!r) return LARE_EINVAL;
  r->boundary_conditions();
  return LARE_OK;
}
int lare_ref_step(lare_ref* r, int step, double* time, double* dt) {
  int rc = lare_ref_neutral_fraction(r);  // lare3d.f90:83
  if (rc) return rc;
  rc = lare_ref_lagrangian_step(r, step);
  if (rc) return rc;
  r->eulerian_remap(step);
  if (r->p.rke) r->energy_correction();  // lare3d.f90:86
  r->eta_calc();
  if (time) *time = r->time;
  if (dt) *dt = r->dt;
  return LARE_OK;
}
int lare_ref_conduct_heat(lare_ref* r, double dt, int* n_stages) {
  if (!r) return LARE_EINVAL;
  double keep = r->dt;
  r->dt = dt;
  r->conduct_heat();
  r->dt = keep;
  if (n_stages) *n_stages = r->n_s_stages;
  return LARE_OK;
}
int lare_ref_energy(lare_ref* r, double out[5]) {
  if (!r || !out) return LARE_EINVAL;
  r->energy_account(out[0], out[1], out[2]);
  out[3] = r->total_visc_heating;
  out[4] = r->total_ohmic_heating;
  return LARE_OK;
}
int lare_ref_download(lare_ref* r, double* rho, double* energy, double* vx, double* vy,
                      double* vz, double* bx, double* by, double* bz) {
  if (!r) return LARE_EINVAL;
  if (rho) copy_out(r->rho, rho);
  if (energy) copy_out(r->energy, energy);
  if (vx) copy_out(r->vx, vx);
  if (vy) copy_out(r->vy, vy);
  if (vz) copy_out(r->vz, vz);
  if (bx) copy_out(r->bx, bx);
  if (by) copy_out(r->by, by);
  if (bz) copy_out(r->bz, bz);
  return LARE_OK;
}
int lare_ref_get_field(lare_ref* r, const char* name, double* host) {
  if (!r || !name || !host) return LARE_EINVAL;
  auto it = r->fields.find(name);
  if (it == r->fields.end()) return fail(r, LARE_ENOTFOUND, "unknown field");
  copy_out(*it->second, host);
  return LARE_OK;
}
int lare_ref_set_field(lare_ref* r, const char* name, const double* host) {
  if (!r || !name || !host) return LARE_EINVAL;
  auto it = r->fields.find(name);
  if (it == r->fields.end()) return fail(r, LARE_ENOTFOUND, "unknown field");
  copy_in(*it->second, host);
  return LARE_OK;
}
int lare_ref_field_bounds(lare_ref* r, const char* name, int lo[3], int hi[3]) {
  if (!r || !name) return LARE_EINVAL;
  auto it = r->fields.find(name);
  if (it == r->fields.end()) return fail(r, LARE_ENOTFOUND, "unknown field");
  for (int d = 0; d < 3; ++d) { lo[d] = it->second->lo[d]; hi[d] = it->second->hi[d]; }
  return LARE_OK;
}
int lare_ref_get_scalars(lare_ref* r, lare_scalars* o) {
  if (!r || !o) return LARE_EINVAL;
  o->time = r->time; o->dt = r->dt; o->dtr = r->dtr;
  o->total_visc_heating = r->total_visc_heating;
  o->total_ohmic_heating = r->total_ohmic_heating;
  o->n_s_stages = r->n_s_stages;
  o->peak_substeps = r->peak_substeps;
  o->last_substeps = r->last_substeps;
  o->steps_taken = r->steps_taken;
  return LARE_OK;
}
int lare_ref_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
const char* lare_ref_last_error(lare_ref* r) { return r ? r->err.c_str() : "null context"; }
void lare_ref_destroy(lare_ref* r) { delete r; }

}  // extern "C"
