// neutral.cuh - partially ionised plasma: neutral.f90.
//
//   neutral_fraction           neutral.f90:158-195  xi_n over the whole cell
//                              array by bisection on the temperature
//   perpendicular_resistivity  neutral.f90:68-124   Cowling resistivity
//                              eta_perp at the vertices 0:n
//   get_neutral                neutral.f90:128-153  the ionisation balance
//
// Both models run in FP64 whatever the engine's precision: they are
// cell-local and compute-bound (a bisection of up to 100 steps, each with an
// exponential, two square roots and three divisions), and the FP32 engine
// rounds the results to FP32 on the store.
//
// The exponential is this file's own (cw_exp below) rather than the CUDA
// library's, so that the device and a host restatement that uses the same
// operations agree bit for bit; the bisection's branches then follow
// identical paths on both.
#pragma once

LARE_BEGIN

// exp(x) by Cody and Waite's argument reduction (W. J. Cody and W. Waite,
// Software Manual for the Elementary Functions, 1980): x = k ln2 + r with
// ln 2 split into a 33-bit head (so k * head is exact for |k| < 2^20) and
// its tail, |r| <= ln2 / 2; exp(r) from its Taylor series through r^13
// (truncation below 2^-60 relative on that interval) by Horner's rule with
// coefficients 1/n! rounded to nearest; and the result scaled by 2^k.
// Measured within 1.03 ulp of the exact exponential.
__host__ __device__ inline double cw_exp(double x) {
  if (!(x == x)) return x;
  if (x > 709.782712893384) return HUGE_VAL;
  if (x < -745.1332191019412) return 0.0;
  const double ln2_hi = 0x1.62e42fee00000p-1, ln2_lo = 0x1.a39ef35793c76p-33;
  const double k = rint(x * 0x1.71547652b82fep+0);
  const double r = (x - k * ln2_hi) - k * ln2_lo;
  double p = 0x1.6124613a86d09p-33;  // 1/13!
  p = p * r + 0x1.1eed8eff8d898p-29;
  p = p * r + 0x1.ae64567f544e4p-26;
  p = p * r + 0x1.27e4fb7789f5cp-22;
  p = p * r + 0x1.71de3a556c734p-19;
  p = p * r + 0x1.a01a01a01a01ap-16;
  p = p * r + 0x1.a01a01a01a01ap-13;
  p = p * r + 0x1.6c16c16c16c17p-10;
  p = p * r + 0x1.1111111111111p-7;
  p = p * r + 0x1.5555555555555p-5;
  p = p * r + 0x1.5555555555555p-3;
  p = p * r + 0.5;
  p = p * r + 1.0;
  p = p * r + 1.0;
  return ldexp(p, (int)k);
}

// Normalised constants of the ionisation model (neutral.f90:46-62 after
// normalise.f90:39-51).
struct NeutralPar {
  double gamma, ionise_pot, f_bar, t_bar, r_bar, tr, eta_bar;
};

// neutral.f90:140-153 get_neutral(t_v, rho_v): the Saha-like balance with a
// diluted photospheric radiation field (t_rad = tr, dilution 0.5).
__device__ __forceinline__ double get_neutral(double t_v, double rho_v, const NeutralPar& q) {
  const double t_rad = q.tr, dilution = 0.5;
  const double bof = 1.0 / (dilution * q.f_bar * t_rad * sqrt(t_v)) *
                     cw_exp((0.25 * (t_v / t_rad - 1.0) + 1.0) * q.t_bar / t_v);
  const double r = 0.5 * (-1.0 + sqrt(1.0 + q.r_bar * rho_v * bof));
  return r / (1.0 + r);
}

template <class R>
NeutralPar neutral_par(const Run<R>& run) {
  const Par& p = run.p;
  return NeutralPar{p.gamma, p.ionise_pot, p.f_bar, p.t_bar, p.r_bar, p.tr, p.eta_bar};
}

// neutral.f90:158-195 neutral_fraction on the energy-like array e (the
// energy itself, or an RKL2 stage that conduct.f90:402-404 has just copied
// into it).  A cell whose bracket [(gamma-1) max((e-chi)/2, tiny),
// (gamma-1) e] is empty raises LARE_EEOS, where the reference prints
// 'Temperature bounds problem' and stops.
template <class R>
void neutral_fraction(Run<R>& run, A3<R> e) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  auto rho = run.a.rho, xi = run.a.xi;
  const NeutralPar q = neutral_par(run);
  double* sc = run.sc;
  LARE_BOXW(run, 3, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
    const double rho0 = (double)rho(ix, iy, iz);
    const double e0 = (double)e(ix, iy, iz);
    const double g1 = q.gamma - 1.0, ip = q.ionise_pot;
    const double ta1 = g1 * fmax((e0 - ip) / 2.0, DBL_MIN), ta2 = g1 * e0;
    if (ta1 > ta2) {
      sc[SC_ERROR] = (double)LARE_EEOS;
      return;
    }
    double dx = ta2 - ta1, t = ta1, x = ta1, xi_a = 0.0;
    for (int loop = 1; loop <= 100; ++loop) {
      dx = dx / 2.0;
      x = t + dx;
      xi_a = get_neutral(x, rho0, q);
      const double fa = x - g1 * (e0 - (1.0 - xi_a) * ip) / (2.0 - xi_a);
      if (fa <= 0.0) t = x;
      if (fabs(dx) < 1.e-8 || fabs(fa) < 1.e-8) break;
    }
    // neutral.f90:191 recomputes get_neutral(x, rho0): the same value
    xi(ix, iy, iz) = (R)xi_a;
  });
}

// neutral.f90:68-124 perpendicular_resistivity.  The vertex field averages
// are the reference's as written: bxv and byv take their z-neighbour terms
// from bz (:95-96), unlike rkstep's averages (lagran.F90:1527-1532).
template <class R>
void perpendicular_resistivity(Run<R>& run) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  auto rho = run.a.rho, cv = run.a.cv, energy = run.a.energy, xi = run.a.xi, eta_perp = run.a.eta_perp;
  auto bx = run.a.bx, by = run.a.by, bz = run.a.bz;
  const NeutralPar q = neutral_par(run);
  LARE_BOXW(run, 9, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz) {
    const int ixp = ix + 1, iyp = iy + 1, izp = iz + 1;
    R rho_v = rho(ix, iy, iz) * cv(ix, iy, iz) + rho(ixp, iy, iz) * cv(ixp, iy, iz) +
              rho(ix, iyp, iz) * cv(ix, iyp, iz) + rho(ixp, iyp, iz) * cv(ixp, iyp, iz) +
              rho(ix, iy, izp) * cv(ix, iy, izp) + rho(ixp, iy, izp) * cv(ixp, iy, izp) +
              rho(ix, iyp, izp) * cv(ix, iyp, izp) + rho(ixp, iyp, izp) * cv(ixp, iyp, izp);
    rho_v = rho_v / (cv(ix, iy, iz) + cv(ixp, iy, iz) + cv(ix, iyp, iz) + cv(ixp, iyp, iz) + cv(ix, iy, izp) +
                     cv(ixp, iy, izp) + cv(ix, iyp, izp) + cv(ixp, iyp, izp));
    R bxv = bx(ix, iy, iz) + bx(ix, iyp, iz) + bz(ix, iy, izp) + bz(ix, iyp, izp);
    R byv = by(ix, iy, iz) + by(ixp, iy, iz) + bz(ix, iy, izp) + bz(ixp, iy, izp);
    R bzv = bz(ix, iy, iz) + bz(ixp, iy, iz) + bz(ix, iyp, iz) + bz(ixp, iyp, iz);
    bxv = R(0.25) * bxv;
    byv = R(0.25) * byv;
    bzv = R(0.25) * bzv;
    const R bfieldsq = bxv * bxv + byv * byv + bzv * bzv;
    const R ip = (R)q.ionise_pot, g = (R)q.gamma;
    R t_v = R(0);
    for (int iz2 = iz; iz2 <= iz + 1; ++iz2)
      for (int iy2 = iy; iy2 <= iy + 1; ++iy2)
        for (int ix2 = ix; ix2 <= ix + 1; ++ix2) {
          const R x = xi(ix2, iy2, iz2);
          t_v = t_v + (energy(ix2, iy2, iz2) - (R(1) - x) * ip) / (R(2) - x);
        }
    t_v = t_v * (g - R(1)) / R(8);
    const R xi_v = (R)get_neutral((double)t_v, (double)rho_v, q);
    const R f = fmax(R(1) - xi_v, Num<R>::tiny());
    R ep = R(0);
    if (f > R(0)) ep = (R)q.eta_bar * xi_v / f * bfieldsq / (rho_v * rho_v) / sqrt(t_v);
    eta_perp(ix, iy, iz) = fmin(ep, R(100));  // eta_perp = MIN(eta_perp, 100) (:122)
  });
}

LARE_END  // namespace lare
