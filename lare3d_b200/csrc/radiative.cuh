// radiative.cuh - optically thin radiative losses, radiative.f90:98-208.
//
// The loss function is the reference's default piecewise power law
// Q(T) = psi_k T^pow_k on kmax = 6 temperature bands (setup_loss_function,
// :38-62), integrated exactly over a step by Townsend's method
// (exact_intergation_method :115-176, set_exact_integration_arrays
// :180-208): the temporal evolution function Y(T) is piecewise analytic,
// so a cell's temperature after dt is Y^-1(Y(T) + dt / t_cool).  The band
// tables are formed once on the host; the per-cell update is one point
// kernel in FP64 (its powers come from CUDA's pow, whose last bit may differ
// from the C library's, so this part is compared with a tolerance).
#pragma once

#include <cmath>

LARE_BEGIN

constexpr int kRadN = 7;  // temperature boundaries (radiative.f90:25)
constexpr int kRadK = kRadN - 1;

struct RadTable {
  double t_boundary[kRadN], pow_[kRadK], yk[kRadN], ratios[kRadN];
  int alpha[kRadK];
  double cool, gamma, temp_norm, time_norm;
};

// radiative.f90:38-62 and :180-208, evaluated in the reference's order.
inline RadTable rad_table(double gamma, double rho_norm, double mf, double temp_norm, double time_norm) {
  RadTable t;
  const double kb_si = 1.3806488e-23, mh_si = 1.672621777e-27;  // shared_data.F90:45-48
  const double tb[kRadN] = {0.02, 0.0398, 0.0794, 0.251, 0.562, 1.995, 10.0};
  for (int i = 0; i < kRadN; ++i) t.t_boundary[i] = tb[i] * 1e6;
  const double frac = -2.0 / 3.0;
  const int alpha[kRadK] = {0, 2, 0, -2, 0, 0};
  const double extra[kRadK] = {0.0, 0.0, 0.0, 0.0, 0.0, frac};
  const double lpsi[kRadK] = {-21.85, -31.0, -21.2, -10.4, -21.94, -17.73};
  double psi[kRadK], qk[kRadN];
  for (int k = 0; k < kRadK; ++k) {
    t.alpha[k] = alpha[k];
    t.pow_[k] = (double)alpha[k] + extra[k];
    psi[k] = 1.e-13 * std::pow(10.0, lpsi[k]);  // RTV fit in cgs, then SI
  }
  for (int k = 0; k < kRadK; ++k) qk[k] = psi[k] * std::pow(t.t_boundary[k], t.pow_[k]);
  qk[kRadN - 1] = qk[kRadN - 2] * std::pow(t.t_boundary[kRadN - 1] / t.t_boundary[kRadN - 2], t.pow_[kRadK - 1]);
  const double ratio = qk[kRadN - 1] / t.t_boundary[kRadN - 1];
  t.cool = 0.5 * ratio * (gamma - 1.0) * rho_norm / (kb_si * mf * mh_si);
  for (int k = 0; k < kRadN; ++k) t.ratios[k] = ratio * (t.t_boundary[k] / qk[k]);
  t.yk[kRadN - 1] = 0.0;
  for (int k = kRadK - 1; k >= 0; --k) {
    if (t.alpha[k] != 1) {
      const double fac = 1.0 / (1.0 - t.pow_[k]);
      t.yk[k] = t.yk[k + 1] -
                fac * t.ratios[k] * (1.0 - std::pow(t.t_boundary[k] / t.t_boundary[k + 1], t.pow_[k] - 1.0));
    } else {
      t.yk[k] = t.yk[k + 1] - t.ratios[k] * std::log(t.t_boundary[k] / t.t_boundary[k + 1]);
    }
  }
  t.gamma = gamma;
  t.temp_norm = temp_norm;
  t.time_norm = time_norm;
  return t;
}

// radiative.f90:115-176 for one cell: the new energy, or e itself where the
// temperature lies outside the table (the reference's CYCLE).
__device__ __forceinline__ double rad_cell(double e, double rho, double dt, const RadTable& t) {
  double temp_si = 0.5 * t.temp_norm * e * (t.gamma - 1.0);
  int k = -1;
  for (int i = 0; i < kRadK; ++i) {
    if (temp_si > t.t_boundary[i] && temp_si <= t.t_boundary[i + 1]) {
      k = i;
      break;
    }
  }
  if (k < 0) return e;
  double yt;
  if (t.alpha[k] != 1) {
    const double fac = 1.0 / (1.0 - t.pow_[k]);
    yt = t.yk[k] + fac * t.ratios[k] * (1.0 - pow(t.t_boundary[k] / temp_si, t.pow_[k] - 1.0));
  } else {
    yt = t.yk[k] + t.ratios[k] * log(t.t_boundary[k] / temp_si);
  }
  const double inverse_t_cool = t.cool * rho;
  yt = yt + dt * inverse_t_cool * t.time_norm;
  k = -1;
  for (int i = 0; i < kRadK; ++i) {
    if ((yt > t.yk[i] && yt <= t.yk[i + 1]) || (yt < t.yk[i] && yt >= t.yk[i + 1])) {
      k = i;
      break;
    }
  }
  if (k < 0) return t.t_boundary[0] * 2.0 / (t.gamma - 1.0) / t.temp_norm;  // cooled below the table
  if (t.alpha[k] != 1) {
    const double fac = 1.0 / (1.0 - t.pow_[k]);
    temp_si = t.t_boundary[k] * pow(1.0 - (1.0 - t.pow_[k]) / t.ratios[k] * (yt - t.yk[k]), fac);
  } else {
    temp_si = t.t_boundary[k] * exp((yt - t.yk[k]) / t.ratios[k]);
  }
  return temp_si * 2.0 / (t.gamma - 1.0) / t.temp_norm;
}

// rad_losses (radiative.f90:98-111) on the energy e0 the reference holds at
// lagran.F90:174 (the energy before conduction), into er: er = e0, the
// interior updated, then energy_bcs on er.  dt from sc[dt_slot].
template <class R>
void rad_losses(Run<R>& run, A3<R> er, A3<R> e0, int dt_slot) {
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  copy_whole(run, er, e0);
  const RadTable t = rad_table(run.p.gamma, run.p.rho_norm, run.p.mf, run.p.temp_norm, run.p.time_norm);
  auto rho = run.a.rho;
  const double* sc = run.sc;
  LARE_BOXW(run, 3, 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz) {
    er(ix, iy, iz) = (R)rad_cell((double)er(ix, iy, iz), (double)rho(ix, iy, iz), sc[dt_slot], t);
  });
  GhostBatch<R> b;
  b.add(run.g_cell, er.p);
  ghost_flush(run, b);
}

LARE_END  // namespace lare
