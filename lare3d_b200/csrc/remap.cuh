// remap.cuh - one directional Van Leer remap sweep, fused.
//
// xremap.f90:37-336 remap_x and its mirrors yremap.f90:37-337 and
// zremap.f90:37-336, for a sweep along axis A (0 = x, 1 = y, 2 = z).  The
// reference runs about 25 loop nests per sweep; here they are grouped into
// eight kernels.  Every element is still computed by exactly the reference's
// expression over exactly the same inputs, so the results are unchanged bit
// for bit; what changes is where intermediates live:
//
//   K1 geometry   cv1, cv2, dxb1 and dxc1 (xremap.f90:57-115); dxb1 at p+e_A
//                 is recomputed in the thread for dxc1.
//   K2 B fluxes   both constrained-transport edge fluxes (:340-470); the
//                 second does not read what the first one's updates change.
//   K3 B update   the four flux-difference updates (:121-157), with each
//                 file's own loop ranges as predicates.
//   K4 mass flux  dm (:474-533) over the whole cell box, with dm_x_bcs
//                 (:899-917) folded in: a ghost element is the flux computed
//                 at its source index (the same value the copy would bring).
//   K5 rho, eflux new rho (:174-182) into a second buffer (old rho stays
//                 readable as rho1) and the energy flux (:539-601).
//   K6 energy     energy update (:187-196).
//   K7 vertex     vertex rho_v, cv1, cv2, dm averages and rho_v1 (:201-290).
//   K8 momentum   the three momentum fluxes (:605-895), each times dm.
//   K9 velocity   the three velocity updates (:292-329).
// The face-averaged vx1 written back at :265 is only read again as
// REAL(xpass)*(...) with xpass = 0, so it is formed in K8 and not stored.
// Predictor sweeps (predictor_step = .TRUE.) stop after K3.
//
// Indexing is linear: c = ix + sx*iy + sxy*iz, neighbours by constant
// offsets, with the axis a compile-time parameter.
#pragma once

#include <utility>

namespace lare {

template <int A>
__device__ __forceinline__ int acoord(int ix, int iy, int iz) {
  return A == 0 ? ix : (A == 1 ? iy : iz);
}

template <int A, class R>
void remap_sweep(Run<R>& run, bool predictor, int dt_slot, int pass[3]) {
  constexpr int T1 = A == 0 ? 1 : 0, T2 = A == 2 ? 1 : 2;  // transverse axes, T1 < T2
  constexpr int B1 = A == 0 ? 1 : 0, B2 = A == 2 ? 1 : 2;  // transported components, in file order
  constexpr int O1 = 3 - A - B1, O2 = 3 - A - B2;          // the remaining axis for each
  const int nx = run.n[0], ny = run.n[1], nz = run.n[2];
  const int nn[3] = {nx, ny, nz};
  const int na = nn[A];
  const int sx = run.sx, sxy = run.sxy;
  const int SA = A == 0 ? 1 : (A == 1 ? sx : sxy);
  const int S1 = T1 == 0 ? 1 : (T1 == 1 ? sx : sxy);
  const int S2 = T2 == 0 ? 1 : (T2 == 1 ? sx : sxy);
  const int SB1 = B1 == 0 ? 1 : (B1 == 1 ? sx : sxy);
  const int SB2 = B2 == 0 ? 1 : (B2 == 1 ? sx : sxy);
  const int SO1 = O1 == 0 ? 1 : (O1 == 1 ? sx : sxy);
  const int SO2 = O2 == 0 ? 1 : (O2 == 1 ? sx : sxy);
  Arrays<R>& Ar = run.a;
  R* const vx1 = Ar.vx1.p;
  R* const vy1 = Ar.vy1.p;
  R* const vz1 = Ar.vz1.p;
  R* const V1[3] = {vx1, vy1, vz1};
  R* const va = V1[A];
  R* const cv = Ar.cv.p;
  R* const cv1 = Ar.cv1.p;
  R* const cv2 = Ar.cv2.p;
  R* const db1 = Ar.db1.p;
  R* const dc1 = Ar.dc1.p;
  const A1<R> dbm[3] = {Ar.dxb, Ar.dyb, Ar.dzb};
  const A1<R> dcm[3] = {Ar.dxc, Ar.dyc, Ar.dzc};
  const A1<R> dba = dbm[A], dbt1 = dbm[T1], dbt2 = dbm[T2], dct1 = dcm[T1], dct2 = dcm[T2];
  const R pass_t1 = (R)pass[T1], pass_t2 = (R)pass[T2];
  const double* sc = run.sc;
  const bool write_cv2 = !predictor;

  // ---- K1: cv1, cv2, db1, dc1 over the whole cell box -1..n+2
  LARE_BOXW(run, 8, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
    const R dt = (R)sc[dt_slot];
    const int c = ix + sx * iy + sxy * iz;
    // v at the two faces normal to each axis (xremap.f90:64-86)
    auto vxf = [&](int q) { return (vx1[q] + vx1[q - sx] + vx1[q - sxy] + vx1[q - sx - sxy]) * R(0.25); };
    auto vyf = [&](int q) { return (vy1[q] + vy1[q - 1] + vy1[q - sxy] + vy1[q - 1 - sxy]) * R(0.25); };
    auto vzf = [&](int q) { return (vz1[q] + vz1[q - 1] + vz1[q - sx] + vz1[q - 1 - sx]) * R(0.25); };
    R vxb = vxf(c), vxbm = vxf(c - 1);
    R vyb = vyf(c), vybm = vyf(c - sx);
    R vzb = vzf(c), vzbm = vzf(c - sxy);
    R dvv[3] = {vxb - vxbm, vyb - vybm, vzb - vzbm};
    const int pp[3] = {ix, iy, iz};
    R term_t1 = pass_t1 * dvv[T1] / dbt1(pp[T1]);
    R term_t2 = pass_t2 * dvv[T2] / dbt2(pp[T2]);
    R term_a = dvv[A] / dba(pp[A]);
    R dv = (term_t1 + term_t2 + term_a) * dt;
    cv1[c] = cv[c] * (R(1) + dv);
    if (write_cv2) {
      dv = (term_t1 + term_t2) * dt;
      cv2[c] = cv[c] * (R(1) + dv);
    }
    R d0 = dba(pp[A]) + dvv[A] * dt;
    db1[c] = d0;
    // dxc1 = (dxb1(p) + dxb1(min(p+1, n+2))) / 2 (xremap.f90:107-115)
    R d1 = d0;
    if (pp[A] < na + 2) {
      const int q = c + SA;
      R f = A == 0 ? vxf(q) : (A == 1 ? vyf(q) : vzf(q));
      R fa = A == 0 ? vxb : (A == 1 ? vyb : vzb);
      d1 = dba(pp[A] + 1) + (f - fa) * dt;
    }
    dc1[c] = R(0.5) * (d0 + d1);
  });

  // ---- K2: both constrained-transport fluxes over -1..n+1
  R* const Bp[3] = {Ar.bx.p, Ar.by.p, Ar.bz.p};
  R* const f1 = Ar.f1.p;
  R* const f2 = Ar.f2.p;
  {
    R* const Bb1 = Bp[B1];
    R* const Bb2 = Bp[B2];
    LARE_BOXW(run, 7, -1, nx + 1, -1, ny + 1, -1, nz + 1, [=] __device__(int ix, int iy, int iz) {
      const R dt = (R)sc[dt_slot];
      const int c = ix + sx * iy + sxy * iz;
      const int ia = acoord<A>(ix, iy, iz);
      const int cm = ia > -1 ? c - SA : c;             // MAX(ix - 1, -1)
      const int cp = c + SA;
      const int cp2 = ia + 2 <= na + 2 ? c + 2 * SA : cp;  // MIN(ix + 2, n + 2)
      auto one = [&](const R* Bb, int SB, int SO) {
        R v_advect = (va[c] + va[c - SO]) * R(0.5);
        auto dbv = [&](int q) { return (db1[q] + db1[q + SB]) * R(0.5); };
        R dbx = dbv(c), dbxp = dbv(cp), dbxp2 = dbv(cp2), dbxm = dbv(cm);
        R fm = Bb[cm] / dbxm;
        R fi = Bb[c] / dbx;
        R fp = Bb[cp] / dbxp;
        R fp2 = Bb[cp2] / dbxp2;
        LimOut<R> L = limiter<R>(v_advect, fm, fi, fp, fp2, dc1[c], dc1[cm], dc1[cp], db1[c], db1[cp], dbx, dbxp,
                                 dt, true);
        return (L.fu + L.Di * (R(1) - L.phi)) * v_advect * dt;
      };
      f1[c] = one(Bb1, SB1, SO1);
      f2[c] = one(Bb2, SB2, SO2);
    });
  }

  // ---- K3: the four updates, each over its file's range
  {
    R* const Ba = Bp[A];
    R* const Bb1 = Bp[B1];
    R* const Bb2 = Bp[B2];
    LARE_BOXW(run, 8, 0, nx + 1, 0, ny + 1, 0, nz + 1, [=] __device__(int ix, int iy, int iz) {
      const int c = ix + sx * iy + sxy * iz;
      // first flux: b1 over 0:n+1 all, a-component over 0:n+1 all
      Bb1[c] = Bb1[c] - f1[c] + f1[c - SA];
      R ba = Ba[c] + f1[c] - f1[c - SB1];
      // second flux ranges (xremap.f90:141-157; yremap.f90:142-158)
      bool r2a = true, r2b = true;
      if (A == 0) {
        r2a = ix >= 1 && ix <= nx && iy >= 1 && iy <= ny && iz <= nz;
        r2b = ix <= nx;
      } else if (A == 1) {
        r2b = ix >= 1 && ix <= nx && iy <= ny && iz >= 1 && iz <= nz;
      }
      if (r2a) Bb2[c] = Bb2[c] - f2[c] + f2[c - SA];
      if (r2b) ba = ba + f2[c] - f2[c - SB2];
      Ba[c] = ba;
    });
  }
  if (predictor) return;  // xremap.f90:159-162 (pass flag not reset)

  R* const rho = Ar.rho.p;        // rho1 of the reference from here on
  R* const rho_new = Ar.rho_alt.p;
  R* const energy = Ar.energy.p;
  R* const dm = Ar.dm.p;
  R* const eflux = Ar.flux.p;
  const bool per = run.p.per[A];
  const int nt1 = nn[T1], nt2 = nn[T2];

  // ---- K4: mass flux with dm_[xyz]_bcs over the whole cell box
  LARE_BOXW(run, 5, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
    const int c = ix + sx * iy + sxy * iz;
    const int pp[3] = {ix, iy, iz};
    const int ia = pp[A], i1 = pp[T1], i2 = pp[T2];
    R out = R(0);
    bool inside_t = i1 >= 0 && i1 <= nt1 + 1 && i2 >= 0 && i2 <= nt2 + 1;
    int sa = ia;  // source index along A
    bool compute = inside_t;
    if (per) {
      if (ia == na + 1) sa = 1;
      else if (ia == na + 2) sa = 2;
      else if (ia == -1) sa = na - 1;
      else if (ia == 0) sa = na;
    } else {
      if (ia == na + 1) sa = na;
      else if (ia == -1) sa = 0;
      else if (ia == na + 2) compute = false;
    }
    if (compute) {
      const R dt = (R)sc[dt_slot];
      const int q = c + (sa - ia) * SA;
      const int qm = q - SA, qp = q + SA, qp2 = q + 2 * SA;
      R area = dbt1(i1) * dbt2(i2);
      R v_advect = (va[q] + va[q - S1] + va[q - S2] + va[q - S1 - S2]) * R(0.25);
      LimOut<R> L = limiter<R>(v_advect, rho[qm], rho[q], rho[qp], rho[qp2], dc1[q], dc1[qm], dc1[qp], db1[q],
                               db1[qp], R(0), R(0), dt, false);
      out = (L.fu + L.Di * (R(1) - L.phi)) * v_advect * dt * area;
    }
    dm[c] = out;
  });

  // ---- K5: new rho (second buffer) and the energy flux (0:n)
  LARE_BOXW(run, 10, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
    const int c = ix + sx * iy + sxy * iz;
    const bool in0 = ix >= 0 && ix <= nx && iy >= 0 && iy <= ny && iz >= 0 && iz <= nz;
    const bool in1 = ix >= 1 && iy >= 1 && iz >= 1 && in0;
    if (in1) rho_new[c] = (rho[c] * cv1[c] + dm[c - SA] - dm[c]) / cv2[c];
    else rho_new[c] = rho[c];
    if (in0) {
      const R dt = (R)sc[dt_slot];
      const int pp[3] = {ix, iy, iz};
      const int cm = c - SA, cp = c + SA, cp2 = c + 2 * SA;
      R area = dbt1(pp[T1]) * dbt2(pp[T2]);
      R v_advect = (va[c] + va[c - S1] + va[c - S2] + va[c - S1 - S2]) * R(0.25);
      LimOut<R> L = limiter<R>(v_advect, energy[cm], energy[c], energy[cp], energy[cp2], dc1[c], dc1[cm], dc1[cp],
                               db1[c], db1[cp], R(0), R(0), dt, false);
      R rhou = rho[c] * L.vad_p + rho[cp] * L.vad_m;
      R dmu = fabs(dm[c]) / area / L.dxbu / rhou;
      eflux[c] = (L.fu + L.Di * (R(1) - dmu)) * dm[c];
    }
  });

  // ---- K6: energy update (1:n)
  LARE_BOXW(run, 7, 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz) {
    const int c = ix + sx * iy + sxy * iz;
    energy[c] = (energy[c] * cv1[c] * rho[c] + eflux[c - SA] - eflux[c]) / (cv2[c] * rho_new[c]);
  });

  // ---- K7: vertex quantities.  rho_v over a -1:n+1, the rest over 0:n;
  // dm vertex averages over a -1:n.
  R* const rv = Ar.r_rho_v.p;
  R* const rv1 = Ar.r_rho_v1.p;
  R* const cv1v = Ar.cv1v.p;
  R* const cv2v = Ar.cv2v.p;
  R* const dmv = Ar.dmv.p;
  {
    int lo[3] = {0, 0, 0}, hi[3] = {nx, ny, nz};
    lo[A] = -1;
    hi[A] = na + 1;
    LARE_BOXW(run, 9, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], [=] __device__(int ix, int iy, int iz) {
      const int c = ix + sx * iy + sxy * iz;
      const int ia = acoord<A>(ix, iy, iz);
      // the eight cells around vertex c, in the reference's summation order
      const int o[8] = {0, 1, sx, 1 + sx, sxy, 1 + sxy, sx + sxy, 1 + sx + sxy};
      R s = rho[c + o[0]] * cv1[c + o[0]];
      R w = cv1[c + o[0]];
      for (int q = 1; q < 8; ++q) {
        s = s + rho[c + o[q]] * cv1[c + o[q]];
        w = w + cv1[c + o[q]];
      }
      R rvc = s / w;
      rv[c] = rvc;
      auto avg_dm = [&](int b) {
        R t = dm[b + o[0]];
        for (int q = 1; q < 8; ++q) t = t + dm[b + o[q]];
        return t;
      };
      if (ia <= na) dmv[c] = avg_dm(c) * R(0.125);
      if (ia >= 0 && ia <= na) {
        R w2 = cv2[c + o[0]];
        for (int q = 1; q < 8; ++q) w2 = w2 + cv2[c + o[q]];
        R c1 = w * R(0.125), c2 = w2 * R(0.125);
        cv1v[c] = c1;
        cv2v[c] = c2;
        R dmm = avg_dm(c - SA) * R(0.125);
        R dmp = avg_dm(c) * R(0.125);
        rv1[c] = (rvc * c1 + dmm - dmp) / c2;
      }
    });
  }

  // ---- K8: momentum fluxes at vertex faces a -1:n, transverse 0:n
  R* const Vp[3] = {Ar.vx.p, Ar.vy.p, Ar.vz.p};
  R* const vxp = Vp[0];
  R* const vyp = Vp[1];
  R* const vzp = Vp[2];
  R* const mfx = Ar.mfx.p;
  R* const mfy = Ar.mfy.p;
  R* const mfz = Ar.mfz.p;
  {
    int lo[3] = {0, 0, 0}, hi[3] = {nx, ny, nz};
    lo[A] = -1;
    hi[A] = na;
    LARE_BOXW(run, 11, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], [=] __device__(int ix, int iy, int iz) {
      const R dt = (R)sc[dt_slot];
      const int c = ix + sx * iy + sxy * iz;
      const int pp[3] = {ix, iy, iz};
      const int cm = c - SA, cp = c + SA, cp2 = c + 2 * SA;
      R area = dct1(pp[T1]) * dct2(pp[T2]);
      R v_advect = (va[c] + va[cp]) * R(0.5);  // the face-averaged v1 of xremap.f90:257-265
      R rvc = rv[c], rvp = rv[cp], dmc = dmv[c];
      const R* Vc[3] = {vxp, vyp, vzp};
      R* Fo[3] = {mfx, mfy, mfz};
      for (int comp = 0; comp < 3; ++comp) {
        const R* vc = Vc[comp];
        LimOut<R> L = limiter<R>(v_advect, vc[cm], vc[c], vc[cp], vc[cp2], db1[cp], db1[c], db1[cp2], dc1[c],
                                 dc1[cp], R(0), R(0), dt, false);
        R rhou = rvc * L.vad_p + rvp * L.vad_m;
        R dmu = fabs(dmc) / area / L.dxbu / rhou;
        R f = L.fu + L.Di * (R(1) - dmu);
        Fo[comp][c] = f * dmc;
      }
    });
  }

  // ---- K9: velocity updates (0:n)
  LARE_BOXW(run, 13, 0, nx, 0, ny, 0, nz, [=] __device__(int ix, int iy, int iz) {
    const int c = ix + sx * iy + sxy * iz;
    R rvc = rv[c], c1 = cv1v[c], den = cv2v[c] * rv1[c];
    vxp[c] = (rvc * vxp[c] * c1 + mfx[c - SA] - mfx[c]) / den;
    vyp[c] = (rvc * vyp[c] * c1 + mfy[c - SA] - mfy[c]) / den;
    vzp[c] = (rvc * vzp[c] * c1 + mfz[c - SA] - mfz[c]) / den;
  });

  // The new density becomes rho; the old buffer is scratch again.
  std::swap(Ar.rho.p, Ar.rho_alt.p);
  boundary_conditions(run);
  pass[A] = 0;
}

}  // namespace lare
