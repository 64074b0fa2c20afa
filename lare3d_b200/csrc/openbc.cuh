// openbc.cuh - open (characteristic) boundaries, openboundary.f90.
//
// A side with BC_OPEN gets no ghost fill from the boundary routines (the
// direction is not periodic and the mirror rules are BC_USER only), so its
// second ghost layer keeps the uploaded far-field state.  Once per step,
// after velocity_bcs in predictor_corrector_step (lagran.F90:409-412), each
// point of an open face solves for the first ghost layer of B, rho and
// energy from the Riemann invariants carried out of the domain and in from
// the far field: the fast-mode solver (openboundary.f90:326-378), or the
// Alfven-mode one (:382-455) where the far field has no transverse B.  One
// kernel per face, in the reference's face order (x min, x max, y min, y
// max, z min, z max): a later face reads edge values an earlier one wrote;
// within a face no point reads what another point writes.
#pragma once

LARE_BEGIN

template <class R>
struct OpenIn {
  R vn, vx1, vy1, vz1, bx1, by1, bz1, r1, e1, pbc, pfar, uxf, uyf, uzf, bxf, byf, bzf, rf;
};
template <class R>
struct OpenOut {
  R bx0, by0, bz0, r0, e0;
};

// openboundary.f90:326-378, transverse far field present
template <class R>
__device__ __forceinline__ OpenOut<R> open_fast(const OpenIn<R>& a, R g) {
  OpenOut<R> o;
  const R c0far = sqrt(g * a.pfar / a.rf);
  const R ctfar = sqrt((a.byf * a.byf + a.bzf * a.bzf) / a.rf);
  const R cffar = sqrt(c0far * c0far + ctfar * ctfar);
  const R c0 = sqrt(g * (g - R(1)) * a.e1);
  const R ct = sqrt((a.by1 * a.by1 + a.bz1 * a.bz1) / a.r1);
  const R cf = sqrt(c0 * c0 + ct * ct);
  const R vtest[3] = {a.vn + cf, a.vn - cf, a.vn};
  R pstar[3], pmag[3], vstar[3], rstar[3], bys[3], bzs[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const bool out = vtest[i] >= R(0);  // carried out of the domain
    pstar[i] = out ? a.pbc + R(0.5) * (a.by1 * a.by1 + a.bz1 * a.bz1)
                   : a.pfar + R(0.5) * (a.byf * a.byf + a.bzf * a.bzf);
    pmag[i] = out ? R(0.5) * (a.by1 * a.by1 + a.bz1 * a.bz1) : R(0.5) * (a.byf * a.byf + a.bzf * a.bzf);
    vstar[i] = out ? a.vx1 : a.uxf;
    rstar[i] = out ? a.r1 : a.rf;
    bys[i] = out ? a.by1 : a.byf;
    bzs[i] = out ? a.bz1 : a.bzf;
  }
  o.bx0 = R(0.5) * (a.bx1 + a.bxf);
  o.by0 = R(0.5) * (bys[0] + bys[1]);
  o.bz0 = R(0.5) * (bzs[0] + bzs[1]);
  R pg = R(0.5) * (pstar[0] + pstar[1] + a.rf * cffar * (vstar[0] - vstar[1])) - R(0.5) * (pmag[0] + pmag[1]);
  pg = fmax(pg, R(0));
  const R rhog = rstar[2] + (pg - (pstar[2] - pmag[2])) / (c0far * c0far);
  o.r0 = fmax(rhog, Num<R>::tiny());
  o.e0 = pg / (g - R(1)) / o.r0;
  return o;
}

// openboundary.f90:382-455, no transverse far field
template <class R>
__device__ __forceinline__ OpenOut<R> open_alfven(const OpenIn<R>& a, R g) {
  OpenOut<R> o;
  const R lyfar = -(a.bxf * a.byf), lzfar = -(a.bxf * a.bzf);
  const R c0far = sqrt(g * a.pfar / a.rf);
  const R cxfar = sqrt(a.bxf * a.bxf / a.rf);
  const R c0 = sqrt(g * (g - R(1)) * a.e1);
  const R cx = sqrt(a.bx1 * a.bx1 / a.r1);
  const R vtest[5] = {a.vn + c0, a.vn - c0, a.vn + cx, a.vn - cx, a.vn};
  R pstar[5], pmag[5], ly[5], lz[5], ux[5], uy[5], uz[5], rstar[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const bool out = vtest[i] >= R(0);
    pstar[i] = out ? a.pbc + R(0.5) * (a.by1 * a.by1 + a.bz1 * a.bz1 - a.bx1 * a.bx1)
                   : a.pfar + R(0.5) * (a.byf * a.byf + a.bzf * a.bzf - a.bxf * a.bxf);
    pmag[i] = out ? R(0.5) * (a.by1 * a.by1 + a.bz1 * a.bz1 - a.bx1 * a.bx1)
                  : R(0.5) * (a.byf * a.byf + a.bzf * a.bzf - a.bxf * a.bxf);
    ly[i] = out ? -(a.by1 * a.bx1) : lyfar;
    lz[i] = out ? -(a.bz1 * a.bx1) : lzfar;
    ux[i] = out ? a.vx1 : a.uxf;
    uy[i] = out ? a.vy1 : a.uyf;
    uz[i] = out ? a.vz1 : a.uzf;
    rstar[i] = out ? a.r1 : a.rf;
  }
  o.bx0 = R(0.5) * (a.bx1 + a.bxf);
  if (fabs(o.bx0) <= Num<R>::tiny()) o.bx0 = Num<R>::tiny();
  R lg = R(0.5) * (ly[2] + ly[3] + a.rf * cxfar * (uy[2] - uy[3]));
  o.by0 = -(lg / o.bx0);
  lg = R(0.5) * (lz[2] + lz[3] + a.rf * cxfar * (uz[2] - uz[3]));
  o.bz0 = -(lg / o.bx0);
  R pg = R(0.5) * (pstar[0] + pstar[1] + a.rf * c0far * (ux[0] - ux[1])) -
         R(0.5) * (o.by0 * o.by0 + o.bz0 * o.bz0 - o.bx0 * o.bx0);
  pg = fmax(pg, Num<R>::tiny());
  const R rhog = rstar[4] + (pg - (pstar[4] - pmag[4])) / (c0far * c0far);
  o.r0 = fmax(rhog, Num<R>::tiny());
  o.e0 = pg / (g - R(1)) / o.r0;
  return o;
}

template <class R>
__device__ __forceinline__ OpenOut<R> open_solve(const OpenIn<R>& a, R g) {
  // solver choice on the far-field transverse field (openboundary.f90:63-71)
  const R bperp = sqrt(a.byf * a.byf + a.bzf * a.bzf);
  return bperp <= Num<R>::tiny() ? open_alfven(a, g) : open_fast(a, g);
}

template <class R>
struct OpenArgs {
  R* vx;
  R* vy;
  R* vz;
  R* bx;
  R* by;
  R* bz;
  R* rho;
  R* energy;
  R g;
  int nx, ny, nz, sx, sxy;
};

// Face F (0 x min, 1 x max, 2 y min, 3 y max, 4 z min, 5 z max) over the
// 0..n+1 range of its two other directions (openboundary.f90:36-37 etc.).
// The normal direction's velocity and field are carried as the solver's x
// components, sign-flipped on a min face; the far field is the second
// ghost layer (openboundary.f90:39-61 and mirrors).
template <int F, class R>
__global__ void __launch_bounds__(128) k_open_face(OpenArgs<R> g) {
  constexpr int D = F / 2;          // normal direction
  constexpr bool MAX = (F & 1) != 0;
  const int u = (int)(blockIdx.x * blockDim.x + threadIdx.x);  // first other direction
  const int w = (int)(blockIdx.y * blockDim.y + threadIdx.y);  // second other direction
  const int nn[3] = {g.nx, g.ny, g.nz};
  const int nu = D == 0 ? g.ny : g.nx, nw = D == 2 ? g.ny : g.nz;
  if (u > nu + 1 || w > nw + 1) return;
  const int sx = g.sx, sxy = g.sxy;
  const int SD = D == 0 ? 1 : (D == 1 ? sx : sxy);                 // stride along the normal
  const int base = D == 0 ? sx * u + sxy * w : (D == 1 ? u + sxy * w : u + sx * w);
  const int n = nn[D];
  // normal index of the boundary point (velocity, normal B), the first
  // interior cell (cell quantities, transverse B), the far-field layers and
  // the ghost written
  const int iv = MAX ? n : 0, ic = MAX ? n : 1, ifv = MAX ? n + 2 : -2, ifc = MAX ? n + 2 : -1;
  // the normal and two transverse components of v and B, in the reference's
  // order for each face: x faces (x, y, z), y faces (y, x, z), z faces (z, y, x)
  R* const vn_a = D == 0 ? g.vx : (D == 1 ? g.vy : g.vz);
  R* const vt1 = D == 1 ? g.vx : g.vy;
  R* const vt2 = D == 2 ? g.vx : g.vz;
  R* const bn_a = D == 0 ? g.bx : (D == 1 ? g.by : g.bz);
  R* const bt1 = D == 1 ? g.bx : g.by;
  R* const bt2 = D == 2 ? g.bx : g.bz;
  const R gm = g.g;
  auto at = [&](int i) { return base + SD * i; };
  auto pres = [&](int i) { return (gm - R(1)) * g.energy[at(i)] * g.rho[at(i)]; };
  OpenIn<R> a;
  a.vn = MAX ? vn_a[at(iv)] : -vn_a[at(iv)];
  a.vx1 = a.vn;
  a.vy1 = vt1[at(iv)];
  a.vz1 = vt2[at(iv)];
  a.bx1 = MAX ? bn_a[at(iv)] : -bn_a[at(iv)];
  a.by1 = bt1[at(ic)];
  a.bz1 = bt2[at(ic)];
  a.r1 = g.rho[at(ic)];
  a.e1 = g.energy[at(ic)];
  a.pbc = pres(ic);
  a.pfar = pres(ifc);
  a.uxf = MAX ? vn_a[at(ifv)] : -vn_a[at(ifv)];
  a.uyf = vt1[at(ifv)];
  a.uzf = vt2[at(ifv)];
  a.bxf = MAX ? bn_a[at(ifv)] : -bn_a[at(ifv)];
  a.byf = bt1[at(ifc)];
  a.bzf = bt2[at(ifc)];
  a.rf = g.rho[at(ifc)];
  const OpenOut<R> o = open_solve(a, gm);
  const int gc = MAX ? n + 1 : 0;     // first ghost layer of cells and transverse B
  const int gn = MAX ? n + 1 : -1;    // the ghost normal-B face
  bn_a[at(gn)] = MAX ? o.bx0 : -o.bx0;
  bt1[at(gc)] = o.by0;
  bt2[at(gc)] = o.bz0;
  g.rho[at(gc)] = o.r0;
  g.energy[at(gc)] = o.e0;
}

LARE_END  // namespace lare
