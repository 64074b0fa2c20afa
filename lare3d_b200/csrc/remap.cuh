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
//                 The y and z sweeps use a marching kernel and the x sweep
//                 a warp-shuffle kernel; both form each quotient once.
//   K3 B update   the four flux-difference updates (:121-157), with each
//                 file's own loop ranges as predicates.
//   K4 mass flux  dm (:474-533) over the whole cell box, with dm_x_bcs
//                 (:899-917) folded in: a ghost element is the flux computed
//                 at its source index (the same value the copy would bring).
//   K5 rho, eflux new rho (:174-182) into a second buffer (old rho stays
//                 readable as rho1) and the energy flux (:539-601).
//   K6 energy     energy update (:187-196).
//   K7 vertex     vertex rho_v, cv1, cv2, dm averages and rho_v1 (:201-290).
//   K8 momentum   the three momentum fluxes (:605-895), each times dm, and
//   K9 velocity   the three velocity updates (:292-329), fused into one
//                 kernel that writes the new velocities to second buffers.
// The face-averaged vx1 written back at :265 is only read again as
// REAL(xpass)*(...) with xpass = 0, so it is formed in K8 and not stored.
// Predictor sweeps (predictor_step = .TRUE.) stop after K3.
// B's conversion to flux form before a remap's three sweeps
// (remap.f90:43-69) and back after them (:101-127) happens in the first
// sweep's K2 and K3 and the last sweep's K3 (remap_sweep's bmode), not in
// passes of their own.
//
// Indexing is linear: c = ix + sx*iy + sxy*iz, neighbours by constant
// offsets, with the axis a compile-time parameter.
#pragma once

#include <utility>

LARE_BEGIN

template <int A>
__device__ __forceinline__ int acoord(int ix, int iy, int iz) {
  return A == 0 ? ix : (A == 1 ? iy : iz);
}

// K2 for the y and z sweeps as a marching kernel.  A thread owns a run of
// kMarch consecutive cells along the sweep axis A at one (x, transverse)
// position and walks it, keeping the quotients B/dbv, the dbv and the db1
// and dc1 values of the four-point stencil in registers: each step loads
// the one new stencil point instead of all four and forms one quotient per
// flux instead of four.  Every value is the same expression of the same
// operands as in the per-cell form, so the fluxes are identical bit for bit.
constexpr int kMarch = 32;
constexpr int kBUpdZ32 = 4, kBUpdZ64 = 1;  // z-points per thread of the B updates (measured)

template <class R>
struct BfArgs {
  const R* va;           // velocity component along A (v1 of the reference)
  const R* b1;           // first transported component
  const R* b2;           // second
  const R* db1;
  const R* dc1;
  R* f1;
  R* f2;
  const double* sc;
  int dt_slot;
  int SA, SB1, SB2, SO1, SO2;  // strides along A, the two components' own axes, and their remaining axes
  int SX, SY;                  // strides of the thread grid's two axes (x and the other transverse axis)
  int na;                      // cells along A
  int n0, n1;                  // extents of the thread grid (-1..n+1 each)
  // for the first sweep of a remap, which reads B itself and forms its
  // flux form on the fly: the metrics, the components' axes, the sweep axis
  A1<R> dbm[3];
  int j1, j2, ax;
};

// remap.f90:43-69 on one value: B component j at (ix, iy, iz) times the
// widths of its face along the other two axes, in axis order, where the
// reference converts (its B arrays start at -1 on the other axes).
template <class R>
__device__ __forceinline__ R to_flux(R b, int j, int ix, int iy, int iz, const A1<R> (&m)[3]) {
  if (j == 0) return (iy >= -1 && iz >= -1) ? b * m[1](iy) * m[2](iz) : b;
  if (j == 1) return (ix >= -1 && iz >= -1) ? b * m[0](ix) * m[2](iz) : b;
  return (ix >= -1 && iy >= -1) ? b * m[0](ix) * m[1](iy) : b;
}
// remap.f90:101-127 on one value: the flux form back to B.
template <class R>
__device__ __forceinline__ R from_flux(R b, int j, int ix, int iy, int iz, const A1<R> (&m)[3],
                                       const A1<R> (&r)[3]) {
  if (j == 0) return (iy >= -1 && iz >= -1) ? div_rcp(div_rcp(b, m[1](iy), r[1](iy)), m[2](iz), r[2](iz)) : b;
  if (j == 1) return (ix >= -1 && iz >= -1) ? div_rcp(div_rcp(b, m[0](ix), r[0](ix)), m[2](iz), r[2](iz)) : b;
  return (ix >= -1 && iy >= -1) ? div_rcp(div_rcp(b, m[0](ix), r[0](ix)), m[1](iy), r[1](iy)) : b;
}

// to_flux along a y/z-sweep march line (the first sweep of a remap): the
// line's points have every coordinate >= -1, so the reference converts them
// all; of component j's two face widths, the one across the line (axis c =
// 3 - j - A, at the thread's x or second grid coordinate) is fixed and is
// formed once, the one along the sweep axis is loaded per point and shared
// by both components; they multiply in axis order as in remap.f90:43-69.
template <class R>
struct LineConv {
  const R* mA;  // widths along the sweep axis
  R cf1, cf2;   // the fixed widths of the two components
  bool af1, af2;  // the sweep axis comes first
};
template <class R>
__device__ __forceinline__ LineConv<R> line_conv(const BfArgs<R>& a, int x, int g2) {
  LineConv<R> L;
  L.mA = a.ax == 1 ? a.dbm[1].p : a.dbm[2].p;
  const int ay = 3 - a.ax;  // the grid's second axis: z for the y sweep, y for the z sweep
  auto fixed = [&](int j) {
    const int c = 3 - j - a.ax;
    return c == 0 ? a.dbm[0](x) : (ay == 1 ? a.dbm[1](g2) : a.dbm[2](g2));
  };
  L.cf1 = fixed(a.j1);
  L.cf2 = fixed(a.j2);
  L.af1 = a.ax < 3 - a.j1 - a.ax;
  L.af2 = a.ax < 3 - a.j2 - a.ax;
  return L;
}
template <class R>
__device__ __forceinline__ R line_form(R b, R ma, R cf, bool afirst) {
  return afirst ? b * ma * cf : b * cf * ma;
}

// B / dbv at q, with dbv (in the carried divisor form dv_of) returned in dvb
template <class R>
__device__ __forceinline__ R bf_quot(R b, const R* db1, int q, int SB, R& dvb) {
  dvb = dv_of((db1[q] + db1[q + SB]) * R(0.5));
  return dv_div(b, dvb);
}

template <class R, bool PRE>
__global__ void __launch_bounds__(256, 2) k_bflux_march(BfArgs<R> a) {
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int t1 = blockIdx.y * blockDim.y + threadIdx.y;
  if (t0 >= a.n0 || t1 >= a.n1) return;
  const int ia0 = -1 + (int)blockIdx.z * kMarch;
  const int ia1 = min(ia0 + kMarch - 1, a.na + 1);
  const int SA = a.SA;
  // cell (t0 - 1, t1 - 1, ia0) in grid / along-A coordinates
  int c = (t0 - 1) * a.SX + (t1 - 1) * a.SY + ia0 * SA;
  const R dt = (R)a.sc[a.dt_slot];
  // four-point windows at cm, c, cp, cp2 (clamped as MAX(ia-1,-1), MIN(ia+2,na+2))
  R q1m, q10, q1p, q1p2, d1m, d10, d1p, d1p2;  // flux 1: quotients, dbv
  R q2m, q20, q2p, q2p2, d2m, d20, d2p, d2p2;  // flux 2
  R dcm, dc0, dcp, dbc0, dbcp;                 // dc1 at cm, c, cp; db1 at c, cp
  const int gx = t0 - 1, g2 = t1 - 1;  // the thread grid's coordinates
  LineConv<R> lc{};
  if constexpr (PRE) lc = line_conv(a, gx, g2);
  {
    const int am = ia0 > -1 ? ia0 - 1 : ia0, ap2 = ia0 + 2 <= a.na + 2 ? ia0 + 2 : ia0 + 1;
    const int cm = c + (am - ia0) * SA;
    const int cp = c + SA;
    const int cp2 = c + (ap2 - ia0) * SA;
    auto b1 = [&](int q, int ia) {
      if constexpr (PRE) return line_form(a.b1[q], lc.mA[ia], lc.cf1, lc.af1);
      return a.b1[q];
    };
    auto b2 = [&](int q, int ia) {
      if constexpr (PRE) return line_form(a.b2[q], lc.mA[ia], lc.cf2, lc.af2);
      return a.b2[q];
    };
    q1m = bf_quot(b1(cm, am), a.db1, cm, a.SB1, d1m);
    q10 = bf_quot(b1(c, ia0), a.db1, c, a.SB1, d10);
    q1p = bf_quot(b1(cp, ia0 + 1), a.db1, cp, a.SB1, d1p);
    q1p2 = bf_quot(b1(cp2, ap2), a.db1, cp2, a.SB1, d1p2);
    q2m = bf_quot(b2(cm, am), a.db1, cm, a.SB2, d2m);
    q20 = bf_quot(b2(c, ia0), a.db1, c, a.SB2, d20);
    q2p = bf_quot(b2(cp, ia0 + 1), a.db1, cp, a.SB2, d2p);
    q2p2 = bf_quot(b2(cp2, ap2), a.db1, cp2, a.SB2, d2p2);
    dcm = dv_of(a.dc1[cm]);
    dc0 = dv_of(a.dc1[c]);
    dcp = dv_of(a.dc1[cp]);
    dbc0 = a.db1[c];
    dbcp = a.db1[cp];
  }
  (void)d1m;
  (void)d2m;
  R va0 = a.va[c], va1 = a.va[c - a.SO1], va2 = a.va[c - a.SO2];
  for (int ia = ia0; ia <= ia1; ++ia) {
    // issue the next step's loads before this step's arithmetic
    const int cn = c + SA;
    const bool more = ia < ia1;
    const bool clamp = ia + 3 > a.na + 2;
    const int qn = cn + 2 * SA;
    const bool fetch = more && !clamp;
    R nb1 = R(0), nb2 = R(0), nd = R(0), nd1 = R(0), nd2 = R(0), ndc = R(0), ndb = R(0);
    R nva0 = R(0), nva1 = R(0), nva2 = R(0);
    if (fetch) {
      nb1 = a.b1[qn];
      nb2 = a.b2[qn];
      if constexpr (PRE) {
        const R ma = lc.mA[ia + 3];
        nb1 = line_form(nb1, ma, lc.cf1, lc.af1);
        nb2 = line_form(nb2, ma, lc.cf2, lc.af2);
      }
      nd = a.db1[qn];
      nd1 = a.db1[qn + a.SB1];
      nd2 = a.db1[qn + a.SB2];
    }
    if (more) {
      ndc = a.dc1[cn + SA];
      ndb = a.db1[cn + SA];
    }
    if (more) {
      nva0 = a.va[cn];
      nva1 = a.va[cn - a.SO1];
      nva2 = a.va[cn - a.SO2];
    }
    {
      const R v_advect = (va0 + va1) * R(0.5);
      LimOut<R> L = limiter_dv<R>(v_advect, q1m, q10, q1p, q1p2, dc0, dcm, dcp, dbc0, dbcp, d10, d1p, dt, true);
      a.f1[c] = (L.fu + L.Di * (R(1) - L.phi)) * v_advect * dt;
    }
    {
      const R v_advect = (va0 + va2) * R(0.5);
      LimOut<R> L = limiter_dv<R>(v_advect, q2m, q20, q2p, q2p2, dc0, dcm, dcp, dbc0, dbcp, d20, d2p, dt, true);
      a.f2[c] = (L.fu + L.Di * (R(1) - L.phi)) * v_advect * dt;
    }
    if (!more) break;
    q1m = q10; q10 = q1p; q1p = q1p2;
    d10 = d1p; d1p = d1p2;
    q2m = q20; q20 = q2p; q2p = q2p2;
    d20 = d2p; d2p = d2p2;
    if (clamp) {
      q1p2 = q1p; d1p2 = d1p;
      q2p2 = q2p; d2p2 = d2p;
    } else {
      d1p2 = dv_of((nd + nd1) * R(0.5));
      q1p2 = dv_div(nb1, d1p2);
      d2p2 = dv_of((nd + nd2) * R(0.5));
      q2p2 = dv_div(nb2, d2p2);
    }
    dcm = dc0; dc0 = dcp; dcp = dv_of(ndc);
    dbc0 = dbcp; dbcp = ndb;
    va0 = nva0; va1 = nva1; va2 = nva2;
    c = cn;
  }
}

// K2 for the x sweep: the lanes of a warp hold consecutive x positions, and
// the stencil neighbours along x (one to the left, two to the right) come
// from the neighbouring lanes by shuffles, so a lane loads its own point
// once and forms one quotient per flux.  A warp spans 32 positions and
// writes the kXOut = 29 whose whole stencil lies inside it; warps overlap by
// three positions.  Same expressions, same operands, same results bit for
// bit as the per-cell form.  The launch bounds cap the FP64 form at 48
// registers: it is latency-bound, and the extra resident warps outweigh the
// few spills (measured at 256^3).
constexpr int kXOut = 29;

template <class R, bool PRE>
__global__ void __launch_bounds__(128, 10) k_bflux_x(BfArgs<R> a, int sx, int sxy, int nx, int ny) {
  const int lane = (int)threadIdx.x;                           // blockDim.x == 32: one warp per row
  const int ix = -2 + (int)blockIdx.x * kXOut + lane;          // this lane's x position
  const int iy = -1 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int iz = -1 + (int)blockIdx.z;
  if (iy > ny + 1) return;                                      // uniform over the warp
  const int cx = min(ix, nx + 2);
  const int c = cx + sx * iy + sxy * iz;                        // positions past n+2 load n+2 (unused)
  R d1, d2;
  R bv1 = a.b1[c], bv2 = a.b2[c];
  if constexpr (PRE) {  // the first sweep of a remap reads B itself (by and bz)
    bv1 = to_flux(bv1, 1, cx, iy, iz, a.dbm);
    bv2 = to_flux(bv2, 2, cx, iy, iz, a.dbm);
  }
  const R q1 = bf_quot(bv1, a.db1, c, a.SB1, d1);
  const R q2 = bf_quot(bv2, a.db1, c, a.SB2, d2);
  const R dc = dv_of(a.dc1[c]), db = a.db1[c];
  const unsigned all = 0xffffffffu;
  const R q1m = __shfl_up_sync(all, q1, 1), q1p = __shfl_down_sync(all, q1, 1), q1p2 = __shfl_down_sync(all, q1, 2);
  const R q2m = __shfl_up_sync(all, q2, 1), q2p = __shfl_down_sync(all, q2, 1), q2p2 = __shfl_down_sync(all, q2, 2);
  const R d1p = __shfl_down_sync(all, d1, 1), d2p = __shfl_down_sync(all, d2, 1);
  const R dcm = __shfl_up_sync(all, dc, 1), dcp = __shfl_down_sync(all, dc, 1);
  const R dbp = __shfl_down_sync(all, db, 1);
  if (lane < 1 || lane > kXOut || ix > nx + 1) return;
  const bool left = ix > -1;            // cm = MAX(ix - 1, -1)
  const bool right = ix + 2 <= nx + 2;  // cp2 = MIN(ix + 2, n + 2)
  const R dt = (R)a.sc[a.dt_slot];
  const R va0 = a.va[c], va1 = a.va[c - a.SO1], va2 = a.va[c - a.SO2];
  {
    const R v_advect = (va0 + va1) * R(0.5);
    LimOut<R> L = limiter_dv<R>(v_advect, left ? q1m : q1, q1, q1p, right ? q1p2 : q1p, dc, left ? dcm : dc, dcp, db,
                             dbp, d1, d1p, dt, true);
    a.f1[c] = (L.fu + L.Di * (R(1) - L.phi)) * v_advect * dt;
  }
  {
    const R v_advect = (va0 + va2) * R(0.5);
    LimOut<R> L = limiter_dv<R>(v_advect, left ? q2m : q2, q2, q2p, right ? q2p2 : q2p, dc, left ? dcm : dc, dcp, db,
                             dbp, d2, d2p, dt, true);
    a.f2[c] = (L.fu + L.Di * (R(1) - L.phi)) * v_advect * dt;
  }
}

// The same march with one flux per thread: blockIdx.z selects the flux
// (even: first, odd: second) and the chunk, so a thread carries one
// four-point window instead of two; twice the threads, about half the
// registers each.
template <class R, bool PRE>
__global__ void __launch_bounds__(128) k_bflux_march1(BfArgs<R> a) {
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int t1 = blockIdx.y * blockDim.y + threadIdx.y;
  if (t0 >= a.n0 || t1 >= a.n1) return;
  const bool second = (blockIdx.z & 1u) != 0;
  const int ia0 = -1 + (int)(blockIdx.z >> 1) * kMarch;
  const int ia1 = min(ia0 + kMarch - 1, a.na + 1);
  const int SA = a.SA;
  const R* B = second ? a.b2 : a.b1;
  const int SB = second ? a.SB2 : a.SB1;
  const int SO = second ? a.SO2 : a.SO1;
  R* const fo = second ? a.f2 : a.f1;
  const int gx = t0 - 1, g2 = t1 - 1;  // the thread grid's coordinates
  R cf = R(0);
  bool af = false;
  const R* mA = nullptr;
  if constexpr (PRE) {
    const LineConv<R> lc = line_conv(a, gx, g2);
    cf = second ? lc.cf2 : lc.cf1;
    af = second ? lc.af2 : lc.af1;
    mA = lc.mA;
  }
  int c = gx * a.SX + g2 * a.SY + ia0 * SA;
  const R dt = (R)a.sc[a.dt_slot];
  R qm, q0, qp, qp2, dm, d0, dp, dp2;  // quotients and dbv at cm, c, cp, cp2
  R dcm, dc0, dcp, dbc0, dbcp;
  {
    const int am = ia0 > -1 ? ia0 - 1 : ia0, ap2 = ia0 + 2 <= a.na + 2 ? ia0 + 2 : ia0 + 1;
    const int cm = c + (am - ia0) * SA;
    const int cp = c + SA;
    const int cp2 = c + (ap2 - ia0) * SA;
    auto b = [&](int q, int ia) {
      if constexpr (PRE) return line_form(B[q], mA[ia], cf, af);
      return B[q];
    };
    qm = bf_quot(b(cm, am), a.db1, cm, SB, dm);
    q0 = bf_quot(b(c, ia0), a.db1, c, SB, d0);
    qp = bf_quot(b(cp, ia0 + 1), a.db1, cp, SB, dp);
    qp2 = bf_quot(b(cp2, ap2), a.db1, cp2, SB, dp2);
    dcm = dv_of(a.dc1[cm]);
    dc0 = dv_of(a.dc1[c]);
    dcp = dv_of(a.dc1[cp]);
    dbc0 = a.db1[c];
    dbcp = a.db1[cp];
  }
  (void)dm;
  R va = a.va[c], vo = a.va[c - SO];
  for (int ia = ia0; ia <= ia1; ++ia) {
    const int cn = c + SA;
    const bool more = ia < ia1;
    const bool clamp = ia + 3 > a.na + 2;
    const int qn = cn + 2 * SA;
    const bool fetch = more && !clamp;
    R nb = R(0), nd = R(0), nds = R(0), ndc = R(0), ndb = R(0), nva = R(0), nvo = R(0);
    if (fetch) {
      nb = B[qn];
      if constexpr (PRE) nb = line_form(nb, mA[ia + 3], cf, af);
      nd = a.db1[qn];
      nds = a.db1[qn + SB];
    }
    if (more) {
      ndc = a.dc1[cn + SA];
      ndb = a.db1[cn + SA];
    }
    if (more) {
      nva = a.va[cn];
      nvo = a.va[cn - SO];
    }
    const R v_advect = (va + vo) * R(0.5);
    LimOut<R> L = limiter_dv<R>(v_advect, qm, q0, qp, qp2, dc0, dcm, dcp, dbc0, dbcp, d0, dp, dt, true);
    fo[c] = (L.fu + L.Di * (R(1) - L.phi)) * v_advect * dt;
    if (!more) break;
    qm = q0; q0 = qp; qp = qp2;
    d0 = dp; dp = dp2;
    if (clamp) {
      qp2 = qp; dp2 = dp;
    } else {
      dp2 = dv_of((nd + nds) * R(0.5));
      qp2 = dv_div(nb, dp2);
    }
    dcm = dc0; dc0 = dcp; dcp = dv_of(ndc);
    dbc0 = dbcp; dbcp = ndb;
    va = nva; vo = nvo;
    c = cn;
  }
}

// K1 as a z-marching kernel: a thread owns an (x, y) column and walks a
// chunk of z.  Each face average (xremap.f90:64-86) sums two values of its
// own plane and two of the plane below in that order, so the lower pair is
// carried from the previous step instead of reloaded, and the z face below a
// cell is the previous step's z face above it: 12 to 15 loads per cell
// instead of 28, the same expressions, the same results bit for bit.
constexpr int kGeomZ = 16;

template <class R>
struct GeomArgs {
  const R* vx1;
  const R* vy1;
  const R* vz1;
  const R* cv;
  R* cv1;
  R* cv2;
  R* db1;
  R* dc1;
  A1<R> dbm[3];
  A1<R> rdbm[3];  // reciprocals of dbm, for div_rcp
  R pass_t1, pass_t2;
  const double* sc;
  int dt_slot, nx, ny, nz, sx, sxy;
  bool write_cv2;
};

template <int A, class R>
__global__ void __launch_bounds__(128) k_geom_march(GeomArgs<R> g) {
  // distinct arrays (no output is an input): restrict lets the compiler
  // hoist the next plane's loads above this plane's stores
  const R* __restrict__ vx1_r = g.vx1;
  const R* __restrict__ vy1_r = g.vy1;
  const R* __restrict__ vz1_r = g.vz1;
  const R* __restrict__ cv_r = g.cv;
  R* __restrict__ cv1_r = g.cv1;
  R* __restrict__ cv2_r = g.cv2;
  R* __restrict__ db1_r = g.db1;
  R* __restrict__ dc1_r = g.dc1;
  constexpr int T1 = A == 0 ? 1 : 0, T2 = A == 2 ? 1 : 2;
  const int ix = -1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int iy = -1 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  if (ix > g.nx + 2 || iy > g.ny + 2) return;
  const int z0 = -1 + (int)blockIdx.z * kGeomZ;
  const int z1 = min(z0 + kGeomZ - 1, g.nz + 2);
  const int sx = g.sx, sxy = g.sxy;
  const int nn[3] = {g.nx, g.ny, g.nz};
  const R q4 = R(0.25);
  const R dt = (R)g.sc[g.dt_slot];
  const R* __restrict__ vx1 = vx1_r;
  const R* __restrict__ vy1 = vy1_r;
  const R* __restrict__ vz1 = vz1_r;
  constexpr int NX = A == 0 ? 3 : 2;  // x faces: c - 1, c (, c + 1)
  constexpr int NY = A == 1 ? 3 : 2;  // y faces: c - sx, c (, c + sx)
  const bool ahead = (A == 0 ? ix : iy) < nn[A] + 2;  // a face beyond c along A exists (A = 0, 1)
  int c = ix + sx * iy + sxy * (z0 - 1);
  // carried lower pairs of the x and y faces, and the z faces
  R xa[NX], xb[NX], ya[NY], yb[NY];
  auto xo = [&](int k) { return k - 1; };        // x offset of x face k
  auto yo = [&](int k) { return (k - 1) * sx; }; // y offset of y face k
#pragma unroll
  for (int k = 0; k < NX; ++k) {
    const bool ok = k < 2 || ahead;
    xa[k] = ok ? vx1[c + xo(k)] : R(0);
    xb[k] = ok ? vx1[c + xo(k) - sx] : R(0);
  }
#pragma unroll
  for (int k = 0; k < NY; ++k) {
    const bool ok = k < 2 || ahead;
    ya[k] = ok ? vy1[c + yo(k)] : R(0);
    yb[k] = ok ? vy1[c + yo(k) - 1] : R(0);
  }
  auto vzf = [&](int q) { return (vz1[q] + vz1[q - 1] + vz1[q - sx] + vz1[q - 1 - sx]) * q4; };
  R vz_prev = vzf(c);          // z face of plane z0 - 1
  c += sxy;
  R vz_cur = vzf(c);           // z face of plane z0
  // the loads of each plane are issued one plane ahead: x and y face pairs,
  // the next z face (its four corners) and cv
  struct Plane {
    R xa[NX], xb[NX], ya[NY], yb[NY], z[4], cv;
  };
  auto fetch = [&](int q, int iz) {
    Plane P;
#pragma unroll
    for (int k = 0; k < NX; ++k) {
      const bool ok = k < 2 || ahead;
      P.xa[k] = ok ? vx1[q + xo(k)] : R(0);
      P.xb[k] = ok ? vx1[q + xo(k) - sx] : R(0);
    }
#pragma unroll
    for (int k = 0; k < NY; ++k) {
      const bool ok = k < 2 || ahead;
      P.ya[k] = ok ? vy1[q + yo(k)] : R(0);
      P.yb[k] = ok ? vy1[q + yo(k) - 1] : R(0);
    }
    // the z face above this plane: read by the z sweep (vz_next) and, for
    // the other sweeps, carried as the next plane's current z face
    const bool zok = A == 2 ? iz < g.nz + 2 : iz < z1;
    const int qz = q + sxy;
    P.z[0] = zok ? vz1[qz] : R(0);
    P.z[1] = zok ? vz1[qz - 1] : R(0);
    P.z[2] = zok ? vz1[qz - sx] : R(0);
    P.z[3] = zok ? vz1[qz - 1 - sx] : R(0);
    P.cv = cv_r[q];
    return P;
  };
  Plane nxt = fetch(c, z0);
  for (int iz = z0; iz <= z1; ++iz, c += sxy) {
    const Plane cur = nxt;
    if (iz < z1) nxt = fetch(c + sxy, iz + 1);
    R vxfc[NX], vyfc[NY];
#pragma unroll
    for (int k = 0; k < NX; ++k) {
      const R a = cur.xa[k], b = cur.xb[k];
      vxfc[k] = (a + b + xa[k] + xb[k]) * q4;
      xa[k] = a;
      xb[k] = b;
    }
#pragma unroll
    for (int k = 0; k < NY; ++k) {
      const R a = cur.ya[k], b = cur.yb[k];
      vyfc[k] = (a + b + ya[k] + yb[k]) * q4;
      ya[k] = a;
      yb[k] = b;
    }
    const R vxb = vxfc[1], vxbm = vxfc[0];
    const R vyb = vyfc[1], vybm = vyfc[0];
    const R vzb = vz_cur, vzbm = vz_prev;
    const R vz_above = (cur.z[0] + cur.z[1] + cur.z[2] + cur.z[3]) * q4;
    R vz_next = R(0);
    if (A == 2 && iz < g.nz + 2) vz_next = vz_above;
    const R dvv[3] = {vxb - vxbm, vyb - vybm, vzb - vzbm};
    const int pp[3] = {ix, iy, iz};
    // quotients by the metrics: through their reciprocals for the z sweep;
    // the x sweep's form (three x faces live) is faster with plain division
    auto quot = [&](R a, int d) {
#if LARE_FAST
      return a * g.rdbm[d](pp[d]);
#else
      return A == 0 ? a / g.dbm[d](pp[d]) : div_rcp(a, g.dbm[d](pp[d]), g.rdbm[d](pp[d]));
#endif
    };
    const R term_t1 = quot(g.pass_t1 * dvv[T1], T1);
    const R term_t2 = quot(g.pass_t2 * dvv[T2], T2);
    const R term_a = quot(dvv[A], A);
    R dv = (term_t1 + term_t2 + term_a) * dt;
    const R cvc = cur.cv;
    cv1_r[c] = cvc * (R(1) + dv);
    if (g.write_cv2) {
      dv = (term_t1 + term_t2) * dt;
      cv2_r[c] = cvc * (R(1) + dv);
    }
    const R d0 = g.dbm[A](pp[A]) + dvv[A] * dt;
    db1_r[c] = d0;
    R d1 = d0;
    if (pp[A] < nn[A] + 2) {
      const R f = A == 0 ? vxfc[NX - 1] : (A == 1 ? vyfc[NY - 1] : vz_next);
      const R fa = A == 0 ? vxb : (A == 1 ? vyb : vzb);
      d1 = g.dbm[A](pp[A] + 1) + (f - fa) * dt;
    }
    dc1_r[c] = R(0.5) * (d0 + d1);
    vz_prev = vz_cur;
    vz_cur = A == 2 ? vz_next : (iz < z1 ? vz_above : R(0));
  }
}

// K7 as a z-marching kernel: a thread owns an (x, y) column of vertices and
// walks a chunk of z.  The eight cells around vertex (x, y, z) are the
// (x..x+1, y..y+1) quads of planes z and z+1, summed lower quad first in
// the reference's order, so each step loads the upper quad of each input
// and carries it down as the next vertex's lower quad: 18 to 20 loads per
// vertex instead of 40, the same sums in the same order, the same results
// bit for bit.  dm around c - e_A needs the quads of planes z-1 and z (A = z,
// one more plane carried) or the quads shifted by one cell in x or y (two
// more loads per plane).
constexpr int kVertZ = 16;

template <class R>
struct VertArgs {
  const R* rho;
  const R* cv1;
  const R* cv2;
  const R* dm;
  R* rv;
  R* rv1;
  R* cv1v;
  R* cv2v;
  R* dmv;
  int lo[3], hi[3];
  int na, sx, sxy;
};

template <int A, class R>
__global__ void __launch_bounds__(128) k_vert_march(VertArgs<R> g) {
  const int ix = g.lo[0] + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int iy = g.lo[1] + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  if (ix > g.hi[0] || iy > g.hi[1]) return;
  const int z0 = g.lo[2] + (int)blockIdx.z * kVertZ;
  const int z1 = min(z0 + kVertZ - 1, g.hi[2]);
  const int sx = g.sx, sxy = g.sxy, na = g.na;
  const int q1 = 1, q2 = sx, q3 = 1 + sx;                     // quad offsets after 0
  const int e0 = A == 0 ? -1 : -sx, e1 = A == 0 ? -1 + sx : 1 - sx;  // shifted-quad cells not in the quad
  int c = ix + sx * iy + sxy * z0;
  // lower quads (plane z0)
  R pr[4], c1[4], c2[4], d[4], dx[2], dz[4];
  auto load = [&](int b, R (&p)[4], R (&w1)[4], R (&w2)[4], R (&m)[4], R (&mx)[2]) {
    const int o[4] = {0, q1, q2, q3};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      w1[q] = g.cv1[b + o[q]];
      p[q] = g.rho[b + o[q]] * w1[q];
      w2[q] = g.cv2[b + o[q]];
      m[q] = g.dm[b + o[q]];
    }
    if (A != 2) {
      mx[0] = g.dm[b + e0];
      mx[1] = g.dm[b + e1];
    }
  };
  load(c, pr, c1, c2, d, dx);
  if (A == 2) {
    const int b = c - sxy;
    dz[0] = g.dm[b];
    dz[1] = g.dm[b + q1];
    dz[2] = g.dm[b + q2];
    dz[3] = g.dm[b + q3];
  }
  for (int iz = z0; iz <= z1; ++iz, c += sxy) {
    R pu[4], cu1[4], cu2[4], du[4], dxu[2];
    load(c + sxy, pu, cu1, cu2, du, dxu);
    const int ia = A == 0 ? ix : (A == 1 ? iy : iz);
    R s = pr[0], w = c1[0];
#pragma unroll
    for (int q = 1; q < 4; ++q) {
      s = s + pr[q];
      w = w + c1[q];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      s = s + pu[q];
      w = w + cu1[q];
    }
    const R rvc = qdiv(s, w);
    g.rv[c] = rvc;
    R tp = d[0];
#pragma unroll
    for (int q = 1; q < 4; ++q) tp = tp + d[q];
#pragma unroll
    for (int q = 0; q < 4; ++q) tp = tp + du[q];
    if (ia <= na) g.dmv[c] = tp * R(0.125);
    if (ia >= 0 && ia <= na) {
      R w2 = c2[0];
#pragma unroll
      for (int q = 1; q < 4; ++q) w2 = w2 + c2[q];
#pragma unroll
      for (int q = 0; q < 4; ++q) w2 = w2 + cu2[q];
      const R cc1 = w * R(0.125), cc2 = w2 * R(0.125);
      g.cv1v[c] = cc1;
      g.cv2v[c] = cc2;
      // dm summed over the cells around c - e_A, lower quad first
      R tm;
      if (A == 2) {
        tm = dz[0] + dz[1] + dz[2] + dz[3] + d[0] + d[1] + d[2] + d[3];
      } else if (A == 0) {  // quad cells (x-1, y), (x, y), (x-1, y+1), (x, y+1)
        tm = dx[0] + d[0] + dx[1] + d[2] + dxu[0] + du[0] + dxu[1] + du[2];
      } else {              // quad cells (x, y-1), (x+1, y-1), (x, y), (x+1, y)
        tm = dx[0] + dx[1] + d[0] + d[1] + dxu[0] + dxu[1] + du[0] + du[1];
      }
      const R dmm = tm * R(0.125);
      const R dmp = tp * R(0.125);
      g.rv1[c] = qdiv(rvc * cc1 + dmm - dmp, cc2);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (A == 2) dz[q] = d[q];
      pr[q] = pu[q];
      c1[q] = cu1[q];
      c2[q] = cu2[q];
      d[q] = du[q];
    }
    if (A != 2) {
      dx[0] = dxu[0];
      dx[1] = dxu[1];
    }
  }
}

// K8 + K9 fused: the momentum fluxes (xremap.f90:605-895, each times dm)
// and the velocity updates that consume them (:292-329).  K9 updates v in
// place while K8's stencil reads v around each face, so the fused kernel
// writes the new velocities to a second set of buffers (swapped in by the
// caller; their ghosts are refilled by boundary_conditions right after) and
// never stores the fluxes: the update at c needs the fluxes at faces c-e_A
// and c.  x sweep: the lanes of a warp hold consecutive faces and pass the
// flux one lane up (31 updates per 32 lanes).  y and z sweeps: a thread
// walks kMomA faces along A, carrying the stencil windows (one new point
// per step) and the flux of the face behind; its register cap (launch
// bounds) is the measured best per precision.  Every flux and update is the
// reference's expression over the same operands, so the results are
// identical bit for bit.
constexpr int kMomA = 32;

template <class R>
struct MomArgs {
  const R* va;  // v1 along A
  const R* rv;
  const R* dmv;
  const R* db1;
  const R* dc1;
  const R* v[3];
  R* vn[3];
  const R* cv1v;
  const R* cv2v;
  const R* rv1;
  R* fp[3];  // rke only: the fluxes before their product with dm
  A1<R> dct1, dct2;
  const double* sc;
  int dt_slot, nx, ny, nz, na, n3, sx, sxy, SA, S3;
};

// the three momentum fluxes through a face (K8's body) from its stencil
// values: w[comp] = v at c-e_A, c, c+e_A, c+2e_A; db1 at c, c+e_A, c+2e_A;
// dc1 at c, c+e_A; v1 (va), rho_v (rv) at c, c+e_A; dm at c
// BOTH: fpre[comp] also receives the flux before its product with dm (what
// rke's kinetic-energy terms use, xremap.f90:664-695).
template <class R, bool BOTH = false>
__device__ __forceinline__ void mom_flux_vals(R area, R va0, R va1, R rvc, R rvp, R dmc, R db0, R db1, R db2, R dc0,
                                              R dc1, const R (&w)[3][4], R dt, R (&F)[3], R* fpre = nullptr) {
  const R v_advect = (va0 + va1) * R(0.5);  // the face-averaged v1 of xremap.f90:257-265
  // The upwind choice, phi and dmu depend only on v_advect and the
  // geometry, so they are formed once for the three components (the same
  // expressions the limiter evaluates per component).
  const R dxci = db1, dxcm = db0, dxcp = db2, dxbi = dc0, dxbp = dc1;
  const R sign_v = copysign(R(1), v_advect);
  const R vad_p = (sign_v + R(1)) * R(0.5);
  const R vad_m = R(1) - vad_p;
  const R dxbu = dxbi * vad_p + dxbp * vad_m;
  const R rhou = rvc * vad_p + rvp * vad_m;
#if LARE_FAST
  // product build: the upwind widths by selection (vad_p is 0 or 1) and one
  // reciprocal per divisor, shared by the three components
  const R rci = fast_rcp(dxci), rcu = fast_rcp(signbit(v_advect) ? dxcp : dxcm), rbu = fast_rcp(dxbu);
  const R phi = fabs(v_advect) * dt * rbu;
  const R dmu = fabs(dmc) * rbu * fast_rcp(area * rhou);
#else
  const R dxcu = dxcm * vad_p + dxcp * vad_m;
  const R phi = fabs(v_advect) * dt / dxbu;
  const R dmu = fabs(dmc) / area / dxbu / rhou;
#endif
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
    const R fm = w[comp][0], fi = w[comp][1], fp = w[comp][2], fp2 = w[comp][3];
    const R dfm = fi - fm, dfi = fp - fi, dfp = fp2 - fp;
    const R fu = fi * vad_p + fp * vad_m;
    const R dfu = dfm * vad_p + dfp * vad_m;
#if LARE_FAST
    R Da = (R(2) - phi) * fabs(dfi) * rci + (R(1) + phi) * fabs(dfu) * rcu;
#else
    R Da = (R(2) - phi) * fabs(dfi) / dxci + (R(1) + phi) * fabs(dfu) / dxcu;
#endif
    Da = Da * (R(1) / R(6));
    const R ss = R(0.5) * (copysign(R(1), dfi) + copysign(R(1), dfu));
    const R Di = sign_v * ss * fmin(fmin(fabs(Da) * dxbu, fabs(dfi)), fabs(dfu));
    const R f = fu + Di * (R(1) - dmu);
    if constexpr (BOTH) fpre[comp] = f;
    F[comp] = f * dmc;
  }
}

// the same, loading the stencil of face c (RKE: also store the fluxes
// before their product with dm in g.fp)
template <class R, bool RKE = false>
__device__ __forceinline__ void mom_flux(const MomArgs<R>& g, int c, int i1, int i2, R dt, R (&F)[3]) {
  const int SA = g.SA;
  R w[3][4];
#pragma unroll
  for (int comp = 0; comp < 3; ++comp)
#pragma unroll
    for (int q = 0; q < 4; ++q) w[comp][q] = g.v[comp][c + (q - 1) * SA];
  R fpre[3];
  mom_flux_vals<R, RKE>(g.dct1(i1) * g.dct2(i2), g.va[c], g.va[c + SA], g.rv[c], g.rv[c + SA], g.dmv[c],
                               g.db1[c], g.db1[c + SA], g.db1[c + 2 * SA], g.dc1[c], g.dc1[c + SA], w, dt, F, fpre);
  if constexpr (RKE) {
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) g.fp[comp][c] = fpre[comp];
  }
}

// rke's kinetic-energy defect of one component through the vertex pair
// (c, c + e_A) (xremap.f90:664-695 and its eight siblings in [xyz]remap.f90,
// all of one form): f the flux before the product with dm, v the velocity
// before the update.
template <class R>
__device__ __forceinline__ R rke_dk(const R* v, const R* f, const R* dmv, const R* rv1, const R* cv2v, int c,
                                    int SA) {
  const R v0 = v[c], v1 = v[c + SA];
  const R fm = f[c - SA], f0 = f[c], fp = f[c + SA];
  const R dmm = dmv[c - SA], dm0 = dmv[c], dmp = dmv[c + SA];
  const R m = rv1[c] * cv2v[c], mp = rv1[c + SA] * cv2v[c + SA];
  const R ai = (v0 - fm) * dmm / m - (v0 - f0) * dm0 / m;
  const R aip = (v1 - f0) * dm0 / mp - (v1 - fp) * dmp / mp;
  R dk = (v1 - v0) * (f0 - R(0.5) * (v1 + v0)) - R(0.5) * ai * (v0 - f0) + R(0.5) * aip * (v1 - f0);
  return dk * dm0 * R(0.5);
}

// K9's update at c from the fluxes at faces c - e_A (Fm) and c (F)
template <class R>
__device__ __forceinline__ void mom_update(const MomArgs<R>& g, int c, const R (&Fm)[3], const R (&F)[3]) {
  const R rvc = g.rv[c], c1 = g.cv1v[c], den = dv_of(g.cv2v[c] * g.rv1[c]);
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) g.vn[comp][c] = dv_div(rvc * g.v[comp][c] * c1 + Fm[comp] - F[comp], den);
}

template <class R, bool RKE>
__global__ void __launch_bounds__(128) k_mom_x(MomArgs<R> g) {
  const int lane = (int)threadIdx.x;                        // blockDim.x == 32: one warp per row
  const int ix = -1 + (int)blockIdx.x * 31 + lane;          // face / vertex x position
  const int iy = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int iz = (int)blockIdx.z;
  if (iy > g.ny) return;                                    // uniform over the warp
  const R dt = (R)g.sc[g.dt_slot];
  const int c = ix + g.sx * iy + g.sxy * iz;
  R F[3] = {R(0), R(0), R(0)};
  if (ix <= g.nx) mom_flux<R, RKE>(g, c, iy, iz, dt, F);    // faces -1..n
  R Fm[3];
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) Fm[comp] = __shfl_up_sync(0xffffffffu, F[comp], 1);
  if (lane >= 1 && ix >= 0 && ix <= g.nx) mom_update(g, c, Fm, F);
}

template <class R, bool RKE>
__global__ void __launch_bounds__(128, sizeof(R) == 8 ? 4 : 8) k_mom_march(MomArgs<R> g) {
  const int t0 = (int)(blockIdx.x * blockDim.x + threadIdx.x);  // x, 0..nx
  const int t1 = (int)(blockIdx.y * blockDim.y + threadIdx.y);  // the third axis, 0..n3
  if (t0 > g.nx || t1 > g.n3) return;
  const int ia0 = (int)blockIdx.z * kMomA;
  const int ia1 = min(ia0 + kMomA - 1, g.na);
  const R dt = (R)g.sc[g.dt_slot];
  const int SA = g.SA;
  const R area = g.dct1(t0) * g.dct2(t1);
  // stencil window of face ia0 - 1; each step shifts it by one and loads
  // the new far point
  int c = t0 + t1 * g.S3 + (ia0 - 1) * SA;
  R w[3][4];
#pragma unroll
  for (int comp = 0; comp < 3; ++comp)
#pragma unroll
    for (int q = 0; q < 4; ++q) w[comp][q] = g.v[comp][c + (q - 1) * SA];
  R va0 = g.va[c], va1 = g.va[c + SA], rvc = g.rv[c], rvn = g.rv[c + SA];
  R dbw0 = g.db1[c], dbw1 = g.db1[c + SA], dbw2 = g.db1[c + 2 * SA], dcw0 = g.dc1[c], dcw1 = g.dc1[c + SA];
  R Fm[3], fpre[3];
  mom_flux_vals<R, RKE>(area, va0, va1, rvc, rvn, g.dmv[c], dbw0, dbw1, dbw2, dcw0, dcw1, w, dt, Fm, fpre);
  if constexpr (RKE) {
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) g.fp[comp][c] = fpre[comp];
  }
  // the loads of face c + SA are issued one step ahead (a face's own values
  // and the new far points of the windows), so each step's arithmetic waits
  // on loads issued a step earlier
  struct Next {
    R w[3], va, rv, db, dc, dm, c1, c2, r1;
  };
  auto fetch = [&](int q) {
    Next n;
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) n.w[comp] = g.v[comp][q + 2 * SA];
    n.va = g.va[q + SA];
    n.rv = g.rv[q + SA];
    n.db = g.db1[q + 2 * SA];
    n.dc = g.dc1[q + SA];
    n.dm = g.dmv[q];
    n.c1 = g.cv1v[q];
    n.c2 = g.cv2v[q];
    n.r1 = g.rv1[q];
    return n;
  };
  Next nx = fetch(c + SA);
  for (int ia = ia0; ia <= ia1; ++ia) {
    c += SA;
    const Next cur = nx;
    if (ia < ia1) nx = fetch(c + SA);
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      w[comp][0] = w[comp][1];
      w[comp][1] = w[comp][2];
      w[comp][2] = w[comp][3];
      w[comp][3] = cur.w[comp];
    }
    va0 = va1;
    va1 = cur.va;
    rvc = rvn;
    rvn = cur.rv;
    dbw0 = dbw1;
    dbw1 = dbw2;
    dbw2 = cur.db;
    dcw0 = dcw1;
    dcw1 = cur.dc;
    R F[3];
    mom_flux_vals<R, RKE>(area, va0, va1, rvc, rvn, cur.dm, dbw0, dbw1, dbw2, dcw0, dcw1, w, dt, F, fpre);
    if constexpr (RKE) {
#pragma unroll
      for (int comp = 0; comp < 3; ++comp) g.fp[comp][c] = fpre[comp];
    }
    // K9's update at c: fluxes at faces c - e_A and c
    const R c1 = cur.c1, den = dv_of(cur.c2 * cur.r1);
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      g.vn[comp][c] = dv_div(rvc * w[comp][1] * c1 + Fm[comp] - F[comp], den);
      Fm[comp] = F[comp];
    }
  }
}

// K3 with kBUpdZ z-points per thread: every load of all the thread's
// points is issued before any store (a point reads and writes B only at
// itself), so each thread keeps several independent loads in flight; the
// FP32 form, 4 bytes a word, is otherwise latency-bound well below HBM
// speed.  Same expressions and predicates as the per-point form.
//
// MODE 0, a middle sweep: the update in place over the box 0..n+1.
// MODE 1, the first sweep of a remap: B is read as stored, put in flux form
// (remap.f90:43-69) and updated over 0..n+1; every point of the arrays' box
// -2..n+2 is written, to the output arrays (the predictor's B0 buffers,
// whose B is kept, or B itself).  MODE 2, the last sweep: updated over
// 0..n+1, then every point of -2..n+2 is put back from flux form
// (remap.f90:101-127).  The conversions are the reference's expressions on
// the same operands, so the result equals converting in separate passes.
template <class R>
struct BUpdArgs {
  const R* f1;
  const R* f2;
  R* Ba;   // B along the sweep axis
  R* Bb1;  // the two transported components
  R* Bb2;
  R* oa;   // where MODE 1 writes them
  R* ob1;
  R* ob2;
  A1<R> dbm[3], rdbm[3];
  int nx, ny, nz, sx, sxy, SA, SB1, SB2;
};

template <int A, int PTS, int MODE, class R>
__global__ void __launch_bounds__(128) k_bupdate(BUpdArgs<R> g) {
  constexpr int JA = A, J1 = A == 0 ? 1 : 0, J2 = A == 2 ? 1 : 2;  // the components' axes
  constexpr int LO = MODE == 0 ? 0 : -2, EXT = MODE == 0 ? 1 : 2;   // the box LO..n+EXT
  const int ix = LO + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int iy = LO + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  if (ix > g.nx + EXT || iy > g.ny + EXT) return;
  const int z0 = LO + (int)blockIdx.z * PTS;
  const bool in_xy = ix >= 0 && ix <= g.nx + 1 && iy >= 0 && iy <= g.ny + 1;
  R b1[PTS], f1c[PTS], f1a[PTS], ba[PTS], f1b[PTS], b2[PTS], f2c[PTS], f2a[PTS], f2b[PTS];
  bool ok[PTS], in[PTS];
#pragma unroll
  for (int p = 0; p < PTS; ++p) {
    const int iz = z0 + p;
    ok[p] = iz <= g.nz + EXT;
    in[p] = in_xy && iz >= 0 && iz <= g.nz + 1;  // the update box
    const int c = ix + g.sx * iy + g.sxy * (ok[p] ? iz : z0);
    b1[p] = g.Bb1[c];
    ba[p] = g.Ba[c];
    b2[p] = g.Bb2[c];
    f1c[p] = f1a[p] = f1b[p] = f2c[p] = f2a[p] = f2b[p] = R(0);
    if (in[p]) {
      f1c[p] = g.f1[c];
      f1a[p] = g.f1[c - g.SA];
      f1b[p] = g.f1[c - g.SB1];
      f2c[p] = g.f2[c];
      f2a[p] = g.f2[c - g.SA];
      f2b[p] = g.f2[c - g.SB2];
    }
  }
#pragma unroll
  for (int p = 0; p < PTS; ++p) {
    if (!ok[p]) continue;
    const int iz = z0 + p;
    const int c = ix + g.sx * iy + g.sxy * iz;
    R v1 = b1[p], va = ba[p], v2 = b2[p];
    if constexpr (MODE == 1) {
      v1 = to_flux(v1, J1, ix, iy, iz, g.dbm);
      va = to_flux(va, JA, ix, iy, iz, g.dbm);
      v2 = to_flux(v2, J2, ix, iy, iz, g.dbm);
    }
    // second flux ranges (xremap.f90:141-157; yremap.f90:142-158)
    bool r2a = true, r2b = true;
    if (A == 0) {
      r2a = ix >= 1 && ix <= g.nx && iy >= 1 && iy <= g.ny && iz <= g.nz;
      r2b = ix <= g.nx;
    } else if (A == 1) {
      r2b = ix >= 1 && ix <= g.nx && iy <= g.ny && iz >= 1 && iz <= g.nz;
    }
    if (in[p]) {
      // first flux: b1 over 0:n+1 all, a-component over 0:n+1 all
      v1 = v1 - f1c[p] + f1a[p];
      R b = va + f1c[p] - f1b[p];
      if (r2a) v2 = v2 - f2c[p] + f2a[p];
      if (r2b) b = b + f2c[p] - f2b[p];
      va = b;
    }
    if constexpr (MODE == 0) {
      g.Bb1[c] = v1;
      if (r2a) g.Bb2[c] = v2;
      g.Ba[c] = va;
    } else {
      if constexpr (MODE == 2) {
        v1 = from_flux(v1, J1, ix, iy, iz, g.dbm, g.rdbm);
        va = from_flux(va, JA, ix, iy, iz, g.dbm, g.rdbm);
        v2 = from_flux(v2, J2, ix, iy, iz, g.dbm, g.rdbm);
      }
      g.ob1[c] = v1;
      g.oa[c] = va;
      g.ob2[c] = v2;
    }
  }
}

// K4 + K5 + K6 for the y and z sweeps as one marching kernel.  A thread owns
// a line along A at one (x, transverse) position of the cell box and walks a
// chunk of it: at each point it forms the mass flux dm (K4, with the ghost
// values of dm_[yz]_bcs taken at their source index), the new density from
// the dm below and here (K5), the energy flux (K5) and the new energy from
// the energy flux below and here (K6).  The fluxes of the point below are
// carried in registers, so the energy flux never reaches memory, and the new
// energy goes to a second buffer (swapped in after the launch) because the
// limiter of the next chunk still reads the old values.  The same
// expressions over the same operands as the three point kernels.
constexpr int kMEChunk = 16;

template <class R>
struct MEArgs {
  const R* va;       // velocity component along A (v1)
  const R* rho;      // old density (rho1)
  R* rho_new;
  const R* energy;   // old energy
  R* energy_new;
  R* dm;
  const R* cv1;
  const R* cv2;
  const R* db1;
  const R* dc1;
  A1<R> dbt1, dbt2;  // widths of the transverse axes
  const double* sc;
  int dt_slot;
  int SA, S1, S2, SY;  // strides along A, T1 (= x), T2, and the thread grid's second axis (= T2)
  int na, nt1, nt2;
  bool per;
};

template <class R>
__global__ void __launch_bounds__(128) k_mass_energy_march(MEArgs<R> a) {
  const int x = (int)(blockIdx.x * blockDim.x + threadIdx.x) - 1;  // T1 = x, -1..nt1+2
  const int t = (int)(blockIdx.y * blockDim.y + threadIdx.y) - 1;  // T2, -1..nt2+2
  if (x > a.nt1 + 2 || t > a.nt2 + 2) return;
  const int na = a.na, SA = a.SA, S1 = a.S1, S2 = a.S2;
  const int ia0 = -1 + (int)blockIdx.z * kMEChunk;
  const int ia1 = min(ia0 + kMEChunk - 1, na + 2);
  const bool inside_t = x >= 0 && x <= a.nt1 + 1 && t >= 0 && t <= a.nt2 + 1;  // dm's transverse range
  const bool line0 = x <= a.nt1 && t <= a.nt2 && x >= 0 && t >= 0;          // the energy flux's
  const bool line1 = line0 && x >= 1 && t >= 1;                              // the updates'
  const R dt = (R)a.sc[a.dt_slot];
  const R area = inside_t ? a.dbt1(x) * a.dbt2(t) : R(0);
  const R* __restrict__ rho = a.rho;
  const R* __restrict__ en = a.energy;
  const R* __restrict__ va = a.va;
  const R* __restrict__ dc1 = a.dc1;
  const R* __restrict__ db1 = a.db1;
  // K4 at ia (cell c), from its source index
  auto mass_flux = [&](int ia, int c) -> R {
    if (!inside_t) return R(0);
    int sa = ia;
    if (a.per) {
      if (ia == na + 1) sa = 1;
      else if (ia == na + 2) sa = 2;
      else if (ia == -1) sa = na - 1;
      else if (ia == 0) sa = na;
    } else {
      if (ia == na + 1) sa = na;
      else if (ia == -1) sa = 0;
      else if (ia == na + 2) return R(0);
    }
    const int q = c + (sa - ia) * SA;
    const int qm = q - SA, qp = q + SA, qp2 = q + 2 * SA;
    const R v_advect = (va[q] + va[q - S1] + va[q - S2] + va[q - S1 - S2]) * R(0.25);
    LimOut<R> L = limiter<R>(v_advect, rho[qm], rho[q], rho[qp], rho[qp2], dc1[q], dc1[qm], dc1[qp], db1[q],
                             db1[qp], R(0), R(0), dt, false);
    return (L.fu + L.Di * (R(1) - L.phi)) * v_advect * dt * area;
  };
  // K5's energy flux at ia (cell c), 0 <= ia <= na on line0
  auto energy_flux = [&](int c, R dmc) -> R {
    const int cm = c - SA, cp = c + SA, cp2 = c + 2 * SA;
    const R v_advect = (va[c] + va[c - S1] + va[c - S2] + va[c - S1 - S2]) * R(0.25);
    LimOut<R> L = limiter<R>(v_advect, en[cm], en[c], en[cp], en[cp2], dc1[c], dc1[cm], dc1[cp], db1[c], db1[cp],
                             R(0), R(0), dt, false);
    const R rhou = rho[c] * L.vad_p + rho[cp] * L.vad_m;
#if LARE_FAST
    const R dmu = fabs(dmc) * fast_rcp(area * L.dxbu * rhou);
#else
    const R dmu = fabs(dmc) / area / L.dxbu / rhou;
#endif
    return (L.fu + L.Di * (R(1) - dmu)) * dmc;
  };
  const int base = x + t * a.SY;
  // loads along the line, clamped to the cell box (a clamped value is never
  // used: the windows reach past n + 2 only at points whose dm is a ghost
  // value and whose energy flux is not formed)
  auto at = [&](int ia) { return base + min(ia, na + 2) * SA; };
  auto vface = [&](int q) { return (va[q] + va[q - S1] + va[q - S2] + va[q - S1 - S2]) * R(0.25); };
  // the fluxes at ia0 - 1, which the first updates of the chunk read
  R dm_prev = R(0), ef_prev = R(0);
  if (ia0 >= 1 && ia0 - 1 <= na) {
    dm_prev = mass_flux(ia0 - 1, at(ia0 - 1));
    if (line0) ef_prev = energy_flux(at(ia0 - 1), dm_prev);
  }
  // register windows of step ia: rho and energy at ia-1..ia+2, dc1 at
  // ia-1..ia+1, db1 at ia..ia+1, and the point's face velocity, cv1, cv2
  R r[4], e[4], dcw[3], dbw[2];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    r[k] = rho[at(ia0 - 1 + k)];
    e[k] = en[at(ia0 - 1 + k)];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) dcw[k] = dc1[at(ia0 - 1 + k)];
  dbw[0] = db1[at(ia0)];
  dbw[1] = db1[at(ia0 + 1)];
  R vf = vface(at(ia0)), c1 = a.cv1[at(ia0)], c2 = a.cv2[at(ia0)];
  for (int ia = ia0; ia <= ia1; ++ia) {
    const int c = at(ia);
    // the next step's new points, a step ahead
    const bool more = ia < ia1;
    R nr = R(0), ne = R(0), ndc = R(0), ndb = R(0), nvf = R(0), nc1 = R(0), nc2 = R(0);
    if (more) {
      nr = rho[at(ia + 3)];
      ne = en[at(ia + 3)];
      ndc = dc1[at(ia + 2)];
      ndb = db1[at(ia + 2)];
      const int cn = at(ia + 1);
      nvf = vface(cn);
      nc1 = a.cv1[cn];
      nc2 = a.cv2[cn];
    }
    // K4 at ia: from the windows, or from the source index for a ghost value
    R dmc = R(0);
    if (inside_t) {
      const bool ghost = a.per ? (ia <= 0 || ia >= na + 1) : (ia == -1 || ia >= na + 1);
      if (!ghost) {
        LimOut<R> L = limiter<R>(vf, r[0], r[1], r[2], r[3], dcw[1], dcw[0], dcw[2], dbw[0], dbw[1], R(0), R(0),
                                 dt, false);
        dmc = (L.fu + L.Di * (R(1) - L.phi)) * vf * dt * area;
      } else {
        dmc = mass_flux(ia, c);
      }
    }
    a.dm[c] = dmc;
    const bool in1 = line1 && ia >= 1 && ia <= na;
    R rn = r[1];
    if (in1) rn = qdiv(r[1] * c1 + dm_prev - dmc, c2);
    a.rho_new[c] = rn;
    R ef = R(0);
    if (line0 && ia >= 0 && ia <= na) {
      LimOut<R> L = limiter<R>(vf, e[0], e[1], e[2], e[3], dcw[1], dcw[0], dcw[2], dbw[0], dbw[1], R(0), R(0), dt,
                               false);
      const R rhou = r[1] * L.vad_p + r[2] * L.vad_m;
#if LARE_FAST
      const R dmu = fabs(dmc) * fast_rcp(area * L.dxbu * rhou);
#else
      const R dmu = fabs(dmc) / area / L.dxbu / rhou;
#endif
      ef = (L.fu + L.Di * (R(1) - dmu)) * dmc;
    }
    R eo = e[1];
    if (in1) eo = qdiv(e[1] * c1 * r[1] + ef_prev - ef, c2 * rn);
    a.energy_new[c] = eo;
    dm_prev = dmc;
    ef_prev = ef;
    r[0] = r[1]; r[1] = r[2]; r[2] = r[3]; r[3] = nr;
    e[0] = e[1]; e[1] = e[2]; e[2] = e[3]; e[3] = ne;
    dcw[0] = dcw[1]; dcw[1] = dcw[2]; dcw[2] = ndc;
    dbw[0] = dbw[1]; dbw[1] = ndb;
    vf = nvf; c1 = nc1; c2 = nc2;
  }
}

// The same for the x sweep: the lanes of a warp hold consecutive x
// positions and take their stencil neighbours (one to the left, two to the
// right) and the fluxes of the point to their left by shuffles.  A warp
// spans 32 positions and writes the kMEXOut = 28 whose stencils and left
// fluxes lie inside it; ghost values of dm (dm_x_bcs) are formed from their
// source index by direct loads.
constexpr int kMEXOut = 28;

template <class R>
__global__ void __launch_bounds__(128) k_mass_energy_x(MEArgs<R> a, int sx, int sxy, int nx) {
  const int lane = (int)threadIdx.x;                               // blockDim.x == 32: one warp per row
  const int ix = -3 + (int)blockIdx.x * kMEXOut + lane;            // lane 2 holds the first output
  const int iy = -1 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int iz = -1 + (int)blockIdx.z;
  if (iy > a.nt1 + 2) return;                                      // uniform over the warp
  const int S1 = a.S1, S2 = a.S2;
  const int xl = min(max(ix, -2), nx + 2);                         // in-box load position
  const int c = xl + sx * iy + sxy * iz;
  const bool inside_t = iy >= 0 && iy <= a.nt1 + 1 && iz >= 0 && iz <= a.nt2 + 1;
  const bool line0 = iy >= 0 && iy <= a.nt1 && iz >= 0 && iz <= a.nt2;
  const bool line1 = line0 && iy >= 1 && iz >= 1;
  const R dt = (R)a.sc[a.dt_slot];
  const R area = inside_t ? a.dbt1(iy) * a.dbt2(iz) : R(0);
  const R* __restrict__ rho = a.rho;
  const R* __restrict__ en = a.energy;
  const R* __restrict__ va = a.va;
  const R* __restrict__ dc1 = a.dc1;
  const R* __restrict__ db1 = a.db1;
  const R r0 = rho[c], e0 = en[c], dc = dc1[c], db = db1[c];
  const unsigned all = 0xffffffffu;
  const R rm = __shfl_up_sync(all, r0, 1), rp = __shfl_down_sync(all, r0, 1), rp2 = __shfl_down_sync(all, r0, 2);
  const R em = __shfl_up_sync(all, e0, 1), ep = __shfl_down_sync(all, e0, 1), ep2 = __shfl_down_sync(all, e0, 2);
  const R dcm = __shfl_up_sync(all, dc, 1), dcp = __shfl_down_sync(all, dc, 1);
  const R dbp = __shfl_down_sync(all, db, 1);
  const R v_c = (va[c] + va[c - S1] + va[c - S2] + va[c - S1 - S2]) * R(0.25);
  const int na = a.na;
  // K4 at ix: from the lane neighbours, or from the source index for a ghost
  R dmc = R(0);
  if (inside_t && lane >= 1 && lane <= 29) {
    int sa = ix;
    bool compute = true;
    if (a.per) {
      if (ix == na + 1) sa = 1;
      else if (ix == na + 2) sa = 2;
      else if (ix == -1) sa = na - 1;
      else if (ix == 0) sa = na;
    } else {
      if (ix == na + 1) sa = na;
      else if (ix == -1) sa = 0;
      else if (ix == na + 2) compute = false;
    }
    if (compute && ix >= -1 && ix <= na + 2) {
      if (sa == ix) {
        LimOut<R> L = limiter<R>(v_c, rm, r0, rp, rp2, dc, dcm, dcp, db, dbp, R(0), R(0), dt, false);
        dmc = (L.fu + L.Di * (R(1) - L.phi)) * v_c * dt * area;
      } else {
        const int q = c + (sa - ix), qm = q - 1, qp = q + 1, qp2 = q + 2;
        const R v_advect = (va[q] + va[q - S1] + va[q - S2] + va[q - S1 - S2]) * R(0.25);
        LimOut<R> L = limiter<R>(v_advect, rho[qm], rho[q], rho[qp], rho[qp2], dc1[q], dc1[qm], dc1[qp], db1[q],
                                 db1[qp], R(0), R(0), dt, false);
        dmc = (L.fu + L.Di * (R(1) - L.phi)) * v_advect * dt * area;
      }
    }
  }
  // K5's energy flux at ix (0 <= ix <= na on line0)
  R ef = R(0);
  if (line0 && ix >= 0 && ix <= na && lane >= 1 && lane <= 29) {
    LimOut<R> L = limiter<R>(v_c, em, e0, ep, ep2, dc, dcm, dcp, db, dbp, R(0), R(0), dt, false);
    const R rhou = r0 * L.vad_p + rp * L.vad_m;
#if LARE_FAST
    const R dmu = fabs(dmc) * fast_rcp(area * L.dxbu * rhou);
#else
    const R dmu = fabs(dmc) / area / L.dxbu / rhou;
#endif
    ef = (L.fu + L.Di * (R(1) - dmu)) * dmc;
  }
  const R dm_prev = __shfl_up_sync(all, dmc, 1), ef_prev = __shfl_up_sync(all, ef, 1);
  if (lane < 2 || lane > 29 || ix > na + 2) return;
  a.dm[c] = dmc;
  const bool in1 = line1 && ix >= 1 && ix <= na;
  R rn = r0;
  if (in1) rn = qdiv(r0 * a.cv1[c] + dm_prev - dmc, a.cv2[c]);
  a.rho_new[c] = rn;
  R e = e0;
  if (in1) e = qdiv(e0 * a.cv1[c] * r0 + ef_prev - ef, a.cv2[c] * rn);
  a.energy_new[c] = e;
}

LARE_END  // namespace lare

#include "remap_vm.cuh"

LARE_BEGIN

template <int A, class R>
// bmode: 1 for the first sweep of a remap (B read as stored, put in flux
// form on the way), 2 for the last (B put back from flux form), 0 between.
void remap_sweep(Run<R>& run, bool predictor, int dt_slot, int pass[3], int bmode) {
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
  const A1<R> rdba = Ar.rdb[A], rdbt1 = Ar.rdb[T1], rdbt2 = Ar.rdb[T2];
  const R pass_t1 = (R)pass[T1], pass_t2 = (R)pass[T2];
  const double* sc = run.sc;
  const bool write_cv2 = !predictor;

  // ---- K1: cv1, cv2, db1, dc1 over the whole cell box -1..n+2 (z-marching for
  // every FP32 sweep, the FP64 z sweep and the exact FP64 x sweep; per cell for
  // the other FP64 sweeps, where the marching form measured no faster)
  if (A == 2 || sizeof(R) == 4 || (A == 0 && !LARE_FAST)) {
    GeomArgs<R> ga;
    ga.vx1 = vx1;
    ga.vy1 = Ar.vy1.p;
    ga.vz1 = vz1;
    ga.cv = cv;
    ga.cv1 = cv1;
    ga.cv2 = cv2;
    ga.db1 = db1;
    ga.dc1 = dc1;
    ga.dbm[0] = Ar.dxb;
    ga.dbm[1] = Ar.dyb;
    ga.dbm[2] = Ar.dzb;
    ga.rdbm[0] = Ar.rdb[0];
    ga.rdbm[1] = Ar.rdb[1];
    ga.rdbm[2] = Ar.rdb[2];
    ga.pass_t1 = pass_t1;
    ga.pass_t2 = pass_t2;
    ga.sc = sc;
    ga.dt_slot = dt_slot;
    ga.nx = nx;
    ga.ny = ny;
    ga.nz = nz;
    ga.sx = sx;
    ga.sxy = sxy;
    ga.write_cv2 = write_cv2;
    dim3 blk(32, 4, 1);
    dim3 grd((nx + 4 + 31) / 32, (ny + 4 + 3) / 4, (nz + 4 + kGeomZ - 1) / kGeomZ);
    const int k = run.prof_begin("remap_sweep_geom_march", 0, 8, (double)(nx + 4) * (ny + 4) * (nz + 4));
    k_geom_march<A, R><<<grd, blk, 0, run.s>>>(ga);
    run.prof_end(k);
    ++run.launches;
  } else {
    LARE_BOXWH(run, 0, 2, 8, -1, nx + 2, -1, ny + 2, -1, nz + 2, [=] __device__(int ix, int iy, int iz) {
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
      R term_t1 = div_rcp(pass_t1 * dvv[T1], dbt1(pp[T1]), rdbt1(pp[T1]));
      R term_t2 = div_rcp(pass_t2 * dvv[T2], dbt2(pp[T2]), rdbt2(pp[T2]));
      R term_a = div_rcp(dvv[A], dba(pp[A]), rdba(pp[A]));
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
  }

  // ---- K2: both constrained-transport fluxes over -1..n+1
  R* const Bp[3] = {Ar.bx.p, Ar.by.p, Ar.bz.p};
  R* const f1 = Ar.f1.p;
  R* const f2 = Ar.f2.p;
  {
    BfArgs<R> ba;
    ba.va = va;
    ba.b1 = Bp[B1];
    ba.b2 = Bp[B2];
    ba.db1 = db1;
    ba.dc1 = dc1;
    ba.f1 = f1;
    ba.f2 = f2;
    ba.sc = sc;
    ba.dt_slot = dt_slot;
    ba.SA = SA;
    ba.SB1 = SB1;
    ba.SB2 = SB2;
    ba.SO1 = SO1;
    ba.SO2 = SO2;
    ba.SX = 1;
    ba.SY = A == 1 ? sxy : sx;     // the grid's second axis: z for the y sweep, y for the z sweep
    ba.na = na;
    ba.n0 = nx + 3;
    ba.n1 = (A == 1 ? nz : ny) + 3;
    ba.dbm[0] = Ar.dxb;
    ba.dbm[1] = Ar.dyb;
    ba.dbm[2] = Ar.dzb;
    ba.j1 = B1;
    ba.j2 = B2;
    ba.ax = A;
    const bool pre = bmode == 1;
    const int k = run.prof_begin(A == 0 ? "remap_sweep_bflux_x" : "remap_sweep_bflux_march", 0, 7,
                                 (double)(nx + 3) * (ny + 3) * (nz + 3));
    if (A != 0) {
      dim3 blk(32, 4, 1);
      dim3 grd((ba.n0 + 31) / 32, (ba.n1 + 3) / 4, (na + 3 + kMarch - 1) / kMarch);
      if (sizeof(R) == 8) {  // one flux per thread in FP64 (half the registers); FP32 measured the same either way
        dim3 grd1((ba.n0 + 31) / 32, (ba.n1 + 3) / 4, 2 * ((na + 3 + kMarch - 1) / kMarch));
        if (pre) {
          k_bflux_march1<R, true><<<grd1, blk, 0, run.s>>>(ba);
        } else {
          k_bflux_march1<R, false><<<grd1, blk, 0, run.s>>>(ba);
        }
      } else if (pre) {
        k_bflux_march<R, true><<<grd, blk, 0, run.s>>>(ba);
      } else {
        k_bflux_march<R, false><<<grd, blk, 0, run.s>>>(ba);
      }
    } else {
      dim3 blk(32, 4, 1);
      dim3 grd((nx + 3 + kXOut - 1) / kXOut, (ny + 3 + 3) / 4, nz + 3);
      if (pre) {
        k_bflux_x<R, true><<<grd, blk, 0, run.s>>>(ba, sx, sxy, nx, ny);
      } else {
        k_bflux_x<R, false><<<grd, blk, 0, run.s>>>(ba, sx, sxy, nx, ny);
      }
    }
    run.prof_end(k);
    ++run.launches;
  }

  // ---- K3: the four updates, each over its file's range (the first sweep
  // of a remap also puts B in flux form, the last puts it back)
  {
    R* const Ba = Bp[A];
    R* const Bb1 = Bp[B1];
    R* const Bb2 = Bp[B2];
    // the predictor keeps B as B0: its first sweep writes the B0 buffers,
    // which are then swapped in (lagran.F90:945-1062)
    const bool keep = bmode == 1 && predictor;
    R* const B0p[3] = {Ar.bx0.p, Ar.by0.p, Ar.bz0.p};
    BUpdArgs<R> gu;
    gu.f1 = f1;
    gu.f2 = f2;
    gu.Ba = Ba;
    gu.Bb1 = Bb1;
    gu.Bb2 = Bb2;
    gu.oa = keep ? B0p[A] : Ba;
    gu.ob1 = keep ? B0p[B1] : Bb1;
    gu.ob2 = keep ? B0p[B2] : Bb2;
    for (int d = 0; d < 3; ++d) {
      gu.dbm[d] = dbm[d];
      gu.rdbm[d] = Ar.rdb[d];
    }
    gu.nx = nx;
    gu.ny = ny;
    gu.nz = nz;
    gu.sx = sx;
    gu.sxy = sxy;
    gu.SA = SA;
    gu.SB1 = SB1;
    gu.SB2 = SB2;
    constexpr int kPts = sizeof(R) == 4 ? kBUpdZ32 : kBUpdZ64;
    const int e = bmode == 0 ? 2 : 5;  // points per axis: the update box 0..n+1, or the arrays' -2..n+2
    dim3 grd((nx + e + 31) / 32, (ny + e + 3) / 4, (nz + e + kPts - 1) / kPts);
    // words: B (3) read and written, the two fluxes read
    const int k = run.prof_begin("remap_sweep_bupd", 0, 8, (double)(nx + e) * (ny + e) * (nz + e));
    if (bmode == 1) {
      k_bupdate<A, kPts, 1, R><<<grd, dim3(32, 4, 1), 0, run.s>>>(gu);
    } else if (bmode == 2) {
      k_bupdate<A, kPts, 2, R><<<grd, dim3(32, 4, 1), 0, run.s>>>(gu);
    } else {
      k_bupdate<A, kPts, 0, R><<<grd, dim3(32, 4, 1), 0, run.s>>>(gu);
    }
    run.prof_end(k);
    ++run.launches;
    if (keep) {
      std::swap(Ar.bx.p, Ar.bx0.p);
      std::swap(Ar.by.p, Ar.by0.p);
      std::swap(Ar.bz.p, Ar.bz0.p);
    }
  }
  if (predictor) return;  // xremap.f90:159-162 (pass flag not reset)

  R* const rho = Ar.rho.p;        // rho1 of the reference from here on
  R* const rho_new = Ar.rho_alt.p;
  R* const energy = Ar.energy.p;
  R* const dm = Ar.dm.p;
  R* const eflux = Ar.flux.p;
  const bool per = run.p.per[A];
  const int nt1 = nn[T1], nt2 = nn[T2];

  {
    // ---- K4 + K5 + K6 in one kernel (marching along A for the y and z
    // sweeps, warp shuffles along x for the x sweep); the new energy is
    // swapped in
    MEArgs<R> me;
    me.va = va;
    me.rho = rho;
    me.rho_new = rho_new;
    me.energy = energy;
    me.energy_new = eflux;  // the energy-flux array is free in this form
    me.dm = dm;
    me.cv1 = cv1;
    me.cv2 = cv2;
    me.db1 = db1;
    me.dc1 = dc1;
    me.dbt1 = dbt1;
    me.dbt2 = dbt2;
    me.sc = sc;
    me.dt_slot = dt_slot;
    me.SA = SA;
    me.S1 = S1;
    me.S2 = S2;
    me.SY = S2;
    me.na = na;
    me.nt1 = nt1;
    me.nt2 = nt2;
    me.per = per;
    dim3 blk(32, 4, 1);
    // words: rho, energy, va, dc1, db1, cv1, cv2 read; dm, rho_new, energy written
    const int k = run.prof_begin(A == 0 ? "remap_sweep_mass_energy_x" : "remap_sweep_mass_energy_march", 0, 10,
                                 (double)(nx + 4) * (ny + 4) * (nz + 4));
    if (A == 0) {
      dim3 grd((nx + 4 + kMEXOut - 1) / kMEXOut, (ny + 4 + 3) / 4, nz + 4);
      k_mass_energy_x<R><<<grd, blk, 0, run.s>>>(me, sx, sxy, nx);
    } else {
      dim3 grd((nt1 + 4 + 31) / 32, (nt2 + 4 + 3) / 4, (na + 4 + kMEChunk - 1) / kMEChunk);
      k_mass_energy_march<R><<<grd, blk, 0, run.s>>>(me);
    }
    run.prof_end(k);
    ++run.launches;
    std::swap(Ar.energy.p, Ar.flux.p);
  }

  // ---- K7: vertex quantities.  rho_v over a -1:n+1, the rest over 0:n;
  // dm vertex averages over a -1:n.
  R* const rv = Ar.r_rho_v.p;
  R* const rv1 = Ar.r_rho_v1.p;
  R* const cv1v = Ar.cv1v.p;
  R* const cv2v = Ar.cv2v.p;
  R* const dmv = Ar.dmv.p;
  // rke off: the vertex averages are formed inside the momentum kernel, in
  // the reference's summation order (remap_vm.cuh)
  const bool fused_vm = !run.p.rke;
  if (!fused_vm) {
    int lo[3] = {0, 0, 0}, hi[3] = {nx, ny, nz};
    lo[A] = -1;
    hi[A] = na + 1;
    VertArgs<R> va7;
    va7.rho = rho;
    va7.cv1 = cv1;
    va7.cv2 = cv2;
    va7.dm = dm;
    va7.rv = rv;
    va7.rv1 = rv1;
    va7.cv1v = cv1v;
    va7.cv2v = cv2v;
    va7.dmv = dmv;
    for (int d = 0; d < 3; ++d) {
      va7.lo[d] = lo[d];
      va7.hi[d] = hi[d];
    }
    va7.na = na;
    va7.sx = sx;
    va7.sxy = sxy;
    dim3 blk(32, 4, 1);
    dim3 grd((hi[0] - lo[0] + 32) / 32, (hi[1] - lo[1] + 4) / 4, (hi[2] - lo[2] + kVertZ) / kVertZ);
    const int k = run.prof_begin("remap_sweep_vert", 0, 9,
                                 (double)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1));
    k_vert_march<A, R><<<grd, blk, 0, run.s>>>(va7);
    run.prof_end(k);
    ++run.launches;
  }

  // ---- K8 + K9: momentum fluxes (faces a -1:n, transverse 0:n) and the
  // velocity updates (0:n) in one kernel, new velocities into the q buffers
  {
    MomArgs<R> gm;
    gm.va = va;
    gm.rv = rv;
    gm.dmv = dmv;
    gm.db1 = db1;
    gm.dc1 = dc1;
    gm.v[0] = Ar.vx.p;
    gm.v[1] = Ar.vy.p;
    gm.v[2] = Ar.vz.p;
    gm.vn[0] = Ar.qx.p;
    gm.vn[1] = Ar.qy.p;
    gm.vn[2] = Ar.qz.p;
    gm.cv1v = cv1v;
    gm.cv2v = cv2v;
    gm.rv1 = rv1;
    gm.dct1 = dct1;
    gm.dct2 = dct2;
    gm.sc = sc;
    gm.dt_slot = dt_slot;
    gm.nx = nx;
    gm.ny = ny;
    gm.nz = nz;
    gm.na = na;
    gm.n3 = A == 1 ? nz : ny;
    gm.sx = sx;
    gm.sxy = sxy;
    gm.SA = SA;
    gm.S3 = A == 1 ? sxy : sx;
    const bool rke = run.p.rke != 0;
    for (int q = 0; q < 3; ++q) gm.fp[q] = rke ? Ar.rke_f[q].p : nullptr;
    // words: fused, v (3), v1, db1, dc1, rho, cv1, cv2, dm read and the new v (3) written
    const char* site = fused_vm ? (A == 0 ? "remap_sweep_vert_mom_x" : "remap_sweep_vert_mom_march")
                                : (A == 0 ? "remap_sweep_mom_x" : "remap_sweep_mom_march");
    const int k = run.prof_begin(site, 0, fused_vm ? 13 : (rke ? 17 : 14), (double)(nx + 1) * (ny + 1) * (nz + 1));
    if (fused_vm) {
      VMArgs<R> vm;
      vm.m = gm;
      vm.rho = rho;
      vm.cv1 = cv1;
      vm.cv2 = cv2;
      vm.dm = dm;
      if constexpr (A == 0) {
        dim3 grd((nx + 1 + kVMXOut - 1) / kVMXOut, (ny + 1 + 3) / 4, nz + 1);
        k_vm_x<R><<<grd, dim3(32, 4, 1), 0, run.s>>>(vm);
      } else {
        dim3 grd((nx + 1 + 31) / 32, (gm.n3 + 1 + 3) / 4, (na + 1 + kMomA - 1) / kMomA);
        k_vm_march<A, R><<<grd, dim3(32, 4, 1), 0, run.s>>>(vm);
      }
    } else if (A == 0) {
      dim3 grd((nx + 1 + 30) / 31, (ny + 1 + 3) / 4, nz + 1);
      if (rke)
        k_mom_x<R, true><<<grd, dim3(32, 4, 1), 0, run.s>>>(gm);
      else
        k_mom_x<R, false><<<grd, dim3(32, 4, 1), 0, run.s>>>(gm);
    } else {
      dim3 grd((nx + 1 + 31) / 32, (gm.n3 + 1 + 3) / 4, (na + 1 + kMomA - 1) / kMomA);
      if (rke)
        k_mom_march<R, true><<<grd, dim3(32, 4, 1), 0, run.s>>>(gm);
      else
        k_mom_march<R, false><<<grd, dim3(32, 4, 1), 0, run.s>>>(gm);
    }
    run.prof_end(k);
    ++run.launches;
  }
  if (run.p.rke) {
    // rke (xremap.f90:664-695 and siblings): the old velocities are still
    // in v (the new ones went to the q buffers), and the momentum kernel
    // above stored the three fluxes before their product with dm (faces
    // -1:n along A).  R2 forms each vertex's defect dk per component; R3
    // adds, per cell 1:n, the dk of each vertex whose update scatters into
    // it, for the components in file order and the vertices in the
    // reference's loop order, so the sums are the reference's bit for bit.
    const R* const rf0 = Ar.rke_f[0].p;
    const R* const rf1 = Ar.rke_f[1].p;
    const R* const rf2 = Ar.rke_f[2].p;
    int lo[3] = {0, 0, 0}, hi[3] = {nx, ny, nz};
    R* const dke = Ar.delta_ke.p;
    const R* const vv0 = Ar.vx.p;
    const R* const vv1 = Ar.vy.p;
    const R* const vv2 = Ar.vz.p;
    R* const dk0 = Ar.rke_dk[0].p;
    R* const dk1 = Ar.rke_dk[1].p;
    R* const dk2 = Ar.rke_dk[2].p;
    // R2: each vertex's defect once (vertices 0:n-1 along A, 0:n across)
    lo[A] = 0;
    hi[A] = na - 1;
    LARE_BOXW(run, 15, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], [=] __device__(int ix, int iy, int iz) {
      const int c = ix + sx * iy + sxy * iz;
      dk0[c] = rke_dk(vv0, rf0, dmv, rv1, cv2v, c, SA);
      dk1[c] = rke_dk(vv1, rf1, dmv, rv1, cv2v, c, SA);
      dk2[c] = rke_dk(vv2, rf2, dmv, rv1, cv2v, c, SA);
    });
    // R3: the gather
    LARE_BOXW(run, 14, 1, nx, 1, ny, 1, nz, [=] __device__(int ix, int iy, int iz) {
      const int c = ix + sx * iy + sxy * iz;
      const int b = c - SA;  // the vertex below along A; its transverse neighbours below
      const int vtx[4] = {b - S1 - S2, b - S2, b - S1, b};
      const R* const dq[3] = {dk0, dk1, dk2};
      R d = dke[c];
#pragma unroll
      for (int comp = 0; comp < 3; ++comp)
#pragma unroll
        for (int q = 0; q < 4; ++q) d = d + dq[comp][vtx[q]];
      dke[c] = d;
    });
  }
  std::swap(Ar.vx.p, Ar.qx.p);
  std::swap(Ar.vy.p, Ar.qy.p);
  std::swap(Ar.vz.p, Ar.qz.p);
  {
    R* const nv[3] = {Ar.vx.p, Ar.vy.p, Ar.vz.p};
    R* const ov[3] = {Ar.qx.p, Ar.qy.p, Ar.qz.p};
    carry_velocity(run, nv, ov);
  }

  // The new density becomes rho; the old buffer is scratch again.
  std::swap(Ar.rho.p, Ar.rho_alt.p);
  boundary_conditions(run);
  pass[A] = 0;
}

LARE_END  // namespace lare
