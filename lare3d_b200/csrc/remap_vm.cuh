// remap_vm.cuh - vertex averages fused into the momentum kernels (FP64
// product build, rke off).
//
// K7 of a sweep (xremap.f90:201-290 and the y/z mirrors) forms at each
// vertex the eight-cell averages rho_v = sum(rho cv1) / sum(cv1),
// cv1_v = sum(cv1) / 8, cv2_v = sum(cv2) / 8, dm_v = sum(dm) / 8 and
// rho_v1 = (rho_v cv1_v + dm_v(below) - dm_v) / cv2_v, and K8 + K9 read them
// back.  Here the march along the sweep axis forms them on the way: the
// eight cells of vertex ia are the 2 x 2 transverse cells of the slices ia
// and ia + 1 along the axis, so each step loads one new slice (rho, cv1,
// cv2, dm at four cells), reduces it to four slice sums, and carries the
// sums of the slices below.  The vertex arrays never reach memory (12 words
// per point instead of 9 + 14).  The eight-cell sums become two four-cell
// sums added, a different association than the reference's left-to-right
// sum, so this form serves the builds that are not bound to the
// reference's rounding: the FP64 product build.  The exact build keeps
// k_vert_march and k_mom_march, and so does the FP32 form, whose error bar
// on the strongest shocks needs the reference's order.  With rke on, the
// vertex arrays are needed by the kinetic energy defect and the split form
// is used as well.
#pragma once

LARE_BEGIN

template <class R>
struct VMArgs {
  MomArgs<R> m;  // the momentum march's operands; rv, dmv, cv1v, cv2v, rv1 unused
  const R* rho;  // rho1 (the density before this sweep)
  const R* cv1;
  const R* cv2;
  const R* dm;
};

// slice sums of the 2 x 2 transverse cells at cell index b (offsets 0, 1, S3, 1 + S3)
template <class R>
struct Slice {
  R p, w, w2, d;  // sum(rho cv1), sum(cv1), sum(cv2), sum(dm)
};

template <class R>
__device__ __forceinline__ Slice<R> slice_sums(const VMArgs<R>& g, int b, int S3) {
  const int o[4] = {0, 1, S3, 1 + S3};
  R c1[4], r[4], c2[4], d[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    c1[q] = g.cv1[b + o[q]];
    r[q] = g.rho[b + o[q]];
    c2[q] = g.cv2[b + o[q]];
    d[q] = g.dm[b + o[q]];
  }
  Slice<R> s;
  s.p = r[0] * c1[0] + r[1] * c1[1] + r[2] * c1[2] + r[3] * c1[3];
  s.w = c1[0] + c1[1] + c1[2] + c1[3];
  s.w2 = c2[0] + c2[1] + c2[2] + c2[3];
  s.d = d[0] + d[1] + d[2] + d[3];
  return s;
}

template <class R>
__global__ void __launch_bounds__(128, sizeof(R) == 8 ? 4 : 8) k_vm_march(VMArgs<R> a) {
  const MomArgs<R>& g = a.m;
  const int t0 = (int)(blockIdx.x * blockDim.x + threadIdx.x);  // x, 0..nx
  const int t1 = (int)(blockIdx.y * blockDim.y + threadIdx.y);  // the third axis, 0..n3
  if (t0 > g.nx || t1 > g.n3) return;
  const int ia0 = (int)blockIdx.z * kMomA;
  const int ia1 = min(ia0 + kMomA - 1, g.na);
  const R dt = (R)g.sc[g.dt_slot];
  const int SA = g.SA, S3 = g.S3;
  const R area = g.dct1(t0) * g.dct2(t1);
  const R eighth = R(0.125);
  int c = t0 + t1 * S3 + (ia0 - 1) * SA;  // vertex (and cell) index of face ia0 - 1
  // slices ia0 - 1, ia0, ia0 + 1
  Slice<R> sm = slice_sums(a, c, S3), s0 = slice_sums(a, c + SA, S3), sp = slice_sums(a, c + 2 * SA, S3);
  R w[3][4];
#pragma unroll
  for (int comp = 0; comp < 3; ++comp)
#pragma unroll
    for (int q = 0; q < 4; ++q) w[comp][q] = g.v[comp][c + (q - 1) * SA];
  R va0 = g.va[c], va1 = g.va[c + SA];
  R dbw0 = g.db1[c], dbw1 = g.db1[c + SA], dbw2 = g.db1[c + 2 * SA], dcw0 = g.dc1[c], dcw1 = g.dc1[c + SA];
  // face ia0 - 1: rho_v at its two vertices, dm_v at the lower one
  R rvc = qdiv(sm.p + s0.p, sm.w + s0.w);
  R rvn = qdiv(s0.p + sp.p, s0.w + sp.w);
  R Fm[3], fpre[3];
  mom_flux_vals<R, false>(area, va0, va1, rvc, rvn, (sm.d + s0.d) * eighth, dbw0, dbw1, dbw2, dcw0, dcw1, w, dt, Fm,
                          fpre);
  // the loads of the next face, a step ahead
  struct Next {
    R w[3], va, db, dc;
  };
  auto fetch = [&](int q) {
    Next n;
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) n.w[comp] = g.v[comp][q + 2 * SA];
    n.va = g.va[q + SA];
    n.db = g.db1[q + 2 * SA];
    n.dc = g.dc1[q + SA];
    return n;
  };
  Next nx = fetch(c + SA);
  for (int ia = ia0; ia <= ia1; ++ia) {
    c += SA;
    const Next cur = nx;
    if (ia < ia1) nx = fetch(c + SA);
    // slice ia + 2: vertex ia + 1's upper cells
    const Slice<R> s2 = slice_sums(a, c + 2 * SA, S3);
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      w[comp][0] = w[comp][1];
      w[comp][1] = w[comp][2];
      w[comp][2] = w[comp][3];
      w[comp][3] = cur.w[comp];
    }
    va0 = va1;
    va1 = cur.va;
    dbw0 = dbw1;
    dbw1 = dbw2;
    dbw2 = cur.db;
    dcw0 = dcw1;
    dcw1 = cur.dc;
    // vertex ia: slices ia (s0) and ia + 1 (sp); ia - 1 (sm) for the dm below
    rvc = rvn;
    rvn = qdiv(sp.p + s2.p, sp.w + s2.w);
    const R dmv = (s0.d + sp.d) * eighth;
    const R cc1 = (s0.w + sp.w) * eighth, cc2 = (s0.w2 + sp.w2) * eighth;
    const R dmm = (sm.d + s0.d) * eighth;
    const R rv1 = qdiv(rvc * cc1 + dmm - dmv, cc2);
    R F[3];
    mom_flux_vals<R, false>(area, va0, va1, rvc, rvn, dmv, dbw0, dbw1, dbw2, dcw0, dcw1, w, dt, F, fpre);
    const R den = dv_of(cc2 * rv1);
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      g.vn[comp][c] = dv_div(rvc * w[comp][1] * cc1 + Fm[comp] - F[comp], den);
      Fm[comp] = F[comp];
    }
    sm = s0;
    s0 = sp;
    sp = s2;
  }
}

// The same for the x sweep: the lanes of a warp hold consecutive x
// positions.  Each lane reduces the slice of cells at its x (the 2 x 2 cells
// in y and z) and takes the slices of the lanes beside it by shuffles: its
// vertex averages from its own slice and the next, the dm average below
// from the previous, the density of the next vertex from the next lane.  A
// lane's face flux needs the two lanes above it, and its update the flux of
// the lane below, so a warp updates the kVMXOut = 29 vertices of lanes 1..29.
constexpr int kVMXOut = 29;

template <class R>
__global__ void __launch_bounds__(128) k_vm_x(VMArgs<R> a) {
  const MomArgs<R>& g = a.m;
  const int lane = (int)threadIdx.x;                          // blockDim.x == 32: one warp per row
  const int ix = -1 + (int)blockIdx.x * kVMXOut + lane;       // vertex / face x position
  const int iy = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int iz = (int)blockIdx.z;
  if (iy > g.ny) return;                                      // uniform over the warp
  const int sx = g.sx, sxy = g.sxy;
  const int c = min(ix, g.nx + 2) + sx * iy + sxy * iz;       // lanes past n + 2 load n + 2 (unused)
  const R dt = (R)g.sc[g.dt_slot];
  const R eighth = R(0.125);
  const unsigned all = 0xffffffffu;
  // this lane's slice: cells (x, y..y+1, z..z+1)
  const int o[4] = {0, sx, sxy, sx + sxy};
  R p = R(0), wv = R(0), w2 = R(0), d = R(0);
  {
    R c1[4], r[4], c2[4], m[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      c1[q] = a.cv1[c + o[q]];
      r[q] = a.rho[c + o[q]];
      c2[q] = a.cv2[c + o[q]];
      m[q] = a.dm[c + o[q]];
    }
    p = r[0] * c1[0] + r[1] * c1[1] + r[2] * c1[2] + r[3] * c1[3];
    wv = c1[0] + c1[1] + c1[2] + c1[3];
    w2 = c2[0] + c2[1] + c2[2] + c2[3];
    d = m[0] + m[1] + m[2] + m[3];
  }
  const R p1 = __shfl_down_sync(all, p, 1), wv1 = __shfl_down_sync(all, wv, 1);
  const R w21 = __shfl_down_sync(all, w2, 1), d1 = __shfl_down_sync(all, d, 1);
  const R dlo = __shfl_up_sync(all, d, 1);
  const R rvc = qdiv(p + p1, wv + wv1);                       // vertex x
  const R rvn = __shfl_down_sync(all, rvc, 1);                // vertex x + 1
  const R dmv = (d + d1) * eighth;
  // the face flux between vertices x and x + 1 (faces -1..n)
  R w[3][4];
#pragma unroll
  for (int comp = 0; comp < 3; ++comp)
#pragma unroll
    for (int q = 0; q < 4; ++q) w[comp][q] = g.v[comp][c + (q - 1)];
  R F[3], fpre[3];
  mom_flux_vals<R, false>(g.dct1(iy) * g.dct2(iz), g.va[c], g.va[c + 1], rvc, rvn, dmv, g.db1[c], g.db1[c + 1],
                          g.db1[c + 2], g.dc1[c], g.dc1[c + 1], w, dt, F, fpre);
  R Fm[3];
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) Fm[comp] = __shfl_up_sync(all, F[comp], 1);
  if (lane < 1 || lane > kVMXOut || ix < 0 || ix > g.nx) return;
  const R cc1 = (wv + wv1) * eighth, cc2 = (w2 + w21) * eighth, dmm = (dlo + d) * eighth;
  const R rv1 = qdiv(rvc * cc1 + dmm - dmv, cc2);
  const R den = dv_of(cc2 * rv1);
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) g.vn[comp][c] = dv_div(rvc * w[comp][1] * cc1 + Fm[comp] - F[comp], den);
}

LARE_END  // namespace lare
