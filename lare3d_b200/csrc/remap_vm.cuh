// remap_vm.cuh - vertex averages fused into the momentum kernels (rke off).
//
// K7 of a sweep (xremap.f90:201-290 and the y/z mirrors) forms at each
// vertex the eight-cell sums of rho cv1, cv1, cv2 and dm, and from them
// rho_v = sum(rho cv1) / sum(cv1), cv1_v = sum(cv1) / 8, cv2_v = sum(cv2) / 8,
// dm_v = sum(dm) / 8 and rho_v1 = (rho_v cv1_v + dm_m - dm_v) / cv2_v, where
// dm_m, the dm average around the vertex below along the sweep axis, is that
// vertex's dm_v: its eight cells are summed in the same order.  K8 + K9
// read these back.  Here the momentum kernel forms them on the way, so no
// vertex array reaches memory (13 words per point instead of 9 + 14).
//
// Every sum keeps the reference's order: the four cells of the z-plane quad
// (x, y), (x+1, y), (x, y+1), (x+1, y+1) at z, then the same at z + 1, added
// left to right.  The eight cells of vertex ia are the 2 x 2 transverse
// cells of two neighbouring slices along the sweep axis, and each sweep
// interleaves the slices differently:
//   z sweep: slice z, then slice z + 1 (its running sum is carried);
//   y sweep: two cells of slice y, two of y + 1, two of y, two of y + 1 (the
//            first pair's sum and the last pair of slice y are carried);
//   x sweep: alternately slice x and slice x + 1 (the next lane's cells).
// The results are the split kernels' bit for bit.  The FP64 product build,
// not bound to the reference's rounding, sums each slice's four cells first
// and adds the two slice sums (kReassoc): fewer live values and shorter
// chains, 0.93 against 1.21 ms a step for the y and z sweeps at 256^3.
// With rke on, the kinetic-energy defect reads the vertex arrays, and the
// split kernels run instead.
#pragma once

LARE_BEGIN

// The product build's association of the eight-cell sums (two slice sums).
template <class R>
constexpr bool kReassoc = LARE_FAST && sizeof(R) == 8;

template <class R>
struct VMArgs {
  MomArgs<R> m;  // the momentum kernel's operands; rv, dmv, cv1v, cv2v, rv1 unused
  const R* rho;  // rho1 (the density before this sweep)
  const R* cv1;
  const R* cv2;
  const R* dm;
};

// The four cells of a slice at cell index b (offsets o[0..3]) for the four
// summed quantities.
template <class R>
struct SliceCells {
  R p[4], w[4], w2[4], d[4];  // rho cv1, cv1, cv2, dm
};

template <class R>
__device__ __forceinline__ SliceCells<R> slice_cells(const VMArgs<R>& g, int b, const int (&o)[4]) {
  SliceCells<R> s;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    s.w[q] = g.cv1[b + o[q]];
    s.p[q] = g.rho[b + o[q]] * s.w[q];
    s.w2[q] = g.cv2[b + o[q]];
    s.d[q] = g.dm[b + o[q]];
  }
  return s;
}

// The eight-cell sums of one vertex.
template <class R>
struct VertexSums {
  R p, w, w2, d;
};

// What a march carries of the slice below the new one: the z sweep its
// running sum (four cells), the y sweep the sum of its first pair
// (x, z), (x+1, z) and its last pair (x, z+1), (x+1, z+1).
template <class R>
struct Carry {
  R h, e2, e3;
};

template <int A, class R>
__device__ __forceinline__ Carry<R> carry_of(const R (&v)[4]) {
  Carry<R> c;
  if (A == 2 || kReassoc<R>) {
    c.h = v[0] + v[1] + v[2] + v[3];
    c.e2 = c.e3 = R(0);
  } else {
    c.h = v[0] + v[1];
    c.e2 = v[2];
    c.e3 = v[3];
  }
  return c;
}

// The vertex sum from the carried lower slice and the upper slice's cells.
// z sweep: (x,y),(x+1,y),(x,y+1),(x+1,y+1) of z, then of z+1.  y sweep
// (slice offsets 0, 1 at z, 2, 3 at z+1): (x,y,z),(x+1,y,z) of the lower
// slice, (x,y+1,z),(x+1,y+1,z) of the upper, (x,y,z+1),(x+1,y,z+1) of the
// lower, (x,y+1,z+1),(x+1,y+1,z+1) of the upper.
template <int A, class R>
__device__ __forceinline__ R vertex_sum(const Carry<R>& lo, const R (&up)[4]) {
  if (kReassoc<R>) return lo.h + (up[0] + up[1] + up[2] + up[3]);
  if (A == 2) return lo.h + up[0] + up[1] + up[2] + up[3];
  return lo.h + up[0] + up[1] + lo.e2 + lo.e3 + up[2] + up[3];
}

template <int A, class R>
__device__ __forceinline__ VertexSums<R> advance(Carry<R> (&cr)[4], const SliceCells<R>& s) {
  VertexSums<R> v;
  v.p = vertex_sum<A>(cr[0], s.p);
  v.w = vertex_sum<A>(cr[1], s.w);
  v.w2 = vertex_sum<A>(cr[2], s.w2);
  v.d = vertex_sum<A>(cr[3], s.d);
  cr[0] = carry_of<A>(s.p);
  cr[1] = carry_of<A>(s.w);
  cr[2] = carry_of<A>(s.w2);
  cr[3] = carry_of<A>(s.d);
  return v;
}

template <int A, class R>
__global__ void __launch_bounds__(128, sizeof(R) == 8 ? 4 : 6) k_vm_march(VMArgs<R> a) {
  const MomArgs<R>& g = a.m;
  const int t0 = (int)(blockIdx.x * blockDim.x + threadIdx.x);  // x, 0..nx
  const int t1 = (int)(blockIdx.y * blockDim.y + threadIdx.y);  // the third axis, 0..n3
  if (t0 > g.nx || t1 > g.n3) return;
  const int ia0 = (int)blockIdx.z * kMomA;
  const int ia1 = min(ia0 + kMomA - 1, g.na);
  const R dt = (R)g.sc[g.dt_slot];
  const int SA = g.SA, S3 = g.S3;
  const int o[4] = {0, 1, S3, 1 + S3};
  const R area = g.dct1(t0) * g.dct2(t1);
  const R eighth = R(0.125);
  int c = t0 + t1 * S3 + (ia0 - 1) * SA;  // vertex (and cell) index of face ia0 - 1
  // slices ia0 - 1, ia0, ia0 + 1: the sums of vertices ia0 - 1 (vlo) and
  // ia0 (vc), and slice ia0 + 1 carried
  Carry<R> cr[4];
  {
    const SliceCells<R> s = slice_cells(a, c, o);
    cr[0] = carry_of<A>(s.p);
    cr[1] = carry_of<A>(s.w);
    cr[2] = carry_of<A>(s.w2);
    cr[3] = carry_of<A>(s.d);
  }
  VertexSums<R> vlo = advance<A>(cr, slice_cells(a, c + SA, o));
  VertexSums<R> vc = advance<A>(cr, slice_cells(a, c + 2 * SA, o));
  R w[3][4];
#pragma unroll
  for (int comp = 0; comp < 3; ++comp)
#pragma unroll
    for (int q = 0; q < 4; ++q) w[comp][q] = g.v[comp][c + (q - 1) * SA];
  R va0 = g.va[c], va1 = g.va[c + SA];
  R dbw0 = g.db1[c], dbw1 = g.db1[c + SA], dbw2 = g.db1[c + 2 * SA], dcw0 = g.dc1[c], dcw1 = g.dc1[c + SA];
  // face ia0 - 1: rho_v at its two vertices, dm_v at the lower one
  R rvc = qdiv(vlo.p, vlo.w);
  R rvn = qdiv(vc.p, vc.w);
  R Fm[3], fpre[3];
  mom_flux_vals<R, false>(area, va0, va1, rvc, rvn, vlo.d * eighth, dbw0, dbw1, dbw2, dcw0, dcw1, w, dt, Fm, fpre);
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
    // slice ia + 2 gives vertex ia + 1's sums
    const VertexSums<R> vn = advance<A>(cr, slice_cells(a, c + 2 * SA, o));
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
    // vertex ia
    rvc = rvn;
    rvn = qdiv(vn.p, vn.w);
    const R dmv = vc.d * eighth;
    const R cc1 = vc.w * eighth, cc2 = vc.w2 * eighth;
    const R dmm = vlo.d * eighth;
    const R rv1 = qdiv(rvc * cc1 + dmm - dmv, cc2);
    R F[3];
    mom_flux_vals<R, false>(area, va0, va1, rvc, rvn, dmv, dbw0, dbw1, dbw2, dcw0, dcw1, w, dt, F, fpre);
    const R den = dv_of(cc2 * rv1);
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      g.vn[comp][c] = dv_div(rvc * w[comp][1] * cc1 + Fm[comp] - F[comp], den);
      Fm[comp] = F[comp];
    }
    vlo = vc;
    vc = vn;
  }
}

// The same for the x sweep: the lanes of a warp hold consecutive x
// positions.  Each lane loads the slice of cells at its x (y, y+1 at z,
// then at z+1) and takes the next lane's by shuffles, alternating the two
// in the reference's order; dm_m is the dm average of the lane below and
// rho_v of the next vertex is the next lane's.  A lane's face flux needs the
// two lanes above it, and its update the flux of the lane below, so a warp
// updates the kVMXOut = 29 vertices of lanes 1..29.
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
  // this lane's slice: (y, z), (y+1, z), (y, z+1), (y+1, z+1) at x
  const int o[4] = {0, sx, sxy, sx + sxy};
  const SliceCells<R> s = slice_cells(a, c, o);
  // vertex x: (x,y,z),(x+1,y,z),(x,y+1,z),(x+1,y+1,z), then the same at z+1
  // (the product build: this slice's sum plus the next lane's)
  auto vsum = [&](const R (&v)[4]) {
    if (kReassoc<R>) {
      const R t = v[0] + v[1] + v[2] + v[3];
      return t + __shfl_down_sync(all, t, 1);
    }
    R t = v[0];
    t = t + __shfl_down_sync(all, v[0], 1);
    t = t + v[1];
    t = t + __shfl_down_sync(all, v[1], 1);
    t = t + v[2];
    t = t + __shfl_down_sync(all, v[2], 1);
    t = t + v[3];
    return t + __shfl_down_sync(all, v[3], 1);
  };
  const R sp = vsum(s.p), sw = vsum(s.w), sw2 = vsum(s.w2), sd = vsum(s.d);
  const R rvc = qdiv(sp, sw);                                 // vertex x
  const R rvn = __shfl_down_sync(all, rvc, 1);                // vertex x + 1
  const R dmv = sd * eighth;
  const R dmm = __shfl_up_sync(all, dmv, 1);                  // vertex x - 1
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
  const R cc1 = sw * eighth, cc2 = sw2 * eighth;
  const R rv1 = qdiv(rvc * cc1 + dmm - dmv, cc2);
  const R den = dv_of(cc2 * rv1);
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) g.vn[comp][c] = dv_div(rvc * w[comp][1] * cc1 + Fm[comp] - F[comp], den);
}

LARE_END  // namespace lare
