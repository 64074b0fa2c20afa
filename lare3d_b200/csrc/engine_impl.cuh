// engine_impl.cuh - EngineT<R>: allocation, transfers and the C-ABI verbs
// of one device context, over the routines of engine.cuh.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "engine.cuh"
#include "engine_base.h"

LARE_BEGIN

// Fortran bounds of each named array (mpi_routines.F90:295-334,
// lagran.F90:56-81, xremap.f90:42-54, conduct.f90:41,319-321).
struct FieldDesc {
  int lo[3], hi[3];
};

// Scatter a Fortran-bounded array into the padded box, flagging any
// non-finite input value in *bad.
template <class R>
__global__ void k_scatter(const double* __restrict__ src, R* __restrict__ dst0, int lo0, int lo1, int lo2, int e0,
                          int e1, int e2, int sx, int sxy, int* bad) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)e0 * e1 * e2;
  if (t >= n) return;
  int i = (int)(t % e0);
  long long r = t / e0;
  int j = (int)(r % e1);
  int k = (int)(r / e1);
  double v = src[t];
  if (!isfinite(v)) atomicOr(bad, 1);
  dst0[(lo0 + i) + (long long)sx * (lo1 + j) + (long long)sxy * (lo2 + k)] = (R)v;
}

template <class R>
__global__ void k_gather(const R* __restrict__ src0, double* __restrict__ dst, int lo0, int lo1, int lo2, int e0,
                         int e1, int e2, int sx, int sxy) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)e0 * e1 * e2;
  if (t >= n) return;
  int i = (int)(t % e0);
  long long r = t / e0;
  int j = (int)(r % e1);
  int k = (int)(r / e1);
  dst[t] = (double)src0[(lo0 + i) + (long long)sx * (lo1 + j) + (long long)sxy * (lo2 + k)];
}

template <class R>
__global__ void k_fill(R* p, size_t n, R v) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) p[t] = v;
}

template <class R>
class EngineT : public EngineBase {
 public:
  Run<R> run;
  std::map<std::string, std::pair<A3<R>*, FieldDesc>> fields;
  double* staging = nullptr;   // device, one array of doubles
  int* dflag = nullptr;        // device non-finite flag for uploads
  double* metric_stage = nullptr;
  R* metrics_dev = nullptr;

  ~EngineT() override {
    if (run.s) cudaStreamSynchronize(run.s);
    for (void* p : run.allocations) cudaFree(p);
    if (run.host_sc) cudaFreeHost(run.host_sc);
    if (run.s) cudaStreamDestroy(run.s);
    if (run.s_body) cudaStreamDestroy(run.s_body);
  }

  int fail(int code, const std::string& m) {
    run.err = m;
    return code;
  }
  int cuda_check(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(LARE_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
    return LARE_OK;
  }

  template <class T>
  T* dalloc(size_t n, std::string& err) {
    void* p = nullptr;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) {
      err = "cudaMalloc failed";
      return nullptr;
    }
    run.allocations.push_back(p);
    return (T*)p;
  }

  static GDim gdim(int stag, int n, bool mpi, bool user_min, bool user_max, bool per) {
    GDim g;
    g.lo = stag == ST_C ? -1 : -2;
    g.hi = n + 2;
    g.nw = 0;
    auto w = [&](int idx, int src) {
      g.widx[g.nw] = idx;
      g.wsrc[g.nw] = src;
      ++g.nw;
    };
    int a = g.lo, b = g.hi;
    if (mpi && per) {
      if (stag == ST_C) { w(n + 1, 1); w(n + 2, 2); w(-1, n - 1); w(0, n); a = 1; b = n; }
      else if (stag == ST_N) { w(n, 0); w(n + 1, 1); w(n + 2, 2); w(-2, n - 2); w(-1, n - 1); a = 0; b = n - 1; }
      else { w(n + 1, 1); w(n + 2, 2); w(-2, n - 2); w(-1, n - 1); w(0, n); a = 1; b = n; }
    }
    if (!per) {
      if (user_min) {
        if (stag == ST_C) { w(0, 1); w(-1, 2); a = 1; }
        else if (stag == ST_N) { w(-2, INT_MIN); w(-1, INT_MIN); w(0, INT_MIN); a = 1; }
        else { w(-1, 1); w(-2, 2); a = 0; }
      }
      if (user_max) {
        if (stag == ST_C) { w(n + 1, n); w(n + 2, n - 1); b = n; }
        else if (stag == ST_N) { w(n, INT_MIN); w(n + 1, INT_MIN); w(n + 2, INT_MIN); b = n - 1; }
        else { w(n + 1, n - 1); w(n + 2, n - 2); b = n; }
      }
    }
    g.a = a;
    g.b = b;
    return g;
  }

  GSpec spec(const int stag[3], bool mpi, bool user, int only_dim = -1) {
    GSpec s;
    for (int d = 0; d < 3; ++d) {
      bool active = only_dim < 0 || only_dim == d;
      bool per = run.p.per[d];
      bool umin = user && !per && run.p.bc[d][0] == LARE_BC_USER;
      bool umax = user && !per && run.p.bc[d][1] == LARE_BC_USER;
      s.d[d] = gdim(stag[d], run.n[d], active && mpi, active && umin, active && umax, per);
      if (!active) {  // nothing written in this dimension
        s.d[d].nw = 0;
        s.d[d].a = s.d[d].lo;
        s.d[d].b = s.d[d].hi;
      }
    }
    auto ext = [](const GDim& g) { return (long long)(g.hi - g.lo + 1); };
    auto inn = [](const GDim& g) { return (long long)(g.b - g.a + 1); };
    s.c0 = (long long)s.d[0].nw * ext(s.d[1]) * ext(s.d[2]);
    s.c1 = inn(s.d[0]) * (long long)s.d[1].nw * ext(s.d[2]);
    s.c2 = inn(s.d[0]) * inn(s.d[1]) * (long long)s.d[2].nw;
    return s;
  }

  int init(const lare_params* prm, int nx, int ny, int nz, const double* const* metrics6, std::string& err) {
    Par& p = run.p;
    p.gamma = prm->gamma; p.visc1 = prm->visc1; p.visc2 = prm->visc2;
    p.eta_background = prm->eta_background; p.eta0 = prm->eta0; p.j_max = prm->j_max;
    p.kappa_0 = prm->kappa_0; p.flux_limiter = prm->flux_limiter; p.ionise_pot = prm->ionise_pot;
    p.xi_n = prm->xi_n; p.va_max = prm->va_max; p.dt_multiplier = prm->dt_multiplier;
    p.dt_from_restart = prm->dt_from_restart; p.kappa_perp_ratio = prm->kappa_perp_ratio;
    p.resistive_mhd = prm->resistive_mhd; p.conduction = prm->conduction;
    p.heat_flux_limiter = prm->heat_flux_limiter; p.use_viscous_damping = prm->use_viscous_damping;
    p.boris = prm->boris; p.restart = prm->restart;
    p.eos_number = prm->eos_number == 0 ? LARE_EOS_IDEAL : prm->eos_number;
    p.cowling_resistivity = prm->cowling_resistivity;
    p.f_bar = prm->f_bar; p.t_bar = prm->t_bar; p.r_bar = prm->r_bar; p.tr = prm->tr; p.eta_bar = prm->eta_bar;
    p.radiation = prm->radiation;
    p.rke = prm->rke;
    p.cooling_term = prm->cooling_term;
    p.alpha_av = prm->alpha_av;
    p.coronal_heating = prm->coronal_heating;
    p.temp_norm = prm->temp_norm; p.time_norm = prm->time_norm; p.rho_norm = prm->rho_norm; p.mf = prm->mf;
    run.pip = p.eos_number != LARE_EOS_IDEAL;
    run.cowling = p.cowling_resistivity != 0;
    int bcs[6] = {prm->xbc_min, prm->xbc_max, prm->ybc_min, prm->ybc_max, prm->zbc_min, prm->zbc_max};
    for (int d = 0; d < 3; ++d) {
      p.bc[d][0] = bcs[2 * d];
      p.bc[d][1] = bcs[2 * d + 1];
      p.per[d] = bcs[2 * d] == LARE_BC_PERIODIC && bcs[2 * d + 1] == LARE_BC_PERIODIC;
    }
    run.any_open = false;
    for (int q = 0; q < 6; ++q) run.any_open = run.any_open || bcs[q] == LARE_BC_OPEN;
    run.n[0] = nx; run.n[1] = ny; run.n[2] = nz;
    run.sx = ((nx + 5) + 3) / 4 * 4;
    int sy = ny + 5, sz = nz + 5;
    long long sxy = (long long)run.sx * sy;
    long long elems = sxy * sz;
    if (elems >= (1LL << 31)) { err = "grid too large for 32-bit indexing"; return LARE_EINVAL; }
    run.sxy = (int)sxy;
    run.elems = (size_t)elems;
    const long long off = 2 + 2LL * run.sx + 2LL * sxy;
    if (cudaStreamCreateWithFlags(&run.s, cudaStreamNonBlocking) != cudaSuccess) { err = "stream"; return LARE_ECUDA; }
    // kernels with more than the default 48 KiB of dynamic shared memory
    if (cudaFuncSetAttribute(k_lp4_tile<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lp4_smem_bytes<R>()) !=
        cudaSuccess) {
      err = "shared memory attribute";
      return LARE_ECUDA;
    }

    std::vector<A3<R>*> all = {
        &run.a.rho, &run.a.energy, &run.a.temperature, &run.a.eta, &run.a.cv, &run.a.cv1, &run.a.p_visc,
        &run.a.visc_dep, &run.a.ohmic_dep, &run.a.gamma_boris, &run.a.vx, &run.a.vy, &run.a.vz, &run.a.vx1,
        &run.a.vy1, &run.a.vz1, &run.a.visc3, &run.a.bx, &run.a.by, &run.a.bz, &run.a.bx0, &run.a.by0,
        &run.a.bz0, &run.a.bx1, &run.a.by1, &run.a.bz1, &run.a.alpha1, &run.a.alpha2, &run.a.alpha3,
        &run.a.visc_heat, &run.a.pressure, &run.a.rho_v, &run.a.cv_v, &run.a.flux_x, &run.a.flux_y,
        &run.a.flux_z, &run.a.curlb, &run.a.fx_visc, &run.a.fy_visc, &run.a.fz_visc, &run.a.qx, &run.a.qy,
        &run.a.qz, &run.a.energy0, &run.a.cs, &run.a.cs_v, &run.a.db1, &run.a.dc1, &run.a.r_rho_v,
        &run.a.r_rho_v1, &run.a.rho1, &run.a.dm, &run.a.cv2, &run.a.flux, &run.a.f1, &run.a.f2,
        &run.a.rho_alt, &run.a.cv1v, &run.a.cv2v, &run.a.dmv, &run.a.mfx, &run.a.mfy, &run.a.mfz};
    if (p.conduction) {
      for (A3<R>* x : {&run.a.larsen, &run.a.Y1, &run.a.Y2, &run.a.Y3, &run.a.Lc_Y0})
        all.push_back(x);
      for (int q = 0; q < 9; ++q) all.push_back(&run.a.kf[q]);
    } else {
      // conduct_heat may still be called on its own; allocate lazily there.
    }
    if (run.pip || run.cowling) all.push_back(&run.a.xi);
    if (run.cowling) all.push_back(&run.a.eta_perp);
    if (p.radiation) all.push_back(&run.a.erad);
    if (p.rke)
      for (A3<R>* x : {&run.a.delta_ke, &run.a.rke_f[0], &run.a.rke_f[1], &run.a.rke_f[2], &run.a.rke_dk[0],
                       &run.a.rke_dk[1], &run.a.rke_dk[2]})
        all.push_back(x);
    if (p.cooling_term)
      for (A3<R>* x : {&run.a.cool_term_v, &run.a.cool_term_b}) all.push_back(x);
    if (p.coronal_heating) all.push_back(&run.a.heat_in);
    for (A3<R>* x : all) {
      R* base = dalloc<R>(run.elems, err);
      if (!base) return LARE_ENOMEM;
      x->p = base + off;
      x->sx = run.sx;
      x->sxy = run.sxy;
      fill(*x, R(0));
    }
    fill(run.a.gamma_boris, R(1));
    if (run.a.xi.p) fill(run.a.xi, (R)p.xi_n);  // the constant until neutral_fraction runs
    run.sc = dalloc<double>(SC_NSLOTS, err);
    run.us = dalloc<unsigned long long>(U_NSLOTS, err);
    size_t nb = (size_t)((nx + 5 + 63) / 64 + 1) * ((ny + 5 + 3) / 4 + 1) * (nz + 6);
    run.partial_cap = nb * 4;
    run.partial = dalloc<double>(run.partial_cap, err);
    staging = dalloc<double>(run.elems, err);
    dflag = dalloc<int>(1, err);
    if (!run.sc || !run.us || !run.partial || !staging || !dflag) return LARE_ENOMEM;
    cudaMemsetAsync(run.sc, 0, SC_NSLOTS * sizeof(double), run.s);
    if (cudaMallocHost(&run.host_sc, SC_NSLOTS * sizeof(double)) != cudaSuccess) { err = "pinned"; return LARE_ENOMEM; }

    // 1-D metrics: dxb(-1:n+2), dxc(-1:n+1) per axis, grav(-1:nz+2).
    int nn[3] = {nx, ny, nz};
    size_t mlen = 0;
    for (int d = 0; d < 3; ++d) mlen += (size_t)(nn[d] + 6) * 5;
    mlen += nz + 6;
    metrics_dev = dalloc<R>(mlen, err);
    if (!metrics_dev) return LARE_ENOMEM;
    std::vector<R> hm(mlen, R(0));
    A1<R>* db[3] = {&run.a.dxb, &run.a.dyb, &run.a.dzb};
    A1<R>* dc[3] = {&run.a.dxc, &run.a.dyc, &run.a.dzc};
    size_t pos = 0;
    for (int d = 0; d < 3; ++d) {
      // dxb stored from index -2 (one pad element) so p points at index 0.
      for (int i = -1; i <= nn[d] + 2; ++i) hm[pos + 2 + i] = (R)metrics6[2 * d][i + 1];
      db[d]->p = metrics_dev + pos + 2;
      pos += nn[d] + 6;
      for (int i = -1; i <= nn[d] + 1; ++i) hm[pos + 2 + i] = (R)metrics6[2 * d + 1][i + 1];
      dc[d]->p = metrics_dev + pos + 2;
      pos += nn[d] + 6;
      // reciprocals used by conduction (computed in double, then rounded)
      for (int i = -1; i <= nn[d] + 2; ++i) hm[pos + 2 + i] = (R)(1.0 / metrics6[2 * d][i + 1]);
      run.a.rdb[d].p = metrics_dev + pos + 2;
      pos += nn[d] + 6;
      for (int i = -1; i <= nn[d] + 1; ++i) hm[pos + 2 + i] = (R)(1.0 / metrics6[2 * d + 1][i + 1]);
      run.a.rdc[d].p = metrics_dev + pos + 2;
      pos += nn[d] + 6;
      for (int i = 0; i <= nn[d] + 1; ++i)
        hm[pos + 2 + i] = (R)(1.0 / (metrics6[2 * d + 1][i + 1] + metrics6[2 * d + 1][i]));
      run.a.rdc2[d].p = metrics_dev + pos + 2;
      pos += nn[d] + 6;
    }
    run.a.grav.p = metrics_dev + pos + 2;
    cudaMemcpy(metrics_dev, hm.data(), mlen * sizeof(R), cudaMemcpyHostToDevice);
    // cv = dxb * dyb * dzb over -1:n+2 (setup.F90:239-245)
    auto cv = run.a.cv;
    auto dxb = run.a.dxb, dyb = run.a.dyb, dzb = run.a.dzb;
    LARE_BOX(run, -1, nx + 2, -1, ny + 2, -1, nz + 2,
             [=] __device__(int i, int j, int k) { cv(i, j, k) = dxb(i) * dyb(j) * dzb(k); });

    // Ghost-fill specifications (boundary.f90, mpiboundary.f90).
    const int sc3[3] = {ST_C, ST_C, ST_C}, sn3[3] = {ST_N, ST_N, ST_N};
    const int sbx[3] = {ST_F, ST_C, ST_C}, sby[3] = {ST_C, ST_F, ST_C}, sbz[3] = {ST_C, ST_C, ST_F};
    run.g_cell = spec(sc3, true, true);
    run.g_node = spec(sn3, true, true);
    run.g_bx = spec(sbx, true, true);
    run.g_by = spec(sby, true, true);
    run.g_bz = spec(sbz, true, true);
    run.g_cell_mpi = spec(sc3, true, false);
    run.g_cell_user = spec(sc3, false, true);
    for (int d = 0; d < 3; ++d) run.g_dm[d] = spec(sc3, true, false, d);
    // the fill kernels index a job's points in 32 bits
    for (const GSpec* g : {&run.g_cell, &run.g_node, &run.g_bx, &run.g_by, &run.g_bz, &run.g_cell_mpi,
                           &run.g_cell_user, &run.g_dm[0], &run.g_dm[1], &run.g_dm[2]})
      if (g->c0 + g->c1 + g->c2 >= (1LL << 31)) return fail(LARE_EINVAL, "grid too large for the ghost fills");

    auto add = [&](const char* name, A3<R>* a, int l0, int h0, int l1, int h1, int l2, int h2) {
      FieldDesc f{{l0, l1, l2}, {h0, h1, h2}};
      fields[name] = {a, f};
    };
    const int X = nx, Y = ny, Z = nz;
    for (auto& kv : std::vector<std::pair<const char*, A3<R>*>>{
             {"rho", &run.a.rho}, {"energy", &run.a.energy}, {"temperature", &run.a.temperature},
             {"eta", &run.a.eta}, {"cv", &run.a.cv}, {"cv1", &run.a.cv1}, {"p_visc", &run.a.p_visc},
             {"visc_dep", &run.a.visc_dep}, {"ohmic_dep", &run.a.ohmic_dep}, {"gamma_boris", &run.a.gamma_boris},
             {"bx1", &run.a.bx1}, {"by1", &run.a.by1}, {"bz1", &run.a.bz1}, {"pressure", &run.a.pressure}}) {
      add(kv.first, kv.second, -1, X + 2, -1, Y + 2, -1, Z + 2);
    }
    for (auto& kv : std::vector<std::pair<const char*, A3<R>*>>{{"vx", &run.a.vx}, {"vy", &run.a.vy},
                                                                 {"vz", &run.a.vz}, {"vx1", &run.a.vx1},
                                                                 {"vy1", &run.a.vy1}, {"vz1", &run.a.vz1},
                                                                 {"visc3", &run.a.visc3}}) {
      add(kv.first, kv.second, -2, X + 2, -2, Y + 2, -2, Z + 2);
    }
    add("bx", &run.a.bx, -2, X + 2, -1, Y + 2, -1, Z + 2);
    add("by", &run.a.by, -1, X + 2, -2, Y + 2, -1, Z + 2);
    add("bz", &run.a.bz, -1, X + 2, -1, Y + 2, -2, Z + 2);
    add("alpha1", &run.a.alpha1, 0, X + 1, 0, Y + 2, 0, Z + 2);
    add("alpha2", &run.a.alpha2, -1, X + 1, 0, Y + 1, 0, Z + 2);
    add("alpha3", &run.a.alpha3, -1, X + 1, -1, Y + 1, 0, Z + 1);
    add("visc_heat", &run.a.visc_heat, 0, X + 1, 0, Y + 1, 0, Z + 1);
    add("rho_v", &run.a.rho_v, -1, X + 1, -1, Y + 1, -1, Z + 1);
    add("cv_v", &run.a.cv_v, -1, X + 1, -1, Y + 1, -1, Z + 1);
    add("fx_visc", &run.a.fx_visc, 0, X, 0, Y, 0, Z);
    add("fy_visc", &run.a.fy_visc, 0, X, 0, Y, 0, Z);
    add("fz_visc", &run.a.fz_visc, 0, X, 0, Y, 0, Z);
    if (p.conduction) add("larsen_factor", &run.a.larsen, 0, X, 0, Y, 0, Z);
    if (run.a.xi.p) add("xi_n", &run.a.xi, -1, X + 2, -1, Y + 2, -1, Z + 2);
    if (run.a.eta_perp.p) add("eta_perp", &run.a.eta_perp, -1, X + 2, -1, Y + 2, -1, Z + 2);
    if (run.a.delta_ke.p) add("delta_ke", &run.a.delta_ke, -1, X + 2, -1, Y + 2, -1, Z + 2);
    if (run.a.heat_in.p) add("heat_in", &run.a.heat_in, -1, X + 2, -1, Y + 2, -1, Z + 2);
    if (run.a.cool_term_v.p) {  // (1:n in the reference; the padding here holds zeros)
      add("cool_term_v", &run.a.cool_term_v, 1, X, 1, Y, 1, Z);
      add("cool_term_b", &run.a.cool_term_b, 1, X, 1, Y, 1, Z);
    }
    cudaError_t e = cudaStreamSynchronize(run.s);
    if (e != cudaSuccess) { err = cudaGetErrorString(e); return LARE_ECUDA; }
    return LARE_OK;
  }

  void fill(A3<R> a, R v) {
    R* base = a.p - (2 + 2 * run.sx + 2 * run.sxy);
    int blocks = (int)((run.elems + 255) / 256);
    k_fill<R><<<blocks, 256, 0, run.s>>>(base, run.elems, v);
    ++run.launches;
  }

  int ensure_conduction_arrays() {
    if (run.a.Y1.p) return LARE_OK;
    std::string err;
    const long long off = 2 + 2LL * run.sx + 2LL * run.sxy;
    std::vector<A3<R>*> list = {&run.a.larsen, &run.a.Y1, &run.a.Y2, &run.a.Y3, &run.a.Lc_Y0};
    for (int q = 0; q < 9; ++q) list.push_back(&run.a.kf[q]);
    for (A3<R>* x : list) {
      R* base = dalloc<R>(run.elems, err);
      if (!base) return fail(LARE_ENOMEM, err);
      x->p = base + off;
      x->sx = run.sx;
      x->sxy = run.sxy;
      fill(*x, R(0));
    }
    FieldDesc f{{0, 0, 0}, {run.n[0], run.n[1], run.n[2]}};
    fields["larsen_factor"] = {&run.a.larsen, f};
    return LARE_OK;
  }

  // host Fortran array -> device padded box
  int put(A3<R> a, const FieldDesc& f, const double* host) {
    int e0 = f.hi[0] - f.lo[0] + 1, e1 = f.hi[1] - f.lo[1] + 1, e2 = f.hi[2] - f.lo[2] + 1;
    size_t n = (size_t)e0 * e1 * e2;
    if (cudaMemcpyAsync(staging, host, n * sizeof(double), cudaMemcpyHostToDevice, run.s) != cudaSuccess)
      return fail(LARE_ECUDA, "host to device copy failed");
    int blocks = (int)((n + 255) / 256);
    k_scatter<R><<<blocks, 256, 0, run.s>>>(staging, a.p, f.lo[0], f.lo[1], f.lo[2], e0, e1, e2, run.sx, run.sxy,
                                            dflag);
    ++run.launches;
    return cuda_check("upload");
  }
  int get(A3<R> a, const FieldDesc& f, double* host) {
    int e0 = f.hi[0] - f.lo[0] + 1, e1 = f.hi[1] - f.lo[1] + 1, e2 = f.hi[2] - f.lo[2] + 1;
    size_t n = (size_t)e0 * e1 * e2;
    int blocks = (int)((n + 255) / 256);
    k_gather<R><<<blocks, 256, 0, run.s>>>(a.p, staging, f.lo[0], f.lo[1], f.lo[2], e0, e1, e2, run.sx, run.sxy);
    ++run.launches;
    if (cudaMemcpyAsync(host, staging, n * sizeof(double), cudaMemcpyDeviceToHost, run.s) != cudaSuccess)
      return fail(LARE_ECUDA, "device to host copy failed");
    cudaError_t e = cudaStreamSynchronize(run.s);
    if (e != cudaSuccess) return fail(LARE_ECUDA, cudaGetErrorString(e));
    return LARE_OK;
  }

  // Upload the state; the scatter kernels flag non-finite values on the
  // device, so the host reads back one int after all copies.
  int upload(const double* const* s8) override {
    static const char* names[8] = {"rho", "energy", "vx", "vy", "vz", "bx", "by", "bz"};
    cudaMemsetAsync(dflag, 0, sizeof(int), run.s);
    for (int q = 0; q < 8; ++q) {
      if (!s8[q]) continue;
      auto& f = fields[names[q]];
      int rc = put(*f.first, f.second, s8[q]);
      if (rc) return rc;
    }
    int bad = 0;
    cudaMemcpyAsync(&bad, dflag, sizeof(int), cudaMemcpyDeviceToHost, run.s);
    cudaError_t e = cudaStreamSynchronize(run.s);
    if (e != cudaSuccess) return fail(LARE_ECUDA, cudaGetErrorString(e));
    if (bad) return fail(LARE_ENONFINITE, "non-finite value in the uploaded state");
    return LARE_OK;
  }

  int profile(int enable) override {
    if (enable) {
      run.prof_collect();
      run.prof.sites.clear();
      run.prof.index.clear();
      run.prof.used = 0;
      run.prof.on = true;
    } else {
      run.prof_collect();
      run.prof.on = false;
    }
    return LARE_OK;
  }

  // One line per launch site: "site<TAB>launches<TAB>ms<TAB>algorithmic bytes<TAB>words".
  int profile_report(char* buf, int len) override {
    run.prof_collect();
    std::vector<ProfSite> v = run.prof.sites;
    std::sort(v.begin(), v.end(), [](const ProfSite& a, const ProfSite& b) { return a.ms > b.ms; });
    std::string out;
    char line[256];
    for (const ProfSite& ps : v) {
      snprintf(line, sizeof(line), "%s:%d\t%lld\t%.6f\t%.0f\t%d\n", ps.func, ps.line, ps.count, ps.ms, ps.bytes,
               ps.words);
      out += line;
    }
    if (buf && len > 0) {
      size_t n = out.size() < (size_t)(len - 1) ? out.size() : (size_t)(len - 1);
      memcpy(buf, out.data(), n);
      buf[n] = 0;
    }
    return (int)out.size() + 1;
  }

  int upload_aux(const double* eta, const double* visc3, const double* grav, const double* gamma_boris) override {
    int rc;
    if (eta && (rc = put(run.a.eta, fields["eta"].second, eta))) return rc;
    if (visc3 && (rc = put(run.a.visc3, fields["visc3"].second, visc3))) return rc;
    if (gamma_boris) {
      if ((rc = put(run.a.gamma_boris, fields["gamma_boris"].second, gamma_boris))) return rc;
      run.gamma_boris_one = false;
    }
    if (grav) {
      std::vector<R> g(run.n[2] + 4);
      for (int i = 0; i < run.n[2] + 4; ++i) g[i] = (R)grav[i];
      cudaMemcpyAsync((R*)run.a.grav.p - 1, g.data(), g.size() * sizeof(R), cudaMemcpyHostToDevice, run.s);
    }
    cudaError_t e = cudaStreamSynchronize(run.s);
    return e == cudaSuccess ? LARE_OK : fail(LARE_ECUDA, cudaGetErrorString(e));
  }

  int set_time(double time, double dt) override {
    double v[2] = {dt, 0.5 * dt};
    cudaMemcpyAsync(run.sc + SC_DT, v, 2 * sizeof(double), cudaMemcpyHostToDevice, run.s);
    cudaMemcpyAsync(run.sc + SC_TIME, &time, sizeof(double), cudaMemcpyHostToDevice, run.s);
    cudaError_t e = cudaStreamSynchronize(run.s);
    return e == cudaSuccess ? LARE_OK : fail(LARE_ECUDA, cudaGetErrorString(e));
  }

  int lagrangian_step(int step) override {
    int rc = lare::lagrangian_step(run, step);
    if (rc) return fail(rc, rc == LARE_EDT ? "dt underflow or non-finite dt" : "lagrangian_step failed");
    if (run.pip) {
      if ((rc = eos_error())) return rc;
    }
    return cuda_check("lagrangian_step");
  }
  // LARE_EEOS raised by a neutral_fraction launch (syncs)
  int eos_error() {
    if (pull_scalars(run) != cudaSuccess) return fail(LARE_ECUDA, "sync failed");
    if ((int)run.host_sc[SC_ERROR] == LARE_EEOS)
      return fail(LARE_EEOS, "neutral_fraction: temperature bounds problem (empty bracket)");
    return LARE_OK;
  }
  int neutral_fraction() override {
    if (!run.pip) return LARE_OK;
    lare::neutral_fraction(run, run.a.energy);
    int rc = eos_error();
    return rc ? rc : cuda_check("neutral_fraction");
  }
  int perpendicular_resistivity() override {
    if (!run.cowling) return fail(LARE_EINVAL, "perpendicular_resistivity: cowling_resistivity is off");
    lare::perpendicular_resistivity(run);
    return cuda_check("perpendicular_resistivity");
  }
  bool partially_ionised() const override { return run.pip; }
  int energy_correction() override {
    if (!run.p.rke) return fail(LARE_EINVAL, "energy_correction: rke is off");
    lare::energy_correction(run);
    return cuda_check("energy_correction");
  }
  bool rke() const override { return run.p.rke != 0; }
  int eulerian_remap(int step) override {
    lare::eulerian_remap(run, step);
    return cuda_check("eulerian_remap");
  }
  int eta_calc() override {
    lare::eta_calc(run);
    return cuda_check("eta_calc");
  }
  int boundary_conditions() override {
    lare::boundary_conditions(run);
    return cuda_check("boundary_conditions");
  }
  int conduct_heat(double dt, int force_stages, int* n_stages) override {
    int rc = ensure_conduction_arrays();
    if (rc) return rc;
    cudaMemcpyAsync(run.sc + SC_DTCOND, &dt, sizeof(double), cudaMemcpyHostToDevice, run.s);
    calc_s_stages(run, SC_DTCOND);
    if (pull_scalars(run) != cudaSuccess) return fail(LARE_ECUDA, "conduct_heat: sync failed");
    int ns = force_stages > 0 ? force_stages : (int)run.host_sc[SC_STAGES];
    if (ns < 1 || ns > 100000) return fail(LARE_ESTAGES, "RKL2 stage count out of range");
    run.n_s_stages = ns;
    heat_conduct_sts2(run, SC_DTCOND);
    if (n_stages) *n_stages = ns;
    return cuda_check("conduct_heat");
  }
  int energy(double out[5]) override {
    energy_account(run);
    if (pull_scalars(run) != cudaSuccess) return fail(LARE_ECUDA, "energy: sync failed");
    out[0] = run.host_sc[SC_EN_B];
    out[1] = run.host_sc[SC_EN_KE];
    out[2] = run.host_sc[SC_EN_INT];
    out[3] = run.host_sc[SC_VISC_TOT];
    out[4] = run.host_sc[SC_OHM_TOT];
    return cuda_check("energy");
  }
  int download(double* const* s8) override {
    static const char* names[8] = {"rho", "energy", "vx", "vy", "vz", "bx", "by", "bz"};
    for (int q = 0; q < 8; ++q) {
      if (!s8[q]) continue;
      auto& f = fields[names[q]];
      int rc = get(*f.first, f.second, s8[q]);
      if (rc) return rc;
    }
    return LARE_OK;
  }
  int get_field(const char* name, double* host) override {
    auto it = fields.find(name);
    if (it == fields.end()) return fail(LARE_ENOTFOUND, std::string("unknown field ") + name);
    return get(*it->second.first, it->second.second, host);
  }
  int set_field(const char* name, const double* host) override {
    auto it = fields.find(name);
    if (it == fields.end()) return fail(LARE_ENOTFOUND, std::string("unknown field ") + name);
    if (std::string(name) == "gamma_boris") run.gamma_boris_one = false;
    int rc = put(*it->second.first, it->second.second, host);
    if (rc) return rc;
    cudaError_t e = cudaStreamSynchronize(run.s);
    return e == cudaSuccess ? LARE_OK : fail(LARE_ECUDA, cudaGetErrorString(e));
  }
  int field_bounds(const char* name, int lo[3], int hi[3]) override {
    auto it = fields.find(name);
    if (it == fields.end()) return fail(LARE_ENOTFOUND, std::string("unknown field ") + name);
    for (int d = 0; d < 3; ++d) {
      lo[d] = it->second.second.lo[d];
      hi[d] = it->second.second.hi[d];
    }
    return LARE_OK;
  }
  int capture_steps(int nsteps) override {
    if (run.p.conduction) return fail(LARE_EINVAL, "capture: conduction steps need the host (stage count)");
    if (run.steps_taken < 1) return fail(LARE_EINVAL, "capture: take one step first (first-call set-up)");
    if (run.prof.on) return fail(LARE_EINVAL, "capture: profiling is on");
    if (!run.s_body && cudaStreamCreateWithFlags(&run.s_body, cudaStreamNonBlocking) != cudaSuccess)
      return fail(LARE_ECUDA, "capture: stream");
    const int first = run.steps_taken + 1;
    const int saved_taken = run.steps_taken, saved_peak = run.peak_substeps;
    run.capturing = true;
    int rc = LARE_OK;
    for (int k = 0; k < nsteps && rc == LARE_OK; ++k) {
      if (run.pip) lare::neutral_fraction(run, run.a.energy);  // lare3d.f90:83
      rc = lare::lagrangian_step(run, first + k);
      if (rc == LARE_OK) lare::eulerian_remap(run, first + k);
      if (rc == LARE_OK && run.p.rke) lare::energy_correction(run);  // lare3d.f90:86
      if (rc == LARE_OK) lare::eta_calc(run);
    }
    run.capturing = false;
    run.steps_taken = saved_taken;
    run.peak_substeps = saved_peak;
    run.last_substeps = -1;
    if (rc) return fail(rc, "capture: step recording failed");
    return cuda_check("capture_steps");
  }
  void add_steps(int n) override { run.steps_taken += n; }
  int set_block(int bx, int by) override {
    if (bx < 1 || by < 1 || bx * by > 256 || (bx * by) % 32) return fail(LARE_EINVAL, "block shape");
    run.blk_x = bx;
    run.blk_y = by;
    return LARE_OK;
  }
  int device_error() override {
    if (pull_scalars(run) != cudaSuccess) return fail(LARE_ECUDA, "device_error: sync failed");
    const int code = (int)run.host_sc[SC_ERROR];
    if (code) fail(code, "raised on the device in a recorded step (bad dt, sub-cycle count or EOS bracket)");
    return code;
  }
  int conduction_stages(double dt, int* n_stages) override {
    int rc = ensure_conduction_arrays();
    if (rc) return rc;
    cudaMemcpyAsync(run.sc + SC_DTCOND, &dt, sizeof(double), cudaMemcpyHostToDevice, run.s);
    calc_s_stages(run, SC_DTCOND);
    if (pull_scalars(run) != cudaSuccess) return fail(LARE_ECUDA, "conduction_stages: sync failed");
    *n_stages = (int)run.host_sc[SC_STAGES];
    return cuda_check("conduction_stages");
  }
  int field_device(const char* name, void** origin, int* sx, int* sxy, int* elem_bytes) override {
    if (std::strcmp(name, "larsen_factor") == 0) {
      int rc = ensure_conduction_arrays();
      if (rc) return rc;
    }
    auto it = fields.find(name);
    if (it == fields.end()) return fail(LARE_ENOTFOUND, std::string("unknown field ") + name);
    *origin = (void*)it->second.first->p;
    *sx = run.sx;
    *sxy = run.sxy;
    *elem_bytes = (int)sizeof(R);
    return LARE_OK;
  }
  int scalars(lare_scalars* o) override {
    if (pull_scalars(run) != cudaSuccess) return fail(LARE_ECUDA, "scalars: sync failed");
    o->time = run.host_sc[SC_TIME];
    o->dt = run.host_sc[SC_DT];
    o->dtr = run.host_sc[SC_DTR];
    o->total_visc_heating = run.host_sc[SC_VISC_TOT];
    o->total_ohmic_heating = run.host_sc[SC_OHM_TOT];
    o->n_s_stages = run.n_s_stages;
    o->peak_substeps = run.peak_substeps;
    o->last_substeps = run.last_substeps;
    o->steps_taken = run.steps_taken;
    return LARE_OK;
  }
  long long launches() const override { return run.launches; }
  void* stream() const override { return (void*)run.s; }
  const char* error() const override { return run.err.c_str(); }
  void set_error(const std::string& e) override { run.err = e; }
};

template <class R>
EngineBase* make_engine(const lare_params* p, int nx, int ny, int nz, const double* const* metrics6,
                        std::string& err) {
  EngineT<R>* e = new EngineT<R>();
  int rc = e->init(p, nx, ny, nz, metrics6, err);
  if (rc != LARE_OK) {
    delete e;
    return nullptr;
  }
  return e;
}

LARE_END  // namespace lare
