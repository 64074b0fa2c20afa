// lare_gpu.cu - the extern "C" boundary declared in include/lare_gpu.h.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/lare_gpu.h"
#include "common.cuh"
#include "engine_base.h"

struct lare_ctx {
  lare::EngineBase* e = nullptr;
  int precision = 64;
  std::string err;
};

namespace {
bool bc_supported(int c) { return c == LARE_BC_PERIODIC || c == LARE_BC_USER || c == LARE_BC_OPEN; }

int guard(lare_ctx* c) { return (c && c->e) ? LARE_OK : LARE_EINVAL; }

__global__ void k_check_division(const double* a, const double* b, long long n, double* out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double rb = 1.0 / b[i];
    out[i] = lare::div_rcp(a[i], b[i], rb);
  }
}

__global__ void k_check_reciprocal(const double* b, long long n, double* out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = lare::fast_rcp(b[i]);
}
}  // namespace

extern "C" {

int lare_gpu_init(const lare_params* p, int nx, int ny, int nz, const double* dxb, const double* dxc,
                  const double* dyb, const double* dyc, const double* dzb, const double* dzc, int precision,
                  lare_ctx** out) {
  if (!out) return LARE_EINVAL;
  *out = nullptr;
  if (!p || !dxb || !dxc || !dyb || !dyc || !dzb || !dzc) return LARE_EINVAL;
  if (nx < 4 || ny < 4 || nz < 4) return LARE_EINVAL;
  if (precision != LARE_FP64 && precision != LARE_FP64_EXACT && precision != LARE_FP32) return LARE_EINVAL;
  const int bcs[6] = {p->xbc_min, p->xbc_max, p->ybc_min, p->ybc_max, p->zbc_min, p->zbc_max};
  for (int q = 0; q < 6; ++q)
    if (!bc_supported(bcs[q])) return LARE_EINVAL;
  // A periodic boundary needs both sides periodic: the reference leaves the
  // ghosts of a half-periodic direction unset (mpi_routines.F90:195-210).
  for (int d = 0; d < 3; ++d)
    if ((bcs[2 * d] == LARE_BC_PERIODIC) != (bcs[2 * d + 1] == LARE_BC_PERIODIC)) return LARE_EINVAL;
  if (!(p->gamma > 1.0) || !(p->dt_multiplier > 0.0)) return LARE_EINVAL;
  if (p->eos_number < 0 || p->eos_number > LARE_EOS_PI) return LARE_EINVAL;
  if ((p->eos_number > LARE_EOS_IDEAL || p->cowling_resistivity) &&
      !(p->f_bar > 0.0 && p->t_bar > 0.0 && p->r_bar > 0.0 && p->tr > 0.0 && p->eta_bar >= 0.0))
    return LARE_EINVAL;  // the ionisation model's constants must be set
  if (p->radiation && !(p->temp_norm > 0.0 && p->time_norm > 0.0 && p->rho_norm > 0.0 && p->mf > 0.0))
    return LARE_EINVAL;  // radiative losses need the normalisation
  // every device index is 32-bit: the padded box must stay below 2^31 points
  if (((long long)nx + 5 + 3) / 4 * 4 * (ny + 5LL) * (nz + 5LL) >= (1LL << 31)) return LARE_ETOOLARGE;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return LARE_ECUDA;
  const double* m6[6] = {dxb, dxc, dyb, dyc, dzb, dzc};
  std::string err;
  lare::EngineBase* e = precision == LARE_FP64         ? lare::make_engine_f64(p, nx, ny, nz, m6, err)
                       : precision == LARE_FP64_EXACT ? lare::make_engine_f64_exact(p, nx, ny, nz, m6, err)
                                                      : lare::make_engine_f32(p, nx, ny, nz, m6, err);
  if (!e) return err.find("cudaMalloc") != std::string::npos ? LARE_ENOMEM : LARE_ECUDA;
  lare_ctx* c = new lare_ctx();
  c->e = e;
  c->precision = precision;
  *out = c;
  return LARE_OK;
}

int lare_gpu_upload(lare_ctx* c, const double* rho, const double* energy, const double* vx, const double* vy,
                    const double* vz, const double* bx, const double* by, const double* bz) {
  if (guard(c)) return LARE_EINVAL;
  const double* s8[8] = {rho, energy, vx, vy, vz, bx, by, bz};
  return c->e->upload(s8);
}

int lare_gpu_upload_aux(lare_ctx* c, const double* eta, const double* visc3, const double* grav,
                        const double* gamma_boris) {
  if (guard(c)) return LARE_EINVAL;
  return c->e->upload_aux(eta, visc3, grav, gamma_boris);
}

int lare_gpu_set_time(lare_ctx* c, double time, double dt) {
  if (guard(c)) return LARE_EINVAL;
  if (!std::isfinite(time) || !std::isfinite(dt) || dt < 0.0) return LARE_EINVAL;
  return c->e->set_time(time, dt);
}

int lare_gpu_lagrangian_step(lare_ctx* c, int step) {
  if (guard(c)) return LARE_EINVAL;
  return c->e->lagrangian_step(step);
}

int lare_gpu_eulerian_remap(lare_ctx* c, int step) {
  if (guard(c)) return LARE_EINVAL;
  return c->e->eulerian_remap(step);
}

int lare_gpu_eta_calc(lare_ctx* c) {
  if (guard(c)) return LARE_EINVAL;
  return c->e->eta_calc();
}

int lare_gpu_boundary_conditions(lare_ctx* c) {
  if (guard(c)) return LARE_EINVAL;
  return c->e->boundary_conditions();
}

int lare_gpu_neutral_fraction(lare_ctx* c) {
  if (guard(c)) return LARE_EINVAL;
  return c->e->neutral_fraction();
}

int lare_gpu_perpendicular_resistivity(lare_ctx* c) {
  if (guard(c)) return LARE_EINVAL;
  return c->e->perpendicular_resistivity();
}

int lare_gpu_energy_correction(lare_ctx* c) {
  if (guard(c)) return LARE_EINVAL;
  return c->e->energy_correction();
}

int lare_gpu_step(lare_ctx* c, int step, double* time, double* dt) {
  if (guard(c)) return LARE_EINVAL;
  int rc = c->e->neutral_fraction();  // lare3d.f90:83 (a no-op under EOS_IDEAL)
  if (rc) return rc;
  rc = c->e->lagrangian_step(step);
  if (rc) return rc;
  if ((rc = c->e->eulerian_remap(step))) return rc;
  if (c->e->rke() && (rc = c->e->energy_correction())) return rc;  // lare3d.f90:86
  if ((rc = c->e->eta_calc())) return rc;
  if (time || dt) {
    lare_scalars s;
    if ((rc = c->e->scalars(&s))) return rc;
    if (time) *time = s.time;
    if (dt) *dt = s.dt;
  }
  return LARE_OK;
}

int lare_gpu_run(lare_ctx* c, int first_step, int nsteps, double t_end, int* steps_done, double* time, double* dt) {
  if (guard(c)) return LARE_EINVAL;
  lare_scalars s;
  int rc = c->e->scalars(&s);
  if (rc) return rc;
  int step = first_step, done = 0;
  // lare3d.f90:80-89
  while (!((done >= nsteps && nsteps >= 0) || s.time >= t_end)) {
    ++step;
    if ((rc = c->e->neutral_fraction())) return rc;
    if ((rc = c->e->lagrangian_step(step))) return rc;
    if ((rc = c->e->eulerian_remap(step))) return rc;
    if (c->e->rke() && (rc = c->e->energy_correction())) return rc;
    if ((rc = c->e->eta_calc())) return rc;
    ++done;
    if ((rc = c->e->scalars(&s))) return rc;
  }
  if (steps_done) *steps_done = done;
  if (time) *time = s.time;
  if (dt) *dt = s.dt;
  return LARE_OK;
}

int lare_gpu_conduct_heat(lare_ctx* c, double dt, int* n_stages) {
  if (guard(c)) return LARE_EINVAL;
  if (!(dt > 0.0) || !std::isfinite(dt)) return LARE_EINVAL;
  return c->e->conduct_heat(dt, 0, n_stages);
}

int lare_gpu_conduct_heat_stages(lare_ctx* c, double dt, int n_stages) {
  if (guard(c)) return LARE_EINVAL;
  if (!(dt > 0.0) || !std::isfinite(dt) || n_stages < 2) return LARE_EINVAL;
  return c->e->conduct_heat(dt, n_stages, nullptr);
}

int lare_gpu_set_block(lare_ctx* c, int bx, int by) {
  if (guard(c)) return LARE_EINVAL;
  return c->e->set_block(bx, by);
}

int lare_gpu_conduction_stages(lare_ctx* c, double dt, int* n_stages) {
  if (guard(c) || !n_stages) return LARE_EINVAL;
  if (!(dt > 0.0) || !std::isfinite(dt)) return LARE_EINVAL;
  return c->e->conduction_stages(dt, n_stages);
}

int lare_gpu_field_device(lare_ctx* c, const char* name, void** origin, int* sx, int* sxy, int* elem_bytes) {
  if (guard(c) || !name || !origin || !sx || !sxy || !elem_bytes) return LARE_EINVAL;
  return c->e->field_device(name, origin, sx, sxy, elem_bytes);
}

int lare_gpu_energy(lare_ctx* c, double out[5]) {
  if (guard(c) || !out) return LARE_EINVAL;
  return c->e->energy(out);
}

int lare_gpu_download(lare_ctx* c, double* rho, double* energy, double* vx, double* vy, double* vz, double* bx,
                      double* by, double* bz) {
  if (guard(c)) return LARE_EINVAL;
  double* s8[8] = {rho, energy, vx, vy, vz, bx, by, bz};
  return c->e->download(s8);
}

int lare_gpu_get_field(lare_ctx* c, const char* name, double* host) {
  if (guard(c) || !name || !host) return LARE_EINVAL;
  return c->e->get_field(name, host);
}

int lare_gpu_set_field(lare_ctx* c, const char* name, const double* host) {
  if (guard(c) || !name || !host) return LARE_EINVAL;
  return c->e->set_field(name, host);
}

int lare_gpu_field_bounds(lare_ctx* c, const char* name, int lo[3], int hi[3]) {
  if (guard(c) || !name || !lo || !hi) return LARE_EINVAL;
  return c->e->field_bounds(name, lo, hi);
}

int lare_gpu_get_scalars(lare_ctx* c, lare_scalars* out) {
  if (guard(c) || !out) return LARE_EINVAL;
  return c->e->scalars(out);
}

int lare_gpu_profile(lare_ctx* c, int enable) {
  if (guard(c)) return LARE_EINVAL;
  return c->e->profile(enable);
}

int lare_gpu_profile_report(lare_ctx* c, char* buf, int len) {
  if (guard(c)) return LARE_EINVAL;
  return c->e->profile_report(buf, len);
}

long long lare_gpu_launch_count(lare_ctx* c) { return (c && c->e) ? c->e->launches() : -1; }

int lare_gpu_check_division(const double* a, const double* b, long long n, double* out, void* stream) {
  if (n < 0 || (n > 0 && (!a || !b || !out))) return LARE_EINVAL;
  if (n == 0) return LARE_OK;
  const long long blocks = (n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16;
  k_check_division<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(a, b, n, out);
  return cudaGetLastError() == cudaSuccess ? LARE_OK : LARE_ECUDA;
}

int lare_gpu_check_reciprocal(const double* b, long long n, double* out, void* stream) {
  if (n < 0 || (n > 0 && (!b || !out))) return LARE_EINVAL;
  if (n == 0) return LARE_OK;
  const long long blocks = (n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16;
  k_check_reciprocal<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(b, n, out);
  return cudaGetLastError() == cudaSuccess ? LARE_OK : LARE_ECUDA;
}

void* lare_gpu_stream(lare_ctx* c) { return (c && c->e) ? c->e->stream() : nullptr; }

const char* lare_gpu_last_error(lare_ctx* c) {
  if (!c) return "null context";
  if (!c->e) return c->err.c_str();
  return c->e->error();
}

void lare_gpu_destroy(lare_ctx* c) {
  if (!c) return;
  delete c->e;
  delete c;
}

// ---------------------------------------------------------------------
// Ensembles: many independent contexts advanced by one CUDA graph launch.

struct lare_ens {
  std::vector<lare_ctx*> m;
  int steps_per_launch = 0;
  cudaStream_t s = nullptr;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t x = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> joins;
  long long launched = 0;  // launches not yet folded into the members' step counters
};

namespace {
void ens_free(lare_ens* e) {
  if (!e) return;
  if (e->s) cudaStreamSynchronize(e->s);
  if (e->x) cudaGraphExecDestroy(e->x);
  if (e->g) cudaGraphDestroy(e->g);
  if (e->fork) cudaEventDestroy(e->fork);
  for (cudaEvent_t j : e->joins)
    if (j) cudaEventDestroy(j);
  if (e->s) cudaStreamDestroy(e->s);
  delete e;
}
}  // namespace

int lare_ens_create(lare_ctx* const* members, int n, int steps_per_launch, lare_ens** out) {
  if (!out) return LARE_EINVAL;
  *out = nullptr;
  if (!members || n < 1 || steps_per_launch < 1 || steps_per_launch % 6) return LARE_EINVAL;
  for (int i = 0; i < n; ++i)
    if (guard(members[i])) return LARE_EINVAL;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < i; ++j)
      if (members[i] == members[j]) return LARE_EINVAL;
  lare_ens* e = new lare_ens();
  e->m.assign(members, members + n);
  e->steps_per_launch = steps_per_launch;
  e->joins.assign(n, nullptr);
  int rc = LARE_OK;
  if (cudaStreamCreateWithFlags(&e->s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess) {
    ens_free(e);
    return LARE_ECUDA;
  }
  for (int i = 0; i < n; ++i) {
    if (cudaEventCreateWithFlags(&e->joins[i], cudaEventDisableTiming) != cudaSuccess) {
      ens_free(e);
      return LARE_ECUDA;
    }
  }
  // Members may still be busy with eager work on their own streams.
  for (int i = 0; i < n; ++i) cudaStreamSynchronize((cudaStream_t)members[i]->e->stream());
  // One capture: fork every member's stream off the ensemble stream, record
  // its steps there, join back.
  if (cudaStreamBeginCapture(e->s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    ens_free(e);
    return LARE_ECUDA;
  }
  cudaEventRecord(e->fork, e->s);
  for (int i = 0; i < n && rc == LARE_OK; ++i) {
    cudaStream_t ms = (cudaStream_t)members[i]->e->stream();
    cudaStreamWaitEvent(ms, e->fork, 0);
    rc = members[i]->e->capture_steps(steps_per_launch);
    cudaEventRecord(e->joins[i], ms);
    cudaStreamWaitEvent(e->s, e->joins[i], 0);
  }
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(e->s, &g);
  e->g = g;
  if (rc == LARE_OK && ce != cudaSuccess) rc = LARE_ECUDA;
  if (rc == LARE_OK && cudaGraphInstantiate(&e->x, e->g, 0) != cudaSuccess) rc = LARE_ECUDA;
  cudaGetLastError();
  if (rc) {
    ens_free(e);
    return rc;
  }
  *out = e;
  return LARE_OK;
}

int lare_ens_launch(lare_ens* e, int nlaunch) {
  if (!e || !e->x || nlaunch < 0) return LARE_EINVAL;
  for (int k = 0; k < nlaunch; ++k) {
    if (cudaGraphLaunch(e->x, e->s) != cudaSuccess) return LARE_ECUDA;
    ++e->launched;
  }
  return LARE_OK;
}

int lare_ens_sync(lare_ens* e, int* first_bad) {
  if (!e) return LARE_EINVAL;
  if (first_bad) *first_bad = -1;
  if (cudaStreamSynchronize(e->s) != cudaSuccess) return LARE_ECUDA;
  const int adv = (int)(e->launched * e->steps_per_launch);
  e->launched = 0;
  int rc = LARE_OK;
  for (size_t i = 0; i < e->m.size(); ++i) {
    e->m[i]->e->add_steps(adv);
    const int code = e->m[i]->e->device_error();
    if (code && rc == LARE_OK) {
      rc = code;
      if (first_bad) *first_bad = (int)i;
    }
  }
  return rc;
}

void* lare_ens_stream(lare_ens* e) { return e ? (void*)e->s : nullptr; }

void lare_ens_destroy(lare_ens* e) { ens_free(e); }

}  // extern "C"
