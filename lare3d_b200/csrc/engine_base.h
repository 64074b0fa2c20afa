// engine_base.h - precision-independent interface of a device context.
#pragma once

#include <string>

#include "../../include/lare_gpu.h"

namespace lare {

class EngineBase {
 public:
  virtual ~EngineBase() {}
  virtual int upload(const double* const* state8) = 0;
  virtual int upload_aux(const double* eta, const double* visc3, const double* grav, const double* gamma_boris) = 0;
  virtual int set_time(double time, double dt) = 0;
  virtual int lagrangian_step(int step) = 0;
  virtual int eulerian_remap(int step) = 0;
  virtual int eta_calc() = 0;
  virtual int boundary_conditions() = 0;
  virtual int neutral_fraction() = 0;           // no-op under EOS_IDEAL
  virtual int perpendicular_resistivity() = 0;
  virtual bool partially_ionised() const = 0;
  virtual int energy_correction() = 0;          // LARE_EINVAL unless rke
  virtual bool rke() const = 0;
  virtual int conduct_heat(double dt, int force_stages, int* n_stages) = 0;
  virtual int conduction_stages(double dt, int* n_stages) = 0;
  virtual int energy(double out[5]) = 0;
  virtual int download(double* const* state8) = 0;
  virtual int get_field(const char* name, double* host) = 0;
  virtual int set_field(const char* name, const double* host) = 0;
  virtual int field_bounds(const char* name, int lo[3], int hi[3]) = 0;
  virtual int field_device(const char* name, void** origin, int* sx, int* sxy, int* elem_bytes) = 0;
  virtual int scalars(lare_scalars* out) = 0;
  virtual int profile(int enable) = 0;
  virtual int profile_report(char* buf, int len) = 0;
  // CUDA-graph recording of whole steps (the ensemble path).  The caller
  // has put stream() into capture mode; capture_steps records nsteps steps
  // numbered from steps_taken + 1 and leaves the host-side counters as they
  // were; add_steps advances them once the graph has run.
  virtual int capture_steps(int nsteps) = 0;
  virtual void add_steps(int n) = 0;
  virtual int set_block(int bx, int by) = 0;
  virtual int device_error() = 0;  // syncs; LARE_E* raised on the device, 0 if none
  virtual long long launches() const = 0;
  virtual void* stream() const = 0;
  virtual const char* error() const = 0;
  virtual void set_error(const std::string& e) = 0;
};

// Factories (engine_f64fast.cu, engine_f64.cu, engine_f32.cu).  Return
// nullptr and fill err on failure.
EngineBase* make_engine_f64(const lare_params* p, int nx, int ny, int nz, const double* const* metrics6,
                            std::string& err);
EngineBase* make_engine_f64_exact(const lare_params* p, int nx, int ny, int nz, const double* const* metrics6,
                                  std::string& err);
EngineBase* make_engine_f32(const lare_params* p, int nx, int ny, int nz, const double* const* metrics6,
                            std::string& err);

}  // namespace lare
