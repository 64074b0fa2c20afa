/*
 * lare_ref.h - C ABI of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * The oracle is a C++ restatement of the reference's Fortran hot path
 * (lagran.F90, remap.f90, [xyz]remap.f90, conduct.f90, boundary.f90 with the
 * periodic semantics of mpiboundary.f90, diagnostics.F90:517-609).  It is
 * used only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg, as the checker; the product path never calls it.
 *
 * Entry points mirror include/lare_gpu.h one for one so that a parity test
 * drives both with the same calls.  Array arguments use the reference's
 * Fortran bounds (see include/lare_gpu.h).
 */
#ifndef LARE_REF_H
#define LARE_REF_H

#include "../include/lare_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lare_ref lare_ref;

int lare_ref_init(const lare_params* params, int nx, int ny, int nz,
                  const double* dxb, const double* dxc,
                  const double* dyb, const double* dyc,
                  const double* dzb, const double* dzc, lare_ref** out);
int lare_ref_upload(lare_ref* r, const double* rho, const double* energy,
                    const double* vx, const double* vy, const double* vz,
                    const double* bx, const double* by, const double* bz);
int lare_ref_upload_aux(lare_ref* r, const double* eta, const double* visc3,
                        const double* grav, const double* gamma_boris);
int lare_ref_set_time(lare_ref* r, double time, double dt);
int lare_ref_lagrangian_step(lare_ref* r, int step);
int lare_ref_eulerian_remap(lare_ref* r, int step);
int lare_ref_eta_calc(lare_ref* r);
int lare_ref_boundary_conditions(lare_ref* r);
int lare_ref_neutral_fraction(lare_ref* r);
int lare_ref_perpendicular_resistivity(lare_ref* r);
int lare_ref_energy_correction(lare_ref* r);
/* the exponential the ionisation model uses (Cody-Waite + Taylor) */
double lare_ref_exp(double x);
int lare_ref_step(lare_ref* r, int step, double* time, double* dt);
int lare_ref_conduct_heat(lare_ref* r, double dt, int* n_stages);
int lare_ref_energy(lare_ref* r, double out[5]);
int lare_ref_download(lare_ref* r, double* rho, double* energy, double* vx,
                      double* vy, double* vz, double* bx, double* by,
                      double* bz);
int lare_ref_get_field(lare_ref* r, const char* name, double* host);
int lare_ref_set_field(lare_ref* r, const char* name, const double* host);
int lare_ref_field_bounds(lare_ref* r, const char* name, int lo[3], int hi[3]);
int lare_ref_get_scalars(lare_ref* r, lare_scalars* out);
int lare_ref_num_threads(void);
const char* lare_ref_last_error(lare_ref* r);
void lare_ref_destroy(lare_ref* r);

#ifdef __cplusplus
}
#endif

#endif
