/*
 * ptrans_oracle.h - TEST INFRASTRUCTURE.  C API of the CPU FP64 oracle: a
 * restatement of the P-TRANS RTMC algorithm (src/RTMCphon.f90) used only by
 * tests/, the smoke check and bench.py's CPU baseline to check the CUDA path.
 * It is never linked into the product library.
 *
 * PARITY UNPINNED: the reference is Fortran, no Fortran compiler exists on
 * either machine, and the reference ships no golden outputs (its RNG is
 * clock-seeded, src/RTMCphon.f90:3314-3330).  The oracle is pinned instead to
 * the published Philox4x32-10 known-answer vectors and to analytic limits the
 * reference formulas imply (tests/test_oracle_analytic.py).
 */
#ifndef PTRANS_ORACLE_H
#define PTRANS_ORACLE_H

#include <stdint.h>
#include "../include/ptrans_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_handle orc_handle;

typedef struct orc_result {
  uint64_t flights;   /* free flights (iterations of the transport loop)   */
  uint64_t lost;      /* phonons that left the box or hit the flight cap   */
  uint64_t capped;    /* of which: hit the flight cap                      */
  uint64_t samples;   /* trajectories simulated                            */
  double seconds;     /* wall time of the transport                         */
  int32_t threads;    /* OpenMP threads used                                */
} orc_result;

int orc_build_model(const ptg_model* m, const ptg_spectrum* s, orc_handle** out);
int orc_from_geometry(const ptg_geometry* g, const ptg_spectrum* s, orc_handle** out);
void orc_free(orc_handle* h);

int orc_geometry_sizes(const orc_handle* h, int32_t* ngrain_total, int32_t* nsurf,
                       int32_t* nvertex_total);
/* Fills caller arrays with the built geometry in the ptg_geometry layout. */
int orc_geometry_export(const orc_handle* h, int32_t* grain_begin, int32_t* grain_incident,
                        double* grain_generatrix, int32_t* shape, int32_t* nvertex,
                        int32_t* vertex_begin, double* vertex, double* normal,
                        double* tangent, double* center, double* radius,
                        int32_t* kind_trans, double* specularity, double* trans_param,
                        int32_t* grain_inside, int32_t* grain_outside, int32_t* internal,
                        int32_t* incident, int32_t* material1, int32_t* material2);

/* Number of tasks of a run (ptg_run numbering). */
int64_t orc_ntask(const orc_handle* h, const ptg_run* run);

/*
 * Transport of the tasks of a run.  task_subset (may be NULL) restricts the
 * run to the listed tasks; counts/lost (length ntask, may be NULL) receive the
 * transmitted / lost counts per task.  nthreads <= 0 uses all OpenMP threads.
 * ref_quirks = 1 adds lost phonons to the transmitted count.
 */
int orc_run_counts(orc_handle* h, const ptg_run* run, int64_t max_flights, int32_t ref_quirks,
                   int32_t nthreads, const int64_t* task_subset, int64_t nsubset,
                   uint64_t* counts, uint64_t* lost, orc_result* res);

/* One task, per particle: exit side (0 lost, 1 x-, 2 x+), flights, final position. */
int orc_replay_task(orc_handle* h, const ptg_run* run, int64_t task, int64_t max_flights,
                    int32_t* end_side, uint32_t* flights, double* final_pos);

/* effectiveMFP + fileoutput kappa from counts (the reference's order of
   operations, including its per-branch exchange sort by omega). */
int orc_kappa_from_counts(orc_handle* h, const ptg_run* run, const uint64_t* counts,
                          ptg_kappa_out* out);

/* fileoutput's thermalproperty.out, effectiveMFP.out and
   phononconductivity.out next to geofile, from the counts of a run. */
int orc_write_outputs(orc_handle* h, const char* geofile, const ptg_run* run,
                      const uint64_t* counts);
/* GammaDeterm (ModeNum 1): gamma of T(omega) = 1/(gamma omega/omega_max + 1)
   whose boundary conductance is TBC [W m^-2 K^-1], on the handle's spectrum. */
int orc_gamma_from_tbc(orc_handle* h, double temperature, double TBC, double* gamma);
/* Raw Philox4x32-10 block (for known-answer tests). */
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* The oracle's log and sincos(2*pi*u) (checked against libm in tests). */
double orc_log(double x);
void orc_sincos2pi(double u, double* s, double* c);

#ifdef __cplusplus
}
#endif
#endif
