/*
 * edm_oracle.h — CPU float64 restatement of the ED-MRDT per-timestep path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
 * against; it is never linked into, imported by or called from the product
 * library.  It follows the reference (Python + Numba, ED-MRDT v1.1) line by
 * line, with every `rng.*` draw replaced by the keyed Philox draw of the same
 * stream, so the reference itself (with the same draws injected) and this
 * oracle produce identical results; the pinning tests check exactly that.
 */
#ifndef EDM_ORACLE_H
#define EDM_ORACLE_H
#include <stdint.h>
#include "../include/edm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- keyed noise (the specification both implementations follow) -------- */
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void orc_uniform2(uint64_t seed, int64_t step, int32_t stream, uint64_t a,
                  uint64_t b, double* u0, double* u1);
void orc_normal2(uint64_t seed, int64_t step, int32_t stream, uint64_t a,
                 double* z0, double* z1);
double orc_ln(double q);
void orc_sincos_2pi(double u, double* c, double* s);
/* vector helpers used by the reference shim */
void orc_fill_uniform(uint64_t seed, int64_t step, int32_t stream,
                      const int64_t* a, const int64_t* b, int64_t n,
                      double* out, int32_t two);
void orc_fill_normal(uint64_t seed, int64_t step, int32_t stream,
                     const int64_t* a, int64_t n, double* out, int32_t two);
int64_t orc_poisson_knuth(uint64_t seed, int64_t step, int32_t stream,
                          uint64_t key, double exp_neg_lambda);

/* ---- dynamics (dynamics.py:2150-2465) ------------------------------------ */
typedef struct {
  int64_t N;
  double* pos;        /* [N][2]               */
  int32_t* species;
  uint8_t* alive;
  int32_t* bond;      /* local index, -1 free */
  int64_t counters[EDM_NCOUNTERS];
  /* outputs of the last step for inspection */
  int32_t* head;      /* [nx*ny]              */
  int32_t* next;      /* [N]                  */
  int32_t* pairs;     /* [max_pairs][2]       */
  int64_t n_pairs, max_pairs;
  double* forces;     /* [N][2]               */
  double* adapt_w;    /* adaptation field w [nx][ny] of the adaptation grid, or NULL */
} OrcDyn;

int orc_dyn_alloc(OrcDyn* s, const EdmDynParams* p, int64_t N);
void orc_dyn_free(OrcDyn* s);
int orc_dyn_step(const EdmDynParams* p, OrcDyn* s, int64_t step);

/* ---- photophysics (photophysics.py:338-683, 1021-1197) ------------------- */
typedef struct {
  int32_t n_fluoro;
  double T_step[EDM_MAX_FLUO][3][3], T_step_fret[EDM_MAX_FLUO][3][3];
  double mean_ph[EDM_MAX_FLUO][2], mean_ph_fret[EDM_MAX_FLUO][2];
  double mean_fret[EDM_MAX_FLUO][2], mean_fret_fret[EDM_MAX_FLUO][2];
  double tau_all[EDM_MAX_FLUO], k_fret_bound[EDM_MAX_FLUO];
  int32_t ground[EDM_MAX_FLUO], excited[EDM_MAX_FLUO], t1[EDM_MAX_FLUO], bl[EDM_MAX_FLUO];
  int32_t n_bond;
  double bond_R0[EDM_MAX_FRET], bond_tauD[EDM_MAX_FRET], bond_icd[EDM_MAX_FRET];
  int32_t bond_donor[EDM_MAX_FRET], bond_acceptor[EDM_MAX_FRET], bond_intra[EDM_MAX_FRET];
  int32_t n_prox;
  double prox_radius_um[EDM_MAX_FRET], prox_khigh[EDM_MAX_FRET], prox_klow[EDM_MAX_FRET];
  int32_t prox_donor[EDM_MAX_FRET], prox_target[EDM_MAX_FRET];
  int64_t max_photons, est_photons;
  double Lx, Ly;
  int32_t periodic_x, periodic_y;
  uint64_t seed;
} OrcPhotParams;

typedef struct {
  int64_t N;
  const double* pos;
  const int32_t* species;
  const uint8_t* alive;
  const int32_t* bond;
  const uint8_t* has_dye;
  const int32_t* dye_type;
  int8_t* ctmc;
  uint8_t* bleached;
  double* k_fret;        /* [N] scratch/output */
  int32_t* acc_idx;      /* [N] scratch/output */
  /* photon batch outputs, capacity max_photons */
  int32_t* ph_particle;
  double* ph_time;
  int8_t* ph_channel;
  uint8_t* ph_is_fret;
  int64_t n_photons;
} OrcPhot;

void orc_update_fret_rates(const OrcPhotParams* p, OrcPhot* s);
int orc_photon_step(const OrcPhotParams* p, OrcPhot* s, int64_t step);

/* ---- microscope (microscope.py:522-631, 716-803, 839-922, 1069-1203) ----- */
typedef struct {
  int64_t n_received, n_detected;
} OrcScopeStats;

int orc_process_photons(const EdmScopeParams* sp, uint64_t seed, int64_t step,
                        const double* pos, int64_t N, const int32_t* ph_particle,
                        const double* ph_time, const int8_t* ph_channel,
                        int64_t n_ph, uint32_t* flim, OrcScopeStats* st);
int orc_finalize_frame(const EdmScopeParams* sp, uint64_t seed, int64_t frame,
                       uint32_t* flim, int64_t* n_dark, int64_t* n_ap);

#ifdef __cplusplus
}
#endif
#endif
