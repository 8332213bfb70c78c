/*
 * edm_b200.h — C ABI of the B200-native ED-MRDT per-timestep hot path.
 *
 * The reference (Edel-datsci/FLIM-Microscopy-Simulator-with-Causal-Inference,
 * "ED-MRDT v1.1") is pure Python + Numba and has no FFI layer; its drop-in
 * boundary is the Python object API.  Each entry point below replaces one call
 * of that API (cited per function), with plain pointers, sizes and a CUDA
 * stream handle passed as `void*` (cudaStream_t), so a ctypes / cgo / JNI
 * binding needs no CUDA or torch headers.
 *
 * Conventions (mirroring the reference's numba kernels, ed_mrdt/dynamics.py):
 *   - particles are indexed per replica 0..N_r-1 ("particle index"), exactly
 *     as ParticleState orders them (ed_mrdt/particles.py:80-187);
 *   - positions are float64 [N][2] in µm, species int32, flags uint8;
 *   - every entry point returns 0 on success and a negative EDM_E* code on
 *     failure; edm_last_error() describes the last failure of this thread;
 *   - runtime overflow (photon buffer, Hill-table range, pair caps) never
 *     truncates silently: it sets a bit in the engine's status word
 *     (EDM_STATUS_*), readable with edm_get_status().
 */
#ifndef EDM_B200_H
#define EDM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EDM_ABI_VERSION 3

/* ---- fixed capacities of the parameter blocks --------------------------- */
#define EDM_MAX_SPECIES 16
#define EDM_MAX_BIND 4
#define EDM_MAX_CAT 8
#define EDM_MAX_EXCH 8
#define EDM_MAX_CONV 8
#define EDM_MAX_GRIDS 8
#define EDM_MAX_RULES 24
#define EDM_MAX_REGIONS 8
#define EDM_MAX_FLUO 4
#define EDM_MAX_FRET 4
#define EDM_MAX_FCLASS 8

/* ---- error codes -------------------------------------------------------- */
#define EDM_OK 0
#define EDM_EINVAL -1   /* bad argument / inconsistent parameters           */
#define EDM_ECUDA -2    /* a CUDA runtime call failed                       */
#define EDM_ENOMEM -3   /* device allocation failed                         */
#define EDM_EUNSUP -4   /* feature not supported by this build              */
#define EDM_ERANGE -5   /* a value does not fit the requested width          */

/* ---- status bits (sticky, per engine) ------------------------------------ */
#define EDM_STATUS_PHOTON_CAP 0x1u     /* photon stream reached max_photons (reference truncates too) */
#define EDM_STATUS_HILL_RANGE 0x2u     /* density count beyond the exact Hill table: device pow used   */
#define EDM_STATUS_FORCE_TERMS 0x4u    /* >EDM_MAX_FORCE_TERMS force terms on one particle             */
#define EDM_STATUS_NONFINITE 0x8u      /* a non-finite position was produced                            */
#define EDM_STATUS_BIND_CAP 0x10u      /* binding candidate buffer overflow                             */
#define EDM_STATUS_RECRUIT_CAP 0x20u   /* recruitment candidate buffer overflow                         */
#define EDM_STATUS_POISSON_NORMAL 0x40u /* a Poisson mean >= 30 used the normal approximation            */
#define EDM_STATUS_CONTACT_CAP 0x80u   /* catalytic contact buffer overflow (events may be missed)      */

/* ---- noise streams (Philox key = seed; counter = (a, b, step, stream)) --- */
enum EdmStream {
  EDM_S_BD_NORMAL = 1,        /* standard_normal((N,2))          dynamics.py:2194 */
  EDM_S_BIND = 16,            /* + 2r: random(M) per binding r   dynamics.py:2207 */
  EDM_S_DISSOC = 17,          /* + 2r: random(N)                 dynamics.py:2219 */
  EDM_S_CAT = 32,             /* + c : random(M) per catalytic   dynamics.py:2246 */
  EDM_S_EX_ACCEPT = 48,       /* + 4e: random(N)                 dynamics.py:2301 */
  EDM_S_EX_POS = 49,          /* + 4e: random((N,2))             dynamics.py:2302 */
  EDM_S_EX_LOC = 50,          /* + 4e: random(N) (local recruit) dynamics.py:2372 */
  EDM_S_EX_DETACH = 51,       /* + 4e: random(N)                 dynamics.py:2407 */
  EDM_S_EX_OFFSET = 96,       /* + e : standard_normal((N,2))    dynamics.py:2373 */
  EDM_S_CONV = 80,            /* + v : random(N)                 dynamics.py:2438 */
  EDM_S_PH_POISSON = 112,     /* random(N)            photophysics.py:1136 */
  EDM_S_PH_TRANS = 113,       /* random(N)            photophysics.py:1137 */
  EDM_S_PH_ARRIVAL = 114,     /* random(est_photons)  photophysics.py:1145 */
  EDM_S_SC_QE = 120,          /* random(n_ph)         microscope.py:848 */
  EDM_S_SC_ASSIGN = 121,      /* random(n_surv)       microscope.py:378 */
  EDM_S_SC_JITTER = 122,      /* normal(0,σ,n)        microscope.py:743 */
  EDM_S_SC_DARK = 123,        /* poisson per pixel    microscope.py:871 */
  EDM_S_SC_DARK_BIN = 124,    /* integers per count   microscope.py:874 */
  EDM_S_SC_AP = 125,          /* binomial per pixel   microscope.py:915 */
  EDM_S_SC_AP_BIN = 126       /* integers per count   microscope.py:917 */
};

/* ---- dynamics parameter block (one per replica) -------------------------- */
typedef struct {
  int32_t sensor;        /* species counted                                   */
  int32_t nx, ny;        /* grid dims, max(3, int(L/res)) (dynamics.py:1958)  */
  int32_t pad;
  double sx, sy;         /* cell sizes L/n                                    */
  int64_t offset;        /* start of this grid in the global count array      */
  double inv_sx, inv_sy; /* 1/sx, 1/sy (division-free cell index, f32 path)   */
} EdmGrid;

typedef struct {
  int32_t grid;          /* index into EdmDynParams.grid                      */
  int32_t inhibition;    /* 1: 1/(1+r^n); 0: a+(1-a) r^n/(1+r^n)              */
  int32_t table_len;     /* exact Hill factors for counts 0..table_len-1      */
  int32_t pad;
  int64_t table_offset;  /* into the engine's hill table (float64)            */
  double K_half, n_hill, basal, inv_area;
} EdmRule;

typedef struct {
  int32_t ra, rb, product, pad;
  double contact_sq;     /* sigma_eff^2 (dynamics.py:1900-1951)               */
  double prob_bind, prob_dissoc;
} EdmBind;

typedef struct {
  int32_t enzyme, substrate, product, rule;  /* rule -1: no feedback          */
  double contact_sq, prob;
} EdmCat;

typedef struct {
  int32_t species, max_recruits;
  int32_t rule_on, rule_on2, rule_off;      /* -1 when absent                 */
  int32_t local_recruit; /* 1: density-biased positions (dynamics.py:1115-1217) */
  double prob_on, prob_off;
} EdmExch;

typedef struct {
  int32_t from, to, rule, pad;
  double prob;
} EdmConv;

enum EdmDField { EDM_DFIELD_NONE = 0, EDM_DFIELD_REGIONS = 1, EDM_DFIELD_SINE_X = 2 };

typedef struct {
  /* domain / time */
  double Lx, Ly, dt;
  int32_t periodic_x, periodic_y;
  /* cell list (dynamics.py:89-114, 1738-1788) */
  int32_t nx, ny;
  double cell_sx, cell_sy, cutoff_sq;
  /* replica slices of the engine's global arrays; a replica owns nx*ny + 1
   * sort buckets: its cells, then one bucket for non-alive particles */
  int64_t particle_offset, n_particles;
  int64_t cell_offset;
  int64_t grid_cells;    /* total density-grid cells of this replica          */
  /* BD (dynamics.py:323-406, 1837-1864) */
  double max_disp, max_disp_sq;
  double force_range_sq; /* max over species pairs of the squared force range */
  double force_reach;    /* sqrt(min(force_range_sq, cutoff_sq)) * 1.0001 + 1e-9 */
  int32_t use_wca, use_harmonic, n_species, dfield;
  double D_base[EDM_MAX_SPECIES];
  double sigma[EDM_MAX_SPECIES * EDM_MAX_SPECIES];
  double eps[EDM_MAX_SPECIES * EDM_MAX_SPECIES];
  double kharm[EDM_MAX_SPECIES * EDM_MAX_SPECIES];
  /* D(x) field */
  int32_t n_regions, pad0;
  double reg_cx[EDM_MAX_REGIONS], reg_cy[EDM_MAX_REGIONS];
  double reg_r[EDM_MAX_REGIONS], reg_f[EDM_MAX_REGIONS];
  double smooth_w;
  double sine_amp, sine_wavelength;  /* D = D0 (1 + amp sin(2 pi x / wl))   */
  /* reactions, in the reference's pass order */
  int32_t n_bind, n_cat, n_exch, n_conv, n_grids, n_rules;
  EdmBind bind[EDM_MAX_BIND];
  EdmCat cat[EDM_MAX_CAT];
  EdmExch exch[EDM_MAX_EXCH];
  EdmConv conv[EDM_MAX_CONV];
  EdmGrid grid[EDM_MAX_GRIDS];
  EdmRule rule[EDM_MAX_RULES];
  /* adaptation field (dynamics.py:1093-1112, 2078-2096, 2227-2242):
   * adapt_grid = the grid counting PIP3 on the 1 µm adaptation grid, -1 off;
   * catalytic reaction c is modulated when bit c of adapt_cat_mask is set */
  int32_t adapt_grid, adapt_cat_mask;
  double adapt_inv_tau;  /* dt / tau_w                                        */
  double adapt_K, adapt_n;
  double adapt_inv_area; /* 1 / (cell_sx cell_sy) of the adaptation grid      */
  double recruit_sigma;  /* Gaussian spread of local recruitment (µm)         */
  /* noise key */
  uint64_t seed;
} EdmDynParams;

/* ---- photophysics parameter block (photophysics.py:690-887) ------------- */
typedef struct {
  int32_t mode;          /* 0 bond, 1 proximity                               */
  int32_t donor_fid, acceptor_fid, intramolecular;
  int32_t cls_bound;     /* FRET class of a bonded donor (bond mode)          */
  int32_t cls_high, cls_low;  /* proximity mode classes                       */
  int32_t target_species;
  double prox_radius_sq;
} EdmFret;

typedef struct {
  int32_t n_fluoro, n_fret;
  int32_t ground[EDM_MAX_FLUO], excited[EDM_MAX_FLUO], t1[EDM_MAX_FLUO], bl[EDM_MAX_FLUO];
  /* per (fluorophore, pss state 0/1, FRET class): class 0 = no FRET */
  double mean_d[EDM_MAX_FLUO][2][EDM_MAX_FCLASS];
  double mean_f[EDM_MAX_FLUO][2][EDM_MAX_FCLASS];
  double exp_neg_d[EDM_MAX_FLUO][2][EDM_MAX_FCLASS];  /* exp(-mean), host libm */
  double exp_neg_f[EDM_MAX_FLUO][2][EDM_MAX_FCLASS];
  double T00[EDM_MAX_FLUO][2][EDM_MAX_FCLASS];
  double T0001[EDM_MAX_FLUO][2][EDM_MAX_FCLASS];      /* T00 + T01          */
  double tau[EDM_MAX_FLUO][EDM_MAX_FCLASS];           /* tau_DA per class   */
  /* exact FRET efficiency k tau_D / (1 + k tau_D) per class (0 without
   * FRET), pipeline.py:410-416 */
  double fret_E[EDM_MAX_FLUO][EDM_MAX_FCLASS];
  /* 1 when the fluorophore is the donor of some FRET pair with a finite
   * positive lifetime: its particles get ground-truth E and tau_DA */
  int32_t gt_donor[EDM_MAX_FLUO];
  double tau_all[EDM_MAX_FLUO];
  int32_t has_fret_cls[EDM_MAX_FCLASS];               /* k_fret > 0         */
  EdmFret fret[EDM_MAX_FRET];
  int32_t donor_channel, acceptor_channel;            /* photophysics.py:782-787 */
  int64_t max_photons, est_photons;
  int64_t photon_offset; /* start of this replica's slice of the photon buffer */
  int64_t emitter_offset, n_emitters;
} EdmPhotParams;

/* ---- microscope parameter block (microscope.py:73-1233) ------------------ */
typedef struct {
  int32_t nx, ny, n_bins, n_channels;   /* n_channels = max(2, n_fluoro)      */
  int32_t psf_range_px, n_sigma;
  double pixel_size, offset_x, offset_y;
  double bin_width, sigma_irf, qe;
  double sigma_ch[EDM_MAX_FLUO];        /* with the reference's fallbacks     */
  double inv_2sig2_ch[EDM_MAX_FLUO];    /* 0.5/(sigma*sigma)                  */
  double dark_lambda, dark_exp_neg;     /* dark_rate*dwell, exp(-lambda)      */
  double ap_prob;
  int64_t flim_offset;   /* start of this replica's stack (uint32 elements)   */
} EdmScopeParams;

/* ---- host-side particle state (id order, replicas concatenated) --------- */
typedef struct {
  int64_t n;             /* total particles over all replicas                 */
  double* positions;     /* [n][2]                                            */
  int32_t* species_id;
  uint8_t* is_alive;
  int32_t* bond_partner; /* replica-local particle index, -1 = free           */
  uint8_t* has_dye;
  int32_t* dye_type_id;
  int8_t* ctmc_state;
  uint8_t* is_bleached;
} EdmHostState;

/* per-replica counters, EDM_NCOUNTERS int64 each */
enum EdmCounter {
  EDM_C_BINDINGS = 0, EDM_C_DISSOC, EDM_C_CATALYTIC, EDM_C_RECRUITED,
  EDM_C_DETACHED, EDM_C_CONVERTED,
  EDM_C_PHOTONS, EDM_C_DONOR_PH, EDM_C_ACCEPTOR_PH, EDM_C_FRET_PH,
  EDM_C_DETECTED, EDM_C_DARK, EDM_C_AFTERPULSE, EDM_C_RECEIVED,
  EDM_NCOUNTERS
};

typedef struct EdmEngine EdmEngine;

/* ---- versioning / layout checks ----------------------------------------- */
int edm_abi_version(void);
/* sizeof of the ABI structs: which = 0 EdmDynParams, 1 EdmPhotParams,
 * 2 EdmScopeParams, 3 EdmHostState, 4 EdmFlimParams; lets a binding verify
 * its mirror. */
int64_t edm_abi_sizeof(int which);
const char* edm_last_error(void);

/* ---- engine lifetime ------------------------------------------------------
 * Replaces DynamicsEngine.__init__ + PhotonSimulator.__init__ +
 * VirtualMicroscope.__init__ (dynamics.py:1724, photophysics.py:693,
 * microscope.py:1045): the host derives every float64 constant exactly as
 * the reference does and hands the blocks over; the engine allocates device
 * memory for all replicas.  precision: 64 = plain float64 path (absolute
 * positions), 32 = float32 cell-relative path.  hill: exact Hill factors,
 * indexed by EdmRule.table_offset.  phot/scope may be NULL (dynamics only). */
int edm_create(const EdmDynParams* dyn, const EdmPhotParams* phot,
               const EdmScopeParams* scope, int32_t n_replicas,
               const double* hill, int64_t n_hill, int32_t precision,
               int32_t device, EdmEngine** out);
int edm_destroy(EdmEngine* eng);

/* Host <-> device particle state, id order (ParticleState arrays).  The
 * copies are ordered on `stream`; when the host arrays are pinned they are
 * read asynchronously, so keep them unchanged until the stream has passed
 * this call.  edm_get_state returns after the state has landed in host
 * memory. */
int edm_set_state(EdmEngine* eng, const EdmHostState* st, void* stream);
int edm_get_state(EdmEngine* eng, EdmHostState* st, void* stream);

/* The same transfers overlapped with computation, for loops that feed a new
 * state and read the result every frame.  No reference counterpart.
 * edm_set_state_async copies the host arrays into a device staging area of
 * its own on the engine's upload stream, without waiting for the work already
 * queued on `stream`, and queues the state's installation on `stream` after
 * that work.  edm_get_state_async queues the state's gathering into a second
 * staging area on `stream` and copies it to the host arrays on the engine's
 * download stream while `stream` goes on.  The host arrays should be pinned,
 * and must stay valid (set) or unread (get) until edm_state_transfers_wait
 * returns.  A set whose dye carriers differ from the last upload rebuilds the
 * emitter list on the host: it falls back to edm_set_state.  The first call
 * allocates both staging areas (2 * 28 bytes per particle). */
int edm_set_state_async(EdmEngine* eng, const EdmHostState* st, void* stream);
int edm_get_state_async(EdmEngine* eng, EdmHostState* st, void* stream);
int edm_state_transfers_wait(EdmEngine* eng);
/* edm_set_state_async in two halves, so that a frame loop can start the next
 * upload before it queues this frame's reads: edm_stage_state_async queues
 * the host-to-staging copy on the upload stream (after the previous
 * installation has left the staging; the dye carriers must equal the last
 * upload's; one staged state at a time), edm_install_state queues the
 * installation of the staged state on `stream`. */
int edm_stage_state_async(EdmEngine* eng, const EdmHostState* st);
int edm_install_state(EdmEngine* eng, void* stream);
int edm_set_step(EdmEngine* eng, int64_t step_index);
int64_t edm_get_step(EdmEngine* eng);

/* DynamicsEngine.step() x n_steps (dynamics.py:2150-2465). */
int edm_dynamics_step(EdmEngine* eng, int32_t n_steps, void* stream);

/* PhotonSimulator.evolve_one_bd_step() (photophysics.py:1116-1197) for the
 * current state; the batch stays on the device until edm_get_photons(). */
int edm_photon_step(EdmEngine* eng, void* stream);
/* Number of photons of the last batch per replica (host array [n_replicas]). */
int edm_get_photon_counts(EdmEngine* eng, int64_t* counts, void* stream);
/* Copy the last batch of one replica to host arrays (PhotonBatch fields). */
int edm_get_photons(EdmEngine* eng, int32_t replica, int32_t* particle_idx,
                    double* arrival_time, int8_t* channel, uint8_t* is_fret,
                    int64_t capacity, void* stream);

/* VirtualMicroscope.process_photons(batch) (microscope.py:1069-1157) on the
 * last device batch, each photon at its particle's position in the current
 * state (as the reference reads it from the particle state it is given). */
int edm_scope_process(EdmEngine* eng, void* stream);

/* Load a host photon batch (PhotonBatch fields, photophysics.py:184-211) of
 * one replica as the current device batch; its per-photon draws are keyed
 * by batch_key.  For batches not produced by edm_photon_step. */
int edm_set_photons(EdmEngine* eng, int32_t replica, const int32_t* particle_idx,
                    const double* arrival_time, const int8_t* channel,
                    const uint8_t* is_fret, int64_t n, int64_t batch_key,
                    void* stream);

/* One fused BD step of the whole pipeline loop body (pipeline.py:554-564):
 * dynamics step, photophysics, photon processing; n_steps times, with the
 * launch sequence captured into CUDA graphs of graph_chunk steps. */
int edm_pipeline_steps(EdmEngine* eng, int32_t n_steps, int32_t with_photons,
                       int32_t graph_chunk, void* stream);

/* VirtualMicroscope.finalize_frame() (microscope.py:1159-1203): dark counts
 * and afterpulsing into the stacks, keyed by frame_index.  Stacks stay on
 * the device; read them with edm_get_flim and clear with edm_reset_flim. */
int edm_scope_finalize(EdmEngine* eng, int64_t frame_index, void* stream);
int edm_get_flim(EdmEngine* eng, int32_t replica, uint32_t* host_out,
                 int64_t n_elems, void* stream);
int edm_reset_flim(EdmEngine* eng, void* stream);

/* Overlapped frame readout, for frame loops that read every stack.
 * edm_frame_out_begin copies the finalized stacks of all replicas into an
 * engine-owned snapshot on `stream` and clears the live stacks (what
 * edm_reset_flim does). Then, on a copy stream of the engine's own, it
 * starts reading the snapshot into host_out, so the read overlaps the work
 * `stream` does next. host_out holds edm_flim_elems() uint32 values,
 * replicas in order, each [n_ch][nx][ny][n_bins] as edm_get_flim returns
 * it; it should be pinned (page-locked) for the copy to be asynchronous.
 * A new begin first waits, on `stream`, for the previous read to leave the
 * snapshot. edm_frame_out_wait blocks until the last read has landed in
 * host memory. The first begin allocates the snapshot (n_flim * 4 bytes).
 * The read occupies the device-to-host link for n_flim * 4 bytes: issue the
 * frame's other reads (edm_get_state) before it, or they queue behind it. */
int64_t edm_flim_elems(EdmEngine* eng);
int edm_frame_out_begin(EdmEngine* eng, uint32_t* host_out, int64_t n_elems,
                        void* stream);
int edm_frame_out_wait(EdmEngine* eng);
/* Every replica's finalized stacks as their nonzero bins only: element index
 * into the concatenated stacks (edm_flim_elems() long; replica r starts at
 * its EdmScopeParams.flim_offset) and count, in index order, copied to host
 * memory; the emitted bins are cleared, so the stacks start the next frame
 * at zero as with edm_frame_out_begin.  A frame's stacks hold about one
 * photon per thousand bins at the rates of the reference's examples, so
 * this moves a few megabytes where the dense read moves gigabytes.  Returns
 * the number of nonzero bins; more than cap is an error and leaves the
 * stacks untouched.  Synchronous on `stream`.  No reference counterpart
 * (finalize_frame returns dense stacks, microscope.py:1159-1203). */
int64_t edm_frame_out_sparse(EdmEngine* eng, int64_t* idx_host, uint32_t* count_host, int64_t cap,
                             void* stream);

/* ---- census rows: sub-frame series and per-frame ground truth -------------
 * One row of EDM_CENSUS_FIELDS int64 per replica holds what the reference's
 * SimulationPipeline reads off the host state after every BD step
 * (pipeline.py:567-642, record_subframe=True) and at every frame end
 * (pipeline.py:399-442, _extract_ground_truth), reduced on the device. */
enum EdmCensusField {
  EDM_CEN_COUNTERS = 0,      /* [0, 7): counters EDM_C_BINDINGS .. EDM_C_PHOTONS (cumulative) */
  EDM_CEN_BOND_ALIVE = 7,    /* alive particles with a bond partner                            */
  EDM_CEN_BOND_ALL = 8,      /* particles with a bond partner                                  */
  EDM_CEN_BLEACHED = 9,      /* bleached particles                                             */
  EDM_CEN_SPECIES = 10,      /* [10, 26): alive particles per species                          */
  EDM_CEN_DONORS = 26,       /* alive unbleached particles carrying dye 0 (pipeline.py:596-598) */
  EDM_CEN_DONOR_CLS = 27,    /* [27, 35): those per FRET class of the step's photon pass       */
  EDM_CEN_FREE_DYE = 35,     /* [35, 39): unbleached particles with dye t and no bond partner  */
  EDM_CENSUS_FIELDS = 40
};

/* Sub-frame recorder.  With capacity_steps > 0, every later
 * edm_pipeline_steps step (eager or inside its CUDA graphs) ends with two
 * kernels that write the step's census row of every replica into a device
 * ring of capacity_steps x n_replicas rows: step s (0-based BD step index)
 * goes to ring slot s % capacity_steps.  capacity_steps = 0 stops recording
 * and frees the ring.  Changing it drops the engine's captured graphs.
 * Replaces the per-step host reductions of pipeline.py:567-642. */
int edm_record_enable(EdmEngine* eng, int32_t capacity_steps);
/* Copies the rows of steps [first_step, first_step + n_steps) to
 * host_out[n_steps][n_replicas][EDM_CENSUS_FIELDS] (host memory; pinned
 * memory makes the copy asynchronous on `stream`).  The steps must be among
 * the last capacity_steps recorded. */
int edm_record_read(EdmEngine* eng, int64_t first_step, int32_t n_steps,
                    int64_t* host_out, void* stream);
/* Per-frame ground truth (pipeline.py:357-455 after
 * PhotonSimulator.update_fret_rates, photophysics.py:1021-1114): every
 * particle's FRET class is evaluated for the current state as the reference's
 * update_fret_rates does (bond and proximity pairs, last matching pair
 * wins), and donors get E = k tau_D / (1 + k tau_D) and tau_DA =
 * tau_D / (1 + k tau_D) (others 0).  Writes fret_E[N] and tau_DA[N] (id
 * order, replicas concatenated) and census[n_replicas][EDM_CENSUS_FIELDS]
 * (counters, bonds, bleaching, species and free-donor counts) to host
 * memory on `stream`; any pointer may be NULL. */
int edm_ground_truth(EdmEngine* eng, double* fret_E, double* tau_DA,
                     int64_t* census, void* stream);

/* ---- launch-shape autotuner ------------------------------------------------
 * No reference counterpart.  For each tuned kernel (k_scatter, k_move,
 * k_contacts, in that order) runs every candidate launch shape (threads per
 * block, minimum resident blocks per SM, which bounds registers per thread)
 * for 1 + steps_per_shape eager dynamics steps, times the kernel alone with
 * CUDA events on `stream` and keeps the fastest.  The steps are real steps:
 * every shape computes the same state, so tuning is simply the first steps
 * of a run.  Choices are cached per (kernel, precision, replicas, log2 of the
 * particle count) for the rest of the process and applied to later engines
 * of the same kind, unless retune != 0.  Drops the engine's captured graphs. */
int edm_autotune(EdmEngine* eng, int32_t steps_per_shape, int32_t retune, void* stream);
/* The launch shape in use per tuned kernel: shapes[k][4] = (threads per block,
 * minimum blocks per SM, candidates, chosen candidate; k_scatter candidates
 * 3-4 give a thread two slots, the others one; k_contacts candidate 0
 * gives a thread a whole sweeper, 1-2 give each lane one neighbour column of
 * a sweeper within a warp, 3-5 within a block, 6-7 over a global sweeper
 * list), ms[k][2] = (time of the default shape, time of the chosen shape) from
 * the last tuning (0 if not tuned).  Either pointer may be NULL.  Returns the
 * number of tuned kernels (3). */
int edm_launch_shapes(EdmEngine* eng, int32_t* shapes, float* ms);
/* Sets the launch shape of each tuned kernel: candidate[k] in
 * [0, candidates of k), or -1 to keep it (a profiler run, where timings mean
 * nothing, replays the shapes a plain run tuned).  Drops the captured graphs. */
int edm_set_launch_shapes(EdmEngine* eng, const int32_t* candidate);

/* Sides of the catalytic contact sweep.  No reference counterpart.  The
 * pairs (enzyme, partner holding the substrate at the step start) of each
 * catalytic reaction are found by sweeping from one side: bit c of the mask
 * set = from the enzyme species, clear = from the substrate species (both
 * find the same pairs; the choice changes only the work).  The first
 * edm_set_state picks the side with fewer alive particles per reaction.
 * force_mask >= 0 sets the sides (bits at or above the reaction count are
 * ignored; later states do not change them) and drops the captured graphs;
 * force_mask < 0 changes nothing.  Returns the mask in use. */
int edm_contact_sides(EdmEngine* eng, int32_t force_mask);

/* Counters [n_replicas][EDM_NCOUNTERS] and the sticky status word. */
int edm_get_counters(EdmEngine* eng, int64_t* out, void* stream);
int edm_get_status(EdmEngine* eng, uint32_t* status, void* stream);

/* Instrumented steps: captures two pipeline steps into a CUDA graph with
 * event-record nodes around each kernel group, replays it until n_steps
 * steps (rounded up to even) have run, and writes the mean device time per
 * step (ms) of ms_out[EDM_NPROF]: cell-list scan, scatter, force+move,
 * reaction passes, photophysics, photon detection, whole step.  The groups
 * are timed as they run inside the pipeline's graphs; the stream must not be
 * the legacy default stream.  No reference counterpart. */
#define EDM_NPROF 7
int edm_profile_steps(EdmEngine* eng, int32_t n_steps, int32_t with_photons,
                      float* ms_out, void* stream);
/* Instrumented eager dynamics steps: runs n_steps dynamics steps with CUDA
 * events between the reaction passes and writes, per pass of the step's
 * schedule, its mean device time (ms) to ms_out[k] and its kind to
 * kinds_out[k] = 100 * kind + index (kind 0 binding candidates, 1 binding
 * apply, 2 dissociation, 3 catalytic contacts, 4 catalytic pass, 6
 * recruitment apply, 9 grid merge, 10 run of recruitment-candidate,
 * detachment and conversion passes over the listed particles, 11 the draw
 * sweep that lists them, 12 adaptation-field update, 13 local-recruitment
 * CDF).  Returns the number of passes (at most
 * cap) or a negative error.  No reference counterpart. */
int edm_profile_passes(EdmEngine* eng, int32_t n_steps, float* ms_out,
                       int32_t* kinds_out, int32_t cap, void* stream);
/* Kernels of this library launched per pipeline step. */
int edm_launches_per_step(EdmEngine* eng, int32_t with_photons);

/* Device pointer to the cell-list arrays of the last dynamics step
 * (CellList.head/next equivalent, dynamics.py:109-138): per replica cell c
 * holds particle indices sorted[start[c] .. start[c+1]) (global indices).  */
int edm_get_cells(EdmEngine* eng, int32_t replica, int32_t* cell_start,
                  int32_t* members, int64_t cap_cells, int64_t cap_members,
                  void* stream);

/* ---- allocation-free cell list ------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory when they call: code that runs inside a pre-sized device memory
 * pool or arena owned by a host framework, a process whose device memory is
 * already handed to another allocator, or a tight loop where cudaMalloc (which
 * may synchronise the device) is not acceptable.
 *
 * Builds the cell list of n caller-owned device positions [n][2] (x, y) on
 * an nx x ny grid over the box [0, Lx) x [0, Ly): cell side = box side /
 * cells, cx = trunc(x / side_x) and cy = trunc(y / side_y), each clamped into
 * the grid (so points outside the box land in the edge cells), cell key
 * cx*ny + cy.  Output: cell_start_dev[nx*ny + 1] and members_dev[n], the
 * particle indices of cell c in members[cell_start[c] .. cell_start[c+1]),
 * ascending.  The work is bounded for any occupancy, including every point in
 * one cell.  It allocates nothing: its scratch is one static device array of
 * about 8 MB (EDM_STATIC_MAX_CELLS-sized counters) that every GPU loading
 * this library holds until the process exits.  nx*ny beyond
 * EDM_STATIC_MAX_CELLS or n beyond EDM_STATIC_MAX_PARTICLES is rejected with
 * EDM_EINVAL.  The first call on a device looks up that array's device
 * address (cudaGetSymbolAddress), so make it before any stream capture.  All
 * calls share the one array: calls that overlap on the GPU race; order them
 * on one stream.  Each call clears what must start at zero. */
#define EDM_STATIC_MAX_PARTICLES (1 << 24)
#define EDM_STATIC_MAX_CELLS (1 << 20)
int edm_cell_list_static(const double* positions_dev, int64_t n, double Lx,
                         double Ly, int32_t nx, int32_t ny,
                         int32_t* cell_start_dev, int32_t* members_dev,
                         void* stream);

/* ---- batched FLIM acquisition from expected intensities ----------------
 * No reference function: the reference forms FLIM stacks photon by photon
 * (VirtualMicroscope.process_photons, microscope.py:1069-1157).  This path
 * takes its pieces from there: the emitter-centric Gaussian PSF with a
 * (2R+1)^2 window renormalised over in-field pixels (microscope.py:522-631),
 * TCSPC bins with negative times in bin 0 and late ones lost
 * (microscope.py:716-803), Gaussian IRF, photon yields and lifetimes of the
 * per-pulse chain (photophysics.py:218-331, computed on the host).
 * For each replica: n_emitters donors at keyed uniform pixels, each bound
 * (FRET) with the replica's bound fraction; intensity maps
 * I = G . counts . G^T on tcgen05 BF16 GEMMs; then per pixel and bin a
 * Poisson count of mean I_free h_free[b] yield_free + I_bound h_bound[b]
 * yield_bound, written as uint32 [replica][x][y][bin]. */
typedef struct EdmFlimParams {
  int32_t nx, ny;          /* pixels per side; 256 x 256 only                   */
  int32_t n_replicas;      /* 1 .. 4096                                         */
  int32_t n_emitters;      /* per replica                                        */
  int32_t n_bins;          /* 128 or 256                                         */
  int32_t half_taps;       /* R: PSF window half-width in pixels (2R+1 taps)    */
  uint64_t seed;
  double bin_width_ns, sigma_irf_ns;
  double sigma_psf_px;     /* PSF sigma in pixels                                */
  double tau_free_ns, tau_bound_ns;
  double yield_free, yield_bound; /* expected detected photons per emitter     */
} EdmFlimParams;

/* Seed of replica r: the acquisition seed mixed with r (also used by hosts
 * that reproduce the emitter draws). */
#if defined(__CUDACC__)
#define EDM_HOST_DEVICE __host__ __device__
#else
#define EDM_HOST_DEVICE
#endif
static inline EDM_HOST_DEVICE uint64_t edm_flim_replica_seed(uint64_t seed, int32_t r) {
  return seed ^ (0x9E3779B97F4A7C15ull * (uint64_t)(r + 1));
}

enum EdmFlimArray {
  EDM_FLIM_HIST = 0,      /* uint32 [R][nx][ny][n_bins]                        */
  EDM_FLIM_INTENSITY = 1, /* float  [R][free, bound][nx][ny]                   */
  EDM_FLIM_COUNTS = 2,    /* int32  [R][free, bound][nx][ny] emitter counts    */
  EDM_FLIM_TAU = 3,       /* double [R][nx][ny] expected mean arrival time, ns */
  EDM_FLIM_BINS = 4,      /* double [free, bound][n_bins] bin probabilities    */
  EDM_FLIM_ERROR = 5      /* uint32 error word (EDM_FLIM_ERR_*)                */
};
#define EDM_FLIM_ERR_LOAD_WAIT 0x1u /* a GEMM stage load did not arrive in time  */
#define EDM_FLIM_ERR_DONE_WAIT 0x2u /* a GEMM accumulator did not complete       */
#define EDM_FLIM_ERR_COUNT 0x4u     /* > 256 emitters in one pixel (bf16 inexact) */

typedef struct EdmFlim EdmFlim;
/* Allocates every device array (histograms: R * nx * ny * n_bins * 4 bytes)
 * and computes the PSF band and bin probabilities. */
int edm_flim_create(const EdmFlimParams* params, int32_t device, EdmFlim** out);
int edm_flim_destroy(EdmFlim* flim);
/* Host bound fractions (n_replicas doubles) and the seed of the next
 * acquisition; the copy is ordered on `stream`. */
int edm_flim_set_inputs(EdmFlim* flim, const double* bound_fraction_host,
                        uint64_t seed, void* stream);
/* Emitter maps and intensity maps (the two GEMMs). */
int edm_flim_project(EdmFlim* flim, void* stream);
/* Poisson histograms from the intensity maps; with_tau also writes the
 * expected mean arrival time per pixel. */
int edm_flim_histograms(EdmFlim* flim, int32_t with_tau, void* stream);
/* project + histograms (with tau). */
int edm_flim_acquire(EdmFlim* flim, void* stream);
/* Device pointer and size in bytes of one of the EdmFlimArray arrays. */
int edm_flim_device_ptr(EdmFlim* flim, int32_t what, void** out, int64_t* bytes);
/* Copies array `what` (one replica's part when replica >= 0 and the array
 * is per replica, else all of it) to host memory and waits for `stream`. */
int edm_flim_read(EdmFlim* flim, int32_t what, int32_t replica,
                  void* host_out, int64_t bytes, void* stream);
int edm_flim_get_error(EdmFlim* flim, uint32_t* word);
/* The histograms (EDM_FLIM_HIST: all replicas, or one when replica >= 0) read
 * as `bits`-bit counts, bits = 8 or 16, narrowed on the device so 1/4 or 1/2
 * of the uint32 bytes cross the link; host_out holds one uint8 / uint16 per
 * bin, in the uint32 array's order.  Lossless or nothing: returns EDM_ERANGE
 * (host_out then undefined) when some count exceeds 2^bits - 1, and the caller
 * reads wider.  The first call allocates a device buffer for the narrow copy.
 * Waits for `stream`. */
int edm_flim_read_hist_narrow(EdmFlim* flim, int32_t replica, int32_t bits,
                              void* host_out, int64_t bytes, void* stream);
/* The same read of every replica's histograms, overlapped with what `stream`
 * does next: narrows on `stream` and waits for the overflow check (EDM_ERANGE
 * as above, before any copy), then copies the narrow array to host_out (one
 * byte or two per bin, pinned memory) on a copy stream of the handle's own
 * and returns; the next acquisition may start at once.  A new read (or a
 * narrow read) waits, on `stream`, for the previous copy to leave the device
 * buffer; edm_flim_read_wait blocks until the last copy has landed. */
int edm_flim_read_hist_narrow_async(EdmFlim* flim, int32_t bits, void* host_out,
                                    int64_t bytes, void* stream);
int edm_flim_read_wait(EdmFlim* flim);

/* ---- lifetime readouts of TCSPC stacks (analysis.py:87-150, 497-566) ----
 * For a device stack [n_px][n_bins] of uint32 counts (an engine stack from
 * edm_flim_stack_ptr, or EDM_FLIM_HIST of an acquisition), writes float64
 * out_dev[6][n_px]: intensity, mean arrival time (ns; NaN below
 * min_counts_mean), phasor g and s of the given harmonic (0 below
 * min_counts_phasor), phase and modulation lifetimes (ns; NaN where the
 * reference leaves them NaN).  n_bins: a multiple of 4, at most 256; the
 * stack 16-byte aligned. */
int edm_readout_lifetimes(const uint32_t* stack_dev, int64_t n_px, int32_t n_bins,
                          double time_range_s, int32_t harmonic,
                          int32_t min_counts_mean, int32_t min_counts_phasor,
                          double* out_dev, void* stream);
/* Device address of replica `replica`'s stack [n_ch][nx][ny][n_bins] and its
 * pixel count n_ch * nx * ny. */
int edm_flim_stack_ptr(EdmEngine* eng, int32_t replica, void** ptr,
                       int64_t* n_px, int32_t* n_bins);

/* Noise of the engine's generator, for injection into the reference:
 * writes n keyed standard normals pairs (2n doubles) / uniforms.  The
 * arrays are device pointers; keys a[i] (particle / photon index). */
int edm_noise_normal_pairs(uint64_t seed, int64_t step, int32_t stream_id,
                           const int64_t* keys_dev, int64_t n, double* out_dev,
                           void* stream);
int edm_noise_uniforms(uint64_t seed, int64_t step, int32_t stream_id,
                       const int64_t* keys_a_dev, const int64_t* keys_b_dev,
                       int64_t n, double* out2_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* EDM_B200_H */
