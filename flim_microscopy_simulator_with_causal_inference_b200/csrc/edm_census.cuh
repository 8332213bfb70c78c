// edm_census.cuh — device reductions the reference's SimulationPipeline takes
// on the host: the per-BD-step sub-frame record (pipeline.py:567-642) and the
// per-frame ground truth (pipeline.py:357-455).
//
// A census row (EDM_CENSUS_FIELDS int64 per replica, fields EdmCensusField)
// holds integer counts only; the host turns them into the reference's
// series (deltas of cumulative counters, complexes = bonded / 2, mean FRET
// efficiency from the donor counts per FRET class).  Rows are either one
// fixed block (ground truth) or a ring indexed by the BD step just finished
// (sub-frame record), so the recorder needs no host input inside a CUDA
// graph: it reads the device step counter.
#pragma once

#include "edm_phot.cuh"

namespace edm {

// Row of replica r: the fixed block when cap == 0, else ring slot
// (step just finished) % cap.
__device__ __forceinline__ int64_t* census_row(int64_t* base, int cap, const int64_t* d_step, int n_rep, int r) {
  if (cap <= 0) return base + (int64_t)r * EDM_CENSUS_FIELDS;
  const int64_t slot = (*d_step - 1) % cap;
  return base + (slot * n_rep + r) * EDM_CENSUS_FIELDS;
}

// Clear every replica's row and copy the cumulative event and photon
// counters (EDM_C_BINDINGS .. EDM_C_PHOTONS are fields 0-6).
__global__ void k_census_begin(int64_t* base, int cap, const int64_t* __restrict__ d_step, int n_rep,
                               const int64_t* __restrict__ counters) {
  const int64_t n = (int64_t)n_rep * EDM_CENSUS_FIELDS;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / EDM_CENSUS_FIELDS), f = (int)(i % EDM_CENSUS_FIELDS);
    census_row(base, cap, d_step, n_rep, r)[f] =
        f < EDM_CEN_BOND_ALIVE ? counters[(int64_t)r * EDM_NCOUNTERS + EDM_C_BINDINGS + f] : 0;
  }
}

// Per slot: bonded (alive / all), bleached, alive per species.  One block
// covers kBlock slots of one replica: warp ballots into shared counters,
// then one global add per non-zero field.
__global__ void __launch_bounds__(kBlock) k_census_particles(const EdmDynParams* __restrict__ P,
                                                             const int2* __restrict__ blk, DevState st,
                                                             const uint8_t* __restrict__ bleached, int64_t* base,
                                                             int cap, int n_species) {
  constexpr int kFields = EDM_CEN_SPECIES + EDM_MAX_SPECIES;
  __shared__ int acc[kFields];
  for (int i = threadIdx.x; i < kFields; i += blockDim.x) acc[i] = 0;
  __syncthreads();
  const Tile t = tile_of(blk);
  const EdmDynParams& p = P[t.r];
  const bool in = t.s < p.particle_offset + p.n_particles;
  bool alive = false, bonded = false, bl = false;
  int sp = -1;
  if (in) {
    const uint8_t f = st.flags[t.s];
    alive = fl_alive(f);
    sp = fl_species(f);
    const int id = st.ids[t.s];
    bonded = st.bond[id] >= 0;
    bl = bleached != nullptr && bleached[id] != 0;
  }
  const int lane = threadIdx.x & 31;
  const unsigned ba = __ballot_sync(0xffffffffu, alive && bonded);
  const unsigned b = __ballot_sync(0xffffffffu, bonded);
  const unsigned bb = __ballot_sync(0xffffffffu, bl);
  if (lane == 0) {
    if (ba) atomicAdd(&acc[EDM_CEN_BOND_ALIVE], __popc(ba));
    if (b) atomicAdd(&acc[EDM_CEN_BOND_ALL], __popc(b));
    if (bb) atomicAdd(&acc[EDM_CEN_BLEACHED], __popc(bb));
  }
  const int key = alive && sp < EDM_MAX_SPECIES ? sp : -1;
  const unsigned peers = __match_any_sync(0xffffffffu, key);
  if (key >= 0 && lane == __ffs(peers) - 1) atomicAdd(&acc[EDM_CEN_SPECIES + key], __popc(peers));
  __syncthreads();
  int64_t* row = census_row(base, cap, st.d_step, st.n_rep, t.r);
  for (int i = EDM_CEN_BOND_ALIVE + threadIdx.x; i < EDM_CEN_SPECIES + n_species; i += blockDim.x)
    if (acc[i]) atomicAdd((unsigned long long*)&row[i], (unsigned long long)acc[i]);
}

// Per dye-carrying particle (the emitter list): the alive unbleached carriers
// of dye 0 (the reference's donors of pipeline.py:596-598), those per FRET
// class of the step's photon pass (with_cls), and the unbleached carriers of
// each dye without a bond partner (pipeline.py:425-437).
__global__ void __launch_bounds__(kBlock) k_census_emitters(const EdmPhotParams* __restrict__ PP,
                                                            const int2* __restrict__ eblk, DevState st, PhotState ph,
                                                            int64_t* base, int cap, int with_cls) {
  __shared__ int acc[EDM_CENSUS_FIELDS];
  for (int i = threadIdx.x; i < EDM_CENSUS_FIELDS; i += blockDim.x) acc[i] = 0;
  __syncthreads();
  const Tile t = tile_of(eblk);
  const EdmPhotParams& pp = PP[t.r];
  if (t.s < pp.emitter_offset + pp.n_emitters) {
    const int gid = ph.emit_id[t.s];
    const bool alive = fl_alive(st.flags[st.slot_of_id[gid]]);
    const bool hd = ph.has_dye[gid] != 0, bl = ph.bleached[gid] != 0;
    const int dye = ph.dye[gid];
    if (hd && alive && !bl && dye == 0) {
      atomicAdd(&acc[EDM_CEN_DONORS], 1);
      const int cls = ph.emit_cls[t.s];
      if (with_cls && cls >= 0 && cls < EDM_MAX_FCLASS) atomicAdd(&acc[EDM_CEN_DONOR_CLS + cls], 1);
    }
    if (hd && !bl && st.bond[gid] < 0 && dye >= 0 && dye < EDM_MAX_FLUO) atomicAdd(&acc[EDM_CEN_FREE_DYE + dye], 1);
  }
  __syncthreads();
  int64_t* row = census_row(base, cap, st.d_step, st.n_rep, t.r);
  for (int i = EDM_CEN_DONORS + threadIdx.x; i < EDM_CENSUS_FIELDS; i += blockDim.x)
    if (acc[i]) atomicAdd((unsigned long long*)&row[i], (unsigned long long)acc[i]);
}

// Ground-truth FRET efficiency and donor lifetime of every unbleached
// carrier of a donor dye (pipeline.py:385-416), with the FRET class of the
// current state (update_fret_rates, photophysics.py:1021-1114).  E and
// tau_DA come from the host's float64 tables of the reference's expressions.
template <bool F64>
__global__ void __launch_bounds__(kBlock) k_ground_truth(const EdmDynParams* __restrict__ DP,
                                                         const EdmPhotParams* __restrict__ PP,
                                                         const int2* __restrict__ eblk, DevState st, PhotState ph,
                                                         int cells_valid, double* __restrict__ fret_E,
                                                         double* __restrict__ tau_DA) {
  const Tile t = tile_of(eblk);
  const EdmPhotParams& pp = PP[t.r];
  if (t.s >= pp.emitter_offset + pp.n_emitters) return;
  const int gid = ph.emit_id[t.s];
  if (!ph.has_dye[gid] || ph.bleached[gid]) return;
  const int dt = ph.dye[gid];
  if (dt < 0 || dt >= pp.n_fluoro || !pp.gt_donor[dt]) return;
  const int64_t slot = st.slot_of_id[gid];
  const bool alive = fl_alive(st.flags[slot]);
  int acc = -1;
  const int cls = fret_class<F64>(DP[t.r], pp, st, ph, t.r, gid, slot, dt, alive, cells_valid, acc);
  fret_E[gid] = pp.fret_E[dt][cls];
  tau_DA[gid] = pp.tau[dt][cls];
}

}  // namespace edm
