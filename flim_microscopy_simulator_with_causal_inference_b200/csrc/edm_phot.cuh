// edm_phot.cuh — photophysics (PhotonSimulator.evolve_one_bd_step,
// ed_mrdt/photophysics.py:338-521, 1021-1197) and photon detection
// (VirtualMicroscope.process_photons / finalize_frame,
// ed_mrdt/microscope.py:522-631, 716-803, 839-922, 1069-1203).
//
// The reference's photon stream is serial: emitters in particle order, each
// emitting its donor photons then its FRET-acceptor photons, one shared
// arrival-time cursor.  Here every emitter draws its counts independently
// (keyed by particle index), an exclusive scan over emitters in particle
// order gives each photon its stream index k, and every per-photon draw is
// keyed by k.  Photons beyond the reference's buffer (max_photons) are
// dropped exactly as its `break` drops them; arrival draws beyond its
// est_photons stream fall back to t = tau as it does.
#pragma once

#include "edm_dyn.cuh"

namespace edm {

constexpr int kPsfMaxR = 16;  // largest PSF window half-width in pixels (4 sigma / pixel, rounded up)

// Mark the 128-element stretch of the stacks holding element e as touched
// (the sparse readout visits only touched stretches).
__device__ __forceinline__ void touch_stretch(uint32_t* touch, int64_t e) {
  if (touch) atomicOr(&touch[e >> 12], 1u << ((e >> 7) & 31));
}

struct PhotState {
  const int32_t* emit_id;   // global particle id of each emitter (particle order per replica)
  int32_t* emit_n;          // photons (donor + acceptor) of the current batch
  int32_t* emit_nd;         // donor photons
  int32_t* emit_acc;        // FRET acceptor (global id) or -1
  int8_t* emit_cls;         // FRET class
  int64_t* emit_off;        // first photon index within the replica
  const uint8_t* has_dye;   // id-indexed
  const int8_t* dye;        // id-indexed
  int8_t* ctmc;             // id-indexed
  uint8_t* bleached;        // id-indexed
  int32_t* ph_pid;          // replica-local particle index
  double* ph_t;
  int8_t* ph_ch;
  uint8_t* ph_fret;
  double2* ph_xy;           // the emitting particle's position when the photon was written
  int64_t* ph_count;        // [R] photons of the batch (after the max_photons cap)
  uint32_t* flim;
  uint32_t* touch;          // one bit per 128-bin stretch of flim that a count has landed in
  int64_t* d_pstep;         // photophysics call counter
  int64_t* d_batch_key;     // key of the last batch
};

// Poisson draw of the reference (photophysics.py:486-521): an LCG seeded from
// one uniform, Knuth's product for mean < 30; exp(-mean) from the host table.
__device__ __forceinline__ int64_t poisson_lcg(double mean, double u_seed, double exp_neg_mean, uint32_t* status) {
  if (mean <= 0.0) return 0;
  uint64_t s = (uint64_t)(int64_t)__dmul_rn(u_seed, 9.007199254740992e15);
  if (mean < 30.0) {
    int64_t k = 0;
    double pr = 1.0;
    for (;;) {
      s = s * 6364136223846793005ull + 1442695040888963407ull;
      const double u = __ddiv_rn(__ull2double_rn(s >> 11), 9.007199254740992e15);
      pr = __dmul_rn(pr, u);
      if (pr <= exp_neg_mean) break;
      k += 1;
      if (k > 10000) break;
    }
    return k;
  }
  set_status(status, EDM_STATUS_POISSON_NORMAL);
  s = s * 6364136223846793005ull + 1442695040888963407ull;
  double u1 = __ddiv_rn(__ull2double_rn(s >> 11), 9.007199254740992e15);
  s = s * 6364136223846793005ull + 1442695040888963407ull;
  const double u2 = __ddiv_rn(__ull2double_rn(s >> 11), 9.007199254740992e15);
  if (u1 < 1e-30) u1 = 1e-30;
  const double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
  const int64_t n = (int64_t)(mean + sqrt(mean) * z + 0.5);
  return n > 0 ? n : 0;
}

// FRET class of donor-capable particle gid (slot `slot`, dye dt) for the
// current state (photophysics.py:528-683, 1021-1114): the reference's
// update_fret_rates visits the bond-mode pairs, then the proximity pairs, and
// the last pair matching the particle's dye sets its rate.  A bonded donor
// gets its pair's bound class (acceptor index `acc` unless intramolecular);
// proximity mode needs an alive donor and sets the high class when an alive
// target lies within the radius, the low class otherwise.
template <bool F64>
__device__ int fret_class(const EdmDynParams& p, const EdmPhotParams& pp, const DevState& st, const PhotState& ph,
                          int r, int gid, int64_t slot, int dt, bool alive, int cells_valid, int& acc) {
  int cls = 0;
  acc = -1;
  for (int b = 0; b < pp.n_fret; ++b) {
    const EdmFret& F = pp.fret[b];
    if (dt != F.donor_fid) continue;
    if (F.mode == 0) {
      const int partner = st.bond[gid];
      if (partner >= 0) {
        if (F.intramolecular) {
          cls = F.cls_bound;
          acc = -1;
        } else if (ph.has_dye[partner] && ph.dye[partner] == F.acceptor_fid) {
          cls = F.cls_bound;
          acc = partner;
        }
      }
    } else {
      if (!alive) continue;  // photophysics.py:640
      // Any alive target within the radius, post-move (the reference's
      // all-pairs search, photophysics.py:591-683).  After a dynamics step
      // it goes through that step's cell list: a target within radius R now
      // was within R + 2 max_disp before the move, so the pre-move cells
      // within that reach of the donor's pre-move cell hold every candidate
      // that moved by Brownian steps; the step's list of particles placed
      // after the sort holds the rest.  Same per-pair test, same answer.  Before any dynamics step since the
      // state was set, the cell list does not exist and every particle of
      // the replica is tested.
      const Geo g(p);
      double xi, yi;
      abs_pos<F64>(st.pos_post, st.lo_post, st.cell_post, slot, g, xi, yi);
      auto near = [&](int64_t j) {
        const uint8_t fj = st.flags[j];
        if (j == slot || !fl_alive(fj) || fl_species(fj) != F.target_species) return false;
        double xj, yj;
        abs_pos<F64>(st.pos_post, st.lo_post, st.cell_post, j, g, xj, yj);
        double dx = xj - xi, dy = yj - yi;
        if (g.px) {
          if (dx > g.Lx() / 2.0) dx -= g.Lx();
          else if (dx < -g.Lx() / 2.0) dx += g.Lx();
        }
        if (g.py) {
          if (dy > g.Ly() / 2.0) dy -= g.Ly();
          else if (dy < -g.Ly() / 2.0) dy += g.Ly();
        }
        return dx * dx + dy * dy < F.prox_radius_sq;
      };
      bool found = false;
      if (!cells_valid) {
        for (int64_t j = p.particle_offset; j < p.particle_offset + p.n_particles && !found; ++j) found = near(j);
        cls = found ? F.cls_high : F.cls_low;
        acc = -1;
        continue;
      }
      const double reach = sqrt(F.prox_radius_sq) + 2.0 * p.max_disp;
      const int kx = (int)ceil(reach / g.sx), ky = (int)ceil(reach / g.sy);
      int cx, cy;
      split_cell(st.cell_pre[slot], g, cx, cy);
      // a window as wide as the grid visits every column / row once
      const int x0 = 2 * kx + 1 >= g.nx ? 0 : cx - kx, x1 = 2 * kx + 1 >= g.nx ? g.nx - 1 : cx + kx;
      const int y0 = 2 * ky + 1 >= g.ny ? 0 : cy - ky, y1 = 2 * ky + 1 >= g.ny ? g.ny - 1 : cy + ky;
      for (int ux = x0; ux <= x1 && !found; ++ux) {
        int ncx = ux;
        if (g.px) ncx = ncx < 0 ? ncx + g.nx : (ncx >= g.nx ? ncx - g.nx : ncx);
        else if (ncx < 0 || ncx >= g.nx) continue;
        for (int uy = y0; uy <= y1 && !found; ++uy) {
          int ncy = uy;
          if (g.py) ncy = ncy < 0 ? ncy + g.ny : (ncy >= g.ny ? ncy - g.ny : ncy);
          else if (ncy < 0 || ncy >= g.ny) continue;
          const int64_t nc = g.cbase + (int64_t)ncx * g.ny + ncy;
          for (int j = st.cell_start[nc], je = st.cell_start[nc + 1]; j < je && !found; ++j) found = near(j);
        }
      }
      // particles placed after the sort (recruitment, dissociation) are not in the cell list
      const int nm = min(st.moved_count[r], (int)p.n_particles);
      for (int k = 0; k < nm && !found; ++k) found = near(st.moved[p.particle_offset + k]);
      cls = found ? F.cls_high : F.cls_low;
      acc = -1;
    }
  }
  return cls;
}

// Per emitter: FRET class, photon counts, photophysical transition.
template <bool F64>
__global__ void __launch_bounds__(kBlock) k_phot_count(const EdmDynParams* __restrict__ DP,
                                                       const EdmPhotParams* __restrict__ PP,
                                                       const int2* __restrict__ eblk, DevState st, PhotState ph,
                                                       int cells_valid) {
  const Tile t = tile_of(eblk);
  const EdmPhotParams& pp = PP[t.r];
  const EdmDynParams& p = DP[t.r];
  const int64_t e = t.s;
  if (e >= pp.emitter_offset + pp.n_emitters) return;
  const int gid = ph.emit_id[e];
  const int lid = gid - (int)p.particle_offset;
  ph.emit_n[e] = 0;
  ph.emit_nd[e] = 0;
  ph.emit_acc[e] = -1;
  const int64_t slot = st.slot_of_id[gid];
  const uint8_t f = st.flags[slot];
  if (!ph.has_dye[gid] || !fl_alive(f) || ph.bleached[gid]) return;
  const int dt = ph.dye[gid];
  if (dt < 0 || dt >= pp.n_fluoro) return;
  const int s0 = pp.ground[dt], s1 = pp.excited[dt], t1 = pp.t1[dt], bl = pp.bl[dt];
  const int cur = ph.ctmc[gid];
  int pss;
  if (cur == s0 || cur == s1) pss = 0;
  else if (t1 >= 0 && cur == t1) pss = 1;
  else if (bl >= 0 && cur == bl) {
    ph.bleached[gid] = 1;
    return;
  } else pss = 0;
  int acc = -1;
  const int cls = fret_class<F64>(p, pp, st, ph, t.r, gid, slot, dt, true, cells_valid, acc);
  const int64_t key = *ph.d_pstep;
  const double up = uniform1(p.seed, key, EDM_S_PH_POISSON, (uint64_t)lid, 0);
  const double ut = uniform1(p.seed, key, EDM_S_PH_TRANS, (uint64_t)lid, 0);
  const double md = pp.mean_d[dt][pss][cls], mf = pp.mean_f[dt][pss][cls];
  const int64_t nd = poisson_lcg(md, up, pp.exp_neg_d[dt][pss][cls], st.status);
  int64_t nf = 0;
  if (mf > 0.0 && pp.has_fret_cls[cls])
    nf = poisson_lcg(mf, __dadd_rn(__dmul_rn(up, 0.5), 0.25), pp.exp_neg_f[dt][pss][cls], st.status);
  const int64_t ntot = nd + ((nf > 0 && acc >= 0) ? nf : 0);
  ph.emit_nd[e] = (int32_t)nd;
  ph.emit_n[e] = (int32_t)ntot;
  ph.emit_acc[e] = acc;
  ph.emit_cls[e] = (int8_t)cls;
  // transition (photophysics.py:474-481)
  if (ut < pp.T00[dt][pss][cls]) ph.ctmc[gid] = (int8_t)s0;
  else if (ut < pp.T0001[dt][pss][cls]) ph.ctmc[gid] = (int8_t)(t1 >= 0 ? t1 : s0);
  else {
    ph.ctmc[gid] = (int8_t)(bl >= 0 ? bl : s0);
    ph.bleached[gid] = 1;
  }
}

// Exclusive scan of emitter photon counts, one block per replica.
__global__ void k_phot_scan(const EdmPhotParams* __restrict__ PP, PhotState ph, int64_t* counters, uint32_t* status) {
  const int r = blockIdx.x;
  const EdmPhotParams& pp = PP[r];
  int64_t carry = 0;
  __shared__ long long sh[32];
  for (int64_t off = 0; off < pp.n_emitters; off += blockDim.x) {
    const int64_t e = pp.emitter_offset + off + threadIdx.x;
    const long long v = (off + threadIdx.x < pp.n_emitters) ? ph.emit_n[e] : 0;
    // block scan (64-bit)
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
      const int nw = blockDim.x >> 5;
      long long w = lane < nw ? sh[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      if (lane < nw) sh[lane] = w;
    }
    __syncthreads();
    const long long base = wid > 0 ? sh[wid - 1] : 0;
    const long long total = sh[(blockDim.x >> 5) - 1];
    if (off + threadIdx.x < pp.n_emitters) ph.emit_off[e] = carry + base + x - v;
    carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int64_t n = carry;
    if (n > pp.max_photons) {
      n = pp.max_photons;
      set_status(status, EDM_STATUS_PHOTON_CAP);
    }
    ph.ph_count[r] = n;
    counters[(int64_t)r * EDM_NCOUNTERS + EDM_C_PHOTONS] += n;
  }
}

// Write the photons of each emitter (photophysics.py:433-472).
// Absolute position of the particle with replica-local index pid.
template <bool F64>
__device__ __forceinline__ double2 particle_pos(const DevState& st, const Geo& g, int pid) {
  double x, y;
  abs_pos<F64>(st.pos_post, st.lo_post, st.cell_post, st.slot_of_id[g.poff + pid], g, x, y);
  return make_double2(x, y);
}

// The photon records, each with the position of the particle it leaves
// (the donor, or the acceptor of a FRET photon), so the detection pass reads
// no particle state and can run beside the next step.
template <bool F64>
__global__ void __launch_bounds__(kBlock) k_phot_write(const EdmDynParams* __restrict__ DP,
                                                       const EdmPhotParams* __restrict__ PP,
                                                       const int2* __restrict__ eblk, DevState st, PhotState ph,
                                                       int64_t* counters) {
  const Tile t = tile_of(eblk);
  const EdmPhotParams& pp = PP[t.r];
  const int64_t e = t.s;
  if (e >= pp.emitter_offset + pp.n_emitters) return;
  const int ntot = ph.emit_n[e];
  if (ntot == 0) return;
  const EdmDynParams& p = DP[t.r];
  const int gid = ph.emit_id[e];
  const int lid = gid - (int)p.particle_offset;
  const int nd = ph.emit_nd[e];
  const int dt = ph.dye[gid];
  const int cls = ph.emit_cls[e];
  const double tau = pp.tau[dt][cls];
  const int64_t off = ph.emit_off[e];
  const int64_t key = *ph.d_pstep;
  const Geo g(p);
  const double2 xy_donor = particle_pos<F64>(st, g, lid);
  double2 xy_acc = xy_donor;
  bool have_acc = false;
  int n_donor_ch = 0, n_acc_ch = 0, n_fret = 0;
  for (int j = 0; j < ntot; ++j) {
    const int64_t k = off + j;
    if (k >= pp.max_photons) break;
    const bool fret = j >= nd;
    int ch = dt, pid = lid;
    double ta = tau;
    if (fret) {
      const int acc = ph.emit_acc[e];
      const int at = ph.dye[acc];
      ta = (at >= 0 && at < pp.n_fluoro) ? pp.tau_all[at] : tau;
      ch = at;
      pid = acc - (int)p.particle_offset;
    }
    double tt;
    if (k < pp.est_photons) {
      double u = uniform1(p.seed, key, EDM_S_PH_ARRIVAL, (uint64_t)k, 0);
      if (u < 1e-30) u = 1e-30;
      tt = -ta * log(u);
    } else {
      tt = ta;
    }
    const int64_t o = pp.photon_offset + k;
    if (fret && !have_acc && pid >= 0 && pid < p.n_particles) {
      xy_acc = particle_pos<F64>(st, g, pid);
      have_acc = true;
    }
    ph.ph_xy[o] = fret ? xy_acc : xy_donor;
    ph.ph_pid[o] = pid;
    ph.ph_t[o] = tt;
    ph.ph_ch[o] = (int8_t)ch;
    ph.ph_fret[o] = fret ? 1 : 0;
    n_donor_ch += ch == pp.donor_channel;
    n_acc_ch += ch == pp.acceptor_channel;
    n_fret += fret;
  }
  int64_t* c = counters + (int64_t)t.r * EDM_NCOUNTERS;
  if (n_donor_ch) atomic_add_i64(c + EDM_C_DONOR_PH, n_donor_ch);
  if (n_acc_ch) atomic_add_i64(c + EDM_C_ACCEPTOR_PH, n_acc_ch);
  if (n_fret) atomic_add_i64(c + EDM_C_FRET_PH, n_fret);
}

__global__ void k_phot_advance(int64_t* d_pstep, int64_t* d_batch_key) {
  *d_batch_key = *d_pstep;
  *d_pstep += 1;
}

// Per photon: detection efficiency, PSF pixel draw, IRF jitter, TCSPC bin.
template <bool F64>
__global__ void __launch_bounds__(kBlock) k_scope(const EdmDynParams* __restrict__ DP,
                                                  const EdmPhotParams* __restrict__ PP,
                                                  const EdmScopeParams* __restrict__ SP,
                                                  const int2* __restrict__ phblk, DevState st, PhotState ph) {
  const Tile t = tile_of(phblk);
  const EdmPhotParams& pp = PP[t.r];
  const int64_t k = t.s - pp.photon_offset;
  if (k >= ph.ph_count[t.r]) return;
  const EdmDynParams& p = DP[t.r];
  const EdmScopeParams& sp = SP[t.r];
  const int64_t key = *ph.d_batch_key;
  const int64_t o = t.s;
  if (!(uniform1(p.seed, key, EDM_S_SC_QE, (uint64_t)k, 0) < sp.qe)) return;
  const int pid = ph.ph_pid[o];
  if (pid < 0 || pid >= p.n_particles) return;
  const double2 xy = ph.ph_xy[o];
  const double x = xy.x, y = xy.y;
  int ch = ph.ph_ch[o];
  int chs = ch;
  if (chs < 0) chs = 0;
  if (chs >= sp.n_sigma) chs = 0;
  const double inv2 = sp.sigma_ch[chs] > 0.0 ? sp.inv_2sig2_ch[chs] : sp.inv_2sig2_ch[0];
  const double fx = (x - sp.offset_x) / sp.pixel_size - 0.5;
  const double fy = (y - sp.offset_y) / sp.pixel_size - 0.5;
  const int i0 = (int)floor(fx + 0.5), j0 = (int)floor(fy + 0.5);
  const int R = sp.psf_range_px;
  if (i0 < -R || i0 >= sp.nx + R) return;
  if (j0 < -R || j0 >= sp.ny + R) return;
  // Pixel weights exp(-(dx^2 + dy^2) / 2 sigma^2) over the in-FOV pixels of
  // the (2R+1)^2 window, summed and searched in the reference's order (di
  // outer, dj inner): the Gaussian factors into exp(-dx^2 / 2 sigma^2)
  // exp(-dy^2 / 2 sigma^2), so a window costs 2(2R+1)+(2R+1) exps, not
  // 2(2R+1)^2 (the weights differ from the unfactored form by an ulp or two).
  double wy[2 * kPsfMaxR + 1];
  const int Rc = R <= kPsfMaxR ? R : kPsfMaxR;  // the host keeps R <= kPsfMaxR
  for (int dj = -Rc; dj <= Rc; ++dj) {
    const int jj = j0 + dj;
    const double dy = y - (((double)jj + 0.5) * sp.pixel_size + sp.offset_y);
    wy[dj + Rc] = (jj < 0 || jj >= sp.ny) ? -1.0 : exp(-(dy * dy) * inv2);
  }
  double total = 0.0;
  int n = 0;
  for (int di = -Rc; di <= Rc; ++di) {
    const int ii = i0 + di;
    if (ii < 0 || ii >= sp.nx) continue;
    const double dx = x - (((double)ii + 0.5) * sp.pixel_size + sp.offset_x);
    const double wx = exp(-(dx * dx) * inv2);
    for (int dj = 0; dj <= 2 * Rc; ++dj) {
      if (wy[dj] < 0.0) continue;
      total += wx * wy[dj];
      ++n;
    }
  }
  if (n == 0 || total <= 0.0) return;
  const double u = uniform1(p.seed, key, EDM_S_SC_ASSIGN, (uint64_t)k, 0) * total;
  int si = -1, sj = -1, fi = -1, fj = -1;
  double cum = 0.0;
  for (int di = -Rc; di <= Rc && si < 0; ++di) {
    const int ii = i0 + di;
    if (ii < 0 || ii >= sp.nx) continue;
    const double dx = x - (((double)ii + 0.5) * sp.pixel_size + sp.offset_x);
    const double wx = exp(-(dx * dx) * inv2);
    for (int dj = 0; dj <= 2 * Rc; ++dj) {
      if (wy[dj] < 0.0) continue;
      const int jj = j0 + dj - Rc;
      if (fi < 0) {
        fi = ii;
        fj = jj;
      }
      cum += wx * wy[dj];
      if (cum >= u) {
        si = ii;
        sj = jj;
        break;
      }
    }
  }
  if (si < 0) {  // no cumulative weight reached u: first pixel (microscope.py:612-619)
    si = fi;
    sj = fj;
  }
  int64_t* cnt = st.counters + (int64_t)t.r * EDM_NCOUNTERS;
  atomic_add_i64(cnt + EDM_C_DETECTED, 1);
  const double z = normal2(p.seed, key, EDM_S_SC_JITTER, (uint64_t)k).u0;
  double tt = __dadd_rn(ph.ph_t[o], __dmul_rn(sp.sigma_irf, z));
  if (ch < 0 || ch >= sp.n_channels) return;
  if (tt < 0.0) tt = 0.0;
  const int64_t b = (int64_t)__ddiv_rn(tt, sp.bin_width);
  if (b >= sp.n_bins) return;
  const int64_t e = sp.flim_offset + (((int64_t)ch * sp.nx + si) * sp.ny + sj) * sp.n_bins + b;
  atomicAdd(&ph.flim[e], 1u);
  touch_stretch(ph.touch, e);
}

// The positions of a photon batch set from the host (edm_set_photons) or left
// by an earlier pass: each photon's particle, from the current state.
template <bool F64>
__global__ void __launch_bounds__(kBlock) k_photon_positions(const EdmDynParams* __restrict__ DP,
                                                             const EdmPhotParams* __restrict__ PP,
                                                             const int2* __restrict__ phblk, DevState st,
                                                             PhotState ph) {
  const Tile t = tile_of(phblk);
  const EdmPhotParams& pp = PP[t.r];
  const int64_t k = t.s - pp.photon_offset;
  if (k >= ph.ph_count[t.r]) return;
  const EdmDynParams& p = DP[t.r];
  const int pid = ph.ph_pid[t.s];
  if (pid < 0 || pid >= p.n_particles) return;
  const Geo g(p);
  ph.ph_xy[t.s] = particle_pos<F64>(st, g, pid);
}

// Photons received per replica (microscope.py:1093).
__global__ void k_scope_received(const EdmPhotParams* __restrict__ PP, int n_rep, PhotState ph, int64_t* counters) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n_rep) counters[(int64_t)r * EDM_NCOUNTERS + EDM_C_RECEIVED] += ph.ph_count[r];
}

// Dark counts (microscope.py:850-887) — one thread per (channel, pixel).
__global__ void __launch_bounds__(kBlock) k_dark(const EdmDynParams* __restrict__ DP,
                                                 const EdmScopeParams* __restrict__ SP, const int2* __restrict__ pxblk,
                                                 uint32_t* flim, uint32_t* touch, int64_t frame,
                                                 int64_t* counters) {
  const Tile t = tile_of(pxblk);
  const EdmScopeParams& sp = SP[t.r];
  const int64_t q = t.s;
  const int64_t npx = (int64_t)sp.n_channels * sp.nx * sp.ny;
  if (q >= npx || !(sp.dark_lambda >= 1e-10)) return;
  const uint64_t seed = DP[t.r].seed;
  double pr = 1.0;
  int64_t n = 0;
  for (uint32_t a = 0; a < 100000; ++a) {
    pr = __dmul_rn(pr, uniform1(seed, frame, EDM_S_SC_DARK, (uint64_t)q, a));
    if (pr <= sp.dark_exp_neg) break;
    ++n;
  }
  const int64_t e0 = sp.flim_offset + q * sp.n_bins;
  for (int64_t m = 0; m < n; ++m) {
    const double u = uniform1(seed, frame, EDM_S_SC_DARK_BIN, (uint64_t)q, (uint64_t)m);
    const int64_t e = e0 + (int64_t)(u * (double)sp.n_bins);
    flim[e] += 1u;
    touch_stretch(touch, e);
  }
  if (n) atomic_add_i64(counters + (int64_t)t.r * EDM_NCOUNTERS + EDM_C_DARK, n);
}

// Afterpulsing (microscope.py:889-922): Binomial(total, p) as keyed Bernoullis.
__global__ void __launch_bounds__(kBlock) k_afterpulse(const EdmDynParams* __restrict__ DP,
                                                       const EdmScopeParams* __restrict__ SP,
                                                       const int2* __restrict__ pxblk, uint32_t* flim,
                                                       uint32_t* touch, int64_t frame, int64_t* counters) {
  const Tile t = tile_of(pxblk);
  const EdmScopeParams& sp = SP[t.r];
  const int64_t q = t.s;
  const int64_t npx = (int64_t)sp.n_channels * sp.nx * sp.ny;
  if (q >= npx || !(sp.ap_prob > 0.0)) return;
  const uint64_t seed = DP[t.r].seed;
  uint32_t* px = flim + sp.flim_offset + q * sp.n_bins;
  int64_t total = 0;
  for (int b = 0; b < sp.n_bins; ++b) total += px[b];
  if (total == 0) return;
  int64_t n = 0;
  for (int64_t m = 0; m < total; ++m)
    if (uniform1(seed, frame, EDM_S_SC_AP, (uint64_t)q, (uint64_t)m) < sp.ap_prob) ++n;
  for (int64_t m = 0; m < n; ++m) {
    const double u = uniform1(seed, frame, EDM_S_SC_AP_BIN, (uint64_t)q, (uint64_t)m);
    const int64_t b = (int64_t)(u * (double)sp.n_bins);
    px[b] += 1u;
    touch_stretch(touch, sp.flim_offset + q * sp.n_bins + b);
  }
  if (n) atomic_add_i64(counters + (int64_t)t.r * EDM_NCOUNTERS + EDM_C_AFTERPULSE, n);
}

}  // namespace edm
