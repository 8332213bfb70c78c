// edm_engine.cu — the engine behind the C ABI of include/edm_b200.h.
//
// One engine holds R replicas (R = 1 for the drop-in single-system API) in
// replica-offset CSR layout: particles, cells, density-grid cells, emitters,
// photon buffers and FLIM stacks of replica r are contiguous slices located
// by the offsets of its parameter blocks.  Every kernel launch covers all
// replicas; per-step work is enqueued on the caller's stream and can be
// captured into CUDA graphs (the BD step index lives in device memory, so a
// captured chunk replays with advancing keys).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "edm_error.h"
#include "edm_census.cuh"
#include "edm_phot.cuh"

using namespace edm;

namespace {
thread_local std::string g_last_error;
}  // namespace

int edm::report_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

namespace {

int fail(int code, const std::string& msg) { return edm::report_error(code, msg); }

#define CUDA_TRY(expr)                                                                  \
  do {                                                                                  \
    cudaError_t _e = (expr);                                                            \
    if (_e != cudaSuccess) return fail(EDM_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

enum PassKind { P_BIND_CAND, P_BIND_APPLY, P_DISSOC, P_CONTACTS, P_CAT, P_REC_CAND, P_REC_APPLY, P_DETACH, P_CONV, P_MERGE,
                P_GROUP, P_DRAWS, P_ADAPT, P_LOCAL_CDF };
struct Pass {
  PassKind kind;
  int index;
  Match match;  // particles a per-particle pass visits
};

template <typename T>
int dalloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) return fail(EDM_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  e = cudaMemset(*p, 0, n * sizeof(T));
  if (e != cudaSuccess) return fail(EDM_ECUDA, cudaGetErrorString(e));
  return EDM_OK;
}

// Tiles of bs items per replica: (replica, first index).
std::vector<int2> tiles(const std::vector<int64_t>& first, const std::vector<int64_t>& count, int bs = kBlock) {
  std::vector<int2> out;
  for (size_t r = 0; r < first.size(); ++r)
    for (int64_t i = 0; i < count[r]; i += bs) out.push_back(make_int2((int)r, (int)(first[r] + i)));
  return out;
}

// ---- launch shapes of the tuned kernels -------------------------------------
// Candidate (threads per block, minimum resident blocks per SM) of each kernel
// the autotuner times; candidate 0 is the fixed shape used without tuning.
struct LaunchShape {
  int block, min_blocks;
};
enum TunedKernel { TK_SCATTER = 0, TK_MOVE = 1, TK_CONTACTS = 2, TK_COUNT = 3 };
constexpr int kMaxShapes = 8;
constexpr LaunchShape kShapes[TK_COUNT][kMaxShapes] = {
    // k_scatter: one slot per thread, then (3-4) two
    {{256, 1}, {128, 1}, {512, 1}, {128, 1}, {256, 1}},
    // k_move: the second number bounds its registers (80 at 256 x 3 down to 32
    // at 128 x 16, with spills below 64): occupancy pays more than the spills
    {{256, 3}, {256, 4}, {128, 8}, {128, 10}, {128, 12}, {128, 16}, {256, 6}, {256, 8}},
    // k_contacts: 0 by sweeper; 1-2 by (sweeper, neighbour column) per warp;
    // 3-5 the same tasks balanced over the block (16, 16, 4 slots per
    // thread); 6-7 over a global sweeper list (k_sweep_list), one wave
    {{256, 6}, {256, 6}, {256, 4}, {256, 6}, {256, 4}, {256, 6}, {256, 6}, {256, 8}},
};
constexpr int kNumShapes[TK_COUNT] = {5, 8, 8};
const char* const kTunedNames[TK_COUNT] = {"k_scatter", "k_move", "k_contacts"};
constexpr int kTileSizes[3] = {128, 256, 512};
int tile_index(int bs) { return bs == 128 ? 0 : (bs == 256 ? 1 : 2); }

// Choices of earlier tunings in this process, by (kernel, precision,
// replicas, log2 of the slot count): later engines of the same kind reuse them.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, int> g_tuned;

}  // namespace

struct EdmEngine {
  int device = 0, precision = 64, R = 0;
  bool f64 = true, has_phot = false, has_scope = false;
  int64_t N = 0, n_cells = 0, n_grid = 0, n_hill = 0, n_emit = 0, n_phcap = 0, n_flim = 0;
  std::vector<EdmDynParams> hdp;
  std::vector<EdmPhotParams> hpp;
  std::vector<EdmScopeParams> hsp;
  EdmDynParams* dp = nullptr;
  EdmPhotParams* pp = nullptr;
  EdmScopeParams* sp = nullptr;
  double* hill = nullptr;
  std::vector<double> rule_max;  // [R][EDM_MAX_RULES] upper bound of each rule's Hill factor (host)
  uint64_t *pass_thr = nullptr, *cat_thr = nullptr;  // draw thresholds ([R][kMaxPP], [R][EDM_MAX_CAT])
  int2 *pblk = nullptr, *eblk = nullptr, *phblk = nullptr, *pxblk = nullptr;
  int npblk = 0, neblk = 0, nphblk = 0, npxblk = 0;
  // slot tiles of 128, 256 and 512 (the 256 table is pblk) for the tuned kernels
  int2* pblk_bs[3] = {nullptr, nullptr, nullptr};
  int npblk_bs[3] = {0, 0, 0};
  // launch shape of each tuned kernel (index into kShapes), tuning timings
  int shape[TK_COUNT] = {0, 0, 0};
  float tuned_ms[TK_COUNT] = {0, 0, 0}, default_ms[TK_COUNT] = {0, 0, 0};
  int tune_kernel = -1;  // the kernel the autotuner is timing, with its event pair
  cudaEvent_t tune_ev[2] = {nullptr, nullptr};
  void* pos_pre = nullptr;
  void* pos_post = nullptr;
  short2 *lo_pre = nullptr, *lo_post = nullptr;
  int32_t *cell_pre = nullptr, *cell_post = nullptr;
  uint8_t* flags[2] = {nullptr, nullptr};
  int32_t* ids[2] = {nullptr, nullptr};
  int cur = 0;
  int32_t *slot_of_id = nullptr, *bond = nullptr;
  uint8_t *has_dye = nullptr, *bleached = nullptr;
  int8_t *dye = nullptr, *ctmc = nullptr;
  int32_t *cell_start = nullptr, *cursor = nullptr, *cnt = nullptr, *bsum = nullptr;
  int nb_scan = 0;
  int32_t *grid_cnt = nullptr, *grid_delta = nullptr;
  int64_t* counters = nullptr;
  uint32_t* status = nullptr;
  int64_t *d_step = nullptr, *d_pstep = nullptr, *d_batch_key = nullptr;
  int32_t *rec_count = nullptr, *rec_id = nullptr, *bind_count = nullptr, *bind_ab = nullptr;
  double* rec_xy = nullptr;
  int64_t* bind_key = nullptr;
  int32_t *emit_id = nullptr, *emit_n = nullptr, *emit_nd = nullptr, *emit_acc = nullptr;
  int8_t* emit_cls = nullptr;
  int64_t* emit_off = nullptr;
  int32_t* ph_pid = nullptr;
  double* ph_t = nullptr;
  int8_t* ph_ch = nullptr;
  uint8_t* ph_fret = nullptr;
  double2* ph_xy = nullptr;
  int64_t* ph_count = nullptr;
  uint32_t* flim = nullptr;
  // host staging for get_state
  double* st_pos = nullptr;
  int32_t *st_sp = nullptr, *st_bond = nullptr;
  uint8_t *st_alive = nullptr, *st_bl = nullptr;
  int8_t* st_ctmc = nullptr;
  std::vector<Pass> passes;
  std::vector<PassGroup> groups;  // runs of per-particle passes (P_GROUP index)
  DrawPlan draw{};                // the draw sweep of the per-particle passes
  bool draws_early = false;       // the sweep runs on side_stream beside the passes before the first run
  cudaStream_t side_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  DrawPlan* d_draw = nullptr;     // device copies of the plan and the runs
  PassGroup* d_groups = nullptr;
  uint32_t rec_after[EDM_MAX_EXCH] = {};  // per recruitment apply: later passes matching a recruit
  int2* contacts = nullptr;
  int32_t* contact_count = nullptr;
  int64_t contact_cap = 0;
  uint32_t enzyme_mask = 0;
  CatLists cat_lists{};
  uint32_t cat_late[EDM_MAX_CAT] = {};
  bool contact_sides_counted = false;  // sides chosen from a state's species counts
  int64_t* rep_first = nullptr;
  int32_t* chunk_rep = nullptr;  // replica of the first slot of each 128-slot chunk
  int32_t *moved = nullptr, *moved_count = nullptr;
  int4* pl = nullptr;  // listed particles of the per-particle passes: (slot, pass bits, replica, id)
  int32_t *pl_count = nullptr, *pl_index = nullptr;
  int32_t *sw_list = nullptr, *sw_count = nullptr;  // the contact search's sweeper list
  uint32_t sensor_grids[EDM_MAX_SPECIES] = {};  // per species: the grids that sense it in some replica
  double *adapt_w = nullptr, *local_cdf = nullptr;  // per global grid cell
  std::vector<int32_t> emit_host;  // emitter list last uploaded
  std::vector<uint8_t> has_dye_host;  // has_dye of the last edm_set_state
  bool cells_valid = false;  // the cell list matches the state (a dynamics step ran since set_state)
  // captured pipeline chunks, keyed by (steps, with photons, slot parity, recording)
  std::map<std::tuple<int, int, int, int>, cudaGraphExec_t> graphs;
  // sub-frame recorder ring [rec_cap][R][EDM_CENSUS_FIELDS] and ground-truth buffers
  int rec_cap = 0;
  int64_t* rec_ring = nullptr;
  int64_t* gt_census = nullptr;
  double *gt_E = nullptr, *gt_tau = nullptr;
  std::vector<void*> allocs;

  DevState dev_state() const {
    DevState s;
    s.pos_pre = pos_pre;
    s.pos_post = pos_post;
    s.lo_pre = lo_pre;
    s.lo_post = lo_post;
    s.cell_pre = cell_pre;
    s.cell_post = cell_post;
    s.flags_old = flags[cur ^ 1];
    s.flags = flags[cur];
    s.ids_old = ids[cur ^ 1];
    s.ids = ids[cur];
    s.slot_of_id = slot_of_id;
    s.bond = bond;
    s.cell_start = cell_start;
    s.cell_cursor = cursor;
    s.cnt_next = cnt;
    s.grid_cnt = grid_cnt;
    s.grid_delta = grid_delta;
    s.hill = hill;
    s.pass_thr = pass_thr;
    s.cat_thr = cat_thr;
    s.counters = counters;
    s.status = status;
    s.d_step = d_step;
    s.rec_count = rec_count;
    s.rec_id = rec_id;
    s.rec_xy = rec_xy;
    s.bind_count = bind_count;
    s.bind_key = bind_key;
    s.bind_ab = bind_ab;
    s.contacts = contacts;
    s.contact_count = contact_count;
    s.contact_cap = contact_cap;
    s.rep_first = rep_first;
    s.chunk_rep = chunk_rep;
    s.moved = moved;
    s.moved_count = moved_count;
    s.pl = pl;
    s.pl_count = pl_count;
    s.pl_index = pl_index;
    for (int sp = 0; sp < EDM_MAX_SPECIES; ++sp) s.sensor_grids[sp] = sensor_grids[sp];
    s.sw_list = sw_list;
    s.sw_count = sw_count;
    s.adapt_w = adapt_w;
    s.local_cdf = local_cdf;
    s.n_rep = R;
    s.n_slots = N;
    return s;
  }

  PhotState phot_state() const {
    PhotState p;
    p.emit_id = emit_id;
    p.emit_n = emit_n;
    p.emit_nd = emit_nd;
    p.emit_acc = emit_acc;
    p.emit_cls = emit_cls;
    p.emit_off = emit_off;
    p.has_dye = has_dye;
    p.dye = dye;
    p.ctmc = ctmc;
    p.bleached = bleached;
    p.ph_pid = ph_pid;
    p.ph_t = ph_t;
    p.ph_ch = ph_ch;
    p.ph_fret = ph_fret;
    p.ph_xy = ph_xy;
    p.ph_count = ph_count;
    p.flim = flim;
    p.touch = touch;
    p.d_pstep = d_pstep;
    p.d_batch_key = d_batch_key;
    return p;
  }

  template <typename T>
  int alloc(T** p, size_t n) {
    int rc = dalloc(p, n);
    if (rc == EDM_OK) allocs.push_back((void*)*p);
    return rc;
  }

  // Host schedule of the reaction passes (reference order, dynamics.py:2205-2465)
  // and the grid merges they need.  Per-particle passes read the current flags,
  // so a pass visits exactly the particles that hold its species when it runs.
  int build_schedule() {
    const EdmDynParams& p = hdp[0];
    std::vector<bool> dirty(EDM_MAX_GRIDS, false);
    auto sensors_of = [&](std::vector<int> species) {
      std::vector<int> gs;
      for (int g = 0; g < p.n_grids; ++g)
        for (int s : species)
          if (p.grid[g].sensor == s) gs.push_back(g);
      return gs;
    };
    auto match = [](std::vector<int> species, int alive) {
      Match m{};
      for (int s : species) m.mask[alive ? 1 : 0] |= 1u << s;
      return m;
    };
    const Match none = match({}, 1);
    auto reads = [&](std::vector<int> rules) {
      bool need = false;
      for (int r : rules)
        if (r >= 0 && dirty[p.rule[r].grid]) need = true;
      if (need) {
        passes.push_back({P_MERGE, 0, none});
        std::fill(dirty.begin(), dirty.end(), false);
      }
    };
    auto writes = [&](std::vector<int> species) {
      for (int g : sensors_of(species)) dirty[g] = true;
    };
    for (int b = 0; b < p.n_bind; ++b) {
      const EdmBind& B = p.bind[b];
      passes.push_back({P_BIND_CAND, b, match({B.ra, B.rb}, 1)});
      passes.push_back({P_BIND_APPLY, b, none});
      passes.push_back({P_DISSOC, b, match({B.product}, 1)});
      writes({B.ra, B.rb, B.product});
    }
    // adaptation field, after binding and before catalysis (dynamics.py:2227-2242)
    if (p.adapt_grid >= 0) {
      if (dirty[p.adapt_grid]) {
        passes.push_back({P_MERGE, 0, none});
        std::fill(dirty.begin(), dirty.end(), false);
      }
      passes.push_back({P_ADAPT, 0, none});
    }
    if (p.n_cat > 0) {
      enzyme_mask = 0;
      uint32_t touched = 0;
      for (int c = 0; c < p.n_cat; ++c) {
        enzyme_mask |= 1u << p.cat[c].enzyme;
        touched |= (1u << p.cat[c].substrate) | (1u << p.cat[c].product);
        // the later reactions whose substrate this pass's product is: a
        // particle it converts gets its late pairs for them at once
        cat_late[c] = 0;
        for (int c2 = c + 1; c2 < p.n_cat; ++c2)
          if (p.cat[c2].substrate == p.cat[c].product) cat_late[c] |= 1u << c2;
      }
      if (enzyme_mask & touched) return fail(EDM_EUNSUP, "an enzyme species is also a catalytic substrate/product");
      passes.push_back({P_CONTACTS, 0, Match{{0u, 0u}}});
      set_contact_sides(nullptr);
    }
    // A pass whose probability is zero in every replica changes nothing (its
    // keyed draws feed no other pass), so it is not scheduled.
    auto any_positive = [&](auto prob_of) {
      for (int r = 0; r < R; ++r)
        if (prob_of(hdp[r]) > 0.0) return true;
      return false;
    };
    for (int c = 0; c < p.n_cat; ++c) {
      if (!any_positive([&](const EdmDynParams& q) { return q.cat[c].prob; })) continue;
      reads({p.cat[c].rule});
      passes.push_back({P_CAT, c, none});
      writes({p.cat[c].substrate, p.cat[c].product});
    }
    for (int e = 0; e < p.n_exch; ++e) {
      if (any_positive([&](const EdmDynParams& q) { return q.exch[e].prob_on; })) {
        reads({p.exch[e].rule_on, p.exch[e].rule_on2});
        if (p.exch[e].local_recruit) passes.push_back({P_LOCAL_CDF, e, none});
        passes.push_back({P_REC_CAND, e, match({p.exch[e].species}, 0)});
        passes.push_back({P_REC_APPLY, e, none});
        writes({p.exch[e].species});
      }
      if (any_positive([&](const EdmDynParams& q) { return q.exch[e].prob_off; })) {
        reads({p.exch[e].rule_off});
        passes.push_back({P_DETACH, e, match({p.exch[e].species}, 1)});
        writes({p.exch[e].species});
      }
    }
    for (int v = 0; v < p.n_conv; ++v) {
      if (!any_positive([&](const EdmDynParams& q) { return q.conv[v].prob; })) continue;
      reads({p.conv[v].rule});
      passes.push_back({P_CONV, v, match({p.conv[v].from}, 1)});
      writes({p.conv[v].from, p.conv[v].to});
    }
    return fuse_particle_passes();
  }

  // Which side of each catalytic reaction sweeps for its direct contact
  // pairs: the species with fewer alive particles (count[sp], summed over
  // the replicas; the enzyme side without counts).  Both sides find the same
  // pairs, so this choice changes only the work.
  // force_mask >= 0: bit c set = reaction c from the enzyme side, whatever
  // the counts.
  void set_contact_sides(const int64_t* count, int32_t force_mask = -1) {
    const EdmDynParams& p = hdp[0];
    cat_lists = CatLists{};
    cat_lists.n_cat = p.n_cat;
    uint32_t sweepers = 0;
    for (int c = 0; c < p.n_cat; ++c) {
      const int e = p.cat[c].enzyme, sub = p.cat[c].substrate;
      const bool from_enzyme = force_mask >= 0 ? ((force_mask >> c) & 1) != 0 : (!count || count[e] <= count[sub]);
      const int sw = from_enzyme ? e : sub, other = from_enzyme ? sub : e;
      if (from_enzyme) cat_lists.from_enzyme |= 1u << c;
      cat_lists.other[c] = other;
      cat_lists.sweep_rx[sw] |= 1u << c;
      cat_lists.sweep_partners[sw] |= 1u << other;
      sweepers |= 1u << sw;
    }
    for (Pass& ps : passes)
      if (ps.kind == P_CONTACTS) ps.match = Match{{0u, sweepers}};
  }

  // The per-particle passes (recruitment candidates, detachments,
  // conversions) get one draw sweep (k_pass_draws) before the first of them;
  // runs of consecutive ones become list passes (k_particle_passes).  The
  // sweep draws, for each particle, the passes it can reach from its state:
  // a detachment turns alive X into dormant X and a conversion alive `from`
  // into alive `to`; a recruitment apply draws the later passes of the
  // particles it recruits itself.
  int fuse_particle_passes() {
    auto per_particle = [](PassKind k) { return k == P_REC_CAND || k == P_DETACH || k == P_CONV; };
    const EdmDynParams& p = hdp[0];
    std::vector<int> pp_of(passes.size(), -1);
    int n_pp = 0;
    size_t first = passes.size();
    for (size_t i = 0; i < passes.size(); ++i)
      if (per_particle(passes[i].kind)) {
        if (first == passes.size()) first = i;
        pp_of[i] = n_pp++;
      }
    groups.clear();
    draw = DrawPlan{};
    if (n_pp == 0) return EDM_OK;
    if (n_pp > kMaxPP) return fail(EDM_EUNSUP, "more than 32 recruitment/detachment/conversion passes");
    draw.n = n_pp;
    for (size_t i = 0; i < passes.size(); ++i) {
      if (pp_of[i] < 0) continue;
      const PassKind k = passes[i].kind;
      draw.kind[pp_of[i]] = k == P_REC_CAND ? kGroupRecruit : (k == P_DETACH ? kGroupDetach : kGroupConvert);
      draw.index[pp_of[i]] = (int8_t)passes[i].index;
    }
    auto state = [](int sp, int alive) { return 1u << (alive * EDM_MAX_SPECIES + sp); };
    // per-particle passes from position `from` on whose match holds a state of R
    auto matching_from = [&](size_t from, uint32_t R) {
      uint32_t mask = 0;
      for (size_t i = from; i < passes.size(); ++i) {
        if (pp_of[i] < 0) continue;
        const Pass& ps = passes[i];
        const uint32_t M = (ps.match.mask[1] << EDM_MAX_SPECIES) | (ps.match.mask[0] & ((1u << EDM_MAX_SPECIES) - 1));
        if (R & M) mask |= 1u << pp_of[i];
      }
      return mask;
    };
    for (int alive = 0; alive < 2; ++alive)
      for (int sp = 0; sp < p.n_species; ++sp) {
        draw.reach[alive][sp] = matching_from(first, state(sp, alive));
        if (draw.reach[alive][sp]) draw.any.mask[alive] |= 1u << sp;
      }
    for (size_t i = 0; i < passes.size(); ++i) {  // the state a detachment / conversion leaves
      if (passes[i].kind == P_DETACH) draw.after[pp_of[i]] = matching_from(i + 1, state(p.exch[passes[i].index].species, 0));
      if (passes[i].kind == P_CONV) draw.after[pp_of[i]] = matching_from(i + 1, state(p.conv[passes[i].index].to, 1));
    }
    // The sweep only reads flags and ids.  When no per-particle pass matches a
    // species the catalytic passes convert, the passes between the binding
    // passes and the first per-particle pass (adaptation, contact search,
    // catalytic passes, merges) change nothing it reads, so it can start right
    // after the binding passes, on a side stream beside them.
    uint32_t touched = 0, pp_species = 0;
    for (int c = 0; c < p.n_cat; ++c) touched |= (1u << p.cat[c].substrate) | (1u << p.cat[c].product);
    for (size_t i = 0; i < passes.size(); ++i)
      if (pp_of[i] >= 0) pp_species |= passes[i].match.mask[0] | passes[i].match.mask[1];
    size_t at = first;
    draws_early = false;
    if (!(touched & pp_species)) {
      size_t b = 0;
      while (b < first && (passes[b].kind == P_BIND_CAND || passes[b].kind == P_BIND_APPLY || passes[b].kind == P_DISSOC))
        ++b;
      if (b < first) {
        at = b;
        draws_early = true;
      }
    }
    std::vector<Pass> fused;
    for (size_t i = 0; i < passes.size();) {
      if (i == at) fused.push_back({P_DRAWS, 0, draw.any});
      if (!per_particle(passes[i].kind)) {
        if (passes[i].kind == P_REC_APPLY) {
          const int e = passes[i].index;
          rec_after[e] = matching_from(i + 1, state(p.exch[e].species, 1));
        }
        fused.push_back(passes[i++]);
        continue;
      }
      PassGroup G{};
      while (i < passes.size() && per_particle(passes[i].kind) && G.n < kMaxGroup) {
        const int k = pp_of[i];
        G.kind[G.n] = draw.kind[k];
        G.index[G.n] = draw.index[k];
        G.pp[G.n] = (int8_t)k;
        G.m[G.n] = passes[i].match;
        G.bits |= 1u << k;
        ++G.n;
        ++i;
      }
      groups.push_back(G);
      fused.push_back({P_GROUP, (int)groups.size() - 1, Match{}});
    }
    passes.swap(fused);
    return EDM_OK;
  }

  // Draw thresholds, per replica: ceil(b 2^53) for the bound b = prob times
  // the largest Hill factor of each of the pass's rules, multiplied in the
  // order the pass multiplies its factors, so that b >= the pass's
  // probability for any grid count.
  int upload_thresholds() {
    auto thr_of = [](double b) -> uint64_t {
      if (!(b > 0.0)) return 0;
      const double B = std::ceil(std::ldexp(b, 53));
      return B >= 9007199254740992.0 ? (1ull << 53) : (uint64_t)B;
    };
    std::vector<uint64_t> pt((size_t)R * kMaxPP, 0), ct((size_t)R * EDM_MAX_CAT, 0);
    for (int r = 0; r < R; ++r) {
      const EdmDynParams& q = hdp[r];
      const double* rm = &rule_max[(size_t)r * EDM_MAX_RULES];
      for (int k = 0; k < draw.n; ++k) {
        const int idx = draw.index[k];
        double b;
        if (draw.kind[k] == kGroupRecruit) {
          const EdmExch& X = q.exch[idx];
          b = X.prob_on;
          if (X.rule_on >= 0) {
            b = b * rm[X.rule_on];
            if (X.rule_on2 >= 0) b = b * rm[X.rule_on2];
          }
        } else if (draw.kind[k] == kGroupDetach) {
          const EdmExch& X = q.exch[idx];
          b = X.rule_off >= 0 ? X.prob_off * rm[X.rule_off] : X.prob_off;
        } else {
          const EdmConv& V = q.conv[idx];
          b = V.rule >= 0 ? V.prob * rm[V.rule] : V.prob;
        }
        pt[(size_t)r * kMaxPP + k] = thr_of(b);
      }
      for (int c = 0; c < q.n_cat; ++c) {
        const EdmCat& C = q.cat[c];
        ct[(size_t)r * EDM_MAX_CAT + c] = thr_of(C.rule >= 0 ? C.prob * rm[C.rule] : C.prob);
      }
    }
    CUDA_TRY(cudaMemcpy(pass_thr, pt.data(), sizeof(uint64_t) * pt.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(cat_thr, ct.data(), sizeof(uint64_t) * ct.size(), cudaMemcpyHostToDevice));
    int rc;
    if ((rc = alloc(&d_draw, 1)) != EDM_OK || (rc = alloc(&d_groups, std::max<size_t>(1, groups.size()))) != EDM_OK)
      return rc;
    CUDA_TRY(cudaMemcpy(d_draw, &draw, sizeof(DrawPlan), cudaMemcpyHostToDevice));
    if (!groups.empty())
      CUDA_TRY(cudaMemcpy(d_groups, groups.data(), sizeof(PassGroup) * groups.size(), cudaMemcpyHostToDevice));
    return EDM_OK;
  }

  // optional CUDA events between kernel groups and between reaction passes (profiling only)
  cudaEvent_t* prof = nullptr;
  cudaEvent_t* pass_prof = nullptr;
  bool prof_capture = false;  // marks become event-record nodes of a graph being captured
  void mark(int k, cudaStream_t s) {
    if (!prof) return;
    if (prof_capture) cudaEventRecordWithFlags(prof[k], s, cudaEventRecordExternal);
    else cudaEventRecord(prof[k], s);
  }

  void tune_mark(int kernel, int k, cudaStream_t s) {
    if (tune_kernel == kernel) cudaEventRecord(tune_ev[k], s);
  }

  // Launches of the BD step's chain on its stream.  When the operation
  // before it on the stream is a kernel of the chain (pdl_chain), the kernel
  // goes as a programmatic dependent of that kernel: its blocks are scheduled
  // while the predecessor drains and wait in pdl_enter() for its completion,
  // so the launch latency between the two overlaps the predecessor's tail.
  // Anything else on the stream (an event wait, a record, a copy) ends the
  // chain: the next kernel goes with the ordinary full dependency.  Off
  // while profiling or tuning, whose event records sit between the kernels,
  // and with EDM_PDL=0 in the environment at engine creation, and on the
  // default streams.
  bool pdl_on = true;
  bool pdl_chain = false;
  template <typename... K, typename... A>
  void go(void (*kernel)(K...), dim3 grid, int block, cudaStream_t s, A&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    // created streams only (not the legacy or per-thread default stream)
    const bool created = reinterpret_cast<uintptr_t>(s) > 2;
    cfg.numAttrs = (pdl_on && pdl_chain && created && !prof && !pass_prof && tune_kernel < 0) ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
    pdl_chain = true;
  }

  template <bool F64>
  void launch_scatter(const DevState& st, cudaStream_t s) {
    const LaunchShape sh = kShapes[TK_SCATTER][shape[TK_SCATTER]];
    const int t = tile_index(sh.block);
    if (npblk_bs[t] == 0) return;
    const int nt = npblk_bs[t];
    const int2* b = pblk_bs[t];
    switch (shape[TK_SCATTER]) {  // the rows of kShapes[TK_SCATTER]
      case 1: go(k_scatter<F64, 128, 1>, nt, 128, s, dp, b, nt, st); break;
      case 2: go(k_scatter<F64, 512, 1>, nt, 512, s, dp, b, nt, st); break;
      case 3: go(k_scatter<F64, 128, 2>, (nt + 1) / 2, 128, s, dp, b, nt, st); break;
      case 4: go(k_scatter<F64, 256, 2>, (nt + 1) / 2, 256, s, dp, b, nt, st); break;
      default: go(k_scatter<F64, 256, 1>, nt, 256, s, dp, b, nt, st); break;
    }
  }

  template <bool F64>
  void launch_move(const DevState& st, cudaStream_t s) {
    const int v = shape[TK_MOVE];
    const int t = tile_index(kShapes[TK_MOVE][v].block);
    if (npblk_bs[t] == 0) return;
    const int n = npblk_bs[t];
    const int2* b = pblk_bs[t];
    switch (v) {  // the rows of kShapes[TK_MOVE]
      case 1: go(k_move<F64, 256, 4>, n, 256, s, dp, b, st); break;
      case 2: go(k_move<F64, 128, 8>, n, 128, s, dp, b, st); break;
      case 3: go(k_move<F64, 128, 10>, n, 128, s, dp, b, st); break;
      case 4: go(k_move<F64, 128, 12>, n, 128, s, dp, b, st); break;
      case 5: go(k_move<F64, 128, 16>, n, 128, s, dp, b, st); break;
      case 6: go(k_move<F64, 256, 6>, n, 256, s, dp, b, st); break;
      case 7: go(k_move<F64, 256, 8>, n, 256, s, dp, b, st); break;
      default: go(k_move<F64, 256, 3>, n, 256, s, dp, b, st); break;
    }
  }

  template <bool F64>
  void launch_contacts(const DevState& st, const Match& m, int grid, cudaStream_t s) {
    const int grid16 = (int)((N + 16 * kBlock - 1) / (16 * kBlock));  // 16 slots per thread
    if (grid16 == 0) return;
    switch (shape[TK_CONTACTS]) {  // the rows of kShapes[TK_CONTACTS]
      case 1: go(k_contacts_cols<F64, 6>, grid, kBlock, s, dp, st, m, cat_lists); break;
      case 2: go(k_contacts_cols<F64, 4>, grid, kBlock, s, dp, st, m, cat_lists); break;
      case 3: go(k_contacts_block<F64, 6, 16>, grid16, kBlock, s, dp, st, m, cat_lists); break;
      case 4: go(k_contacts_block<F64, 4, 16>, grid16, kBlock, s, dp, st, m, cat_lists); break;
      case 5: go(k_contacts_block<F64, 6, 4>, grid, kBlock, s, dp, st, m, cat_lists); break;
      case 6:
      case 7:
        go(k_sweep_list, grid16, kBlock, s, st, m);
        if (shape[TK_CONTACTS] == 6) go(k_contacts_list<F64, 6>, 148 * 6, kBlock, s, dp, st, cat_lists);
        else go(k_contacts_list<F64, 8>, 148 * 8, kBlock, s, dp, st, cat_lists);
        break;
      default: go(k_contacts<F64, 6>, grid, kBlock, s, dp, st, m, cat_lists); break;
    }
  }

  template <bool F64>
  void enqueue_dynamics_t(cudaStream_t s) {
    const int nbs = nb_scan;
    mark(0, s);
    StepZero z{};
    z.p[0] = grid_cnt, z.n[0] = grid_cnt ? n_grid : 0;
    z.p[1] = grid_delta, z.n[1] = grid_delta ? n_grid : 0;
    z.p[2] = moved_count, z.n[2] = R;
    z.p[3] = contact_count, z.n[3] = contact_count ? EDM_MAX_CAT : 0;
    z.p[4] = pl_count, z.n[4] = pl_count ? 1 : 0;
    z.p[5] = sw_count, z.n[5] = sw_count ? 1 : 0;
    k_scan_reduce<<<nbs, kScanThreads, 0, s>>>(cnt, n_cells, bsum, z);  // starts the chain
    pdl_chain = true;
    go(k_scan_bsum, 1, 1024, s, bsum, nbs);
    // the previous step's photon pass reads the slots and positions the sort
    // rewrites, and with proximity FRET the bucket starts
    if (phot_uses_cells) join_photons(s);
    go(k_scan_down, nbs, kScanThreads, s, cnt, n_cells, bsum, cell_start, cursor);
    join_photons(s);
    mark(1, s);
    cur ^= 1;
    DevState st = dev_state();
    tune_mark(TK_SCATTER, 0, s);
    launch_scatter<F64>(st, s);
    tune_mark(TK_SCATTER, 1, s);
    mark(2, s);
    tune_mark(TK_MOVE, 0, s);
    launch_move<F64>(st, s);
    tune_mark(TK_MOVE, 1, s);
    mark(3, s);
    const int rb = (R + 127) / 128;
    const int sgrid = (int)std::max<int64_t>(1, (N / 4 + kBlock) / kBlock);  // 4 slots per thread
    const int cgrid = 148 * 8;
    const int gm = (int)std::min<int64_t>((n_grid + 255) / 256, 4096);
    bool joined = true;  // the side stream's draw sweep has been waited for
    for (size_t i = 0; i < passes.size(); ++i) {
      const Pass& ps = passes[i];
      if (pass_prof) cudaEventRecord(pass_prof[i], s);
      switch (ps.kind) {
        case P_BIND_CAND: go(k_bind_candidates<F64>, sgrid, kBlock, s, dp, st, ps.match, ps.index); break;
        case P_BIND_APPLY: go(k_bind_apply<F64>, rb, 128, s, dp, R, st, ps.index); break;
        case P_DISSOC: go(k_dissociate<F64>, sgrid, kBlock, s, dp, st, ps.match, ps.index); break;
        case P_CONTACTS:
          tune_mark(TK_CONTACTS, 0, s);
          launch_contacts<F64>(st, ps.match, sgrid, s);
          tune_mark(TK_CONTACTS, 1, s);
          break;
        case P_CAT: go(k_catalytic<F64>, cgrid, kBlock, s, dp, st, ps.index, cat_late[ps.index]); break;
        case P_REC_APPLY: go(k_recruit_apply<F64>, rb, 128, s, dp, R, st, ps.index, d_draw, rec_after[ps.index]); break;
        case P_DRAWS: {
          // beside the following passes on the side stream (not while timing passes one by one)
          const bool fork = draws_early && !pass_prof && side_stream;
          cudaStream_t ds = s;
          if (fork) {
            cudaEventRecord(ev_fork, s);
            cudaStreamWaitEvent(side_stream, ev_fork, 0);
            ds = side_stream;
            pdl_chain = false;
          }
          if (fork) k_pass_draws<<<sgrid, kBlock, 0, ds>>>(dp, st, d_draw, draw.any);
          else go(k_pass_draws, sgrid, kBlock, s, dp, st, d_draw, draw.any);
          if (fork) {
            cudaEventRecord(ev_join, side_stream);
            joined = false;
          }
          break;
        }
        case P_GROUP:
          if (!joined) {
            cudaStreamWaitEvent(s, ev_join, 0);
            joined = true;
            pdl_chain = false;
          }
          go(k_particle_passes<F64>, 148, kBlock, s, dp, st, d_groups + ps.index, d_draw);
          break;
        case P_ADAPT: go(k_adapt, dim3(4, R), 256, s, dp, grid_cnt, adapt_w); break;
        case P_LOCAL_CDF: go(k_local_cdf, R, 256, s, dp, grid_cnt, local_cdf, ps.index); break;
        case P_REC_CAND:
        case P_DETACH:
        case P_CONV: break;  // fused into P_GROUP passes
        case P_MERGE: go(k_grid_merge, gm > 0 ? gm : 1, 256, s, grid_cnt, grid_delta, n_grid); break;
      }
    }
    if (pass_prof) cudaEventRecord(pass_prof[passes.size()], s);
    go(k_step_inc, 1, 1, s, d_step);
    cells_valid = true;
    mark(4, s);
  }

  int launches_per_step(bool with_photons) const {
    int n = 3 + 1 + 1 + (int)passes.size() + 1;
    for (const Pass& ps : passes)  // the sweeper-list contact shapes launch two kernels
      if (ps.kind == P_CONTACTS && shape[TK_CONTACTS] >= 6) ++n;
    if (with_photons) n += (neblk > 0 ? 3 : 1) + 1 + (nphblk > 0 ? 1 : 0) + 1;
    if (rec_cap > 0) n += 2 + ((has_phot && neblk > 0) ? 1 : 0);
    return n;
  }

  void enqueue_dynamics(cudaStream_t s) {
    if (f64) enqueue_dynamics_t<true>(s);
    else enqueue_dynamics_t<false>(s);
  }

  template <bool F64>
  void enqueue_photons_t(cudaStream_t s) {
    DevState st = dev_state();
    PhotState ph = phot_state();
    if (neblk > 0) k_phot_count<F64><<<neblk, kBlock, 0, s>>>(dp, pp, eblk, st, ph, cells_valid ? 1 : 0);
    k_phot_scan<<<R, 256, 0, s>>>(pp, ph, counters, status);
    if (neblk > 0) k_phot_write<F64><<<neblk, kBlock, 0, s>>>(dp, pp, eblk, st, ph, counters);
    k_phot_advance<<<1, 1, 0, s>>>(d_pstep, d_batch_key);
  }

  void enqueue_photons(cudaStream_t s) {
    if (f64) enqueue_photons_t<true>(s);
    else enqueue_photons_t<false>(s);
  }

  template <bool F64>
  void enqueue_scope_t(cudaStream_t s) {
    DevState st = dev_state();
    PhotState ph = phot_state();
    if (nphblk > 0) k_scope<F64><<<nphblk, kBlock, 0, s>>>(dp, pp, sp, phblk, st, ph);
    k_scope_received<<<(R + 127) / 128, 128, 0, s>>>(pp, R, ph, counters);
  }

  void enqueue_scope(cudaStream_t s) {
    if (f64) enqueue_scope_t<true>(s);
    else enqueue_scope_t<false>(s);
  }

  // The positions of the current photon batch from the current state (a batch
  // the host set, before a standalone detection pass).
  void enqueue_photon_positions(cudaStream_t s) {
    if (nphblk == 0) return;
    DevState st = dev_state();
    PhotState ph = phot_state();
    if (f64) k_photon_positions<true><<<nphblk, kBlock, 0, s>>>(dp, pp, phblk, st, ph);
    else k_photon_positions<false><<<nphblk, kBlock, 0, s>>>(dp, pp, phblk, st, ph);
  }

  // A step's photon pass and detection pass beside the next step, each on a
  // stream of its own.  The photon pass reads the step's final state: the next
  // step's bucket scan may run beside it, its bucket starts and sort may not
  // (enqueue_dynamics joins it before them).  The detection pass reads only the
  // photon records, which carry their positions: the next step's dynamics run
  // beside it, the next photon pass waits for it.  A census and the end of the
  // call wait for both.  Errors surface at the call's cudaGetLastError or at
  // the capture's end.
  cudaStream_t phot_stream = nullptr, scope_stream = nullptr;
  bool phot_uses_cells = true;  // some replica's FRET is by proximity (a cell-list search)
  cudaEvent_t ev_phot_fork = nullptr, ev_phot_join = nullptr, ev_scope_join = nullptr;
  bool phot_pending = false, scope_pending = false;
  void enqueue_photons_beside(cudaStream_t s) {
    cudaEventRecord(ev_phot_fork, s);
    cudaStreamWaitEvent(phot_stream, ev_phot_fork, 0);
    if (scope_pending) cudaStreamWaitEvent(phot_stream, ev_scope_join, 0);  // the records are free again
    enqueue_photons(phot_stream);
    cudaEventRecord(ev_phot_join, phot_stream);
    cudaStreamWaitEvent(scope_stream, ev_phot_join, 0);
    enqueue_scope(scope_stream);
    cudaEventRecord(ev_scope_join, scope_stream);
    phot_pending = scope_pending = true;
  }
  void join_photons(cudaStream_t s) {
    if (!phot_pending) return;
    cudaStreamWaitEvent(s, ev_phot_join, 0);
    phot_pending = false;
    pdl_chain = false;
  }
  void join_beside(cudaStream_t s) {
    join_photons(s);
    if (!scope_pending) return;
    cudaStreamWaitEvent(s, ev_scope_join, 0);
    scope_pending = false;
    pdl_chain = false;
  }

  // Census of the state into `base` (ring of `cap` steps, or one block when
  // cap == 0): counters, bonds, bleaching, species; with photophysics the
  // donor and free-dye counts (with_cls: donors per FRET class of the step's
  // photon pass).
  void enqueue_census(cudaStream_t s, int64_t* base, int cap, bool with_cls) {
    DevState st = dev_state();
    PhotState ph = phot_state();
    const int nrow = R * EDM_CENSUS_FIELDS;
    k_census_begin<<<(nrow + 255) / 256, 256, 0, s>>>(base, cap, d_step, R, counters);
    k_census_particles<<<npblk, kBlock, 0, s>>>(dp, pblk, st, has_phot ? bleached : nullptr, base, cap,
                                               hdp[0].n_species);
    if (has_phot && neblk > 0) k_census_emitters<<<neblk, kBlock, 0, s>>>(pp, eblk, st, ph, base, cap, with_cls ? 1 : 0);
  }

  std::tuple<int, int, int, int> tune_key(int kernel) const {
    int lg = 0;
    while ((int64_t(1) << (lg + 1)) <= N) ++lg;
    return std::make_tuple(kernel, precision, R, lg);
  }

  void drop_graphs() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    graphs.clear();
  }

  // overlapped frame readout (edm_frame_out_begin / _wait)
  uint32_t* flim_snap = nullptr;
  // one bit per 128-bin stretch of the stacks that a count has landed in
  // since the last clear: the sparse readout visits only these
  uint32_t* touch = nullptr;
  int64_t n_touch = 0;  // words
  // sparse frame readout: block counts and offsets, device output of sp_cap entries
  int32_t* sp_bcount = nullptr;
  int64_t* sp_off = nullptr;
  int64_t* sp_idx = nullptr;
  uint32_t* sp_cnt = nullptr;
  int64_t sp_cap = 0;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_snap = nullptr, ev_read = nullptr;
  bool read_pending = false;

  // asynchronous state transfers (edm_set_state_async / edm_get_state_async):
  // the host arrays land in (leave from) device staging of their own, on an
  // upload (download) stream, so the link works while `stream` computes
  struct Xfer {
    double* pos = nullptr;
    int32_t *sp = nullptr, *bond = nullptr, *dye = nullptr;
    uint8_t *alive = nullptr, *has_dye = nullptr, *bleached = nullptr;
    int8_t* ctmc = nullptr;
  } in, out;
  cudaStream_t up_stream = nullptr, down_stream = nullptr;
  cudaEvent_t ev_staged = nullptr, ev_in_free = nullptr, ev_out_ready = nullptr, ev_out_free = nullptr;
  bool in_used = false, out_used = false, staged = false;

  int xfer_setup() {
    if (up_stream) return EDM_OK;
    int rc;
    const size_t n = (size_t)std::max<int64_t>(N, 1);
    for (Xfer* x : {&in, &out}) {
      if ((rc = alloc(&x->pos, 2 * n)) != EDM_OK || (rc = alloc(&x->sp, n)) != EDM_OK ||
          (rc = alloc(&x->bond, n)) != EDM_OK || (rc = alloc(&x->dye, n)) != EDM_OK ||
          (rc = alloc(&x->alive, n)) != EDM_OK || (rc = alloc(&x->has_dye, n)) != EDM_OK ||
          (rc = alloc(&x->bleached, n)) != EDM_OK || (rc = alloc(&x->ctmc, n)) != EDM_OK)
        return rc;
    }
    CUDA_TRY(cudaStreamCreateWithFlags(&up_stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaStreamCreateWithFlags(&down_stream, cudaStreamNonBlocking));
    for (cudaEvent_t* ev : {&ev_staged, &ev_in_free, &ev_out_ready, &ev_out_free})
      CUDA_TRY(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
    return EDM_OK;
  }

  ~EdmEngine() {
    for (auto& ev : tune_ev)
      if (ev) cudaEventDestroy(ev);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side_stream) cudaStreamDestroy(side_stream);
    if (ev_snap) cudaEventDestroy(ev_snap);
    if (ev_read) cudaEventDestroy(ev_read);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (up_stream) cudaStreamDestroy(up_stream);
    if (phot_stream) cudaStreamDestroy(phot_stream);
    if (scope_stream) cudaStreamDestroy(scope_stream);
    for (cudaEvent_t ev : {ev_phot_fork, ev_phot_join, ev_scope_join})
      if (ev) cudaEventDestroy(ev);
    if (down_stream) cudaStreamDestroy(down_stream);
    for (cudaEvent_t ev : {ev_staged, ev_in_free, ev_out_ready, ev_out_free})
      if (ev) cudaEventDestroy(ev);
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    for (void* p : allocs) cudaFree(p);
  }
};

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

int edm_abi_version(void) { return EDM_ABI_VERSION; }

int64_t edm_abi_sizeof(int which) {
  switch (which) {
    case 0: return (int64_t)sizeof(EdmDynParams);
    case 1: return (int64_t)sizeof(EdmPhotParams);
    case 2: return (int64_t)sizeof(EdmScopeParams);
    case 3: return (int64_t)sizeof(EdmHostState);
    case 4: return (int64_t)sizeof(EdmFlimParams);
    default: return -1;
  }
}

const char* edm_last_error(void) { return g_last_error.c_str(); }

// Upper bound of a rule's Hill factor over every grid count: the largest
// exact table entry, and beyond the table the device expression, which is at
// most 1 for inhibition and at most max(1, basal) for activation (1 without
// K_half); the relative margin covers the expression's last-place rounding.
static double rule_factor_bound(const EdmRule& R, const double* hill) {
  double m = 1.0;
  for (int64_t i = 0; i < R.table_len; ++i) m = std::max(m, hill[R.table_offset + i]);
  if (R.K_half > 0 && !R.inhibition) m = std::max(m, R.basal);
  return m * (1.0 + 1e-12);
}

int edm_create(const EdmDynParams* dyn, const EdmPhotParams* phot, const EdmScopeParams* scope, int32_t n_replicas,
               const double* hill, int64_t n_hill, int32_t precision, int32_t device, EdmEngine** out) {
  if (!dyn || !out || n_replicas <= 0) return fail(EDM_EINVAL, "edm_create: null argument or no replicas");
  if (precision != 32 && precision != 64) return fail(EDM_EINVAL, "edm_create: precision must be 32 or 64");
  *out = nullptr;
  CUDA_TRY(cudaSetDevice(device));
  EdmEngine* E = new EdmEngine();
  E->device = device;
  E->precision = precision;
  E->f64 = precision == 64;
  E->R = n_replicas;
  if (const char* pdl = std::getenv("EDM_PDL")) E->pdl_on = pdl[0] != '0';
  E->hdp.assign(dyn, dyn + n_replicas);
  E->has_phot = phot != nullptr;
  E->has_scope = scope != nullptr && phot != nullptr;
  if (E->has_phot) E->hpp.assign(phot, phot + n_replicas);
  if (E->has_scope) E->hsp.assign(scope, scope + n_replicas);
  for (int r = 0; E->has_scope && r < n_replicas; ++r)
    if (E->hsp[r].psf_range_px < 0 || E->hsp[r].psf_range_px > kPsfMaxR) {
      delete E;
      return fail(EDM_EUNSUP, "edm_create: PSF window wider than 16 pixels each side (pixels below sigma/4)");
    }
  // validate the CSR layout and that every replica has the same pass structure
  int64_t np = 0, nc = 0, ng = 0, ne = 0, nph = 0, nfl = 0;
  std::vector<int64_t> pfirst, pcount, efirst, ecount, phfirst, phcount, pxfirst, pxcount;
  const EdmDynParams& p0 = E->hdp[0];
  for (int r = 0; r < n_replicas; ++r) {
    const EdmDynParams& p = E->hdp[r];
    if (p.particle_offset != np || p.cell_offset != nc) {
      delete E;
      return fail(EDM_EINVAL, "edm_create: replica offsets must be contiguous and in order");
    }
    if (p.n_species > EDM_MAX_SPECIES || p.n_species > 127 || p.nx < 3 || p.ny < 3 || p.n_bind > EDM_MAX_BIND ||
        p.n_cat > EDM_MAX_CAT || p.n_exch > EDM_MAX_EXCH || p.n_conv > EDM_MAX_CONV || p.n_grids > EDM_MAX_GRIDS ||
        p.n_rules > EDM_MAX_RULES) {
      delete E;
      return fail(EDM_EINVAL, "edm_create: parameter block out of range");
    }
    if (p.n_bind != p0.n_bind || p.n_cat != p0.n_cat || p.n_exch != p0.n_exch || p.n_conv != p0.n_conv ||
        p.n_grids != p0.n_grids) {
      delete E;
      return fail(EDM_EINVAL, "edm_create: replicas must share one reaction structure");
    }
    for (int g = 0; g < p.n_grids; ++g) {
      if (p.grid[g].offset != ng) {
        delete E;
        return fail(EDM_EINVAL, "edm_create: density-grid offsets must be contiguous");
      }
      ng += (int64_t)p.grid[g].nx * p.grid[g].ny;
    }
    for (int k = 0; k < p.n_rules; ++k) {
      if (p.rule[k].table_offset < 0 || p.rule[k].table_offset + p.rule[k].table_len > n_hill) {
        delete E;
        return fail(EDM_EINVAL, "edm_create: Hill table out of range");
      }
    }
    if (p.adapt_grid >= p.n_grids || p.adapt_grid != p0.adapt_grid) {
      delete E;
      return fail(EDM_EINVAL, "edm_create: adaptation grid out of range or not shared by the replicas");
    }
    for (int e = 0; e < p.n_exch; ++e) {
      if (p.exch[e].local_recruit != p0.exch[e].local_recruit ||
          (p.exch[e].local_recruit && (p.exch[e].rule_on < 0 || p.exch[e].rule_on >= p.n_rules))) {
        delete E;
        return fail(EDM_EINVAL, "edm_create: local recruitment needs a feedback rule, the same in every replica");
      }
    }
    pfirst.push_back(np);
    pcount.push_back(p.n_particles);
    np += p.n_particles;
    nc += (int64_t)p.nx * p.ny + 1;
    if (E->has_phot) {
      const EdmPhotParams& q = E->hpp[r];
      if (q.photon_offset != nph) {
        delete E;
        return fail(EDM_EINVAL, "edm_create: photon buffer offsets must be contiguous");
      }
      phfirst.push_back(nph);
      phcount.push_back(q.max_photons);
      nph += q.max_photons;
    }
    if (E->has_scope) {
      const EdmScopeParams& s = E->hsp[r];
      if (s.flim_offset != nfl) {
        delete E;
        return fail(EDM_EINVAL, "edm_create: FLIM stack offsets must be contiguous");
      }
      const int64_t npx = (int64_t)s.n_channels * s.nx * s.ny;
      pxfirst.push_back(0);
      pxcount.push_back(npx);
      nfl += npx * s.n_bins;
    }
  }
  if (np >= (int64_t)1 << 31) {
    delete E;
    return fail(EDM_EINVAL, "edm_create: more than 2^31 particles");
  }
  E->N = np;
  E->n_cells = nc;
  E->n_grid = ng;
  E->n_hill = n_hill;
  E->n_phcap = nph;
  E->n_flim = nfl;
  int rc = EDM_OK;
#define ALLOC(ptr, n)                        \
  if ((rc = E->alloc(&(ptr), (n))) != EDM_OK) { \
    delete E;                                \
    return rc;                               \
  }
  ALLOC(E->dp, (size_t)n_replicas);
  CUDA_TRY(cudaMemcpy(E->dp, dyn, sizeof(EdmDynParams) * n_replicas, cudaMemcpyHostToDevice));
  ALLOC(E->hill, (size_t)n_hill);
  if (n_hill > 0) CUDA_TRY(cudaMemcpy(E->hill, hill, sizeof(double) * n_hill, cudaMemcpyHostToDevice));
  E->rule_max.assign((size_t)n_replicas * EDM_MAX_RULES, 1.0);
  for (int r = 0; r < n_replicas; ++r)
    for (int k = 0; k < dyn[r].n_rules; ++k) E->rule_max[(size_t)r * EDM_MAX_RULES + k] = rule_factor_bound(dyn[r].rule[k], hill);
  ALLOC(E->pass_thr, (size_t)n_replicas * kMaxPP);
  ALLOC(E->cat_thr, (size_t)n_replicas * EDM_MAX_CAT);
  const size_t psz = E->f64 ? sizeof(double2) : sizeof(float2);
  uint8_t *pp0 = nullptr, *pp1 = nullptr;
  ALLOC(pp0, psz * np);
  ALLOC(pp1, psz * np);
  E->pos_pre = pp0;
  E->pos_post = pp1;
  if (!E->f64) {  // float32 remainders of the offsets
    ALLOC(E->lo_pre, np);
    ALLOC(E->lo_post, np);
  }
  ALLOC(E->cell_pre, np);
  ALLOC(E->cell_post, np);
  ALLOC(E->flags[0], np + 4);
  ALLOC(E->flags[1], np + 4);
  ALLOC(E->ids[0], np);
  ALLOC(E->ids[1], np);
  ALLOC(E->slot_of_id, np);
  ALLOC(E->bond, np);
  ALLOC(E->has_dye, np);
  ALLOC(E->bleached, np);
  ALLOC(E->dye, np);
  ALLOC(E->ctmc, np);
  ALLOC(E->cell_start, nc + 1);
  ALLOC(E->cursor, nc);
  ALLOC(E->cnt, nc);
  E->nb_scan = (int)((nc + kScanTile - 1) / kScanTile);
  if (E->nb_scan < 1) E->nb_scan = 1;
  ALLOC(E->bsum, (size_t)E->nb_scan);
  ALLOC(E->grid_cnt, ng);
  ALLOC(E->grid_delta, ng);
  ALLOC(E->counters, (size_t)n_replicas * EDM_NCOUNTERS);
  ALLOC(E->status, 1);
  ALLOC(E->d_step, 1);
  ALLOC(E->d_pstep, 1);
  ALLOC(E->d_batch_key, 1);
  ALLOC(E->rec_count, n_replicas);
  ALLOC(E->rec_id, (size_t)n_replicas * kRecCap);
  ALLOC(E->rec_xy, (size_t)n_replicas * kRecCap * 2);
  ALLOC(E->bind_count, n_replicas);
  ALLOC(E->bind_key, (size_t)n_replicas * kBindCap);
  ALLOC(E->bind_ab, (size_t)n_replicas * kBindCap * 2);
  for (const EdmDynParams& q : E->hdp)
    for (int g = 0; g < q.n_grids && g < EDM_MAX_GRIDS; ++g)
      if (q.grid[g].sensor >= 0 && q.grid[g].sensor < EDM_MAX_SPECIES) E->sensor_grids[q.grid[g].sensor] |= 1u << g;
  if ((rc = E->build_schedule()) != EDM_OK || (rc = E->upload_thresholds()) != EDM_OK) {
    delete E;
    return rc;
  }
  if (E->has_phot) {
    E->phot_uses_cells = false;
    for (const EdmPhotParams& q : E->hpp)
      for (int f = 0; f < q.n_fret && f < EDM_MAX_FRET; ++f)
        if (q.fret[f].mode != 0) E->phot_uses_cells = true;
  }
  if (E->has_scope) {
    CUDA_TRY(cudaStreamCreateWithFlags(&E->phot_stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaStreamCreateWithFlags(&E->scope_stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&E->ev_phot_fork, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&E->ev_phot_join, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&E->ev_scope_join, cudaEventDisableTiming));
  }
  if (E->draws_early) {
    CUDA_TRY(cudaStreamCreateWithFlags(&E->side_stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&E->ev_fork, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&E->ev_join, cudaEventDisableTiming));
  }
  E->contact_cap = std::max<int64_t>(4 * np, 1 << 20);  // per catalytic reaction
  ALLOC(E->contacts, (size_t)E->contact_cap * std::max(1, E->hdp[0].n_cat));
  ALLOC(E->contact_count, EDM_MAX_CAT);
  ALLOC(E->moved, np);
  ALLOC(E->moved_count, (size_t)n_replicas);
  ALLOC(E->pl, (size_t)np);
  ALLOC(E->pl_count, 1);
  ALLOC(E->pl_index, (size_t)np);
  ALLOC(E->sw_list, (size_t)np);
  ALLOC(E->sw_count, 1);
  ALLOC(E->adapt_w, (size_t)std::max<int64_t>(ng, 1));
  ALLOC(E->local_cdf, (size_t)std::max<int64_t>(ng, 1));
  CUDA_TRY(cudaMemset(E->pl_index, 0xFF, sizeof(int32_t) * np));
  CUDA_TRY(cudaMemset(E->pl_count, 0, sizeof(int32_t)));
  ALLOC(E->rep_first, (size_t)n_replicas + 1);
  {
    std::vector<int64_t> rf(pfirst);
    rf.push_back(np);
    CUDA_TRY(cudaMemcpy(E->rep_first, rf.data(), sizeof(int64_t) * rf.size(), cudaMemcpyHostToDevice));
    const int64_t nchunks = (np + kSweepChunk - 1) / kSweepChunk;
    std::vector<int32_t> cr((size_t)std::max<int64_t>(1, nchunks), 0);
    int r = 0;
    for (int64_t c = 0; c < nchunks; ++c) {
      while (r + 1 < n_replicas && rf[r + 1] <= c * kSweepChunk) ++r;
      cr[(size_t)c] = r;
    }
    ALLOC(E->chunk_rep, cr.size());
    CUDA_TRY(cudaMemcpy(E->chunk_rep, cr.data(), sizeof(int32_t) * cr.size(), cudaMemcpyHostToDevice));
  }
  for (int t = 0; t < 3; ++t) {
    std::vector<int2> pt = tiles(pfirst, pcount, kTileSizes[t]);
    E->npblk_bs[t] = (int)pt.size();
    ALLOC(E->pblk_bs[t], std::max<size_t>(1, pt.size()));
    if (!pt.empty())
      CUDA_TRY(cudaMemcpy(E->pblk_bs[t], pt.data(), sizeof(int2) * pt.size(), cudaMemcpyHostToDevice));
  }
  E->pblk = E->pblk_bs[1];
  E->npblk = E->npblk_bs[1];
  {  // launch shapes chosen by an earlier tuning of an engine of this kind
    std::lock_guard<std::mutex> lock(g_tune_mu);
    for (int k = 0; k < TK_COUNT; ++k) {
      auto it = g_tuned.find(E->tune_key(k));
      if (it != g_tuned.end()) E->shape[k] = it->second;
    }
  }
  if (E->has_phot) {
    ALLOC(E->pp, (size_t)n_replicas);
    ALLOC(E->emit_id, np);
    ALLOC(E->emit_n, np);
    ALLOC(E->emit_nd, np);
    ALLOC(E->emit_acc, np);
    ALLOC(E->emit_cls, np);
    ALLOC(E->emit_off, np);
    ALLOC(E->ph_pid, nph);
    ALLOC(E->ph_t, nph);
    ALLOC(E->ph_ch, nph);
    ALLOC(E->ph_fret, nph);
    ALLOC(E->ph_xy, nph);
    ALLOC(E->ph_count, n_replicas);
    std::vector<int2> ph = tiles(phfirst, phcount);
    E->nphblk = (int)ph.size();
    ALLOC(E->phblk, ph.size());
    if (!ph.empty()) CUDA_TRY(cudaMemcpy(E->phblk, ph.data(), sizeof(int2) * ph.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(E->pp, E->hpp.data(), sizeof(EdmPhotParams) * n_replicas, cudaMemcpyHostToDevice));
  }
  if (E->has_scope) {
    ALLOC(E->sp, (size_t)n_replicas);
    CUDA_TRY(cudaMemcpy(E->sp, E->hsp.data(), sizeof(EdmScopeParams) * n_replicas, cudaMemcpyHostToDevice));
    ALLOC(E->flim, (size_t)nfl);
    E->n_touch = (nfl + 4095) / 4096;
    ALLOC(E->touch, (size_t)std::max<int64_t>(E->n_touch, 1));  // zeroed, as every allocation
    std::vector<int2> px = tiles(pxfirst, pxcount);
    E->npxblk = (int)px.size();
    ALLOC(E->pxblk, px.size());
    if (!px.empty()) CUDA_TRY(cudaMemcpy(E->pxblk, px.data(), sizeof(int2) * px.size(), cudaMemcpyHostToDevice));
  }
  ALLOC(E->st_sp, np);
  ALLOC(E->st_bond, np);
  ALLOC(E->st_alive, np);
  ALLOC(E->st_bl, np);
  ALLOC(E->st_ctmc, np);
  ALLOC(E->st_pos, (size_t)np * 2);
#undef ALLOC
  CUDA_TRY(cudaDeviceSynchronize());
  *out = E;
  return EDM_OK;
}

int edm_destroy(EdmEngine* eng) {
  if (!eng) return EDM_OK;
  cudaSetDevice(eng->device);
  cudaDeviceSynchronize();
  delete eng;
  return EDM_OK;
}

}  // extern "C"

// ---- state upload / download ------------------------------------------------
namespace {

// ---- sparse frame readout ----------------------------------------------------
// A frame's TCSPC stacks are mostly zero (about one bin in a thousand holds a
// photon at the bench's rates), so the readout can move only the nonzero
// bins.  Warp w owns the elements [w chunk, (w + 1) chunk) of the
// concatenated stacks; a counting pass and a scan of the warp counts give
// each warp its output offset, and the writing pass emits (element index,
// count) in index order and clears the bins it emits.  Warps work alone (no
// block barrier), and a 128-element stretch without a photon costs the
// writing pass one ballot.
constexpr int kSpBlocks = 148 * 8;
constexpr int kSpThreads = 256;
constexpr int kSpWarps = kSpBlocks * (kSpThreads / 32);

__device__ __forceinline__ uint4 sp_load(const uint32_t* f, int64_t i, int64_t end) {
  if (i + 3 < end) return *reinterpret_cast<const uint4*>(f + i);
  uint4 v = make_uint4(0u, 0u, 0u, 0u);
  if (i < end) v.x = f[i];
  if (i + 1 < end) v.y = f[i + 1];
  if (i + 2 < end) v.z = f[i + 2];
  return v;
}

__device__ __forceinline__ int sp_nonzero(const uint4& v) {
  return (v.x != 0u) + (v.y != 0u) + (v.z != 0u) + (v.w != 0u);
}

// Whether the 128-element stretch starting at t0 (a multiple of 128) has been
// touched since the last clear.
__device__ __forceinline__ bool sp_touched(const uint32_t* __restrict__ touch, int64_t t0) {
  return (touch[t0 >> 12] >> ((t0 >> 7) & 31)) & 1u;
}

__global__ void __launch_bounds__(kSpThreads) k_sp_count(const uint32_t* __restrict__ flim, int64_t n, int64_t chunk,
                                                         const uint32_t* __restrict__ touch,
                                                         int32_t* __restrict__ wcount) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t b0 = w * chunk, b1 = b0 + chunk < n ? b0 + chunk : n;
  int c = 0;
  for (int64_t t0 = b0; t0 < b1; t0 += 128)  // only the touched stretches (the same test in every lane)
    if (sp_touched(touch, t0)) c += sp_nonzero(sp_load(flim, t0 + 4 * lane, b1));
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if (lane == 0) wcount[w] = c;
}

// exclusive scan of the warp counts (one block); off[nb] = total
__global__ void k_sp_scan(const int32_t* __restrict__ bcount, int nb, int64_t* __restrict__ off) {
  int64_t carry = 0;
  for (int base = 0; base < nb; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int v = i < nb ? bcount[i] : 0;
    int total;
    const int ex = block_exclusive_scan(v, total);
    if (i < nb) off[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) off[nb] = carry;
}

// Emit and clear the nonzero bins; writes nothing (and clears nothing) when
// the frame holds more nonzero bins than the output's capacity.
__global__ void __launch_bounds__(kSpThreads) k_sp_write(uint32_t* __restrict__ flim, int64_t n, int64_t chunk,
                                                         const uint32_t* __restrict__ touch,
                                                         const int64_t* __restrict__ off, int nb,
                                                         int64_t* __restrict__ idx_out, uint32_t* __restrict__ cnt_out,
                                                         int64_t cap) {
  if (off[nb] > cap) return;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t b0 = w * chunk, b1 = b0 + chunk < n ? b0 + chunk : n;
  int64_t base = off[w];
  for (int64_t t0 = b0; t0 < b1; t0 += 128) {  // the same trip count in every lane of the warp
    if (!sp_touched(touch, t0)) continue;
    const int64_t i = t0 + 4 * lane;
    const uint4 v = sp_load(flim, i, b1);
    const int c = sp_nonzero(v);
    if (__ballot_sync(0xffffffffu, c != 0) == 0u) continue;
    int q = c;  // inclusive scan over the lanes
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, q, o);
      if (lane >= o) q += t;
    }
    const int total = __shfl_sync(0xffffffffu, q, 31);
    q -= c;
    const uint32_t e[4] = {v.x, v.y, v.z, v.w};
    for (int k = 0; k < 4; ++k) {
      if (e[k] != 0u) {
        idx_out[base + q] = i + k;
        cnt_out[base + q] = e[k];
        flim[i + k] = 0u;
        ++q;
      }
    }
    base += total;
  }
}

template <bool F64>
__global__ void k_set_state(const EdmDynParams* __restrict__ P, const int2* __restrict__ blk, const double* pos,
                            const int32_t* species, const uint8_t* alive, void* pos_post, short2* lo_post,
                            int32_t* cell_post, uint8_t* flags, int32_t* ids, int32_t* slot_of_id, int32_t* cnt) {
  const Tile t = tile_of(blk);
  const EdmDynParams& p = P[t.r];
  const int64_t s = t.s;
  if (s >= p.particle_offset + p.n_particles) return;
  const Geo g(p);
  const double x = pos[2 * s], y = pos[2 * s + 1];
  const int cx = cell_index(x, g.sx, g.nx), cy = cell_index(y, g.sy, g.ny);
  if constexpr (F64) {
    ((double2*)pos_post)[s] = make_double2(x, y);
  } else {
    float2 o;
    short2 l;
    split_offset(x - (double)cx * g.sx, g.sxf, o.x, l.x);
    split_offset(y - (double)cy * g.sy, g.syf, o.y, l.y);
    ((float2*)pos_post)[s] = o;
    lo_post[s] = l;
  }
  const int c = cx * g.ny + cy;
  cell_post[s] = c;
  flags[s] = fl_make(species[s], alive[s] != 0);
  ids[s] = (int32_t)s;
  slot_of_id[s] = (int32_t)s;
  atomicAdd(&cnt[g.cbase + (alive[s] ? c : g.grave)], 1);
}

template <bool F64>
__global__ void k_get_state(const EdmDynParams* __restrict__ P, const int2* __restrict__ blk, const void* pos_post,
                            const short2* lo_post, const int32_t* cell_post, const uint8_t* flags, const int32_t* slot_of_id,
                            const int32_t* bond, double* pos, int32_t* species, uint8_t* alive, int32_t* bond_local) {
  const Tile t = tile_of(blk);
  const EdmDynParams& p = P[t.r];
  const int64_t id = t.s;
  if (id >= p.particle_offset + p.n_particles) return;
  const Geo g(p);
  const int64_t s = slot_of_id[id];
  double x, y;
  abs_pos<F64>(pos_post, lo_post, cell_post, s, g, x, y);
  pos[2 * id] = x;
  pos[2 * id + 1] = y;
  const uint8_t f = flags[s];
  species[id] = fl_species(f);
  alive[id] = fl_alive(f) ? 1 : 0;
  const int b = bond[id];
  bond_local[id] = b >= 0 ? (int32_t)(b - p.particle_offset) : -1;
}

__global__ void k_narrow_i8(const int32_t* __restrict__ in, int8_t* __restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int8_t)in[i];
}

__global__ void k_bond_to_global(const EdmDynParams* __restrict__ P, const int2* __restrict__ blk, int32_t* bond) {
  const Tile t = tile_of(blk);
  const EdmDynParams& p = P[t.r];
  const int64_t id = t.s;
  if (id >= p.particle_offset + p.n_particles) return;
  const int b = bond[id];
  bond[id] = b >= 0 ? (int32_t)(b + p.particle_offset) : -1;
}

}  // namespace

extern "C" {

int edm_set_state(EdmEngine* E, const EdmHostState* st, void* stream) {
  if (!E || !st || st->n != E->N) return fail(EDM_EINVAL, "edm_set_state: size mismatch");
  E->cells_valid = false;
  cudaStream_t s = (cudaStream_t)stream;
  CUDA_TRY(cudaSetDevice(E->device));
  const int64_t N = E->N;
  double* dpos = E->st_pos;
  CUDA_TRY(cudaMemcpyAsync(dpos, st->positions, sizeof(double) * 2 * N, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(E->st_sp, st->species_id, sizeof(int32_t) * N, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(E->st_alive, st->is_alive, N, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(E->bond, st->bond_partner, sizeof(int32_t) * N, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(E->has_dye, st->has_dye, N, cudaMemcpyHostToDevice, s));
  // dye types arrive as int32 and are narrowed on the device (st_bond is free here)
  CUDA_TRY(cudaMemcpyAsync(E->st_bond, st->dye_type_id, sizeof(int32_t) * N, cudaMemcpyHostToDevice, s));
  if (N > 0) k_narrow_i8<<<148 * 8, 256, 0, s>>>(E->st_bond, E->dye, N);
  CUDA_TRY(cudaMemcpyAsync(E->ctmc, st->ctmc_state, N, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(E->bleached, st->is_bleached, N, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemsetAsync(E->cnt, 0, sizeof(int32_t) * (E->n_cells > 0 ? E->n_cells : 1), s));
  if (!E->contact_sides_counted && E->hdp[0].n_cat > 0) {
    // the contact sweep's sides from the first state's alive species counts
    int64_t count[EDM_MAX_SPECIES] = {};
    for (int64_t i = 0; i < N; ++i) {
      const int32_t sp = st->species_id[i];
      if (st->is_alive[i] && sp >= 0 && sp < EDM_MAX_SPECIES) ++count[sp];
    }
    E->set_contact_sides(count);
    E->drop_graphs();
    E->contact_sides_counted = true;
  }
  if (E->npblk > 0) {
    if (E->f64)
      k_set_state<true><<<E->npblk, kBlock, 0, s>>>(E->dp, E->pblk, dpos, E->st_sp, E->st_alive, E->pos_post, E->lo_post,
                                                    E->cell_post, E->flags[E->cur], E->ids[E->cur], E->slot_of_id,
                                                    E->cnt);
    else
      k_set_state<false><<<E->npblk, kBlock, 0, s>>>(E->dp, E->pblk, dpos, E->st_sp, E->st_alive, E->pos_post, E->lo_post,
                                                     E->cell_post, E->flags[E->cur], E->ids[E->cur], E->slot_of_id,
                                                     E->cnt);
    k_bond_to_global<<<E->npblk, kBlock, 0, s>>>(E->dp, E->pblk, E->bond);
  }
  // emitters: particles carrying a dye, in particle order per replica.  When
  // has_dye equals the last upload the emitter list, its tiles and the
  // captured graphs stay, and nothing here waits for the stream.
  if (E->has_phot && E->has_dye_host.size() == (size_t)N &&
      std::memcmp(E->has_dye_host.data(), st->has_dye, (size_t)N) == 0) {
    CUDA_TRY(cudaGetLastError());
    return EDM_OK;
  }
  if (E->has_phot) {
    E->has_dye_host.assign(st->has_dye, st->has_dye + N);
    std::vector<int32_t> eid;
    eid.reserve(N);
    int64_t off = 0;
    std::vector<int64_t> efirst, ecount;
    for (int r = 0; r < E->R; ++r) {
      const EdmDynParams& p = E->hdp[r];
      const int64_t before = (int64_t)eid.size();
      for (int64_t i = p.particle_offset; i < p.particle_offset + p.n_particles; ++i)
        if (st->has_dye[i]) eid.push_back((int32_t)i);
      E->hpp[r].emitter_offset = before;
      E->hpp[r].n_emitters = (int64_t)eid.size() - before;
      efirst.push_back(before);
      ecount.push_back((int64_t)eid.size() - before);
      off = (int64_t)eid.size();
    }
    (void)off;
    if (eid == E->emit_host) {  // same emitters: keep tiles and captured graphs
      CUDA_TRY(cudaStreamSynchronize(s));
      CUDA_TRY(cudaGetLastError());
      return EDM_OK;
    }
    E->emit_host = eid;
    E->n_emit = (int64_t)eid.size();
    if (!eid.empty())
      CUDA_TRY(cudaMemcpyAsync(E->emit_id, eid.data(), sizeof(int32_t) * eid.size(), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(E->pp, E->hpp.data(), sizeof(EdmPhotParams) * E->R, cudaMemcpyHostToDevice, s));
    std::vector<int2> et = tiles(efirst, ecount);
    if (E->eblk) cudaFree(E->eblk);
    for (auto& a : E->allocs)
      if (a == (void*)E->eblk) a = nullptr;
    E->eblk = nullptr;
    E->neblk = (int)et.size();
    if (!et.empty()) {
      CUDA_TRY(cudaMalloc(&E->eblk, sizeof(int2) * et.size()));
      E->allocs.push_back(E->eblk);
      CUDA_TRY(cudaMemcpyAsync(E->eblk, et.data(), sizeof(int2) * et.size(), cudaMemcpyHostToDevice, s));
    }
    CUDA_TRY(cudaStreamSynchronize(s));  // host vectors above go out of scope
    E->drop_graphs();
  } else {
    CUDA_TRY(cudaStreamSynchronize(s));
  }
  CUDA_TRY(cudaGetLastError());
  return EDM_OK;
}

int edm_get_state(EdmEngine* E, EdmHostState* st, void* stream) {
  if (!E || !st || st->n != E->N) return fail(EDM_EINVAL, "edm_get_state: size mismatch");
  cudaStream_t s = (cudaStream_t)stream;
  CUDA_TRY(cudaSetDevice(E->device));
  const int64_t N = E->N;
  if (E->npblk > 0) {
    if (E->f64)
      k_get_state<true><<<E->npblk, kBlock, 0, s>>>(E->dp, E->pblk, E->pos_post, E->lo_post, E->cell_post, E->flags[E->cur],
                                                    E->slot_of_id, E->bond, E->st_pos, E->st_sp, E->st_alive,
                                                    E->st_bond);
    else
      k_get_state<false><<<E->npblk, kBlock, 0, s>>>(E->dp, E->pblk, E->pos_post, E->lo_post, E->cell_post, E->flags[E->cur],
                                                     E->slot_of_id, E->bond, E->st_pos, E->st_sp, E->st_alive,
                                                     E->st_bond);
  }
  CUDA_TRY(cudaGetLastError());
  if (st->positions) CUDA_TRY(cudaMemcpyAsync(st->positions, E->st_pos, sizeof(double) * 2 * N, cudaMemcpyDeviceToHost, s));
  if (st->species_id) CUDA_TRY(cudaMemcpyAsync(st->species_id, E->st_sp, sizeof(int32_t) * N, cudaMemcpyDeviceToHost, s));
  if (st->is_alive) CUDA_TRY(cudaMemcpyAsync(st->is_alive, E->st_alive, N, cudaMemcpyDeviceToHost, s));
  if (st->bond_partner) CUDA_TRY(cudaMemcpyAsync(st->bond_partner, E->st_bond, sizeof(int32_t) * N, cudaMemcpyDeviceToHost, s));
  if (st->ctmc_state) CUDA_TRY(cudaMemcpyAsync(st->ctmc_state, E->ctmc, N, cudaMemcpyDeviceToHost, s));
  if (st->is_bleached) CUDA_TRY(cudaMemcpyAsync(st->is_bleached, E->bleached, N, cudaMemcpyDeviceToHost, s));
  if (st->has_dye) CUDA_TRY(cudaMemcpyAsync(st->has_dye, E->has_dye, N, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return EDM_OK;
}

int edm_stage_state_async(EdmEngine* E, const EdmHostState* st) {
  if (!E || !st || st->n != E->N) return fail(EDM_EINVAL, "edm_stage_state_async: size mismatch");
  if (E->has_phot && !(E->has_dye_host.size() == (size_t)E->N &&
                       std::memcmp(E->has_dye_host.data(), st->has_dye, (size_t)E->N) == 0))
    return fail(EDM_EINVAL, "edm_stage_state_async: the dye carriers differ from the last upload (edm_set_state)");
  if (E->staged) return fail(EDM_EINVAL, "edm_stage_state_async: a staged state waits for edm_install_state");
  CUDA_TRY(cudaSetDevice(E->device));
  int rc = E->xfer_setup();
  if (rc != EDM_OK) return rc;
  cudaStream_t u = E->up_stream;
  const int64_t N = E->N;
  const EdmEngine::Xfer& in = E->in;
  // waits only for the previous installation to leave the staging
  if (E->in_used) CUDA_TRY(cudaStreamWaitEvent(u, E->ev_in_free, 0));
  CUDA_TRY(cudaMemcpyAsync(in.pos, st->positions, sizeof(double) * 2 * N, cudaMemcpyHostToDevice, u));
  CUDA_TRY(cudaMemcpyAsync(in.sp, st->species_id, sizeof(int32_t) * N, cudaMemcpyHostToDevice, u));
  CUDA_TRY(cudaMemcpyAsync(in.alive, st->is_alive, N, cudaMemcpyHostToDevice, u));
  CUDA_TRY(cudaMemcpyAsync(in.bond, st->bond_partner, sizeof(int32_t) * N, cudaMemcpyHostToDevice, u));
  CUDA_TRY(cudaMemcpyAsync(in.has_dye, st->has_dye, N, cudaMemcpyHostToDevice, u));
  CUDA_TRY(cudaMemcpyAsync(in.dye, st->dye_type_id, sizeof(int32_t) * N, cudaMemcpyHostToDevice, u));
  CUDA_TRY(cudaMemcpyAsync(in.ctmc, st->ctmc_state, N, cudaMemcpyHostToDevice, u));
  CUDA_TRY(cudaMemcpyAsync(in.bleached, st->is_bleached, N, cudaMemcpyHostToDevice, u));
  CUDA_TRY(cudaEventRecord(E->ev_staged, u));
  E->staged = true;
  return EDM_OK;
}

int edm_install_state(EdmEngine* E, void* stream) {
  if (!E) return fail(EDM_EINVAL, "edm_install_state: null engine");
  if (!E->staged) return fail(EDM_EINVAL, "edm_install_state: no staged state");
  CUDA_TRY(cudaSetDevice(E->device));
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t N = E->N;
  const EdmEngine::Xfer& in = E->in;
  E->cells_valid = false;
  // in order on `stream`: as edm_set_state, from the staging
  CUDA_TRY(cudaStreamWaitEvent(s, E->ev_staged, 0));
  CUDA_TRY(cudaMemcpyAsync(E->bond, in.bond, sizeof(int32_t) * N, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(E->has_dye, in.has_dye, N, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(E->ctmc, in.ctmc, N, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(E->bleached, in.bleached, N, cudaMemcpyDeviceToDevice, s));
  if (N > 0) k_narrow_i8<<<148 * 8, 256, 0, s>>>(in.dye, E->dye, N);
  CUDA_TRY(cudaMemsetAsync(E->cnt, 0, sizeof(int32_t) * (E->n_cells > 0 ? E->n_cells : 1), s));
  if (E->npblk > 0) {
    if (E->f64)
      k_set_state<true><<<E->npblk, kBlock, 0, s>>>(E->dp, E->pblk, in.pos, in.sp, in.alive, E->pos_post, E->lo_post,
                                                    E->cell_post, E->flags[E->cur], E->ids[E->cur], E->slot_of_id,
                                                    E->cnt);
    else
      k_set_state<false><<<E->npblk, kBlock, 0, s>>>(E->dp, E->pblk, in.pos, in.sp, in.alive, E->pos_post, E->lo_post,
                                                     E->cell_post, E->flags[E->cur], E->ids[E->cur], E->slot_of_id,
                                                     E->cnt);
    k_bond_to_global<<<E->npblk, kBlock, 0, s>>>(E->dp, E->pblk, E->bond);
  }
  CUDA_TRY(cudaEventRecord(E->ev_in_free, s));
  E->in_used = true;
  E->staged = false;
  CUDA_TRY(cudaGetLastError());
  return EDM_OK;
}

int edm_set_state_async(EdmEngine* E, const EdmHostState* st, void* stream) {
  if (!E || !st || st->n != E->N) return fail(EDM_EINVAL, "edm_set_state_async: size mismatch");
  // new dye carriers rebuild the emitter list on the host: the synchronous path
  if (E->has_phot && !(E->has_dye_host.size() == (size_t)E->N &&
                       std::memcmp(E->has_dye_host.data(), st->has_dye, (size_t)E->N) == 0))
    return edm_set_state(E, st, stream);
  if (!E->contact_sides_counted && E->hdp[0].n_cat > 0) return edm_set_state(E, st, stream);
  const int rc = edm_stage_state_async(E, st);
  return rc != EDM_OK ? rc : edm_install_state(E, stream);
}

int edm_get_state_async(EdmEngine* E, EdmHostState* st, void* stream) {
  if (!E || !st || st->n != E->N) return fail(EDM_EINVAL, "edm_get_state_async: size mismatch");
  CUDA_TRY(cudaSetDevice(E->device));
  int rc = E->xfer_setup();
  if (rc != EDM_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream, d = E->down_stream;
  const int64_t N = E->N;
  const EdmEngine::Xfer& out = E->out;
  // the gathering, in order on `stream`, once the previous download has left the staging
  if (E->out_used) CUDA_TRY(cudaStreamWaitEvent(s, E->ev_out_free, 0));
  if (E->npblk > 0) {
    if (E->f64)
      k_get_state<true><<<E->npblk, kBlock, 0, s>>>(E->dp, E->pblk, E->pos_post, E->lo_post, E->cell_post, E->flags[E->cur],
                                                    E->slot_of_id, E->bond, out.pos, out.sp, out.alive, out.bond);
    else
      k_get_state<false><<<E->npblk, kBlock, 0, s>>>(E->dp, E->pblk, E->pos_post, E->lo_post, E->cell_post, E->flags[E->cur],
                                                     E->slot_of_id, E->bond, out.pos, out.sp, out.alive, out.bond);
  }
  CUDA_TRY(cudaMemcpyAsync(out.ctmc, E->ctmc, N, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(out.bleached, E->bleached, N, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(out.has_dye, E->has_dye, N, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaEventRecord(E->ev_out_ready, s));
  // the download, on the engine's stream, while `stream` goes on
  CUDA_TRY(cudaStreamWaitEvent(d, E->ev_out_ready, 0));
  if (st->positions) CUDA_TRY(cudaMemcpyAsync(st->positions, out.pos, sizeof(double) * 2 * N, cudaMemcpyDeviceToHost, d));
  if (st->species_id) CUDA_TRY(cudaMemcpyAsync(st->species_id, out.sp, sizeof(int32_t) * N, cudaMemcpyDeviceToHost, d));
  if (st->is_alive) CUDA_TRY(cudaMemcpyAsync(st->is_alive, out.alive, N, cudaMemcpyDeviceToHost, d));
  if (st->bond_partner) CUDA_TRY(cudaMemcpyAsync(st->bond_partner, out.bond, sizeof(int32_t) * N, cudaMemcpyDeviceToHost, d));
  if (st->ctmc_state) CUDA_TRY(cudaMemcpyAsync(st->ctmc_state, out.ctmc, N, cudaMemcpyDeviceToHost, d));
  if (st->is_bleached) CUDA_TRY(cudaMemcpyAsync(st->is_bleached, out.bleached, N, cudaMemcpyDeviceToHost, d));
  if (st->has_dye) CUDA_TRY(cudaMemcpyAsync(st->has_dye, out.has_dye, N, cudaMemcpyDeviceToHost, d));
  CUDA_TRY(cudaEventRecord(E->ev_out_free, d));
  E->out_used = true;
  CUDA_TRY(cudaGetLastError());
  return EDM_OK;
}

int edm_state_transfers_wait(EdmEngine* E) {
  if (!E) return fail(EDM_EINVAL, "edm_state_transfers_wait: null engine");
  CUDA_TRY(cudaSetDevice(E->device));
  if (E->up_stream) CUDA_TRY(cudaStreamSynchronize(E->up_stream));
  if (E->down_stream) CUDA_TRY(cudaStreamSynchronize(E->down_stream));
  return EDM_OK;
}

int edm_set_step(EdmEngine* E, int64_t step_index) {
  if (!E) return fail(EDM_EINVAL, "null engine");
  CUDA_TRY(cudaSetDevice(E->device));
  CUDA_TRY(cudaMemcpy(E->d_step, &step_index, sizeof(int64_t), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(E->d_pstep, &step_index, sizeof(int64_t), cudaMemcpyHostToDevice));
  return EDM_OK;
}

int64_t edm_get_step(EdmEngine* E) {
  if (!E) return -1;
  int64_t v = -1;
  cudaSetDevice(E->device);
  if (cudaMemcpy(&v, E->d_step, sizeof(int64_t), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  return v;
}

int edm_dynamics_step(EdmEngine* E, int32_t n_steps, void* stream) {
  if (!E || n_steps < 0) return fail(EDM_EINVAL, "edm_dynamics_step: bad argument");
  CUDA_TRY(cudaSetDevice(E->device));
  cudaStream_t s = (cudaStream_t)stream;
  for (int i = 0; i < n_steps; ++i) E->enqueue_dynamics(s);
  CUDA_TRY(cudaGetLastError());
  return EDM_OK;
}

int edm_photon_step(EdmEngine* E, void* stream) {
  if (!E || !E->has_phot) return fail(EDM_EINVAL, "edm_photon_step: engine has no photophysics");
  CUDA_TRY(cudaSetDevice(E->device));
  E->enqueue_photons((cudaStream_t)stream);
  CUDA_TRY(cudaGetLastError());
  return EDM_OK;
}

int edm_get_photon_counts(EdmEngine* E, int64_t* counts, void* stream) {
  if (!E || !E->has_phot || !counts) return fail(EDM_EINVAL, "edm_get_photon_counts: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  CUDA_TRY(cudaMemcpyAsync(counts, E->ph_count, sizeof(int64_t) * E->R, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return EDM_OK;
}

int edm_get_photons(EdmEngine* E, int32_t replica, int32_t* particle_idx, double* arrival_time, int8_t* channel,
                    uint8_t* is_fret, int64_t capacity, void* stream) {
  if (!E || !E->has_phot || replica < 0 || replica >= E->R) return fail(EDM_EINVAL, "edm_get_photons: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  int64_t n = 0;
  CUDA_TRY(cudaMemcpyAsync(&n, E->ph_count + replica, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (n > capacity) return fail(EDM_EINVAL, "edm_get_photons: capacity too small");
  const int64_t o = E->hpp[replica].photon_offset;
  if (n > 0) {
    if (particle_idx) CUDA_TRY(cudaMemcpyAsync(particle_idx, E->ph_pid + o, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
    if (arrival_time) CUDA_TRY(cudaMemcpyAsync(arrival_time, E->ph_t + o, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    if (channel) CUDA_TRY(cudaMemcpyAsync(channel, E->ph_ch + o, n, cudaMemcpyDeviceToHost, s));
    if (is_fret) CUDA_TRY(cudaMemcpyAsync(is_fret, E->ph_fret + o, n, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
  }
  return (int)n;
}

int edm_scope_process(EdmEngine* E, void* stream) {
  if (!E || !E->has_scope) return fail(EDM_EINVAL, "edm_scope_process: engine has no microscope");
  CUDA_TRY(cudaSetDevice(E->device));
  E->enqueue_photon_positions((cudaStream_t)stream);  // the batch may come from the host
  E->enqueue_scope((cudaStream_t)stream);
  CUDA_TRY(cudaGetLastError());
  return EDM_OK;
}

int edm_set_photons(EdmEngine* E, int32_t replica, const int32_t* particle_idx, const double* arrival_time,
                    const int8_t* channel, const uint8_t* is_fret, int64_t n, int64_t batch_key, void* stream) {
  if (!E || !E->has_phot || replica < 0 || replica >= E->R || n < 0) return fail(EDM_EINVAL, "edm_set_photons: bad argument");
  if (n > E->hpp[replica].max_photons) return fail(EDM_EINVAL, "edm_set_photons: batch larger than the photon buffer");
  CUDA_TRY(cudaSetDevice(E->device));
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t o = E->hpp[replica].photon_offset;
  if (n > 0) {
    CUDA_TRY(cudaMemcpyAsync(E->ph_pid + o, particle_idx, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(E->ph_t + o, arrival_time, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(E->ph_ch + o, channel, n, cudaMemcpyHostToDevice, s));
    if (is_fret) CUDA_TRY(cudaMemcpyAsync(E->ph_fret + o, is_fret, n, cudaMemcpyHostToDevice, s));
  }
  std::vector<int64_t> counts(E->R, 0);
  counts[replica] = n;
  CUDA_TRY(cudaMemcpyAsync(E->ph_count, counts.data(), sizeof(int64_t) * E->R, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(E->d_batch_key, &batch_key, sizeof(int64_t), cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return EDM_OK;
}

int edm_pipeline_steps(EdmEngine* E, int32_t n_steps, int32_t with_photons, int32_t graph_chunk, void* stream) {
  if (!E || n_steps < 0) return fail(EDM_EINVAL, "edm_pipeline_steps: bad argument");
  if (with_photons && !E->has_scope) return fail(EDM_EINVAL, "edm_pipeline_steps: no photophysics/microscope");
  CUDA_TRY(cudaSetDevice(E->device));
  cudaStream_t s = (cudaStream_t)stream;
  auto body = [&](cudaStream_t st) {
    E->enqueue_dynamics(st);  // beside the previous step's photon and detection passes
    if (with_photons) E->enqueue_photons_beside(st);
    if (E->rec_cap > 0) {
      E->join_beside(st);  // the census reads the photon state and the detection counters
      E->enqueue_census(st, E->rec_ring, E->rec_cap, with_photons != 0);
    }
  };
  int done = 0;
  if (graph_chunk > 0 && s != nullptr) {
    while (n_steps - done >= graph_chunk) {
      const auto key = std::make_tuple(graph_chunk, with_photons ? 1 : 0, E->cur, E->rec_cap > 0 ? 1 : 0);
      auto it = E->graphs.find(key);
      if (it == E->graphs.end()) {
        const int cur0 = E->cur;
        cudaGraph_t g;
        CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < graph_chunk; ++i) body(s);
        E->join_beside(s);  // the capture ends on the origin stream
        CUDA_TRY(cudaStreamEndCapture(s, &g));
        cudaGraphExec_t ge;
        CUDA_TRY(cudaGraphInstantiate(&ge, g, 0));
        cudaGraphDestroy(g);
        E->cur = cur0;  // capture advanced the parity; the launch below replays it
        it = E->graphs.emplace(key, ge).first;
      }
      CUDA_TRY(cudaGraphLaunch(it->second, s));
      if (graph_chunk & 1) E->cur ^= 1;
      done += graph_chunk;
    }
  }
  for (; done < n_steps; ++done) body(s);
  E->join_beside(s);  // whatever the caller queues next sees the photon and detection passes done
  CUDA_TRY(cudaGetLastError());
  return EDM_OK;
}

int edm_profile_steps(EdmEngine* E, int32_t n_steps, int32_t with_photons, float* ms_out, void* stream) {
  if (!E || n_steps <= 0 || !ms_out) return fail(EDM_EINVAL, "edm_profile_steps: bad argument");
  if (with_photons && !E->has_scope) return fail(EDM_EINVAL, "edm_profile_steps: no photophysics/microscope");
  if (!stream) return fail(EDM_EINVAL, "edm_profile_steps: needs a non-default stream (the steps are captured)");
  CUDA_TRY(cudaSetDevice(E->device));
  cudaStream_t s = (cudaStream_t)stream;
  // Two steps (both parities of the double-buffered slot arrays) are captured
  // into one graph with event-record nodes between the kernel groups, so the
  // groups are timed as they run inside the pipeline's graphs.
  cudaEvent_t ev[2][7];
  for (int h = 0; h < 2; ++h)
    for (int k = 0; k < 7; ++k) CUDA_TRY(cudaEventCreate(&ev[h][k]));
  auto destroy = [&]() {
    for (int h = 0; h < 2; ++h)
      for (int k = 0; k < 7; ++k) cudaEventDestroy(ev[h][k]);
  };
  const int cur0 = E->cur;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  E->prof_capture = true;
  cudaError_t ce = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (ce == cudaSuccess) {
    for (int h = 0; h < 2; ++h) {
      E->prof = ev[h];
      E->enqueue_dynamics(s);
      if (with_photons) {
        E->enqueue_photons(s);
        E->mark(5, s);
        E->enqueue_scope(s);
        E->mark(6, s);
      }
    }
    ce = cudaStreamEndCapture(s, &g);
  }
  E->prof = nullptr;
  E->prof_capture = false;
  E->cur = cur0;  // the capture advanced the parity twice: unchanged
  if (ce == cudaSuccess) ce = cudaGraphInstantiate(&ge, g, 0);
  if (g) cudaGraphDestroy(g);
  if (ce != cudaSuccess) {
    destroy();
    return fail(EDM_ECUDA, cudaGetErrorString(ce));
  }
  double acc[EDM_NPROF] = {0, 0, 0, 0, 0, 0, 0};
  const int reps = (n_steps + 1) / 2;
  for (int i = 0; i < reps; ++i) {
    ce = cudaGraphLaunch(ge, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) break;
    for (int h = 0; h < 2; ++h) {
      float t;
      for (int k = 0; k < 4; ++k) {
        cudaEventElapsedTime(&t, ev[h][k], ev[h][k + 1]);
        acc[k] += t;
      }
      if (with_photons) {
        cudaEventElapsedTime(&t, ev[h][4], ev[h][5]);
        acc[4] += t;
        cudaEventElapsedTime(&t, ev[h][5], ev[h][6]);
        acc[5] += t;
      }
      cudaEventElapsedTime(&t, ev[h][0], with_photons ? ev[h][6] : ev[h][4]);
      acc[6] += t;
    }
  }
  cudaGraphExecDestroy(ge);
  destroy();
  if (ce != cudaSuccess) return fail(EDM_ECUDA, cudaGetErrorString(ce));
  for (int k = 0; k < EDM_NPROF; ++k) ms_out[k] = (float)(acc[k] / (2.0 * reps));
  return EDM_OK;
}

int edm_profile_passes(EdmEngine* E, int32_t n_steps, float* ms_out, int32_t* kinds_out, int32_t cap, void* stream) {
  if (!E || n_steps <= 0 || !ms_out || !kinds_out) return fail(EDM_EINVAL, "edm_profile_passes: bad argument");
  const int n = (int)E->passes.size();
  if (cap < n) return fail(EDM_EINVAL, "edm_profile_passes: cap below the number of passes");
  CUDA_TRY(cudaSetDevice(E->device));
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<cudaEvent_t> ev(n + 1);
  for (auto& e : ev) CUDA_TRY(cudaEventCreate(&e));
  std::vector<double> acc(n, 0.0);
  E->pass_prof = ev.data();
  int rc = EDM_OK;
  for (int i = 0; i < n_steps && rc == EDM_OK; ++i) {
    E->enqueue_dynamics(s);
    const cudaError_t e = cudaEventSynchronize(ev[n]);
    if (e != cudaSuccess) {
      rc = fail(EDM_ECUDA, cudaGetErrorString(e));
      break;
    }
    for (int k = 0; k < n; ++k) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
      acc[k] += t;
    }
  }
  E->pass_prof = nullptr;
  for (auto& e : ev) cudaEventDestroy(e);
  if (rc != EDM_OK) return rc;
  for (int k = 0; k < n; ++k) {
    ms_out[k] = (float)(acc[k] / n_steps);
    kinds_out[k] = 100 * (int)E->passes[k].kind + E->passes[k].index;
  }
  return n;
}

int edm_record_enable(EdmEngine* E, int32_t capacity_steps) {
  if (!E || capacity_steps < 0) return fail(EDM_EINVAL, "edm_record_enable: bad argument");
  CUDA_TRY(cudaSetDevice(E->device));
  if (capacity_steps == E->rec_cap) return EDM_OK;
  CUDA_TRY(cudaDeviceSynchronize());  // no captured chunk or kernel may still use the old ring
  E->drop_graphs();
  if (E->rec_ring) {
    for (auto& a : E->allocs)
      if (a == (void*)E->rec_ring) a = nullptr;
    cudaFree(E->rec_ring);
    E->rec_ring = nullptr;
  }
  E->rec_cap = 0;
  if (capacity_steps > 0) {
    int rc = E->alloc(&E->rec_ring, (size_t)capacity_steps * E->R * EDM_CENSUS_FIELDS);
    if (rc != EDM_OK) return rc;
    CUDA_TRY(cudaMemset(E->rec_ring, 0, sizeof(int64_t) * (size_t)capacity_steps * E->R * EDM_CENSUS_FIELDS));
    E->rec_cap = capacity_steps;
  }
  return EDM_OK;
}

int edm_record_read(EdmEngine* E, int64_t first_step, int32_t n_steps, int64_t* host_out, void* stream) {
  if (!E || first_step < 0 || n_steps < 0 || (n_steps > 0 && !host_out))
    return fail(EDM_EINVAL, "edm_record_read: bad argument");
  if (n_steps > E->rec_cap) return fail(EDM_EINVAL, "edm_record_read: more steps than the recorder holds");
  CUDA_TRY(cudaSetDevice(E->device));
  cudaStream_t s = (cudaStream_t)stream;
  const size_t row = (size_t)E->R * EDM_CENSUS_FIELDS;
  int done = 0;
  while (done < n_steps) {  // at most two runs of ring slots
    const int64_t slot = (first_step + done) % E->rec_cap;
    const int run = (int)std::min<int64_t>(n_steps - done, E->rec_cap - slot);
    CUDA_TRY(cudaMemcpyAsync(host_out + done * row, E->rec_ring + slot * row, sizeof(int64_t) * row * run,
                             cudaMemcpyDeviceToHost, s));
    done += run;
  }
  return EDM_OK;
}

int edm_ground_truth(EdmEngine* E, double* fret_E, double* tau_DA, int64_t* census, void* stream) {
  if (!E) return fail(EDM_EINVAL, "edm_ground_truth: null engine");
  CUDA_TRY(cudaSetDevice(E->device));
  cudaStream_t s = (cudaStream_t)stream;
  int rc;
  if (!E->gt_census) {
    if ((rc = E->alloc(&E->gt_census, (size_t)E->R * EDM_CENSUS_FIELDS)) != EDM_OK) return rc;
    if ((rc = E->alloc(&E->gt_E, (size_t)std::max<int64_t>(E->N, 1))) != EDM_OK) return rc;
    if ((rc = E->alloc(&E->gt_tau, (size_t)std::max<int64_t>(E->N, 1))) != EDM_OK) return rc;
  }
  E->enqueue_census(s, E->gt_census, 0, false);
  CUDA_TRY(cudaMemsetAsync(E->gt_E, 0, sizeof(double) * E->N, s));
  CUDA_TRY(cudaMemsetAsync(E->gt_tau, 0, sizeof(double) * E->N, s));
  if (E->has_phot && E->neblk > 0) {
    const DevState st = E->dev_state();
    const PhotState ph = E->phot_state();
    const int cv = E->cells_valid ? 1 : 0;
    if (E->f64) k_ground_truth<true><<<E->neblk, kBlock, 0, s>>>(E->dp, E->pp, E->eblk, st, ph, cv, E->gt_E, E->gt_tau);
    else k_ground_truth<false><<<E->neblk, kBlock, 0, s>>>(E->dp, E->pp, E->eblk, st, ph, cv, E->gt_E, E->gt_tau);
  }
  CUDA_TRY(cudaGetLastError());
  if (fret_E) CUDA_TRY(cudaMemcpyAsync(fret_E, E->gt_E, sizeof(double) * E->N, cudaMemcpyDeviceToHost, s));
  if (tau_DA) CUDA_TRY(cudaMemcpyAsync(tau_DA, E->gt_tau, sizeof(double) * E->N, cudaMemcpyDeviceToHost, s));
  if (census)
    CUDA_TRY(cudaMemcpyAsync(census, E->gt_census, sizeof(int64_t) * E->R * EDM_CENSUS_FIELDS,
                             cudaMemcpyDeviceToHost, s));
  return EDM_OK;
}

int edm_autotune(EdmEngine* E, int32_t steps_per_shape, int32_t retune, void* stream) {
  if (!E || steps_per_shape <= 0) return fail(EDM_EINVAL, "edm_autotune: bad argument");
  CUDA_TRY(cudaSetDevice(E->device));
  cudaStream_t s = (cudaStream_t)stream;
  for (int k = 0; k < 2; ++k)
    if (!E->tune_ev[k]) CUDA_TRY(cudaEventCreate(&E->tune_ev[k]));
  bool has_contacts = false;
  for (const Pass& ps : E->passes) has_contacts |= ps.kind == P_CONTACTS;
  cudaError_t ce = cudaSuccess;
  for (int k = 0; k < TK_COUNT && ce == cudaSuccess; ++k) {
    if (E->npblk == 0 || (k == TK_CONTACTS && !has_contacts)) continue;
    const auto key = E->tune_key(k);
    if (!retune) {
      std::lock_guard<std::mutex> lock(g_tune_mu);
      auto it = g_tuned.find(key);
      if (it != g_tuned.end()) {
        E->shape[k] = it->second;
        continue;
      }
    }
    // Each candidate runs real steps (every shape computes the same state),
    // one untimed, then steps_per_shape timed around the kernel alone.
    double best = 1e30;
    int best_v = 0;
    for (int v = 0; v < kNumShapes[k] && ce == cudaSuccess; ++v) {
      E->shape[k] = v;
      E->tune_kernel = -1;
      E->enqueue_dynamics(s);
      double acc = 0.0;
      for (int i = 0; i < steps_per_shape && ce == cudaSuccess; ++i) {
        E->tune_kernel = k;
        E->enqueue_dynamics(s);
        E->tune_kernel = -1;
        ce = cudaEventSynchronize(E->tune_ev[1]);
        float t = 0.f;
        if (ce == cudaSuccess) ce = cudaEventElapsedTime(&t, E->tune_ev[0], E->tune_ev[1]);
        acc += t;
      }
      const double ms = acc / steps_per_shape;
      if (v == 0) E->default_ms[k] = (float)ms;
      if (ms < best) {
        best = ms;
        best_v = v;
      }
    }
    E->shape[k] = best_v;
    E->tuned_ms[k] = (float)best;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tuned[key] = best_v;
  }
  E->tune_kernel = -1;
  E->drop_graphs();  // captured chunks hold the previous shapes
  if (ce != cudaSuccess) return fail(EDM_ECUDA, std::string("edm_autotune: ") + cudaGetErrorString(ce));
  CUDA_TRY(cudaGetLastError());
  return EDM_OK;
}

int edm_set_launch_shapes(EdmEngine* E, const int32_t* candidate) {
  if (!E || !candidate) return fail(EDM_EINVAL, "edm_set_launch_shapes: bad argument");
  for (int k = 0; k < TK_COUNT; ++k)
    if (candidate[k] < -1 || candidate[k] >= kNumShapes[k])
      return fail(EDM_EINVAL, "edm_set_launch_shapes: no such candidate");
  for (int k = 0; k < TK_COUNT; ++k)
    if (candidate[k] >= 0) E->shape[k] = candidate[k];
  E->drop_graphs();
  return EDM_OK;
}

int edm_contact_sides(EdmEngine* E, int32_t force_mask) {
  if (!E) return fail(EDM_EINVAL, "edm_contact_sides: null engine");
  if (force_mask >= 0 && E->hdp[0].n_cat > 0) {
    E->set_contact_sides(nullptr, force_mask);
    E->contact_sides_counted = true;
    E->drop_graphs();
  }
  return (int)(E->cat_lists.from_enzyme & 0x7FFFFFFFu);
}

int edm_launch_shapes(EdmEngine* E, int32_t* shapes, float* ms) {
  if (!E) return fail(EDM_EINVAL, "edm_launch_shapes: null engine");
  for (int k = 0; k < TK_COUNT; ++k) {
    const LaunchShape sh = kShapes[k][E->shape[k]];
    if (shapes) {
      shapes[4 * k] = sh.block;
      shapes[4 * k + 1] = sh.min_blocks;
      shapes[4 * k + 2] = kNumShapes[k];
      shapes[4 * k + 3] = E->shape[k];
    }
    if (ms) {
      ms[2 * k] = E->default_ms[k];
      ms[2 * k + 1] = E->tuned_ms[k];
    }
  }
  return TK_COUNT;
}

int edm_launches_per_step(EdmEngine* E, int32_t with_photons) {
  if (!E) return fail(EDM_EINVAL, "null engine");
  return E->launches_per_step(with_photons != 0);
}

int edm_scope_finalize(EdmEngine* E, int64_t frame_index, void* stream) {
  if (!E || !E->has_scope) return fail(EDM_EINVAL, "edm_scope_finalize: engine has no microscope");
  CUDA_TRY(cudaSetDevice(E->device));
  cudaStream_t s = (cudaStream_t)stream;
  if (E->npxblk > 0) {
    k_dark<<<E->npxblk, kBlock, 0, s>>>(E->dp, E->sp, E->pxblk, E->flim, E->touch, frame_index, E->counters);
    k_afterpulse<<<E->npxblk, kBlock, 0, s>>>(E->dp, E->sp, E->pxblk, E->flim, E->touch, frame_index,
                                              E->counters);
  }
  CUDA_TRY(cudaGetLastError());
  return EDM_OK;
}

int edm_get_flim(EdmEngine* E, int32_t replica, uint32_t* host_out, int64_t n_elems, void* stream) {
  if (!E || !E->has_scope || replica < 0 || replica >= E->R) return fail(EDM_EINVAL, "edm_get_flim: bad argument");
  const EdmScopeParams& p = E->hsp[replica];
  const int64_t n = (int64_t)p.n_channels * p.nx * p.ny * p.n_bins;
  if (n_elems < n) return fail(EDM_EINVAL, "edm_get_flim: buffer too small");
  cudaStream_t s = (cudaStream_t)stream;
  CUDA_TRY(cudaMemcpyAsync(host_out, E->flim + p.flim_offset, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return EDM_OK;
}

int edm_reset_flim(EdmEngine* E, void* stream) {
  if (!E || !E->has_scope) return fail(EDM_EINVAL, "edm_reset_flim: engine has no microscope");
  CUDA_TRY(cudaMemsetAsync(E->flim, 0, sizeof(uint32_t) * E->n_flim, (cudaStream_t)stream));
  CUDA_TRY(cudaMemsetAsync(E->touch, 0, sizeof(uint32_t) * E->n_touch, (cudaStream_t)stream));
  return EDM_OK;
}

int64_t edm_flim_elems(EdmEngine* E) { return (E && E->has_scope) ? E->n_flim : 0; }

int edm_flim_stack_ptr(EdmEngine* E, int32_t replica, void** ptr, int64_t* n_px, int32_t* n_bins) {
  if (!E || !E->has_scope || !ptr || replica < 0 || replica >= E->R)
    return fail(EDM_EINVAL, "edm_flim_stack_ptr: bad argument");
  const EdmScopeParams& p = E->hsp[replica];
  *ptr = E->flim + p.flim_offset;
  if (n_px) *n_px = (int64_t)p.n_channels * p.nx * p.ny;
  if (n_bins) *n_bins = p.n_bins;
  return EDM_OK;
}

int edm_frame_out_begin(EdmEngine* E, uint32_t* host_out, int64_t n_elems, void* stream) {
  if (!E || !E->has_scope || !host_out) return fail(EDM_EINVAL, "edm_frame_out_begin: bad argument");
  if (n_elems < E->n_flim) return fail(EDM_EINVAL, "edm_frame_out_begin: host buffer too small");
  CUDA_TRY(cudaSetDevice(E->device));
  cudaStream_t s = (cudaStream_t)stream;
  if (!E->flim_snap) {
    int rc;
    if ((rc = E->alloc(&E->flim_snap, (size_t)E->n_flim)) != EDM_OK) return rc;
    CUDA_TRY(cudaStreamCreateWithFlags(&E->copy_stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&E->ev_snap, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&E->ev_read, cudaEventDisableTiming));
  }
  const size_t bytes = sizeof(uint32_t) * (size_t)E->n_flim;
  if (E->read_pending) CUDA_TRY(cudaStreamWaitEvent(s, E->ev_read, 0));  // snapshot free again
  CUDA_TRY(cudaMemcpyAsync(E->flim_snap, E->flim, bytes, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemsetAsync(E->flim, 0, bytes, s));
  CUDA_TRY(cudaMemsetAsync(E->touch, 0, sizeof(uint32_t) * E->n_touch, s));
  CUDA_TRY(cudaEventRecord(E->ev_snap, s));
  CUDA_TRY(cudaStreamWaitEvent(E->copy_stream, E->ev_snap, 0));
  CUDA_TRY(cudaMemcpyAsync(host_out, E->flim_snap, bytes, cudaMemcpyDeviceToHost, E->copy_stream));
  CUDA_TRY(cudaEventRecord(E->ev_read, E->copy_stream));
  E->read_pending = true;
  return EDM_OK;
}

int64_t edm_frame_out_sparse(EdmEngine* E, int64_t* idx_host, uint32_t* count_host, int64_t cap, void* stream) {
  if (!E || !E->has_scope || cap < 0 || (cap > 0 && (!idx_host || !count_host)))
    return fail(EDM_EINVAL, "edm_frame_out_sparse: bad argument");
  CUDA_TRY(cudaSetDevice(E->device));
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t dcap = cap < E->n_flim ? cap : E->n_flim;
  int rc;
  if (!E->sp_bcount) {
    if ((rc = E->alloc(&E->sp_bcount, kSpWarps)) != EDM_OK) return rc;
    if ((rc = E->alloc(&E->sp_off, kSpWarps + 1)) != EDM_OK) return rc;
  }
  if (dcap > E->sp_cap) {  // (re)size the device output
    for (auto& a : E->allocs)
      if (a == (void*)E->sp_idx || a == (void*)E->sp_cnt) a = nullptr;
    CUDA_TRY(cudaStreamSynchronize(s));
    cudaFree(E->sp_idx);
    cudaFree(E->sp_cnt);
    E->sp_idx = nullptr;
    E->sp_cnt = nullptr;
    E->sp_cap = 0;
    if ((rc = E->alloc(&E->sp_idx, (size_t)std::max<int64_t>(dcap, 1))) != EDM_OK) return rc;
    if ((rc = E->alloc(&E->sp_cnt, (size_t)std::max<int64_t>(dcap, 1))) != EDM_OK) return rc;
    E->sp_cap = dcap;
  }
  const int64_t n = E->n_flim;
  const int64_t per = (n + kSpWarps - 1) / kSpWarps;
  const int64_t quantum = 128;  // 4 elements per lane: uint4 loads stay 16-byte aligned
  const int64_t chunk = std::max<int64_t>(quantum, (per + quantum - 1) / quantum * quantum);
  k_sp_count<<<kSpBlocks, kSpThreads, 0, s>>>(E->flim, n, chunk, E->touch, E->sp_bcount);
  k_sp_scan<<<1, 1024, 0, s>>>(E->sp_bcount, kSpWarps, E->sp_off);
  k_sp_write<<<kSpBlocks, kSpThreads, 0, s>>>(E->flim, n, chunk, E->touch, E->sp_off, kSpWarps, E->sp_idx, E->sp_cnt,
                                              dcap);
  CUDA_TRY(cudaGetLastError());
  int64_t total = 0;
  CUDA_TRY(cudaMemcpyAsync(&total, E->sp_off + kSpWarps, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (total > dcap)
    return fail(EDM_EINVAL, "edm_frame_out_sparse: " + std::to_string((long long)total) +
                                " nonzero bins exceed the capacity; the stacks are left in place");
  CUDA_TRY(cudaMemsetAsync(E->touch, 0, sizeof(uint32_t) * E->n_touch, s));  // every touched bin is cleared
  if (total > 0) {
    CUDA_TRY(cudaMemcpyAsync(idx_host, E->sp_idx, sizeof(int64_t) * total, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(count_host, E->sp_cnt, sizeof(uint32_t) * total, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
  }
  return total;
}

int edm_frame_out_wait(EdmEngine* E) {
  if (!E) return fail(EDM_EINVAL, "edm_frame_out_wait: null engine");
  if (!E->read_pending) return EDM_OK;
  CUDA_TRY(cudaSetDevice(E->device));
  CUDA_TRY(cudaEventSynchronize(E->ev_read));
  return EDM_OK;
}

int edm_get_counters(EdmEngine* E, int64_t* out, void* stream) {
  if (!E || !out) return fail(EDM_EINVAL, "edm_get_counters: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  CUDA_TRY(cudaMemcpyAsync(out, E->counters, sizeof(int64_t) * E->R * EDM_NCOUNTERS, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return EDM_OK;
}

int edm_get_status(EdmEngine* E, uint32_t* status, void* stream) {
  if (!E || !status) return fail(EDM_EINVAL, "edm_get_status: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  CUDA_TRY(cudaMemcpyAsync(status, E->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return EDM_OK;
}

int edm_get_cells(EdmEngine* E, int32_t replica, int32_t* cell_start, int32_t* members, int64_t cap_cells,
                  int64_t cap_members, void* stream) {
  if (!E || replica < 0 || replica >= E->R) return fail(EDM_EINVAL, "edm_get_cells: bad argument");
  const EdmDynParams& p = E->hdp[replica];
  const int64_t nc = (int64_t)p.nx * p.ny;
  if (cap_cells < nc + 1 || cap_members < p.n_particles) return fail(EDM_EINVAL, "edm_get_cells: buffers too small");
  // The sort buckets hold alive particles only; the reference's cell list
  // holds every particle (dynamics.py:181-196), so group all slots by the
  // reference cell each slot stores.
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<int32_t> cells(p.n_particles), ids(p.n_particles);
  CUDA_TRY(cudaMemcpyAsync(cells.data(), E->cell_pre + p.particle_offset, sizeof(int32_t) * p.n_particles,
                           cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(ids.data(), E->ids[E->cur] + p.particle_offset, sizeof(int32_t) * p.n_particles,
                           cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  for (int64_t c = 0; c <= nc; ++c) cell_start[c] = 0;
  for (int64_t i = 0; i < p.n_particles; ++i) cell_start[cells[i] + 1] += 1;
  for (int64_t c = 0; c < nc; ++c) cell_start[c + 1] += cell_start[c];
  std::vector<int32_t> fill(cell_start, cell_start + nc);
  for (int64_t i = 0; i < p.n_particles; ++i) members[fill[cells[i]]++] = ids[i] - (int32_t)p.particle_offset;
  return EDM_OK;
}

}  // extern "C"

// ---- noise hooks ----------------------------------------------------------------
namespace {
__global__ void k_noise_normals(uint64_t seed, int64_t step, int stream, const int64_t* keys, int64_t n, double* out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const U2 z = normal2(seed, step, stream, (uint64_t)keys[i]);
  out[2 * i] = z.u0;
  out[2 * i + 1] = z.u1;
}
__global__ void k_noise_uniforms(uint64_t seed, int64_t step, int stream, const int64_t* a, const int64_t* b, int64_t n,
                                 double* out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const U2 u = uniform2(seed, step, stream, (uint64_t)a[i], b ? (uint64_t)b[i] : 0u);
  out[2 * i] = u.u0;
  out[2 * i + 1] = u.u1;
}
}  // namespace

extern "C" {
int edm_noise_normal_pairs(uint64_t seed, int64_t step, int32_t stream_id, const int64_t* keys_dev, int64_t n,
                           double* out_dev, void* stream) {
  if (n < 0 || (n > 0 && (!keys_dev || !out_dev))) return fail(EDM_EINVAL, "edm_noise_normal_pairs: bad argument");
  if (n == 0) return EDM_OK;
  k_noise_normals<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(seed, step, stream_id, keys_dev, n,
                                                                               out_dev);
  CUDA_TRY(cudaGetLastError());
  return EDM_OK;
}
int edm_noise_uniforms(uint64_t seed, int64_t step, int32_t stream_id, const int64_t* keys_a_dev,
                       const int64_t* keys_b_dev, int64_t n, double* out2_dev, void* stream) {
  if (n < 0 || (n > 0 && (!keys_a_dev || !out2_dev))) return fail(EDM_EINVAL, "edm_noise_uniforms: bad argument");
  if (n == 0) return EDM_OK;
  k_noise_uniforms<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(seed, step, stream_id, keys_a_dev,
                                                                                keys_b_dev, n, out2_dev);
  CUDA_TRY(cudaGetLastError());
  return EDM_OK;
}
}  // extern "C"
