// edm_dyn.cuh — dynamics kernels (one BD step of DynamicsEngine.step,
// ed_mrdt/dynamics.py:2150-2465) for all replicas of an engine.
//
// Layout.  Every step the particles of every replica are counting-sorted into
// "slots" by a key: the reference cell cx*ny + cy of alive particles
// (dynamics.py:176-196: cx = int(x/cell_sx) clamped), and one extra bucket
// (key nx*ny) holding every particle that is not alive.  Replica r owns slots
// [particle_offset, +n_particles) and sort buckets [cell_offset, +nx*ny+1).
// Non-alive particles never take part in a pair computation
// (dynamics.py:680-681, 767-768, 850-851), so keeping them out of the cells
// leaves the neighbour sweeps with alive particles only; their reference
// cell is still stored per slot.  Slot arrays: position (float64 absolute, or
// float32 offset inside the cell), the cell, one flag byte (species |
// alive<<7) and the particle id.  Id-indexed arrays (bond partner, dye,
// photophysical state) do not move.
//
// Order independence.  The slot order inside a bucket comes from atomics and
// is not deterministic; nothing downstream depends on it:
//  - pair forces are summed per particle in the reference's own pair order
//    (its (j, i) pairs by ascending j, then its (i, j) pairs by neighbour-cell
//    ordinal and descending j; WCA terms before harmonic terms), recovered
//    from particle ids and cells;
//  - every random draw is keyed by particle ids, not by storage position;
//  - reaction passes are set-valued (catalysis) or per particle; the two
//    order-dependent rules (binding's greedy pair order, the recruitment cap
//    in index order) are resolved on small candidate lists sorted by the
//    reference's order key.
#pragma once

#include "edm_common.cuh"

namespace edm {

constexpr int kBlock = 256;
constexpr int kSweepChunk = 128;  // slots per warp in the flag sweeps (4 per lane)
constexpr int kMaxPP = 32;        // recruitment-candidate, detachment and conversion passes per step
constexpr int kRecCap = 128;
constexpr int kBindCap = 512;

struct DevState {
  void* pos_pre;      // double2 (f64) or float2 (f32 offsets), slot order, before the move
  void* pos_post;     // same, after the move
  // f32 path: the float32 remainder of each offset (offset = hi + lo, hi in
  // pos_*); range tests read hi alone, exact arithmetic reads both
  short2* lo_pre;
  short2* lo_post;
  int32_t* cell_pre;  // reference cell of each slot, before the move
  int32_t* cell_post;
  const uint8_t* flags_old;
  uint8_t* flags;     // slot flags of the current step
  const int32_t* ids_old;
  int32_t* ids;       // global particle id of each slot
  int32_t* slot_of_id;
  int32_t* bond;      // id-indexed, global id or -1
  int32_t* cell_start;   // sort-bucket starts [n_buckets + 1]
  int32_t* cell_cursor;
  int32_t* cnt_next;     // bucket counts for the next step's sort
  int32_t* grid_cnt;     // density-grid counts (snapshot of the current pass)
  int32_t* grid_delta;   // pending changes of the current pass
  const double* hill;
  // draw thresholds: a keyed draw u = m 2^-53 with m >= the threshold is
  // rejected by its pass whatever the grid counts (threshold = ceil(b 2^53),
  // b = prob times the largest Hill factor of each rule of the pass)
  const uint64_t* pass_thr;  // [R][kMaxPP] per-particle passes, in schedule order
  const uint64_t* cat_thr;   // [R][EDM_MAX_CAT] catalytic passes
  int64_t* counters;     // [R][EDM_NCOUNTERS]
  uint32_t* status;
  const int64_t* d_step;
  // candidate buffers
  int32_t* rec_count;    // [R]
  int32_t* rec_id;       // [R][kRecCap] local id
  double* rec_xy;        // [R][kRecCap][2]
  int32_t* bind_count;   // [R]
  int64_t* bind_key;     // [R][kBindCap]
  int32_t* bind_ab;      // [R][kBindCap][2] local ids (a = reactant A role, b = B role)
  // catalytic contacts of the step: (enzyme slot, substrate-capable slot)
  int2* contacts;
  int32_t* contact_count;  // [EDM_MAX_CAT]
  int64_t contact_cap;      // per catalytic reaction
  const int64_t* rep_first;  // [R + 1] first slot of each replica
  const int32_t* chunk_rep;  // replica of the first slot of each kSweepChunk-slot chunk
  // slots that left their sort bucket's neighbourhood after the sort this step
  // (recruited, or placed by dissociation): per replica at particle_offset
  int32_t* moved;
  int32_t* moved_count;  // [R]
  // particles whose keyed draws pass some per-particle pass's bound this step:
  // (slot, bit mask of those passes, replica, local id); pl_index[slot] = its entry
  int4* pl;
  int32_t* pl_count;
  int32_t* pl_index;
  // per species: the density grids (bit g) that sense it in some replica
  uint32_t sensor_grids[EDM_MAX_SPECIES];
  // the contact search's sweepers of this step (k_sweep_list), block by block
  int32_t* sw_list;
  int32_t* sw_count;
  // per global grid cell: the adaptation field w (float64, on the adaptation
  // grid's cells) and the local-recruitment CDF (on a feedback grid's cells)
  double* adapt_w;
  double* local_cdf;
  int n_rep;
  int64_t n_slots;
};

__device__ __forceinline__ int replica_of(const int64_t* __restrict__ rep_first, int R, int64_t s) {
  int lo = 0, hi = R - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (rep_first[mid] <= s) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Particles a per-particle pass visits: the species set mask[1] of alive
// particles and mask[0] of particles that are not alive.
struct Match {
  uint32_t mask[2];
};
__device__ __forceinline__ bool matches(uint8_t f, const Match& m) {
  return ((fl_alive(f) ? m.mask[1] : m.mask[0]) >> fl_species(f)) & 1u;
}

// Flag sweep with warp-local compaction: each warp reads the flags of its
// kSweepChunk slots (4 per lane, one 32-bit load), gathers the matching
// slots in its shared-memory list (ballot + popc, no block barrier), then
// runs body(replica, slot) on them with every lane busy.  Launch with
// blockDim == kBlock and ceil(n_slots / (4*kBlock)) blocks.
template <typename Body>
__device__ __forceinline__ void sweep4(const DevState& st, const Match& m, Body body) {
  __shared__ int32_t list[kBlock / 32][kSweepChunk];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) * 4;
  if (w0 >= st.n_slots) return;  // whole warps only
  const int64_t s0 = w0 + (int64_t)lane * 4;
  uchar4 f4 = make_uchar4(0, 0, 0, 0);
  if (s0 < st.n_slots) f4 = *reinterpret_cast<const uchar4*>(st.flags + s0);
  const uint8_t f[4] = {f4.x, f4.y, f4.z, f4.w};
  const unsigned below = (1u << lane) - 1u;
  int n = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const bool hit = s0 + k < st.n_slots && matches(f[k], m);
    const unsigned bits = __ballot_sync(0xffffffffu, hit);
    if (hit) list[wid][n + __popc(bits & below)] = (int32_t)(s0 + k);
    n += __popc(bits);
  }
  __syncwarp();
  if (n == 0) return;
  const int r0 = st.chunk_rep[w0 / kSweepChunk];
  for (int q = lane; q < n; q += 32) {
    const int64_t s = list[wid][q];
    int r = r0;
    while (r + 1 < st.n_rep && st.rep_first[r + 1] <= s) ++r;
    body(r, s);
  }
}

// One atomicAdd per group of lanes adding 1 to the same address; returns
// the value each lane would have got from its own atomicAdd(addr, 1).
__device__ __forceinline__ int atomic_inc_aggregated(int32_t* addr) {
  const unsigned act = __activemask();
  const unsigned peers = __match_any_sync(act, (unsigned long long)(uintptr_t)addr);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(peers) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(addr, __popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + __popc(peers & ((1u << lane) - 1u));
}

// ---- replica geometry --------------------------------------------------------
// The box side and the pair-list cutoff are read from the parameter block
// where they are used (rare branches), so they hold no registers meanwhile.
// Slot, particle and bucket offsets fit 32 bits (slot indices are int32).
struct Geo {
  const EdmDynParams* prm;
  int nx, ny, px, py;
  double sx, sy;
  float sxf, syf, inv_ny;
  int cbase, poff;
  int grave;  // bucket of non-alive particles
  __device__ __forceinline__ double Lx() const { return prm->Lx; }
  __device__ __forceinline__ double Ly() const { return prm->Ly; }
  __device__ __forceinline__ double cutoff_sq() const { return prm->cutoff_sq; }
  __device__ __forceinline__ explicit Geo(const EdmDynParams& p)
      : prm(&p), nx(p.nx), ny(p.ny), px(p.periodic_x), py(p.periodic_y),
        sx(p.cell_sx), sy(p.cell_sy), sxf((float)p.cell_sx),
        syf((float)p.cell_sy), inv_ny(0.0f), cbase((int)p.cell_offset), poff((int)p.particle_offset),
        grave(p.nx * p.ny) {
#ifdef __CUDA_ARCH__  // device-only intrinsic: the reciprocal without a division's slow path
    inv_ny = __frcp_rn((float)p.ny);
#endif
  }
};

// Cell key c = cx * ny + cy -> (cx, cy) without an integer division: the
// float quotient (c + 0.5) / ny is within one of cx for any c < 2^24 and the
// remainder check corrects it, so the result is exact.
__device__ __forceinline__ void split_cell(int c, const Geo& g, int& cx, int& cy) {
  int q = __float2int_rz(((float)c + 0.5f) * g.inv_ny);
  int r = c - q * g.ny;
  if (r < 0) {
    --q;
    r += g.ny;
  } else if (r >= g.ny) {
    ++q;
    r -= g.ny;
  }
  cx = q;
  cy = r;
}

// float32 path: a cell offset o (float64) is stored as hi = its float32
// rounding, clamped into [0, cell side), and lo = o - hi as an int16 count of
// the quantum q = 2^(e - 37), 2^e <= side < 2^(e + 1).  |o - hi| stays within
// 1.5 float32 ulps of the side, 3 * 2^13 q, so lo fits, and hi + lo q is
// within q / 2 of o (3e-13 µm for a 0.165 µm cell).  The scalings by q are
// exact.
__device__ __forceinline__ int lo_exponent(float side_f) {
  return (int)((__float_as_uint(side_f) >> 23) & 0xFFu) - 127 - 37;
}
__device__ __forceinline__ double pow2(int e) { return __longlong_as_double((long long)(1023 + e) << 52); }
__device__ __forceinline__ double lo_value(short l, float side_f) { return (double)l * pow2(lo_exponent(side_f)); }
__device__ __forceinline__ void split_offset(double o, float side_f, float& hi, short& lo) {
  float h = (float)o;
  if (!(h >= 0.0f)) h = 0.0f;
  else if (h >= side_f) h = __int_as_float(__float_as_int(side_f) - 1);  // largest float below the side
  hi = h;
  int q = __double2int_rn((o - (double)h) * pow2(-lo_exponent(side_f)));
  q = q > 32767 ? 32767 : (q < -32767 ? -32767 : q);
  lo = (short)q;
}

// Absolute position of a slot (float64); lo is the f32 path's remainder array.
template <bool F64>
__device__ __forceinline__ void abs_pos(const void* pos, const short2* lo, const int32_t* cell, int64_t s,
                                        const Geo& g, double& x, double& y) {
  if constexpr (F64) {
    const double2 v = ((const double2*)pos)[s];
    x = v.x;
    y = v.y;
  } else {
    const float2 v = ((const float2*)pos)[s];
    const short2 l = lo[s];
    int cx, cy;
    split_cell(cell[s], g, cx, cy);
    x = __dadd_rn(__dmul_rn((double)cx, g.sx), __dadd_rn((double)v.x, lo_value(l.x, g.sxf)));
    y = __dadd_rn(__dmul_rn((double)cy, g.sy), __dadd_rn((double)v.y, lo_value(l.y, g.syf)));
  }
}

// Reference minimum-image separation (dynamics.py:199-216) of absolute points.
__device__ __forceinline__ double min_image_sq(double x1, double y1, double x2, double y2, const Geo& g,
                                               double& dx, double& dy) {
  dx = x1 - x2;
  dy = y1 - y2;
  if (g.px) {
    if (dx > 0.5 * g.Lx()) dx -= g.Lx();
    else if (dx < -0.5 * g.Lx()) dx += g.Lx();
  }
  if (g.py) {
    if (dy > 0.5 * g.Ly()) dy -= g.Ly();
    else if (dy < -0.5 * g.Ly()) dy += g.Ly();
  }
  return dx * dx + dy * dy;
}

// float32 separation of two cell-relative points, i in cell (cxi, cyi), j in
// cell key cj.
__device__ __forceinline__ float rel_sq_f32_xy(int cxi, int cyi, float2 oi, int cj, float2 oj, const Geo& g,
                                               float& dx, float& dy) {
  int cxj, cyj;
  split_cell(cj, g, cxj, cyj);
  int dcx = cxi - cxj, dcy = cyi - cyj;
  if (g.px) {
    if (2 * dcx > g.nx) dcx -= g.nx;
    else if (2 * dcx < -g.nx) dcx += g.nx;
  }
  if (g.py) {
    if (2 * dcy > g.ny) dcy -= g.ny;
    else if (2 * dcy < -g.ny) dcy += g.ny;
  }
  dx = __fmaf_rn((float)dcx, g.sxf, oi.x - oj.x);
  dy = __fmaf_rn((float)dcy, g.syf, oi.y - oj.y);
  return __fmaf_rn(dx, dx, dy * dy);
}

// float32 separation of two cell-relative points (cells ci, cj).
__device__ __forceinline__ float rel_sq_f32(int ci, float2 oi, int cj, float2 oj, const Geo& g, float& dx,
                                            float& dy) {
  int cxi, cyi;
  split_cell(ci, g, cxi, cyi);
  return rel_sq_f32_xy(cxi, cyi, oi, cj, oj, g, dx, dy);
}

// Squared separation of slots a and b in the given position array.
template <bool F64>
__device__ __forceinline__ double sep_sq(const void* pos, const int32_t* cell, int64_t a, int64_t b,
                                         const Geo& g) {
  if constexpr (F64) {
    const double2 pa = ((const double2*)pos)[a], pb = ((const double2*)pos)[b];
    double dx, dy;
    return min_image_sq(pa.x, pa.y, pb.x, pb.y, g, dx, dy);
  } else {
    float dx, dy;
    return (double)rel_sq_f32(cell[a], ((const float2*)pos)[a], cell[b], ((const float2*)pos)[b], g, dx, dy);
  }
}

// Replica r and slot s of this thread (block table of kBlock-slot tiles).
struct Tile {
  int r;
  int64_t s;
};
__device__ __forceinline__ Tile tile_of(const int2* blk) {
  const int2 b = blk[blockIdx.x];
  Tile t;
  t.r = b.x;
  t.s = (int64_t)(uint32_t)b.y + threadIdx.x;
  return t;
}

// Visit the slots of the 3x3 neighbour cells of cell c: f(slot, ordinal,
// dcx, dcy), ordinal = (dcx + 1) * 3 + (dcy + 1) as in dynamics.py:243-260.
// The cells of one neighbour column are consecutive sort buckets, so each
// column is one slot run (two where the column wraps in y); a slot's dcy
// follows from its bucket (its pre-move cell).
template <typename F>
__device__ __forceinline__ void for_neighbour_slots_box(const Geo& g, const DevState& st, int c, int dxlo, int dxhi,
                                                        int dylo, int dyhi, F f) {
  int cx, cy;
  split_cell(c, g, cx, cy);
  // rows cy+dylo .. cy+dyhi (dylo <= 0 <= dyhi) as one or two runs
  int ya0 = cy + dylo, yb0 = cy + dyhi, ya1 = 0, yb1 = -1;
  if (!g.py) {
    ya0 = ya0 < 0 ? 0 : ya0;
    yb0 = yb0 >= g.ny ? g.ny - 1 : yb0;
  } else if (ya0 < 0) {
    ya0 = 0;
    ya1 = yb1 = g.ny - 1;
  } else if (yb0 >= g.ny) {
    yb0 = g.ny - 1;
    ya1 = yb1 = 0;
  }
  for (int dcx = dxlo; dcx <= dxhi; ++dcx) {
    int ncx = cx + dcx;
    if (g.px) ncx = ncx < 0 ? ncx + g.nx : (ncx >= g.nx ? ncx - g.nx : ncx);
    else if (ncx < 0 || ncx >= g.nx) continue;
    const int col = ncx * g.ny;
    for (int run = 0; run < 2; ++run) {
      const int ya = run == 0 ? ya0 : ya1, yb = run == 0 ? yb0 : yb1;
      if (yb < ya) break;
      const int j0 = st.cell_start[g.cbase + col + ya], j1 = st.cell_start[g.cbase + col + yb + 1];
      for (int j = j0; j < j1; ++j) {
        int dcy = st.cell_pre[j] - col - cy;
        dcy = dcy > 1 ? dcy - g.ny : (dcy < -1 ? dcy + g.ny : dcy);
        f(j, (dcx + 1) * 3 + (dcy + 1), dcx, dcy);
      }
    }
  }
}

template <typename F>
__device__ __forceinline__ void for_neighbour_slots(const Geo& g, const DevState& st, int c, F f) {
  for_neighbour_slots_box(g, st, c, -1, 1, -1, 1, f);
}

// ---- density grids -----------------------------------------------------------
// int(x / s) as the reference computes it (a rounded float64 quotient,
// truncated), without the division when it cannot matter: the product x * inv
// lies within a few ulps of the quotient, so when it is farther than 1e-6
// from an integer both truncate to the same value; closer than that (about
// one call in 10^6) the quotient itself is taken.
__device__ __forceinline__ int grid_index(double x, double s, double inv) {
  const double q = x * inv;
  const double f = q - floor(q);
  return (f > 1e-6 && f < 1.0 - 1e-6) ? (int)q : (int)__ddiv_rn(x, s);
}

__device__ __forceinline__ int64_t grid_cell_of(const EdmGrid& G, double x, double y) {
  const int gx = clampi(grid_index(x, G.sx, G.inv_sx), G.nx);
  const int gy = clampi(grid_index(y, G.sy, G.inv_sy), G.ny);
  return G.offset + (int64_t)gx * G.ny + gy;
}

// Density of a grid cell holding k particles: the reference's k-fold
// sequential float64 sum of inv_area (dynamics.py:1685-1703).
__device__ __forceinline__ double kfold_density(int k, double inv_area) {
  double rho = 0.0;
  for (int i = 0; i < k; ++i) rho = __dadd_rn(rho, inv_area);
  return rho;
}

// Adaptation factor 1/(1 + (w/K)^n) of catalytic feedback rule `rule` at
// (x, y) (dynamics.py:1077-1083): w is read as adaptation_field[gx, gy] with
// the feedback grid's (gx, gy), i.e. at flat index gx * ny_adapt + gy of the
// adaptation grid (the host rejects grids where that leaves the array); w = 0
// without a PIP3 grid.
__device__ __forceinline__ double adapt_factor(const EdmDynParams& p, const double* __restrict__ w_all, int rule,
                                               double x, double y) {
  const EdmGrid& G = p.grid[p.rule[rule].grid];
  const int gx = clampi(grid_index(x, G.sx, G.inv_sx), G.nx);
  const int gy = clampi(grid_index(y, G.sy, G.inv_sy), G.ny);
  double w = 0.0;
  if (p.adapt_grid >= 0) {
    const EdmGrid& A = p.grid[p.adapt_grid];
    w = w_all[A.offset + (int64_t)gx * A.ny + gy];
  }
  if (p.adapt_K > 0) return __ddiv_rn(1.0, __dadd_rn(1.0, pow(__ddiv_rn(w, p.adapt_K), p.adapt_n)));
  return 1.0;
}

// Add d to every grid counting species sp, at (x, y) — into `arr`.
__device__ __forceinline__ void grid_add(const EdmDynParams& p, int32_t* arr, int sp, double x, double y, int d) {
  for (int g = 0; g < p.n_grids; ++g) {
    if (p.grid[g].sensor == sp) atomicAdd(&arr[grid_cell_of(p.grid[g], x, y)], d);
  }
}

__device__ __forceinline__ double rule_factor(const EdmDynParams& p, int rule, const DevState& st, double x,
                                              double y) {
  const EdmRule& R = p.rule[rule];
  const int k = st.grid_cnt[grid_cell_of(p.grid[R.grid], x, y)];
  return hill_of(R, st.hill, k, st.status);
}

// Grid bookkeeping of a particle changing (species, alive) at one position.
__device__ __forceinline__ void grid_change(const EdmDynParams& p, int32_t* delta, int sp_old, bool alive_old,
                                            int sp_new, bool alive_new, double x, double y) {
  if (alive_old) grid_add(p, delta, sp_old, x, y, -1);
  if (alive_new) grid_add(p, delta, sp_new, x, y, +1);
}

// Record a slot placed away from its sort bucket after this step's sort.
__device__ __forceinline__ void note_moved(const DevState& st, int r, const EdmDynParams& p, int64_t slot) {
  const int k = atomicAdd(&st.moved_count[r], 1);
  if (k < p.n_particles) st.moved[p.particle_offset + k] = (int32_t)slot;
}

// Next step's bucket counts when a particle changes bucket.
__device__ __forceinline__ void rebucket(const DevState& st, const Geo& g, int from, int to) {
  if (from == to) return;
  atomicAdd(&st.cnt_next[g.cbase + from], -1);
  atomicAdd(&st.cnt_next[g.cbase + to], 1);
}

// =============================================================================
// Sort: exclusive scan of the bucket counts, scatter into slots.
// =============================================================================
constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;  // one int4 per thread: a warp touches 512 contiguous bytes
constexpr int kScanTile = kScanThreads * kScanItems;

// The kScanItems counts at [base, base + 4) (zero past n); arrays are
// 16-byte aligned and base is a multiple of 4.
__device__ __forceinline__ int4 load4(const int32_t* __restrict__ a, int64_t base, int64_t n) {
  if (base + 3 < n) return *reinterpret_cast<const int4*>(a + base);
  int4 v = make_int4(0, 0, 0, 0);
  if (base < n) v.x = a[base];
  if (base + 1 < n) v.y = a[base + 1];
  if (base + 2 < n) v.z = a[base + 2];
  return v;
}
__device__ __forceinline__ void store4(int32_t* __restrict__ a, int64_t base, int64_t n, int4 v) {
  if (base + 3 < n) {
    *reinterpret_cast<int4*>(a + base) = v;
    return;
  }
  if (base < n) a[base] = v.x;
  if (base + 1 < n) a[base + 1] = v.y;
  if (base + 2 < n) a[base + 2] = v.z;
}

__device__ __forceinline__ int block_exclusive_scan(int v, int& total) {
  __shared__ int warp_sums[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    int w = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) warp_sums[lane] = w;
  }
  __syncthreads();
  const int base = wid > 0 ? warp_sums[wid - 1] : 0;
  total = warp_sums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return base + x - v;
}

// Buffers the step clears before its kernels use them (density grids and
// their deltas, the placed-after-sort and contact counters, the draw list
// length): cleared by the first scan kernel instead of one memset each.
struct StepZero {
  int32_t* p[6];
  int64_t n[6];
};

__global__ void k_scan_reduce(const int32_t* __restrict__ cnt, int64_t n, int32_t* __restrict__ bsum, StepZero z) {
  for (int k = 0; k < 6; ++k)
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < z.n[k]; i += (int64_t)gridDim.x * blockDim.x)
      z.p[k][i] = 0;
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  const int4 c = load4(cnt, base, n);
  const int v = c.x + c.y + c.z + c.w;
  int total;
  block_exclusive_scan(v, total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void k_scan_bsum(int32_t* __restrict__ bsum, int nb) {
  pdl_enter();
  int carry = 0;
  for (int off = 0; off < nb; off += blockDim.x) {
    const int i = off + threadIdx.x;
    const int v = i < nb ? bsum[i] : 0;
    int total;
    const int ex = block_exclusive_scan(v, total);
    if (i < nb) bsum[i] = carry + ex;
    carry += total;
  }
}

__global__ void k_scan_down(int32_t* __restrict__ cnt, int64_t n, const int32_t* __restrict__ bsum,
                            int32_t* __restrict__ start, int32_t* __restrict__ cursor) {
  pdl_enter();
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  const int4 c = load4(cnt, base, n);
  int total;
  const int run = block_exclusive_scan(c.x + c.y + c.z + c.w, total) + bsum[blockIdx.x];
  const int4 st4 = make_int4(run, run + c.x, run + c.x + c.y, run + c.x + c.y + c.z);
  store4(start, base, n, st4);
  store4(cursor, base, n, st4);
  store4(cnt, base, n, make_int4(0, 0, 0, 0));
  // the thread holding element n-1 writes the sentinel start[n]
  if (base < n && base + kScanItems >= n) start[n] = run + c.x + c.y + c.z + c.w;
  if (n == 0 && blockIdx.x == 0 && threadIdx.x == 0) start[0] = 0;
}

template <bool F64, int BS, int SPT>
__global__ void __launch_bounds__(BS) k_scatter(const EdmDynParams* __restrict__ P, const int2* __restrict__ blk,
                                                    int ntiles, DevState st) {
  pdl_enter();
  // SPT tiles per block (blockIdx.x * SPT + k): each thread reads its slots'
  // buckets and takes all their cursor positions before the first dependent
  // store, so SPT atomics are in flight per thread
  int64_t src[SPT], bkt[SPT];
  uint8_t fl[SPT];
  int cl[SPT], dst[SPT];
#pragma unroll
  for (int k = 0; k < SPT; ++k) {
    src[k] = -1;
    const int tile = (int)blockIdx.x * SPT + k;
    if (tile >= ntiles) continue;
    const int2 b = blk[tile];
    const EdmDynParams& p = P[b.x];
    const int64_t s = (int64_t)(uint32_t)b.y + threadIdx.x;
    if (s >= p.particle_offset + p.n_particles) continue;
    src[k] = s;
    cl[k] = st.cell_post[s];
    fl[k] = st.flags_old[s];
    bkt[k] = p.cell_offset + (fl_alive(fl[k]) ? cl[k] : p.nx * p.ny);
  }
#pragma unroll
  for (int k = 0; k < SPT; ++k) {
    if (src[k] < 0) continue;
    // alive particles mostly have a cell to themselves: a plain atomic; the
    // non-alive ones all share their replica's last bucket: aggregated per warp
    dst[k] = fl_alive(fl[k]) ? atomicAdd(&st.cell_cursor[bkt[k]], 1) : atomic_inc_aggregated(&st.cell_cursor[bkt[k]]);
  }
#pragma unroll
  for (int k = 0; k < SPT; ++k) {
    if (src[k] < 0) continue;
    const int64_t s = src[k];
    const int d = dst[k];
    if constexpr (F64) {
      ((double2*)st.pos_pre)[d] = ((const double2*)st.pos_post)[s];
    } else {
      ((float2*)st.pos_pre)[d] = ((const float2*)st.pos_post)[s];
      st.lo_pre[d] = st.lo_post[s];
    }
    st.cell_pre[d] = cl[k];
    st.flags[d] = fl[k];
    const int id = st.ids_old[s];
    st.ids[d] = id;
    st.slot_of_id[id] = d;
  }
}

// =============================================================================
// Forces + Ermak–McCammon move (dynamics.py:440-519, 665-816, 323-406).
// =============================================================================

// Enumerate the pair-force terms of slot s; pass `emit(key, fx, fy)`.
constexpr int kForceCand = 2;  // float32 force candidates listed per sweep

template <bool F64, typename Emit>
__device__ __forceinline__ void for_each_force_term(const EdmDynParams& p, const Geo& g, const DevState& st,
                                                    int64_t s, int sp, int id, Emit emit, int2* cand = nullptr,
                                                    int cand_stride = 0) {
  double xi = 0, yi = 0;
  float2 oi = make_float2(0.f, 0.f);
  if constexpr (F64) {
    const double2 v = ((const double2*)st.pos_pre)[s];
    xi = v.x;
    yi = v.y;
  } else {
    oi = ((const float2*)st.pos_pre)[s];
  }
  // pairs beyond both the pair-list cutoff and every potential's range carry no force
  const double range_sq = p.force_range_sq < g.cutoff_sq() ? p.force_range_sq : g.cutoff_sq();
  const float range_sqf = (float)range_sq * 1.0001f;
  // Only neighbour cells within that range of the particle can hold a force
  // partner (a partner in a skipped column or row is farther than its offset
  // to the cell side, itself beyond the range), so the sweep skips the others.
  // Range <= cutoff <= cell side keeps every partner inside the 3x3 block.
  const int c_pre = st.cell_pre[s];
  double ox, oy;
  if constexpr (F64) {
    int cx, cy;
    split_cell(c_pre, g, cx, cy);
    ox = xi - (double)cx * g.sx;
    oy = yi - (double)cy * g.sy;
  } else {
    ox = (double)oi.x;
    oy = (double)oi.y;
  }
  const double reach = p.force_reach;  // sqrt(range_sq) * 1.0001 + 1e-9, from the host
  const int dxlo = ox < reach ? -1 : 0, dxhi = ox > g.sx - reach ? 1 : 0;
  const int dylo = oy < reach ? -1 : 0, dyhi = oy > g.sy - reach ? 1 : 0;
  auto term = [&](int j, int ordinal, int dcx, int dcy) {
    {
      if (j == s) return;
      double dx, dy, dsq;
      if constexpr (F64) {
        const double2 v = ((const double2*)st.pos_pre)[j];
        dsq = min_image_sq(xi, yi, v.x, v.y, g, dx, dy);
        if (!(dsq < range_sq)) return;
      } else {
        // float32 range test (with a 1e-4 relative margin) on every
        // neighbour; the few pairs inside it get their separation in float64
        // from (cell, offset): the float32 sum below rounds at the ulp of a
        // cell side, a large fraction of |dx| for nearly coincident pairs
        const float2 oj = ((const float2*)st.pos_pre)[j];
        const float fdx = __fmaf_rn(-(float)dcx, g.sxf, oi.x - oj.x);
        const float fdy = __fmaf_rn(-(float)dcy, g.syf, oi.y - oj.y);
        const float fdsq = __fmaf_rn(fdx, fdx, fdy * fdy);
        if (!(fdsq < range_sqf)) return;
        const short2 li = st.lo_pre[s], lj = st.lo_pre[j];
        dx = (double)(-dcx) * g.sx +
             (((double)oi.x - (double)oj.x) + (double)((int)li.x - (int)lj.x) * pow2(lo_exponent(g.sxf)));
        dy = (double)(-dcy) * g.sy +
             (((double)oi.y - (double)oj.y) + (double)((int)li.y - (int)lj.y) * pow2(lo_exponent(g.syf)));
        dsq = dx * dx + dy * dy;
        if (!(dsq < range_sq)) return;
      }
      const uint8_t fj = st.flags[j];
      if (!fl_alive(fj)) return;
      const int spj = fl_species(fj);
      const double sig = p.sigma[sp * EDM_MAX_SPECIES + spj];
      if (!(sig > 0.0)) return;
      const int idj = st.ids[j] - (int)g.poff;
      const uint64_t order = idj < id ? (uint64_t)idj
                                      : ((1ull << 60) | ((uint64_t)ordinal << 32) | (uint64_t)(0xFFFFFFFFu - (uint32_t)idj));
      // The pair force itself is float64 on both paths: a pair inside force
      // range is rare (a few per thousand particles at the membrane
      // densities), and a capped move takes the direction of this force.
      if (p.use_wca) {
        const double eps = p.eps[sp * EDM_MAX_SPECIES + spj];
        if (eps > 0.0) {
          const double rcut2 = sig * sig * 1.2599210498948732;
          if (dsq < rcut2 && dsq >= 1e-30) {
            const double inv_r2 = 1.0 / dsq;
            const double s2 = sig * sig * inv_r2;
            const double s6 = s2 * s2 * s2;
            const double s12 = s6 * s6;
            double f = 24.0 * eps * (2.0 * s12 - s6) * inv_r2;
            const double fmax = 2400.0 * eps / (sig * sig);
            if (f > fmax) f = fmax;
            emit(order, f * dx, f * dy);
          }
        }
      }
      if (p.use_harmonic) {
        const double k = p.kharm[sp * EDM_MAX_SPECIES + spj];
        if (k > 0.0) {
          const double s2 = sig * sig;
          if (dsq < s2 && dsq >= 1e-30) {
            const double r = sqrt(dsq);
            const double f = k * (sig - r) / r;
            emit(order | (1ull << 62), f * dx, f * dy);
          }
        }
      }
    }
  };
  if constexpr (F64) {
    for_neighbour_slots_box(g, st, c_pre, dxlo, dxhi, dylo, dyhi, term);
  } else {
    // The sweep only lists the neighbours that pass the float32 range test
    // (rarely any) in cand[0], cand[cand_stride], ...; their float64
    // separation and force follow after it, so the sweep's loop does not
    // hold the float64 pair code's registers.  More than kForceCand of them
    // take further sweeps, each listing the next kForceCand in sweep order.
    for (int done = 0;; done += kForceCand) {
      int found = 0, kept = 0;
      for_neighbour_slots_box(g, st, c_pre, dxlo, dxhi, dylo, dyhi, [&](int j, int ordinal, int dcx, int dcy) {
        if (j == s) return;
        const float2 oj = ((const float2*)st.pos_pre)[j];
        const float fdx = __fmaf_rn(-(float)dcx, g.sxf, oi.x - oj.x);
        const float fdy = __fmaf_rn(-(float)dcy, g.syf, oi.y - oj.y);
        if (!(__fmaf_rn(fdx, fdx, fdy * fdy) < range_sqf)) return;
        const int rank = found++;
        if (rank >= done && rank < done + kForceCand) cand[(kept++) * cand_stride] = make_int2(j, ordinal);
      });
      for (int k = 0; k < kept; ++k) {
        const int2 e = cand[k * cand_stride];
        term(e.x, e.y, e.y / 3 - 1, e.y % 3 - 1);
      }
      if (found <= done + kForceCand) break;
    }
  }
}

// D(x) and grad D at an absolute position (dynamics.py:440-519; sine-x field).
__device__ __forceinline__ void dfield(const EdmDynParams& p, int sp, double x, double y, double& D, double& gx,
                                       double& gy) {
  const double base = p.D_base[sp];
  double factor = 1.0, gfx = 0.0, gfy = 0.0;
  if (p.dfield == EDM_DFIELD_REGIONS) {
    for (int reg = 0; reg < p.n_regions; ++reg) {
      const double dxc = x - p.reg_cx[reg], dyc = y - p.reg_cy[reg];
      const double dsq = dxc * dxc + dyc * dyc;
      const double d = dsq > 1e-30 ? sqrt(dsq) : 1e-15;
      const double arg = (d - p.reg_r[reg]) / p.smooth_w;
      double sig, dsig;
      if (arg > 100.0) {
        sig = 0.0;
        dsig = 0.0;
      } else if (arg < -100.0) {
        sig = 1.0;
        dsig = 0.0;
      } else {
        const double ea = exp(arg);
        const double den = 1.0 + ea;
        sig = 1.0 / den;
        dsig = -ea / (den * den * p.smooth_w);
      }
      const double local = 1.0 + (p.reg_f[reg] - 1.0) * sig;
      if (sig > 0.01) {
        factor = local;
        const double inv_d = 1.0 / d;
        gfx = (p.reg_f[reg] - 1.0) * dsig * dxc * inv_d;
        gfy = (p.reg_f[reg] - 1.0) * dsig * dyc * inv_d;
        break;
      }
    }
    D = base * factor;
    gx = base * gfx;
    gy = base * gfy;
  } else if (p.dfield == EDM_DFIELD_SINE_X) {
    const double w = 2.0 * 3.141592653589793 / p.sine_wavelength;
    const double ph = w * x;
    double sn, cs;
    sincos(ph, &sn, &cs);
    D = base * (1.0 + p.sine_amp * sn);
    gx = base * p.sine_amp * w * cs;
    gy = 0.0;
  } else {
    D = base * factor;
    gx = base * gfx;
    gy = base * gfy;
  }
}

// dfield out of line, for the float32 move: most systems have no D(x) field,
// and the field's float64 code would otherwise share the move's registers.
__device__ __noinline__ void dfield_call(const EdmDynParams& p, int sp, double x, double y, double& D, double& gx,
                                         double& gy) {
  dfield(p, sp, x, y, D, gx, gy);
}

// BS threads per block over tiles of BS slots; MINB resident blocks per SM
// requested from the register allocator (1 = no constraint).
template <bool F64, int BS, int MINB>
__global__ void __launch_bounds__(BS, MINB) k_move(const EdmDynParams* __restrict__ P, const int2* __restrict__ blk,
                                                 DevState st) {
  pdl_enter();
  const Tile t = tile_of(blk);
  const EdmDynParams& p = P[t.r];
  const int64_t s = t.s;
  if (s >= p.particle_offset + p.n_particles) return;
  const Geo g(p);
  const uint8_t f = st.flags[s];
  const int c = st.cell_pre[s];
  if (!fl_alive(f)) {  // dead / dormant particles do not move (dynamics.py:360)
    if constexpr (F64) {
      ((double2*)st.pos_post)[s] = ((const double2*)st.pos_pre)[s];
    } else {
      ((float2*)st.pos_post)[s] = ((const float2*)st.pos_pre)[s];
      st.lo_post[s] = st.lo_pre[s];
    }
    st.cell_post[s] = c;
    atomic_inc_aggregated(&st.cnt_next[g.cbase + g.grave]);
    return;
  }
  const int sp = fl_species(f);
  // the float32 path reads its id and the step index after the force sweep,
  // which needs neither, so that they hold no registers during it
  int id = 0;
  int64_t step = 0;
  if constexpr (F64) {
    id = st.ids[s] - (int)g.poff;
    step = *st.d_step;
  }

  // Pair forces.  The float64 path sums them in the reference's accumulation
  // order (a sum of two terms is the same either way, so only three or more
  // terms are re-summed in order).  The float32 path sums them in 2^-20
  // fixed point, exact and independent of the sweep order, so runs repeat
  // bit for bit.
  double Fx = 0.0, Fy = 0.0;
  long long qx = 0, qy = 0;
  int nterms = 0;
  __shared__ int2 cand_smem[F64 ? 1 : kForceCand * BS];
  for_each_force_term<F64>(p, g, st, s, sp, id, [&](uint64_t, double fx, double fy) {
    ++nterms;
    if constexpr (F64) {
      Fx += fx;
      Fy += fy;
    } else {
      qx += __double2ll_rn(fx * 0x1p20);
      qy += __double2ll_rn(fy * 0x1p20);
    }
  }, cand_smem + threadIdx.x, BS);
  if constexpr (F64) {
    if (nterms > 2) {
      Fx = 0.0;
      Fy = 0.0;
      uint64_t last = 0;
      bool first = true;
      for (int k = 0; k < nterms; ++k) {
        uint64_t best = ~0ull;
        double bx = 0.0, by = 0.0;
        for_each_force_term<F64>(p, g, st, s, sp, id, [&](uint64_t key, double fx, double fy) {
          if ((first || key > last) && key < best) {
            best = key;
            bx = fx;
            by = fy;
          }
        });
        Fx += bx;
        Fy += by;
        last = best;
        first = false;
      }
    }
  } else if (nterms > 0) {  // most particles have no partner in force range
    Fx = (double)qx * 0x1p-20;
    Fy = (double)qy * 0x1p-20;
  }

  double x = 0.0, y = 0.0;
  // the float32 path needs the absolute position here only for a D(x) field
  if (F64 || p.dfield != EDM_DFIELD_NONE) abs_pos<F64>(st.pos_pre, st.lo_pre, st.cell_pre, s, g, x, y);
  double Di, gDx, gDy;
  if constexpr (F64) {
    dfield(p, sp, x, y, Di, gDx, gDy);
  } else if (p.dfield == EDM_DFIELD_NONE) {
    Di = p.D_base[sp];
    gDx = gDy = 0.0;
  } else {
    dfield_call(p, sp, x, y, Di, gDx, gDy);
  }
  const double dt = p.dt;
  int newc;
  if constexpr (F64) {
    const U2 z = normal2(p.seed, step, EDM_S_BD_NORMAL, (uint64_t)id);
    const double sn = sqrt(2.0 * Di * dt);
    double dxt = gDx * dt, dyt = gDy * dt;
    dxt += sn * z.u0;
    dyt += sn * z.u1;
    dxt += Di * Fx * dt;
    dyt += Di * Fy * dt;
    const double dr2 = dxt * dxt + dyt * dyt;
    if (dr2 > p.max_disp_sq) {
      const double scale = p.max_disp / sqrt(dr2);
      dxt *= scale;
      dyt *= scale;
    }
    x += dxt;
    y += dyt;
    if (g.px) x = py_fmod(x, g.Lx());
    else if (x < 0.0) x = -x;
    else if (x >= g.Lx()) x = 2.0 * g.Lx() - x;
    if (g.py) y = py_fmod(y, g.Ly());
    else if (y < 0.0) y = -y;
    else if (y >= g.Ly()) y = 2.0 * g.Ly() - y;
    if (!isfinite(x) || !isfinite(y)) set_status(st.status, EDM_STATUS_NONFINITE);
    ((double2*)st.pos_post)[s] = make_double2(x, y);
    newc = cell_index(x, g.sx, g.nx) * g.ny + cell_index(y, g.sy, g.ny);
  } else {
    id = st.ids[s] - (int)g.poff;
    step = *st.d_step;
    float z0, z1;
    normal2_f32(p.seed, step, EDM_S_BD_NORMAL, (uint64_t)id, z0, z1);
    const float Dif = (float)Di, dtf = (float)dt;
    const float sn = sqrtf(2.0f * Dif * dtf);
    float dxt = __fmaf_rn(sn, z0, __fmaf_rn((float)gDx, dtf, Dif * (float)Fx * dtf));
    float dyt = __fmaf_rn(sn, z1, __fmaf_rn((float)gDy, dtf, Dif * (float)Fy * dtf));
    const float dr2 = __fmaf_rn(dxt, dxt, dyt * dyt);
    double ddx = (double)dxt, ddy = (double)dyt;
    if (dr2 > (float)(p.max_disp_sq * 0.999)) {
      // at (or within rounding of) the displacement cap the move keeps only
      // its direction: form and cap it in float64 as dynamics.py:378-385 do
      ddx = gDx * dt;
      ddy = gDy * dt;
      const double sn64 = sqrt(2.0 * Di * dt);
      ddx += sn64 * (double)z0;
      ddy += sn64 * (double)z1;
      ddx += Di * Fx * dt;
      ddy += Di * Fy * dt;
      const double d2 = ddx * ddx + ddy * ddy;
      if (d2 > p.max_disp_sq) {
        const double scale = p.max_disp / sqrt(d2);
        ddx *= scale;
        ddy *= scale;
      }
    }
    // the new offset in float64 from hi + lo, carried into the next cell
    // against the float64 cell side, then stored as hi + lo again
    const float2 oh = ((const float2*)st.pos_pre)[s];
    const short2 ol = st.lo_pre[s];
    int cx, cy;
    split_cell(c, g, cx, cy);
    double ax = ((double)oh.x + lo_value(ol.x, g.sxf)) + ddx;
    double ay = ((double)oh.y + lo_value(ol.y, g.syf)) + ddy;
    if (!(ax >= 0.0 && ax < g.sx)) {
      const int k = (int)floor(ax / g.sx);
      cx += k;
      ax -= (double)k * g.sx;
    }
    if (!(ay >= 0.0 && ay < g.sy)) {
      const int k = (int)floor(ay / g.sy);
      cy += k;
      ay -= (double)k * g.sy;
    }
    if (g.px) {  // |cx| stays within 64 cells of the box: a few wraps at most
      while (cx >= g.nx) cx -= g.nx;
      while (cx < 0) cx += g.nx;
    } else if (cx < 0 || cx >= g.nx) {  // reflecting wall, in float64
      double bx = (double)cx * g.sx + ax;
      if (bx < 0.0) bx = -bx;
      else if (bx >= g.Lx()) bx = 2.0 * g.Lx() - bx;
      cx = cell_index(bx, g.sx, g.nx);
      ax = bx - (double)cx * g.sx;
    }
    if (g.py) {
      while (cy >= g.ny) cy -= g.ny;
      while (cy < 0) cy += g.ny;
    } else if (cy < 0 || cy >= g.ny) {
      double by = (double)cy * g.sy + ay;
      if (by < 0.0) by = -by;
      else if (by >= g.Ly()) by = 2.0 * g.Ly() - by;
      cy = cell_index(by, g.sy, g.ny);
      ay = by - (double)cy * g.sy;
    }
    if (!isfinite(ax) || !isfinite(ay)) set_status(st.status, EDM_STATUS_NONFINITE);
    float2 o;
    short2 l;
    split_offset(ax, g.sxf, o.x, l.x);
    split_offset(ay, g.syf, o.y, l.y);
    ((float2*)st.pos_post)[s] = o;
    st.lo_post[s] = l;
    newc = cx * g.ny + cy;
    x = (double)cx * g.sx + ax;
    y = (double)cy * g.sy + ay;
  }
  st.cell_post[s] = newc;
  atomicAdd(&st.cnt_next[g.cbase + newc], 1);  // result unused: a fire-and-forget reduction
  // grid_add over only the grids that can sense this species (most species have none)
  for (uint32_t gm = st.sensor_grids[sp]; gm; gm &= gm - 1) {
    const int gi = __ffs(gm) - 1;
    if (p.grid[gi].sensor == sp) atomicAdd(&st.grid_cnt[grid_cell_of(p.grid[gi], x, y)], 1);
  }
}

// =============================================================================
// Reactions.
// =============================================================================

// Catalytic contacts (pairs of the reference's pre-move pair list, dynamics.py
// :219-278, in post-move contact).  During the catalytic passes enzymes keep
// their species and nobody moves or dies, so pass c needs the pairs (enzyme
// of species E_c, partner) within c's contact radius whose partner holds c's
// substrate S_c when pass c runs:
// * direct pairs, whose partner holds S_c at the step start, are found by
//   one sweep after the move, from the rarer side of each reaction: the
//   alive particles of the sweeping species (E_c or S_c) visit their
//   neighbour cells for the other species.  Both distance tests are
//   symmetric in the two particles (the float32 differences change sign
//   exactly), so either side finds the same pairs;
// * late pairs, whose partner an earlier catalytic pass of the step turns
//   into S_c, are few: the pass that converts a particle looks up its
//   enzymes of the later reactions at once (late_contacts).
// A late pair is filed only when its keyed draw for the pass lies below the
// pass's threshold (the pass rejects it otherwise); the sweep files every
// direct pair and leaves the draws to the passes (a Philox per pair inside
// the sweep measured slower).  A pair can be filed twice (a partner converted
// away and back); the passes accept a substrate once, so duplicates change
// nothing.
constexpr int kContactSmem = 2048;

struct CatLists {
  uint32_t sweep_rx[EDM_MAX_SPECIES];        // reactions whose direct pairs the species sweeps for
  uint32_t sweep_partners[EDM_MAX_SPECIES];  // species those sweeps look for
  int32_t other[EDM_MAX_CAT];                // species the sweeper of reaction c looks for
  uint32_t from_enzyme;                      // reactions swept from the enzyme side
  int n_cat;
};

// Whether pass c's keyed draw for the pair of local ids (a, b) of replica r
// lies below the pass's threshold.  The pass rejects the pair otherwise,
// whatever the state, so a pair whose draw fails is not filed.
__device__ __forceinline__ bool cat_draw_passes(const EdmDynParams& p, const DevState& st, int r, int c, int a,
                                                int b, int64_t step) {
  const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
  return draw_u53(p.seed, step, EDM_S_CAT + c, lo, hi) < st.cat_thr[(int64_t)r * EDM_MAX_CAT + c];
}

// One neighbour j (pre-move cell offset dcx, dcy) of sweeper s: the pair
// tests, then stage(c, enzyme, substrate) for each reaction of rx it meets.
// oi_pre / oi_post / (cxs, cys): the sweeper's float32 offsets and post-move
// cell (float32 path).
template <bool F64, typename Stage>
__device__ __forceinline__ void contact_candidate(const EdmDynParams& p, const Geo& g, const DevState& st,
                                                  const CatLists& L, int64_t s, int j, int dcx, int dcy,
                                                  uint32_t rx, uint32_t pmask,
                                                  float2 oi_pre, float2 oi_post, int cxs, int cys, Stage stage) {
  if (j == s) return;
  const uint8_t fj = st.flags[j];
  const int spj = fl_species(fj);
  if (!fl_alive(fj) || !((pmask >> spj) & 1u)) return;
  double d2;
  if constexpr (F64) {
    if (!(sep_sq<F64>(st.pos_pre, st.cell_pre, s, j, g) < g.cutoff_sq())) return;
    d2 = sep_sq<F64>(st.pos_post, st.cell_post, s, j, g);
  } else {
    // pre-move: j sits in the neighbour cell at (dcx, dcy)
    const float2 oj = ((const float2*)st.pos_pre)[j];
    const float fdx = __fmaf_rn(-(float)dcx, g.sxf, oi_pre.x - oj.x);
    const float fdy = __fmaf_rn(-(float)dcy, g.syf, oi_pre.y - oj.y);
    if (!((double)__fmaf_rn(fdx, fdx, fdy * fdy) < g.cutoff_sq())) return;
    float dx, dy;
    d2 = (double)rel_sq_f32_xy(cxs, cys, oi_post, st.cell_post[j], ((const float2*)st.pos_post)[j], g, dx, dy);
  }
  for (uint32_t bits = rx; bits; bits &= bits - 1) {
    const int c = __ffs(bits) - 1;
    if (spj != L.other[c] || d2 > p.cat[c].contact_sq) continue;
    if ((L.from_enzyme >> c) & 1u) stage(c, (int)s, j);
    else stage(c, j, (int)s);
  }
}

// Shared-memory staging of a block's contact pairs, per reaction, then one
// global append per reaction; a full stage appends directly.
struct ContactStage {
  int2* buf;
  int* nbuf;
  int per;
  __device__ __forceinline__ void operator()(const DevState& st, int c, int e, int sub) const {
    const int k = atomicAdd(&nbuf[c], 1);
    if (k < per) {
      buf[c * per + k] = make_int2(e, sub);
    } else {
      const int q = atomicAdd(&st.contact_count[c], 1);
      if (q < st.contact_cap) st.contacts[(int64_t)c * st.contact_cap + q] = make_int2(e, sub);
      else set_status(st.status, EDM_STATUS_CONTACT_CAP);
    }
  }
};

__device__ __forceinline__ void flush_contacts(const DevState& st, const CatLists& L, const ContactStage& S,
                                               int* base) {
  __syncthreads();
  if (threadIdx.x < L.n_cat) {
    const int n = S.nbuf[threadIdx.x] < S.per ? S.nbuf[threadIdx.x] : S.per;
    base[threadIdx.x] = n > 0 ? atomicAdd(&st.contact_count[threadIdx.x], n) : 0;
  }
  __syncthreads();
  for (int c = 0; c < L.n_cat; ++c) {
    const int n = S.nbuf[c] < S.per ? S.nbuf[c] : S.per;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const int64_t q = (int64_t)base[c] + k;
      if (q < st.contact_cap) st.contacts[(int64_t)c * st.contact_cap + q] = S.buf[c * S.per + k];
      else set_status(st.status, EDM_STATUS_CONTACT_CAP);
    }
  }
}

template <bool F64, int MINB>
__global__ void __launch_bounds__(kBlock, MINB) k_contacts(const EdmDynParams* __restrict__ P, DevState st, Match m,
                                                     CatLists L) {
  pdl_enter();
  __shared__ int2 buf[kContactSmem];
  __shared__ int nbuf[EDM_MAX_CAT], base[EDM_MAX_CAT];
  const ContactStage S{buf, nbuf, L.n_cat > 0 ? kContactSmem / L.n_cat : kContactSmem};
  if (threadIdx.x < EDM_MAX_CAT) nbuf[threadIdx.x] = 0;
  __syncthreads();
  sweep4(st, m, [&](int r, int64_t s) {
    const EdmDynParams& p = P[r];
    const Geo g(p);
    const int sps = fl_species(st.flags[s]);
    const uint32_t rx = L.sweep_rx[sps], pmask = L.sweep_partners[sps];
    float2 oi_pre = make_float2(0.f, 0.f), oi_post = make_float2(0.f, 0.f);
    int cxs = 0, cys = 0;
    if constexpr (!F64) {
      oi_pre = ((const float2*)st.pos_pre)[s];
      oi_post = ((const float2*)st.pos_post)[s];
      split_cell(st.cell_post[s], g, cxs, cys);
    }
    for_neighbour_slots(g, st, st.cell_pre[s], [&](int j, int, int dcx, int dcy) {
      contact_candidate<F64>(p, g, st, L, s, j, dcx, dcy, rx, pmask, oi_pre, oi_post, cxs, cys,
                             [&](int c, int e, int sub) { S(st, c, e, sub); });
    });
  });
  flush_contacts(st, L, S, base);
}

// The per-sweeper work of the column-task contact search: sweeper s, its
// neighbour column dcx (-1, 0, 1); r0 is a replica at or before s's.
template <bool F64, typename Stage>
__device__ __forceinline__ void contact_column_task(const EdmDynParams* __restrict__ P, const DevState& st,
                                                    const CatLists& L, int64_t s, int dcx, int r0, Stage stage) {
  int r = r0;
  while (r + 1 < st.n_rep && st.rep_first[r + 1] <= s) ++r;
  const EdmDynParams& p = P[r];
  const Geo g(p);
  const int sps = fl_species(st.flags[s]);
  const uint32_t rx = L.sweep_rx[sps], pmask = L.sweep_partners[sps];
  float2 oi_pre = make_float2(0.f, 0.f), oi_post = make_float2(0.f, 0.f);
  int cxs = 0, cys = 0;
  if constexpr (!F64) {
    oi_pre = ((const float2*)st.pos_pre)[s];
    oi_post = ((const float2*)st.pos_post)[s];
    split_cell(st.cell_post[s], g, cxs, cys);
  }
  for_neighbour_slots_box(g, st, st.cell_pre[s], dcx, dcx, -1, 1, [&](int j, int, int dcx_, int dcy) {
    contact_candidate<F64>(p, g, st, L, s, j, dcx_, dcy, rx, pmask, oi_pre, oi_post, cxs, cys, stage);
  });
}

// The same contact search with the work spread over (sweeper, neighbour
// column) tasks: a warp compacts the sweepers of its kSweepChunk slots in
// shared memory (as sweep4 does), then each lane takes tasks t = lane,
// lane + 32, ... (sweeper t / 3, column t % 3 - 1) and walks that column's
// one or two slot runs.  A lane's loop is about three candidates instead of
// nine, so lanes idle less while the longest run finishes.  Same tests, same
// contact set (in another order, which the catalytic passes do not depend
// on).
template <bool F64, int MINB>
__global__ void __launch_bounds__(kBlock, MINB) k_contacts_cols(const EdmDynParams* __restrict__ P, DevState st,
                                                              Match m, CatLists L) {
  pdl_enter();
  __shared__ int2 buf[kContactSmem];
  __shared__ int nbuf[EDM_MAX_CAT], base[EDM_MAX_CAT];
  __shared__ int32_t list[kBlock / 32][kSweepChunk];
  const ContactStage S{buf, nbuf, L.n_cat > 0 ? kContactSmem / L.n_cat : kContactSmem};
  if (threadIdx.x < EDM_MAX_CAT) nbuf[threadIdx.x] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) * 4;
  int n = 0, r0 = 0;
  if (w0 < st.n_slots) {  // whole warps: compact the chunk's sweepers
    const int64_t s0 = w0 + (int64_t)lane * 4;
    uchar4 f4 = make_uchar4(0, 0, 0, 0);
    if (s0 < st.n_slots) f4 = *reinterpret_cast<const uchar4*>(st.flags + s0);
    const uint8_t fl[4] = {f4.x, f4.y, f4.z, f4.w};
    const unsigned below = (1u << lane) - 1u;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const bool hit = s0 + k < st.n_slots && matches(fl[k], m);
      const unsigned bits = __ballot_sync(0xffffffffu, hit);
      if (hit) list[wid][n + __popc(bits & below)] = (int32_t)(s0 + k);
      n += __popc(bits);
    }
    r0 = st.chunk_rep[w0 / kSweepChunk];
  }
  __syncwarp();
  for (int t = lane; t < 3 * n; t += 32) {
    const int q = t / 3;
    contact_column_task<F64>(P, st, L, list[wid][q], t - 3 * q - 1, r0,
                             [&](int c, int e, int sub) { S(st, c, e, sub); });
  }
  flush_contacts(st, L, S, base);
}

// Block compaction of the slots matching m among the block's kBlock * SPT
// slots from b0 (SPT per thread, in slot order per thread): writes them to
// list (kBlock * SPT entries of shared memory) and returns their number.
// Every thread of the block calls it.
template <int SPT>
__device__ __forceinline__ int block_compact(const DevState& st, const Match& m, int64_t b0, int32_t* list,
                                             int* woff) {
  static_assert(SPT == 4 || SPT == 16, "4 or 16 slots per thread");
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t s0 = b0 + (int64_t)threadIdx.x * SPT;
  uint8_t fl[SPT];
  if (s0 + SPT <= st.n_slots) {  // s0 and SPT are multiples of SPT bytes: aligned
    if constexpr (SPT == 16) {
      const uint4 v = *reinterpret_cast<const uint4*>(st.flags + s0);
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int k = 0; k < 16; ++k) fl[k] = (uint8_t)(w[k >> 2] >> (8 * (k & 3)));
    } else {
      const uchar4 f4 = *reinterpret_cast<const uchar4*>(st.flags + s0);
      fl[0] = f4.x, fl[1] = f4.y, fl[2] = f4.z, fl[3] = f4.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < SPT; ++k) fl[k] = s0 + k < st.n_slots ? st.flags[s0 + k] : (uint8_t)0;
  }
  unsigned hits = 0;  // bit k: slot s0 + k matches
#pragma unroll
  for (int k = 0; k < SPT; ++k)
    if (s0 + k < st.n_slots && matches(fl[k], m)) hits |= 1u << k;
  int wn = 0;
#pragma unroll
  for (int k = 0; k < SPT; ++k) wn += __popc(__ballot_sync(0xffffffffu, (hits >> k) & 1u));
  if (lane == 0) woff[wid + 1] = wn;
  __syncthreads();
  if (threadIdx.x == 0) {
    woff[0] = 0;
    for (int w = 1; w <= kBlock / 32; ++w) woff[w] += woff[w - 1];
  }
  __syncthreads();
  const unsigned below = (1u << lane) - 1u;
  int at = woff[wid];
#pragma unroll
  for (int k = 0; k < SPT; ++k) {
    const bool hit = (hits >> k) & 1u;
    const unsigned bits = __ballot_sync(0xffffffffu, hit);
    if (hit) list[at + __popc(bits & below)] = (int32_t)(s0 + k);
    at += __popc(bits);
  }
  __syncthreads();
  return woff[kBlock / 32];
}

// The contact search's sweepers as one global list: each block compacts its
// kBlock * 16 slots and appends them with one atomic (launch with
// ceil(n_slots / (16 kBlock)) blocks of kBlock).
__global__ void __launch_bounds__(kBlock) k_sweep_list(DevState st, Match m) {
  pdl_enter();
  __shared__ int32_t list[kBlock * 16];
  __shared__ int woff[kBlock / 32 + 1];
  __shared__ int at;
  const int n = block_compact<16>(st, m, (int64_t)blockIdx.x * kBlock * 16, list, woff);
  if (threadIdx.x == 0) at = n > 0 ? atomicAdd(st.sw_count, n) : 0;
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) st.sw_list[at + k] = list[k];
}

// The column tasks over the global sweeper list, one wave of blocks walking
// the tasks grid-stride: every lane has a task however the sweepers cluster.
template <bool F64, int MINB>
__global__ void __launch_bounds__(kBlock, MINB) k_contacts_list(const EdmDynParams* __restrict__ P, DevState st,
                                                              CatLists L) {
  pdl_enter();
  __shared__ int2 buf[kContactSmem];
  __shared__ int nbuf[EDM_MAX_CAT], base[EDM_MAX_CAT];
  const ContactStage S{buf, nbuf, L.n_cat > 0 ? kContactSmem / L.n_cat : kContactSmem};
  if (threadIdx.x < EDM_MAX_CAT) nbuf[threadIdx.x] = 0;
  __syncthreads();
  const int64_t tasks = 3 * (int64_t)*st.sw_count;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < tasks; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = t / 3;
    const int64_t s = st.sw_list[q];
    contact_column_task<F64>(P, st, L, s, (int)(t - 3 * q) - 1, st.chunk_rep[s / kSweepChunk],
                             [&](int c, int e, int sub) { S(st, c, e, sub); });
  }
  flush_contacts(st, L, S, base);
}

// The column tasks balanced over the whole block: the block compacts the
// sweepers of its kBlock * SPT slots (SPT per thread) into one shared list,
// so a warp whose slots hold a cluster of sweepers shares them with the
// block's other warps instead of keeping the block waiting.
template <bool F64, int MINB, int SPT>
__global__ void __launch_bounds__(kBlock, MINB) k_contacts_block(const EdmDynParams* __restrict__ P, DevState st,
                                                               Match m, CatLists L) {
  pdl_enter();
  __shared__ int2 buf[kContactSmem];
  __shared__ int nbuf[EDM_MAX_CAT], base[EDM_MAX_CAT];
  __shared__ int32_t list[kBlock * SPT];
  __shared__ int woff[kBlock / 32 + 1];
  const ContactStage S{buf, nbuf, L.n_cat > 0 ? kContactSmem / L.n_cat : kContactSmem};
  if (threadIdx.x < EDM_MAX_CAT) nbuf[threadIdx.x] = 0;
  const int64_t b0 = (int64_t)blockIdx.x * blockDim.x * SPT;
  const int n = block_compact<SPT>(st, m, b0, list, woff);  // its barriers also publish nbuf
  const int r0 = n > 0 ? st.chunk_rep[b0 / kSweepChunk] : 0;
  for (int t = threadIdx.x; t < 3 * n; t += blockDim.x) {
    const int q = t / 3;
    contact_column_task<F64>(P, st, L, list[q], t - 3 * q - 1, r0,
                             [&](int c, int e, int sub) { S(st, c, e, sub); });
  }
  flush_contacts(st, L, S, base);
}

// Late pairs of particle j, which a catalytic pass has just turned into the
// substrate of the later reactions `late`: its alive neighbours of those
// reactions' enzyme species passing the tests an enzyme-side sweep makes
// (j seen from enzyme e at the opposite cell offset, the same float32
// expressions), appended to the reactions' lists.
template <bool F64>
__device__ __forceinline__ void late_contacts(const EdmDynParams& p, const Geo& g, const DevState& st, int r,
                                           int64_t j, int id_j, int64_t step, uint32_t late) {
  uint32_t emask = 0;
  for (uint32_t b = late; b; b &= b - 1) emask |= 1u << p.cat[__ffs(b) - 1].enzyme;
  for_neighbour_slots(g, st, st.cell_pre[j], [&](int e, int, int dcx, int dcy) {
    if (e == j) return;
    const uint8_t fe = st.flags[e];
    const int spe = fl_species(fe);
    if (!fl_alive(fe) || !((emask >> spe) & 1u)) return;
    double d2;
    if constexpr (F64) {
      if (!(sep_sq<F64>(st.pos_pre, st.cell_pre, e, j, g) < g.cutoff_sq())) return;
      d2 = sep_sq<F64>(st.pos_post, st.cell_post, e, j, g);
    } else {
      const float2 oe = ((const float2*)st.pos_pre)[e], oj = ((const float2*)st.pos_pre)[j];
      const float fdx = __fmaf_rn(-(float)(-dcx), g.sxf, oe.x - oj.x);
      const float fdy = __fmaf_rn(-(float)(-dcy), g.syf, oe.y - oj.y);
      if (!((double)__fmaf_rn(fdx, fdx, fdy * fdy) < g.cutoff_sq())) return;
      d2 = sep_sq<F64>(st.pos_post, st.cell_post, e, j, g);
    }
    for (uint32_t b = late; b; b &= b - 1) {
      const int c = __ffs(b) - 1;
      if (spe != p.cat[c].enzyme || d2 > p.cat[c].contact_sq) continue;
      if (!cat_draw_passes(p, st, r, c, st.ids[e] - (int)g.poff, id_j, step)) continue;
      const int q = atomicAdd(&st.contact_count[c], 1);
      if (q < st.contact_cap) st.contacts[(int64_t)c * st.contact_cap + q] = make_int2(e, (int)j);
      else set_status(st.status, EDM_STATUS_CONTACT_CAP);
    }
  });
}

// Catalytic pass c (dynamics.py:825-983) over its contact list: the set of
// substrates with at least one accepted (enzyme, substrate) pair converts.
// Every listed pair is alive, has the pass's enzyme and is within its contact
// radius; only the partner's current species is left to test.
// `late`: the later reactions whose substrate is this pass's product.
template <bool F64>
__global__ void __launch_bounds__(kBlock, 4) k_catalytic(const EdmDynParams* __restrict__ P, DevState st, int cidx,
                                                       uint32_t late) {
  pdl_enter();
  const int n = st.contact_count[cidx];
  const int lim = (int64_t)n < st.contact_cap ? n : (int)st.contact_cap;
  const int2* list = st.contacts + (int64_t)cidx * st.contact_cap;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < lim; q += (int64_t)gridDim.x * blockDim.x) {
    const int2 es = list[q];
    const uint8_t fs = st.flags[es.y];
    int r = st.chunk_rep[es.x / kSweepChunk];
    while (r + 1 < st.n_rep && st.rep_first[r + 1] <= es.x) ++r;
    const EdmDynParams& p = P[r];
    const EdmCat& C = p.cat[cidx];
    if (!fl_alive(fs) || fl_species(fs) != C.substrate) continue;
    const Geo g(p);
    const int ide = st.ids[es.x] - (int)g.poff, ids = st.ids[es.y] - (int)g.poff;
    const uint32_t lo = ide < ids ? ide : ids, hi = ide < ids ? ids : ide;
    const uint64_t m = draw_u53(p.seed, *st.d_step, EDM_S_CAT + cidx, lo, hi);
    if (m >= st.cat_thr[(int64_t)r * EDM_MAX_CAT + cidx]) continue;
    const double u = __dmul_rn(__ull2double_rn(m), 0x1p-53);
    double xs, ys;
    abs_pos<F64>(st.pos_post, st.lo_post, st.cell_post, es.y, g, xs, ys);
    double peff = C.prob;
    if (C.rule >= 0) peff = C.prob * rule_factor(p, C.rule, st, xs, ys);
    if (C.rule >= 0 && ((p.adapt_cat_mask >> cidx) & 1)) peff = peff * adapt_factor(p, st.adapt_w, C.rule, xs, ys);
    if (u < peff) {
      if (cas_u8(&st.flags[es.y], fs, fl_make(C.product, true))) {
        atomic_add_i64(&st.counters[(int64_t)r * EDM_NCOUNTERS + EDM_C_CATALYTIC], 1);
        grid_change(p, st.grid_delta, C.substrate, true, C.product, true, xs, ys);
        if (late) late_contacts<F64>(p, g, st, r, es.y, ids, *st.d_step, late);
      }
    }
  }
}

// ---- per-particle passes: recruitment candidates, detachments, conversions ----
// Each decides for one particle from its flags, its keyed draw u, and (only
// when u is below the pass's threshold, pass_thr) its position and the grid
// counts.  One sweep before the first of these passes (k_pass_draws) draws,
// for every particle, the passes whose match holds its state; the few
// particles with some draw below its threshold go to a list, and the passes
// visit only that list.  A pass that changes a listed particle's state
// (detachment, conversion, recruitment) draws at once the later passes that
// match the new state.  A particle left off the list for a pass would be
// rejected by it, so skipping it changes nothing.
enum GroupPass : int8_t { kGroupRecruit = 0, kGroupDetach = 1, kGroupConvert = 2 };
struct DrawPlan {
  Match any;                           // states that some pass matches
  uint32_t reach[2][EDM_MAX_SPECIES];  // passes matching (alive, species), from the sweep on
  uint32_t after[kMaxPP];              // passes after pass k matching the state pass k leaves
  int8_t kind[kMaxPP];                 // GroupPass of each per-particle pass
  int8_t index[kMaxPP];                // its exchange or conversion
  int n;
};

__device__ __forceinline__ int pass_stream(int kind, int idx) {
  return kind == kGroupRecruit ? EDM_S_EX_ACCEPT + 4 * idx
                               : (kind == kGroupDetach ? EDM_S_EX_DETACH + 4 * idx : EDM_S_CONV + idx);
}

// Bits of the passes in `todo` whose keyed draw for local id `id` lies below
// the pass's threshold (the others reject the particle).
__device__ __forceinline__ uint32_t draw_passes(const DevState& st, const DrawPlan* __restrict__ D, uint64_t seed,
                                                int r, int id, int64_t step, uint32_t todo) {
  uint32_t bits = 0;
  for (; todo; todo &= todo - 1) {
    const int k = __ffs(todo) - 1;
    const uint64_t m = draw_u53(seed, step, pass_stream(D->kind[k], D->index[k]), (uint64_t)id, 0);
    if (m < st.pass_thr[(int64_t)r * kMaxPP + k]) bits |= 1u << k;
  }
  return bits;
}

__global__ void __launch_bounds__(kBlock, 8) k_pass_draws(const EdmDynParams* __restrict__ P, DevState st,
                                                       const DrawPlan* __restrict__ D, Match any) {
  pdl_enter();
  sweep4(st, any, [&](int r, int64_t s) {
    const uint8_t f = st.flags[s];
    const int sp = fl_species(f);
    const uint32_t todo = sp < EDM_MAX_SPECIES ? D->reach[fl_alive(f) ? 1 : 0][sp] : 0u;
    const int id = st.ids[s] - (int)P[r].particle_offset;
    const uint32_t bits = draw_passes(st, D, P[r].seed, r, id, *st.d_step, todo);
    if (bits) {
      const int q = atomicAdd(st.pl_count, 1);
      st.pl[q] = make_int4((int)s, (int)bits, r, id);
      st.pl_index[s] = q;
    }
  });
}

// Apply the first max_recruits accepted candidates in particle order.
// A recruited particle is alive from here on, so the passes after this one
// that match it (`after`) get its draws now, in its list entry (the entry
// exists: the particle was listed for this exchange's candidates).
template <bool F64>
__global__ void k_recruit_apply(const EdmDynParams* __restrict__ P, int n_rep, DevState st, int e,
                                const DrawPlan* __restrict__ D,
                                uint32_t after) {
  pdl_enter();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rep) return;
  const EdmDynParams& p = P[r];
  const EdmExch& X = p.exch[e];
  int n = st.rec_count[r];
  if (n > kRecCap) n = kRecCap;
  st.rec_count[r] = 0;
  if (n == 0) return;
  int32_t* ids = st.rec_id + (int64_t)r * kRecCap;
  double* xy = st.rec_xy + (int64_t)r * kRecCap * 2;
  for (int a = 1; a < n; ++a) {  // insertion sort by particle index
    const int id = ids[a];
    const double x = xy[2 * a], y = xy[2 * a + 1];
    int b = a - 1;
    while (b >= 0 && ids[b] > id) {
      ids[b + 1] = ids[b];
      xy[2 * (b + 1)] = xy[2 * b];
      xy[2 * (b + 1) + 1] = xy[2 * b + 1];
      --b;
    }
    ids[b + 1] = id;
    xy[2 * (b + 1)] = x;
    xy[2 * (b + 1) + 1] = y;
  }
  const Geo g(p);
  const int take = n < X.max_recruits ? n : X.max_recruits;
  for (int a = 0; a < take; ++a) {
    const int64_t slot = st.slot_of_id[g.poff + ids[a]];
    const double x = xy[2 * a], y = xy[2 * a + 1];
    const int cxn = cell_index(x, g.sx, g.nx), cyn = cell_index(y, g.sy, g.ny);
    const int newc = cxn * g.ny + cyn;
    if constexpr (F64) {
      ((double2*)st.pos_post)[slot] = make_double2(x, y);
    } else {
      float2 o;
      short2 l;
      split_offset(x - (double)cxn * g.sx, g.sxf, o.x, l.x);
      split_offset(y - (double)cyn * g.sy, g.syf, o.y, l.y);
      ((float2*)st.pos_post)[slot] = o;
      st.lo_post[slot] = l;
    }
    st.cell_post[slot] = newc;
    rebucket(st, g, g.grave, newc);
    st.flags[slot] = fl_make(X.species, true);
    note_moved(st, r, p, slot);
    grid_add(p, st.grid_delta, X.species, x, y, 1);
    if (after) {
      const uint32_t bits = draw_passes(st, D, p.seed, r, ids[a], *st.d_step, after);
      const int q = st.pl_index[slot];
      if (q >= 0 && q < *st.pl_count && st.pl[q].x == (int)slot) st.pl[q].y |= (int)bits;
      else set_status(st.status, EDM_STATUS_RECRUIT_CAP);  // cannot happen: see above
    }
  }
  atomic_add_i64(&st.counters[(int64_t)r * EDM_NCOUNTERS + EDM_C_RECRUITED], take);
}

// Recruitment candidate of exchange e (dynamics.py:1229-1458): a dormant
// particle of the species whose keyed draw accepts at the keyed position.
// The per-particle passes below run on listed particles only.
__device__ __forceinline__ void recruit_candidate(const EdmDynParams& p, const DevState& st, int r, int id, int e) {
  const EdmExch& X = p.exch[e];
  const int64_t step = *st.d_step;
  const double ua = uniform1(p.seed, step, EDM_S_EX_ACCEPT + 4 * e, (uint64_t)id, 0);
  double cx, cy;
  if (X.local_recruit) {  // density-biased position (dynamics.py:1115-1217)
    const EdmGrid& G = p.grid[p.rule[X.rule_on].grid];
    const double rl = uniform1(p.seed, step, EDM_S_EX_LOC + 4 * e, (uint64_t)id, 0);
    const U2 off = normal2(p.seed, step, EDM_S_EX_OFFSET + e, (uint64_t)id);
    const double* cdf = st.local_cdf + G.offset;
    int lo = 0, hi = G.nx * G.ny - 1;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (cdf[mid] < rl) lo = mid + 1;
      else hi = mid;
    }
    const int gx = lo / G.ny, gy = lo - gx * G.ny;
    cx = py_fmod(__dadd_rn(__dmul_rn(__dadd_rn((double)gx, 0.5), G.sx), __dmul_rn(off.u0, p.recruit_sigma)), p.Lx);
    cy = py_fmod(__dadd_rn(__dmul_rn(__dadd_rn((double)gy, 0.5), G.sy), __dmul_rn(off.u1, p.recruit_sigma)), p.Ly);
  } else {
    const U2 up = uniform2(p.seed, step, EDM_S_EX_POS + 4 * e, (uint64_t)id, 0);
    cx = up.u0 * p.Lx;
    cy = up.u1 * p.Ly;
  }
  double peff = X.prob_on;
  if (X.rule_on >= 0 && X.rule_on2 >= 0) {
    peff = X.prob_on * rule_factor(p, X.rule_on, st, cx, cy) * rule_factor(p, X.rule_on2, st, cx, cy);
  } else if (X.rule_on >= 0) {
    peff = X.prob_on * rule_factor(p, X.rule_on, st, cx, cy);
  }
  if (ua < peff) {
    const int k = atomicAdd(&st.rec_count[r], 1);
    if (k < kRecCap) {
      st.rec_id[(int64_t)r * kRecCap + k] = id;
      st.rec_xy[((int64_t)r * kRecCap + k) * 2] = cx;
      st.rec_xy[((int64_t)r * kRecCap + k) * 2 + 1] = cy;
    } else {
      set_status(st.status, EDM_STATUS_RECRUIT_CAP);
    }
  }
}

// Position of slot s after the move, fetched once for the passes that need it.
template <bool F64>
struct LazyPos {
  bool have = false;
  double x = 0.0, y = 0.0;
  __device__ __forceinline__ void get(const DevState& st, int64_t s, const Geo& g) {
    if (!have) abs_pos<F64>(st.pos_post, st.lo_post, st.cell_post, s, g, x, y);
    have = true;
  }
};

// Detachment of exchange e (dynamics.py:1461-1555) of the alive particle in
// slot s; returns its flags afterwards.
template <bool F64>
__device__ __forceinline__ uint8_t detach_one(const EdmDynParams& p, const Geo& g, const DevState& st, int r,
                                              int64_t s, int id, LazyPos<F64>& pos, int e, uint8_t f) {
  const EdmExch& X = p.exch[e];
  const double u = uniform1(p.seed, *st.d_step, EDM_S_EX_DETACH + 4 * e, (uint64_t)id, 0);
  pos.get(st, s, g);
  double peff = X.prob_off;
  if (X.rule_off >= 0) peff = X.prob_off * rule_factor(p, X.rule_off, st, pos.x, pos.y);
  if (u < peff) {
    f = fl_make(X.species, false);
    st.flags[s] = f;
    rebucket(st, g, st.cell_post[s], g.grave);
    atomic_add_i64(&st.counters[(int64_t)r * EDM_NCOUNTERS + EDM_C_DETACHED], 1);
    grid_add(p, st.grid_delta, X.species, pos.x, pos.y, -1);
  }
  return f;
}

// Unimolecular conversion v (dynamics.py:1565-1657) of the alive particle in
// slot s; returns its flags afterwards.
template <bool F64>
__device__ __forceinline__ uint8_t convert_one(const EdmDynParams& p, const Geo& g, const DevState& st, int r,
                                               int64_t s, int id, LazyPos<F64>& pos, int v, uint8_t f) {
  const EdmConv& V = p.conv[v];
  const double u = uniform1(p.seed, *st.d_step, EDM_S_CONV + v, (uint64_t)id, 0);
  pos.get(st, s, g);
  double peff = V.prob;
  if (V.rule >= 0) peff = V.prob * rule_factor(p, V.rule, st, pos.x, pos.y);
  if (u < peff) {
    f = fl_make(V.to, true);
    st.flags[s] = f;
    atomic_add_i64(&st.counters[(int64_t)r * EDM_NCOUNTERS + EDM_C_CONVERTED], 1);
    grid_change(p, st.grid_delta, V.from, true, V.to, true, pos.x, pos.y);
  }
  return f;
}

// A run of consecutive per-particle passes over the listed particles.  Each
// of these passes decides for a particle from its own flags, position and
// keyed draws and from the grid counts, which no pass of the run changes
// (their grid changes go to the delta grid), and a particle's flags change
// only in its own passes.  So taking every listed particle through the run's
// passes in order gives the result of the passes one after another.
constexpr int kMaxGroup = 16;
struct PassGroup {
  Match m[kMaxGroup];      // particles each pass visits
  int8_t kind[kMaxGroup];  // GroupPass
  int8_t index[kMaxGroup]; // exchange or conversion index
  int8_t pp[kMaxGroup];    // the pass's bit in the list entries
  uint32_t bits;           // union of the passes' bits
  int n;
};

template <bool F64>
__global__ void __launch_bounds__(kBlock) k_particle_passes(const EdmDynParams* __restrict__ P, DevState st,
                                                            const PassGroup* __restrict__ G,
                                                            const DrawPlan* __restrict__ D) {
  pdl_enter();
  const PassGroup& sg = *G;
  const int n = *st.pl_count;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int4 e = st.pl[q];
    uint32_t bits = (uint32_t)e.y;
    if (!(bits & sg.bits)) continue;
    const int64_t s = e.x;
    const int r = e.z, id = e.w;
    const EdmDynParams& p = P[r];
    const Geo g(p);
    uint8_t f = st.flags[s];
    const uint32_t bits0 = bits;
    LazyPos<F64> pos;  // these passes move no particle
    for (int k = 0; k < sg.n; ++k) {
      const int pk = sg.pp[k];
      if (!((bits >> pk) & 1u) || !matches(f, sg.m[k])) continue;
      const int kind = sg.kind[k], idx = sg.index[k];
      if (kind == kGroupRecruit) {
        recruit_candidate(p, st, r, id, idx);
        continue;
      }
      const uint8_t f0 = f;
      f = kind == kGroupDetach ? detach_one<F64>(p, g, st, r, s, id, pos, idx, f)
                               : convert_one<F64>(p, g, st, r, s, id, pos, idx, f);
      if (f != f0) bits |= draw_passes(st, D, p.seed, r, id, *st.d_step, D->after[pk] & ~bits);
    }
    if (bits != bits0) st.pl[q].y = (int)bits;
  }
}

// Binding candidates of reaction b (dynamics.py:528-606): pairs (i < j)
// passing every test of the pass-start state, keyed by the reference's pair
// order (i, neighbour-cell ordinal, descending j).
template <bool F64>
__global__ void __launch_bounds__(kBlock) k_bind_candidates(const EdmDynParams* __restrict__ P, DevState st,
                                                            Match m, int b) {
  pdl_enter();
  sweep4(st, m, [&](int r, int64_t s) {
    const EdmDynParams& p = P[r];
    const EdmBind& B = p.bind[b];
    const int spi = fl_species(st.flags[s]);
    const Geo g(p);
    const int id = st.ids[s] - (int)g.poff;
    if (st.bond[g.poff + id] >= 0) return;
    const int64_t step = *st.d_step;
    for_neighbour_slots(g, st, st.cell_pre[s], [&](int j, int ordinal, int, int) {
      {
        const int idj = st.ids[j] - (int)g.poff;
        if (idj <= id) return;
        const uint8_t fj = st.flags[j];
        if (!fl_alive(fj)) return;
        if (st.bond[g.poff + idj] >= 0) return;
        const int spj = fl_species(fj);
        int a, bb;
        if (spi == B.ra && spj == B.rb) {
          a = id;
          bb = idj;
        } else if (spi == B.rb && spj == B.ra) {
          a = idj;
          bb = id;
        } else {
          return;
        }
        if (!(sep_sq<F64>(st.pos_pre, st.cell_pre, s, j, g) < g.cutoff_sq())) return;
        if (sep_sq<F64>(st.pos_post, st.cell_post, s, j, g) > B.contact_sq) return;
        const double u = uniform1(p.seed, step, EDM_S_BIND + 2 * b, (uint64_t)id, (uint64_t)idj);
        if (!(u < B.prob_bind)) return;
        const int k = atomicAdd(&st.bind_count[r], 1);
        if (k < kBindCap) {
          st.bind_key[(int64_t)r * kBindCap + k] =
              ((int64_t)id << 36) | ((int64_t)ordinal << 32) | (int64_t)(0xFFFFFFFFu - (uint32_t)idj);
          st.bind_ab[((int64_t)r * kBindCap + k) * 2] = a;
          st.bind_ab[((int64_t)r * kBindCap + k) * 2 + 1] = bb;
        } else {
          set_status(st.status, EDM_STATUS_BIND_CAP);
        }
      }
    });
  });
}

// Sequential greedy application in pair order, re-checking the live state.
template <bool F64>
__global__ void k_bind_apply(const EdmDynParams* __restrict__ P, int n_rep, DevState st, int b) {
  pdl_enter();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rep) return;
  const EdmDynParams& p = P[r];
  const EdmBind& B = p.bind[b];
  int n = st.bind_count[r];
  if (n > kBindCap) n = kBindCap;
  st.bind_count[r] = 0;
  if (n == 0) return;
  int64_t* key = st.bind_key + (int64_t)r * kBindCap;
  int32_t* ab = st.bind_ab + (int64_t)r * kBindCap * 2;
  for (int i = 1; i < n; ++i) {
    const int64_t k = key[i];
    const int a = ab[2 * i], bb = ab[2 * i + 1];
    int j = i - 1;
    while (j >= 0 && key[j] > k) {
      key[j + 1] = key[j];
      ab[2 * (j + 1)] = ab[2 * j];
      ab[2 * (j + 1) + 1] = ab[2 * j + 1];
      --j;
    }
    key[j + 1] = k;
    ab[2 * (j + 1)] = a;
    ab[2 * (j + 1) + 1] = bb;
  }
  const Geo g(p);
  int64_t nb = 0;
  for (int i = 0; i < n; ++i) {
    const int a = ab[2 * i], bb = ab[2 * i + 1];
    const int64_t sa = st.slot_of_id[g.poff + a], sb = st.slot_of_id[g.poff + bb];
    const uint8_t fa = st.flags[sa], fb = st.flags[sb];
    if (!fl_alive(fa) || !fl_alive(fb)) continue;
    if (st.bond[g.poff + a] >= 0 || st.bond[g.poff + bb] >= 0) continue;
    if (fl_species(fa) != B.ra || fl_species(fb) != B.rb) continue;
    double xa, ya, xb, yb;
    abs_pos<F64>(st.pos_post, st.lo_post, st.cell_post, sa, g, xa, ya);
    abs_pos<F64>(st.pos_post, st.lo_post, st.cell_post, sb, g, xb, yb);
    st.flags[sa] = fl_make(B.product, true);
    st.flags[sb] = fl_make(B.rb, false);
    rebucket(st, g, st.cell_post[sb], g.grave);
    st.bond[g.poff + a] = (int32_t)(g.poff + bb);
    st.bond[g.poff + bb] = (int32_t)(g.poff + a);
    grid_change(p, st.grid_delta, B.ra, true, B.product, true, xa, ya);
    grid_change(p, st.grid_delta, B.rb, true, B.rb, false, xb, yb);
    ++nb;
  }
  atomic_add_i64(&st.counters[(int64_t)r * EDM_NCOUNTERS + EDM_C_BINDINGS], nb);
}

// Dissociation of reaction b (dynamics.py:609-654).
template <bool F64>
__global__ void __launch_bounds__(kBlock) k_dissociate(const EdmDynParams* __restrict__ P, DevState st, Match m,
                                                       int b) {
  pdl_enter();
  sweep4(st, m, [&](int r, int64_t s) {
    const EdmDynParams& p = P[r];
    const EdmBind& B = p.bind[b];
    const Geo g(p);
    const int id = st.ids[s] - (int)g.poff;
    const int partner = st.bond[g.poff + id];
    if (partner < 0) return;
    const double u = uniform1(p.seed, *st.d_step, EDM_S_DISSOC + 2 * b, (uint64_t)id, 0);
    if (!(u < B.prob_dissoc)) return;
    const int64_t sj = st.slot_of_id[partner];
    double x, y;
    abs_pos<F64>(st.pos_post, st.lo_post, st.cell_post, s, g, x, y);
    const uint8_t fj = st.flags[sj];
    st.flags[s] = fl_make(B.ra, true);
    st.flags[sj] = fl_make(B.rb, true);
    const int newc = st.cell_post[s];
    if constexpr (F64) {
      ((double2*)st.pos_post)[sj] = ((const double2*)st.pos_post)[s];
    } else {
      ((float2*)st.pos_post)[sj] = ((const float2*)st.pos_post)[s];
      st.lo_post[sj] = st.lo_post[s];
    }
    rebucket(st, g, fl_alive(fj) ? st.cell_post[sj] : g.grave, newc);
    st.cell_post[sj] = newc;
    note_moved(st, r, p, sj);
    st.bond[g.poff + id] = -1;
    st.bond[partner] = -1;
    grid_change(p, st.grid_delta, B.product, true, B.ra, true, x, y);
    grid_change(p, st.grid_delta, fl_species(fj), fl_alive(fj), B.rb, true, x, y);
    atomic_add_i64(&st.counters[(int64_t)r * EDM_NCOUNTERS + EDM_C_DISSOC], 1);
  });
}

// grid_cnt += grid_delta; grid_delta = 0
// Adaptation field update w += dt/tau_w (rho_PIP3 - w) on every cell of each
// replica's adaptation grid (dynamics.py:1093-1112, 2227-2242); block row =
// replica.
__global__ void k_adapt(const EdmDynParams* __restrict__ P, const int32_t* __restrict__ cnt,
                        double* __restrict__ w) {
  pdl_enter();
  const EdmDynParams& p = P[blockIdx.y];
  if (p.adapt_grid < 0) return;
  const EdmGrid& A = p.grid[p.adapt_grid];
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < A.nx * A.ny; c += gridDim.x * blockDim.x) {
    const int64_t i = A.offset + c;
    const double rho = kfold_density(cnt[i], p.adapt_inv_area);
    w[i] = __dadd_rn(w[i], __dmul_rn(p.adapt_inv_tau, __dadd_rn(rho, -w[i])));
  }
}

// Local-recruitment CDF of exchange e for each replica (block = replica):
// cumulative max(density, 0.01) over the feedback grid's cells in (gx, gy)
// order, sequentially as the reference sums it, then divided by the total
// (dynamics.py:2356-2371).
__global__ void k_local_cdf(const EdmDynParams* __restrict__ P, const int32_t* __restrict__ cnt,
                            double* __restrict__ cdf_all, int e) {
  pdl_enter();
  const EdmDynParams& p = P[blockIdx.x];
  const EdmExch& X = p.exch[e];
  if (!X.local_recruit || X.rule_on < 0) return;
  const EdmRule& R = p.rule[X.rule_on];
  const EdmGrid& G = p.grid[R.grid];
  const int n = G.nx * G.ny;
  double* cdf = cdf_all + G.offset;
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    const double rho = kfold_density(cnt[G.offset + c], R.inv_area);
    cdf[c] = rho > 0.01 ? rho : 0.01;
  }
  __syncthreads();
  __shared__ double total_s;
  if (threadIdx.x == 0) {
    double total = 0.0;
    for (int c = 0; c < n; ++c) {
      total = __dadd_rn(total, cdf[c]);
      cdf[c] = total;
    }
    total_s = total;
  }
  __syncthreads();
  const double total = total_s;
  for (int c = threadIdx.x; c < n; c += blockDim.x)
    cdf[c] = total > 0 ? __ddiv_rn(cdf[c], total) : __ddiv_rn((double)c + 1.0, (double)n);
}

__global__ void k_grid_merge(int32_t* __restrict__ cnt, int32_t* __restrict__ delta, int64_t n) {
  pdl_enter();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int d = delta[i];
    if (d) {
      cnt[i] += d;
      delta[i] = 0;
    }
  }
}

__global__ void k_step_inc(int64_t* step) {
  pdl_enter();
  *step += 1;
}

}  // namespace edm
