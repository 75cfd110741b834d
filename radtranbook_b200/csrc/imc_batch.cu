// imc_batch.cu — batched independent 1-D gray slab problems (imc_batch_* of
// include/imcb200.h): source fill, the persistent tracking kernel with one work queue over
// every instance's histories, the comb, and the C entry points.
//
// Layout.  Instance k owns cells [cell_off[k], cell_off[k+1]) of every per-cell array and
// bank slots [slot_off[k], slot_off[k+1]) of both banks.  Its live entries this step are
// its census followed by its new particles (left face | right face | emission), so the
// flattened index space "entry q of the batch" is instance-major: entry q belongs to the
// last k with live_pref[k] <= q.  Kernels that run over entries find k by a binary search
// of the (K+1)-entry prefix held in shared memory.
//
// Equivalence with the single-problem path.  Every per-particle computation (source
// sampling, event geometry, implicit capture, tallies, weight floor, comb copies) is the
// single-problem slab code with the instance's own Philox key and the entry's index inside
// its instance as the counter, so instance k reproduces an imc_step_transport / imc_comb
// run with seed[k] (IMC/IMC1D.py:75-200 events, 319-329 boundary, 203-291 emission,
// 770-828 comb).
#include <algorithm>
#include <cmath>
#include <cstring>
#include "imc_batch.h"
#include "imc_device.cuh"
#include "imc_sample.cuh"

using namespace imcdev;
using namespace imcsample;

namespace {

enum : int { B_CENSUS = 0, B_FLOOR, B_REFLECT, B_CAP, B_ESCAPE, B_N };

// last k with pref[k] <= q; for q < pref[K] this is the instance that owns entry q
// (instances without entries share their prefix value with the next one)
__device__ __forceinline__ int find_inst(const long long* pref, int K, long long q) {
  int lo = 0, hi = K - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pref[mid] <= q) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ void load_pref(long long* sh, const long long* pref, int K) {
  for (int q = threadIdx.x; q <= K; q += blockDim.x) sh[q] = pref[q];
  __syncthreads();
}

// ---------------------------------------------------------------- sources
// ic = 1: the initial census (tag IC, step 0, uniform in the cell, birth time 0).
__global__ void k_bfill(BatchArgs a, int ic) {
  extern __shared__ long long pref[];
  load_pref(pref, a.new_pref, a.K);
  const long long total = pref[a.K];
  const BatchBank B = a.bank[*a.sel];
  const uint32_t step = ic ? 0u : *a.step;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += stride) {
    const int k = find_inst(pref, a.K, q);
    const long long local = q - pref[k];
    const int cb = a.cell_off[k], nc = a.cell_off[k + 1] - cb;
    const double* e1 = a.edges + cb + k;
    const uint64_t seed = a.seed[k];
    const long long b = a.slot_off[k] + a.n_census[k] + local;
    const long long n0 = a.n_side[2 * k], n1 = a.n_side[2 * k + 1];
    if (local < n0 + n1) {
      // boundary particle (IMC/IMC1D.py:319-329): at the face, mu = +-sqrt(u), t ~ U(0, dt)
      const int side = local < n0 ? 0 : 1;
      const uint32_t kk = (uint32_t)(side == 0 ? local : local - n0);
      const U4 ra = draw(seed, kk, 0, step, TAG_BOUNDARY | (uint32_t)side);
      const U4 rb = draw(seed, kk, 1, step, TAG_BOUNDARY | (uint32_t)side);
      const double mu_n = sqrt(u01d(ra.z));
      const double t = u01d(rb.x) * a.dt;
      B.p1[b] = (float)(side == 0 ? e1[0] : e1[nc]);
      B.d1[b] = (float)(side == 0 ? mu_n : -mu_n);
      B.w[b] = a.w_side[2 * k + side];
      B.t[b] = (float)t;
      B.cell[b] = side == 0 ? 0 : nc - 1;
    } else {
      // emission / initial-census particle: cell from the instance's count prefix
      const long long m = local - (n0 + n1);
      const long long* off = a.emit_off + cb + k;
      int lo = 0, hi = nc;
      while (lo < hi) { const int mid = (lo + hi) >> 1; if (off[mid + 1] <= m) lo = mid + 1; else hi = mid; }
      const int c = lo;
      const uint32_t tag = ic ? TAG_IC : TAG_EMISSION;
      const U4 r = draw(seed, (uint32_t)m, 0, step, tag);
      const U4 s = draw(seed, (uint32_t)m, 1, step, tag);
      const double u0 = u01d(r.x), u2 = u01d(r.z), u3 = u01d(r.w);
      const double s0 = u01d(s.x);
      const double ea = e1[c], eb = e1[c + 1];
      double p1 = ea + (ic ? u0 * (eb - ea) : slab_linear(eb - ea, a.tilt[cb + c], a.T[cb + c], u0));
      p1 = fmin(fmax(p1, ea), eb);
      double d1, d2;
      iso_dir(G_SLAB, u2, u3, d1, d2);
      B.p1[b] = (float)p1;
      B.d1[b] = (float)d1;
      B.w[b] = a.emit_w[cb + c];
      B.t[b] = (float)(s0 * (ic ? 0.0 : a.dt));
      B.cell[b] = c;
    }
  }
}

// per-instance sum of the tracked entries' weights (the weight floor is 1e-10 * sum / n)
// wsum[k] = sum of instance k's live weights.  Block b sums the contiguous entries
// [b*per, (b+1)*per) (coalesced, block-strided by blockDim); each thread finds its entry's
// instance once and advances it as its index passes instance boundaries (the entry space is
// instance-major), adding its partial sum to wsum when it leaves an instance and, at the end,
// through one warp-aggregated add per instance.
__global__ void __launch_bounds__(256) k_bwsum(BatchArgs a) {
  extern __shared__ long long pref[];
  __shared__ WarpStage stages[8];
  load_pref(pref, a.live_pref, a.K);
  WarpStage* st = stages + (threadIdx.x >> 5);
  const BatchBank B = a.bank[*a.sel];
  const long long total = pref[a.K];
  const long long per = (total + gridDim.x - 1) / gridDim.x;
  const long long lo = min(total, per * (long long)blockIdx.x), hi = min(total, lo + per);
  int k = lo + threadIdx.x < hi ? find_inst(pref, a.K, lo + threadIdx.x) : 0;
  long long slot0 = a.slot_off[k] - pref[k];  // bank slot of entry q is slot0 + q within instance k
  double s = 0.0;
  for (long long q = lo + threadIdx.x; q < hi; q += blockDim.x) {
    if (q >= pref[k + 1]) {  // left instance k (k < K - 1 here: q < total = pref[K])
      if (s != 0.0) atomicAdd(a.wsum + k, s);
      s = 0.0;
      do { ++k; } while (q >= pref[k + 1]);
      slot0 = a.slot_off[k] - pref[k];
    }
    const float wf = B.w[slot0 + q];
    if (wf > 0.f) s += (double)wf;
  }
  warp_tally1(s != 0.0, k, s, a.wsum, st);
}

// ---------------------------------------------------------------- tracking
// The single-problem slab kernel's event loop (k_track<G_SLAB>) over every instance:
// persistent warps claim runs of the flattened entry index with guided atomic tickets; a
// lane that takes entry q looks up its instance once and keeps the instance's constants
// (cell and edge bases, cell count, reflect mask, weight floor, Philox key) in registers.
// refill_min: a warp refills its idle lanes once at least that many are idle (1 = at
// every event boundary, as the single-problem kernel), or when all are idle.
__global__ void __launch_bounds__(256) k_btrack(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ unsigned blk_cnt[B_N];
  WarpStage* stages = reinterpret_cast<WarpStage*>(smem);
  const int nwarps = blockDim.x >> 5;
  long long* pref = reinterpret_cast<long long*>(stages + nwarps);
  if (threadIdx.x < B_N) blk_cnt[threadIdx.x] = 0u;
  load_pref(pref, a.live_pref, a.K);

  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  WarpStage* st = stages + (threadIdx.x >> 5);
  const unsigned long long n = (unsigned long long)pref[a.K];
  const BatchBank B = a.bank[*a.sel];
  const uint32_t step = *a.step;
  const float dt = (float)a.dt;
  const float c_light = (float)C_LIGHT;
  const unsigned refill_min = (unsigned)max(1, min(32, a.refill_min));

  unsigned long long chunk_next = 0, chunk_end = 0;
  bool drained = false;

  bool has = false;
  long long pid = 0;
  uint32_t lid = 0, ev = 0;
  int k = 0, cb = 0, eb = 0, nc = 0, rmask = 0, ci = 0;
  uint64_t seed = 0;
  float wfloor = 0.f, x = 0.f, u = 0.f, w = 0.f, dcen = 0.f;
  double inv_q = 0.0;  // the instance's fixed-point energy quantum, inverted
  double acc_lost = 0.0, acc_wd = 0.0;
  unsigned s_bd = 0, s_sc = 0;
  // events of finished histories, summed per lane while they belong to one instance (a
  // warp's claims are contiguous runs of one instance's entries) and added to the
  // instance's ledger when the instance changes: one atomic per run, not per history
  unsigned long long ev_acc = 0ull;
  int ev_k = 0;

  for (;;) {
    unsigned need = __ballot_sync(FULL, !has);
    if ((unsigned)__popc(need) >= refill_min) {
      while (need && !drained) {
        if (chunk_next >= chunk_end) {
          unsigned long long base = 0, claim = 0;
          if (lane == 0) {
            const unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(a.queue);
            const unsigned long long left = cur < n ? n - cur : 0ull;
            const unsigned long long nw = (unsigned long long)gridDim.x * (blockDim.x >> 5);
            claim = min((unsigned long long)a.chunk, max(32ull, left / (2ull * nw)));
            base = atomicAdd(a.queue, claim);
          }
          base = __shfl_sync(FULL, base, 0);
          claim = __shfl_sync(FULL, claim, 0);
          if (base >= n) { drained = true; break; }
          chunk_next = base;
          chunk_end = min(base + claim, n);
        }
        const unsigned long long avail = chunk_end - chunk_next;
        const unsigned rank = __popc(need & lt_mask);
        if (!has && rank < avail) {
          const long long q = (long long)(chunk_next + rank);
          k = find_inst(pref, a.K, q);
          lid = (uint32_t)(q - pref[k]);
          pid = a.slot_off[k] + lid;
          w = B.w[pid];
          dcen = (dt - B.t[pid]) * c_light;
          if (w > 0.f && dcen > 0.f) {
            x = B.p1[pid]; u = B.d1[pid]; ci = B.cell[pid];
            cb = a.cell_off[k]; nc = a.cell_off[k + 1] - cb; eb = cb + k;
            rmask = a.reflect[k]; seed = a.seed[k];
            const long long nb = a.n_bank[k];
            const double W = a.wsum[k];
            wfloor = (float)(1e-10 * W / (double)(nb > 0 ? nb : 1));
            inv_q = fx_inv_quantum(W);
            ev = 0;
            has = true;
          }
        }
        chunk_next += min((unsigned long long)__popc(need), avail);
        need = __ballot_sync(FULL, !has);
      }
    }
    if (!__any_sync(FULL, has)) break;

    bool flush = false;
    int flush_cell = 0;
    double f_lost = 0.0, f_wd = 0.0;
    if (has) {
      const int cg = cb + ci;
      const float2 sq = __ldg(a.sass + cg);
      const float sa = sq.x, ss = sq.y;
      bool finished = false;
      if (ev >= (1u << 30)) {
        atomicAdd(&blk_cnt[B_CAP], 1u);
        atomicOr(a.flags, (int)IMC_FLAG_EVENT_CAP);
        finished = true;
      } else {
        const U4 r = draw(seed, lid, ev, step, TAG_TRANSPORT);
        ++ev;
        const float xl = __ldg(a.ef + eb + ci), xr = __ldg(a.ef + eb + ci + 1);
        const float L = xr - xl;
        const float sb = slab_face(x, u, xl, xr);
        float ds = BIGF;
        {
          const bool capped = ss * L > 10000.0f;
          const float sig = capped ? 10000.0f / L : (ss > 1e-10f ? ss : 0.f);
          if (sig > 0.f) {
            const float s_other = fminf(sb, dcen);
            const double t = (double)sig * (double)s_other;
            bool may = true;
            if (t < 0.01) {
              const double thr = 1.0 - t * (1.0 - t * (0.5 - t * (1.0 / 6.0)));
              may = u01d(r.x) > thr;
            }
            if (may) ds = capped ? neglog_u(r.x) * (L * 1e-4f) : __fdividef(neglog_u(r.x), ss);
          }
        }
        float d = sb;
        int evt = EV_BOUNDARY, cross = X_NONE;
        if (ds < d) { d = ds; evt = EV_SCATTER; }
        if (dcen < d) { d = dcen; evt = EV_CENSUS; }
        float xn = fmaf(u, d, x), un = u;
        if (evt == EV_BOUNDARY) { if (u > 0.f) { xn = xr; cross = X_IP; } else { xn = xl; cross = X_IM; } }
        else { if (evt == EV_SCATTER) un = fmaf(2.f, u01f(r.y), -1.f); xn = fminf(fmaxf(xn, xl), xr); }
        const float wn = w * __expf(-sa * d);
        acc_lost += (double)w - (double)wn;
        acc_wd += (double)(w * d);
        dcen -= d;
        if (evt == EV_BOUNDARY) ++s_bd; else if (evt == EV_SCATTER) ++s_sc;
        else atomicAdd(&blk_cnt[B_CENSUS], 1u);
        w = wn; x = xn; u = un;
        if (cross != X_NONE) {
          flush = true; flush_cell = cg; f_lost = acc_lost; f_wd = acc_wd;
          acc_lost = 0.0; acc_wd = 0.0;
          int ni = cross == X_IP ? ci + 1 : ci - 1;
          const int side = ni < 0 ? 0 : (ni >= nc ? 1 : -1);
          if (side >= 0) {
            if ((rmask >> side) & 1) {
              u = -u;
              ni = side == 0 ? 0 : nc - 1;
              atomicAdd(&blk_cnt[B_REFLECT], 1u);
            } else {
              atomicAdd(a.esc_fx + 2 * k + side, fx_units((double)w, inv_q));
              atomicAdd(&blk_cnt[B_ESCAPE], 1u);
              w = 0.f;
              finished = true;
              ni = ci;
            }
          }
          ci = ni;
        }
        if (!finished && w < wfloor) {
          // IMC/IMC1D.py:188-195: kill and deposit the remainder in the current cell
          atomicAdd(&blk_cnt[B_FLOOR], 1u);
          atomicAdd(a.dep_fx + cb + ci, fx_units((double)w, inv_q));  // its intensity follows from it
          w = 0.f;
          finished = true;
        }
        if (!finished && !(dcen > 0.f)) finished = true;
      }
      if (finished) {
        if (!flush && (acc_lost != 0.0 || acc_wd != 0.0)) {
          flush = true; flush_cell = cb + ci; f_lost = acc_lost; f_wd = acc_wd;
        }
        acc_lost = 0.0; acc_wd = 0.0;
        B.w[pid] = w;
        if (w > 0.f) { B.p1[pid] = x; B.d1[pid] = u; B.cell[pid] = ci; }
        if (k != ev_k) {
          if (ev_acc) atomicAdd(a.ledger + (size_t)ev_k * IMC_BL_N + IMC_BL_EVENTS, (double)ev_acc);
          ev_k = k;
          ev_acc = 0ull;
        }
        ev_acc += ev;
        has = false;
      }
    }
    unsigned long long ud = 0ull;
    double vs = 0.0;
    if (flush) {
      const double2 cf = __ldg(a.cellf + flush_cell);
      ud = fx_units(f_lost, inv_q);  // lanes of one cell share its instance's quantum
      vs = cf.y > 0.0 ? 0.0 : f_wd;  // raw w*s of a cell without absorption (the rest follows from ud)
    }
    warp_tally_fx(flush, flush_cell, ud, vs, a.dep_fx, a.si, st);
  }

  if (ev_acc) atomicAdd(a.ledger + (size_t)ev_k * IMC_BL_N + IMC_BL_EVENTS, (double)ev_acc);
  const unsigned long long t_bd = warp_sum_u(s_bd), t_sc = warp_sum_u(s_sc);
  if (lane == 0) {
    if (t_bd) atomicAdd(a.stats + S_BOUNDARY, t_bd);
    if (t_sc) atomicAdd(a.stats + S_SCATTER, t_sc);
    if (t_bd + t_sc) atomicAdd(a.stats + S_EVENTS, t_bd + t_sc);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned long long cen = blk_cnt[B_CENSUS], cap = blk_cnt[B_CAP];
    if (cen) atomicAdd(a.stats + S_CENSUS, cen);
    if (cen + cap) atomicAdd(a.stats + S_EVENTS, cen + cap);
    if (blk_cnt[B_FLOOR]) atomicAdd(a.stats + S_FLOOR, (unsigned long long)blk_cnt[B_FLOOR]);
    if (blk_cnt[B_REFLECT]) atomicAdd(a.stats + S_REFLECT, (unsigned long long)blk_cnt[B_REFLECT]);
    if (cap) atomicAdd(a.stats + S_CAP, cap);
    if (blk_cnt[B_ESCAPE]) atomicAdd(a.stats + S_ESCAPE, (unsigned long long)blk_cnt[B_ESCAPE]);
  }
}

// Work-unit form of the tracking, for batches whose largest instance has at most
// IMC_BATCH_SMEM_CELLS cells.  A block claims a unit of chunk x (warps per block) consecutive
// entries of the batch (instance-major: one instance, or the end of one and the start of the
// next) and tracks it instance by instance with all its warps, each warp refilling idle lanes
// from a shared-memory cursor.  For the instance at hand the block keeps the cell table
// (sigma_a, sigma_s), the edges and the intensity factor in shared memory and sums the
// deposition (fixed point) and intensity tallies there, adding them to the instance's global
// tallies when it moves to another instance: the single-problem kernel's on-chip tables, which
// the entry-granular queue of k_btrack cannot keep because its warps draw entries of any
// instance.  Per history the computation is k_btrack's (same Philox counters and arithmetic).
// Five resident 256-thread blocks per SM (48 registers, 20 bytes of spills): 55.5 G segments/s on
// the 256-instance uneven batch against 53.9 G at four blocks (57 registers).
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v += __shfl_down_sync(FULL, v, o);
  return v;
}

__host__ __device__ inline size_t units_smem(int K, int M) {
  return sizeof(long long) * (size_t)(K + 1) + (size_t)M * (8 + 8 + 8 + 8) + sizeof(float) * (size_t)(M + 1);
}

// Prefetched refills (form 3): every lane holds the bank record of its next history in a
// shared-memory slot, copied there by cp.async while it tracks the current one, so a lane whose
// history ends takes its next one from shared memory instead of stalling the warp on two
// dependent HBM reads (weight and birth time, then position, direction and cell).
constexpr int PF_FIELDS = 6;  // w, t, x, u, cell, entry index inside the instance
__host__ __device__ inline size_t units_pf_smem(int block) { return sizeof(float) * PF_FIELDS * (size_t)block; }

template <bool PF>
__global__ void __launch_bounds__(256, 5) k_btrack_units(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ unsigned blk_cnt[B_N];
  __shared__ unsigned long long s_base, s_cur, s_unit;
  __shared__ __align__(16) uint32_t s_rk[20];  // Philox round keys of the staged instance's seed
  const int M = a.max_cells;
  long long* pref = reinterpret_cast<long long*>(smem);                                 // [K+1]
  unsigned long long* TD = reinterpret_cast<unsigned long long*>(pref + (a.K + 1));    // [M] deposition
  double* TS = reinterpret_cast<double*>(TD + M);                                       // [M] intensity
  double* CF = TS + M;                                                                  // [M] cellf.y
  float2* SS = reinterpret_cast<float2*>(CF + M);                                       // [M] (sa, ss)
  float* EF = reinterpret_cast<float*>(SS + M);                                         // [M+1] edges
  // PF: the lane's next bank record, field f of thread i at PQ[f * blockDim.x + i]
  float* PQ = reinterpret_cast<float*>(smem + units_smem(a.K, M));
  float* const my_pf = PQ + threadIdx.x;
  const int pf_stride = blockDim.x;
  if (threadIdx.x < B_N) blk_cnt[threadIdx.x] = 0u;
  load_pref(pref, a.live_pref, a.K);

  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  const unsigned long long n = (unsigned long long)pref[a.K];
  const BatchBank B = a.bank[*a.sel];
  const uint32_t step = *a.step;
  const float dt = (float)a.dt;
  const float c_light = (float)C_LIGHT;
  const unsigned long long unit = (unsigned long long)max(a.chunk, 32) * (blockDim.x >> 5);
  unsigned s_bd = 0, s_sc = 0;
  int cur_k = -1, cur_nc = 0, cur_cb = 0;  // block-uniform: the instance whose tallies are staged

  for (;;) {
    if (threadIdx.x == 0) {
      // full units while at least one per block is left; after that the rest shared over the
      // blocks (a multiple of 32, at least one row per warp), so the blocks finish together
      // instead of the last full units running on a few SMs
      unsigned long long u = unit;
      const unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(a.queue);
      const unsigned long long left = cur < n ? n - cur : 0ull;
      const unsigned long long nb = gridDim.x;
      if (left < nb * unit) {
        const unsigned long long floor_u = 32ull * (blockDim.x >> 5);
        u = min(unit, max(floor_u, (left / nb + 31ull) & ~31ull));
      }
      s_unit = u;
      s_base = atomicAdd(a.queue, u);
    }
    __syncthreads();
    const unsigned long long base = s_base;
    if (base >= n) break;  // uniform: every thread read the same claim
    const unsigned long long end = min(base + s_unit, n);
    for (unsigned long long q0 = base; q0 < end;) {
      const int k = find_inst(pref, a.K, (long long)q0);
      const unsigned long long q1 = min(end, (unsigned long long)pref[k + 1]);
      if (k != cur_k) {
        // the staged tallies to the previous instance, then this instance's tables
        for (int c = threadIdx.x; c < cur_nc; c += blockDim.x) {
          if (TD[c]) atomicAdd(a.dep_fx + cur_cb + c, TD[c]);
          if (TS[c] != 0.0) atomicAdd(a.si + cur_cb + c, TS[c]);
        }
        __syncthreads();
        cur_k = k; cur_cb = a.cell_off[k]; cur_nc = a.cell_off[k + 1] - cur_cb;
        for (int c = threadIdx.x; c < cur_nc; c += blockDim.x) {
          TD[c] = 0ull; TS[c] = 0.0;
          CF[c] = a.cellf[cur_cb + c].y;
          SS[c] = a.sass[cur_cb + c];
        }
        for (int c = threadIdx.x; c <= cur_nc; c += blockDim.x) EF[c] = a.ef[cur_cb + k + c];
        if (threadIdx.x == 0) philox_round_keys(a.seed[k], s_rk);
      }
      if (threadIdx.x == 0) s_cur = q0;
      __syncthreads();
      // the instance's constants (block-uniform)
      const int nc = cur_nc;
      const int rmask = a.reflect[k];
      const long long nbk = a.n_bank[k];
      const double W = a.wsum[k];
      const float wfloor = (float)(1e-10 * W / (double)(nbk > 0 ? nbk : 1));
      const double inv_q = fx_inv_quantum(W);
      const long long pk = pref[k], so = a.slot_off[k];
      unsigned long long ev_acc = 0ull;
      bool has = false, drained = false;
      bool pv = false;  // PF: the lane's slot holds a claimed record (copy issued)
      long long pid = 0;
      uint32_t lid = 0, ev = 0;
      int ci = 0;
      float x = 0.f, u = 0.f, w = 0.f, dcen = 0.f;
      float w_in = 0.f;     // weight at the start of the current cell visit
      double acc_wd = 0.0;  // w*s in the current cell (cells without absorption only)
      for (;;) {
        // ---- refill idle lanes from the block's cursor over [q0, q1) ----
        if (PF) {
          // An idle lane takes the record in its slot; every lane without a claimed record
          // claims the next entry of the unit (one shared atomic per warp) and starts its copy.
          // Leaves with every lane either tracking or holding no claim; at the unit's end the
          // cursor is past q1 and no claim is left untaken.
          for (;;) {
            if (!has && pv) {
              cp_async_wait_all();
              pv = false;
              lid = __float_as_uint(my_pf[5 * pf_stride]);
              pid = so + lid;
              w = my_pf[0];
              dcen = (dt - my_pf[pf_stride]) * c_light;
              if (w > 0.f && dcen > 0.f) {
                x = my_pf[2 * pf_stride]; u = my_pf[3 * pf_stride]; ci = __float_as_int(my_pf[4 * pf_stride]);
                ev = 0;
                w_in = w;
                has = true;
              }
            }
            if (!drained) {
              const unsigned pneed = __ballot_sync(FULL, !pv);
              if (pneed) {
                unsigned long long b0 = 0;
                if (lane == 0) b0 = atomicAdd(&s_cur, (unsigned long long)__popc(pneed));
                b0 = __shfl_sync(FULL, b0, 0);
                if (b0 >= q1) {
                  drained = true;
                } else {
                  const unsigned rank = __popc(pneed & lt_mask);
                  if (!pv && b0 + rank < q1) {
                    const uint32_t nl = (uint32_t)((long long)(b0 + rank) - pk);
                    const long long np = so + nl;
                    my_pf[5 * pf_stride] = __uint_as_float(nl);
                    cp_async4(my_pf, B.w + np);
                    cp_async4(my_pf + pf_stride, B.t + np);
                    cp_async4(my_pf + 2 * pf_stride, B.p1 + np);
                    cp_async4(my_pf + 3 * pf_stride, B.d1 + np);
                    cp_async4(my_pf + 4 * pf_stride, B.cell + np);
                    cp_async_commit();
                    pv = true;
                  }
                }
              }
            }
            if (!__any_sync(FULL, !has && pv)) break;
          }
          if (!__any_sync(FULL, has)) break;
        }
        unsigned need = PF ? 0u : __ballot_sync(FULL, !has);
        while (need && !drained) {
          unsigned long long b0 = 0;
          if (lane == 0) b0 = atomicAdd(&s_cur, (unsigned long long)__popc(need));
          b0 = __shfl_sync(FULL, b0, 0);
          if (b0 >= q1) { drained = true; break; }
          const unsigned rank = __popc(need & lt_mask);
          if (!has && b0 + rank < q1) {
            lid = (uint32_t)((long long)(b0 + rank) - pk);
            pid = so + lid;
            w = B.w[pid];
            dcen = (dt - B.t[pid]) * c_light;
            if (w > 0.f && dcen > 0.f) {
              x = B.p1[pid]; u = B.d1[pid]; ci = B.cell[pid];
              ev = 0;
              w_in = w;
              has = true;
            }
          }
          need = __ballot_sync(FULL, !has);
        }
        if (!__any_sync(FULL, has)) break;
        bool flush = false;
        int flush_cell = 0;
        double f_lost = 0.0, f_wd = 0.0;
        if (has) {
          const float2 sq = SS[ci];
          const float sa = sq.x, ss = sq.y;
          bool finished = false;
          if (ev >= (1u << 30)) {
            atomicAdd(&blk_cnt[B_CAP], 1u);
            atomicOr(a.flags, (int)IMC_FLAG_EVENT_CAP);
            finished = true;
          } else {
            const U4 r = draw_rk4(reinterpret_cast<const uint4*>(s_rk), lid, ev, step, TAG_TRANSPORT);
            ++ev;
            const float xl = EF[ci], xr = EF[ci + 1];
            const float L = xr - xl;
            const float sb = slab_face(x, u, xl, xr);
            float ds = BIGF;
            {
              const bool capped = ss * L > 10000.0f;
              const float sig = capped ? 10000.0f / L : (ss > 1e-10f ? ss : 0.f);
              if (sig > 0.f) {
                const float s_other = fminf(sb, dcen);
                const double t = (double)sig * (double)s_other;
                bool may = true;
                if (t < 0.01) {
                  const double thr = 1.0 - t * (1.0 - t * (0.5 - t * (1.0 / 6.0)));
                  may = u01d(r.x) > thr;
                }
                if (may) ds = capped ? neglog_u(r.x) * (L * 1e-4f) : __fdividef(neglog_u(r.x), ss);
              }
            }
            float d = sb;
            int evt = EV_BOUNDARY, cross = X_NONE;
            if (ds < d) { d = ds; evt = EV_SCATTER; }
            if (dcen < d) { d = dcen; evt = EV_CENSUS; }
            float xn = fmaf(u, d, x), un = u;
            if (evt == EV_BOUNDARY) { if (u > 0.f) { xn = xr; cross = X_IP; } else { xn = xl; cross = X_IM; } }
            else { if (evt == EV_SCATTER) un = fmaf(2.f, u01f(r.y), -1.f); xn = fminf(fmaxf(xn, xl), xr); }
            // implicit capture: the energy removed in a visit is counted at its flush, w_in - w
            const float wn = w * __expf(-sa * d);
            if (CF[ci] <= 0.0) acc_wd += (double)(w * d);
            dcen -= d;
            if (evt == EV_BOUNDARY) ++s_bd; else if (evt == EV_SCATTER) ++s_sc;
            else atomicAdd(&blk_cnt[B_CENSUS], 1u);
            w = wn; x = xn; u = un;
            if (cross != X_NONE) {
              flush = true; flush_cell = ci; f_lost = (double)w_in - (double)w; f_wd = acc_wd;
              w_in = w; acc_wd = 0.0;
              int ni = cross == X_IP ? ci + 1 : ci - 1;
              const int side = ni < 0 ? 0 : (ni >= nc ? 1 : -1);
              if (side >= 0) {
                if ((rmask >> side) & 1) {
                  u = -u;
                  ni = side == 0 ? 0 : nc - 1;
                  atomicAdd(&blk_cnt[B_REFLECT], 1u);
                } else {
                  atomicAdd(a.esc_fx + 2 * k + side, fx_units((double)w, inv_q));
                  atomicAdd(&blk_cnt[B_ESCAPE], 1u);
                  w = 0.f;
                  finished = true;
                  ni = ci;
                }
              }
              ci = ni;
            }
            if (!finished && w < wfloor) {
              // IMC/IMC1D.py:188-195: kill and deposit the remainder in the current cell.
              // Without a crossing in this event the visit's flush at the history end (w_in - 0)
              // carries it; after one, the old cell holds the flush slot and the remainder goes
              // to the new cell here (its intensity follows from the deposition)
              atomicAdd(&blk_cnt[B_FLOOR], 1u);
              if (flush) atomicAdd(TD + ci, fx_units((double)w, inv_q));
              w = 0.f;
              finished = true;
            }
            if (!finished && !(dcen > 0.f)) finished = true;
          }
          if (finished) {
            if (!flush) {  // the visit the history ends in
              const double lost = (double)w_in - (double)w;
              if (lost != 0.0 || acc_wd != 0.0) { flush = true; flush_cell = ci; f_lost = lost; f_wd = acc_wd; }
            }
            acc_wd = 0.0;
            B.w[pid] = w;
            if (w > 0.f) { B.p1[pid] = x; B.d1[pid] = u; B.cell[pid] = ci; }
            ev_acc += ev;
            has = false;
          }
        }
        if (flush) {
          // the cell visit's tallies into the block's staged ones (one shared atomic per lane):
          // deposition in fixed point, raw w*s only from a cell without absorption (an
          // absorbing cell's intensity follows from its deposition in the material update)
          const unsigned long long ud = fx_units(f_lost, inv_q);
          if (ud) atomicAdd(TD + flush_cell, ud);
          if (f_wd != 0.0) atomicAdd(TS + flush_cell, f_wd);
        }
      }
      // the unit's events of this instance to its ledger, one atomic per warp
      const unsigned long long t_ev = warp_sum_u64(ev_acc);
      if (lane == 0 && t_ev) atomicAdd(a.ledger + (size_t)k * IMC_BL_N + IMC_BL_EVENTS, (double)t_ev);
      __syncthreads();  // every warp is done with s_cur and the tables of this range
      q0 = q1;
    }
  }
  for (int c = threadIdx.x; c < cur_nc; c += blockDim.x) {
    if (TD[c]) atomicAdd(a.dep_fx + cur_cb + c, TD[c]);
    if (TS[c] != 0.0) atomicAdd(a.si + cur_cb + c, TS[c]);
  }
  const unsigned long long t_bd = warp_sum_u(s_bd), t_sc = warp_sum_u(s_sc);
  if (lane == 0) {
    if (t_bd) atomicAdd(a.stats + S_BOUNDARY, t_bd);
    if (t_sc) atomicAdd(a.stats + S_SCATTER, t_sc);
    if (t_bd + t_sc) atomicAdd(a.stats + S_EVENTS, t_bd + t_sc);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned long long cen = blk_cnt[B_CENSUS], cap = blk_cnt[B_CAP];
    if (cen) atomicAdd(a.stats + S_CENSUS, cen);
    if (cen + cap) atomicAdd(a.stats + S_EVENTS, cen + cap);
    if (blk_cnt[B_FLOOR]) atomicAdd(a.stats + S_FLOOR, (unsigned long long)blk_cnt[B_FLOOR]);
    if (blk_cnt[B_REFLECT]) atomicAdd(a.stats + S_REFLECT, (unsigned long long)blk_cnt[B_REFLECT]);
    if (cap) atomicAdd(a.stats + S_CAP, cap);
    if (blk_cnt[B_ESCAPE]) atomicAdd(a.stats + S_ESCAPE, (unsigned long long)blk_cnt[B_ESCAPE]);
  }
}

// ---------------------------------------------------------------- comb
// ecen[c] = sum of live weights per cell (all instances)
__global__ void __launch_bounds__(256) k_bcomb_ecen(BatchArgs a) {
  extern __shared__ long long pref[];
  __shared__ WarpStage stages[8];
  load_pref(pref, a.live_pref, a.K);
  WarpStage* st = stages + (threadIdx.x >> 5);
  const BatchBank B = a.bank[*a.sel];
  const long long total = pref[a.K];
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = (long long)blockIdx.x * blockDim.x; base < total; base += stride) {
    const long long q = base + threadIdx.x;
    bool live = false;
    int bin = 0;
    double w = 0.0;
    if (q < total) {
      const int k = find_inst(pref, a.K, q);
      const long long pid = a.slot_off[k] + (q - pref[k]);
      const float wf = B.w[pid];
      if (wf > 0.f) { live = true; bin = a.cell_off[k] + B.cell[pid]; w = (double)wf; }
    }
    warp_tally1(live, bin, w, a.ecen, st);
  }
}

// copies per entry n = floor(w / ew + xi), xi from Philox (entry index in its instance,
// 0, step, TAG_COMB); copies per cell, per instance and per tile of BATCH_TILE entries
__global__ void __launch_bounds__(BATCH_TILE) k_bcomb_count(BatchArgs a) {
  extern __shared__ long long pref[];
  __shared__ long long sh[BATCH_TILE / 32];
  __shared__ WarpStage stages[BATCH_TILE / 32];
  load_pref(pref, a.live_pref, a.K);
  WarpStage* st = stages + (threadIdx.x >> 5);
  const BatchBank B = a.bank[*a.sel];
  const uint32_t step = *a.step;
  const long long total = pref[a.K];
  const long long ntiles = (total + BATCH_TILE - 1) / BATCH_TILE;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long q = tile * BATCH_TILE + threadIdx.x;
    int n = 0, bin = 0, k = 0;
    if (q < total) {
      k = find_inst(pref, a.K, q);
      const long long lid = q - pref[k];
      const long long pid = a.slot_off[k] + lid;
      const float wf = B.w[pid];
      if (wf > 0.f) {
        bin = a.cell_off[k] + B.cell[pid];
        const double ew = a.ew[bin];
        if (ew > 0.0) {
          const U4 r = draw(a.seed[k], (uint32_t)(lid >> 2), 1, step, TAG_COMB);  // word lid % 4
          n = (int)floor((double)wf / ew + u01d(u4_word(r, (int)(lid & 3))));
        }
      }
      a.cnt[q] = n;
    }
    warp_tally1(n > 0, bin, (double)n, a.ncopy, st);
    warp_tally1(n > 0, k, (double)n, a.copies_d, st);
    const unsigned ws = __reduce_add_sync(FULL, (unsigned)n);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = ws;
    __syncthreads();
    if (threadIdx.x < 32) {
      unsigned long long v = sh[threadIdx.x];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
      if (threadIdx.x == 0) a.blk[tile] = (long long)v;
    }
    __syncthreads();
  }
}

// exclusive scans: tile totals (output position of each tile) and copies per instance;
// the new census of each instance, capped at what its slots hold next to a step's sources
__global__ void __launch_bounds__(1024) k_bcomb_scan(BatchArgs a) {
  __shared__ long long sh[1024];
  const int t = threadIdx.x;
  const long long total = a.live_pref[a.K];
  const long long nblk = (total + BATCH_TILE - 1) / BATCH_TILE;
  auto scan = [&](long long* x, long long m) {
    const long long per = (m + 1023) / 1024;
    const long long lo = min((long long)t * per, m), hi = min(lo + per, m);
    long long s = 0;
    for (long long q = lo; q < hi; ++q) s += x[q];
    sh[t] = s;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
      const long long v = t >= d ? sh[t - d] : 0;
      __syncthreads();
      sh[t] += v;
      __syncthreads();
    }
    long long run = sh[t] - s;
    for (long long q = lo; q < hi; ++q) { const long long v = x[q]; x[q] = run; run += v; }
    if (t == 1023) x[m] = sh[1023];
    __syncthreads();
  };
  scan(a.blk, nblk);
  for (int k = t; k < a.K; k += 1024) {
    const long long c = (long long)a.copies_d[k];
    a.inst_pref[k] = c;
    long long keep = c;
    if (c > a.census_cap[k]) { atomicOr(a.flags, (int)IMC_FLAG_COMB_OVERFLOW); keep = a.census_cap[k]; }
    a.n_census[k] = keep;
  }
  __syncthreads();
  scan(a.inst_pref, a.K);
}

// Copies written in entry order into the instance's slots of the other bank, one thread per
// output copy: the tile's copy counts are scanned in shared memory and each thread finds the
// entry of its copy by a binary search there, so the stores are contiguous across the warp
// however many copies a single entry makes (the census piles up in a few hot entries).
__global__ void __launch_bounds__(BATCH_TILE) k_bcomb_scatter(BatchArgs a) {
  extern __shared__ long long pref[];
  __shared__ int incl[BATCH_TILE];
  __shared__ int sh[BATCH_TILE / 32];
  load_pref(pref, a.live_pref, a.K);
  const int sel = *a.sel;
  const BatchBank B = a.bank[sel];
  const BatchBank O = a.bank[1 - sel];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long total = pref[a.K];
  const long long ntiles = (total + BATCH_TILE - 1) / BATCH_TILE;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long tile0 = tile * BATCH_TILE;
    const long long q = tile0 + threadIdx.x;
    const int n = (q < total) ? a.cnt[q] : 0;
    int x = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(FULL, x, o); if (lane >= o) x += y; }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int v = sh[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(FULL, v, o); if (lane >= o) v += y; }
      sh[lane] = v;
    }
    __syncthreads();
    incl[threadIdx.x] = x + (wid ? sh[wid - 1] : 0);
    __syncthreads();
    const int tot = incl[BATCH_TILE - 1];
    const long long out0 = a.blk[tile];
    for (int o = threadIdx.x; o < tot; o += BATCH_TILE) {
      int lo = 0, hi = BATCH_TILE - 1;  // the entry j with incl[j-1] <= o < incl[j]
      while (lo < hi) { const int mid = (lo + hi) >> 1; if (incl[mid] > o) hi = mid; else lo = mid + 1; }
      const long long src = tile0 + lo;
      const int k = find_inst(pref, a.K, src);
      const long long within = out0 + o - a.inst_pref[k];
      if (within >= a.census_cap[k]) continue;  // overflow: flagged by the scan
      const long long pid = a.slot_off[k] + (src - pref[k]);
      const int c = B.cell[pid];
      const long long dst = a.slot_off[k] + within;
      O.p1[dst] = B.p1[pid]; O.d1[dst] = B.d1[pid];
      O.w[dst] = (float)a.ew[a.cell_off[k] + c]; O.t[dst] = 0.f; O.cell[dst] = c;
    }
    __syncthreads();  // incl and sh are reused by the next tile
  }
}

// census energy after the comb per instance: sum over cells of copies * FP32(ew)
__global__ void __launch_bounds__(256) k_bcomb_disc(BatchArgs a) {
  __shared__ WarpStage stages[8];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double after = 0.0;
  int k = 0;
  if (c < a.n_cells) {
    k = a.cell_inst[c];
    after = a.ncopy[c] * (double)(float)a.ew[c];
  }
  warp_tally1(after != 0.0, k, after, a.comb_after, stages + (threadIdx.x >> 5));
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

int grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  if (g > 148LL * 16) g = 148LL * 16;
  return (int)(g < 1 ? 1 : g);
}

size_t pref_bytes(const BatchArgs& a) { return sizeof(long long) * (size_t)(a.K + 1); }

}  // namespace

cudaError_t imc_batch_launch_fill(const BatchArgs& a, int ic, long long bound, cudaStream_t s) {
  if (bound <= 0) return cudaSuccess;
  ++g_imc_launches;
  k_bfill<<<grid_for(bound, 256), 256, pref_bytes(a), s>>>(a, ic);
  return cudaGetLastError();
}

cudaError_t imc_batch_launch_wsum(const BatchArgs& a, cudaStream_t s) {
  ++g_imc_launches;
  k_bwsum<<<grid_for(a.n_slots, 256), 256, pref_bytes(a), s>>>(a);
  return cudaGetLastError();
}

cudaError_t imc_batch_launch_track(const BatchArgs& a, int block, int grid, cudaStream_t s) {
  ++g_imc_launches;
  if (a.form != 2 && a.max_cells > 0 && a.max_cells <= IMC_BATCH_SMEM_CELLS) {
    const bool pf = a.form == 3;
    const size_t sh = units_smem(a.K, a.max_cells) + (pf ? units_pf_smem(block) : 0);
    auto kern = pf ? k_btrack_units<true> : k_btrack_units<false>;
    if (sh > 48 * 1024) {
      const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
      if (e != cudaSuccess) return e;
    }
    kern<<<grid, block, sh, s>>>(a);
    return cudaGetLastError();
  }
  const size_t sh = (size_t)(block / 32) * sizeof(WarpStage) + pref_bytes(a);
  if (sh > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(k_btrack, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    if (e != cudaSuccess) return e;
  }
  k_btrack<<<grid, block, sh, s>>>(a);
  return cudaGetLastError();
}

cudaError_t imc_batch_launch_comb_ecen(const BatchArgs& a, cudaStream_t s) {
  ++g_imc_launches;
  k_bcomb_ecen<<<grid_for(a.n_slots, 256), 256, pref_bytes(a), s>>>(a);
  return cudaGetLastError();
}

cudaError_t imc_batch_launch_comb_copy(const BatchArgs& a, cudaStream_t s) {
  const int g = (int)std::min<long long>(std::max<long long>(a.max_tiles, 1), (long long)sm_count() * 2);
  g_imc_launches += 4;
  k_bcomb_count<<<g, BATCH_TILE, pref_bytes(a), s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_bcomb_scan<<<1, 1024, 0, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_bcomb_scatter<<<g, BATCH_TILE, pref_bytes(a), s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_bcomb_disc<<<(a.n_cells + 255) / 256, 256, 0, s>>>(a);
  return cudaGetLastError();
}

// ================================================================== C entry points
namespace {

#define BCUDA(call)                                 \
  do {                                              \
    cudaError_t e__ = (call);                       \
    if (e__ != cudaSuccess) {                       \
      imc_note_cuda_error((int)e__);                \
      return IMC_ERR_CUDA;                          \
    }                                               \
  } while (0)

inline size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

struct BatchLayout {
  size_t cell_inst, ef, vol, sass, cellf, emit_E, emit_n, emit_off, emit_w, tilt, ecen, ew, ncopy;
  size_t n_side, w_side, n_bank, n_new, census_cap, live_pref, new_pref, inst_pref, copies_d, wsum, esc_fx, dep_fx;
  size_t comb_after, e_side, e_emit, comb_before, cnt, blk, queue, total;
  long long max_tiles;
};

BatchLayout batch_layout(const imc_batch* b) {
  BatchLayout L{};
  size_t o = 0;
  auto take = [&](size_t bytes) { const size_t r = o; o += al256(bytes); return r; };
  const size_t nc = (size_t)b->n_cells, K = (size_t)b->n_inst, ns = (size_t)std::max<int64_t>(b->n_slots, 1);
  L.max_tiles = (long long)((ns + BATCH_TILE - 1) / BATCH_TILE);
  L.cell_inst = take(4 * nc); L.ef = take(4 * (nc + K)); L.vol = take(8 * nc);
  L.sass = take(8 * nc); L.cellf = take(16 * nc); L.emit_E = take(8 * nc); L.emit_n = take(8 * nc);
  L.emit_off = take(8 * (nc + K)); L.emit_w = take(4 * nc); L.tilt = take(8 * nc);
  L.ecen = take(8 * nc); L.ew = take(8 * nc); L.ncopy = take(8 * nc);
  L.n_side = take(8 * 2 * K); L.w_side = take(4 * 2 * K); L.n_bank = take(8 * K); L.n_new = take(8 * K);
  L.census_cap = take(8 * K); L.live_pref = take(8 * (K + 1)); L.new_pref = take(8 * (K + 1));
  L.inst_pref = take(8 * (K + 1)); L.copies_d = take(8 * K); L.wsum = take(8 * K); L.esc_fx = take(8 * 2 * K); L.dep_fx = take(8 * nc);
  L.comb_after = take(8 * K); L.e_side = take(8 * 2 * K); L.e_emit = take(8 * K); L.comb_before = take(8 * K);
  L.cnt = take(4 * ns); L.blk = take(8 * ((size_t)L.max_tiles + 1)); L.queue = take(8);
  L.total = o;
  return L;
}

template <class T>
T* wp(void* ws, size_t off) { return reinterpret_cast<T*>(static_cast<char*>(ws) + off); }

BatchArgs make_args(const imc_batch* b, const imc_batch_state* s, void* ws, const BatchLayout& L) {
  BatchArgs a{};
  a.K = b->n_inst; a.n_cells = b->n_cells; a.n_slots = b->n_slots; a.max_tiles = L.max_tiles;
  a.dt = b->dt; a.theta = b->theta;
  a.cell_off = b->cell_off; a.edges = b->edges; a.slot_off = reinterpret_cast<const long long*>(b->slot_off);
  a.seed = b->seed; a.n_target = reinterpret_cast<const long long*>(b->n_target);
  a.n_boundary = reinterpret_cast<const long long*>(b->n_boundary);
  a.n_max = reinterpret_cast<const long long*>(b->n_max);
  a.face_T = b->face_T; a.reflect = b->reflect; a.op_a = b->opacity_a; a.op_p = b->opacity_p; a.cv = b->cv;
  for (int q = 0; q < 2; ++q)
    a.bank[q] = BatchBank{s->bank[q].pos1, s->bank[q].dir1, s->bank[q].weight, s->bank[q].time, s->bank[q].cell};
  a.sel = s->sel; a.step = s->step; a.n_census = reinterpret_cast<long long*>(s->n_census);
  a.T = s->T; a.e = s->e; a.tr = s->tr; a.dep = s->dep; a.si = s->si; a.emitted = s->emitted;
  a.ledger = s->ledger; a.stats = s->stats; a.flags = s->flags;
  a.cell_inst = wp<int>(ws, L.cell_inst); a.ef = wp<float>(ws, L.ef); a.vol = wp<double>(ws, L.vol);
  a.sass = wp<float2>(ws, L.sass); a.cellf = wp<double2>(ws, L.cellf); a.emit_E = wp<double>(ws, L.emit_E);
  a.emit_n = wp<long long>(ws, L.emit_n); a.emit_off = wp<long long>(ws, L.emit_off);
  a.emit_w = wp<float>(ws, L.emit_w); a.tilt = wp<double>(ws, L.tilt);
  a.ecen = wp<double>(ws, L.ecen); a.ew = wp<double>(ws, L.ew); a.ncopy = wp<double>(ws, L.ncopy);
  a.n_side = wp<long long>(ws, L.n_side); a.w_side = wp<float>(ws, L.w_side);
  a.n_bank = wp<long long>(ws, L.n_bank); a.n_new = wp<long long>(ws, L.n_new);
  a.census_cap = wp<long long>(ws, L.census_cap); a.live_pref = wp<long long>(ws, L.live_pref);
  a.new_pref = wp<long long>(ws, L.new_pref); a.inst_pref = wp<long long>(ws, L.inst_pref);
  a.copies_d = wp<double>(ws, L.copies_d); a.wsum = wp<double>(ws, L.wsum);
  a.esc_fx = wp<unsigned long long>(ws, L.esc_fx); a.dep_fx = wp<unsigned long long>(ws, L.dep_fx);
  a.comb_after = wp<double>(ws, L.comb_after); a.e_side = wp<double>(ws, L.e_side);
  a.e_emit = wp<double>(ws, L.e_emit); a.comb_before = wp<double>(ws, L.comb_before);
  a.cnt = wp<int>(ws, L.cnt); a.blk = wp<long long>(ws, L.blk); a.queue = wp<unsigned long long>(ws, L.queue);
  a.chunk = 1024; a.refill_min = 1;
  a.max_cells = b->max_cells;
  return a;
}

constexpr int kMaxInstances = 4096;

imc_status batch_check(const imc_batch* b, const imc_batch_state* s, void* ws, size_t wsb) {
  if (!b || !s || !ws) return IMC_ERR_INVALID_ARG;
  if (b->n_inst < 1 || b->n_inst > kMaxInstances || b->n_cells < b->n_inst || b->n_slots < 1) return IMC_ERR_INVALID_ARG;
  if (b->n_slots >= (1LL << 31) || b->max_new < 0 || !(b->dt > 0.0)) return IMC_ERR_INVALID_ARG;
  if (!b->cell_off || !b->edges || !b->slot_off || !b->seed || !b->n_target || !b->n_boundary || !b->n_max ||
      !b->face_T || !b->reflect || !b->opacity_a || !b->opacity_p || !b->cv)
    return IMC_ERR_INVALID_ARG;
  for (int q = 0; q < 2; ++q) {
    const imc_bank& k = s->bank[q];
    if (!k.pos1 || !k.dir1 || !k.weight || !k.time || !k.cell || k.capacity < b->n_slots) return IMC_ERR_INVALID_ARG;
  }
  if (!s->sel || !s->step || !s->n_census || !s->T || !s->e || !s->tr || !s->dep || !s->si || !s->emitted ||
      !s->ledger || !s->stats || !s->flags)
    return IMC_ERR_INVALID_ARG;
  if (wsb < batch_layout(b).total) return IMC_ERR_WORKSPACE;
  return IMC_OK;
}

int track_grid(const imc_batch_launch* l, int* block) {
  int bs = (l && l->block_size > 0) ? l->block_size : 256;
  bs = std::max(32, std::min(256, bs / 32 * 32));
  const int bps = (l && l->blocks_per_sm > 0) ? l->blocks_per_sm : 4;
  *block = bs;
  return sm_count() * bps;
}

}  // namespace

extern "C" {

size_t imc_batch_workspace_bytes(const imc_batch* b) {
  if (!b || b->n_inst < 1 || b->n_cells < 1) return 0;
  return batch_layout(b).total;
}

imc_status imc_batch_init(const imc_batch* b, imc_batch_state* s, const double* T0, const double* Tr0,
                          void* workspace, size_t workspace_bytes, void* stream) {
  imc_status st = batch_check(b, s, workspace, workspace_bytes);
  if (st != IMC_OK) return st;
  if (!T0 || !Tr0) return IMC_ERR_INVALID_ARG;
  cudaStream_t cs = (cudaStream_t)stream;
  const BatchLayout L = batch_layout(b);
  BatchArgs a = make_args(b, s, workspace, L);
  BCUDA(cudaMemsetAsync(s->sel, 0, sizeof(int32_t), cs));
  BCUDA(cudaMemsetAsync(s->step, 0, sizeof(uint32_t), cs));
  BCUDA(cudaMemsetAsync(s->flags, 0, sizeof(int32_t), cs));
  BCUDA(cudaMemsetAsync(s->stats, 0, sizeof(unsigned long long) * IMC_STAT_N, cs));
  BCUDA(cudaMemsetAsync(s->n_census, 0, sizeof(int64_t) * b->n_inst, cs));
  BCUDA(cudaMemsetAsync(s->dep, 0, sizeof(double) * b->n_cells, cs));
  BCUDA(cudaMemsetAsync(s->si, 0, sizeof(double) * b->n_cells, cs));
  BCUDA(cudaMemsetAsync(s->emitted, 0, sizeof(double) * b->n_cells, cs));
  BCUDA(cudaMemsetAsync(s->tr, 0, sizeof(double) * b->n_cells, cs));
  BCUDA(imc_batch_launch_setup(a, T0, cs));
  BCUDA(imc_batch_launch_ic_plan(a, Tr0, cs));
  BCUDA(imc_batch_launch_prefix(a, cs));
  long long bound = 0;
  {
    // host bound of the initial census: n_target + nc per instance
    bound = b->max_new;
  }
  BCUDA(imc_batch_launch_fill(a, 1, bound, cs));
  BCUDA(imc_batch_launch_ledger(a, 1, cs));
  BCUDA(imc_batch_launch_material_fleck(a, 0, cs));
  int flags = 0;
  BCUDA(cudaMemcpyAsync(&flags, s->flags, sizeof(int), cudaMemcpyDeviceToHost, cs));
  BCUDA(cudaStreamSynchronize(cs));
  if (flags & IMC_FLAG_COMB_OVERFLOW) return IMC_ERR_BANK_OVERFLOW;
  if (flags & IMC_FLAG_NONFINITE) return IMC_ERR_NONFINITE;
  return IMC_OK;
}

imc_status imc_batch_step(const imc_batch* b, imc_batch_state* s, const imc_batch_launch* launch, void* workspace,
                          size_t workspace_bytes, void* stream) {
  imc_status st = batch_check(b, s, workspace, workspace_bytes);
  if (st != IMC_OK) return st;
  cudaStream_t cs = (cudaStream_t)stream;
  const BatchLayout L = batch_layout(b);
  BatchArgs a = make_args(b, s, workspace, L);
  if (launch && launch->chunk > 0) a.chunk = launch->chunk;
  if (launch && launch->refill_min > 0) a.refill_min = std::min(32, launch->refill_min);
  if (launch) a.form = launch->form;
  int block = 256;
  const int grid = track_grid(launch, &block);
  BCUDA(imc_batch_launch_plan(a, cs));
  BCUDA(imc_batch_launch_prefix(a, cs));
  BCUDA(imc_batch_launch_fill(a, 0, b->max_new, cs));
  BCUDA(imc_batch_launch_wsum(a, cs));
  BCUDA(imc_batch_launch_track(a, block, grid, cs));
  BCUDA(imc_batch_launch_material_fleck(a, 1, cs));
  BCUDA(imc_batch_launch_comb_ecen(a, cs));
  BCUDA(imc_batch_launch_comb_plan(a, cs));
  BCUDA(imc_batch_launch_comb_copy(a, cs));
  BCUDA(imc_batch_launch_ledger(a, 0, cs));
  return IMC_OK;
}

}  // extern "C"
