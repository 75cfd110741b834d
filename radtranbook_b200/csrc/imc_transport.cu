// imc_transport.cu — event-based tracking of a census/source bank to census.
//
// Reference behaviour (per event and per history):
//   slab   IMC/IMC1D.py:75-130 (move_particle), 133-200 (move_particles)
//   sphere IMC/IMC1D.py:336-436, 439-532
//   xy/rz  IMC/IMC2D.py:711-935 (events), 938-1107 (history loop)
//   multigroup  MG_IMC/MG_IMC2D.py:580-989 (xy, rz), MG_IMC/MG_IMC1D.py:276-461 (sphere)
//
// Execution model: a persistent grid (blocks_per_sm x SMs).  Each warp claims a chunk of
// bank indices with one atomic ticket and keeps 32 histories in registers.  Every loop
// iteration advances every live lane by one event (distance to face / effective scatter /
// census, implicit capture w *= exp(-sigma_a s)); at each event boundary, lanes whose
// history ended are refilled from the warp's chunk, so warps do not carry dead lanes until
// the bank drains (the in-warp form of bank compaction between events).  Particle state is
// FP32; energy removed from a history is accounted as the exact FP64 difference of its
// FP32 weights, accumulated in registers while the history stays in one cell and flushed
// through warp-aggregated FP64 reductions when it leaves.  Random numbers: Philox keyed by
// the run seed, counter (id_base + bank index, event number, step, TAG_TRANSPORT).
#include <algorithm>

#include "imc_device.cuh"
#include "imc_internal.h"

using namespace imcdev;

namespace {

// Block-level counters for rare events (shared-memory atomics keep them out of registers).
enum : int { B_CENSUS = 0, B_FLOOR, B_REFLECT, B_CAP, B_ESCAPE, B_CAPTURE, B_N };

// MG: group-indexed tables and tallies, escaped energy also by group.  In 2-D the rules of
// MG_IMC/MG_IMC2D.py:580-989 (no effective-scatter cap, no absorption for sigma_a <= 1e-12,
// the weight floor ends a history after its event is committed); on the 1-D sphere those of
// MG_IMC/MG_IMC1D.py:276-461, which are the gray spherical ones (cap, floor kill with local
// deposit) with the floor coefficient 1e-14.
// CF: Carter-Forest (IMC/IMC1D_CarterForest.py:63-331, 614-820; IMC/IMC2D_CarterForest.py:
// 102-508).  The table holds (0, sigma_a): the flight samples the absorption distance in the
// scatter slot (same threshold and cap) and captures nothing on the way; at an absorption the
// photon is re-emitted in the new direction the event drew after a delay ~ Exp(cf_rate) if that
// falls inside the step, else captured (its weight deposited).  Histories at or below the
// weight floor are not moved (they stay in census).
// One event of one history (distance to the cell boundary / effective scatter / census,
// implicit capture, crossing with reflection or escape, weight floor, events cap) and, when
// the history ends, its final state written back to the bank.  Shared by the persistent
// kernel k_track (the history in registers, refilled in-warp) and the event-by-event kernel
// k_event (the history in device arrays, survivors compacted between launches): both follow
// a history through the same arithmetic and the same Philox draws.
struct Hist {
  uint32_t pid, ev;
  float x, y, u, v, w, dcen, w_in;
  int ci, cj, grp;
  float2 tab;      // (sigma_a, sigma_s) of the current (group, cell)
  double acc_wd;   // w*s in the current cell (cells without absorption only)
};
struct EvOut {
  bool flush;      // a cell visit to flush: deposition f_lost, path length f_wd, into flush_cell
  int flush_cell;
  double f_lost, f_wd;
  bool cen;        // the history ended alive: its weight goes to the comb's census sums
  int cen_bin;
  bool finished;
};

template <int GEOM, bool SMEM_CELLS, bool MG, bool CF>
__device__ __forceinline__ void history_event(const TrackArgs& a, Hist& h, EvOut& o, const float* E1,
                                              const float* E2, const float2* CS, unsigned* blk_cnt,
                                              unsigned long long* blk_esc, unsigned long long* dep_t,
                                              uint32_t stepk, float weight_floor, double inv_q,
                                              unsigned& s_bd, unsigned& s_sc) {
  constexpr bool ONED = GEOM == G_SLAB || GEOM == G_SPHERE;
  constexpr bool MG2 = MG && !ONED;  // MG_IMC2D history rules
  const float c_light = (float)C_LIGHT;
  const float ss_thr = ONED ? 1e-10f : 1e-12f;
  auto table = [&](int cq) { return SMEM_CELLS ? CS[cq] : __ldg(a.sass + cq); };
  uint32_t& pid = h.pid;
  uint32_t& ev = h.ev;
  float &x = h.x, &y = h.y, &u = h.u, &v = h.v, &w = h.w, &dcen = h.dcen, &w_in = h.w_in;
  int &ci = h.ci, &cj = h.cj, &grp = h.grp;
  float2& tab = h.tab;
  double& acc_wd = h.acc_wd;
  bool& flush = o.flush;
  int& flush_cell = o.flush_cell;
  double &f_lost = o.f_lost, &f_wd = o.f_wd;
  bool& cen = o.cen;
  int& cen_bin = o.cen_bin;
  const int c = ci + a.nx * cj;
  const int cq = MG ? c + a.nc * grp : c;  // (group, cell) table / tally index
  const float sa = tab.x, ss = tab.y;
  bool finished = false, frozen = false;
  if (ev >= (uint32_t)a.max_events) {
    // events-per-history cap (IMC/IMC2D.py:974-977): stops, weight stays in census
    atomicAdd(&blk_cnt[B_CAP], 1u);
    if (!a.cap_is_reference) atomicOr(a.flags, (int)IMC_FLAG_EVENT_CAP);
    finished = true;
  } else {
    const U4 r = draw_rk(a.rk, a.id_base + pid, ev, stepk, TAG_TRANSPORT);
    ++ev;
    float d, sb, L, xn = x, yn = y, un = u, vn = v;
    int evt, cross = X_NONE;
    // ---- distance to the cell boundary ----
    float s_rin = BIGF, s_rout = BIGF, s_zlo = BIGF, s_zhi = BIGF, st_ = 0.f, sx = BIGF, sy = BIGF;
    float din = BIGF, dout = BIGF;
    if (GEOM == G_SLAB) {
      const float xl = E1[ci], xr = E1[ci + 1];
      L = xr - xl;
      sb = slab_face(x, u, xl, xr);
    } else if (GEOM == G_SPHERE) {
      const float r0 = E1[ci], r1 = E1[ci + 1];
      L = r1 - r0;
      const float b2 = x * x * ((1.f - u) * (1.f + u));
      dout = outer_root(x, u, r1, b2);
      din = inner_root(x, u, r0, b2);
      sb = fminf(dout, din);
    } else if (GEOM == G_XY) {
      const float xl = E1[ci], xr = E1[ci + 1], yl = E2[cj], yr = E2[cj + 1];
      L = fminf(xr - xl, yr - yl);
      if (u > 0.f) sx = __fdividef(xr - x, u); else if (u < 0.f) sx = __fdividef(xl - x, u);
      if (v > 0.f) sy = __fdividef(yr - y, v); else if (v < 0.f) sy = __fdividef(yl - y, v);
      sx = fmaxf(sx, 0.f); sy = fmaxf(sy, 0.f);
      sb = fminf(sx, sy);
    } else {
      const float rin = E1[ci], rout = E1[ci + 1], zlo = E2[cj], zhi = E2[cj + 1];
      L = fminf(rout - rin, zhi - zlo);
      const float sin2 = (1.f - v) * (1.f + v);
      if (sin2 >= 1e-15f) {
        const float ist = rsqrtf(sin2);
        st_ = sin2 * ist;
        const float b2 = x * x * ((1.f - u) * (1.f + u));
        s_rout = outer_root(x, u, rout, b2) * ist;
        const float li = inner_root(x, u, rin, b2);
        if (li < BIGF) s_rin = li * ist;
      }
      if (v > 1e-15f) s_zhi = fmaxf(__fdividef(zhi - y, v), 0.f);
      else if (v < -1e-15f) s_zlo = fmaxf(__fdividef(zlo - y, v), 0.f);
      sb = fminf(fminf(s_rin, s_rout), fminf(s_zlo, s_zhi));
    }
    // ---- effective-scatter distance (reference cap: sigma_s*L > 1e4 -> 1e4/L) ----
    // -log(u)/sigma competes with s_other = min(boundary, census); when sigma*s_other
    // is small the scatter loses unless u > exp(-sigma*s_other), tested in FP64 with a
    // short series, so the logarithm is evaluated only when it can win.
    float ds = BIGF;
    {
      const bool capped = !MG2 && ss * L > 10000.0f;
      const float sig = capped ? 10000.0f / L : (ss > ss_thr ? ss : 0.f);
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
    d = sb; evt = EV_BOUNDARY;
    if (ds < d) { d = ds; evt = EV_SCATTER; }
    if (dcen < d) { d = dcen; evt = EV_CENSUS; }
    // ---- move ----
    if (GEOM == G_SLAB) {
      const float xl = E1[ci], xr = E1[ci + 1];
      xn = fmaf(u, d, x);
      if (evt == EV_BOUNDARY) { if (u > 0.f) { xn = xr; cross = X_IP; } else { xn = xl; cross = X_IM; } }
      else { if (evt == EV_SCATTER) un = fmaf(2.f, u01f(r.y), -1.f); xn = fminf(fmaxf(xn, xl), xr); }
    } else if (GEOM == G_SPHERE) {
      const float r0 = E1[ci], r1 = E1[ci + 1];
      const float ax = fmaf(u, d, x);
      float rn = sqrt_nn(fmaf(ax, ax, d * d * ((1.f - u) * (1.f + u))));
      float mun = rn > 1e-15f ? (x * u + d) / rn : 1.f;
      if (evt == EV_BOUNDARY) {
        if (dout <= din) { rn = r1; mun = (x * u + d) / r1; cross = X_IP; }
        else { rn = r0; mun = (x * u + d) / r0; cross = X_IM; }
      } else {
        if (evt == EV_SCATTER) mun = fmaf(2.f, u01f(r.y), -1.f);
        rn = fminf(fmaxf(rn, r0), r1);
      }
      xn = rn; un = fminf(1.f, fmaxf(-1.f, mun));
    } else if (GEOM == G_XY) {
      const float xl = E1[ci], xr = E1[ci + 1], yl = E2[cj], yr = E2[cj + 1];
      xn = fmaf(u, d, x); yn = fmaf(v, d, y);
      if (evt == EV_BOUNDARY) {
        if (sx <= sy) { if (u > 0.f) { xn = xr; cross = X_IP; } else { xn = xl; cross = X_IM; } yn = fminf(fmaxf(yn, yl), yr); }
        else { if (v > 0.f) { yn = yr; cross = X_JP; } else { yn = yl; cross = X_JM; } xn = fminf(fmaxf(xn, xl), xr); }
      } else {
        if (evt == EV_SCATTER) {
          const float uz = fmaf(2.f, u01f(r.y), -1.f);
          const float rxy = sqrt_nn((1.f - uz) * (1.f + uz));
          float sp, cp;
          sincospif(2.f * u01f(r.z), &sp, &cp);
          un = rxy * cp; vn = rxy * sp;
        }
        xn = fminf(fmaxf(xn, xl), xr); yn = fminf(fmaxf(yn, yl), yr);
      }
    } else {
      const float rin = E1[ci], rout = E1[ci + 1], zlo = E2[cj], zhi = E2[cj + 1];
      const float l = d * st_;
      const float ax = fmaf(u, l, x);
      float rn = sqrt_nn(fmaf(ax, ax, l * l * ((1.f - u) * (1.f + u))));
      yn = fmaf(d, v, y);
      if (rn > 1e-15f && l > 0.f) un = fminf(1.f, fmaxf(-1.f, __fdividef(fmaf(x, u, l), rn)));
      if (evt == EV_BOUNDARY) {
        if (sb == s_rin) { rn = rin; cross = X_IM; }
        else if (sb == s_rout) { rn = rout; cross = X_IP; }
        else if (sb == s_zlo) { yn = zlo; cross = X_JM; }
        else { yn = zhi; cross = X_JP; }
      } else if (evt == EV_SCATTER) {
        vn = fmaf(2.f, u01f(r.y), -1.f);
        un = cospif(2.f * u01f(r.z));
      }
      if (cross != X_IM && cross != X_IP) rn = fminf(fmaxf(rn, rin), rout);
      if (cross != X_JM && cross != X_JP) yn = fminf(fmaxf(yn, zlo), zhi);
      xn = rn;
    }
    // implicit capture (the energy removed is counted at the flush, w_in - w)
    const float wn = (MG2 && !(sa > 1e-12f)) ? w : w * __expf(-sa * d);
    // path-length intensity: w*s is needed only in cells without absorption (table
    // entry 0: below the estimator's threshold, or Carter-Forest); elsewhere it is
    // lost / (sigma_a V dt), formed from the deposition tally when the step ends
    if (!(sa > 0.f)) acc_wd += (double)(w * d);
    dcen -= d;
    bool captured = false;
    if (CF && evt == EV_SCATTER) {
      // absorption (IMC/IMC1D_CarterForest.py:146-194, IMC/IMC2D_CarterForest.py:189-210)
      const float rate = __ldg(a.cf_rate + c);
      const float tr = dcen / c_light;  // time left after the flight
      const uint32_t ub = ONED ? r.z : r.w;
      if (!(rate > 0.f)) {
        captured = !ONED;  // no re-emission: 1-D redirects, 2-D captures
      } else if (a.cf_fastpath > 0.f && tr > 1e-14f && rate * tr > a.cf_fastpath) {
        captured = u01f(ub) < __expf(-rate * tr);
      } else {
        const float delay = __fdividef(neglog_u(ub), rate);
        if (ONED ? (tr > 1e-14f && delay < tr) : (delay < tr - 1e-15f)) dcen = fmaxf(0.f, (tr - delay) * c_light);
        else captured = true;
      }
      // a capture deposits the whole weight: w becomes 0 below, so w_in - w includes it
    }
    if (evt == EV_BOUNDARY) ++s_bd;
    else if (captured) atomicAdd(&blk_cnt[B_CAPTURE], 1u);
    else if (evt == EV_SCATTER) ++s_sc;
    else atomicAdd(&blk_cnt[B_CENSUS], 1u);

    if (!MG && !CF && (GEOM == G_XY || GEOM == G_RZ)) {
      if (wn <= weight_floor) {
        // IMC/IMC2D.py:1043-1047: history stops in place keeping its weight
        atomicAdd(&blk_cnt[B_FLOOR], 1u);
        w = wn;
        frozen = true;
        finished = true;
      }
    }
    if (!frozen) {
      w = captured ? 0.f : wn; x = xn; y = yn; u = un; v = vn;
      if (CF && captured) finished = true;
      if (cross != X_NONE) {
        // leaving the cell: flush the visit (before an escape zeroes w) and start the next
        flush = true; flush_cell = cq; f_lost = (double)w_in - (double)w; f_wd = acc_wd;
        w_in = w; acc_wd = 0.0;
        int ni = ci, nj = cj;
        if (cross == X_IP) ++ni; else if (cross == X_IM) --ni; else if (cross == X_JP) ++nj; else --nj;
        int side = -1;
        if (ni < 0) side = 0; else if (ni >= a.nx) side = 1; else if (nj < 0) side = 2; else if (nj >= a.ny) side = 3;
        if (side >= 0) {
          if ((a.reflect_mask >> side) & 1) {
            if (side < 2) { u = -u; ni = side == 0 ? 0 : a.nx - 1; }
            else { v = -v; nj = side == 2 ? 0 : a.ny - 1; }
            atomicAdd(&blk_cnt[B_REFLECT], 1u);
          } else {
            const unsigned long long uw = fx_units((double)w, inv_q);
            atomicAdd(&blk_esc[side], uw);
            if (MG) atomicAdd(a.esc_fx + 4 + grp, uw);
            atomicAdd(&blk_cnt[B_ESCAPE], 1u);
            w = 0.f;
            finished = true;
            ni = ci; nj = cj;
          }
        }
        ci = ni; cj = nj;
        if (!finished) tab = table(MG ? ci + a.nx * cj + a.nc * grp : ci + a.nx * cj);
      }
      if (GEOM == G_SLAB || GEOM == G_SPHERE) {
        if (!CF && !finished && w < weight_floor) {
          // IMC/IMC1D.py:188-195: kill and deposit the remainder in the current cell
          // (every cell, including the two edge cells the reference skips).  Without a
          // crossing in this event the visit's flush at the history end (w_in - 0) carries
          // it; after one, the old cell holds the flush slot and the remainder is added to
          // the new cell here.  Its intensity share, lost / (sigma_a V dt), follows from the
          // deposition tally.
          atomicAdd(&blk_cnt[B_FLOOR], 1u);
          if (flush) {
            const int c2 = ci + a.nx * cj + (MG ? a.nc * grp : 0);
            atomicAdd(dep_t + c2, fx_units((double)w, inv_q));
          }
          w = 0.f;
          finished = true;
        }
      } else if (MG2 && !finished && dcen > 0.f && w <= weight_floor) {
        // MG_IMC/MG_IMC2D.py:858-860: the next event would stop at the floor (a weight
        // that underflowed to 0 included)
        atomicAdd(&blk_cnt[B_FLOOR], 1u);
        finished = true;
      } else if (!finished && !(w > 0.f)) {
        w = 0.f;
        finished = true;
      }
      if (!finished && !(dcen > 0.f)) finished = true;
    }
  }
  if (finished) {
    // A history that ends without leaving its cell flushes that cell's visit now.  (One
    // that ended by crossing has already queued the old cell and holds nothing new: a
    // 1-D weight-floor kill after a crossing deposits directly.)
    if (!flush) {
      const double lost = (double)w_in - (double)w;
      if (lost != 0.0 || acc_wd != 0.0) { flush = true; flush_cell = cq; f_lost = lost; f_wd = acc_wd; }
    }
    acc_wd = 0.0;
    a.w[pid] = w;
    // census, cap and frozen histories keep their (pre-event, when frozen) state
    if (w > 0.f) {
      a.p1[pid] = x; a.d1[pid] = u;
      if (GEOM == G_XY || GEOM == G_RZ) { a.p2[pid] = y; a.d2[pid] = v; }
      a.cell[pid] = ci + a.nx * cj;
      cen = true;
      cen_bin = ci + a.nx * cj + (a.ecen_by_group ? a.nc * grp : 0);
    }
  }
  o.finished = finished;
}

// SMEM_TALLY (small meshes): the block sums its deposition (fixed point) and intensity per
// (group, cell) in shared memory and adds them to the global tallies once, at its end.  On a
// mesh of a few hundred cells every crossing would otherwise send its reductions to the few
// dozen cells the wave occupies, which serialise in the L2.
//
// PF (prefetched refills): every lane keeps the bank record of its next history in a
// shared-memory slot, copied there by cp.async while it tracks the current one, so a lane
// whose history ends starts the next one from shared memory instead of holding its warp on two
// dependent HBM reads (weight and birth time, then the rest of the record).  The histories,
// their Philox counters and the tallies are the same; only which lane tracks which differs.
enum : int { PF_W = 0, PF_T, PF_P1, PF_D1, PF_CELL, PF_P2, PF_D2, PF_GROUP, PF_PID, PF_NF };
inline size_t pf_smem(int block) { return sizeof(float) * PF_NF * (size_t)block; }

template <int GEOM, bool SMEM_CELLS, bool MG, bool CF, bool SMEM_TALLY, bool PF>
__global__ void __launch_bounds__(256, PF ? 4 : 1) k_track(TrackArgs a) {  // PF: at most 64 registers
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  const float dtk = a.dt_dev ? (float)*a.dt_dev : a.dt;  // graph replay: step length and Philox
  const uint32_t stepk = a.step_dev ? *a.step_dev : a.step;  // step counter from device memory
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ unsigned blk_cnt[B_N];
  __shared__ unsigned long long blk_esc[4];
  constexpr bool ONED = GEOM == G_SLAB || GEOM == G_SPHERE;
  constexpr bool MG2 = MG && !ONED;  // MG_IMC2D history rules
  WarpStage* stages = reinterpret_cast<WarpStage*>(smem);
  const int nwarps = blockDim.x >> 5;
  float* E1 = reinterpret_cast<float*>(stages + nwarps);
  float* E2 = E1 + (a.nx + 1);
  float2* CS = reinterpret_cast<float2*>(E2 + (a.ny + 1) + ((a.nx + a.ny) & 1));
  const int ncg = a.nc * a.ng;
  // block tallies after the table (8-byte aligned: CS is), deposition then intensity
  unsigned long long* TD = reinterpret_cast<unsigned long long*>(CS + (SMEM_CELLS ? ncg : 0));
  double* TS = reinterpret_cast<double*>(TD + ncg);
  unsigned long long* const dep_t = SMEM_TALLY ? TD : a.dep_fx;
  double* const si_t = SMEM_TALLY ? TS : a.si;
  for (int q = threadIdx.x; q <= a.nx; q += blockDim.x) E1[q] = a.e1[q];
  for (int q = threadIdx.x; q <= a.ny; q += blockDim.x) E2[q] = a.e2[q];
  if (SMEM_CELLS)
    for (int q = threadIdx.x; q < ncg; q += blockDim.x) CS[q] = a.sass[q];
  if (SMEM_TALLY)
    for (int q = threadIdx.x; q < ncg; q += blockDim.x) { TD[q] = 0ull; TS[q] = 0.0; }
  if (threadIdx.x < B_N) blk_cnt[threadIdx.x] = 0u;
  if (threadIdx.x < 4) blk_esc[threadIdx.x] = 0ull;
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  WarpStage* st = stages + (threadIdx.x >> 5);
  const uint32_t n = (uint32_t)*a.n_dev;

  // warp-uniform chunk cursor
  uint32_t chunk_next = 0, chunk_end = 0;
  bool drained = false;

  // lane state
  bool has = false;
  uint32_t pid = 0, ev = 0;
  float x = 0, y = 0, u = 0, v = 0, w = 0, dcen = 0;
  int ci = 0, cj = 0, grp = 0;
  // (sigma_a, sigma_s) of the current (group, cell), loaded as soon as the cell is known (at
  // refill, after a crossing) so the load overlaps the tally flush and refill of the loop end
  float2 tab = make_float2(0.f, 0.f);
  auto table = [&](int cq) { return SMEM_CELLS ? CS[cq] : __ldg(a.sass + cq); };
  // energy removed in the current cell visit: the per-flight differences telescope, so it is
  // the weight at the visit's start minus the weight now (one FP64 difference at the flush)
  float w_in = 0.f;
  double acc_wd = 0.0;  // w*s in the current cell (cells without absorption only)
  unsigned s_bd = 0, s_sc = 0;          // per-event counters (census/cap counted at finish)
  unsigned n_alive = 0;                 // entries alive at the end (census sums for the comb)

  const float c_light = (float)C_LIGHT;
  // weight floor, IMC/IMC1D.py:1007 / IMC/IMC2D.py:1771 (1e-10); MG_IMC/MG_IMC1D.py:1127 (1e-14)
  const float weight_floor = (float)(a.floor_coef * (*a.wsum) / (double)(n > 0 ? n : 1));
  const double inv_q = fx_inv_quantum(*a.wsum);  // fixed-point energy tallies
  const float inv_nx = 1.0f / (float)a.nx;  // cell -> (i, j) at refill without an integer divide

  // PF: the lane's next bank record, field f of thread i at PQ[f * blockDim.x + i] (after the
  // block tallies, or after the cell table without them)
  float* const my_pf = (SMEM_TALLY ? reinterpret_cast<float*>(TS + ncg) : reinterpret_cast<float*>(TD)) + threadIdx.x;
  const int pfs = blockDim.x;
  bool pv = false;  // PF: the slot holds a claimed record (copies issued)

  for (;;) {
    // ---------------- refill idle lanes from the warp's chunk ----------------
    if (PF) {
      // An idle lane takes the record in its slot; every lane without a claim takes the next
      // entry of the warp's chunk (a new guided ticket when it runs out) and starts its copies,
      // which land while the lane tracks.  Leaves with every lane tracking or holding no claim;
      // when the warp stops, the queue is past n and no claim is left untaken.
      for (;;) {
        if (!has && pv) {
          cp_async_wait_all();
          pv = false;
          pid = __float_as_uint(my_pf[PF_PID * pfs]);
          w = my_pf[0];
          dcen = (dtk - my_pf[pfs]) * c_light;
          const int c = __float_as_int(my_pf[PF_CELL * pfs]);
          const int g = MG ? __float_as_int(my_pf[PF_GROUP * pfs]) : 0;
          const bool moves = (MG2 || CF ? w > weight_floor : w > 0.f) && dcen > 0.f;
          if (!moves && w > 0.f && a.ecen) {
            const int b = c + (a.ecen_by_group ? a.nc * g : 0);
#ifdef IMC_CHECKED
            if (b >= 0 && b < a.nc * (a.ecen_by_group ? a.ng : 1))
#endif
            { atomicAdd(a.ecen + b, (double)w); ++n_alive; }
          }
          if (moves) {
            x = my_pf[2 * pfs]; u = my_pf[3 * pfs];
            if (MG) grp = g;
            if (GEOM == G_XY || GEOM == G_RZ) { y = my_pf[PF_P2 * pfs]; v = my_pf[PF_D2 * pfs]; }
#ifdef IMC_CHECKED
            if (c < 0 || c >= a.nc || (MG && (grp < 0 || grp >= a.ng)) || !isfinite(w)) {
              atomicOr(a.flags, (int)IMC_FLAG_BOUNDS);
            } else
#endif
            {
              cj = __float2int_rd(((float)c + 0.5f) * inv_nx);
              ci = c - cj * a.nx;
              if (ci < 0) { --cj; ci += a.nx; } else if (ci >= a.nx) { ++cj; ci -= a.nx; }
              tab = table(MG ? c + a.nc * grp : c);
              ev = 0;
              w_in = w;
              has = true;
            }
          }
        }
        if (!drained) {
          const unsigned pneed = __ballot_sync(FULL, !pv);
          if (pneed) {
            if (chunk_next >= chunk_end) {
              unsigned long long base = 0, claim = 0;
              if (lane == 0) {
                const unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(a.queue);
                const unsigned long long left = cur < (unsigned long long)n ? (unsigned long long)n - cur : 0ull;
                const unsigned long long nw = (unsigned long long)gridDim.x * (blockDim.x >> 5);
                claim = min((unsigned long long)a.chunk, max(32ull, left / (2ull * nw)));
                base = atomicAdd(a.queue, claim);
              }
              base = __shfl_sync(FULL, base, 0);
              claim = __shfl_sync(FULL, claim, 0);
              if (base >= (unsigned long long)n) {
                drained = true;
              } else {
                chunk_next = (uint32_t)base;
                chunk_end = (uint32_t)min(base + claim, (unsigned long long)n);
              }
            }
            if (!drained) {
              const uint32_t avail = chunk_end - chunk_next;
              const uint32_t rank = __popc(pneed & lt_mask);
              if (!pv && rank < avail) {
                const uint32_t np = chunk_next + rank;
                my_pf[PF_PID * pfs] = __uint_as_float(np);
                cp_async4(my_pf, a.w + np);
                cp_async4(my_pf + pfs, a.t + np);
                cp_async4(my_pf + 2 * pfs, a.p1 + np);
                cp_async4(my_pf + 3 * pfs, a.d1 + np);
                cp_async4(my_pf + PF_CELL * pfs, a.cell + np);
                if (GEOM == G_XY || GEOM == G_RZ) {
                  cp_async4(my_pf + PF_P2 * pfs, a.p2 + np);
                  cp_async4(my_pf + PF_D2 * pfs, a.d2 + np);
                }
                if (MG) cp_async4(my_pf + PF_GROUP * pfs, a.group + np);
                cp_async_commit();
                pv = true;
              }
              chunk_next += min((uint32_t)__popc(pneed), avail);
            }
          }
        }
        if (!__any_sync(FULL, !has && pv)) break;
      }
    }
    unsigned need = PF ? 0u : __ballot_sync(FULL, !has);
    while (need && !drained) {
      if (chunk_next >= chunk_end) {
        // guided claim: a share of what is left, at most `chunk`, at least 32, so early
        // claims are long contiguous (coherent) runs and the drain is finely balanced
        unsigned long long base = 0, claim = 0;
        if (lane == 0) {
          const unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(a.queue);
          const unsigned long long left = cur < (unsigned long long)n ? (unsigned long long)n - cur : 0ull;
          const unsigned long long nw = (unsigned long long)gridDim.x * (blockDim.x >> 5);
          claim = min((unsigned long long)a.chunk, max(32ull, left / (2ull * nw)));
          base = atomicAdd(a.queue, claim);
        }
        base = __shfl_sync(FULL, base, 0);
        claim = __shfl_sync(FULL, claim, 0);
        if (base >= (unsigned long long)n) { drained = true; break; }
        chunk_next = (uint32_t)base;
        chunk_end = (uint32_t)min(base + claim, (unsigned long long)n);
      }
      const uint32_t avail = chunk_end - chunk_next;
      const uint32_t rank = __popc(need & lt_mask);
      if (!has && rank < avail) {
        pid = chunk_next + rank;
        w = a.w[pid];
        dcen = (dtk - a.t[pid]) * c_light;
        const bool moves = (MG2 || CF ? w > weight_floor : w > 0.f) && dcen > 0.f;
        if (!moves && w > 0.f && a.ecen) {
          // not tracked but alive: part of the census the comb sees
          const int b = a.cell[pid] + (a.ecen_by_group ? a.nc * a.group[pid] : 0);
#ifdef IMC_CHECKED
          if (b >= 0 && b < a.nc * (a.ecen_by_group ? a.ng : 1))
#endif
          { atomicAdd(a.ecen + b, (double)w); ++n_alive; }
        }
        if (moves) {
          x = a.p1[pid]; u = a.d1[pid];
          if (MG) grp = a.group[pid];
          if (GEOM == G_XY || GEOM == G_RZ) { y = a.p2[pid]; v = a.d2[pid]; }
          const int c = a.cell[pid];
#ifdef IMC_CHECKED
          // bounds-checked build: an entry outside the mesh (or group range), or with a
          // non-finite weight, is reported and left untouched
          if (c < 0 || c >= a.nc || (MG && (grp < 0 || grp >= a.ng)) || !isfinite(w)) {
            atomicOr(a.flags, (int)IMC_FLAG_BOUNDS);
          } else
#endif
          {
            // j from a float estimate, corrected to the exact quotient (the estimate is off
            // by at most one for any int c)
            cj = __float2int_rd(((float)c + 0.5f) * inv_nx);
            ci = c - cj * a.nx;
            if (ci < 0) { --cj; ci += a.nx; } else if (ci >= a.nx) { ++cj; ci -= a.nx; }
            tab = table(MG ? c + a.nc * grp : c);
            ev = 0;
            w_in = w;
            has = true;
          }
        }
      }
      chunk_next += min((uint32_t)__popc(need), avail);
      need = __ballot_sync(FULL, !has);
    }
    if (!__any_sync(FULL, has)) break;
#ifdef IMC_CHECKED
    if (has && (ci < 0 || ci >= a.nx || cj < 0 || cj >= a.ny || !isfinite(w) || !isfinite(x) || !isfinite(dcen))) {
      atomicOr(a.flags, (int)IMC_FLAG_BOUNDS);
      w_in = w; acc_wd = 0.0;  // nothing is tallied at an invalid index
      has = false;
    }
#endif

    EvOut o{false, 0, 0.0, 0.0, false, 0, false};
    if (has) {
      Hist h{pid, ev, x, y, u, v, w, dcen, w_in, ci, cj, grp, tab, acc_wd};
      history_event<GEOM, SMEM_CELLS, MG, CF>(a, h, o, E1, E2, CS, blk_cnt, blk_esc, dep_t, stepk, weight_floor,
                                              inv_q, s_bd, s_sc);
      pid = h.pid; ev = h.ev; x = h.x; y = h.y; u = h.u; v = h.v; w = h.w; dcen = h.dcen; w_in = h.w_in;
      ci = h.ci; cj = h.cj; grp = h.grp; tab = h.tab; acc_wd = h.acc_wd;
      if (o.finished) has = false;
    }
    const bool flush = o.flush, cen = o.cen;
    const int flush_cell = o.flush_cell, cen_bin = o.cen_bin;
    const double f_lost = o.f_lost, f_wd = o.f_wd;
    // ---------------- converged tally flush ----------------
    // deposited energy in fixed point; w*s (raw, only from cells without absorption) in FP64
    unsigned long long ud = 0ull;
    double vs = 0.0;
    if (flush) {
      ud = fx_units(f_lost, inv_q);
      vs = f_wd;
    }
    if (SMEM_TALLY) {
      // block tallies in shared memory: one shared atomic per flushing lane costs less than
      // grouping the warp's lanes by cell first (the grouping pays off for global tallies)
      if (flush) { if (ud) atomicAdd(dep_t + flush_cell, ud); if (vs != 0.0) atomicAdd(si_t + flush_cell, vs); }
    } else {
      warp_tally_fx(flush, flush_cell, ud, vs, dep_t, si_t, st);
    }
    if (a.ecen) {
      warp_tally1(cen, cen_bin, (double)w, a.ecen, st);
      n_alive += cen ? 1u : 0u;
    }
  }

  // ---------------- statistics ----------------
  const unsigned long long t_bd = warp_sum_u(s_bd), t_sc = warp_sum_u(s_sc);
  if (a.ecen) {
    const unsigned long long t_alive = warp_sum_u(n_alive);
    if (lane == 0 && t_alive) atomicAdd(a.n_live, t_alive);
  }
  if (lane == 0) {
    if (t_bd) atomicAdd(a.stats + S_BOUNDARY, t_bd);
    if (t_sc) atomicAdd(a.stats + S_SCATTER, t_sc);
    if (t_bd + t_sc) atomicAdd(a.stats + S_EVENTS, t_bd + t_sc);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned long long cen = blk_cnt[B_CENSUS], cap = blk_cnt[B_CAP], capt = blk_cnt[B_CAPTURE];
    if (cen) atomicAdd(a.stats + S_CENSUS, cen);
    if (capt) atomicAdd(a.stats + S_CAPTURE, capt);
    if (cen + cap + capt) atomicAdd(a.stats + S_EVENTS, cen + cap + capt);
    if (blk_cnt[B_FLOOR]) atomicAdd(a.stats + S_FLOOR, (unsigned long long)blk_cnt[B_FLOOR]);
    if (blk_cnt[B_REFLECT]) atomicAdd(a.stats + S_REFLECT, (unsigned long long)blk_cnt[B_REFLECT]);
    if (cap) atomicAdd(a.stats + S_CAP, cap);
    if (blk_cnt[B_ESCAPE]) atomicAdd(a.stats + S_ESCAPE, (unsigned long long)blk_cnt[B_ESCAPE]);
  }
  if (threadIdx.x < 4 && blk_esc[threadIdx.x] != 0ull) atomicAdd(a.esc_fx + threadIdx.x, blk_esc[threadIdx.x]);
  if (SMEM_TALLY) {
    // the block's tallies (every warp's last flush is behind the __syncthreads above)
    for (int q = threadIdx.x; q < ncg; q += blockDim.x) {
      if (TD[q]) atomicAdd(a.dep_fx + q, TD[q]);
      if (TS[q] != 0.0) atomicAdd(a.si + q, TS[q]);
    }
  }
}

template <int GEOM, bool SM, bool MG, bool CF, bool ST, bool PF>
cudaError_t launch_one(const TrackArgs& a, int block, int grid, cudaStream_t s) {
  const int nwarps = block / 32;
  size_t sh = nwarps * sizeof(WarpStage) + sizeof(float) * (a.nx + a.ny + 4);
  if (SM) sh += sizeof(float2) * a.nc * a.ng;
  if (ST) sh += (sizeof(unsigned long long) + sizeof(double)) * a.nc * a.ng;
  if (PF) sh += pf_smem(block);
  if (sh > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_track<GEOM, SM, MG, CF, ST, PF>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    if (e != cudaSuccess) return e;
  }
  IMC_LAUNCH_PDL((k_track<GEOM, SM, MG, CF, ST, PF>), grid, block, sh, s, a);
  return cudaGetLastError();
}

// the block tallies are built only with the shared-memory cell table (small meshes)
template <int GEOM, bool MG, bool CF, bool PF>
cudaError_t launch_pf(const TrackArgs& a, int block, int grid, bool sm, bool st, cudaStream_t s) {
  if (sm && st) return launch_one<GEOM, true, MG, CF, true, PF>(a, block, grid, s);
  return sm ? launch_one<GEOM, true, MG, CF, false, PF>(a, block, grid, s)
            : launch_one<GEOM, false, MG, CF, false, PF>(a, block, grid, s);
}

template <int GEOM, bool MG, bool CF = false>
cudaError_t launch_geom(const TrackArgs& a, int block, int grid, bool sm, bool st, bool pf, cudaStream_t s) {
  return pf ? launch_pf<GEOM, MG, CF, true>(a, block, grid, sm, st, s)
            : launch_pf<GEOM, MG, CF, false>(a, block, grid, sm, st, s);
}

// ---------------------------------------------------------------------------------
// Event-by-event form (the textbook event-based loop): one launch advances every live
// history by one event; the histories still alive are compacted into the next launch's list.
// The history state lives in the bank (position, direction, weight, cell) and in scratch
// arrays (event count, distance to census, weight at the visit's start, w*s); the physics is
// history_event, so a history follows exactly the path and draws it follows in k_track.
// ---------------------------------------------------------------------------------
struct EventScratch {
  uint32_t* live[2];        // lists of live bank indices
  unsigned* count;          // [2] their lengths
  uint32_t* ev; float* dcen; float* w_in; double* acc_wd;  // [capacity]
};

// The histories that move (as k_track's refill decides) into list 0, with their scratch state.
template <bool MG2CF>
__global__ void k_event_init(TrackArgs a, EventScratch e) {
  const float dtk = a.dt_dev ? (float)*a.dt_dev : a.dt;
  const uint32_t n = (uint32_t)*a.n_dev;
  const float weight_floor = (float)(a.floor_coef * (*a.wsum) / (double)(n > 0 ? n : 1));
  const int lane = threadIdx.x & 31;
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t trips = (n + stride - 1) / stride;  // uniform: every lane reaches the ballot
  for (uint32_t it = 0; it < trips; ++it) {
    const uint32_t k = it * stride + blockIdx.x * blockDim.x + threadIdx.x;
    bool moves = false;
    if (k < n) {
      const float w = a.w[k];
      const float dc = (dtk - a.t[k]) * (float)C_LIGHT;
      moves = (MG2CF ? w > weight_floor : w > 0.f) && dc > 0.f;
      if (moves) { e.ev[k] = 0u; e.dcen[k] = dc; e.w_in[k] = w; e.acc_wd[k] = 0.0; }
    }
    const unsigned m = __ballot_sync(FULL, moves);
    unsigned base = 0;
    if (lane == 0 && m) base = atomicAdd(e.count, (unsigned)__popc(m));
    base = __shfl_sync(FULL, base, 0);
    if (moves) e.live[0][base + __popc(m & ((1u << lane) - 1u))] = k;
  }
}

template <int GEOM, bool MG, bool CF>
__global__ void __launch_bounds__(256) k_event(TrackArgs a, EventScratch e, int cur) {
  const uint32_t stepk = a.step_dev ? *a.step_dev : a.step;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ unsigned blk_cnt[B_N];
  __shared__ unsigned long long blk_esc[4];
  WarpStage* stages = reinterpret_cast<WarpStage*>(smem);
  const int nwarps = blockDim.x >> 5;
  float* E1 = reinterpret_cast<float*>(stages + nwarps);
  float* E2 = E1 + (a.nx + 1);
  for (int q = threadIdx.x; q <= a.nx; q += blockDim.x) E1[q] = a.e1[q];
  for (int q = threadIdx.x; q <= a.ny; q += blockDim.x) E2[q] = a.e2[q];
  if (threadIdx.x < B_N) blk_cnt[threadIdx.x] = 0u;
  if (threadIdx.x < 4) blk_esc[threadIdx.x] = 0ull;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  WarpStage* st = stages + (threadIdx.x >> 5);
  const uint32_t n = (uint32_t)*a.n_dev;  // the whole bank: the weight floor is k_track's
  const float weight_floor = (float)(a.floor_coef * (*a.wsum) / (double)(n > 0 ? n : 1));
  const double inv_q = fx_inv_quantum(*a.wsum);
  const uint32_t n_in = e.count[cur];
  const uint32_t* live_in = e.live[cur];
  uint32_t* live_out = e.live[cur ^ 1];
  unsigned* n_out = e.count + (cur ^ 1);
  unsigned s_bd = 0, s_sc = 0;
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t trips = (n_in + stride - 1) / stride;
  for (uint32_t it = 0; it < trips; ++it) {
    const uint32_t i = it * stride + blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n_in;
    EvOut o{false, 0, 0.0, 0.0, false, 0, false};
    bool alive = false;
    uint32_t pid = 0;
    if (active) {
      Hist h;
      pid = live_in[i];
      h.pid = pid;
      h.x = a.p1[pid]; h.u = a.d1[pid]; h.w = a.w[pid];
      h.y = 0.f; h.v = 0.f;
      if (GEOM == G_XY || GEOM == G_RZ) { h.y = a.p2[pid]; h.v = a.d2[pid]; }
      h.grp = MG ? a.group[pid] : 0;
      const int c = a.cell[pid];
      h.ev = e.ev[pid]; h.dcen = e.dcen[pid]; h.w_in = e.w_in[pid]; h.acc_wd = e.acc_wd[pid];
#ifdef IMC_CHECKED
      // bounds-checked build: an entry outside the mesh or group range, or with a non-finite
      // weight or position, is reported and dropped from the loop untouched
      if (c < 0 || c >= a.nc || (MG && (h.grp < 0 || h.grp >= a.ng)) || !isfinite(h.w) || !isfinite(h.x) ||
          !isfinite(h.dcen)) {
        atomicOr(a.flags, (int)IMC_FLAG_BOUNDS);
        o.finished = true;
      } else
#endif
      {
        h.cj = c / a.nx; h.ci = c - h.cj * a.nx;
        h.tab = __ldg(a.sass + (MG ? c + a.nc * h.grp : c));
        history_event<GEOM, false, MG, CF>(a, h, o, E1, E2, nullptr, blk_cnt, blk_esc, a.dep_fx, stepk,
                                           weight_floor, inv_q, s_bd, s_sc);
      }
      if (!o.finished) {
        alive = true;
        a.p1[pid] = h.x; a.d1[pid] = h.u; a.w[pid] = h.w;
        if (GEOM == G_XY || GEOM == G_RZ) { a.p2[pid] = h.y; a.d2[pid] = h.v; }
        a.cell[pid] = h.ci + a.nx * h.cj;
        e.ev[pid] = h.ev; e.dcen[pid] = h.dcen; e.w_in[pid] = h.w_in; e.acc_wd[pid] = h.acc_wd;
      }
    }
    // survivors into the next list (warp-aggregated append)
    const unsigned m = __ballot_sync(FULL, alive);
    unsigned base = 0;
    if (lane == 0 && m) base = atomicAdd(n_out, (unsigned)__popc(m));
    base = __shfl_sync(FULL, base, 0);
    if (alive) live_out[base + __popc(m & ((1u << lane) - 1u))] = pid;
    const unsigned long long ud = o.flush ? fx_units(o.f_lost, inv_q) : 0ull;
    warp_tally_fx(o.flush, o.flush_cell, ud, o.flush ? o.f_wd : 0.0, a.dep_fx, a.si, st);
  }
  const unsigned long long t_bd = warp_sum_u(s_bd), t_sc = warp_sum_u(s_sc);
  if (lane == 0) {
    if (t_bd) atomicAdd(a.stats + S_BOUNDARY, t_bd);
    if (t_sc) atomicAdd(a.stats + S_SCATTER, t_sc);
    if (t_bd + t_sc) atomicAdd(a.stats + S_EVENTS, t_bd + t_sc);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned long long cen = blk_cnt[B_CENSUS], cap = blk_cnt[B_CAP], capt = blk_cnt[B_CAPTURE];
    if (cen) atomicAdd(a.stats + S_CENSUS, cen);
    if (capt) atomicAdd(a.stats + S_CAPTURE, capt);
    if (cen + cap + capt) atomicAdd(a.stats + S_EVENTS, cen + cap + capt);
    if (blk_cnt[B_FLOOR]) atomicAdd(a.stats + S_FLOOR, (unsigned long long)blk_cnt[B_FLOOR]);
    if (blk_cnt[B_REFLECT]) atomicAdd(a.stats + S_REFLECT, (unsigned long long)blk_cnt[B_REFLECT]);
    if (cap) atomicAdd(a.stats + S_CAP, cap);
    if (blk_cnt[B_ESCAPE]) atomicAdd(a.stats + S_ESCAPE, (unsigned long long)blk_cnt[B_ESCAPE]);
  }
  if (threadIdx.x < 4 && blk_esc[threadIdx.x] != 0ull) atomicAdd(a.esc_fx + threadIdx.x, blk_esc[threadIdx.x]);
}

template <int GEOM, bool MG, bool CF>
cudaError_t launch_event(const TrackArgs& a, const EventScratch& e, int cur, int block, int grid, cudaStream_t s) {
  const size_t sh = (block / 32) * sizeof(WarpStage) + sizeof(float) * (a.nx + a.ny + 4);
  if (sh > 48 * 1024) {
    cudaError_t err = cudaFuncSetAttribute(k_event<GEOM, MG, CF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    if (err != cudaSuccess) return err;
  }
  k_event<GEOM, MG, CF><<<grid, block, sh, s>>>(a, e, cur);
  return cudaGetLastError();
}

cudaError_t launch_event_geom(const TrackArgs& a, int geom, const EventScratch& e, int cur, int block, int grid,
                              cudaStream_t s) {
  if (a.ng > 1) {
    switch (geom) {
      case G_SPHERE: return launch_event<G_SPHERE, true, false>(a, e, cur, block, grid, s);
      case G_XY: return launch_event<G_XY, true, false>(a, e, cur, block, grid, s);
      case G_RZ: return launch_event<G_RZ, true, false>(a, e, cur, block, grid, s);
      default: return cudaErrorInvalidValue;
    }
  }
  if (a.cf_rate) {
    switch (geom) {
      case G_SLAB: return launch_event<G_SLAB, false, true>(a, e, cur, block, grid, s);
      case G_SPHERE: return launch_event<G_SPHERE, false, true>(a, e, cur, block, grid, s);
      case G_XY: return launch_event<G_XY, false, true>(a, e, cur, block, grid, s);
      case G_RZ: return launch_event<G_RZ, false, true>(a, e, cur, block, grid, s);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (geom) {
    case G_SLAB: return launch_event<G_SLAB, false, false>(a, e, cur, block, grid, s);
    case G_SPHERE: return launch_event<G_SPHERE, false, false>(a, e, cur, block, grid, s);
    case G_XY: return launch_event<G_XY, false, false>(a, e, cur, block, grid, s);
    case G_RZ: return launch_event<G_RZ, false, false>(a, e, cur, block, grid, s);
    default: return cudaErrorInvalidValue;
  }
}

// Fixed-point tallies to the FP64 outputs: deposition per unit volume per (group, cell),
// escaped energy per side and (MG) per group, and the path-length intensity.
// cellf[q] = (1/V, si factor): a factor > 0 is 1/(sigma_a V dt) and the cell's intensity is
// its deposited energy times it (the sum over the cell's flights of (w - w') / (sigma_a V dt));
// < 0 is -1/(V dt), the cell has no absorption and si holds the raw sum of w*s.
__global__ void k_tally_finalize(TrackArgs a) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const double W = *a.wsum;
  const int ncg = a.nc * a.ng;
  if (q < ncg) {
    const double2 cf = a.cellf[q];
    const double E = fx_energy(a.dep_fx[q], W);
    a.dep[q] = E * cf.x;
    a.si[q] = cf.y > 0.0 ? E * cf.y : a.si[q] * -cf.y;
  }
  else if (q < ncg + 4) a.escaped[q - ncg] = fx_energy(a.esc_fx[q - ncg], W);
  else if (q < ncg + 4 + a.ng && a.ng > 1) a.escaped_group[q - ncg - 4] = fx_energy(a.esc_fx[q - ncg], W);
}

}  // namespace

cudaError_t imc_launch_tally_finalize(const TrackArgs& a, cudaStream_t s) {
  ++g_imc_launches;
  const int n = a.nc * a.ng + 4 + a.ng;
  IMC_LAUNCH_PDL(k_tally_finalize, (n + 255) / 256, 256, 0, s, a);
  return cudaGetLastError();
}

size_t imc_event_scratch_bytes(long long capacity) {
  const size_t cap = (size_t)(capacity > 0 ? capacity : 1);
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  return al(8) + 2 * al(4 * cap) + 3 * al(4 * cap) + al(8 * cap);
}

cudaError_t imc_run_event_tracking(const TrackArgs& a, int geom, void* scratch, long long capacity,
                                   long long n_upper, int block, int sms, long long max_launches, bool* cap_hit,
                                   cudaStream_t s) {
  const size_t cap = (size_t)(capacity > 0 ? capacity : 1);
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  char* p = static_cast<char*>(scratch);
  EventScratch e;
  e.count = reinterpret_cast<unsigned*>(p); p += al(8);
  e.live[0] = reinterpret_cast<uint32_t*>(p); p += al(4 * cap);
  e.live[1] = reinterpret_cast<uint32_t*>(p); p += al(4 * cap);
  e.ev = reinterpret_cast<uint32_t*>(p); p += al(4 * cap);
  e.dcen = reinterpret_cast<float*>(p); p += al(4 * cap);
  e.w_in = reinterpret_cast<float*>(p); p += al(4 * cap);
  e.acc_wd = reinterpret_cast<double*>(p);
  *cap_hit = false;
  cudaError_t err = cudaMemsetAsync(e.count, 0, 8, s);
  if (err != cudaSuccess) return err;
  const bool mg2cf = (a.ng > 1 && geom >= G_XY) || a.cf_rate != nullptr;
  const int init_grid = (int)std::min<long long>((n_upper + 255) / 256 + 1, (long long)sms * 16);
  ++g_imc_launches;
  if (mg2cf) k_event_init<true><<<init_grid, 256, 0, s>>>(a, e);
  else k_event_init<false><<<init_grid, 256, 0, s>>>(a, e);
  if ((err = cudaGetLastError()) != cudaSuccess) return err;
  // one launch per event; every 8 launches the live count comes back to size the grid and to
  // stop (each launch advances every live history by one event, so at most max_events + 1
  // launches are needed)
  long long bound = n_upper;
  int cur = 0;
  for (long long it = 0; bound > 0; ++it) {
    if (it > max_launches) { *cap_hit = true; break; }
    if ((err = cudaMemsetAsync(e.count + (cur ^ 1), 0, 4, s)) != cudaSuccess) return err;
    const int grid = (int)std::max<long long>(1, std::min<long long>((bound + block - 1) / block, (long long)sms * 8));
    ++g_imc_launches;
    if ((err = launch_event_geom(a, geom, e, cur, block, grid, s)) != cudaSuccess) return err;
    cur ^= 1;
    if ((it & 7) == 7) {
      unsigned live = 0;
      if ((err = cudaMemcpyAsync(&live, e.count + cur, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return err;
      if ((err = cudaStreamSynchronize(s)) != cudaSuccess) return err;
      bound = live;
    }
  }
  return cudaSuccess;
}

cudaError_t imc_launch_track(const TrackArgs& a, int geom, int block, int grid, bool sm, bool st, bool pf,
                             cudaStream_t s) {
  ++g_imc_launches;
  if (a.ng > 1) {  // multigroup: 2-D (MG_IMC/MG_IMC2D.py) and the 1-D sphere (MG_IMC/MG_IMC1D.py)
    switch (geom) {
      case G_SPHERE: return launch_geom<G_SPHERE, true>(a, block, grid, sm, st, pf, s);
      case G_XY: return launch_geom<G_XY, true>(a, block, grid, sm, st, pf, s);
      case G_RZ: return launch_geom<G_RZ, true>(a, block, grid, sm, st, pf, s);
      default: return cudaErrorInvalidValue;
    }
  }
  if (a.cf_rate) {  // Carter-Forest, gray
    switch (geom) {
      case G_SLAB: return launch_geom<G_SLAB, false, true>(a, block, grid, sm, st, pf, s);
      case G_SPHERE: return launch_geom<G_SPHERE, false, true>(a, block, grid, sm, st, pf, s);
      case G_XY: return launch_geom<G_XY, false, true>(a, block, grid, sm, st, pf, s);
      case G_RZ: return launch_geom<G_RZ, false, true>(a, block, grid, sm, st, pf, s);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (geom) {
    case G_SLAB: return launch_geom<G_SLAB, false>(a, block, grid, sm, st, pf, s);
    case G_SPHERE: return launch_geom<G_SPHERE, false>(a, block, grid, sm, st, pf, s);
    case G_XY: return launch_geom<G_XY, false>(a, block, grid, sm, st, pf, s);
    case G_RZ: return launch_geom<G_RZ, false>(a, block, grid, sm, st, pf, s);
    default: return cudaErrorInvalidValue;
  }
}
