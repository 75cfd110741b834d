// imc_adjoint.cu — vector-Jacobian product of one step's deposition tally with respect to
// the per-cell opacity sigma, for 2-D gray steps (xy, rz; IMC/IMC2D.py:711-1107 events).
//
// Tally and its derivative.  For cotangent g, the step's score is T = sum_c g_c dep_c and
// a history contributes L = sum_i a_i d_i over its segments i (cell c_i, length s_i,
// entering weight w_i, leaving weight w_{i+1} = w_i exp(-sigma_a,c_i s_i), deposit
// d_i = w_i - w_{i+1}, a_i = g_{c_i} / V_{c_i}).  Two effects of sigma_j:
//  * implicit capture (path-length / pathwise term): holding the path fixed,
//      dL/dsigma_a,j = sum_{k in j} s_k (a_k w_{k+1} + L_{<=k} - L),
//    L_{<=k} = sum_{i<=k} a_i d_i (what the history scored before it left segment k);
//  * effective scatter (likelihood-ratio term): the path density carries
//    exp(-sigma_s,j s_k) per segment in j and a factor sigma_s,j per scatter in j, so
//      dE[L]/dsigma_s,j = E[ sum_{k in j} (L - L_{<k}) (-s_k + [scatter at k] / sigma_s,j) ],
//    with only the score accrued from segment k on (earlier scores are independent of it).
//    A cell whose scatter distance is capped (sigma_s L > 1e4) or off (sigma_s <= 1e-12)
//    samples independently of sigma_s and contributes no such term.
//  * Fleck factor: sigma_a = f sigma, f = 1 / (1 + b sigma), so dsigma_a/dsigma = f^2 and
//    dsigma_s/dsigma = 1 - f^2.
// Replay.  Each lane tracks a history twice from its Philox counter (bank index, event,
// step, TAG_TRANSPORT): pass 0 computes L, pass 1 accumulates the per-visit sums
// gp = sum s_k (a_k w_{k+1} + L_{<=k} - L), gs1 = sum (L - L_{<k}) s_k,
// gs2 = sum_{scatters} (L - L_{<k}) and flushes f^2 gp + (1 - f^2)(gs2 / sigma_s - gs1)
// into grad[cell] (warp-aggregated FP64) when the history leaves the cell.  No path is
// stored; the bank is read, never written.  The event arithmetic is the forward tracking
// kernel's, so each replay follows the forward step's path.
#include "imc_device.cuh"
#include "imc_internal.h"

using namespace imcdev;

namespace {

template <int GEOM>
__global__ void __launch_bounds__(256) k_adjoint(AdjointArgs A) {
  const TrackArgs& a = A.t;
  extern __shared__ __align__(16) unsigned char smem[];
  WarpStage* stages = reinterpret_cast<WarpStage*>(smem);
  const int nwarps = blockDim.x >> 5;
  float* E1 = reinterpret_cast<float*>(stages + nwarps);
  float* E2 = E1 + (a.nx + 1);
  for (int q = threadIdx.x; q <= a.nx; q += blockDim.x) E1[q] = a.e1[q];
  for (int q = threadIdx.x; q <= a.ny; q += blockDim.x) E2[q] = a.e2[q];
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  WarpStage* st = stages + (threadIdx.x >> 5);
  const uint32_t n = (uint32_t)*a.n_dev;
  const float c_light = (float)C_LIGHT;
  const float weight_floor = (float)(1e-10 * (*a.wsum) / (double)(n > 0 ? n : 1));
  const float ss_thr = 1e-12f;

  uint32_t chunk_next = 0, chunk_end = 0;
  bool drained = false;

  bool has = false;
  int phase = 0;
  uint32_t pid = 0, ev = 0;
  float x = 0, y = 0, u = 0, v = 0, w = 0, dcen = 0;
  int ci = 0, cj = 0;
  double L = 0.0, Lcum = 0.0, gp = 0.0, gs1 = 0.0, gs2 = 0.0;

  auto load = [&](uint32_t p) {
    w = a.w[p];
    dcen = (a.dt - a.t[p]) * c_light;
    x = a.p1[p]; u = a.d1[p]; y = a.p2[p]; v = a.d2[p];
    const int c = a.cell[p];
    cj = c / a.nx; ci = c - cj * a.nx;
    ev = 0;
  };

  for (;;) {
    unsigned need = __ballot_sync(FULL, !has);
    while (need && !drained) {
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
        if (base >= (unsigned long long)n) { drained = true; break; }
        chunk_next = (uint32_t)base;
        chunk_end = (uint32_t)min(base + claim, (unsigned long long)n);
      }
      const uint32_t avail = chunk_end - chunk_next;
      const uint32_t rank = __popc(need & lt_mask);
      if (!has && rank < avail) {
        pid = chunk_next + rank;
        load(pid);
        if (w > 0.f && dcen > 0.f) {
          has = true; phase = 0; L = 0.0;
        }
      }
      chunk_next += min((uint32_t)__popc(need), avail);
      need = __ballot_sync(FULL, !has);
    }
    if (!__any_sync(FULL, has)) break;

    bool flush = false;
    int flush_cell = 0;
    double f_gp = 0.0, f_gs1 = 0.0, f_gs2 = 0.0;
    if (has) {
      const int c = ci + a.nx * cj;
      const float2 q = __ldg(a.sass + c);
      const float sa = q.x, ss = q.y;
      bool finished = false;
      if (ev >= (uint32_t)a.max_events) {
        finished = true;  // cap: the history stops where it is, in both passes
      } else {
        const U4 r = draw_rk(a.rk, a.id_base + pid, ev, a.step, TAG_TRANSPORT);
        ++ev;
        float d, sb, Lc, xn = x, yn = y, un = u, vn = v;
        int evt, cross = X_NONE;
        float s_rin = BIGF, s_rout = BIGF, s_zlo = BIGF, s_zhi = BIGF, st_ = 0.f, sx = BIGF, sy = BIGF;
        if (GEOM == G_XY) {
          const float xl = E1[ci], xr = E1[ci + 1], yl = E2[cj], yr = E2[cj + 1];
          Lc = fminf(xr - xl, yr - yl);
          if (u > 0.f) sx = __fdividef(xr - x, u); else if (u < 0.f) sx = __fdividef(xl - x, u);
          if (v > 0.f) sy = __fdividef(yr - y, v); else if (v < 0.f) sy = __fdividef(yl - y, v);
          sx = fmaxf(sx, 0.f); sy = fmaxf(sy, 0.f);
          sb = fminf(sx, sy);
        } else {
          const float rin = E1[ci], rout = E1[ci + 1], zlo = E2[cj], zhi = E2[cj + 1];
          Lc = fminf(rout - rin, zhi - zlo);
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
        // effective scatter, as the forward kernel (cap sigma_s L > 1e4; series test)
        float ds = BIGF;
        const bool capped = ss * Lc > 10000.0f;
        const bool scores = !capped && ss > ss_thr;  // sampling depends on sigma_s here
        {
          const float sig = capped ? 10000.0f / Lc : (ss > ss_thr ? ss : 0.f);
          if (sig > 0.f) {
            const float s_other = fminf(sb, dcen);
            const double t = (double)sig * (double)s_other;
            bool may = true;
            if (t < 0.01) {
              const double thr = 1.0 - t * (1.0 - t * (0.5 - t * (1.0 / 6.0)));
              may = u01d(r.x) > thr;
            }
            if (may) ds = capped ? neglog_u(r.x) * (Lc * 1e-4f) : __fdividef(neglog_u(r.x), ss);
          }
        }
        d = sb; evt = EV_BOUNDARY;
        if (ds < d) { d = ds; evt = EV_SCATTER; }
        if (dcen < d) { d = dcen; evt = EV_CENSUS; }
        if (GEOM == G_XY) {
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
        const float wn = w * __expf(-sa * d);
        const double dd = (double)w - (double)wn;  // exact
        const double ac = A.cot[c] * __ldg(&a.cellf[c].x);
        if (phase == 0) {
          L += ac * dd;
        } else {
          const double Lprev = Lcum;
          Lcum += ac * dd;
          gp += (double)d * (ac * (double)wn + Lcum - L);
          if (scores) {
            const double R = L - Lprev;
            gs1 += R * (double)d;
            if (evt == EV_SCATTER) gs2 += R;
          }
        }
        dcen -= d;
        if (wn <= weight_floor) {
          finished = true;  // IMC/IMC2D.py:1043-1047: the history stops at the floor
        } else {
          w = wn; x = xn; y = yn; u = un; v = vn;
          if (cross != X_NONE) {
            if (phase == 1) {
              flush = true; flush_cell = c; f_gp = gp; f_gs1 = gs1; f_gs2 = gs2;
              gp = 0.0; gs1 = 0.0; gs2 = 0.0;
            }
            int ni = ci, nj = cj;
            if (cross == X_IP) ++ni; else if (cross == X_IM) --ni; else if (cross == X_JP) ++nj; else --nj;
            int side = -1;
            if (ni < 0) side = 0; else if (ni >= a.nx) side = 1; else if (nj < 0) side = 2; else if (nj >= a.ny) side = 3;
            if (side >= 0) {
              if ((a.reflect_mask >> side) & 1) {
                if (side < 2) { u = -u; ni = side == 0 ? 0 : a.nx - 1; }
                else { v = -v; nj = side == 2 ? 0 : a.ny - 1; }
              } else {
                w = 0.f;
                finished = true;
                ni = ci; nj = cj;
              }
            }
            ci = ni; cj = nj;
          }
          if (!finished && !(w > 0.f)) finished = true;
          if (!finished && !(dcen > 0.f)) finished = true;
        }
      }
      if (finished) {
        if (phase == 0) {
          // replay the same history for the sensitivities
          load(pid);
          phase = 1; Lcum = 0.0; gp = 0.0; gs1 = 0.0; gs2 = 0.0;
        } else {
          if (!flush && (gp != 0.0 || gs1 != 0.0 || gs2 != 0.0)) {
            flush = true; flush_cell = c; f_gp = gp; f_gs1 = gs1; f_gs2 = gs2;
          }
          gp = 0.0; gs1 = 0.0; gs2 = 0.0;
          has = false;
        }
      }
    }
    double val = 0.0;
    if (flush) {
      const double sig = A.sig64[flush_cell];
      const double f = sig > 0.0 ? A.sa64[flush_cell] / sig : 1.0;
      const double ssd = A.ss64[flush_cell];
      val = f * f * f_gp;
      if (ssd > 0.0 && (f_gs1 != 0.0 || f_gs2 != 0.0)) val += (1.0 - f * f) * (f_gs2 / ssd - f_gs1);
    }
    warp_tally1(flush, flush_cell, val, A.grad, st);
  }
}

template <int GEOM>
cudaError_t launch_adj(const AdjointArgs& a, int block, int grid, cudaStream_t s) {
  const size_t sh = (size_t)(block / 32) * sizeof(WarpStage) + sizeof(float) * (a.t.nx + a.t.ny + 4);
  if (sh > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(k_adjoint<GEOM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    if (e != cudaSuccess) return e;
  }
  k_adjoint<GEOM><<<grid, block, sh, s>>>(a);
  return cudaGetLastError();
}

}  // namespace

cudaError_t imc_launch_adjoint(const AdjointArgs& a, int geom, int block, int grid, cudaStream_t s) {
  ++g_imc_launches;
  switch (geom) {
    case G_XY: return launch_adj<G_XY>(a, block, grid, s);
    case G_RZ: return launch_adj<G_RZ>(a, block, grid, s);
    default: return cudaErrorInvalidValue;
  }
}
