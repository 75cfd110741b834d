// imc_batch_plan.cu — per-cell and per-instance FP64 work of the batched 1-D slab engine.
//
// Compiled without FMA contraction, like imc_bookkeeping.cu: each instance's Fleck
// factors, source counts (ceil(N E_c / E)), comb targets and ledger sums are computed with
// the operations, in the order, of the single-problem kernels, so an instance of the batch
// reproduces its single-problem run.  Per-instance kernels run one 1024-thread block per
// instance (grid = K); per-cell kernels run one thread per cell of the whole batch.
//
//   Fleck factor     IMC/IMC1D.py:933-938
//   material update  IMC/IMC1D.py:1021-1035 (e += dep - emitted/V; Tr from the intensity)
//   emission plan    IMC/IMC1D.py:251-291 (ceil counts, linear-T tilt)
//   boundary         IMC/IMC1D.py:319-329
//   initial census   IMC/IMC1D.py:220-248
//   comb targets     IMC/IMC1D.py:786-799
#include <cmath>
#include "imc_batch.h"
#include "imc_block.cuh"
#include "imc_device.cuh"

using namespace imcdev;
using namespace imcblk;

namespace {

__device__ __forceinline__ int inst_of_cell(const int* cell_off, int K, int c) {
  int lo = 0, hi = K - 1;  // last k with cell_off[k] <= c
  while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (cell_off[mid] <= c) lo = mid; else hi = mid - 1; }
  return lo;
}

// cell -> instance map, FP32 edges, dx, T = T0, e = cv T0, slot capacities
__global__ void k_bsetup(BatchArgs a, const double* T0) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < a.n_cells + a.K) a.ef[q] = (float)a.edges[q];
  if (q < a.n_cells) {
    const int k = inst_of_cell(a.cell_off, a.K, q);
    a.cell_inst[q] = k;
    const int e0 = q + k;
    a.vol[q] = a.edges[e0 + 1] - a.edges[e0];
    a.T[q] = T0[q];
    a.e[q] = a.cv[k] * T0[q];
  }
  if (q < a.K) {
    const int k = q;
    const long long nck = a.cell_off[k + 1] - a.cell_off[k];
    long long sides = 0;
    for (int side = 0; side < 2; ++side) if (a.face_T[2 * k + side] > 0.0) ++sides;
    const long long new_max = sides * a.n_boundary[k] + a.n_target[k] + nck;
    a.census_cap[k] = (a.slot_off[k + 1] - a.slot_off[k]) - new_max;
    if (a.census_cap[k] < a.n_target[k] + nck) atomicOr(a.flags, (int)IMC_FLAG_COMB_OVERFLOW);
  }
}

// Fleck factor (and, with update, the material update first) for every cell of the batch.
__global__ void k_bmaterial_fleck(BatchArgs a, int update) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.n_cells) return;
  const int k = a.cell_inst[c];
  const double V = a.vol[c];
  const double cv = a.cv[k];
  double T;
  if (update) {
    // deposition of the step from its fixed-point sum (units of wsum * 2^-60)
    const double E = fx_energy(a.dep_fx[c], a.wsum[k]);
    const double dep = E * (1.0 / V);  // as the single-problem finalize
    a.dep[c] = dep;
    const double e = a.e[c] + dep - a.emitted[c] / V;
    a.e[c] = e;
    // path-length intensity: an absorbing cell's from its deposition, E / (sigma_a V dt); the
    // others' from their w*s tally, times 1 / (V dt) (the single-problem finalize)
    const double cfy = a.cellf[c].y;
    const double si = cfy > 0.0 ? E * cfy : a.si[c] * -cfy;
    a.si[c] = si;
    const double x = si / A_RAD / C_LIGHT;
    a.tr[c] = x > 0.0 ? sqrt(sqrt(x)) : 0.0;
    T = e / cv;  // e = cv T
    a.T[c] = T;
  } else {
    T = a.T[c];
  }
  const double sig = a.op_a[k] * pow(T, a.op_p[k]);
  if (!isfinite(T) || !(T > 0.0) || !isfinite(sig) || !(cv > 0.0)) atomicOr(a.flags, (int)IMC_FLAG_NONFINITE);
  const double beta = 4.0 * A_RAD * pow3(T) / cv;
  double f = 1.0 / (1.0 + a.theta * beta * sig * C_LIGHT * a.dt);
  f = fmin(1.0, fmax(0.0, f));
  const double ss = sig * (1.0 - f);
  const double sa = sig * f;
  a.sass[c] = make_float2((float)sa, (float)ss);
  const double iv = 1.0 / V;
  a.cellf[c] = make_double2(iv, sa > 1e-10 ? 1.0 / (sa * V * a.dt) : -1.0 / (V * a.dt));
  a.emit_E[c] = A_RAD * C_LIGHT * pow4(fmax(T, 0.0)) * sa * a.dt * V;
}

// Per-instance source plan: emission counts/weights/offsets, linear-T slopes, boundary
// faces, this step's bank layout inside the instance's slot range.  Also clears the
// instance's tallies and accumulators for the step.
__global__ void __launch_bounds__(NT) k_bplan(BatchArgs a) {
  __shared__ double red[NT];
  __shared__ long long sh[NT];
  const int k = blockIdx.x, t = threadIdx.x;
  const int cb = a.cell_off[k], nc = a.cell_off[k + 1] - cb;
  const double* e1 = a.edges + cb + k;
  const double* T = a.T + cb;
  for (int c = t; c < nc; c += NT) {
    a.dep_fx[cb + c] = 0ull; a.si[cb + c] = 0.0; a.ecen[cb + c] = 0.0; a.ncopy[cb + c] = 0.0;
  }
  const long long n_emit = plan_volume(a.emit_E + cb, a.n_target[k], nc, 1, nc, a.emit_n + cb,
                                       a.emit_off + cb + k, a.emit_w + cb, a.emitted + cb, red, sh);
  const double e_emit = block_canon_sum(a.emitted + cb, nc, red);
  // centred slopes of T, zeroed when an edge value goes negative (IMC/IMC1D.py:254-262)
  for (int i = t; i < nc; i += NT) {
    double s = 0.0;
    if (nc > 1) {
      auto dx = [&](int q) { return e1[q + 1] - e1[q]; };
      if (i == 0) s = (T[1] - T[0]) / (dx(1) + dx(0)) * 2.0;
      else if (i == nc - 1) s = (T[i] - T[i - 1]) / (dx(i) + dx(i - 1)) * 2.0;
      else s = (T[i + 1] - T[i - 1]) / (dx(i + 1) + dx(i - 1)) * 2.0;
      if (T[i] - s * dx(i) / 2.0 < 0.0) s = 0.0;
      else if (T[i] + s * dx(i) / 2.0 < 0.0) s = 0.0;
    }
    a.tilt[cb + i] = s;
  }
  if (t < 2) {
    const int side = t;
    const double Tf = a.face_T[2 * k + side];
    long long n = 0;
    float wq = 0.f;
    double e = 0.0;
    if (a.n_boundary[k] > 0) {
      const double area = 1.0;
      const double Et = (Tf > 0.0) ? A_RAD * C_LIGHT * Tf * Tf * Tf * Tf / 4.0 * area * a.dt : 0.0;
      if (Et > 0.0) {
        n = a.n_boundary[k];
        wq = (float)(Et / (double)n);
        e = (double)n * (double)wq;
      }
    }
    a.n_side[2 * k + side] = n; a.w_side[2 * k + side] = wq; a.e_side[2 * k + side] = e;
    a.esc_fx[2 * k + side] = 0ull;
  }
  __syncthreads();
  if (t == 0) {
    const long long nb = a.n_side[2 * k] + a.n_side[2 * k + 1];
    long long n_new = nb + n_emit;
    const long long cen = a.n_census[k];
    if (cen + n_new > a.slot_off[k + 1] - a.slot_off[k]) {
      // cannot happen while the census respects census_cap; never write outside the slots
      atomicOr(a.flags, (int)IMC_FLAG_COMB_OVERFLOW);
      a.n_side[2 * k] = a.n_side[2 * k + 1] = 0;
      n_new = 0;
    }
    a.n_new[k] = n_new;
    a.n_bank[k] = cen + n_new;
    a.e_emit[k] = e_emit;
    a.wsum[k] = 0.0; a.comb_after[k] = 0.0; a.copies_d[k] = 0.0;
    double* L = a.ledger + (size_t)k * IMC_BL_N;
    L[IMC_BL_BOUNDARY] = a.e_side[2 * k] + a.e_side[2 * k + 1];
    L[IMC_BL_EMISSION] = e_emit;
  }
}

// Per-instance initial census plan: E_c = a Tr^4 V, n_c = ceil(E_c / E N) (1-D rule).
__global__ void __launch_bounds__(NT) k_bic_plan(BatchArgs a, const double* tr) {
  __shared__ double red[NT];
  __shared__ long long sh[NT];
  const int k = blockIdx.x, t = threadIdx.x;
  const int cb = a.cell_off[k], nc = a.cell_off[k + 1] - cb;
  double* E = a.emit_E + cb;
  for (int c = t; c < nc; c += NT) E[c] = A_RAD * pow4(tr[cb + c]) * a.vol[cb + c];
  __syncthreads();
  const double Et = block_canon_sum(E, nc, red);
  const long long N = a.n_target[k];
  for (int c = t; c < nc; c += NT) {
    long long n = 0;
    if (N > 0) n = Et > 0.0 ? (long long)ceil(E[c] / Et * (double)N) : 0;
    a.emit_n[cb + c] = n;
    a.emit_w[cb + c] = n > 0 ? (float)(E[c] / (double)n) : 0.f;
  }
  __syncthreads();
  long long tot = block_scan_counts(a.emit_n + cb, a.emit_off + cb + k, nc, sh);
  if (t == 0) {
    if (tot > a.census_cap[k]) { atomicOr(a.flags, (int)IMC_FLAG_COMB_OVERFLOW); tot = 0; }
    a.n_new[k] = tot;
    a.n_bank[k] = tot;
    a.n_census[k] = 0;
    a.n_side[2 * k] = a.n_side[2 * k + 1] = 0;
  }
}

// Exclusive prefix sums over instances of the entries tracked and of the new particles.
__global__ void __launch_bounds__(NT) k_bprefix(BatchArgs a) {
  __shared__ long long sh[NT];
  block_scan_counts(a.n_bank, a.live_pref, a.K, sh);
  block_scan_counts(a.n_new, a.new_pref, a.K, sh);
  if (threadIdx.x == 0) *a.queue = 0ull;
}

// Per-instance comb targets: ew_c = ecen_c / max(1, rint(Nmax ecen_c / E)).
__global__ void __launch_bounds__(NT) k_bcomb_plan(BatchArgs a) {
  __shared__ double red[NT];
  const int k = blockIdx.x;
  const int cb = a.cell_off[k], nc = a.cell_off[k + 1] - cb;
  const double E = block_canon_sum(a.ecen + cb, nc, red);
  const long long nmax = a.n_max[k];
  for (int c = threadIdx.x; c < nc; c += NT) {
    const double ec = a.ecen[cb + c];
    double ew = 0.0;
    if (E > 0.0 && ec > 0.0) ew = ec / fmax(1.0, rint((double)nmax * ec / E));
    a.ew[cb + c] = ew;
  }
  if (threadIdx.x == 0) a.comb_before[k] = E;
}

// Per-instance energy ledger (IMC/IMC1D.py:1063-1074 plus the comb discrepancy), then the
// bank swap and step increment.  init: record the starting total only.
__global__ void __launch_bounds__(NT) k_bledger(BatchArgs a, int init) {
  __shared__ double red[NT];
  const int k = blockIdx.x, t = threadIdx.x;
  const int cb = a.cell_off[k], nc = a.cell_off[k + 1] - cb;
  double s = 0.0;
  for (int c = t; c < nc; c += NT) s += a.e[cb + c] * a.vol[cb + c];
  red[t] = s;
  __syncthreads();
  for (int h = NT / 2; h >= 1; h >>= 1) { if (t < h) red[t] += red[t + h]; __syncthreads(); }
  const double internal = red[0];
  __syncthreads();
  double rad;
  if (init) {
    // census energy of the initial bank (bank 0), which becomes the census
    const long long s0 = a.slot_off[k], n = a.n_new[k];
    double w = 0.0;
    for (long long q = t; q < n; q += NT) w += (double)a.bank[0].w[s0 + q];
    red[t] = w;
    __syncthreads();
    for (int h = NT / 2; h >= 1; h >>= 1) { if (t < h) red[t] += red[t + h]; __syncthreads(); }
    rad = red[0];
  } else {
    rad = a.comb_after[k];
  }
  if (t == 0) {
    double* L = a.ledger + (size_t)k * IMC_BL_N;
    const double total = internal + rad;
    if (init) {
      a.n_census[k] = a.n_new[k];
      for (int f = 0; f < IMC_BL_N; ++f) L[f] = 0.0;
      L[IMC_BL_TOTAL] = total; L[IMC_BL_PREV] = total;
      L[IMC_BL_INTERNAL] = internal; L[IMC_BL_RADIATION] = rad;
    } else {
      const double prev = L[IMC_BL_TOTAL];
      const double escaped = fx_energy(a.esc_fx[2 * k] + a.esc_fx[2 * k + 1], a.wsum[k]);
      const double disc = a.comb_before[k] - a.comb_after[k];
      const double closure = total - prev - L[IMC_BL_BOUNDARY] + escaped + disc;
      L[IMC_BL_PREV] = prev; L[IMC_BL_TOTAL] = total;
      L[IMC_BL_INTERNAL] = internal; L[IMC_BL_RADIATION] = rad;
      L[IMC_BL_ESCAPED] = escaped; L[IMC_BL_COMB_DISC] = disc; L[IMC_BL_CLOSURE] = closure;
      const double rel = fabs(closure) / fmax(fabs(total), 1e-300);
      if (rel > L[IMC_BL_MAX_REL]) L[IMC_BL_MAX_REL] = rel;
    }
  }
  if (!init && k == 0 && t == 0) {
    // the comb wrote the census into the other bank; nothing after this kernel reads sel
    *a.sel = 1 - *a.sel;
    *a.step = *a.step + 1u;
  }
}

}  // namespace

cudaError_t imc_batch_launch_setup(const BatchArgs& a, const double* T0, cudaStream_t s) {
  ++g_imc_launches;
  const int n = a.n_cells + a.K;
  k_bsetup<<<(n + 255) / 256, 256, 0, s>>>(a, T0);
  return cudaGetLastError();
}
cudaError_t imc_batch_launch_material_fleck(const BatchArgs& a, int update, cudaStream_t s) {
  ++g_imc_launches;
  k_bmaterial_fleck<<<(a.n_cells + 255) / 256, 256, 0, s>>>(a, update);
  return cudaGetLastError();
}
cudaError_t imc_batch_launch_plan(const BatchArgs& a, cudaStream_t s) {
  ++g_imc_launches;
  k_bplan<<<a.K, NT, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t imc_batch_launch_ic_plan(const BatchArgs& a, const double* tr, cudaStream_t s) {
  ++g_imc_launches;
  k_bic_plan<<<a.K, NT, 0, s>>>(a, tr);
  return cudaGetLastError();
}
cudaError_t imc_batch_launch_prefix(const BatchArgs& a, cudaStream_t s) {
  ++g_imc_launches;
  k_bprefix<<<1, NT, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t imc_batch_launch_comb_plan(const BatchArgs& a, cudaStream_t s) {
  ++g_imc_launches;
  k_bcomb_plan<<<a.K, NT, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t imc_batch_launch_ledger(const BatchArgs& a, int init, cudaStream_t s) {
  ++g_imc_launches;
  k_bledger<<<a.K, NT, 0, s>>>(a, init);
  return cudaGetLastError();
}
