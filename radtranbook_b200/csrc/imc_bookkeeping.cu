// imc_bookkeeping.cu — per-cell FP64 work of the time step.
//
// Compiled with -fmad=false: every number here is computed with the same operation order
// as the FP64 CPU oracle, so the integer particle counts per cell (ceil(N E_c / E)) and the
// comb targets agree exactly.
//
//   Fleck factor   IMC/IMC1D.py:933-938, IMC/IMC2D.py:1646-1651
//   emission plan  IMC/IMC1D.py:251-291 (slab), 629-707 (sphere), IMC/IMC2D.py:1731-1764
//                  with _sample_source_{xy,rz_uniform,rz_linear} :1191-1445
//   fixed source   IMC/IMC1D.py:294-316, 710-741; IMC/IMC2D.py:1709-1728
//   boundary       IMC/IMC1D.py:319-329, 744-763; IMC/IMC2D.py:157-489
//   IC             IMC/IMC1D.py:220-248, 535-575; IMC/IMC2D.py:1110-1188
//   material       IMC/IMC1D.py:1021-1035; IMC/IMC2D.py:1801-1810
//   comb targets   IMC/IMC1D.py:786-799; IMC/IMC2D.py:1461-1468; MG_IMC/MG_IMC1D.py:1194-1200
//   multigroup     MG_IMC/MG_IMC2D.py:1703-1943 (xy, rz); MG_IMC/MG_IMC1D.py:941-1120 (sphere)
#include <algorithm>
#include <cmath>
#include "imc_block.cuh"
#include "imc_device.cuh"
#include "imc_internal.h"

using namespace imcdev;

namespace {

constexpr double PI = 3.14159265358979323846;
using imcblk::NT;
using namespace imcblk;

// Per-cell part of the plan, one thread per cell: Fleck factor, absorption / effective
// scatter tables, emission energy, linear tilt constants, FP32 edges.
__global__ void k_plan_cells(PlanArgs a) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;  // device-resident step length (graph replay)
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c <= a.nx) a.e1f[c] = (float)a.e1[c];
  if (c <= a.ny) a.e2f[c] = (float)a.e2[c];
  if (c >= a.nc) return;
  const bool oned = (a.geom == G_SLAB || a.geom == G_SPHERE);
  // ---- Fleck factor and emission energy per cell (gray) ----
  const double sa_thr = oned ? 1e-10 : 1e-12;  // IMC/IMC1D.py:117, IMC/IMC2D.py:917
  {
    const double T = a.T[c];
    if (!isfinite(T) || (oned && !(T > 0.0)) || !isfinite(a.sigma[c]) || !(a.cv[c] > 0.0))
      atomicOr(&a.sum->flags, (int)IMC_FLAG_NONFINITE);
    const double beta = 4.0 * A_RAD * pow3(T) / a.cv[c];
    double f = 1.0 / (1.0 + a.theta * beta * a.sigma[c] * C_LIGHT * dt);
    f = fmin(1.0, fmax(0.0, f));
    const double ss = a.sigma[c] * (1.0 - f);
    const double sa = a.sigma[c] * f;
    a.sa[c] = sa; a.ss[c] = ss;
    // tracking table: sigma_a below the estimator's threshold is entered as 0 (no capture; in
    // FP32 exp(-sigma_a s) is 1 there anyway), which also marks the cell's intensity as the
    // path-length sum w*s; elsewhere the intensity follows from the deposition
    a.sass[c] = make_float2(sa > sa_thr ? (float)sa : 0.f, (float)ss);
    const double iv = 1.0 / a.vol[c];
    a.cellf[c] = make_double2(iv, sa > sa_thr ? 1.0 / (sa * a.vol[c] * dt) : -1.0 / (a.vol[c] * dt));
    double E = A_RAD * C_LIGHT * pow4(fmax(T, 0.0)) * sa * dt * a.vol[c];
    if (a.method == IMC_METHOD_CARTER_FOREST) {
      // Carter-Forest (IMC/IMC1D_CarterForest.py:1181-1185, 485-494; IMC/IMC2D_CarterForest.py:
      // 947-948, 877-883): true opacity, no effective scatter (the tracking kernel samples the
      // absorption distance from the scatter slot), path-length intensity only, emission
      // a T^4 (1 - e^{-k dt}) / beta V with k = c sigma beta
      const double sig = a.sigma[c];
      const double Tm = oned ? T : fmax(T, 1e-12);
      const double beta = 4.0 * A_RAD * pow3(Tm) / a.cv[c];
      const double rate = C_LIGHT * sig * beta;
      a.sa[c] = sig; a.ss[c] = 0.0;
      a.sass[c] = make_float2(0.f, (float)sig);
      a.cellf[c] = make_double2(iv, -1.0 / (a.vol[c] * dt));
      a.cf_rate[c] = (beta > 1e-15 && sig > 1e-15) ? (float)rate : 0.f;
      const double T4 = pow4(fmax(T, 0.0));
      const bool decays = oned ? rate > 1e-10 : (rate > 1e-12 && beta > 1e-15);
      E = decays ? A_RAD * T4 * -expm1(-rate * dt) / beta * a.vol[c] : A_RAD * T4 * C_LIGHT * sig * dt * a.vol[c];
    }
    if (a.t_emit_floor > 0.0 && T < a.t_emit_floor) E = 0.0;
    a.emit_E[c] = E * a.share;  // a rank of a partitioned step issues its share
  }
  // ---- tilt constants (emission; fixed-source RZ tilt uses the same T) ----
  {
    const int i = c % a.nx, j = c / a.nx;
    double* tl = a.tilt + 4 * c;
    tl[0] = tl[1] = tl[2] = tl[3] = 0.0;
    if (a.geom == G_SLAB && a.nx > 1) {
      // IMC/IMC1D.py:254-262: centred slopes of T, zeroed when an edge value goes negative
      auto dx = [&](int k) { return a.e1[k + 1] - a.e1[k]; };
      double s;
      if (i == 0) s = (a.T[1] - a.T[0]) / (dx(1) + dx(0)) * 2.0;
      else if (i == a.nx - 1) s = (a.T[i] - a.T[i - 1]) / (dx(i) + dx(i - 1)) * 2.0;
      else s = (a.T[i + 1] - a.T[i - 1]) / (dx(i + 1) + dx(i - 1)) * 2.0;
      if (a.T[i] - s * dx(i) / 2.0 < 0.0) s = 0.0;
      else if (a.T[i] + s * dx(i) / 2.0 < 0.0) s = 0.0;
      tl[0] = s;
    } else if (a.geom == G_SPHERE && a.nx > 1) {
      // IMC/IMC1D.py:643-659: slope of T^4 between cell-centre radii
      auto rm = [&](int k) { return 0.5 * (a.e1[k] + a.e1[k + 1]); };
      double M;
      if (i == 0) M = (pow4(a.T[1]) - pow4(a.T[0])) / (rm(1) - rm(0));
      else if (i == a.nx - 1) M = (pow4(a.T[i]) - pow4(a.T[i - 1])) / (rm(i) - rm(i - 1));
      else M = (pow4(a.T[i + 1]) - pow4(a.T[i - 1])) / (rm(i + 1) - rm(i - 1));
      const double lo = pow4(a.T[i]) - M * (rm(i) - a.e1[i]);
      const double hi = pow4(a.T[i]) + M * (a.e1[i + 1] - rm(i));
      if (lo < 0.0 || hi < 0.0) M = 0.0;
      tl[0] = M;
      tl[1] = pow4(a.T[i]) - M * (0.5 * (a.e1[i] + a.e1[i + 1]) - a.e1[i]);
    } else if (a.geom == G_RZ && a.rz_linear) {
      // IMC/IMC2D.py:1350-1417
      auto T4 = [&](int ii, int jj) { return pow4(fmax(a.T[ii + a.nx * jj], 0.0)); };
      auto rc = [&](int k) { return 0.5 * (a.e1[k] + a.e1[k + 1]); };
      auto zc = [&](int k) { return 0.5 * (a.e2[k] + a.e2[k + 1]); };
      double Mr, Mz;
      if (a.nx == 1) Mr = 0.0;
      else if (i == 0) Mr = (T4(i + 1, j) - T4(i, j)) / (rc(i + 1) - rc(i));
      else if (i == a.nx - 1) Mr = (T4(i, j) - T4(i - 1, j)) / (rc(i) - rc(i - 1));
      else Mr = (T4(i + 1, j) - T4(i - 1, j)) / (rc(i + 1) - rc(i - 1));
      if (a.ny == 1) Mz = 0.0;
      else if (j == 0) Mz = (T4(i, j + 1) - T4(i, j)) / (zc(j + 1) - zc(j));
      else if (j == a.ny - 1) Mz = (T4(i, j) - T4(i, j - 1)) / (zc(j) - zc(j - 1));
      else Mz = (T4(i, j + 1) - T4(i, j - 1)) / (zc(j + 1) - zc(j - 1));
      const double r0 = a.e1[i], r1 = a.e1[i + 1], z0 = a.e2[j], z1 = a.e2[j + 1];
      const double T4c = pow4(fmax(a.T[c], 0.0));
      double ar = T4c - Mr * (0.5 * (r0 + r1) - r0);
      double Mloc;
      const double t0 = ar, t1 = ar + Mr * (r1 - r0);
      if (t0 < 0.0 || t1 < 0.0) { ar = fmax(T4c, 0.0); Mloc = 0.0; } else Mloc = Mr;
      const double az = T4c - Mz * (0.5 * (z0 + z1) - z0);
      const double q0 = fmax(az, 0.0), q1 = fmax(az + Mz * (z1 - z0), 0.0);
      const double Pn = (q0 + q1 > 0.0) ? q0 / (q0 + q1) : 0.5;
      tl[0] = ar; tl[1] = Mloc; tl[2] = Pn;
    }
    if (a.method == IMC_METHOD_CARTER_FOREST) {
      const double Tm = oned ? a.T[c] : fmax(a.T[c], 1e-12);
      tl[3] = C_LIGHT * a.sigma[c] * (4.0 * A_RAD * pow3(Tm) / a.cv[c]);  // birth-time rate
    }
  }
}

// Boundary-face source energies of one side, E_q = a c T_q^4 / 4 * area_q * dt * share, all
// faces in parallel over the block; block_face_cdf then forms the side's cumulative sums.
__device__ void block_face_energy(int geom, bool oned, int side, int nf, const double* Tf, const double* e1,
                                  const double* e2, int nx, double dt, double share, double* Ef) {
  const bool along2 = side < 2;
  for (int q = threadIdx.x; q < nf; q += blockDim.x) {
    double area;
    if (oned) {
      if (geom == G_SLAB) area = 1.0;
      else { const double R = side == 0 ? e1[0] : e1[nx]; area = 4.0 * PI * R * R; }
    } else if (geom == G_XY) {
      area = along2 ? (e2[q + 1] - e2[q]) : (e1[q + 1] - e1[q]);
    } else {
      if (along2) { const double R = side == 0 ? e1[0] : e1[nx]; area = 2.0 * PI * R * (e2[q + 1] - e2[q]); }
      else area = PI * (e1[q + 1] * e1[q + 1] - e1[q] * e1[q]);
    }
    const double T = Tf[q];
    Ef[q] = (T > 0.0) ? A_RAD * C_LIGHT * T * T * T * T / 4.0 * area * dt * share : 0.0;
  }
}

// one thread: cdf[q] = E_0 + ... + E_q in face order; returns the side's total
__device__ double face_cdf_serial(const double* Ef, double* cdf, int nf) {
  constexpr int B = 16;
  double Et = 0.0;
  for (int q0 = 0; q0 < nf; q0 += B) {
    double v[B];
#pragma unroll
    for (int j = 0; j < B; ++j) v[j] = q0 + j < nf ? Ef[q0 + j] : 0.0;
#pragma unroll
    for (int j = 0; j < B; ++j) if (q0 + j < nf) { Et += v[j]; cdf[q0 + j] = Et; }
  }
  return Et;
}

__global__ void __launch_bounds__(NT) k_plan(PlanArgs a) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;  // device-resident step length (graph replay)
  __shared__ double red[NT];
  __shared__ long long sh[NT];
  const int t = threadIdx.x;
  const int nc = a.nc;
  const bool oned = (a.geom == G_SLAB || a.geom == G_SPHERE);

  // ---- emission counts / weights / offsets ----
  // Carter-Forest 1-D emission counts are max(1, round) in every cell
  // (IMC/IMC1D_CarterForest.py:499, :932); otherwise ceil
  const bool cf1 = a.method == IMC_METHOD_CARTER_FOREST && oned;
  const long long n_emit = plan_volume(a.emit_E, a.n_target, a.nx, a.ny, nc, a.emit_n, a.emit_off,
                                       a.emit_w, a.emitted, red, sh, cf1);
  const double e_emit = block_canon_sum(a.emitted, nc, red);

  // ---- fixed source (reference: only when max(source) > 0) ----
  long long n_src = 0;
  double e_src = 0.0;
  if (a.source && a.n_source > 0) {
    double smax = 0.0;
    for (int c = t; c < nc; c += NT) {
      smax = fmax(smax, a.source[c]);
      a.src_QV[c] = a.source[c] * dt * a.vol[c] * a.share;
    }
    red[t] = smax;
    __syncthreads();
    for (int h = NT / 2; h >= 1; h >>= 1) { if (t < h) red[t] = fmax(red[t], red[t + h]); __syncthreads(); }
    const bool any = red[0] > 0.0;
    __syncthreads();
    if (any) {
      n_src = plan_volume(a.src_QV, a.n_source, a.nx, a.ny, nc, a.src_n, a.src_off, a.src_w,
                          a.src_issued, red, sh);
      e_src = block_canon_sum(a.src_issued, nc, red);
    }
  }

  // ---- boundary faces: energies in parallel, then one thread per side forms the side's
  // cumulative sums in face order ----
  for (int side = 0; side < 4; ++side) {
    if (a.face_T[side] && a.n_side[side] > 0 && !(oned && side >= 2))
      block_face_energy(a.geom, oned, side, oned ? 1 : (side < 2 ? a.ny : a.nx), a.face_T[side], a.e1, a.e2, a.nx,
                        dt, a.share, a.face + (size_t)(side * 2 + 0) * a.nf);
  }
  __syncthreads();
  if (t < 4) {
    const int side = t;
    a.sum->n_side[side] = 0;
    a.sum->e_side[side] = 0.0;
    const double* Tf = a.face_T[side];
    const long long nbs = a.n_side[side];
    if (Tf && nbs > 0 && !(oned && side >= 2)) {
      const int nf = oned ? 1 : (side < 2 ? a.ny : a.nx);
      const double Et = face_cdf_serial(a.face + (size_t)(side * 2 + 0) * a.nf,
                                        a.face + (size_t)(side * 2 + 1) * a.nf, nf);
      if (Et > 0.0) {
        a.sum->n_side[side] = nbs;
        const float wq = (float)(Et / (double)nbs);
        a.sum->e_side[side] = (double)nbs * (double)wq;
      }
    }
  }
  __syncthreads();
  if (t == 0) {
    // bank layout of this step: census | boundary sides 0..3 | fixed source | emission
    long long base = a.sum->n_census;
    for (int q = 0; q < 4; ++q) { a.sum->base_side[q] = base; base += a.sum->n_side[q]; }
    a.sum->n_source = n_src; a.sum->base_source = base; base += n_src;
    a.sum->n_emission = n_emit; a.sum->base_emission = base; base += n_emit;
    a.sum->n_bank = base;
    a.sum->source_emission = e_src;
    a.sum->emission_total = e_emit;
  }
}

__global__ void __launch_bounds__(NT) k_ic_plan(IcArgs a) {
  __shared__ double red[NT];
  __shared__ long long sh[NT];
  const int t = threadIdx.x;
  const int nc = a.nc;
  const bool oned = (a.geom == G_SLAB || a.geom == G_SPHERE);
  double* E = a.E;
  for (int c = t; c < nc; c += NT) {
    double e = A_RAD * pow4(a.tr[c]) * a.vol[c];
    if (a.t_emit_floor > 0.0 && a.tr[c] < a.t_emit_floor) e = 0.0;
    E[c] = e;
  }
  __syncthreads();
  const double Et = block_canon_sum(E, nc, red);
  const long long N = a.n_target;
  for (int o = t; o < nc; o += NT) {
    const int c = order_to_cell(o, a.nx, a.ny);
    long long n = 0;
    if (N > 0) {
      if (a.rule == 2) n = (Et > 0.0 && E[c] > 0.0) ? max(1LL, (long long)rint((double)N * E[c] / Et)) : 0;
      else if (oned) n = Et > 0.0 ? (long long)ceil(E[c] / Et * (double)N) : 0;
      else n = max(1LL, (long long)ceil((double)N * E[c] / fmax(Et, 1e-300)));
    }
    a.n[o] = n;
    a.w[c] = n > 0 ? (float)(E[c] / (double)n) : 0.f;
  }
  __syncthreads();
  const long long tot = block_scan_counts(a.n, a.off, nc, sh);
  if (t == 0) { a.sum->n_emission = tot; a.sum->base_emission = 0; a.sum->n_bank = tot; }
}

__global__ void k_material(MatArgs a) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.nc) return;
  double dep = 0.0, si = 0.0;
  for (int g = 0; g < a.ng; ++g) { dep += a.dep[(size_t)g * a.nc + c]; si += a.si[(size_t)g * a.nc + c]; }
  a.e[c] = a.e[c] + dep - a.emitted[c] / a.vol[c];
  const double x = si / A_RAD / C_LIGHT;
  a.tr[c] = x > 0.0 ? sqrt(sqrt(x)) : 0.0;
}

// k_material, then T = e / cv_eos and the law's opacity of every group and cv at that T for
// the next step.  e and tr are k_material's sums (same order, so the same bits).
__global__ void k_material_law(MatArgs a, imc_material_law law, double* T, double* sigma_next, double* cv_next) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.nc) return;
  double dep = 0.0, si = 0.0;
  for (int g = 0; g < a.ng; ++g) { dep += a.dep[(size_t)g * a.nc + c]; si += a.si[(size_t)g * a.nc + c]; }
  const double e = a.e[c] + dep - a.emitted[c] / a.vol[c];
  a.e[c] = e;
  const double x = si / A_RAD / C_LIGHT;
  a.tr[c] = x > 0.0 ? sqrt(sqrt(x)) : 0.0;
  const double t = e / (law.cv_eos_array ? law.cv_eos_array[c] : law.cv_eos);
  T[c] = t;
  cv_next[c] = law.cv_array ? law.cv_array[c] : law.cv;
  if (law.sigma_array) {
    for (int g = 0; g < a.ng; ++g) sigma_next[(size_t)g * a.nc + c] = law.sigma_array[(size_t)g * a.nc + c];
    return;
  }
  const double tp = law.sigma_T_floor > 0.0 ? fmax(t, law.sigma_T_floor) : t;
  double base = law.sigma_n == 0.0 ? law.sigma_A : law.sigma_A * pow(tp, -law.sigma_n);
  if (law.sigma_scale) base = base * law.sigma_scale[c];
  for (int g = 0; g < a.ng; ++g) {
    double sg = law.sigma_group ? base * law.sigma_group[g] : base;
    if (law.sigma_lo > 0.0) sg = fmax(sg, law.sigma_lo);
    if (law.sigma_hi > 0.0) sg = fmin(sg, law.sigma_hi);
    sigma_next[(size_t)g * a.nc + c] = sg;
  }
}

// Single block: the canonical total of the census energy and the comb mode.
__global__ void __launch_bounds__(NT) k_comb_plan(CombPlanArgs a) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  __shared__ double red[NT];
  const double E = block_canon_sum<16>(a.ecen, a.nb, red);
  // MG_IMC/MG_IMC1D.py:1194-1200: Nmax = 0 never combs; Nmax < 0 combs once |Nmax| entries live
  const bool compact = a.force_compact || (a.threshold > 0 && (long long)*a.n_live < a.threshold);
  if (threadIdx.x == 0) { *a.mode = compact ? 1 : 0; a.sum->comb_before = E; a.sum->comb_after = 0.0; }
}

// Wide: the comb weight of every bin, ecen / max(1, rint(Nmax ecen / E)).
__global__ void k_comb_weights(CombPlanArgs a) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.nb) return;
  const double E = a.sum->comb_before;
  const long long n_max = a.n_max_dev ? (long long)*a.n_max_dev : a.n_max;
  const double ec = a.ecen[b];
  double ew = 0.0;
  if (E > 0.0 && ec > 0.0) ew = ec / fmax(1.0, rint((double)n_max * ec / E));
  a.ew[b] = ew;
  a.ncopy[b] = 0ull;
}

// Zero the regions of a ZeroList (one launch for a step's accumulators).
__global__ void k_zero(ZeroList z) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  const size_t t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x, stride = (size_t)gridDim.x * blockDim.x;
  for (int r = 0; r < z.n; ++r) {
    unsigned long long* q = static_cast<unsigned long long*>(z.p[r]);
    const size_t n8 = z.bytes[r] / 8;
    for (size_t i = t0; i < n8; i += stride) q[i] = 0ull;
  }
}

__global__ void __launch_bounds__(NT) k_canon_eV(const double* e, const double* vol, int nc, double* out) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  __shared__ double red[NT];
  const int t = threadIdx.x;
  double s = 0.0;
  for (int c = t; c < nc; c += NT) s += e[c] * vol[c];
  red[t] = s;
  __syncthreads();
  for (int h = NT / 2; h >= 1; h >>= 1) { if (t < h) red[t] += red[t + h]; __syncthreads(); }
  if (t == 0) *out = red[0];
}

}  // namespace

cudaError_t imc_launch_plan(const PlanArgs& a, cudaStream_t s) {
  g_imc_launches += 2;
  IMC_LAUNCH_PDL(k_plan_cells, (std::max(a.nc, std::max(a.nx, a.ny) + 1) + 255) / 256, 256, 0, s, a);
  IMC_LAUNCH_PDL(k_plan, 1, NT, 0, s, a);
  return cudaGetLastError();
}
cudaError_t imc_launch_ic_plan(const IcArgs& a, cudaStream_t s) {
  ++g_imc_launches;
  k_ic_plan<<<1, NT, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t imc_launch_material(const MatArgs& a, cudaStream_t s) {
  ++g_imc_launches;
  IMC_LAUNCH_PDL(k_material, (a.nc + 255) / 256, 256, 0, s, a);
  return cudaGetLastError();
}
cudaError_t imc_launch_material_law(const MatArgs& a, const imc_material_law& law, double* T, double* sigma_next,
                                    double* cv_next, cudaStream_t s) {
  ++g_imc_launches;
  IMC_LAUNCH_PDL(k_material_law, (a.nc + 255) / 256, 256, 0, s, a, law, T, sigma_next, cv_next);
  return cudaGetLastError();
}
cudaError_t imc_launch_zero(const ZeroList& z, cudaStream_t s) {
  unsigned long long most = 0;
  for (int r = 0; r < z.n; ++r) most = std::max(most, z.bytes[r] / 8);
  if (most == 0) return cudaSuccess;
  ++g_imc_launches;
  const unsigned blocks = (unsigned)std::min<unsigned long long>(1184ull, (most + 255) / 256);
  IMC_LAUNCH_PDL(k_zero, blocks, 256, 0, s, z);
  return cudaGetLastError();
}
cudaError_t imc_launch_comb_plan(const CombPlanArgs& a, cudaStream_t s) {
  g_imc_launches += 2;
  IMC_LAUNCH_PDL(k_comb_plan, 1, NT, 0, s, a);
  if (a.nb > 0) IMC_LAUNCH_PDL(k_comb_weights, (a.nb + 255) / 256, 256, 0, s, a);
  return cudaGetLastError();
}
// The multigroup step's reported fields in the reference's (nx, ny) order, one output each:
// si / c and after / V by group, then e, T, Tr, then the two group sums (imc_mg_report_fields).
__global__ void k_mg_report(ReportArgs a) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  const long long nc = (long long)a.nx * a.ny, gnc = nc * a.ng;
  for (long long q = a.q0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; q < a.q1;
       q += (long long)gridDim.x * blockDim.x) {
    double v;
    if (q < 2 * gnc + 3 * nc) {
      const long long part = q < 2 * gnc ? q / gnc : 2 + (q - 2 * gnc) / nc;  // 0 pre, 1 post, 2.. e T Tr
      const double* src = part == 0 ? a.si : part == 1 ? a.after : part == 2 ? a.e : part == 3 ? a.T : a.Tr;
      if (!src) continue;  // a section left to another call
      const long long r = q < 2 * gnc ? q % nc : (q - 2 * gnc) % nc;         // reference order i*ny + j
      const long long g = q < 2 * gnc ? (q % gnc) / nc : 0;
      const int i = (int)(r / a.ny), j = (int)(r - (long long)i * a.ny);
      const long long c = i + (long long)a.nx * j;
      if (part == 0) v = src[g * nc + c] / C_LIGHT;
      else if (part == 1) v = src[g * nc + c] / a.vol[c];
      else v = src[c];
    } else {
      const long long k = q - 2 * gnc - 3 * nc;
      const double* src = k < a.ng ? a.bnd : a.esc;
      if (!src) continue;
      v = src[k < a.ng ? k : k - a.ng];
    }
    a.out[q] = v;
  }
}

cudaError_t imc_launch_mg_report(const ReportArgs& a, cudaStream_t s) {
  if (a.q1 <= a.q0) return cudaSuccess;
  ++g_imc_launches;
  const unsigned blocks = (unsigned)std::min<long long>(4736LL, (a.q1 - a.q0 + 255) / 256);
  IMC_LAUNCH_PDL(k_mg_report, blocks, 256, 0, s, a);
  return cudaGetLastError();
}

cudaError_t imc_launch_canon_sum_eV(const double* e, const double* vol, int nc, double* out, cudaStream_t s) {
  ++g_imc_launches;
  IMC_LAUNCH_PDL(k_canon_eV, 1, NT, 0, s, e, vol, nc, out);
  return cudaGetLastError();
}

// =====================================================================================
// Multigroup planning (MG_IMC/MG_IMC2D.py:1703-1943): Planck group fractions, Fleck factor
// with the Planck-mean opacity, categorical emission / fixed-source tables.
// =====================================================================================
namespace {

// Planck fraction F(x) = (15/pi^4) int_0^x t^3/(e^t-1) dt: Bernoulli series below x = 1,
// exponential series above (Widger & Woodall 1976).  Same expansion as the oracle.
// sum_k e^{-kx}(x^3/k + 3x^2/k^2 + 6x/k^3 + 6/k^4) = (pi^4/15)(1 - F(x)), for x >= 1
// 1/k for the tail's terms, k < 64 (K = 2 + 40/x <= 42 for x >= 1): the correctly rounded
// quotients, so each term is the one the division gives
struct InvK { double v[64]; };
constexpr InvK inv_k_table() {
  InvK t{};
  for (int k = 1; k < 64; ++k) t.v[k] = 1.0 / (double)k;
  return t;
}
__device__ const InvK g_inv_k = inv_k_table();

__device__ double planck_tail(double x) {
  double tail = 0.0;
  const int K = (int)(2.0 + 40.0 / x);
  for (int k = K; k >= 1; --k) {
    const double kx = k * x, ik = k < 64 ? g_inv_k.v[k] : 1.0 / k;
    tail += exp(-kx) * ik * (x * x * x + ik * (3.0 * x * x + ik * (6.0 * x + ik * 6.0)));
  }
  return tail;
}

// Bernoulli series of (pi^4/15) F(x) for 0 < x < 1
__device__ double planck_series(double x) {
  const double B[21] = {1.0, -0.5, 1.0 / 6.0, 0.0, -1.0 / 30.0, 0.0, 1.0 / 42.0, 0.0, -1.0 / 30.0, 0.0,
                        5.0 / 66.0, 0.0, -691.0 / 2730.0, 0.0, 7.0 / 6.0, 0.0, -3617.0 / 510.0, 0.0,
                        43867.0 / 798.0, 0.0, -174611.0 / 330.0};
  double sum = 0.0, xp = x * x * x, fact = 1.0;
  for (int n = 0; n <= 20; ++n) {
    if (n > 0) fact *= n;
    if (B[n] != 0.0) sum += B[n] * xp / ((n + 3) * fact);
    xp *= x;
  }
  return sum;
}

// One group edge x = E/T with its series (0 < x < 1) or tail (x >= 1) value, evaluated once
// and shared by the two groups the edge bounds.
struct PlanckEdge { double x, s; };

__device__ PlanckEdge planck_edge(double x) {
  if (!(x > 0.0)) return PlanckEdge{x, 0.0};
  return PlanckEdge{x, x < 1.0 ? planck_series(x) : planck_tail(x)};
}

__device__ double planck_F(const PlanckEdge& e) {
  const double c = 15.0 / (PI * PI * PI * PI);
  if (!(e.x > 0.0)) return 0.0;
  return e.x < 1.0 ? c * e.s : 1.0 - c * e.s;
}

// F(x1) - F(x0); above x = 1 as a difference of tails, which keeps its relative precision
// far into the Wien tail (1 - F cancels to 0 there)
__device__ double planck_frac(const PlanckEdge& e0, const PlanckEdge& e1) {
  if (!(e1.x > e0.x)) return 0.0;
  if (e0.x >= 1.0) return 15.0 / (PI * PI * PI * PI) * (e0.s - e1.s);
  return planck_F(e1) - planck_F(e0);
}

// canonical inclusive prefix sum of n values (the oracle's canon_prefix order)
// The sequential parts load their operands a batch at a time into registers before the
// dependent adds, so each add waits for the previous add only, not for a load issued after
// the previous store (the compiler cannot reorder those: out may alias x); the adds and
// their order are unchanged.
__device__ void block_canon_prefix(const double* x, int n, double* out, double* sh) {
  constexpr int B = 16;
  const int t = threadIdx.x;
  const int per = (n + NT - 1) / NT;
  const int lo = min(t * per, n), hi = min(lo + per, n);
  double s = 0.0;
  for (int i = lo; i < hi; ++i) s += x[i];
  sh[t] = s;
  __syncthreads();
  if (t == 0) {
    double off = 0.0;
    for (int q0 = 0; q0 < NT; q0 += 32) {
      double v[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = sh[q0 + j];
#pragma unroll
      for (int j = 0; j < 32; ++j) { sh[q0 + j] = off; off += v[j]; }
    }
  }
  __syncthreads();
  double run = sh[t];
  for (int i0 = lo; i0 < hi; i0 += B) {
    double v[B];
#pragma unroll
    for (int j = 0; j < B; ++j) v[j] = i0 + j < hi ? x[i0 + j] : 0.0;
#pragma unroll
    for (int j = 0; j < B; ++j) if (i0 + j < hi) { run += v[j]; out[i0 + j] = run; }
  }
  __syncthreads();
}

// Mixture-of-Gammas CDF of the Planck group sampler, weights 1/n^4 over n = 1..200
// (MG_IMC/MG_IMC2D.py:105-107), summed in order n = 1..200.  A constant: the compiler
// evaluates it once (IEEE double, the order of the loop), the plan kernels copy it into the
// step's workspace.
struct MixCdf { double v[200]; };
constexpr MixCdf mix_cdf_table() {
  MixCdf m{};
  double tot = 0.0, run = 0.0;
  for (int n = 1; n <= 200; ++n) { const double d = (double)n; tot += 1.0 / (d * d * d * d); }
  for (int n = 1; n <= 200; ++n) { const double d = (double)n; run += 1.0 / (d * d * d * d); m.v[n - 1] = run / tot; }
  return m;
}
__device__ const MixCdf g_mix_cdf = mix_cdf_table();

// The Planck edge integrals of the block's cells [c0, c0 + ncb) at the G + 1 group edges,
// one (cell, edge) pair per thread: x and its series or tail value at [(c - c0)(G + 1) + k].
// The tail costs up to 2 + 40/x exponentials, so this is most of a plan's arithmetic; spread
// over all the block's threads it is no longer one long chain per cell.
__device__ void block_planck_edges(const double* T, const double* gedges, int G, int c0, int ncb, double* sx,
                                   double* ss) {
  const int E = G + 1;
  for (int i = threadIdx.x; i < ncb * E; i += blockDim.x) {
    const int cl = i / E, k = i - cl * E;
    const double Tc = T[c0 + cl];
    const PlanckEdge pe = planck_edge(Tc > 0.0 ? gedges[k] / Tc : 0.0);
    sx[i] = pe.x;
    ss[i] = pe.s;
  }
  __syncthreads();
}

// Per-cell part of the 2-D multigroup plan.  A block takes cb consecutive cells: its threads
// evaluate the cells' Planck edges into shared memory, then one thread per cell forms the
// fractions, Planck-mean opacity, Fleck factor and emission by group (each cell's numbers
// depend on that cell alone, so the result is the single-block loop's).
__global__ void __launch_bounds__(256) k_plan_mg_cells(PlanMgArgs a, int cb) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  extern __shared__ double plan_sh[];
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;  // device-resident step length (graph replay)
  const int nc = a.nc, G = a.ng;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int q = t0; q <= a.nx; q += stride) a.e1f[q] = (float)a.e1[q];
  for (int q = t0; q <= a.ny; q += stride) a.e2f[q] = (float)a.e2[q];
  for (int q = t0; q < 200; q += stride) a.mixcdf[q] = g_mix_cdf.v[q];
  const int c0 = blockIdx.x * cb, ncb = min(cb, nc - c0);
  double* sx = plan_sh;
  double* sv = plan_sh + (size_t)cb * (G + 1);
  block_planck_edges(a.T, a.gedges, G, c0, ncb, sx, sv);
  // ---- per cell: Planck fractions, Planck-mean opacity, Fleck, emission by group ----
  if ((int)threadIdx.x < ncb) {
    const int c = c0 + threadIdx.x;
    const int eb = threadIdx.x * (G + 1);
    const double T = a.T[c];
    if (!isfinite(T) || !(a.cv[c] > 0.0)) atomicOr(&a.sum->flags, (int)IMC_FLAG_NONFINITE);
    double* gc = a.Egc + (size_t)c * G;  // scratch: fractions, then cumulative emission
    double tot = 0.0;
    PlanckEdge lo{sx[eb], sv[eb]};
    for (int g = 0; g < G; ++g) {
      const PlanckEdge hi{sx[eb + g + 1], sv[eb + g + 1]};
      const double f = (T > 0.0) ? planck_frac(lo, hi) : 0.0;
      lo = hi;
      gc[g] = f > 0.0 ? f : 0.0;
      tot += gc[g];
    }
    double sp = 0.0;
    for (int g = 0; g < G; ++g) {
      gc[g] = tot > 0.0 ? gc[g] / tot : 0.0;
      sp += a.sigma[(size_t)g * nc + c] * gc[g];
    }
    const double beta = 4.0 * A_RAD * pow3(T) / a.cv[c];
    double f = 1.0 / (1.0 + a.theta * beta * sp * C_LIGHT * dt);
    f = fmin(1.0, fmax(0.0, f));
    const double aT4 = (a.t_emit_floor > 0.0 && T < a.t_emit_floor) ? 0.0
                                                                      : A_RAD * C_LIGHT * pow4(T) * dt * a.vol[c] * a.share;
    double run = 0.0;
    for (int g = 0; g < G; ++g) {
      const size_t q = (size_t)g * nc + c;
      const double ss = a.sigma[q] * (1.0 - f);
      const double sa = a.sigma[q] * f;
      a.sa[q] = sa; a.ss[q] = ss;
      a.sass[q] = make_float2(sa > 1e-12 ? (float)sa : 0.f, (float)ss);  // 0: no capture, w*s intensity
      a.cellf[q] = make_double2(1.0 / a.vol[c], sa > 1e-12 ? 1.0 / (sa * a.vol[c] * dt) : -1.0 / (a.vol[c] * dt));
      const double bg = a.emission_fractions ? a.emission_fractions[g] : gc[g];
      run += sa * bg * aT4;
      gc[g] = run;  // cumulative over groups
    }
    a.Ec[c] = run;
  }
  // fixed source [g][c] (MG_IMC/MG_IMC2D.py:1098-1170): per-cell cumulative over groups
  if (a.source && a.n_source > 0) {
    for (int c = t0; c < nc; c += stride) {
      double run = 0.0;
      for (int g = 0; g < G; ++g) {
        run += a.source[(size_t)g * nc + c] * a.vol[c] * dt * a.share;
        a.Sgc[(size_t)c * G + g] = run;
      }
      a.Sc[c] = run;
    }
  }
}

// Single-block part: canonical prefix sums and totals, counts, boundary faces, bank layout.
__global__ void __launch_bounds__(NT) k_plan_mg(PlanMgArgs a) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;  // device-resident step length (graph replay)
  __shared__ double sh[NT];
  const int t = threadIdx.x;
  const int nc = a.nc;
  block_canon_prefix(a.Ec, nc, a.cdf, sh);
  const double Eemit = a.cdf[nc - 1];
  long long n_emit = 0;
  double issued = 0.0;
  if (a.n_target > 0 && Eemit > 0.0) {
    n_emit = a.n_target;
    const float w32 = (float)(Eemit / (double)n_emit);
    issued = (double)n_emit * (double)w32;
  }
  const double scale = Eemit > 0.0 ? issued / Eemit : 0.0;
  for (int c = t; c < nc; c += NT) a.emitted[c] = a.Ec[c] * scale;

  // ---- fixed source [g][c] (MG_IMC/MG_IMC2D.py:1098-1170) ----
  long long n_src = 0;
  double e_src = 0.0;
  if (a.source && a.n_source > 0) {
    block_canon_prefix(a.Sc, nc, a.Scdf, sh);
    const double St = a.Scdf[nc - 1];
    if (St > 0.0) {
      n_src = a.n_source;
      e_src = (double)n_src * (double)(float)(St / (double)n_src);
    }
  }

  // ---- boundary faces (as gray: energies in parallel, cumulative sums per side) ----
  for (int side = 0; side < 4; ++side) {
    if (a.face_T[side] && a.n_side[side] > 0)
      block_face_energy(a.geom, false, side, side < 2 ? a.ny : a.nx, a.face_T[side], a.e1, a.e2, a.nx, dt, a.share,
                        a.face + (size_t)(side * 2 + 0) * a.nf);
  }
  __syncthreads();
  if (t < 4) {
    const int side = t;
    a.sum->n_side[side] = 0;
    a.sum->e_side[side] = 0.0;
    const double* Tf = a.face_T[side];
    const long long nbs = a.n_side[side];
    if (Tf && nbs > 0) {
      const int nf = side < 2 ? a.ny : a.nx;
      const double Et = face_cdf_serial(a.face + (size_t)(side * 2 + 0) * a.nf,
                                        a.face + (size_t)(side * 2 + 1) * a.nf, nf);
      if (Et > 0.0) {
        a.sum->n_side[side] = nbs;
        a.sum->e_side[side] = (double)nbs * (double)(float)(Et / (double)nbs);
      }
    }
  }
  __syncthreads();
  if (t == 0) {
    long long base = a.sum->n_census;
    for (int q = 0; q < 4; ++q) { a.sum->base_side[q] = base; base += a.sum->n_side[q]; }
    a.sum->n_source = n_src; a.sum->base_source = base; base += n_src;
    a.sum->n_emission = n_emit; a.sum->base_emission = base; base += n_emit;
    a.sum->n_bank = base;
    a.sum->source_emission = e_src;
    a.sum->emission_total = issued;
  }
}

// Multigroup 1-D sphere planning (MG_IMC/MG_IMC1D.py:941-1120): Planck fractions, Fleck
// factor with the Planck-mean opacity, emission E_gc = a c T^4 sigma_a,g b*_g dt V per
// (group, cell) bin b = g*nc + c with stratified counts max(1, round(N E_b / E)) (fixed
// source: round, no minimum), inner / outer sphere boundary faces.
// Per-shell part of the sphere plan, one thread per shell over a wide grid (each shell's
// numbers depend on that shell alone, so the result is the single-block loop's).
__global__ void __launch_bounds__(256) k_plan_mg1d_cells(PlanMgArgs a, int cb) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  extern __shared__ double plan_sh[];
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;  // device-resident step length (graph replay)
  const int nc = a.nc, G = a.ng;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int q = t0; q <= a.nx; q += stride) a.e1f[q] = (float)a.e1[q];
  for (int q = t0; q <= a.ny; q += stride) a.e2f[q] = (float)a.e2[q];
  for (int q = t0; q < 200; q += stride) a.mixcdf[q] = g_mix_cdf.v[q];
  const int c0 = blockIdx.x * cb, ncb = min(cb, nc - c0);
  double* sx = plan_sh;
  double* sv = plan_sh + (size_t)cb * (G + 1);
  block_planck_edges(a.T, a.gedges, G, c0, ncb, sx, sv);
  if ((int)threadIdx.x < ncb) {
    const int c = c0 + threadIdx.x;
    const int eb = threadIdx.x * (G + 1);
    const double T = a.T[c];
    if (!isfinite(T) || !(a.cv[c] > 0.0)) atomicOr(&a.sum->flags, (int)IMC_FLAG_NONFINITE);
    double* b = a.Egc + (size_t)c * G;  // scratch: Planck fractions of this cell
    double tot = 0.0;
    PlanckEdge lo{sx[eb], sv[eb]};
    for (int g = 0; g < G; ++g) {
      const PlanckEdge hi{sx[eb + g + 1], sv[eb + g + 1]};
      const double f = (T > 0.0) ? planck_frac(lo, hi) : 0.0;
      lo = hi;
      b[g] = f > 0.0 ? f : 0.0;
      tot += b[g];
    }
    double sp = 0.0;
    for (int g = 0; g < G; ++g) {
      b[g] = tot > 0.0 ? b[g] / tot : 0.0;
      sp += a.sigma[(size_t)g * nc + c] * b[g];
    }
    const double beta = 4.0 * A_RAD * pow3(T) / a.cv[c];
    double f = 1.0 / (1.0 + a.theta * beta * sp * C_LIGHT * dt);
    f = fmin(1.0, fmax(0.0, f));
    const bool cold = a.t_emit_floor > 0.0 && T < a.t_emit_floor;
    for (int g = 0; g < G; ++g) {
      const size_t q = (size_t)g * nc + c;
      const double sa = a.sigma[q] * f;
      const double ss = a.sigma[q] * (1.0 - f);
      a.sa[q] = sa; a.ss[q] = ss;
      a.sass[q] = make_float2(sa > 1e-10 ? (float)sa : 0.f, (float)ss);  // 0: no capture, w*s intensity
      // MG_IMC/MG_IMC1D.py:346-350: path-length estimator below sigma_a = 1e-10
      a.cellf[q] = make_double2(1.0 / a.vol[c], sa > 1e-10 ? 1.0 / (sa * a.vol[c] * dt) : -1.0 / (a.vol[c] * dt));
      a.emit_E[q] = cold ? 0.0 : A_RAD * C_LIGHT * pow4(T) * sa * b[g] * dt * a.vol[c] * a.share;
    }
  }
}

// Single-block part of the sphere plan: canonical totals, stratified counts and scans,
// fixed source, boundary faces, bank layout.
__global__ void __launch_bounds__(NT) k_plan_mg1d(PlanMgArgs a) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;  // device-resident step length (graph replay)
  __shared__ double red[NT];
  __shared__ long long sh[NT];
  const int t = threadIdx.x;
  const int nc = a.nc, G = a.ng, ncg = nc * G;
  // ---- emission: stratified counts, FP32 weights, energy issued per bin and per cell ----
  const double Et = block_canon_sum(a.emit_E, ncg, red);
  for (int q = t; q < ncg; q += NT) {
    const double E = a.emit_E[q];
    long long n = 0;
    if (a.n_target > 0 && Et > 0.0 && E > 0.0) n = max(1LL, (long long)rint((double)a.n_target * E / Et));
    const float w = n > 0 ? (float)(E / (double)n) : 0.f;
    a.emit_n[q] = n; a.emit_w[q] = w; a.emit_issued[q] = (double)n * (double)w;
  }
  __syncthreads();
  const long long n_emit = block_scan_counts(a.emit_n, a.emit_off, ncg, sh);
  const double e_emit = block_canon_sum(a.emit_issued, ncg, red);
  for (int c = t; c < nc; c += NT) {
    double e = 0.0;
    for (int g = 0; g < G; ++g) e += a.emit_issued[(size_t)g * nc + c];
    a.emitted[c] = e;
  }
  // ---- fixed source [g][c] (MG_IMC/MG_IMC1D.py:679-743; only when max(source) > 0) ----
  long long n_src = 0;
  double e_src = 0.0;
  if (a.source && a.n_source > 0) {
    double smax = 0.0;
    for (int q = t; q < ncg; q += NT) {
      smax = fmax(smax, a.source[q]);
      a.src_QV[q] = a.source[q] * a.vol[q % nc] * dt * a.share;
    }
    red[t] = smax;
    __syncthreads();
    for (int h = NT / 2; h >= 1; h >>= 1) { if (t < h) red[t] = fmax(red[t], red[t + h]); __syncthreads(); }
    const bool any = red[0] > 0.0;
    __syncthreads();
    if (any) {
      const double Qt = block_canon_sum(a.src_QV, ncg, red);
      for (int q = t; q < ncg; q += NT) {
        const double Q = a.src_QV[q];
        long long n = 0;
        if (Qt > 0.0 && Q > 0.0) n = max(0LL, (long long)rint((double)a.n_source * Q / Qt));
        const float w = n > 0 ? (float)(Q / (double)n) : 0.f;
        a.src_n[q] = n; a.src_w[q] = w; a.src_issued[q] = (double)n * (double)w;
      }
      __syncthreads();
      n_src = block_scan_counts(a.src_n, a.src_off, ncg, sh);
      e_src = block_canon_sum(a.src_issued, ncg, red);
    }
  }
  // ---- boundary: a c T^4 / 4 * 4 pi R^2 * dt on the inner and outer sphere ----
  if (t < 4) {
    const int side = t;
    a.sum->n_side[side] = 0;
    a.sum->e_side[side] = 0.0;
    const double* Tf = a.face_T[side];
    const long long nbs = a.n_side[side];
    if (side < 2 && Tf && nbs > 0) {
      double* Ef = a.face + (size_t)(side * 2 + 0) * a.nf;
      double* cdf = a.face + (size_t)(side * 2 + 1) * a.nf;
      const double R = side == 0 ? a.e1[0] : a.e1[a.nx];
      const double T = Tf[0];
      const double E = (T > 0.0) ? A_RAD * C_LIGHT * T * T * T * T / 4.0 * (4.0 * PI * R * R) * dt * a.share : 0.0;
      Ef[0] = E;
      cdf[0] = E;
      if (E > 0.0) {
        a.sum->n_side[side] = nbs;
        a.sum->e_side[side] = (double)nbs * (double)(float)(E / (double)nbs);
      }
    }
  }
  __syncthreads();
  if (t == 0) {
    long long base = a.sum->n_census;
    for (int q = 0; q < 4; ++q) { a.sum->base_side[q] = base; base += a.sum->n_side[q]; }
    a.sum->n_source = n_src; a.sum->base_source = base; base += n_src;
    a.sum->n_emission = n_emit; a.sum->base_emission = base; base += n_emit;
    a.sum->n_bank = base;
    a.sum->source_emission = e_src;
    a.sum->emission_total = e_emit;
  }
}

// multigroup initial census plan: cell CDF of a Tr^4 V, N particles of weight E/N
__global__ void __launch_bounds__(NT) k_ic_plan_mg(IcMgArgs a) {
  __shared__ double sh[NT];
  const int t = threadIdx.x;
  for (int q = t; q < 200; q += NT) a.mixcdf[q] = g_mix_cdf.v[q];
  for (int c = t; c < a.nc; c += NT) {
    double e = A_RAD * pow4(a.tr[c]) * a.vol[c];
    if (a.t_emit_floor > 0.0 && a.tr[c] < a.t_emit_floor) e = 0.0;
    a.E[c] = e;
  }
  __syncthreads();
  block_canon_prefix(a.E, a.nc, a.cdf, sh);
  if (t == 0) {
    const double Et = a.cdf[a.nc - 1];
    const long long n = (a.n_target > 0 && Et > 0.0) ? a.n_target : 0;
    a.sum->n_emission = n; a.sum->base_emission = 0; a.sum->n_bank = n;
  }
}

}  // namespace

// Launch shape of the per-cell multigroup plan: as many cells a block as leave one
// (cell, group edge) pair per thread (the edge integrals are the long part; at most 32 cells),
// two doubles per pair of shared memory; above 48 KB the kernel is opted in to more.
template <typename K>
cudaError_t launch_plan_cells(K kernel, const PlanMgArgs& a, cudaStream_t s) {
  const long long E = (long long)a.ng + 1;
  const int cb = (int)std::max(1LL, std::min(32LL, 256LL / E));
  const size_t smem = (size_t)2 * cb * E * sizeof(double);
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const int blocks = (a.nc + cb - 1) / cb;
  IMC_LAUNCH_PDL(kernel, blocks, 256, smem, s, a, cb);
  return cudaSuccess;
}

cudaError_t imc_launch_plan_mg(const PlanMgArgs& a, cudaStream_t s) {
  g_imc_launches += 2;
  const cudaError_t e = launch_plan_cells(k_plan_mg_cells, a, s);
  if (e != cudaSuccess) return e;
  IMC_LAUNCH_PDL(k_plan_mg, 1, NT, 0, s, a);
  return cudaGetLastError();
}

cudaError_t imc_launch_plan_mg1d(const PlanMgArgs& a, cudaStream_t s) {
  g_imc_launches += 2;
  const cudaError_t e = launch_plan_cells(k_plan_mg1d_cells, a, s);
  if (e != cudaSuccess) return e;
  IMC_LAUNCH_PDL(k_plan_mg1d, 1, NT, 0, s, a);
  return cudaGetLastError();
}

cudaError_t imc_launch_ic_plan_mg(const IcMgArgs& a, cudaStream_t s) {
  ++g_imc_launches;
  k_ic_plan_mg<<<1, NT, 0, s>>>(a);
  return cudaGetLastError();
}
