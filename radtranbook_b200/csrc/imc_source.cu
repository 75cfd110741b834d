// imc_source.cu — fill the structure-of-arrays bank with new particles.
//
// One thread per new particle.  The particle's cell comes from a binary search of the
// per-cell prefix sums computed by the planning kernel (source order: the reference's
// i-outer / j-inner loops), so writes of consecutive threads are consecutive bank slots.
// Sampling math is FP64 (Newton-bisection CDF inversions included) and stored as FP32.
//
//   volume sources  IMC/IMC1D.py:203-316 (slab emission, linear-T tilt, fixed source),
//                   IMC/IMC1D.py:578-741 (sphere), IMC/IMC2D.py:1191-1445 (xy, rz),
//                   MG_IMC/MG_IMC1D.py:569-743 (sphere, stratified per (group, cell))
//   initial census  IMC/IMC1D.py:220-248, 535-575; IMC/IMC2D.py:1110-1188; MG_IMC/MG_IMC1D.py:514-566
//   boundary        IMC/IMC1D.py:319-329, 744-763; IMC/IMC2D.py:157-489
// Random numbers: Philox (particle index within this source, block 0/1, step, tag).
#include <cmath>
#include "imc_device.cuh"
#include "imc_internal.h"
#include "imc_sample.cuh"

using namespace imcdev;
using namespace imcsample;

namespace {

// Offsets sampled into shared memory for the first levels of the particle -> bin search.
constexpr int kOffSamples = 1024;

// Adds the block's sum of v to *out (one FP64 atomic per block).  Every thread of the block
// calls it.
__device__ __forceinline__ void block_add_d(double v, double* out) {
  __shared__ double sh[32];
  v = warp_sum_d(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();  // the body's own shared-memory use is over
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    double t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    t = warp_sum_d(t);
    if (lane == 0 && t != 0.0) atomicAdd(out, t);
  }
}

// The bodies below run on blocks blk of nblk (a kernel of their own, or a job of
// k_fill_sources); the boundary body with wsum adds the weights it writes to *wsum.
__device__ __forceinline__ void fill_volume(const uint32_t* __restrict__ rk, const FillArgs& a, int blk, int nblk) {
  const double time_scale = a.time_scale_dev ? *a.time_scale_dev : a.time_scale;  // graph replay
  const uint32_t step = a.step_dev ? *a.step_dev : a.step;
  const long long stride = (long long)nblk * blockDim.x;
  const long long n = *a.d_n, base = *a.d_base;
  // s_off[q] = off[min((q + 1) * span, nbins)]: the search for the bin of particle k (the
  // smallest o with off[o + 1] > k) first finds its span of `span` bins in shared memory,
  // then bisects the span in global memory.
  __shared__ long long s_off[kOffSamples];
  const int nbins = a.nbins;
  if (nbins <= 0) return;  // uniform across the grid
  const int span = (nbins + kOffSamples - 1) / kOffSamples;
  const int m = (nbins + span - 1) / span;
  for (int q = threadIdx.x; q < m; q += blockDim.x) s_off[q] = a.off[min((q + 1) * span, nbins)];
  __syncthreads();
  for (long long k = (long long)blk * blockDim.x + threadIdx.x; k < n; k += stride) {
    // order position o with off[o] <= k < off[o+1] (k < n = off[nbins], so o < nbins)
    int qlo = 0, qhi = m - 1;
    while (qlo < qhi) { const int mid = (qlo + qhi) >> 1; if (s_off[mid] > k) qhi = mid; else qlo = mid + 1; }
    int lo = qlo * span, hi = min(lo + span, nbins) - 1;
    while (lo < hi) { const int mid = (lo + hi) >> 1; if (a.off[mid + 1] <= k) lo = mid + 1; else hi = mid; }
    const int o = lo;
    const int g = a.bins_by_group ? o / a.nc : 0;  // MG 1-D bins b = g*nc + c
    const int oc = o - g * a.nc;
    const int i = oc / a.ny, j = oc - i * a.ny;
    const int c = i + a.nx * j;
    const U4 r = draw_rk(rk, (uint32_t)k + a.id_base, 0, step, a.tag);
    const U4 s = draw_rk(rk, (uint32_t)k + a.id_base, 1, step, a.tag);
    const double u0 = u01d(r.x), u1 = u01d(r.y), u2 = u01d(r.z), u3 = u01d(r.w);
    const double s0 = u01d(s.x), s1 = u01d(s.y);
    const double ea = a.e1[i], eb = a.e1[i + 1];
    double p1, p2 = 0.0;
    switch (a.geom) {
      case G_SLAB:
        p1 = ea + (a.tilt_kind == 1 ? slab_linear(eb - ea, a.tilt[4 * c], a.T[c], u0) : u0 * (eb - ea));
        break;
      case G_SPHERE: {
        const double M = a.tilt_kind == 2 ? a.tilt[4 * c] : 0.0;
        const double ac = a.tilt_kind == 2 ? a.tilt[4 * c + 1] : 0.0;
        if (a.tilt_kind == 2 && !(fabs(M) < 1e-30 || fabs(ac) < 1e-30)) p1 = sphere_cdf(ea, eb, ac, M, u0);
        else p1 = cbrt(ea * ea * ea + (eb * eb * eb - ea * ea * ea) * u0);
        break;
      }
      case G_XY:
        p1 = ea + u0 * (eb - ea);
        p2 = a.e2[j] + u1 * (a.e2[j + 1] - a.e2[j]);
        break;
      default: {
        const double zl = a.e2[j], zh = a.e2[j + 1];
        if (a.tilt_kind == 3) {
          const double* tl = a.tilt + 4 * c;
          p1 = rz_r_cdf(ea, eb, tl[0], tl[1], u0);
          const double sq = sqrt(u1);
          p2 = (s1 <= tl[2]) ? zh - (zh - zl) * sq : zl + (zh - zl) * sq;
        } else {
          p1 = sqrt(ea * ea + (eb * eb - ea * ea) * u0);
          p2 = zl + u1 * (zh - zl);
        }
        break;
      }
    }
    p1 = fmin(fmax(p1, ea), eb);
    if (a.geom == G_XY || a.geom == G_RZ) p2 = fmin(fmax(p2, a.e2[j]), a.e2[j + 1]);
    double d1, d2;
    iso_dir(a.geom, u2, u3, d1, d2);
    const long long b = base + k;
    a.p1[b] = (float)p1; a.d1[b] = (float)d1;
    if (a.p2) a.p2[b] = (float)p2;
    if (a.d2) a.d2[b] = (float)d2;
    a.wb[b] = a.w[a.bins_by_group ? o : c];
    double tb = s0 * time_scale;
    if (a.cf_rate4) {
      // Carter-Forest birth time, density ~ exp(-k t) on [0, dt]: t = -ln(1 - xi (1 - e^{-k dt})) / k
      // (IMC/IMC1D_CarterForest.py:529-536, IMC/IMC2D_CarterForest.py:51-56)
      const double k = a.cf_rate4[4 * c];
      if (k > a.cf_thr) tb = -log1p(s0 * expm1(-k * time_scale)) / k;
    }
    a.t[b] = (float)tb;
    a.cell[b] = c;
    if (a.group) {
      int gb = g;
      if (a.tr) {  // MG 1-D initial census: Planck group at the cell's Tr (MG_IMC/MG_IMC1D.py:557-560)
        const U4 d = draw_rk(rk, (uint32_t)k + a.id_base, 2, step, a.tag);
        gb = planck_group(a.tr[c], a.gedges, a.ng, a.mixcdf, s1, u01d(s.z), u01d(s.w), u01d(d.x), u01d(d.y), true);
      }
      a.group[b] = gb;
    }
  }
}

__global__ void k_fill_volume(FillArgs a) { fill_volume(a.rk, a, blockIdx.x, gridDim.x); }

// Boundary energy by group: every particle of a face has the same FP32 weight wq, so the
// tally is (count of the group) x wq.  Counts go to shared memory per block (groups below
// kBndGroups) and each block adds count x wq once per group: exact and order-independent
// (every partial sum is an integer multiple of wq below 2^29 wq), and free of the contention
// of one FP64 atomic per particle on a handful of addresses.
constexpr int kBndGroups = 256;

__device__ __forceinline__ void fill_boundary(const uint32_t* __restrict__ rk, const BndArgs& a, int blk, int nblk,
                                              double* wsum) {
  __shared__ unsigned s_gcnt[kBndGroups];
  const bool tally_groups = a.group && a.ng > 1;
  if (tally_groups)
    for (int g = threadIdx.x; g < kBndGroups; g += blockDim.x) s_gcnt[g] = 0u;
  __syncthreads();
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;  // graph replay
  const uint32_t step = a.step_dev ? *a.step_dev : a.step;
  const long long stride = (long long)nblk * blockDim.x;
  const bool oned = (a.geom == G_SLAB || a.geom == G_SPHERE);
  const bool along2 = a.side < 2;
  const int nf = oned ? 1 : (along2 ? a.ny : a.nx);
  const double* Ef = a.face;
  const double* cdf = a.face + a.nf;
  const long long n = *a.d_n, base = *a.d_base;
  if (n <= 0) return;  // uniform across the grid: no block passes the barrier below alone
  const double total = cdf[nf - 1];
  const float wq = (float)(total / (double)n);
  unsigned n_mine = 0;  // particles this thread writes, each of weight wq
  for (long long k = (long long)blk * blockDim.x + threadIdx.x; k < n; k += stride) {
    ++n_mine;
    const U4 ra = draw_rk(rk, (uint32_t)k + a.id_base, 0, step, TAG_BOUNDARY | (uint32_t)a.side);
    const U4 rb = draw_rk(rk, (uint32_t)k + a.id_base, 1, step, TAG_BOUNDARY | (uint32_t)a.side);
    const double ua0 = u01d(ra.x), ua1 = u01d(ra.y), ua2 = u01d(ra.z), ua3 = u01d(ra.w);
    const double x = ua0 * total;
    int lo = 0, hi = nf;  // lower_bound(cdf, x)
    while (lo < hi) { const int mid = (lo + hi) >> 1; if (cdf[mid] < x) lo = mid + 1; else hi = mid; }
    int q = min(lo, nf - 1);
    while (q > 0 && Ef[q] <= 0.0) --q;
    const double mu_n = sqrt(ua2);
    const double t = u01d(rb.x) * dt;
    double p1, p2 = 0.0, d1, d2 = 0.0;
    int i, j = 0;
    const int side = a.side;
    if (oned) {
      i = side == 0 ? 0 : a.nx - 1;
      p1 = side == 0 ? a.e1[0] : a.e1[a.nx];
      d1 = side == 0 ? mu_n : -mu_n;
    } else if (a.geom == G_XY) {
      const double mu_t = sqrt(fmax(0.0, 1.0 - mu_n * mu_n));
      const double ct = mu_t * cospi(2.0 * ua3);
      if (along2) {
        j = q; i = side == 0 ? 0 : a.nx - 1;
        p1 = side == 0 ? a.e1[0] : a.e1[a.nx];
        p2 = a.e2[q] + ua1 * (a.e2[q + 1] - a.e2[q]);
        d1 = side == 0 ? mu_n : -mu_n; d2 = ct;
      } else {
        i = q; j = side == 2 ? 0 : a.ny - 1;
        p2 = side == 2 ? a.e2[0] : a.e2[a.ny];
        p1 = a.e1[q] + ua1 * (a.e1[q + 1] - a.e1[q]);
        d2 = side == 2 ? mu_n : -mu_n; d1 = ct;
      }
    } else {
      if (along2) {
        j = q; i = side == 0 ? 0 : a.nx - 1;
        p1 = side == 0 ? a.e1[0] : a.e1[a.nx];
        p2 = a.e2[q] + ua1 * (a.e2[q + 1] - a.e2[q]);
        d1 = side == 0 ? mu_n : -mu_n;
        d2 = 2.0 * ua3 - 1.0;
      } else {
        i = q; j = side == 2 ? 0 : a.ny - 1;
        const double r0 = a.e1[q], r1 = a.e1[q + 1];
        p1 = sqrt(r0 * r0 + ua1 * (r1 * r1 - r0 * r0));
        p2 = side == 2 ? a.e2[0] : a.e2[a.ny];
        d2 = side == 2 ? mu_n : -mu_n;
        d1 = cospi(2.0 * ua3);
      }
    }
    const long long b = base + k;
    a.p1[b] = (float)p1; a.d1[b] = (float)d1;
    if (a.p2) a.p2[b] = (float)p2;
    if (a.d2) a.d2[b] = (float)d2;
    a.wb[b] = wq;
    a.t[b] = (float)t;
    a.cell[b] = i + a.nx * j;
    if (a.group) {
      int g = 0;
      if (a.ng > 1) {
        const U4 rd = draw_rk(rk, (uint32_t)k + a.id_base, 2, step, TAG_BOUNDARY | (uint32_t)a.side);
        g = planck_group(a.faceT[q], a.gedges, a.ng, a.mixcdf, u01d(rb.y), u01d(rb.z), u01d(rb.w), u01d(rd.x),
                         u01d(rd.y), a.below_last != 0);
        if (g < kBndGroups) atomicAdd(&s_gcnt[g], 1u);
        else atomicAdd(a.boundary_group + g, (double)wq);
      }
      a.group[b] = g;
    }
  }
  if (tally_groups) {
    __syncthreads();
    for (int g = threadIdx.x; g < min(a.ng, kBndGroups); g += blockDim.x)
      if (s_gcnt[g]) atomicAdd(a.boundary_group + g, (double)s_gcnt[g] * (double)wq);
  }
  if (wsum) block_add_d((double)n_mine * (double)wq, wsum);
}

__global__ void k_fill_boundary(BndArgs a) { fill_boundary(a.rk, a, blockIdx.x, gridDim.x, nullptr); }

// multigroup categorical sources (MG_IMC/MG_IMC2D.py:1098-1170, 1866-1943) and the MG
// initial census (:992-1097): cell ~ canonical CDF over cells, group ~ the cell's cumulative
// group emission (or the Planck spectrum at tr for the IC), equal weights, uniform position.
__device__ __forceinline__ void fill_mg(const uint32_t* __restrict__ rk, const FillMgArgs& a, int blk, int nblk) {
  const double time_scale = a.time_scale_dev ? *a.time_scale_dev : a.time_scale;  // graph replay
  const uint32_t step = a.step_dev ? *a.step_dev : a.step;
  const long long stride = (long long)nblk * blockDim.x;
  const long long n = *a.d_n, base = *a.d_base;
  if (n <= 0) return;
  const double total = a.cdf[a.nc - 1];
  const float wq = (float)(total / (double)n);
  const bool ic = a.gcdf == nullptr;
  for (long long k = (long long)blk * blockDim.x + threadIdx.x; k < n; k += stride) {
    const U4 ra = draw_rk(rk, (uint32_t)k + a.id_base, 0, step, a.tag);
    const U4 rb = draw_rk(rk, (uint32_t)k + a.id_base, 1, step, a.tag);
    const double x = u01d(ra.x) * total;
    int lo = 0, hi = a.nc;  // first c with cdf[c] > x
    while (lo < hi) { const int mid = (lo + hi) >> 1; if (a.cdf[mid] <= x) lo = mid + 1; else hi = mid; }
    const int c = min(lo, a.nc - 1);
    const int i = c % a.nx, j = c / a.nx;
    const double e1a = a.e1[i], e1b = a.e1[i + 1], e2a = a.e2[j], e2b = a.e2[j + 1];
    int g;
    double up1, up2, ua, ub, ut;
    if (!ic) {
      const double* gc = a.gcdf + (size_t)c * a.ng;
      const double y = u01d(ra.y) * gc[a.ng - 1];
      g = a.ng - 1;
      for (int q = 0; q < a.ng; ++q) if (gc[q] >= y) { g = q; break; }
      up1 = u01d(ra.z); up2 = u01d(ra.w); ua = u01d(rb.x); ub = u01d(rb.y); ut = u01d(rb.z);
    } else {
      const U4 rd = draw_rk(rk, (uint32_t)k + a.id_base, 2, step, a.tag);
      up1 = u01d(ra.y); up2 = u01d(ra.z); ua = u01d(ra.w); ub = u01d(rb.x); ut = 0.0;
      g = planck_group(a.tr[c], a.gedges, a.ng, a.mixcdf, u01d(rb.y), u01d(rb.z), u01d(rb.w), u01d(rd.x), u01d(rd.y));
    }
    double p1 = (a.geom == G_RZ) ? sqrt(e1a * e1a + up1 * (e1b * e1b - e1a * e1a)) : e1a + up1 * (e1b - e1a);
    const double p2 = e2a + up2 * (e2b - e2a);
    double d1, d2;
    iso_dir(a.geom, ua, ub, d1, d2);
    const long long b = base + k;
    a.p1[b] = (float)p1; a.p2[b] = (float)p2;
    a.d1[b] = (float)d1; a.d2[b] = (float)d2;
    a.wb[b] = wq;
    a.t[b] = (float)(ut * time_scale);
    a.cell[b] = c;
    a.group[b] = g;
  }
}

__global__ void k_fill_mg(FillMgArgs a) { fill_mg(a.rk, a, blockIdx.x, gridDim.x); }

// The weights of the census entries [0, *n_census) and of every volume source of the job
// table, from its plan: order position o issues off[o+1] - off[o] particles of weight
// w[c(o)] (w[o] with bins by group); a multigroup fill issues n particles of weight
// (float)(total / n).  With the boundary jobs' own sums, *wsum ends as the sum of the
// weights of every tracked entry.
__device__ __forceinline__ void census_wsum(const SourceJobs& j, int blk, int nblk) {
  const long long stride = (long long)nblk * blockDim.x;
  const long long t0 = (long long)blk * blockDim.x + threadIdx.x;
  const long long n = *j.n_census;
  double s = 0.0;
  for (long long k = t0; k < n; k += stride) s += (double)j.census_w[k];
  for (int v = 0; v < j.n_vol; ++v) {
    const FillArgs& a = j.vol[v];
    for (long long o = t0; o < a.nbins; o += stride) {
      const long long cnt = a.off[o + 1] - a.off[o];
      if (cnt <= 0) continue;
      int wi = (int)o;
      if (!a.bins_by_group) { const int i = (int)o / a.ny, jj = (int)o - i * a.ny; wi = i + a.nx * jj; }
      s += (double)cnt * (double)a.w[wi];
    }
  }
  if (t0 == 0)
    for (int v = 0; v < j.n_vmg; ++v) {
      const long long nm = *j.vmg[v].d_n;
      if (nm > 0) s += (double)nm * (double)(float)(j.vmg[v].cdf[j.vmg[v].nc - 1] / (double)nm);
    }
  block_add_d(s, j.wsum);
}

// Source jobs in one launch: block b runs the job whose range holds b.  KINDS (bits
// 1 << JOB_*) selects the bodies compiled into an instance, so the volume fills keep the
// registers of their own kernel instead of the largest of all the bodies.
template <int KINDS>
__global__ void __launch_bounds__(256) k_fill_sources(const __grid_constant__ SourceJobs j) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  int q = 0;
  while (q + 1 < j.n_jobs && (int)blockIdx.x >= j.first_block[q + 1]) ++q;
  const int blk = (int)blockIdx.x - j.first_block[q];
  const int nblk = j.first_block[q + 1] - j.first_block[q];
  constexpr bool VOL = KINDS & (1 << JOB_VOLUME), VMG = KINDS & (1 << JOB_VOLUME_MG);
  constexpr bool BND = KINDS & (1 << JOB_BOUNDARY), CEN = KINDS & (1 << JOB_CENSUS_WSUM);
  // one case per (kind, slot): constant indices keep every argument a direct operand of
  // the parameter block (a run-time index would load them into registers)
  switch (j.kind[q] * 4 + j.slot[q]) {
    case JOB_VOLUME * 4 + 0: if (VOL) fill_volume(j.rk, j.vol[0], blk, nblk); break;
    case JOB_VOLUME * 4 + 1: if (VOL) fill_volume(j.rk, j.vol[1], blk, nblk); break;
    case JOB_VOLUME_MG * 4 + 0: if (VMG) fill_mg(j.rk, j.vmg[0], blk, nblk); break;
    case JOB_VOLUME_MG * 4 + 1: if (VMG) fill_mg(j.rk, j.vmg[1], blk, nblk); break;
    case JOB_BOUNDARY * 4 + 0: if (BND) fill_boundary(j.rk, j.bnd[0], blk, nblk, j.wsum); break;
    case JOB_BOUNDARY * 4 + 1: if (BND) fill_boundary(j.rk, j.bnd[1], blk, nblk, j.wsum); break;
    case JOB_BOUNDARY * 4 + 2: if (BND) fill_boundary(j.rk, j.bnd[2], blk, nblk, j.wsum); break;
    case JOB_BOUNDARY * 4 + 3: if (BND) fill_boundary(j.rk, j.bnd[3], blk, nblk, j.wsum); break;
    default: if (CEN) census_wsum(j, blk, nblk); break;
  }
}

__global__ void k_wsum(const float* w, const int64_t* d_n, double* out) {
  __shared__ double sh[32];
  const long long n = *d_n;
  double s = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) s += (double)w[k];
  s = warp_sum_d(s);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    v = warp_sum_d(v);
    if (threadIdx.x == 0 && v != 0.0) atomicAdd(out, v);
  }
}

int grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  if (g > 148LL * 16) g = 148LL * 16;
  return (int)(g < 1 ? 1 : g);
}

}  // namespace

cudaError_t imc_launch_fill_volume(const FillArgs& a, cudaStream_t s) {
  if (a.n_bound <= 0) return cudaSuccess;
  ++g_imc_launches;
  k_fill_volume<<<grid_for(a.n_bound, 256), 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t imc_launch_fill_boundary(const BndArgs& a, cudaStream_t s) {
  if (a.n_bound <= 0) return cudaSuccess;
  ++g_imc_launches;
  k_fill_boundary<<<grid_for(a.n_bound, 256), 256, 0, s>>>(a);
  return cudaGetLastError();
}

int imc_source_blocks(long long n_bound) { return grid_for(n_bound, 256); }

cudaError_t imc_launch_sources(const SourceJobs& j, cudaStream_t s) {
  if (j.n_jobs <= 0) return cudaSuccess;
  if (j.n_jobs > kSourceJobsMax) return cudaErrorInvalidValue;
  int kinds = 0;
  for (int q = 0; q < j.n_jobs; ++q) kinds |= 1 << j.kind[q];
  const int grid = j.first_block[j.n_jobs];
  constexpr int kVol = 1 << JOB_VOLUME, kVmg = 1 << JOB_VOLUME_MG;
  constexpr int kAux = (1 << JOB_BOUNDARY) | (1 << JOB_CENSUS_WSUM);
  ++g_imc_launches;
  // an instance per kind of fill: the gray and the multigroup volume fills never share a step
  if (kinds == kVol) IMC_LAUNCH_PDL(k_fill_sources<kVol>, grid, 256, 0, s, j);
  else if (kinds == kVmg) IMC_LAUNCH_PDL(k_fill_sources<kVmg>, grid, 256, 0, s, j);
  else if ((kinds & ~kAux) == 0) IMC_LAUNCH_PDL(k_fill_sources<kAux>, grid, 256, 0, s, j);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t imc_launch_fill_mg(const FillMgArgs& a, cudaStream_t s) {
  if (a.n_bound <= 0) return cudaSuccess;
  ++g_imc_launches;
  k_fill_mg<<<grid_for(a.n_bound, 256), 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t imc_launch_wsum(const float* w, const int64_t* d_n, long long n_bound, double* out, cudaStream_t s) {
  if (n_bound <= 0) return cudaSuccess;
  ++g_imc_launches;
  k_wsum<<<grid_for(n_bound, 256), 256, 0, s>>>(w, d_n, out);
  return cudaGetLastError();
}
