// imc_comb.cu — stochastic comb of the census bank (IMC/IMC1D.py:770-828,
// IMC/IMC2D.py:1448-1511, MG_IMC/MG_IMC2D.py:1270-1378).
//
//   1. ecen[b]  = sum of live weights per bin (cell, or cell + nc*group)      k_comb_ecen
//   2. ew[b]    = ecen / max(1, rint(Nmax ecen / E))                          k_comb_plan
//   3. n_k      = floor(w_k / ew[b] + xi_k), xi word k % 4 of Philox block
//      (k / 4, 1, step, TAG_COMB); per-block totals                          k_comb_count
//   4. exclusive scan of block totals                                         k_comb_scan
//   5. copies written in bank order (block-local scan + block offset; entries
//      staged in shared memory, one thread per output copy)                  k_comb_scatter
//   6. disc[b] = ecen - (copies in b) * FP32(ew), and optionally that energy
//      after the comb per bin (exact: equal FP32 weights summed in FP64)         k_comb_disc
// Order of the output bank = order of the input bank, so the result is deterministic.
// Modes (MG_IMC/MG_IMC1D.py:1187-1200, 808-820): when the comb plan decides not to comb
// (Nmax = 0, or fewer live entries than a threshold) every live entry is copied once with its
// weight (disc = 0); with conserve_rad each bin's copies share its pre-comb energy equally.
#include "imc_device.cuh"
#include "imc_internal.h"

using namespace imcdev;

namespace {

constexpr int TILE = 4096;      // entries per count / scatter block (one block total each for the scan)
constexpr int CNT_T = 256;      // count threads per block (TILE / CNT_T entries each)
constexpr int CNT_SLOTS = 512;  // count: shared-memory bins per block

__device__ __forceinline__ int bin_of(const CombArgs& a, long long k) {
  return a.per_group ? a.cell[k] + a.nc * a.group[k] : a.cell[k];
}

// Bounds-checked build: a bin outside [0, nb) is reported and its entry treated as dead.
__device__ __forceinline__ bool bin_ok(const CombArgs& a, int b) {
#ifdef IMC_CHECKED
  if (b >= 0 && b < a.nb) return true;
  if (a.sum) atomicOr(&a.sum->flags, (int)IMC_FLAG_BOUNDS);
  return false;
#else
  (void)a; (void)b;
  return true;
#endif
}

// weight of every copy in bin b: the comb weight, or the bin's energy shared equally
__device__ __forceinline__ float copy_weight(const CombArgs& a, int b) {
  if (!a.conserve_rad) return (float)a.ew[b];
  const double n = (double)a.ncopy[b];
  return n > 0.0 ? (float)(a.ecen[b] / n) : 0.f;
}

constexpr int ECH = 4096;       // consecutive entries per k_comb_ecen block
constexpr int EBINS = 1024;     // shared-memory bins per block

// Each block sums a contiguous run of ECH entries into its shared bins (warp groups first),
// then adds one value per distinct bin to ecen.
__global__ void __launch_bounds__(256) k_comb_ecen(CombArgs a) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  __shared__ BlockBins<EBINS> t;
  __shared__ WarpStage stages[8];
  WarpStage* st = stages + (threadIdx.x >> 5);
  bins_init(t);
  __syncthreads();
  const long long n_in = min((long long)*a.d_n_in, (long long)a.n_bound);  // a count above the bound is never read
  const long long base = (long long)blockIdx.x * ECH;
  // block-uniform trip count keeps every warp converged for the aggregated reduction
  unsigned n_live = 0;
  for (int i = 0; i < ECH; i += 256) {
    const long long k = base + i + threadIdx.x;
    bool live = false;
    int b = 0;
    double w = 0.0;
    if (k < n_in) {
      const float wf = a.w[k];
      if (wf > 0.f) { b = bin_of(a, k); live = bin_ok(a, b); w = live ? (double)wf : 0.0; if (!live) b = 0; }
    }
    n_live += live ? 1u : 0u;
    warp_bins_add(live, b, w, t, a.ecen, st);
  }
  n_live = __reduce_add_sync(FULL, n_live);
  if ((threadIdx.x & 31) == 0 && n_live && a.n_live) atomicAdd(a.n_live, (unsigned long long)n_live);
  __syncthreads();
  bins_flush(t, a.ecen);
}

// Each block combs a tile of TILE consecutive entries; each of its CNT_T threads takes CNT_PER
// consecutive entries (16-byte vector loads and stores when the bank arrays allow them):
// copies per entry, the tile's total for the scan, and copies per bin, summed in registers
// over runs of equal bins (the bank is largely grouped by cell) and added to the block's
// table when the bin changes, so the loop has no warp-wide step.
constexpr int CNT_PER = TILE / CNT_T;

// copies of one entry: floor(w / ew + xi), xi its comb uniform (word k % 4 of Philox block
// (k / 4, 1, step, TAG_COMB), k the pre-comb index)
__device__ __forceinline__ int comb_copies(const CombArgs& a, float wf, int bk, bool compact, uint32_t xw, int& b) {
  b = 0;
  if (!(wf > 0.f) || !bin_ok(a, bk)) return 0;
  b = bk;
  if (compact) return 1;
  const double ew = a.ew[b];
  if (!(ew > 0.0)) return 0;
  return (int)floor((double)wf / ew + u01d(xw));
}

__global__ void __launch_bounds__(CNT_T) k_comb_count(CombArgs a) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  const uint32_t step = a.step_dev ? *a.step_dev : a.step;  // graph replay
  __shared__ unsigned sh[CNT_T / 32];
  __shared__ BlockCounts<CNT_SLOTS> t;
  counts_init(t);
  __syncthreads();
  const long long n_in = min((long long)*a.d_n_in, (long long)a.n_bound);  // the grid covers n_bound entries
  const bool compact = *a.mode != 0;
  const long long k0 = (long long)blockIdx.x * TILE + (long long)threadIdx.x * CNT_PER;
  unsigned tsum = 0, run_n = 0;
  int run_b = -1;
#pragma unroll 1
  for (int j = 0; j < CNT_PER; j += 4) {
    const long long kj = k0 + j;
    float wv[4] = {0.f, 0.f, 0.f, 0.f};
    int bv[4] = {0, 0, 0, 0};
    if (a.vec16 && kj + 3 < n_in) {  // kj % 4 == 0: the 16-byte loads are aligned
      const float4 W = *reinterpret_cast<const float4*>(a.w + kj);
      const int4 C = *reinterpret_cast<const int4*>(a.cell + kj);
      wv[0] = W.x; wv[1] = W.y; wv[2] = W.z; wv[3] = W.w;
      bv[0] = C.x; bv[1] = C.y; bv[2] = C.z; bv[3] = C.w;
      if (a.per_group) {
        const int4 g = *reinterpret_cast<const int4*>(a.group + kj);
        bv[0] += a.nc * g.x; bv[1] += a.nc * g.y; bv[2] += a.nc * g.z; bv[3] += a.nc * g.w;
      }
    } else {
      for (int q = 0; q < 4; ++q)
        if (kj + q < n_in) { wv[q] = a.w[kj + q]; bv[q] = bin_of(a, kj + q); }
    }
    // one Philox block for the four entries kj..kj+3 (kj % 4 == 0), drawn when one of them is alive
    U4 r{0u, 0u, 0u, 0u};
    if (!compact && (wv[0] > 0.f || wv[1] > 0.f || wv[2] > 0.f || wv[3] > 0.f))
      r = draw_rk(a.rk, (uint32_t)(kj >> 2), 1, step, TAG_COMB);
    int nv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int b;
      const int n = kj + q < n_in ? comb_copies(a, wv[q], bv[q], compact, u4_word(r, q), b) : 0;
      nv[q] = n;
      tsum += (unsigned)n;
      if (n > 0) {
        if (b != run_b) {
          if (run_n) counts_add(t, run_b, run_n, a.ncopy);
          run_b = b;
          run_n = 0;
        }
        run_n += (unsigned)n;
      }
    }
    if (kj + 3 < n_in) {
      *reinterpret_cast<int4*>(a.cnt + kj) = make_int4(nv[0], nv[1], nv[2], nv[3]);  // workspace: aligned
    } else {
      for (int q = 0; q < 4; ++q) if (kj + q < n_in) a.cnt[kj + q] = nv[q];
    }
  }
  if (run_n) counts_add(t, run_b, run_n, a.ncopy);
  const unsigned ws = __reduce_add_sync(FULL, tsum);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = ws;
  __syncthreads();
  counts_flush(t, a.ncopy);
  if (threadIdx.x == 0) {
    unsigned long long v = 0;
    for (int q = 0; q < CNT_T / 32; ++q) v += sh[q];
    a.blk[blockIdx.x] = (long long)v;
  }
}

// exclusive scan of nblk block totals in place (blk[nblk] = total), single block
__global__ void __launch_bounds__(1024) k_comb_scan(long long* blk, long long nblk, long long out_capacity,
                                                    imc_step_summary* sum) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  __shared__ long long sh[1024];
  const int t = threadIdx.x;
  const long long per = (nblk + 1023) / 1024;
  const long long lo = min((long long)t * per, nblk), hi = min(lo + per, nblk);
  long long s = 0;
  for (long long q = lo; q < hi; ++q) s += blk[q];
  sh[t] = s;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    const long long v = t >= d ? sh[t - d] : 0;
    __syncthreads();
    sh[t] += v;
    __syncthreads();
  }
  long long run = sh[t] - s;
  for (long long q = lo; q < hi; ++q) { const long long x = blk[q]; blk[q] = run; run += x; }
  if (t == 1023) {
    const long long total = sh[1023];
    blk[nblk] = total;
    sum->n_out = total;
    if (total > out_capacity) { atomicOr(&sum->flags, (int)IMC_FLAG_COMB_OVERFLOW); sum->n_census = 0; }
    else sum->n_census = total;  // the combed bank is the next step's census
  }
}

// One thread per output copy: the tile's copy counts are scanned in shared memory (each
// thread owns 4 consecutive entries), each thread finds the entry of its copy by a binary
// search there and gathers the entry's fields (cached: a tile's entries are few), so the
// output stores are contiguous across the warp.
// Shared memory of k_comb_scatter: the tile's inclusive copy counts, then its entries'
// fields (pos1, dir1, cell; pos2, dir2 in 2-D; group when the bank has one), TILE each.
__host__ __device__ inline int scatter_fields(bool two_d, bool grp) { return 3 + (two_d ? 2 : 0) + (grp ? 1 : 0); }
__host__ __device__ inline size_t scatter_smem(bool two_d, bool grp) {
  return sizeof(int) * (size_t)TILE * (1 + scatter_fields(two_d, grp));
}

// The tile's entries are staged in shared memory with 16-byte loads (one thread per four
// entries, as the count kernel tiled them), then one thread per output copy finds its entry
// by a binary search of the scanned counts and copies its fields from shared memory, so the
// global loads and the stores of a warp are both contiguous.
__global__ void __launch_bounds__(1024) k_comb_scatter(CombArgs a) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  extern __shared__ __align__(16) int sm_tile[];
  __shared__ int sh[32];
  const bool two_d = a.p2 != nullptr, grp = a.group != nullptr;
  int* incl = sm_tile;
  float* sP1 = reinterpret_cast<float*>(incl + TILE);
  float* sD1 = sP1 + TILE;
  int* sC = reinterpret_cast<int*>(sD1 + TILE);
  float* sP2 = reinterpret_cast<float*>(sC + TILE);   // 2-D only
  float* sD2 = sP2 + TILE;                            // 2-D only
  int* sG = reinterpret_cast<int*>(two_d ? sD2 + TILE : sP2);  // with a group array only
  const long long tile0 = (long long)blockIdx.x * TILE;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long n_in = min((long long)*a.d_n_in, (long long)a.n_bound);
  const int q0 = 4 * threadIdx.x;
  const long long k0 = tile0 + q0;
  const bool full = k0 + 3 < n_in;
  int c[4] = {0, 0, 0, 0};
  if (full) {
    const int4 v = *reinterpret_cast<const int4*>(a.cnt + k0);  // 16-byte aligned: k0 % 4 == 0
    c[0] = v.x; c[1] = v.y; c[2] = v.z; c[3] = v.w;
  } else {
    for (int j = 0; j < 4; ++j) if (k0 + j < n_in) c[j] = a.cnt[k0 + j];
  }
  const int s4 = c[0] + c[1] + c[2] + c[3];
  // stage the fields of the four entries (only where they have copies)
  const uintptr_t al = reinterpret_cast<uintptr_t>(a.p1) | reinterpret_cast<uintptr_t>(a.d1) |
                       reinterpret_cast<uintptr_t>(a.p2) | reinterpret_cast<uintptr_t>(a.d2);
  if (s4 > 0) {
    if (full && a.vec16 && (al & 15u) == 0) {
      *reinterpret_cast<float4*>(sP1 + q0) = *reinterpret_cast<const float4*>(a.p1 + k0);
      *reinterpret_cast<float4*>(sD1 + q0) = *reinterpret_cast<const float4*>(a.d1 + k0);
      *reinterpret_cast<int4*>(sC + q0) = *reinterpret_cast<const int4*>(a.cell + k0);
      if (two_d) {
        *reinterpret_cast<float4*>(sP2 + q0) = *reinterpret_cast<const float4*>(a.p2 + k0);
        *reinterpret_cast<float4*>(sD2 + q0) = *reinterpret_cast<const float4*>(a.d2 + k0);
      }
      if (grp) *reinterpret_cast<int4*>(sG + q0) = *reinterpret_cast<const int4*>(a.group + k0);
    } else {
      for (int j = 0; j < 4; ++j) {
        if (c[j] == 0) continue;
        const long long k = k0 + j;
        sP1[q0 + j] = a.p1[k]; sD1[q0 + j] = a.d1[k]; sC[q0 + j] = a.cell[k];
        if (two_d) { sP2[q0 + j] = a.p2[k]; sD2[q0 + j] = a.d2[k]; }
        if (grp) sG[q0 + j] = a.group[k];
      }
    }
  }
  // block-exclusive scan of the threads' sums, then the entries' inclusive sums
  int x = s4;
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
  int run = x - s4 + (wid ? sh[wid - 1] : 0);
#pragma unroll
  for (int j = 0; j < 4; ++j) { run += c[j]; incl[q0 + j] = run; }
  __syncthreads();
  const int total = incl[TILE - 1];
  const long long out0 = a.blk[blockIdx.x];
  const bool compact = *a.mode != 0;
  for (int o = threadIdx.x; o < total; o += blockDim.x) {
    const long long dst = out0 + o;
    if (dst >= a.out_capacity) break;  // overflow: flagged by the scan, caller regrows
    int lo = 0, hi = TILE - 1;  // the entry j with incl[j-1] <= o < incl[j]
    while (lo < hi) { const int mid = (lo + hi) >> 1; if (incl[mid] > o) hi = mid; else lo = mid + 1; }
    const int cl = sC[lo];
    const int gr = grp ? sG[lo] : 0;
    a.op1[dst] = sP1[lo]; a.od1[dst] = sD1[lo];
    if (two_d) { a.op2[dst] = sP2[lo]; a.od2[dst] = sD2[lo]; }
    a.ow[dst] = compact ? a.w[tile0 + lo] : copy_weight(a, a.per_group ? cl + a.nc * gr : cl);
    a.ot[dst] = 0.f; a.ocell[dst] = cl;
    if (a.ogroup) a.ogroup[dst] = gr;
  }
}

__global__ void k_comb_disc(CombArgs a) {
  pdl_wait();     // the previous kernel of the stream has completed
  pdl_trigger();  // the next one may be scheduled
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  double after = 0.0;
  if (b < a.nb) {
    // compact only: every live entry kept with its weight, nothing is lost
    after = *a.mode != 0 ? a.ecen[b] : (double)a.ncopy[b] * (double)copy_weight(a, b);
    a.disc[b] = a.ecen[b] - after;
    if (a.after) a.after[b] = after;
  }
  after = warp_sum_d(after);
  if ((threadIdx.x & 31) == 0 && after != 0.0) atomicAdd(&a.sum->comb_after, after);
}

}  // namespace

cudaError_t imc_launch_comb_ecen(const CombArgs& a, cudaStream_t s) {
  if (a.n_bound <= 0) return cudaSuccess;
  ++g_imc_launches;
  IMC_LAUNCH_PDL(k_comb_ecen, (unsigned)((a.n_bound + ECH - 1) / ECH), 256, 0, s, a);
  return cudaGetLastError();
}

cudaError_t imc_launch_comb_count(const CombArgs& a, cudaStream_t s) {
  const long long nblk = (a.n_bound + TILE - 1) / TILE;
  if (nblk > 0) {
    ++g_imc_launches;
    IMC_LAUNCH_PDL(k_comb_count, (unsigned)nblk, CNT_T, 0, s, a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  ++g_imc_launches;
  IMC_LAUNCH_PDL(k_comb_scan, 1, 1024, 0, s, a.blk, nblk, a.out_capacity, a.sum);
  return cudaGetLastError();
}

cudaError_t imc_launch_comb_scatter(const CombArgs& a, cudaStream_t s) {
  const long long nblk = (a.n_bound + TILE - 1) / TILE;
  if (nblk > 0) {
    ++g_imc_launches;
    // the attribute allows the largest layout (2-D with groups), set once per device
    static bool attr_set[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
      e = cudaFuncSetAttribute(k_comb_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)scatter_smem(true, true));
      if (e != cudaSuccess) return e;
      if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
    IMC_LAUNCH_PDL(k_comb_scatter, (unsigned)nblk, 1024, scatter_smem(a.p2 != nullptr, a.group != nullptr), s, a);
  }
  ++g_imc_launches;
  IMC_LAUNCH_PDL(k_comb_disc, (a.nb + 255) / 256, 256, 0, s, a);
  return cudaGetLastError();
}
