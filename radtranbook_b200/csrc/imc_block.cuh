// imc_block.cuh — single-block FP64 building blocks shared by the per-problem planning
// kernels (one 1024-thread block per problem): the canonical summation order, the count
// scan and the volume-source plan.  Files that include this are compiled without FMA
// contraction, so the numbers match the CPU oracle's (canon_sum, ceil counts) exactly.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace imcblk {

constexpr int NT = 1024;

__device__ __forceinline__ double pow4(double T) { const double t2 = T * T; return t2 * t2; }
__device__ __forceinline__ double pow3(double T) { return T * T * T; }

// 1024 strided partial sums, then a halving tree (the oracle's canon_sum).  Each partial
// loads B of its terms at a time before adding them in order (same sum, fewer waits; B = 16
// only where the kernel has registers to spare at 1024 threads).
template <int B = 8>
__device__ inline double block_canon_sum(const double* x, long long n, double* red) {
  const int t = threadIdx.x;
  double s = 0.0;
  for (long long i0 = t; i0 < n; i0 += (long long)B * NT) {
    double v[B];
#pragma unroll
    for (int j = 0; j < B; ++j) { const long long i = i0 + (long long)j * NT; v[j] = i < n ? x[i] : 0.0; }
#pragma unroll
    for (int j = 0; j < B; ++j) if (i0 + (long long)j * NT < n) s += v[j];
  }
  red[t] = s;
  __syncthreads();
  for (int h = NT / 2; h >= 1; h >>= 1) {
    if (t < h) red[t] += red[t + h];
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

// Exclusive scan of per-order-position counts n[0..m) into off[0..m]; returns the total.
// Integer sums are exact in any order: each thread sums a contiguous chunk, the chunk totals
// are scanned by warp shuffles (then the 32 warp totals by one warp), and each thread writes
// its chunk's offsets.  sh needs 32 entries.
__device__ inline long long block_scan_counts(const long long* n, long long* off, int m, long long* sh) {
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const int per = (m + NT - 1) / NT;
  const int lo = min(t * per, m), hi = min(lo + per, m);
  long long s = 0;
  for (int o = lo; o < hi; ++o) s += n[o];
  long long x = s;  // inclusive scan within the warp
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) { const long long y = __shfl_up_sync(0xffffffffu, x, d); if (lane >= d) x += y; }
  if (lane == 31) sh[wid] = x;
  __syncthreads();
  if (wid == 0) {
    long long v = lane < NT / 32 ? sh[lane] : 0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) { const long long y = __shfl_up_sync(0xffffffffu, v, d); if (lane >= d) v += y; }
    sh[lane] = v;  // inclusive over the warps
  }
  __syncthreads();
  long long run = x - s + (wid ? sh[wid - 1] : 0);  // this thread's exclusive offset
  const long long total = sh[NT / 32 - 1];
  __syncthreads();  // sh is the caller's again
  for (int o = lo; o < hi; ++o) { const long long v = n[o]; off[o] = run; run += v; }
  if (t == 0) off[m] = total;
  __syncthreads();
  return total;
}

// order position o = i*ny + j (the reference's i-outer, j-inner source loops)
__device__ __forceinline__ int order_to_cell(int o, int nx, int ny) {
  const int i = o / ny, j = o - (o / ny) * ny;
  return i + nx * j;
}

// Volume-source counts (ceil(N QV_c / Q), in source order; min1_round: max(1, round), the
// Carter-Forest 1-D emission rule), per-cell weights and the energy actually issued per
// cell (n_c times the FP32 weight, exact in FP64).
__device__ inline long long plan_volume(const double* QV, long long N, int nx, int ny, int nc, long long* cnt,
                                 long long* off, float* w, double* issued, double* red, long long* sh,
                                 bool min1_round = false) {
  const double Qt = block_canon_sum(QV, nc, red);
  // cells in storage order (coalesced loads); the count goes to the cell's order position
  for (int c = threadIdx.x; c < nc; c += NT) {
    const int ci = c % nx, o = ci * ny + c / nx;
    long long n = 0;
    if (Qt > 0.0 && N > 0)
      n = min1_round ? max(1LL, (long long)rint((double)N * QV[c] / Qt)) : (long long)ceil((double)N * QV[c] / Qt);
    cnt[o] = n;
    const float wc = n > 0 ? (float)(QV[c] / (double)n) : 0.f;
    w[c] = wc;
    issued[c] = (double)n * (double)wc;
  }
  __syncthreads();
  return block_scan_counts(cnt, off, nc, sh);
}

}  // namespace imcblk
