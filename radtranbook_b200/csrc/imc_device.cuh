// imc_device.cuh — device building blocks of the B200 IMC engine.
//
//  * Philox-4x32-10 (Salmon et al., SC'11), keyed by the run seed, counter
//    (particle index, draw block / event number, step, stream tag).
//  * 23-bit open-interval uniforms, identical in FP32 and FP64.
//  * FP32 event geometry for slab / sphere / xy / rz (the reference's event
//    functions IMC/IMC1D.py:75-130, 336-436 and IMC/IMC2D.py:711-935, rewritten in
//    cancellation-free form; the cell index, not the position, decides the cell).
//  * Warp-aggregated FP64 tally reduction (match_any + per-warp shared staging).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace imcdev {

constexpr double C_LIGHT = 29.98;
constexpr double A_RAD = 0.01372;
constexpr float BIGF = 1e30f;
constexpr unsigned FULL = 0xffffffffu;

enum : int { G_SLAB = 0, G_SPHERE = 1, G_XY = 2, G_RZ = 3 };
enum : int { EV_CENSUS = 0, EV_BOUNDARY = 1, EV_SCATTER = 2 };
enum : int { X_NONE = 0, X_IP = 1, X_IM = 2, X_JP = 3, X_JM = 4 };
enum : int { S_EVENTS = 0, S_BOUNDARY, S_SCATTER, S_CENSUS, S_CAPTURE, S_FLOOR, S_REFLECT, S_CAP, S_ESCAPE, S_N };

enum : uint32_t {
  TAG_TRANSPORT = 0x10000000u,
  TAG_BOUNDARY = 0x20000000u,
  TAG_SOURCE = 0x30000000u,
  TAG_EMISSION = 0x40000000u,
  TAG_IC = 0x50000000u,
  TAG_COMB = 0x60000000u,
};

struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
  }
  return c;
}

// ((x>>9) + 0.5) * 2^-23 = (2k+1) * 2^-24, k < 2^23: 24 significant bits, so exact in
// float and double alike, and never 0 or 1.
__device__ __forceinline__ float u01f(uint32_t x) { return __uint2float_rn(((x >> 9) << 1) | 1u) * 5.9604644775390625e-8f; }
__device__ __forceinline__ double u01d(uint32_t x) { return (double)(((x >> 9) << 1) | 1u) * 5.9604644775390625e-8; }

__device__ __forceinline__ U4 draw(uint64_t seed, uint32_t idx, uint32_t block, uint32_t step, uint32_t tag) {
  return philox4x32_10(U4{idx, block, step, tag}, (uint32_t)seed, (uint32_t)(seed >> 32));
}

// The 20 round keys of a seed (k0 + r*0x9E3779B9, k1 + r*0xBB67AE85, r = 0..9), for kernels
// that carry them in their parameter block: the rounds then read them as constant operands
// instead of stepping the key in registers.  Same outputs as draw().
__host__ __device__ inline void philox_round_keys(uint64_t seed, uint32_t* rk) {
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  for (int r = 0; r < 10; ++r) {
    rk[2 * r] = k0; rk[2 * r + 1] = k1;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
}

__device__ __forceinline__ U4 draw_rk(const uint32_t* rk, uint32_t idx, uint32_t block, uint32_t step,
                                      uint32_t tag) {
  U4 c{idx, block, step, tag};
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = U4{hi1 ^ c.y ^ rk[2 * r], lo1, hi0 ^ c.w ^ rk[2 * r + 1], lo0};
  }
  return c;
}

// draw_rk with the round keys read as five 16-byte words (rk4: the 20 keys of
// philox_round_keys, 16-byte aligned, e.g. staged in shared memory): the same numbers, five
// vector loads where draw_rk makes twenty scalar ones.
__device__ __forceinline__ U4 draw_rk4(const uint4* rk4, uint32_t idx, uint32_t block, uint32_t step,
                                       uint32_t tag) {
  U4 c{idx, block, step, tag};
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const uint4 k = rk4[q];
    const uint32_t a0 = 0xD2511F53u * c.x, b0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t a1 = 0xCD9E8D57u * c.z, b1 = __umulhi(0xCD9E8D57u, c.z);
    c = U4{b1 ^ c.y ^ k.x, a1, b0 ^ c.w ^ k.y, a0};
    const uint32_t e0 = 0xD2511F53u * c.x, f0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t e1 = 0xCD9E8D57u * c.z, f1 = __umulhi(0xCD9E8D57u, c.z);
    c = U4{f1 ^ c.y ^ k.z, e1, f0 ^ c.w ^ k.w, e0};
  }
  return c;
}

// Word q (0..3) of a Philox block: the comb's uniform of pre-comb entry k is word k % 4 of
// block (k / 4, 1), so four consecutive entries share one block.
__device__ __forceinline__ uint32_t u4_word(const U4& r, int q) {
  return q == 0 ? r.x : q == 1 ? r.y : q == 2 ? r.z : r.w;
}

// -log(u) for u = u01: distance in mean free paths.
__device__ __forceinline__ float neglog_u(uint32_t x) { return -logf(u01f(x)); }

// Effective-scatter distance with the optically-thick cap of the reference
// (IMC/IMC1D.py:83-88; IMC/IMC2D.py:758-765): sigma_s*L > 1e4 uses sigma = 1e4/L.
__device__ __forceinline__ float scatter_distance(float ss, float L, uint32_t x, float thresh, bool cap) {
  if (cap && ss * L > 10000.0f) return neglog_u(x) * (L * 1e-4f);
  if (ss > thresh) return neglog_u(x) / ss;
  return BIGF;
}

struct Ev {
  float d;       // path length of this event
  int evt;       // EV_*
  int cross;     // X_*
};

// ---- 1-D slab: distance to the exit face in the direction of mu ----
__device__ __forceinline__ float slab_face(float x, float mu, float xl, float xr) {
  const float db = __fdividef(mu > 0.f ? (xr - x) : (xl - x), mu);
  return fmaxf(db, 0.f);
}

// ---- sphere / cylinder: cancellation-free roots of l^2 + 2 r mu l + (r^2 - R^2) = 0 ----
// sqrt(x) = x * x^(-1/2): one hardware reciprocal square root and a multiply (a few ulp,
// against the ~10-instruction correctly rounded sqrtf); 0 for x <= 0.  Tracking is FP32
// with statistical tolerances, and every kernel that replays a history uses the same form.
__device__ __forceinline__ float sqrt_nn(float x) { return x > 0.f ? x * rsqrtf(x) : 0.f; }

__device__ __forceinline__ float outer_root(float r, float mu, float R, float b2) {
  const float q = sqrt_nn(fmaf(R, R, -b2));
  float l = (mu >= 0.f) ? __fdividef((R - r) * (R + r), fmaxf(fmaf(r, mu, q), 1e-30f)) : q - r * mu;
  return fmaxf(l, 0.f);
}
__device__ __forceinline__ float inner_root(float r, float mu, float R, float b2) {
  if (!(R > 0.f) || !(mu < 0.f)) return BIGF;
  const float disc = fmaf(R, R, -b2);
  if (!(disc > 0.f)) return BIGF;
  const float l = __fdividef((r - R) * (r + R), disc * rsqrtf(disc) - r * mu);
  return fmaxf(l, 0.f);
}

// ---- warp-aggregated FP64 reduction into global tallies ----
// Every lane of the warp must call this (converged).  Lanes with flush=false pass any
// key.  Lanes flushing the same cell are grouped with __match_any_sync; the lowest lane
// of each group sums the group's values (staged in per-warp shared memory) and issues
// one FP64 red per tally.
struct WarpStage { double a[32]; double b[32]; };

// Asynchronous 4-byte global -> shared copies (cp.async): a thread starts the copies of a bank
// record it will need later and waits for its own copies only when it reads them.
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ void warp_tally2(bool flush, int key, double va, double vb,
                                            double* __restrict__ ta, double* __restrict__ tb,
                                            WarpStage* st) {
  const unsigned fm = __ballot_sync(FULL, flush);
  if (fm == 0u) return;
  const int lane = threadIdx.x & 31;
  const int k = flush ? key : -1 - lane;  // keys >= 0 for flushing lanes are cells
  const unsigned peers = __match_any_sync(FULL, k);
  if (__all_sync(FULL, !flush || __popc(peers) == 1)) {
    if (flush) { atomicAdd(ta + key, va); atomicAdd(tb + key, vb); }
    return;
  }
  st->a[lane] = va; st->b[lane] = vb;
  __syncwarp();
  if (flush && (__ffs(peers) - 1) == lane) {
    double sa = 0.0, sb = 0.0;
    unsigned m = peers;
    while (m) {
      const int l = __ffs(m) - 1;
      m &= m - 1;
      sa += st->a[l]; sb += st->b[l];
    }
    atomicAdd(ta + key, sa);
    atomicAdd(tb + key, sb);
  }
  __syncwarp();
}

__device__ __forceinline__ void warp_tally1(bool flush, int key, double va, double* __restrict__ ta,
                                            WarpStage* st) {
  const unsigned fm = __ballot_sync(FULL, flush);
  if (fm == 0u) return;
  const int lane = threadIdx.x & 31;
  const unsigned peers = __match_any_sync(FULL, flush ? key : -1 - lane);
  if (__all_sync(FULL, !flush || __popc(peers) == 1)) {
    if (flush) atomicAdd(ta + key, va);
    return;
  }
  st->a[lane] = va;
  __syncwarp();
  if (flush && (__ffs(peers) - 1) == lane) {
    double sa = 0.0;
    unsigned m = peers;
    while (m) { const int l = __ffs(m) - 1; m &= m - 1; sa += st->a[l]; }
    atomicAdd(ta + key, sa);
  }
  __syncwarp();
}

// ---- block-aggregated per-bin sums ----
// The census of a step piles up in a few cells (the hottest radiation), so even after
// per-warp aggregation thousands of FP64 atomics land on each of those addresses and
// serialise in the L2.  A block first sums its (bin, value) pairs in a shared-memory hash
// table (per-warp groups add once), then flushes one global atomic per distinct bin.
// Probing is bounded: a bin that finds no slot in BINS_PROBES tries adds to global memory.
constexpr int BINS_PROBES = 8;
template <int S>
struct BlockBins {
  int key[S];
  double val[S];
};

template <int S>
__device__ __forceinline__ void bins_init(BlockBins<S>& t) {
  for (int i = threadIdx.x; i < S; i += blockDim.x) { t.key[i] = -1; t.val[i] = 0.0; }
}

template <int S>
__device__ __forceinline__ void bins_add(BlockBins<S>& t, int bin, double v, double* __restrict__ global) {
  const unsigned h = ((unsigned)bin * 2654435761u) >> 8;
#pragma unroll 1
  for (int p = 0; p < BINS_PROBES; ++p) {
    const int s = (int)((h + (unsigned)p) & (unsigned)(S - 1));
    const int old = atomicCAS(&t.key[s], -1, bin);
    if (old == -1 || old == bin) { atomicAdd(&t.val[s], v); return; }
  }
  atomicAdd(global + bin, v);
}

// warp_tally1 whose group sums go into the block's table (every lane calls it, converged)
template <int S>
__device__ __forceinline__ void warp_bins_add(bool flush, int key, double v, BlockBins<S>& t,
                                              double* __restrict__ global, WarpStage* st) {
  const unsigned fm = __ballot_sync(FULL, flush);
  if (fm == 0u) return;
  const int lane = threadIdx.x & 31;
  const unsigned peers = __match_any_sync(FULL, flush ? key : -1 - lane);
  st->a[lane] = v;
  __syncwarp();
  if (flush && (__ffs(peers) - 1) == lane) {
    double s = 0.0;
    unsigned m = peers;
    while (m) { const int l = __ffs(m) - 1; m &= m - 1; s += st->a[l]; }
    bins_add(t, key, s, global);
  }
  __syncwarp();
}

// after a __syncthreads(): one global atomic per occupied slot
template <int S>
__device__ __forceinline__ void bins_flush(BlockBins<S>& t, double* __restrict__ global) {
  for (int i = threadIdx.x; i < S; i += blockDim.x)
    if (t.key[i] >= 0) atomicAdd(global + t.key[i], t.val[i]);
}

// The same per-block aggregation for integer counts (32-bit shared-memory adds, exact).
template <int S>
struct BlockCounts {
  int key[S];
  unsigned val[S];
};

template <int S>
__device__ __forceinline__ void counts_init(BlockCounts<S>& t) {
  for (int i = threadIdx.x; i < S; i += blockDim.x) { t.key[i] = -1; t.val[i] = 0u; }
}

template <int S>
__device__ __forceinline__ void counts_add(BlockCounts<S>& t, int bin, unsigned v,
                                           unsigned long long* __restrict__ global) {
  const unsigned h = ((unsigned)bin * 2654435761u) >> 8;
#pragma unroll 1
  for (int p = 0; p < BINS_PROBES; ++p) {
    const int s = (int)((h + (unsigned)p) & (unsigned)(S - 1));
    const int old = atomicCAS(&t.key[s], -1, bin);
    if (old == -1 || old == bin) { atomicAdd(&t.val[s], v); return; }
  }
  atomicAdd(global + bin, (unsigned long long)v);
}

// every lane calls it (converged): per-warp groups by bin (lanes' counts summed with the
// group's leader), then one shared-memory add per group
template <int S>
__device__ __forceinline__ void warp_counts_add(bool add, int key, unsigned v, BlockCounts<S>& t,
                                                unsigned long long* __restrict__ global) {
  const unsigned fm = __ballot_sync(FULL, add);
  if (fm == 0u) return;
  const int lane = threadIdx.x & 31;
  const unsigned peers = __match_any_sync(FULL, add ? key : -1 - lane);
  const unsigned s = __reduce_add_sync(peers, add ? v : 0u);  // the group's sum, on every member
  if (add && (__ffs(peers) - 1) == lane) counts_add(t, key, s, global);
}

template <int S>
__device__ __forceinline__ void counts_flush(BlockCounts<S>& t, unsigned long long* __restrict__ global) {
  for (int i = threadIdx.x; i < S; i += blockDim.x)
    if (t.key[i] >= 0) atomicAdd(global + t.key[i], (unsigned long long)t.val[i]);
}

// ---- energy tallies in 64-bit fixed point ----
// Deposited and escaped energy are summed as integers in units of q = W * 2^-60, W the
// total weight tracked in the step (an upper bound of every such sum, so no total exceeds
// 2^60 units).  Integer adds are exact and independent of order: each deposit is rounded
// once, by at most q/2, however many adds a cell receives, which keeps the step's energy
// balance far inside 1e-12 where FP64 atomics would drift with the square root of the
// number of adds.
constexpr double FX_ONE = 1152921504606846976.0;  // 2^60
__device__ __forceinline__ double fx_inv_quantum(double wsum) { return wsum > 0.0 ? FX_ONE / wsum : 0.0; }
__device__ __forceinline__ unsigned long long fx_units(double e, double inv_q) { return __double2ull_rn(e * inv_q); }
__device__ __forceinline__ double fx_energy(unsigned long long u, double wsum) { return (double)u * (wsum / FX_ONE); }

// warp_tally2 with the first tally in fixed point (a zero value issues no reduction)
__device__ __forceinline__ void warp_tally_fx(bool flush, int key, unsigned long long ua, double vb,
                                              unsigned long long* __restrict__ ta, double* __restrict__ tb,
                                              WarpStage* st) {
  const unsigned fm = __ballot_sync(FULL, flush);
  if (fm == 0u) return;
  const int lane = threadIdx.x & 31;
  const unsigned peers = __match_any_sync(FULL, flush ? key : -1 - lane);
  if (__all_sync(FULL, !flush || __popc(peers) == 1)) {
    if (flush) { if (ua) atomicAdd(ta + key, ua); if (vb != 0.0) atomicAdd(tb + key, vb); }
    return;
  }
  unsigned long long* sa_u = reinterpret_cast<unsigned long long*>(st->a);
  sa_u[lane] = ua; st->b[lane] = vb;
  __syncwarp();
  if (flush && (__ffs(peers) - 1) == lane) {
    unsigned long long su = 0ull;
    double sb = 0.0;
    unsigned m = peers;
    while (m) {
      const int l = __ffs(m) - 1;
      m &= m - 1;
      su += sa_u[l]; sb += st->b[l];
    }
    if (su) atomicAdd(ta + key, su);
    if (sb != 0.0) atomicAdd(tb + key, sb);
  }
  __syncwarp();
}

// Group of a photon sampled from the Planck spectrum at T (mixture of Gammas,
// MG_IMC/MG_IMC2D.py:202-254): n from the 1/n^4 mixture CDF, x = (four Exp(1)) / n,
// energy T*x located in the group edges.
// below_last: an energy below the lowest edge goes to the last group (MG_IMC/MG_IMC1D.py:180-186);
// otherwise to the first (MG_IMC/MG_IMC2D.py:242-243)
__device__ __forceinline__ int planck_group(double T, const double* edges, int G, const double* mixcdf, double un,
                                            double u1, double u2, double u3, double u4, bool below_last = false) {
  if (!(T > 0.0)) return 0;
  double ns = 200.0;
  for (int i = 0; i < 200; ++i) if (un <= mixcdf[i]) { ns = (double)(i + 1); break; }
  const double x = (-log(u1) - log(u2) - log(u3) - log(u4)) / ns;
  const double f = T * x;
  if (f < edges[0]) return below_last ? G - 1 : 0;
  if (f >= edges[G]) return G - 1;
  for (int g = 0; g < G; ++g) if (f >= edges[g] && f < edges[g + 1]) return g;
  return G - 1;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}
__device__ __forceinline__ unsigned long long warp_sum_u(unsigned v) {
  return (unsigned long long)__reduce_add_sync(FULL, v);
}

}  // namespace imcdev
