// imc_internal.h — launch-argument structs and workspace layout shared by the kernels
// of the IMC engine.  Not part of the public ABI.
//
// Sizes flow between phases in device memory (imc_step_summary): the host passes only
// upper bounds used to size grids, and every kernel reads its true element count from the
// summary, so a whole step runs without a host round trip.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/imcb200.h"

// ---------------------------------------------------------------------------------
// Tracking
// ---------------------------------------------------------------------------------
struct TrackArgs {
  uint32_t rk[20];           // Philox round keys of seed (philox_round_keys)
  int nx, ny, nc, ng;
  const float* e1;           // nx+1 edges (FP32 copy)
  const float* e2;           // ny+1
  const float2* sass;        // [g][c] (Fleck absorption, effective scatter), FP32
  const double2* cellf;      // [g][c] (1/V, 1/(sigma_a V dt) or -1/(V dt))
  double* dep;               // [g][c]
  double* si;                // [g][c]
  double* escaped;           // [4 + ng]
  unsigned long long* stats; // [IMC_STAT_N]
  float* p1; float* p2; float* d1; float* d2; float* w; float* t;
  int* cell;
  int* group;
  const int64_t* n_dev;      // bank entries to track (device)
  const double* wsum;        // sum of their weights (device): floor = floor_coef * wsum / n
  double floor_coef;         // 1e-10 (IMC1D, IMC2D, MG_IMC2D); 1e-14 (MG_IMC1D)
  unsigned long long* queue; // ticket counter (zeroed before launch)
  int* flags;                // IMC_FLAG_* (device)
  float dt;
  int reflect_mask;
  long long max_events;
  int cap_is_reference;      // 1: the cap is the reference's (no error flag)
  uint64_t seed;
  uint32_t step;
  int chunk;
  const double* group_edges; // MG
  double* escaped_group;     // MG: [ng]
  unsigned long long* dep_fx; // [g][c] deposited energy, fixed point (zeroed before launch)
  unsigned long long* esc_fx; // [4 + ng] escaped energy by side, then by group (MG)
  const float* cf_rate;      // Carter-Forest: [c] re-emission rate c sigma_a beta (0: none), else NULL
  float cf_fastpath;         // Carter-Forest stiff fast-path threshold (0 = off)
  const double* dt_dev;      // non-NULL: the step length is read from device memory (graph replay)
  const uint32_t* step_dev;  // non-NULL: the Philox step counter is read from device memory
  uint32_t id_base;          // Philox particle id of bank entry k is id_base + k
  // census sums for the comb (NULL: none): energy of the entries alive at the end of the
  // step per bin (cell, + nc * group when ecen_by_group) and their count
  double* ecen;
  unsigned long long* n_live;
  int ecen_by_group;
};

// smem_tally: per-block deposition / intensity tallies in shared memory (with smem_cells only);
// prefetch: lanes copy their next history's bank record into shared memory while they track
cudaError_t imc_launch_track(const TrackArgs& a, int geom, int block, int grid, bool smem_cells, bool smem_tally,
                             bool prefetch, cudaStream_t s);
// Event-by-event tracking (reserved bit 3 of imc_step_params): scratch bytes for a bank of
// `capacity` entries, and the launch loop (synchronises the stream every 8 launches to read the
// live count; *cap_hit when more than max_launches launches would be needed)
size_t imc_event_scratch_bytes(long long capacity);
cudaError_t imc_run_event_tracking(const TrackArgs& a, int geom, void* scratch, long long capacity,
                                   long long n_upper, int block, int sms, long long max_launches, bool* cap_hit,
                                   cudaStream_t s);
// dep = fixed-point deposition / V, escaped (and escaped_group) from their fixed-point sums
cudaError_t imc_launch_tally_finalize(const TrackArgs& a, cudaStream_t s);

// Adjoint tracking (imc_adjoint.cu): the step's histories replayed from their Philox
// counters, accumulating the vector-Jacobian product of the deposition tally with respect
// to the per-cell opacity.
struct AdjointArgs {
  TrackArgs t;            // the forward step's tracking arguments (tallies unused)
  const double* cot;      // [c] cotangent of the deposition tally (per unit volume)
  double* grad;           // [c] += d(cot . dep) / d sigma
  const double* sa64;     // [c] Fleck absorption opacity (FP64)
  const double* ss64;     // [c] effective scatter opacity (FP64)
  const double* sig64;    // [c] opacity sigma
};
cudaError_t imc_launch_adjoint(const AdjointArgs& a, int geom, int block, int grid, cudaStream_t s);

// ---------------------------------------------------------------------------------
// Workspace layout (byte offsets into the caller's workspace, 256-aligned pieces)
// ---------------------------------------------------------------------------------
struct WsLayout {
  size_t e1f, e2f;            // float edges
  size_t sass;                // float2 [ncg]
  size_t cellf;               // double2 [ncg]
  size_t emit_E;              // double [ncg]  emission energy per (group,) cell
  size_t emit_n;              // int64 [ncg]   emission count per order position (MG 1-D: per bin)
  size_t emit_off;            // int64 [ncg+1] exclusive offsets in source order
  size_t emit_w;              // float [ncg]
  size_t emit_issued;         // double [ncg]  MG 1-D: energy issued per bin
  size_t tilt;                // double [4*nc] per-cell tilt constants
  size_t src_n, src_off, src_w, src_QV, src_issued;  // fixed source ([ncg] / [ncg+1])
  size_t face;                // double [4][2][nf] per-side face energies and CDF
  size_t mg_gcdf, mg_ec, mg_cdf, mg_sgcdf, mg_sc, mg_scdf, mixcdf;  // multigroup tables
  size_t summary;             // imc_step_summary used by the synchronous wrappers
  size_t queue;               // uint64 ticket counter
  size_t ecen, ew, ncopy;     // comb: double [nb], double [nb], uint64 [nb]
  size_t cnt;                 // int32 [cap]    comb copies per entry
  size_t blk;                 // int64 [nblk+1] comb block totals / offsets
  size_t comb_mode;           // int32 mode + uint64 live-entry count (comb)
  size_t dep_fx, esc_fx;      // uint64 [ncg], [4 + ng] fixed-point energy tallies
  size_t cf_rate;             // float [nc] Carter-Forest re-emission rate
  size_t total;
};

WsLayout imc_ws_layout(const imc_mesh* m, int64_t capacity);

template <typename T>
inline T* ws_ptr(void* ws, size_t off) { return reinterpret_cast<T*>(static_cast<char*>(ws) + off); }

// ---------------------------------------------------------------------------------
// Bookkeeping kernels (FP64, compiled without FMA contraction so the oracle, which is
// plain C++ on x86-64, can reproduce every per-cell number and integer count exactly)
// ---------------------------------------------------------------------------------
struct PlanArgs {
  int geom, nx, ny, nc, ng;
  const double* e1; const double* e2; const double* vol;
  const double* T; const double* sigma; const double* cv; const double* source;
  double dt, theta;
  long long n_target, n_source, n_boundary;
  long long n_side[4];             // boundary particles per side (n_boundary unless overridden)
  const double* face_T[4];
  int rz_linear;
  double t_emit_floor;
  int method;                      // IMC_METHOD_*
  float* cf_rate;                  // Carter-Forest: [c] re-emission rate (tilt[4c+3]: emission rate)
  const double* dt_dev;            // non-NULL: dt read from device memory (graph replay)
  double share;                    // fraction of the source energy issued (1: all of it)
  // outputs
  double* sa; double* ss;          // FP64 [ncg]
  float2* sass;                    // FP32 [ncg]
  double2* cellf;                  // [c]
  float* e1f; float* e2f;
  double* emit_E; long long* emit_n; long long* emit_off; float* emit_w; double* tilt;
  long long* src_n; long long* src_off; float* src_w; double* src_QV; double* src_issued;
  double* emitted;                 // [c] issued emission energy per cell
  double* face;                    // [4][2][nf]
  int nf;
  imc_step_summary* sum;
};
cudaError_t imc_launch_plan(const PlanArgs& a, cudaStream_t s);

struct IcArgs {
  int geom, nx, ny, nc;
  int rule;                        // counts: 0 ceil(N E/Et) (IMC1D), 1 max(1, ceil) (IMC2D),
                                   // 2 max(1, round) for E > 0 (MG_IMC1D)
  const double* e1; const double* e2; const double* vol;
  const double* tr;
  long long n_target;
  double t_emit_floor;
  long long* n; long long* off; float* w; double* E;
  imc_step_summary* sum;           // n_emission = total, base_emission = 0
};
cudaError_t imc_launch_ic_plan(const IcArgs& a, cudaStream_t s);

struct MatArgs {
  int nc, ng;
  const double* vol; const double* dep; const double* si; const double* emitted;
  double* e; double* tr;
};
cudaError_t imc_launch_material(const MatArgs& a, cudaStream_t s);
// the material update with the law's inverse EOS and next-step opacity / heat capacity
cudaError_t imc_launch_material_law(const MatArgs& a, const imc_material_law& law, double* T, double* sigma_next,
                                    double* cv_next, cudaStream_t s);

struct CombPlanArgs {
  int nb;
  long long n_max;
  const int64_t* n_max_dev;        // when set, the comb target (read at run time)
  long long threshold;             // > 0: comb only when at least this many entries are alive
  int force_compact;               // 1: no comb, only drop dead entries
  const unsigned long long* n_live;
  int* mode;                       // out: 0 comb, 1 compact only
  const double* ecen;
  double* ew;
  unsigned long long* ncopy;       // zeroed with the weights (the count accumulates into it)
  imc_step_summary* sum;
};
cudaError_t imc_launch_comb_plan(const CombPlanArgs& a, cudaStream_t s);

// Up to 12 device regions zeroed by one launch (8-byte aligned, sizes multiples of 8): the
// per-step tallies, counters and summary fields that a step's kernels accumulate into.
struct ZeroList {
  int n;
  void* p[12];
  unsigned long long bytes[12];
  void add(void* ptr, size_t b) { if (ptr && b) { p[n] = ptr; bytes[n] = b; ++n; } }
};
cudaError_t imc_launch_zero(const ZeroList& z, cudaStream_t s);

cudaError_t imc_launch_canon_sum_eV(const double* e, const double* vol, int nc, double* out, cudaStream_t s);
struct ReportArgs {
  int nx, ny, ng;
  const double* vol; const double* si; const double* after;
  const double* e; const double* T; const double* Tr; const double* bnd; const double* esc;
  double* out;
  long long q0, q1;  // the entries of out written: [q0, q1), sections whose input is NULL skipped
};
cudaError_t imc_launch_mg_report(const ReportArgs& a, cudaStream_t s);

// ---------------------------------------------------------------------------------
// Source fill kernels (element count and first bank index read from device memory)
// ---------------------------------------------------------------------------------
struct FillArgs {
  uint32_t rk[20];             // Philox round keys of seed (philox_round_keys)
  int geom, nx, ny, nc;
  const double* e1; const double* e2;
  const double* T;
  const int64_t* d_n;          // particles to write (device)
  const int64_t* d_base;       // first bank index (device)
  long long n_bound;           // host upper bound of *d_n (grid sizing)
  int nbins;                   // order positions in off (nc; bins_by_group: ng*nc)
  int bins_by_group;           // 1: bin b = g*nc + c carries group g (MG 1-D sources)
  const long long* off;        // [nbins+1] offsets in source order
  const float* w;              // [nc] per-cell weight ([nbins] when bins_by_group)
  const double* tilt;          // [4*nc] or NULL
  int tilt_kind;               // 0 none, 1 slab linear-T, 2 sphere linear-T^4, 3 rz linear
  double time_scale;           // birth time = u * time_scale (dt; 0 for the IC)
  uint64_t seed; uint32_t step; uint32_t tag;
  float* p1; float* p2; float* d1; float* d2; float* wb; float* t; int* cell; int* group;
  // MG 1-D initial census: group from the Planck spectrum at tr[c] (NULL otherwise)
  const double* tr; const double* gedges; const double* mixcdf; int ng;
  // Carter-Forest emission: birth time of density ~ exp(-k t) on [0, dt], k = cf_rate4[4c]
  // when k > cf_thr (else uniform); NULL otherwise
  const double* cf_rate4; double cf_thr;
  const double* time_scale_dev; const uint32_t* step_dev;  // non-NULL: read from device memory
  uint32_t id_base;            // Philox particle id of source particle k is id_base + k
};
cudaError_t imc_launch_fill_volume(const FillArgs& a, cudaStream_t s);

struct BndArgs {
  uint32_t rk[20];             // Philox round keys of seed (philox_round_keys)
  int geom, nx, ny, side, nf;
  const double* e1; const double* e2;
  const double* face;          // [2][nf]: energies, cumulative (total = last)
  const int64_t* d_n;
  const int64_t* d_base;
  long long n_bound;
  double dt;
  uint64_t seed; uint32_t step;
  float* p1; float* p2; float* d1; float* d2; float* wb; float* t; int* cell; int* group;
  // multigroup: Planck group at the face cell's temperature
  int ng; const double* faceT; const double* gedges; const double* mixcdf; double* boundary_group;
  int below_last;              // MG 1-D: an energy below the lowest edge goes to the last group
  const double* dt_dev; const uint32_t* step_dev;  // non-NULL: read from device memory
  uint32_t id_base;            // Philox particle id of face particle k is id_base + k
};
cudaError_t imc_launch_fill_boundary(const BndArgs& a, cudaStream_t s);

cudaError_t imc_launch_wsum(const float* w, const int64_t* d_n, long long n_bound, double* out, cudaStream_t s);


// ---------------------------------------------------------------------------------
// Comb kernels
// ---------------------------------------------------------------------------------
struct CombArgs {
  uint32_t rk[20];             // Philox round keys of seed (philox_round_keys)
  int nc, nb, per_group;
  int vec16;                   // w, cell (and group) 16-byte aligned: vector loads in the count
  int conserve_rad;            // copies in bin b weigh ecen[b] / ncopy[b] (bin energy kept)
  int* mode;                   // set by the comb plan: 0 comb, 1 compact only (copy live entries)
  const uint32_t* step_dev;    // non-NULL: the Philox step counter is read from device memory
  unsigned long long* n_live;  // live entries (counted by k_comb_ecen; zeroed before)
  const int64_t* d_n_in;       // entries to comb (device)
  long long n_bound;           // host upper bound of *d_n_in (grid sizing)
  long long out_capacity;
  const float* w; const int* cell; const int* group;
  const float* p1; const float* p2; const float* d1; const float* d2;
  double* ecen; double* ew; unsigned long long* ncopy; int* cnt; long long* blk;  // ncopy: copies per bin
  uint64_t seed; uint32_t step;
  float* op1; float* op2; float* od1; float* od2; float* ow; float* ot; int* ocell; int* ogroup;
  double* disc;
  double* after;               // nullable: energy after the comb per bin [nb]
  imc_step_summary* sum;
};
cudaError_t imc_launch_comb_ecen(const CombArgs& a, cudaStream_t s);
cudaError_t imc_launch_comb_count(const CombArgs& a, cudaStream_t s);
cudaError_t imc_launch_comb_scatter(const CombArgs& a, cudaStream_t s);

cudaError_t imc_launch_philox(const uint32_t* ctr, uint32_t k0, uint32_t k1, uint32_t* out, long long n, cudaStream_t s);

extern unsigned long long g_imc_launches;

// Programmatic dependent launch for the kernels of a step's chain: a kernel launched with
// launch_pdl may be scheduled while the previous kernel of its stream drains, so its launch
// latency hides behind that kernel's tail.  Such a kernel calls pdl_wait() before it touches
// global memory (griddepcontrol.wait returns once the previous kernel has completed and its
// writes are visible: a hardware dependency, no spin) and pdl_trigger() to let its own
// successor be scheduled.  Without the attribute both are no-ops.  IMCB200_PDL=0 in the
// environment launches without it.
extern bool g_imc_pdl;

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" :::); }

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
                       Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = g_imc_pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<Args&&>(args)...);
}
// launch_pdl(...) in a function returning cudaError_t: returns its error
#define IMC_LAUNCH_PDL(...)                                     \
  do {                                                          \
    const cudaError_t e_pdl_ = launch_pdl(__VA_ARGS__);         \
    if (e_pdl_ != cudaSuccess) return e_pdl_;                   \
  } while (0)

// ---------------------------------------------------------------------------------
// Multigroup planning and sources
// ---------------------------------------------------------------------------------
struct PlanMgArgs {
  int geom, nx, ny, nc, ng;
  const double* e1; const double* e2; const double* vol;
  const double* T; const double* sigma; const double* cv; const double* source;  // sigma, source [g][c]
  const double* gedges; const double* emission_fractions;
  double dt, theta;
  long long n_target, n_source, n_boundary;
  long long n_side[4];             // boundary particles per side
  const double* face_T[4];
  double t_emit_floor;
  double* sa; double* ss; float2* sass; double2* cellf;  // [g][c]
  float* e1f; float* e2f;
  double* Egc; double* Ec; double* cdf;       // emission: [c][g] cumulative, [c], [c] canonical prefix
  double* Sgc; double* Sc; double* Scdf;      // fixed source, same shapes
  double* emitted;                            // [c]
  double* face; int nf;
  double* mixcdf;                             // [200]
  imc_step_summary* sum;
  // 1-D sphere (MG_IMC1D): stratified (group, cell) bins b = g*nc + c
  double* emit_E; long long* emit_n; long long* emit_off; float* emit_w; double* emit_issued;
  double* src_QV; long long* src_n; long long* src_off; float* src_w; double* src_issued;
  const double* dt_dev;            // non-NULL: dt read from device memory (graph replay)
  double share;                    // fraction of the source energy issued (1: all of it)
};
cudaError_t imc_launch_plan_mg(const PlanMgArgs& a, cudaStream_t s);
cudaError_t imc_launch_plan_mg1d(const PlanMgArgs& a, cudaStream_t s);

struct IcMgArgs {
  int nc;
  const double* vol; const double* tr;
  long long n_target; double t_emit_floor;
  double* E; double* cdf; double* mixcdf;
  imc_step_summary* sum;
};
cudaError_t imc_launch_ic_plan_mg(const IcMgArgs& a, cudaStream_t s);

// categorical (cell ~ total, group ~ per-cell cumulative) multigroup source fill; the IC
// variant samples the group from the Planck spectrum at tr[c] instead
struct FillMgArgs {
  uint32_t rk[20];             // Philox round keys of seed (philox_round_keys)
  int geom, nx, ny, nc, ng;
  const double* e1; const double* e2;
  const double* cdf;           // [c] canonical inclusive prefix of cell totals
  const double* gcdf;          // [c][g] cumulative over groups (NULL: Planck group at tr)
  const double* tr;            // IC: [c]
  const double* gedges; const double* mixcdf;
  const int64_t* d_n; const int64_t* d_base; long long n_bound;
  double time_scale;
  uint64_t seed; uint32_t step; uint32_t tag;
  float* p1; float* p2; float* d1; float* d2; float* wb; float* t; int* cell; int* group;
  const double* time_scale_dev; const uint32_t* step_dev;  // non-NULL: read from device memory
  uint32_t id_base;            // Philox particle id of source particle k is id_base + k
};
cudaError_t imc_launch_fill_mg(const FillMgArgs& a, cudaStream_t s);

// All of a step's sources in one launch: each job (a boundary side, a volume source or its
// multigroup form, the census weights) owns a contiguous range of blocks and runs the
// body of its own kernel there, so the short jobs fill the SMs beside the long one instead
// of waiting behind it.  With wsum set, every fill adds the weights it writes and the
// census job adds the weights of entries [0, *n_census): wsum ends as the sum of all the
// tracked weights (what imc_launch_wsum computes after separate fills).
constexpr int kSourceJobsMax = 8;
enum SourceJobKind { JOB_BOUNDARY = 0, JOB_VOLUME = 1, JOB_VOLUME_MG = 2, JOB_CENSUS_WSUM = 3 };
struct SourceJobs {
  uint32_t rk[20];             // Philox round keys of the run seed (every job's)
  int n_jobs;
  int kind[kSourceJobsMax];
  int slot[kSourceJobsMax];    // index into bnd / vol / vmg
  int first_block[kSourceJobsMax + 1];
  BndArgs bnd[4];
  FillArgs vol[2];
  FillMgArgs vmg[2];
  const float* census_w; const int64_t* n_census;
  double* wsum;                // NULL: the weights are not summed
  int n_bnd, n_vol, n_vmg;
  // appends a job of kind k (its args already in bnd / vol / vmg at slot) with `blocks` blocks
  bool add(int k, int sl, int blocks) {
    if (n_jobs >= kSourceJobsMax || blocks < 1) return false;
    if (n_jobs == 0) first_block[0] = 0;
    kind[n_jobs] = k; slot[n_jobs] = sl;
    first_block[n_jobs + 1] = first_block[n_jobs] + blocks;
    ++n_jobs;
    return true;
  }
};
int imc_source_blocks(long long n_bound);
cudaError_t imc_launch_sources(const SourceJobs& j, cudaStream_t s);
