/*
 * imcb200.h — C ABI of the B200 implicit Monte Carlo (Fleck-Cummings) time-step engine.
 *
 * The reference (DrRyanMc/RadTranBook) exposes its time step as Python functions; the
 * calls below are what a binding of those functions needs, split where the reference
 * hands control back to user material callables:
 *
 *   IMC/IMC1D.py:908    step(state, Ntarget, Nboundary, Nsource, NMax, T_boundary, dt, mesh,
 *                            sigma_a_func, inv_eos, cv, source, reflect, theta, ...)
 *   IMC/IMC2D.py:1591   step(state, ..., edges1, edges2, ..., geometry='xy'|'rz', ...)
 *   MG_IMC/MG_IMC2D.py:1635  step(state, ..., energy_edges, sigma_a_funcs, ...)
 *   MG_IMC/MG_IMC1D.py:917   step(state, ..., mesh, energy_edges, sigma_a_funcs, ...)
 *
 *   imc_step_transport  = reference lines from the Fleck factor through the transport
 *                         kernel (IMC/IMC1D.py:932-1017, IMC/IMC2D.py:1646-1797,
 *                         MG_IMC/MG_IMC2D.py:1703-1976, MG_IMC/MG_IMC1D.py:941-1140)
 *   imc_material_update = internal_energy += dep - emitted / V; Tr from the path-length
 *                         intensity (IMC/IMC1D.py:1021-1035, IMC/IMC2D.py:1801-1810)
 *   imc_comb            = the stochastic comb (IMC/IMC1D.py:770-828, IMC/IMC2D.py:1448-1511,
 *                         MG_IMC/MG_IMC2D.py:1314-1378, MG_IMC/MG_IMC1D.py:746-847)
 *   imc_init_census     = the equilibrium initial census of init_simulation
 *                         (IMC/IMC1D.py:220-248,535-575; IMC/IMC2D.py:1110-1188;
 *                         MG_IMC/MG_IMC1D.py:514-566)
 *
 * Conventions
 *   - Every pointer in a struct is DEVICE memory, caller-owned.  The library never
 *     allocates or frees; scratch lives in a caller-provided workspace of
 *     imc_workspace_bytes() bytes (256-byte aligned).
 *   - All work is stream-ordered on the cudaStream_t passed in (a CUstream is accepted).
 *     Calls that return sizes synchronise that stream before returning.
 *   - Errors are returned as imc_status; nothing throws across the ABI.
 *   - Cells are flattened c = i + nx*j (1-D: ny = 1).  Multigroup arrays are [g][c].
 *   - Particle state is FP32 (tracking precision); tallies, energies and the ledger are
 *     FP64.
 */
#ifndef IMCB200_H
#define IMCB200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define IMC_API __attribute__((visibility("default")))
#else
#define IMC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum imc_status {
  IMC_OK = 0,
  IMC_ERR_BANK_OVERFLOW = 1,   /* report.required_capacity says how much is needed */
  IMC_ERR_EVENT_CAP = 2,       /* safety cap on events per history reached */
  IMC_ERR_NONFINITE = 3,       /* NaN/Inf or non-positive temperature in inputs */
  IMC_ERR_BAD_GEOMETRY = 4,    /* unknown geometry / inconsistent mesh */
  IMC_ERR_TIMEOUT = 5,         /* a bounded device wait gave up */
  IMC_ERR_CUDA = 6,            /* CUDA runtime error (see imc_last_cuda_error) */
  IMC_ERR_INVALID_ARG = 7,
  IMC_ERR_WORKSPACE = 8,       /* workspace too small, or not 256-byte aligned */
  IMC_ERR_BOUNDS = 9           /* bounds-checked build only: an index or weight out of range */
} imc_status;

enum { IMC_GEOM_SLAB = 0, IMC_GEOM_SPHERE = 1, IMC_GEOM_XY = 2, IMC_GEOM_RZ = 3 };

/* statistics slots (uint64) */
enum {
  IMC_STAT_EVENTS = 0, IMC_STAT_BOUNDARY = 1, IMC_STAT_SCATTER = 2, IMC_STAT_CENSUS = 3,
  IMC_STAT_CAPTURE = 4, IMC_STAT_FLOOR = 5, IMC_STAT_REFLECT = 6, IMC_STAT_CAP = 7,
  IMC_STAT_ESCAPE = 8, IMC_STAT_N = 9
};

typedef struct imc_mesh {
  int32_t geometry;        /* IMC_GEOM_* */
  int32_t nx, ny;          /* cells per direction; ny = 1 in 1-D */
  int32_t n_groups;        /* 1 = gray; > 1 with xy / rz: MG_IMC2D rules; with the
                              sphere: MG_IMC1D rules (stratified (group, cell) sources,
                              scatter cap, weight floor 1e-14 * sum / n) */
  const double* edges1;    /* nx+1 (x | r) */
  const double* edges2;    /* ny+1 (y | z); 1-D: {0, 1} */
  const double* volume;    /* nx*ny cell volumes (1-D slab: dx; sphere: 4/3 pi dr^3) */
  const double* group_edges; /* n_groups+1 photon energies (keV), MG only */
} imc_mesh;

typedef struct imc_bank {  /* structure-of-arrays particle bank */
  float* pos1;             /* x | r */
  float* pos2;             /* y | z (unused in 1-D) */
  float* dir1;             /* mu | u_x | mu_perp */
  float* dir2;             /* u_y | eta (unused in 1-D) */
  float* weight;           /* energy weight (GJ); 0 = dead */
  float* time;             /* birth time within the step (ns); census = 0 */
  int32_t* cell;           /* flat cell */
  int32_t* group;          /* photon group (MG) or NULL */
  int64_t size;            /* live entries (host-side count) */
  int64_t capacity;
} imc_bank;

typedef struct imc_material {   /* per-cell state at the start of the step (FP64) */
  const double* temperature;    /* T (keV), [c] */
  const double* sigma;          /* true absorption opacity (1/cm), [g][c] */
  const double* cv;             /* rho c_v (GJ/cm^3/keV), [c] */
  const double* source;         /* fixed source power density, [c] (MG: [g][c]), or NULL */
} imc_material;

typedef struct imc_step_params {
  uint64_t seed;                /* Philox key */
  uint32_t step;                /* time-step index (Philox counter word 2) */
  int32_t reflect[4];           /* -dir1, +dir1, -dir2, +dir2 faces */
  double dt, theta;
  int64_t n_target, n_boundary, n_source;
  const double* face_T[4];      /* per-face-cell boundary temperatures or NULL
                                   (sides 0/1: ny entries, 2/3: nx entries; 1-D: 1) */
  int64_t max_events;           /* events per history cap (2-D reference); <= 0: none */
  int32_t rz_linear_source;     /* RZ emission with the linear r/z tilt */
  int32_t census_bins;          /* 0, or IMC_CENSUS_BY_CELL / IMC_CENSUS_BY_GROUP_CELL: the tracking
                                   kernel also sums the energy of the entries alive at the end of
                                   the step per comb bin (cell, or (group, cell)) and counts them,
                                   into the workspace, as each history ends; an imc_comb_async /
                                   imc_comb_async_dev that follows on the same workspace and bank
                                   with the flag IMC_COMB_CENSUS_READY (and the matching
                                   IMC_COMB_PER_GROUP) uses them instead of a pass of its own */
  double t_emit_floor;
  int32_t block_size;           /* tracking launch shape; 0 = tuned default */
  int32_t blocks_per_sm;
  int32_t chunk;                /* histories claimed per warp ticket (guided: at most this) */
  int32_t reserved;             /* bit 0: shared-memory cell table (default: up to 4096 (group, cell)
                                   entries); bit 1: per-block tallies in shared memory with that
                                   table, bit 2: never (default: up to 2048 entries); bit 3:
                                   event-by-event tracking (workspace of imc_workspace_bytes_event);
                                   bit 4: prefetched refills (each lane copies its next history's
                                   bank record into shared memory while it tracks the current one;
                                   the same histories and tallies); others ignored */
  const double* emission_fractions; /* MG: [g] fixed emission spectrum, or NULL = Planck */
  int64_t n_boundary_side[4];   /* > 0: boundary particles on that side instead of n_boundary
                                   (per-side budgets, MG_IMC/MG_IMC1D.py:1000-1040) */
  int32_t method;               /* IMC_METHOD_FLECK_CUMMINGS or IMC_METHOD_CARTER_FOREST (gray) */
  uint32_t id_base;             /* Philox particle-id offset: the k-th source particle of each kind
                                   and the k-th bank entry draw with particle id id_base + k.  0 for
                                   a single process; the ranks of a partitioned step (each tracks
                                   its share of the particles, IMC/IMC2DMPI.py:172-175) take
                                   disjoint id ranges so their histories are independent */
  double cf_fastpath;           /* Carter-Forest stiff fast path: when rate * t_left exceeds it,
                                   capture with probability exp(-rate t_left) (0 = off) */
  const uint32_t* step_dev;     /* DEVICE pointer or NULL: when set, every kernel of the step reads
                                   the Philox step counter from it at run time instead of `step` */
  const double* dt_dev;         /* DEVICE pointer or NULL: likewise for dt.  With both set, a
                                   captured step is replayed (CUDA graph) for any step and dt. */
  double energy_share;          /* fraction of the step's source energy (emission, fixed source,
                                   boundary faces) this call issues; 0 or 1 = all of it.  A rank of a
                                   partitioned step issues 1/ranks of it with its share of the
                                   particles, so the ranks' sources together carry the energy once */
} imc_step_params;

/* Carter-Forest (IMC/IMC1D_CarterForest.py, IMC/IMC2D_CarterForest.py): no Fleck factor;
 * sigma_a is the true opacity and there is no effective scatter; emission a T^4 (1 - e^{-k dt})
 * / beta V per cell (k = c sigma_a beta, beta = 4 a T^3 / cv) with birth times of density
 * ~ e^{-k t}; an absorbed photon is re-emitted isotropically after a delay ~ Exp(k) when that
 * falls inside the step and is captured (its weight deposited) otherwise. */
enum { IMC_METHOD_FLECK_CUMMINGS = 0, IMC_METHOD_CARTER_FOREST = 1 };

typedef struct imc_tallies {    /* device outputs, overwritten by each step */
  double* dep;                  /* [g][c] energy deposited per unit volume */
  double* si;                   /* [g][c] path-length scalar intensity */
  double* emitted;              /* [c] emission energy issued from matter (GJ) */
  double* sigma_a;              /* [g][c] Fleck absorption (out) */
  double* sigma_s;              /* [g][c] effective scatter (out) */
  double* escaped;              /* [4] escaped energy by side */
  unsigned long long* stats;    /* [IMC_STAT_N] */
  double* escaped_group;        /* MG: [n_groups] escaped energy by group (NULL for gray) */
  double* boundary_group;       /* MG: [n_groups] issued boundary energy by group */
} imc_tallies;

typedef struct imc_step_report {  /* host-side summary of imc_step_transport */
  int64_t n_boundary, n_source, n_emission;
  int64_t n_transported;
  int64_t required_capacity;
  double boundary_emission, source_emission, emission_total;
  double weight_floor;
  float ms_sources, ms_transport;  /* device time of source fill and of tracking */
} imc_step_report;

typedef struct imc_comb_report {
  int64_t n_in, n_out;
  int64_t required_capacity;
  double energy_before, energy_after;
} imc_comb_report;

/* Device-resident summary of one step, written by the asynchronous calls (the caller
 * allocates it in device memory and copies it to the host once per step).  Bank sizes
 * live here between the phases, so no phase needs the host to know them. */
/* IMC_FLAG_BOUNDS is set only by the bounds-checked build of this library
 * (libimcb200_checked.so: every source compiled with IMC_CHECKED): a tracking or comb kernel
 * met a cell, group or bin index outside the mesh, or a non-finite particle weight; it
 * skipped that access and the host call reports IMC_ERR_BOUNDS.  No reference counterpart
 * (the reference asserts particle-in-cell in its event loop, IMC/IMC1D.py:98-113). */
enum { IMC_FLAG_EVENT_CAP = 1, IMC_FLAG_NONFINITE = 2, IMC_FLAG_COMB_OVERFLOW = 4, IMC_FLAG_BOUNDS = 8 };
typedef struct imc_step_summary {
  int64_t n_census;             /* bank entries before the sources (set by the caller) */
  int64_t n_side[4];            /* boundary particles per side */
  int64_t n_source, n_emission;
  int64_t base_side[4];         /* first bank index of each source block */
  int64_t base_source, base_emission;
  int64_t n_bank;               /* entries tracked = census + sources */
  int64_t n_out;                /* entries the comb produced (or wanted: see flags) */
  int32_t flags;                /* IMC_FLAG_* */
  int32_t pad;
  double e_side[4];             /* issued boundary energy per side (GJ) */
  double source_emission, emission_total;
  double weight_sum;            /* sum of tracked weights; floor = 1e-10 * sum / n_bank
                                   (MG sphere: 1e-14) */
  double comb_before, comb_after;
  double internal_energy;       /* sum_c e[c] V[c] after imc_comb_async */
  unsigned long long stats[IMC_STAT_N];
  double escaped[4];
} imc_step_summary;

/* Workspace bytes for a mesh and a bank capacity. */
IMC_API size_t imc_workspace_bytes(const imc_mesh* mesh, int64_t bank_capacity);

/* Workspace for a step with event-by-event tracking (imc_step_params.reserved bit 3): the
 * history-based tracking kernel is replaced by the textbook event-based loop, one launch per
 * event over the live histories with the survivors compacted between launches (the same
 * physics and Philox draws per history; it synchronises the stream every few launches to read
 * the live count, and does not take census_bins).  No reference counterpart: a second form of
 * the tracking of IMC/IMC2D.py:938-1107, kept to compare the two on the hardware. */
IMC_API size_t imc_workspace_bytes_event(const imc_mesh* mesh, int64_t bank_capacity);

/* Equilibrium initial census at radiation temperature tr[c] into an empty bank.
 * (IMC/IMC1D.py:220-248, IMC/IMC2D.py:1110-1188, MG_IMC/MG_IMC2D.py:992-1235,
 * MG_IMC/MG_IMC1D.py:514-566) */
IMC_API imc_status imc_init_census(const imc_mesh* mesh, const double* tr, int64_t n_target,
                           double t_emit_floor, uint64_t seed, imc_bank* bank, void* workspace,
                           size_t workspace_bytes, int64_t* n_out, void* stream);

/* Fleck factor, boundary / fixed / emission sources appended to the bank in the
 * reference's order, then tracking of the whole bank to census.  Tallies are zeroed
 * and written.  Returns IMC_ERR_BANK_OVERFLOW (bank untouched) when the sources do not
 * fit; report->required_capacity says how much does. */
IMC_API imc_status imc_step_transport(const imc_mesh* mesh, const imc_material* mat,
                              const imc_step_params* par, imc_bank* bank, imc_tallies* tal,
                              void* workspace, size_t workspace_bytes, imc_step_report* report,
                              void* stream);

/* e[c] += sum_g dep[g][c] - emitted[c]/V[c]; tr[c] = (sum_g si[g][c] / (a c))^(1/4). */
IMC_API imc_status imc_material_update(const imc_mesh* mesh, const imc_tallies* tal, double* e,
                               double* tr, void* stream);

/* A material whose laws the device evaluates itself: linear EOS e = cv_eos * T, heat
 * capacity cv, and opacity
 *   sigma_g(T)[c] = sigma_A * max(T, sigma_T_floor)^-sigma_n * sigma_scale[c] * sigma_group[g]
 * clamped to [sigma_lo, sigma_hi] (multiplied in that order; a bound <= 0 is no bound,
 * sigma_T_floor <= 0 no floor, sigma_n = 0 a constant, a null sigma_scale / sigma_group a
 * factor of 1).  cv_eos_array, cv_array and sigma_scale, when set, are DEVICE arrays [c];
 * sigma_group is a DEVICE array [g] (multigroup meshes need it, or sigma_array).
 * sigma_array, when set, replaces the whole opacity law by temperature-independent values,
 * a DEVICE array [g][c]. */
typedef struct imc_material_law {
  double cv_eos;          const double* cv_eos_array;
  double cv;              const double* cv_array;
  double sigma_A, sigma_n, sigma_lo, sigma_hi;
  const double* sigma_array;
  const double* sigma_scale;
  double sigma_T_floor;
  const double* sigma_group;
} imc_material_law;

/* imc_material_update and the material temperature of the next step in one kernel: e and
 * tr as imc_material_update, then T = e / cv_eos (the inverse EOS, IMC/IMC1D.py:1024
 * inv_eos; MG_IMC/MG_IMC2D.py:2037), and the next step's opacity and cv(T) of the law into
 * sigma_next ([g][c]) and cv_next ([c]) (IMC/IMC1D.py:932-935 sigma_a_func(T), cv(T);
 * MG_IMC/MG_IMC2D.py:1703-1710 one sigma_a_funcs[g](T) per group), which a step's
 * imc_material then takes as they are. */
IMC_API imc_status imc_material_update_law(const imc_mesh* mesh, const imc_tallies* tal,
                                           const imc_material_law* law, double* e, double* tr,
                                           double* T, double* sigma_next, double* cv_next,
                                           void* stream);

/* Stochastic comb of bank `in` into bank `out` (census times reset to 0).
 * per_group is a set of flags: IMC_COMB_PER_GROUP combs per (cell, group) bin (MG);
 * IMC_COMB_CONSERVE_RADIATION gives every copy in a bin the bin's pre-comb energy divided
 * by its copy count (MG_IMC/MG_IMC1D.py:808-820, conserve_comb_energy='radiation').
 * n_max > 0 combs to n_max; n_max == 0 only drops dead entries (every live entry copied
 * once with its weight); n_max < 0 combs to |n_max| when at least |n_max| entries are
 * alive, else only drops dead entries (MG_IMC/MG_IMC1D.py:1194-1200).
 * disc[bin] = energy before - after. */
enum { IMC_COMB_PER_GROUP = 1, IMC_COMB_CONSERVE_RADIATION = 2,
       IMC_COMB_CENSUS_READY = 4, /* async forms: the census sums come from the tracking call */
       IMC_COMB_WRITE_AFTER = 8   /* disc holds 2 x bins: [bins, 2 bins) the energy after the
                                     comb per bin (sum of its copies' FP32 weights in FP64;
                                     divided by V: MG_IMC/MG_IMC2D.py:2017-2025) */ };
enum { IMC_CENSUS_BY_CELL = 1, IMC_CENSUS_BY_GROUP_CELL = 2 };
IMC_API imc_status imc_comb(const imc_mesh* mesh, const imc_bank* in, imc_bank* out, int64_t n_max,
                    uint64_t seed, uint32_t step, int32_t per_group, double* disc,
                    void* workspace, size_t workspace_bytes, imc_comb_report* report,
                    void* stream);

/* Vector-Jacobian product of one step's deposition tally with respect to the per-cell
 * opacity mat->sigma, 2-D gray (xy or rz):
 *   grad[c] += sum_c' cotangent[c'] * d dep[c'] / d sigma[c].
 * The arguments are those of the forward imc_step_transport call, with `bank` holding the
 * same census entries (its first bank->size entries) as before the forward call.  The
 * step's source particles are regenerated from the same Philox streams and every history
 * is tracked twice from its counter (no path is stored): once for its total cotangent-
 * weighted score, once to accumulate the path-length derivative of implicit capture and
 * the likelihood-ratio derivative of effective scattering, chained through the Fleck
 * factor (d sigma_a / d sigma = f^2, d sigma_s / d sigma = 1 - f^2).  The bank entries
 * after bank->size and the tallies' sigma_a / sigma_s / emitted are used as scratch; the
 * census entries and bank->size are unchanged.  Synchronises the stream.
 * No reference counterpart: the reference has no derivative of its tallies. */
IMC_API imc_status imc_adjoint_vjp(const imc_mesh* mesh, const imc_material* mat,
                                   const imc_step_params* par, imc_bank* bank,
                                   const double* cotangent, double* grad, imc_tallies* tal,
                                   void* workspace, size_t workspace_bytes, void* stream);

/* imc_comb without a workspace argument.  No reference counterpart: the reference combs
 * NumPy arrays and has no device scratch to provide.
 *
 * For callers that cannot allocate device memory, e.g. a C or Fortran host that links only
 * this library and the CUDA runtime and owns no device allocator, or code that must not
 * change the device's memory map.  Scratch is a fixed array of IMC_NOALLOC_SCRATCH_BYTES
 * compiled into the library, one per device; this call allocates and frees nothing.
 *   - Limit: imc_workspace_bytes(mesh, in->size) must be <= IMC_NOALLOC_SCRATCH_BYTES
 *     (8 MiB; e.g. a 60 x 210 gray mesh with up to about 1.5 million entries in `in`).
 *     Larger inputs return IMC_ERR_WORKSPACE without launching anything.
 *   - The first call on a device, made with that device current, looks up the array's
 *     device address; make that first call before any stream capture.
 *   - The array is shared by every call on the device: calls that overlap in time (other
 *     host threads, or work still running on another stream) race on it.
 * Inputs, outputs and report are those of imc_comb; the stream is synchronised. */
#define IMC_NOALLOC_SCRATCH_BYTES ((size_t)8 << 20)
IMC_API imc_status imc_comb_noalloc(const imc_mesh* mesh, const imc_bank* in, imc_bank* out,
                                    int64_t n_max, uint64_t seed, uint32_t step,
                                    int32_t per_group, double* disc,
                                    imc_comb_report* report, void* stream);

/* Asynchronous forms.  Nothing is synchronised and no size is returned to the host:
 * imc_step_transport_async reads summary->n_census (set it to the bank's live size),
 * requires bank->capacity >= n_census + imc_source_bound(...), and writes the source
 * counts, n_bank, weight_sum, stats and escaped energy into the device summary (the
 * tallies' stats/escaped pointers may point into the summary).  imc_comb_async combs
 * summary->n_bank entries of `in` into `out`, writing at most out->capacity entries; if
 * more were needed it sets IMC_FLAG_COMB_OVERFLOW and n_out = the count needed (`in` is
 * untouched, so the caller can grow `out` and call again).  It also writes comb_before,
 * comb_after (= the radiation energy of `out`) and internal_energy = sum e*V. */
IMC_API int64_t imc_source_bound(const imc_mesh* mesh, const imc_step_params* par);
IMC_API imc_status imc_step_transport_async(const imc_mesh* mesh, const imc_material* mat,
                                            const imc_step_params* par, imc_bank* bank,
                                            imc_tallies* tal, void* workspace,
                                            size_t workspace_bytes,
                                            imc_step_summary* summary, void* stream);
IMC_API imc_status imc_comb_async(const imc_mesh* mesh, const imc_bank* in, imc_bank* out,
                                  int64_t n_max, uint64_t seed, uint32_t step, int32_t per_group,
                                  double* disc, const double* e, void* workspace,
                                  size_t workspace_bytes, imc_step_summary* summary,
                                  void* stream);
/* imc_comb_async with the Philox step counter read from device memory when the comb runs
 * (step_dev, a DEVICE pointer), so a captured comb can be replayed for every step; when
 * n_max_dev (DEVICE, nullable) is given, the comb target is read from it too (a growing
 * Nmax, MG_IMC/MG_IMC2D.py:2067-2120 'Nmax_next'), and n_max only selects the mode (> 0).
 * No reference counterpart (the reference time loop runs on the host). */
IMC_API imc_status imc_comb_async_dev(const imc_mesh* mesh, const imc_bank* in, imc_bank* out,
                                      int64_t n_max, const int64_t* n_max_dev, uint64_t seed,
                                      const uint32_t* step_dev, int32_t per_group, double* disc,
                                      const double* e, void* workspace, size_t workspace_bytes,
                                      imc_step_summary* summary, void* stream);
/* Energy (sum of live FP32 weights, FP64) per bin of a bank: per (group, cell) bin
 * g*nc + c when per_group is set (needs bank->group), else per cell; out[bins] is
 * overwritten.  The entry count is read from device memory when the kernel runs (n_dev, a
 * DEVICE pointer, e.g. the summary's n_out after imc_comb_async; counts above bank->capacity
 * are clipped to it), so it can follow a queued comb without a host synchronisation.  Divided
 * by the cell volumes this is MG_IMC2D's post-comb radiation_energy_by_group
 * (MG_IMC/MG_IMC2D.py:2017-2025). */
/* The fields a multigroup 2-D step reports, gathered in one device buffer in the reference's
 * array order (cells as (nx, ny) C order, j fastest; groups outermost), so that one
 * device-to-host copy of (2G + 3) nc + 2G doubles carries them all:
 *   out[0, G nc)            si[g][c] / c, the radiation energy density by group before the comb
 *                           (MG_IMC/MG_IMC2D.py:2017-2025 radiation_energy_by_group)
 *   out[G nc, 2G nc)        after[g][c] / V[c], the same after the comb (after: the second half
 *                           of an IMC_COMB_WRITE_AFTER disc)
 *   out[2G nc, (2G+3) nc)   e, T, Tr (nc each)
 *   then boundary_group and escaped_group (G each).
 * A NULL input skips its section (out keeps those entries), so the sections that are final
 * before the comb (everything but `after`) can be gathered and copied while the comb runs and
 * the post-comb section by a second call with only `after` set.  At least one input is set.
 * No reference counterpart (the reference's arrays are host arrays already). */
IMC_API imc_status imc_mg_report_fields(const imc_mesh* mesh, const double* si, const double* after,
                                        const double* e, const double* T, const double* Tr,
                                        const double* boundary_group, const double* escaped_group,
                                        double* out, void* stream);
IMC_API imc_status imc_bank_energy_by_bin(const imc_mesh* mesh, const imc_bank* bank, const int64_t* n_dev,
                                          int32_t per_group, double* out, void* stream);
/* Device time (ms) of the source fill and of tracking in this host thread's last
 * imc_step_transport[_async].  Waits for that step's tracking to end (not for work queued
 * after it, such as the comb), so a host can read the times while the comb runs. */
IMC_API imc_status imc_phase_times(float* ms_sources, float* ms_transport);

/* Sum of live weights (FP64) and of e[c]*V[c]; host results. */
IMC_API imc_status imc_energy_totals(const imc_mesh* mesh, const imc_bank* bank, const double* e,
                             double* radiation, double* internal, void* workspace,
                             size_t workspace_bytes, void* stream);

/* Philox-4x32-10 on the device, for known-answer tests: n counters (4 words each) with
 * one key -> n outputs. */
IMC_API imc_status imc_philox(const uint32_t* ctr, uint32_t key0, uint32_t key1, uint32_t* out,
                      int64_t n, void* stream);

IMC_API const char* imc_status_str(imc_status s);
IMC_API int imc_last_cuda_error(void);
/* number of kernels this library launched since load (diagnostic) */
IMC_API unsigned long long imc_kernel_launches(void);

/* ------------------------------------------------------------------------------------
 * Batched independent 1-D gray slab problems.
 *
 * Replaces a host loop of IMC/IMC1D.py:908 step(..., geometry='slab') over independent
 * problems.  Instance k is a slab of nc_k cells with
 *   sigma_a(T) = opacity_a[k] * T^opacity_p[k], constant cv[k] (e = cv T),
 *   boundary temperature face_T[2k + side] on the left (side 0) / right (side 1) face
 *   (<= 0: no source), reflect bit mask (bit 0 left, bit 1 right),
 *   n_target[k] emission and n_boundary[k] boundary particles per source face per step,
 *   comb target n_max[k] and Philox key seed[k].
 * Instance k's particles draw the same random numbers, in the same bank order, as a
 * single-problem run of imc_step_transport / imc_comb with seed[k] (census | left face |
 * right face | emission), so each instance reproduces that run.
 *
 * One imc_batch_step is a fixed sequence of kernels over all instances: sources, the
 * persistent tracking kernel (one work queue over every instance's histories), the fused
 * material + Fleck update, the per-cell comb and a per-instance energy ledger.  It reads
 * every count from device memory, synchronises nothing and allocates nothing, so the
 * caller may capture it in a CUDA graph and replay the graph once per step.
 * ------------------------------------------------------------------------------------ */
typedef struct imc_batch {
  int32_t n_inst;               /* K */
  int32_t n_cells;              /* sum of nc_k */
  int64_t n_slots;              /* bank slots per bank = slot_off[K] (host copy) */
  int64_t max_new;              /* host bound: sum over k of the new particles of one step,
                                   sides_k * n_boundary[k] + n_target[k] + nc_k */
  double dt, theta;
  const int32_t* cell_off;      /* [K+1] instance k owns cells [cell_off[k], cell_off[k+1]) */
  const double* edges;          /* [n_cells + K] instance k's nc_k+1 edges start at cell_off[k]+k */
  const int64_t* slot_off;      /* [K+1] bank slots of instance k */
  const uint64_t* seed;         /* [K] */
  const int64_t* n_target;      /* [K] */
  const int64_t* n_boundary;    /* [K] */
  const int64_t* n_max;         /* [K] */
  const double* face_T;         /* [2K] */
  const int32_t* reflect;       /* [K] */
  const double* opacity_a;      /* [K] */
  const double* opacity_p;      /* [K] */
  const double* cv;             /* [K] */
  int32_t max_cells;            /* the largest nc_k (host copy; 0: not given).  With 0 < max_cells <=
                                   IMC_BATCH_SMEM_CELLS the tracking keeps the instance's cell
                                   table and tallies of each work unit in shared memory */
} imc_batch;

/* largest instance whose cell table and tallies the batched tracking stages in shared memory */
#define IMC_BATCH_SMEM_CELLS 2048

/* per-instance energy ledger of the last step (FP64), ledger[k * IMC_BL_N + field] */
enum {
  IMC_BL_TOTAL = 0,      /* internal + radiation after the comb */
  IMC_BL_PREV = 1,       /* the same at the start of the step */
  IMC_BL_INTERNAL = 2,
  IMC_BL_RADIATION = 3,  /* census energy after the comb */
  IMC_BL_BOUNDARY = 4,   /* boundary energy issued */
  IMC_BL_ESCAPED = 5,
  IMC_BL_EMISSION = 6,   /* emission energy issued */
  IMC_BL_COMB_DISC = 7,  /* census energy before - after the comb */
  IMC_BL_CLOSURE = 8,    /* TOTAL - PREV - BOUNDARY + ESCAPED + COMB_DISC */
  IMC_BL_MAX_REL = 9,    /* max over steps of |CLOSURE| / TOTAL */
  IMC_BL_EVENTS = 10,    /* track segments of this instance, accumulated over steps */
  IMC_BL_N = 11
};

typedef struct imc_batch_state {   /* device memory, caller-owned */
  imc_bank bank[2];             /* 1-D banks (pos1, dir1, weight, time, cell), n_slots each */
  int32_t* sel;                 /* [1] the bank that holds the census */
  uint32_t* step;               /* [1] step index (Philox counter word 2) */
  int64_t* n_census;            /* [K] census entries of instance k, at its first slot */
  double* T;                    /* [n_cells] material temperature */
  double* e;                    /* [n_cells] internal energy density */
  double* tr;                   /* [n_cells] radiation temperature */
  double* dep;                  /* [n_cells] deposition of the last step */
  double* si;                   /* [n_cells] path-length intensity of the last step */
  double* emitted;              /* [n_cells] emission issued in the last step */
  double* ledger;               /* [K * IMC_BL_N] */
  unsigned long long* stats;    /* [IMC_STAT_N], accumulated over steps */
  int32_t* flags;               /* [1] IMC_FLAG_* (sticky; the caller clears it) */
} imc_batch_state;

typedef struct imc_batch_launch {  /* tracking kernel shape; 0 = default */
  int32_t block_size;
  int32_t blocks_per_sm;
  int32_t chunk;                /* histories per work-queue ticket (at most) */
  int32_t refill_min;           /* idle lanes a warp waits for before it refills (1..32) */
  int32_t form;                 /* tracking form: 1 work units (a block takes chunk x warps entries
                                   and stages each instance's tables and tallies in shared memory;
                                   needs imc_batch.max_cells), 2 the entry queue (warps take entries
                                   of any instance, tables and tallies in global memory; for many
                                   small instances), 3 work units with prefetched refills (each
                                   lane copies its next history's bank record into shared memory
                                   while it tracks the current one), 0 the library's choice (work
                                   units when max_cells allows) */
} imc_batch_launch;

IMC_API size_t imc_batch_workspace_bytes(const imc_batch* b);
/* T = T0, e = cv T0, equilibrium initial census of n_target[k] particles at Tr0
 * (IMC/IMC1D.py:220-248), ledger PREV, step = 0, sel = 0, stats and flags cleared, and
 * the Fleck tables of the first step.  Synchronises the stream. */
IMC_API imc_status imc_batch_init(const imc_batch* b, imc_batch_state* s, const double* T0,
                                  const double* Tr0, void* workspace, size_t workspace_bytes,
                                  void* stream);
/* One time step of every instance, asynchronous (see above).  Errors found on the device
 * (non-finite material state, a bank slot overflow) set bits in *s->flags. */
IMC_API imc_status imc_batch_step(const imc_batch* b, imc_batch_state* s,
                                  const imc_batch_launch* launch, void* workspace,
                                  size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* IMCB200_H */
