// imc_capi.cu — the extern "C" entry points of libimcb200.so (declared in
// include/imcb200.h): argument checks, workspace carving and phase ordering on the
// caller's stream.
//
// The step runs asynchronously: every element count a kernel needs lives in the device
// step summary, and the host supplies only upper bounds for grid sizes.  The synchronous
// entry points wrap the asynchronous ones with one host<->device round trip each.
#include <algorithm>
#include <cstdlib>
#include <cstddef>
#include <cstring>
#include <mutex>
#include "imc_device.cuh"
#include "imc_internal.h"

unsigned long long g_imc_launches = 0;
bool g_imc_pdl = [] {
  const char* e = std::getenv("IMCB200_PDL");
  return !(e && e[0] == '0');
}();

namespace {

thread_local int g_last_cuda = 0;

inline size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

#define IMC_CUDA(call)                              \
  do {                                              \
    cudaError_t e__ = (call);                       \
    if (e__ != cudaSuccess) {                       \
      g_last_cuda = (int)e__;                       \
      return IMC_ERR_CUDA;                          \
    }                                               \
  } while (0)

// Timing events for the last step in this host thread (created on first use).
struct PhaseEvents {
  cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
  bool ok = false, recorded = false;
  explicit PhaseEvents(bool create = true) {
    ok = create;
    if (create)
      for (auto& x : e) ok = ok && cudaEventCreate(&x) == cudaSuccess;
  }
};
PhaseEvents& phase_events() {
  static thread_local PhaseEvents pe;
  return pe;
}

// A second stream per device and host thread (non-blocking, created on first use) with a
// fork and a join event: a step's boundary faces and tracked-weight sums are made on it beside
// the volume fill.  NULL when it cannot be created (the step then runs both on its stream).
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  bool ok = false, tried = false;
};
SideStream* side_stream() {
  static thread_local SideStream ss[16];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 16) return nullptr;
  SideStream& x = ss[dev];
  if (!x.tried) {
    x.tried = true;
    x.ok = cudaStreamCreateWithFlags(&x.s, cudaStreamNonBlocking) == cudaSuccess &&
           cudaEventCreateWithFlags(&x.fork, cudaEventDisableTiming) == cudaSuccess &&
           cudaEventCreateWithFlags(&x.join, cudaEventDisableTiming) == cudaSuccess;
  }
  return x.ok ? &x : nullptr;
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

imc_status check_mesh(const imc_mesh* m) {
  if (!m || !m->edges1 || !m->edges2 || !m->volume) return IMC_ERR_INVALID_ARG;
  if (m->geometry < IMC_GEOM_SLAB || m->geometry > IMC_GEOM_RZ) return IMC_ERR_BAD_GEOMETRY;
  if (m->nx <= 0 || m->ny <= 0) return IMC_ERR_BAD_GEOMETRY;
  const bool oned = m->geometry == IMC_GEOM_SLAB || m->geometry == IMC_GEOM_SPHERE;
  if (oned && m->ny != 1) return IMC_ERR_BAD_GEOMETRY;
  if (m->n_groups < 1) return IMC_ERR_INVALID_ARG;
  // multigroup: xy / rz (MG_IMC2D) and the 1-D sphere (MG_IMC1D)
  if (m->n_groups > 1 && (m->geometry == IMC_GEOM_SLAB || !m->group_edges)) return IMC_ERR_INVALID_ARG;
  return IMC_OK;
}

bool bank_ok(const imc_bank* b, bool two_d, bool mg = false) {
  if (!b || !b->pos1 || !b->dir1 || !b->weight || !b->time || !b->cell) return false;
  if (mg && !b->group) return false;
  if (two_d && (!b->pos2 || !b->dir2)) return false;
  return b->size >= 0 && b->capacity >= b->size && b->capacity < (1LL << 31);
}

// the workspace is 256-byte aligned by contract (its tables hold 8- and 16-byte vectors)
inline bool ws_misaligned(const void* workspace) { return (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0; }
inline bool mg_sphere(const imc_mesh* m) { return m->n_groups > 1 && m->geometry == IMC_GEOM_SPHERE; }

inline long long side_count(const imc_step_params* p, int q) {
  return p->n_boundary_side[q] > 0 ? p->n_boundary_side[q] : p->n_boundary;
}

long long source_bound(const imc_mesh* m, const imc_step_params* p) {
  // ceil adds at most one per cell; MG 1-D: round (+1/2) and the minimum of one per bin
  const long long nb = (long long)m->nx * m->ny * (mg_sphere(m) ? m->n_groups : 1);
  long long b = 0;
  for (int q = 0; q < 4; ++q)
    if (p->face_T[q] && side_count(p, q) > 0) b += side_count(p, q);
  if (p->n_target > 0) b += p->n_target + nb;
  if (p->n_source > 0) b += p->n_source + nb;
  return b;
}

inline void set_bank(float*& p2, float*& d2, const imc_bank* b, bool two_d) {
  p2 = two_d ? b->pos2 : nullptr;
  d2 = two_d ? b->dir2 : nullptr;
}

// adj != NULL: the sources are made as for the forward step, then the adjoint kernel
// replays the histories instead of tracking them (bank and tallies are not written).
imc_status transport_async(const imc_mesh* mesh, const imc_material* mat, const imc_step_params* par,
                           imc_bank* bank, imc_tallies* tal, void* workspace, size_t workspace_bytes,
                           imc_step_summary* sum, cudaStream_t s, const AdjointArgs* adj = nullptr) {
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  const bool two_d = mesh->geometry >= IMC_GEOM_XY;
  const int ng = mesh->n_groups;
  const bool mg = ng > 1;
  const bool mg1 = mg_sphere(mesh);  // MG_IMC1D: stratified (group, cell) sources
  if (!mat || !mat->temperature || !mat->sigma || !mat->cv || !par || !tal || !sum) return IMC_ERR_INVALID_ARG;
  if (!tal->dep || !tal->si || !tal->emitted || !tal->sigma_a || !tal->sigma_s || !tal->escaped || !tal->stats)
    return IMC_ERR_INVALID_ARG;
  if (mg && (!tal->escaped_group || !tal->boundary_group)) return IMC_ERR_INVALID_ARG;
  if (!bank_ok(bank, two_d, mg) || !workspace) return IMC_ERR_INVALID_ARG;
  if (!(par->dt > 0.0) || par->n_target < 0 || par->n_boundary < 0 || par->n_source < 0) return IMC_ERR_INVALID_ARG;
  if (!(par->energy_share >= 0.0 && par->energy_share <= 1.0)) return IMC_ERR_INVALID_ARG;
  if (par->census_bins < 0 || par->census_bins > IMC_CENSUS_BY_GROUP_CELL ||
      (par->census_bins == IMC_CENSUS_BY_GROUP_CELL && mesh->n_groups < 2))
    return IMC_ERR_INVALID_ARG;
  const double share = par->energy_share > 0.0 ? par->energy_share : 1.0;
  for (int q = 0; q < 4; ++q) if (par->n_boundary_side[q] < 0) return IMC_ERR_INVALID_ARG;
  const bool cf = par->method == IMC_METHOD_CARTER_FOREST;
  if (par->method != IMC_METHOD_FLECK_CUMMINGS && !cf) return IMC_ERR_INVALID_ARG;
  if (cf && (mg || adj)) return IMC_ERR_INVALID_ARG;  // Carter-Forest: gray forward steps
  const long long bound = source_bound(mesh, par);
  const long long n_upper = bank->size + bound;
  if (n_upper > bank->capacity) return IMC_ERR_BANK_OVERFLOW;
  const WsLayout L = imc_ws_layout(mesh, bank->capacity);
  if (workspace_bytes < L.total || ws_misaligned(workspace)) return IMC_ERR_WORKSPACE;
  const int nc = mesh->nx * mesh->ny;
  // reserved bit 3: event-by-event tracking, its scratch after the workspace layout
  const bool event_mode = (par->reserved & 8) != 0;
  if (event_mode) {
    if (par->census_bins || adj) return IMC_ERR_INVALID_ARG;
    if (workspace_bytes < L.total + imc_event_scratch_bytes(bank->capacity)) return IMC_ERR_WORKSPACE;
  }

  // every per-step accumulator starts at zero, in one launch: the summary's per-step fields
  // (everything after n_census), the group energies, the fixed-point tallies, the intensity,
  // the statistics, the tracking ticket and the census sums for the comb
  unsigned long long* dep_fx = ws_ptr<unsigned long long>(workspace, L.dep_fx);
  unsigned long long* esc_fx = ws_ptr<unsigned long long>(workspace, L.esc_fx);
  unsigned long long* queue = ws_ptr<unsigned long long>(workspace, L.queue);
  {
    ZeroList zl{};
    zl.add(reinterpret_cast<char*>(sum) + sizeof(int64_t), sizeof(imc_step_summary) - sizeof(int64_t));
    if (mg) {
      zl.add(tal->boundary_group, sizeof(double) * ng);
      zl.add(tal->escaped_group, sizeof(double) * ng);
    }
    zl.add(dep_fx, sizeof(unsigned long long) * nc * ng);
    zl.add(esc_fx, sizeof(unsigned long long) * (4 + ng));
    zl.add(tal->si, sizeof(double) * nc * ng);
    zl.add(tal->stats, sizeof(unsigned long long) * IMC_STAT_N);
    zl.add(queue, 8);
    if (par->census_bins && !adj) {
      const int nb = par->census_bins == IMC_CENSUS_BY_GROUP_CELL ? nc * ng : nc;
      zl.add(ws_ptr<double>(workspace, L.ecen), sizeof(double) * nb);
      zl.add(ws_ptr<unsigned long long>(workspace, L.comb_mode + 8), sizeof(unsigned long long));
    }
    IMC_CUDA(imc_launch_zero(zl, s));
  }

  // ---- plan: Fleck, per-cell source counts / weights / offsets, boundary faces ----
  PlanArgs pa{};
  pa.geom = mesh->geometry; pa.nx = mesh->nx; pa.ny = mesh->ny; pa.nc = nc; pa.ng = 1;
  pa.e1 = mesh->edges1; pa.e2 = mesh->edges2; pa.vol = mesh->volume;
  pa.T = mat->temperature; pa.sigma = mat->sigma; pa.cv = mat->cv; pa.source = mat->source;
  pa.dt = par->dt; pa.theta = par->theta;
  pa.n_target = par->n_target; pa.n_source = par->n_source; pa.n_boundary = par->n_boundary;
  for (int q = 0; q < 4; ++q) pa.n_side[q] = side_count(par, q);
  for (int q = 0; q < 4; ++q) pa.face_T[q] = par->face_T[q];
  pa.rz_linear = par->rz_linear_source; pa.t_emit_floor = par->t_emit_floor;
  pa.method = par->method; pa.cf_rate = ws_ptr<float>(workspace, L.cf_rate);
  pa.dt_dev = par->dt_dev;
  pa.share = share;
  pa.sa = tal->sigma_a; pa.ss = tal->sigma_s;
  pa.sass = ws_ptr<float2>(workspace, L.sass); pa.cellf = ws_ptr<double2>(workspace, L.cellf);
  pa.e1f = ws_ptr<float>(workspace, L.e1f); pa.e2f = ws_ptr<float>(workspace, L.e2f);
  pa.emit_E = ws_ptr<double>(workspace, L.emit_E); pa.emit_n = ws_ptr<long long>(workspace, L.emit_n);
  pa.emit_off = ws_ptr<long long>(workspace, L.emit_off); pa.emit_w = ws_ptr<float>(workspace, L.emit_w);
  pa.tilt = ws_ptr<double>(workspace, L.tilt);
  pa.src_n = ws_ptr<long long>(workspace, L.src_n); pa.src_off = ws_ptr<long long>(workspace, L.src_off);
  pa.src_w = ws_ptr<float>(workspace, L.src_w); pa.src_QV = ws_ptr<double>(workspace, L.src_QV);
  pa.src_issued = ws_ptr<double>(workspace, L.src_issued);
  pa.emitted = tal->emitted;
  pa.face = ws_ptr<double>(workspace, L.face); pa.nf = std::max(mesh->nx, mesh->ny);
  pa.sum = sum;
  PlanMgArgs pm{};
  if (!mg) {
    IMC_CUDA(imc_launch_plan(pa, s));
  } else if (mg1) {
    pm.geom = mesh->geometry; pm.nx = mesh->nx; pm.ny = mesh->ny; pm.nc = nc; pm.ng = ng;
    pm.e1 = mesh->edges1; pm.e2 = mesh->edges2; pm.vol = mesh->volume;
    pm.T = mat->temperature; pm.sigma = mat->sigma; pm.cv = mat->cv; pm.source = mat->source;
    pm.gedges = mesh->group_edges;
    pm.dt = par->dt; pm.theta = par->theta;
    pm.n_target = par->n_target; pm.n_source = par->n_source; pm.n_boundary = par->n_boundary;
    for (int q = 0; q < 4; ++q) pm.n_side[q] = side_count(par, q);
    for (int q = 0; q < 4; ++q) pm.face_T[q] = par->face_T[q];
    pm.t_emit_floor = par->t_emit_floor;
    pm.sa = tal->sigma_a; pm.ss = tal->sigma_s; pm.sass = pa.sass; pm.cellf = pa.cellf;
    pm.e1f = pa.e1f; pm.e2f = pa.e2f;
    pm.Egc = ws_ptr<double>(workspace, L.mg_gcdf);
    pm.emitted = tal->emitted; pm.face = pa.face; pm.nf = pa.nf;
    pm.mixcdf = ws_ptr<double>(workspace, L.mixcdf);
    pm.emit_E = pa.emit_E; pm.emit_n = pa.emit_n; pm.emit_off = pa.emit_off; pm.emit_w = pa.emit_w;
    pm.emit_issued = ws_ptr<double>(workspace, L.emit_issued);
    pm.src_QV = pa.src_QV; pm.src_n = pa.src_n; pm.src_off = pa.src_off; pm.src_w = pa.src_w;
    pm.src_issued = pa.src_issued;
    pm.sum = sum;
    pm.dt_dev = par->dt_dev;
    pm.share = share;
    IMC_CUDA(imc_launch_plan_mg1d(pm, s));
  } else {
    pm.geom = mesh->geometry; pm.nx = mesh->nx; pm.ny = mesh->ny; pm.nc = nc; pm.ng = ng;
    pm.e1 = mesh->edges1; pm.e2 = mesh->edges2; pm.vol = mesh->volume;
    pm.T = mat->temperature; pm.sigma = mat->sigma; pm.cv = mat->cv; pm.source = mat->source;
    pm.gedges = mesh->group_edges; pm.emission_fractions = par->emission_fractions;
    pm.dt = par->dt; pm.theta = par->theta;
    pm.n_target = par->n_target; pm.n_source = par->n_source; pm.n_boundary = par->n_boundary;
    for (int q = 0; q < 4; ++q) pm.n_side[q] = side_count(par, q);
    for (int q = 0; q < 4; ++q) pm.face_T[q] = par->face_T[q];
    pm.t_emit_floor = par->t_emit_floor;
    pm.sa = tal->sigma_a; pm.ss = tal->sigma_s; pm.sass = pa.sass; pm.cellf = pa.cellf;
    pm.e1f = pa.e1f; pm.e2f = pa.e2f;
    pm.Egc = ws_ptr<double>(workspace, L.mg_gcdf); pm.Ec = ws_ptr<double>(workspace, L.mg_ec);
    pm.cdf = ws_ptr<double>(workspace, L.mg_cdf);
    pm.Sgc = ws_ptr<double>(workspace, L.mg_sgcdf); pm.Sc = ws_ptr<double>(workspace, L.mg_sc);
    pm.Scdf = ws_ptr<double>(workspace, L.mg_scdf);
    pm.emitted = tal->emitted; pm.face = pa.face; pm.nf = pa.nf;
    pm.mixcdf = ws_ptr<double>(workspace, L.mixcdf);
    pm.sum = sum;
    pm.dt_dev = par->dt_dev;
    pm.share = share;
    IMC_CUDA(imc_launch_plan_mg(pm, s));
  }

  // ---- sources, appended in the reference's order: census | boundary | fixed | emission ----
  // (the phase-timing events are left out of a stream capture)
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  IMC_CUDA(cudaStreamIsCapturing(s, &capture));
  PhaseEvents& pe_all = phase_events();
  PhaseEvents pe_off(false);
  PhaseEvents& pe = capture == cudaStreamCaptureStatusNone ? pe_all : pe_off;
  if (pe.ok) IMC_CUDA(cudaEventRecord(pe.e[0], s));
  float *p2, *d2;
  set_bank(p2, d2, bank, two_d);
  // every source of the step (and the sum of the tracked weights) in one launch
  SourceJobs sj{};
  imcdev::philox_round_keys(par->seed, sj.rk);
  sj.wsum = &sum->weight_sum;
  sj.census_w = bank->weight;
  sj.n_census = &sum->n_census;
  for (int side = 0; side < 4; ++side) {
    if (!par->face_T[side] || side_count(par, side) <= 0) continue;
    BndArgs& ba = sj.bnd[sj.n_bnd++];
    ba.geom = mesh->geometry; ba.nx = mesh->nx; ba.ny = mesh->ny; ba.side = side; ba.nf = pa.nf;
    ba.e1 = mesh->edges1; ba.e2 = mesh->edges2;
    ba.face = pa.face + (size_t)side * 2 * pa.nf;
    ba.d_n = &sum->n_side[side]; ba.d_base = &sum->base_side[side]; ba.n_bound = side_count(par, side);
    ba.dt = par->dt; ba.seed = par->seed; ba.step = par->step;
    imcdev::philox_round_keys(ba.seed, ba.rk);
    ba.p1 = bank->pos1; ba.p2 = p2; ba.d1 = bank->dir1; ba.d2 = d2; ba.wb = bank->weight;
    ba.t = bank->time; ba.cell = bank->cell; ba.group = bank->group;
    ba.ng = ng; ba.faceT = par->face_T[side]; ba.gedges = mesh->group_edges;
    ba.mixcdf = ws_ptr<double>(workspace, L.mixcdf); ba.boundary_group = tal->boundary_group;
    ba.below_last = mg1 ? 1 : 0;
    ba.dt_dev = par->dt_dev; ba.step_dev = par->step_dev;
    ba.id_base = par->id_base;
  }
  const int nbins = mg1 ? nc * ng : nc;  // source order positions (MG 1-D: (group, cell) bins)
  bool cf_times = false;
  auto fill = [&](const int64_t* d_n, const int64_t* d_base, long long n_bound, const long long* off,
                  const float* w, const double* tilt, int kind, uint32_t tag) -> cudaError_t {
    if (sj.n_vol >= 2) return cudaErrorInvalidValue;
    FillArgs& fa = sj.vol[sj.n_vol++];
    fa.geom = mesh->geometry; fa.nx = mesh->nx; fa.ny = mesh->ny; fa.nc = nc;
    fa.nbins = nbins; fa.bins_by_group = mg1 ? 1 : 0;
    fa.time_scale_dev = par->dt_dev; fa.step_dev = par->step_dev;
    fa.id_base = par->id_base;
    fa.e1 = mesh->edges1; fa.e2 = mesh->edges2; fa.T = mat->temperature;
    fa.d_n = d_n; fa.d_base = d_base; fa.n_bound = n_bound;
    fa.off = off; fa.w = w; fa.tilt = tilt; fa.tilt_kind = kind;
    fa.time_scale = par->dt; fa.seed = par->seed; fa.step = par->step; fa.tag = tag;
    imcdev::philox_round_keys(fa.seed, fa.rk);
    fa.p1 = bank->pos1; fa.p2 = p2; fa.d1 = bank->dir1; fa.d2 = d2; fa.wb = bank->weight;
    fa.t = bank->time; fa.cell = bank->cell; fa.group = bank->group;
    if (cf_times) {
      fa.cf_rate4 = pa.tilt + 3;
      fa.cf_thr = (mesh->geometry == IMC_GEOM_SLAB || mesh->geometry == IMC_GEOM_SPHERE) ? 1e-10 : 1e-12;
    }
    return cudaSuccess;
  };
  auto fill_mg = [&](const int64_t* d_n, const int64_t* d_base, long long n_bound, const double* cdf,
                     const double* gcdf, uint32_t tag) -> cudaError_t {
    if (sj.n_vmg >= 2) return cudaErrorInvalidValue;
    FillMgArgs& fm = sj.vmg[sj.n_vmg++];
    fm.geom = mesh->geometry; fm.nx = mesh->nx; fm.ny = mesh->ny; fm.nc = nc; fm.ng = ng;
    fm.e1 = mesh->edges1; fm.e2 = mesh->edges2; fm.cdf = cdf; fm.gcdf = gcdf; fm.tr = nullptr;
    fm.gedges = mesh->group_edges; fm.mixcdf = ws_ptr<double>(workspace, L.mixcdf);
    fm.d_n = d_n; fm.d_base = d_base; fm.n_bound = n_bound;
    fm.time_scale = par->dt; fm.seed = par->seed; fm.step = par->step; fm.tag = tag;
    imcdev::philox_round_keys(fm.seed, fm.rk);
    fm.p1 = bank->pos1; fm.p2 = p2; fm.d1 = bank->dir1; fm.d2 = d2; fm.wb = bank->weight;
    fm.t = bank->time; fm.cell = bank->cell; fm.group = bank->group;
    fm.time_scale_dev = par->dt_dev; fm.step_dev = par->step_dev;
    fm.id_base = par->id_base;
    return cudaSuccess;
  };
  const bool rzlin = mesh->geometry == IMC_GEOM_RZ && par->rz_linear_source;
  if (mg1) {
    if (mat->source && par->n_source > 0)
      IMC_CUDA(fill(&sum->n_source, &sum->base_source, par->n_source + nbins, pa.src_off, pa.src_w, nullptr, 0,
                    imcdev::TAG_SOURCE));
    if (par->n_target > 0)
      IMC_CUDA(fill(&sum->n_emission, &sum->base_emission, par->n_target + nbins, pa.emit_off, pa.emit_w, nullptr, 0,
                    imcdev::TAG_EMISSION));
  } else if (mg) {
    if (mat->source && par->n_source > 0)
      IMC_CUDA(fill_mg(&sum->n_source, &sum->base_source, par->n_source, pm.Scdf, pm.Sgc, imcdev::TAG_SOURCE));
    if (par->n_target > 0)
      IMC_CUDA(fill_mg(&sum->n_emission, &sum->base_emission, par->n_target, pm.cdf, pm.Egc, imcdev::TAG_EMISSION));
  } else if (mat->source && par->n_source > 0)
    IMC_CUDA(fill(&sum->n_source, &sum->base_source, par->n_source + nc, pa.src_off, pa.src_w,
                  rzlin ? pa.tilt : nullptr, rzlin ? 3 : 0, imcdev::TAG_SOURCE));
  int ekind = 0;
  if (mesh->geometry == IMC_GEOM_SLAB) ekind = 1;
  else if (mesh->geometry == IMC_GEOM_SPHERE) ekind = 2;
  else if (rzlin) ekind = 3;
  if (!mg && par->n_target > 0) {
    cf_times = cf;  // Carter-Forest birth times for the emission only
    IMC_CUDA(fill(&sum->n_emission, &sum->base_emission, par->n_target + nc, pa.emit_off, pa.emit_w,
                  ekind ? pa.tilt : nullptr, ekind, imcdev::TAG_EMISSION));
    cf_times = false;
  }

  // two launches of the job table: the faces with the tracked-weight sums and the volume fills
  // (one kernel holding every body would run the volume fill with fewer resident blocks).  With
  // a large volume fill (crooked pipe RZ: 5 us less from plan to tracking) the first launch is
  // forked onto the side stream and tracking waits for both; a small one (the multigroup
  // crooked pipe's, where the fork's events cost 4 us more) runs after it on the step's stream.
  long long vol_bound = 0;
  for (int q = 0; q < sj.n_vol; ++q) vol_bound += sj.vol[q].n_bound;
  SideStream* side = vol_bound >= (1LL << 19) ? side_stream() : nullptr;
  {
    const int nb = sj.n_jobs;
    for (int q = 0; q < sj.n_bnd; ++q) sj.add(JOB_BOUNDARY, q, imc_source_blocks(sj.bnd[q].n_bound));
    sj.add(JOB_CENSUS_WSUM, 0, std::min(imc_source_blocks(std::max<long long>(bank->size, 1)), 4 * sm_count()));
    if (side) {
      IMC_CUDA(cudaEventRecord(side->fork, s));
      IMC_CUDA(cudaStreamWaitEvent(side->s, side->fork, 0));
    }
    IMC_CUDA(imc_launch_sources(sj, side ? side->s : s));
    if (side) IMC_CUDA(cudaEventRecord(side->join, side->s));
    sj.n_jobs = nb;
    for (int q = 0; q < sj.n_vol; ++q) sj.add(JOB_VOLUME, q, imc_source_blocks(sj.vol[q].n_bound));
    IMC_CUDA(imc_launch_sources(sj, s));
    sj.n_jobs = nb;
    for (int q = 0; q < sj.n_vmg; ++q) sj.add(JOB_VOLUME_MG, q, imc_source_blocks(sj.vmg[q].n_bound));
    IMC_CUDA(imc_launch_sources(sj, s));
    if (side) IMC_CUDA(cudaStreamWaitEvent(s, side->join, 0));
  }

  // ---- tracking ----
  if (pe.ok) IMC_CUDA(cudaEventRecord(pe.e[1], s));

  TrackArgs ta{};
  ta.nx = mesh->nx; ta.ny = mesh->ny; ta.nc = nc; ta.ng = ng;
  ta.e1 = pa.e1f; ta.e2 = pa.e2f; ta.sass = pa.sass; ta.cellf = pa.cellf;
  ta.dep = tal->dep; ta.si = tal->si; ta.escaped = tal->escaped; ta.stats = tal->stats;
  ta.p1 = bank->pos1; ta.p2 = p2; ta.d1 = bank->dir1; ta.d2 = d2; ta.w = bank->weight; ta.t = bank->time;
  ta.cell = bank->cell; ta.group = bank->group;
  ta.n_dev = &sum->n_bank; ta.wsum = &sum->weight_sum; ta.queue = queue; ta.flags = &sum->flags;
  ta.dt = (float)par->dt;
  ta.floor_coef = mg1 ? 1e-14 : 1e-10;
  ta.cf_rate = cf ? pa.cf_rate : nullptr;
  ta.cf_fastpath = (float)par->cf_fastpath;
  ta.dt_dev = par->dt_dev; ta.step_dev = par->step_dev;
  ta.id_base = par->id_base;
  if (par->census_bins && !adj) {
    // census sums for the comb that follows on this workspace (IMC_COMB_CENSUS_READY),
    // zeroed with the step's accumulators
    ta.ecen = ws_ptr<double>(workspace, L.ecen);
    ta.n_live = ws_ptr<unsigned long long>(workspace, L.comb_mode + 8);
    ta.ecen_by_group = par->census_bins == IMC_CENSUS_BY_GROUP_CELL ? 1 : 0;
  }
  int rm = 0;
  for (int q = 0; q < 4; ++q) if (par->reflect[q]) rm |= 1 << q;
  ta.reflect_mask = rm;
  ta.max_events = par->max_events > 0 ? par->max_events : (long long)1 << 30;
  ta.cap_is_reference = par->max_events > 0 ? 1 : 0;
  ta.seed = par->seed; ta.step = par->step;
  imcdev::philox_round_keys(ta.seed, ta.rk);
  ta.chunk = par->chunk > 0 ? par->chunk : 64;
  ta.group_edges = mesh->group_edges;
  ta.escaped_group = tal->escaped_group;
  ta.dep_fx = dep_fx; ta.esc_fx = esc_fx;
  const int block = par->block_size > 0 ? par->block_size : 256;
  const int bps = par->blocks_per_sm > 0 ? par->blocks_per_sm : 3;
  // reserved: bit 0 = stage the cell table in shared memory; bit 1 = block tallies in shared
  // memory, bit 2 = never (default: with the staged table up to 2048 (group, cell) entries)
  const bool smem_cells = (par->reserved & 1) ? true : ((long long)nc * ng <= 4096);
  const bool smem_tally = smem_cells && !(par->reserved & 4) && ((par->reserved & 2) || (long long)nc * ng <= 2048);
  // bit 4: prefetched refills (each lane's next bank record copied to shared memory ahead)
  const bool prefetch = (par->reserved & 16) != 0;
  if (adj) {
    AdjointArgs A = *adj;
    A.t = ta; A.sa64 = tal->sigma_a; A.ss64 = tal->sigma_s; A.sig64 = mat->sigma;
    IMC_CUDA(imc_launch_adjoint(A, mesh->geometry, block, sm_count() * bps, s));
    if (pe.ok) { IMC_CUDA(cudaEventRecord(pe.e[2], s)); pe.recorded = true; }
    return IMC_OK;
  }
  if (event_mode) {
    bool cap_hit = false;
    IMC_CUDA(imc_run_event_tracking(ta, mesh->geometry, static_cast<char*>(workspace) + L.total, bank->capacity,
                                    n_upper, block, sm_count(), ta.max_events + 2, &cap_hit, s));
    if (cap_hit) return IMC_ERR_EVENT_CAP;
  } else {
    IMC_CUDA(imc_launch_track(ta, mesh->geometry, block, sm_count() * bps, smem_cells, smem_tally, prefetch, s));
  }
  if (pe.ok) { IMC_CUDA(cudaEventRecord(pe.e[2], s)); pe.recorded = true; }
  IMC_CUDA(imc_launch_tally_finalize(ta, s));
  return IMC_OK;
}

imc_status comb_async(const imc_mesh* mesh, const imc_bank* in, imc_bank* out, int64_t n_max, uint64_t seed,
                      uint32_t step, int32_t per_group, double* disc, const double* e, void* workspace,
                      size_t workspace_bytes, imc_step_summary* sum, cudaStream_t s,
                      const uint32_t* step_dev = nullptr, const int64_t* n_max_dev = nullptr) {
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  const bool two_d = mesh->geometry >= IMC_GEOM_XY;
  if (!bank_ok(in, two_d) || !bank_ok(out, two_d) || !disc || !workspace || !sum) return IMC_ERR_INVALID_ARG;
  if (in->pos1 == out->pos1 || in->weight == out->weight) return IMC_ERR_INVALID_ARG;
  const bool by_group = (per_group & IMC_COMB_PER_GROUP) != 0;
  const bool census_ready = (per_group & IMC_COMB_CENSUS_READY) != 0;  // sums made by the tracking
  if (by_group && (!in->group || !out->group)) return IMC_ERR_INVALID_ARG;
  const WsLayout L = imc_ws_layout(mesh, in->size);
  if (workspace_bytes < L.total || ws_misaligned(workspace)) return IMC_ERR_WORKSPACE;
  const int nc = mesh->nx * mesh->ny;
  const int nb = by_group ? nc * mesh->n_groups : nc;

  CombArgs ca{};
  ca.nc = nc; ca.nb = nb; ca.per_group = by_group ? 1 : 0;
  ca.conserve_rad = (per_group & IMC_COMB_CONSERVE_RADIATION) ? 1 : 0;
  ca.mode = ws_ptr<int>(workspace, L.comb_mode);
  ca.n_live = ws_ptr<unsigned long long>(workspace, L.comb_mode + 8);
  ca.d_n_in = &sum->n_bank; ca.n_bound = in->size; ca.out_capacity = out->capacity;
  ca.w = in->weight; ca.cell = in->cell; ca.group = in->group;
  ca.p1 = in->pos1; ca.p2 = two_d ? in->pos2 : nullptr; ca.d1 = in->dir1; ca.d2 = two_d ? in->dir2 : nullptr;
  ca.ecen = ws_ptr<double>(workspace, L.ecen); ca.ew = ws_ptr<double>(workspace, L.ew);
  ca.ncopy = ws_ptr<unsigned long long>(workspace, L.ncopy); ca.cnt = ws_ptr<int>(workspace, L.cnt);
  ca.blk = ws_ptr<long long>(workspace, L.blk);
  ca.seed = seed; ca.step = step; ca.step_dev = step_dev;
  imcdev::philox_round_keys(seed, ca.rk);
  ca.op1 = out->pos1; ca.op2 = two_d ? out->pos2 : nullptr; ca.od1 = out->dir1; ca.od2 = two_d ? out->dir2 : nullptr;
  ca.ow = out->weight; ca.ot = out->time; ca.ocell = out->cell; ca.ogroup = out->group;
  ca.vec16 = ((reinterpret_cast<uintptr_t>(in->weight) | reinterpret_cast<uintptr_t>(in->cell) |
               reinterpret_cast<uintptr_t>(by_group ? in->group : in->cell)) & 15u) == 0;
  ca.disc = disc;
  ca.after = (per_group & IMC_COMB_WRITE_AFTER) ? disc + nb : nullptr;
  ca.sum = sum;

  // ncopy is zeroed by the comb plan's weights kernel, comb_after and the mode by the plan
  if (!census_ready) {  // else the census sums and the live count are the tracking's
    IMC_CUDA(cudaMemsetAsync(ca.ecen, 0, sizeof(double) * nb, s));
    IMC_CUDA(cudaMemsetAsync(ca.mode, 0, 16, s));
    IMC_CUDA(imc_launch_comb_ecen(ca, s));
  }
  CombPlanArgs cp{};
  cp.nb = nb; cp.ecen = ca.ecen; cp.ew = ca.ew; cp.ncopy = ca.ncopy; cp.sum = sum;
  // n_max > 0: comb to n_max; 0: keep every live entry; < 0: comb to |n_max| once at least
  // |n_max| entries are alive (MG_IMC/MG_IMC1D.py:1194-1200)
  cp.n_max = n_max < 0 ? -n_max : n_max;
  cp.n_max_dev = n_max > 0 ? n_max_dev : nullptr;
  cp.threshold = n_max < 0 ? -n_max : 0;
  cp.force_compact = n_max == 0 ? 1 : 0;
  cp.n_live = ca.n_live; cp.mode = ca.mode;
  IMC_CUDA(imc_launch_comb_plan(cp, s));
  IMC_CUDA(imc_launch_comb_count(ca, s));
  IMC_CUDA(imc_launch_comb_scatter(ca, s));
  if (e) IMC_CUDA(imc_launch_canon_sum_eV(e, mesh->volume, nc, &sum->internal_energy, s));
  return IMC_OK;
}

imc_step_summary* internal_summary(void* workspace, const WsLayout& L) {
  return ws_ptr<imc_step_summary>(workspace, L.summary);
}

}  // namespace

void imc_note_cuda_error(int e) { g_last_cuda = e; }

WsLayout imc_ws_layout(const imc_mesh* m, int64_t capacity) {
  WsLayout L{};
  size_t o = 0;
  const size_t nx = (size_t)m->nx, ny = (size_t)m->ny, nc = nx * ny;
  const size_t ng = (size_t)std::max(1, m->n_groups), ncg = nc * ng;
  const size_t nf = std::max(nx, ny);
  const size_t cap = (size_t)std::max<int64_t>(capacity, 1);
  auto take = [&](size_t bytes) { const size_t r = o; o += al256(bytes); return r; };
  L.summary = take(sizeof(imc_step_summary)); L.queue = take(8);
  L.e1f = take(4 * (nx + 1)); L.e2f = take(4 * (ny + 1));
  L.sass = take(8 * ncg); L.cellf = take(16 * ncg);
  L.emit_E = take(8 * ncg); L.emit_n = take(8 * ncg); L.emit_off = take(8 * (ncg + 1)); L.emit_w = take(4 * ncg);
  L.emit_issued = take(8 * ncg);
  L.tilt = take(8 * 4 * nc);
  L.src_n = take(8 * ncg); L.src_off = take(8 * (ncg + 1)); L.src_w = take(4 * ncg);
  L.src_QV = take(8 * ncg); L.src_issued = take(8 * ncg);
  L.face = take(8 * 4 * 2 * nf);
  if (ng > 1) {
    L.mg_gcdf = take(8 * ncg); L.mg_ec = take(8 * nc); L.mg_cdf = take(8 * nc);
    L.mg_sgcdf = take(8 * ncg); L.mg_sc = take(8 * nc); L.mg_scdf = take(8 * nc);
  }
  L.mixcdf = take(8 * 200);
  L.ecen = take(8 * ncg); L.ew = take(8 * ncg); L.ncopy = take(8 * ncg);
  L.comb_mode = take(16);
  L.dep_fx = take(8 * ncg); L.esc_fx = take(8 * (4 + ng));
  L.cf_rate = take(4 * nc);
  // The regions sized by the capacity come last, so every other offset is the same for any
  // capacity: a comb, laid out for its input's size, finds the census sums and the live count
  // where the tracking, laid out for the bank's capacity, left them.
  L.cnt = take(4 * cap); L.blk = take(8 * ((cap + 1023) / 1024 + 2));
  L.total = o;
  return L;
}

// ---- library-owned comb scratch (imc_comb_noalloc) ----
// A caller that owns no device allocator cannot provide a workspace, so this entry point
// carves its scratch from a fixed array linked into the library.  The array is a module
// global: the runtime creates one per device when the module is loaded there, which
// happens at the latest on the first cudaGetSymbolAddress with that device current.
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[IMC_NOALLOC_SCRATCH_BYTES];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of this device's scratch array, looked up once per device.
imc_status noalloc_scratch(void** ptr) {
  int dev = -1;
  IMC_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return IMC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    IMC_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    if (!p) return IMC_ERR_CUDA;
    g_noalloc_ptr[dev] = p;
  }
  *ptr = g_noalloc_ptr[dev];
  return IMC_OK;
}

}  // namespace

extern "C" {

size_t imc_workspace_bytes(const imc_mesh* mesh, int64_t bank_capacity) {
  if (!mesh) return 0;
  return imc_ws_layout(mesh, bank_capacity).total;
}

size_t imc_workspace_bytes_event(const imc_mesh* mesh, int64_t bank_capacity) {
  if (!mesh) return 0;
  return imc_ws_layout(mesh, bank_capacity).total + imc_event_scratch_bytes(bank_capacity);
}

int64_t imc_source_bound(const imc_mesh* mesh, const imc_step_params* par) {
  if (!mesh || !par) return 0;
  return source_bound(mesh, par);
}

const char* imc_status_str(imc_status s) {
  switch (s) {
    case IMC_OK: return "ok";
    case IMC_ERR_BANK_OVERFLOW: return "particle bank capacity exceeded";
    case IMC_ERR_EVENT_CAP: return "event safety cap reached";
    case IMC_ERR_NONFINITE: return "non-finite or non-positive material input";
    case IMC_ERR_BAD_GEOMETRY: return "bad geometry";
    case IMC_ERR_TIMEOUT: return "bounded device wait timed out";
    case IMC_ERR_CUDA: return "CUDA runtime error";
    case IMC_ERR_INVALID_ARG: return "invalid argument";
    case IMC_ERR_WORKSPACE: return "workspace too small";
    case IMC_ERR_BOUNDS: return "bounds check failed (an index or weight out of range)";
  }
  return "unknown status";
}

int imc_last_cuda_error(void) { return g_last_cuda; }
unsigned long long imc_kernel_launches(void) { return g_imc_launches; }

imc_status imc_phase_times(float* ms_sources, float* ms_transport) {
  PhaseEvents& pe = phase_events();
  if (!pe.ok || !pe.recorded || !ms_sources || !ms_transport) return IMC_ERR_INVALID_ARG;
  // waits for the tracking to end, not for the rest of the stream (the comb may still run)
  IMC_CUDA(cudaEventSynchronize(pe.e[2]));
  IMC_CUDA(cudaEventElapsedTime(ms_sources, pe.e[0], pe.e[1]));
  IMC_CUDA(cudaEventElapsedTime(ms_transport, pe.e[1], pe.e[2]));
  return IMC_OK;
}

imc_status imc_init_census(const imc_mesh* mesh, const double* tr, int64_t n_target, double t_emit_floor,
                           uint64_t seed, imc_bank* bank, void* workspace, size_t workspace_bytes,
                           int64_t* n_out, void* stream) {
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  const bool two_d = mesh->geometry >= IMC_GEOM_XY;
  if (!tr || !bank_ok(bank, two_d) || !workspace) return IMC_ERR_INVALID_ARG;
  const WsLayout L = imc_ws_layout(mesh, bank->capacity);
  if (workspace_bytes < L.total || ws_misaligned(workspace)) return IMC_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  const int nc = mesh->nx * mesh->ny;
  const long long bound = n_target + (long long)nc * (two_d ? 2 : 1);  // ceil (+1) and 2-D min 1 per cell
  if (bound > bank->capacity) { if (n_out) *n_out = bound; return IMC_ERR_BANK_OVERFLOW; }
  imc_step_summary* sum = internal_summary(workspace, L);
  IMC_CUDA(cudaMemsetAsync(sum, 0, sizeof(imc_step_summary), s));
  const bool mg1 = mg_sphere(mesh);
  if (mesh->n_groups > 1 && !mg1) {
    if (!bank->group) return IMC_ERR_INVALID_ARG;
    IcMgArgs im{};
    im.nc = nc; im.vol = mesh->volume; im.tr = tr; im.n_target = n_target; im.t_emit_floor = t_emit_floor;
    im.E = ws_ptr<double>(workspace, L.mg_ec); im.cdf = ws_ptr<double>(workspace, L.mg_cdf);
    im.mixcdf = ws_ptr<double>(workspace, L.mixcdf); im.sum = sum;
    IMC_CUDA(imc_launch_ic_plan_mg(im, s));
    FillMgArgs fm{};
    fm.geom = mesh->geometry; fm.nx = mesh->nx; fm.ny = mesh->ny; fm.nc = nc; fm.ng = mesh->n_groups;
    fm.e1 = mesh->edges1; fm.e2 = mesh->edges2; fm.cdf = im.cdf; fm.gcdf = nullptr; fm.tr = tr;
    fm.gedges = mesh->group_edges; fm.mixcdf = im.mixcdf;
    fm.d_n = &sum->n_emission; fm.d_base = &sum->base_emission; fm.n_bound = n_target;
    fm.time_scale = 0.0; fm.seed = seed; fm.step = 0; fm.tag = imcdev::TAG_IC;
    imcdev::philox_round_keys(fm.seed, fm.rk);
    fm.p1 = bank->pos1; fm.p2 = bank->pos2; fm.d1 = bank->dir1; fm.d2 = bank->dir2; fm.wb = bank->weight;
    fm.t = bank->time; fm.cell = bank->cell; fm.group = bank->group;
    IMC_CUDA(imc_launch_fill_mg(fm, s));
    long long n = 0;
    IMC_CUDA(cudaMemcpyAsync(&n, &sum->n_emission, sizeof(n), cudaMemcpyDeviceToHost, s));
    IMC_CUDA(cudaStreamSynchronize(s));
    bank->size = n;
    if (n_out) *n_out = n;
    return IMC_OK;
  }
  if (mg1) {
    if (!bank->group || !mesh->group_edges) return IMC_ERR_INVALID_ARG;
    // the Planck group sampler's mixture table (MG_IMC/MG_IMC1D.py:105-107)
    double mix[200];
    double tot = 0.0, run = 0.0;
    for (int n = 1; n <= 200; ++n) { const double d = (double)n; tot += 1.0 / (d * d * d * d); }
    for (int n = 1; n <= 200; ++n) { const double d = (double)n; run += 1.0 / (d * d * d * d); mix[n - 1] = run / tot; }
    IMC_CUDA(cudaMemcpyAsync(ws_ptr<double>(workspace, L.mixcdf), mix, sizeof(mix), cudaMemcpyHostToDevice, s));
    IMC_CUDA(cudaStreamSynchronize(s));  // mix is a stack array
  }
  IcArgs ia{};
  ia.geom = mesh->geometry; ia.nx = mesh->nx; ia.ny = mesh->ny; ia.nc = nc;
  ia.rule = mg1 ? 2 : (two_d ? 1 : 0);
  ia.e1 = mesh->edges1; ia.e2 = mesh->edges2; ia.vol = mesh->volume; ia.tr = tr;
  ia.n_target = n_target; ia.t_emit_floor = t_emit_floor;
  ia.n = ws_ptr<long long>(workspace, L.emit_n); ia.off = ws_ptr<long long>(workspace, L.emit_off);
  ia.w = ws_ptr<float>(workspace, L.emit_w); ia.E = ws_ptr<double>(workspace, L.emit_E);
  ia.sum = sum;
  IMC_CUDA(imc_launch_ic_plan(ia, s));
  FillArgs fa{};
  fa.geom = mesh->geometry; fa.nx = mesh->nx; fa.ny = mesh->ny; fa.nc = nc;
  fa.e1 = mesh->edges1; fa.e2 = mesh->edges2; fa.T = nullptr;
  fa.d_n = &sum->n_emission; fa.d_base = &sum->base_emission; fa.n_bound = bound;
  fa.off = ia.off; fa.w = ia.w; fa.tilt = nullptr; fa.tilt_kind = 0;
  fa.time_scale = 0.0; fa.seed = seed; fa.step = 0; fa.tag = imcdev::TAG_IC;
  imcdev::philox_round_keys(fa.seed, fa.rk);
  fa.nbins = nc; fa.bins_by_group = 0;
  if (mg1) {
    fa.tr = tr; fa.gedges = mesh->group_edges; fa.mixcdf = ws_ptr<double>(workspace, L.mixcdf);
    fa.ng = mesh->n_groups;
  }
  set_bank(fa.p2, fa.d2, bank, two_d);
  fa.p1 = bank->pos1; fa.d1 = bank->dir1;
  fa.wb = bank->weight; fa.t = bank->time; fa.cell = bank->cell; fa.group = bank->group;
  IMC_CUDA(imc_launch_fill_volume(fa, s));
  long long n = 0;
  IMC_CUDA(cudaMemcpyAsync(&n, &sum->n_emission, sizeof(n), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaStreamSynchronize(s));
  bank->size = n;
  if (n_out) *n_out = n;
  return IMC_OK;
}

imc_status imc_step_transport_async(const imc_mesh* mesh, const imc_material* mat, const imc_step_params* par,
                                    imc_bank* bank, imc_tallies* tal, void* workspace, size_t workspace_bytes,
                                    imc_step_summary* summary, void* stream) {
  return transport_async(mesh, mat, par, bank, tal, workspace, workspace_bytes, summary, (cudaStream_t)stream);
}

imc_status imc_step_transport(const imc_mesh* mesh, const imc_material* mat, const imc_step_params* par,
                              imc_bank* bank, imc_tallies* tal, void* workspace, size_t workspace_bytes,
                              imc_step_report* report, void* stream) {
  if (!report || !mesh || !par || !bank) return IMC_ERR_INVALID_ARG;
  std::memset(report, 0, sizeof(*report));
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  const WsLayout L = imc_ws_layout(mesh, bank->capacity);
  if (!workspace || workspace_bytes < L.total || ws_misaligned(workspace)) return IMC_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  report->required_capacity = bank->size + source_bound(mesh, par);
  imc_step_summary* sum = internal_summary(workspace, L);
  long long n_census = bank->size;
  IMC_CUDA(cudaMemcpyAsync(&sum->n_census, &n_census, sizeof(n_census), cudaMemcpyHostToDevice, s));
  st = transport_async(mesh, mat, par, bank, tal, workspace, workspace_bytes, sum, s);
  if (st != IMC_OK) return st;
  imc_step_summary h;
  IMC_CUDA(cudaMemcpyAsync(&h, sum, sizeof(h), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaStreamSynchronize(s));
  long long nb = 0;
  for (int q = 0; q < 4; ++q) { nb += h.n_side[q]; report->boundary_emission += h.e_side[q]; }
  report->n_boundary = nb; report->n_source = h.n_source; report->n_emission = h.n_emission;
  report->source_emission = h.source_emission; report->emission_total = h.emission_total;
  report->n_transported = h.n_bank;
  report->weight_floor = (mg_sphere(mesh) ? 1e-14 : 1e-10) * h.weight_sum / (double)std::max<long long>(h.n_bank, 1);
  imc_phase_times(&report->ms_sources, &report->ms_transport);
  bank->size = h.n_bank;
  if (h.flags & IMC_FLAG_BOUNDS) return IMC_ERR_BOUNDS;
  if (h.flags & IMC_FLAG_NONFINITE) return IMC_ERR_NONFINITE;
  if (h.flags & IMC_FLAG_EVENT_CAP) return IMC_ERR_EVENT_CAP;
  return IMC_OK;
}

imc_status imc_adjoint_vjp(const imc_mesh* mesh, const imc_material* mat, const imc_step_params* par,
                           imc_bank* bank, const double* cotangent, double* grad, imc_tallies* tal, void* workspace,
                           size_t workspace_bytes, void* stream) {
  if (!mesh || !par || !bank || !cotangent || !grad) return IMC_ERR_INVALID_ARG;
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  if ((mesh->geometry != IMC_GEOM_XY && mesh->geometry != IMC_GEOM_RZ) || mesh->n_groups != 1)
    return IMC_ERR_BAD_GEOMETRY;
  const WsLayout L = imc_ws_layout(mesh, bank->capacity);
  if (!workspace || workspace_bytes < L.total || ws_misaligned(workspace)) return IMC_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  imc_step_summary* sum = internal_summary(workspace, L);
  long long n_census = bank->size;
  IMC_CUDA(cudaMemcpyAsync(&sum->n_census, &n_census, sizeof(n_census), cudaMemcpyHostToDevice, s));
  AdjointArgs A{};
  A.cot = cotangent; A.grad = grad;
  st = transport_async(mesh, mat, par, bank, tal, workspace, workspace_bytes, sum, s, &A);
  if (st != IMC_OK) return st;
  int flags = 0;
  IMC_CUDA(cudaMemcpyAsync(&flags, &sum->flags, sizeof(int), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaStreamSynchronize(s));
  if (flags & IMC_FLAG_BOUNDS) return IMC_ERR_BOUNDS;
  if (flags & IMC_FLAG_NONFINITE) return IMC_ERR_NONFINITE;
  return IMC_OK;
}

imc_status imc_material_update(const imc_mesh* mesh, const imc_tallies* tal, double* e, double* tr, void* stream) {
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  if (!tal || !tal->dep || !tal->si || !tal->emitted || !e || !tr) return IMC_ERR_INVALID_ARG;
  MatArgs ma{};
  ma.nc = mesh->nx * mesh->ny; ma.ng = mesh->n_groups; ma.vol = mesh->volume;
  ma.dep = tal->dep; ma.si = tal->si; ma.emitted = tal->emitted; ma.e = e; ma.tr = tr;
  IMC_CUDA(imc_launch_material(ma, (cudaStream_t)stream));
  return IMC_OK;
}

imc_status imc_material_update_law(const imc_mesh* mesh, const imc_tallies* tal, const imc_material_law* law,
                                   double* e, double* tr, double* T, double* sigma_next, double* cv_next,
                                   void* stream) {
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  if (!tal || !tal->dep || !tal->si || !tal->emitted || !law || !e || !tr || !T || !sigma_next || !cv_next)
    return IMC_ERR_INVALID_ARG;
  if ((!law->cv_eos_array && !(law->cv_eos > 0.0)) || (!law->cv_array && !(law->cv > 0.0))) return IMC_ERR_INVALID_ARG;
  const int ng = std::max(1, mesh->n_groups);
  if (ng > 1 && !law->sigma_group && !law->sigma_array) return IMC_ERR_INVALID_ARG;  // one factor per group
  MatArgs ma{};
  ma.nc = mesh->nx * mesh->ny; ma.ng = ng; ma.vol = mesh->volume;
  ma.dep = tal->dep; ma.si = tal->si; ma.emitted = tal->emitted; ma.e = e; ma.tr = tr;
  IMC_CUDA(imc_launch_material_law(ma, *law, T, sigma_next, cv_next, (cudaStream_t)stream));
  return IMC_OK;
}

imc_status imc_comb_async(const imc_mesh* mesh, const imc_bank* in, imc_bank* out, int64_t n_max, uint64_t seed,
                          uint32_t step, int32_t per_group, double* disc, const double* e, void* workspace,
                          size_t workspace_bytes, imc_step_summary* summary, void* stream) {
  return comb_async(mesh, in, out, n_max, seed, step, per_group, disc, e, workspace, workspace_bytes, summary,
                    (cudaStream_t)stream);
}

imc_status imc_comb_async_dev(const imc_mesh* mesh, const imc_bank* in, imc_bank* out, int64_t n_max,
                              const int64_t* n_max_dev, uint64_t seed, const uint32_t* step_dev, int32_t per_group,
                              double* disc, const double* e, void* workspace, size_t workspace_bytes,
                              imc_step_summary* summary, void* stream) {
  if (!step_dev) return IMC_ERR_INVALID_ARG;
  return comb_async(mesh, in, out, n_max, seed, 0u, per_group, disc, e, workspace, workspace_bytes, summary,
                    (cudaStream_t)stream, step_dev, n_max_dev);
}

imc_status imc_mg_report_fields(const imc_mesh* mesh, const double* si, const double* after, const double* e,
                                const double* T, const double* Tr, const double* boundary_group,
                                const double* escaped_group, double* out, void* stream) {
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  if (mesh->n_groups < 2 || mesh->geometry < IMC_GEOM_XY) return IMC_ERR_INVALID_ARG;  // 2-D multigroup
  if (!out || !(si || after || e || T || Tr || boundary_group || escaped_group)) return IMC_ERR_INVALID_ARG;
  ReportArgs ra{};
  ra.nx = mesh->nx; ra.ny = mesh->ny; ra.ng = mesh->n_groups; ra.vol = mesh->volume;
  ra.si = si; ra.after = after; ra.e = e; ra.T = T; ra.Tr = Tr; ra.bnd = boundary_group; ra.esc = escaped_group;
  ra.out = out;
  // the post-comb section alone (the rest gathered by an earlier call) spans G nc entries
  const long long gnc = (long long)mesh->nx * mesh->ny * mesh->n_groups;
  const bool post_only = after && !si && !e && !T && !Tr && !boundary_group && !escaped_group;
  ra.q0 = post_only ? gnc : 0;
  ra.q1 = post_only ? 2 * gnc : 2 * gnc + 3LL * mesh->nx * mesh->ny + 2LL * mesh->n_groups;
  IMC_CUDA(imc_launch_mg_report(ra, (cudaStream_t)stream));
  return IMC_OK;
}

imc_status imc_bank_energy_by_bin(const imc_mesh* mesh, const imc_bank* bank, const int64_t* n_dev,
                                  int32_t per_group, double* out, void* stream) {
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  if (!bank || !bank->weight || !bank->cell || !n_dev || !out || bank->capacity < 0) return IMC_ERR_INVALID_ARG;
  if (per_group && !bank->group) return IMC_ERR_INVALID_ARG;
  const cudaStream_t s = (cudaStream_t)stream;
  const int nc = mesh->nx * mesh->ny;
  const int nb = per_group ? nc * std::max(1, mesh->n_groups) : nc;
  IMC_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * nb, s));
  CombArgs ca{};
  ca.nc = nc; ca.nb = nb; ca.per_group = per_group ? 1 : 0;
  ca.w = bank->weight; ca.cell = bank->cell; ca.group = bank->group;
  ca.d_n_in = n_dev; ca.n_bound = bank->capacity;
  ca.ecen = out;
  IMC_CUDA(imc_launch_comb_ecen(ca, s));
  return IMC_OK;
}

imc_status imc_comb(const imc_mesh* mesh, const imc_bank* in, imc_bank* out, int64_t n_max, uint64_t seed,
                    uint32_t step, int32_t per_group, double* disc, void* workspace, size_t workspace_bytes,
                    imc_comb_report* report, void* stream) {
  if (!report || !mesh || !in || !out) return IMC_ERR_INVALID_ARG;
  std::memset(report, 0, sizeof(*report));
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  const WsLayout L = imc_ws_layout(mesh, in->size);
  if (!workspace || workspace_bytes < L.total || ws_misaligned(workspace)) return IMC_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  report->n_in = in->size;
  imc_step_summary* sum = internal_summary(workspace, L);
  long long n_in = in->size;
  IMC_CUDA(cudaMemsetAsync(&sum->flags, 0, sizeof(int), s));
  IMC_CUDA(cudaMemcpyAsync(&sum->n_bank, &n_in, sizeof(n_in), cudaMemcpyHostToDevice, s));
  st = comb_async(mesh, in, out, n_max, seed, step, per_group, disc, nullptr, workspace, workspace_bytes, sum, s);
  if (st != IMC_OK) return st;
  imc_step_summary h;
  IMC_CUDA(cudaMemcpyAsync(&h, sum, sizeof(h), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaStreamSynchronize(s));
  report->required_capacity = h.n_out;
  report->energy_before = h.comb_before;
  report->energy_after = h.comb_after;
  if (h.flags & IMC_FLAG_BOUNDS) return IMC_ERR_BOUNDS;
  if (h.flags & IMC_FLAG_COMB_OVERFLOW) return IMC_ERR_BANK_OVERFLOW;
  out->size = h.n_out;
  report->n_out = h.n_out;
  return IMC_OK;
}

imc_status imc_comb_noalloc(const imc_mesh* mesh, const imc_bank* in, imc_bank* out, int64_t n_max,
                            uint64_t seed, uint32_t step, int32_t per_group, double* disc,
                            imc_comb_report* report, void* stream) {
  if (!report || !mesh || !in || !out) return IMC_ERR_INVALID_ARG;
  std::memset(report, 0, sizeof(*report));
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  if (in->size < 0) return IMC_ERR_INVALID_ARG;
  const WsLayout L = imc_ws_layout(mesh, in->size);
  if (L.total > IMC_NOALLOC_SCRATCH_BYTES) return IMC_ERR_WORKSPACE;
  void* scratch = nullptr;
  st = noalloc_scratch(&scratch);
  if (st != IMC_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  report->n_in = in->size;
  // The array outlives every call: clear the whole summary (flags, counters, energies) so
  // nothing from an earlier call is read.  The comb clears its own bin accumulators.
  imc_step_summary* sum = internal_summary(scratch, L);
  IMC_CUDA(cudaMemsetAsync(sum, 0, sizeof(*sum), s));
  long long n_in = in->size;
  IMC_CUDA(cudaMemcpyAsync(&sum->n_bank, &n_in, sizeof(n_in), cudaMemcpyHostToDevice, s));
  st = comb_async(mesh, in, out, n_max, seed, step, per_group, disc, nullptr, scratch, IMC_NOALLOC_SCRATCH_BYTES,
                  sum, s);
  if (st != IMC_OK) return st;
  imc_step_summary h;
  IMC_CUDA(cudaMemcpyAsync(&h, sum, sizeof(h), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaStreamSynchronize(s));
  report->required_capacity = h.n_out;
  report->energy_before = h.comb_before;
  report->energy_after = h.comb_after;
  if (h.flags & IMC_FLAG_BOUNDS) return IMC_ERR_BOUNDS;
  if (h.flags & IMC_FLAG_COMB_OVERFLOW) return IMC_ERR_BANK_OVERFLOW;
  out->size = h.n_out;
  report->n_out = h.n_out;
  return IMC_OK;
}

imc_status imc_energy_totals(const imc_mesh* mesh, const imc_bank* bank, const double* e, double* radiation,
                             double* internal, void* workspace, size_t workspace_bytes, void* stream) {
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  if (!bank || !bank->weight || !e || !radiation || !internal || !workspace) return IMC_ERR_INVALID_ARG;
  const WsLayout L = imc_ws_layout(mesh, 1);
  if (workspace_bytes < L.total || ws_misaligned(workspace)) return IMC_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  imc_step_summary* sum = internal_summary(workspace, L);
  long long n = bank->size;
  IMC_CUDA(cudaMemcpyAsync(&sum->n_bank, &n, sizeof(n), cudaMemcpyHostToDevice, s));
  IMC_CUDA(cudaMemsetAsync(&sum->weight_sum, 0, sizeof(double), s));
  IMC_CUDA(imc_launch_wsum(bank->weight, &sum->n_bank, std::max<long long>(n, 1), &sum->weight_sum, s));
  IMC_CUDA(imc_launch_canon_sum_eV(e, mesh->volume, mesh->nx * mesh->ny, &sum->internal_energy, s));
  double h[2];
  IMC_CUDA(cudaMemcpyAsync(&h[0], &sum->weight_sum, sizeof(double), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaMemcpyAsync(&h[1], &sum->internal_energy, sizeof(double), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaStreamSynchronize(s));
  *radiation = h[0];
  *internal = h[1];
  return IMC_OK;
}

imc_status imc_philox(const uint32_t* ctr, uint32_t key0, uint32_t key1, uint32_t* out, int64_t n, void* stream) {
  if (!ctr || !out || n < 0) return IMC_ERR_INVALID_ARG;
  IMC_CUDA(imc_launch_philox(ctr, key0, key1, out, n, (cudaStream_t)stream));
  return IMC_OK;
}

}  // extern "C"

namespace {
__global__ void k_philox(const uint32_t* ctr, uint32_t k0, uint32_t k1, uint32_t* out, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const imcdev::U4 c{ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3]};
  const imcdev::U4 r = imcdev::philox4x32_10(c, k0, k1);
  out[4 * i] = r.x; out[4 * i + 1] = r.y; out[4 * i + 2] = r.z; out[4 * i + 3] = r.w;
}
}  // namespace

cudaError_t imc_launch_philox(const uint32_t* ctr, uint32_t k0, uint32_t k1, uint32_t* out, long long n,
                              cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  ++g_imc_launches;
  k_philox<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(ctr, k0, k1, out, n);
  return cudaGetLastError();
}
