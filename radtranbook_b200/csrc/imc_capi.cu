// imc_capi.cu — the extern "C" entry points of libimcb200.so (declared in
// include/imcb200.h): argument checks, workspace carving, phase ordering on the caller's
// stream, and the few small device->host copies that return sizes and totals.
#include <algorithm>
#include <cstring>
#include "imc_device.cuh"
#include "imc_internal.h"

unsigned long long g_imc_launches = 0;

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

// one pair of timing events per host thread (created on first use, never destroyed)
struct PhaseEvents {
  cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
  bool ok = false;
  PhaseEvents() {
    ok = true;
    for (auto& x : e) ok = ok && cudaEventCreate(&x) == cudaSuccess;
  }
};
PhaseEvents& phase_events() {
  static thread_local PhaseEvents pe;
  return pe;
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
  if (m->n_groups != 1) return IMC_ERR_INVALID_ARG;  // multigroup tracking: not in this build
  return IMC_OK;
}

bool bank_ok(const imc_bank* b, bool two_d) {
  if (!b || !b->pos1 || !b->dir1 || !b->weight || !b->time || !b->cell) return false;
  if (two_d && (!b->pos2 || !b->dir2)) return false;
  return b->size >= 0 && b->capacity >= b->size;
}

}  // namespace

WsLayout imc_ws_layout(const imc_mesh* m, int64_t capacity) {
  WsLayout L{};
  size_t o = 0;
  const size_t nx = (size_t)m->nx, ny = (size_t)m->ny, nc = nx * ny;
  const size_t ng = (size_t)std::max(1, m->n_groups), ncg = nc * ng;
  const size_t nf = std::max(nx, ny);
  const size_t cap = (size_t)std::max<int64_t>(capacity, 1);
  auto take = [&](size_t bytes) { const size_t r = o; o += al256(bytes); return r; };
  L.e1f = take(4 * (nx + 1)); L.e2f = take(4 * (ny + 1));
  L.saf = take(4 * ncg); L.ssf = take(4 * ncg);
  L.emit_E = take(8 * ncg); L.emit_n = take(8 * nc); L.emit_off = take(8 * (nc + 1)); L.emit_w = take(4 * nc);
  L.tilt = take(8 * 4 * nc);
  L.src_n = take(8 * nc); L.src_off = take(8 * (nc + 1)); L.src_w = take(4 * nc);
  L.src_QV = take(8 * nc); L.src_issued = take(8 * nc);
  L.face = take(8 * 4 * 2 * nf);
  L.plan = take(sizeof(PlanDev)); L.queue = take(8); L.err = take(8); L.wsum = take(8 * 4);
  L.ecen = take(8 * ncg); L.ew = take(8 * ncg); L.ncopy = take(8 * ncg);
  L.cnt = take(4 * cap); L.blk = take(8 * ((cap + 1023) / 1024 + 2));
  L.total = o;
  return L;
}

extern "C" {

size_t imc_workspace_bytes(const imc_mesh* mesh, int64_t bank_capacity) {
  if (!mesh) return 0;
  return imc_ws_layout(mesh, bank_capacity).total;
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
  }
  return "unknown status";
}

int imc_last_cuda_error(void) { return g_last_cuda; }
unsigned long long imc_kernel_launches(void) { return g_imc_launches; }

imc_status imc_init_census(const imc_mesh* mesh, const double* tr, int64_t n_target,
                           double t_emit_floor, uint64_t seed, imc_bank* bank, void* workspace,
                           size_t workspace_bytes, int64_t* n_out, void* stream) {
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  const bool two_d = mesh->geometry >= IMC_GEOM_XY;
  if (!tr || !bank_ok(bank, two_d) || !workspace) return IMC_ERR_INVALID_ARG;
  const WsLayout L = imc_ws_layout(mesh, bank->capacity);
  if (workspace_bytes < L.total) return IMC_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  const int nc = mesh->nx * mesh->ny;
  IcArgs ia{};
  ia.geom = mesh->geometry; ia.nx = mesh->nx; ia.ny = mesh->ny; ia.nc = nc;
  ia.e1 = mesh->edges1; ia.e2 = mesh->edges2; ia.vol = mesh->volume; ia.tr = tr;
  ia.n_target = n_target; ia.t_emit_floor = t_emit_floor;
  ia.n = ws_ptr<long long>(workspace, L.emit_n); ia.off = ws_ptr<long long>(workspace, L.emit_off);
  ia.w = ws_ptr<float>(workspace, L.emit_w); ia.E = ws_ptr<double>(workspace, L.emit_E);
  ia.plan = ws_ptr<PlanDev>(workspace, L.plan);
  IMC_CUDA(imc_launch_ic_plan(ia, s));
  PlanDev hp{};
  IMC_CUDA(cudaMemcpyAsync(&hp, ia.plan, sizeof(PlanDev), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaStreamSynchronize(s));
  if (hp.n_emit > bank->capacity) { if (n_out) *n_out = hp.n_emit; return IMC_ERR_BANK_OVERFLOW; }
  FillArgs fa{};
  fa.geom = mesh->geometry; fa.nx = mesh->nx; fa.ny = mesh->ny; fa.nc = nc;
  fa.e1 = mesh->edges1; fa.e2 = mesh->edges2; fa.T = nullptr;
  fa.n = hp.n_emit; fa.base = 0; fa.off = ia.off; fa.w = ia.w; fa.tilt = nullptr; fa.tilt_kind = 0;
  fa.dt = 0.0; fa.time_scale = 0.0; fa.seed = seed; fa.step = 0; fa.tag = imcdev::TAG_IC;
  fa.p1 = bank->pos1; fa.p2 = two_d ? bank->pos2 : bank->pos1; fa.d1 = bank->dir1;
  fa.d2 = two_d ? bank->dir2 : bank->dir1;
  fa.wb = bank->weight; fa.t = bank->time; fa.cell = bank->cell; fa.group = bank->group;
  if (!two_d) { fa.p2 = nullptr; fa.d2 = nullptr; }
  IMC_CUDA(imc_launch_fill_volume(fa, s));
  bank->size = hp.n_emit;
  if (n_out) *n_out = hp.n_emit;
  return IMC_OK;
}

imc_status imc_step_transport(const imc_mesh* mesh, const imc_material* mat,
                              const imc_step_params* par, imc_bank* bank, imc_tallies* tal,
                              void* workspace, size_t workspace_bytes, imc_step_report* report,
                              void* stream) {
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  const bool two_d = mesh->geometry >= IMC_GEOM_XY;
  if (!mat || !mat->temperature || !mat->sigma || !mat->cv || !par || !tal || !report) return IMC_ERR_INVALID_ARG;
  if (!tal->dep || !tal->si || !tal->emitted || !tal->sigma_a || !tal->sigma_s || !tal->escaped || !tal->stats) return IMC_ERR_INVALID_ARG;
  if (!bank_ok(bank, two_d) || !workspace) return IMC_ERR_INVALID_ARG;
  if (!(par->dt > 0.0)) return IMC_ERR_INVALID_ARG;
  const WsLayout L = imc_ws_layout(mesh, bank->capacity);
  if (workspace_bytes < L.total) return IMC_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  const int nc = mesh->nx * mesh->ny;
  std::memset(report, 0, sizeof(*report));

  int* err = ws_ptr<int>(workspace, L.err);
  PlanDev* plan = ws_ptr<PlanDev>(workspace, L.plan);
  IMC_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));

  // ---- plan: Fleck, per-cell source counts / weights / offsets, boundary faces ----
  PlanArgs pa{};
  pa.geom = mesh->geometry; pa.nx = mesh->nx; pa.ny = mesh->ny; pa.nc = nc; pa.ng = 1;
  pa.e1 = mesh->edges1; pa.e2 = mesh->edges2; pa.vol = mesh->volume;
  pa.T = mat->temperature; pa.sigma = mat->sigma; pa.cv = mat->cv; pa.source = mat->source;
  pa.dt = par->dt; pa.theta = par->theta;
  pa.n_target = par->n_target; pa.n_source = par->n_source; pa.n_boundary = par->n_boundary;
  for (int q = 0; q < 4; ++q) pa.face_T[q] = par->face_T[q];
  pa.rz_linear = par->rz_linear_source; pa.t_emit_floor = par->t_emit_floor;
  pa.sa = tal->sigma_a; pa.ss = tal->sigma_s;
  pa.saf = ws_ptr<float>(workspace, L.saf); pa.ssf = ws_ptr<float>(workspace, L.ssf);
  pa.e1f = ws_ptr<float>(workspace, L.e1f); pa.e2f = ws_ptr<float>(workspace, L.e2f);
  pa.emit_E = ws_ptr<double>(workspace, L.emit_E); pa.emit_n = ws_ptr<long long>(workspace, L.emit_n);
  pa.emit_off = ws_ptr<long long>(workspace, L.emit_off); pa.emit_w = ws_ptr<float>(workspace, L.emit_w);
  pa.tilt = ws_ptr<double>(workspace, L.tilt);
  pa.src_n = ws_ptr<long long>(workspace, L.src_n); pa.src_off = ws_ptr<long long>(workspace, L.src_off);
  pa.src_w = ws_ptr<float>(workspace, L.src_w); pa.src_QV = ws_ptr<double>(workspace, L.src_QV);
  pa.src_issued = ws_ptr<double>(workspace, L.src_issued);
  pa.emitted = tal->emitted;
  pa.face = ws_ptr<double>(workspace, L.face); pa.nf = std::max(mesh->nx, mesh->ny);
  pa.plan = plan; pa.err = err;
  IMC_CUDA(imc_launch_plan(pa, s));
  PlanDev hp{};
  int herr = 0;
  IMC_CUDA(cudaMemcpyAsync(&hp, plan, sizeof(PlanDev), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaStreamSynchronize(s));
  if (herr & 2) return IMC_ERR_NONFINITE;

  long long n_bnd = 0;
  double e_bnd = 0.0;
  for (int q = 0; q < 4; ++q) { n_bnd += hp.n_bnd[q]; e_bnd += hp.e_bnd[q]; }
  const long long n_new = n_bnd + hp.n_src + hp.n_emit;
  report->n_boundary = n_bnd; report->n_source = hp.n_src; report->n_emission = hp.n_emit;
  report->boundary_emission = e_bnd; report->source_emission = hp.e_src; report->emission_total = hp.e_emit;
  report->required_capacity = bank->size + n_new;
  if (bank->size + n_new > bank->capacity) return IMC_ERR_BANK_OVERFLOW;

  // ---- sources, appended in the reference's order: census | boundary | fixed | emission ----
  PhaseEvents& pe = phase_events();
  if (pe.ok) IMC_CUDA(cudaEventRecord(pe.e[0], s));
  long long base = bank->size;
  float* p2 = two_d ? bank->pos2 : nullptr;
  float* d2 = two_d ? bank->dir2 : nullptr;
  for (int side = 0; side < 4; ++side) {
    if (hp.n_bnd[side] <= 0) continue;
    BndArgs ba{};
    ba.geom = mesh->geometry; ba.nx = mesh->nx; ba.ny = mesh->ny; ba.side = side; ba.nf = pa.nf;
    ba.e1 = mesh->edges1; ba.e2 = mesh->edges2;
    ba.face = pa.face + (size_t)side * 2 * pa.nf;
    ba.n = hp.n_bnd[side]; ba.base = base; ba.dt = par->dt; ba.seed = par->seed; ba.step = par->step;
    ba.p1 = bank->pos1; ba.p2 = p2; ba.d1 = bank->dir1; ba.d2 = d2; ba.wb = bank->weight;
    ba.t = bank->time; ba.cell = bank->cell; ba.group = bank->group;
    IMC_CUDA(imc_launch_fill_boundary(ba, s));
    base += ba.n;
  }
  auto fill = [&](long long n, const long long* off, const float* w, const double* tilt, int kind,
                  uint32_t tag) -> imc_status {
    FillArgs fa{};
    fa.geom = mesh->geometry; fa.nx = mesh->nx; fa.ny = mesh->ny; fa.nc = nc;
    fa.e1 = mesh->edges1; fa.e2 = mesh->edges2; fa.T = mat->temperature;
    fa.n = n; fa.base = base; fa.off = off; fa.w = w; fa.tilt = tilt; fa.tilt_kind = kind;
    fa.dt = par->dt; fa.time_scale = par->dt; fa.seed = par->seed; fa.step = par->step; fa.tag = tag;
    fa.p1 = bank->pos1; fa.p2 = p2; fa.d1 = bank->dir1; fa.d2 = d2; fa.wb = bank->weight;
    fa.t = bank->time; fa.cell = bank->cell; fa.group = bank->group;
    IMC_CUDA(imc_launch_fill_volume(fa, s));
    base += n;
    return IMC_OK;
  };
  const bool rzlin = mesh->geometry == IMC_GEOM_RZ && par->rz_linear_source;
  st = fill(hp.n_src, pa.src_off, pa.src_w, rzlin ? pa.tilt : nullptr, rzlin ? 3 : 0, imcdev::TAG_SOURCE);
  if (st != IMC_OK) return st;
  int ekind = 0;
  if (mesh->geometry == IMC_GEOM_SLAB) ekind = 1;
  else if (mesh->geometry == IMC_GEOM_SPHERE) ekind = 2;
  else if (rzlin) ekind = 3;
  st = fill(hp.n_emit, pa.emit_off, pa.emit_w, ekind ? pa.tilt : nullptr, ekind, imcdev::TAG_EMISSION);
  if (st != IMC_OK) return st;
  bank->size = base;

  // ---- tracking ----
  if (pe.ok) IMC_CUDA(cudaEventRecord(pe.e[1], s));
  const int ng = 1;
  IMC_CUDA(cudaMemsetAsync(tal->dep, 0, sizeof(double) * nc * ng, s));
  IMC_CUDA(cudaMemsetAsync(tal->si, 0, sizeof(double) * nc * ng, s));
  IMC_CUDA(cudaMemsetAsync(tal->escaped, 0, sizeof(double) * (4 + ng), s));
  IMC_CUDA(cudaMemsetAsync(tal->stats, 0, sizeof(unsigned long long) * IMC_STAT_N, s));
  unsigned long long* queue = ws_ptr<unsigned long long>(workspace, L.queue);
  double* wsum = ws_ptr<double>(workspace, L.wsum);
  IMC_CUDA(cudaMemsetAsync(queue, 0, 8, s));
  IMC_CUDA(cudaMemsetAsync(wsum, 0, 8 * 4, s));
  IMC_CUDA(imc_launch_wsum(bank->weight, bank->size, wsum, s));

  TrackArgs ta{};
  ta.nx = mesh->nx; ta.ny = mesh->ny; ta.nc = nc; ta.ng = ng;
  ta.e1 = pa.e1f; ta.e2 = pa.e2f; ta.sa = pa.saf; ta.ss = pa.ssf; ta.vol = mesh->volume;
  ta.dep = tal->dep; ta.si = tal->si; ta.escaped = tal->escaped; ta.stats = tal->stats;
  ta.p1 = bank->pos1; ta.p2 = p2; ta.d1 = bank->dir1; ta.d2 = d2; ta.w = bank->weight; ta.t = bank->time;
  ta.cell = bank->cell; ta.group = bank->group;
  ta.n = bank->size; ta.queue = queue; ta.err = err;
  ta.dt = (float)par->dt; ta.dt_d = par->dt;
  ta.wsum = wsum;
  int rm = 0;
  for (int q = 0; q < 4; ++q) if (par->reflect[q]) rm |= 1 << q;
  ta.reflect_mask = rm;
  ta.max_events = par->max_events > 0 ? par->max_events : (long long)1 << 30;
  ta.cap_is_reference = par->max_events > 0 ? 1 : 0;
  ta.seed = par->seed; ta.step = par->step;
  ta.chunk = par->chunk > 0 ? par->chunk : 64;
  ta.group_edges = mesh->group_edges;
  const int block = par->block_size > 0 ? par->block_size : 256;
  const int bps = par->blocks_per_sm > 0 ? par->blocks_per_sm : 4;
  const int grid = sm_count() * bps;
  if (bank->size > 0) {
    ++g_imc_launches;
    IMC_CUDA(imc_launch_track(ta, mesh->geometry, block, grid, s));
  }
  if (pe.ok) IMC_CUDA(cudaEventRecord(pe.e[2], s));
  double hw = 0.0;
  IMC_CUDA(cudaMemcpyAsync(&hw, wsum, sizeof(double), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaStreamSynchronize(s));
  report->n_transported = bank->size;
  if (pe.ok) {
    cudaEventElapsedTime(&report->ms_sources, pe.e[0], pe.e[1]);
    cudaEventElapsedTime(&report->ms_transport, pe.e[1], pe.e[2]);
  }
  report->weight_floor = 1e-10 * hw / (double)std::max<long long>(bank->size, 1);
  if (herr & 1) return IMC_ERR_EVENT_CAP;
  return IMC_OK;
}

imc_status imc_material_update(const imc_mesh* mesh, const imc_tallies* tal, double* e, double* tr,
                               void* stream) {
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  if (!tal || !tal->dep || !tal->si || !tal->emitted || !e || !tr) return IMC_ERR_INVALID_ARG;
  MatArgs ma{};
  ma.nc = mesh->nx * mesh->ny; ma.ng = 1; ma.vol = mesh->volume;
  ma.dep = tal->dep; ma.si = tal->si; ma.emitted = tal->emitted; ma.e = e; ma.tr = tr;
  IMC_CUDA(imc_launch_material(ma, (cudaStream_t)stream));
  return IMC_OK;
}

imc_status imc_comb(const imc_mesh* mesh, const imc_bank* in, imc_bank* out, int64_t n_max,
                    uint64_t seed, uint32_t step, int32_t per_group, double* disc, void* workspace,
                    size_t workspace_bytes, imc_comb_report* report, void* stream) {
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  const bool two_d = mesh->geometry >= IMC_GEOM_XY;
  if (!bank_ok(in, two_d) || !bank_ok(out, two_d) || !disc || !workspace || !report) return IMC_ERR_INVALID_ARG;
  if (in->pos1 == out->pos1 || in->weight == out->weight) return IMC_ERR_INVALID_ARG;
  if (per_group && (!in->group || !out->group)) return IMC_ERR_INVALID_ARG;
  const WsLayout L = imc_ws_layout(mesh, in->size);
  if (workspace_bytes < L.total) return IMC_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  const int nc = mesh->nx * mesh->ny;
  const int nb = per_group ? nc * mesh->n_groups : nc;
  std::memset(report, 0, sizeof(*report));
  report->n_in = in->size;

  CombArgs ca{};
  ca.nc = nc; ca.nb = nb; ca.per_group = per_group; ca.n_in = in->size;
  ca.w = in->weight; ca.cell = in->cell; ca.group = in->group;
  ca.p1 = in->pos1; ca.p2 = two_d ? in->pos2 : nullptr; ca.d1 = in->dir1; ca.d2 = two_d ? in->dir2 : nullptr;
  ca.ecen = ws_ptr<double>(workspace, L.ecen); ca.ew = ws_ptr<double>(workspace, L.ew);
  ca.ncopy = ws_ptr<long long>(workspace, L.ncopy); ca.cnt = ws_ptr<int>(workspace, L.cnt);
  ca.blk = ws_ptr<long long>(workspace, L.blk);
  ca.seed = seed; ca.step = step;
  ca.op1 = out->pos1; ca.op2 = two_d ? out->pos2 : nullptr; ca.od1 = out->dir1; ca.od2 = two_d ? out->dir2 : nullptr;
  ca.ow = out->weight; ca.ot = out->time; ca.ocell = out->cell; ca.ogroup = out->group;
  ca.disc = disc;
  ca.plan = ws_ptr<PlanDev>(workspace, L.plan);

  IMC_CUDA(cudaMemsetAsync(ca.ecen, 0, sizeof(double) * nb, s));
  IMC_CUDA(cudaMemsetAsync(ca.ncopy, 0, sizeof(long long) * nb, s));
  IMC_CUDA(cudaMemsetAsync(ca.plan, 0, sizeof(PlanDev), s));
  IMC_CUDA(imc_launch_comb_ecen(ca, s));
  CombPlanArgs cp{};
  cp.nb = nb; cp.n_max = n_max; cp.ecen = ca.ecen; cp.ew = ca.ew; cp.plan = ca.plan;
  IMC_CUDA(imc_launch_comb_plan(cp, s));
  IMC_CUDA(imc_launch_comb_count(ca, s));
  PlanDev hp{};
  IMC_CUDA(cudaMemcpyAsync(&hp, ca.plan, sizeof(PlanDev), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaStreamSynchronize(s));
  report->required_capacity = hp.comb_total;
  report->energy_before = hp.comb_e_before;
  if (hp.comb_total > out->capacity) return IMC_ERR_BANK_OVERFLOW;
  IMC_CUDA(imc_launch_comb_scatter(ca, s));
  IMC_CUDA(cudaMemcpyAsync(&hp, ca.plan, sizeof(PlanDev), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaStreamSynchronize(s));
  out->size = hp.comb_total;
  report->n_out = hp.comb_total;
  report->energy_after = hp.comb_e_after;
  return IMC_OK;
}

imc_status imc_energy_totals(const imc_mesh* mesh, const imc_bank* bank, const double* e,
                             double* radiation, double* internal, void* workspace,
                             size_t workspace_bytes, void* stream) {
  imc_status st = check_mesh(mesh);
  if (st != IMC_OK) return st;
  if (!bank || !bank->weight || !e || !radiation || !internal || !workspace) return IMC_ERR_INVALID_ARG;
  const WsLayout L = imc_ws_layout(mesh, 1);
  if (workspace_bytes < L.total) return IMC_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  double* wsum = ws_ptr<double>(workspace, L.wsum);
  IMC_CUDA(cudaMemsetAsync(wsum, 0, 8 * 4, s));
  IMC_CUDA(imc_launch_wsum(bank->weight, bank->size, wsum, s));
  IMC_CUDA(imc_launch_canon_sum_eV(e, mesh->volume, mesh->nx * mesh->ny, wsum + 1, s));
  double h[2];
  IMC_CUDA(cudaMemcpyAsync(h, wsum, sizeof(h), cudaMemcpyDeviceToHost, s));
  IMC_CUDA(cudaStreamSynchronize(s));
  *radiation = h[0];
  *internal = h[1];
  return IMC_OK;
}

imc_status imc_philox(const uint32_t* ctr, uint32_t key0, uint32_t key1, uint32_t* out, int64_t n,
                      void* stream) {
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
