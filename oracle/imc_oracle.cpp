/*
 * ORACLE — test infrastructure only.  Never linked into, or called by, the product
 * (radtranbook_b200).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it, as the checker / CPU baseline.
 *
 * An FP64, history-based CPU restatement of the reference implicit Monte Carlo
 * (Fleck-Cummings) time step of DrRyanMc/RadTranBook:
 *   gray 1-D slab    IMC/IMC1D.py:75-130 (move_particle), 133-200 (move_particles),
 *                    203-291 (emission + linear-T tilt), 220-248 (IC), 294-316 (fixed
 *                    source), 319-329 (boundary), 770-828 (comb), 908-1124 (step)
 *   gray 1-D sphere  IMC/IMC1D.py:336-436, 439-532, 535-763
 *   gray 2-D xy/rz   IMC/IMC2D.py:157-489 (boundary), 711-935 (events), 938-1107
 *                    (history loop), 1110-1445 (IC / sources), 1448-1511 (comb),
 *                    1591-1897 (step)
 *   multigroup xy/rz MG_IMC/MG_IMC2D.py:202-254 (Planck sampler), 580-771 (events),
 *                    774-989 (history loop), 1237-1267 (emission groups),
 *                    1270-1378 (comb), 1635-2122 (step)
 *   multigroup 1-D sphere  MG_IMC/MG_IMC1D.py:276-461 (events, history loop), 514-743
 *                    (IC and sources), 746-847 (comb), 917-1140 (step)
 * It differs from the reference in exactly one way on purpose: random numbers come
 * from Philox-4x32-10 streams keyed by (seed) with counter (index, block, step, tag),
 * the same streams the CUDA path draws, so the two can be compared history by history.
 * The uniforms are 24-bit values exactly representable in FP32 and FP64.
 * Everything else (geometry, estimators, caps, ordering of the census bank, comb) is
 * the reference's algorithm; the few deliberate reference-quirk decisions are noted
 * where they occur.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "philox_ref.h"

using oracle::draw;
using oracle::Draw4;

namespace {

constexpr double C_LIGHT = 29.98;   /* cm/ns        IMC/IMC1D.py:68 */
constexpr double A_RAD = 0.01372;   /* GJ/cm^3/keV^4 IMC/IMC1D.py:69 */
constexpr double PI = 3.14159265358979323846;
constexpr double BIG = 1e30;

enum { G_SLAB = 0, G_SPHERE = 1, G_XY = 2, G_RZ = 3 };
enum { EV_CENSUS = 0, EV_BOUNDARY = 1, EV_SCATTER = 2 };
/* face crossed: 0 none, 1 +dir1, 2 -dir1, 3 +dir2, 4 -dir2 */
enum { X_NONE = 0, X_IP = 1, X_IM = 2, X_JP = 3, X_JM = 4 };
/* unified statistics layout */
enum { S_EVENTS = 0, S_BOUNDARY, S_SCATTER, S_CENSUS, S_CAPTURE, S_FLOOR, S_REFLECT, S_CAP, S_ESCAPE, S_N };

struct EventOut {
  double w, d1, d2, p1, p2, dep, dep_i, dcen;
  double s;  /* path length of the event */
  int cross, evt;
};

/* ---- effective-scatter distance with the reference's optically-thick cap ----
 * IMC/IMC1D.py:83-88, IMC/IMC2D.py:758-765: a sigma_s*L > 1e4 cell uses sigma = 1e4/L.
 * The capped distance reuses the same uniform (the reference draws a fresh one; the
 * distribution is identical). */
inline double scatter_distance(double ss, double L, double u, double thresh, bool cap = true) {
  if (cap && ss * L > 10000.0) return -std::log(u) / (10000.0 / L);
  if (ss > thresh) return -std::log(u) / ss;
  return BIG;
}

/* ---- 1-D slab event: IMC/IMC1D.py:75-130 ---- */
EventOut event_slab(double w, double mu, double x, double xl, double xr, double sa, double ss,
                    double dcen, double u0, double u1) {
  EventOut o{};
  const double dx = xr - xl;
  double db = (mu > 0) ? (xr - x) / mu : (xl - x) / mu;
  if (db < 0) db = 0;
  const double ds = scatter_distance(ss, dx, u0, 1e-10);
  double d = db;
  int evt = EV_BOUNDARY;
  if (ds < d) { d = ds; evt = EV_SCATTER; }
  if (dcen < d) { d = dcen; evt = EV_CENSUS; }
  double xn = x + mu * d, mun = mu;
  int cross = X_NONE;
  if (evt == EV_BOUNDARY) {
    if (mu > 0) { xn = xr; cross = X_IP; } else { xn = xl; cross = X_IM; }
  } else if (evt == EV_SCATTER) {
    mun = 2.0 * u1 - 1.0;
  }
  xn = std::min(std::max(xn, xl), xr);
  const double wf = std::exp(-sa * d);
  const double wn = w * wf;
  const double lost = w - wn;
  o.dep = lost / dx;
  o.dep_i = (sa > 1e-10) ? lost / sa / dx : w * d / dx;
  o.w = wn; o.d1 = mun; o.p1 = xn; o.dcen = dcen - d; o.cross = cross; o.evt = evt;
  return o;
}

/* ---- 1-D spherical event: IMC/IMC1D.py:336-436 (stable root forms) ---- */
EventOut event_sphere(double w, double mu, double r, double r0, double r1, double sa, double ss,
                      double dcen, double u0, double u1) {
  EventOut o{};
  const double b2 = r * r * (1.0 - mu * mu);
  double q = std::sqrt(std::max(r1 * r1 - b2, 0.0));
  double d_out = (mu >= 0) ? (r1 - r) * (r1 + r) / std::max(q + r * mu, 1e-300) : q - r * mu;
  if (d_out < 0) d_out = 0;
  double d_in = BIG;
  if (mu < 0 && r0 > 0) {
    const double disc = r0 * r0 - b2;
    if (disc > 0) {
      d_in = (r - r0) * (r + r0) / (std::sqrt(disc) - r * mu);
      if (d_in < 0) d_in = 0;
    }
  }
  const bool hit_outer = d_out <= d_in;
  const double db = hit_outer ? d_out : d_in;
  const double ds = scatter_distance(ss, r1 - r0, u0, 1e-10);
  double d = db;
  int evt = EV_BOUNDARY;
  if (ds < d) { d = ds; evt = EV_SCATTER; }
  if (dcen < d) { d = dcen; evt = EV_CENSUS; }
  const double rn2 = r * r + 2.0 * r * d * mu + d * d;
  double rn = rn2 > 0 ? std::sqrt(rn2) : 0.0;
  double mun = rn > 1e-15 ? (r * mu + d) / rn : 1.0;
  int cross = X_NONE;
  if (evt == EV_BOUNDARY) {
    if (hit_outer) { rn = r1; mun = r1 > 1e-15 ? (r * mu + d) / r1 : 1.0; cross = X_IP; }
    else { rn = r0; mun = r0 > 1e-15 ? (r * mu + d) / r0 : -1.0; cross = X_IM; }
  } else if (evt == EV_SCATTER) {
    mun = 2.0 * u1 - 1.0;
  }
  mun = std::min(1.0, std::max(-1.0, mun));
  rn = std::min(std::max(rn, r0), r1);
  const double vol = (4.0 / 3.0) * PI * (r1 * r1 * r1 - r0 * r0 * r0);
  const double wn = w * std::exp(-sa * d);
  const double lost = w - wn;
  o.dep = lost / vol;
  o.dep_i = (sa > 1e-10) ? lost / sa / vol : w * d / vol;
  o.w = wn; o.d1 = mun; o.p1 = rn; o.dcen = dcen - d; o.cross = cross; o.evt = evt;
  return o;
}

/* ---- 2-D Cartesian event: IMC/IMC2D.py:739-823 ---- */
EventOut event_xy(double w, double ux, double uy, double x, double y, double xl, double xr,
                  double yl, double yr, double sa, double ss, double dcen, double u0, double u1,
                  double u2, bool cap = true) {
  EventOut o{};
  double sx = BIG, sy = BIG;
  if (ux > 0) sx = (xr - x) / ux; else if (ux < 0) sx = (xl - x) / ux;
  if (uy > 0) sy = (yr - y) / uy; else if (uy < 0) sy = (yl - y) / uy;
  if (sx < 0) sx = 0;
  if (sy < 0) sy = 0;
  const double ds = scatter_distance(ss, std::min(xr - xl, yr - yl), u0, 1e-12, cap);
  const double sb = sx < sy ? sx : sy;
  double s = sb;
  int evt = EV_BOUNDARY;
  if (ds < s) { s = ds; evt = EV_SCATTER; }
  if (dcen < s) { s = dcen; evt = EV_CENSUS; }
  double xn = x + ux * s, yn = y + uy * s, uxn = ux, uyn = uy;
  int cross = X_NONE;
  if (evt == EV_BOUNDARY) {
    if (sx <= sy) { if (ux > 0) { xn = xr; cross = X_IP; } else { xn = xl; cross = X_IM; } }
    else { if (uy > 0) { yn = yr; cross = X_JP; } else { yn = yl; cross = X_JM; } }
  } else if (evt == EV_SCATTER) {
    /* IMC/IMC2D.py:695-701: 3-D isotropic, u_z dropped */
    const double uz = 2.0 * u1 - 1.0, phi = 2.0 * PI * u2;
    const double rxy = std::sqrt(std::max(0.0, 1.0 - uz * uz));
    uxn = rxy * std::cos(phi); uyn = rxy * std::sin(phi);
  }
  const double wn = w * std::exp(-sa * s);
  const double lost = w - wn;
  o.dep = lost;
  o.dep_i = (sa > 1e-12) ? lost / sa : w * s;
  o.w = wn; o.d1 = uxn; o.d2 = uyn; o.p1 = xn; o.p2 = yn; o.dcen = dcen - s; o.s = s;
  o.cross = cross; o.evt = evt;
  return o;
}

/* ---- cylinder distances, IMC/IMC2D.py:711-736, written with the cancellation-free
 * root forms.  l^2 + 2 r mu l + (r^2 - R^2) = 0, path length s = l / sqrt(1-eta^2). ---- */
inline double rz_outer_l(double r, double mu, double R, double b2) {
  const double q = std::sqrt(std::max(R * R - b2, 0.0));
  double l = (mu >= 0) ? (R - r) * (R + r) / std::max(q + r * mu, 1e-300) : q - r * mu;
  return l < 0 ? 0 : l;
}
inline double rz_inner_l(double r, double mu, double R, double b2) {
  if (!(R > 0) || !(mu < 0)) return BIG;
  const double disc = R * R - b2;
  if (!(disc > 0)) return BIG;
  double l = (r - R) * (r + R) / (std::sqrt(disc) - r * mu);
  return l < 0 ? 0 : l;
}

/* ---- 2-D cylindrical r-z event: IMC/IMC2D.py:826-935 ---- */
EventOut event_rz(double w, double mu, double eta, double r, double z, double rin, double rout,
                  double zlo, double zhi, double sa, double ss, double dcen, double u0, double u1,
                  double u2, bool cap = true) {
  EventOut o{};
  const double sin2 = 1.0 - eta * eta;
  double s_rin = BIG, s_rout = BIG;
  if (sin2 >= 1e-15) {
    const double st = std::sqrt(sin2);
    const double b2 = r * r * (1.0 - mu * mu);
    s_rout = rz_outer_l(r, mu, rout, b2) / st;
    const double li = rz_inner_l(r, mu, rin, b2);
    if (li < BIG) s_rin = li / st;
  }
  double s_zlo = BIG, s_zhi = BIG;
  if (eta > 1e-15) s_zhi = std::max((zhi - z) / eta, 0.0);
  else if (eta < -1e-15) s_zlo = std::max((zlo - z) / eta, 0.0);
  const double ds = scatter_distance(ss, std::min(rout - rin, zhi - zlo), u0, 1e-12, cap);
  double sb = s_rin;
  if (s_rout < sb) sb = s_rout;
  if (s_zlo < sb) sb = s_zlo;
  if (s_zhi < sb) sb = s_zhi;
  double s = sb;
  int evt = EV_BOUNDARY;
  if (ds < s) { s = ds; evt = EV_SCATTER; }
  if (dcen < s) { s = dcen; evt = EV_CENSUS; }
  const double l = s * std::sqrt(std::max(sin2, 0.0));
  double rn = std::sqrt(std::max(r * r + 2.0 * r * mu * l + l * l, 0.0));
  double zn = z + s * eta;
  double mun = mu, etan = eta;
  if (rn > 1e-15 && l > 0) mun = std::min(1.0, std::max(-1.0, (r * mu + l) / rn));
  int cross = X_NONE;
  if (evt == EV_BOUNDARY) {
    /* no 1e-12 nudges: the cell index, not the position, decides the cell */
    if (sb == s_rin) { rn = rin; cross = X_IM; }
    else if (sb == s_rout) { rn = rout; cross = X_IP; }
    else if (sb == s_zlo) { zn = zlo; cross = X_JM; }
    else { zn = zhi; cross = X_JP; }
  } else if (evt == EV_SCATTER) {
    /* IMC/IMC2D.py:704-708 */
    etan = 2.0 * u1 - 1.0;
    mun = std::cos(2.0 * PI * u2);
  }
  if (cross != X_IM && cross != X_IP) rn = std::min(std::max(rn, rin), rout);
  if (cross != X_JM && cross != X_JP) zn = std::min(std::max(zn, zlo), zhi);
  const double wn = w * std::exp(-sa * s);
  const double lost = w - wn;
  o.dep = lost;
  o.dep_i = (sa > 1e-12) ? lost / sa : w * s;
  o.w = wn; o.d1 = mun; o.d2 = etan; o.p1 = rn; o.p2 = zn; o.dcen = dcen - s; o.s = s;
  o.cross = cross; o.evt = evt;
  return o;
}

/* ---- problem / bank ---- */
struct Problem {
  int geom = 0, nx = 1, ny = 1, ng = 1;
  std::vector<double> e1, e2, vol;
  uint64_t seed = 0;
};

struct Bank {
  std::vector<double> w, d1, d2, t, p1, p2;
  std::vector<int> cell, grp;
  size_t size() const { return w.size(); }
  void resize(size_t n) {
    w.resize(n); d1.resize(n); d2.resize(n); t.resize(n);
    p1.resize(n); p2.resize(n); cell.resize(n); grp.resize(n);
  }
  void push(double w_, double d1_, double d2_, double t_, double p1_, double p2_, int c, int g) {
    w.push_back(w_); d1.push_back(d1_); d2.push_back(d2_); t.push_back(t_);
    p1.push_back(p1_); p2.push_back(p2_); cell.push_back(c); grp.push_back(g);
  }
};

struct Oracle {
  Problem P;
  Bank B;
};

inline int ncells(const Problem& P) { return P.nx * P.ny; }

/* Canonical FP64 total: 1024 strided partial sums, then a halving tree.  The CUDA path
 * reduces in exactly this order (one 1024-thread block), so totals, and the integer
 * source counts derived from them, agree bit for bit. */
double canon_sum(const double* x, long long n) {
  double part[1024];
  for (int t = 0; t < 1024; ++t) {
    double s = 0;
    for (long long i = t; i < n; i += 1024) s += x[i];
    part[t] = s;
  }
  for (int h = 512; h >= 1; h >>= 1)
    for (int i = 0; i < h; ++i) part[i] += part[i + h];
  return part[0];
}
inline double pow4(double T) { const double t2 = T * T; return t2 * t2; }

/* Neumaier-compensated accumulator: millions of event tallies per cell sum to FP64 round-off
 * of the total, so the ledger check measures the algorithm, not the summation order. */
struct KSum {
  double s = 0.0, c = 0.0;
  inline void add(double x) {
    const double t = s + x;
    c += (std::fabs(s) >= std::fabs(x)) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  inline double value() const { return s + c; }
};
inline double pow3(double T) { return T * T * T; }
inline bool is1d(const Problem& P) { return P.geom == G_SLAB || P.geom == G_SPHERE; }

int locate(const std::vector<double>& e, double v) {
  /* np.searchsorted(edges, v, side='right') - 1, clamped into the mesh */
  int i = (int)(std::upper_bound(e.begin(), e.end(), v) - e.begin()) - 1;
  const int n = (int)e.size() - 1;
  return std::min(std::max(i, 0), n - 1);
}

/* isotropic direction for the geometry from two uniforms */
inline void iso_dir(int geom, double ua, double ub, double& d1, double& d2) {
  if (is1d(Problem{geom})) { d1 = 2.0 * ua - 1.0; d2 = 0; return; }
  if (geom == G_XY) {
    const double uz = 2.0 * ua - 1.0, phi = 2.0 * PI * ub;
    const double rxy = std::sqrt(std::max(0.0, 1.0 - uz * uz));
    d1 = rxy * std::cos(phi); d2 = rxy * std::sin(phi);
  } else {
    d2 = 2.0 * ua - 1.0;            /* eta */
    d1 = std::cos(2.0 * PI * ub);    /* mu_perp */
  }
}

/* Carter-Forest absorption (IMC/IMC1D_CarterForest.py:146-194, :678-709;
 * IMC/IMC2D_CarterForest.py:189-210, :318-340), for an event whose absorption distance won
 * (EV_SCATTER of the flight run with sigma_s := sigma_a and no implicit capture, which also
 * drew the new isotropic direction).  rate = c sigma_a beta, 0 when beta or sigma_a <=
 * 1e-15.  Re-emission after a delay ~ Exp(rate) when it falls inside the step (e.dcen becomes
 * the distance left after the delay); otherwise capture (returns true).  Without a rate the
 * 1-D modules redirect the photon and the 2-D module captures it.  The stiff fast path
 * (threshold > 0) captures with probability exp(-rate t_left), else redirects at once. */
bool cf_absorb(bool oned, double rate, double fastpath, double ud, EventOut& e) {
  const double tr = e.dcen / C_LIGHT;
  if (!(rate > 0)) return !oned;
  if (fastpath > 0 && tr > 1e-14 && rate * tr > fastpath) return ud < std::exp(-rate * tr);
  const double delay = -std::log(std::max(ud, 1e-15)) / rate;
  if (oned ? (tr > 1e-14 && delay < tr) : (delay < tr - 1e-15)) {
    e.dcen = std::max(0.0, (tr - delay) * C_LIGHT);
    return false;
  }
  return true;
}

}  // namespace

/* ======================================================================================
 * C API
 * ==================================================================================== */
extern "C" {

/* per-event pins (used against golden vectors recorded from the reference) */
void orc_event(int geom, const double* in, double* out) {
  /* in: w d1 d2 p1 p2 lo1 hi1 lo2 hi2 sa ss dcen u0 u1 u2 */
  EventOut o;
  switch (geom) {
    case G_SLAB: o = event_slab(in[0], in[1], in[3], in[5], in[6], in[9], in[10], in[11], in[12], in[13]); break;
    case G_SPHERE: o = event_sphere(in[0], in[1], in[3], in[5], in[6], in[9], in[10], in[11], in[12], in[13]); break;
    case G_XY: o = event_xy(in[0], in[1], in[2], in[3], in[4], in[5], in[6], in[7], in[8], in[9], in[10], in[11], in[12], in[13], in[14]); break;
    default: o = event_rz(in[0], in[1], in[2], in[3], in[4], in[5], in[6], in[7], in[8], in[9], in[10], in[11], in[12], in[13], in[14]); break;
  }
  out[0] = o.w; out[1] = o.d1; out[2] = o.d2; out[3] = o.p1; out[4] = o.p2;
  out[5] = o.dep; out[6] = o.dep_i; out[7] = o.dcen; out[8] = o.cross; out[9] = o.evt;
}

/* one Carter-Forest event (pins): in = w d1 d2 p1 p2 lo1 hi1 lo2 hi2 sigma_a rate dcen
 * fastpath u0 u1 u2 u3 (u0 distance; 1-D: u1 direction, u2 delay; 2-D: u1 u2 direction, u3
 * delay); out = w d1 d2 p1 p2 dep_w dep_i dcen cross evt (0 census, 1 boundary,
 * 2 absorbed and continuing, 4 captured).  dep_i is w*s (1-D: per unit length / volume). */
void orc_event_cf(int geom, const double* in, double* out) {
  EventOut e;
  const bool oned = geom == G_SLAB || geom == G_SPHERE;
  switch (geom) {
    case G_SLAB: e = event_slab(in[0], in[1], in[3], in[5], in[6], 0.0, in[9], in[11], in[13], in[14]); break;
    case G_SPHERE: e = event_sphere(in[0], in[1], in[3], in[5], in[6], 0.0, in[9], in[11], in[13], in[14]); break;
    case G_XY: e = event_xy(in[0], in[1], in[2], in[3], in[4], in[5], in[6], in[7], in[8], 0.0, in[9], in[11], in[13], in[14], in[15]); break;
    default: e = event_rz(in[0], in[1], in[2], in[3], in[4], in[5], in[6], in[7], in[8], 0.0, in[9], in[11], in[13], in[14], in[15]); break;
  }
  int evt = e.evt == EV_SCATTER ? 2 : e.evt;
  double dep_w = 0.0, w = e.w;
  if (e.evt == EV_SCATTER && cf_absorb(oned, in[10], in[12], oned ? in[15] : in[16], e)) {
    evt = 4; dep_w = w; w = 0.0; e.dcen = 0.0;
  }
  out[0] = w; out[1] = e.d1; out[2] = e.d2; out[3] = e.p1; out[4] = e.p2;
  out[5] = dep_w; out[6] = e.dep_i; out[7] = e.dcen; out[8] = e.cross; out[9] = evt;
}

void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  oracle::philox4x32_10(ctr, key, out);
}

void* orc_create(int geom, int nx, int ny, int ng, const double* e1, const double* e2,
                 const double* vol, uint64_t seed) {
  Oracle* o = new Oracle();
  o->P.geom = geom; o->P.nx = nx; o->P.ny = ny; o->P.ng = ng; o->P.seed = seed;
  o->P.e1.assign(e1, e1 + nx + 1);
  o->P.e2.assign(e2, e2 + ny + 1);
  /* cell volumes come from the caller (the host computes them once, as the reference
   * does, and hands the same array to every implementation) */
  o->P.vol.assign(vol, vol + (size_t)nx * ny);
  return o;
}

void orc_destroy(void* h) { delete (Oracle*)h; }

long long orc_size(void* h) { return (long long)((Oracle*)h)->B.size(); }

void orc_volumes(void* h, double* out) {
  Oracle* o = (Oracle*)h;
  std::copy(o->P.vol.begin(), o->P.vol.end(), out);
}

void orc_get_bank(void* h, double* w, double* d1, double* d2, double* t, double* p1, double* p2,
                  int* cell, int* grp) {
  Bank& B = ((Oracle*)h)->B;
  const size_t n = B.size();
  std::copy(B.w.begin(), B.w.begin() + n, w);
  std::copy(B.d1.begin(), B.d1.begin() + n, d1);
  std::copy(B.d2.begin(), B.d2.begin() + n, d2);
  std::copy(B.t.begin(), B.t.begin() + n, t);
  std::copy(B.p1.begin(), B.p1.begin() + n, p1);
  std::copy(B.p2.begin(), B.p2.begin() + n, p2);
  std::copy(B.cell.begin(), B.cell.begin() + n, cell);
  std::copy(B.grp.begin(), B.grp.begin() + n, grp);
}

void orc_set_bank(void* h, long long n, const double* w, const double* d1, const double* d2,
                  const double* t, const double* p1, const double* p2, const int* cell,
                  const int* grp) {
  Bank& B = ((Oracle*)h)->B;
  B.w.assign(w, w + n); B.d1.assign(d1, d1 + n); B.d2.assign(d2, d2 + n);
  B.t.assign(t, t + n); B.p1.assign(p1, p1 + n); B.p2.assign(p2, p2 + n);
  B.cell.assign(cell, cell + n);
  if (grp) B.grp.assign(grp, grp + n); else B.grp.assign(n, 0);
}

/* ---------------- initial census (gray) ----------------
 * slab: IMC/IMC1D.py:220-248 (counts ceil(N E_c/E), no minimum)
 * sphere: IMC/IMC1D.py:535-575
 * xy/rz: IMC/IMC2D.py:1110-1188 (counts max(1, ceil(N E_c/E)))
 * Draws: index k of the IC particle, block 0, step 0, TAG_IC. */
long long orc_init_ic(void* h, long long N, const double* Tr, double T_emit_floor) {
  Oracle* o = (Oracle*)h;
  Problem& P = o->P;
  Bank& B = o->B;
  B.resize(0);
  const int nc = ncells(P);
  std::vector<double> E(nc);
  for (int c = 0; c < nc; ++c) {
    E[c] = A_RAD * pow4(Tr[c]) * P.vol[c];
    if (T_emit_floor > 0 && Tr[c] < T_emit_floor) E[c] = 0;
  }
  const double Et = canon_sum(E.data(), nc);
  if (N <= 0 || (is1d(P) && Et <= 0)) return 0;
  uint32_t k = 0;
  /* 1-D orders by cell i; 2-D by (i outer, j inner) as the reference loops */
  std::vector<int> order;
  if (is1d(P)) { for (int i = 0; i < P.nx; ++i) order.push_back(i); }
  else { for (int i = 0; i < P.nx; ++i) for (int j = 0; j < P.ny; ++j) order.push_back(i + P.nx * j); }
  for (int c : order) {
    long long n;
    if (is1d(P)) n = (long long)std::ceil(E[c] / Et * (double)N);
    else n = std::max(1LL, (long long)std::ceil((double)N * E[c] / std::max(Et, 1e-300)));
    if (n <= 0) continue;
    const double wgt = E[c] / (double)n;
    const int i = c % P.nx, j = c / P.nx;
    const double a = P.e1[i], b = P.e1[i + 1], lo = P.e2[j], hi = P.e2[j + 1];
    for (long long q = 0; q < n; ++q, ++k) {
      Draw4 r = draw(P.seed, k, 0, 0, oracle::TAG_IC);
      double p1, p2 = 0, d1, d2;
      switch (P.geom) {
        case G_SLAB: p1 = a + r.u[0] * (b - a); break;
        case G_SPHERE: p1 = std::cbrt(a * a * a + (b * b * b - a * a * a) * r.u[0]); break;
        case G_XY: p1 = a + r.u[0] * (b - a); p2 = lo + r.u[1] * (hi - lo); break;
        default: p1 = std::sqrt(a * a + (b * b - a * a) * r.u[0]); p2 = lo + r.u[1] * (hi - lo); break;
      }
      iso_dir(P.geom, r.u[2], r.u[3], d1, d2);
      B.push(wgt, d1, d2, 0.0, p1, p2, c, 0);
    }
  }
  return (long long)B.size();
}

/* ---------------- step phase 1: Fleck, sources, transport ---------------- */
typedef struct {
  uint32_t step;
  double dt, theta;
  const double* T;        /* material temperature per cell */
  const double* sigma;    /* true absorption opacity per cell */
  const double* cv;       /* heat capacity per cell */
  long long Ntarget, Nboundary, Nsource;
  const double* source;   /* fixed source power density per cell or NULL */
  const double* face_T[4];/* per-face-cell boundary temperature, NULL = no source */
  int reflect[4];
  long long max_events;   /* <= 0: no cap (1-D reference has none) */
  int rz_linear_source;
  double T_emit_floor;
  int nthreads;
  int sources_only;       /* 1: Fleck + sources appended, no transport (pins) */
  int method;             /* 0 Fleck-Cummings, 1 Carter-Forest */
  double cf_fastpath;     /* Carter-Forest stiff fast path threshold (0 = off) */
} orc_step_in;

typedef struct {
  double* dep;            /* energy deposited per unit volume, per cell */
  double* si;             /* path-length scalar intensity per cell */
  double* emitted;        /* emission energy removed from matter per cell (GJ) */
  double* sigma_a;        /* Fleck-modified absorption per cell (out) */
  double* sigma_s;        /* effective scatter per cell (out) */
  double boundary_emission, source_emission;
  double escaped[4];
  long long stats[S_N];
  long long n_transported;
  double weight_floor;
} orc_step_out;

}  // extern "C"

namespace {

/* Fleck factor, IMC/IMC1D.py:933-938 (1-D asserts f in [0,1]); IMC/IMC2D.py:1646-1651 (clip). */
void fleck(const Problem& P, const orc_step_in* in, std::vector<double>& sa, std::vector<double>& ss) {
  const int nc = ncells(P);
  sa.resize(nc); ss.resize(nc);
  for (int c = 0; c < nc; ++c) {
    const double T = in->T[c];
    const double beta = 4.0 * A_RAD * pow3(T) / in->cv[c];
    double f = 1.0 / (1.0 + in->theta * beta * in->sigma[c] * C_LIGHT * in->dt);
    f = std::min(1.0, std::max(0.0, f));
    ss[c] = in->sigma[c] * (1.0 - f);
    sa[c] = in->sigma[c] * f;
  }
}

/* Boundary source, shared by every geometry.  For each side with a face-temperature
 * array: face cell chosen with probability proportional to a c T^4/4 * area * dt (the
 * reference's multinomial, IMC/IMC2D.py:183-206, 350-412; uniform T reduces to the
 * uniform face sampling of :284-319), equal weights total/n, position uniform in the
 * face cell's area, half-Lambertian direction.
 * Draws: k, blocks 0 and 1, step, TAG_BOUNDARY|side. */
double boundary_source(const Problem& P, const orc_step_in* in, Bank& B) {
  double total = 0;
  for (int side = 0; side < 4; ++side) {
    const double* Tf = in->face_T[side];
    if (!Tf || in->Nboundary <= 0) continue;
    if (is1d(P) && side >= 2) continue;
    const bool along2 = (side < 2);           /* rmin/rmax/left/right: cells indexed by j */
    const int nf = is1d(P) ? 1 : (along2 ? P.ny : P.nx);
    std::vector<double> Ef(nf), cdf(nf);
    double Et = 0;
    for (int q = 0; q < nf; ++q) {
      double area;
      if (is1d(P)) {
        if (P.geom == G_SLAB) area = 1.0;
        else { const double R = side == 0 ? P.e1[0] : P.e1[P.nx]; area = 4.0 * PI * R * R; }
      } else if (P.geom == G_XY) {
        area = along2 ? (P.e2[q + 1] - P.e2[q]) : (P.e1[q + 1] - P.e1[q]);
      } else {
        if (along2) { const double R = side == 0 ? P.e1[0] : P.e1[P.nx]; area = 2.0 * PI * R * (P.e2[q + 1] - P.e2[q]); }
        else area = PI * (P.e1[q + 1] * P.e1[q + 1] - P.e1[q] * P.e1[q]);
      }
      const double T = Tf[q];
      Ef[q] = (T > 0) ? A_RAD * C_LIGHT * T * T * T * T / 4.0 * area * in->dt : 0.0;
      Et += Ef[q];
      cdf[q] = Et;
    }
    if (!(Et > 0)) continue;
    const long long n = in->Nboundary;
    const double wgt = Et / (double)n;
    for (long long k = 0; k < n; ++k) {
      Draw4 a = draw(P.seed, (uint32_t)k, 0, in->step, oracle::TAG_BOUNDARY | side);
      Draw4 b = draw(P.seed, (uint32_t)k, 1, in->step, oracle::TAG_BOUNDARY | side);
      int q = (int)(std::lower_bound(cdf.begin(), cdf.end(), a.u[0] * Et) - cdf.begin());
      q = std::min(q, nf - 1);
      while (Ef[q] <= 0 && q > 0) --q;  /* never land in a non-emitting face cell */
      const double mu_n = std::sqrt(a.u[2]);
      const double t = b.u[0] * in->dt;
      double p1, p2 = 0, d1, d2 = 0;
      int i, j = 0;
      if (is1d(P)) {
        i = side == 0 ? 0 : P.nx - 1;
        p1 = side == 0 ? P.e1[0] : P.e1[P.nx];
        d1 = side == 0 ? mu_n : -mu_n;
      } else if (P.geom == G_XY) {
        const double mu_t = std::sqrt(std::max(0.0, 1.0 - mu_n * mu_n));
        const double ct = mu_t * std::cos(2.0 * PI * a.u[3]);
        if (along2) {
          j = q; i = side == 0 ? 0 : P.nx - 1;
          p1 = side == 0 ? P.e1[0] : P.e1[P.nx];
          p2 = P.e2[q] + a.u[1] * (P.e2[q + 1] - P.e2[q]);
          d1 = side == 0 ? mu_n : -mu_n; d2 = ct;
        } else {
          i = q; j = side == 2 ? 0 : P.ny - 1;
          p2 = side == 2 ? P.e2[0] : P.e2[P.ny];
          p1 = P.e1[q] + a.u[1] * (P.e1[q + 1] - P.e1[q]);
          d2 = side == 2 ? mu_n : -mu_n; d1 = ct;
        }
      } else { /* rz */
        if (along2) {
          j = q; i = side == 0 ? 0 : P.nx - 1;
          p1 = side == 0 ? P.e1[0] : P.e1[P.nx];
          p2 = P.e2[q] + a.u[1] * (P.e2[q + 1] - P.e2[q]);
          d1 = side == 0 ? mu_n : -mu_n;      /* mu_perp */
          d2 = 2.0 * a.u[3] - 1.0;            /* eta */
        } else {
          i = q; j = side == 2 ? 0 : P.ny - 1;
          const double r0 = P.e1[q], r1 = P.e1[q + 1];
          p1 = std::sqrt(r0 * r0 + a.u[1] * (r1 * r1 - r0 * r0));
          p2 = side == 2 ? P.e2[0] : P.e2[P.ny];
          d2 = side == 2 ? mu_n : -mu_n;      /* eta */
          d1 = std::cos(2.0 * PI * a.u[3]);   /* mu_perp */
        }
      }
      B.push(wgt, d1, d2, t, p1, p2, i + P.nx * j, 0);
      total += wgt;
    }
  }
  return total;
}

/* slab linear-T position sampler, IMC/IMC1D.py:203-217 (closed-form inversion) */
double slab_linear(double dx, double s, double T, double xi) {
  if (std::fabs(s) < 1e-6) return xi * dx;
  const double smax = 2.0 * T / (dx * dx);
  s = std::max(-smax, std::min(s, smax));
  const double disc = (s / (2.0 * T) - 1.0 / dx) * (s / (2.0 * T) - 1.0 / dx) + 2.0 * s * xi / (T * dx);
  return (-2.0 * T + s * dx + 2.0 * T * dx * std::sqrt(std::max(disc, 0.0))) / (2.0 * s);
}

/* sphere linear-T^4 CDF inversion, IMC/IMC1D.py:578-626 */
double sphere_cdf(double r0, double r1, double a, double M, double xi) {
  const double C = a / 3.0 * (r1 * r1 * r1 - r0 * r0 * r0) + M / 4.0 * (pow4(r1) - pow4(r0));
  if (C <= 0) return r0 + xi * (r1 - r0);
  const double rhs = xi * C + (a / 3.0 * r0 * r0 * r0 + M / 4.0 * pow4(r0));
  double lo = r0, hi = r1, r = r0 + xi * (r1 - r0);
  for (int it = 0; it < 60; ++it) {
    const double r3 = r * r * r, r4 = r3 * r;
    const double g = a / 3.0 * r3 + M / 4.0 * r4 - rhs;
    if (std::fabs(g) < 1e-14 * (std::fabs(rhs) + 1e-30)) break;
    if (g < 0) lo = r; else hi = r;
    const double dg = r * r * (a + M * r);
    double rn = std::fabs(dg) > 1e-30 ? r - g / dg : 0.5 * (lo + hi);
    if (rn <= lo || rn >= hi) rn = 0.5 * (lo + hi);
    if (std::fabs(rn - r) < 1e-14 * (r1 - r0 + 1e-30)) { r = rn; break; }
    r = rn;
  }
  return r;
}

/* cylinder linear-in-r CDF inversion, IMC/IMC2D.py:1293-1323 */
double rz_r_cdf(double r0, double r1, double a, double M, double xi) {
  const double C = a * 0.5 * (r1 * r1 - r0 * r0) + M / 3.0 * (r1 * r1 * r1 - r0 * r0 * r0);
  if (C <= 0) return std::sqrt(r0 * r0 + (r1 * r1 - r0 * r0) * xi);
  const double rhs = xi * C + a * 0.5 * r0 * r0 + M / 3.0 * r0 * r0 * r0;
  double lo = r0, hi = r1, r = std::sqrt(r0 * r0 + (r1 * r1 - r0 * r0) * xi);
  for (int it = 0; it < 50; ++it) {
    const double g = a * 0.5 * r * r + M / 3.0 * r * r * r - rhs;
    if (std::fabs(g) < 1e-14 * (std::fabs(rhs) + 1e-30)) break;
    if (g < 0) lo = r; else hi = r;
    const double dg = a * r + M * r * r;
    double rn = std::fabs(dg) > 1e-30 ? r - g / dg : 0.5 * (lo + hi);
    if (rn <= lo || rn >= hi) rn = 0.5 * (lo + hi);
    if (std::fabs(rn - r) < 1e-14 * (r1 - r0 + 1e-30)) { r = rn; break; }
    r = rn;
  }
  return r;
}

/* Volume source with per-cell energies QV (counts ceil(N QV/Qtot), weights QV/n).
 * kind: 0 = material emission (times U(0,dt), 1-D linear tilts),
 *       1 = fixed source.  Draws: k, blocks 0 and 1, step, tag.
 * slab: IMC/IMC1D.py:251-316; sphere :629-741; xy IMC/IMC2D.py:1191-1238;
 * rz uniform :1241-1290, rz linear :1326-1445. */
double volume_source(const Problem& P, const std::vector<double>& QV, const double* T, long long N,
                     double dt, uint32_t step, uint32_t tag, bool tilt, bool rz_linear, Bank& B,
                     bool min1_round = false, const std::vector<double>* cf_rate = nullptr,
                     double cf_thr = 0.0) {
  const int nc = ncells(P);
  const double Qt = canon_sum(QV.data(), nc);
  if (!(Qt > 0) || N <= 0) return 0;
  /* tilt data */
  std::vector<double> slope(nc, 0.0), Mr(nc, 0.0), Mz(nc, 0.0);
  if (tilt && P.geom == G_SLAB && P.nx > 1) {
    const int I = P.nx;
    auto dx = [&](int i) { return P.e1[i + 1] - P.e1[i]; };
    for (int i = 1; i < I - 1; ++i) slope[i] = (T[i + 1] - T[i - 1]) / (dx(i + 1) + dx(i - 1)) * 2;
    slope[0] = (T[1] - T[0]) / (dx(1) + dx(0)) * 2;
    slope[I - 1] = (T[I - 1] - T[I - 2]) / (dx(I - 1) + dx(I - 2)) * 2;
    for (int i = 0; i < I; ++i) {
      if (T[i] - slope[i] * dx(i) / 2 < 0) slope[i] = 0;
      else if (T[i] + slope[i] * dx(i) / 2 < 0) slope[i] = 0;
    }
  }
  if (tilt && P.geom == G_SPHERE && P.nx > 1) {
    const int I = P.nx;
    std::vector<double> rm(I), T4(I);
    for (int i = 0; i < I; ++i) { rm[i] = 0.5 * (P.e1[i] + P.e1[i + 1]); T4[i] = pow4(T[i]); }
    for (int i = 1; i < I - 1; ++i) slope[i] = (T4[i + 1] - T4[i - 1]) / (rm[i + 1] - rm[i - 1]);
    slope[0] = (T4[1] - T4[0]) / (rm[1] - rm[0]);
    slope[I - 1] = (T4[I - 1] - T4[I - 2]) / (rm[I - 1] - rm[I - 2]);
    for (int i = 0; i < I; ++i) {
      const double a = T4[i] - slope[i] * (rm[i] - P.e1[i]);
      const double b = T4[i] + slope[i] * (P.e1[i + 1] - rm[i]);
      if (a < 0 || b < 0) slope[i] = 0;
    }
  }
  if (P.geom == G_RZ && rz_linear) {
    std::vector<double> rc(P.nx), zc(P.ny);
    for (int i = 0; i < P.nx; ++i) rc[i] = 0.5 * (P.e1[i] + P.e1[i + 1]);
    for (int j = 0; j < P.ny; ++j) zc[j] = 0.5 * (P.e2[j] + P.e2[j + 1]);
    auto T4 = [&](int i, int j) { return pow4(std::max(T[i + P.nx * j], 0.0)); };
    for (int i = 0; i < P.nx; ++i)
      for (int j = 0; j < P.ny; ++j) {
        const int c = i + P.nx * j;
        if (P.nx == 1) Mr[c] = 0;
        else if (i == 0) Mr[c] = (T4(i + 1, j) - T4(i, j)) / (rc[i + 1] - rc[i]);
        else if (i == P.nx - 1) Mr[c] = (T4(i, j) - T4(i - 1, j)) / (rc[i] - rc[i - 1]);
        else Mr[c] = (T4(i + 1, j) - T4(i - 1, j)) / (rc[i + 1] - rc[i - 1]);
        if (P.ny == 1) Mz[c] = 0;
        else if (j == 0) Mz[c] = (T4(i, j + 1) - T4(i, j)) / (zc[j + 1] - zc[j]);
        else if (j == P.ny - 1) Mz[c] = (T4(i, j) - T4(i, j - 1)) / (zc[j] - zc[j - 1]);
        else Mz[c] = (T4(i, j + 1) - T4(i, j - 1)) / (zc[j + 1] - zc[j - 1]);
      }
  }
  std::vector<int> order;
  if (is1d(P)) { for (int i = 0; i < P.nx; ++i) order.push_back(i); }
  else { for (int i = 0; i < P.nx; ++i) for (int j = 0; j < P.ny; ++j) order.push_back(i + P.nx * j); }
  double total = 0;
  uint32_t k = 0;
  for (int c : order) {
    /* Carter-Forest 1-D emission (IMC/IMC1D_CarterForest.py:499, :932): max(1, round) in
     * every cell, a zero-energy cell included */
    const long long n = min1_round ? std::max(1LL, (long long)std::nearbyint((double)N * QV[c] / Qt))
                                   : (long long)std::ceil((double)N * QV[c] / Qt);
    if (n <= 0) continue;
    const double wgt = QV[c] / (double)n;
    const int i = c % P.nx, j = c / P.nx;
    const double a = P.e1[i], b = P.e1[i + 1], lo = P.e2[j], hi = P.e2[j + 1];
    /* per-cell tilt constants */
    double ar = 0, Mloc = 0, Pn = 0.5, sa_c = 0, M4 = 0;
    if (P.geom == G_RZ && rz_linear) {
      const double rcen = 0.5 * (a + b), zcen = 0.5 * (lo + hi), T4c = pow4(std::max(T[c], 0.0));
      ar = T4c - Mr[c] * (rcen - a);
      const double t0 = ar, t1 = ar + Mr[c] * (b - a);
      if (t0 < 0 || t1 < 0) { ar = std::max(T4c, 0.0); Mloc = 0; } else Mloc = Mr[c];
      const double az = T4c - Mz[c] * (zcen - lo);
      const double z0 = std::max(az, 0.0), z1 = std::max(az + Mz[c] * (hi - lo), 0.0);
      Pn = (z0 + z1 > 0) ? z0 / (z0 + z1) : 0.5;
    }
    if (P.geom == G_SPHERE && tilt) {
      M4 = slope[i];
      sa_c = pow4(T[i]) - M4 * (0.5 * (a + b) - a);
    }
    for (long long q = 0; q < n; ++q, ++k) {
      Draw4 r = draw(P.seed, k, 0, step, tag);
      Draw4 s = draw(P.seed, k, 1, step, tag);
      double p1, p2 = 0, d1, d2;
      switch (P.geom) {
        case G_SLAB:
          p1 = a + (tilt ? slab_linear(b - a, slope[i], T[i], r.u[0]) : r.u[0] * (b - a));
          break;
        case G_SPHERE:
          if (tilt && !(std::fabs(M4) < 1e-30 || std::fabs(sa_c) < 1e-30)) p1 = sphere_cdf(a, b, sa_c, M4, r.u[0]);
          else p1 = std::cbrt(a * a * a + (b * b * b - a * a * a) * r.u[0]);
          break;
        case G_XY:
          p1 = a + r.u[0] * (b - a); p2 = lo + r.u[1] * (hi - lo);
          break;
        default:
          if (rz_linear) {
            p1 = rz_r_cdf(a, b, ar, Mloc, r.u[0]);
            const double sq = std::sqrt(r.u[1]);
            p2 = (s.u[1] <= Pn) ? hi - (hi - lo) * sq : lo + (hi - lo) * sq;
          } else {
            p1 = std::sqrt(a * a + (b * b - a * a) * r.u[0]);
            p2 = lo + r.u[1] * (hi - lo);
          }
          break;
      }
      p1 = std::min(std::max(p1, a), b);
      p2 = is1d(P) ? 0.0 : std::min(std::max(p2, lo), hi);
      iso_dir(P.geom, r.u[2], r.u[3], d1, d2);
      double t = s.u[0] * dt;  /* reference 1-D fixed source uses U(0,1): fixed to U(0,dt) */
      if (cf_rate) {
        /* Carter-Forest emission time, density ~ exp(-rate t) on [0, dt]
         * (IMC/IMC1D_CarterForest.py:529-536, IMC/IMC2D_CarterForest.py:51-56):
         * t = -ln(1 - xi (1 - e^{-rate dt})) / rate, written with log1p / expm1 */
        const double rt = (*cf_rate)[c];
        if (rt > cf_thr) t = -std::log1p(s.u[0] * std::expm1(-rt * dt)) / rt;
      }
      B.push(wgt, d1, d2, t, p1, p2, c, 0);
      total += wgt;
    }
  }
  return total;
}

}  // namespace

extern "C" {

int orc_step_transport(void* h, const orc_step_in* in, orc_step_out* out) {
  Oracle* o = (Oracle*)h;
  Problem& P = o->P;
  Bank& B = o->B;
  const int nc = ncells(P);
  std::vector<double> sa, ss;
  fleck(P, in, sa, ss);
  for (int c = 0; c < nc; ++c)
    if (!(in->T[c] > 0) && is1d(P)) return 1; /* IMC/IMC1D.py:264 asserts T > 0 */
  /* Carter-Forest (IMC/IMC1D_CarterForest.py:1151-1244, IMC/IMC2D_CarterForest.py:909-1045):
   * no Fleck factor, sigma_a is the true opacity, no effective scatter; beta = 4aT^3/cv
   * (2-D: T floored at 1e-12) sets the re-emission rate c sigma_a beta, which is zero when
   * beta or sigma_a <= 1e-15 (no re-emission) */
  const bool cf = in->method == 1;
  std::vector<double> rate_e(nc, 0.0), rate_re(nc, 0.0), beta_c(nc, 0.0);
  if (cf) {
    for (int c = 0; c < nc; ++c) {
      const double Tm = is1d(P) ? in->T[c] : std::max(in->T[c], 1e-12);
      const double beta = 4.0 * A_RAD * pow3(Tm) / in->cv[c];
      beta_c[c] = beta;
      sa[c] = in->sigma[c];
      ss[c] = 0.0;
      rate_e[c] = C_LIGHT * in->sigma[c] * beta;
      rate_re[c] = (beta > 1e-15 && in->sigma[c] > 1e-15) ? rate_e[c] : 0.0;
    }
  }
  if (out->sigma_a) std::copy(sa.begin(), sa.end(), out->sigma_a);
  if (out->sigma_s) std::copy(ss.begin(), ss.end(), out->sigma_s);

  /* sources appended in the reference's order: census | boundary | fixed | emission */
  out->boundary_emission = boundary_source(P, in, B);
  out->source_emission = 0;
  if (in->Nsource > 0 && in->source) {
    double smax = 0;
    for (int c = 0; c < nc; ++c) smax = std::max(smax, in->source[c]);
    if (smax > 0) {
      std::vector<double> QV(nc);
      for (int c = 0; c < nc; ++c) QV[c] = in->source[c] * in->dt * P.vol[c];
      const bool tilt_rz = (P.geom == G_RZ) && in->rz_linear_source;
      out->source_emission = volume_source(P, QV, in->T, in->Nsource, in->dt, in->step,
                                           oracle::TAG_SOURCE, false, tilt_rz, B);
    }
  }
  std::vector<double> E(nc);
  for (int c = 0; c < nc; ++c) {
    E[c] = A_RAD * C_LIGHT * pow4(std::max(in->T[c], 0.0)) * sa[c] * in->dt * P.vol[c];
    if (cf) {
      /* a T^4 (1 - e^{-rate dt}) / beta V (IMC/IMC1D_CarterForest.py:485-494,
       * IMC/IMC2D_CarterForest.py:877-883), 1 - e^{-x} without cancellation */
      const double T4 = pow4(std::max(in->T[c], 0.0));
      const double beta = beta_c[c];
      const bool decays = is1d(P) ? rate_e[c] > 1e-10 : (rate_e[c] > 1e-12 && beta > 1e-15);
      E[c] = decays ? A_RAD * T4 * -std::expm1(-rate_e[c] * in->dt) / beta * P.vol[c]
                    : A_RAD * T4 * C_LIGHT * in->sigma[c] * in->dt * P.vol[c];
    }
    if (in->T_emit_floor > 0 && in->T[c] < in->T_emit_floor) E[c] = 0;
    out->emitted[c] = 0;
  }
  {
    const size_t n0 = B.size();
    if (in->Ntarget > 0)
      volume_source(P, E, in->T, in->Ntarget, in->dt, in->step, oracle::TAG_EMISSION, true,
                    (P.geom == G_RZ) && in->rz_linear_source, B, cf && is1d(P), cf ? &rate_e : nullptr,
                    is1d(P) ? 1e-10 : 1e-12);
    /* matter loses exactly the energy carried by the issued emission particles */
    std::vector<KSum> em(nc);
    for (size_t k = n0; k < B.size(); ++k) em[B.cell[k]].add(B.w[k]);
    for (int c = 0; c < nc; ++c) out->emitted[c] = em[c].value();
  }

  if (in->sources_only) return 0;

  /* weight floor, IMC/IMC1D.py:1007, IMC/IMC2D.py:1771 */
  const long long N = (long long)B.size();
  double wsum = 0;
  for (long long k = 0; k < N; ++k) wsum += B.w[k];
  const double floor_w = 1e-10 * wsum / (double)std::max(N, 1LL);
  out->weight_floor = floor_w;
  out->n_transported = N;

  int nth = in->nthreads > 0 ? in->nthreads : 1;
#ifndef _OPENMP
  nth = 1;
#endif
  std::vector<std::vector<KSum>> dep_t(nth, std::vector<KSum>(nc)), si_t(nth, std::vector<KSum>(nc));
  std::vector<std::vector<long long>> st_t(nth, std::vector<long long>(S_N, 0));
  std::vector<std::vector<KSum>> esc_t(nth, std::vector<KSum>(4));
  const double dt = in->dt;
  const bool oned = is1d(P);

#pragma omp parallel for schedule(dynamic, 256) num_threads(nth)
  for (long long k = 0; k < N; ++k) {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    KSum* dep = dep_t[tid].data();
    KSum* si = si_t[tid].data();
    long long* st = st_t[tid].data();
    KSum* esc = esc_t[tid].data();
    double w = B.w[k], d1 = B.d1[k], d2 = B.d2[k], p1 = B.p1[k], p2 = B.p2[k];
    int c = B.cell[k];
    /* Carter-Forest: an entry at or below the floor is not moved and stays in census
     * (IMC/IMC2D_CarterForest.py:381; the 1-D module deletes it, :320-322) */
    if (!(w > 0) || (cf && !(w > floor_w))) continue;
    double dcen = (dt - B.t[k]) * C_LIGHT;
    uint32_t ev = 0;
    bool frozen = false;
    while (dcen > 0) {
      int i = c % P.nx, j = c / P.nx;
      st[S_EVENTS]++;
      if ((cf || !oned) && in->max_events > 0 && (long long)ev >= in->max_events) {
        /* IMC/IMC2D.py:974-977: cap hit, particle stays in census with its weight */
        st[S_CAP]++;
        break;
      }
      Draw4 r = draw(P.seed, (uint32_t)k, ev, in->step, oracle::TAG_TRANSPORT);
      ++ev;
      /* Carter-Forest: the absorption distance is the capped "scatter" distance of sigma_a
       * and nothing is captured along the flight (weights change only at a capture) */
      const double sa_e = cf ? 0.0 : sa[c], ss_e = cf ? sa[c] : ss[c];
      EventOut e;
      switch (P.geom) {
        case G_SLAB: e = event_slab(w, d1, p1, P.e1[i], P.e1[i + 1], sa_e, ss_e, dcen, r.u[0], r.u[1]); break;
        case G_SPHERE: e = event_sphere(w, d1, p1, P.e1[i], P.e1[i + 1], sa_e, ss_e, dcen, r.u[0], r.u[1]); break;
        case G_XY: e = event_xy(w, d1, d2, p1, p2, P.e1[i], P.e1[i + 1], P.e2[j], P.e2[j + 1], sa_e, ss_e, dcen, r.u[0], r.u[1], r.u[2]); break;
        default: e = event_rz(w, d1, d2, p1, p2, P.e1[i], P.e1[i + 1], P.e2[j], P.e2[j + 1], sa_e, ss_e, dcen, r.u[0], r.u[1], r.u[2]); break;
      }
      const bool captured = cf && e.evt == EV_SCATTER && cf_absorb(oned, rate_re[c], in->cf_fastpath,
                                                                   oned ? r.u[2] : r.u[3], e);
      if (e.evt == EV_BOUNDARY) st[S_BOUNDARY]++;
      else if (captured) st[S_CAPTURE]++;
      else if (e.evt == EV_SCATTER) st[S_SCATTER]++;
      else st[S_CENSUS]++;
      if (oned) { dep[c].add(e.dep); si[c].add(e.dep_i / dt); }
      else { dep[c].add(e.dep / P.vol[c]); si[c].add(e.dep_i / (dt * P.vol[c])); }
      dcen = e.dcen;
      if (captured) {
        dep[c].add(w / P.vol[c]);
        w = 0; dcen = 0;
        break;
      }
      if (cf) {
        w = e.w;
      } else if (!oned) {
        /* IMC/IMC2D.py:1042-1047: at/below the floor the history stops in place,
         * keeping its weight (position and cell from before the event) */
        w = e.w;
        if (w <= floor_w) { st[S_FLOOR]++; frozen = true; break; }
      } else {
        w = e.w;
      }
      d1 = e.d1; d2 = e.d2; p1 = e.p1; p2 = e.p2;
      bool escaped = false;
      if (e.cross != X_NONE) {
        if (e.cross == X_IP) ++i; else if (e.cross == X_IM) --i;
        else if (e.cross == X_JP) ++j; else --j;
        int side = -1;
        if (i < 0) side = 0; else if (i >= P.nx) side = 1; else if (j < 0) side = 2; else if (j >= P.ny) side = 3;
        if (side >= 0) {
          if (in->reflect[side]) {
            if (side < 2) { d1 = -d1; i = side == 0 ? 0 : P.nx - 1; }
            else { d2 = -d2; j = side == 2 ? 0 : P.ny - 1; }
            st[S_REFLECT]++;
          } else {
            esc[side].add(w); st[S_ESCAPE]++; w = 0; dcen = 0; escaped = true;
          }
        }
        if (!escaped) c = i + P.nx * j;
      }
      if (oned && !cf && !escaped && w < floor_w) {
        /* IMC/IMC1D.py:188-195; the reference deposits only for interior cells and loses
         * the energy in the two edge cells: here every cell gets it (ledger closes). */
        st[S_FLOOR]++;
        dep[c].add(w / P.vol[c]);
        if (sa[c] > 0) si[c].add(w / dt / sa[c] / P.vol[c]);
        w = 0; dcen = 0;
      }
      if (!oned && w <= 1e-300) { w = 0; dcen = 0; }
    }
    /* a frozen history keeps the state from before its last event (IMC/IMC2D.py:1042-1051) */
    (void)frozen;
    B.w[k] = w; B.d1[k] = d1; B.d2[k] = d2; B.p1[k] = p1; B.p2[k] = p2; B.cell[k] = c;
  }
  for (int c = 0; c < nc; ++c) { out->dep[c] = 0; out->si[c] = 0; }
  for (int s = 0; s < S_N; ++s) out->stats[s] = 0;
  for (int s = 0; s < 4; ++s) out->escaped[s] = 0;
  for (int c = 0; c < nc; ++c) {
    KSum d, q;
    for (int t = 0; t < nth; ++t) { d.add(dep_t[t][c].value()); q.add(si_t[t][c].value()); }
    out->dep[c] = d.value(); out->si[c] = q.value();
  }
  for (int s = 0; s < 4; ++s) {
    KSum x;
    for (int t = 0; t < nth; ++t) x.add(esc_t[t][s].value());
    out->escaped[s] = x.value();
  }
  for (int t = 0; t < nth; ++t)
    for (int s = 0; s < S_N; ++s) out->stats[s] += st_t[t][s];
  return 0;
}

/* Vector-Jacobian product of the deposition tally with respect to the per-cell opacity
 * (2-D gray), in FP64: the estimator of the GPU adjoint kernel restated on the same
 * histories.  Per history, a first replay gives its cotangent-weighted score
 * L = sum_i a_i d_i (a = cot / V, d = deposit of event i); a second replay accumulates
 * per cell visit gp = sum s_k (a_k w_{k+1} + L_{<=k} - L) (implicit capture, path fixed)
 * and, where the scatter distance depends on sigma_s (not capped, sigma_s > 1e-12),
 * gs1 = sum (L - L_{<k}) s_k, gs2 = sum over scatters of (L - L_{<k}) (likelihood ratio),
 * and adds f^2 gp + (1 - f^2)(gs2 / sigma_s - gs1) to grad[cell] (f = sigma_a / sigma, the
 * Fleck factor).  The bank holds the step's census and sources (orc_step_transport with
 * sources_only) and is not modified.  History rules as orc_step_transport (2-D). */
int orc_adjoint_vjp(void* h, const orc_step_in* in, const double* cot, double* grad) {
  Oracle* o = (Oracle*)h;
  Problem& P = o->P;
  Bank& B = o->B;
  if (P.geom != G_XY && P.geom != G_RZ) return 2;
  const int nc = ncells(P);
  std::vector<double> sa, ss;
  fleck(P, in, sa, ss);
  const long long N = (long long)B.size();
  double wsum = 0;
  for (long long k = 0; k < N; ++k) wsum += B.w[k];
  const double floor_w = 1e-10 * wsum / (double)std::max(N, 1LL);
  int nth = in->nthreads > 0 ? in->nthreads : 1;
#ifndef _OPENMP
  nth = 1;
#endif
  std::vector<std::vector<KSum>> g_t(nth, std::vector<KSum>(nc));
  const double dt = in->dt;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nth)
  for (long long k = 0; k < N; ++k) {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    KSum* g = g_t[tid].data();
    if (!(B.w[k] > 0) || !((dt - B.t[k]) * C_LIGHT > 0)) continue;
    auto replay = [&](int phase, double Ltot) -> double {
      double w = B.w[k], d1 = B.d1[k], d2 = B.d2[k], p1 = B.p1[k], p2 = B.p2[k];
      int c = B.cell[k];
      double dcen = (dt - B.t[k]) * C_LIGHT;
      uint32_t ev = 0;
      double L = 0.0, Lc = 0.0, gp = 0.0, gs1 = 0.0, gs2 = 0.0;
      auto flush = [&](int cell) {
        if (phase == 1 && (gp != 0.0 || gs1 != 0.0 || gs2 != 0.0)) {
          const double sig = in->sigma[cell];
          const double f = sig > 0 ? sa[cell] / sig : 1.0;
          double val = f * f * gp;
          if (ss[cell] > 0 && (gs1 != 0.0 || gs2 != 0.0)) val += (1.0 - f * f) * (gs2 / ss[cell] - gs1);
          g[cell].add(val);
        }
        gp = gs1 = gs2 = 0.0;
      };
      while (dcen > 0) {
        int i = c % P.nx, j = c / P.nx;
        if (in->max_events > 0 && (long long)ev >= in->max_events) break;
        Draw4 r = draw(P.seed, (uint32_t)k, ev, in->step, oracle::TAG_TRANSPORT);
        ++ev;
        const double xl = P.e1[i], xr = P.e1[i + 1], yl = P.e2[j], yr = P.e2[j + 1];
        EventOut e = P.geom == G_XY
                         ? event_xy(w, d1, d2, p1, p2, xl, xr, yl, yr, sa[c], ss[c], dcen, r.u[0], r.u[1], r.u[2])
                         : event_rz(w, d1, d2, p1, p2, xl, xr, yl, yr, sa[c], ss[c], dcen, r.u[0], r.u[1], r.u[2]);
        const double Lcell = std::min(xr - xl, yr - yl);
        const bool scores = !(ss[c] * Lcell > 10000.0) && ss[c] > 1e-12;
        const double ac = cot[c] / P.vol[c];
        const double dd = w - e.w;
        if (phase == 0) {
          L += ac * dd;
        } else {
          const double Lprev = Lc;
          Lc += ac * dd;
          gp += e.s * (ac * e.w + Lc - Ltot);
          if (scores) {
            const double R = Ltot - Lprev;
            gs1 += R * e.s;
            if (e.evt == EV_SCATTER) gs2 += R;
          }
        }
        dcen = e.dcen;
        w = e.w;
        if (w <= floor_w) break; /* 2-D floor: the history stops */
        d1 = e.d1; d2 = e.d2; p1 = e.p1; p2 = e.p2;
        if (e.cross != X_NONE) {
          flush(c);
          if (e.cross == X_IP) ++i; else if (e.cross == X_IM) --i;
          else if (e.cross == X_JP) ++j; else --j;
          int side = -1;
          if (i < 0) side = 0; else if (i >= P.nx) side = 1; else if (j < 0) side = 2; else if (j >= P.ny) side = 3;
          if (side >= 0) {
            if (in->reflect[side]) {
              if (side < 2) { d1 = -d1; i = side == 0 ? 0 : P.nx - 1; }
              else { d2 = -d2; j = side == 2 ? 0 : P.ny - 1; }
            } else {
              w = 0; dcen = 0;
              break;
            }
          }
          c = i + P.nx * j;
        }
        if (w <= 1e-300) break;
      }
      flush(c);
      return L;
    };
    const double Ltot = replay(0, 0.0);
    replay(1, Ltot);
  }
  for (int c = 0; c < nc; ++c) {
    KSum x;
    for (int t = 0; t < nth; ++t) x.add(g_t[t][c].value());
    grad[c] = x.value();
  }
  return 0;
}

/* Stochastic comb, IMC/IMC1D.py:770-828 and IMC/IMC2D.py:1448-1511 (per cell), or
 * MG_IMC/MG_IMC2D.py:1314-1378 (per cell and group, bin = cell + ncell*group).
 *   ecen[b] = sum of live weights; desired = max(1, round_half_even(Nmax ecen/E));
 *   ew = ecen/desired; copies = floor(w/ew + xi), each of weight ew, in bank order.
 * xi: word k % 4 of Philox block (k / 4, 1, step, TAG_COMB), k the pre-comb index.
 * Sets census times to 0.
 * disc (per bin) = ecen - ecen_after.  Returns the new bank size. */
/* Stochastic comb.  flags: bit 0 = bins per (cell, group), bit 1 = each bin's copies share
 * the bin's pre-comb energy equally (MG_IMC/MG_IMC1D.py:808-820, conserve_comb_energy =
 * 'radiation').  Nmax > 0 combs to Nmax; Nmax == 0 only drops dead entries; Nmax < 0 combs
 * to |Nmax| when at least |Nmax| entries are alive, else only drops dead entries
 * (MG_IMC/MG_IMC1D.py:1194-1200).  Surviving entries start the next step at t = 0. */
long long orc_comb(void* h, long long Nmax, uint32_t step, int flags, double* disc) {
  Oracle* o = (Oracle*)h;
  Problem& P = o->P;
  Bank& B = o->B;
  const int nc = ncells(P);
  const bool per_group = (flags & 1) != 0, conserve_rad = (flags & 2) != 0;
  const int nb = per_group ? nc * P.ng : nc;
  std::vector<double> ecen(nb, 0.0), ew(nb, 0.0);
  std::vector<long long> ncopy(nb, 0);
  const long long N = (long long)B.size();
  auto bin = [&](long long k) { return per_group ? B.cell[k] + nc * B.grp[k] : B.cell[k]; };
  long long live = 0;
  {
    std::vector<KSum> acc(nb);
    for (long long k = 0; k < N; ++k) if (B.w[k] > 0) { acc[bin(k)].add(B.w[k]); ++live; }
    for (int b = 0; b < nb; ++b) ecen[b] = acc[b].value();
  }
  double E = 0;
  for (int b = 0; b < nb; ++b) E += ecen[b];
  const bool compact_only = Nmax == 0 || (Nmax < 0 && live < -Nmax);
  if (Nmax < 0) Nmax = -Nmax;
  if (!(E > 0) || compact_only) {
    Bank nbk;
    for (long long k = 0; k < N; ++k)
      if (B.w[k] > 0) nbk.push(B.w[k], B.d1[k], B.d2[k], 0.0, B.p1[k], B.p2[k], B.cell[k], B.grp[k]);
    B = nbk;
    for (int b = 0; b < nb; ++b) disc[b] = 0;
    return (long long)B.size();
  }
  for (int b = 0; b < nb; ++b) {
    if (ecen[b] > 0) {
      const double d = std::max(1.0, std::nearbyint((double)Nmax * ecen[b] / E));
      ew[b] = ecen[b] / d;
    }
  }
  Bank nbk;
  std::vector<long long> nk(N, 0);
  for (long long k = 0; k < N; ++k) {
    if (!(B.w[k] > 0)) continue;
    const int b = bin(k);
    if (!(ew[b] > 0)) continue;
    // four consecutive entries share one Philox block: entry k takes word k % 4 of block k / 4
    Draw4 r = draw(P.seed, (uint32_t)(k >> 2), 1, step, oracle::TAG_COMB);
    nk[k] = (long long)std::floor(B.w[k] / ew[b] + r.u[k & 3]);
    if (nk[k] > 0) ncopy[b] += nk[k];
  }
  std::vector<double> wout(ew);
  if (conserve_rad)
    for (int b = 0; b < nb; ++b) wout[b] = ncopy[b] > 0 ? ecen[b] / (double)ncopy[b] : 0.0;
  for (long long k = 0; k < N; ++k) {
    const int b = nk[k] > 0 ? bin(k) : 0;
    for (long long q = 0; q < nk[k]; ++q)
      nbk.push(wout[b], B.d1[k], B.d2[k], 0.0, B.p1[k], B.p2[k], B.cell[k], B.grp[k]);
  }
  B = nbk;
  /* energy after the comb in bin b is exactly ncopy * (copy weight): identical copies */
  for (int b = 0; b < nb; ++b) disc[b] = ecen[b] - (double)ncopy[b] * wout[b];
  return (long long)B.size();
}

/* position samplers, exposed for the pins against the reference's own samplers */
double orc_slab_linear(double dx, double s, double T, double xi) { return slab_linear(dx, s, T, xi); }
double orc_sphere_cdf(double r0, double r1, double a, double M, double xi) { return sphere_cdf(r0, r1, a, M, xi); }
double orc_rz_r_cdf(double r0, double r1, double a, double M, double xi) { return rz_r_cdf(r0, r1, a, M, xi); }

/* comb with caller-supplied uniforms (one per bank entry, pre-comb order, used only by
 * the pin against the reference's own seeded comb) */
long long orc_comb_with_xi(void* h, long long Nmax, const double* xi, double* disc) {
  Oracle* o = (Oracle*)h;
  Problem& P = o->P;
  Bank& B = o->B;
  const int nc = ncells(P);
  std::vector<double> ecen(nc, 0.0), after(nc, 0.0), ew(nc, 0.0);
  const long long N = (long long)B.size();
  for (long long k = 0; k < N; ++k) if (B.w[k] > 0) ecen[B.cell[k]] += B.w[k];
  double E = 0;
  for (int c = 0; c < nc; ++c) E += ecen[c];
  for (int c = 0; c < nc; ++c)
    if (ecen[c] > 0) ew[c] = ecen[c] / std::max(1.0, std::nearbyint((double)Nmax * ecen[c] / E));
  Bank nbk;
  long long live = 0;
  for (long long k = 0; k < N; ++k) {
    if (!(B.w[k] > 0)) continue;
    const double x = xi[live++];
    const int c = B.cell[k];
    if (!(ew[c] > 0)) continue;
    const long long n = (long long)std::floor(B.w[k] / ew[c] + x);
    for (long long q = 0; q < n; ++q) {
      nbk.push(ew[c], B.d1[k], B.d2[k], B.t[k], B.p1[k], B.p2[k], c, B.grp[k]);
      after[c] += ew[c];
    }
  }
  B = nbk;
  for (int c = 0; c < nc; ++c) disc[c] = ecen[c] - after[c];
  return (long long)B.size();
}

/* per-(cell, group) comb with caller-supplied uniforms (one per live entry, pre-comb
 * order), for the pin against MG_IMC/MG_IMC1D.py:746-847 _comb_mg_1d; bit 1 of flags
 * shares each bin's energy equally among its copies ('radiation') */
long long orc_comb_mg_with_xi(void* h, long long Nmax, const double* xi, int flags, double* disc) {
  Oracle* o = (Oracle*)h;
  Problem& P = o->P;
  Bank& B = o->B;
  const int nc = ncells(P), nb = nc * P.ng;
  std::vector<double> ecen(nb, 0.0), ew(nb, 0.0), wout(nb, 0.0);
  std::vector<long long> ncopy(nb, 0);
  const long long N = (long long)B.size();
  for (long long k = 0; k < N; ++k) if (B.w[k] > 0) ecen[B.cell[k] + nc * B.grp[k]] += B.w[k];
  double E = 0;
  for (int b = 0; b < nb; ++b) E += ecen[b];
  for (int b = 0; b < nb; ++b)
    if (ecen[b] > 0) ew[b] = ecen[b] / std::max(1.0, std::nearbyint((double)Nmax * ecen[b] / E));
  std::vector<long long> nk(N, 0);
  long long live = 0;
  for (long long k = 0; k < N; ++k) {
    if (!(B.w[k] > 0)) continue;
    const double x = xi[live++];
    const int b = B.cell[k] + nc * B.grp[k];
    if (!(ew[b] > 0)) continue;
    nk[k] = (long long)std::floor(B.w[k] / ew[b] + x);
    ncopy[b] += nk[k];
  }
  for (int b = 0; b < nb; ++b) wout[b] = (flags & 2) ? (ncopy[b] > 0 ? ecen[b] / (double)ncopy[b] : 0.0) : ew[b];
  Bank nbk;
  for (long long k = 0; k < N; ++k) {
    const int b = B.cell[k] + nc * B.grp[k];
    for (long long q = 0; q < nk[k]; ++q)
      nbk.push(wout[b], B.d1[k], B.d2[k], B.t[k], B.p1[k], B.p2[k], B.cell[k], B.grp[k]);
  }
  B = nbk;
  for (int b = 0; b < nb; ++b) disc[b] = ecen[b] - (double)ncopy[b] * wout[b];
  return (long long)B.size();
}

}  // extern "C"

/* =====================================================================================
 * Multigroup (MG_IMC/MG_IMC2D.py)
 * =================================================================================== */
namespace {

/* Planck fraction F(x) = (15/pi^4) * int_0^x t^3/(e^t - 1) dt: Bernoulli power series for
 * x < 1, exponential series sum_k e^{-kx}(x^3/k + 3x^2/k^2 + 6x/k^3 + 6/k^4) above (the
 * standard expansions of the incomplete Planck integral; Widger & Woodall, Bull. Amer.
 * Meteor. Soc. 57 (1976) 1217).  Stands in for the external planck_integrals module
 * (MG_IMC/MG_IMC2D.py:62) whose group fractions the step normalises anyway. */
/* sum_k e^{-kx}(x^3/k + 3x^2/k^2 + 6x/k^3 + 6/k^4) = (pi^4/15)(1 - F(x)), for x >= 1 */
double planck_tail(double x) {
  double tail = 0.0;
  const int K = (int)(2.0 + 40.0 / x);
  for (int k = K; k >= 1; --k) {
    const double kx = k * x, ik = 1.0 / k;
    tail += std::exp(-kx) * ik * (x * x * x + ik * (3.0 * x * x + ik * (6.0 * x + ik * 6.0)));
  }
  return tail;
}

double planck_F(double x) {
  const double c = 15.0 / (PI * PI * PI * PI);
  if (!(x > 0.0)) return 0.0;
  if (x < 1.0) {
    /* t^3/(e^t-1) = sum_n B_n t^(n+2)/n!; integrate term by term */
    static const double B[] = {1.0, -0.5, 1.0 / 6.0, 0.0, -1.0 / 30.0, 0.0, 1.0 / 42.0, 0.0, -1.0 / 30.0, 0.0,
                               5.0 / 66.0, 0.0, -691.0 / 2730.0, 0.0, 7.0 / 6.0, 0.0, -3617.0 / 510.0, 0.0,
                               43867.0 / 798.0, 0.0, -174611.0 / 330.0};
    double sum = 0.0, xp = x * x * x, fact = 1.0;
    for (int n = 0; n <= 20; ++n) {
      if (n > 0) fact *= n;
      if (B[n] != 0.0) sum += B[n] * xp / ((n + 3) * fact);
      xp *= x;
    }
    return c * sum;
  }
  return 1.0 - c * planck_tail(x);
}

/* F(x1) - F(x0); above x = 1 as a difference of tails, which keeps its relative precision
 * far into the Wien tail (1 - F cancels to 0 there) */
double planck_frac(double x0, double x1) {
  if (!(x1 > x0)) return 0.0;
  if (x0 >= 1.0) return 15.0 / (PI * PI * PI * PI) * (planck_tail(x0) - planck_tail(x1));
  return planck_F(x1) - planck_F(x0);
}

/* normalised group fractions b*_g of the Planck spectrum at T (sum = 1 unless T <= 0) */
void planck_fractions(const double* edges, int G, double T, double* b) {
  double tot = 0.0;
  for (int g = 0; g < G; ++g) {
    const double f = (T > 0.0) ? planck_frac(edges[g] / T, edges[g + 1] / T) : 0.0;
    b[g] = f > 0.0 ? f : 0.0;
    tot += b[g];
  }
  for (int g = 0; g < G; ++g) b[g] = tot > 0.0 ? b[g] / tot : 0.0;
}

/* mixture-of-Gammas CDF over n = 1..200 with weights 1/n^4 (MG_IMC/MG_IMC2D.py:105-107) */
struct MixCdf {
  double cdf[200];
  MixCdf() {
    double tot = 0.0;
    for (int n = 1; n <= 200; ++n) { const double d = (double)n; tot += 1.0 / (d * d * d * d); }
    double run = 0.0;
    for (int n = 1; n <= 200; ++n) { const double d = (double)n; run += 1.0 / (d * d * d * d); cdf[n - 1] = run / tot; }
  }
};
const MixCdf& mixcdf() { static MixCdf m; return m; }

/* group of a photon sampled from the Planck spectrum at T (MG_IMC/MG_IMC2D.py:202-254):
 * n from the 1/n^4 mixture, x = (sum of four Exp(1)) / n, energy T*x, group by edges */
int planck_group(double T, const double* edges, int G, double un, double u1, double u2, double u3, double u4,
                 bool below_to_last = false) {
  if (!(T > 0.0)) return 0;
  const MixCdf& m = mixcdf();
  double ns = 200.0;
  for (int i = 0; i < 200; ++i) if (un <= m.cdf[i]) { ns = (double)(i + 1); break; }
  const double x = (-std::log(u1) - std::log(u2) - std::log(u3) - std::log(u4)) / ns;
  const double f = T * x;
  /* MG_IMC/MG_IMC1D.py:180-186 assigns an energy below the lowest edge to the last group;
   * MG_IMC/MG_IMC2D.py:242-243 to the first.  Each module's rule is kept. */
  if (f < edges[0]) return below_to_last ? G - 1 : 0;
  if (f >= edges[G]) return G - 1;
  for (int g = 0; g < G; ++g) if (f >= edges[g] && f < edges[g + 1]) return g;
  return G - 1;
}

/* canonical prefix sum of n values (inclusive): 1024 contiguous segments summed in order,
 * segment offsets added in order — the order the CUDA path uses */
void canon_prefix(const double* x, long long n, double* out) {
  const long long per = (n + 1023) / 1024;
  std::vector<double> seg(1024, 0.0);
  for (int t = 0; t < 1024; ++t) {
    const long long lo = std::min((long long)t * per, n), hi = std::min(lo + per, n);
    double s = 0.0;
    for (long long i = lo; i < hi; ++i) s += x[i];
    seg[t] = s;
  }
  double off = 0.0;
  for (int t = 0; t < 1024; ++t) {
    const long long lo = std::min((long long)t * per, n), hi = std::min(lo + per, n);
    double run = off;
    for (long long i = lo; i < hi; ++i) { run += x[i]; out[i] = run; }
    off += seg[t];
  }
}

/* first index with cdf[i] > x (np.searchsorted side='right'), clamped */
int search_right(const double* cdf, int n, double x) {
  int lo = 0, hi = n;
  while (lo < hi) { const int mid = (lo + hi) >> 1; if (cdf[mid] <= x) lo = mid + 1; else hi = mid; }
  return std::min(lo, n - 1);
}
/* first index with cdf[i] >= x */
int search_left(const double* cdf, int n, double x) {
  int lo = 0, hi = n;
  while (lo < hi) { const int mid = (lo + hi) >> 1; if (cdf[mid] < x) lo = mid + 1; else hi = mid; }
  return std::min(lo, n - 1);
}

}  // namespace

extern "C" {

double orc_planck_F(double x) { return planck_F(x); }
void orc_planck_fractions(const double* edges, int G, double T, double* b) { planck_fractions(edges, G, T, b); }
int orc_planck_group(double T, const double* edges, int G, const double* u) {
  return planck_group(T, edges, G, u[0], u[1], u[2], u[3], u[4]);
}
int orc_planck_group_mg1d(double T, const double* edges, int G, const double* u) {
  return planck_group(T, edges, G, u[0], u[1], u[2], u[3], u[4], true);
}

typedef struct {
  uint32_t step;
  double dt, theta;
  const double* T;          /* [c] */
  const double* sigma;      /* [g][c] true absorption opacity */
  const double* cv;         /* [c] */
  long long Ntarget, Nboundary, Nsource;
  const double* source;     /* [g][c] power density or NULL */
  const double* face_T[4];
  int reflect[4];
  long long max_events;
  const double* emission_fractions;  /* [g] or NULL */
  const double* group_edges;         /* [G+1] */
  double T_emit_floor;
  int nthreads;
  int sources_only;
} orc_mg_in;

typedef struct {
  double* dep; double* si;         /* [g][c] */
  double* emitted;                 /* [c] */
  double* sigma_a; double* sigma_s;/* [g][c] */
  double* bnd_by_group;            /* [g] */
  double* esc_by_group;            /* [g] */
  double boundary_emission, source_emission, emission_total;
  double bnd_by_side[4];
  double escaped[4];
  long long stats[S_N];
  long long n_transported;
  double weight_floor;
} orc_mg_out;

/* multigroup initial census, MG_IMC/MG_IMC2D.py:992-1097: N particles of equal weight
 * E/N, cell ~ a Tr^4 V, position uniform in the cell, isotropic, time 0, group from the
 * Planck spectrum at the local Tr.  Draws: k, blocks 0-2, step 0, TAG_IC. */
long long orc_init_ic_mg(void* h, long long N, const double* Tr, const double* edges, double T_emit_floor) {
  Oracle* o = (Oracle*)h;
  Problem& P = o->P;
  Bank& B = o->B;
  B.resize(0);
  const int nc = ncells(P), G = P.ng;
  std::vector<double> E(nc), cdf(nc);
  for (int c = 0; c < nc; ++c) {
    E[c] = A_RAD * pow4(Tr[c]) * P.vol[c];
    if (T_emit_floor > 0 && Tr[c] < T_emit_floor) E[c] = 0;
  }
  canon_prefix(E.data(), nc, cdf.data());
  const double Et = cdf[nc - 1];
  if (N <= 0 || !(Et > 0)) return 0;
  const double wgt = Et / (double)N;
  for (long long k = 0; k < N; ++k) {
    Draw4 a = draw(P.seed, (uint32_t)k, 0, 0, oracle::TAG_IC);
    Draw4 b = draw(P.seed, (uint32_t)k, 1, 0, oracle::TAG_IC);
    Draw4 d = draw(P.seed, (uint32_t)k, 2, 0, oracle::TAG_IC);
    const int c = search_right(cdf.data(), nc, a.u[0] * Et);
    const int i = c % P.nx, j = c / P.nx;
    const double e1a = P.e1[i], e1b = P.e1[i + 1], e2a = P.e2[j], e2b = P.e2[j + 1];
    double p1, p2 = e2a + a.u[2] * (e2b - e2a), d1, d2;
    if (P.geom == G_RZ) p1 = std::sqrt(e1a * e1a + a.u[1] * (e1b * e1b - e1a * e1a));
    else p1 = e1a + a.u[1] * (e1b - e1a);
    iso_dir(P.geom, a.u[3], b.u[0], d1, d2);
    const int g = planck_group(Tr[c], edges, G, b.u[1], b.u[2], b.u[3], d.u[0], d.u[1]);
    B.push(wgt, d1, d2, 0.0, p1, p2, c, g);
  }
  return (long long)B.size();
}

int orc_step_transport_mg(void* h, const orc_mg_in* in, orc_mg_out* out) {
  Oracle* o = (Oracle*)h;
  Problem& P = o->P;
  Bank& B = o->B;
  const int nc = ncells(P), G = P.ng;
  const double* edges = in->group_edges;
  /* Fleck factor with the Planck-mean opacity, MG_IMC/MG_IMC2D.py:1703-1719 */
  std::vector<double> bstar((size_t)G * nc), sa((size_t)G * nc), ss((size_t)G * nc), b(G);
  for (int c = 0; c < nc; ++c) {
    planck_fractions(edges, G, in->T[c], b.data());
    double sp = 0.0;
    for (int g = 0; g < G; ++g) { bstar[(size_t)g * nc + c] = b[g]; sp += in->sigma[(size_t)g * nc + c] * b[g]; }
    const double T = in->T[c];
    const double beta = 4.0 * A_RAD * pow3(T) / in->cv[c];
    double f = 1.0 / (1.0 + in->theta * beta * sp * C_LIGHT * in->dt);
    f = std::min(1.0, std::max(0.0, f));
    for (int g = 0; g < G; ++g) {
      const size_t q = (size_t)g * nc + c;
      ss[q] = in->sigma[q] * (1.0 - f);
      sa[q] = in->sigma[q] * f;
    }
  }
  std::copy(sa.begin(), sa.end(), out->sigma_a);
  std::copy(ss.begin(), ss.end(), out->sigma_s);
  for (int g = 0; g < G; ++g) { out->bnd_by_group[g] = 0; out->esc_by_group[g] = 0; }
  for (int q = 0; q < 4; ++q) { out->bnd_by_side[q] = 0; out->escaped[q] = 0; }

  /* ---- boundary: the gray face sampling plus a Planck group at the face cell's T ---- */
  double bnd_total = 0.0;
  for (int side = 0; side < 4; ++side) {
    const double* Tf = in->face_T[side];
    if (!Tf || in->Nboundary <= 0) continue;
    const bool along2 = side < 2;
    const int nf = along2 ? P.ny : P.nx;
    std::vector<double> Ef(nf), cdf(nf);
    double Et = 0;
    for (int q = 0; q < nf; ++q) {
      double area;
      if (P.geom == G_XY) area = along2 ? (P.e2[q + 1] - P.e2[q]) : (P.e1[q + 1] - P.e1[q]);
      else if (along2) { const double R = side == 0 ? P.e1[0] : P.e1[P.nx]; area = 2.0 * PI * R * (P.e2[q + 1] - P.e2[q]); }
      else area = PI * (P.e1[q + 1] * P.e1[q + 1] - P.e1[q] * P.e1[q]);
      const double T = Tf[q];
      Ef[q] = (T > 0) ? A_RAD * C_LIGHT * T * T * T * T / 4.0 * area * in->dt : 0.0;
      Et += Ef[q];
      cdf[q] = Et;
    }
    if (!(Et > 0)) continue;
    const long long n = in->Nboundary;
    const double wgt = Et / (double)n;
    for (long long k = 0; k < n; ++k) {
      Draw4 a = draw(P.seed, (uint32_t)k, 0, in->step, oracle::TAG_BOUNDARY | side);
      Draw4 bb = draw(P.seed, (uint32_t)k, 1, in->step, oracle::TAG_BOUNDARY | side);
      Draw4 d = draw(P.seed, (uint32_t)k, 2, in->step, oracle::TAG_BOUNDARY | side);
      int q = (int)(std::lower_bound(cdf.begin(), cdf.end(), a.u[0] * Et) - cdf.begin());
      q = std::min(q, nf - 1);
      while (Ef[q] <= 0 && q > 0) --q;
      const double mu_n = std::sqrt(a.u[2]);
      const double t = bb.u[0] * in->dt;
      double p1, p2, d1, d2;
      int i, j;
      if (P.geom == G_XY) {
        const double mu_t = std::sqrt(std::max(0.0, 1.0 - mu_n * mu_n));
        const double ct = mu_t * std::cos(2.0 * PI * a.u[3]);
        if (along2) {
          j = q; i = side == 0 ? 0 : P.nx - 1;
          p1 = side == 0 ? P.e1[0] : P.e1[P.nx];
          p2 = P.e2[q] + a.u[1] * (P.e2[q + 1] - P.e2[q]);
          d1 = side == 0 ? mu_n : -mu_n; d2 = ct;
        } else {
          i = q; j = side == 2 ? 0 : P.ny - 1;
          p2 = side == 2 ? P.e2[0] : P.e2[P.ny];
          p1 = P.e1[q] + a.u[1] * (P.e1[q + 1] - P.e1[q]);
          d2 = side == 2 ? mu_n : -mu_n; d1 = ct;
        }
      } else {
        if (along2) {
          j = q; i = side == 0 ? 0 : P.nx - 1;
          p1 = side == 0 ? P.e1[0] : P.e1[P.nx];
          p2 = P.e2[q] + a.u[1] * (P.e2[q + 1] - P.e2[q]);
          d1 = side == 0 ? mu_n : -mu_n; d2 = 2.0 * a.u[3] - 1.0;
        } else {
          i = q; j = side == 2 ? 0 : P.ny - 1;
          const double r0 = P.e1[q], r1 = P.e1[q + 1];
          p1 = std::sqrt(r0 * r0 + a.u[1] * (r1 * r1 - r0 * r0));
          p2 = side == 2 ? P.e2[0] : P.e2[P.ny];
          d2 = side == 2 ? mu_n : -mu_n; d1 = std::cos(2.0 * PI * a.u[3]);
        }
      }
      const int g = planck_group(Tf[q], edges, G, bb.u[1], bb.u[2], bb.u[3], d.u[0], d.u[1]);
      B.push(wgt, d1, d2, t, p1, p2, i + P.nx * j, g);
      out->bnd_by_group[g] += wgt;
      out->bnd_by_side[side] += wgt;
      bnd_total += wgt;
    }
  }
  out->boundary_emission = bnd_total;

  /* ---- categorical volume sources: cell ~ sum_g E_gc, group ~ E_gc, equal weights ----
   * (fixed source MG_IMC/MG_IMC2D.py:1098-1170; emission :1866-1943) */
  auto categorical = [&](const std::vector<double>& Egc, long long N, uint32_t tag) -> double {
    std::vector<double> Ec(nc, 0.0), cdf(nc);
    for (int c = 0; c < nc; ++c) { double s2 = 0.0; for (int g = 0; g < G; ++g) s2 += Egc[(size_t)g * nc + c]; Ec[c] = s2; }
    canon_prefix(Ec.data(), nc, cdf.data());
    const double Et = cdf[nc - 1];
    if (!(Et > 0) || N <= 0) return 0.0;
    const double wgt = Et / (double)N;
    std::vector<double> gc(G);
    for (long long k = 0; k < N; ++k) {
      Draw4 a = draw(P.seed, (uint32_t)k, 0, in->step, tag);
      Draw4 bb = draw(P.seed, (uint32_t)k, 1, in->step, tag);
      const int c = search_right(cdf.data(), nc, a.u[0] * Et);
      double run = 0.0;
      for (int g = 0; g < G; ++g) { run += Egc[(size_t)g * nc + c]; gc[g] = run; }
      const int g = search_left(gc.data(), G, a.u[1] * run);
      const int i = c % P.nx, j = c / P.nx;
      const double e1a = P.e1[i], e1b = P.e1[i + 1], e2a = P.e2[j], e2b = P.e2[j + 1];
      double p1 = P.geom == G_RZ ? std::sqrt(e1a * e1a + a.u[2] * (e1b * e1b - e1a * e1a)) : e1a + a.u[2] * (e1b - e1a);
      const double p2 = e2a + a.u[3] * (e2b - e2a);
      double d1, d2;
      iso_dir(P.geom, bb.u[0], bb.u[1], d1, d2);
      B.push(wgt, d1, d2, bb.u[2] * in->dt, p1, p2, c, g);
    }
    return wgt * (double)N;
  };
  out->source_emission = 0.0;
  if (in->source && in->Nsource > 0) {
    std::vector<double> Sgc((size_t)G * nc);
    for (int g = 0; g < G; ++g)
      for (int c = 0; c < nc; ++c) Sgc[(size_t)g * nc + c] = in->source[(size_t)g * nc + c] * P.vol[c] * in->dt;
    out->source_emission = categorical(Sgc, in->Nsource, oracle::TAG_SOURCE);
  }
  std::vector<double> Egc((size_t)G * nc, 0.0);
  for (int c = 0; c < nc; ++c) {
    const double T = in->T[c];
    if (in->T_emit_floor > 0 && T < in->T_emit_floor) continue;
    const double aT4 = A_RAD * C_LIGHT * pow4(T) * in->dt * P.vol[c];
    for (int g = 0; g < G; ++g) {
      const size_t q = (size_t)g * nc + c;
      const double bg = in->emission_fractions ? in->emission_fractions[g] : bstar[q];
      Egc[q] = sa[q] * bg * aT4;
    }
  }
  double Eemit = 0.0;
  for (int c = 0; c < nc; ++c) { out->emitted[c] = 0.0; for (int g = 0; g < G; ++g) out->emitted[c] += Egc[(size_t)g * nc + c]; Eemit += out->emitted[c]; }
  out->emission_total = 0.0;
  if (in->Ntarget > 0) {
    const double issued = categorical(Egc, in->Ntarget, oracle::TAG_EMISSION);
    /* matter loses E_c scaled so the total is exactly the issued particle energy */
    const double scale = Eemit > 0 ? issued / Eemit : 0.0;
    for (int c = 0; c < nc; ++c) out->emitted[c] *= scale;
    out->emission_total = issued;
  } else {
    for (int c = 0; c < nc; ++c) out->emitted[c] = 0.0;
  }
  if (in->sources_only) return 0;

  /* ---- transport, MG_IMC/MG_IMC2D.py:774-989 ---- */
  const long long N = (long long)B.size();
  double wsum = 0;
  for (long long k = 0; k < N; ++k) wsum += B.w[k];
  const double floor_w = 1e-10 * wsum / (double)std::max(N, 1LL);
  out->weight_floor = floor_w;
  out->n_transported = N;
  int nth = in->nthreads > 0 ? in->nthreads : 1;
#ifndef _OPENMP
  nth = 1;
#endif
  const size_t ncg = (size_t)nc * G;
  std::vector<std::vector<KSum>> dep_t(nth, std::vector<KSum>(ncg)), si_t(nth, std::vector<KSum>(ncg));
  std::vector<std::vector<long long>> st_t(nth, std::vector<long long>(S_N, 0));
  std::vector<std::vector<KSum>> esc_t(nth, std::vector<KSum>(4 + G));
  const double dt = in->dt;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nth)
  for (long long k = 0; k < N; ++k) {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    KSum* dep = dep_t[tid].data();
    KSum* si = si_t[tid].data();
    long long* st = st_t[tid].data();
    KSum* esc = esc_t[tid].data();
    double w = B.w[k], d1 = B.d1[k], d2 = B.d2[k], p1 = B.p1[k], p2 = B.p2[k];
    int c = B.cell[k];
    const int g = B.grp[k];
    if (!(w > floor_w)) continue;  /* reference: skipped without an event */
    double dcen = (dt - B.t[k]) * C_LIGHT;
    uint32_t ev = 0;
    while (dcen > 0) {
      if (in->max_events > 0 && (long long)ev >= in->max_events) { st[S_CAP]++; break; }
      int i = c % P.nx, j = c / P.nx;
      const size_t q = (size_t)g * nc + c;
      Draw4 r = draw(P.seed, (uint32_t)k, ev, in->step, oracle::TAG_TRANSPORT);
      ++ev;
      st[S_EVENTS]++;
      /* MG events: no effective-scatter cap (MG_IMC/MG_IMC2D.py:601-604) */
      EventOut e;
      if (P.geom == G_XY) e = event_xy(w, d1, d2, p1, p2, P.e1[i], P.e1[i + 1], P.e2[j], P.e2[j + 1], sa[q], ss[q], dcen, r.u[0], r.u[1], r.u[2], false);
      else e = event_rz(w, d1, d2, p1, p2, P.e1[i], P.e1[i + 1], P.e2[j], P.e2[j + 1], sa[q], ss[q], dcen, r.u[0], r.u[1], r.u[2], false);
      if (e.evt == EV_BOUNDARY) st[S_BOUNDARY]++; else if (e.evt == EV_SCATTER) st[S_SCATTER]++; else st[S_CENSUS]++;
      if (sa[q] > 1e-12) {
        dep[q].add(e.dep / P.vol[c]);
        si[q].add(e.dep_i / (dt * P.vol[c]));
      } else {
        si[q].add(w * (dcen - e.dcen) / (dt * P.vol[c]));
        e.w = w;  /* no absorption below the threshold */
      }
      w = e.w; d1 = e.d1; d2 = e.d2; p1 = e.p1; p2 = e.p2; dcen = e.dcen;
      if (e.cross != X_NONE) {
        if (e.cross == X_IP) ++i; else if (e.cross == X_IM) --i; else if (e.cross == X_JP) ++j; else --j;
        int side = -1;
        if (i < 0) side = 0; else if (i >= P.nx) side = 1; else if (j < 0) side = 2; else if (j >= P.ny) side = 3;
        if (side >= 0) {
          if (in->reflect[side]) {
            /* the reference does not reset the index after a -dir1 reflection
             * (MG_IMC/MG_IMC2D.py:916-919): here the particle stays in cell 0 */
            if (side < 2) { d1 = -d1; i = side == 0 ? 0 : P.nx - 1; }
            else { d2 = -d2; j = side == 2 ? 0 : P.ny - 1; }
            st[S_REFLECT]++;
          } else {
            esc[side].add(w); esc[4 + g].add(w); st[S_ESCAPE]++;
            w = 0; dcen = 0;
          }
        }
        if (w > 0) c = i + P.nx * j;
      }
      /* MG_IMC/MG_IMC2D.py:858-860: the next event's floor test stops the history; an
       * escape set dcen = 0 and a weight that underflowed to 0 is at the floor too */
      if (dcen > 0 && w <= floor_w) { st[S_FLOOR]++; break; }
    }
    B.w[k] = w; B.d1[k] = d1; B.d2[k] = d2; B.p1[k] = p1; B.p2[k] = p2; B.cell[k] = c;
  }
  for (size_t q = 0; q < ncg; ++q) {
    KSum d, s2;
    for (int t = 0; t < nth; ++t) { d.add(dep_t[t][q].value()); s2.add(si_t[t][q].value()); }
    out->dep[q] = d.value(); out->si[q] = s2.value();
  }
  for (int s2 = 0; s2 < S_N; ++s2) { out->stats[s2] = 0; for (int t = 0; t < nth; ++t) out->stats[s2] += st_t[t][s2]; }
  for (int q = 0; q < 4 + G; ++q) {
    KSum x;
    for (int t = 0; t < nth; ++t) x.add(esc_t[t][q].value());
    if (q < 4) out->escaped[q] = x.value(); else out->esc_by_group[q - 4] = x.value();
  }
  return 0;
}

}  // extern "C"

/* =====================================================================================
 * Multigroup 1-D sphere (MG_IMC/MG_IMC1D.py)
 *
 * Sources are stratified per (group, cell) bin, bins in the reference's g-outer / i-inner
 * order: n_b = max(1, round(N E_b / E)) for emitting bins (fixed source: round, no
 * minimum), weight E_b / n_b, radius uniform in the shell's volume, mu ~ U(-1, 1).
 * Tracking is the gray spherical event with group-indexed opacities, the sigma_s*dr > 1e4
 * cap, a weight floor of 1e-14 * sum(w) / N and the floor kill after every event.
 * Draws per particle k of a source: blocks 0 (radius, -, direction, -) and 1 (time, then
 * the Planck group sampler's five uniforms with block 2 for the IC).
 * =================================================================================== */
namespace {

/* stratified (group, cell) counts; minimum one per positive bin when min1 */
long long strat_counts(const std::vector<double>& E, long long N, bool min1, std::vector<long long>& n) {
  const long long nb = (long long)E.size();
  n.assign(nb, 0);
  const double Et = canon_sum(E.data(), nb);
  if (N <= 0 || !(Et > 0)) return 0;
  long long tot = 0;
  for (long long b = 0; b < nb; ++b) {
    if (!(E[b] > 0)) continue;
    const double r = std::nearbyint((double)N * E[b] / Et);
    n[b] = min1 ? std::max(1LL, (long long)r) : std::max(0LL, (long long)r);
    tot += n[b];
  }
  return tot;
}

/* append the particles of stratified bins (b = g*nc + c); returns the energy issued */
double strat_fill(const Problem& P, const std::vector<double>& E, const std::vector<long long>& n, double dt,
                  uint32_t step, uint32_t tag, Bank& B) {
  const int nc = ncells(P);
  double total = 0.0;
  uint32_t k = 0;
  for (size_t b = 0; b < E.size(); ++b) {
    if (n[b] <= 0) continue;
    const int g = (int)(b / nc), c = (int)(b % nc);
    const double wgt = E[b] / (double)n[b];
    const double r0 = P.e1[c], r1 = P.e1[c + 1];
    for (long long q = 0; q < n[b]; ++q, ++k) {
      Draw4 r = draw(P.seed, k, 0, step, tag);
      Draw4 s = draw(P.seed, k, 1, step, tag);
      double p1 = std::cbrt(r0 * r0 * r0 + (r1 * r1 * r1 - r0 * r0 * r0) * r.u[0]);
      p1 = std::min(std::max(p1, r0), r1);
      B.push(wgt, 2.0 * r.u[2] - 1.0, 0.0, s.u[0] * dt, p1, 0.0, c, g);
      total += wgt;
    }
  }
  return total;
}

}  // namespace

extern "C" {

/* initial census, MG_IMC/MG_IMC1D.py:514-566: per shell max(1, round(N E_i / E)) particles
 * of weight E_i / n_i (E_i = a Tr^4 V, zero below T_emit_floor), group from the Planck
 * spectrum at the shell's Tr.  Draws: k, blocks 0-2, step 0, TAG_IC. */
long long orc_init_ic_mg1d(void* h, long long N, const double* Tr, const double* edges, double T_emit_floor) {
  Oracle* o = (Oracle*)h;
  Problem& P = o->P;
  Bank& B = o->B;
  B.resize(0);
  const int nc = ncells(P), G = P.ng;
  std::vector<double> E(nc);
  for (int c = 0; c < nc; ++c) {
    E[c] = A_RAD * pow4(Tr[c]) * P.vol[c];
    if (T_emit_floor > 0 && Tr[c] < T_emit_floor) E[c] = 0;
  }
  std::vector<long long> n;
  strat_counts(E, N, true, n);
  uint32_t k = 0;
  for (int c = 0; c < nc; ++c) {
    if (n[c] <= 0) continue;
    const double wgt = E[c] / (double)n[c];
    const double r0 = P.e1[c], r1 = P.e1[c + 1];
    for (long long q = 0; q < n[c]; ++q, ++k) {
      Draw4 r = draw(P.seed, k, 0, 0, oracle::TAG_IC);
      Draw4 s = draw(P.seed, k, 1, 0, oracle::TAG_IC);
      Draw4 d = draw(P.seed, k, 2, 0, oracle::TAG_IC);
      double p1 = std::cbrt(r0 * r0 * r0 + (r1 * r1 * r1 - r0 * r0 * r0) * r.u[0]);
      p1 = std::min(std::max(p1, r0), r1);
      const int g = planck_group(Tr[c], edges, G, s.u[1], s.u[2], s.u[3], d.u[0], d.u[1], true);
      B.push(wgt, 2.0 * r.u[2] - 1.0, 0.0, 0.0, p1, 0.0, c, g);
    }
  }
  return (long long)B.size();
}

/* one MG_IMC1D step up to the material update (MG_IMC/MG_IMC1D.py:917-1140):
 * Fleck with the Planck-mean opacity, boundary (inner, outer) | fixed source | emission,
 * then transport (MG_IMC/MG_IMC1D.py:367-461).  source is [g][c] (a gray source is
 * placed in group 0 by the caller, as the reference does). */
int orc_step_transport_mg1d(void* h, const orc_mg_in* in, orc_mg_out* out) {
  Oracle* o = (Oracle*)h;
  Problem& P = o->P;
  Bank& B = o->B;
  if (P.geom != G_SPHERE) return 2;
  const int nc = ncells(P), G = P.ng;
  const size_t ncg = (size_t)nc * G;
  const double* edges = in->group_edges;
  std::vector<double> bstar(ncg), sa(ncg), ss(ncg), b(G);
  for (int c = 0; c < nc; ++c) {
    planck_fractions(edges, G, in->T[c], b.data());
    double sp = 0.0;
    for (int g = 0; g < G; ++g) { bstar[(size_t)g * nc + c] = b[g]; sp += in->sigma[(size_t)g * nc + c] * b[g]; }
    const double T = in->T[c];
    const double beta = 4.0 * A_RAD * pow3(T) / in->cv[c];
    double f = 1.0 / (1.0 + in->theta * beta * sp * C_LIGHT * in->dt);
    f = std::min(1.0, std::max(0.0, f));
    for (int g = 0; g < G; ++g) {
      const size_t q = (size_t)g * nc + c;
      sa[q] = in->sigma[q] * f;
      ss[q] = in->sigma[q] * (1.0 - f);
    }
  }
  std::copy(sa.begin(), sa.end(), out->sigma_a);
  std::copy(ss.begin(), ss.end(), out->sigma_s);
  for (int g = 0; g < G; ++g) { out->bnd_by_group[g] = 0; out->esc_by_group[g] = 0; }
  for (int q = 0; q < 4; ++q) { out->bnd_by_side[q] = 0; out->escaped[q] = 0; }

  /* ---- boundary, MG_IMC/MG_IMC1D.py:653-676: a c T^4 / 4 * 4 pi R^2 * dt on the inner
   * (outward) and outer (inward) sphere, half-Lambertian, Planck group at the face T ---- */
  double bnd_total = 0.0;
  for (int side = 0; side < 2; ++side) {
    const double* Tf = in->face_T[side];
    if (!Tf || in->Nboundary <= 0) continue;
    const double R = side == 0 ? P.e1[0] : P.e1[P.nx];
    const double T = Tf[0];
    const double Et = (T > 0) ? A_RAD * C_LIGHT * T * T * T * T / 4.0 * (4.0 * PI * R * R) * in->dt : 0.0;
    if (!(Et > 0)) continue;
    const long long n = in->Nboundary;
    const double wgt = Et / (double)n;
    for (long long k = 0; k < n; ++k) {
      Draw4 a = draw(P.seed, (uint32_t)k, 0, in->step, oracle::TAG_BOUNDARY | side);
      Draw4 bb = draw(P.seed, (uint32_t)k, 1, in->step, oracle::TAG_BOUNDARY | side);
      Draw4 d = draw(P.seed, (uint32_t)k, 2, in->step, oracle::TAG_BOUNDARY | side);
      const double mu_n = std::sqrt(a.u[2]);
      const int g = planck_group(T, edges, G, bb.u[1], bb.u[2], bb.u[3], d.u[0], d.u[1], true);
      B.push(wgt, side == 0 ? mu_n : -mu_n, 0.0, bb.u[0] * in->dt, R, 0.0, side == 0 ? 0 : P.nx - 1, g);
      out->bnd_by_group[g] += wgt;
      out->bnd_by_side[side] += wgt;
      bnd_total += wgt;
    }
  }
  out->boundary_emission = bnd_total;

  /* ---- fixed source, MG_IMC/MG_IMC1D.py:679-743 (only when max(source) > 0) ---- */
  out->source_emission = 0.0;
  if (in->source && in->Nsource > 0) {
    double smax = 0.0;
    for (size_t q = 0; q < ncg; ++q) smax = std::max(smax, in->source[q]);
    if (smax > 0) {
      std::vector<double> QV(ncg);
      for (int g = 0; g < G; ++g)
        for (int c = 0; c < nc; ++c) QV[(size_t)g * nc + c] = in->source[(size_t)g * nc + c] * P.vol[c] * in->dt;
      std::vector<long long> n;
      strat_counts(QV, in->Nsource, false, n);
      out->source_emission = strat_fill(P, QV, n, in->dt, in->step, oracle::TAG_SOURCE, B);
    }
  }

  /* ---- emission, MG_IMC/MG_IMC1D.py:569-650 ---- */
  std::vector<double> Egc(ncg, 0.0);
  for (int c = 0; c < nc; ++c) {
    const double T = in->T[c];
    if (in->T_emit_floor > 0 && T < in->T_emit_floor) continue;
    for (int g = 0; g < G; ++g) {
      const size_t q = (size_t)g * nc + c;
      Egc[q] = A_RAD * C_LIGHT * pow4(T) * sa[q] * bstar[q] * in->dt * P.vol[c];
    }
  }
  for (int c = 0; c < nc; ++c) out->emitted[c] = 0.0;
  out->emission_total = 0.0;
  if (in->Ntarget > 0) {
    std::vector<long long> n;
    strat_counts(Egc, in->Ntarget, true, n);
    const size_t n0 = B.size();
    out->emission_total = strat_fill(P, Egc, n, in->dt, in->step, oracle::TAG_EMISSION, B);
    std::vector<KSum> em(nc);
    for (size_t k = n0; k < B.size(); ++k) em[B.cell[k]].add(B.w[k]);
    for (int c = 0; c < nc; ++c) out->emitted[c] = em[c].value();
  }
  if (in->sources_only) return 0;

  /* ---- transport, MG_IMC/MG_IMC1D.py:367-461; weight floor :1127 ---- */
  const long long N = (long long)B.size();
  double wsum = 0;
  for (long long k = 0; k < N; ++k) wsum += B.w[k];
  const double floor_w = 1e-14 * wsum / (double)std::max(N, 1LL);
  out->weight_floor = floor_w;
  out->n_transported = N;
  int nth = in->nthreads > 0 ? in->nthreads : 1;
#ifndef _OPENMP
  nth = 1;
#endif
  std::vector<std::vector<KSum>> dep_t(nth, std::vector<KSum>(ncg)), si_t(nth, std::vector<KSum>(ncg));
  std::vector<std::vector<long long>> st_t(nth, std::vector<long long>(S_N, 0));
  std::vector<std::vector<KSum>> esc_t(nth, std::vector<KSum>(4 + G));
  const double dt = in->dt;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nth)
  for (long long k = 0; k < N; ++k) {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    KSum* dep = dep_t[tid].data();
    KSum* si = si_t[tid].data();
    long long* st = st_t[tid].data();
    KSum* esc = esc_t[tid].data();
    double w = B.w[k], mu = B.d1[k], r = B.p1[k];
    int c = B.cell[k];
    const int g = B.grp[k];
    /* a zero-weight entry carries nothing (the reference moves it without effect) */
    if (!(w > 0)) continue;
    double dcen = (dt - B.t[k]) * C_LIGHT;
    uint32_t ev = 0;
    while (dcen > 0) {
      const size_t q = (size_t)g * nc + c;
      Draw4 u = draw(P.seed, (uint32_t)k, ev, in->step, oracle::TAG_TRANSPORT);
      ++ev;
      st[S_EVENTS]++;
      EventOut e = event_sphere(w, mu, r, P.e1[c], P.e1[c + 1], sa[q], ss[q], dcen, u.u[0], u.u[1]);
      if (e.evt == EV_BOUNDARY) st[S_BOUNDARY]++; else if (e.evt == EV_SCATTER) st[S_SCATTER]++; else st[S_CENSUS]++;
      dep[q].add(e.dep);
      si[q].add(e.dep_i / dt);
      w = e.w; mu = e.d1; r = e.p1; dcen = e.dcen;
      bool escaped = false;
      if (e.cross != X_NONE) {
        int i = c + (e.cross == X_IP ? 1 : -1);
        const int side = i < 0 ? 0 : (i >= P.nx ? 1 : -1);
        if (side >= 0) {
          if (in->reflect[side]) { mu = -mu; i = side == 0 ? 0 : P.nx - 1; st[S_REFLECT]++; }
          else { esc[side].add(w); esc[4 + g].add(w); st[S_ESCAPE]++; w = 0; dcen = 0; escaped = true; }
        }
        if (!escaped) c = i;
      }
      if (!escaped && w < floor_w) {
        /* MG_IMC/MG_IMC1D.py:439-452: kill, the remainder deposited in the current shell */
        const size_t q2 = (size_t)g * nc + c;
        st[S_FLOOR]++;
        dep[q2].add(w / P.vol[c]);
        if (sa[q2] > 1e-10) si[q2].add(w / dt / sa[q2] / P.vol[c]);
        w = 0; dcen = 0;
      }
    }
    B.w[k] = w; B.d1[k] = mu; B.p1[k] = r; B.cell[k] = c;
  }
  for (size_t q = 0; q < ncg; ++q) {
    KSum d, s2;
    for (int t = 0; t < nth; ++t) { d.add(dep_t[t][q].value()); s2.add(si_t[t][q].value()); }
    out->dep[q] = d.value(); out->si[q] = s2.value();
  }
  for (int s2 = 0; s2 < S_N; ++s2) { out->stats[s2] = 0; for (int t = 0; t < nth; ++t) out->stats[s2] += st_t[t][s2]; }
  for (int q = 0; q < 4 + G; ++q) {
    KSum x;
    for (int t = 0; t < nth; ++t) x.add(esc_t[t][q].value());
    if (q < 4) out->escaped[q] = x.value(); else out->esc_by_group[q - 4] = x.value();
  }
  return 0;
}

}  // extern "C"
