// Native host side of the rank-adaptive BUG step: `cbe_bug_step!` run inside the library.
//
// The whole step -- half-sweeps, DD-QR controlled bond expansion, local Krylov enrichment, the
// order-p closure, the root exponential and the budgeted compression -- is driven from C++ over
// the engine's planners (engine.h), so a step costs kernel launches and the host syncs its
// rank decisions need, and no interpreter overhead. The step follows the reference in order:
//   cbe_bug_step!            src/BUG/TimeEvolution/bug_step.jl:17-513
//   _half_left!/_half_right! src/BUG/Core/Sweeps/half_sweeps.jl:218-410
//   dd_cbe_expand            src/BUG/Randomised/dd_cbe_expand.jl:19-419 (:rank_tail, :adaptive)
//   _dd_controller           src/BUG/Randomised/dd_cbe_controller.jl:26-212
//   _krylov_enrich           src/BUG/Core/RankAdaptation/krylov_enrichment.jl:58-307
//   lanczos/arnoldi chains   krylov_lanczos.jl:18-71, krylov_arnoldi.jl:13-58
//   _single_pass_closure!    krylov_closure_loop.jl:203-281, frontier_closure.jl:42-222,
//                            frontier_sweeps.jl:20-354, krylov_frontier_bonds.jl:13-106
//   expv                     src/BUG/Core/LocalSolvers/krylov.jl:128-442, root_methods.jl:94-402
//   truncate_recursive!      truncation.jl:49-158; _assemble_and_compress! diagnostics.jl:269-337
//   basis budget / ledger    src/BUG/Core/RankAdaptation/basis_budget.jl:12-568
// Gaussian probes are drawn on the host through a caller-supplied callback (the caller's seeded
// generator), in the order documented in include/bug_b200.h, and uploaded.
#include "engine.h"
#include "smallla.h"

#include <complex>
#include <exception>
#include <limits>
#include <numeric>
#include <set>
#include <thread>

namespace bugs {

using namespace bugi;
using cd = std::complex<double>;
using T = std::shared_ptr<bug_tensor>;
using smallla::CMat;
using smallla::RMat;

constexpr double EPS = 2.220446049250313e-16;
constexpr double CBE_EPS = 100 * EPS;

// _tridiag_eigen's check (krylov.jl:77-86): a non-finite Lanczos coefficient comes from the input
// vector or the operator, not from the eigensolver, and is reported as such (BUG_ENONFINITE)
// instead of as a convergence failure.
inline void require_finite_tridiag(const double* alpha, size_t na, const double* beta, size_t nb) {
  size_t ca = 0, cb = 0;
  for (size_t i = 0; i < na; ++i) ca += !std::isfinite(alpha[i]);
  for (size_t i = 0; i < nb; ++i) cb += !std::isfinite(beta[i]);
  if (ca || cb)
    throw BugError(BUG_ENONFINITE, "Lanczos tridiagonal has non-finite entries (" + std::to_string(ca) +
                                       " of " + std::to_string(na) + " alpha, " + std::to_string(cb) +
                                       " of " + std::to_string(nb) +
                                       " beta): the input vector or the operator is not finite");
}
constexpr double KRY_BREAKDOWN = 1e-13;
constexpr int KRY_MAXDEPTH = 64;
constexpr double KRY_SKEW_TOL = 1e-12;
constexpr int RESIDUAL_MAX_PANELS = 4096;
constexpr int TAIL_NODES = 8;
constexpr double EXPV_SHIFT_TRIGGER = 30.0;
constexpr double EXPV_MAX_NORM = 1e150;
constexpr double FRONTIER_FLOOR = 1e-14;
constexpr double REORTH_KEEP = 0.70710678118654752440;  // _REORTH_KEEP, dd_cbe.jl:273
constexpr double UNION_KEEP = 0.5;                        // _UNION_KEEP, half_sweeps.jl:127
constexpr int DD_HOLDOUT = 4;                             // _DD_HOLDOUT, dd_cbe_controller.jl:12
constexpr double ADAPTIVE_GROWTH = 1.2;                   // basis_budget.jl:565

enum Unmet { U_SAMPLE = 0, U_TAIL, U_KRYLOV, U_TRUNC, U_PROJECTION, U_EXPV, U_CLOSURE };

// ── engine wrappers ──────────────────────────────────────────────────────────────────────────

// The step's Gaussian draws, fetched from the caller's stream in chunks instead of one callback per
// probe. The caller's generator is saved when the step starts (rng_ctl op 0); values are handed out
// in stream order from the buffer; a save/restore pair inside the step (a measurement drawing from
// a copy of the stream) becomes a mark on the buffer position; when the step ends, the caller's
// generator is restored (op 1) and advanced by exactly the values handed out, so it ends where
// one draw per probe would have left it. Needs a normal stream that splits freely (a draw of a + b
// values equals a draw of a then b, as numpy's standard_normal does).
struct DrawBuf {
  bug_normal_fn draw = nullptr;
  void* user = nullptr;
  bug_rng_ctl_fn ctl = nullptr;
  void* ctl_user = nullptr;
  std::vector<double> x;      // values drawn from the caller's stream; x[0] is at position `base`
  int64_t base = 0, pos = 0;  // pos: stream position of the next value handed out
  std::vector<int64_t> marks;
  bool open = false;
  static constexpr int64_t kChunk = 4096;
  void begin() {
    ctl(ctl_user, 0);
    open = true;
  }
  void take(int64_t n, double* out) {
    const int64_t have = base + int64_t(x.size()) - pos;
    if (have < n) {
      const int64_t keep_from = marks.empty() ? pos : std::min(pos, marks.front());
      x.erase(x.begin(), x.begin() + (keep_from - base));
      base = keep_from;
      const int64_t get = std::max(n - have, kChunk);
      const size_t old = x.size();
      x.resize(old + size_t(get));
      draw(user, get, x.data() + old);
    }
    std::memcpy(out, x.data() + (pos - base), size_t(n) * sizeof(double));
    pos += n;
  }
  void save() { marks.push_back(pos); }
  void restore() {
    pos = marks.back();
    marks.pop_back();
  }
  void drop() { marks.pop_back(); }  // forget the last mark, keeping the position
  // The caller's generator exactly where the values handed out so far leave it, for a draw of
  // another kind from it (pause); resume() then saves the generator after that draw and buffers
  // from there.
  bool paused = false;
  void pause() {
    if (!open) return;
    require(marks.empty(), "a stream fork inside a measurement of a copied stream");
    finish();
    x.clear();
    base = pos = 0;
    paused = true;
  }
  void resume() {
    if (!paused) return;
    paused = false;
    begin();
  }
  // the caller's generator back to the step's start, then forward by the values handed out
  void finish() {
    if (!open) return;
    open = false;
    ctl(ctl_user, 1);
    std::vector<double> tmp(size_t(std::max<int64_t>(pos, 1)));
    if (pos > 0) draw(user, pos, tmp.data());
  }
  ~DrawBuf() { finish(); }
};

struct Eng {
  bug_ctx* c;
  bug_normal_fn draw;
  void* user;
  DrawBuf* buf = nullptr;  // when set, draws come from the buffer

  static T sh(TensorPtr p) { return T(p.release()); }

  T contract(const T& a, std::vector<int> ia, const T& b, std::vector<int> ib, bool ca = false,
             bool cb = false) const {
    return sh(contract_impl(c, *a, int(ia.size()), ia.data(), *b, ib.data(), ca, cb));
  }
  double norm(const T& t) const {
    double r[2];
    dots(c, {{t.get(), t.get()}}, r);
    return std::sqrt(std::max(r[0], 0.0));
  }
  cd inner(const T& a, const T& b) const {
    double r[2];
    dots(c, {{a.get(), b.get()}}, r);
    return cd(r[0], r[1]);
  }
  std::vector<cd> inner_many(const std::vector<T>& vs, const T& w) const {
    std::vector<std::pair<const bug_tensor*, const bug_tensor*>> ps;
    for (auto& v : vs) ps.push_back({v.get(), w.get()});
    std::vector<double> r(2 * std::max<size_t>(vs.size(), 1));
    if (!vs.empty()) dots(c, ps, r.data());
    std::vector<cd> out(vs.size());
    for (size_t i = 0; i < vs.size(); ++i) out[i] = cd(r[2 * i], r[2 * i + 1]);
    return out;
  }
  T lin(const std::vector<std::pair<cd, T>>& terms) const {
    std::vector<double> coef;
    std::vector<const bug_tensor*> ts;
    for (auto& t : terms) {
      coef.push_back(t.first.real());
      coef.push_back(t.first.imag());
      ts.push_back(t.second.get());
    }
    return sh(lincomb_impl(c, int(ts.size()), coef.data(), ts.data()));
  }
  T scale(const T& t, cd s) const { return lin({{s, t}}); }
  T sub(const T& a, const T& b) const { return lin({{1.0, a}, {-1.0, b}}); }
  T permute(const T& t, std::vector<int> p) const { return sh(permute_impl(c, *t, p.data())); }
  T flip(const T& t, int leg) const { return sh(flip_leg_impl(c, *t, leg)); }
  T oplus(const std::vector<T>& ts, int leg) const {
    std::vector<const bug_tensor*> p;
    for (auto& t : ts) p.push_back(t.get());
    return sh(oplus_impl(c, int(p.size()), p.data(), leg));
  }
  T trim(const T& t, int leg, const std::map<int, int>& counts) const {
    bool any = false;
    for (auto& kv : counts) any |= kv.second > 0;
    if (!any) return nullptr;
    std::vector<int> cs;
    for (int q : t->legs[leg].q) {
      auto it = counts.find(q);
      cs.push_back(it == counts.end() ? 0 : it->second);
    }
    auto r = trim_impl(c, *t, leg, cs.data());
    return r ? sh(std::move(r)) : nullptr;
  }
  T trim_total(const T& t, int leg, int64_t ncols) const {
    if (ncols <= 0) return nullptr;
    if (t->legs[leg].total() <= ncols) return t;
    int64_t left = ncols;
    std::map<int, int> keep;
    for (size_t s = 0; s < t->legs[leg].q.size(); ++s) {
      int k = int(std::min<int64_t>(t->legs[leg].d[s], left));
      keep[t->legs[leg].q[s]] = k;
      left -= k;
    }
    return trim(t, leg, keep);
  }
  T scale_leg(const T& t, int leg, const std::map<int, std::vector<double>>& w) const {
    std::vector<double> flat;
    for (int q : t->legs[leg].q) {
      auto& v = w.at(q);
      flat.insert(flat.end(), v.begin(), v.end());
    }
    if (flat.empty()) flat.push_back(0.0);
    return sh(scale_leg_impl(c, *t, leg, flat.data()));
  }
  T upload(int rank, const std::vector<Leg>& legs, const std::map<Key, std::vector<cd>>& blocks) const {
    std::vector<Key> keys;
    std::vector<cd> data;
    for (auto& kv : blocks) {
      keys.push_back(kv.first);
      data.insert(data.end(), kv.second.begin(), kv.second.end());
    }
    return sh(upload_impl(c, rank, legs, keys, reinterpret_cast<const double*>(data.data())));
  }
  // pivoted thin QR basis of the leg-`leg` columns per sector (engine: bug_thin_qr), or null
  T thin_qr(const T& t, int leg, int ref_dir, double thr) const {
    auto r = thin_qr_impl(c, *t, leg, ref_dir, thr);
    return r ? sh(std::move(r)) : nullptr;
  }
  std::pair<double, double> norms(const T& a, const T& b) const {
    double r[4];
    dots(c, {{a.get(), a.get()}, {b.get(), b.get()}}, r);
    return {std::sqrt(std::max(r[0], 0.0)), std::sqrt(std::max(r[2], 0.0))};
  }
  std::vector<cd> complex_normals(int64_t n) const {
    std::vector<double> x(static_cast<size_t>(2 * n));
    if (n > 0) {
      if (buf) buf->take(2 * n, x.data());
      else draw(user, 2 * n, x.data());
    }
    std::vector<cd> z(static_cast<size_t>(n));
    const double s = std::sqrt(0.5);
    for (int64_t i = 0; i < n; ++i) z[i] = cd(x[2 * i] * s, x[2 * i + 1] * s);
    return z;
  }
};

inline int64_t dim(const T& t, int leg) { return t->legs[leg].total(); }

struct SVDRes {
  T U, Vd, Us, SVd_;  // Us = U*S and SVd_ = S*Vd when requested
  std::map<int, std::vector<double>> S;
  std::vector<std::pair<double, int>> kept, trunc;  // (sigma, charge), descending
};

// want: 1 = U, 2 = Vd, 4 = U*S, 8 = S*Vd (one unpack launch writes all requested factors)
SVDRes svd(const Eng& e, const T& t, std::vector<int> left, double cutoff, int nkeep = -1,
           int want = 3) {
  TensorPtr U, V, US_, SV_;
  std::vector<double> sv;
  std::vector<int> q;
  int nk = 0;
  svd_impl(e.c, *t, int(left.size()), left.data(), cutoff, nkeep, U, V, sv, q, nk, want, &US_, &SV_);
  SVDRes r;
  if (U) r.U = Eng::sh(std::move(U));
  if (V) r.Vd = Eng::sh(std::move(V));
  if (US_) r.Us = Eng::sh(std::move(US_));
  if (SV_) r.SVd_ = Eng::sh(std::move(SV_));
  for (size_t i = 0; i < sv.size(); ++i) {
    if (int(i) < nk) {
      r.kept.push_back({sv[i], q[i]});
      r.S[q[i]].push_back(sv[i]);
    } else {
      r.trunc.push_back({sv[i], q[i]});
    }
  }
  return r;
}

// An SVD with cutoff 0 taken ahead of its read-back (svd_ahead: every sector keeps min(m, n)
// columns); false when the context's region for them is full. Only the factors are returned (no
// singular value lists): ask for U*S / S*Vd through `want`. Valid once svd_ahead_check says so.
bool svd_ahead1(const Eng& e, const T& t, std::vector<int> left, int want, SVDRes& r) {
  TensorPtr U, V, US_, SV_;
  std::vector<double> sv;
  std::vector<int> q;
  int nk = 0;
  if (!svd_ahead(e.c, {SvdReq{t.get(), int(left.size()), left.data(), 0.0, -1, want, &U, &V, &sv,
                              &q, &nk, &US_, &SV_}}))
    return false;
  r = SVDRes{};
  if (U) r.U = Eng::sh(std::move(U));
  if (V) r.Vd = Eng::sh(std::move(V));
  if (US_) r.Us = Eng::sh(std::move(US_));
  if (SV_) r.SVd_ = Eng::sh(std::move(SV_));
  return true;
}

// Two such SVDs taken ahead in one launch; false (nothing launched) when the region is full.
bool svd2_ahead(const Eng& e, const T& t1, std::vector<int> left1, int want1, const T& t2,
                std::vector<int> left2, int want2, std::pair<SVDRes, SVDRes>& out) {
  TensorPtr U[2], V[2], US_[2], SV_[2];
  std::vector<double> sv[2];
  std::vector<int> q[2];
  int nk[2] = {0, 0};
  if (!svd_ahead(e.c, {SvdReq{t1.get(), int(left1.size()), left1.data(), 0.0, -1, want1, &U[0],
                              &V[0], &sv[0], &q[0], &nk[0], &US_[0], &SV_[0]},
                       SvdReq{t2.get(), int(left2.size()), left2.data(), 0.0, -1, want2, &U[1],
                              &V[1], &sv[1], &q[1], &nk[1], &US_[1], &SV_[1]}}))
    return false;
  SVDRes* r[2] = {&out.first, &out.second};
  for (int i = 0; i < 2; ++i) {
    *r[i] = SVDRes{};
    if (U[i]) r[i]->U = Eng::sh(std::move(U[i]));
    if (V[i]) r[i]->Vd = Eng::sh(std::move(V[i]));
    if (US_[i]) r[i]->Us = Eng::sh(std::move(US_[i]));
    if (SV_[i]) r[i]->SVd_ = Eng::sh(std::move(SV_[i]));
  }
  return true;
}

// Two independent SVDs (cutoff 0, no Nkeep) in one launch and one read-back, each result as svd()
// gives it.
std::pair<SVDRes, SVDRes> svd2(const Eng& e, const T& t1, std::vector<int> left1, int want1,
                               const T& t2, std::vector<int> left2, int want2) {
  struct Raw {
    TensorPtr U, V, US_, SV_;
    std::vector<double> sv;
    std::vector<int> q;
    int nk = 0;
  } a, b;
  svd_many(e.c, {SvdReq{t1.get(), int(left1.size()), left1.data(), 0.0, -1, want1, &a.U, &a.V,
                        &a.sv, &a.q, &a.nk, &a.US_, &a.SV_},
                 SvdReq{t2.get(), int(left2.size()), left2.data(), 0.0, -1, want2, &b.U, &b.V,
                        &b.sv, &b.q, &b.nk, &b.US_, &b.SV_}});
  auto conv = [](Raw& x) {
    SVDRes r;
    if (x.U) r.U = Eng::sh(std::move(x.U));
    if (x.V) r.Vd = Eng::sh(std::move(x.V));
    if (x.US_) r.Us = Eng::sh(std::move(x.US_));
    if (x.SV_) r.SVd_ = Eng::sh(std::move(x.SV_));
    for (size_t i = 0; i < x.sv.size(); ++i) {
      if (int(i) < x.nk) {
        r.kept.push_back({x.sv[i], x.q[i]});
        r.S[x.q[i]].push_back(x.sv[i]);
      } else {
        r.trunc.push_back({x.sv[i], x.q[i]});
      }
    }
    return r;
  };
  return {conv(a), conv(b)};
}

T US(const Eng& e, const SVDRes& r) { return r.Us ? r.Us : e.scale_leg(r.U, r.U->rank - 1, r.S); }
T SVd(const Eng& e, const SVDRes& r) { return r.SVd_ ? r.SVd_ : e.scale_leg(r.Vd, 0, r.S); }
constexpr int W_U = 1, W_VD = 2, W_US = 4, W_SVD = 8;

double sq_weight(const std::vector<std::pair<double, int>>& l) {
  double s = 0.0;
  for (auto& x : l) s += x.first * x.first;
  return s;
}

double trunc_weight(const SVDRes& r) {
  const double k = sq_weight(r.kept), c = sq_weight(r.trunc), tot = k + c;
  return tot == 0.0 ? 0.0 : std::sqrt(c / tot);
}

// ── budget and ledger (basis_budget.jl) ─────────────────────────────────────────────────────

struct Alloc {
  double per_bond, sample, tail, krylov, scale;
  bool linear;
  double krylov_rank;
};

struct Ledger {
  double max_sample = 0, max_sample_l = 0, max_sample_r = 0, max_tail = 0, max_krylov = 0,
         max_krylov_c = 0, max_krylov_d = 0, discarded = 0, expv_err = 0;
  int64_t n_probes = 0, n_holdout = 0, n_selected = 0, n_krylov = 0, n_h1 = 0, n_targeted = 0,
          n_c_pass = 0, n_d_after_c = 0;
  bool workcap_reached = false, tolerance_met = true, maxdim_reached = false;
  double proj_err = 0;
  int64_t r_old = 0, r_aug = 0, r_final = 0, expv_iters = 0;
  std::vector<int> unmet;
  std::vector<bug_bond_log> bond_log;
  int order = 1;
  int64_t n_passes = 0, n_closure_sweeps = 0;
  std::vector<double> leak;
  double defect = 0;
  int64_t n_root_frontier = 0, n_h2_leak = 0, n_h1_closure = 0, n_compress = 0;

  void unmet_(int what) {
    tolerance_met = false;
    if (std::find(unmet.begin(), unmet.end(), what) == unmet.end()) unmet.push_back(what);
  }
  void merge(const Ledger& o) {
    max_sample = std::max(max_sample, o.max_sample);
    max_sample_l = std::max(max_sample_l, o.max_sample_l);
    max_sample_r = std::max(max_sample_r, o.max_sample_r);
    max_tail = std::max(max_tail, o.max_tail);
    max_krylov = std::max(max_krylov, o.max_krylov);
    max_krylov_c = std::max(max_krylov_c, o.max_krylov_c);
    max_krylov_d = std::max(max_krylov_d, o.max_krylov_d);
    n_c_pass += o.n_c_pass;
    n_d_after_c += o.n_d_after_c;
    discarded = std::max(discarded, o.discarded);
    expv_err = std::max(expv_err, o.expv_err);
    n_probes += o.n_probes;
    n_holdout += o.n_holdout;
    n_selected += o.n_selected;
    n_krylov += o.n_krylov;
    n_h1 += o.n_h1;
    n_targeted += o.n_targeted;
    workcap_reached |= o.workcap_reached;
    tolerance_met &= o.tolerance_met;
    maxdim_reached |= o.maxdim_reached;
    proj_err = std::max(proj_err, o.proj_err);
    r_old = std::max(r_old, o.r_old);
    r_aug = std::max(r_aug, o.r_aug);
    r_final = std::max(r_final, o.r_final);
    expv_iters += o.expv_iters;
    for (int u : o.unmet)
      if (std::find(unmet.begin(), unmet.end(), u) == unmet.end()) unmet.push_back(u);
    bond_log.insert(bond_log.end(), o.bond_log.begin(), o.bond_log.end());
    order = std::max(order, o.order);
    n_passes += o.n_passes;
    n_closure_sweeps += o.n_closure_sweeps;
    leak.insert(leak.end(), o.leak.begin(), o.leak.end());
    defect = std::max(defect, o.defect);
    n_root_frontier += o.n_root_frontier;
    n_h2_leak += o.n_h2_leak;
    n_h1_closure += o.n_h1_closure;
    n_compress += o.n_compress;
  }
};

int unmet_mask(const std::vector<int>& u) {
  int m = 0;
  for (int x : u) m |= 1 << x;
  return m;
}

void log_bond(Ledger& ledger, Ledger& bl, int bond, int side, int width) {
  bug_bond_log e{};
  e.bond = bond;
  e.side = side;
  e.sample = bl.max_sample;
  e.tail = bl.max_tail;
  e.krylov_c = bl.max_krylov_c;
  e.krylov_d = bl.max_krylov_d;
  e.n_probes = bl.n_probes;
  e.n_selected = bl.n_selected;
  e.n_krylov = bl.n_krylov;
  e.n_h1 = bl.n_h1;
  e.c_pass = bl.n_c_pass > 0;
  e.d_after_c = bl.n_d_after_c > 0;
  e.workcap = bl.workcap_reached;
  e.met = bl.tolerance_met;
  e.unmet_mask = unmet_mask(bl.unmet);
  e.width = width;
  bl.bond_log.push_back(e);
  ledger.merge(bl);
}

Alloc basis_allocation(double basis, int nbonds, cd tau, double nrm, int nfront, double krylov,
                       double krylov_rank) {
  const int nb = std::max(nbonds, 1), nf = std::max(nfront, 1);
  const double kr = krylov > 0 ? krylov / basis : 1.0;
  const double rank_share = krylov_rank / basis;
  const double at = std::abs(tau);
  const double scale = at == 0.0 ? 1.0 : at / std::max(nrm, EPS);
  const double per_test = basis / (2.0 * (nb + 1) * nf);
  return Alloc{2 * per_test, per_test, per_test, kr * per_test, scale, true, rank_share * per_test};
}

inline double indicator(const Alloc& a, double r) { return a.scale * r; }

std::pair<int, double> tail_rank(const std::vector<std::pair<double, int>>& lst, double scale,
                                 double allowance, int kmax, double base = 0.0) {
  const int n = int(lst.size());
  kmax = std::min(kmax, n);
  if (kmax <= 0) return {0, scale * std::sqrt(base + sq_weight(lst))};
  std::vector<double> w(n);
  for (int i = 0; i < n; ++i) w[i] = lst[i].first * lst[i].first;
  double tail = base;
  for (int i = kmax; i < n; ++i) tail += w[i];
  int keep = kmax;
  while (keep > 0) {
    const double trial = tail + w[keep - 1];
    if (!(scale * std::sqrt(trial) <= allowance)) break;
    tail = trial;
    --keep;
  }
  return {keep, scale * std::sqrt(tail)};
}

// ── environments and effective operators (mpo_environments.jl, effective_operators.jl) ─────

struct Env {
  const Eng& e;
  T left_boundary() const {
    std::vector<Leg> legs(3);
    legs[0] = Leg{-1, {0}, {1}};
    legs[1] = Leg{+1, {0}, {1}};
    legs[2] = Leg{+1, {0}, {1}};
    std::map<Key, std::vector<cd>> b;
    b[Key{0, 0, 0, 0, 0, 0}] = {cd(1.0)};
    return e.upload(3, legs, b);
  }
  T right_boundary(int q) const {
    std::vector<Leg> legs(3);
    legs[0] = Leg{+1, {q}, {1}};
    legs[1] = Leg{-1, {0}, {1}};
    legs[2] = Leg{-1, {q}, {1}};
    std::map<Key, std::vector<cd>> b;
    b[Key{q, 0, q, 0, 0, 0}] = {cd(1.0)};
    return e.upload(3, legs, b);
  }
  T left_step(const T& E, const T& A, const T& W) const {
    T t = e.contract(E, {2}, A, {0});
    t = e.contract(t, {1, 2}, W, {0, 1});
    t = e.contract(t, {0, 2}, A, {0, 1}, false, true);
    return e.permute(t, {2, 1, 0});
  }
  T right_step(const T& R, const T& A, const T& W) const {
    T t = e.contract(A, {2}, R, {2});
    t = e.contract(t, {1, 3}, W, {1, 3});
    t = e.contract(t, {1, 3}, A, {2, 1}, false, true);
    return e.permute(t, {2, 1, 0});
  }
  // H Theta for a two-site tensor (l, s1, s2, r) (apply_h_two_site, mpo_environments.jl:316-344)
  T two_site(const T& Le, const T& Wl, const T& Wr, const T& Re, const T& x) const {
    T t = e.contract(Le, {2}, x, {0});
    t = e.contract(t, {1, 2}, Wl, {0, 1});
    t = e.contract(t, {4, 1}, Wr, {0, 1});
    return e.contract(t, {4, 1}, Re, {1, 2});
  }
  T one_site(const T& Le, const T& W, const T& Re, const T& x) const {
    T t = e.contract(Le, {2}, x, {0});
    t = e.contract(t, {1, 2}, W, {0, 1});
    return e.contract(t, {3, 1}, Re, {1, 2});
  }
  T stream_left(const T& lamp, const T& riso, const T& Wl, const T& Wr, const T& lenv,
                const T& renv, const T& Om) const {
    T t = e.contract(Om, {2}, renv, {0}, true, false);
    T rc = e.contract(t, {1, 2}, Wr, {2, 3});
    T bp = e.contract(riso, {1, 2}, rc, {3, 1});
    T sp = e.contract(lamp, {2}, bp, {0});
    T wm = e.contract(sp, {1, 3}, Wl, {1, 3});
    t = e.contract(wm, {0, 2}, lenv, {2, 1});
    return e.permute(t, {2, 1, 0});
  }
  T stream_right(const T& liso, const T& ramp, const T& Wl, const T& Wr, const T& lenv,
                 const T& renv, const T& Om) const {
    T t = e.contract(Om, {0}, lenv, {0}, true, false);
    T gf = e.contract(t, {0, 2}, Wl, {2, 0});
    T lc = e.permute(gf, {1, 0, 2, 3});
    T bp = e.contract(liso, {0, 1}, lc, {0, 2});
    T sp = e.contract(ramp, {0}, bp, {0});
    T wm = e.contract(sp, {0, 3}, Wr, {1, 0});
    return e.contract(wm, {0, 3}, renv, {2, 1});
  }
};

// H0 - shift (apply_zero_site, effective_operators.jl:91-107; shift_h, :110-129)
struct ZeroSiteH {
  T l, r;
  double shift = 0.0;
  T apply(const Eng& e, const T& core) const {
    T t = e.contract(l, {2}, core, {0});
    T y = e.contract(t, {1, 2}, r, {1, 2});
    return shift == 0.0 ? y : e.lin({{1.0, y}, {-shift, core}});
  }
};

// ── projections, probes, DD-QR CBE (cbe.jl, dd_cbe.jl, dd_cbe_expand.jl, sketch.jl) ─────────

T perp_left(const Eng& e, const T& U, const T& K) {
  T ov = e.contract(U, {0, 1}, K, {0, 1}, true, false);
  T pr = e.contract(U, {2}, ov, {0});
  return e.sub(K, pr);
}

T perp_right(const Eng& e, const T& V, const T& K) {
  T ov = e.contract(K, {1, 2}, V, {1, 2}, false, true);
  T pr = e.contract(ov, {1}, V, {0});
  return e.sub(K, pr);
}

T rows_from_u(const Eng& e, const T& U) { return e.flip(e.permute(U, {2, 0, 1}), 0); }

double rank_cut(double stol, double sketch_norm, double outside_norm) {
  return stol > 0 ? stol : CBE_EPS * std::max(sketch_norm, outside_norm) / outside_norm;
}

T reortho(const Eng& e, const T& frame, const T& block, bool left) {
  if (!block) return nullptr;
  T out = left ? perp_left(e, frame, block) : perp_right(e, frame, block);
  const auto nb = e.norms(out, block);  // one read-back for both
  if (nb.first <= CBE_EPS * std::max(nb.second, 1.0)) return nullptr;
  if (left) return svd(e, out, {0, 1}, 1e-14, -1, W_U).U;
  return rows_from_u(e, svd(e, out, {1, 2}, 1e-14, -1, W_U).U);
}

// fused local space of a frame: charge -> list of (qa, qb) pairs, and per charge dims
struct Fused {
  std::map<int, std::vector<std::pair<int, int>>> pairs;
  std::map<int, int64_t> dfull, dT;
};

Fused fused_of(const Leg& la, const Leg& lb, int out_dir) {
  Fused f;
  for (size_t i = 0; i < la.q.size(); ++i)
    for (size_t j = 0; j < lb.q.size(); ++j) {
      const int c = -(la.dir * la.q[i] + lb.dir * lb.q[j]) * out_dir;
      f.pairs[c].push_back({la.q[i], lb.q[j]});
      f.dfull[c] += int64_t(la.d[i]) * lb.d[j];
    }
  for (auto& kv : f.pairs) std::sort(kv.second.begin(), kv.second.end());
  return f;
}

Fused fused_dims(const T& frame, bool left) {
  Fused f = left ? fused_of(frame->legs[0], frame->legs[1], +1)
                 : fused_of(frame->legs[1], frame->legs[2], -1);
  const Leg& bl = left ? frame->legs[2] : frame->legs[0];
  for (auto& kv : f.dfull) {
    const int w = bl.dim_of(kv.first);
    require(w <= kv.second, "a frame holds more directions in a sector than its local space");
    f.dT[kv.first] = w;
  }
  return f;
}

T cap_to_local_room(const Eng& e, const T& frame, const T& cand, bool left) {
  if (!cand) return nullptr;
  const int fl = left ? 2 : 0;
  Fused f = fused_dims(frame, left);
  std::map<int, int> counts;
  bool over = false;
  for (auto& kv : f.dfull) {
    const int du = cand->legs[fl].dim_of(kv.first);
    if (du == 0) continue;
    const int c = int(std::min<int64_t>(du, kv.second - f.dT[kv.first]));
    counts[kv.first] = c;
    over |= c < du;
  }
  if (!over) return cand;
  return e.trim(cand, fl, counts);
}

std::map<int, int> alloc_columns(const std::map<int, int64_t>& dims, int budget) {
  int64_t tot = 0;
  for (auto& kv : dims) tot += kv.second;
  std::map<int, int> out;
  for (auto& kv : dims) {
    if (tot == 0 || budget <= 0) {
      out[kv.first] = 0;
      continue;
    }
    const double r = double(kv.second) / double(tot) * double(budget);
    out[kv.first] = int(std::min<int64_t>(kv.second, int64_t(std::ceil(r))));
  }
  return out;
}

// Gaussian on the fused space; layout (la, lb, g:+1) or (g:-1, la, lb)
T gaussian_fused(const Eng& e, const Leg& la, const Leg& lb, const std::map<int, int>& cols,
                 bool new_first, bool* nonzero = nullptr) {
  if (nonzero) *nonzero = false;
  const int gdir = new_first ? -1 : +1;
  Fused f = fused_of(la, lb, gdir);
  Leg g;
  g.dir = gdir;
  for (auto& kv : f.pairs) {
    auto it = cols.find(kv.first);
    if (it != cols.end() && it->second > 0) {
      g.q.push_back(kv.first);
      g.d.push_back(it->second);
    }
  }
  if (g.q.empty()) return nullptr;
  std::vector<Leg> legs = new_first ? std::vector<Leg>{g, la, lb} : std::vector<Leg>{la, lb, g};
  std::map<Key, std::vector<cd>> blocks;
  for (auto& kv : f.pairs) {
    const int c = kv.first;
    const int k = g.dim_of(c);
    if (k == 0) continue;
    int64_t n = 0;
    for (auto& pr : kv.second) n += int64_t(la.dim_of(pr.first)) * lb.dim_of(pr.second);
    std::vector<cd> M = e.complex_normals(n * k);  // (n, k) C order
    if (nonzero && !*nonzero)
      *nonzero = std::any_of(M.begin(), M.end(), [](const cd& z) { return z != cd(0); });
    int64_t off = 0;
    for (auto& pr : kv.second) {
      const int da = la.dim_of(pr.first), db = lb.dim_of(pr.second);
      const int64_t r = int64_t(da) * db;
      std::vector<cd> blk(size_t(r * k));
      if (new_first) {  // (k, da, db) from rows (da*db) x k
        for (int64_t i = 0; i < r; ++i)
          for (int j = 0; j < k; ++j) blk[size_t(j * r + i)] = M[size_t((off + i) * k + j)];
        blocks[Key{c, pr.first, pr.second, 0, 0, 0}] = std::move(blk);
      } else {
        for (int64_t i = 0; i < r; ++i)
          for (int j = 0; j < k; ++j) blk[size_t(i * k + j)] = M[size_t((off + i) * k + j)];
        blocks[Key{pr.first, pr.second, c, 0, 0, 0}] = std::move(blk);
      }
      off += r;
    }
  }
  return e.upload(3, legs, blocks);
}

// the complete fused basis of la (x) lb (fusion_basis, dd_cbe.jl:140-148): the n_c x n_c identity
// in every fused sector, rows and columns in gaussian_fused's (qa, qb)-pair order and layouts
T identity_fused(const Eng& e, const Leg& la, const Leg& lb, bool new_first) {
  const int gdir = new_first ? -1 : +1;
  Fused f = fused_of(la, lb, gdir);
  Leg g;
  g.dir = gdir;
  for (auto& kv : f.pairs) {
    int64_t n = 0;
    for (auto& pr : kv.second) n += int64_t(la.dim_of(pr.first)) * lb.dim_of(pr.second);
    if (n > 0) {
      g.q.push_back(kv.first);
      g.d.push_back(int(n));
    }
  }
  if (g.q.empty()) return nullptr;
  std::vector<Leg> legs = new_first ? std::vector<Leg>{g, la, lb} : std::vector<Leg>{la, lb, g};
  std::map<Key, std::vector<cd>> blocks;
  for (auto& kv : f.pairs) {
    const int c = kv.first;
    const int64_t n = g.dim_of(c);
    if (n == 0) continue;
    int64_t off = 0;
    for (auto& pr : kv.second) {
      const int da = la.dim_of(pr.first), db = lb.dim_of(pr.second);
      const int64_t r = int64_t(da) * db;
      if (r == 0) continue;
      std::vector<cd> blk(size_t(r * n), cd(0));
      // row off + i of the identity has its one in column off + i
      for (int64_t i = 0; i < r; ++i)
        blk[size_t(new_first ? (off + i) * r + i : i * n + off + i)] = cd(1);
      blocks[new_first ? Key{c, pr.first, pr.second, 0, 0, 0} : Key{pr.first, pr.second, c, 0, 0, 0}] =
          std::move(blk);
      off += r;
    }
  }
  return e.upload(3, legs, blocks);
}

// _dd_probe(...; exact = true) (dd_cbe.jl:140-161): the complete fused basis with the opposite
// frame projected out, or null when there is no discarded space or nothing survives. No draws.
T dd_probe_exact(const Eng& e, const T& opp, bool oleft) {
  Fused f = fused_dims(opp, oleft);
  int64_t tot = 0;
  for (auto& kv : f.dfull) tot += std::max<int64_t>(kv.second - f.dT[kv.first], 0);
  if (tot == 0) return nullptr;
  T om = oleft ? identity_fused(e, opp->legs[0], opp->legs[1], false)
               : identity_fused(e, opp->legs[1], opp->legs[2], true);
  if (!om) return nullptr;
  T pr = oleft ? perp_left(e, opp, om) : perp_right(e, opp, om);
  return e.norm(pr) > 0 ? pr : nullptr;
}

// _boost! (cbe.jl:206-216): raise the targeted sectors' columns, capped by the room `cap`
void boost_columns(std::map<int, int>& cols, const std::map<int, int64_t>& boost,
                   const std::map<int, int64_t>& cap) {
  for (auto& kv : boost) {
    auto ci = cap.find(kv.first);
    if (ci == cap.end()) continue;
    const int64_t have = cols.count(kv.first) ? cols[kv.first] : 0;
    const int64_t add = std::min<int64_t>(std::max<int64_t>(kv.second, 0),
                                          std::max<int64_t>(ci->second - have, 0));
    cols[kv.first] = int(have + add);
  }
}

// sector-graded Gaussian probe in the opposite frame's discarded space (dd_cbe.jl:132-161). With
// `norm_slot` the probe's |.|^2 is queued into that device slot and the probe returned unchecked:
// the caller reads the slot back with its own next result and treats |probe| = 0 as no probe.
T dd_probe(const Eng& e, const T& opp, bool oleft, int width,
           const std::map<int, int64_t>* boost = nullptr, double2* norm_slot = nullptr) {
  Fused f = fused_dims(opp, oleft);
  std::map<int, int64_t> dC;
  int64_t tot = 0;
  for (auto& kv : f.dfull) {
    dC[kv.first] = std::max<int64_t>(kv.second - f.dT[kv.first], 0);
    tot += dC[kv.first];
  }
  if (tot == 0) return nullptr;
  auto cols = alloc_columns(dC, width);
  if (boost && !boost->empty()) boost_columns(cols, *boost, dC);
  T om = oleft ? gaussian_fused(e, opp->legs[0], opp->legs[1], cols, false)
               : gaussian_fused(e, opp->legs[1], opp->legs[2], cols, true);
  if (!om) return nullptr;
  T pr = oleft ? perp_left(e, opp, om) : perp_right(e, opp, om);
  if (norm_slot) {
    dots_device(e.c, {{pr.get(), pr.get()}}, norm_slot);
    return pr;
  }
  return e.norm(pr) > 0 ? pr : nullptr;
}

T graded_sketch(const Eng& e, const T& frame, bool left, int npre) {
  Fused f = fused_dims(frame, left);
  auto cols = alloc_columns(f.dfull, npre);
  // the drawn values are on the host: |r| > 0 exactly when one of them is not zero (a Gaussian
  // value whose square underflows, |x| < 1e-161, does not occur)
  bool nonzero = false;
  T r = left ? gaussian_fused(e, frame->legs[0], frame->legs[1], cols, false, &nonzero)
             : gaussian_fused(e, frame->legs[1], frame->legs[2], cols, true, &nonzero);
  if (!r) return nullptr;
  return nonzero ? r : nullptr;
}

// Test B's two read-backs in one: |res| (returned) and the per-sector squared norms `n2` of the
// residual the test measures, `fin` (res itself, or res projected off `basis` once more), the
// latter formed and measured ahead of the |res| <= CBE_EPS test and unused when that test returns
// early.
double residual_norms(const Eng& e, const T& res, const T& basis,
                      const std::function<T(const T&)>& project, bool left, std::vector<double>& n2,
                      T& fin) {
  const int rleg = left ? 2 : 0;
  fin = basis ? project(left ? perp_left(e, basis, res) : perp_right(e, basis, res)) : res;
  const int ns = int(fin->legs[rleg].q.size());
  double2* q = static_cast<double2*>(e.c->scratch(size_t(1 + ns) * sizeof(double2)));
  dots_device(e.c, {{res.get(), res.get()}}, q);
  sector_norms2_device(e.c, *fin, rleg, q + 1);
  double* host = e.c->readback(size_t(2 * (1 + ns)));
  e.c->drain();  // the queued dot stages write the slots: they run before the copy
  BUG_CUDA(cudaMemcpyAsync(host, q, size_t(1 + ns) * sizeof(double2), cudaMemcpyDeviceToHost,
                           e.c->stream));
  e.c->wait();
  n2.resize(size_t(ns));
  for (int s = 0; s < ns; ++s) n2[size_t(s)] = host[2 * (1 + s)];
  return std::sqrt(std::max(host[0], 0.0));
}

// Test B with one fixed probe (sketch.jl:141-180)
double sample_residual(const Eng& e, const T& basis, const std::function<T(const T&)>& project,
                       const std::function<T(const T&)>& sketch, const T& Om, int wleg, bool left) {
  if (!Om) return 0.0;
  std::map<int, int> cols;
  for (size_t s = 0; s < Om->legs[wleg].q.size(); ++s)
    if (Om->legs[wleg].d[s] > 0) cols[Om->legs[wleg].q[s]] = Om->legs[wleg].d[s];
  if (cols.empty()) return 0.0;
  T sk = sketch(Om);
  if (!sk) return 0.0;
  T res = project(sk);
  const int rleg = left ? 2 : 0;
  std::vector<double> n2;
  T fin;
  if (residual_norms(e, res, basis, project, left, n2, fin) <= CBE_EPS) return 0.0;
  res = fin;
  double tot = 0.0;
  const Leg& rl = res->legs[rleg];
  for (size_t s = 0; s < rl.q.size(); ++s) {
    auto it = cols.find(rl.q[s]);
    require(it != cols.end() && it->second > 0, "Test B: residual sector has no holdout column");
    tot += n2[s] / it->second;
  }
  return std::sqrt(tot);
}

// Test B with one fixed, already sketched holdout (sketch.jl:141-180), per sector: `est`, the
// per-sector residual share r2 = |residual_q|^2 / holdout columns_q, and the holdout columns.
struct TestB {
  double est = 0.0;
  std::map<int, double> per;
  std::map<int, int> cols;
};

TestB sample_residual_sectors(const Eng& e, const T& basis, const std::function<T(const T&)>& project,
                              const T& sketched, const T& Om, int wleg, bool left) {
  TestB r;
  if (!Om) return r;
  for (size_t s = 0; s < Om->legs[wleg].q.size(); ++s)
    if (Om->legs[wleg].d[s] > 0) r.cols[Om->legs[wleg].q[s]] = Om->legs[wleg].d[s];
  if (r.cols.empty() || !sketched) return r;
  T res = project(sketched);
  std::vector<double> n2;
  T fin;
  if (residual_norms(e, res, basis, project, left, n2, fin) <= CBE_EPS) return r;
  res = fin;
  const int rleg = left ? 2 : 0;
  const Leg& rl = res->legs[rleg];
  double tot = 0.0;
  for (size_t s = 0; s < rl.q.size(); ++s) {
    if (rl.d[s] <= 0) continue;
    auto it = r.cols.find(rl.q[s]);
    require(it != r.cols.end() && it->second > 0, "Test B: residual sector has no holdout column");
    r.per[rl.q[s]] = n2[s] / it->second;
    tot += r.per[rl.q[s]];
  }
  r.est = std::sqrt(tot);
  return r;
}

// _dd_select (dd_cbe.jl:290-321): P^D sketch, a first pivoted QR at the floor
// CBE_EPS max(|sketch|, |projected|), then a pivoted QR of P^D of the first pass keeping pivots
// above 1/sqrt(2) ("twice is enough"). Null when nothing survives.
T dd_select(const Eng& e, const T& frame, const T& sketch, bool left) {
  const int fl = left ? 2 : 0;
  T projected = left ? perp_left(e, frame, sketch) : perp_right(e, frame, sketch);
  const auto nn = e.norms(sketch, projected);
  const double nz = nn.first, ny = nn.second;
  if (ny <= CBE_EPS * std::max(nz, 1.0)) return nullptr;
  const int ref_dir = frame->legs[fl].dir;
  T first = e.thin_qr(projected, fl, ref_dir, CBE_EPS * std::max(nz, ny));
  if (!first) return nullptr;
  T again = left ? perp_left(e, frame, first) : perp_right(e, frame, first);
  return e.thin_qr(again, fl, ref_dir, REORTH_KEEP);
}

// _target_sectors! (sketch.jl:188-201): sectors whose residual share exceeds an even split of
// the sample allowance get max(holdout columns, 1) more probe columns; returns how many
int target_sectors(std::map<int, int64_t>& boost, const TestB& tb, const T& Om, int wleg,
                   double scale, double sample) {
  if (tb.per.empty()) return 0;
  const double share = sample * sample / double(tb.per.size());
  int n = 0;
  for (auto& kv : tb.per) {
    if (!(scale * scale * kv.second > share)) continue;
    const int have = Om ? Om->legs[wleg].dim_of(kv.first) : 0;
    boost[kv.first] += std::max(have, 1);
    ++n;
  }
  return n;
}

struct BondFrame {
  T U0, S0, V0;
  int64_t old_rank;
};

T frame_theta(const Eng& e, const BondFrame& f) {
  return e.contract(e.contract(f.U0, {2}, f.S0, {0}), {2}, f.V0, {0});
}

struct Expansion {
  T U_ex, V_ex;
  int64_t n_new_l = 0, n_new_r = 0;
};

struct Step;  // forward

struct MPOv {
  std::vector<T> W;  // 0-based sites
  const T& operator[](int site) const { return W[site - 1]; }
};

// ── the step ────────────────────────────────────────────────────────────────────────────────

// Per-bond work ceilings from the bonds before the step (basis_budget.jl:454-555): rule 0 :bond
// (ceil(f d D_b), 2 d D_b at f = 0), 1 :maxdim (one ceiling d max(maxdim, max D_b)),
// 2 :bond_strict (ceil(f D_b), f > 1), 3 :frame_root (ceil(f D_b), f = 2 at 0, and
// ceil(root_factor D_root) at the root bond); each within [1, maxdim] except :maxdim's. `factor`
// < 0 is the keyword's default (1.2 under :bond, 0 otherwise), `root_factor` <= 0 is 1.2. Products
// are rounded to nine decimals before the ceiling, as the reference rounds them.
std::vector<int64_t> work_ceilings(int rule, const std::vector<int64_t>& bonds, int64_t dloc,
                                   int64_t maxdim, double factor, int root_link, double root_factor) {
  require(rule >= 0 && rule <= 3, "work_ceiling_rule must be 0 (:bond), 1 (:maxdim), 2 (:bond_strict) or 3 (:frame_root)");
  if (factor < 0) factor = rule == 0 ? 1.2 : 0.0;
  require(factor == 0 || (factor > 1 && rule != 1),
          "bond_ceiling_factor must be 0, or > 1 with work_ceiling_rule = bond");
  auto ceil9 = [](double x) { return int64_t(std::ceil(std::round(x * 1e9) / 1e9)); };
  std::vector<int64_t> w;
  if (rule == 1) {
    const int64_t mx = bonds.empty() ? 0 : *std::max_element(bonds.begin(), bonds.end());
    w.assign(bonds.size(), std::max<int64_t>({dloc * maxdim, dloc * mx, 1}));
    return w;
  }
  if (rule == 2) require(factor > 1, "strict bond factor must exceed 1");
  if (rule == 3) {
    if (factor == 0) factor = 2.0;
    if (root_factor <= 0) root_factor = 1.2;
    require(root_factor > 1, "root_ceiling_factor must exceed one");
    require(root_factor <= factor, "root_ceiling_factor must not exceed the frame factor");
    require(root_link >= 1 && root_link <= int(bonds.size()), "root bond outside the chain");
  }
  for (size_t b = 0; b < bonds.size(); ++b) {
    const int64_t r = bonds[b];
    int64_t c;
    if (rule == 0) c = factor > 0 ? ceil9(factor * double(dloc) * double(r)) : 2 * dloc * r;
    else if (rule == 2) c = ceil9(factor * double(r));
    else c = ceil9((int(b) + 1 == root_link ? root_factor : factor) * double(r));
    w.push_back(std::max<int64_t>(std::min<int64_t>(c, maxdim), 1));
  }
  return w;
}

struct Params {
  double tol_basis, tol_trunc, tol_expv, tol_krylov;
  int order, maxdim, hermitian, root, reorth, truncate, root_maxiter, fixed_width;
  double tail_factor, bond_ceiling_factor;
  int lanczos, fixed_depth;
  int dd_mode;  // 0 :rank_tail, 1 :adaptive
  int holdout_width, batch_blocks, cap_selection_svd;
  double acceptance_factor;
  int closure_checks = 0;  // the measured, multi-pass closure (_krylov_closure!, checks = true)
  int root_method = 0;     // 0 exp, 1 trapezoid, 2 radau2, 3 radau3
  bool root_shift = true;  // the implicit roots' imaginary-time spectral shift
  bool parallel = false;   // parallel = true: halves on two streams, right halves on forked streams
  bug_rng_fork_fn rng_fork = nullptr;
  void* rng_fork_user = nullptr;
  bool exact = false;  // exact = true: DD expansions sketch the complete fused basis (no draws)
  bool fold = true;    // fold_omega: frontier leaks from folded closures (sampled), else exact
  std::vector<std::vector<T>> keep;  // keep_states: each kept state's L sites (borrowed)
  std::vector<double> keep_tols;     // per kept state: 0 contained exactly, > 0 admitted at it
  bool cap_keep = false;             // :bond ceiling: admitted states fill frames to the ceiling
};

struct MPS {
  std::vector<T> s;  // 0-based storage, 1-based access
  int center;
  T& operator[](int i) { return s[i - 1]; }
  const T& operator[](int i) const { return s[i - 1]; }
  int size() const { return int(s.size()); }
  std::vector<int64_t> bond_dims() const {
    std::vector<int64_t> d;
    for (int b = 1; b < size(); ++b) d.push_back(dim((*this)[b], 2));
    return d;
  }
};

// |tau| int_0^1 |(exp(s g) e_1)[comp]| ds by composite Simpson in log space
// (krylov_enrichment.jl:89-120): the nodes are s_j = j / N of the shifted generator's propagator
// P = exp(g / N). Only component `comp` of P^j e_1 enters a node, so the nodes are evaluated in
// blocks of B: the rows e_comp^T P^r (r < B) once, the vectors P^(qB) e_1 by one matvec with P^B
// per block, and node qB + r as their dot product -- the same Simpson sum for ~1/10 of the work
// of N full matvecs at N = 8192, n = 64. With `state_seed` the integral is normalised by
// |P^N e_1| e^sigma, the propagated seed's norm.
double residual_integral(int comp, const CMat& g, cd tau_eff, bool state_seed) {
  const int n = g.n;
  CMat gh(n, n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) gh(i, j) = g(i, j) + std::conj(g(j, i));
  const bool unitary = smallla::frob(gh) <= KRY_SKEW_TOL * smallla::frob(g);
  double sigma = 0.0;
  if (!unitary) {
    auto ev = smallla::eigvals_hess(g);
    sigma = -std::numeric_limits<double>::infinity();
    for (auto& v : ev) sigma = std::max(sigma, v.real());
  }
  CMat shifted = g;
  for (int i = 0; i < n; ++i) shifted(i, i) -= sigma;
  const int intervals =
      2 * std::min(std::max(int(std::ceil(2 * smallla::norm1(shifted))), 8), RESIDUAL_MAX_PANELS);
  const double spacing = 1.0 / intervals;
  CMat sc = shifted;
  for (auto& v : sc.a) v *= spacing;
  const CMat prop = smallla::expm(sc);
  // split real/imaginary copies for the inner loops (explicit FMAs, no complex-multiply calls)
  auto split = [n](const CMat& m, std::vector<double>& re, std::vector<double>& im) {
    re.resize(size_t(n) * n);
    im.resize(size_t(n) * n);
    for (size_t i = 0; i < m.a.size(); ++i) {
      re[i] = m.a[i].real();
      im[i] = m.a[i].imag();
    }
  };
  // y = M x (M row-major n x n)
  auto matvec = [n](const std::vector<double>& mr, const std::vector<double>& mi,
                    const std::vector<double>& xr, const std::vector<double>& xi,
                    std::vector<double>& yr, std::vector<double>& yi) {
    for (int i = 0; i < n; ++i) {
      const double* ar = &mr[size_t(i) * n];
      const double* ai = &mi[size_t(i) * n];
      double sr = 0.0, si = 0.0;
      for (int j = 0; j < n; ++j) {
        sr = std::fma(ar[j], xr[j], std::fma(-ai[j], xi[j], sr));
        si = std::fma(ar[j], xi[j], std::fma(ai[j], xr[j], si));
      }
      yr[i] = sr;
      yi[i] = si;
    }
  };
  std::vector<double> pr, pi;
  split(prop, pr, pi);
  const int B = intervals >= 256 ? 64 : 1;
  // rows e_comp^T P^r, r = 0 .. B-1
  std::vector<double> rowr(size_t(B) * n, 0.0), rowi(size_t(B) * n, 0.0);
  rowr[size_t(comp)] = 1.0;
  // P transposed, so that (u P)_j runs along a contiguous row (same sums in the same order)
  std::vector<double> ptr_(size_t(n) * n), pti_(size_t(n) * n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      ptr_[size_t(j) * n + i] = pr[size_t(i) * n + j];
      pti_[size_t(j) * n + i] = pi[size_t(i) * n + j];
    }
  for (int r = 1; r < B; ++r) {
    const double* ur = &rowr[size_t(r - 1) * n];
    const double* ui = &rowi[size_t(r - 1) * n];
    double* vr = &rowr[size_t(r) * n];
    double* vi = &rowi[size_t(r) * n];
    for (int j = 0; j < n; ++j) {
      const double* ar = &ptr_[size_t(j) * n];
      const double* ai = &pti_[size_t(j) * n];
      double sr = 0.0, si = 0.0;
      for (int i = 0; i < n; ++i) {  // (u P)_j = sum_i u_i P_ij
        sr = std::fma(ur[i], ar[i], std::fma(-ui[i], ai[i], sr));
        si = std::fma(ur[i], ai[i], std::fma(ui[i], ar[i], si));
      }
      vr[j] = sr;
      vi[j] = si;
    }
  }
  // P^B by squaring (B is a power of two)
  std::vector<double> qre = pr, qim = pi;
  if (B > 1) {
    CMat Q = prop;
    for (int m = 1; m < B; m *= 2) Q = smallla::matmul(Q, Q);
    split(Q, qre, qim);
  }
  std::vector<double> vr(n, 0.0), vi(n, 0.0), tr(n), ti(n);
  vr[0] = 1.0;
  std::vector<double> logs(intervals + 1);
  for (int base = 0; base <= intervals; base += B) {
    for (int r = 0; r < B && base + r <= intervals; ++r) {
      const int node = base + r;
      double cr = vr[comp], ci = vi[comp];
      if (B > 1) {
        const double* ur = &rowr[size_t(r) * n];
        const double* ui = &rowi[size_t(r) * n];
        cr = 0.0;
        ci = 0.0;
        for (int j = 0; j < n; ++j) {
          cr = std::fma(ur[j], vr[j], std::fma(-ui[j], vi[j], cr));
          ci = std::fma(ur[j], vi[j], std::fma(ui[j], vr[j], ci));
        }
      }
      const double w = (node == 0 || node == intervals) ? 1.0 : (node % 2 == 1 ? 4.0 : 2.0);
      const double mag = std::hypot(cr, ci);
      logs[node] = mag == 0 ? -std::numeric_limits<double>::infinity()
                            : std::log(w * spacing / 3 * mag) + node * spacing * sigma;
    }
    if (base + B <= intervals) {
      matvec(qre, qim, vr, vi, tr, ti);
      vr.swap(tr);
      vi.swap(ti);
    }
  }
  double peak = -std::numeric_limits<double>::infinity();
  for (double x : logs) peak = std::max(peak, x);
  if (peak == -std::numeric_limits<double>::infinity()) return 0.0;
  double s = 0.0;
  for (double x : logs) s += std::exp(x - peak);
  const double lw = std::log(std::abs(tau_eff)) + peak + std::log(s);
  if (unitary || !state_seed) return std::exp(lw);
  // the last node's full vector P^N e_1: from the last block's start, the remaining steps by P
  const int last_base = (intervals / B) * B;
  for (int m = last_base; m < intervals; ++m) {
    matvec(pr, pi, vr, vi, tr, ti);
    vr.swap(tr);
    vi.swap(ti);
  }
  double cn = 0.0;
  for (int i = 0; i < n; ++i) cn += vr[i] * vr[i] + vi[i] * vi[i];
  cn = std::sqrt(cn);
  return std::exp(lw - sigma - std::log(std::max(cn, std::numeric_limits<double>::min())));
}

struct Step {
  Eng e;
  Env env{e};
  const MPOv& mpo;
  Params P;
  cd tau;
  double eshift = 0.0;  // the generators are H - eshift
  int L, root_link;
  Alloc alloc{};
  std::vector<int64_t> wcap;
  int64_t nmv = 0;

  Step(const Eng& eng, const MPOv& m, const Params& p, cd t, int l) : e(eng), env{e}, mpo(m), P(p), tau(t), L(l) {}
  Step(const Step&) = delete;
  Step& operator=(const Step&) = delete;

  int64_t cap_at(int bond) const { return wcap[bond - 1]; }

  // ── parallel = true (bug_step.jl:222-268, frontier_closure.jl:121-145) ──
  // this step's settings on a step bound to another engine (context and draw stream); a Step is
  // never copied (its Env refers to its own Eng)
  void share_settings(Step& s) const {
    s.eshift = eshift;
    s.root_link = root_link;
    s.alloc = alloc;
    s.wcap = wcap;
  }
  // The right half's stream: ONE 64-bit draw from the step's stream at this point seeds it (the
  // caller makes it through rng_fork); a buffered step stream is first brought to this point.
  std::pair<bug_normal_fn, void*> fork_stream() {
    if (e.buf) e.buf->pause();
    bug_normal_fn d = nullptr;
    void* u = nullptr;
    const int rc = P.rng_fork(P.rng_fork_user, &d, &u);
    if (e.buf) e.buf->resume();
    require(rc == 0 && d, "parallel: the draw-stream fork failed");
    return {d, u};
  }
  // `left` on this step, `right` at the same time on a copy of it bound to the context's second
  // stream (fork_begin) and the forked draw stream, driven by a thread of its own; both are done
  // and the parent stream is ordered after both when this returns. The halves share no mutable
  // state: each writes its own outputs (the one shared vector, `expanded`, at disjoint bonds).
  // A profiled context (every launch timed on its one stream), or BUG_PARALLEL_SERIAL=1, runs the
  // halves in turn on this context instead: the same draws and results, no second stream.
  void run_halves(const std::function<void(Step&)>& left, const std::function<void(Step&)>& right,
                  std::pair<bug_normal_fn, void*> stream) {
    static const bool in_turn = [] {
      const char* v = std::getenv("BUG_PARALLEL_SERIAL");
      return v && std::string(v) == "1";
    }();
    DrawBuf rbuf;  // the forked stream is the half's alone: it is read ahead freely, never rewound
    rbuf.draw = stream.first;
    rbuf.user = stream.second;
    if (in_turn || e.c->profiling) {
      Eng er{e.c, stream.first, stream.second};
      er.buf = &rbuf;
      Step SR(er, mpo, P, tau, L);
      share_settings(SR);
      left(*this);
      right(SR);
      nmv += SR.nmv;
      return;
    }
    bug_ctx* ch = bugi::fork_begin(e.c);
    Eng er{ch, stream.first, stream.second};
    er.buf = &rbuf;
    Step SR(er, mpo, P, tau, L);
    share_settings(SR);
    std::exception_ptr rerr, lerr;
    std::thread th([&] {
      bool ok = true;
      try {
        right(SR);
      } catch (...) {
        rerr = std::current_exception();
        ok = false;
      }
      try {
        bugi::fork_child_done(ch, ok);
      } catch (...) {
        if (!rerr) rerr = std::current_exception();
      }
    });
    try {
      left(*this);
    } catch (...) {
      lerr = std::current_exception();
    }
    th.join();
    try {
      bugi::fork_end(e.c);
    } catch (...) {
      if (!lerr) lerr = std::current_exception();
    }
    nmv += SR.nmv;
    if (lerr) std::rethrow_exception(lerr);
    if (rerr) std::rethrow_exception(rerr);
  }

  // canonical form (canonical_form.jl)
  // `ahead`: the move's SVD is taken ahead of its read-back (svd_ahead) when there is room
  void move_right(MPS& psi, int site, bool ahead = false) {
    SVDRes r;
    if (!ahead || !svd_ahead1(e, psi[site], {0, 1}, W_U | W_SVD, r))
      r = svd(e, psi[site], {0, 1}, 0.0, -1, W_U | W_SVD);
    psi[site + 1] = e.contract(SVd(e, r), {1}, psi[site + 1], {0});
    psi[site] = r.U;
  }
  void move_left(MPS& psi, int site, bool ahead = false) {
    SVDRes r;
    if (!ahead || !svd_ahead1(e, psi[site], {0}, W_VD | W_US, r))
      r = svd(e, psi[site], {0}, 0.0, -1, W_VD | W_US);
    psi[site - 1] = e.contract(psi[site - 1], {2}, US(e, r), {0});
    psi[site] = r.Vd;
  }
  // The moves are a pure function of psi, so their SVDs are taken ahead (no read-back per move)
  // and checked once at the end; if a move met an exactly zero or non-finite singular value (or an
  // unconverged sector), the moves are redone from the saved state with read-backs, as the
  // reference's svd with cutoff 0 takes them.
  void canonical(MPS& psi, int site) {
    if (psi.center == site) return;
    MPS saved = psi;
    for (bool ahead : {true, false}) {
      if (!ahead) psi = saved;
      while (psi.center < site) {
        move_right(psi, psi.center, ahead);
        psi.center += 1;
      }
      while (psi.center > site) {
        move_left(psi, psi.center, ahead);
        psi.center -= 1;
      }
      if (!ahead || svd_ahead_check(e.c)) return;
    }
  }
  int total_charge(const MPS& psi) const { return psi[psi.size()]->legs[2].q.at(0); }

  std::vector<T> right_env_stack(const MPS& psi, int downto) {
    std::vector<T> envs(L + 2);
    T cur = env.right_boundary(total_charge(psi));
    envs[L + 1] = cur;
    for (int site = L; site >= downto; --site) {
      cur = env.right_step(cur, psi[site], mpo[site]);
      envs[site] = cur;
    }
    return envs;
  }
  std::vector<T> left_env_stack(const MPS& psi, int upto) {
    std::vector<T> envs(L + 2);
    T cur = env.left_boundary();
    envs[1] = cur;
    for (int site = 1; site <= upto; ++site) {
      cur = env.left_step(cur, psi[site], mpo[site]);
      envs[site + 1] = cur;
    }
    return envs;
  }

  BondFrame frame_from(const T& left, const T& right) {
    auto both = svd2x(left, {0, 1}, W_U | W_SVD, right, {0}, W_US | W_VD);
    SVDRes& rl = both.first;
    SVDRes& rr = both.second;
    T core = e.contract(SVd(e, rl), {1}, US(e, rr), {0});
    return BondFrame{rl.U, core, rr.Vd, dim(rl.U, 2)};
  }
  BondFrame frame_onto_left(const T& liso, const T& carry, const T& right) {
    return frame_onto_left(liso, carry, svd(e, right, {0}, 0.0, -1, W_US | W_VD));
  }
  BondFrame frame_onto_left(const T& liso, const T& carry, const SVDRes& rr) {
    T ov = e.contract(liso, {0, 1}, carry, {0, 1}, true, false);
    return BondFrame{liso, e.contract(ov, {1}, US(e, rr), {0}), rr.Vd, dim(liso, 2)};
  }
  BondFrame frame_onto_right(const T& left, const T& carry, const T& riso) {
    return frame_onto_right(svd(e, left, {0, 1}, 0.0, -1, W_U | W_SVD), carry, riso);
  }
  BondFrame frame_onto_right(const SVDRes& rl, const T& carry, const T& riso) {
    T ov = e.contract(carry, {1, 2}, riso, {1, 2}, false, true);
    return BondFrame{rl.U, e.contract(SVd(e, rl), {1}, ov, {0}), riso, dim(riso, 0)};
  }
  T polar_frame(const T& frame, bool left) {
    return polar_of(left ? svd(e, frame, {0, 1}, 0.0) : svd(e, frame, {0}, 0.0), left);
  }
  T polar_of(const SVDRes& r, bool left) { return e.contract(r.U, {left ? 2 : 1}, r.Vd, {0}); }

  // _record_sample! (sketch.jl:215-258): the ledger's sample maxima
  static void record_sample(Ledger* ledger, bool left, double ind) {
    if (!ledger) return;
    ledger->max_sample = std::max(ledger->max_sample, ind);
    if (left) ledger->max_sample_l = std::max(ledger->max_sample_l, ind);
    else ledger->max_sample_r = std::max(ledger->max_sample_r, ind);
  }

  // _dd_controller (dd_cbe_controller.jl:26-212, no audit): grows the DD basis block by block
  // until an independent holdout of `holdout_width` probe columns finds the rest within
  // acceptance_factor x the sample allowance. Probe draws in the reference's order. Streaming a
  // block (probe or holdout) sets `width` to its column count: the reference's `stream` closure
  // assigns the enclosing `width` (dd_cbe_controller.jl:108-118).
  T dd_controller(const T& frame, const T& opp, bool left, const std::function<T(const T&)>& sketch,
                  const std::function<T(const T&)>& project, int64_t initial_width, int64_t wcap,
                  int64_t ncap, Ledger* ledger) {
    const int fl = left ? 2 : 0, wleg = left ? 0 : 2;
    const int64_t holdout_width = P.holdout_width;
    T aug = frame, basis;
    int64_t count = 0, discovered = 0, width = 0;
    std::map<int, int64_t> boost;
    auto remaining = [&]() -> int64_t { return ncap - (basis ? dim(basis, fl) : 0); };
    auto draw = [&](int64_t w, bool boosted) {
      return dd_probe(e, opp, !left, int(w), boosted && !boost.empty() ? &boost : nullptr);
    };
    auto absorb = [&](const T& sketched) -> int64_t {
      if (!sketched) return 0;
      T nb = dd_select(e, aug, sketched, left);
      if (!nb) return 0;
      const int64_t room = remaining();
      if (room <= 0) return 0;
      if (dim(nb, fl) > room) {
        if (P.cap_selection_svd) {
          // the strongest sampled directions across sectors: an SVD of the thin projected
          // sketch (dd_cbe_controller.jl:67-96)
          T off = left ? perp_left(e, aug, sketched) : perp_right(e, aug, sketched);
          const double noff = e.norm(off);
          SVDRes fac = svd(e, off, left ? std::vector<int>{0, 1} : std::vector<int>{1, 2},
                           rank_cut(0.0, noff, noff), int(room), W_U);
          nb = fac.kept.empty() ? nullptr
                                : (left ? reortho(e, aug, fac.U, true)
                                        : reortho(e, aug, rows_from_u(e, fac.U), false));
        } else {
          nb = e.trim_total(nb, fl, room);
        }
        if (!nb) return 0;
      }
      basis = basis ? e.oplus({basis, nb}, fl) : nb;
      aug = e.oplus({aug, nb}, fl);
      return dim(nb, fl);
    };
    auto stream = [&](const T& Om, bool probe) {
      width = dim(Om, wleg);
      if (probe) {
        discovered += width;
        if (ledger) ledger->n_probes += width;
      } else if (ledger) {
        ledger->n_holdout += width;
      }
      return sketch(Om);
    };
    struct Check {
      T Om, sk;
    };
    auto fresh = [&](int64_t columns) -> Check {
      T Om = draw(columns, false);
      if (!Om) return Check{};
      return Check{Om, stream(Om, false)};
    };
    auto newsector = [&]() {
      if (!basis) return false;
      for (int q : basis->legs[fl].q)
        if (frame->legs[fl].dim_of(q) == 0) return true;
      return false;
    };
    if (P.cap_selection_svd)
      width = std::min(std::max<int64_t>(std::max(initial_width, ncap + std::min<int64_t>(4, ncap)), 1),
                       std::max<int64_t>(wcap, 1));
    else
      width = std::min(std::max<int64_t>(initial_width, 1), std::max<int64_t>(std::min(wcap, ncap), 1));
    T last = draw(width, false);
    if (!last) return nullptr;
    count += absorb(stream(last, true));
    Check check = fresh(holdout_width);
    bool escalated = false;
    while (true) {
      if (!check.Om) return basis;
      const TestB tb = sample_residual_sectors(e, basis, project, check.sk, check.Om, wleg, left);
      const double ind = indicator(alloc, tb.est);
      const bool ok = ind <= P.acceptance_factor * alloc.sample;
      if (ok && !escalated && (ind > alloc.sample / 2 || newsector())) {
        escalated = true;
        Check wide = fresh(2 * holdout_width);
        if (wide.Om) {
          check = wide;
          continue;
        }
      }
      const bool capped = discovered >= wcap || count >= ncap;
      if (ok || capped) {
        record_sample(ledger, left, ind);
        if (ok) return basis;
        if (ledger) {
          ledger->unmet_(U_SAMPLE);
          ledger->workcap_reached = true;
        }
        return basis;
      }
      const int nt = target_sectors(boost, tb, check.Om, wleg, alloc.scale, alloc.sample);
      if (ledger) ledger->n_targeted += nt;
      int64_t added = 0;
      if (P.batch_blocks == 1) {
        Check next_check = fresh(holdout_width);
        added = absorb(check.sk);
        if (nt == 0) width = std::min(2 * width, wcap);
        if (remaining() > 0) {
          T blk = draw(std::min(width, std::max<int64_t>(remaining() + 2, 1)), true);
          if (blk) {
            last = blk;
            added += absorb(stream(blk, true));
          }
        }
        check = next_check;
      } else {
        // the failed holdout is absorbed, then up to batch_blocks targeted blocks before the next
        // holdout is drawn (dd_cbe_controller.jl:186-202)
        added = absorb(check.sk);
        for (int b = 0; b < P.batch_blocks; ++b) {
          if (remaining() <= 0) break;
          if (nt == 0) width = std::min(2 * width, wcap);
          T blk = draw(std::min(width, std::max<int64_t>(remaining() + 2, 1)), true);
          if (!blk) break;
          last = blk;
          added += absorb(stream(blk, true));
        }
        check = fresh(holdout_width);
      }
      count += added;
      if (added == 0) {
        record_sample(ledger, left, ind);
        if (ledger) ledger->unmet_(U_SAMPLE);
        return basis;
      }
    }
  }

  // DD-QR CBE (dd_cbe_expand.jl:19-419): rank by tail bisection (:rank_tail, tail_dd) or by the
  // incremental controller (:adaptive, _dd_controller)
  Expansion dd_cbe_expand(const BondFrame& fr, int bond, const T& lenv, const T& renv, bool left,
                          Ledger* ledger, int64_t workcap) {
    const T& U0 = fr.U0;
    const T& V0 = fr.V0;
    const int64_t old_rank = fr.old_rank;
    const T& frame = left ? U0 : V0;
    const T& opp = left ? V0 : U0;
    const int fl = left ? 2 : 0, wleg = left ? 0 : 2;
    Expansion none{U0, V0, 0, 0};
    const int64_t full_self = left ? dim(U0, 0) * dim(U0, 1) : dim(V0, 1) * dim(V0, 2);
    const int64_t full_opp = left ? dim(V0, 1) * dim(V0, 2) : dim(U0, 0) * dim(U0, 1);
    int64_t cap = full_self - old_rank;
    bool wbind = false;
    if (workcap > 0) {
      const int64_t wk = std::max<int64_t>(workcap - old_rank, 0);
      wbind = wk < cap;
      cap = std::min(cap, wk);
    }
    if (cap <= 0) return none;
    const T& Wl = mpo[bond];
    const T& Wr = mpo[bond + 1];
    T core = left ? e.contract(U0, {2}, fr.S0, {0}) : e.contract(fr.S0, {1}, V0, {0});
    auto sketch = [&](const T& Om) {
      return left ? env.stream_left(core, V0, Wl, Wr, lenv, renv, Om)
                  : env.stream_right(U0, core, Wl, Wr, lenv, renv, Om);
    };
    auto project = [&](const T& b) { return left ? perp_left(e, U0, b) : perp_right(e, V0, b); };
    T Om, directions, Y;
    double nY = 0.0;
    int64_t direction_count = 0;
    if (P.exact) {
      // exact = true: the complete DD-projected fused basis sketched once and _dd_select's QR; the
      // certified range without an allocation stops after this pass, its width cap being its start
      // width (dd_cbe_expand.jl:91,346-360; sketch.jl:119-132). The mode is not consulted.
      T probe = dd_probe_exact(e, opp, !left);
      if (probe) {
        directions = dd_select(e, frame, sketch(probe), left);
        direction_count = directions ? dim(directions, fl) : 0;
      }
    } else if (P.dd_mode == 1) {
      const int64_t dmax = std::max({dim(U0, 0), old_rank, dim(V0, 2)});
      const int64_t grow = int64_t(std::ceil(ADAPTIVE_GROWTH * double(dmax))) - old_rank;
      const int64_t initial_width = int64_t(std::ceil(1.2 * double(std::max<int64_t>(grow, 1))));
      int64_t wcap = full_opp;
      if (workcap > 0) wcap = std::min(wcap, workcap);
      directions = dd_controller(frame, opp, left, sketch, project, initial_width, wcap, cap, ledger);
      direction_count = directions ? dim(directions, fl) : 0;
    } else {
      // the probe's non-zero test and |Y| come back together: Y is formed before the test is known
      double2* q = static_cast<double2*>(e.c->scratch(2 * sizeof(double2)));
      Om = dd_probe(e, opp, !left, int(std::min<int64_t>(P.fixed_width, full_opp)), nullptr, q);
      if (Om) {
        Y = project(sketch(Om));
        dots_device(e.c, {{Y.get(), Y.get()}}, q + 1);
        double* host = e.c->readback(4);
        e.c->drain();  // the queued dot stages write the slots: they run before the copy
        BUG_CUDA(cudaMemcpyAsync(host, q, 2 * sizeof(double2), cudaMemcpyDeviceToHost, e.c->stream));
        e.c->wait();
        if (!(std::sqrt(std::max(host[0], 0.0)) > 0)) Om = nullptr;
        nY = std::sqrt(std::max(host[2], 0.0));
      }
    }
    if (Om) {
      if (ledger) ledger->n_probes += dim(Om, wleg);
      if (!(nY <= CBE_EPS)) {
        std::vector<int> legs = left ? std::vector<int>{0, 1} : std::vector<int>{1, 2};
        const int64_t rmax = std::min(cap, dim(Om, wleg));
        std::map<int64_t, T> cache;
        auto candidate = [&](int64_t k) -> T {
          if (k <= 0) return nullptr;
          auto it = cache.find(k);
          if (it != cache.end()) return it->second;
          SVDRes fac = svd(e, Y, legs, rank_cut(0.0, nY, nY), int(k), W_U);
          T res;
          if (!fac.kept.empty()) res = left ? reortho(e, frame, fac.U, true)
                                            : reortho(e, frame, rows_from_u(e, fac.U), false);
          cache[k] = res;
          return res;
        };
        const double limit = P.tail_factor * alloc.sample;
        auto metric = [&](int64_t k) {
          const double est = sample_residual(e, candidate(k), project, [&](const T&) { return Y; },
                                             Om, wleg, left);
          return indicator(alloc, est);
        };
        if (!(metric(0) <= limit)) {
          int64_t hi = rmax;
          if (metric(hi) > limit) {
            directions = candidate(hi);
            direction_count = hi;
          } else {
            int64_t lo = 0;
            while (hi - lo > 1) {
              const int64_t k = (hi + lo) / 2;
              if (metric(k) <= limit) hi = k;
              else lo = k;
            }
            directions = candidate(hi);
            direction_count = directions ? dim(directions, fl) : 0;
          }
        }
      }
    }
    if (!directions) return none;
    if (direction_count > cap) {
      directions = e.trim_total(directions, fl, cap);
      if (!directions) return none;
    }
    if (ledger && wbind && direction_count >= cap) ledger->workcap_reached = true;
    directions = cap_to_local_room(e, frame, directions, left);
    if (!directions) return none;
    const int64_t nq = dim(directions, fl);
    if (ledger) ledger->n_selected += nq;
    T grown = e.oplus({frame, directions}, fl);
    if (left) return Expansion{grown, V0, nq, 0};
    return Expansion{U0, grown, 0, nq};
  }

  // ── Krylov weights and chains ──
  cd tau_eff;

  double kry_weight(const CMat& Hm, int k, bool state_seed) {
    const double beta = std::abs(Hm(k, k - 1));
    if (beta == 0) return 0.0;
    CMat g(k, k);
    for (int i = 0; i < k; ++i)
      for (int j = 0; j < k; ++j) g(i, j) = tau_eff * Hm(i, j);
    return beta * residual_integral(k - 1, g, tau_eff, state_seed);
  }

  struct Chain {
    std::vector<T> basis;
    int64_t n_h1 = 0;
    bool closed = false, capped = false;
  };

  // The chain's scalars stay on the device until ONE read-back per step: the Lanczos alpha
  // (slot 0), |image|^2 (slot 1), the score residual's |r|^2 (slot 2), the seed's |s|^2 (slot 3,
  // step 1) and, for Arnoldi, the two CGS passes' coefficients (slots 4 .. 4 + 2k). The
  // combinations that need them read them from device memory (DevTerm modes), so every value is
  // the one a chain with host scalars computes. Work whose need the read-back decides runs ahead
  // of it and is dropped when not needed: the first application before the seed is known to be
  // non-zero (not counted then), the score residual before the breakdown test. `applyH` must not
  // count its applications: `n_h1` holds the chain's. `prep` forms the score residual of a new
  // direction and queues its squared norm into a slot; `decide` takes the read-back norm and
  // returns false to cap.
  Chain krylov_basis(const T& seed, const std::function<T(const T&)>& applyH, double allowance,
                     const std::function<T(const T&, double2*)>& prep,
                     const std::function<bool(const T&, const T&, double, double, bool)>& decide,
                     double amp, bool state_seed, bool lanczos) {
    Chain ch;
    tau_eff = tau == cd(0) ? cd(1.0) : tau;
    const int maxdepth = KRY_MAXDEPTH;
    CMat Hm(maxdepth + 1, maxdepth + 1);
    double2* slot = static_cast<double2*>(e.c->scratch(size_t(4 + 2 * maxdepth) * sizeof(double2)));
    auto re = [](const double2* q) { return reinterpret_cast<const double*>(q); };
    dots_device(e.c, {{seed.get(), seed.get()}}, slot + 3);
    ch.basis.push_back(lin_dev({{0.0, 2, re(slot + 3), seed}}));  // seed / |seed|
    std::vector<T>& vs = ch.basis;
    double prev_beta = 0.0;
    for (int step = 1; step <= maxdepth; ++step) {
      T image = applyH(lanczos ? vs[step - 1] : vs.back());
      ch.n_h1 += 1;
      const int k = int(vs.size());
      if (lanczos) {
        if (step > 1) image = e.lin({{1.0, image}, {-prev_beta, vs[step - 2]}});
        dots_device(e.c, {{vs[step - 1].get(), image.get()}}, slot);
        image = lin_dev({{1.0, 0, nullptr, image}, {0.0, 1, re(slot), vs[step - 1]}});
        if (step >= 20 && step % 2 == 0) {
          auto cs = e.inner_many(vs, image);
          std::vector<std::pair<cd, T>> terms{{1.0, image}};
          for (size_t i = 0; i < vs.size(); ++i) terms.push_back({-cs[i], vs[i]});
          image = e.lin(terms);
        }
      } else {
        for (int pass = 0; pass < 2; ++pass) {
          double2* cs = slot + 4 + pass * k;
          std::vector<std::pair<const bug_tensor*, const bug_tensor*>> ps;
          for (auto& v : vs) ps.push_back({v.get(), image.get()});
          dots_device(e.c, ps, cs);
          std::vector<DevTerm> terms{{1.0, 0, nullptr, image}};
          for (int i = 0; i < k; ++i) terms.push_back({0.0, 4, re(cs + i), vs[size_t(i)]});
          image = lin_dev(terms);
        }
      }
      dots_device(e.c, {{image.get(), image.get()}}, slot + 1);
      T nv = lin_dev({{0.0, 2, re(slot + 1), image}});
      T residual = prep(nv, slot + 2);
      const int nread = lanczos ? 4 : 4 + 2 * k;
      double* host = e.c->readback(size_t(2 * nread));
      e.c->drain();  // the queued stages write the slots: they run before the copy
      BUG_CUDA(cudaMemcpyAsync(host, slot, size_t(nread) * sizeof(double2), cudaMemcpyDeviceToHost,
                               e.c->stream));
      e.c->wait();
      if (step == 1 && !(std::sqrt(std::max(host[6], 0.0)) > 0)) {
        ch = Chain{};  // a zero seed: no basis and no application
        ch.closed = true;
        return ch;
      }
      if (lanczos) {
        const cd alpha(host[0], host[1]);
        // with tensor-core contractions the matvec carries FP32-level error (about 1e-7 relative),
        // so the Hermiticity test allows that much instead of FP64 rounding
        const double herm_tol = e.c->mixed_min_dim > 0 ? 1e-5 : 1e-9;
        require(std::abs(alpha.imag()) <= herm_tol * std::max(std::abs(alpha), 1.0),
                "Lanczos needs a Hermitian one-site generator");
        Hm(step - 1, step - 1) = alpha.real();
      } else {
        for (int pass = 0; pass < 2; ++pass)
          for (int i = 0; i < k; ++i) {
            const double* c2 = host + 2 * (4 + pass * k + i);
            Hm(i, step - 1) += cd(c2[0], c2[1]);
          }
      }
      const double beta = std::sqrt(std::max(host[2], 0.0));
      if (beta <= KRY_BREAKDOWN) {
        ch.closed = true;
        break;
      }
      Hm(step, step - 1) = beta;
      if (lanczos) Hm(step - 1, step) = beta;
      vs.push_back(nv);
      const double w = amp * kry_weight(Hm, step, state_seed);
      if (!decide(residual, nv, w, std::sqrt(std::max(host[4], 0.0)), step == 1)) {
        ch.capped = true;
        break;
      }
      // _krylov_stop with fixed_depth
      bool stop, closed;
      if (P.fixed_depth > 0) {
        stop = step >= P.fixed_depth;
        closed = stop && w <= allowance;
      } else {
        stop = w <= allowance;
        closed = stop;
      }
      ch.closed = closed;
      if (stop) break;
      prev_beta = beta;
    }
    if (!ch.closed) ch.capped = true;
    return ch;
  }

  struct KStats {
    double eta_c = 0, eta_d = 0;
    int64_t added = 0, n_h1 = 0;
    bool d_after_c = false, capped = false, met = false;
  };

  std::tuple<T, int64_t, bool> extend_frame(const T& frame, const T& residual, const T& direction,
                                            bool left, double weight, double allowance, int64_t room) {
    std::vector<int> legs = left ? std::vector<int>{0, 1} : std::vector<int>{1, 2};
    const auto nrd = e.norms(residual, direction);  // one read-back for both
    const double nres = nrd.first;
    const double cut = rank_cut(0.0, nrd.second, nres);
    SVDRes res = svd(e, residual, legs, cut, -1, W_U);
    const int nk = int(res.kept.size());
    auto tr = tail_rank(res.kept, weight, allowance, int(std::min<int64_t>(nk, room)), sq_weight(res.trunc));
    const bool fits = tr.second <= allowance;
    if (tr.first == 0) return {frame, 0, fits};
    if (tr.first < nk) res = svd(e, residual, legs, cut, tr.first, W_U);
    T nb = left ? reortho(e, frame, res.U, true) : reortho(e, frame, rows_from_u(e, res.U), false);
    nb = cap_to_local_room(e, frame, nb, left);
    if (!nb) return {frame, 0, fits};
    const int fl = left ? 2 : 0;
    return {e.oplus({frame, nb}, fl), dim(nb, fl), fits};
  }

  std::pair<T, KStats> krylov_enrich(const T& seed, const std::function<T(const T&)>& applyH,
                                     const T& start_frame, bool left, int64_t workcap, double amp,
                                     bool state_seed) {
    const int fl = left ? 2 : 0;
    const double allow = alloc.krylov;
    T frame = start_frame;
    KStats st;
    int64_t added_d = 0;
    auto prep = [&](const T& dir, double2* slot) {
      T residual = left ? perp_left(e, frame, dir) : perp_right(e, frame, dir);
      dots_device(e.c, {{residual.get(), residual.get()}}, slot);
      return residual;
    };
    auto decide = [&](const T& residual, const T& dir, double w, double rnorm, bool first) {
      const double eta = w * rnorm;
      if (first) st.eta_c = eta;
      else st.eta_d = std::max(st.eta_d, eta);
      if (!(eta > allow)) return true;
      const int64_t room = workcap > 0 ? workcap - dim(frame, fl) : (int64_t(1) << 62);
      if (room <= 0) return false;
      auto r = extend_frame(frame, residual, dir, left, w, allow, room);
      frame = std::get<0>(r);
      st.added += std::get<1>(r);
      if (!first) added_d += std::get<1>(r);
      return std::get<2>(r);
    };
    Chain ch = krylov_basis(seed, applyH, alloc.krylov, prep, decide, amp, state_seed,
                            P.lanczos != 0);
    st.n_h1 = ch.n_h1;
    st.capped = ch.capped;
    st.d_after_c = st.eta_c <= alloc.krylov && added_d > 0;
    st.met = ch.closed && !ch.capped;
    return {frame, st};
  }

  void record_krylov(Ledger& l, const KStats& st) {
    l.max_krylov_c = std::max(l.max_krylov_c, st.eta_c);
    l.max_krylov_d = std::max(l.max_krylov_d, st.eta_d);
    l.max_krylov = std::max({l.max_krylov, st.eta_c, st.eta_d});
    l.n_krylov += st.added;
    l.n_h1 += st.n_h1;
    if (st.eta_c <= alloc.krylov) l.n_c_pass += 1;
    if (st.d_after_c) l.n_d_after_c += 1;
    if (st.capped) l.workcap_reached = true;
    if (!st.met) l.unmet_(U_KRYLOV);
  }

  // ── half-sweeps (half_sweeps.jl) ──
  // A half-sweep is a function of its inputs and its draws: its frames' cutoff-0 SVDs are taken
  // ahead (frame_from) and checked at its end; on a zero singular value the half runs again from
  // the saved state and draw position. Only this half's outputs are restored (the other half
  // writes its own bonds of `expanded`, possibly at the same time).
  template <class F>
  void half_ahead(MPS& psi, std::map<int, T>& frames, std::vector<int64_t>& expanded,
                  int b_lo, int b_hi, std::vector<int64_t>& nn, Ledger& hl, F body) {
    if (!e.buf) {
      body();
      return;
    }
    const MPS s_psi = psi;
    const std::map<int, T> s_frames = frames;
    const std::vector<int64_t> s_exp(expanded.begin() + (b_lo - 1),
                                     expanded.begin() + std::max(b_lo - 1, b_hi));
    const std::vector<int64_t> s_nn = nn;
    const Ledger s_hl = hl;
    const int64_t s_nmv = nmv;
    e.buf->save();
    frames_ahead = true;
    body();
    frames_ahead = false;
    if (svd_ahead_check(e.c)) {
      e.buf->drop();
      return;
    }
    e.buf->restore();
    psi = s_psi;
    frames = s_frames;
    std::copy(s_exp.begin(), s_exp.end(), expanded.begin() + (b_lo - 1));
    nn = s_nn;
    hl = s_hl;
    nmv = s_nmv;
    body();
  }
  T half_left(MPS& psiL, std::map<int, T>& lf, std::vector<int64_t>& expanded,
              std::vector<int64_t>& nn, Ledger& hl) {
    T out;
    half_ahead(psiL, lf, expanded, 1, root_link, nn, hl,
               [&] { out = half_left_body(psiL, lf, expanded, nn, hl); });
    return out;
  }
  std::pair<T, T> half_right(MPS& psiR, std::map<int, T>& rf, std::vector<int64_t>& expanded,
                             std::vector<int64_t>& nn, Ledger& hl) {
    std::pair<T, T> out;
    half_ahead(psiR, rf, expanded, root_link + 1, L - 1, nn, hl,  // bond root_link is the left's
               [&] { out = half_right_body(psiR, rf, expanded, nn, hl); });
    return out;
  }
  // ── kept states (keep_states / keep_tols, half_sweeps.jl:127-204) ──
  // _union_fresh: orthonormal directions of `cand` outside `frame` that survive a second
  // projection, at most `room` of them (the strongest), or null. tol = 0 admits every direction
  // above the numerical floor (`cand` is contained exactly); tol > 0 only those carrying more
  // than about tol |cand|.
  T union_fresh(const T& frame, const T& cand, bool left, double tol, int64_t room) {
    if (room <= 0) return nullptr;
    const std::vector<int> legs = left ? std::vector<int>{0, 1} : std::vector<int>{1, 2};
    auto perp = [&](const T& x) { return left ? perp_left(e, frame, x) : perp_right(e, frame, x); };
    auto orient = [&](const T& U) { return left ? U : rows_from_u(e, U); };
    T res = perp(cand);
    const auto nn = e.norms(cand, res);
    const double ncand = nn.first, nres = nn.second;
    if (nres <= CBE_EPS * std::max(ncand, 1.0) || nres <= tol * ncand) return nullptr;
    const double first_cut = std::max(rank_cut(0.0, ncand, nres), tol * ncand / nres);
    T basis = orient(svd(e, e.scale(res, cd(1.0 / nres)), legs, first_cut, -1, W_U).U);
    res = perp(basis);
    double smax = 0.0;
    for (auto& k : svd(e, res, legs, 1e-13, -1, W_U).kept) smax = std::max(smax, k.first);
    if (smax < UNION_KEEP) return nullptr;
    const int nkeep = room >= int64_t(INT32_MAX) ? -1 : int(room);
    return orient(svd(e, res, legs, UNION_KEEP / smax, nkeep, W_U).U);
  }
  // every kept state's carried site tensor unioned into `frame` in turn (_union_left/_right and
  // the loops at half_sweeps.jl:281-297, 385-398); under the :bond ceiling a tolerance-admitted
  // state fills the frame only up to the bond's work ceiling (_keep_room, :179-181)
  T union_kept(T frame, const std::vector<T>& cands, bool left, int bond) {
    const int fl = left ? 2 : 0;
    for (size_t i = 0; i < cands.size(); ++i) {
      const double tol = P.keep_tols[i];
      const int64_t room = P.cap_keep && tol > 0 ? cap_at(bond) - dim(frame, fl) : INT64_MAX;
      T fresh = union_fresh(frame, cands[i], left, tol, room);
      if (fresh) frame = e.oplus({frame, fresh}, fl);
    }
    return frame;
  }

  T half_left_body(MPS& psiL, std::map<int, T>& lf, std::vector<int64_t>& expanded,
                   std::vector<int64_t>& nn, Ledger& hl) {
    canonical(psiL, 1);
    auto rstack = right_env_stack(psiL, 3);
    T lch = env.left_boundary();
    T lroot = lch;
    T carry;
    std::vector<T> kcar(P.keep.size());  // each kept state's carry (b_i, link)
    for (int bond = 1; bond <= root_link; ++bond) {
      T carried = carry ? e.contract(carry, {1}, psiL[bond], {0}) : psiL[bond];
      BondFrame fr = frame_from(carried, psiL[bond + 1]);
      Ledger bl;
      Expansion ex = dd_cbe_expand(fr, bond, lch, rstack[bond + 2], true, &bl, cap_at(bond));
      nn[bond - 1] = ex.n_new_l;
      T rp = e.contract(psiL[bond + 1], {1, 2}, ex.V_ex, {1, 2}, false, true);
      T Kex = e.contract(carried, {2}, rp, {0});
      T rch1 = env.right_step(rstack[bond + 2], ex.V_ex, mpo[bond + 1]);
      const T& W = mpo[bond];
      auto applyH = [&](const T& v) { return h1(lch, W, rch1, v); };
      auto kr = krylov_enrich(Kex, applyH, ex.U_ex, true, cap_at(bond), 1.0, true);
      nmv += kr.second.n_h1;
      record_krylov(bl, kr.second);
      T Wk = kr.first;
      if (!P.keep.empty()) {
        std::vector<T> kx;
        for (size_t i = 0; i < P.keep.size(); ++i) {
          const T& site = P.keep[i][size_t(bond - 1)];
          kx.push_back(kcar[i] ? e.contract(kcar[i], {1}, site, {0}) : site);
        }
        Wk = union_kept(Wk, kx, true, bond);  // every union before any carry
        for (size_t i = 0; i < kx.size(); ++i) kcar[i] = e.contract(Wk, {0, 1}, kx[i], {0, 1}, true, false);
      }
      lf[bond] = Wk;
      expanded[bond - 1] = dim(Wk, 2);
      log_bond(hl, bl, bond, 0, int(expanded[bond - 1]));
      carry = e.contract(Wk, {0, 1}, carried, {0, 1}, true, false);
      if (bond == root_link) lroot = lch;
      if (bond < root_link) lch = env.left_step(lch, Wk, mpo[bond]);
    }
    return lroot;
  }

  std::pair<T, T> half_right_body(MPS& psiR, std::map<int, T>& rf, std::vector<int64_t>& expanded,
                                  std::vector<int64_t>& nn, Ledger& hl) {
    canonical(psiR, L);
    auto lstack = left_env_stack(psiR, L - 2);
    T rch = env.right_boundary(total_charge(psiR));
    T rroot = rch;
    T carry;
    std::vector<T> kcar(P.keep.size());  // each kept state's carry (link, b_j)
    for (int bond = L - 1; bond >= root_link; --bond) {
      T carried = carry ? e.contract(psiR[bond + 1], {2}, carry, {0}) : psiR[bond + 1];
      BondFrame fr = frame_from(psiR[bond], carried);
      Ledger bl;
      Expansion ex = dd_cbe_expand(fr, bond, lstack[bond], rch, false, &bl, cap_at(bond));
      nn[bond - 1] = ex.n_new_r;
      T lp = e.contract(ex.U_ex, {0, 1}, psiR[bond], {0, 1}, true, false);
      T Bex = e.contract(lp, {1}, carried, {0});
      T lch1 = env.left_step(lstack[bond], ex.U_ex, mpo[bond]);
      const T& W = mpo[bond + 1];
      auto applyH = [&](const T& v) { return h1(lch1, W, rch, v); };
      auto kr = krylov_enrich(Bex, applyH, ex.V_ex, false, cap_at(bond), 1.0, true);
      nmv += kr.second.n_h1;
      record_krylov(bl, kr.second);
      T Zk = kr.first;
      if (!P.keep.empty()) {
        std::vector<T> kx;
        for (size_t i = 0; i < P.keep.size(); ++i) {
          const T& site = P.keep[i][size_t(bond)];
          kx.push_back(kcar[i] ? e.contract(site, {2}, kcar[i], {0}) : site);
        }
        Zk = union_kept(Zk, kx, false, bond);
        for (size_t i = 0; i < kx.size(); ++i) kcar[i] = e.contract(kx[i], {1, 2}, Zk, {1, 2}, false, true);
      }
      rf[bond] = Zk;
      if (bond != root_link) expanded[bond - 1] = dim(Zk, 0);
      log_bond(hl, bl, bond, 1, int(dim(Zk, 0)));
      carry = e.contract(carried, {1, 2}, Zk, {1, 2}, false, true);
      if (bond == root_link) rroot = rch;
      if (bond > root_link) rch = env.right_step(rch, Zk, mpo[bond + 1]);
    }
    return {rroot, carry};
  }

  // ── overlaps and projections (krylov_closure_frames.jl) ──
  T overlap_left(const MPS& psi, std::map<int, T>& lf) {
    T AL;
    for (int site = 1; site <= root_link; ++site) {
      T carried = AL ? e.contract(AL, {1}, psi[site], {0}) : psi[site];
      AL = e.contract(lf[site], {0, 1}, carried, {0, 1}, true, false);
    }
    return AL;
  }
  T overlap_right(const MPS& psi, std::map<int, T>& rf) {
    T AR;
    for (int bond = L - 1; bond >= root_link; --bond) {
      T carried = AR ? e.contract(psi[bond + 1], {2}, AR, {0}) : psi[bond + 1];
      AR = e.contract(carried, {1, 2}, rf[bond], {1, 2}, false, true);
    }
    return AR;
  }
  // The outside components' squared norms go to device slots and come back in one read-back at
  // the end, summed in the order the terms arise; the factors' SVDs are taken ahead (svd_ahead)
  // and checked with that read-back, the measurement redone with read-backs if one failed.
  double projection_miss(const MPS& psi, std::map<int, T>& lf, std::map<int, T>& rf) {
    double out = 0.0;
    if (!projection_miss_once(psi, lf, rf, true, out)) projection_miss_once(psi, lf, rf, false, out);
    return out;
  }
  bool projection_miss_once(const MPS& psi, std::map<int, T>& lf, std::map<int, T>& rf, bool ahead,
                            double& out) {
    double2* n2 = static_cast<double2*>(e.c->scratch(size_t(L + 1) * sizeof(double2)));
    int nterm = 0;
    auto miss_term = [&](const T& x) { dots_device(e.c, {{x.get(), x.get()}}, n2 + nterm++); };
    auto factor = [&](const T& t, std::vector<int> left, int want) {
      SVDRes r;
      if (!ahead || !svd_ahead1(e, t, left, want, r)) r = svd(e, t, left, 0.0, -1, want);
      return r;
    };
    std::vector<T> rfac(L + 2);
    for (int site = L; site >= 2; --site) {
      T carried = site == L ? psi[L] : e.contract(psi[site], {2}, rfac[site + 1], {0});
      rfac[site] = US(e, factor(carried, {0}, W_US));
    }
    T AL;
    for (int site = 1; site <= root_link; ++site) {
      T carried = AL ? e.contract(AL, {1}, psi[site], {0}) : psi[site];
      T outside = perp_left(e, lf[site], carried);
      miss_term(e.contract(outside, {2}, rfac[site + 1], {0}));
      AL = e.contract(lf[site], {0, 1}, carried, {0, 1}, true, false);
    }
    std::vector<T> lfac(L + 1);
    lfac[root_link] = SVd(e, factor(AL, {0}, W_SVD));
    for (int bond = root_link + 1; bond <= L - 1; ++bond)
      lfac[bond] = SVd(e, factor(e.contract(lfac[bond - 1], {1}, psi[bond], {0}), {0, 1}, W_SVD));
    T AR;
    for (int bond = L - 1; bond >= root_link; --bond) {
      T carried = AR ? e.contract(psi[bond + 1], {2}, AR, {0}) : psi[bond + 1];
      T outside = perp_right(e, rf[bond], carried);
      miss_term(e.contract(lfac[bond], {1}, outside, {0}));
      AR = e.contract(carried, {1, 2}, rf[bond], {1, 2}, false, true);
    }
    double* host = e.c->readback(size_t(2 * std::max(nterm, 1)));
    if (nterm > 0) {
      e.c->drain();  // the queued dot stages write the slots: they run before the copy
      BUG_CUDA(cudaMemcpyAsync(host, n2, size_t(nterm) * sizeof(double2), cudaMemcpyDeviceToHost,
                               e.c->stream));
    }
    const bool waited = !e.c->ahead.empty();  // the check waits, for the copy too
    if (!svd_ahead_check(e.c)) return false;
    if (nterm > 0 && !waited) e.c->wait();
    double miss2 = 0.0;
    for (int i = 0; i < nterm; ++i) miss2 += std::pow(std::sqrt(std::max(host[2 * i], 0.0)), 2);
    out = std::sqrt(miss2);
    return true;
  }

  // ── closure (single pass, folded leak) ──
  struct KL {
    std::map<int, T> lf, rf;
    T lenv, renv;
    int gen = 0;
  };
  ZeroSiteH root_generator(KL& fr) {
    return ZeroSiteH{env.left_step(fr.lenv, fr.lf[root_link], mpo[root_link]),
                     env.right_step(fr.renv, fr.rf[root_link], mpo[root_link + 1]), eshift};
  }
  // H1 - eshift on a site tensor (shift_h: eshift = 0 is the unshifted action itself)
  T h1(const T& lch, const T& W, const T& rch, const T& v) const {
    T y = env.one_site(lch, W, rch, v);
    return eshift == 0.0 ? y : e.lin({{1.0, y}, {-eshift, v}});
  }
  T project_root(const MPS& psi, KL& fr) {
    return e.contract(overlap_left(psi, fr.lf), {1}, overlap_right(psi, fr.rf), {0});
  }
  MPS frontier_mps(const MPS& /*psi*/, KL& fr, const T& core) {
    MPS m;
    for (int s = 1; s < root_link; ++s) m.s.push_back(fr.lf[s]);
    m.s.push_back(e.contract(fr.lf[root_link], {2}, core, {0}));
    for (int b = root_link; b < L; ++b) m.s.push_back(fr.rf[b]);
    m.center = root_link;
    return m;
  }

  // _bond_action (krylov_frontier_bonds.jl:80-100). Folded: the sketch closures with the probe
  // folded into the environment contractions and the sampled leak (cbe.jl:62-144, 355-391).
  // Unfolded (fold_omega = false): the two-site action X = H Theta_F formed once and the exact
  // leak |(I - U0 U0^dag) X| or |X (I - V0^dag V0)| (_left_leak/_right_leak, :37-66), no draws.
  double bond_action(const BondFrame& fr, int bond, const T& lenv, const T& renv, bool left) {
    const T& Wl = mpo[bond];
    const T& Wr = mpo[bond + 1];
    T theta = frame_theta(e, fr);
    if (!P.fold) {
      T X = env.two_site(lenv, Wl, Wr, renv, theta);  // (l, s1, s2, r)
      if (left) return e.norm(perp_left(e, fr.U0, X));
      T ov = e.contract(X, {2, 3}, fr.V0, {1, 2}, false, true);  // (l, s1, bond)
      return e.norm(e.lin({{1.0, X}, {-1.0, e.contract(ov, {2}, fr.V0, {0})}}));
    }
    const int64_t grown = left ? dim(fr.U0, 2) : dim(fr.V0, 0);
    const int count = int(std::max<int64_t>(8, (grown + 3) / 4));
    if (left) {
      auto skl = [&](const T& Om) {
        T t = e.contract(Om, {2}, renv, {0}, true, false);
        T rc = e.contract(t, {1, 2}, Wr, {2, 3});
        T tc = e.contract(theta, {2, 3}, rc, {3, 1});
        T wm = e.contract(tc, {1, 3}, Wl, {1, 3});
        t = e.contract(wm, {0, 2}, lenv, {2, 1});
        return perp_left(e, fr.U0, e.permute(t, {2, 1, 0}));
      };
      T Om = graded_sketch(e, fr.V0, false, count);
      return sample_residual(e, nullptr, [&](const T& s) { return perp_left(e, fr.U0, s); }, skl,
                             Om, 0, true);
    }
    auto skr = [&](const T& Om) {
      T t = e.contract(Om, {0}, lenv, {0}, true, false);
      T cap = e.permute(e.contract(t, {0, 2}, Wl, {2, 0}), {1, 0, 2, 3});
      T tc = e.contract(theta, {0, 1}, cap, {0, 2});
      T wm = e.contract(tc, {0, 3}, Wr, {1, 0});
      t = e.contract(wm, {0, 3}, renv, {2, 1});
      return perp_right(e, fr.V0, t);
    };
    T Om = graded_sketch(e, fr.U0, true, count);
    return sample_residual(e, nullptr, [&](const T& s) { return perp_right(e, fr.V0, s); }, skr, Om,
                           2, false);
  }

  struct FrontierHalf {
    std::map<int, T> frames;
    T env;
    Ledger ledger;
    std::vector<double> leak;
    int64_t added = 0, n_h1 = 0, n_h2 = 0;
  };

  // A frontier half is a function of its inputs and its draws, so its cutoff-0 SVDs (the frames
  // and polar factors) are taken ahead of their read-back (svd_ahead) and checked once at its end;
  // if a singular value was exactly zero, the half is run again from the same draw position with
  // read-backs. Without a buffered draw stream (nothing to rewind) it runs with read-backs.
  bool frames_ahead = false;
  SVDRes svdx(const T& t, std::vector<int> left, int want) {
    SVDRes r;
    if (!frames_ahead || !svd_ahead1(e, t, left, want, r)) r = svd(e, t, left, 0.0, -1, want);
    return r;
  }
  std::pair<SVDRes, SVDRes> svd2x(const T& t1, std::vector<int> l1, int w1, const T& t2,
                                  std::vector<int> l2, int w2) {
    if (!frames_ahead) return svd2(e, t1, l1, w1, t2, l2, w2);
    std::pair<SVDRes, SVDRes> r;
    if (svd2_ahead(e, t1, l1, w1, t2, l2, w2, r)) return r;
    return svd2(e, t1, l1, w1, t2, l2, w2);
  }
  template <class F> auto with_frames_ahead(F body) -> decltype(body()) {
    if (e.buf) {
      e.buf->save();
      frames_ahead = true;
      auto out = body();
      frames_ahead = false;
      if (svd_ahead_check(e.c)) {
        e.buf->drop();
        return out;
      }
      e.buf->restore();
    }
    return body();
  }
  FrontierHalf frontier_left(const MPS& Fm, KL& fr, double amp, bool enrich = true) {
    return with_frames_ahead([&] { return frontier_left_body(Fm, fr, amp, enrich); });
  }
  FrontierHalf frontier_right(const MPS& Fm, KL& fr, double amp, bool enrich = true) {
    return with_frames_ahead([&] { return frontier_right_body(Fm, fr, amp, enrich); });
  }

  // enrich = false measures only (estimate_global_complement_action): the frames stay, the
  // environments are the frames' own
  FrontierHalf frontier_left_body(const MPS& Fm0, KL& fr, double amp, bool enrich) {
    MPS Fm = Fm0;
    FrontierHalf out;
    canonical(Fm, 1);
    auto rstack = right_env_stack(Fm, 3);
    T lch = env.left_boundary();
    T lenv = lch;
    T carry, Pm;
    std::map<int, T> chain;
    if (!enrich) {
      T ch = env.left_boundary();
      for (int bond = 1; bond <= root_link; ++bond) {
        chain[bond] = ch;
        if (bond < root_link) ch = env.left_step(ch, fr.lf.at(bond), mpo[bond]);
      }
    }
    for (int bond = 1; bond <= root_link; ++bond) {
      if (!enrich) lch = chain[bond];
      T old = Pm ? e.contract(Pm, {1}, fr.lf.at(bond), {0}) : fr.lf.at(bond);
      T site_core = carry ? e.contract(carry, {1}, Fm[bond], {0}) : Fm[bond];
      // enriching: the frame's SVD and, ahead of the quiet test, the polar factor of `old` (the
      // new frame of a quiet bond) come back together
      SVDRes pol;
      BondFrame tsf;
      if (enrich) {
        auto both = svd2x(Fm[bond + 1], {0}, W_US | W_VD, old, {0, 1}, W_U | W_VD);
        tsf = frame_onto_left(old, site_core, both.first);
        pol = std::move(both.second);
      } else {
        tsf = frame_onto_left(old, site_core, svdx(Fm[bond + 1], {0}, W_US | W_VD));
      }
      const T& rch = rstack[bond + 2];
      const double lk = bond_action(tsf, bond, lch, rch, true);
      if (!P.fold) out.n_h2 += 1;
      out.leak.push_back(lk);
      Ledger bl;
      const bool quiet = indicator(alloc, lk) <= alloc.per_bond;
      T Wi;
      if (enrich && !quiet) {
        Expansion ex = dd_cbe_expand(tsf, bond, lch, rch, true, &bl, cap_at(bond));
        T rp = e.contract(Fm[bond + 1], {1, 2}, ex.V_ex, {1, 2}, false, true);
        T Kex = e.contract(site_core, {2}, rp, {0});
        T rch1 = env.right_step(rch, ex.V_ex, mpo[bond + 1]);
        const T& W = mpo[bond];
        auto applyH = [&](const T& v) { return h1(lch, W, rch1, v); };
        auto kr = krylov_enrich(Kex, applyH, ex.U_ex, true, cap_at(bond), amp, false);
        out.n_h1 += kr.second.n_h1;
        record_krylov(bl, kr.second);
        Wi = kr.first;
      } else {
        Wi = old;
      }
      T Wn = !enrich ? old : (quiet ? polar_of(pol, true) : polar_of(svdx(Wi, {0, 1}, W_U | W_VD), true));
      out.frames[bond] = Wn;
      out.added += dim(Wn, 2) - dim(old, 2);
      log_bond(out.ledger, bl, bond, 0, int(dim(Wn, 2)));
      if (enrich) Pm = e.contract(Wn, {0, 1}, old, {0, 1}, true, false);
      carry = e.contract(Wn, {0, 1}, site_core, {0, 1}, true, false);
      if (bond == root_link) lenv = lch;
      if (enrich && bond < root_link) lch = env.left_step(lch, Wn, mpo[bond]);
    }
    out.env = lenv;
    return out;
  }

  FrontierHalf frontier_right_body(const MPS& Fm0, KL& fr, double amp, bool enrich) {
    MPS Fm = Fm0;
    FrontierHalf out;
    canonical(Fm, L);
    auto lstack = left_env_stack(Fm, L - 2);
    T rch = env.right_boundary(total_charge(Fm));
    T renv = rch;
    T carry, Pm;
    std::vector<double> leak(L + 1, 0.0);
    std::map<int, T> chain;
    if (!enrich) {
      T ch = env.right_boundary(total_charge(Fm));
      for (int bond = L - 1; bond >= root_link; --bond) {
        chain[bond] = ch;
        if (bond > root_link) ch = env.right_step(ch, fr.rf.at(bond), mpo[bond + 1]);
      }
    }
    for (int bond = L - 1; bond >= root_link; --bond) {
      if (!enrich) rch = chain[bond];
      T old = Pm ? e.contract(fr.rf.at(bond), {2}, Pm, {0}) : fr.rf.at(bond);
      T site_core = carry ? e.contract(Fm[bond + 1], {2}, carry, {0}) : Fm[bond + 1];
      SVDRes pol;
      BondFrame tsf;
      if (enrich) {
        auto both = svd2x(Fm[bond], {0, 1}, W_U | W_SVD, old, {0}, W_U | W_VD);
        tsf = frame_onto_right(both.first, site_core, old);
        pol = std::move(both.second);
      } else {
        tsf = frame_onto_right(svdx(Fm[bond], {0, 1}, W_U | W_SVD), site_core, old);
      }
      const T& lch = lstack[bond];
      const double lk = bond_action(tsf, bond, lch, rch, false);
      if (!P.fold) out.n_h2 += 1;
      leak[bond] = lk;
      Ledger bl;
      const bool quiet = indicator(alloc, lk) <= alloc.per_bond;
      T Zj;
      if (enrich && !quiet) {
        Expansion ex = dd_cbe_expand(tsf, bond, lch, rch, false, &bl, cap_at(bond));
        T lp = e.contract(ex.U_ex, {0, 1}, Fm[bond], {0, 1}, true, false);
        T Bex = e.contract(lp, {1}, site_core, {0});
        T lch1 = env.left_step(lch, ex.U_ex, mpo[bond]);
        const T& W = mpo[bond + 1];
        auto applyH = [&](const T& v) { return h1(lch1, W, rch, v); };
        auto kr = krylov_enrich(Bex, applyH, ex.V_ex, false, cap_at(bond), amp, false);
        out.n_h1 += kr.second.n_h1;
        record_krylov(bl, kr.second);
        Zj = kr.first;
      } else {
        Zj = old;
      }
      T Zn = !enrich ? old : (quiet ? polar_of(pol, false) : polar_of(svdx(Zj, {0}, W_U | W_VD), false));
      out.frames[bond] = Zn;
      out.added += dim(Zn, 0) - dim(old, 0);
      log_bond(out.ledger, bl, bond, 1, int(dim(Zn, 0)));
      if (enrich) Pm = e.contract(old, {1, 2}, Zn, {1, 2}, false, true);
      carry = e.contract(site_core, {1, 2}, Zn, {1, 2}, false, true);
      if (bond == root_link) renv = rch;
      if (enrich && bond > root_link) rch = env.right_step(rch, Zn, mpo[bond + 1]);
    }
    for (int b = root_link; b < L; ++b) out.leak.push_back(leak[b]);
    out.env = renv;
    return out;
  }

  struct Sweep {
    int64_t added = 0;
    double leak = 0;
    bool met = true, capped = false;
    Ledger ledger;
    std::vector<double> leaks_left, leaks_right;  // per bond: 1..root, root..L-1
  };

  // `halves`: false keeps the two halves serial on the step's stream even under parallel = true
  // (the outside-residual measurement, which the reference takes without `parallel`)
  Sweep frontier_sweep(KL& fr, const MPS& psi, const T& core, double nrm, bool enrich = true,
                       bool halves = true) {
    Sweep sw;
    const double nF = e.norm(core);
    if (nF <= FRONTIER_FLOOR * std::max(nrm, EPS)) return sw;
    MPS Fm = frontier_mps(psi, fr, core);
    const double amp = nF / std::max(nrm, EPS);
    FrontierHalf rl, rr;
    if (P.parallel && halves) {
      run_halves([&](Step& s) { rl = s.frontier_left(Fm, fr, amp, enrich); },
                 [&](Step& s) { rr = s.frontier_right(Fm, fr, amp, enrich); }, fork_stream());
    } else {
      rl = frontier_left(Fm, fr, amp, enrich);
      rr = frontier_right(Fm, fr, amp, enrich);
    }
    sw.leaks_left = rl.leak;
    sw.leaks_right = rr.leak;
    sw.ledger.merge(rl.ledger);
    sw.ledger.merge(rr.ledger);
    double lL = 0, lR = 0;
    for (double x : rl.leak) lL += x * x;
    for (double x : rr.leak) lR += x * x;
    sw.leak = indicator(alloc, std::sqrt(lL + lR));
    if (enrich) {
      sw.met = sw.ledger.tolerance_met;
    } else {  // a measurement meets its shares when every bond's action is within per_bond
      sw.met = true;
      for (double x : rl.leak) sw.met &= indicator(alloc, x) <= alloc.per_bond;
      for (double x : rr.leak) sw.met &= indicator(alloc, x) <= alloc.per_bond;
    }
    sw.added = rl.added + rr.added;
    if (sw.added > 0) {
      for (int b = 1; b <= root_link; ++b) fr.lf[b] = rl.frames[b];
      for (int b = root_link; b < L; ++b) fr.rf[b] = rr.frames[b];
      fr.lenv = rl.env;
      fr.renv = rr.env;
      fr.gen += 1;
    }
    sw.ledger.n_closure_sweeps = 1;
    sw.ledger.n_h1_closure = rl.n_h1 + rr.n_h1;
    sw.ledger.n_h2_leak = rl.n_h2 + rr.n_h2;
    sw.capped = sw.ledger.workcap_reached;
    return sw;
  }

  // _krylov_closure! with checks = true (krylov_closure_loop.jl:18-194; serial, include_zero =
  // false): every frontier is first measured on the incoming frames (_measure_frontiers,
  // frontier_closure.jl:289-359), which stay untouched if all close; otherwise the closure loop
  // (_closure_loop!, :370-409) sweeps degrees 1..order-1 until a pass adds nothing (converged if
  // every share is met), a capped pass misses a share, or 2 order + 2 passes; degree 0 is then
  // measured again on the final frames.
  struct ClosureOut {
    T root;
    Ledger lg;
    int64_t nroot = 0;
  };
  ClosureOut checked_closure(KL& fr, const MPS& psi, const T& root_start, double nrm) {
    ClosureOut out;
    Ledger& lg = out.lg;
    lg.order = P.order;
    T current = root_start;
    ZeroSiteH op = root_generator(fr);
    auto projected = [&](const T& root, int count) {
      std::vector<T> Fs;
      T F = root;
      for (int d = 1; d <= count; ++d) {
        out.nroot += 1;
        F = e.scale(op.apply(e, F), tau / double(d));
        Fs.push_back(F);
      }
      return Fs;
    };
    std::vector<T> cores{root_start};
    for (auto& F : projected(root_start, P.order - 1)) cores.push_back(F);
    std::vector<double> final_leak(P.order, 0.0);
    bool met = true;
    for (int d = 0; d < P.order; ++d) {
      auto sw = frontier_sweep(fr, psi, cores[d], nrm, false);
      lg.merge(sw.ledger);
      final_leak[d] = sw.leak;
      if (d >= 1) met &= sw.met;
    }
    const int gen0 = fr.gen;
    int passes = 0;
    bool converged = true;
    if (!met) {
      op = root_generator(fr);
      auto frontier = [&](int degree) { return degree == 0 ? current : projected(current, degree).back(); };
      const int maxpass = 2 * P.order + 2;
      passes = maxpass;
      converged = false;
      for (int pass = 1; pass <= maxpass; ++pass) {
        bool grew = false, allmet = true, capped = false;
        for (int degree = 1; degree < P.order; ++degree) {
          T F = frontier(degree);
          auto sw = frontier_sweep(fr, psi, F, nrm, true);
          lg.merge(sw.ledger);
          final_leak[degree] = sw.leak;
          if (sw.added > 0) {
            op = root_generator(fr);
            current = project_root(psi, fr);
          }
          grew |= sw.added > 0;
          allmet &= sw.met;
          capped |= sw.capped;
        }
        if (!grew) {
          passes = pass;
          converged = allmet;
          break;
        }
        if (capped && !allmet) {
          passes = pass;
          break;
        }
      }
      if (fr.gen != gen0) {
        auto sw = frontier_sweep(fr, psi, frontier(0), nrm, false);
        lg.merge(sw.ledger);
        final_leak[0] = sw.leak;
      }
    }
    lg.n_passes = passes;
    lg.leak = final_leak;
    double defect = 0.0;
    for (int d = 0; d < P.order; ++d) defect += final_leak[d] / (d + 1);
    lg.defect = defect;
    lg.n_root_frontier = out.nroot;
    if (!converged) lg.unmet_(U_CLOSURE);
    out.root = current;
    return out;
  }

  // ── root exponential (krylov.jl, root_methods.jl) ──
  struct Eig {
    std::vector<double> vals;
    RMat vecs;
  };
  static double shift(const std::vector<cd>& vals, cd t) {
    if (vals.empty()) return 0.0;
    int top = 0;
    double best = -std::numeric_limits<double>::infinity();
    for (size_t i = 0; i < vals.size(); ++i) {
      const double ex = (t * vals[i]).real();
      if (ex > best) {
        best = ex;
        top = int(i);
      }
    }
    return best > EXPV_SHIFT_TRIGGER ? vals[top].real() : 0.0;
  }
  static std::pair<std::vector<cd>, cd> coeffs_from_eigen(const Eig& eg, cd t) {
    std::vector<cd> cv(eg.vals.begin(), eg.vals.end());
    const double sigma = shift(cv, t);
    const int n = int(eg.vals.size());
    std::vector<cd> w(n);
    for (int j = 0; j < n; ++j) w[j] = std::exp(t * (cd(eg.vals[j]) - sigma)) * eg.vecs(0, j);
    std::vector<cd> c(n, 0.0);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) c[i] += eg.vecs(i, j) * w[j];
    return {c, t * sigma};
  }
  static Eig tridiag_eigen(const std::vector<double>& a, const std::vector<double>& b) {
    require_finite_tridiag(a.data(), a.size(), b.data(), b.size());
    Eig eg;
    smallla::eigh_tridiag(a, std::vector<double>(b.begin(), b.begin() + std::max<ptrdiff_t>(ptrdiff_t(a.size()) - 1, 0)),
                          eg.vals, eg.vecs);
    return eg;
  }
  static double tail(const std::vector<cd>& c, double betak) { return c.empty() ? 0.0 : betak * std::abs(c.back()); }
  template <class F>
  static double tail_sup(F evalcoeff, cd step, double betak, double above = std::numeric_limits<double>::infinity()) {
    double t = tail(evalcoeff(step).first, betak);
    if (step.real() != 0) return t;
    for (int node = 1; node < TAIL_NODES; ++node) {
      if (t >= above) return t;
      t = std::max(t, tail(evalcoeff(step * (double(node) / TAIL_NODES)).first, betak));
    }
    return t;
  }
  template <class F>
  static cd pick_tau(F evalcoeff, cd tau_rem, double betak, double conv_tol) {
    auto accepted = [&](cd trial) {
      const double tl = tail_sup(evalcoeff, trial, betak,
                                 conv_tol > 0 ? conv_tol : std::numeric_limits<double>::infinity());
      return std::isfinite(tl) && (conv_tol <= 0 || tl <= conv_tol);
    };
    if (accepted(tau_rem)) return tau_rem;
    double lo = 0.0, hi = 1.0;
    for (int i = 0; i < 40; ++i) {
      const double mid = 0.5 * (lo + hi);
      if (accepted(mid * tau_rem)) lo = mid;
      else hi = mid;
    }
    return std::max(lo, 1e-6) * tau_rem;
  }
  T combine(const std::vector<cd>& coeff, const std::vector<T>& basis, double beta0) {
    std::vector<std::pair<cd, T>> terms;
    for (size_t c = 0; c < coeff.size(); ++c) terms.push_back({coeff[c] * beta0, basis[c]});
    return e.lin(terms);
  }
  T apply_scale(const T& cur, cd logscale) {
    const cd sc = std::exp(logscale);
    if (!(std::isfinite(std::abs(sc)) && sc != cd(0))) return cur;
    const double n = e.norm(cur);
    if (std::isfinite(n) && n > 0 && std::abs(sc) * n > EXPV_MAX_NORM) return cur;
    if (sc == cd(1)) return cur;
    return e.scale(cur, sc);
  }

  struct ExpvRep {
    int64_t iters = 0, nsub = 0, wasted = 0;  // wasted: applications past a deferred chain's cut
    double err = 0;
  };

  // A linear combination whose coefficients may be device-resident dot products (bugk::LinSrc):
  // mode 0 uses `coef`; 1, 2, 3 give -x, 1/sqrt(max(x, 0)), -sqrt(max(x, 0)) of the real part x
  // at `ref`; 4 gives -(x + iy) of the complex value (x, y) at `ref`.
  struct DevTerm {
    cd coef;
    int mode;
    const double* ref;
    T t;
  };
  T lin_dev(const std::vector<DevTerm>& terms) {
    std::vector<double> coef;
    std::vector<const bug_tensor*> ts;
    std::vector<const double*> refs;
    std::vector<int> modes;
    for (auto& x : terms) {
      coef.push_back(x.coef.real());
      coef.push_back(x.coef.imag());
      ts.push_back(x.t.get());
      refs.push_back(x.ref);
      modes.push_back(x.mode);
    }
    return Eng::sh(lincomb_impl(e.c, int(ts.size()), coef.data(), ts.data(), refs.data(), modes.data()));
  }

  // The Lanczos chain (no reorthogonalisation, no convergence test) with its coefficients left on
  // the device: alpha_k and |r_k|^2 are written by the dot launches into device memory, and the
  // combinations that need them compute -alpha, 1/|r| and -|r| in the kernel. The host reads the
  // coefficients back once per chunk of iterations and replays the host-driven chain's stop (the
  // first |r| below `tol`) on them: the arithmetic is the host-driven chain's, launch for launch,
  // with one read-back per chunk instead of two per iteration. The first chunk is at most the
  // vector's dimension long (a Krylov chain breaks down by then), later chunks kDeferredChunk; the
  // iterations of the last chunk past the stop are discarded. Returns their applications.
  static constexpr int kDeferredChunk = 8;
  int64_t deferred_chain(const std::function<T(const T&)>& apply, const T& v0, int maxiter,
                         double tol, std::vector<T>& basis, std::vector<double>& alpha,
                         std::vector<double>& betas, double& betak) {
    double2* A = static_cast<double2*>(e.c->scratch(size_t(2 * maxiter) * sizeof(double2)));
    double2* N = A + maxiter;  // N[k] = |r|^2 after iteration k + 1
    auto re = [](const double2* q) { return reinterpret_cast<const double*>(q); };
    basis.assign(1, v0);
    T residual = apply(v0);
    dots_device(e.c, {{v0.get(), residual.get()}}, A);
    residual = lin_dev({{1.0, 0, nullptr, residual}, {0.0, 1, re(A), v0}});
    dots_device(e.c, {{residual.get(), residual.get()}}, N);
    int ran = 1;  // iterations run on the device
    int chunk = int(std::max<int64_t>(1, std::min<int64_t>(kDeferredChunk, v0->nelem)));
    alpha.clear();
    betas.clear();
    betak = -1.0;
    int used = -1;
    int tested = 1;  // iterations whose continuation has been replayed on the host
    while (true) {
      const int target = std::min(maxiter, ran + chunk - (ran == 1 ? 1 : 0));
      for (int it = ran + 1; it <= target; ++it) {
        T v = lin_dev({{0.0, 2, re(N + (it - 2)), residual}});
        basis.push_back(v);
        residual = apply(v);
        dots_device(e.c, {{v.get(), residual.get()}}, A + (it - 1));
        residual = lin_dev({{1.0, 0, nullptr, residual},
                            {0.0, 1, re(A + (it - 1)), v},
                            {0.0, 3, re(N + (it - 2)), basis[basis.size() - 2]}});
        dots_device(e.c, {{residual.get(), residual.get()}}, N + (it - 1));
      }
      ran = target;
      double* host = e.c->readback(size_t(4 * maxiter));
      e.c->drain();  // the queued recurrence writes A and N: it runs before the copies
      BUG_CUDA(cudaMemcpyAsync(host, A, size_t(maxiter) * sizeof(double2), cudaMemcpyDeviceToHost,
                               e.c->stream));
      BUG_CUDA(cudaMemcpyAsync(host + 2 * maxiter, N, size_t(maxiter) * sizeof(double2),
                               cudaMemcpyDeviceToHost, e.c->stream));
      e.c->wait();
      auto nrm = [&](int k) { return std::sqrt(std::max(host[2 * (maxiter + k)], 0.0)); };
      if (alpha.empty()) alpha.push_back(host[0]);
      // replay the stop test of iterations tested+1 .. ran+1 (the test of `it` reads N[it-2])
      for (int it = tested + 1; it <= std::min(maxiter, ran + 1); ++it) {
        const double off = nrm(it - 2);
        if (off < tol) {
          used = it - 1;
          betak = off;
          break;
        }
        if (it > ran) break;  // continues: the next chunk runs it
        betas.push_back(off);
        alpha.push_back(host[2 * (it - 1)]);
        tested = it;
      }
      if (used > 0) break;
      if (ran == maxiter) {
        used = maxiter;
        betak = nrm(maxiter - 1);
        break;
      }
      tested = ran;
      chunk = kDeferredChunk;
    }
    basis.resize(size_t(used));
    alpha.resize(size_t(used));
    betas.resize(size_t(used - 1));
    return int64_t(ran - used);
  }

  // substeps: 1 one step of the whole tau, > 1 that many equal substeps, 0 the adaptive substep
  // search (pick_tau)
  T lanczos_expv(const std::function<T(const T&)>& apply, const T& vec, int maxiter, double tol,
                 bool reorth, double conv_tol, ExpvRep& rep, int substeps = 0, bool deferred = false,
                 int rmethod = 0, bool rshift = true) {
    if (rmethod) substeps = 1;  // an implicit root takes the whole step in one stage
    const double beta0 = e.norm(vec);
    if (beta0 == 0) return vec;
    T cur = vec;
    cd tau_rem = tau, logscale = 0.0;
    int nsub = 0;
    while (true) {
      rep.nsub += 1;
      nsub += 1;
      const double cur_norm = e.norm(cur);
      if (cur_norm == 0) break;
      T v = e.scale(cur, 1.0 / cur_norm);
      std::vector<T> basis;
      std::vector<double> alpha, betas;
      double betak = 0.0;
      if (deferred && !reorth && conv_tol <= 0) {
        rep.wasted += deferred_chain(apply, v, maxiter, tol, basis, alpha, betas, betak);
        rep.iters += int64_t(basis.size());
      } else {
        basis.push_back(v);
        T residual = apply(v);
        rep.iters += 1;
        double a = e.inner(v, residual).real();
        alpha.push_back(a);
        residual = e.lin({{1.0, residual}, {-a, v}});
        for (int it = 2; it <= maxiter; ++it) {
          const double off = e.norm(residual);
          if (off < tol) break;
          if (conv_tol > 0) {
            Eig eg = tridiag_eigen(alpha, betas);
            auto ev = [&](cd s) { return rmethod ? rational_coeffs(eg, s, rmethod, rshift) : coeffs_from_eigen(eg, s); };
            if (tail_sup(ev, tau_rem, off, conv_tol) < conv_tol) break;
          }
          betas.push_back(off);
          v = e.scale(residual, 1.0 / off);
          basis.push_back(v);
          residual = apply(v);
          rep.iters += 1;
          a = e.inner(v, residual).real();
          alpha.push_back(a);
          residual = e.lin({{1.0, residual}, {-a, v}, {-off, basis[basis.size() - 2]}});
          if (reorth) {
            for (int pass = 0; pass < 2; ++pass) {
              auto cs = e.inner_many(basis, residual);
              std::vector<std::pair<cd, T>> terms{{1.0, residual}};
              for (size_t i = 0; i < basis.size(); ++i) terms.push_back({-cs[i], basis[i]});
              residual = e.lin(terms);
            }
          }
        }
        betak = e.norm(residual);
      }
      Eig eg = tridiag_eigen(alpha, betas);
      auto ev = [&](cd s) { return rmethod ? rational_coeffs(eg, s, rmethod, rshift) : coeffs_from_eigen(eg, s); };
      const cd tau_s = substeps == 1 ? tau_rem
                       : substeps > 1 ? tau_rem / double(substeps - nsub + 1)
                                      : pick_tau(ev, tau_rem, betak, conv_tol);
      auto cl = ev(tau_s);
      rep.err += tail_sup(ev, tau_s, betak) * cur_norm / beta0;
      cur = combine(cl.first, basis, cur_norm);
      logscale += cl.second;
      tau_rem -= tau_s;
      if (substeps == 1 || std::abs(tau_rem) <= 1e-14 * std::max(std::abs(tau), 1.0)) break;
      require(rep.nsub < 10000, "expv: substep search failed to advance");
    }
    return apply_scale(cur, logscale);
  }


  // ── implicit roots (root_methods.jl:12-75, 143-168): R(z) = N(z) / D(z) of one implicit RK
  // step, the (k, k+1) Pade approximants of exp (coefficients constant term first): 1 trapezoid,
  // 2 Radau IIA with two stages, 3 with three. The spectrum is shifted to the Ritz value that
  // maximises Re(tau lambda) (none in real time or without `shift`); no scale is carried.
  static cd root_stability(int m, cd z) {
    static const std::vector<double> num[4] = {{}, {1.0, 0.5}, {1.0, 1.0 / 3.0}, {1.0, 0.4, 0.05}};
    static const std::vector<double> den[4] = {
        {}, {1.0, -0.5}, {1.0, -2.0 / 3.0, 1.0 / 6.0}, {1.0, -0.6, 0.15, -1.0 / 60.0}};
    auto horner = [&](const std::vector<double>& c) {
      cd r = c.back();
      for (int k = int(c.size()) - 2; k >= 0; --k) r = r * z + c[k];
      return r;
    };
    return horner(num[m]) / horner(den[m]);
  }
  static cd rational_shift(const std::vector<cd>& vals, cd t, bool shift) {
    if (!shift || vals.empty() || t.real() == 0) return 0.0;
    size_t top = 0;
    for (size_t i = 1; i < vals.size(); ++i)
      if ((t * vals[i]).real() > (t * vals[top]).real()) top = i;
    return vals[top];
  }
  static std::pair<std::vector<cd>, cd> rational_coeffs(const Eig& eg, cd t, int m, bool shift) {
    std::vector<cd> cv(eg.vals.begin(), eg.vals.end());
    const cd sigma = rational_shift(cv, t, shift);
    const int n = int(eg.vals.size());
    std::vector<cd> w(n), c(n, 0.0);
    for (int j = 0; j < n; ++j) w[j] = root_stability(m, t * (cd(eg.vals[j]) - sigma)) * eg.vecs(0, j);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) c[i] += eg.vecs(i, j) * w[j];
    return {c, 0.0};
  }
  std::pair<std::vector<cd>, cd> hess_rational(const CMat& Hm, cd t, int m, bool shift) {
    const int n = Hm.n;
    if (n == 0) return {{}, 0.0};
    const cd sigma = rational_shift(smallla::eigvals_hess(Hm), t, shift);
    CMat M(n, n);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) M(i, j) = t * (Hm(i, j) - (i == j ? sigma : cd(0)));
    static const std::vector<double> num[4] = {{}, {1.0, 0.5}, {1.0, 1.0 / 3.0}, {1.0, 0.4, 0.05}};
    static const std::vector<double> den[4] = {
        {}, {1.0, -0.5}, {1.0, -2.0 / 3.0, 1.0 / 6.0}, {1.0, -0.6, 0.15, -1.0 / 60.0}};
    auto poly = [&](const std::vector<double>& c) {
      CMat r(n, n);
      for (int i = 0; i < n; ++i) r(i, i) = c.back();
      for (int k = int(c.size()) - 2; k >= 0; --k) {
        r = smallla::matmul(r, M);
        for (int i = 0; i < n; ++i) r(i, i) += c[k];
      }
      return r;
    };
    CMat N = poly(num[m]), e1(n, 1);
    for (int i = 0; i < n; ++i) e1(i, 0) = N(i, 0);
    CMat x = smallla::solve(poly(den[m]), e1);
    std::vector<cd> c(n);
    for (int i = 0; i < n; ++i) c[i] = x(i, 0);
    return {c, 0.0};
  }

  // ── radau2_gmres (root_methods.jl:170-345): one Radau IIA(2) step, the coupled stages
  // (I - tau A (x) B) Y = 1 (x) x decoupled by A = P Lambda P^-1 into (I - tau lambda_k (B - sigma))
  // Z_k = d_k x, d = P^-1 1, solved on ONE Arnoldi basis of B (a Krylov space is shift
  // invariant), then Y = (P (x) I) Z; restarted on the true stage residual at most 4 times. The
  // method is stiffly accurate: the result is Y_2.
  struct Gmres {
    std::vector<T> Z;
    double res = 0.0;
    int64_t nmv = 0;
    cd sigma = 0.0;
  };
  // _shifted_gmres: the systems (I - z_k (B - sigma)) Z_k = d_k rhs on one basis; Wt[s][k] the
  // entry of P the solution of system k enters stage s with
  Gmres shifted_gmres(const std::function<T(const T&)>& apply, const T& rhs, const std::vector<cd>& zs,
                      const std::vector<cd>& ds, const std::vector<std::vector<cd>>& Wt,
                      bool have_sigma, cd sigma_in, double target, int maxiter, double tol) {
    Gmres g;
    const double beta = e.norm(rhs);
    std::vector<T> basis{e.scale(rhs, 1.0 / beta)};
    CMat H(maxiter + 1, maxiter);
    std::vector<std::vector<cd>> ys;
    for (int k = 1; k <= maxiter; ++k) {
      T nv = apply(basis[size_t(k - 1)]);
      for (int pass = 0; pass < 2; ++pass) {  // CGS2 (krylov.jl:321-332)
        auto cs = e.inner_many(basis, nv);
        std::vector<std::pair<cd, T>> terms{{1.0, nv}};
        for (size_t i = 0; i < basis.size(); ++i) {
          H(int(i), k - 1) += cs[i];
          terms.push_back({-cs[i], basis[i]});
        }
        nv = e.lin(terms);
      }
      g.nmv += 1;
      const double nn = e.norm(nv);
      H(k, k - 1) = nn;
      CMat lead(k, k);
      for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) lead(i, j) = H(i, j);
      g.sigma = have_sigma ? sigma_in : rational_shift(smallla::eigvals_hess(lead), tau, true);
      ys.assign(zs.size(), {});
      std::vector<std::vector<cd>> sres(zs.size());
      for (size_t sidx = 0; sidx < zs.size(); ++sidx) {
        CMat M(k + 1, k);
        for (int i = 0; i <= k; ++i)
          for (int j = 0; j < k; ++j)
            M(i, j) = (i == j ? cd(1.0) : cd(0.0)) - zs[sidx] * (H(i, j) - (i == j ? g.sigma : cd(0.0)));
        std::vector<cd> rhs_k(size_t(k + 1), 0.0);
        rhs_k[0] = ds[sidx] * beta;
        ys[sidx] = smallla::lstsq(M, rhs_k);
        sres[sidx] = rhs_k;
        for (int i = 0; i <= k; ++i)
          for (int j = 0; j < k; ++j) sres[sidx][size_t(i)] -= M(i, j) * ys[sidx][size_t(j)];
      }
      double r2 = 0.0;  // |SR Wt^T|_F
      for (size_t st = 0; st < Wt.size(); ++st)
        for (int i = 0; i <= k; ++i) {
          cd acc = 0.0;
          for (size_t sidx = 0; sidx < zs.size(); ++sidx) acc += sres[sidx][size_t(i)] * Wt[st][sidx];
          r2 += std::norm(acc);
        }
      g.res = std::sqrt(r2);
      if (nn < tol || g.res <= target || k == maxiter) break;
      basis.push_back(e.scale(nv, 1.0 / nn));
    }
    for (auto& c : ys) {
      std::vector<T> b(basis.begin(), basis.begin() + long(c.size()));
      g.Z.push_back(combine(c, b, 1.0));
    }
    return g;
  }

  T radau2_gmres_expv(const std::function<T(const T&)>& apply, const T& vec, int maxiter, double tol,
                      double conv_tol, bool rshift, ExpvRep& rep) {
    const double beta0 = e.norm(vec);
    if (beta0 == 0) return vec;
    const double A[2][2] = {{5.0 / 12.0, -1.0 / 12.0}, {0.75, 0.25}};
    const cd half_tr = 0.5 * (A[0][0] + A[1][1]);
    const cd disc = std::sqrt(half_tr * half_tr - cd(A[0][0] * A[1][1] - A[0][1] * A[1][0]));
    const cd lam[2] = {half_tr + disc, half_tr - disc};
    cd Pm[2][2];
    for (int k = 0; k < 2; ++k) {  // eigenvector (A12, lambda - A11), unit norm
      const cd v0 = A[0][1], v1 = lam[k] - A[0][0];
      const double nv = std::sqrt(std::norm(v0) + std::norm(v1));
      Pm[0][k] = v0 / nv;
      Pm[1][k] = v1 / nv;
    }
    const cd det = Pm[0][0] * Pm[1][1] - Pm[0][1] * Pm[1][0];
    const cd Pi[2][2] = {{Pm[1][1] / det, -Pm[0][1] / det}, {-Pm[1][0] / det, Pm[0][0] / det}};
    const std::vector<cd> zs{tau * lam[0], tau * lam[1]};
    const double target = conv_tol > 0 ? conv_tol * beta0 : 0.0;
    const std::vector<cd> ds{Pi[0][0] + Pi[0][1], Pi[1][0] + Pi[1][1]};
    const std::vector<std::vector<cd>> W2{{Pm[0][0], Pm[0][1]}, {Pm[1][0], Pm[1][1]}};
    Gmres g = shifted_gmres(apply, vec, zs, ds, W2, !rshift, 0.0, target, maxiter, tol);
    int64_t nmv = g.nmv;
    const cd sigma = g.sigma;
    auto stage = [&](const std::vector<T>& Z, int i) { return e.lin({{Pm[i][0], Z[0]}, {Pm[i][1], Z[1]}}); };
    std::vector<T> Y{stage(g.Z, 0), stage(g.Z, 1)};
    std::vector<T> R(2);
    auto residual = [&]() {
      std::vector<T> BY;
      for (auto& y : Y) {
        T img = apply(y);
        BY.push_back(sigma == cd(0.0) ? img : e.lin({{1.0, img}, {-sigma, y}}));
      }
      nmv += 2;
      for (int i = 0; i < 2; ++i)
        R[i] = e.lin({{1.0, vec}, {-1.0, Y[i]}, {tau * A[i][0], BY[0]}, {tau * A[i][1], BY[1]}});
      const auto nR = e.norms(R[0], R[1]);
      return std::sqrt(std::pow(nR.first, 2) + std::pow(nR.second, 2));
    };
    double res = residual();
    int cycles = 1;
    while (target > 0 && res > target && cycles < 4) {
      cycles += 1;
      std::vector<T> dZ;
      for (int i = 0; i < 2; ++i) {
        T rho = e.lin({{Pi[i][0], R[0]}, {Pi[i][1], R[1]}});
        if (e.norm(rho) == 0) {
          dZ.push_back(rho);
          continue;
        }
        Gmres gk = shifted_gmres(apply, rho, {zs[size_t(i)]}, {1.0}, {{Pm[0][i]}, {Pm[1][i]}}, true,
                                 sigma, target / std::sqrt(2.0), maxiter, tol);
        nmv += gk.nmv;
        dZ.push_back(gk.Z[0]);
      }
      for (int i = 0; i < 2; ++i) Y[i] = e.lin({{1.0, Y[i]}, {1.0, stage(dZ, i)}});
      res = residual();
    }
    rep.iters += nmv;
    rep.nsub += 1;
    rep.err += res / beta0;
    return Y[1];
  }

  std::pair<std::vector<cd>, cd> hess_coeffs(const CMat& Hm, cd t) {
    const int n = Hm.n;
    if (n == 0) return {{}, 0.0};
    const double sigma = shift(smallla::eigvals_hess(Hm), t);
    CMat M(n, n);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) M(i, j) = t * (Hm(i, j) - (i == j ? cd(sigma) : cd(0)));
    CMat Pm = smallla::expm(M);
    std::vector<cd> c(n);
    for (int i = 0; i < n; ++i) c[i] = Pm(i, 0);
    return {c, t * sigma};
  }

  T arnoldi_expv(const std::function<T(const T&)>& apply, const T& vec, int maxiter, double tol,
                 double conv_tol, ExpvRep& rep, int substeps = 0, int rmethod = 0, bool rshift = true) {
    if (rmethod) substeps = 1;
    const double beta0 = e.norm(vec);
    if (beta0 == 0) return vec;
    T cur = vec;
    cd tau_rem = tau, logscale = 0.0;
    int nsub = 0;
    while (true) {
      rep.nsub += 1;
      nsub += 1;
      const double cur_norm = e.norm(cur);
      if (cur_norm == 0) break;
      std::vector<T> basis{e.scale(cur, 1.0 / cur_norm)};
      CMat H(maxiter + 1, maxiter);
      int dimk = 0;
      double betak = 0.0;
      for (int k = 0; k < maxiter; ++k) {
        T residual = apply(basis[k]);
        for (int pass = 0; pass < 2; ++pass) {
          auto cs = e.inner_many(basis, residual);
          std::vector<std::pair<cd, T>> terms{{1.0, residual}};
          for (size_t i = 0; i < basis.size(); ++i) {
            H(int(i), k) += cs[i];
            terms.push_back({-cs[i], basis[i]});
          }
          residual = e.lin(terms);
        }
        rep.iters += 1;
        dimk = k + 1;
        const double rn = e.norm(residual);
        betak = rn;
        if (rn < tol) break;
        if (conv_tol > 0) {
          CMat lead(dimk, dimk);
          for (int i = 0; i < dimk; ++i)
            for (int j = 0; j < dimk; ++j) lead(i, j) = H(i, j);
          auto ev = [&](cd s) { return rmethod ? hess_rational(lead, s, rmethod, rshift) : hess_coeffs(lead, s); };
          if (tail_sup(ev, tau_rem, rn, conv_tol) < conv_tol) break;
        }
        H(k + 1, k) = rn;
        if (k + 1 == maxiter) break;
        basis.push_back(e.scale(residual, 1.0 / rn));
      }
      CMat Hm(dimk, dimk);
      for (int i = 0; i < dimk; ++i)
        for (int j = 0; j < dimk; ++j) Hm(i, j) = H(i, j);
      auto ev = [&](cd s) { return rmethod ? hess_rational(Hm, s, rmethod, rshift) : hess_coeffs(Hm, s); };
      const cd tau_s = substeps == 1 ? tau_rem
                       : substeps > 1 ? tau_rem / double(substeps - nsub + 1)
                                      : pick_tau(ev, tau_rem, betak, conv_tol);
      auto cl = ev(tau_s);
      rep.err += tail_sup(ev, tau_s, betak) * cur_norm / beta0;
      basis.resize(dimk);
      cur = combine(cl.first, basis, cur_norm);
      logscale += cl.second;
      tau_rem -= tau_s;
      if (substeps == 1 || std::abs(tau_rem) <= 1e-14 * std::max(std::abs(tau), 1.0)) break;
      require(rep.nsub < 10000, "expv: substep search failed to advance");
    }
    return apply_scale(cur, logscale);
  }

  // ── compression (truncation.jl) ──
  std::pair<SVDRes, bool> budget_svd(const T& t, std::vector<int> split, int maxdim,
                                     const std::function<double(double)>& share_of) {
    const int want = split.size() == 1 ? (W_VD | W_US) : (W_U | W_SVD);
    SVDRes res = svd(e, t, split, 0.0, maxdim, want);
    const double share = share_of(sq_weight(res.kept) + sq_weight(res.trunc));
    const int nk = int(res.kept.size());
    auto tr = tail_rank(res.kept, 1.0, share, nk, sq_weight(res.trunc));
    const bool capped = tr.second > share && !res.trunc.empty();
    const int keep = std::max(tr.first, 1);
    if (keep < nk) res = svd(e, t, split, 0.0, keep, want);
    return {res, capped};
  }

  std::tuple<double, double, bool> truncate_recursive(MPS& psi, int root, int maxdim, double wtol,
                                                      std::vector<double>& bw) {
    double worst = 0.0, nrm2 = -1.0;
    bool capped = false;
    double cum[2] = {0.0, 0.0};
    const double sdiv = std::sqrt(double(root - 1)) + std::sqrt(double(L - root));
    auto share_of = [&](double total) {
      if (nrm2 < 0) nrm2 = total;
      return sdiv > 0 ? wtol * std::sqrt(std::max(nrm2, 0.0)) / sdiv : 0.0;
    };
    auto account = [&](const SVDRes& r, int side, int bond) {
      worst = std::max(worst, trunc_weight(r));
      cum[side] += sq_weight(r.trunc);
      bw[bond - 1] = sq_weight(r.trunc);
      if (nrm2 < 0) nrm2 = sq_weight(r.kept) + sq_weight(r.trunc);
    };
    for (int site = root; site >= 2; --site) {
      auto rc = budget_svd(psi[site], {0}, maxdim, share_of);
      capped |= rc.second;
      account(rc.first, 0, site - 1);
      psi[site] = rc.first.Vd;
      psi[site - 1] = e.contract(psi[site - 1], {2}, US(e, rc.first), {0});
      psi.center = site - 1;
    }
    canonical(psi, root);
    for (int site = root; site < L; ++site) {
      auto rc = budget_svd(psi[site], {0, 1}, maxdim, share_of);
      capped |= rc.second;
      account(rc.first, 1, site);
      psi[site] = rc.first.U;
      psi[site + 1] = e.contract(SVd(e, rc.first), {1}, psi[site + 1], {0});
      psi.center = site + 1;
    }
    const double cumulative = nrm2 > 0 ? (std::sqrt(cum[0]) + std::sqrt(cum[1])) / std::sqrt(nrm2) : 0.0;
    for (auto& x : bw) x = nrm2 > 0 ? std::sqrt(x / nrm2) : 0.0;
    return {worst, cumulative, capped};
  }
};

}  // namespace bugs

using namespace bugs;

// ── C-ABI ────────────────────────────────────────────────────────────────────────────────────

extern "C" int bug_mps_step(bug_ctx* c, int L, bug_tensor** psi_io, int* center_io,
                            const bug_tensor* const* mpo_in, double tau_re, double tau_im,
                            const bug_step_params* prm, bug_normal_fn draw, void* user,
                            bug_step_info* info, bug_bond_log* bond_log, int bond_log_cap,
                            int* n_bond_log) {
  return guard([&] {
    require(c && psi_io && center_io && mpo_in && prm && draw && info, "null argument");
    require(L >= 2, "cbe_bug_step needs at least two sites");
    Params P{};
    P.tol_basis = prm->tol_basis > 0 ? prm->tol_basis : 1e-5;
    P.tol_trunc = prm->tol_trunc >= 0 ? prm->tol_trunc : 1e-7;
    P.tol_expv = prm->tol_expv > 0 ? prm->tol_expv : 1e-10;
    P.tol_krylov = prm->tol_krylov;
    P.order = prm->order;
    require(P.order >= 1, "order must be >= 1");
    P.maxdim = prm->maxdim > 0 ? prm->maxdim : 128;
    P.hermitian = prm->hermitian;
    P.root = prm->root;
    P.reorth = prm->reorth;
    P.truncate = prm->truncate;
    P.root_maxiter = prm->root_maxiter > 0 ? prm->root_maxiter : 30;
    P.fixed_width = prm->fixed_width > 0 ? prm->fixed_width : 8;
    P.tail_factor = prm->tail_factor > 0 ? prm->tail_factor : 0.10;
    P.bond_ceiling_factor = prm->bond_ceiling_factor;
    P.lanczos = prm->krylov_mode == 0 ? (P.hermitian ? 1 : 0) : (prm->krylov_mode == 1 ? 1 : 0);
    P.fixed_depth = prm->krylov_fixed_depth;
    require(prm->dd_mode == 0 || prm->dd_mode == 1, "dd_mode must be 0 (:rank_tail) or 1 (:adaptive)");
    P.dd_mode = prm->dd_mode;
    P.closure_checks = prm->closure_checks != 0;
    require(prm->root_method >= 0 && prm->root_method <= 4,
            "root_method must be 0 (exp), 1 (trapezoid), 2 (radau2), 3 (radau3) or 4 (radau2_gmres)");
    P.root_method = prm->root_method;
    P.root_shift = prm->root_noshift == 0;
    P.parallel = prm->parallel != 0;
    P.rng_fork = prm->rng_fork;
    P.rng_fork_user = prm->rng_fork_user;
    require(!P.parallel || (P.rng_fork && draw), "parallel needs rng_fork and a draw stream");
    P.exact = prm->exact != 0;
    require(prm->fold_omega >= 0 && prm->fold_omega <= 2, "fold_omega must be 0 (default), 1 or 2");
    // bug_step_stages.jl:67: the folded closures are the default above order 1 unless exact
    P.fold = prm->fold_omega == 0 ? (P.order > 1 && !P.exact) : prm->fold_omega == 1;
    require(prm->n_keep >= 0 && (prm->n_keep == 0 || prm->keep_sites), "keep_states: no site handles");
    for (int k = 0; k < prm->n_keep; ++k) {
      std::vector<T> sites;
      for (int i = 0; i < L; ++i) {
        const bug_tensor* t = prm->keep_sites[size_t(k) * size_t(L) + size_t(i)];
        require(t != nullptr && t->rank == 3, "keep_states: a site is not a rank-3 tensor");
        sites.push_back(T(const_cast<bug_tensor*>(t), [](bug_tensor*) {}));
      }
      P.keep.push_back(std::move(sites));
      const double tol = prm->keep_tols ? prm->keep_tols[k] : 0.0;
      require(tol >= 0, "keep_tols must be >= 0");
      P.keep_tols.push_back(tol);
    }
    P.cap_keep = prm->work_ceiling_rule != 1;  // :bond, :bond_strict and :frame_root
    require(!prm->frames_only || (!prm->root_report && !prm->truncate),
            "frames_only needs root_report = nothing, kls = nothing and truncate = false");
    P.holdout_width = prm->holdout_width > 0 ? prm->holdout_width : DD_HOLDOUT;
    P.batch_blocks = prm->batch_blocks > 0 ? prm->batch_blocks : 1;
    require(P.batch_blocks <= 8, "batch_blocks must lie in 1:8");
    require(prm->cap_selection == 0 || prm->cap_selection == 1, "cap_selection must be 0 (:storage) or 1 (:svd)");
    P.cap_selection_svd = prm->cap_selection;
    P.acceptance_factor = prm->acceptance_factor > 0 ? prm->acceptance_factor : 1.0;
    require(P.acceptance_factor <= 1.0, "acceptance_factor must lie in (0,1]");
    require(P.tail_factor > 0 && P.tail_factor <= 1, "tail_factor must lie in (0,1]");

    DrawBuf dbuf;
    Eng e{c, draw, user};
    if (prm->rng_ctl && draw) {
      dbuf.draw = draw;
      dbuf.user = user;
      dbuf.ctl = prm->rng_ctl;
      dbuf.ctl_user = prm->rng_ctl_user;
      dbuf.begin();
      e.buf = &dbuf;
    }
    MPOv mpo;
    for (int i = 0; i < L; ++i) {
      // the MPO handles stay owned by the caller: alias them without taking ownership
      mpo.W.push_back(T(const_cast<bug_tensor*>(mpo_in[i]), [](bug_tensor*) {}));
    }
    MPS psi;
    for (int i = 0; i < L; ++i) psi.s.push_back(T(psi_io[i], [](bug_tensor*) {}));
    psi.center = *center_io;
    const cd tau(tau_re, tau_im);
    Step S(e, mpo, P, tau, L);
    S.eshift = prm->eshift;
    require(!prm->outside_residual || prm->root_report, "outside_residual needs root_report");
    require(!prm->outside_residual || prm->rng_ctl, "outside_residual needs rng_ctl (a copy of the draw stream)");
    require(!prm->outside_residual || P.fold, "the outside residual with the exact (unfolded) leak is not built");
    S.root_link = P.root > 0 ? P.root : std::max(1, std::min(L - 1, L / 2));
    require(S.root_link >= 1 && S.root_link <= L - 1, "root must be a bond in 1:L-1");

    // options (bug_step_stages.jl:15-142)
    std::vector<int64_t> bd0 = psi.bond_dims();
    int64_t dloc = 1;
    for (int s = 1; s <= L; ++s) dloc = std::max<int64_t>(dloc, dim(psi[s], 1));
    S.wcap = work_ceilings(prm->work_ceiling_rule, bd0, dloc, P.maxdim, P.bond_ceiling_factor,
                           S.root_link, prm->root_ceiling_factor);
    const double nrm = (psi.center >= 1 && psi.center <= L) ? e.norm(psi[psi.center]) : 1.0;
    S.alloc = basis_allocation(P.tol_basis, L - 1, tau, nrm, P.order, P.tol_krylov, 0.0);
    Ledger ledger;
    ledger.order = P.order;
    ledger.r_old = bd0.empty() ? 0 : *std::max_element(bd0.begin(), bd0.end());
    std::vector<double> bwts(L - 1, 0.0);
    std::vector<int64_t> expanded(L - 1, 0), nL(L - 1, 0), nR(L - 1, 0);
    Ledger ledgerL, ledgerR;
    std::map<int, T> lf, rf;
    MPS psiL = psi;
    T lenv_root;
    std::pair<T, T> rr;
    if (P.parallel) {
      S.run_halves([&](Step& s) { lenv_root = s.half_left(psiL, lf, expanded, nL, ledgerL); },
                   [&](Step& s) { rr = s.half_right(psi, rf, expanded, nR, ledgerR); },
                   S.fork_stream());
    } else {
      lenv_root = S.half_left(psiL, lf, expanded, nL, ledgerL);
      rr = S.half_right(psi, rf, expanded, nR, ledgerR);
    }
    T renv_root = rr.first, AR = rr.second;
    ledger.merge(ledgerL);
    ledger.merge(ledgerR);
    std::vector<int64_t> n_new(L - 1);
    for (int b = 1; b <= L - 1; ++b) n_new[b - 1] = b < S.root_link ? nL[b - 1] : nR[b - 1];
    T AL = S.overlap_left(psi, lf);
    T root_start = e.contract(AL, {1}, AR, {0});
    int64_t nclose = 0;
    Step::KL fr{lf, rf, lenv_root, renv_root, 0};
    if (P.order > 1 && P.closure_checks) {
      auto cl = S.checked_closure(fr, psi, root_start, nrm);
      ledger.merge(cl.lg);
      lf = fr.lf;
      rf = fr.rf;
      for (int b = 1; b < S.root_link; ++b) expanded[b - 1] = dim(lf[b], 2);
      for (int b = S.root_link + 1; b < L; ++b) expanded[b - 1] = dim(rf[b], 0);
      lenv_root = fr.lenv;
      renv_root = fr.renv;
      root_start = cl.root;
      nclose = cl.lg.n_h1_closure + cl.nroot;
    } else if (P.order > 1) {
      Ledger lg;
      lg.order = P.order;
      int64_t nroot = 0;
      T current = root_start;
      ZeroSiteH op = S.root_generator(fr);
      std::vector<double> leak(P.order, std::numeric_limits<double>::quiet_NaN());
      bool met = true;
      for (int degree = 1; degree < P.order; ++degree) {
        T F = current;
        for (int d = 1; d <= degree; ++d) {
          nroot += 1;
          F = e.scale(op.apply(e, F), tau / double(d));
        }
        auto sw = S.frontier_sweep(fr, psi, F, nrm);
        lg.merge(sw.ledger);
        leak[degree] = sw.leak;
        met &= sw.met;
        if (sw.added > 0) {
          op = S.root_generator(fr);
          current = S.project_root(psi, fr);
        }
      }
      lg.n_passes = 1;
      lg.leak = leak;
      double defect = 0.0;
      for (int d = 0; d < P.order; ++d)
        if (!std::isnan(leak[d])) defect += leak[d] / (d + 1);
      lg.defect = defect;
      lg.n_root_frontier = nroot;
      if (!met) lg.unmet_(U_CLOSURE);
      ledger.merge(lg);
      lf = fr.lf;
      rf = fr.rf;
      for (int b = 1; b < S.root_link; ++b) expanded[b - 1] = dim(lf[b], 2);
      for (int b = S.root_link + 1; b < L; ++b) expanded[b - 1] = dim(rf[b], 0);
      lenv_root = fr.lenv;
      renv_root = fr.renv;
      root_start = current;
      nclose = lg.n_h1_closure + nroot;
    }
    const double npsi = e.norm(psi[psi.center]);
    int64_t mexp = 0;
    for (auto x : expanded) mexp = std::max(mexp, x);
    ledger.r_aug = std::max(mexp, dim(rf[S.root_link], 0));
    ledger.proj_err = npsi > 0 ? S.projection_miss(psi, lf, rf) / npsi : 0.0;
    if (ledger.proj_err > P.tol_basis) ledger.unmet_(U_PROJECTION);
    ZeroSiteH gen{S.env.left_step(lenv_root, lf[S.root_link], mpo[S.root_link]),
                  S.env.right_step(renv_root, rf[S.root_link], mpo[S.root_link + 1]), S.eshift};
    int64_t nroot_apps = 0;
    auto apply_root = [&](const T& v) {
      nroot_apps += 1;
      return gen.apply(e, v);
    };
    auto solve_root = [&](const T& start, Step::ExpvRep& r) {
      if (P.root_method == 4)
        return S.radau2_gmres_expv(apply_root, start, P.root_maxiter, 1e-15, P.tol_expv, P.root_shift, r);
      return P.hermitian ? S.lanczos_expv(apply_root, start, P.root_maxiter, 1e-15, P.reorth != 0, P.tol_expv, r,
                                          0, false, P.root_method, P.root_shift)
                         : S.arnoldi_expv(apply_root, start, P.root_maxiter, 1e-15, P.tol_expv, r, 0,
                                          P.root_method, P.root_shift);
    };
    Step::ExpvRep rep;
    // frames_only: the caller solves its own root on these frames, so the start is carried and no
    // expv report is read (bug_step.jl:381-382)
    T root_result = prm->frames_only ? root_start : solve_root(root_start, rep);
    if (prm->frames_out) {
      // frames_report (bug_step.jl:455-467): new handles owned by the caller, payloads shared
      auto out = [](const T& t) { return t ? std::make_unique<bug_tensor>(*t).release() : nullptr; };
      for (int b = 1; b < L; ++b) {
        prm->frames_out[b - 1] = b <= S.root_link ? out(lf[b]) : nullptr;
        prm->frames_out[L - 1 + b - 1] = b >= S.root_link ? out(rf[b]) : nullptr;
      }
      prm->frames_out[2 * L - 2] = out(lenv_root);
      prm->frames_out[2 * L - 1] = out(renv_root);
    }
    // the root report (_report_root!, bug_step_stages.jl:243-390)
    const double NaN = std::numeric_limits<double>::quiet_NaN();
    double r_e_pre = NaN, r_e_root = NaN, r_resid = NaN, r_init = NaN, r_out = NaN, r_outl = NaN,
           r_outr = NaN;
    int r_passes = 0, r_added = 0;
    if (prm->root_report) {
      auto rayleigh = [&](const T& v) {
        const double n2 = std::pow(e.norm(v), 2);
        if (!(n2 > 0)) return NaN;
        return e.inner(v, gen.apply(e, v)).real() / n2 + S.eshift;
      };
      // estimate_global_complement_action (frontier_closure.jl:238-277, nsample = 0): the
      // per-bond two-site misses of a non-enriching frontier sweep, drawn from a copy of the stream
      struct Action {
        double left = 0, right = 0, bound = 0;
        bool have = false;
      };
      auto outside_of = [&](const T& core) {
        Action a;
        Step::KL kf{lf, rf, lenv_root, renv_root, 0};
        if (e.buf) e.buf->save();
        else prm->rng_ctl(prm->rng_ctl_user, 0);
        auto sw = S.frontier_sweep(kf, psi, core, std::max(e.norm(core), EPS), false, false);
        if (e.buf) e.buf->restore();
        else prm->rng_ctl(prm->rng_ctl_user, 1);
        for (double x : sw.leaks_left) a.left += x * x;
        for (double x : sw.leaks_right) a.right += x * x;
        a.bound = std::sqrt(a.left + a.right);
        a.left = std::sqrt(a.left);
        a.right = std::sqrt(a.right);
        a.have = true;
        return a;
      };
      auto residual_of = [&](const Action& a, const T& v) {
        return a.have ? std::abs(tau) * a.bound / std::max(e.norm(v), EPS) : NaN;
      };
      r_e_pre = rayleigh(root_start);
      Action outside;
      if (prm->outside_residual) outside = outside_of(root_result);
      r_init = residual_of(outside, root_result);
      if (prm->outside_residual) {
        while (!(residual_of(outside, root_result) <= P.tol_basis) && r_passes < 2 * P.order + 2) {
          Step::KL kf{lf, rf, lenv_root, renv_root, 0};
          r_passes += 1;
          auto sw = S.frontier_sweep(kf, psi, root_result, nrm, true);
          ledger.merge(sw.ledger);
          if (sw.added == 0) break;
          r_added += int(sw.added);
          lf = kf.lf;
          rf = kf.rf;
          lenv_root = kf.lenv;
          renv_root = kf.renv;
          root_start = S.project_root(psi, kf);
          gen = S.root_generator(kf);
          rep = Step::ExpvRep{};
          root_result = solve_root(root_start, rep);
          outside = outside_of(root_result);
          if (sw.capped) break;
        }
        if (r_added > 0) {
          for (int b = 1; b < S.root_link; ++b) expanded[b - 1] = dim(lf[b], 2);
          for (int b = S.root_link + 1; b < L; ++b) expanded[b - 1] = dim(rf[b], 0);
          int64_t mx = 0;
          for (auto x : expanded) mx = std::max(mx, x);
          ledger.r_aug = std::max(mx, dim(rf[S.root_link], 0));
        }
      }
      r_e_root = rayleigh(root_result);
      if (outside.have) {
        const double rn = std::max(e.norm(root_result), EPS);
        r_out = outside.bound / rn;
        r_outl = outside.left / rn;
        r_outr = outside.right / rn;
        r_resid = std::abs(tau) * outside.bound / rn;
      }
    }
    ledger.expv_err = rep.err;
    ledger.expv_iters = rep.iters;
    if (rep.err > P.tol_expv * (1 + 1e-8)) ledger.unmet_(U_EXPV);
    SVDRes res = svd(e, root_result, {0}, 0.0, -1, W_U | W_SVD);
    expanded[S.root_link - 1] = dim(lf[S.root_link], 2);
    const int64_t root_frame_width = dim(rf[S.root_link], 0);
    // assemble and compress (diagnostics.jl:269-337)
    double discarded = trunc_weight(res);
    for (int s = 1; s < S.root_link; ++s) psi[s] = lf[s];
    psi[S.root_link] = e.contract(lf[S.root_link], {2}, res.U, {0});
    psi[S.root_link + 1] = e.contract(SVd(e, res), {1}, rf[S.root_link], {0});
    for (int b = S.root_link + 1; b < L; ++b) psi[b + 1] = rf[b];
    psi.center = S.root_link + 1;
    const int64_t root_rank = dim(psi[S.root_link], 2);
    if (P.truncate) {
      auto tr = S.truncate_recursive(psi, S.root_link + 1, P.maxdim, P.tol_trunc, bwts);
      discarded = std::max(discarded, std::get<0>(tr));
      ledger.n_compress += 1;
      ledger.discarded = std::get<1>(tr);
      ledger.maxdim_reached = std::get<2>(tr);
      if (std::get<1>(tr) > P.tol_trunc * (1 + 1e-8)) ledger.unmet_(U_TRUNC);
    }
    std::vector<int64_t> bd1 = psi.bond_dims();
    ledger.r_final = bd1.empty() ? 0 : *std::max_element(bd1.begin(), bd1.end());
    for (auto& bl : ledger.bond_log) {
      bl.r_old = int(bd0[bl.bond - 1]);
      bl.r_final = int(bd1[bl.bond - 1]);
      bl.discarded = bwts[bl.bond - 1];
    }
    // outputs: new site handles (the caller owns them), info, bond log
    for (int i = 0; i < L; ++i) {
      T& t = psi.s[i];
      bug_tensor* raw = t.get();
      if (raw == psi_io[i]) {
        psi_io[i] = nullptr;  // unchanged slot: the caller keeps its handle
        continue;
      }
      // transfer ownership out of the shared_ptr: copy the metadata, share the payload
      auto copy = std::make_unique<bug_tensor>(*raw);
      psi_io[i] = copy.release();
    }
    *center_io = psi.center;
    bug_step_info& o = *info;
    o.status = ledger.tolerance_met ? 0 : 1;
    o.unmet_mask = unmet_mask(ledger.unmet);
    o.root_link = S.root_link;
    o.root_rank = int(root_rank);
    o.root_frame_width = int(root_frame_width);
    o.discarded = discarded;
    o.n_matvec = S.nmv + nroot_apps + nclose;
    o.max_sample = ledger.max_sample;
    o.max_tail = ledger.max_tail;
    o.max_krylov = ledger.max_krylov;
    o.max_krylov_c = ledger.max_krylov_c;
    o.max_krylov_d = ledger.max_krylov_d;
    o.ledger_discarded = ledger.discarded;
    o.expv_err = ledger.expv_err;
    o.expv_iters = ledger.expv_iters;
    o.n_probes = ledger.n_probes;
    o.n_holdout = ledger.n_holdout;
    o.e_pre = r_e_pre;
    o.e_root = r_e_root;
    o.resid = r_resid;
    o.resid_initial = r_init;
    o.outside = r_out;
    o.outside_left = r_outl;
    o.outside_right = r_outr;
    o.outside_passes = r_passes;
    o.outside_added = r_added;
    o.n_targeted = ledger.n_targeted;
    o.n_selected = ledger.n_selected;
    o.n_krylov = ledger.n_krylov;
    o.n_h1 = ledger.n_h1;
    o.n_c_pass = ledger.n_c_pass;
    o.n_d_after_c = ledger.n_d_after_c;
    o.workcap_reached = ledger.workcap_reached;
    o.maxdim_reached = ledger.maxdim_reached;
    o.proj_err = ledger.proj_err;
    o.r_old = ledger.r_old;
    o.r_aug = ledger.r_aug;
    o.r_final = ledger.r_final;
    o.n_passes = ledger.n_passes;
    o.n_closure_sweeps = ledger.n_closure_sweeps;
    o.defect = ledger.defect;
    o.n_root_frontier = ledger.n_root_frontier;
    o.n_h1_closure = ledger.n_h1_closure;
    o.n_h2_leak = ledger.n_h2_leak;
    o.n_compress = ledger.n_compress;
    o.leak1 = ledger.leak.size() > 1 ? ledger.leak[1] : 0.0;
    for (int b = 0; b < L - 1 && b < BUG_MAX_SITES; ++b) {
      o.expanded[b] = int(expanded[b]);
      o.n_new[b] = int(n_new[b]);
      o.workcap[b] = int(S.wcap[b]);
    }
    for (int i = 0; i < 8 && i < int(ledger.unmet.size()); ++i) o.unmet_order[i] = ledger.unmet[i] + 1;
    if (n_bond_log) *n_bond_log = int(ledger.bond_log.size());
    if (bond_log)
      for (int i = 0; i < bond_log_cap && i < int(ledger.bond_log.size()); ++i) bond_log[i] = ledger.bond_log[i];
  });
}

// ── kernel-granular entry points ───────────────────────────────────────────────────────────
// The pieces of the step for a host that keeps the sweep logic itself: each takes borrowed
// handles and returns a new handle owned by the caller (metadata copied, payload shared: tensors
// are never mutated in place).

namespace {

T borrow(const bug_tensor* t) {
  require(t != nullptr, "null tensor handle");
  return T(const_cast<bug_tensor*>(t), [](bug_tensor*) {});
}

bug_tensor* hand_out(const T& t) { return t ? std::make_unique<bug_tensor>(*t).release() : nullptr; }

// local populations of the site whose tensor is `t` (centre there; leg 1 the site leg): the
// norm^2 of every local basis index, in leg order (sectors ascending, then index)
std::vector<double> site_populations(bug_ctx* c, const bug_tensor& t) {
  const Leg& sl = t.legs[1];
  const std::vector<double> n2 = sector_norms2(c, t, 1);
  std::vector<double> out;
  for (size_t s = 0; s < sl.q.size(); ++s) {
    if (sl.d[s] == 1) {
      out.push_back(n2[s]);
      continue;
    }
    double prev = 0.0;
    for (int k = 1; k <= sl.d[s]; ++k) {
      double cum = n2[s];
      if (k < sl.d[s]) {
        std::vector<int> counts(sl.q.size(), 0);
        counts[s] = k;
        auto tr = trim_impl(c, t, 1, counts.data());
        double r[2] = {0.0, 0.0};
        if (tr) dots(c, {{tr.get(), tr.get()}}, r);
        cum = r[0];
      }
      out.push_back(cum - prev);
      prev = cum;
    }
  }
  return out;
}

// normalised local populations of every site (centre moved to each in turn), flattened
std::vector<double> populations_impl(bug_ctx* c, int L, const bug_tensor* const* psi, int center) {
  require(c && psi && L >= 1 && center >= 1 && center <= L, "bad argument");
  Eng e{c, nullptr, nullptr};
  MPOv none;
  Step S(e, none, Params{}, cd(0.0), L);
  MPS phi;
  for (int i = 0; i < L; ++i) phi.s.push_back(borrow(psi[i]));
  phi.center = center;
  std::vector<double> out;
  S.canonical(phi, 1);
  for (int j = 1; j <= L; ++j) {
    if (j > 1) S.canonical(phi, j);
    std::vector<double> pop = site_populations(c, *phi[j]);
    double tot = 0.0;
    for (double x : pop) tot += x;
    for (double x : pop) out.push_back(tot > 0 ? x / tot : 0.0);
  }
  return out;
}

}  // namespace

extern "C" int bug_env_boundary(bug_ctx* c, int side, int charge, bug_tensor** out) {
  return guard([&] {
    require(c && out && (side == 0 || side == 1), "bad argument");
    Eng e{c, nullptr, nullptr};
    Env env{e};
    *out = hand_out(side == 0 ? env.left_boundary() : env.right_boundary(charge));
  });
}

extern "C" int bug_env_step(bug_ctx* c, int side, const bug_tensor* env_in, const bug_tensor* A,
                            const bug_tensor* W, bug_tensor** out) {
  return guard([&] {
    require(c && out && (side == 0 || side == 1), "bad argument");
    Eng e{c, nullptr, nullptr};
    Env env{e};
    *out = hand_out(side == 0 ? env.left_step(borrow(env_in), borrow(A), borrow(W))
                              : env.right_step(borrow(env_in), borrow(A), borrow(W)));
  });
}

extern "C" int bug_apply_one_site(bug_ctx* c, const bug_tensor* lenv, const bug_tensor* W,
                                  const bug_tensor* renv, const bug_tensor* x, bug_tensor** out) {
  return guard([&] {
    require(c && out, "null argument");
    Eng e{c, nullptr, nullptr};
    Env env{e};
    *out = hand_out(env.one_site(borrow(lenv), borrow(W), borrow(renv), borrow(x)));
  });
}

extern "C" int bug_apply_zero_site(bug_ctx* c, const bug_tensor* lgen, const bug_tensor* rgen,
                                   const bug_tensor* core, bug_tensor** out) {
  return guard([&] {
    require(c && out, "null argument");
    Eng e{c, nullptr, nullptr};
    ZeroSiteH h{borrow(lgen), borrow(rgen)};
    *out = hand_out(h.apply(e, borrow(core)));
  });
}

extern "C" int bug_sketch_stream(bug_ctx* c, int side, const bug_tensor* a, const bug_tensor* b,
                                 const bug_tensor* Wl, const bug_tensor* Wr, const bug_tensor* lenv,
                                 const bug_tensor* renv, const bug_tensor* probe, bug_tensor** out) {
  return guard([&] {
    require(c && out && (side == 0 || side == 1), "bad argument");
    Eng e{c, nullptr, nullptr};
    Env env{e};
    *out = hand_out(side == 0 ? env.stream_left(borrow(a), borrow(b), borrow(Wl), borrow(Wr),
                                                borrow(lenv), borrow(renv), borrow(probe))
                              : env.stream_right(borrow(a), borrow(b), borrow(Wl), borrow(Wr),
                                                 borrow(lenv), borrow(renv), borrow(probe)));
  });
}

extern "C" int bug_perp(bug_ctx* c, int side, const bug_tensor* frame, const bug_tensor* K,
                        bug_tensor** out) {
  return guard([&] {
    require(c && out && (side == 0 || side == 1), "bad argument");
    Eng e{c, nullptr, nullptr};
    *out = hand_out(side == 0 ? perp_left(e, borrow(frame), borrow(K))
                              : perp_right(e, borrow(frame), borrow(K)));
  });
}

extern "C" int bug_root_expv(bug_ctx* c, const bug_tensor* lgen, const bug_tensor* rgen,
                             const bug_tensor* core, double tau_re, double tau_im, int hermitian,
                             int maxiter, int reorth, double tol_expv, bug_tensor** out,
                             int64_t* iters, double* err) {
  return guard([&] {
    require(c && out, "null argument");
    require(maxiter >= 1, "maxiter must be positive");
    Eng e{c, nullptr, nullptr};
    MPOv none;
    Params P{};
    P.tol_expv = tol_expv;
    Step S(e, none, P, cd(tau_re, tau_im), 2);
    ZeroSiteH h{borrow(lgen), borrow(rgen)};
    auto apply = [&](const T& v) { return h.apply(e, v); };
    Step::ExpvRep rep;
    T r = hermitian ? S.lanczos_expv(apply, borrow(core), maxiter, 1e-15, reorth != 0, tol_expv, rep)
                    : S.arnoldi_expv(apply, borrow(core), maxiter, 1e-15, tol_expv, rep);
    *out = hand_out(r);
    if (iters) *iters = rep.iters;
    if (err) *err = rep.err;
  });
}

extern "C" int bug_site_populations(bug_ctx* c, int L, const bug_tensor* const* psi, int center,
                                    double* out, int cap, int* n_out) {
  return guard([&] {
    require(n_out != nullptr, "null argument");
    const std::vector<double> pop = populations_impl(c, L, psi, center);
    for (int i = 0; i < int(pop.size()) && i < cap; ++i)
      if (out) out[i] = pop[i];
    *n_out = int(pop.size());
  });
}

extern "C" int bug_observable_sz(bug_ctx* c, int L, const bug_tensor* const* psi, int center,
                                 double* out) {
  return guard([&] {
    require(out != nullptr, "null argument");
    const std::vector<double> pop = populations_impl(c, L, psi, center);
    size_t k = 0;
    for (int j = 0; j < L; ++j) {
      const Leg& sl = psi[j]->legs[1];
      double sz = 0.0;
      if (sl.q.size() == 1) {  // :none -- one charge-0 sector, index 0 up, 1 down
        require(sl.q[0] == 0 && sl.d[0] == 2, "S^z needs a spin-1/2 site");
        sz = 0.5 * pop[k] - 0.5 * pop[k + 1];
        k += 2;
      } else {  // U(1) -- the charge is 2 S^z, one state per sector
        for (size_t s = 0; s < sl.q.size(); ++s) {
          require(sl.d[s] == 1, "S^z needs a spin-1/2 site");
          sz += 0.5 * sl.q[s] * pop[k++];
        }
      }
      out[j] = sz;
    }
  });
}

// ── two-site TDVP (src/Baselines/TDVP/tdvp2.jl) ────────────────────────────────────────────
// One symmetric step: a forward sweep of two-site updates exp(tau/2 H2) with SVD splits and
// backward one-site half-steps exp(-tau/2 H1), then the mirror sweep (tdvp2_step!, :229-297;
// _tdvp2_bond!, :39-136; _tdvp2_backward, :145-173). The environments are carried bond to bond on
// the sweep's own side and read from one prebuilt stack on the other.

extern "C" int bug_tdvp2_step(bug_ctx* c, int L, bug_tensor** psi_io, int* center_io,
                              const bug_tensor* const* mpo_in, double tau_re, double tau_im,
                              const bug_tdvp2_params* prm, bug_tdvp2_info* info) {
  return guard([&] {
    require(c && psi_io && center_io && mpo_in && prm && info, "null argument");
    require(L >= 2, "tdvp2_step needs at least two sites");
    const int maxdim = prm->maxdim > 0 ? prm->maxdim : 200;
    const double trunc_thresh = prm->trunc_thresh >= 0 ? prm->trunc_thresh : 1e-12;
    const int maxiter = prm->maxiter > 0 ? prm->maxiter : 30;
    const double tol = prm->tol > 0 ? prm->tol : 1e-15;
    const bool hermitian = prm->hermitian != 0;
    const double conv_tol = prm->conv_tol;
    const int substeps = prm->substeps;
    require(substeps >= 0, "substeps must be >= 0");
    const double weight_tol = prm->weight_tol;
    const double eshift = prm->eshift;
    Eng e{c, nullptr, nullptr};
    MPOv mpo;
    for (int i = 0; i < L; ++i) mpo.W.push_back(borrow(mpo_in[i]));
    MPS psi;
    for (int i = 0; i < L; ++i) psi.s.push_back(borrow(psi_io[i]));
    psi.center = *center_io;
    require(psi.center >= 1 && psi.center <= L, "centre out of range");
    const cd tau(tau_re, tau_im), half = tau / 2.0;
    Step S(e, mpo, Params{}, half, L);
    const int root = std::max(1, std::min(L - 1, L / 2)) + 1;
    const double wdiv = std::sqrt(double(root - 1)) + std::sqrt(double(L - root));
    int64_t apps = 0, theta_max = 0, peak = 0;
    double worst = 0.0, wsum[2] = {0.0, 0.0}, total = 0.0;
    auto stored = [&]() {
      int64_t n = 0;
      for (auto& t : psi.s) n += t->nelem;
      return n;
    };
    auto expv = [&](const std::function<T(const T&)>& op, cd t, const T& v) {
      S.tau = t;
      Step::ExpvRep rep;
      auto counted = [&](const T& x) {
        apps += 1;
        T y = op(x);
        return eshift == 0.0 ? y : e.lin({{1.0, y}, {-eshift, x}});
      };
      // Lanczos keeps its recurrence coefficients on the device (one read-back per chunk of
      // iterations); applications past the host-driven chain's stop are not counted
      T r = hermitian ? S.lanczos_expv(counted, v, maxiter, tol, false, conv_tol, rep, substeps, true)
                      : S.arnoldi_expv(counted, v, maxiter, tol, conv_tol, rep, substeps);
      apps -= rep.wasted;
      return r;
    };
    auto split = [&](const T& theta, int want) {
      if (weight_tol < 0) return svd(e, theta, {0, 1}, std::max(trunc_thresh, 1e-14), maxdim, want);
      SVDRes res = svd(e, theta, {0, 1}, 0.0, maxdim, want);
      const double share = weight_tol * std::sqrt(sq_weight(res.kept) + sq_weight(res.trunc)) / wdiv;
      const int nk = int(res.kept.size());
      const int keep = std::max(tail_rank(res.kept, 1.0, share, nk, sq_weight(res.trunc)).first, 1);
      if (keep < nk) res = svd(e, theta, {0, 1}, 0.0, keep, want);
      return res;
    };
    auto bond = [&](int i, bool right, const T& lch, const T& rch, int sweep) -> T {
      T theta = e.contract(psi[i], {2}, psi[i + 1], {0});
      theta_max = std::max(theta_max, theta->nelem);
      peak = std::max(peak, stored() + theta->nelem);
      const T& Wl = mpo[i];
      const T& Wr = mpo[i + 1];
      theta = expv([&](const T& x) { return S.env.two_site(lch, Wl, Wr, rch, x); }, half, theta);
      SVDRes res = split(theta, right ? (W_U | W_SVD) : (W_VD | W_US));
      worst = std::max(worst, trunc_weight(res));
      wsum[sweep] += sq_weight(res.trunc);
      total = std::max(total, sq_weight(res.kept) + sq_weight(res.trunc));
      if (right) {
        psi[i] = res.U;
        T lnext = S.env.left_step(lch, psi[i], Wl);
        T M = SVd(e, res);
        if (i < L - 1) M = expv([&](const T& x) { return S.env.one_site(lnext, Wr, rch, x); }, -half, M);
        psi[i + 1] = M;
        psi.center = i + 1;
        return lnext;
      }
      psi[i + 1] = res.Vd;
      T rnext = S.env.right_step(rch, psi[i + 1], Wr);
      T M = US(e, res);
      if (i > 1) M = expv([&](const T& x) { return S.env.one_site(lch, Wl, rnext, x); }, -half, M);
      psi[i] = M;
      psi.center = i;
      return rnext;
    };
    S.canonical(psi, 1);
    std::vector<T> rstack = S.right_env_stack(psi, 3);
    T lch = S.env.left_boundary();
    for (int i = 1; i <= L - 1; ++i) lch = bond(i, true, lch, rstack[i + 2], 0);
    std::vector<T> lstack = S.left_env_stack(psi, L - 2);
    T rch = S.env.right_boundary(S.total_charge(psi));
    for (int i = L - 1; i >= 1; --i) {
      S.canonical(psi, i);
      rch = bond(i, false, lstack[i], rch, 1);
    }
    // outputs: new site handles (the caller owns them); an unchanged slot returns NULL
    for (int i = 0; i < L; ++i) {
      bug_tensor* raw = psi.s[i].get();
      if (raw == psi_io[i]) {
        psi_io[i] = nullptr;
        continue;
      }
      psi_io[i] = std::make_unique<bug_tensor>(*raw).release();
    }
    *center_io = psi.center;
    int64_t mb = 0;
    for (auto d : psi.bond_dims()) mb = std::max(mb, d);
    info->max_bond = int(mb);
    info->theta_elements = theta_max;
    info->discarded = worst;
    info->peak_elements = peak;
    info->krylov_dims = apps;
    info->cumulative = total > 0 ? (std::sqrt(wsum[0]) + std::sqrt(wsum[1])) / std::sqrt(total) : 0.0;
  });
}

extern "C" int bug_apply_two_site(bug_ctx* c, const bug_tensor* lenv, const bug_tensor* Wl,
                                  const bug_tensor* Wr, const bug_tensor* renv,
                                  const bug_tensor* theta, bug_tensor** out) {
  return guard([&] {
    require(c && out, "null argument");
    Eng e{c, nullptr, nullptr};
    Env env{e};
    *out = hand_out(env.two_site(borrow(lenv), borrow(Wl), borrow(Wr), borrow(renv), borrow(theta)));
  });
}

extern "C" int bug_work_ceilings(int rule, int nbonds, const int64_t* bonds, int64_t site_dim,
                                 int64_t maxdim, double factor, int root_link, double root_factor,
                                 int64_t* out) {
  return guard([&] {
    require(nbonds >= 0 && (nbonds == 0 || (bonds && out)), "bad arguments");
    std::vector<int64_t> b(bonds, bonds + nbonds);
    const std::vector<int64_t> w = work_ceilings(rule, b, site_dim, maxdim, factor, root_link, root_factor);
    std::copy(w.begin(), w.end(), out);
  });
}

extern "C" int bug_la_expm(int n, const double* a, double* out) {
  return guard([&] {
    require(n >= 0, "bad size");
    smallla::CMat A(n, n);
    for (int i = 0; i < n * n; ++i) A.a[i] = cd(a[2 * i], a[2 * i + 1]);
    smallla::CMat R = smallla::expm(A);
    for (int i = 0; i < n * n; ++i) {
      out[2 * i] = R.a[i].real();
      out[2 * i + 1] = R.a[i].imag();
    }
  });
}

extern "C" int bug_la_eigh_tridiag(int n, const double* d, const double* e, double* vals,
                                   double* vecs) {
  return guard([&] {
    require(n >= 0, "bad size");
    std::vector<double> dd(d, d + n), ee;
    if (n > 1) ee.assign(e, e + n - 1);
    require_finite_tridiag(dd.data(), dd.size(), ee.data(), ee.size());
    std::vector<double> v;
    smallla::RMat V;
    smallla::eigh_tridiag(dd, ee, v, V);
    for (int i = 0; i < n; ++i) vals[i] = v[i];
    for (int i = 0; i < n * n; ++i) vecs[i] = V.a[i];
  });
}

extern "C" int bug_la_eigh(int n, const double* a, double* vals, double* vecs) {
  return guard([&] {
    smallla::RMat A(n, n);
    for (int i = 0; i < n * n; ++i) A.a[i] = a[i];
    std::vector<double> v;
    smallla::RMat V;
    smallla::eigh_jacobi(A, v, V);
    for (int i = 0; i < n; ++i) vals[i] = v[i];
    for (int i = 0; i < n * n; ++i) vecs[i] = V.a[i];
  });
}

extern "C" int bug_la_kry_weight(int n, const double* hm, int k, double tau_re, double tau_im,
                                 int state_seed, double* out) {
  return guard([&] {
    require(n >= 2 && k >= 1 && k < n && hm && out, "bug_la_kry_weight: need 1 <= k < n");
    const size_t sub = 2 * (size_t(k) * n + size_t(k - 1));
    const double beta = std::hypot(hm[sub], hm[sub + 1]);
    if (beta == 0) {
      *out = 0.0;
      return;
    }
    const cd tau(tau_re, tau_im);
    smallla::CMat g(k, k);
    for (int i = 0; i < k; ++i)
      for (int j = 0; j < k; ++j)
        g(i, j) = tau * cd(hm[2 * (size_t(i) * n + j)], hm[2 * (size_t(i) * n + j) + 1]);
    *out = beta * bugs::residual_integral(k - 1, g, tau, state_seed != 0);
  });
}

extern "C" int bug_la_eigvals_hess(int n, const double* a, double* out) {
  return guard([&] {
    smallla::CMat A(n, n);
    for (int i = 0; i < n * n; ++i) A.a[i] = cd(a[2 * i], a[2 * i + 1]);
    auto ev = smallla::eigvals_hess(A);
    for (int i = 0; i < n; ++i) {
      out[2 * i] = ev[i].real();
      out[2 * i + 1] = ev[i].imag();
    }
  });
}
