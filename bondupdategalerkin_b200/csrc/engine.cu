// Host side of the B200 block-sparse engine: the contraction and SVD planners, descriptor staging,
// and the C-ABI of include/bug_b200.h.
//
// A tensor keeps its block table on the host (sorted keys, shapes, offsets) and its payload in
// one HBM allocation from the device's stream-ordered memory pool. Every operation plans on the
// host from the block tables, ships one descriptor array per kernel through a pinned staging
// ring, and launches a handful of kernels on the context stream; only operations whose result
// the host must read (norms, inner products, singular values, downloads) synchronise.
#include "engine.h"
#include "tcgemm.cuh"

namespace bugi {

thread_local std::string g_err;
thread_local bug_ctx* g_active_ctx = nullptr;

Buffer::~Buffer() {
  if (ptr && ctx) {
    ctx->dev_free(ptr);
    ctx->bytes -= n * int64_t(sizeof(double2));
  }
}

void run_copies(bug_ctx* c, std::vector<CopyDesc>& descs);

// Zero n elements at p: a copy stage whose source is null.
void zero_fill(bug_ctx* c, double2* p, int64_t n) {
  std::vector<CopyDesc> d;
  const int64_t chunk = int64_t(1) << 30;
  for (int64_t off = 0; off < n; off += chunk) {
    CopyDesc cd{};
    cd.src = nullptr;
    cd.dst = p + off;
    cd.n = std::min(chunk, n - off);
    cd.ndim = 1;
    cd.dims[0] = int(cd.n);
    cd.sstr[0] = 0;
    cd.dstr[0] = 1;
    cd.alpha = make_double2(1.0, 0.0);
    cd.wdim = -1;
    d.push_back(cd);
  }
  run_copies(c, d);
}

std::shared_ptr<Buffer> alloc_buffer(bug_ctx* c, int64_t n, bool zero) {
  auto b = std::make_shared<Buffer>();
  b->n = n;
  b->ctx = c->allocator();  // a second stream's tensors are returned to the allocator they came from
  if (n > 0) {
    b->ptr = static_cast<double2*>(c->dev_alloc(size_t(n) * sizeof(double2)));
    if (zero) zero_fill(c, b->ptr, n);
    b->ctx->bytes += n * int64_t(sizeof(double2));
  }
  return b;
}

int64_t block_size(const bug_tensor& t, const Key& k, std::array<int, BUG_MAX_RANK>& shape) {
  int64_t s = 1;
  for (int l = 0; l < t.rank; ++l) {
    int dd = t.legs[l].dim_of(k[l]);
    require(dd > 0, "block key uses a charge its leg does not carry");
    shape[l] = dd;
    s *= dd;
  }
  for (int l = t.rank; l < BUG_MAX_RANK; ++l) shape[l] = 1;
  return s;
}

// Finalise a tensor whose legs are set and whose keys are given (any order, no duplicates).
std::unique_ptr<bug_tensor> make_tensor(bug_ctx* c, int rank, std::vector<Leg> legs,
                                        std::vector<Key> keys, bool zero) {
  auto t = std::make_unique<bug_tensor>();
  t->rank = rank;
  t->legs = std::move(legs);
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  int64_t off = 0;
  for (auto& k : keys) {
    int flux = 0;
    for (int l = 0; l < rank; ++l) flux += t->legs[l].dir * k[l];
    require(flux == 0, "block key violates charge conservation");
    Block b;
    b.key = k;
    b.size = block_size(*t, k, b.shape);
    b.off = off;
    off += b.size;
    t->blocks.push_back(b);
  }
  t->nelem = off;
  t->buf = alloc_buffer(c, off, zero);
  return t;
}

Leg flipped(const Leg& l) {
  Leg o = l;
  o.dir = -l.dir;
  return o;
}

Leg merged(const Leg& a, const Leg& b) {
  require(a.dir == b.dir, "leg arrows differ");
  Leg o;
  o.dir = a.dir;
  std::map<int, int> m;
  for (size_t i = 0; i < a.q.size(); ++i) m[a.q[i]] = a.d[i];
  for (size_t i = 0; i < b.q.size(); ++i) {
    auto it = m.find(b.q[i]);
    if (it != m.end()) require(it->second == b.d[i], "sector dimensions differ");
    m[b.q[i]] = b.d[i];
  }
  for (auto& kv : m) {
    o.q.push_back(kv.first);
    o.d.push_back(kv.second);
  }
  return o;
}

std::array<int64_t, BUG_MAX_RANK> c_strides(const std::array<int, BUG_MAX_RANK>& shape, int rank) {
  std::array<int64_t, BUG_MAX_RANK> s{};
  int64_t acc = 1;
  for (int l = rank - 1; l >= 0; --l) {
    s[l] = acc;
    acc *= shape[l];
  }
  return s;
}

void run_copies(bug_ctx* c, std::vector<CopyDesc>& descs) {
  std::vector<CopyDesc> nz;
  nz.reserve(descs.size());
  int64_t total = 0;
  for (auto& d : descs) {
    if (d.n <= 0) continue;
    d.prefix = total;
    total += d.n;
    nz.push_back(d);
  }
  if (nz.empty()) return;
  CopyDesc* dd = c->push(nz);
  bugk::Stage st{};
  st.kind = bugk::kStageCopy;
  st.n = int(nz.size());
  st.total = total;
  st.a = dd;
  c->run_stage(st, BUG_K_COPY, 0.0, 32.0 * double(total));
}

CopyDesc plain_copy(const double2* src, double2* dst, int64_t n, bool conj, double2 alpha,
                    bool acc) {
  CopyDesc d{};
  d.src = src;
  d.dst = dst;
  d.n = n;
  d.ndim = 1;
  d.dims[0] = int(n);
  d.sstr[0] = 1;
  d.dstr[0] = 1;
  d.conj = conj;
  d.alpha = alpha;
  d.accumulate = acc;
  return d;
}

// Permuted copy: the result has legs perm[0..r) of t.
std::unique_ptr<bug_tensor> permute_impl(bug_ctx* c, const bug_tensor& t, const int* perm) {
  std::vector<Leg> legs(t.rank);
  std::vector<bool> seen(t.rank, false);
  for (int i = 0; i < t.rank; ++i) {
    require(perm[i] >= 0 && perm[i] < t.rank && !seen[perm[i]], "bad permutation");
    seen[perm[i]] = true;
    legs[i] = t.legs[perm[i]];
  }
  std::vector<Key> keys;
  for (auto& b : t.blocks) {
    Key k{};
    for (int i = 0; i < t.rank; ++i) k[i] = b.key[perm[i]];
    keys.push_back(k);
  }
  auto out = make_tensor(c, t.rank, legs, keys, false);
  std::vector<CopyDesc> descs;
  for (auto& b : t.blocks) {
    Key k{};
    for (int i = 0; i < t.rank; ++i) k[i] = b.key[perm[i]];
    const Block& ob = out->blocks[out->find(k)];
    auto ss = c_strides(b.shape, t.rank);
    auto ds = c_strides(ob.shape, t.rank);
    CopyDesc d{};
    d.src = t.data(&b - &t.blocks[0]);
    d.dst = out->mdata(out->find(k));
    d.n = b.size;
    d.ndim = t.rank;
    for (int i = 0; i < t.rank; ++i) {
      d.dims[i] = ob.shape[i];
      d.sstr[i] = ss[perm[i]];
      d.dstr[i] = ds[i];
    }
    d.alpha = make_double2(1.0, 0.0);
    descs.push_back(d);
  }
  run_copies(c, descs);
  return out;
}

// ── contraction ──

// View one block as a matrix: rows = legs `rl` (C order), cols = legs `cl`; adjacent dims whose
// strides chain are merged, so the kernel decomposes as few indices as possible.
void make_group(const Block& b, const std::array<int64_t, BUG_MAX_RANK>& st,
                const std::vector<int>& legs, int& n, int* d, int64_t* s) {
  int dd[BUG_MAX_RANK];
  int64_t ss[BUG_MAX_RANK];
  int k = 0;
  for (int l : legs) {
    if (k > 0 && ss[k - 1] == int64_t(b.shape[l]) * st[l]) {
      dd[k - 1] *= b.shape[l];
      ss[k - 1] = st[l];
    } else {
      dd[k] = b.shape[l];
      ss[k] = st[l];
      ++k;
    }
  }
  // drop unit dims
  n = 0;
  for (int i = 0; i < k; ++i)
    if (dd[i] != 1) {
      require(n < bugk::kGroup, "contract: operand index group too deep");
      d[n] = dd[i];
      s[n] = ss[i];
      ++n;
    }
}

void make_operand(bugk::Operand& op, const double2* p, const Block& b, const std::vector<int>& rows,
                  const std::vector<int>& cols, bool conj) {
  // shape entries past the tensor's rank are 1, so full-rank C strides equal the tensor's own
  const auto st = c_strides(b.shape, BUG_MAX_RANK);
  op.p = p;
  op.conj = conj ? 1 : 0;
  make_group(b, st, rows, op.nr, op.rd, op.rs);
  make_group(b, st, cols, op.nc, op.cd, op.cs);
  op.row_fast = (op.nr > 0 && op.rs[op.nr - 1] == 1) ? 1 : 0;
}

// Per-thread planning arrays of contract_impl.
struct BRef {
  std::array<int, BUG_MAX_RANK> ck;  // the block's charges on the contracted legs
  int bi;
};
struct OutPair {
  Key ok;  // output block key
  int ai, bi;
};
struct ContractPlan {
  std::vector<BRef> bref;
  std::vector<OutPair> ops;
  std::vector<GemmOut> outs;
  std::vector<GemmPair> pairs;
  std::vector<GemmTile> tiles;
  std::vector<int> mixed;
};

std::unique_ptr<bug_tensor> contract_impl(bug_ctx* c, const bug_tensor& A0, int n, const int* ia,
                                          const bug_tensor& B0, const int* ib, bool conja,
                                          bool conjb) {
  require(n >= 0 && n <= A0.rank && n <= B0.rank, "bad contraction arity");
  std::vector<bool> ca(A0.rank, false), cb(B0.rank, false);
  for (int k = 0; k < n; ++k) {
    require(ia[k] >= 0 && ia[k] < A0.rank && !ca[ia[k]], "bad contracted leg of A");
    require(ib[k] >= 0 && ib[k] < B0.rank && !cb[ib[k]], "bad contracted leg of B");
    ca[ia[k]] = true;
    cb[ib[k]] = true;
    const Leg& la = A0.legs[ia[k]];
    const Leg& lb = B0.legs[ib[k]];
    int da = conja ? -la.dir : la.dir, db = conjb ? -lb.dir : lb.dir;
    require(da == -db, "contract: paired legs must have opposite arrows");
    for (size_t i = 0; i < la.q.size(); ++i) {
      int dbb = lb.dim_of(la.q[i]);
      require(dbb == 0 || dbb == la.d[i], "contract: sector dimensions differ");
    }
  }
  std::vector<int> fa, fb;
  for (int i = 0; i < A0.rank; ++i)
    if (!ca[i]) fa.push_back(i);
  for (int i = 0; i < B0.rank; ++i)
    if (!cb[i]) fb.push_back(i);
  const int ro = int(fa.size() + fb.size());
  require(ro <= BUG_MAX_RANK, "result rank exceeds the engine limit");
  std::vector<Leg> legs;
  for (int i : fa) legs.push_back(conja ? flipped(A0.legs[i]) : A0.legs[i]);
  for (int i : fb) legs.push_back(conjb ? flipped(B0.legs[i]) : B0.legs[i]);

  const bug_tensor* A = &A0;
  const bug_tensor* B = &B0;
  std::vector<int> iaa(ia, ia + n), ibb(ib, ib + n);
  const std::vector<int>& fa2 = fa;
  const std::vector<int>& fb2 = fb;
  // match blocks: B's blocks ordered by their contracted charges (a stable sort keeps equal ones
  // in block order), each A block against its run; the (A block, B block) pairs of every output
  // key then in A-block-major order, output keys ascending (a stable sort of the pair list)
  // the planning arrays live per thread across calls (their capacity is reused, no allocation)
  thread_local ContractPlan plan;
  auto ck_less = [n](const BRef& x, const BRef& y) {
    return std::lexicographical_compare(x.ck.begin(), x.ck.begin() + n, y.ck.begin(),
                                        y.ck.begin() + n);
  };
  std::vector<BRef>& bref = plan.bref;
  bref.resize(B->blocks.size());
  for (int bi = 0; bi < int(B->blocks.size()); ++bi) {
    bref[size_t(bi)].bi = bi;
    for (int k = 0; k < n; ++k) bref[size_t(bi)].ck[size_t(k)] = B->blocks[bi].key[ibb[k]];
  }
  std::stable_sort(bref.begin(), bref.end(), ck_less);
  std::vector<OutPair>& ops = plan.ops;
  ops.clear();
  BRef probe{};
  for (int ai = 0; ai < int(A->blocks.size()); ++ai) {
    for (int k = 0; k < n; ++k) probe.ck[size_t(k)] = A->blocks[ai].key[iaa[k]];
    auto run = std::equal_range(bref.begin(), bref.end(), probe, ck_less);
    for (auto it = run.first; it != run.second; ++it) {
      OutPair e{};
      int p = 0;
      for (int i : fa2) e.ok[p++] = A->blocks[ai].key[i];
      for (int i : fb2) e.ok[p++] = B->blocks[it->bi].key[i];
      e.ai = ai;
      e.bi = it->bi;
      ops.push_back(e);
    }
  }
  std::stable_sort(ops.begin(), ops.end(),
                   [](const OutPair& x, const OutPair& y) { return x.ok < y.ok; });
  std::vector<Key> keys;
  for (size_t i = 0; i < ops.size(); ++i)
    if (i == 0 || ops[i].ok != ops[i - 1].ok) keys.push_back(ops[i].ok);
  auto out = make_tensor(c, ro, legs, keys, false);
  if (keys.empty()) return out;
  std::vector<GemmOut>& outs = plan.outs;
  std::vector<GemmPair>& pairs = plan.pairs;
  std::vector<GemmTile>& tiles = plan.tiles;
  std::vector<int>& mixed = plan.mixed;  // outputs the tensor-core path computes
  outs.clear();
  pairs.clear();
  tiles.clear();
  mixed.clear();
  for (size_t r0 = 0, oj = 0; r0 < ops.size(); ++oj) {
    size_t r1 = r0 + 1;
    while (r1 < ops.size() && ops[r1].ok == ops[r0].ok) ++r1;
    require(out->blocks[oj].key == ops[r0].ok, "contract: output block order");
    const Block& ob = out->blocks[oj];
    GemmOut go{};
    go.C = out->mdata(oj);
    int64_t m = 1, nn = 1;
    for (size_t i = 0; i < fa2.size(); ++i) m *= ob.shape[i];
    for (size_t i = 0; i < fb2.size(); ++i) nn *= ob.shape[fa2.size() + i];
    go.m = int(m);
    go.n = int(nn);
    go.pair_begin = int(pairs.size());
    for (size_t r = r0; r < r1; ++r) {
      const Block& ab = A->blocks[ops[r].ai];
      const Block& bb = B->blocks[ops[r].bi];
      int64_t K = 1;
      for (int k = 0; k < n; ++k) K *= ab.shape[iaa[k]];
      GemmPair gp{};
      gp.k = int(K);
      make_operand(gp.A, A->data(ops[r].ai), ab, fa2, iaa, conja);
      make_operand(gp.B, B->data(ops[r].bi), bb, ibb, fb2, conjb);
      pairs.push_back(gp);
    }
    go.pair_end = int(pairs.size());
    r0 = r1;
    int o = int(outs.size());
    outs.push_back(go);
    if (c->mixed_min_dim > 0 && bugtc::mixed_block(int(m), int(nn), c->mixed_min_dim)) {
      mixed.push_back(o);
      continue;
    }
    for (int tm = 0; tm * 32 < m; ++tm)
      for (int tn = 0; tn * 32 < nn; ++tn) tiles.push_back(GemmTile{o, tm, tn});
  }
  if (!mixed.empty()) bugtc::run_mixed(c, outs, pairs, mixed);
  if (tiles.empty()) return out;
  GemmOut* d_outs = c->push(outs);
  GemmPair* d_pairs = c->push(pairs);
  GemmTile* d_tiles = c->push(tiles);
  double flops = 0.0, gbytes = 0.0;
  std::vector<char> is_mixed(outs.size(), 0);
  for (int o : mixed) is_mixed[size_t(o)] = 1;
  for (size_t o = 0; o < outs.size(); ++o) {
    if (is_mixed[o]) continue;
    const GemmOut& go = outs[o];
    gbytes += 16.0 * double(go.m) * double(go.n);
    for (int p = go.pair_begin; p < go.pair_end; ++p) {
      flops += 8.0 * double(go.m) * double(go.n) * double(pairs[p].k);
      gbytes += 16.0 * (double(go.m) + double(go.n)) * double(pairs[p].k);
    }
  }
  bugk::Stage st{};
  st.kind = bugk::kStageGemm;
  st.n = int(tiles.size());
  st.a = d_outs;
  st.b = d_pairs;
  st.c = d_tiles;
  c->run_stage(st, BUG_K_GEMM, flops, gbytes);
  return out;
}

// ── SVD ──────────────────────────────────────────────────────────────────────────────────────

struct SectorPlan {
  int charge;
  std::vector<std::vector<int>> rows, cols;  // left / right charge tuples
  std::vector<int64_t> rdim, cdim, roff, coff;
  int64_t m = 0, n = 0;
};

// One tensor's SVD inside a multi-tensor launch: its sector plans and its offsets into the shared
// workspace, singular values and read-back arrays.
struct SvdJob {
  const bug_tensor* t = nullptr;
  std::vector<int> L, R;
  std::map<int, SectorPlan> plans;
  std::vector<SectorPlan*> order;
  std::vector<int64_t> woff, vwoff, uoff, voff, soff;
  int64_t wtot = 0, stot = 0;
  int np = 0;
};

void svd_plan(SvdJob& j, const bug_tensor& t, int nleft, const int* left) {
  require(nleft >= 0 && nleft <= t.rank, "bad split");
  j.t = &t;
  std::vector<bool> isl(t.rank, false);
  j.L.assign(left, left + nleft);
  for (int i : j.L) {
    require(i >= 0 && i < t.rank && !isl[i], "bad left leg");
    isl[i] = true;
  }
  for (int i = 0; i < t.rank; ++i)
    if (!isl[i]) j.R.push_back(i);
  const std::vector<int>& L = j.L;
  const std::vector<int>& R = j.R;
  for (auto& b : t.blocks) {
    int cq = 0;
    for (int i : L) cq -= t.legs[i].dir * b.key[i];
    std::vector<int> rk, ck;
    for (int i : L) rk.push_back(b.key[i]);
    for (int i : R) ck.push_back(b.key[i]);
    auto& p = j.plans[cq];
    p.charge = cq;
    p.rows.push_back(rk);
    p.cols.push_back(ck);
  }
  for (auto& kv : j.plans) {
    auto& p = kv.second;
    std::sort(p.rows.begin(), p.rows.end());
    p.rows.erase(std::unique(p.rows.begin(), p.rows.end()), p.rows.end());
    std::sort(p.cols.begin(), p.cols.end());
    p.cols.erase(std::unique(p.cols.begin(), p.cols.end()), p.cols.end());
    for (auto& rk : p.rows) {
      int64_t sz = 1;
      for (size_t q = 0; q < L.size(); ++q) sz *= t.legs[L[q]].dim_of(rk[q]);
      p.roff.push_back(p.m);
      p.rdim.push_back(sz);
      p.m += sz;
    }
    for (auto& ck : p.cols) {
      int64_t sz = 1;
      for (size_t q = 0; q < R.size(); ++q) sz *= t.legs[R[q]].dim_of(ck[q]);
      p.coff.push_back(p.n);
      p.cdim.push_back(sz);
      p.n += sz;
    }
    j.order.push_back(&p);
  }
  j.np = int(j.order.size());
  // workspace per sector: work (mm*r), vwork (r*r), U (m*r), V (n*r), S (r)
  j.woff.resize(j.np);
  j.vwoff.resize(j.np);
  j.uoff.resize(j.np);
  j.voff.resize(j.np);
  j.soff.resize(j.np);
  for (int q = 0; q < j.np; ++q) {
    auto& p = *j.order[q];
    int64_t mm = std::max(p.m, p.n), r = std::min(p.m, p.n);
    require(r <= 1024, "SVD sector wider than the engine's 1024-column limit");
    j.woff[q] = j.wtot;
    j.wtot += mm * r;
    j.vwoff[q] = j.wtot;
    j.wtot += r * r;
    j.uoff[q] = j.wtot;
    j.wtot += p.m * r;
    j.voff[q] = j.wtot;
    j.wtot += p.n * r;
    j.soff[q] = j.stot;
    j.stot += r;
  }
}

// Selection and factors of one job after the launch's read-back.
void svd_finish(bug_ctx* c, SvdJob& job, const SvdReq& q, double2* W, double* S, const double* host) {
  const bug_tensor& t = *job.t;
  const std::vector<int>& L = job.L;
  const std::vector<int>& R = job.R;
  const int np = job.np;
  auto& order = job.order;
  auto& uoff = job.uoff;
  auto& voff = job.voff;
  auto& soff = job.soff;
  const double cutoff = q.cutoff;
  const int nkeep = q.nkeep;
  const int want = q.want;
  std::vector<double>& sv_sorted = *q.sv_sorted;
  std::vector<int>& sv_q = *q.sv_q;
  int& nkept = *q.nkept;
  std::unique_ptr<bug_tensor>& U = *q.U;
  std::unique_ptr<bug_tensor>& Vd = *q.Vd;
  std::unique_ptr<bug_tensor>* USo = q.USo;
  std::unique_ptr<bug_tensor>* SVdo = q.SVdo;
  std::vector<int> kc(np, 0);
  sv_sorted.clear();
  sv_q.clear();
  if (!host) {
    // taken ahead (svd_ahead): every sector keeps all min(m, n) columns, which is the selection
    // below exactly when cutoff is 0, no Nkeep applies and every singular value is positive
    nkept = 0;
    for (int s = 0; s < np; ++s) {
      kc[s] = int(std::min(order[s]->m, order[s]->n));
      nkept += kc[s];
    }
  } else {
    // selection (Telum): sigma > cutoff*smax, stable descending sort, Nkeep
    struct Entry {
      double sv;
      int s, j;
    };
    std::vector<Entry> entries;
    double smax = 0.0;
    for (int s = 0; s < np; ++s) {
      int64_t r = std::min(order[s]->m, order[s]->n);
      for (int j = 0; j < r; ++j) {
        double v = host[soff[s] + j];
        require(std::isfinite(v), "non-finite singular value");
        smax = std::max(smax, v);
        entries.push_back({v, s, j});
      }
    }
    std::stable_sort(entries.begin(), entries.end(),
                     [](const Entry& a, const Entry& b) { return a.sv > b.sv; });
    const double thresh = cutoff * smax;
    int nsel = 0;
    for (auto& e : entries)
      if (e.sv > thresh) ++nsel;
    if (nkeep >= 0) nsel = std::min(nsel, nkeep);
    for (int i = 0; i < nsel; ++i) kc[entries[i].s]++;
    for (auto& e : entries) {
      sv_sorted.push_back(e.sv);
      sv_q.push_back(order[e.s]->charge);
    }
    nkept = nsel;
  }
  // build U and Vd
  Leg bondU, bondV;
  bondU.dir = +1;
  bondV.dir = -1;
  for (int s = 0; s < np; ++s)
    if (kc[s] > 0) {
      bondU.q.push_back(order[s]->charge);
      bondU.d.push_back(kc[s]);
    }
  bondV.q = bondU.q;
  bondV.d = bondU.d;
  std::vector<Leg> ulegs, vlegs;
  for (int i : L) ulegs.push_back(t.legs[i]);
  ulegs.push_back(bondU);
  vlegs.push_back(bondV);
  for (int i : R) vlegs.push_back(t.legs[i]);
  std::vector<Key> ukeys, vkeys;
  for (int s = 0; s < np; ++s) {
    if (kc[s] == 0) continue;
    auto& p = *order[s];
    for (auto& rk : p.rows) {
      Key k{};
      for (size_t j = 0; j < rk.size(); ++j) k[j] = rk[j];
      k[rk.size()] = p.charge;
      ukeys.push_back(k);
    }
    for (auto& ck : p.cols) {
      Key k{};
      k[0] = p.charge;
      for (size_t j = 0; j < ck.size(); ++j) k[j + 1] = ck[j];
      vkeys.push_back(k);
    }
  }
  if (want & 1) U = make_tensor(c, int(L.size()) + 1, ulegs, ukeys, false);
  if (want & 2) Vd = make_tensor(c, int(R.size()) + 1, vlegs, vkeys, false);
  if ((want & 4) && USo) *USo = make_tensor(c, int(L.size()) + 1, ulegs, ukeys, false);
  if ((want & 8) && SVdo) *SVdo = make_tensor(c, int(R.size()) + 1, vlegs, vkeys, false);
  std::vector<CopyDesc> out;
  for (int s = 0; s < np; ++s) {
    if (kc[s] == 0) continue;
    auto& p = *order[s];
    for (size_t ri = 0; ri < p.rows.size(); ++ri) {
      Key k{};
      for (size_t j = 0; j < p.rows[ri].size(); ++j) k[j] = p.rows[ri][j];
      k[p.rows[ri].size()] = p.charge;
      CopyDesc d{};
      d.src = W + uoff[s] + p.roff[ri];
      d.n = p.rdim[ri] * kc[s];
      d.ndim = 2;
      d.dims[0] = int(p.rdim[ri]);
      d.dims[1] = kc[s];
      d.sstr[0] = 1;
      d.sstr[1] = p.m;
      d.dstr[0] = kc[s];
      d.dstr[1] = 1;
      d.alpha = make_double2(1.0, 0.0);
      if (want & 1) {
        d.dst = U->mdata(U->find(k));
        out.push_back(d);
      }
      if ((want & 4) && USo) {
        d.dst = (*USo)->mdata((*USo)->find(k));
        d.w = S + soff[s];
        d.wdim = 1;
        out.push_back(d);
      }
    }
    for (size_t ci = 0; ci < p.cols.size(); ++ci) {
      Key k{};
      k[0] = p.charge;
      for (size_t j = 0; j < p.cols[ci].size(); ++j) k[j + 1] = p.cols[ci][j];
      CopyDesc d{};
      d.src = W + voff[s] + p.coff[ci];
      d.n = p.cdim[ci] * kc[s];
      d.ndim = 2;
      d.dims[0] = kc[s];
      d.dims[1] = int(p.cdim[ci]);
      d.sstr[0] = p.n;
      d.sstr[1] = 1;
      d.dstr[0] = p.cdim[ci];
      d.dstr[1] = 1;
      d.conj = 1;
      d.alpha = make_double2(1.0, 0.0);
      if (want & 2) {
        d.dst = Vd->mdata(Vd->find(k));
        out.push_back(d);
      }
      if ((want & 8) && SVdo) {
        d.dst = (*SVdo)->mdata((*SVdo)->find(k));
        d.w = S + soff[s];
        d.wdim = 0;
        out.push_back(d);
      }
    }
  }
  run_copies(c, out);
}


// The SVDs of several tensors: one Jacobi launch over all their sectors and one read-back; then
// each tensor's Telum selection and its factors, exactly as one call per tensor would give them
// (a sector's arithmetic does not depend on the other sectors of the launch).
// The jobs of one SVD launch: plans, workspace and where each job's parts start.
struct SvdBatch {
  std::vector<SvdJob> jobs;
  std::vector<int64_t> wbase, sbase, pbase;
  int64_t wtot = 0, stot = 0, nptot = 0;
  double2* W0 = nullptr;
  double* S0 = nullptr;
};

static void svd_plan_batch(bug_ctx* c, const std::vector<SvdReq>& reqs, SvdBatch& B) {
  B.jobs.resize(reqs.size());
  B.wbase.resize(reqs.size());
  B.sbase.resize(reqs.size());
  B.pbase.resize(reqs.size());
  for (size_t r = 0; r < reqs.size(); ++r) {
    svd_plan(B.jobs[r], *reqs[r].t, reqs[r].nleft, reqs[r].left);
    B.wbase[r] = B.wtot;
    B.sbase[r] = B.stot;
    B.pbase[r] = B.nptot;
    B.wtot += B.jobs[r].wtot;
    B.stot += B.jobs[r].stot;
    B.nptot += B.jobs[r].np;
  }
  B.W0 = static_cast<double2*>(c->scratch(size_t(std::max<int64_t>(B.wtot, 1)) * sizeof(double2)));
  B.S0 = static_cast<double*>(c->scratch(size_t(std::max<int64_t>(B.stot, 1)) * sizeof(double)));
}

// The Jacobi launch of a planned batch; singular values and sweep counts also go straight to the
// host-mapped pinned memory at host0 (stot values) and sweeps0 (nptot counts).
static void svd_launch_batch(bug_ctx* c, SvdBatch& B, double* host0, int* sweeps0) {
  std::vector<SvdJob>& jobs = B.jobs;
  double2* W0 = B.W0;
  double* S0 = B.S0;
  const std::vector<int64_t>& wbase = B.wbase;
  const std::vector<int64_t>& sbase = B.sbase;
  const std::vector<int64_t>& pbase = B.pbase;
  for (int64_t q = 0; q < B.nptot; ++q) sweeps0[q] = 0;
  const int smem_limit = bugk::svd_smem_limit();
  std::vector<SvdDesc> sd;
  std::vector<CopyDesc> packs;
  int max_smem = 0;
  int64_t max_r = 0;
  double sbytes = 0.0, sflops = 0.0;
  for (size_t r = 0; r < jobs.size(); ++r) {
    SvdJob& j = jobs[r];
    const bug_tensor& t = *j.t;
    const std::vector<int>& L = j.L;
    const std::vector<int>& R = j.R;
    double2* W = W0 + wbase[r];
    double* S = S0 + sbase[r];
    double* host = host0 + sbase[r];
    // gather descriptors of the sector matrices (column-major M, or M^H when m < n), run inside
    // the Jacobi kernel itself
    std::vector<std::vector<CopyDesc>> packs_of(j.order.size());
    for (int bi = 0; bi < int(t.blocks.size()); ++bi) {
      const Block& b = t.blocks[bi];
      int cq = 0;
      for (int i : L) cq -= t.legs[i].dir * b.key[i];
      auto& p = j.plans[cq];
      int sec = int(std::find(j.order.begin(), j.order.end(), &p) - j.order.begin());
      std::vector<int> rk, ck;
      for (int i : L) rk.push_back(b.key[i]);
      for (int i : R) ck.push_back(b.key[i]);
      int ri = int(std::lower_bound(p.rows.begin(), p.rows.end(), rk) - p.rows.begin());
      int ci = int(std::lower_bound(p.cols.begin(), p.cols.end(), ck) - p.cols.begin());
      const bool trans = p.m < p.n;
      auto ss = c_strides(b.shape, t.rank);
      CopyDesc d{};
      d.src = t.data(bi);
      d.dst = W + j.woff[sec];
      d.n = b.size;
      d.ndim = t.rank;
      d.conj = trans ? 1 : 0;
      d.alpha = make_double2(1.0, 0.0);
      // element multi-index in (L..., R...) order; row = C-order over L dims, col over R dims
      int p_i = 0;
      int64_t rs = 1, cs = 1;
      std::array<int64_t, BUG_MAX_RANK> rstr{}, cstr{};
      for (int q = int(L.size()) - 1; q >= 0; --q) {
        rstr[q] = rs;
        rs *= b.shape[L[q]];
      }
      for (int q = int(R.size()) - 1; q >= 0; --q) {
        cstr[q] = cs;
        cs *= b.shape[R[q]];
      }
      const int64_t ldw = trans ? p.n : p.m;  // leading dimension of the column-major work
      for (size_t q = 0; q < L.size(); ++q, ++p_i) {
        d.dims[p_i] = b.shape[L[q]];
        d.sstr[p_i] = ss[L[q]];
        d.dstr[p_i] = trans ? rstr[q] * ldw : rstr[q];
      }
      for (size_t q = 0; q < R.size(); ++q, ++p_i) {
        d.dims[p_i] = b.shape[R[q]];
        d.sstr[p_i] = ss[R[q]];
        d.dstr[p_i] = trans ? cstr[q] : cstr[q] * ldw;
      }
      const int64_t base = trans ? (p.coff[ci] + p.roff[ri] * ldw) : (p.roff[ri] + p.coff[ci] * ldw);
      d.dst += base;
      packs_of[sec].push_back(d);
    }
    for (int sec = 0; sec < j.np; ++sec) {
      auto& p = *j.order[sec];
      int64_t mm = std::max(p.m, p.n), rr = std::min(p.m, p.n);
      SvdDesc d{};
      d.work = W + j.woff[sec];
      d.vwork = W + j.vwoff[sec];
      d.U = W + j.uoff[sec];
      d.V = W + j.voff[sec];
      d.S = S + j.soff[sec];
      d.S_host = host + j.soff[sec];
      d.sweeps = sweeps0 + pbase[r] + sec;
      d.m = int(p.m);
      d.n = int(p.n);
      d.trans = p.m < p.n ? 1 : 0;
      // shared memory for A and V if both fit, else for A alone, else none
      const int64_t both = (mm * rr + rr * rr) * int64_t(sizeof(double2));
      const int64_t a_only = mm * rr * int64_t(sizeof(double2));
      d.use_smem = both <= smem_limit ? 2 : (a_only <= smem_limit ? 1 : 0);
      if (d.use_smem) max_smem = std::max<int>(max_smem, int(d.use_smem == 2 ? both : a_only));
      max_r = std::max(max_r, rr);
      d.pack_begin = int(packs.size());
      packs.insert(packs.end(), packs_of[sec].begin(), packs_of[sec].end());
      d.pack_end = int(packs.size());
      sd.push_back(d);
      sbytes += 16.0 * (2.0 * double(mm) * double(rr) + double(rr) * double(rr) + double(p.m + p.n) * double(rr));
      sflops += 8.0 * 2.0 * double(mm) * double(rr) * double(rr);  // one QR-equivalent pass
    }
  }
  const int np = int(sd.size());
  if (np > 0) {
    SvdDesc* dsd = c->push(sd);
    CopyDesc* dpk = c->push(packs);
    // one warp per column pair of a round (8 to 32 warps): a round's pairs run side by side
    // instead of in turns. Which warp takes a pair or a column changes no reduction order, so
    // the factors are the same bits for any warp count.
    const int warps = int(std::min<int64_t>(32, std::max<int64_t>(8, (max_r + 1) / 2)));
    const bugk::Blob blob = c->begin();
    bugk::launch_svd(blob, dsd, np, dpk, max_smem, 32 * warps, c->stream);
    c->launched(BUG_K_SVD, sflops, sbytes);
  }
}

void svd_many(bug_ctx* c, const std::vector<SvdReq>& reqs) {
  SvdBatch B;
  svd_plan_batch(c, reqs, B);
  double* host0 = c->readback(size_t(B.stot) + size_t(B.nptot) + 1);
  int* sweeps0 = reinterpret_cast<int*>(host0 + B.stot);
  svd_launch_batch(c, B, host0, sweeps0);
  // the kernel wrote singular values and sweep counts into `host`
  c->wait();
  for (int64_t q = 0; q < B.nptot; ++q)
    if (sweeps0[q] < 0) throw BugError(BUG_ENOTCONV, "Jacobi SVD did not converge within its sweep bound");
  for (size_t r = 0; r < reqs.size(); ++r)
    svd_finish(c, B.jobs[r], reqs[r], B.W0 + B.wbase[r], B.S0 + B.sbase[r], host0 + B.sbase[r]);
}

bool svd_ahead(bug_ctx* c, const std::vector<SvdReq>& reqs) {
  for (auto& q : reqs)
    require(q.cutoff == 0.0 && q.nkeep < 0, "an SVD taken ahead keeps every column");
  if (!c->ahead_host) {
    BUG_CUDA(cudaHostAlloc((void**)&c->ahead_host, bug_ctx::kAheadCap * sizeof(double),
                           cudaHostAllocDefault));
  }
  SvdBatch B;
  svd_plan_batch(c, reqs, B);
  const size_t need = size_t(B.stot) + size_t(B.nptot) + 1;
  if (c->ahead_used + need > bug_ctx::kAheadCap) return false;
  double* host0 = c->ahead_host + c->ahead_used;
  int* sweeps0 = reinterpret_cast<int*>(host0 + B.stot);
  c->ahead.push_back({c->ahead_used, size_t(B.stot), size_t(B.nptot)});
  c->ahead_used += need;
  svd_launch_batch(c, B, host0, sweeps0);
  for (size_t r = 0; r < reqs.size(); ++r)
    svd_finish(c, B.jobs[r], reqs[r], B.W0 + B.wbase[r], B.S0 + B.sbase[r], nullptr);
  return true;
}

bool svd_ahead_check(bug_ctx* c) {
  // BUG_SVD_AHEAD_REDO=1 fails every check that had SVDs ahead, so that the exact redo of every
  // caller runs after its ahead attempt (same results, twice the work; for testing the redo)
  static const bool redo = [] {
    const char* v = std::getenv("BUG_SVD_AHEAD_REDO");
    return v && std::string(v) == "1";
  }();
  bool ok = !(redo && !c->ahead.empty());
  if (!c->ahead.empty()) {
    c->wait();
    for (auto& a : c->ahead) {
      const double* sv = c->ahead_host + a.off;
      for (size_t i = 0; i < a.nsv; ++i) ok &= std::isfinite(sv[i]) && sv[i] > 0.0;
      const int* sw = reinterpret_cast<const int*>(sv + a.nsv);
      for (size_t i = 0; i < a.nsweeps; ++i) ok &= sw[i] >= 0;
    }
  }
  c->ahead.clear();
  c->ahead_used = 0;
  return ok;
}

int svd_impl(bug_ctx* c, const bug_tensor& t, int nleft, const int* left, double cutoff, int nkeep,
             std::unique_ptr<bug_tensor>& U, std::unique_ptr<bug_tensor>& Vd,
             std::vector<double>& sv_sorted, std::vector<int>& sv_q, int& nkept, int want,
             std::unique_ptr<bug_tensor>* USo, std::unique_ptr<bug_tensor>* SVdo) {
  svd_many(c, {SvdReq{&t, nleft, left, cutoff, nkeep, want, &U, &Vd, &sv_sorted, &sv_q, &nkept, USo,
                      SVdo}});
  return BUG_OK;
}

// ── column-pivoted thin QR per charge sector of one leg ────────────────────────────────────

// Orthonormal basis of the span of `t`'s leg-`fl` columns (``_thin_qr``, dd_cbe.jl:184-259): per
// charge sector of leg `fl`, the sector's blocks stacked row-wise (blocks in ascending key order,
// rows = the other legs in C order, columns = leg `fl`), a column-pivoted Householder QR on
// device, and the leading Q columns whose |R_kk| exceeds `thr`. The new leg has arrow `ref_dir`;
// its charges keep the flux (negated when the arrow flips). nullptr when nothing is kept.
TensorPtr thin_qr_impl(bug_ctx* c, const bug_tensor& t, int fl, int ref_dir, double thr) {
  require(fl >= 0 && fl < t.rank && (ref_dir == 1 || ref_dir == -1), "thin_qr: bad leg or arrow");
  const Leg& F = t.legs[fl];
  std::map<int, std::vector<int>> groups;  // charge on fl -> block indices (ascending keys)
  for (int bi = 0; bi < int(t.blocks.size()); ++bi) groups[t.blocks[bi].key[fl]].push_back(bi);
  struct Sec {
    int charge;
    int64_t m = 0, n = 0, woff = 0, qoff = 0, roff = 0;
    std::vector<int64_t> row_of;  // row offset of each block of the sector
  };
  std::vector<Sec> secs;
  int64_t wtot = 0, rtot = 0;
  for (auto& kv : groups) {
    Sec sc;
    sc.charge = kv.first;
    sc.n = F.dim_of(kv.first);
    for (int bi : kv.second) {
      sc.row_of.push_back(sc.m);
      sc.m += t.blocks[bi].size / std::max<int64_t>(sc.n, 1);
    }
    if (sc.m == 0 || sc.n == 0) continue;
    require(sc.n <= 1024, "thin_qr: a sector wider than 1024 columns");
    const int64_t kq = std::min(sc.m, sc.n);
    sc.woff = wtot;
    wtot += sc.m * sc.n;
    sc.qoff = wtot;
    wtot += sc.m * kq;
    sc.roff = rtot;
    rtot += kq;
    secs.push_back(sc);
  }
  if (secs.empty()) return nullptr;
  double2* W = static_cast<double2*>(c->scratch(size_t(wtot) * sizeof(double2)));
  double* host = c->readback(size_t(rtot) + 1);
  // strides of an element of a block inside its sector matrix (column-major m x n): the other
  // legs in C order give the row, leg fl the column
  auto matrix_strides = [&](const Block& b, int64_t m, std::array<int64_t, BUG_MAX_RANK>& st) {
    int64_t acc = 1;
    for (int l = t.rank - 1; l >= 0; --l) {
      if (l == fl) continue;
      st[l] = acc;
      acc *= b.shape[l];
    }
    st[fl] = m;
  };
  std::vector<QrDesc> qd;
  std::vector<CopyDesc> packs;
  std::map<int, int> sec_of;
  for (size_t s2 = 0; s2 < secs.size(); ++s2) {
    Sec& sc = secs[s2];
    sec_of[sc.charge] = int(s2);
    QrDesc d{};
    d.work = W + sc.woff;
    d.Q = W + sc.qoff;
    d.rdiag_host = host + sc.roff;
    d.m = int(sc.m);
    d.n = int(sc.n);
    d.pack_begin = int(packs.size());
    const auto& bis = groups[sc.charge];
    for (size_t j = 0; j < bis.size(); ++j) {
      const Block& b = t.blocks[bis[j]];
      std::array<int64_t, BUG_MAX_RANK> ms{};
      matrix_strides(b, sc.m, ms);
      auto ss = c_strides(b.shape, t.rank);
      CopyDesc cd{};
      cd.src = t.data(bis[j]);
      cd.dst = d.work + sc.row_of[j];
      cd.n = b.size;
      cd.ndim = t.rank;
      cd.alpha = make_double2(1.0, 0.0);
      cd.wdim = -1;
      for (int l = 0; l < t.rank; ++l) {
        cd.dims[l] = b.shape[l];
        cd.sstr[l] = ss[l];
        cd.dstr[l] = ms[l];
      }
      packs.push_back(cd);
    }
    d.pack_end = int(packs.size());
    qd.push_back(d);
  }
  QrDesc* dq = c->push(qd);
  CopyDesc* dp = c->push(packs);
  // one warp per column of the widest sector (8 to 32 warps): a reflector reaches the remaining
  // columns side by side. Which warp takes a column changes no reduction order, so Q and R are the
  // same bits for any warp count.
  int64_t max_n = 0;
  for (auto& sc : secs) max_n = std::max<int64_t>(max_n, sc.n);
  const int qwarps = int(std::min<int64_t>(32, std::max<int64_t>(8, max_n)));
  const bugk::Blob blob = c->begin();
  bugk::launch_qr(blob, dq, int(qd.size()), dp, 32 * qwarps, c->stream);
  double qflops = 0.0;
  for (auto& sc : secs) qflops += 8.0 * 2.0 * double(sc.m) * double(sc.n) * double(std::min(sc.m, sc.n));
  c->launched(BUG_K_SVD, qflops, 0.0);
  c->wait();
  // ranks, the new leg, the output tensor
  Leg NL;
  NL.dir = ref_dir;
  std::vector<int> kept(secs.size(), 0);
  std::map<int, int> dims;
  for (size_t s2 = 0; s2 < secs.size(); ++s2) {
    const Sec& sc = secs[s2];
    const int64_t kq = std::min(sc.m, sc.n);
    int k = 0;
    for (int64_t j = 0; j < kq; ++j) k += host[sc.roff + j] > thr ? 1 : 0;
    kept[s2] = k;
    if (k > 0) dims[F.dir == ref_dir ? sc.charge : -sc.charge] = k;
  }
  if (dims.empty()) return nullptr;
  for (auto& kv : dims) {
    NL.q.push_back(kv.first);
    NL.d.push_back(kv.second);
  }
  std::vector<Leg> legs = t.legs;
  legs[fl] = NL;
  std::vector<Key> keys;
  for (auto& b : t.blocks) {
    const int s2 = sec_of.count(b.key[fl]) ? sec_of[b.key[fl]] : -1;
    if (s2 < 0 || kept[s2] == 0) continue;
    Key k = b.key;
    k[fl] = F.dir == ref_dir ? b.key[fl] : -b.key[fl];
    keys.push_back(k);
  }
  auto out = make_tensor(c, t.rank, legs, keys, false);
  std::vector<CopyDesc> copies;
  for (size_t s2 = 0; s2 < secs.size(); ++s2) {
    const Sec& sc = secs[s2];
    if (kept[s2] == 0) continue;
    const auto& bis = groups[sc.charge];
    for (size_t j = 0; j < bis.size(); ++j) {
      const Block& b = t.blocks[bis[j]];
      Key k = b.key;
      k[fl] = F.dir == ref_dir ? b.key[fl] : -b.key[fl];
      const int ob = out->find(k);
      const Block& o = out->blocks[ob];
      std::array<int64_t, BUG_MAX_RANK> ms{};
      matrix_strides(b, sc.m, ms);
      auto ds = c_strides(o.shape, t.rank);
      CopyDesc cd{};
      cd.src = W + sc.qoff + sc.row_of[j];
      cd.dst = out->mdata(ob);
      cd.n = o.size;
      cd.ndim = t.rank;
      cd.alpha = make_double2(1.0, 0.0);
      cd.wdim = -1;
      for (int l = 0; l < t.rank; ++l) {
        cd.dims[l] = o.shape[l];
        cd.sstr[l] = ms[l];
        cd.dstr[l] = ds[l];
      }
      copies.push_back(cd);
    }
  }
  run_copies(c, copies);
  return out;
}

// ── reductions and linear combinations ───────────────────────────────────────────────────────

constexpr int64_t kDotChunk = 16384;

// Run a descriptor list whose descriptors are grouped by output slot (seg[o]..seg[o+1]) through
// the one-launch reduction; returns nout complex sums (read back, synchronising).
// The dot launch itself: sums of every output (re, im) written to `q` (device or host-mapped).
void launch_dots(bug_ctx* c, const std::vector<DotDesc>& descs, const std::vector<int>& seg,
                 int nout, double2* q, double bytes_per_elem) {
  double2* partial = static_cast<double2*>(c->scratch(descs.size() * sizeof(double2)));
  DotDesc* dd = c->push(descs);
  int* dseg = c->push(seg);
  double dbytes = 0.0;
  for (auto& d : descs) dbytes += bytes_per_elem * double(d.n);
  bugk::Stage st{};
  st.kind = bugk::kStageDot;
  st.n = int(descs.size());
  st.total = nout;
  st.a = dd;
  st.b = dseg;
  st.p = partial;
  st.q = q;
  st.counter = c->counter();
  c->run_stage(st, BUG_K_DOT, 0.0, dbytes);
}

void run_dots(bug_ctx* c, const std::vector<DotDesc>& descs, const std::vector<int>& seg, int nout,
              double* out_re_im, double bytes_per_elem) {
  if (nout <= 0) return;
  if (descs.empty()) {
    for (int i = 0; i < 2 * nout; ++i) out_re_im[i] = 0.0;
    return;
  }
  double* host = c->readback(size_t(2 * nout));  // the kernel writes the sums here (host-mapped)
  launch_dots(c, descs, seg, nout, reinterpret_cast<double2*>(host), bytes_per_elem);
  c->wait();
  std::memcpy(out_re_im, host, size_t(nout) * sizeof(double2));
}

// descriptors of <a_o, b_o> for every pair o: matching blocks in chunks of kDotChunk
void dot_descs(const std::vector<std::pair<const bug_tensor*, const bug_tensor*>>& pairs,
               std::vector<DotDesc>& descs, std::vector<int>& seg) {
  seg.assign(pairs.size() + 1, 0);
  for (size_t o = 0; o < pairs.size(); ++o) {
    seg[o] = int(descs.size());
    const bug_tensor& a = *pairs[o].first;
    const bug_tensor& b = *pairs[o].second;
    for (int ai = 0; ai < int(a.blocks.size()); ++ai) {
      int bi = b.find(a.blocks[ai].key);
      if (bi < 0) continue;
      require(a.blocks[ai].size == b.blocks[bi].size, "inner: block shapes differ");
      for (int64_t s = 0; s < a.blocks[ai].size; s += kDotChunk) {
        DotDesc d{};
        d.a = a.data(ai) + s;
        d.b = b.data(bi) + s;
        d.n = std::min(kDotChunk, a.blocks[ai].size - s);
        d.out = int(o);
        descs.push_back(d);
      }
    }
  }
  seg[pairs.size()] = int(descs.size());
}

void dots(bug_ctx* c, const std::vector<std::pair<const bug_tensor*, const bug_tensor*>>& pairs,
          double* out_re_im) {
  std::vector<DotDesc> descs;
  std::vector<int> seg;
  dot_descs(pairs, descs, seg);
  run_dots(c, descs, seg, int(pairs.size()), out_re_im, 32.0);
}

void dots_device(bug_ctx* c, const std::vector<std::pair<const bug_tensor*, const bug_tensor*>>& pairs,
                 double2* q) {
  std::vector<DotDesc> descs;
  std::vector<int> seg;
  dot_descs(pairs, descs, seg);
  if (descs.empty()) {
    zero_fill(c, q, int64_t(pairs.size()));  // a (queued) stage: stays in order with the others
    return;
  }
  launch_dots(c, descs, seg, int(pairs.size()), q, 32.0);
}

// sum of |x|^2 over the blocks of `t` whose charge on `leg` is sector s, for every sector s of
// that leg (ascending), in one launch and one read-back.
static void sector_descs(const bug_tensor& t, int leg, std::vector<DotDesc>& descs,
                         std::vector<int>& seg) {
  const Leg& L = t.legs[leg];
  const int nout = int(L.q.size());
  std::vector<std::vector<DotDesc>> per(nout);
  for (int bi = 0; bi < int(t.blocks.size()); ++bi) {
    const int s = L.index_of(t.blocks[bi].key[leg]);
    for (int64_t o = 0; o < t.blocks[bi].size; o += kDotChunk) {
      DotDesc d{};
      d.a = t.data(bi) + o;
      d.b = t.data(bi) + o;
      d.n = std::min(kDotChunk, t.blocks[bi].size - o);
      d.out = s;
      per[s].push_back(d);
    }
  }
  descs.clear();
  seg.assign(nout + 1, 0);
  for (int s = 0; s < nout; ++s) {
    seg[s] = int(descs.size());
    descs.insert(descs.end(), per[s].begin(), per[s].end());
  }
  seg[nout] = int(descs.size());
}

std::vector<double> sector_norms2(bug_ctx* c, const bug_tensor& t, int leg) {
  const int nout = int(t.legs[leg].q.size());
  std::vector<DotDesc> descs;
  std::vector<int> seg;
  sector_descs(t, leg, descs, seg);
  std::vector<double> out(nout, 0.0);
  if (nout == 0) return out;
  std::vector<double> tmp(2 * size_t(nout));
  run_dots(c, descs, seg, nout, tmp.data(), 16.0);
  for (int s = 0; s < nout; ++s) out[s] = tmp[2 * s];
  return out;
}

// The same sums (re, im) written to device memory `q` (one slot per sector of `leg`), no read-back.
void sector_norms2_device(bug_ctx* c, const bug_tensor& t, int leg, double2* q) {
  const int nout = int(t.legs[leg].q.size());
  if (nout == 0) return;
  std::vector<DotDesc> descs;
  std::vector<int> seg;
  sector_descs(t, leg, descs, seg);
  if (descs.empty()) {
    zero_fill(c, q, int64_t(nout));
    return;
  }
  launch_dots(c, descs, seg, nout, q, 16.0);
}

std::unique_ptr<bug_tensor> lincomb_impl(bug_ctx* c, int n, const double* coef,
                                         const bug_tensor* const* ts, const double* const* cref,
                                         const int* cmode) {
  require(n >= 1, "lincomb needs at least one tensor");
  const int rank = ts[0]->rank;
  std::vector<Leg> legs = ts[0]->legs;
  for (int i = 1; i < n; ++i) {
    require(ts[i]->rank == rank, "lincomb: ranks differ");
    for (int l = 0; l < rank; ++l) legs[l] = merged(legs[l], ts[i]->legs[l]);
  }
  std::vector<Key> keys;
  for (int i = 0; i < n; ++i)
    for (auto& b : ts[i]->blocks) keys.push_back(b.key);
  auto out = make_tensor(c, rank, legs, keys, false);
  std::vector<LinOut> outs;
  std::vector<LinSrc> srcs;
  int64_t total = 0;
  for (int j = 0; j < int(out->blocks.size()); ++j) {
    LinOut o{};
    o.dst = out->mdata(j);
    o.n = out->blocks[j].size;
    o.prefix = total;
    total += o.n;
    o.src_begin = int(srcs.size());
    for (int i = 0; i < n; ++i) {
      int b = ts[i]->find(out->blocks[j].key);
      if (b < 0) continue;
      LinSrc ls{};
      ls.src = ts[i]->data(b);
      ls.coef = make_double2(coef[2 * i], coef[2 * i + 1]);
      if (cmode && cmode[i]) {
        ls.cref = cref[i];
        ls.cmode = cmode[i];
      }
      srcs.push_back(ls);
    }
    o.src_end = int(srcs.size());
    outs.push_back(o);
  }
  if (!outs.empty()) {
    LinOut* dout = c->push(outs);
    LinSrc* dsrc = c->push(srcs);
    double lbytes = 0.0;
    for (auto& o : outs) lbytes += 16.0 * double(o.n) * double(o.src_end - o.src_begin + 1);
    bugk::Stage st{};
    st.kind = bugk::kStageLincomb;
    st.n = int(outs.size());
    st.total = total;
    st.a = dout;
    st.b = dsrc;
    c->run_stage(st, BUG_K_LINCOMB, 0.0, lbytes);
  }
  return out;
}

}  // namespace bugi

namespace bugi {
int guard_body(const std::function<void()>& f);

// Runs one C-ABI call. When it returns, the stages the call queued on its context are launched
// (or dropped if the call failed) and the call's scratch is released, so every call leaves all of
// its work enqueued on the context stream, in order.
int guard(const std::function<void()>& f) {
  int rc = guard_body(f);
  if (bug_ctx* c = g_active_ctx) {
    if (rc == BUG_OK) rc = guard_body([c] { c->drain(); });
    if (rc != BUG_OK) c->discard_queue();
    for (void* p : c->deferred) c->dev_free(p);
    c->deferred.clear();
    c->ahead.clear();  // SVDs taken ahead and left unchecked by a failed call
    c->ahead_used = 0;
  }
  g_active_ctx = nullptr;
  return rc;
}

int guard_body(const std::function<void()>& f) {
  try {
    f();
    return BUG_OK;
  } catch (const BugError& e) {
    g_err = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_err = "host allocation failed";
    return BUG_ENOMEM;
  } catch (const std::exception& e) {
    g_err = e.what();
    return BUG_EINVAL;
  }
}
}  // namespace bugi


namespace bugi {

TensorPtr scale_leg_impl(bug_ctx* c, const bug_tensor& tt, int leg, const double* w) {
  const bug_tensor* t = &tt;
  TensorPtr result;

    require(c && t && leg >= 0 && leg < t->rank, "bad argument");
    const Leg& L = t->legs[leg];
    std::vector<double> wv(w, w + L.total());
    std::vector<int64_t> woff(L.q.size());
    int64_t acc = 0;
    for (size_t s = 0; s < L.q.size(); ++s) {
      woff[s] = acc;
      acc += L.d[s];
    }
    std::vector<Key> keys;
    for (auto& b : t->blocks) keys.push_back(b.key);
    auto o = make_tensor(c, t->rank, t->legs, keys, false);
    double* dw = c->push(wv);
    std::vector<ScaleDesc> descs;
    int64_t total = 0;
    for (int bi = 0; bi < int(t->blocks.size()); ++bi) {
      const Block& b = t->blocks[bi];
      auto st = c_strides(b.shape, t->rank);
      ScaleDesc d{};
      d.src = t->data(bi);
      d.dst = o->mdata(bi);
      d.n = b.size;
      d.prefix = total;
      total += b.size;
      d.leg_stride = st[leg];
      d.leg_dim = b.shape[leg];
      d.w = dw + woff[L.index_of(b.key[leg])];
      descs.push_back(d);
    }
    if (!descs.empty()) {
      ScaleDesc* dd = c->push(descs);
      bugk::Stage st{};
      st.kind = bugk::kStageScale;
      st.n = int(descs.size());
      st.total = total;
      st.a = dd;
      c->run_stage(st, BUG_K_SCALE, 0.0, 32.0 * double(total));
    }
    result = std::move(o);
    return result;
}

TensorPtr conj_impl(bug_ctx* c, const bug_tensor& tt) {
  const bug_tensor* t = &tt;
  TensorPtr result;

    std::vector<Leg> legs;
    for (auto& l : t->legs) legs.push_back(flipped(l));
    std::vector<Key> keys;
    for (auto& b : t->blocks) keys.push_back(b.key);
    auto o = make_tensor(c, t->rank, legs, keys, false);
    std::vector<CopyDesc> d;
    if (t->nelem > 0)
      d.push_back(plain_copy(t->buf->ptr, o->buf->ptr, t->nelem, true, make_double2(1.0, 0.0), false));
    run_copies(c, d);
    result = std::move(o);
    return result;
}

TensorPtr flip_leg_impl(bug_ctx* c, const bug_tensor& tt, int leg) {
  const bug_tensor* t = &tt;
  TensorPtr result;

    require(leg >= 0 && leg < t->rank, "bad leg");
    std::vector<Leg> legs = t->legs;
    Leg L;
    L.dir = -t->legs[leg].dir;
    for (int s = int(t->legs[leg].q.size()) - 1; s >= 0; --s) {
      L.q.push_back(-t->legs[leg].q[s]);
      L.d.push_back(t->legs[leg].d[s]);
    }
    legs[leg] = L;
    std::vector<Key> keys;
    for (auto& b : t->blocks) {
      Key k = b.key;
      k[leg] = -k[leg];
      keys.push_back(k);
    }
    auto o = make_tensor(c, t->rank, legs, keys, false);
    std::vector<CopyDesc> d;
    for (int bi = 0; bi < int(t->blocks.size()); ++bi) {
      Key k = t->blocks[bi].key;
      k[leg] = -k[leg];
      int ob = o->find(k);
      d.push_back(plain_copy(t->data(bi), o->mdata(ob), t->blocks[bi].size, false,
                             make_double2(1.0, 0.0), false));
    }
    run_copies(c, d);
    result = std::move(o);
    return result;
}

TensorPtr oplus_impl(bug_ctx* c, int n, const bug_tensor* const* ts, int leg) {
  TensorPtr result;

    require(n >= 1, "oplus needs at least one tensor");
    const int rank = ts[0]->rank;
    require(leg >= 0 && leg < rank, "bad leg");
    std::map<int, int> dims;
    std::vector<Leg> legs = ts[0]->legs;
    for (int i = 0; i < n; ++i) {
      require(ts[i]->rank == rank, "oplus: ranks differ");
      require(ts[i]->legs[leg].dir == ts[0]->legs[leg].dir, "oplus: arrows differ");
      for (size_t s = 0; s < ts[i]->legs[leg].q.size(); ++s) dims[ts[i]->legs[leg].q[s]] += ts[i]->legs[leg].d[s];
      if (i > 0)
        for (int l = 0; l < rank; ++l)
          if (l != leg) legs[l] = merged(legs[l], ts[i]->legs[l]);
    }
    Leg L;
    L.dir = ts[0]->legs[leg].dir;
    for (auto& kv : dims) {
      L.q.push_back(kv.first);
      L.d.push_back(kv.second);
    }
    legs[leg] = L;
    std::vector<Key> keys;
    for (int i = 0; i < n; ++i)
      for (auto& b : ts[i]->blocks) keys.push_back(b.key);
    auto o = make_tensor(c, rank, legs, keys, true);
    std::map<int, int> offs;
    std::vector<CopyDesc> d;
    for (int i = 0; i < n; ++i) {
      for (int bi = 0; bi < int(ts[i]->blocks.size()); ++bi) {
        const Block& b = ts[i]->blocks[bi];
        int ob = o->find(b.key);
        const Block& obb = o->blocks[ob];
        auto ss = c_strides(b.shape, rank);
        auto ds = c_strides(obb.shape, rank);
        CopyDesc cd{};
        cd.src = ts[i]->data(bi);
        cd.dst = o->mdata(ob) + int64_t(offs[b.key[leg]]) * ds[leg];
        cd.n = b.size;
        cd.ndim = rank;
        for (int l = 0; l < rank; ++l) {
          cd.dims[l] = b.shape[l];
          cd.sstr[l] = ss[l];
          cd.dstr[l] = ds[l];
        }
        cd.alpha = make_double2(1.0, 0.0);
        d.push_back(cd);
      }
      for (size_t s = 0; s < ts[i]->legs[leg].q.size(); ++s) offs[ts[i]->legs[leg].q[s]] += ts[i]->legs[leg].d[s];
    }
    run_copies(c, d);
    result = std::move(o);
    return result;
}

TensorPtr trim_impl(bug_ctx* c, const bug_tensor& tt, int leg, const int* counts) {
  const bug_tensor* t = &tt;
  TensorPtr result;

    require(leg >= 0 && leg < t->rank, "bad leg");
    const Leg& L0 = t->legs[leg];
    Leg L;
    L.dir = L0.dir;
    std::map<int, int> keep;
    for (size_t s = 0; s < L0.q.size(); ++s) {
      int k = std::min(std::max(counts[s], 0), L0.d[s]);
      if (k > 0) {
        L.q.push_back(L0.q[s]);
        L.d.push_back(k);
        keep[L0.q[s]] = k;
      }
    }
    if (L.q.empty()) return nullptr;
    std::vector<Leg> legs = t->legs;
    legs[leg] = L;
    std::vector<Key> keys;
    for (auto& b : t->blocks)
      if (keep.count(b.key[leg])) keys.push_back(b.key);
    auto o = make_tensor(c, t->rank, legs, keys, false);
    std::vector<CopyDesc> d;
    for (int bi = 0; bi < int(t->blocks.size()); ++bi) {
      const Block& b = t->blocks[bi];
      if (!keep.count(b.key[leg])) continue;
      int ob = o->find(b.key);
      const Block& obb = o->blocks[ob];
      auto ss = c_strides(b.shape, t->rank);
      auto ds = c_strides(obb.shape, t->rank);
      CopyDesc cd{};
      cd.src = t->data(bi);
      cd.dst = o->mdata(ob);
      cd.n = obb.size;
      cd.ndim = t->rank;
      for (int l = 0; l < t->rank; ++l) {
        cd.dims[l] = obb.shape[l];
        cd.sstr[l] = ss[l];
        cd.dstr[l] = ds[l];
      }
      cd.alpha = make_double2(1.0, 0.0);
      d.push_back(cd);
    }
    run_copies(c, d);
    result = std::move(o);
    return result;
}

TensorPtr upload_impl(bug_ctx* c, int rank, const std::vector<Leg>& legs, const std::vector<Key>& keys,
                      const double* data) {
  auto t = make_tensor(c, rank, legs, keys, false);
  require(int(t->blocks.size()) == int(keys.size()), "duplicate block keys");
  if (t->nelem > 0) {
    // through the pinned staging ring: no wait, and `data` may be reused at once. The payload is
    // a new allocation that no queued stage reads, so the copy may precede them in the stream.
    const size_t bytes = size_t(t->nelem) * sizeof(double2);
    void* h = c->stage(bytes);
    std::memcpy(h, data, bytes);
    BUG_CUDA(cudaMemcpyAsync(t->buf->ptr, h, bytes, cudaMemcpyHostToDevice, c->stream));
    c->stage_done();
  }
  return t;
}

}  // namespace bugi

using namespace bugi;

// ── C-ABI ────────────────────────────────────────────────────────────────────────────────────

extern "C" {

const char* bug_last_error(void) { return g_err.c_str(); }
const char* bug_version(void) { return "bug_b200 0.1 (sm_100a, complex FP64)"; }

int bug_ctx_create(int device, bug_ctx** out) {
  return guard([&] {
    require(out != nullptr, "null output");
    int count = 0;
    BUG_CUDA(cudaGetDeviceCount(&count));
    require(device >= 0 && device < count, "no such CUDA device");
    BUG_CUDA(cudaSetDevice(device));
    auto c = std::make_unique<bug_ctx>();
    ctx_init(c.get(), device);
    *out = c.release();
  });
}

int bug_ctx_destroy(bug_ctx* c) {
  return guard([&] {
    if (!c) return;
    if (c->child) {
      ctx_release(c->child);
      delete c->child;
      c->child = nullptr;
    }
    ctx_release(c);
    delete c;
  });
}
}  // extern "C"

namespace bugi {

void ctx_init(bug_ctx* c, int device) {
  c->device = device;
  BUG_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  c->list_cluster = bugk::stage_list_cluster();
  // BUG_STAGE_LISTS=0 launches every stage on its own (same results; for comparisons)
  const char* lists = std::getenv("BUG_STAGE_LISTS");
  c->queue_enabled = !(lists && std::string(lists) == "0");
  if (const char* qm = std::getenv("BUG_STAGE_LIST_MAX")) {
    const long v = std::strtol(qm, nullptr, 10);
    if (v >= 1 && v <= 4096) c->queue_max_stages = size_t(v);
  }
  if (const char* qr = std::getenv("BUG_STAGE_LIST_ROUNDS")) {
    const long v = std::strtol(qr, nullptr, 10);
    if (v >= 1 && v <= 64) c->queue_rounds = int(v);
  }
  for (int i = 0; i < bug_ctx::kSlots; ++i)
    BUG_CUDA(cudaEventCreateWithFlags(&c->stage_ev[i], cudaEventDisableTiming));
  cudaMemPool_t pool;
  BUG_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t thr = UINT64_MAX;
  BUG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
}

// Everything a context holds, after its stream has finished (the object itself stays).
void ctx_release(bug_ctx* c) {
  cudaStreamSynchronize(c->stream);
  for (int i = 0; i < bug_ctx::kSlots; ++i) {
    if (c->stage_ptr[i]) cudaFreeHost(c->stage_ptr[i]);
    cudaEventDestroy(c->stage_ev[i]);
  }
  if (c->pinned_out) cudaFreeHost(c->pinned_out);
  if (c->ahead_host) cudaFreeHost(c->ahead_host);
  if (c->tc_err_host) cudaFreeHost(c->tc_err_host);
  if (c->arena) cudaFreeAsync(c->arena, c->stream);
  c->release_cached();
  cudaStreamSynchronize(c->stream);
  if (c->dot_counter) cudaFree(c->dot_counter);
  if (c->sync_ev) cudaEventDestroy(c->sync_ev);
  if (c->fork_ev) cudaEventDestroy(c->fork_ev);
  if (c->owns_stream) cudaStreamDestroy(c->stream);
}

// ── concurrent halves: the second stream ─────────────────────────────────────────────────────

bug_ctx* fork_begin(bug_ctx* c) {
  require(!c->alloc_owner && !c->forking, "a fork inside a fork");
  require(!c->combiner, "parallel half-sweeps need a context with a stream of its own, not a "
                        "combining batch");
  if (!c->child) {
    auto ch = std::make_unique<bug_ctx>();
    ctx_init(ch.get(), c->device);
    ch->alloc_owner = c;
    c->child = ch.release();
  }
  bug_ctx* ch = c->child;
  ch->queue_enabled = c->queue_enabled;
  ch->queue_max_stages = c->queue_max_stages;
  ch->queue_rounds = c->queue_rounds;
  ch->mixed_min_dim = c->mixed_min_dim;
  ch->ahead.clear();  // anything a failed half left unchecked
  ch->ahead_used = 0;
  if (!c->fork_ev) BUG_CUDA(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
  if (!ch->fork_ev) BUG_CUDA(cudaEventCreateWithFlags(&ch->fork_ev, cudaEventDisableTiming));
  c->drain();  // every queued stage of the parent is enqueued before the fork event
  BUG_CUDA(cudaEventRecord(c->fork_ev, c->stream));
  BUG_CUDA(cudaStreamWaitEvent(ch->stream, c->fork_ev, 0));
  c->forking = true;  // set before the child's thread starts
  return ch;
}

// On the child's thread when its half is done (or failed): its queue enqueued (or dropped) and the
// join event recorded after it.
void fork_child_done(bug_ctx* ch, bool ok) {
  if (ok) ch->drain();
  else ch->discard_queue();
  BUG_CUDA(cudaEventRecord(ch->fork_ev, ch->stream));
}

// After the child's thread has been joined: the parent stream waits for the child's work, the
// releases parked during the fork and the child's scratch go back, and the child's accounting is
// folded into the parent's.
void fork_end(bug_ctx* c) {
  bug_ctx* ch = c->child;
  cudaError_t e = cudaStreamWaitEvent(c->stream, ch->fork_ev, 0);
  c->forking = false;
  std::vector<void*> parked;
  parked.swap(c->fork_frees);
  for (void* p : parked) c->dev_free(p);
  for (void* p : ch->deferred) ch->dev_free(p);
  ch->deferred.clear();
  c->launches += ch->launches;
  c->syncs += ch->syncs;
  c->sync_wait_s += ch->sync_wait_s;
  c->launch_s += ch->launch_s;
  c->alloc_s += ch->alloc_s;
  c->list_launches += ch->list_launches;
  c->queued_stages += ch->queued_stages;
  for (int f = 0; f < BUG_K_NFAMILIES; ++f) {
    c->k_launches[f] += ch->k_launches[f];
    c->k_flops[f] += ch->k_flops[f];
    c->k_bytes[f] += ch->k_bytes[f];
  }
  ch->launches = ch->syncs = ch->list_launches = ch->queued_stages = 0;
  ch->sync_wait_s = ch->launch_s = ch->alloc_s = 0.0;
  for (int f = 0; f < BUG_K_NFAMILIES; ++f) {
    ch->k_launches[f] = 0;
    ch->k_flops[f] = ch->k_bytes[f] = 0.0;
  }
  BUG_CUDA(e);
}

}  // namespace bugi

extern "C" {

int bug_ctx_synchronize(bug_ctx* c) {
  return guard([&] {
    require(c != nullptr, "null context");
    c->sync_stream();
    c->check_tc_error();
  });
}

int64_t bug_ctx_launches(const bug_ctx* c) { return c ? c->launches : 0; }

void* bug_ctx_stream(bug_ctx* c) { return c ? (void*)c->stream : nullptr; }

int bug_ctx_set_mixed(bug_ctx* c, int min_dim) {
  return guard([&] {
    require(c != nullptr, "null context");
    c->mixed_min_dim = min_dim > 0 ? min_dim : 0;
  });
}

int bug_ctx_set_profiling(bug_ctx* c, int on) {
  return guard([&] {
    require(c != nullptr, "null context");
    c->harvest();
    c->profiling = on != 0;
  });
}

int bug_ctx_kernel_stats(bug_ctx* c, int family, int64_t* launches, double* flops, double* bytes,
                         double* device_ms) {
  return guard([&] {
    require(c && family >= 0 && family < BUG_K_NFAMILIES, "bad argument");
    c->harvest();
    *launches = c->k_launches[family];
    *flops = c->k_flops[family];
    *bytes = c->k_bytes[family];
    *device_ms = c->k_ms[family];
  });
}

int bug_ctx_reset_stats(bug_ctx* c) {
  return guard([&] {
    require(c != nullptr, "null context");
    c->harvest();
    for (int f = 0; f < BUG_K_NFAMILIES; ++f) {
      c->k_launches[f] = 0;
      c->k_flops[f] = c->k_bytes[f] = c->k_ms[f] = 0.0;
    }
    c->syncs = 0;
    c->sync_wait_s = c->launch_s = c->alloc_s = 0.0;
  });
}

int bug_ctx_host_stats(bug_ctx* c, int64_t* syncs, double* wait_s, double* launch_s,
                       double* alloc_s) {
  return guard([&] {
    require(c && syncs && wait_s && launch_s && alloc_s, "bad argument");
    *syncs = c->syncs;
    *wait_s = c->sync_wait_s;
    *launch_s = c->launch_s;
    *alloc_s = c->alloc_s;
  });
}
int64_t bug_ctx_bytes_in_use(const bug_ctx* c) { return c ? c->bytes.load() : 0; }

int bug_tensor_create(bug_ctx* c, int rank, const int* dirs, const int* nsec, const int* charges,
                      const int* dims, int nblocks, const int* keys, bug_tensor** out) {
  return guard([&] {
    require(c && out, "null argument");
    require(rank >= 0 && rank <= BUG_MAX_RANK, "rank out of range");
    std::vector<Leg> legs(rank);
    int p = 0;
    for (int l = 0; l < rank; ++l) {
      require(dirs[l] == 1 || dirs[l] == -1, "leg arrow must be +1 or -1");
      legs[l].dir = dirs[l];
      for (int s = 0; s < nsec[l]; ++s, ++p) {
        require(dims[p] > 0, "sector dimension must be positive");
        require(legs[l].q.empty() || charges[p] > legs[l].q.back(), "sector charges must ascend");
        legs[l].q.push_back(charges[p]);
        legs[l].d.push_back(dims[p]);
      }
    }
    std::vector<Key> ks(nblocks);
    for (int b = 0; b < nblocks; ++b) {
      Key k{};
      for (int l = 0; l < rank; ++l) k[l] = keys[b * rank + l];
      ks[b] = k;
    }
    auto t = make_tensor(c, rank, legs, ks, true);
    require(int(t->blocks.size()) == nblocks, "duplicate block keys");
    *out = t.release();
  });
}

int bug_tensor_upload(bug_ctx* c, bug_tensor* t, const double* host, int64_t nelem) {
  return guard([&] {
    require(c && t, "null argument");
    require(nelem == t->nelem, "upload: element count mismatch");
    if (nelem > 0)
      BUG_CUDA(cudaMemcpyAsync(t->buf->ptr, host, size_t(nelem) * sizeof(double2),
                               cudaMemcpyHostToDevice, c->stream));
    c->sync_stream();
  });
}

int bug_tensor_download(bug_ctx* c, const bug_tensor* t, double* host, int64_t nelem) {
  return guard([&] {
    require(c && t, "null argument");
    require(nelem == t->nelem, "download: element count mismatch");
    if (nelem > 0)
      BUG_CUDA(cudaMemcpyAsync(host, t->buf->ptr, size_t(nelem) * sizeof(double2),
                               cudaMemcpyDeviceToHost, c->stream));
    c->sync_stream();
  });
}

int bug_tensor_free(bug_ctx* /*ctx: the ABI names the owner; the handle frees itself*/, bug_tensor* t) {
  return guard([&] { delete t; });
}

int bug_tensor_shape(const bug_tensor* t, int* rank, int* nblocks, int64_t* nelem,
                     int* total_sectors) {
  return guard([&] {
    require(t != nullptr, "null tensor");
    *rank = t->rank;
    *nblocks = int(t->blocks.size());
    *nelem = t->nelem;
    int s = 0;
    for (auto& l : t->legs) s += int(l.q.size());
    *total_sectors = s;
  });
}

int bug_tensor_meta(const bug_tensor* t, int* dirs, int* nsec, int* charges, int* dims, int* keys) {
  return guard([&] {
    int p = 0;
    for (int l = 0; l < t->rank; ++l) {
      dirs[l] = t->legs[l].dir;
      nsec[l] = int(t->legs[l].q.size());
      for (size_t s = 0; s < t->legs[l].q.size(); ++s, ++p) {
        charges[p] = t->legs[l].q[s];
        dims[p] = t->legs[l].d[s];
      }
    }
    for (size_t b = 0; b < t->blocks.size(); ++b)
      for (int l = 0; l < t->rank; ++l) keys[b * t->rank + l] = t->blocks[b].key[l];
  });
}

// The flat host layout of many tensors (include/bug_b200.h): per tensor, at meta + meta_off[i],
// rank r, r arrows, r sector counts, the charges and the dims of all sectors leg by leg, the block
// count nb and nb x r block keys; its payload at payload_off[i] complex values into `payload`.
int bug_tensors_from_host(bug_ctx* c, int n, const int* meta, const int64_t* meta_off,
                          const double* payload, const int64_t* payload_off, bug_tensor** out) {
  return guard([&] {
    require(c && n >= 0, "bad argument");
    require(n == 0 || (meta && meta_off && payload && payload_off && out), "null argument");
    std::vector<TensorPtr> made;
    for (int i = 0; i < n; ++i) {
      const int* m = meta + meta_off[i];
      const int rank = m[0];
      require(rank >= 0 && rank <= BUG_MAX_RANK, "rank out of range");
      const int* dirs = m + 1;
      const int* nsec = m + 1 + rank;
      int ns = 0;
      for (int l = 0; l < rank; ++l) {
        require(nsec[l] >= 0, "negative sector count");
        ns += nsec[l];
      }
      const int* ch = m + 1 + 2 * rank;
      const int* dm = ch + ns;
      std::vector<Leg> legs(rank);
      for (int l = 0, p = 0; l < rank; ++l) {
        require(dirs[l] == 1 || dirs[l] == -1, "leg arrow must be +1 or -1");
        legs[l].dir = dirs[l];
        for (int q = 0; q < nsec[l]; ++q, ++p) {
          require(dm[p] > 0, "sector dimension must be positive");
          require(legs[l].q.empty() || ch[p] > legs[l].q.back(), "sector charges must ascend");
          legs[l].q.push_back(ch[p]);
          legs[l].d.push_back(dm[p]);
        }
      }
      const int nb = dm[ns];
      require(nb >= 0, "negative block count");
      const int* keys = dm + ns + 1;
      std::vector<Key> ks(nb);
      for (int b = 0; b < nb; ++b) {
        Key k{};
        for (int l = 0; l < rank; ++l) k[l] = keys[b * rank + l];
        ks[b] = k;
      }
      made.push_back(upload_impl(c, rank, legs, ks, payload + 2 * payload_off[i]));
    }
    for (int i = 0; i < n; ++i) out[i] = made[size_t(i)].release();
  });
}

int bug_tensors_layout(int n, const bug_tensor* const* t, int64_t* meta_len, int64_t* nelem) {
  return guard([&] {
    require(n >= 0 && (n == 0 || (t && meta_len && nelem)), "bad argument");
    for (int i = 0; i < n; ++i) {
      require(t[i] != nullptr, "null tensor");
      int64_t ns = 0;
      for (auto& l : t[i]->legs) ns += int64_t(l.q.size());
      meta_len[i] = 2 + 2 * int64_t(t[i]->rank) + 2 * ns + int64_t(t[i]->blocks.size()) * t[i]->rank;
      nelem[i] = t[i]->nelem;
    }
  });
}

int bug_tensors_to_host(bug_ctx* c, int n, const bug_tensor* const* t, int* meta,
                        const int64_t* meta_off, double* payload, const int64_t* payload_off) {
  return guard([&] {
    require(c && n >= 0, "bad argument");
    require(n == 0 || (t && meta && meta_off && payload && payload_off), "null argument");
    int64_t total = 0;
    for (int i = 0; i < n; ++i) {
      require(t[i] != nullptr, "null tensor");
      total += t[i]->nelem;
    }
    double* pin = c->readback(size_t(2 * std::max<int64_t>(total, 1)));
    c->drain();
    int64_t acc = 0;
    for (int i = 0; i < n; ++i) {
      if (t[i]->nelem > 0)
        BUG_CUDA(cudaMemcpyAsync(pin + 2 * acc, t[i]->buf->ptr, size_t(t[i]->nelem) * sizeof(double2),
                                 cudaMemcpyDeviceToHost, c->stream));
      acc += t[i]->nelem;
    }
    for (int i = 0; i < n; ++i) {  // metadata from the host-side block tables meanwhile
      const bug_tensor& x = *t[i];
      int* m = meta + meta_off[i];
      int p = 0;
      m[p++] = x.rank;
      for (int l = 0; l < x.rank; ++l) m[p++] = x.legs[l].dir;
      for (int l = 0; l < x.rank; ++l) m[p++] = int(x.legs[l].q.size());
      for (int l = 0; l < x.rank; ++l)
        for (int q : x.legs[l].q) m[p++] = q;
      for (int l = 0; l < x.rank; ++l)
        for (int d : x.legs[l].d) m[p++] = d;
      m[p++] = int(x.blocks.size());
      for (auto& b : x.blocks)
        for (int l = 0; l < x.rank; ++l) m[p++] = b.key[l];
    }
    c->wait();
    acc = 0;
    for (int i = 0; i < n; ++i) {
      if (t[i]->nelem > 0)
        std::memcpy(payload + 2 * payload_off[i], pin + 2 * acc, size_t(t[i]->nelem) * sizeof(double2));
      acc += t[i]->nelem;
    }
  });
}

int bug_contract(bug_ctx* c, const bug_tensor* a, int n, const int* ia, const bug_tensor* b,
                 const int* ib, int conja, int conjb, bug_tensor** out) {
  return guard([&] {
    require(c && a && b && out, "null argument");
    *out = contract_impl(c, *a, n, ia, *b, ib, conja != 0, conjb != 0).release();
  });
}

int bug_thin_qr(bug_ctx* c, const bug_tensor* t, int leg, int ref_dir, double thr, bug_tensor** out) {
  return guard([&] {
    require(c && t && out, "null argument");
    *out = thin_qr_impl(c, *t, leg, ref_dir, thr).release();
  });
}

int bug_svd(bug_ctx* c, const bug_tensor* t, int nleft, const int* left, double cutoff, int nkeep,
            bug_tensor** U, bug_tensor** Vd, double* sv_all, int* sv_charge, int cap, int* nsv_all,
            int* nkept) {
  return guard([&] {
    require(c && t && U && Vd, "null argument");
    std::unique_ptr<bug_tensor> u, v;
    std::vector<double> sv;
    std::vector<int> q;
    int nk = 0;
    svd_impl(c, *t, nleft, left, cutoff, nkeep, u, v, sv, q, nk, 3, nullptr, nullptr);
    int ncopy = std::min<int>(cap, int(sv.size()));
    for (int i = 0; i < ncopy; ++i) {
      sv_all[i] = sv[i];
      sv_charge[i] = q[i];
    }
    *nsv_all = int(sv.size());
    *nkept = nk;
    *U = u.release();
    *Vd = v.release();
  });
}


int bug_norm2(bug_ctx* c, const bug_tensor* t, double* out) {
  return guard([&] {
    double r[2];
    dots(c, {{t, t}}, r);
    *out = r[0];
  });
}

int bug_inner(bug_ctx* c, const bug_tensor* a, const bug_tensor* b, double* out) {
  return guard([&] { dots(c, {{a, b}}, out); });
}

int bug_inner_many(bug_ctx* c, int n, const bug_tensor* const* v, const bug_tensor* w,
                   double* out) {
  return guard([&] {
    std::vector<std::pair<const bug_tensor*, const bug_tensor*>> ps;
    for (int i = 0; i < n; ++i) ps.push_back({v[i], w});
    if (n > 0) dots(c, ps, out);
  });
}

int bug_lincomb(bug_ctx* c, int n, const double* coef, const bug_tensor* const* t,
                bug_tensor** out) {
  return guard([&] { *out = lincomb_impl(c, n, coef, t).release(); });
}

int bug_permute(bug_ctx* c, const bug_tensor* t, const int* perm, bug_tensor** out) {
  return guard([&] { *out = permute_impl(c, *t, perm).release(); });
}






int bug_scale_leg(bug_ctx* c, const bug_tensor* t, int leg, const double* w, bug_tensor** out) {
  return guard([&] {
    require(c && t && out, "null argument");
    *out = scale_leg_impl(c, *t, leg, w).release();
  });
}

int bug_conj(bug_ctx* c, const bug_tensor* t, bug_tensor** out) {
  return guard([&] { *out = conj_impl(c, *t).release(); });
}

int bug_flip_leg(bug_ctx* c, const bug_tensor* t, int leg, bug_tensor** out) {
  return guard([&] { *out = flip_leg_impl(c, *t, leg).release(); });
}

int bug_oplus(bug_ctx* c, int n, const bug_tensor* const* ts, int leg, bug_tensor** out) {
  return guard([&] { *out = oplus_impl(c, n, ts, leg).release(); });
}

int bug_trim(bug_ctx* c, const bug_tensor* t, int leg, const int* counts, bug_tensor** out) {
  return guard([&] { *out = trim_impl(c, *t, leg, counts).release(); });
}

}  // extern "C"
