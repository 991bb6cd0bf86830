// Host-side set-up of a drape instance (see setup.h).
#include "setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <condition_variable>
#include <memory>
#include <mutex>
#include <numeric>
#include <unordered_map>

namespace vistio {
namespace {

// Symbolic factors (numeric == false) keyed by the exact adjacency and
// dissection order they were computed from. Everything factorize_csr derives
// after the dissection (postorder, supernodes, row structures, schedules)
// depends on nothing else, so a hit returns the Factor a fresh analysis would
// build: garments that share a mesh pay for the analysis once. Entries hold
// their key arrays and are compared in full; the cache is bounded in bytes and
// evicts the least recently used entry first. An analysis in progress is
// listed as pending: a thread that needs the same one waits for it instead of
// repeating it (set-up threads tend to start on the same mesh together).
struct SymEntry {
  std::vector<uint32_t> ptr, adj, order;
  std::shared_ptr<const Factor> factor;
  uint64_t bytes = 0, used = 0;
  bool same(const std::vector<uint32_t>& p, const std::vector<uint32_t>& a, const std::vector<uint32_t>& o) const {
    return order == o && ptr == p && adj == a;
  }
};
struct SymPending {
  uint64_t key = 0;
  SymEntry entry;     // the key arrays; `factor` is set when done
  bool done = false;  // done without a factor: the analysis was abandoned
};
struct SymCache {
  std::mutex mu;
  std::condition_variable cv;
  std::unordered_multimap<uint64_t, SymEntry> map;
  std::vector<std::shared_ptr<SymPending>> pending;
  uint64_t bytes = 0, clock = 0, hits = 0, misses = 0, limit = uint64_t(1) << 30;
};
SymCache& sym_cache() {
  static SymCache c;
  return c;
}

uint64_t fnv_words(uint64_t h, const std::vector<uint32_t>& v) {
  for (uint32_t w : v)
    for (int b = 0; b < 4; ++b) { h ^= (w >> (8 * b)) & 0xffu; h *= 1099511628211ull; }
  return h;
}

template <class T> uint64_t vec_bytes(const std::vector<T>& v) { return v.size() * sizeof(T); }

uint64_t factor_bytes(const Factor& f) {
  return vec_bytes(f.perm) + vec_bytes(f.iperm) + vec_bytes(f.sn) + vec_bytes(f.rows) + vec_bytes(f.row_sn) +
         vec_bytes(f.level_ptr) + vec_bytes(f.level_rows) + vec_bytes(f.level_sn_ptr) + vec_bytes(f.level_sn) +
         vec_bytes(f.sub_first) + vec_bytes(f.sub_last) + vec_bytes(f.fwd_ptr) + vec_bytes(f.fwd_sn) +
         vec_bytes(f.fwd_pos);
}

struct F3 {
  float x, y, z;
};
inline F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3 add(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline F3 mul(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline F3 dvs(F3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float len(F3 a) { return std::sqrt(dot(a, a)); }

// Rest-state Dm^-1 in the triangle's local 2D frame
// (crates/vistio-solver/src/element.rs:228-263).
void dm_inverse(F3 e1, F3 e2, float out[4]) {
  out[0] = 1.f; out[1] = 0.f; out[2] = 0.f; out[3] = 1.f;
  float l1 = len(e1);
  if (l1 < 1e-10f) return;
  F3 u = dvs(e1, l1);
  F3 n = cross(e1, e2);
  if (len(n) < 1e-10f) return;
  F3 vv = cross(n, u);
  F3 v = mul(vv, 1.f / len(vv));
  float d00 = dot(e1, u), d10 = dot(e1, v), d01 = dot(e2, u), d11 = dot(e2, v);
  float det = d00 * d11 - d01 * d10;
  if (std::fabs(det) < 1e-10f) return;
  float id = 1.f / det;
  out[0] = d11 * id;
  out[1] = -d10 * id;
  out[2] = -d01 * id;
  out[3] = d00 * id;
}

// Dihedral angle between the wings seen from the shared edge
// (crates/vistio-solver/src/bending.rs:56-91).
float dihedral(F3 p0, F3 p1, F3 pa, F3 pb) {
  const float PI = 3.14159265358979323846f;
  F3 e = sub(p1, p0);
  float l = len(e);
  if (l < 1e-10f) return PI;
  F3 ed = dvs(e, l);
  F3 ta = sub(pa, p0), tb = sub(pb, p0);
  F3 qa = sub(ta, mul(ed, dot(ta, ed))), qb = sub(tb, mul(ed, dot(tb, ed)));
  float la = len(qa), lb = len(qb);
  if (la < 1e-10f || lb < 1e-10f) return PI;
  qa = dvs(qa, la);
  qb = dvs(qb, lb);
  float c = dot(qa, qb);
  c = c < -1.f ? -1.f : (c > 1.f ? 1.f : c);
  return std::acos(c);
}

float clamp_rest(float a) {  // bending.rs:122-128
  const float PI = 3.14159265358979323846f;
  if (std::fabs(a - PI) < 1e-3f) return PI;
  if (std::fabs(a) < 1e-3f) return 0.f;
  return a;
}

// ------------------------------------------------------------ ordering
struct Graph {
  uint32_t n;
  std::vector<uint32_t> ptr, adj;
};

// Nested dissection. With coordinates: split at the median of the longest
// extent; the first half's vertices adjacent to the second half separate
// them. Without: BFS level structure from a pseudo-peripheral vertex, the
// median level separates. Separators are numbered after both halves.
class Dissector {
 public:
  Dissector(const Graph& g, const float* xyz) : g_(g), xyz_(xyz), mark_(g.n, 0), lvl_(g.n, -1) {}
  void run(std::vector<uint32_t>& order) {
    std::vector<uint32_t> all(g_.n);
    std::iota(all.begin(), all.end(), 0u);
    order.clear();
    order.reserve(g_.n);
    rec(all, order, 0);
  }

 private:
  const Graph& g_;
  const float* xyz_;
  std::vector<uint32_t> mark_;
  std::vector<int> lvl_;
  uint32_t stamp_ = 0;
  static constexpr size_t kLeaf = 24;

  void rec(std::vector<uint32_t>& verts, std::vector<uint32_t>& out, int depth) {
    if (verts.size() <= kLeaf || depth > 64) {
      out.insert(out.end(), verts.begin(), verts.end());
      return;
    }
    std::vector<uint32_t> A, B, S;
    if (xyz_) split_geometric(verts, A, B, S);
    else split_bfs(verts, A, B, S);
    if (A.empty() && B.empty()) {
      out.insert(out.end(), S.begin(), S.end());
      return;
    }
    rec(A, out, depth + 1);
    rec(B, out, depth + 1);
    out.insert(out.end(), S.begin(), S.end());
  }

  void split_geometric(std::vector<uint32_t>& verts, std::vector<uint32_t>& A, std::vector<uint32_t>& B,
                       std::vector<uint32_t>& S) {
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    for (uint32_t v : verts)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], xyz_[3 * v + k]);
        hi[k] = std::max(hi[k], xyz_[3 * v + k]);
      }
    // The longest axis, a later one only when clearly longer: extents equal up
    // to rounding (a square sheet) give the same axis at every scale, so a
    // uniformly scaled mesh gets the same ordering (and its symbolic factor
    // comes from the cache).
    int ax = 0;
    for (int k = 1; k < 3; ++k)
      if (hi[k] - lo[k] > (hi[ax] - lo[ax]) * (1.f + 1e-4f)) ax = k;
    std::stable_sort(verts.begin(), verts.end(),
                     [&](uint32_t a, uint32_t b) { return xyz_[3 * a + ax] < xyz_[3 * b + ax]; });
    size_t mid = verts.size() / 2;
    ++stamp_;
    for (size_t i = mid; i < verts.size(); ++i) mark_[verts[i]] = stamp_;
    for (size_t i = 0; i < mid; ++i) {
      uint32_t v = verts[i];
      bool touch = false;
      for (uint32_t p = g_.ptr[v]; p < g_.ptr[v + 1]; ++p)
        if (mark_[g_.adj[p]] == stamp_) { touch = true; break; }
      (touch ? S : A).push_back(v);
    }
    B.assign(verts.begin() + mid, verts.end());
  }

  void bfs(const std::vector<uint32_t>& verts, uint32_t src, std::vector<uint32_t>& order) {
    order.clear();
    for (uint32_t v : verts) lvl_[v] = -1;
    lvl_[src] = 0;
    order.push_back(src);
    for (size_t h = 0; h < order.size(); ++h) {
      uint32_t v = order[h];
      for (uint32_t p = g_.ptr[v]; p < g_.ptr[v + 1]; ++p) {
        uint32_t u = g_.adj[p];
        if (mark_[u] == stamp_ && lvl_[u] < 0) { lvl_[u] = lvl_[v] + 1; order.push_back(u); }
      }
    }
  }

  void split_bfs(std::vector<uint32_t>& verts, std::vector<uint32_t>& A, std::vector<uint32_t>& B,
                 std::vector<uint32_t>& S) {
    ++stamp_;
    for (uint32_t v : verts) mark_[v] = stamp_;
    std::vector<uint32_t> order;
    bfs(verts, verts[0], order);
    bfs(verts, order.back(), order);  // pseudo-peripheral start
    if (order.size() < verts.size()) {
      // Disconnected: the reached component and the rest are independent.
      std::vector<uint32_t> rest;
      for (uint32_t v : verts) if (lvl_[v] < 0) rest.push_back(v);
      A = order;
      B = rest;
      return;
    }
    int maxl = lvl_[order.back()];
    if (maxl < 2) { S = verts; return; }
    std::vector<size_t> cnt(maxl + 1, 0);
    for (uint32_t v : verts) cnt[lvl_[v]]++;
    size_t acc = 0;
    int sl = 1;
    for (int l = 0; l <= maxl; ++l) {
      acc += cnt[l];
      if (acc * 2 >= verts.size()) { sl = std::max(1, std::min(l, maxl - 1)); break; }
    }
    for (uint32_t v : verts) {
      if (lvl_[v] < sl) A.push_back(v);
      else if (lvl_[v] == sl) S.push_back(v);
      else B.push_back(v);
    }
  }
};

}  // namespace

// ------------------------------------------------------------- factorize
std::string factorize_csr(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx, const double* vals,
                          const float* coords, Factor& f, int* status, bool numeric) {
  *status = 0;
  f = Factor();
  f.n = n;
  f.numeric = numeric;
  if (n == 0) { *status = 3; return "cannot factorize an empty matrix"; }
  // Symmetric adjacency (pattern of A + A^T without the diagonal).
  Graph g;
  g.n = n;
  {
    // Bucket both directions of every off-diagonal entry by row (two counting
    // passes), then sort and deduplicate each short row in place.
    std::vector<uint32_t> deg(n + 1, 0);
    for (uint32_t i = 0; i < n; ++i)
      for (uint32_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
        uint32_t j = col_idx[p];
        if (j >= n) { *status = 3; return "column index out of range"; }
        if (j != i) { deg[i + 1]++; deg[j + 1]++; }
      }
    for (uint32_t i = 0; i < n; ++i) deg[i + 1] += deg[i];
    std::vector<uint32_t> raw(deg[n]), fill(deg.begin(), deg.end() - 1);
    for (uint32_t i = 0; i < n; ++i)
      for (uint32_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
        uint32_t j = col_idx[p];
        if (j != i) { raw[fill[i]++] = j; raw[fill[j]++] = i; }
      }
    g.ptr.assign(n + 1, 0);
    g.adj.clear();
    g.adj.reserve(raw.size());
    for (uint32_t i = 0; i < n; ++i) {
      auto b = raw.begin() + deg[i], e = raw.begin() + deg[i + 1];
      std::sort(b, e);
      g.adj.insert(g.adj.end(), b, std::unique(b, e));
      g.ptr[i + 1] = uint32_t(g.adj.size());
    }
  }
  std::vector<uint32_t> order;
  Dissector(g, coords).run(order);
  std::shared_ptr<SymPending> mine;  // this call's analysis, while pending
  if (!numeric) {
    const uint64_t key = fnv_words(fnv_words(fnv_words(14695981039346656037ull, g.ptr), g.adj), order);
    SymCache& C = sym_cache();
    std::unique_lock<std::mutex> lk(C.mu);
    for (;;) {
      auto range = C.map.equal_range(key);
      for (auto it = range.first; it != range.second; ++it)
        if (it->second.same(g.ptr, g.adj, order)) {
          it->second.used = ++C.clock;
          C.hits++;
          f = *it->second.factor;
          return "";
        }
      std::shared_ptr<SymPending> other;
      for (auto& p : C.pending)
        if (p->key == key && p->entry.same(g.ptr, g.adj, order)) { other = p; break; }
      if (!other) break;
      C.cv.wait(lk, [&] { return other->done; });
      if (other->entry.factor) {
        C.hits++;
        f = *other->entry.factor;
        return "";
      }  // abandoned: look again
    }
    C.misses++;
    mine = std::make_shared<SymPending>();
    mine->key = key;
    mine->entry.ptr = g.ptr;
    mine->entry.adj = g.adj;
    mine->entry.order = order;
    C.pending.push_back(mine);
  }
  // An early return leaves the pending analysis abandoned, and its waiters
  // compute their own.
  struct Abandon {
    std::shared_ptr<SymPending>& p;
    ~Abandon() {
      if (!p) return;
      SymCache& C = sym_cache();
      std::lock_guard<std::mutex> lk(C.mu);
      p->done = true;
      C.pending.erase(std::find(C.pending.begin(), C.pending.end(), p));
      C.cv.notify_all();
    }
  } abandon{mine};
  // Elimination tree of the permuted matrix, then a postorder so every
  // subtree is a contiguous column range.
  auto etree_of = [&](const std::vector<uint32_t>& perm, std::vector<uint32_t>& ip, std::vector<int>& parent) {
    ip.assign(n, 0);
    for (uint32_t k = 0; k < n; ++k) ip[perm[k]] = k;
    parent.assign(n, -1);
    std::vector<int> anc(n, -1);
    for (uint32_t k = 0; k < n; ++k) {
      uint32_t old = perm[k];
      for (uint32_t p = g.ptr[old]; p < g.ptr[old + 1]; ++p) {
        int i = int(ip[g.adj[p]]);
        while (i != -1 && i < int(k)) {
          int nx = anc[i];
          anc[i] = int(k);
          if (nx == -1) { parent[i] = int(k); break; }
          i = nx;
        }
      }
    }
  };
  std::vector<uint32_t> ip;
  std::vector<int> parent;
  etree_of(order, ip, parent);
  {
    std::vector<std::vector<uint32_t>> kids(n);
    std::vector<uint32_t> roots;
    for (uint32_t k = 0; k < n; ++k) (parent[k] < 0 ? roots : kids[parent[k]]).push_back(k);
    std::vector<uint32_t> post;
    post.reserve(n);
    std::vector<std::pair<uint32_t, size_t>> st;
    for (uint32_t r : roots) {
      st.push_back({r, 0});
      while (!st.empty()) {
        auto& top = st.back();
        if (top.second < kids[top.first].size()) {
          uint32_t c = kids[top.first][top.second++];
          st.push_back({c, 0});
        } else {
          post.push_back(top.first);
          st.pop_back();
        }
      }
    }
    std::vector<uint32_t> perm2(n);
    for (uint32_t k = 0; k < n; ++k) perm2[k] = order[post[k]];
    order.swap(perm2);
  }
  etree_of(order, ip, parent);
  f.perm = order;
  f.iperm = ip;
  // Upper triangle of B = P A P^T by columns (values summed).
  std::vector<uint32_t> bp(n + 1, 0);
  std::vector<std::pair<uint32_t, double>> bent;
  {
    // Entries bucketed by permuted column (counting passes), each column then
    // sorted by row; an entry given in both triangles counts once (the two
    // copies of a symmetric matrix's entry hold the same value).
    std::vector<uint32_t> cptr(n + 1, 0);
    for (uint32_t i = 0; i < n; ++i)
      for (uint32_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) cptr[std::max(ip[i], ip[col_idx[p]]) + 1]++;
    for (uint32_t c = 0; c < n; ++c) cptr[c + 1] += cptr[c];
    std::vector<std::pair<uint32_t, double>> raw(cptr[n]);
    std::vector<uint32_t> fill(cptr.begin(), cptr.end() - 1);
    for (uint32_t i = 0; i < n; ++i)
      for (uint32_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
        uint32_t r = ip[i], c = ip[col_idx[p]];
        raw[fill[std::max(r, c)]++] = {std::min(r, c), vals[p]};  // accept lower-triangle-only input as well
      }
    bent.reserve(raw.size());
    for (uint32_t c = 0; c < n; ++c) {
      auto b = raw.begin() + cptr[c], e = raw.begin() + cptr[c + 1];
      std::stable_sort(b, e, [](const auto& x, const auto& y) { return x.first < y.first; });
      for (auto it = b; it != e; ++it)
        if (bent.size() == bp[c] || bent.back().first != it->first) bent.push_back(*it);
      bp[c + 1] = uint32_t(bent.size());
    }
  }
  // Up-looking simplicial LL^T in FP64 (row k of L from the etree reach).
  std::vector<int> mark(n, -1), stack(n), pat(n);
  auto ereach = [&](uint32_t k) -> int {
    int top = int(n);
    mark[k] = int(k);
    for (uint32_t p = bp[k]; p < bp[k + 1]; ++p) {
      int i = int(bent[p].first);
      if (i >= int(k)) continue;
      int l = 0;
      for (; mark[i] != int(k); i = parent[i]) { stack[l++] = i; mark[i] = int(k); }
      while (l > 0) pat[--top] = stack[--l];
    }
    return top;
  };
  std::vector<uint32_t> cnt(n, 1);
  for (uint32_t k = 0; k < n; ++k) {
    int top = ereach(k);
    for (int p = top; p < int(n); ++p) cnt[pat[p]]++;
  }
  std::vector<uint64_t> Lp(n + 1, 0);
  for (uint32_t k = 0; k < n; ++k) Lp[k + 1] = Lp[k] + cnt[k];
  std::vector<uint32_t> Li(Lp[n]);
  std::vector<double> Lx(numeric ? Lp[n] : 0);
  std::vector<uint64_t> cur(Lp.begin(), Lp.end() - 1);
  std::vector<double> x(n, 0.0);
  std::fill(mark.begin(), mark.end(), -1);
  if (!numeric) {  // the pattern of L only (row k from the etree reach)
    for (uint32_t k = 0; k < n; ++k) {
      int top = ereach(k);
      for (int p = top; p < int(n); ++p) Li[cur[uint32_t(pat[p])]++] = k;
      Li[cur[k]++] = k;
    }
  }
  for (uint32_t k = 0; k < n && numeric; ++k) {
    int top = ereach(k);
    for (uint32_t p = bp[k]; p < bp[k + 1]; ++p) x[bent[p].first] += bent[p].second;
    double d = x[k];
    x[k] = 0;
    for (int p = top; p < int(n); ++p) {
      uint32_t i = uint32_t(pat[p]);
      double lki = x[i] / Lx[Lp[i]];
      x[i] = 0;
      for (uint64_t q = Lp[i] + 1; q < cur[i]; ++q) x[Li[q]] -= Lx[q] * lki;
      d -= lki * lki;
      uint64_t q = cur[i]++;
      Li[q] = k;
      Lx[q] = lki;
    }
    if (!(d > 0.0) || !std::isfinite(d)) {
      *status = 11;
      return "matrix is not symmetric positive definite (Cholesky pivot " + std::to_string(k) + ")";
    }
    uint64_t q = cur[k]++;
    Li[q] = k;
    Lx[q] = std::sqrt(d);
  }
  f.nnz_L = Lp[n];
  // Fundamental supernodes, then relaxed amalgamation of a child whose
  // columns directly precede its parent's.
  // Column j continues the supernode of j-1 when j is j-1's parent, j has no
  // other child, and struct(L_{j-1}) = {j-1} u struct(L_j).
  std::vector<uint32_t> sfirst;  // supernode first columns
  {
    std::vector<uint32_t> nkids(n, 0);
    for (uint32_t j = 0; j < n; ++j) if (parent[j] >= 0) nkids[parent[j]]++;
    for (uint32_t j = 0; j < n; ++j) {
      bool cont = j > 0 && parent[j - 1] == int(j) && nkids[j] == 1 && cnt[j - 1] == cnt[j] + 1 &&
                  j - sfirst.back() < kMaxSupernodeCols;
      if (!cont) sfirst.push_back(j);
    }
  }
  // Row structure (below diagonal block) of a supernode = structure of its
  // last column minus that column. For amalgamated supernodes use the
  // union, which equals the structure of the first column minus own columns.
  struct SN { uint32_t f, s; std::vector<uint32_t> below; };
  std::vector<SN> sns;
  for (size_t k = 0; k < sfirst.size(); ++k) {
    uint32_t f0 = sfirst[k], f1 = (k + 1 < sfirst.size()) ? sfirst[k + 1] : n;
    SN s;
    s.f = f0;
    s.s = f1 - f0;
    uint32_t last = f1 - 1;
    for (uint64_t q = Lp[last] + 1; q < Lp[last + 1]; ++q) s.below.push_back(Li[q]);
    sns.push_back(std::move(s));
  }
  // Relaxed amalgamation: merge supernode k into k+1 when k+1 is k's parent
  // (k's parent column is the first column of k+1) and the zero fill stays small.
  {
    std::vector<SN> out;
    for (size_t k = 0; k < sns.size(); ++k) {
      SN cur_sn = std::move(sns[k]);
      while (k + 1 < sns.size()) {
        SN& nxt = sns[k + 1];
        uint32_t lastc = cur_sn.f + cur_sn.s - 1;
        if (parent[lastc] != int(nxt.f)) break;
        // merged structure below = nxt.below; cur's below must be within nxt cols ∪ nxt.below
        uint64_t s_new = uint64_t(cur_sn.s) + nxt.s;
        uint64_t rows_full = s_new + nxt.below.size();
        uint64_t dense = 0, actual = 0;
        for (uint32_t j = cur_sn.f; j < nxt.f + nxt.s; ++j) {
          dense += rows_full - (j - cur_sn.f);
          actual += cnt[j];
        }
        uint64_t zeros = dense - actual;
        bool ok = (s_new <= 8) || (s_new <= 32 && zeros * 5 <= dense) ||
                  (s_new <= kMaxSupernodeCols && zeros * 20 <= dense);
        if (!ok) break;
        SN m;
        m.f = cur_sn.f;
        m.s = uint32_t(s_new);
        m.below = nxt.below;
        cur_sn = std::move(m);
        ++k;
      }
      out.push_back(std::move(cur_sn));
    }
    sns.swap(out);
  }
  // Owner map, parents, levels.
  uint32_t nsn = uint32_t(sns.size());
  f.row_sn.assign(n, 0);
  for (uint32_t k = 0; k < nsn; ++k)
    for (uint32_t j = sns[k].f; j < sns[k].f + sns[k].s; ++j) f.row_sn[j] = k;
  f.sn.resize(nsn);
  uint64_t off = 0;
  for (uint32_t k = 0; k < nsn; ++k) {
    Supernode& S = f.sn[k];
    S.first = sns[k].f;
    S.ncols = sns[k].s;
    S.nrows = uint32_t(sns[k].below.size());
    S.rows_off = uint32_t(f.rows.size());
    f.rows.insert(f.rows.end(), sns[k].below.begin(), sns[k].below.end());
    S.panel_off = off;
    off += uint64_t(S.nrows) * S.ncols;
    S.diag_off = off;
    off += uint64_t(S.ncols) * S.ncols;
    S.parent = S.nrows ? f.row_sn[sns[k].below[0]] : UINT32_MAX;
    S.level = 0;
  }
  // Bottom subtrees whose packed data fits kSubtreeFloats and whose columns
  // number at most kSubtreeCols are swept whole by one warp; the supernodes
  // above them are swept level by level, a top
  // supernode's level being one more than its highest top child (children
  // that are bottom subtrees count as below level 0).
  {
    std::vector<uint64_t> sub(nsn, 0), cols(nsn, 0);
    std::vector<uint32_t> cnt_sub(nsn, 1);
    for (uint32_t k = 0; k < nsn; ++k) {  // children precede parents (postorder)
      sub[k] += sn_floats(f.sn[k].ncols, f.sn[k].nrows);
      cols[k] += f.sn[k].ncols;
      uint32_t p = f.sn[k].parent;
      if (p != UINT32_MAX) { sub[p] += sub[k]; cols[p] += cols[k]; cnt_sub[p] += cnt_sub[k]; }
    }
    std::vector<char> bottom(nsn, 0);
    for (int k = int(nsn) - 1; k >= 0; --k) {  // parents first
      uint32_t p = f.sn[k].parent;
      bool fits = sub[k] <= kSubtreeFloats && cols[k] <= kSubtreeCols;
      if (p != UINT32_MAX && bottom[p]) bottom[k] = 1;
      else if (fits) {
        bottom[k] = 1;
        f.sub_first.push_back(uint32_t(k) + 1 - cnt_sub[k]);
        f.sub_last.push_back(uint32_t(k));
      }
    }
    std::reverse(f.sub_first.begin(), f.sub_first.end());
    std::reverse(f.sub_last.begin(), f.sub_last.end());
    std::vector<int> top_lvl(nsn, -1);
    for (uint32_t k = 0; k < nsn; ++k) {
      if (bottom[k]) { f.sn[k].level = kBottomLevel; continue; }
      if (top_lvl[k] < 0) top_lvl[k] = 0;
      f.sn[k].level = uint32_t(top_lvl[k]);
      uint32_t p = f.sn[k].parent;
      if (p != UINT32_MAX) top_lvl[p] = std::max(top_lvl[p], top_lvl[k] + 1);
    }
  }
  f.nnz_stored = off;
  if (numeric) f.vals.assign(off, 0.0);
  // Scatter the simplicial columns into panels and diagonal blocks.
  std::vector<int> pos(n, -1);
  std::vector<double> Lkk;
  for (uint32_t k = 0; k < nsn && numeric; ++k) {
    Supernode& S = f.sn[k];
    const uint32_t* R = f.rows.data() + S.rows_off;
    for (uint32_t r = 0; r < S.nrows; ++r) pos[R[r]] = int(r);
    uint32_t s = S.ncols;
    Lkk.assign(size_t(s) * s, 0.0);
    for (uint32_t c = 0; c < s; ++c) {
      uint32_t j = S.first + c;
      for (uint64_t q = Lp[j]; q < Lp[j + 1]; ++q) {
        uint32_t i = Li[q];
        if (i < S.first + s) Lkk[size_t(c) * s + (i - S.first)] = Lx[q];  // column-major
        else {
          int pr = pos[i];
          if (pr < 0) { *status = 3; return "internal: supernode structure mismatch"; }
          f.vals[S.panel_off + uint64_t(pr) * s + c] = Lx[q];
        }
      }
    }
    for (uint32_t r = 0; r < S.nrows; ++r) pos[R[r]] = -1;
    // inv(L_kk) by forward substitution on the identity (column-major).
    double* Inv = f.vals.data() + S.diag_off;
    for (uint32_t c = 0; c < s; ++c) {
      // column c of inverse: solve L y = e_c
      for (uint32_t i = 0; i < s; ++i) {
        double v = (i == c) ? 1.0 : 0.0;
        for (uint32_t m = c; m < i; ++m) v -= Lkk[size_t(m) * s + i] * Inv[size_t(c) * s + m];
        Inv[size_t(c) * s + i] = (i < c) ? 0.0 : v / Lkk[size_t(i) * s + i];
      }
    }
  }
  // Level schedule of the top supernodes.
  uint32_t nl = 0;
  for (auto& S : f.sn) if (S.level != kBottomLevel) nl = std::max(nl, S.level + 1);
  f.nlevels = nl;
  f.level_ptr.assign(nl + 1, 0);
  std::vector<std::vector<uint32_t>> bylvl(nl);
  for (uint32_t k = 0; k < nsn; ++k) if (f.sn[k].level != kBottomLevel) bylvl[f.sn[k].level].push_back(k);
  f.level_sn_ptr.assign(nl + 1, 0);
  for (uint32_t l = 0; l < nl; ++l) {
    std::stable_sort(bylvl[l].begin(), bylvl[l].end(), [&](uint32_t a, uint32_t b) {
      uint64_t wa = uint64_t(f.sn[a].ncols) * (f.sn[a].ncols + f.sn[a].nrows);
      uint64_t wb = uint64_t(f.sn[b].ncols) * (f.sn[b].ncols + f.sn[b].nrows);
      return wa > wb;
    });
    for (uint32_t k : bylvl[l]) {
      f.level_sn.push_back(k);
      for (uint32_t c = 0; c < f.sn[k].ncols; ++c) f.level_rows.push_back(f.sn[k].first + c);
    }
    f.level_ptr[l + 1] = uint32_t(f.level_rows.size());
    f.level_sn_ptr[l + 1] = uint32_t(f.level_sn.size());
  }
  // Forward pull lists.
  f.fwd_ptr.assign(n + 1, 0);
  for (uint32_t k = 0; k < nsn; ++k)
    for (uint32_t r = 0; r < f.sn[k].nrows; ++r) f.fwd_ptr[f.rows[f.sn[k].rows_off + r] + 1]++;
  for (uint32_t i = 0; i < n; ++i) f.fwd_ptr[i + 1] += f.fwd_ptr[i];
  f.fwd_sn.resize(f.fwd_ptr[n]);
  f.fwd_pos.resize(f.fwd_ptr[n]);
  std::vector<uint32_t> fc(f.fwd_ptr.begin(), f.fwd_ptr.end() - 1);
  for (uint32_t k = 0; k < nsn; ++k)
    for (uint32_t r = 0; r < f.sn[k].nrows; ++r) {
      uint32_t row = f.rows[f.sn[k].rows_off + r];
      uint32_t q = fc[row]++;
      f.fwd_sn[q] = k;
      f.fwd_pos[q] = r;
    }
  if (mine) {
    SymCache& C = sym_cache();
    std::lock_guard<std::mutex> lk(C.mu);
    SymEntry& e = mine->entry;
    e.factor = std::make_shared<const Factor>(f);
    e.bytes = factor_bytes(f) + vec_bytes(e.ptr) + vec_bytes(e.adj) + vec_bytes(e.order);
    if (e.bytes <= C.limit) {
      while (C.bytes + e.bytes > C.limit && !C.map.empty()) {
        auto victim = C.map.begin();
        for (auto it = C.map.begin(); it != C.map.end(); ++it)
          if (it->second.used < victim->second.used) victim = it;
        C.bytes -= victim->second.bytes;
        C.map.erase(victim);
      }
      e.used = ++C.clock;
      C.bytes += e.bytes;
      C.map.emplace(mine->key, e);
    }
    mine->done = true;  // waiters take the factor from the pending record
    C.pending.erase(std::find(C.pending.begin(), C.pending.end(), mine));
    C.cv.notify_all();
    mine.reset();
  }
  return "";
}

void symbolic_cache_info(uint64_t* hits, uint64_t* misses, uint64_t* bytes, uint64_t* entries) {
  SymCache& C = sym_cache();
  std::lock_guard<std::mutex> lk(C.mu);
  if (hits) *hits = C.hits;
  if (misses) *misses = C.misses;
  if (bytes) *bytes = C.bytes;
  if (entries) *entries = C.map.size();
}

void symbolic_cache_set_limit(uint64_t limit_bytes) {
  SymCache& C = sym_cache();
  std::lock_guard<std::mutex> lk(C.mu);
  C.limit = limit_bytes;
  while (C.bytes > C.limit && !C.map.empty()) {
    auto victim = C.map.begin();
    for (auto it = C.map.begin(); it != C.map.end(); ++it)
      if (it->second.used < victim->second.used) victim = it;
    C.bytes -= victim->second.bytes;
    C.map.erase(victim);
  }
}

// ----------------------------------------------------------- instance
std::string build_instance(uint32_t nv, const float* px, const float* py, const float* pz, uint32_t nt,
                           const uint32_t* tris, const uint8_t* pinned, const SetupParams& prm,
                           InstanceSetup& I, int* status) {
  *status = 0;
  if (nv == 0 || nt == 0) { *status = 1; return "mesh has no vertices or no triangles"; }
  for (uint64_t k = 0; k < 3ull * nt; ++k)
    if (tris[k] >= nv) { *status = 1; return "triangle index out of range"; }
  for (uint32_t i = 0; i < nv; ++i)
    if (!std::isfinite(px[i]) || !std::isfinite(py[i]) || !std::isfinite(pz[i])) {
      *status = 1;
      return "non-finite vertex position";
    }
  if (!(prm.matrix_dt > 0.f)) { *status = 3; return "matrix_dt must be positive"; }
  I = InstanceSetup();
  I.nv = nv;
  I.nt = nt;
  I.prm = prm;
  I.rest.resize(3 * size_t(nv));
  for (uint32_t i = 0; i < nv; ++i) { I.rest[3 * i] = px[i]; I.rest[3 * i + 1] = py[i]; I.rest[3 * i + 2] = pz[i]; }
  I.tris.assign(tris, tris + 3 * size_t(nt));
  I.pinned.assign(pinned, pinned + nv);
  auto P = [&](uint32_t i) { return F3{px[i], py[i], pz[i]}; };
  // ElementData::from_mesh (element.rs:54-91)
  I.dm_inv.resize(4 * size_t(nt));
  I.area.resize(nt);
  I.tri_w.resize(nt);
  for (uint32_t t = 0; t < nt; ++t) {
    F3 p0 = P(tris[3 * t]), p1 = P(tris[3 * t + 1]), p2 = P(tris[3 * t + 2]);
    F3 e1 = sub(p1, p0), e2 = sub(p2, p0);
    I.area[t] = 0.5f * len(cross(e1, e2));
    dm_inverse(e1, e2, &I.dm_inv[4 * size_t(t)]);
    I.tri_w[t] = prm.stiffness * I.area[t];
  }
  // Lumped masses (pd_solver.rs:1219-1242)
  I.mass.assign(nv, 0.f);
  float dens = prm.density_gsm / 1000.f;
  for (uint32_t t = 0; t < nt; ++t) {
    float third = (I.area[t] * dens) / 3.0f;
    for (int k = 0; k < 3; ++k) I.mass[tris[3 * t + k]] += third;
  }
  for (uint32_t i = 0; i < nv; ++i) {
    if (pinned[i]) I.mass[i] = 1e8f;
    else if (I.mass[i] < 1e-8f) I.mass[i] = 1e-8f;
  }
  // Interior edges (topology.rs:58-121), kept sorted by (v0, v1). The wing of
  // tri_a comes from the lower-indexed triangle.
  if (prm.bending != BEND_NONE) {
    // Half-edges (edge key, triangle) in stable (lo, hi) order: bucketed by the
    // lower vertex in triangle order, then each short bucket insertion-sorted
    // by the higher one.
    std::vector<uint32_t> lo_ptr(nv + 1, 0);
    for (size_t q = 0; q < 3 * size_t(nt); ++q) {
      uint32_t x = tris[q], y = tris[q % 3 == 2 ? q - 2 : q + 1];
      lo_ptr[std::min(x, y) + 1]++;
    }
    for (uint32_t i = 0; i < nv; ++i) lo_ptr[i + 1] += lo_ptr[i];
    std::vector<std::pair<uint64_t, uint32_t>> he(3 * size_t(nt));
    {
      std::vector<uint32_t> fill(lo_ptr.begin(), lo_ptr.end() - 1);
      for (uint32_t t = 0; t < nt; ++t) {
        uint32_t a = tris[3 * t], b = tris[3 * t + 1], c = tris[3 * t + 2];
        uint32_t e[3][2] = {{a, b}, {b, c}, {c, a}};
        for (auto& x : e) {
          uint32_t lo = std::min(x[0], x[1]), hi = std::max(x[0], x[1]);
          he[fill[lo]++] = {(uint64_t(lo) << 32) | hi, t};
        }
      }
    }
    for (uint32_t v = 0; v < nv; ++v)
      for (uint32_t i = lo_ptr[v] + 1; i < lo_ptr[v + 1]; ++i) {
        auto x = he[i];
        uint32_t j = i;
        for (; j > lo_ptr[v] && he[j - 1].first > x.first; --j) he[j] = he[j - 1];
        he[j] = x;
      }
    auto wing = [&](uint32_t t, uint32_t v0, uint32_t v1) {
      uint32_t a = tris[3 * t], b = tris[3 * t + 1], c = tris[3 * t + 2];
      if (a != v0 && a != v1) return a;
      if (b != v0 && b != v1) return b;
      return c;
    };
    const float PI = 3.14159265358979323846f;
    for (size_t i = 0; i < he.size();) {
      size_t j = i;
      while (j < he.size() && he[j].first == he[i].first) ++j;
      if (j - i == 2) {
        uint32_t v0 = uint32_t(he[i].first >> 32), v1 = uint32_t(he[i].first & 0xffffffffu);
        uint32_t wa = wing(he[i].second, v0, v1), wb = wing(he[i + 1].second, v0, v1);
        F3 p0 = P(v0), p1 = P(v1), pa = P(wa), pb = P(wb);
        float rest = clamp_rest(dihedral(p0, p1, pa, pb));
        F3 e = sub(p1, p0);
        float el = len(e);
        float st[4] = {-1.f, -1.f, 1.f, 1.f};
        float w = prm.bend_stiffness * el;
        bool keep = true;
        if (prm.bending == BEND_DS || prm.bending == BEND_DS_ANISO) {
          // DiscreteShellsBendingData::from_topology (discrete_shells.rs:106-199)
          float area_a = 0.5f * len(cross(sub(p1, p0), sub(pa, p0)));
          float area_b = 0.5f * len(cross(sub(p1, p0), sub(pb, p0)));
          if (el < 1e-10f) keep = false;
          else {
            float inv_e2 = 1.f / (el * el);
            float c_wa = el / (2.f * std::max(area_a, 1e-8f));
            float c_wb = el / (2.f * std::max(area_b, 1e-8f));
            float d0a = dot(sub(p1, pa), e) * inv_e2, d0b = dot(sub(p1, pb), e) * inv_e2;
            float c0 = -d0a * c_wa - d0b * c_wb;
            float d1a = dot(sub(pa, p0), e) * inv_e2, d1b = dot(sub(pb, p0), e) * inv_e2;
            float c1 = -d1a * c_wa - d1b * c_wb;
            float raw[4] = {c0, c1, c_wa, c_wb};
            float nrm = std::sqrt(raw[0] * raw[0] + raw[1] * raw[1] + raw[2] * raw[2] + raw[3] * raw[3]);
            if (nrm > 1e-10f) for (int k = 0; k < 4; ++k) st[k] = raw[k] / nrm;
            else { st[0] = st[1] = -0.5f; st[2] = st[3] = 0.5f; }
            if (prm.bending == BEND_DS_ANISO) {  // discrete_shells.rs:219-269
              float kw = prm.bend_warp, kf = prm.bend_weft, avg = (kw + kf) / 2.f;
              if (avg > 1e-8f) {
                F3 ed = dvs(e, el);
                F3 hz{ed.x, 0.f, ed.z};
                float hl = len(hz);
                if (hl >= 1e-10f) {
                  F3 hd = dvs(hz, hl);
                  float cs = std::fabs(hd.x), cos2 = cs * cs, sin2 = 1.f - cos2;
                  w *= (kf * cos2 + kw * sin2) / avg;
                }
              }
            }
          }
        }
        (void)PI;
        if (keep) {
          I.hinge_v.insert(I.hinge_v.end(), {v0, v1, wa, wb});
          I.hinge_st.insert(I.hinge_st.end(), st, st + 4);
          I.hinge_w.push_back(w);
          I.hinge_rest.push_back(rest);
        }
      }
      i = j;
    }
  }
  I.nh = uint32_t(I.hinge_w.size());
  // assemble_system_matrix (assembly.rs:44-135): the f32 triplets in the
  // reference's order (diagonal masses, then triangles, then hinges), summed
  // per (row, col) in f64 in that order. Assembled row by row: a vertex's
  // incidences (element, corner) are listed in increasing element order, so
  // each (row, col) meets its triplets in the same order as the reference's
  // single list; a column gets a slot on first sight and the slots are
  // emitted by column.
  float h = prm.matrix_dt;
  float inv_h2 = 1.f / (h * h);
  std::vector<uint32_t> tptr(nv + 1, 0), hptr(nv + 1, 0);
  for (size_t q = 0; q < 3 * size_t(nt); ++q) tptr[tris[q] + 1]++;
  for (size_t q = 0; q < 4 * size_t(I.nh); ++q) hptr[I.hinge_v[q] + 1]++;
  for (uint32_t i = 0; i < nv; ++i) { tptr[i + 1] += tptr[i]; hptr[i + 1] += hptr[i]; }
  std::vector<uint32_t> tinc(tptr[nv]), hinc(hptr[nv]);
  {
    std::vector<uint32_t> ft(tptr.begin(), tptr.end() - 1), fh(hptr.begin(), hptr.end() - 1);
    for (size_t q = 0; q < 3 * size_t(nt); ++q) tinc[ft[tris[q]]++] = uint32_t(q);
    for (size_t q = 0; q < 4 * size_t(I.nh); ++q) hinc[fh[I.hinge_v[q]]++] = uint32_t(q);
  }
  I.A_ptr.assign(nv + 1, 0);
  I.A_col.reserve(size_t(nv) * 16);
  I.A_val.reserve(size_t(nv) * 16);
  std::vector<int32_t> slot_of(nv, -1);
  std::vector<std::pair<uint32_t, double>> slots;
  auto add = [&](uint32_t c, float v) {
    int32_t& sl = slot_of[c];
    if (sl < 0) { sl = int32_t(slots.size()); slots.push_back({c, 0.0}); }
    slots[size_t(sl)].second += double(v);
  };
  for (uint32_t r = 0; r < nv; ++r) {
    slots.clear();
    add(r, I.mass[r] * inv_h2);
    for (uint32_t e = tptr[r]; e < tptr[r + 1]; ++e) {
      const uint32_t t = tinc[e] / 3, a = tinc[e] % 3;
      const float* d = &I.dm_inv[4 * size_t(t)];
      float g[3][2] = {{-(d[0] + d[1]), -(d[2] + d[3])}, {d[0], d[2]}, {d[1], d[3]}};
      for (int b2 = 0; b2 < 3; ++b2) {
        float dt_ = g[a][0] * g[b2][0] + g[a][1] * g[b2][1];
        if (std::fabs(dt_) > 1e-12f) add(tris[3 * size_t(t) + b2], I.tri_w[t] * dt_);
      }
    }
    for (uint32_t e = hptr[r]; e < hptr[r + 1]; ++e) {
      const uint32_t k = hinc[e] / 4, a = hinc[e] % 4;
      const float* st = &I.hinge_st[4 * size_t(k)];
      for (int b2 = 0; b2 < 4; ++b2) {
        float v = I.hinge_w[k] * st[a] * st[b2];
        if (std::fabs(v) > 1e-12f) add(I.hinge_v[4 * size_t(k) + b2], v);
      }
    }
    for (auto& x : slots) slot_of[x.first] = -1;
    std::sort(slots.begin(), slots.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    for (auto& x : slots) { I.A_col.push_back(x.first); I.A_val.push_back(x.second); }
    I.A_ptr[r + 1] = uint32_t(I.A_col.size());
  }
  mirror_upper(nv, I.A_ptr, I.A_col, I.A_val);
  std::string err = factorize_csr(nv, I.A_ptr.data(), I.A_col.data(), I.A_val.data(), I.rest.data(), I.factor, status,
                                  prm.numeric);
  if (!err.empty()) return "Cholesky factorization failed: " + err;
  return "";
}

void mirror_upper(uint32_t n, std::vector<uint32_t>& ptr, std::vector<uint32_t>& col, std::vector<double>& val) {
  std::vector<uint32_t> P(n + 1, 0);
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t q = ptr[i]; q < ptr[i + 1]; ++q) {
      const uint32_t j = col[q];
      if (j < i) continue;
      P[i + 1]++;
      if (j != i) P[j + 1]++;
    }
  for (uint32_t i = 0; i < n; ++i) P[i + 1] += P[i];
  std::vector<uint32_t> C(P[n]), cur(P.begin(), P.end() - 1);
  std::vector<double> V(P[n]);
  // row i receives its lower entries while the rows j < i are visited, before
  // its own upper ones: every row comes out sorted
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t q = ptr[i]; q < ptr[i + 1]; ++q) {
      const uint32_t j = col[q];
      if (j < i) continue;
      C[cur[i]] = j; V[cur[i]++] = val[q];
      if (j != i) { C[cur[j]] = i; V[cur[j]++] = val[q]; }
    }
  ptr.swap(P);
  col.swap(C);
  val.swap(V);
}

void append_permuted_matrix(const InstanceSetup& I, uint32_t base, std::vector<uint32_t>& ptr,
                            std::vector<uint32_t>& col, std::vector<double>& val) {
  const Factor& F = I.factor;
  for (uint32_t r = 0; r < I.nv; ++r) {
    const uint32_t i = F.perm[r];
    for (uint32_t q = I.A_ptr[i]; q < I.A_ptr[i + 1]; ++q) {
      col.push_back(base + F.iperm[I.A_col[q]]);
      val.push_back(I.A_val[q]);
    }
    ptr.push_back(uint32_t(col.size()));
  }
}

}  // namespace vistio
