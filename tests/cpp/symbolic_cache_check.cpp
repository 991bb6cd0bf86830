// CPU check of the symbolic-analysis cache of the host set-up
// (vistio_b200/csrc/setup.cpp, factorize_csr with numeric == false):
// * a cache hit gives the same Factor, field for field, as an analysis with
//   the cache disabled, for quad grids with and without pins, DS bending and
//   a perturbed (non-grid) geometry;
// * the same grid at other uniform scales hits the entry of the first;
// * eight threads that analyse the same mesh at once run one analysis (the
//   others wait for it) and all get the same Factor;
// * the byte bound evicts the least recently used entry, 0 empties it.
// Prints one JSON object; exit status 0 when every check holds.
#include <cstdio>
#include <random>
#include <thread>
#include <vector>

#include "../../vistio_b200/csrc/setup.h"

using namespace vistio;

namespace {

template <class T> void put(std::vector<char>& o, const std::vector<T>& v) {
  size_t n = v.size();
  o.insert(o.end(), (const char*)&n, (const char*)&n + sizeof(n));
  o.insert(o.end(), (const char*)v.data(), (const char*)v.data() + n * sizeof(T));
}

std::vector<char> blob(const Factor& F) {
  std::vector<char> o;
  put(o, F.perm); put(o, F.iperm); put(o, F.rows); put(o, F.row_sn); put(o, F.level_ptr); put(o, F.level_rows);
  put(o, F.level_sn_ptr); put(o, F.level_sn); put(o, F.sub_first); put(o, F.sub_last); put(o, F.fwd_ptr);
  put(o, F.fwd_sn); put(o, F.fwd_pos);
  std::vector<uint64_t> sn;
  for (const Supernode& s : F.sn) {
    sn.insert(sn.end(), {s.first, s.ncols, s.nrows, s.rows_off, s.panel_off, s.diag_off, s.parent, s.level});
  }
  put(o, sn);
  uint64_t tail[3] = {F.n, F.nnz_L, F.nnz_stored};
  o.insert(o.end(), (const char*)tail, (const char*)tail + sizeof(tail));
  return o;
}

struct Grid {
  std::vector<float> px, py, pz;
  std::vector<uint32_t> tris;
  std::vector<uint8_t> pin;
};

Grid grid(int side, float len, bool pinned, float jitter, unsigned seed) {
  Grid g;
  int vx = side + 1;
  std::mt19937 rng(seed);
  std::uniform_real_distribution<float> u(-jitter, jitter);
  for (int j = 0; j < vx; ++j)
    for (int i = 0; i < vx; ++i) {
      g.px.push_back(-len / 2 + len * float(i) / float(side) + u(rng));
      g.py.push_back(1.f);
      g.pz.push_back(len / 2 - len * float(j) / float(side) + u(rng));
    }
  for (int j = 0; j < side; ++j)
    for (int i = 0; i < side; ++i) {
      uint32_t a = j * vx + i, b = a + 1, c = a + vx, d = c + 1;
      if ((i + j) % 2) g.tris.insert(g.tris.end(), {a, c, b, b, c, d});
      else g.tris.insert(g.tris.end(), {a, c, d, a, d, b});
    }
  g.pin.assign(g.px.size(), 0);
  if (pinned)
    for (int i = 0; i < vx; ++i) g.pin[i] = 1;
  return g;
}

std::vector<char> analyse(const Grid& g, int bending) {
  SetupParams p;
  p.numeric = false;
  p.bending = bending;
  InstanceSetup I;
  int st = 0;
  std::string e = build_instance(uint32_t(g.px.size()), g.px.data(), g.py.data(), g.pz.data(),
                                 uint32_t(g.tris.size() / 3), g.tris.data(), g.pin.data(), p, I, &st);
  if (!e.empty()) { std::fprintf(stderr, "%s\n", e.c_str()); std::exit(2); }
  return blob(I.factor);
}

}  // namespace

int main() {
  int failures = 0;
  uint64_t h0, m0, b0, e0, h1, m1, b1, e1;
  struct Case { int side; float len; bool pinned; float jitter; int bending; };
  const Case cases[] = {{12, 1.f, true, 0.f, BEND_DIHEDRAL}, {33, 0.7f, false, 0.f, BEND_DS},
                        {50, 1.3f, true, 2e-3f, BEND_DIHEDRAL}, {64, 1.f, false, 0.f, BEND_NONE}};
  int identical = 0;
  for (const Case& c : cases) {
    Grid g = grid(c.side, c.len, c.pinned, c.jitter, 7u + unsigned(c.side));
    symbolic_cache_set_limit(0);
    std::vector<char> fresh = analyse(g, c.bending);
    symbolic_cache_set_limit(uint64_t(1) << 30);
    std::vector<char> first = analyse(g, c.bending);   // computed, then kept
    symbolic_cache_info(&h0, &m0, &b0, &e0);
    std::vector<char> again = analyse(g, c.bending);   // served by the cache
    symbolic_cache_info(&h1, &m1, &b1, &e1);
    bool ok = fresh == first && first == again && h1 == h0 + 1 && m1 == m0 && e1 == e0;
    identical += ok;
    failures += !ok;
  }
  // scaled copies of one grid: one entry, hits for every other scale
  symbolic_cache_set_limit(0);
  symbolic_cache_set_limit(uint64_t(1) << 30);
  symbolic_cache_info(&h0, &m0, nullptr, nullptr);
  std::vector<char> base;
  int scaled_same = 0, scales = 0;
  for (float len = 0.5f; len <= 2.01f; len += 0.25f, ++scales) {
    std::vector<char> b = analyse(grid(40, len, true, 0.f, 1), BEND_DIHEDRAL);
    if (base.empty()) base = b;
    scaled_same += (b == base);
  }
  symbolic_cache_info(&h1, &m1, &b1, &e1);
  bool scaled_ok = scaled_same == scales && m1 - m0 == 1 && h1 - h0 == uint64_t(scales - 1) && e1 == 1;
  failures += !scaled_ok;
  // concurrent set-ups of one mesh: one analysis, the same result everywhere
  symbolic_cache_set_limit(0);
  symbolic_cache_set_limit(uint64_t(1) << 30);
  symbolic_cache_info(&h0, &m0, nullptr, nullptr);
  Grid shared = grid(90, 1.f, true, 0.f, 3);
  std::vector<std::vector<char>> got(8);
  {
    std::vector<std::thread> ts;
    for (int k = 0; k < 8; ++k) ts.emplace_back([&, k] { got[k] = analyse(shared, BEND_DIHEDRAL); });
    for (auto& t : ts) t.join();
  }
  symbolic_cache_info(&h1, &m1, nullptr, nullptr);
  int concurrent_same = 0;
  for (auto& b : got) concurrent_same += (b == got[0]);
  bool concurrent_ok = concurrent_same == 8 && m1 - m0 == 1 && h1 - h0 == 7;
  failures += !concurrent_ok;
  symbolic_cache_set_limit(0);
  symbolic_cache_set_limit(uint64_t(1) << 30);
  analyse(grid(40, 1.f, true, 0.f, 1), BEND_DIHEDRAL);
  symbolic_cache_info(nullptr, nullptr, &b1, nullptr);
  // byte bound: room for one entry of this size evicts the older one
  uint64_t one = b1;
  symbolic_cache_set_limit(one + one / 2);
  analyse(grid(41, 1.f, true, 0.f, 1), BEND_DIHEDRAL);
  uint64_t b2, e2;
  symbolic_cache_info(nullptr, nullptr, &b2, &e2);
  bool evict_ok = e2 == 1 && b2 <= one + one / 2;
  symbolic_cache_set_limit(0);
  uint64_t b3, e3;
  symbolic_cache_info(nullptr, nullptr, &b3, &e3);
  bool zero_ok = b3 == 0 && e3 == 0;
  failures += !evict_ok + !zero_ok;
  std::printf("{\"identical\": %d, \"cases\": %d, \"scaled_same\": %d, \"scales\": %d, \"scaled_ok\": %d, "
              "\"concurrent_ok\": %d, \"evict_ok\": %d, \"zero_ok\": %d}\n",
              identical, int(sizeof(cases) / sizeof(cases[0])), scaled_same, scales, int(scaled_ok),
              int(concurrent_ok), int(evict_ok),
              int(zero_ok));
  return failures ? 1 : 0;
}
