// Checks utl::pieces::cut_pieces (the host-buffer pipeline's batch cut) on
// seeded random stream tables: the pieces partition the values and blocks
// in order, each piece's table describes exactly its sub-streams, a cut
// inside a stream falls on a multiple of 128 values from the stream's
// start, and the pieces' blocks laid end to end are the batch's blocks.
// Prints "ok <cases>" or the first failure and exits non-zero.
#include <stdint.h>
#include <stdio.h>

#include <random>
#include <utility>
#include <vector>

#include "utl_pieces.h"

using utl::pieces::Piece;

static int fail(int c, const char* what) {
  printf("case %d: %s\n", c, what);
  return 1;
}

int main() {
  std::mt19937_64 rng(20240601);
  const uint64_t B = utl::pieces::kBlockValues;
  int cases = 0;
  for (int c = 0; c < 4000; c++) {
    const int ns = 1 + (int)(rng() % 40);
    std::vector<uint64_t> vo(ns + 1);
    vo[0] = rng() % 500;
    for (int s = 0; s < ns; s++) {
      uint64_t len = rng() % 5 == 0 ? 0 : rng() % (rng() % 2 ? 300 : 6000);
      vo[s + 1] = vo[s] + len;
    }
    const uint64_t nv = vo[ns] - vo[0];
    if (nv == 0) continue;
    const uint64_t targets[4] = {B, 2 * B, (nv + 7) / 8, 1000};
    uint64_t target = targets[rng() % 4];
    target = (target + B - 1) / B * B;
    std::vector<Piece> ps;
    std::vector<uint64_t> tab;
    utl::pieces::cut_pieces(vo.data(), ns, target, ps, tab);
    cases++;
    // the whole batch's blocks, as value ranges
    std::vector<std::pair<uint64_t, uint64_t>> whole, got;
    int64_t nb = 0;
    for (int s = 0; s < ns; s++)
      for (uint64_t x = vo[s]; x < vo[s + 1]; x += B) {
        whole.push_back({x, x + B < vo[s + 1] ? x + B : vo[s + 1]});
        nb++;
      }
    if (ps.empty()) return fail(c, "no pieces");
    if (ps.front().v0 != vo[0] || ps.back().v1 != vo[ns] || ps.back().b1 != nb) return fail(c, "ends");
    size_t entries = 0;
    for (size_t k = 0; k < ps.size(); k++) {
      const Piece& q = ps[k];
      if (k && (q.v0 != ps[k - 1].v1 || q.b0 != ps[k - 1].b1)) return fail(c, "not contiguous");
      if (q.ns < 1 || q.v1 - q.v0 > target) return fail(c, "piece size");
      if (q.t0 + q.ns + 1 > tab.size() || tab[q.t0] != 0 || tab[q.t0 + q.ns] != q.v1 - q.v0) return fail(c, "table");
      entries += q.ns + 1;
      int64_t blocks = 0;
      for (int i = 0; i < q.ns; i++) {
        const uint64_t a = q.v0 + tab[q.t0 + i], b = q.v0 + tab[q.t0 + i + 1];
        if (b <= a) return fail(c, "empty sub-stream");
        for (uint64_t x = a; x < b; x += B) got.push_back({x, x + B < b ? x + B : b});
        blocks += (int64_t)((b - a + B - 1) / B);
      }
      if (blocks != q.b1 - q.b0) return fail(c, "block count");
    }
    if (entries != tab.size()) return fail(c, "table size");
    if (got != whole) return fail(c, "blocks differ from the batch's");
  }
  printf("ok %d\n", cases);
  return 0;
}
