// utl_pieces.h -- how a host-buffer batch is cut into pieces for the
// pipelined utl_pack_streams_* / utl_unpack_streams_* calls (host code only).
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <vector>

namespace utl {
namespace pieces {

constexpr uint64_t kBlockValues = 128;

// A piece of a host-buffer batch: values [v0, v1) and blocks [b0, b1) of
// the caller's arrays, as ns sub-streams whose value-offset table (ns + 1
// entries, rebased to v0) starts at tab[t0].
struct Piece {
  uint64_t v0, v1;
  int64_t b0, b1;
  size_t t0;
  int ns;
};

// Cut the batch into pieces of about `target` values.  A piece ends at a
// stream end or, inside a stream, at a multiple of 128 values from the
// stream's start: every block's bytes depend on its own values only, so a
// stream cut there packs to the same blocks and the pieces' outputs laid
// end to end are the whole batch's.
inline void cut_pieces(const uint64_t* vo, int n_streams, uint64_t target, std::vector<Piece>& ps,
                       std::vector<uint64_t>& tab) {
  const uint64_t B = kBlockValues;
  ps.clear();
  tab.clear();
  Piece p{vo[0], vo[0], 0, 0, 0, 0};
  tab.push_back(0);
  auto close = [&]() {
    ps.push_back(p);
    p = Piece{p.v1, p.v1, p.b1, p.b1, tab.size(), 0};
    tab.push_back(0);
  };
  for (int s = 0; s < n_streams; s++) {
    uint64_t left = vo[s + 1] - vo[s];
    while (left) {
      const uint64_t room = target - (p.v1 - p.v0);
      uint64_t take = left;
      if (take > room) {
        take = room / B * B;
        if (take == 0) {  // the piece holds more than target - 128 values
          close();
          continue;
        }
      }
      left -= take;
      p.v1 += take;
      p.b1 += (int64_t)((take + B - 1) / B);
      p.ns++;
      tab.push_back(p.v1 - p.v0);
      if (p.v1 - p.v0 == target) close();
    }
  }
  if (p.ns) ps.push_back(p);
  else tab.pop_back();
}

}  // namespace pieces
}  // namespace utl
