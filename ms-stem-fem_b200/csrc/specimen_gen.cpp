// Seeded amorphous specimens: random sequential addition with a minimum
// periodic separation, on the host.  For benchmark and serving inputs of
// 10^5 - 10^6 atoms (the reference reads specimens from files and has no
// generator).
//
// Proposals are uniform in the box from std::mt19937_64 (u = (x >> 11) *
// 2^-53, so the sequence does not depend on the standard library's
// distributions); a proposal within min_sep of an accepted atom (periodic
// images included) is rejected.  Accepted atoms live in a cell list with
// cells no smaller than min_sep, so a test visits the 27 cells around the
// proposal.
#include <cmath>
#include <cstdint>
#include <random>
#include <string>
#include <vector>

#include "engine.hpp"
#include "msf.h"

extern "C" msf_status msf_amorphous_positions(int64_t n_atoms, const double* box, double min_sep,
                                              uint64_t seed, int64_t max_proposals,
                                              double* q) {
  using msf::set_error;
  if (n_atoms < 0 || !box || !q || !(min_sep >= 0) || box[0] <= 0 || box[1] <= 0 ||
      box[2] <= 0) {
    set_error("msf_amorphous_positions: invalid arguments");
    return MSF_ERR_ARG;
  }
  if (max_proposals <= 0) max_proposals = 1000 * (n_atoms + 1);
  int nc[3];
  double cell[3];
  for (int d = 0; d < 3; ++d) {
    nc[d] = min_sep > 0 ? std::max(1, (int)std::floor(box[d] / min_sep)) : 1;
    if (nc[d] > 1024) nc[d] = 1024;
    cell[d] = box[d] / nc[d];
  }
  const int64_t n_cells = (int64_t)nc[0] * nc[1] * nc[2];
  std::vector<std::vector<int32_t>> cells((size_t)n_cells);
  std::mt19937_64 rng(seed);
  auto uniform = [&rng] { return (double)(rng() >> 11) * (1.0 / 9007199254740992.0); };
  const double r2 = min_sep * min_sep;
  int64_t accepted = 0;
  for (int64_t tries = 0; accepted < n_atoms && tries < max_proposals; ++tries) {
    const double p[3] = {uniform() * box[0], uniform() * box[1], uniform() * box[2]};
    int c[3];
    for (int d = 0; d < 3; ++d) c[d] = std::min(nc[d] - 1, (int)(p[d] / cell[d]));
    bool ok = true;
    // with fewer than 3 cells along an axis, visit each cell once
    const int span[3] = {nc[0] >= 3 ? 1 : 0, nc[1] >= 3 ? 1 : 0, nc[2] >= 3 ? 1 : 0};
    for (int dx = -span[0]; dx <= span[0] && ok; ++dx)
      for (int dy = -span[1]; dy <= span[1] && ok; ++dy)
        for (int dz = -span[2]; dz <= span[2] && ok; ++dz) {
          auto wrap = [](int v, int n) { return (v % n + n) % n; };
          const int64_t idx = ((int64_t)wrap(c[0] + dx, nc[0]) * nc[1] + wrap(c[1] + dy, nc[1])) *
                                  nc[2] + wrap(c[2] + dz, nc[2]);
          const std::vector<int32_t>& list = cells[(size_t)idx];
          // cells spanning a whole short axis hold all its atoms: test them all
          for (int32_t a : list) {
            double s = 0;
            for (int d = 0; d < 3; ++d) {
              double dd = std::fabs(p[d] - q[3 * (int64_t)a + d]);
              dd = std::min(dd, box[d] - dd);
              s += dd * dd;
            }
            if (s < r2) {
              ok = false;
              break;
            }
          }
        }
    if (nc[0] < 3 || nc[1] < 3 || nc[2] < 3) {
      // short axes: the loops above skipped neighbouring cells; test every atom
      for (int64_t a = 0; a < accepted && ok; ++a) {
        double s = 0;
        for (int d = 0; d < 3; ++d) {
          double dd = std::fabs(p[d] - q[3 * a + d]);
          dd = std::min(dd, box[d] - dd);
          s += dd * dd;
        }
        if (s < r2) ok = false;
      }
    }
    if (!ok) continue;
    for (int d = 0; d < 3; ++d) q[3 * accepted + d] = p[d];
    const int64_t idx = ((int64_t)c[0] * nc[1] + c[1]) * nc[2] + c[2];
    cells[(size_t)idx].push_back((int32_t)accepted);
    ++accepted;
  }
  if (accepted < n_atoms) {
    set_error("msf_amorphous_positions: only " + std::to_string(accepted) + " of " +
              std::to_string(n_atoms) + " atoms placed within the proposal limit");
    return MSF_ERR_ARG;
  }
  return MSF_OK;
}
