// Host check of the chi2 correlation orders (gtls_b200/csrc/chi2_core.cuh):
// correlate_rounds (a lane's offsets as overlapped rounds) must give the
// bitwise sums of correlate_pre applied offset by offset, and the clamped and
// unclamped forms of correlate_pre must agree where no read passes the tile.
// Prints one line per failure and "ok <cases>" at the end; exit status 1 on
// any failure.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "chi2_core.cuh"

using namespace gtls;

static bool same(const double2 (&a)[kR], const double2 (&b)[kR]) { return std::memcmp(a, b, sizeof(a)) == 0; }

int main() {
  std::mt19937_64 rng(12345);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  int cases = 0, bad = 0;
  const int skips[] = {32, 33, 47, 64, 100, 257, 1050};
  for (int s : skips) {
    for (int extra : {0, 3, 7}) {
      const int w = 8 * s + (extra < s ? extra : 0);
      const int Q = (w + s - 1) / s;
      const int Qr = (Q + kR - 1) / kR * kR;
      // template row: (s_i, s_i^2) for i < w, zeros up to (Qr + 1) * s
      std::vector<double2> trow((size_t)(Qr + 1) * s);
      for (size_t i = 0; i < trow.size(); ++i) {
        const double v = (int)i < w ? u(rng) : 0.0;
        trow[i] = make_double2(v, v * v);
      }
      // records of a tile: the task's reads reach base + (s - 1) + 16 s
      const int base = 5 * s + 3;
      const int L = base + 18 * s + 11;
      std::vector<double2> tile(L);
      for (auto& r : tile) r = make_double2(u(rng), 1.0 + 0.5 * u(rng));
      for (int lane = 0; lane < 32; ++lane) {
        double2 ref[kR], got[kR], clamped[kR];
        for (int r = 0; r < kR; ++r) ref[r] = got[r] = clamped[r] = make_double2(0.25 * u(rng), 0.25 * u(rng));
        for (int r = 0; r < kR; ++r) got[r] = clamped[r] = ref[r];
        for (int rho = lane; rho < s; rho += 32) {
          correlate_pre<double, false, false>(tile.data(), L, base + rho, s, trow.data(), rho, Q, ref);
          correlate_pre<double, false, true>(tile.data(), L, base + rho, s, trow.data(), rho, Q, clamped);
        }
        correlate_rounds<double>(tile.data(), base, s, trow.data(), lane, got);
        ++cases;
        if (!same(ref, got)) {
          ++bad;
          std::printf("rounds differ: s %d w %d lane %d\n", s, w, lane);
        }
        if (!same(ref, clamped)) {
          ++bad;
          std::printf("clamped differs: s %d w %d lane %d\n", s, w, lane);
        }
      }
    }
  }
  if (bad) return 1;
  std::printf("ok %d\n", cases);
  return 0;
}
