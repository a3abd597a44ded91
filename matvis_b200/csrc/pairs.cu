// Redundant-baseline pair selection (host code; no device work).
//
// Restates get_redundancies (cli.py:273-290): baselines are rounded to
// `ndecimals` decimals as numpy's round does (x * 10^d, round half to even,
// / 10^d; for d < 0 the divide and multiply swap), and pairs (i, j), i < j, are
// visited with i slow; a pair is kept when neither its rounded (u, v) nor
// (-u, -v) has been kept before.  Both signs of a baseline form one class, so
// a hash set holds one canonical member per class (the larger of the two in
// lexicographic order, with -0.0 folded into +0.0).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_set>

#include "common.cuh"

using mvb::fail;

namespace {

inline uint64_t bits(double x) {
  x += 0.0;  // -0.0 -> +0.0
  uint64_t b;
  std::memcpy(&b, &x, sizeof b);
  return b;
}

struct ClassKey {
  uint64_t u, v;
  bool operator==(const ClassKey &o) const { return u == o.u && v == o.v; }
};

struct ClassHash {
  size_t operator()(const ClassKey &k) const {
    uint64_t h = k.u * 0x9E3779B97F4A7C15ull;
    h ^= (k.v + 0x632BE59BD9B4E019ull + (h << 6) + (h >> 2));
    return (size_t)(h ^ (h >> 31));
  }
};

inline double round_decimals(double x, int nd, double scale) {
  if (nd >= 0) return std::nearbyint(x * scale) / scale;
  return std::nearbyint(x / scale) * scale;
}

}  // namespace

extern "C" int mvb_redundant_pairs(const double *bls, int64_t nant, int ndecimals, int32_t *pairs_out, int64_t cap,
                                   int64_t *n_out) {
  if (nant < 0 || !n_out || (nant > 0 && !bls) || cap < 0 || (cap > 0 && !pairs_out))
    return fail(MVB_ERR_ARG, "mvb_redundant_pairs: bad arguments");
  if (nant > INT32_MAX) return fail(MVB_ERR_ARG, "mvb_redundant_pairs: too many antennas");
  if (ndecimals < -22 || ndecimals > 22) return fail(MVB_ERR_ARG, "mvb_redundant_pairs: ndecimals out of range");
  // 10^|d| is exact in double for |d| <= 22, as numpy's integer power converted to float is
  double scale = 1.0;
  for (int k = 0; k < std::abs(ndecimals); ++k) scale *= 10.0;
  std::unordered_set<ClassKey, ClassHash> seen;
  int64_t n = 0;
  for (int64_t i = 0; i < nant; ++i) {
    for (int64_t j = i + 1; j < nant; ++j) {
      const double *b = bls + 2 * (i * nant + j);
      const double u = round_decimals(b[0], ndecimals, scale), v = round_decimals(b[1], ndecimals, scale);
      if (std::isnan(u) || std::isnan(v)) return fail(MVB_ERR_ARG, "mvb_redundant_pairs: non-finite baseline");
      const double nu = -u, nv = -v;
      const bool pos = (u > nu) || (u == nu && v >= nv);
      const ClassKey key = pos ? ClassKey{bits(u), bits(v)} : ClassKey{bits(nu), bits(nv)};
      if (seen.insert(key).second) {
        if (n < cap) {
          pairs_out[2 * n] = (int32_t)i;
          pairs_out[2 * n + 1] = (int32_t)j;
        }
        ++n;
      }
    }
  }
  *n_out = n;
  if (n > cap) return fail(MVB_ERR_OVERFLOW, "mvb_redundant_pairs: output capacity too small");
  return MVB_OK;
}
