// CPU check of o2f::qdiv and o2f::qdiv_flag (optimisation2forme_b200/csrc/qdiv.h):
// the quotient from a shared reciprocal must equal the IEEE division a/b bit
// for bit, and qdiv_flag must flag exactly the quotients qdiv sends to a/b.
//
// Three sets of cases:
//   random   random 53-bit significands, signs and exponents (a narrow and a
//            wide exponent range, so the fallback ranges are crossed too);
//   hard     quotients that lie as close to a rounding midpoint as two
//            53-bit operands allow: a = A, b = B with A * 2^j - B * M = +-1
//            (or a small odd k) for an odd 54-bit M, so a/b sits 1/(B 2^j)
//            from the midpoint M / 2^j; the divisors include the
//            significands just below 2 and just above 1 where RN(1/b) is
//            least accurate relative to b;
//   special  zeros, infinities, NaNs, subnormals and extreme magnitudes.
//
// Usage: qdiv_check [n_random] [n_hard] [seed]; prints the counts, exits 1
// on the first mismatches.
#include <cinttypes>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <limits>

#include "qdiv.h"

namespace {

using u128 = unsigned __int128;
using i128 = __int128;

uint64_t g_state = 0x9e3779b97f4a7c15ull;
uint64_t next_u64() {  // splitmix64
  uint64_t z = (g_state += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

uint64_t bits(double x) {
  uint64_t u;
  std::memcpy(&u, &x, 8);
  return u;
}

long g_bad = 0;
long g_flagged = 0;
bool equal_bits(double x, double y) { return (std::isnan(x) && std::isnan(y)) || bits(x) == bits(y); }

// qdiv must equal a/b; qdiv_flag must equal a/b whenever it leaves ok set,
// and clear ok exactly when qdiv takes its fallback.
bool same(double a, double b) {
  const double ref = a / b;
  const double y = o2f::recip_for_div(b);
  const double got = o2f::qdiv(a, b, y);
  bool ok = true;
  const double got_flag = o2f::qdiv_flag(a, b, y, ok);
  const double q0 = a * y;
  const bool in_range = std::fabs(q0) >= 0x1p-400 && std::fabs(q0) <= 0x1p+400;
  if (!ok) ++g_flagged;
  const bool good = equal_bits(ref, got) && ok == in_range && (!ok || equal_bits(ref, got_flag)) &&
                    equal_bits(y, o2f::recip_for_div(b, 1.0 / b));
  if (good) return true;
  if (g_bad++ < 10)
    std::printf("MISMATCH a=%a b=%a ref=%a got=%a flag=%a ok=%d\n", a, b, ref, got, got_flag, (int)ok);
  return false;
}

double random_double(int emin, int emax) {
  const uint64_t mant = (next_u64() >> 12) | (1ull << 52);  // 53-bit significand
  const int e = emin + (int)(next_u64() % (uint64_t)(emax - emin + 1));
  const double x = std::ldexp((double)mant, e - 52);
  return (next_u64() & 1) ? -x : x;
}

// Inverse of x modulo m (m odd, gcd(x, m) = 1).
uint64_t inv_mod(uint64_t x, uint64_t m) {
  i128 r0 = m, r1 = x % m, s0 = 0, s1 = 1;
  while (r1 != 0) {
    const i128 q = r0 / r1;
    i128 t = r0 - q * r1;
    r0 = r1;
    r1 = t;
    t = s0 - q * s1;
    s0 = s1;
    s1 = t;
  }
  if (s0 < 0) s0 += m;
  return (uint64_t)s0;
}

// For the odd 53-bit significand B, every 53-bit A with A * 2^j = B * M + k,
// M odd and 54 bits (a/b then lies k / (B 2^j) from the midpoint M / 2^j).
// Each pair is checked at a few exponent offsets and all four sign choices.
long hard_cases_for(uint64_t B, int j, long k, long* checked) {
  long bad = 0;
  const u128 pow2j = (u128)1 << j;
  const uint64_t p = (uint64_t)(pow2j % B);
  const uint64_t kk = (uint64_t)((k % (long)B + (long)B) % (long)B);
  // A = k * inv(2^j) mod B, plus multiples of B inside [2^52, 2^53).
  const uint64_t a0 = (uint64_t)(((u128)kk * inv_mod(p, B)) % B);
  for (uint64_t A = a0; A < (1ull << 53); A += B) {
    if (A < (1ull << 52)) continue;
    const i128 num = (i128)((u128)A << j) - (i128)k;
    if (num % (i128)B != 0) continue;
    const i128 M = num / (i128)B;
    if ((M & 1) == 0 || M < ((i128)1 << 53) || M >= ((i128)1 << 54)) continue;
    for (int ea : {0, 37, -41}) {
      for (int eb : {0, -29, 53}) {
        const double a = std::ldexp((double)A, ea), b = std::ldexp((double)B, eb);
        for (int s = 0; s < 4; ++s) {
          ++*checked;
          if (!same((s & 1) ? -a : a, (s & 2) ? -b : b)) ++bad;
        }
      }
    }
  }
  return bad;
}

}  // namespace

int main(int argc, char** argv) {
  const long n_random = argc > 1 ? std::atol(argv[1]) : 2000000;
  const long n_hard = argc > 2 ? std::atol(argv[2]) : 20000;
  if (argc > 3) g_state = std::strtoull(argv[3], nullptr, 10);

  long checked = 0;
  // random: operands of the residual's magnitudes, then the full range
  for (long i = 0; i < n_random; ++i) {
    ++checked;
    same(random_double(-40, 40), random_double(-40, 40));
    ++checked;
    same(random_double(-1074, 1023), random_double(-1074, 1023));
  }
  const long random_checked = checked;

  // hard: odd divisors near 2 (largest relative error of RN(1/b)), near 1,
  // and random; j chosen so that A * 2^j / B has 54 bits
  long hard_checked = 0;
  for (long i = 0; i < n_hard; ++i) {
    uint64_t B;
    switch (i % 3) {
      case 0: B = ((1ull << 53) - 1) - 2 * (next_u64() % (1ull << 20)); break;
      case 1: B = (1ull << 52) + 1 + 2 * (next_u64() % (1ull << 20)); break;
      default: B = ((next_u64() >> 11) | (1ull << 52)) | 1ull; break;
    }
    const long k = (i & 8) ? 3 : 1;
    for (int j : {53, 54}) {
      hard_cases_for(B, j, k, &hard_checked);
      hard_cases_for(B, j, -k, &hard_checked);
    }
  }
  checked += hard_checked;

  // special values
  const double inf = std::numeric_limits<double>::infinity();
  const double nan = std::numeric_limits<double>::quiet_NaN();
  const double dmin = std::numeric_limits<double>::denorm_min();
  const double nmin = std::numeric_limits<double>::min();
  const double dmax = std::numeric_limits<double>::max();
  const double vals[] = {0.0, -0.0, 1.0, -1.0, 3.0, 0.1, -7.5e-300, 1e300, inf, -inf, nan, dmin, -dmin,
                         nmin, 3 * nmin, dmax, -dmax, 0x1p-500, 0x1p+500, 0x1.0000000000001p-400,
                         0x1.fffffffffffffp+399, 1e-160, 1e160};
  long special_checked = 0;
  for (double a : vals)
    for (double b : vals) {
      ++special_checked;
      same(a, b);
    }
  checked += special_checked;

  std::printf("qdiv_check: %ld random, %ld hard, %ld special, %ld mismatches (%ld sent to the fallback)\n",
              random_checked, hard_checked, special_checked, g_bad, g_flagged);
  return g_bad == 0 ? 0 : 1;
}
