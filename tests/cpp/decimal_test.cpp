// Host check of the device decimal conversion (sparseops_b200/csrc/decimal.cuh)
// against the C library's strtod, which scanf("%lf") -- the reference's Matrix
// Market reader -- uses: every token must give the same bits.
//
// Cases: random doubles printed with 3..40 significant digits; random digit
// strings with random exponents (over- and underflow included); the exact
// decimal expansions of midpoints between neighbouring doubles and strings a
// hair above and below them (these take the big-integer pass); fixed edge
// cases.  Usage: decimal_test [random cases]
#include <cfloat>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>

#include "decimal.cuh"

using namespace spops::dec;

static std::vector<Pow10> g_tab;
static long g_fast = 0, g_dd = 0, g_big = 0, g_fail = 0, g_count = 0;

static bool parse(const std::string& s, double* out) {
  Decimal d;
  if (!scan_decimal(s.data(), s.data() + s.size(), &d)) return false;
  double cand = 0;
  if (fast_value(d, g_tab.data(), out, &cand)) {
    ++g_fast;
    return true;
  }
  ++g_big;
  static Big L, R;
  return big_round(s.data(), s.data() + s.size(), cand, out, L, R);
}

static void check(const std::string& s) {
  ++g_count;
  double got = 0;
  const bool ok = parse(s, &got);
  const double want = std::strtod(s.c_str(), nullptr);
  uint64_t a, b;
  std::memcpy(&a, &got, 8);
  std::memcpy(&b, &want, 8);
  const bool same = ok && (a == b || (std::isnan(got) && std::isnan(want) && std::signbit(got) == std::signbit(want)));
  if (!same) {
    if (g_fail < 20) std::printf("MISMATCH %s: got %.17g (%d) want %.17g\n", s.c_str(), got, (int)ok, want);
    ++g_fail;
  }
}

int main(int argc, char** argv) {
  const long n = argc > 1 ? std::atol(argv[1]) : 200000;
  g_tab = make_pow10_table();
  std::mt19937_64 rng(12345);
  char buf[2048];
  // fixed edge cases
  const char* fixed[] = {"0", "-0", "0.0", "1", "-1", "1e0", "1E+0", ".5", "5.", "+3.25", "1e-400", "1e400",
                         "2.2250738585072011e-308", "2.2250738585072014e-308", "4.9406564584124654e-324",
                         "2.4703282292062327e-324", "2.4703282292062328e-324", "1.7976931348623157e308",
                         "1.7976931348623158e308", "1.7976931348623159e308", "9007199254740993",
                         "9007199254740992.5", "0.1", "0.3", "123456789012345678901234567890", "inf", "-Infinity",
                         "NaN", "-nan", "1e22", "1e23", "8.98846567431158e307", "0.000000000000000000000000001",
                         "3.14159265358979323846264338327950288419716939937510582097494459",
                         "1.00000000000000011102230246251565404236316680908203125",
                         "1.00000000000000011102230246251565404236316680908203124",
                         "1.00000000000000011102230246251565404236316680908203126"};
  for (const char* f : fixed) check(f);
  std::uniform_int_distribution<int> prec(3, 40), len(1, 40), dig(0, 9), exd(-350, 330);
  for (long i = 0; i < n; ++i) {
    // a random finite double, printed at a random precision
    uint64_t bits = rng() & 0x7fffffffffffffffULL;
    if (((bits >> 52) & 0x7ff) == 0x7ff) bits &= ~((uint64_t)1 << 62);
    double x;
    std::memcpy(&x, &bits, 8);
    if (rng() & 1) x = -x;
    std::snprintf(buf, sizeof buf, (rng() & 1) ? "%.*g" : "%.*e", prec(rng), x);
    check(buf);
    std::snprintf(buf, sizeof buf, "%.17g", x);
    check(buf);
    // a random digit string with a decimal point and exponent
    std::string s;
    const int L = len(rng), dp = (int)(rng() % (uint64_t)(L + 1));
    for (int k = 0; k < L; ++k) {
      if (k == dp) s += '.';
      s += (char)('0' + dig(rng));
    }
    s += "e" + std::to_string(exd(rng));
    check(s);
    // the exact midpoint between x and its upper neighbour, and a hair either side
    if (i % 8 == 0) {
      const double ax = std::fabs(x);
      const double up = std::nextafter(ax, INFINITY);
      if (std::isfinite(up)) {
        const long double mid = ((long double)ax + (long double)up) / 2;
        std::snprintf(buf, sizeof buf, "%.780Le", mid);
        std::string m(buf);
        check(m);
        const size_t epos = m.find('e');
        std::string lo = m, hi = m;
        // strip trailing zeros of the mantissa, then nudge the last digit
        size_t last = epos - 1;
        while (last > 0 && m[last] == '0') --last;
        hi.insert(last + 1, "1");
        check(hi);
        if (lo[last] != '.' && lo[last] > '0') {
          lo[last] = (char)(lo[last] - 1);
          lo.insert(last + 1, "9999");
          check(lo);
        }
      }
    }
  }
  // integers
  long ifail = 0;
  for (long i = 0; i < n / 10; ++i) {
    const int64_t v = (int64_t)(rng() >> (rng() % 63));
    std::snprintf(buf, sizeof buf, "%" PRId64, (rng() & 1) ? -v : v);
    int64_t got = 0;
    if (!parse_int64(buf, buf + std::strlen(buf), &got) || got != std::strtoll(buf, nullptr, 10)) ++ifail;
  }
  std::printf("tokens %ld  fast-or-dd %ld  exact pass %ld  mismatches %ld  integer mismatches %ld\n", g_count,
              g_fast, g_big, g_fail, ifail);
  (void)g_dd;
  return (g_fail || ifail) ? 1 : 0;
}
