// Decimal text to IEEE double / int64, correctly rounded (to nearest, ties to
// even) as C's strtod and scanf("%lf") convert, for the device Matrix Market
// reader (mtx.cu).  Everything is __host__ __device__ so that a test program
// can compare these functions with the C library on the host.
//
// A decimal D * 10^q (D = all significant digits) becomes a double in one of
// three ways:
//   1. exact: D <= 2^53 and |q| <= 22 -- one correctly rounded IEEE multiply
//      or divide of two exact operands (Clinger's fast path);
//   2. double-double: the first 19 digits w times 10^q from a table of
//      (hi + lo) * 2^e (the leading 107 bits of 10^q, made with big-integer
//      arithmetic on the host) give the value to about 2^-100 relative; unless
//      that lies within 2^-93 of a rounding midpoint its rounding is the
//      answer (with more than 19 digits, w and w + 1 must round alike);
//   3. otherwise big_round() decides exactly, comparing D * 10^q with the
//      midpoints around a nearby double as integers (rare; the reader runs it
//      as a separate pass over the tokens the first two left open).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef __CUDACC__
#define SPOPS_HD __host__ __device__ __forceinline__
#define SPOPS_HDN __host__ __device__
#else
#define SPOPS_HD inline
#define SPOPS_HDN inline
#endif

namespace spops {
namespace dec {

constexpr int kPowMin = -360, kPowMax = 320;
constexpr int kPowCount = kPowMax - kPowMin + 1;
constexpr int kMaxDigits = 800;  // significant digits the exact pass accepts

// 10^q = (hi + lo) * 2^e2 with 1 <= hi < 2 and |lo| <= ulp(hi) / 2
struct Pow10 {
  double hi, lo;
  int32_t e2;
  int32_t pad;
};

// ------------------------------------------------------------ host table
namespace host_big {  // little-endian 32-bit limbs
inline void mul_small(std::vector<uint32_t>& a, uint32_t m) {
  uint64_t c = 0;
  for (auto& x : a) {
    const uint64_t t = (uint64_t)x * m + c;
    x = (uint32_t)t;
    c = t >> 32;
  }
  if (c) a.push_back((uint32_t)c);
}
inline int bit_length(const std::vector<uint32_t>& a) {
  for (int i = (int)a.size() - 1; i >= 0; --i)
    if (a[(size_t)i]) {
      int b = 31;
      while (!((a[(size_t)i] >> b) & 1u)) --b;
      return i * 32 + b + 1;
    }
  return 0;
}
inline uint64_t bit(const std::vector<uint32_t>& a, int i) {
  return (i >= 0 && (size_t)(i >> 5) < a.size()) ? (uint64_t)((a[(size_t)(i >> 5)] >> (i & 31)) & 1u) : 0;
}
inline int cmp(const std::vector<uint32_t>& a, const std::vector<uint32_t>& b) {
  const size_t n = a.size() > b.size() ? a.size() : b.size();
  for (size_t i = n; i-- > 0;) {
    const uint32_t x = i < a.size() ? a[i] : 0, y = i < b.size() ? b[i] : 0;
    if (x != y) return x < y ? -1 : 1;
  }
  return 0;
}
inline void sub(std::vector<uint32_t>& a, const std::vector<uint32_t>& b) {  // a -= b (a >= b)
  int64_t br = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    int64_t t = (int64_t)a[i] - (i < b.size() ? (int64_t)b[i] : 0) - br;
    br = t < 0;
    if (t < 0) t += (int64_t)1 << 32;
    a[i] = (uint32_t)t;
  }
}
inline void shl1(std::vector<uint32_t>& a) {
  uint32_t c = 0;
  for (auto& x : a) {
    const uint32_t n = x >> 31;
    x = (x << 1) | c;
    c = n;
  }
  if (c) a.push_back(c);
}
}  // namespace host_big

// hi + lo from the leading 107 bits of a mantissa, m1 (53 bits, the top one
// set) followed by m2 (54 bits); truncated
inline void split107(uint64_t m1, uint64_t m2, double* hi, double* lo) {
  const double h = (double)m1 * 0x1p-52;   // [1, 2)
  const double l = (double)m2 * 0x1p-106;  // < ulp(h)
  const double s = h + l;
  *lo = l - (s - h);
  *hi = s;
}

inline std::vector<Pow10> make_pow10_table() {
  using namespace host_big;
  std::vector<Pow10> t((size_t)kPowCount);
  std::vector<uint32_t> p(1, 1u);  // 10^q, q >= 0: exact
  for (int q = 0; q <= kPowMax; ++q) {
    const int nb = bit_length(p);
    uint64_t m1 = 0, m2 = 0;
    for (int i = 0; i < 53; ++i) m1 = (m1 << 1) | bit(p, nb - 1 - i);
    for (int i = 0; i < 54; ++i) m2 = (m2 << 1) | bit(p, nb - 54 - i);
    Pow10& e = t[(size_t)(q - kPowMin)];
    split107(m1, m2, &e.hi, &e.lo);
    e.e2 = nb - 1;
    e.pad = 0;
    mul_small(p, 10u);
  }
  std::vector<uint32_t> den(1, 1u);  // 10^-q: binary long division of 2^s by 10^q
  for (int q = 1; q <= -kPowMin; ++q) {
    mul_small(den, 10u);
    std::vector<uint32_t> rem(1, 1u);
    int s = 0;
    while (cmp(rem, den) < 0) {
      shl1(rem);
      ++s;
    }
    uint64_t m1 = 0, m2 = 0;
    for (int i = 0; i < 107; ++i) {
      uint64_t qb = 0;
      if (cmp(rem, den) >= 0) {
        sub(rem, den);
        qb = 1;
      }
      if (i < 53) m1 = (m1 << 1) | qb; else m2 = (m2 << 1) | qb;
      shl1(rem);
    }
    Pow10& e = t[(size_t)(-q - kPowMin)];
    split107(m1, m2, &e.hi, &e.lo);
    e.e2 = -s;
    e.pad = 0;
  }
  return t;
}

// ------------------------------------------------------- double-double
struct DD {
  double hi, lo;
};
SPOPS_HD DD quick_two_sum(double a, double b) {
  const double s = a + b;
  return DD{s, b - (s - a)};
}
SPOPS_HD DD dd_mul(DD a, DD b) {
  const double p = a.hi * b.hi;
  double e = fma(a.hi, b.hi, -p);
  e += a.hi * b.lo + a.lo * b.hi;
  return quick_two_sum(p, e);
}
SPOPS_HD double from_bits(uint64_t b) {
  double d;
  memcpy(&d, &b, 8);
  return d;
}
SPOPS_HD uint64_t to_bits(double d) {
  uint64_t b;
  memcpy(&b, &d, 8);
  return b;
}
SPOPS_HD double inf_value() { return from_bits(0x7ff0000000000000ULL); }
SPOPS_HD double nan_value() { return from_bits(0x7ff8000000000000ULL); }
SPOPS_HD double pow2(int k) {  // 2^k, -1074 <= k <= 1023, exact
  return k >= -1022 ? from_bits((uint64_t)(k + 1023) << 52) : from_bits((uint64_t)1 << (k + 1074));
}
SPOPS_HD double scale2(double x, int k) {  // x * 2^k in steps that stay exact
  while (k > 1000) {
    x *= pow2(1000);
    k -= 1000;
  }
  while (k < -1000) {
    x *= pow2(-1000);
    k += 1000;
  }
  return x * pow2(k);
}

// ------------------------------------------------------------- tokens
struct Decimal {
  bool neg = false, special = false, trunc = false;
  double special_value = 0;
  uint64_t w = 0;  // first (up to 19) significant digits
  int nw = 0;      // digits in w
  int nd = 0;      // all significant digits
  int64_t q = 0;   // value = w * 10^q, plus the truncated digits
};

SPOPS_HD char lower_ascii(char c) { return (c >= 'A' && c <= 'Z') ? (char)(c + 32) : c; }
SPOPS_HD bool word_is(const char* p, const char* e, const char* w) {
  while (*w) {
    if (p >= e || lower_ascii(*p) != *w) return false;
    ++p;
    ++w;
  }
  return p == e;
}

// The whole token [p, e) in strtod's decimal syntax -- [+-] digits [. digits]
// [(e|E) [+-] digits] -- or inf, infinity, nan (any case).  False for anything
// else, the hexadecimal forms included.
SPOPS_HD bool scan_decimal(const char* p, const char* e, Decimal* d) {
  if (p < e && (*p == '+' || *p == '-')) {
    d->neg = *p == '-';
    ++p;
  }
  if (p < e && (lower_ascii(*p) == 'i' || lower_ascii(*p) == 'n')) {
    d->special = true;
    if (word_is(p, e, "inf") || word_is(p, e, "infinity")) {
      d->special_value = d->neg ? -inf_value() : inf_value();
      return true;
    }
    if (word_is(p, e, "nan")) {
      d->special_value = d->neg ? -nan_value() : nan_value();
      return true;
    }
    return false;
  }
  bool any = false, dot = false;
  int64_t adj = 0;
  for (; p < e; ++p) {
    const char c = *p;
    if (c == '.') {
      if (dot) return false;
      dot = true;
      continue;
    }
    if (c < '0' || c > '9') break;
    any = true;
    const int dg = c - '0';
    if (d->nd == 0 && dg == 0) {  // a leading zero
      if (dot) --adj;
      continue;
    }
    ++d->nd;
    if (d->nw < 19) {
      d->w = d->w * 10 + (uint64_t)dg;
      ++d->nw;
      if (dot) --adj;
    } else {
      if (dg) d->trunc = true;
      if (!dot) ++adj;
    }
  }
  if (!any) return false;
  int64_t ex = 0;
  if (p < e && (*p == 'e' || *p == 'E')) {
    ++p;
    bool en = false;
    if (p < e && (*p == '+' || *p == '-')) {
      en = *p == '-';
      ++p;
    }
    if (p >= e || *p < '0' || *p > '9') return false;
    for (; p < e && *p >= '0' && *p <= '9'; ++p)
      if (ex < 100000000) ex = ex * 10 + (*p - '0');
    if (en) ex = -ex;
  }
  if (p != e) return false;
  d->q = adj + ex;
  return true;
}

// The rounding of m * 2^eb (m a double-double within 2^-100 of the true
// mantissa, 1 <= m.hi < 2) to a double, or false when the true value may lie
// on the other side of a rounding midpoint.
SPOPS_HD bool dd_round(DD m, int64_t eb, double* out) {
  const double margin = 0x1p-93;
  if (eb > 1023) {
    *out = inf_value();
    return true;
  }
  if (eb >= -1022) {  // normal: midpoints at hi +- ulp/2 (ulp/4 below a power of two)
    const double a = m.lo < 0 ? -m.lo : m.lo;
    const double half = (m.lo < 0 && m.hi == 1.0) ? 0x1p-54 : 0x1p-53;
    if (half - a <= margin) return false;
    *out = scale2(m.hi, (int)eb);
    return true;
  }
  // subnormal: the grid is 2^-1074; s = m * 2^(eb + 1074) < 2^52
  const int sh = (int)(eb + 1074);
  if (sh <= -2) {  // below a quarter of the smallest subnormal
    *out = 0.0;
    return true;
  }
  const double sh_hi = scale2(m.hi, sh), sh_lo = scale2(m.lo, sh);
  const double n0 = floor(sh_hi);
  const double frac = (sh_hi - n0) + sh_lo;
  const double tol = (sh_hi + 1.0) * margin;
  if (fabs(frac - 0.5) <= tol || fabs(frac + 0.5) <= tol) return false;
  const double n = frac > 0.5 ? n0 + 1 : (frac < -0.5 ? n0 - 1 : n0);
  *out = n * pow2(-1074);  // exact
  return true;
}

// w * 10^q through the table, or false if that is not decisive
SPOPS_HD bool dd_value(uint64_t w, int64_t q, const Pow10* tab, double* out) {
  if (q < kPowMin || q > kPowMax) return false;
  const Pow10 P = tab[q - kPowMin];
  const double whi = (double)w;
  const double wlo = (double)(int64_t)(w - (uint64_t)whi);  // |w - whi| < 2^11: exact
  int ew = 0;
  for (double t = whi; t >= 2.0; t *= 0.5) ++ew;
  const double sc = pow2(-ew);
  DD x = dd_mul(DD{whi * sc, wlo * sc}, DD{P.hi, P.lo});
  int64_t eb = (int64_t)ew + P.e2;
  if (x.hi >= 2.0) {
    x.hi *= 0.5;
    x.lo *= 0.5;
    ++eb;
  } else if (x.hi < 1.0) {  // w just below a power of two rounded up in whi
    x.hi *= 2.0;
    x.lo *= 2.0;
    --eb;
  }
  return dd_round(x, eb, out);
}

// The value when the first two ways settle it (true); otherwise false with
// *cand a double within a few units of the answer.
SPOPS_HD bool fast_value(const Decimal& d, const Pow10* tab, double* out, double* cand) {
  *cand = 0;
  if (d.special) {
    *out = d.special_value;
    return true;
  }
  if (d.w == 0) {
    *out = d.neg ? -0.0 : 0.0;
    return true;
  }
  const int64_t lead = (int64_t)d.nw - 1 + d.q;  // decimal exponent of the leading digit
  if (lead > 309) {
    *out = d.neg ? -inf_value() : inf_value();
    return true;
  }
  if (lead < -326) {
    *out = d.neg ? -0.0 : 0.0;
    return true;
  }
  double v = 0;
  if (!d.trunc && d.w <= ((uint64_t)1 << 53) && d.q >= -22 && d.q <= 22) {
    double p10 = 1.0;
    for (int64_t i = 0; i < (d.q < 0 ? -d.q : d.q); ++i) p10 *= 10.0;  // exact up to 10^22
    v = d.q >= 0 ? (double)d.w * p10 : (double)d.w / p10;
    *out = d.neg ? -v : v;
    return true;
  }
  bool ok = dd_value(d.w, d.q, tab, &v);
  if (ok && d.trunc) {  // the dropped digits put the value between w and w + 1
    double v2 = 0;
    ok = dd_value(d.w + 1, d.q, tab, &v2) && v2 == v;
  }
  if (ok) {
    *out = d.neg ? -v : v;
    return true;
  }
  const int64_t qc = d.q < kPowMin ? kPowMin : (d.q > kPowMax ? kPowMax : d.q);
  const Pow10 P = tab[qc - kPowMin];
  const double c = scale2((double)d.w * P.hi, P.e2);
  *cand = d.neg ? -c : c;
  return false;
}

// ------------------------------------------------------ exact pass
constexpr int kBigLimbs = 240;  // 7680 bits: 800 digits, 10^1200 and 2^1100 fit
struct Big {
  uint32_t a[kBigLimbs];
  int n;
};
SPOPS_HD void big_set(Big& b, uint64_t v) {
  b.n = 0;
  while (v) {
    b.a[b.n++] = (uint32_t)v;
    v >>= 32;
  }
}
SPOPS_HD bool big_mul_add(Big& b, uint32_t m, uint32_t add) {
  uint64_t c = add;
  for (int i = 0; i < b.n; ++i) {
    const uint64_t t = (uint64_t)b.a[i] * m + c;
    b.a[i] = (uint32_t)t;
    c = t >> 32;
  }
  if (c) {
    if (b.n >= kBigLimbs) return false;
    b.a[b.n++] = (uint32_t)c;
  }
  return true;
}
SPOPS_HD bool big_pow10(Big& b, int64_t k) {
  for (; k >= 9; k -= 9)
    if (!big_mul_add(b, 1000000000u, 0)) return false;
  uint32_t m = 1;
  for (; k > 0; --k) m *= 10;
  return big_mul_add(b, m, 0);
}
SPOPS_HD bool big_shl(Big& b, int64_t s) {
  if (b.n == 0 || s == 0) return true;
  const int w = (int)(s / 32), r = (int)(s % 32);
  if (b.n + w + 1 > kBigLimbs) return false;
  if (r) {
    uint32_t c = 0;
    for (int i = 0; i < b.n; ++i) {
      const uint32_t n = b.a[i] >> (32 - r);
      b.a[i] = (b.a[i] << r) | c;
      c = n;
    }
    if (c) b.a[b.n++] = c;
  }
  if (w) {
    for (int i = b.n - 1; i >= 0; --i) b.a[i + w] = b.a[i];
    for (int i = 0; i < w; ++i) b.a[i] = 0;
    b.n += w;
  }
  return true;
}
SPOPS_HD int big_cmp(const Big& x, const Big& y) {
  if (x.n != y.n) return x.n < y.n ? -1 : 1;
  for (int i = x.n - 1; i >= 0; --i)
    if (x.a[i] != y.a[i]) return x.a[i] < y.a[i] ? -1 : 1;
  return 0;
}

// D * 10^qd (D the token's significant digits) against (2m + 1) * 2^(e - 1):
// -1 / 0 / +1, or -2 if the integers do not fit
SPOPS_HDN int cmp_midpoint(const char* p, const char* end, int64_t qd, uint64_t m, int e, Big& L, Big& R) {
  big_set(L, 0);
  int nd = 0;
  for (; p < end; ++p) {
    const char c = *p;
    if (c == 'e' || c == 'E') break;
    if (c < '0' || c > '9') continue;
    if (nd == 0 && c == '0') continue;
    if (++nd > kMaxDigits) return -2;
    if (L.n == 0) big_set(L, (uint64_t)(c - '0'));
    else if (!big_mul_add(L, 10u, (uint32_t)(c - '0'))) return -2;
  }
  big_set(R, 2 * m + 1);
  if (qd > 0 && !big_pow10(L, qd)) return -2;
  if (qd < 0 && !big_pow10(R, -qd)) return -2;
  if (e - 1 > 0 && !big_shl(R, e - 1)) return -2;
  if (e - 1 < 0 && !big_shl(L, 1 - (int64_t)e)) return -2;
  return big_cmp(L, R);
}

SPOPS_HD void mant_exp(uint64_t bits, uint64_t* m, int* e) {  // |x| = m * 2^e
  const int be = (int)((bits >> 52) & 0x7ff);
  *m = bits & (((uint64_t)1 << 52) - 1);
  if (be == 0) {
    *e = -1074;
  } else {
    *m |= (uint64_t)1 << 52;
    *e = be - 1075;
  }
}

// The correctly rounded value of the token [p, end), starting from a double
// within a few units; false if the token is not a decimal or has more than
// kMaxDigits significant digits.
SPOPS_HDN bool big_round(const char* p, const char* end, double cand, double* out, Big& L, Big& R) {
  Decimal d;
  if (!scan_decimal(p, end, &d) || d.special) return false;
  const int64_t qd = d.q - (d.nd - d.nw);  // value = D * 10^qd
  double c = cand < 0 ? -cand : cand;
  if (!(c > 0)) c = pow2(-1074);
  if (c > 1.7976931348623157e308) c = 1.7976931348623157e308;
  for (int step = 0; step < 64; ++step) {
    uint64_t b = to_bits(c), m;
    int e;
    mant_exp(b, &m, &e);
    const int up = cmp_midpoint(p, end, qd, m, e, L, R);  // against c + ulp/2
    if (up == -2) return false;
    if (up > 0 || (up == 0 && (m & 1))) {
      if (b == 0x7fefffffffffffffULL) {
        c = inf_value();
        break;
      }
      c = from_bits(b + 1);
      continue;
    }
    if (b == 0) break;
    uint64_t mlo;
    int elo;
    mant_exp(b - 1, &mlo, &elo);
    const int dn = cmp_midpoint(p, end, qd, mlo, elo, L, R);  // against the midpoint below c
    if (dn == -2) return false;
    if (dn < 0 || (dn == 0 && (mlo & 1) == 0)) {
      c = from_bits(b - 1);
      continue;
    }
    break;
  }
  *out = d.neg ? -c : c;
  return true;
}

// ------------------------------------------------------------- integers
// [+-]digits over the whole token (at most 19 digits)
SPOPS_HD bool parse_int64(const char* p, const char* e, int64_t* out) {
  bool neg = false;
  if (p < e && (*p == '+' || *p == '-')) {
    neg = *p == '-';
    ++p;
  }
  if (p >= e) return false;
  uint64_t v = 0;
  int n = 0;
  for (; p < e; ++p) {
    if (*p < '0' || *p > '9') return false;
    v = v * 10 + (uint64_t)(*p - '0');
    if (++n > 19) return false;
  }
  *out = neg ? -(int64_t)v : (int64_t)v;
  return true;
}

}  // namespace dec
}  // namespace spops
