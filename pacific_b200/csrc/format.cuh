// format.cuh -- exact decimal formatting of doubles in C's "%.{P}e" form
// (what an iostream prints with std::scientific and precision P), on the
// device and on the host.
//
// The reference writes every double of its reload and RawData files through
// GrainsExec::doubleToString (Base/src/GrainsExec.cpp:213-225): scientific
// notation with P digits after the point (16 for reload files, Basic.hh:35;
// 6 for RawData, RawDataPostProcessingWriter.cpp:17), except that exact zeros
// take the default iostream form "0" / "-0".  libstdc++ formats those through
// vsnprintf("%.*e"), i.e. the correctly rounded decimal value, ties to even.
//
// Method (exact integer arithmetic, no floating point): x = M 2^q with M an
// integer of at most 53 bits.  With E = floor(log10 |x|) and k = P - E, the
// (P+1)-digit significand is N = round(M 2^q 10^k) = round(M 5^k 2^(q+k)),
// computed as a quotient and a remainder of integers of at most 256 bits, and
// rounded half to even.  E starts from floor(e2 log10 2), e2 the binary
// exponent of the leading bit, and is raised by one when the quotient shows
// it low.  Values whose integers would not fit (|x| below ~1e-71 or above
// ~1e44 at P = 16) and NaN / infinity report failure on the device; the host
// entry falls back to snprintf for them.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>

#include "common.cuh"

namespace gg {
namespace fmt {

// 64 x 64 -> 128-bit product, high word
GG_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// little-endian 4 x 64-bit unsigned integer
struct U256 {
  uint64_t w[4];
};

// a *= m (m < 2^64); returns false on overflow past 256 bits
GG_HD bool mul_small(U256& a, uint64_t m) {
  uint64_t carry = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint64_t lo = a.w[i] * m;
    const uint64_t hi = mulhi64(a.w[i], m);
    const uint64_t s = lo + carry;
    carry = hi + (s < lo ? 1 : 0);
    a.w[i] = s;
  }
  return carry == 0;
}

GG_HD int bitlen64(uint64_t v) {
#ifdef __CUDA_ARCH__
  return v ? 64 - __clzll((long long)v) : 0;
#else
  return v ? 64 - __builtin_clzll(v) : 0;
#endif
}

GG_HD int bitlen(const U256& a) {
  for (int i = 3; i >= 0; --i)
    if (a.w[i]) return 64 * i + bitlen64(a.w[i]);
  return 0;
}

// bit t of a (t < 256)
GG_HD int bit(const U256& a, int t) { return (int)((a.w[t >> 6] >> (t & 63)) & 1u); }

// any of bits [0, t) set
GG_HD bool any_below(const U256& a, int t) {
  for (int i = 0; i < 4 && t > 0; ++i, t -= 64) {
    const uint64_t m = t >= 64 ? ~0ull : ((1ull << t) - 1);
    if (a.w[i] & m) return true;
  }
  return false;
}

// a >> t, when the result fits 64 bits
GG_HD uint64_t shr_to64(const U256& a, int t) {
  const int i = t >> 6, r = t & 63;
  uint64_t lo = i < 4 ? a.w[i] : 0;
  uint64_t hi = i + 1 < 4 ? a.w[i + 1] : 0;
  return r ? (lo >> r) | (hi << (64 - r)) : lo;
}

GG_HD uint64_t pow10u(int n) {
  uint64_t p = 1;
  for (int i = 0; i < n; ++i) p *= 10u;
  return p;
}

GG_HD uint64_t pow5u(int n) {  // n <= 27
  uint64_t p = 1;
  for (int i = 0; i < n; ++i) p *= 5u;
  return p;
}

// 128-bit (hi:lo) / d for d < 2^64 with hi < d: quotient, remainder
GG_HD uint64_t div128(uint64_t hi, uint64_t lo, uint64_t d, uint64_t* rem) {
#ifdef __CUDA_ARCH__
  // bitwise long division (the quotient fits 64 bits since hi < d)
  uint64_t q = 0, r = hi;
  for (int i = 63; i >= 0; --i) {
    const uint64_t top = r >> 63;
    r = (r << 1) | ((lo >> i) & 1u);
    if (top || r >= d) {
      r -= d;
      q |= 1ull << i;
    }
  }
  *rem = r;
  return q;
#else
  const unsigned __int128 n = ((unsigned __int128)hi << 64) | lo;
  *rem = (uint64_t)(n % d);
  return (uint64_t)(n / d);
#endif
}

// Significand N (truncated), and the rounding class of the discarded part:
// 0 = exactly zero, 1 = below half, 2 = exactly half, 3 = above half.
// Returns false when the integers do not fit the fast path.
GG_HD bool scaled(uint64_t M, int q, int k, uint64_t* N, int* cls) {
  const int s = q + k;
  if (k >= 0) {
    if (k > 87) return false;
    U256 a{{M, 0, 0, 0}};
    for (int left = k; left > 0;) {
      const int c = left > 27 ? 27 : left;
      if (!mul_small(a, pow5u(c))) return false;
      left -= c;
    }
    if (s >= 0) {
      if (bitlen(a) + s > 64) return false;
      *N = a.w[0] << s;
      *cls = 0;
      return true;
    }
    const int t = -s;
    if (t >= 256) {
      // the whole value is below 1: not a (P+1)-digit significand
      return false;
    }
    if (bitlen(a) - t > 64) return false;
    *N = shr_to64(a, t);
    const int half = bit(a, t - 1);
    const bool rest = any_below(a, t - 1);
    *cls = half ? (rest ? 3 : 2) : (rest ? 1 : 0);
    return true;
  }
  // k < 0: divide by 5^(-k), and by 2^(-s) when s < 0
  const int kk = -k;
  if (kk > 27) return false;
  const uint64_t d5 = pow5u(kk);
  uint64_t rem;
  if (s < 0) {
    const int t = -s;
    if (t + bitlen64(d5) > 63) {
      // the denominator exceeds M: the quotient is 0
      *N = 0;
      *cls = 1;
      return true;
    }
    const uint64_t d = d5 << t;
    *N = M / d;
    rem = M % d;
    const uint64_t twice = rem << 1;  // d < 2^63
    *cls = rem == 0 ? 0 : (twice < d ? 1 : (twice == d ? 2 : 3));
    return true;
  }
  // numerator M 2^s, at most 128 bits
  if (bitlen64(M) + s > 127) return false;
  const uint64_t hi = s == 0 ? 0 : (s >= 64 ? (M << (s - 64)) : (M >> (64 - s)));
  const uint64_t lo = s >= 64 ? 0 : (M << s);
  if (hi >= d5) return false;  // quotient above 64 bits
  *N = div128(hi, lo, d5, &rem);
  const uint64_t twice = rem << 1;  // d5 < 2^63
  *cls = rem == 0 ? 0 : (twice < d5 ? 1 : (twice == d5 ? 2 : 3));
  return true;
}

// "%.{P}e" of x into out (at least P + 9 bytes); returns the length, or -1
// when x is NaN, infinite or outside the fast path.  0 <= P <= 16.
GG_HD int sci(double x, int P, char* out) {
  uint64_t bits;
  memcpy(&bits, &x, 8);
  const bool neg = (bits >> 63) != 0;
  const int eb = (int)((bits >> 52) & 0x7ff);
  const uint64_t frac = bits & ((1ull << 52) - 1);
  if (eb == 0x7ff) return -1;
  int len = 0;
  if (neg) out[len++] = '-';
  uint64_t N = 0;
  int E = 0;
  if (eb == 0 && frac == 0) {
    N = 0;
    E = 0;
  } else {
    const uint64_t M = eb ? (frac | (1ull << 52)) : frac;
    const int q = eb ? eb - 1075 : -1074;
    const int e2 = q + bitlen64(M) - 1;
    // floor(e2 log10 2): 78913 / 2^18 = 0.30102920..., exact for |e2| < 1700
    E = (int)(((int64_t)e2 * 78913) >> 18);
    const uint64_t lo = pow10u(P), hi = lo * 10u;
    int cls = 0;
    for (int tries = 0;; ++tries) {
      if (!scaled(M, q, P - E, &N, &cls)) return -1;
      if (N >= hi) {
        ++E;
      } else if (N < lo) {
        --E;
      } else {
        break;
      }
      if (tries > 2) return -1;
    }
    if (cls == 3 || (cls == 2 && (N & 1u))) ++N;
    if (N == hi) {
      N = lo;
      ++E;
    }
  }
  // digits of N, most significant first
  char d[17];
  for (int i = P; i >= 0; --i) {
    d[i] = (char)('0' + (int)(N % 10u));
    N /= 10u;
  }
  out[len++] = d[0];
  if (P > 0) {
    out[len++] = '.';
    for (int i = 1; i <= P; ++i) out[len++] = d[i];
  }
  out[len++] = 'e';
  out[len++] = E < 0 ? '-' : '+';
  int ae = E < 0 ? -E : E;
  if (ae >= 100) {
    out[len++] = (char)('0' + ae / 100);
    ae %= 100;
  }
  out[len++] = (char)('0' + ae / 10);
  out[len++] = (char)('0' + ae % 10);
  return len;
}

// GrainsExec::doubleToString(ios::scientific, P, x): "%.{P}e", but an exact
// zero keeps the default iostream form ("0", "-0").
GG_HD int grains_double(double x, int P, char* out) {
  if (x == 0.) {
    uint64_t bits;
    memcpy(&bits, &x, 8);
    if (bits >> 63) {
      out[0] = '-';
      out[1] = '0';
      return 2;
    }
    out[0] = '0';
    return 1;
  }
  return sci(x, P, out);
}

// decimal form of a 32-bit integer (what ostream << int prints)
GG_HD int int32(int v, char* out) {
  int len = 0;
  uint32_t u = (uint32_t)v;
  if (v < 0) {
    out[len++] = '-';
    u = 0u - u;
  }
  char d[10];
  int n = 0;
  do {
    d[n++] = (char)('0' + u % 10u);
    u /= 10u;
  } while (u);
  while (n) out[len++] = d[--n];
  return len;
}

// host form with the snprintf fallback outside the fast path
#if defined(__CUDACC__)
__host__
#endif
inline int grains_double_host(double x, int P, char* out, size_t cap) {
  char tmp[64];
  int n = grains_double(x, P, tmp);
  if (n < 0) n = std::snprintf(tmp, sizeof(tmp), "%.*e", P, x);
  if (n < 0 || (size_t)n >= cap) return -1;
  memcpy(out, tmp, (size_t)n);
  out[n] = 0;
  return n;
}

}  // namespace fmt
}  // namespace gg
