// Correctly rounded sine and cosine of a pose angle, for host and device.
//
// The reference rotates every scan point by R(theta) with std::cos/std::sin
// (src/core/pose.hpp:19-25, src/problem/residual_math.hpp:99-100), and the
// cell a point falls in (src/core/grid_map.hpp:58-70) must come out the same
// on the GPU bit for bit. glibc's double sin/cos return the correctly
// rounded result except in rare hard cases, so the GPU computes the correctly
// rounded values itself instead of calling the CUDA math library (whose
// results may differ from glibc's in the last bit):
//
//  * argument reduction after Cody and Waite ("Software Manual for the
//    Elementary Functions", 1980): k = rint(x * 2/pi), r = x - k * pi/2 with
//    pi/2 held as a sum of four doubles, products split exactly with fma and
//    the differences carried as double-double (hi + lo) numbers;
//  * sin(r) and cos(r) for |r| <= pi/4 from their Taylor series, evaluated by
//    Horner's rule in double-double arithmetic (Dekker 1971; Knuth's TwoSum)
//    to about 2^-100 relative, with the 1/n! coefficients held as
//    double-double constants;
//  * one final rounding of hi + lo, which is the correctly rounded value of
//    sin/cos unless the exact value lies within ~2^-100 of a rounding
//    boundary between two doubles.
//
// Constants: pi/2 split into four doubles, 2/pi and 1/n! (n <= 30) rounded
// to double-double, computed from pi to 115 digits by Machin's formula.
// Domain: |x| < 2^30 (pose angles); the reduction stays exact there.
// Every operation is an explicitly rounded +, -, * or fma, so host and device
// builds of these functions return identical bits.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define SDFGPU_HD __host__ __device__ __forceinline__
#else
#define SDFGPU_HD inline
#endif

namespace sdfgpu {
namespace trig {

struct DD {
  double hi;
  double lo;
};

SDFGPU_HD double Fma(double a, double b, double c) {
#ifdef __CUDA_ARCH__
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}

/// Knuth's TwoSum: s + e == a + b exactly.
SDFGPU_HD DD TwoSum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  const double e = (a - (s - bb)) + (b - bb);
  return {s, e};
}

/// Dekker's FastTwoSum, |a| >= |b|.
SDFGPU_HD DD QuickTwoSum(double a, double b) {
  const double s = a + b;
  return {s, b - (s - a)};
}

/// p + e == a * b exactly.
SDFGPU_HD DD TwoProd(double a, double b) {
  const double p = a * b;
  return {p, Fma(a, b, -p)};
}

/// Double-double sum with the low parts carried (accurate form).
SDFGPU_HD DD Add(DD a, DD b) {
  DD s = TwoSum(a.hi, b.hi);
  DD t = TwoSum(a.lo, b.lo);
  s.lo += t.hi;
  s = QuickTwoSum(s.hi, s.lo);
  s.lo += t.lo;
  return QuickTwoSum(s.hi, s.lo);
}

SDFGPU_HD DD Mul(DD a, DD b) {
  DD p = TwoProd(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return QuickTwoSum(p.hi, p.lo);
}

/// Horner's rule over the double-double coefficients c[0..n-1] (c[0] the
/// constant term) at z.
SDFGPU_HD DD Horner(const double (*c)[2], int n, DD z) {
  DD p = {c[n - 1][0], c[n - 1][1]};
  for (int m = n - 2; m >= 0; --m) {
    p = Add(Mul(p, z), DD{c[m][0], c[m][1]});
  }
  return p;
}

/// sin(r) = r * S(r^2), cos(r) = C(r^2) for |r| <= pi/4 (plus the rounding
/// slack of k); S and C are the Taylor series in z = r^2 to z^14.
SDFGPU_HD void KernelSinCos(DD r, DD* s, DD* c) {
  // (-1)^m / (2m+1)!, m = 0..14
  constexpr double kS[15][2] = {
      {1.0, 0.0},
      {-0x1.5555555555555p-3, -0x1.5555555555555p-57},
      {0x1.1111111111111p-7, 0x1.1111111111111p-63},
      {-0x1.a01a01a01a01ap-13, -0x1.a01a01a01a01ap-73},
      {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73},
      {-0x1.ae64567f544e4p-26, 0x1.c062e06d1f209p-80},
      {0x1.6124613a86d09p-33, 0x1.f28e0cc748ebep-87},
      {-0x1.ae7f3e733b81fp-41, -0x1.1d8656b0ee8cbp-97},
      {0x1.952c77030ad4ap-49, 0x1.ac981465ddc6cp-103},
      {-0x1.2f49b46814157p-57, -0x1.2650f61dbdcb4p-112},
      {0x1.71b8ef6dcf572p-66, -0x1.d043ae40c4647p-120},
      {-0x1.761b41316381ap-75, 0x1.3423c7d91404fp-130},
      {0x1.3f3ccdd165fa9p-84, -0x1.58ddadf344487p-139},
      {-0x1.d1ab1c2dccea3p-94, -0x1.054d0c78aea14p-149},
      {0x1.259f98b4358adp-103, 0x1.eaf8c39dd9bc5p-157},
  };
  // (-1)^m / (2m)!, m = 0..14
  constexpr double kC[15][2] = {
      {1.0, 0.0},
      {-0x1.0000000000000p-1, 0.0},
      {0x1.5555555555555p-5, 0x1.5555555555555p-59},
      {-0x1.6c16c16c16c17p-10, 0x1.f49f49f49f49fp-65},
      {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76},
      {-0x1.27e4fb7789f5cp-22, -0x1.cbbc05b4fa99ap-76},
      {0x1.1eed8eff8d898p-29, -0x1.2aec959e14c06p-83},
      {-0x1.93974a8c07c9dp-37, -0x1.05d6f8a2efd1fp-92},
      {0x1.ae7f3e733b81fp-45, 0x1.1d8656b0ee8cbp-101},
      {-0x1.6827863b97d97p-53, -0x1.eec01221a8b0bp-107},
      {0x1.e542ba4020225p-62, 0x1.ea72b4afe3c2fp-120},
      {-0x1.0ce396db7f853p-70, 0x1.aebcdbd20331cp-124},
      {0x1.f2cf01972f578p-80, -0x1.9ada5fcc1ab14p-135},
      {-0x1.88e85fc6a4e5ap-89, 0x1.71c37ebd16540p-143},
      {0x1.0a18a2635085dp-98, 0x1.b9e2e28e1aa54p-153},
  };
  const DD z = Mul(r, r);
  *s = Mul(r, Horner(kS, 15, z));
  *c = Horner(kC, 15, z);
}

}  // namespace trig

/// Correctly rounded sin(x) and cos(x) (see the file comment); x = +-0 gives
/// (+-0, 1), non-finite x gives NaN.
SDFGPU_HD void SinCosRn(double x, double* sin_out, double* cos_out) {
  using trig::DD;
  constexpr double kTwoOverPi = 0x1.45f306dc9c883p-1;
  constexpr double kPio2_1 = 0x1.921fb54442d18p+0;
  constexpr double kPio2_2 = 0x1.1a62633145c07p-54;
  constexpr double kPio2_3 = -0x1.f1976b7ed8fbcp-110;
  constexpr double kPio2_4 = 0x1.4cf98e804177dp-164;
  if (x == 0.0) {
    *sin_out = x;  // keeps the sign of zero
    *cos_out = 1.0;
    return;
  }
  if (!(x - x == 0.0)) {  // infinity or NaN
    *sin_out = x - x;
    *cos_out = x - x;
    return;
  }
#ifdef __CUDA_ARCH__
  const double k = rint(x * kTwoOverPi);
#else
  const double k = std::rint(x * kTwoOverPi);
#endif
  // r = x - k pi/2: x - k*P1 is exact (Sterbenz) once its low part is split off
  const DD p1 = trig::TwoProd(k, kPio2_1);
  DD r = trig::TwoSum(x - p1.hi, -p1.lo);
  const DD p2 = trig::TwoProd(k, kPio2_2);
  r = trig::Add(r, DD{-p2.hi, -p2.lo});
  r = trig::Add(r, DD{-(k * kPio2_3), -(k * kPio2_4)});
  DD s;
  DD c;
  trig::KernelSinCos(r, &s, &c);
  const double sv = s.hi + s.lo;
  const double cv = c.hi + c.lo;
  // quadrant k mod 4 (two's complement keeps negative k right)
  const int q = static_cast<int>(static_cast<int64_t>(k) & 3);
  switch (q) {
    case 0:
      *sin_out = sv;
      *cos_out = cv;
      break;
    case 1:
      *sin_out = cv;
      *cos_out = -sv;
      break;
    case 2:
      *sin_out = -sv;
      *cos_out = -cv;
      break;
    default:
      *sin_out = -cv;
      *cos_out = sv;
      break;
  }
}

}  // namespace sdfgpu
