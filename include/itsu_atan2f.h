/*
 * itsu_atan2f.h - correctly rounded binary32 atan2, bit-identical on host and device.
 *
 * The reference computes every azimuth with the C library's atan2f:
 *   cluster phi   = atan2f(-dy, -dx) + Pi   (MathUtils.h:37-39, via Cluster.cxx:35-45)
 *   tracklet phi  = atan2f(y1 - y2, x1 - x2) (Tracklet.cxx:32-37)
 * The result feeds hard cuts (Tracker.cxx:93-100, :161-166), so a one-ulp difference can
 * flip a tracklet or cell. glibc's atan2f is not correctly rounded and CUDA's differs again,
 * so this library replaces both with ONE function whose result is the binary32 value nearest
 * the exact atan2(y, x) (round-to-nearest-even). The oracle and the reference harness link
 * the same definition, which makes the device path and the CPU path agree by construction.
 *
 * Method (a published one, restated here): Ziv's two-step rounding test.
 *  1. Fast path in binary64. With num = min(|x|,|y|), den = max(|x|,|y|), pick k = round(32 t)
 *     for t = num/den (from a binary32 quotient) and reduce with atan(t) = atan(k/32) + atan(u),
 *     u = (num - (k/32) den) / (den + (k/32) num). The numerator is exact (both products have
 *     <= 30 significant bits and their exponents are at most two apart), |u| <= 1/64 + 2^-20, and
 *     atan(u) is a 6-term Taylor polynomial. Octant reconstruction uses pi/2 - a and pi - a.
 *     The relative error is below 2^-48; the result is returned when the interval
 *     [a - 2^-44 a, a + 2^-44 a] does not contain a binary32 rounding boundary.
 *  2. Otherwise (about 2e-6 of inputs) the same reduction is re-evaluated in double-double
 *     arithmetic (Dekker's exact product and Knuth's two-sum) with a 10-term series
 *     (relative error ~2^-100) and rounded with the low word deciding exact midpoints.
 * Only IEEE binary64 +, -, *, / and conversions are used. On the device every one of them is
 * an explicitly rounded intrinsic (__dadd_rn, ...), so nvcc cannot contract them into FMAs;
 * host code must be compiled without FP contraction (-ffp-contract=off), as the library's
 * build does. The tables atan(k/32), pi, pi/2 and 1/(2m+1) are double-double values computed
 * with 300-bit mpmath.
 */
#ifndef ITSU_ATAN2F_H
#define ITSU_ATAN2F_H

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define ITSU_CR_FN static __host__ __device__ __forceinline__
#else
#define ITSU_CR_FN static inline
#endif

#if defined(__CUDA_ARCH__)
#define ITSU_DADD(a, b) __dadd_rn((a), (b))
#define ITSU_DSUB(a, b) __dsub_rn((a), (b))
#define ITSU_DMUL(a, b) __dmul_rn((a), (b))
#define ITSU_DDIV(a, b) __ddiv_rn((a), (b))
#define ITSU_D2F(a) __double2float_rn(a)
#define ITSU_D2I_RZ(a) __double2int_rz(a)
#define ITSU_FDIV(a, b) __fdiv_rn((a), (b))
#define ITSU_FMUL(a, b) __fmul_rn((a), (b))
#define ITSU_FADD(a, b) __fadd_rn((a), (b))
#define ITSU_F2I_RZ(a) __float2int_rz(a)
#else
#define ITSU_DADD(a, b) ((a) + (b))
#define ITSU_DSUB(a, b) ((a) - (b))
#define ITSU_DMUL(a, b) ((a) * (b))
#define ITSU_DDIV(a, b) ((a) / (b))
#define ITSU_D2F(a) ((float)(a))
#define ITSU_D2I_RZ(a) ((int)(a))
#define ITSU_FDIV(a, b) ((a) / (b))
#define ITSU_FMUL(a, b) ((a) * (b))
#define ITSU_FADD(a, b) ((a) + (b))
#define ITSU_F2I_RZ(a) ((int)(a))
#endif

/* atan(k/32), k = 0..32, as (hi, lo) pairs. */
#define ITSU_CR_ATAN_K32_VALUES \
  { \
    {0x0.0p+0, 0x0.0p+0}, \
    {0x1.ffd55bba97625p-6, -0x1.5ec431444912cp-60}, \
    {0x1.ff55bb72cfdeap-5, -0x1.c934d86d23f1dp-60}, \
    {0x1.7ee182602f10fp-4, -0x1.cfb654c0c3d98p-58}, \
    {0x1.fd5ba9aac2f6ep-4, -0x1.cd37686760c17p-59}, \
    {0x1.3d6eee8c6626cp-3, 0x1.61a3b0ce9281bp-57}, \
    {0x1.7b97b4bce5b02p-3, 0x1.347b0b4f881cap-58}, \
    {0x1.b90d7529260a2p-3, 0x1.17b10d2e0e5abp-61}, \
    {0x1.f5b75f92c80ddp-3, 0x1.8ab6e3cf7afbdp-57}, \
    {0x1.18bf5a30bf178p-2, 0x1.30ca4748b1bf9p-57}, \
    {0x1.362773707ebccp-2, -0x1.963a544b672d8p-57}, \
    {0x1.530ad9951cd4ap-2, -0x1.2566480884082p-57}, \
    {0x1.6f61941e4def1p-2, -0x1.c63aae6f6e918p-56}, \
    {0x1.8b24d394a1b25p-2, 0x1.b6d0ba3748fa8p-56}, \
    {0x1.a64eec3cc23fdp-2, -0x1.24dec1b50b7ffp-56}, \
    {0x1.c0db4c94ec9f0p-2, -0x1.cc1ce70934c34p-56}, \
    {0x1.dac670561bb4fp-2, 0x1.a2b7f222f65e2p-56}, \
    {0x1.f40dd0b541418p-2, -0x1.a3992dc382a23p-57}, \
    {0x1.0657e94db30d0p-1, -0x1.d5b495f6349e6p-56}, \
    {0x1.1255d9bfbd2a9p-1, -0x1.2bdaee1c0ee35p-58}, \
    {0x1.1e00babdefeb4p-1, -0x1.928df287a668fp-58}, \
    {0x1.2958e59308e31p-1, -0x1.09e73b0c6c087p-56}, \
    {0x1.345f01cce37bbp-1, 0x1.1021137c71102p-55}, \
    {0x1.3f13fb89e96f4p-1, 0x1.ecf8b492644f0p-56}, \
    {0x1.4978fa3269ee1p-1, 0x1.2419a87f2a458p-56}, \
    {0x1.538f57b89061fp-1, -0x1.1bb74abda520cp-55}, \
    {0x1.5d58987169b18p-1, 0x1.0028e4bc5e7cap-57}, \
    {0x1.66d663923e087p-1, -0x1.6ea6febe8bbbap-56}, \
    {0x1.700a7c5784634p-1, -0x1.8c34d25aadef6p-56}, \
    {0x1.78f6bbd5d315ep-1, 0x1.406a089803740p-55}, \
    {0x1.819d0b7158a4dp-1, -0x1.bf76229d3b917p-56}, \
    {0x1.89ff5ff57f1f8p-1, -0x1.55b9a5e177a1bp-55}, \
    {0x1.921fb54442d18p-1, 0x1.1a62633145c07p-55}, \
  }

/* 1/(2m+1), m = 0..9, as (hi, lo) pairs: coefficients of atan(u) = u sum (-1)^m u^2m/(2m+1). */
#define ITSU_CR_INV_ODD_VALUES \
  { \
    {0x1.0p+0, 0x0.0p+0}, \
    {0x1.5555555555555p-2, 0x1.5555555555555p-56}, \
    {0x1.999999999999ap-3, -0x1.999999999999ap-57}, \
    {0x1.2492492492492p-3, 0x1.2492492492492p-57}, \
    {0x1.c71c71c71c71cp-4, 0x1.c71c71c71c71cp-58}, \
    {0x1.745d1745d1746p-4, -0x1.745d1745d1746p-59}, \
    {0x1.3b13b13b13b14p-4, -0x1.3b13b13b13b14p-58}, \
    {0x1.1111111111111p-4, 0x1.1111111111111p-60}, \
    {0x1.e1e1e1e1e1e1ep-5, 0x1.e1e1e1e1e1e1ep-61}, \
    {0x1.af286bca1af28p-5, 0x1.af286bca1af28p-59}, \
  }

/* One copy of each table per side: device code reads the __device__ copy, host code its own. */
#if defined(__CUDACC__)
static __device__ const double itsu_cr_atan_k32_dev[33][2] = ITSU_CR_ATAN_K32_VALUES;
static __device__ const double itsu_cr_inv_odd_dev[10][2] = ITSU_CR_INV_ODD_VALUES;
#endif
static const double itsu_cr_atan_k32_host[33][2] = ITSU_CR_ATAN_K32_VALUES;
static const double itsu_cr_inv_odd_host[10][2] = ITSU_CR_INV_ODD_VALUES;
#if defined(__CUDA_ARCH__)
#define itsu_cr_atan_k32 itsu_cr_atan_k32_dev
#define itsu_cr_inv_odd itsu_cr_inv_odd_dev
#else
#define itsu_cr_atan_k32 itsu_cr_atan_k32_host
#define itsu_cr_inv_odd itsu_cr_inv_odd_host
#endif


#define ITSU_CR_PI_HI 0x1.921fb54442d18p+1
#define ITSU_CR_PI_LO 0x1.1a62633145c07p-53
#define ITSU_CR_PIO2_HI 0x1.921fb54442d18p+0
#define ITSU_CR_PIO2_LO 0x1.1a62633145c07p-54
#define ITSU_CR_PIO4_HI 0x1.921fb54442d18p-1
#define ITSU_CR_3PIO4_HI 0x1.2d97c7f3321d2p+1

ITSU_CR_FN uint32_t itsu_cr_f2u(float f)
{
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, sizeof u);
  return u;
#endif
}

ITSU_CR_FN float itsu_cr_u2f(uint32_t u)
{
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, sizeof f);
  return f;
#endif
}

/* ---- double-double primitives (Knuth two-sum, Dekker/Veltkamp exact product) ---- */
typedef struct {
  double hi, lo;
} itsu_cr_dd;

ITSU_CR_FN itsu_cr_dd itsu_cr_two_sum(double a, double b)
{
  itsu_cr_dd r;
  double s = ITSU_DADD(a, b);
  double v = ITSU_DSUB(s, a);
  r.hi = s;
  r.lo = ITSU_DADD(ITSU_DSUB(a, ITSU_DSUB(s, v)), ITSU_DSUB(b, v));
  return r;
}

/* requires |a| >= |b| or a == 0 */
ITSU_CR_FN itsu_cr_dd itsu_cr_fast_two_sum(double a, double b)
{
  itsu_cr_dd r;
  double s = ITSU_DADD(a, b);
  r.hi = s;
  r.lo = ITSU_DSUB(b, ITSU_DSUB(s, a));
  return r;
}

ITSU_CR_FN void itsu_cr_split(double a, double *hi, double *lo)
{
  double t = ITSU_DMUL(134217729.0, a); /* 2^27 + 1 */
  *hi = ITSU_DSUB(t, ITSU_DSUB(t, a));
  *lo = ITSU_DSUB(a, *hi);
}

ITSU_CR_FN itsu_cr_dd itsu_cr_two_prod(double a, double b)
{
  double ah, al, bh, bl;
  itsu_cr_dd r;
  double p = ITSU_DMUL(a, b);
  itsu_cr_split(a, &ah, &al);
  itsu_cr_split(b, &bh, &bl);
  r.hi = p;
  r.lo = ITSU_DADD(ITSU_DADD(ITSU_DADD(ITSU_DSUB(ITSU_DMUL(ah, bh), p), ITSU_DMUL(ah, bl)), ITSU_DMUL(al, bh)),
                   ITSU_DMUL(al, bl));
  return r;
}

ITSU_CR_FN itsu_cr_dd itsu_cr_dd_add(itsu_cr_dd x, itsu_cr_dd y)
{
  itsu_cr_dd s = itsu_cr_two_sum(x.hi, y.hi);
  itsu_cr_dd t = itsu_cr_two_sum(x.lo, y.lo);
  s.lo = ITSU_DADD(s.lo, t.hi);
  s = itsu_cr_fast_two_sum(s.hi, s.lo);
  s.lo = ITSU_DADD(s.lo, t.lo);
  return itsu_cr_fast_two_sum(s.hi, s.lo);
}

ITSU_CR_FN itsu_cr_dd itsu_cr_dd_neg(itsu_cr_dd x)
{
  x.hi = -x.hi;
  x.lo = -x.lo;
  return x;
}

ITSU_CR_FN itsu_cr_dd itsu_cr_dd_mul(itsu_cr_dd x, itsu_cr_dd y)
{
  itsu_cr_dd p = itsu_cr_two_prod(x.hi, y.hi);
  p.lo = ITSU_DADD(p.lo, ITSU_DADD(ITSU_DMUL(x.hi, y.lo), ITSU_DMUL(x.lo, y.hi)));
  return itsu_cr_fast_two_sum(p.hi, p.lo);
}

/* x / y with three quotient digits */
ITSU_CR_FN itsu_cr_dd itsu_cr_dd_div(itsu_cr_dd x, itsu_cr_dd y)
{
  itsu_cr_dd q, r, t;
  double q1, q2, q3;
  q1 = ITSU_DDIV(x.hi, y.hi);
  t.hi = q1;
  t.lo = 0.0;
  r = itsu_cr_dd_add(x, itsu_cr_dd_neg(itsu_cr_dd_mul(y, t)));
  q2 = ITSU_DDIV(r.hi, y.hi);
  t.hi = q2;
  r = itsu_cr_dd_add(r, itsu_cr_dd_neg(itsu_cr_dd_mul(y, t)));
  q3 = ITSU_DDIV(r.hi, y.hi);
  q = itsu_cr_fast_two_sum(q1, q2);
  t.hi = q3;
  return itsu_cr_dd_add(q, t);
}

/* Round a positive double-double to the nearest binary32; the low word breaks exact ties of hi. */
ITSU_CR_FN float itsu_cr_dd_to_float(itsu_cr_dd a)
{
  float f = ITSU_D2F(a.hi);
  double fd = (double)f;
  if (fd != a.hi) {
    uint32_t fb = itsu_cr_f2u(f);
    double other;
    if (a.hi > fd) {
      other = (double)itsu_cr_u2f(fb + 1u);
    } else {
      other = fb == 0u ? -(double)itsu_cr_u2f(1u) : (double)itsu_cr_u2f(fb - 1u);
    }
    if (a.hi == ITSU_DMUL(ITSU_DADD(fd, other), 0.5)) {
      if (a.lo > 0.0) {
        f = ITSU_D2F(fd > other ? fd : other);
      } else if (a.lo < 0.0) {
        f = ITSU_D2F(fd < other ? fd : other);
      }
    }
  }
  return f;
}

/* Correctly rounded atan2 for binary32 arguments (C99 Annex F special cases). */
ITSU_CR_FN float itsu_atan2f(float y, float x)
{
  const uint32_t ux = itsu_cr_f2u(x), uy = itsu_cr_f2u(y);
  const uint32_t axb = ux & 0x7fffffffu, ayb = uy & 0x7fffffffu;
  const int yneg = (int)(uy >> 31), xneg = (int)(ux >> 31);
  float res;

  if (axb > 0x7f800000u || ayb > 0x7f800000u) {
    return x + y; /* NaN */
  }
  if (ayb == 0u) {
    res = xneg ? ITSU_D2F(ITSU_CR_PI_HI) : 0.0f;
    return yneg ? -res : res;
  }
  if (axb == 0u) {
    res = ITSU_D2F(ITSU_CR_PIO2_HI);
    return yneg ? -res : res;
  }
  if (ayb == 0x7f800000u) {
    if (axb == 0x7f800000u) {
      res = xneg ? ITSU_D2F(ITSU_CR_3PIO4_HI) : ITSU_D2F(ITSU_CR_PIO4_HI);
    } else {
      res = ITSU_D2F(ITSU_CR_PIO2_HI);
    }
    return yneg ? -res : res;
  }
  if (axb == 0x7f800000u) {
    res = xneg ? ITSU_D2F(ITSU_CR_PI_HI) : 0.0f;
    return yneg ? -res : res;
  }

  {
    const float axf = itsu_cr_u2f(axb), ayf = itsu_cr_u2f(ayb);
    const int swap = ayf > axf;
    const float numf = swap ? axf : ayf, denf = swap ? ayf : axf;
    const double num = (double)numf, den = (double)denf;
    /* k = round(32 t) from a binary32 quotient: |32 t - k| <= 1/2 + 2^-19, which keeps |u| within
     * 1/64 + 2^-20 and the numerator below exact (both products have <= 30 significant bits and
     * exponents at most two apart). */
    const float tf = ITSU_FDIV(numf, denf);
    const int k = ITSU_F2I_RZ(ITSU_FADD(ITSU_FMUL(tf, 32.0f), 0.5f));
    const double c = ITSU_DMUL((double)k, 0.03125);
    const double nn = ITSU_DSUB(num, ITSU_DMUL(c, den)); /* exact */
    const double cn = ITSU_DMUL(c, num);                 /* exact */
    const double u = ITSU_DDIV(nn, ITSU_DADD(den, cn));
    const double s = ITSU_DMUL(u, u);
    double p = ITSU_DMUL(s, -0x1.745d1745d1746p-4); /* -1/11 */
    double a, e, mlo, mhi, fd;
    uint32_t fb;
    p = ITSU_DMUL(s, ITSU_DADD(0x1.c71c71c71c71cp-4, p));  /* 1/9 */
    p = ITSU_DMUL(s, ITSU_DADD(-0x1.2492492492492p-3, p)); /* -1/7 */
    p = ITSU_DMUL(s, ITSU_DADD(0x1.999999999999ap-3, p));  /* 1/5 */
    p = ITSU_DMUL(s, ITSU_DADD(-0x1.5555555555555p-2, p)); /* -1/3 */
    p = ITSU_DADD(u, ITSU_DMUL(u, p));
    a = ITSU_DADD(itsu_cr_atan_k32[k][0], p);
    if (swap) {
      a = ITSU_DSUB(ITSU_CR_PIO2_HI, a);
    }
    if (xneg) {
      a = ITSU_DSUB(ITSU_CR_PI_HI, a);
    }
    res = ITSU_D2F(a);
    fd = (double)res;
    fb = itsu_cr_f2u(res);
    mhi = ITSU_DMUL(ITSU_DADD(fd, (double)itsu_cr_u2f(fb + 1u)), 0.5);
    mlo = fb == 0u ? -(double)itsu_cr_u2f(1u) : ITSU_DMUL(ITSU_DADD(fd, (double)itsu_cr_u2f(fb - 1u)), 0.5);
    e = ITSU_DMUL(a, 0x1.0p-44);
    if (ITSU_DSUB(a, e) > mlo && ITSU_DADD(a, e) < mhi) {
      return yneg ? -res : res;
    }

    /* Slow path: the same reduction in double-double. */
    {
#if defined(ITSU_CR_SLOW_PATH_HOOK)
      ITSU_CR_SLOW_PATH_HOOK;
#endif
      itsu_cr_dd dn, dden, du, ds, dp, dc, dr;
      int m;
      dn.hi = nn;
      dn.lo = 0.0;
      dden = itsu_cr_two_sum(den, cn);
      du = itsu_cr_dd_div(dn, dden);
      ds = itsu_cr_dd_mul(du, du);
      dp.hi = itsu_cr_inv_odd[9][0];
      dp.lo = itsu_cr_inv_odd[9][1];
      dp = itsu_cr_dd_neg(dp); /* (-1)^9 / 19 */
      for (m = 8; m >= 0; --m) {
        dc.hi = itsu_cr_inv_odd[m][0];
        dc.lo = itsu_cr_inv_odd[m][1];
        if (m & 1) {
          dc = itsu_cr_dd_neg(dc);
        }
        dp = itsu_cr_dd_add(dc, itsu_cr_dd_mul(ds, dp));
      }
      dr = itsu_cr_dd_mul(du, dp);
      dc.hi = itsu_cr_atan_k32[k][0];
      dc.lo = itsu_cr_atan_k32[k][1];
      dr = itsu_cr_dd_add(dc, dr);
      if (swap) {
        dc.hi = ITSU_CR_PIO2_HI;
        dc.lo = ITSU_CR_PIO2_LO;
        dr = itsu_cr_dd_add(dc, itsu_cr_dd_neg(dr));
      }
      if (xneg) {
        dc.hi = ITSU_CR_PI_HI;
        dc.lo = ITSU_CR_PI_LO;
        dr = itsu_cr_dd_add(dc, itsu_cr_dd_neg(dr));
      }
      res = itsu_cr_dd_to_float(dr);
      return yneg ? -res : res;
    }
  }
}

#endif /* ITSU_ATAN2F_H */
