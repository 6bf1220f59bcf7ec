/* cns_pmath.h -- one exponential and one real power for the device kernels
 * and for the CPU checker alike.
 *
 * The reference evaluates b**gam6 (clidd.f90:128) and the Spalart-Allmaras
 * exp / real power (met_smsa.f90) through its Fortran runtime's libm, and a
 * GPU's libm and the host's glibc differ by an ulp here and there.  These
 * functions are written from the mathematics in plain IEEE double operations
 * (each product and sum rounded on its own, never contracted into a fused
 * multiply-add: device code spells the roundings out, host code is built with
 * -ffp-contract=off), so a kernel and a host restatement that both call them
 * get the same bits.  They agree with glibc's exp and pow to a few ulp on the
 * arguments these routines see (the CPU tests check it).
 *
 *   cns_exp(t):    t = k ln2 + r with |r| <= ln2/2 (Cody-Waite reduction,
 *                  ln2 split into a 24-bit head, so k*head is exact, and a
 *                  tail), exp(r) by its Taylor series to degree 14 in Horner
 *                  form, times 2^k.
 *   cns_log(x):    x = 2^e m with m in [sqrt(1/2), sqrt(2)), log(m) = 2 atanh(s)
 *                  with s = (m - 1)/(m + 1) by its Taylor series in s^2
 *                  (|s| <= 0.1716: 12 terms), plus e ln2, as a double-double.
 *   cns_pow(x, y): exp(y log x) for x > 0, y log x formed in double-double
 *                  (Dekker's product); 0 or inf for x = 0; NaN for x < 0.
 *   cns_asin(x):   the Taylor series of asin for |x| <= 1/2, the half-angle
 *                  identity above (the wall laws' Van Driest transform).
 */
#ifndef CNS_PMATH_H
#define CNS_PMATH_H

#include <math.h>

#ifdef __CUDACC__
#define CNS_PM_FN static __host__ __device__ __forceinline__
#define CNS_PM_UNROLL _Pragma("unroll")
#else
#define CNS_PM_FN static inline
#define CNS_PM_UNROLL
#endif

#if defined(__CUDA_ARCH__)
#define CNS_PM_MUL(a, b) __dmul_rn((a), (b))
#define CNS_PM_ADD(a, b) __dadd_rn((a), (b))
#define CNS_PM_SUB(a, b) __dsub_rn((a), (b))
#define CNS_PM_DIV(a, b) __ddiv_rn((a), (b))
#else
#define CNS_PM_MUL(a, b) ((a) * (b))
#define CNS_PM_ADD(a, b) ((a) + (b))
#define CNS_PM_SUB(a, b) ((a) - (b))
#define CNS_PM_DIV(a, b) ((a) / (b))
#endif

/* ln 2 = 0.6931471805599453094172321214581765680755...: a 24-bit head and
 * the rest rounded to double; 1/ln 2 rounded to double */
#define CNS_PM_LN2_HI 0x1.62e43p-1
#define CNS_PM_LN2_LO (-0x1.05c610ca86c39p-29)
#define CNS_PM_INV_LN2 0x1.71547652b82fep+0

/* error-free transformations (Knuth's two-sum; Dekker's product with
 * Veltkamp's split, which needs no fused multiply-add) */
CNS_PM_FN void cns_two_sum(double a, double b, double* s, double* e) {
  const double t = CNS_PM_ADD(a, b);
  const double bb = CNS_PM_SUB(t, a);
  *s = t;
  *e = CNS_PM_ADD(CNS_PM_SUB(a, CNS_PM_SUB(t, bb)), CNS_PM_SUB(b, bb));
}
CNS_PM_FN void cns_split(double a, double* hi, double* lo) {
  const double c = CNS_PM_MUL(134217729.0, a); /* 2^27 + 1 */
  *hi = CNS_PM_SUB(c, CNS_PM_SUB(c, a));
  *lo = CNS_PM_SUB(a, *hi);
}
CNS_PM_FN void cns_two_prod(double a, double b, double* p, double* e) {
  double ah, al, bh, bl;
  const double t = CNS_PM_MUL(a, b);
  cns_split(a, &ah, &al);
  cns_split(b, &bh, &bl);
  *p = t;
  *e = CNS_PM_ADD(CNS_PM_ADD(CNS_PM_ADD(CNS_PM_SUB(CNS_PM_MUL(ah, bh), t), CNS_PM_MUL(ah, bl)),
                             CNS_PM_MUL(al, bh)),
                  CNS_PM_MUL(al, bl));
}

/* exp(th + tl) for a double-double argument (|tl| <= ulp(th)) */
CNS_PM_FN double cns_exp_dd(double th, double tl) {
  if (th != th) return th;
  if (th > 709.8) return INFINITY;
  if (th < -745.2) return 0.0;
  const double kf = floor(CNS_PM_ADD(CNS_PM_MUL(th, CNS_PM_INV_LN2), 0.5));
  /* th - k ln2_hi is exact (k ln2_hi has 24 + 11 bits and lies within a
     factor two of th) */
  const double r = CNS_PM_ADD(CNS_PM_SUB(CNS_PM_SUB(th, CNS_PM_MUL(kf, CNS_PM_LN2_HI)),
                                         CNS_PM_MUL(kf, CNS_PM_LN2_LO)),
                              tl);
  /* 1 + r (1 + r/2 (1 + r/3 (... (1 + r/14)))), each r/n as r times the
     double nearest 1/n */
  double p = 1.0;
  CNS_PM_UNROLL
  for (int n = 14; n >= 1; --n) p = CNS_PM_ADD(1.0, CNS_PM_MUL(CNS_PM_MUL(r, 1.0 / n), p));
  return ldexp(p, (int)kf);
}

CNS_PM_FN double cns_exp(double t) { return cns_exp_dd(t, 0.0); }

/* log(x) = hi + lo for finite x > 0: x = 2^e (1 + f) with 1 + f in
 * [sqrt(1/2), sqrt(2)) (f exact), s = f / (2 + f),
 * log(1 + f) = 2 s (1 + q), q = s^2/3 + s^4/5 + ... + s^22/23, written as
 * f - s (f - 2 q) (2 s = f - s f), whose leading term f is exact */
CNS_PM_FN void cns_log_dd(double x, double* hi, double* lo) {
  int e = 0;
  double m = frexp(x, &e); /* x = m 2^e, m in [1/2, 1) */
  if (m < 0.70710678118654757) {
    m = CNS_PM_MUL(m, 2.0);
    e -= 1;
  }
  const double f = CNS_PM_SUB(m, 1.0);
  const double s = CNS_PM_DIV(f, CNS_PM_ADD(2.0, f));
  const double s2 = CNS_PM_MUL(s, s);
  double q = 0.0;
  CNS_PM_UNROLL
  for (int k = 11; k >= 1; --k) q = CNS_PM_MUL(s2, CNS_PM_ADD(1.0 / (2 * k + 1), q));
  const double corr = CNS_PM_MUL(s, CNS_PM_SUB(f, CNS_PM_MUL(2.0, q)));
  const double ef = (double)e;
  double h, err;
  cns_two_sum(CNS_PM_MUL(ef, CNS_PM_LN2_HI), f, &h, &err);
  *hi = h;
  *lo = CNS_PM_ADD(err, CNS_PM_SUB(CNS_PM_MUL(ef, CNS_PM_LN2_LO), corr));
}

CNS_PM_FN double cns_log(double x) {
  double h, l;
  cns_log_dd(x, &h, &l);
  return CNS_PM_ADD(h, l);
}

/* x^y = exp(y log x) with y log x carried in double-double */
CNS_PM_FN double cns_pow(double x, double y) {
  if (x != x || y != y) return x + y;
  if (x < 0.0) return NAN;
  if (x == 0.0) return y > 0.0 ? 0.0 : (y < 0.0 ? INFINITY : 1.0);
  if (y == 0.0 || x == 1.0) return 1.0;
  if (isinf(x)) return y > 0.0 ? INFINITY : 0.0;
  double lh, ll, th, te;
  cns_log_dd(x, &lh, &ll);
  cns_two_prod(y, lh, &th, &te);
  return cns_exp_dd(th, CNS_PM_ADD(te, CNS_PM_MUL(y, ll)));
}

/* pi/2 = 1.5707963267948966192313216916397514...: the nearest double and
 * the rest */
#define CNS_PM_PIO2_HI 0x1.921fb54442d18p+0
#define CNS_PM_PIO2_LO 0x1.1a62633145c07p-54

/* asin(x) for |x| <= 1/2 by its Taylor series
 *   asin(x) = x (1 + r1 z (1 + r2 z (1 + ... (1 + r29 z)))),  z = x^2,
 *   r_n = (2n - 1)^2 / ((2n) (2n + 1))   (the ratio of consecutive terms),
 * whose tail after 29 terms is below 2^-58 relative for z <= 1/4 */
CNS_PM_FN double cns_asin_small(double x) {
  const double z = CNS_PM_MUL(x, x);
  double p = 1.0;
  CNS_PM_UNROLL
  for (int n = 29; n >= 1; --n)
    p = CNS_PM_ADD(1.0, CNS_PM_MUL(CNS_PM_MUL(CNS_PM_DIV((double)((2 * n - 1) * (2 * n - 1)),
                                                         (double)((2 * n) * (2 * n + 1))),
                                              z),
                                   p));
  return CNS_PM_MUL(x, p);
}

/* asin(x): the series for |x| <= 1/2; above, asin(|x|) = pi/2 - 2 asin(s)
 * with s = sqrt((1 - |x|)/2) <= 1/2 (1 - |x| and the halving are exact);
 * NaN outside [-1, 1] */
CNS_PM_FN double cns_asin(double x) {
  if (x != x) return x;
  const double a = fabs(x);
  if (a > 1.0) return NAN;
  if (a <= 0.5) return cns_asin_small(x);
  const double s = sqrt(CNS_PM_MUL(CNS_PM_SUB(1.0, a), 0.5));
  const double r =
      CNS_PM_ADD(CNS_PM_SUB(CNS_PM_PIO2_HI, CNS_PM_MUL(2.0, cns_asin_small(s))), CNS_PM_PIO2_LO);
  return x < 0.0 ? -r : r;
}

#endif /* CNS_PMATH_H */
