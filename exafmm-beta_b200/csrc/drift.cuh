// Closed form of the reference bounding-box recurrence.
//
// BoundBox::getBounds (include/bound_box.h:17-21) walks the bodies in order with
//     Xmin = min(X_i, Xmin - 1e-5),   Xmax = max(X_i, Xmax + 1e-5),
// which is a sequential chain over all N bodies.  Because x -> fl(x - c) is
// monotone, min commutes with it and the result is
//     Xmin = min( min_j g^(N-1-j)(X_j), g^N(X_0) ),   g(x) = fl(x - 1e-5),
// so every body contributes independently once g^k can be evaluated without
// stepping k times.  drift_down(x, k) does that exactly: inside one binade the
// spacing u of doubles is constant and every step subtracts the same rounded
// amount D*u (D = rint(c/u); no ties arise for |x| >= 2^-12), so a run of steps
// is one integer update; the few steps that touch a binade edge, and all steps
// with |x| < 2^-12, are taken one at a time in IEEE round-to-nearest.
#pragma once
#include <math.h>

namespace exafmm_b200 {

__host__ __device__ inline double sub_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dsub_rn(a, b);
#else
  volatile double r = a - b;
  return r;
#endif
}

// g^k(x) with g(x) = fl(x - 1e-5).
__host__ __device__ inline double drift_down(double x, long long k) {
  const double c = 1e-5;
  while (k > 0) {
    const double a = fabs(x);
    if (!(a >= 0x1p-12) || isinf(x)) {   // tiny (or NaN/inf): one exact step
      if (isinf(x) || isnan(x)) return x;
      x = sub_rn(x, c);
      k--;
      continue;
    }
    const int e = ilogb(a);                 // a in [2^e, 2^(e+1))
    const double u = ldexp(1.0, e - 52);    // spacing of doubles in this binade
    const double cu = c / u;                // exact power-of-two scaling
    const double Dd = rint(cu);
    if (Dd == 0.0) return x;                // a step no longer moves x
    const long long D = (long long)Dd;
    const long long A = (long long)(a / u); // integer in [2^52, 2^53)
    const long long cc = (long long)ceil(cu);
    long long room;                          // extra steps beyond the first that stay inside
    if (x > 0) {
      // toward zero: each exact intermediate A - i*D - cu must stay >= 2^52
      room = A - (1LL << 52) - cc;
    } else {
      // away from zero: each exact intermediate A + i*D + cu must stay < 2^53
      room = (1LL << 53) - 1 - A - cc;
    }
    if (room < 0) {
      x = sub_rn(x, c);
      k--;
      continue;
    }
    long long s = room / D + 1;
    if (s > k) s = k;
    const long long A2 = (x > 0) ? A - s * D : A + s * D;
    const double mag = ldexp((double)A2, e - 52);
    x = (x > 0) ? mag : -mag;
    k -= s;
  }
  return x;
}

// g^k(x) with g(x) = fl(x + 1e-5): round-to-nearest is symmetric under negation.
__host__ __device__ inline double drift_up(double x, long long k) { return -drift_down(-x, k); }

}  // namespace exafmm_b200
