// Fixed-step natural log and exp in IEEE double (internal to libgowalker.so).
//
// Every operation is rounded to nearest with no contraction, so any IEEE
// implementation of the same steps -- the CPU oracle's C and Python
// restatements included -- gives the same bits.  They serve draws whose
// outcome must be reproducible off the device: the annealing acceptance and
// the power-law degrees of the web-shaped graph.  They are written from the
// series below, not from any library's implementation.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gw {

// 1/(2j+1) and 1/k, each a correctly rounded quotient.
static __constant__ double kFmInvOdd[12] = {1.0 / 1,  1.0 / 3,  1.0 / 5,  1.0 / 7,  1.0 / 9,  1.0 / 11,
                                     1.0 / 13, 1.0 / 15, 1.0 / 17, 1.0 / 19, 1.0 / 21, 1.0 / 23};
static __constant__ double kFmInv[14] = {0.0,     1.0 / 1, 1.0 / 2, 1.0 / 3,  1.0 / 4,  1.0 / 5,  1.0 / 6,
                                  1.0 / 7, 1.0 / 8, 1.0 / 9, 1.0 / 10, 1.0 / 11, 1.0 / 12, 1.0 / 13};

// ln(z * 2^-32) for a 32-bit draw z: u = m 2^e with m in [sqrt(1/2), sqrt(2)),
// ln u = e ln2 + 2 atanh(s), s = (m-1)/(m+1), the atanh series to s^23/23 by
// Horner in s^2 (|s| < 0.172: truncation below 1e-19); ln2 split as
// 45426 * 2^-16 (exact products) plus the remainder.  z = 0 gives -inf.
__device__ inline double fm_log_u32(uint32_t z)
{
    if (z == 0) return -__longlong_as_double(0x7FF0000000000000ll);
    int e = 31 - __clz(z);                  // z = 2^e * (1.f), e in [0, 31]
    double m = (double)z * ldexp(1.0, -e);  // exact: [1, 2)
    if (m >= 1.4142135623730951) {
        m = __dmul_rn(m, 0.5);  // exact
        e += 1;
    }
    const double s = __ddiv_rn(__dsub_rn(m, 1.0), __dadd_rn(m, 1.0));
    const double s2 = __dmul_rn(s, s);
    double q = kFmInvOdd[11];
    for (int j = 10; j >= 0; --j) q = __dadd_rn(kFmInvOdd[j], __dmul_rn(s2, q));
    const double lnm = __dmul_rn(__dmul_rn(2.0, s), q);
    const double ex = (double)(e - 32);
    return __dadd_rn(__dadd_rn(__dmul_rn(ex, 0.693145751953125), __dmul_rn(ex, 1.4286068203094172e-06)), lnm);
}

// exp(x) for x <= 0: x = n ln2 + r (n = nearest integer of x / ln2, ln2 split
// as above), the Taylor series of exp(r), |r| <= ln2/2, to r^13/13! by Horner
// (q = 1 + r q (1/k)), then 2^n.  x <= -700 gives 0, x >= 0 gives 1.
__device__ inline double fm_exp_nonpos(double x)
{
    if (!(x > -700.0)) return 0.0;
    if (x >= 0.0) return 1.0;
    const double nd = rint(__dmul_rn(x, 1.4426950408889634));
    const double r = __dsub_rn(__dsub_rn(x, __dmul_rn(nd, 0.693145751953125)), __dmul_rn(nd, 1.4286068203094172e-06));
    double q = 1.0;
    for (int k = 13; k >= 1; --k) q = __dadd_rn(1.0, __dmul_rn(__dmul_rn(r, q), kFmInv[k]));
    return ldexp(q, (int)nd);
}

}  // namespace gw
