// dsmc_physics.h -- per-atom and per-cell arithmetic of the DSMC timestep.
//
// Included by the sm_100a kernels (nvcc, compiled with --fmad=false) and by the CPU
// oracle (g++, -ffp-contract=off).  Every value is produced by IEEE-754 operations that
// are correctly rounded on both sides (+ - * /, sqrt, fma, floor/rint, integer ops), so the
// GPU and the CPU restatement give bit-identical results for the same inputs in float and
// in double.  Elementary functions (sin/cos/log/exp) are written here from their series
// (Cody-Waite argument reduction, Taylor / atanh series) instead of calling libm or the
// CUDA math library, whose implementations differ between host and device.
//
// Physics follows CUDADSMC (paths inside that project):
//   trap field and Jacobian           src/moveAtoms.cu:135-157 (Ioffe-Pritchard),
//                                     energyComparison.py:53 (quadrupole |B| = B' sqrt(x^2/4+y^2/4+z^2))
//   acceleration a = -(mu/m) grad|B|  src/moveAtoms.cu:93-116
//   velocity Verlet                   src/moveAtoms.cu:51-65
//   Larmor rotation exp(-i theta s.B^) src/wavefunction.cu:39-73
//   normalisation                     src/wavefunction.cu:279-299
//   Majorana test <s.B^> < 0          src/evaporation.cu:86-95
//   cell index                        src/collisions.cu:187-219
//   NTC collisions                    src/collisions.cu:291-437, 529-546
//   random numbers: Philox4x32-10, Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
//   as easy as 1, 2, 3", SC'11 (replaces the cuRAND XORWOW states of src/setUp.cu:63-75).
#ifndef DSMC_PHYSICS_H
#define DSMC_PHYSICS_H

#include <stdint.h>

#if defined(__CUDACC__)
#define DSMC_HD __host__ __device__ __forceinline__
#else
#include <math.h>
#include <string.h>
#define DSMC_HD inline
#endif

namespace dsmc {

typedef __int128 i128;

// ---------------------------------------------------------------------------------------
// Correctly rounded primitives (identical on host and device)
// ---------------------------------------------------------------------------------------
DSMC_HD float xfma(float a, float b, float c) { return fmaf(a, b, c); }
DSMC_HD double xfma(double a, double b, double c) { return fma(a, b, c); }
DSMC_HD float xsqrt(float x) { return sqrtf(x); }
DSMC_HD double xsqrt(double x) { return sqrt(x); }
DSMC_HD float xabs(float x) { return fabsf(x); }
DSMC_HD double xabs(double x) { return fabs(x); }
DSMC_HD float xfloor(float x) { return floorf(x); }
DSMC_HD double xfloor(double x) { return floor(x); }
DSMC_HD float xceil(float x) { return ceilf(x); }
DSMC_HD double xceil(double x) { return ceil(x); }
DSMC_HD float xrint(float x) { return rintf(x); }
DSMC_HD double xrint(double x) { return rint(x); }

// ---------------------------------------------------------------------------------------
// Two independent lanes of arithmetic.  On sm_100 a float pair is one paired FP32 instruction
// (FADD2 / FMUL2 / FFMA2), each lane an ordinary round-to-nearest IEEE operation; elsewhere
// (double, the host) it is two scalar operations with the same results.
// ---------------------------------------------------------------------------------------
template <class R> struct V2 {
    R x, y;
};
template <class R> DSMC_HD V2<R> v2(R a, R b) {
    V2<R> r;
    r.x = a;
    r.y = b;
    return r;
}
template <class R> DSMC_HD V2<R> v2s(R a) { return v2(a, a); }
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
DSMC_HD V2<float> add2(V2<float> a, V2<float> b) {
    const float2 r = __fadd2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
    return v2(r.x, r.y);
}
DSMC_HD V2<float> mul2(V2<float> a, V2<float> b) {
    const float2 r = __fmul2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
    return v2(r.x, r.y);
}
DSMC_HD V2<float> fma2(V2<float> a, V2<float> b, V2<float> c) {
    const float2 r = __ffma2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y), make_float2(c.x, c.y));
    return v2(r.x, r.y);
}
#else
DSMC_HD V2<float> add2(V2<float> a, V2<float> b) { return v2(a.x + b.x, a.y + b.y); }
DSMC_HD V2<float> mul2(V2<float> a, V2<float> b) { return v2(a.x * b.x, a.y * b.y); }
DSMC_HD V2<float> fma2(V2<float> a, V2<float> b, V2<float> c) { return v2(xfma(a.x, b.x, c.x), xfma(a.y, b.y, c.y)); }
#endif
DSMC_HD V2<double> add2(V2<double> a, V2<double> b) { return v2(a.x + b.x, a.y + b.y); }
DSMC_HD V2<double> mul2(V2<double> a, V2<double> b) { return v2(a.x * b.x, a.y * b.y); }
DSMC_HD V2<double> fma2(V2<double> a, V2<double> b, V2<double> c) {
    return v2(xfma(a.x, b.x, c.x), xfma(a.y, b.y, c.y));
}
template <class R> DSMC_HD V2<R> sub2(V2<R> a, V2<R> b) { return add2(a, v2(-b.x, -b.y)); }

DSMC_HD uint32_t f2u(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u; memcpy(&u, &f, 4); return u;
#endif
}
DSMC_HD float u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f; memcpy(&f, &u, 4); return f;
#endif
}
DSMC_HD uint64_t d2u(double f) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(f);
#else
    uint64_t u; memcpy(&u, &f, 8); return u;
#endif
}
DSMC_HD double u2d(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double f; memcpy(&f, &u, 8); return f;
#endif
}

// 4th-lane integer payloads (atom id in pos.w, flag bits in vel.w)
DSMC_HD float lane_from_u32(uint32_t u, float) { return u2f(u); }
DSMC_HD double lane_from_u32(uint32_t u, double) { return u2d((uint64_t)u); }
DSMC_HD uint32_t lane_to_u32(float f) { return f2u(f); }
DSMC_HD uint32_t lane_to_u32(double f) { return (uint32_t)d2u(f); }

// ---------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11): 10 rounds of the 4x32 S-P network with the
// multipliers M0 = 0xD2511F53, M1 = 0xCD9E8D57 and key schedule constants (Weyl
// sequence) W0 = 0x9E3779B9, W1 = 0xBB67AE85 given in the paper.
// ---------------------------------------------------------------------------------------
struct u32x4 { uint32_t x, y, z, w; };

DSMC_HD u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        u32x4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// Stream purposes (third counter word, high byte); the low 24 bits carry the cloud id.
enum : uint32_t {
    PURPOSE_INIT_POS = 1u,
    PURPOSE_INIT_VEL = 2u,
    PURPOSE_COLLIDE = 3u,
    PURPOSE_FLIP = 4u
};

DSMC_HD u32x4 draw(uint32_t id, uint32_t step, uint32_t purpose, uint32_t cloud, uint32_t sub,
                   uint64_t seed) {
    u32x4 c;
    c.x = id;
    c.y = step;
    c.z = (purpose << 24) | (cloud & 0xFFFFFFu);
    c.w = sub;
    return philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
}

// uniform in the open interval (0,1): float from 24 bits, double from 53 bits (two words)
DSMC_HD float u01f(uint32_t a) { return ((float)(a >> 8) + 0.5f) * 0x1p-24f; }
DSMC_HD double u01d(uint32_t a, uint32_t b) {
    uint64_t m = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);
    return ((double)m + 0.5) * 0x1p-53;
}
template <class R> DSMC_HD R u01(uint32_t a, uint32_t b);
template <> DSMC_HD float u01<float>(uint32_t a, uint32_t) { return u01f(a); }
template <> DSMC_HD double u01<double>(uint32_t a, uint32_t b) { return u01d(a, b); }

// unbiased-enough index in [0, n): high word of a 32x32 product (bias < n / 2^32)
DSMC_HD uint32_t index_below(uint32_t r, uint32_t n) {
    return (uint32_t)(((uint64_t)r * (uint64_t)n) >> 32);
}

// ---------------------------------------------------------------------------------------
// Elementary functions from their series.
// sin/cos: x = k pi/2 + r with pi/2 split in three parts (the leading parts have trailing
// zero bits, so k*part is exact), |r| <= pi/4, Taylor series evaluated with fma (Horner).
// log: x = m 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh((m-1)/(m+1)) series.
// exp: x = k ln2 + r, |r| <= ln2/2, Taylor series, scaled by 2^k.
// The split constants were derived from Machin's formula for pi and the atanh(1/3)
// series for ln 2 in exact rational arithmetic.
// ---------------------------------------------------------------------------------------
DSMC_HD void xsincos(float x, float* s, float* c) {
    const float two_over_pi = 0x1.45f306p-1f;
    const float p1 = 0x1.922p+0f, p2 = -0x1.2aep-18f, p3 = -0x1.de973ep-31f;
    // k = x 2/pi rounded to the nearest integer (ties to even) by adding and removing 1.5 * 2^23:
    // exact for |x 2/pi| < 2^22, and the sum's low mantissa bits are then k modulo 4 (1.5 * 2^23
    // is a multiple of 4) -- two adds instead of a rounding and a conversion on the slow pipe
    const float t = x * two_over_pi;
    const float shifter = 12582912.0f;
    float k, km;
    if (xabs(t) < 4194304.0f) {
        km = t + shifter;
        k = km - shifter;
    } else {
        k = xrint(t);
        km = 0.0f;
    }
    float r = xfma(-k, p1, x);
    r = xfma(-k, p2, r);
    r = xfma(-k, p3, r);
    float r2 = r * r;
    // sin r = r + r^3 (-1/3! + r^2 (1/5! + r^2 (-1/7! + r^2/9!)))
    // cos r = 1 + r^2 (-1/2 + r^2 (1/4! + r^2 (-1/6! + r^2 (1/8! - r^2/10!))))
    // evaluated as one two-lane Horner chain (sin lane, cos lane)
    const V2<float> rr = v2s(r2);
    const float pc0 = xfma(r2, -2.75573192e-7f, 2.48015873e-5f);
    V2<float> p = fma2(rr, v2(2.75573192e-6f, pc0), v2(-1.98412698e-4f, -1.38888889e-3f));
    p = fma2(rr, p, v2(8.33333333e-3f, 4.16666667e-2f));
    p = fma2(rr, p, v2(-1.66666667e-1f, -0.5f));
    const V2<float> sc = fma2(v2(r * r2, r2), p, v2(r, 1.0f));
    const float sr = sc.x, cr = sc.y;
    int q = xabs(t) < 4194304.0f ? (int)(f2u(km) & 3u) : (((int)k) & 3);
    float ss = (q & 1) ? cr : sr;
    float cc = (q & 1) ? sr : cr;
    if (q == 1 || q == 2) cc = -cc;
    if (q >= 2) ss = -ss;
    *s = ss;
    *c = cc;
}

DSMC_HD void xsincos(double x, double* s, double* c) {
    const double two_over_pi = 0x1.45f306dc9c883p-1;
    const double p1 = 0x1.921fb58p+0, p2 = -0x1.dde974p-27, p3 = 0x1.1a62633145c07p-54;
    // nearest integer by adding and removing 1.5 * 2^52 (exact for |x 2/pi| < 2^51; the sum's low
    // mantissa bits are k modulo 4), as in the float version
    const double t = x * two_over_pi;
    const double shifter = 6755399441055744.0;
    double k, km;
    if (xabs(t) < 2251799813685248.0) {
        km = t + shifter;
        k = km - shifter;
    } else {
        k = xrint(t);
        km = 0.0;
    }
    double r = xfma(-k, p1, x);
    r = xfma(-k, p2, r);
    r = xfma(-k, p3, r);
    double r2 = r * r;
    // Taylor coefficients 1/n!, alternating signs
    double ps = xfma(r2, 2.8114572543455206e-15, -7.6471637318198164e-13);   // 1/17!, -1/15!
    ps = xfma(r2, ps, 1.6059043836821613e-10);                                // 1/13!
    ps = xfma(r2, ps, -2.5052108385441720e-8);                                // -1/11!
    ps = xfma(r2, ps, 2.7557319223985893e-6);                                 // 1/9!
    ps = xfma(r2, ps, -1.9841269841269841e-4);                                // -1/7!
    ps = xfma(r2, ps, 8.3333333333333333e-3);                                 // 1/5!
    ps = xfma(r2, ps, -1.6666666666666667e-1);                                // -1/3!
    double sr = xfma(r * r2, ps, r);
    double pc = xfma(r2, 1.5619206968586225e-16, -4.7794773323873853e-14);   // 1/18!, -1/16!
    pc = xfma(r2, pc, 1.1470745597729725e-11);                                // 1/14!
    pc = xfma(r2, pc, -2.0876756987868099e-9);                                // -1/12!
    pc = xfma(r2, pc, 2.7557319223985891e-7);                                 // 1/10!
    pc = xfma(r2, pc, -2.4801587301587302e-5);                                // -1/8!
    pc = xfma(r2, pc, 1.3888888888888889e-3);                                 // 1/6!
    pc = xfma(r2, pc, -4.1666666666666667e-2);                                // -1/4!
    pc = xfma(r2, pc, 0.5);                                                   // 1/2!
    double cr = xfma(-r2, pc, 1.0);
    int q = xabs(t) < 2251799813685248.0 ? (int)(d2u(km) & 3ull) : (((int)(long long)k) & 3);
    double ss = (q & 1) ? cr : sr;
    double cc = (q & 1) ? sr : cr;
    if (q == 1 || q == 2) cc = -cc;
    if (q >= 2) ss = -ss;
    *s = ss;
    *c = cc;
}

// 1/sqrt(x) for positive normal x by Newton's iteration y <- y (3/2 - x y^2 / 2) from the
// bit-level initial guess of Lomont, "Fast inverse square root" (2003): 3 iterations in float,
// 5 in double reach the working precision (within ~2 ulp; deterministic, not correctly rounded).
// Newton steps y <- y (3/2 - x y^2 / 2) from Lomont's initial guess.  The early steps are written
// as 1.5 y - (x/2 y) y^2, whose three products are independent and joined by one multiply-add (two
// dependent operations instead of three: the field's rsqrt is on the step's critical path); the
// last keeps the form y (1.5 - (x/2 y) y), which rounds less.
DSMC_HD float rsqrt_step(float y, float hx) { return xfma(-(hx * y), y * y, 1.5f * y); }
DSMC_HD double rsqrt_step(double y, double hx) { return xfma(-(hx * y), y * y, 1.5 * y); }
DSMC_HD float xrsqrt(float x) {
    float y = u2f(0x5f375a86u - (f2u(x) >> 1));
    const float hx = 0.5f * x;
    y = rsqrt_step(y, hx);
    y = rsqrt_step(y, hx);
    y = y * xfma(-(hx * y), y, 1.5f);
    return y;
}
DSMC_HD double xrsqrt(double x) {
    double y = u2d(0x5fe6eb50c7b537a9ull - (d2u(x) >> 1));
    const double hx = 0.5 * x;
    y = rsqrt_step(y, hx);
    y = rsqrt_step(y, hx);
    y = rsqrt_step(y, hx);
    y = rsqrt_step(y, hx);
    y = y * xfma(-(hx * y), y, 1.5);
    return y;
}

// 1/sqrt(n2) for the squared norm of a spinor the step keeps normalised: a unitary rotation moves
// n2 from 1 only by rounding, so with d = 1 - n2 (exact for n2 near 1) the series
// 1/sqrt(1 - d) = 1 + d/2 + 3 d^2/8 + ..., cut after d^2, is exact to well under an ulp when
// |d| < 2^-12 (float; 2^-18 for double); anything further from 1 takes the Newton rsqrt.  Two
// dependent multiply-adds in place of the rsqrt's chain on the step's critical path.
DSMC_HD float inv_norm(float n2) {
    const float d = 1.0f - n2;
    if (xabs(d) < 0x1p-12f) return xfma(d, xfma(d, 0.375f, 0.5f), 1.0f);
    return xrsqrt(n2);
}
DSMC_HD double inv_norm(double n2) {
    const double d = 1.0 - n2;
    if (xabs(d) < 0x1p-18) return xfma(d, xfma(d, 0.375, 0.5), 1.0);
    return xrsqrt(n2);
}

// natural log for normal positive x
DSMC_HD float xlog(float x) {
    uint32_t u = f2u(x);
    int e = (int)(u >> 23) - 127;
    float m = u2f((u & 0x7FFFFFu) | 0x3F800000u);
    if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
    float s = (m - 1.0f) / (m + 1.0f);
    float s2 = s * s;
    // atanh series: 2 s (1 + s^2/3 + s^4/5 + s^6/7 + s^8/9)
    float p = xfma(s2, 0.111111111f, 0.142857143f);
    p = xfma(s2, p, 0.2f);
    p = xfma(s2, p, 0.333333333f);
    float lm = xfma(2.0f * s * s2, p, 2.0f * s);
    const float ln2_hi = 0x1.62ep-1f, ln2_lo = 0x1.0bfbe8p-15f;
    float fe = (float)e;
    return xfma(fe, ln2_hi, xfma(fe, ln2_lo, lm));
}

DSMC_HD double xlog(double x) {
    uint64_t u = d2u(x);
    int e = (int)(u >> 52) - 1023;
    double m = u2d((u & 0xFFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
    if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
    double s = (m - 1.0) / (m + 1.0);
    double s2 = s * s;
    double p = xfma(s2, 1.0 / 21.0, 1.0 / 19.0);
    p = xfma(s2, p, 1.0 / 17.0);
    p = xfma(s2, p, 1.0 / 15.0);
    p = xfma(s2, p, 1.0 / 13.0);
    p = xfma(s2, p, 1.0 / 11.0);
    p = xfma(s2, p, 1.0 / 9.0);
    p = xfma(s2, p, 1.0 / 7.0);
    p = xfma(s2, p, 1.0 / 5.0);
    p = xfma(s2, p, 1.0 / 3.0);
    double lm = xfma(2.0 * s * s2, p, 2.0 * s);
    const double ln2_hi = 0x1.62e42ffp-1, ln2_lo = -0x1.718432a1b0e26p-35;
    double fe = (double)e;
    return xfma(fe, ln2_hi, xfma(fe, ln2_lo, lm));
}

DSMC_HD float xexp(float x) {
    if (x < -87.0f) return 0.0f;
    if (x > 88.0f) x = 88.0f;
    float k = xrint(x * 0x1.715476p+0f);
    float r = xfma(-k, 0x1.62ep-1f, x);
    r = xfma(-k, 0x1.0bfbe8p-15f, r);
    float p = xfma(r, 1.98412698e-4f, 1.38888889e-3f);  // 1/7!, 1/6!
    p = xfma(r, p, 8.33333333e-3f);
    p = xfma(r, p, 4.16666667e-2f);
    p = xfma(r, p, 1.66666667e-1f);
    p = xfma(r, p, 0.5f);
    p = xfma(r, p, 1.0f);
    p = xfma(r, p, 1.0f);
    return p * u2f((uint32_t)((int)k + 127) << 23);
}

DSMC_HD double xexp(double x) {
    if (x < -708.0) return 0.0;
    if (x > 709.0) x = 709.0;
    double k = xrint(x * 0x1.71547652b82fep+0);
    double r = xfma(-k, 0x1.62e42ffp-1, x);
    r = xfma(-k, -0x1.718432a1b0e26p-35, r);
    double p = xfma(r, 1.6059043836821613e-10, 2.0876756987868099e-9);  // 1/13!, 1/12!
    p = xfma(r, p, 2.5052108385441720e-8);
    p = xfma(r, p, 2.7557319223985891e-7);
    p = xfma(r, p, 2.7557319223985893e-6);
    p = xfma(r, p, 2.4801587301587302e-5);
    p = xfma(r, p, 1.9841269841269841e-4);
    p = xfma(r, p, 1.3888888888888889e-3);
    p = xfma(r, p, 8.3333333333333333e-3);
    p = xfma(r, p, 4.1666666666666667e-2);
    p = xfma(r, p, 1.6666666666666667e-1);
    p = xfma(r, p, 0.5);
    p = xfma(r, p, 1.0);
    p = xfma(r, p, 1.0);
    return p * u2d((uint64_t)((long long)k + 1023) << 52);
}

// ---------------------------------------------------------------------------------------
// Exact fixed-point accumulation for diagnostics: a value d, its magnitude clamped to 2^38 (no
// physical v^2 or |B| comes near; NaN clamps too), maps to sign(d) floor(|d| 2^64) as a 128-bit
// integer.  Sums of these are exact and therefore independent of summation order (GPU tiles,
// CPU loop, batched or single clouds).  The integer part of |d| and its fraction scaled by 2^64
// are both exact in the value's own precision, so the float and double forms agree bit for bit
// on every float input.
// ---------------------------------------------------------------------------------------
template <class R> DSMC_HD i128 fx_from_magnitude(R m) {
    if (!(m < R(0x1p38))) m = R(0x1p38);
    const R h = xfloor(m);
    const int64_t hi = (int64_t)h;
    const uint64_t lo = (uint64_t)((m - h) * R(0x1p64));
    return (i128)(((unsigned __int128)(uint64_t)hi << 64) | (unsigned __int128)lo);
}
DSMC_HD i128 fx_from(double d) { return d < 0.0 ? -fx_from_magnitude(-d) : fx_from_magnitude(d); }
DSMC_HD i128 fx_from(float f) { return f < 0.0f ? -fx_from_magnitude(-f) : fx_from_magnitude(f); }
DSMC_HD double fx_to_double(i128 q) {
    int64_t hi = (int64_t)(q >> 64);
    uint64_t lo = (uint64_t)q;
    return (double)hi + (double)lo * 0x1p-64;
}

// knife temperature after a step: T = m sum(v^2) / (3 kB n) from the exact fixed-point sum
DSMC_HD double knife_temperature(double mass, double kB, double T0, bool fixed_T, i128 sum_v2, long long n) {
    if (fixed_T || n <= 0) return T0;
    return mass * fx_to_double(sum_v2) / (3.0 * kB * (double)n);
}

// ---------------------------------------------------------------------------------------
// Parameters of one cloud as the kernels see them (derived on the host from
// dsmc_cloud_params + dsmc_params, identically for the GPU engine and the oracle).
// ---------------------------------------------------------------------------------------
enum { TRAP_QUADRUPOLE = 0, TRAP_IOFFE_PRITCHARD = 1, TRAP_BOX = 2 };
enum {
    F_COLLIDE = 1, F_LARMOR = 2, F_MAJORANA = 4, F_KNIFE = 8, F_NORMALISE = 16, F_KNIFE_FIXED_T = 32,
    F_MCWF = 64
};

template <class R> struct CloudPhys {
    int32_t trap, flags;
    int32_t nx, ny, nz;
    int32_t cell_base;   // global id of grid cell (0,0,0)
    int32_t ovf_cell;    // global id of the overflow cell = cell_base + nx*ny*nz
    int32_t cloud_id;
    R gmin_x, gmin_y, gmin_z;
    R inv_dx, inv_dy, inv_dz;
    R box_x, box_y, box_z;       // grid box edge lengths (periodic wrap)
    R inv_box_x, inv_box_y, inv_box_z;
    R fnx, fny, fnz;              // nx, ny, nz as reals (the grid's extent in cell units)
    R Bp, Bpp, B0, B_floor;       // gradient, curvature, bias, trap-bottom |B|
    R dt, half_dt;
    R accel_scale;                // mu / m
    R theta_per_B;                // mu dt / hbar
    R kappa;                      // 2 mu / m: energy per (m/2) in units of v^2 per tesla
    R sigma;                      // cross-section
    R cand_pref;                  // alpha * dt_collide / V_cell
    R v_init;                     // sqrt(kB T0 / m)
    R r0_init;                    // kB T0 / mu  (quadrupole thermal length)
    R inv_kT_over_mu;             // mu / (kB T0) for rejection sampling
    R mcwf_cp;                    // 1.163 sqrt(sigma): tau_pos = mcwf_cp / sqrt(2 |a|)
    R mcwf_cv;                    // sqrt(2/pi) hbar / (m sigma): tau_vel = mcwf_cv / (2 |a|)
    R dt_period;                  // collide_every * dt: the MCWF period
    R prop_min_x, prop_min_y, prop_min_z;  // proposal box of the rejection sampler
    R prop_len_x, prop_len_y, prop_len_z;
    int32_t knife_nknots;
    int32_t id_base;  // first slot of this cloud in by-atom-id records (the capacities of the clouds before it)
    int32_t id_cap;   // atom ids of this cloud that have a slot there (its capacity)
    int32_t pad0;
    double knife_step[9];
    double knife_eta[9];
    double mass, moment, kB, T0;  // for diagnostics and the knife cut
};

// piecewise-linear knife eta(step), constant outside the knots
DSMC_HD double knife_eta(const int32_t nk, const double* ks, const double* ke, double step) {
    if (nk <= 0) return 1e300;
    if (step <= ks[0]) return ke[0];
    for (int i = 1; i < nk; ++i) {
        if (step <= ks[i]) {
            double f = (step - ks[i - 1]) / (ks[i] - ks[i - 1]);
            return ke[i - 1] + f * (ke[i] - ke[i - 1]);
        }
    }
    return ke[nk - 1];
}

// knife cut in units of v^2 (E / (m/2)): 2 eta kB T / m
DSMC_HD double knife_cut_v2(double eta, double kB, double T, double mass) {
    return 2.0 * eta * kB * T / mass;
}

// ---------------------------------------------------------------------------------------
// Trap field: B, |B|, B^ and grad|B| at a point.
// ---------------------------------------------------------------------------------------
template <class R> struct Field {
    R bx, by, bz;     // unit vector B^
    R absB;           // |B|
    R gx, gy, gz;     // grad |B|
};

template <class R>
DSMC_HD void trap_field(const CloudPhys<R>& P, R x, R y, R z, Field<R>& f) {
    if (P.trap == TRAP_QUADRUPOLE) {
        // B = (h x, h y, B0 - B' z), h = B'/2;  grad|B| = (h B^x, h B^y, -B' B^z)
        const R h = R(0.5) * P.Bp;
        const V2<R> Bxy = mul2(v2s(h), v2(x, y));
        const R Bz = xfma(-P.Bp, z, P.B0);
        const R b2 = xfma(Bz, Bz, xfma(Bxy.y, Bxy.y, Bxy.x * Bxy.x));
        if (b2 > R(0)) {
            const R inv = xrsqrt(b2);
            f.absB = b2 * inv;
            const V2<R> bxy = mul2(Bxy, v2s(inv));
            f.bx = bxy.x; f.by = bxy.y; f.bz = Bz * inv;
        } else {
            f.absB = R(0);
            f.bx = R(0); f.by = R(0); f.bz = R(1);
        }
        const V2<R> gxy = mul2(v2s(h), v2(f.bx, f.by));
        f.gx = gxy.x;
        f.gy = gxy.y;
        f.gz = -(P.Bp * f.bz);
        return;
    }
    if (P.trap == TRAP_IOFFE_PRITCHARD) {
        // CUDADSMC/src/moveAtoms.cu:135-157
        const R hc = R(0.5) * P.Bpp;
        const R Bx = P.Bp * x - hc * (x * z);
        const R By = -(P.Bp * y) - hc * (y * z);
        const R Bz = P.B0 + hc * (z * z - R(0.5) * (x * x + y * y));
        const R b2 = Bx * Bx + By * By + Bz * Bz;
        if (b2 > R(0)) {
            const R inv = xrsqrt(b2);
            f.absB = b2 * inv;
            f.bx = Bx * inv; f.by = By * inv; f.bz = Bz * inv;
        } else {
            f.absB = R(0);
            f.bx = R(0); f.by = R(0); f.bz = R(1);
        }
        // d|B|/dx_j = B^ . dB/dx_j  (columns of the Jacobian, moveAtoms.cu:144-157)
        const R jxx = P.Bp - hc * z, jxz = -(hc * x);
        const R jyy = -P.Bp - hc * z, jyz = -(hc * y);
        const R jzx = -(hc * x), jzy = -(hc * y), jzz = P.Bpp * z;
        f.gx = f.bx * jxx + f.bz * jzx;
        f.gy = f.by * jyy + f.bz * jzy;
        f.gz = f.bx * jxz + f.by * jyz + f.bz * jzz;
        return;
    }
    f.bx = R(0); f.by = R(0); f.bz = R(1);
    f.absB = R(0);
    f.gx = R(0); f.gy = R(0); f.gz = R(0);
}

// ---------------------------------------------------------------------------------------
// Cell index (collisions.cu:194-219): floor((x - xmin) / dx) per axis, linear id
// z*nx*ny + y*nx + x, atoms outside the grid go to the cloud's overflow cell.
// Evaluated as (x - xmin) * (1/dx) without contraction, identically on host and device.
// ---------------------------------------------------------------------------------------
template <class R>
DSMC_HD int32_t cell_of(const CloudPhys<R>& P, R x, R y, R z, bool periodic) {
    const V2<R> fxy = mul2(sub2(v2(x, y), v2(P.gmin_x, P.gmin_y)), v2(P.inv_dx, P.inv_dy));
    R fx = fxy.x;
    R fy = fxy.y;
    R fz = (z - P.gmin_z) * P.inv_dz;
    if (periodic) {
        int ix = (fx >= R(0)) ? (int)fx : 0;
        int iy = (fy >= R(0)) ? (int)fy : 0;
        int iz = (fz >= R(0)) ? (int)fz : 0;
        if (!(fx == fx) || !(fy == fy) || !(fz == fz)) return P.ovf_cell;
        ix = ix < P.nx ? ix : P.nx - 1;
        iy = iy < P.ny ? iy : P.ny - 1;
        iz = iz < P.nz ? iz : P.nz - 1;
        return P.cell_base + (iz * P.ny + iy) * P.nx + ix;
    }
    if (!(fx >= R(0) && fx < P.fnx && fy >= R(0) && fy < P.fny && fz >= R(0) && fz < P.fnz))
        return P.ovf_cell;
    int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    return P.cell_base + (iz * P.ny + iy) * P.nx + ix;
}

// ---------------------------------------------------------------------------------------
// One timestep of one atom: Larmor rotation about B^(x) (evolveWavefunction runs before
// moveAtoms, main.cu:465-476), renormalisation, velocity Verlet kick-drift-kick with the
// acceleration recomputed from the position (no stored a), periodic wrap for the box,
// then the evaporation tests at the new position (evaporationTag, evaporation.cu:68-106)
// and the new cell.
// ---------------------------------------------------------------------------------------
template <class R> struct Atom {
    R x, y, z, vx, vy, vz;
    R ur, ui, dr, di;  // psi_up, psi_dn
    uint32_t flags;    // bit 0: anti-trapped; bits 2..31: MCWF period-start population (mcwf_store)
};

// Per-atom context of a step: the atom id, the step number and seed for the spin-flip random
// number, and the MCWF phase (bit 0: record the trapped population, bit 1: flip and decay)
struct StepCtx {
    uint32_t id;
    uint32_t step;
    uint32_t cloud;
    uint32_t mcwf;
    uint64_t seed;
};

enum { FATE_ALIVE = 0, FATE_MAJORANA = 1, FATE_KNIFE = 2 };

template <class R> struct AtomOut {
    int32_t cell;
    int32_t fate;
    R v2;     // |v|^2 after the step
    R absB;   // s |B| after the step: s = +1 trapped, -1 anti-trapped (potential energy / mu)
};

// ---------------------------------------------------------------------------------------
// MCWF spin flips and decoherence (wavefunction.cu:75-237; scheduled by main.cu:457-520: the
// populations are taken after the collisions, the flip and the decay follow the last motion
// step of the collision period).
// ---------------------------------------------------------------------------------------
// trapped-state population (1 + <s.B^>)/2 in the reference's form for a normalised spinor:
// 1/2 + Bx Re(u* d) + By Im(u* d) - Bz (1/2 - |u|^2)   (projectLocalPopulations, :162-170)
template <class R> DSMC_HD R trapped_population(const Field<R>& f, const Atom<R>& a) {
    const R re = a.ur * a.dr + a.ui * a.di;
    const R im = a.ur * a.di - a.ui * a.dr;
    const R u2 = a.ur * a.ur + a.ui * a.ui;
    return R(0.5) + f.bx * re + f.by * im - f.bz * (R(0.5) - u2);
}
// the period-start population kept in flag bits 2..31 as floor(x 2^30), x clamped to [0, 1)
template <class R> DSMC_HD uint32_t mcwf_store(uint32_t flags, R x) {
    const R xc = x >= R(0) ? (x < R(1) ? x : R(1) - R(1) / R(1 << 24)) : R(0);  // NaN -> 0
    uint32_t q = (uint32_t)(xc * R(1 << 30));
    q = q < (1u << 30) ? q : (1u << 30) - 1u;
    return (flags & 3u) | (q << 2);
}
template <class R> DSMC_HD R mcwf_load(uint32_t flags) { return (R)(flags >> 2) * (R(1) / R(1 << 30)); }

// End of a collision period: the jump to the other state with probability (y1 - y0)/x0 for a
// trapped atom, (x1 - x0)/y0 for an anti-trapped one (y = 1 - x), taken when the kinetic
// energy stays positive after the change 2 mu |B| of potential energy, the speed rescaled to
// conserve energy (flipAtoms, :99-156); then decoherence towards the eigenstates of s.B^ over
// the period, psi <- [(1 - e) (s.B^) psi + (1 + e) psi] / 2 with e = exp(-dt_c / tau), tau from the
// local acceleration (exponentialDecay + calculateTau, :175-223), and renormalisation.
template <class R>
DSMC_HD void mcwf_end(const CloudPhys<R>& P, const Field<R>& f, Atom<R>& a, const StepCtx& sc) {
    const R x0 = mcwf_load<R>(a.flags);
    const R x1 = trapped_population(f, a);
    const bool trapped = !(a.flags & 1u);
    const R pflip = trapped ? ((R(1) - x1) - (R(1) - x0)) / x0 : (x1 - x0) / (R(1) - x0);
    const R dv2 = trapped ? R(2) * P.kappa * f.absB : -(R(2) * P.kappa * f.absB);  // dE / (m/2)
    const R vv = xfma(a.vz, a.vz, xfma(a.vy, a.vy, a.vx * a.vx));
    const u32x4 w = draw(sc.id, sc.step, PURPOSE_FLIP, sc.cloud, 0u, sc.seed);
    const R u = u01<R>(w.x, w.y);
    if (pflip > u && vv + dv2 > R(0) && vv > R(0)) {
        a.flags ^= 1u;
        const R s = xsqrt(vv + dv2) / xsqrt(vv);
        const V2<R> vxy = mul2(v2(a.vx, a.vy), v2s(s));
        a.vx = vxy.x;
        a.vy = vxy.y;
        a.vz = a.vz * s;
    }
    // decoherence: 1/tau = (tau_pos^-3 + tau_vel^-3)^(1/3), relative acceleration 2 |a|
    const R g = xsqrt(xfma(f.gz, f.gz, xfma(f.gy, f.gy, f.gx * f.gx)));
    const R rel = R(2) * P.accel_scale * g;
    R e = R(1);
    if (rel > R(0)) {
        const R ip = xsqrt(rel) / P.mcwf_cp;  // 1 / tau_pos
        const R iv = rel / P.mcwf_cv;         // 1 / tau_vel
        const R s3 = ip * ip * ip + iv * iv * iv;
        const R rate = xexp(xlog(s3) * (R(1) / R(3)));
        e = xexp(-(P.dt_period * rate));
    }
    const R om = R(1) - e, op = R(1) + e;
    const R ur = R(0.5) * ((f.bx * a.dr + f.by * a.di + f.bz * a.ur) * om + a.ur * op);
    const R ui = R(0.5) * ((f.bx * a.di - f.by * a.dr + f.bz * a.ui) * om + a.ui * op);
    const R dr = R(0.5) * ((f.bx * a.ur - f.by * a.ui - f.bz * a.dr) * om + a.dr * op);
    const R di = R(0.5) * ((f.bx * a.ui + f.by * a.ur - f.bz * a.di) * om + a.di * op);
    const R n2 = ur * ur + ui * ui + dr * dr + di * di;
    const R inv = xrsqrt(n2);
    a.ur = ur * inv; a.ui = ui * inv; a.dr = dr * inv; a.di = di * inv;
}

template <class R>
DSMC_HD void advance_atom(const CloudPhys<R>& P, R cut_v2, Atom<R>& a, AtomOut<R>& o, const StepCtx& sc) {
    const bool box = (P.trap == TRAP_BOX);
    Field<R> f0;
    trap_field(P, a.x, a.y, a.z, f0);
    if ((P.flags & F_MCWF) && !box && (sc.mcwf & 1u)) a.flags = mcwf_store(a.flags, trapped_population(f0, a));

    if ((P.flags & F_LARMOR) && !box) {
        // psi <- [cos t - i sin t (s.B^)] psi, t = mu |B| dt / hbar   (wavefunction.cu:39-73):
        //   ur' = ur c + ( bx di - by dr + bz ui) s     ui' = ui c + (-bx dr - by di - bz ur) s
        //   dr' = dr c + ( bx ui + by ur - bz di) s     di' = di c + (-bx ur + by ui + bz dr) s
        // with the (up, down) rows as two-lane pairs
        R th = P.theta_per_B * f0.absB;
        R s, c;
        xsincos(th, &s, &c);
        const V2<R> u = v2(a.ur, a.ui), d = v2(a.dr, a.di);
        const V2<R> tu = fma2(v2(f0.bz, -f0.bz), v2(a.ui, a.ur),
                              fma2(v2s(-f0.by), d, mul2(v2(f0.bx, -f0.bx), v2(a.di, a.dr))));
        const V2<R> td = fma2(v2(-f0.bz, f0.bz), v2(a.di, a.dr),
                              fma2(v2s(f0.by), v2(a.ur, a.ui), mul2(v2(f0.bx, -f0.bx), v2(a.ui, a.ur))));
        V2<R> nu = fma2(tu, v2s(s), mul2(u, v2s(c)));
        V2<R> nd = fma2(td, v2s(s), mul2(d, v2s(c)));
        if (P.flags & F_NORMALISE) {
            const V2<R> q = fma2(nd, nd, mul2(nu, nu));
            const R inv = inv_norm(q.x + q.y);
            nu = mul2(nu, v2s(inv));
            nd = mul2(nd, v2s(inv));
        }
        a.ur = nu.x; a.ui = nu.y; a.dr = nd.x; a.di = nd.y;
    }

    // velocity Verlet (moveAtoms.cu:51-65); anti-trapped atoms feel +grad|B|
    const R sgn = (a.flags & 1u) ? R(1) : R(-1);
    const R kick = P.half_dt * (sgn * P.accel_scale);
    V2<R> vxy = fma2(v2s(kick), v2(f0.gx, f0.gy), v2(a.vx, a.vy));
    a.vz = xfma(kick, f0.gz, a.vz);
    const V2<R> xy = fma2(v2s(P.dt), vxy, v2(a.x, a.y));
    a.x = xy.x;
    a.y = xy.y;
    a.z = xfma(P.dt, a.vz, a.z);
    if (box) {
        a.x = a.x - P.box_x * xfloor((a.x - P.gmin_x) * P.inv_box_x);
        a.y = a.y - P.box_y * xfloor((a.y - P.gmin_y) * P.inv_box_y);
        a.z = a.z - P.box_z * xfloor((a.z - P.gmin_z) * P.inv_box_z);
    }
    Field<R> f1;
    trap_field(P, a.x, a.y, a.z, f1);
    vxy = fma2(v2s(kick), v2(f1.gx, f1.gy), vxy);
    a.vx = vxy.x;
    a.vy = vxy.y;
    a.vz = xfma(kick, f1.gz, a.vz);

    o.v2 = xfma(a.vz, a.vz, xfma(a.vy, a.vy, a.vx * a.vx));
    o.absB = f1.absB;
    o.fate = FATE_ALIVE;
    if ((P.flags & F_MAJORANA) && !box) {
        // <s.B^> = 2 Bx Re(u* d) + 2 By Im(u* d) + Bz (|u|^2 - |d|^2)   (evaporation.cu:88-90)
        const V2<R> ri = fma2(v2(a.ui, -a.ui), v2(a.di, a.dr), mul2(v2s(a.ur), v2(a.dr, a.di)));  // Re, Im
        const V2<R> nn = fma2(v2(a.ui, a.di), v2(a.ui, a.di), mul2(v2(a.ur, a.dr), v2(a.ur, a.dr)));
        const R sz = nn.x - nn.y;
        const R proj = xfma(f1.bz, sz, R(2) * xfma(f1.bx, ri.x, f1.by * ri.y));
        if (proj < R(0)) o.fate = FATE_MAJORANA;
    }
    if ((P.flags & F_KNIFE) && o.fate == FATE_ALIVE) {
        R e = xfma(P.kappa, f1.absB - P.B_floor, o.v2);
        if (e > cut_v2) o.fate = FATE_KNIFE;
    }
    if ((P.flags & F_MCWF) && !box && (sc.mcwf & 2u) && o.fate == FATE_ALIVE) {
        mcwf_end(P, f1, a, sc);
        o.v2 = xfma(a.vz, a.vz, xfma(a.vy, a.vy, a.vx * a.vx));
    }
    if (a.flags & 1u) o.absB = -o.absB;
    o.cell = cell_of(P, a.x, a.y, a.z, box);
}

// ---------------------------------------------------------------------------------------
// No-time-counter collisions in one cell (collisions.cu:306-437 with the intended
// semantics): Mc = n(n-1)/2 candidate pairs, Ncand = ceil(Mc alpha dt_c (sigma v_r)max / V),
// each candidate is a uniformly chosen distinct pair (i, j) accepted with probability
// sigma v_r alpha dt_c Mc / (V Ncand); accepted pairs scatter isotropically about their
// centre of mass (collisions.cu:425-437, 537-546).  vel points at n consecutive atoms
// (4 reals each).  Random numbers: one Philox block per candidate keyed by
// (cell, step, cloud, candidate), the second one only for accepted pairs.
// ---------------------------------------------------------------------------------------
template <class R> struct CollideResult {
    int32_t accepted;
    int32_t candidates;
};

// receives every accepted collision (cell-local indices i, j and the direction n^); the
// default records nothing
struct NoCollisionLog {
    template <class R> DSMC_HD void accept(uint32_t, uint32_t, R, R, R) {}
};

// Element access of the velocities a cell's collisions update: a plain array of n consecutive
// 4-lane vectors here; the GPU step passes an accessor that reaches each atom through the sorted
// order's permutation (vload / vstore overloads beside it).
template <class V4> DSMC_HD V4 vload(V4* vel, uint32_t i) { return vel[i]; }
template <class V4> DSMC_HD void vstore(V4* vel, uint32_t i, const V4& v) { vel[i] = v; }

template <class R, class VA, class Log = NoCollisionLog>
DSMC_HD CollideResult<R> collide_cell(VA vel, int n, R& sigvrmax, const CloudPhys<R>& P,
                                      uint32_t local_cell, uint32_t step, uint64_t seed, Log* log = nullptr) {
    CollideResult<R> res;
    res.accepted = 0;
    res.candidates = 0;
    if (n < 2) return res;
    const R Mc = R(0.5) * ((R)n * (R)(n - 1));
    const R x = Mc * P.cand_pref * sigvrmax;
    const R ncf = xceil(x);
    if (!(ncf >= R(1))) return res;
    const int ncand = ncf < R(1 << 24) ? (int)ncf : (1 << 24);
    const R pacc = (P.cand_pref * Mc) / ncf;
    const R two_pi = R(6.283185307179586476925286766559);
    for (int k = 0; k < ncand; ++k) {
        const u32x4 w = draw(local_cell, step, PURPOSE_COLLIDE, (uint32_t)P.cloud_id, 2u * (uint32_t)k, seed);
        uint32_t i = index_below(w.x, (uint32_t)n);
        uint32_t j = index_below(w.y, (uint32_t)(n - 1));
        j += (j >= i) ? 1u : 0u;
        auto vi = vload(vel, i);
        auto vj = vload(vel, j);
        R dx = vi.x - vj.x, dy = vi.y - vj.y, dz = vi.z - vj.z;
        R vr = xsqrt(dx * dx + dy * dy + dz * dz);
        R svr = P.sigma * vr;
        if (svr > sigvrmax) sigvrmax = svr;
        R pa = svr * pacc;
        R u = u01<R>(w.z, w.w);
        if (u < pa) {
            // the scattering angles come from a second block, drawn only for accepted pairs
            const u32x4 w2 = draw(local_cell, step, PURPOSE_COLLIDE, (uint32_t)P.cloud_id, 2u * (uint32_t)k + 1u, seed);
            R ct = R(2) * u01<R>(w2.x, w2.y) - R(1);
            R st2 = R(1) - ct * ct;
            R st = xsqrt(st2 > R(0) ? st2 : R(0));
            R phi = two_pi * u01<R>(w2.z, w2.w);
            R sp, cp;
            xsincos(phi, &sp, &cp);
            R hv = R(0.5) * vr;
            R nx = st * cp, ny = st * sp, nz = ct;
            R cx = R(0.5) * (vi.x + vj.x), cy = R(0.5) * (vi.y + vj.y), cz = R(0.5) * (vi.z + vj.z);
            vi.x = cx + hv * nx; vi.y = cy + hv * ny; vi.z = cz + hv * nz;
            vj.x = cx - hv * nx; vj.y = cy - hv * ny; vj.z = cz - hv * nz;
            vstore(vel, i, vi);
            vstore(vel, j, vj);
            res.accepted += 1;
            if (log) log->accept(i, j, nx, ny, nz);
        }
    }
    res.candidates = ncand;
    return res;
}

// ---------------------------------------------------------------------------------------
// Initial state of one atom (generateInitialDist, setUp.cu:129-165, with an exact sampler):
//   quadrupole: scaled radius rho = sqrt(x^2/4+y^2/4+z^2) has density ~ rho^2 exp(-rho/r0),
//     i.e. Gamma(3, r0): rho = -r0 log(u1 u2 u3); direction isotropic in (x/2, y/2, z);
//   Ioffe-Pritchard: bounded rejection sampling, uniform proposal over a box of +-7 thermal
//     widths of the harmonic approximation (clipped to the grid box), acceptance
//     exp(-mu (|B| - B_floor) / kT);
//   box: uniform over the grid box.
// Velocities: Maxwellian N(0, kT/m) per axis by Box-Muller.  Spinor aligned with B^
// (the +1 eigenvector of s.B^, without the rsqrt(1 + B^x) singularity of setUp.cu:240).
// Returns false if rejection sampling gave up (the atom is then placed at the trap centre).
// ---------------------------------------------------------------------------------------
template <class R>
DSMC_HD bool init_atom(const CloudPhys<R>& P, int init_mode, uint32_t local_id, uint64_t seed,
                       Atom<R>& a) {
    const R two_pi = R(6.283185307179586476925286766559);
    bool ok = true;
    if (init_mode == 1 || P.trap == TRAP_BOX) {
        u32x4 w = draw(local_id, 0u, PURPOSE_INIT_POS, (uint32_t)P.cloud_id, 0u, seed);
        u32x4 w2 = draw(local_id, 0u, PURPOSE_INIT_POS, (uint32_t)P.cloud_id, 1u, seed);
        a.x = P.gmin_x + P.box_x * u01<R>(w.x, w2.x);
        a.y = P.gmin_y + P.box_y * u01<R>(w.y, w2.y);
        a.z = P.gmin_z + P.box_z * u01<R>(w.z, w2.z);
    } else if (P.trap == TRAP_QUADRUPOLE) {
        u32x4 w = draw(local_id, 0u, PURPOSE_INIT_POS, (uint32_t)P.cloud_id, 0u, seed);
        u32x4 w2 = draw(local_id, 0u, PURPOSE_INIT_POS, (uint32_t)P.cloud_id, 1u, seed);
        R u1 = u01<R>(w.x, w2.x), u2 = u01<R>(w.y, w2.y), u3 = u01<R>(w.z, w2.z);
        R rho = -P.r0_init * (xlog(u1) + xlog(u2) + xlog(u3));
        R ct = R(2) * u01<R>(w.w, w2.w) - R(1);
        u32x4 w3 = draw(local_id, 0u, PURPOSE_INIT_POS, (uint32_t)P.cloud_id, 2u, seed);
        R phi = two_pi * u01<R>(w3.x, w3.y);
        R st2 = R(1) - ct * ct;
        R st = xsqrt(st2 > R(0) ? st2 : R(0));
        R sp, cp;
        xsincos(phi, &sp, &cp);
        // scaled coordinates (x/2, y/2, z) are isotropic; the bias shifts the zero along z
        a.x = R(2) * (rho * (st * cp));
        a.y = R(2) * (rho * (st * sp));
        a.z = rho * ct + (P.Bp != R(0) ? P.B0 / P.Bp : R(0));
    } else {
        ok = false;
        a.x = R(0); a.y = R(0); a.z = R(0);
        for (uint32_t t = 0; t < 4096u; ++t) {
            u32x4 w = draw(local_id, t, PURPOSE_INIT_POS, (uint32_t)P.cloud_id, 0u, seed);
            u32x4 w2 = draw(local_id, t, PURPOSE_INIT_POS, (uint32_t)P.cloud_id, 1u, seed);
            R x = P.prop_min_x + P.prop_len_x * u01<R>(w.x, w2.x);
            R y = P.prop_min_y + P.prop_len_y * u01<R>(w.y, w2.y);
            R z = P.prop_min_z + P.prop_len_z * u01<R>(w.z, w2.z);
            Field<R> f;
            trap_field(P, x, y, z, f);
            R pr = xexp(-(P.inv_kT_over_mu * (f.absB - P.B_floor)));
            if (u01<R>(w.w, w2.w) < pr) {
                a.x = x; a.y = y; a.z = z;
                ok = true;
                break;
            }
        }
    }
    // Maxwellian velocities by Box-Muller
    u32x4 v = draw(local_id, 0u, PURPOSE_INIT_VEL, (uint32_t)P.cloud_id, 0u, seed);
    u32x4 v2 = draw(local_id, 0u, PURPOSE_INIT_VEL, (uint32_t)P.cloud_id, 1u, seed);
    R g[4];
    {
        R r1 = xsqrt(R(-2) * xlog(u01<R>(v.x, v2.x)));
        R s1, c1;
        xsincos(two_pi * u01<R>(v.y, v2.y), &s1, &c1);
        R r2 = xsqrt(R(-2) * xlog(u01<R>(v.z, v2.z)));
        R s2, c2;
        xsincos(two_pi * u01<R>(v.w, v2.w), &s2, &c2);
        g[0] = r1 * c1; g[1] = r1 * s1; g[2] = r2 * c2; g[3] = r2 * s2;
    }
    a.vx = P.v_init * g[0];
    a.vy = P.v_init * g[1];
    a.vz = P.v_init * g[2];
    // aligned spinor
    Field<R> f;
    trap_field(P, a.x, a.y, a.z, f);
    if (f.bz >= R(0)) {
        R h = xsqrt(R(0.5) * (R(1) + f.bz));
        R inv = R(1) / (R(2) * h);
        a.ur = h; a.ui = R(0);
        a.dr = f.bx * inv; a.di = f.by * inv;
    } else {
        R h = xsqrt(R(0.5) * (R(1) - f.bz));
        R inv = R(1) / (R(2) * h);
        a.ur = f.bx * inv; a.ui = -(f.by * inv);
        a.dr = h; a.di = R(0);
    }
    a.flags = 0u;
    return ok;
}

}  // namespace dsmc

#endif  // DSMC_PHYSICS_H
