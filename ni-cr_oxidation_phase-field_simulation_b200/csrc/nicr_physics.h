// Pointwise physics of the Ni-Cr oxidation model, shared by host C++ and the
// CUDA kernels. Every expression keeps the reference's operand order and
// association, so that with FMA contraction disabled (nvcc -fmad=false, gcc on
// x86-64 without -march) device and host results are bit-identical to the
// reference's. Reference: 3S = mpi3d-slab/NiCr3D_grains.cpp,
// 2D = mpi2d/NiCr2D_grains.cpp.
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define NICR_HD __host__ __device__ __forceinline__
#else
#define NICR_HD inline
#endif

namespace nicr {

// struct Physics (3S:73-79). Vm = 1 divides exactly and is left out.
struct Phys {
    static constexpr double W = 1e4, ko = 1e-9, kc = 7.5e-9, kp = 1.7e-10, L = 0.2;
    static constexpr double bmo = 2.21e-16, bmc = 3.5436e-20, boo = 2.21e-18, boc = 3.5436e-21;
    static constexpr double ckO = 2e-10, ckCr = 2e-10, ksp = 1.28e-7;
    static constexpr double bulkO = 0., bulkCr = 0.1986, layerO = 0.0023, layerCr = 0.182;
    static constexpr double oxideO = 0.56300203, oxideCr = 0.35677915;
};

constexpr double PI = 3.14159265358979323846;

// h(phi) interpolation (3S:171) and its derivative (3S:87)
NICR_HD double h(double p) { return p * p * p * (10. - 15. * p + 6. * p * p); }
NICR_HD double hp(double p) { return 30. * p * p * (p - 1.) * (p - 1.); }
// minimum-image offset for a periodic axis (3S:172)
NICR_HD double min_image(double d, double period) { return d - period * round(d / period); }

// chemical free energies (3S:198-206)
NICR_HD double fmetal(double o, double cr) {
    return (6000000. * o * o + 583264.303945031 * cr * cr + 3200000. * o * cr
            - 298432. * o - 97045.64 * cr - 61732.2974223055);
}
NICR_HD double foxide(double o, double cr) {
    return (12000000. * o * o + 7000000. * cr * cr - 13800000. * o * cr
            - 8880000. * o + 2680000. * cr + 1860990.);
}
// chemical potentials without the gradient term (refresh, 3S:604-612)
NICR_HD double mu_o_local(double o, double cr, double hh) {
    return (1. - hh) * (12000000. * o + 3200000. * cr - 298432.) + hh * (24000000. * o - 13800000. * cr - 8880000.);
}
NICR_HD double mu_cr_local(double o, double cr, double hh) {
    return (1. - hh) * (1166528.60789006 * cr + 3200000. * o - 97045.64)
         + hh * (14000000. * cr - 13800000. * o + 2680000.);
}
// mobility(conc, p, gb) (3S:207-215); active_gb is gb when grains are on, else 0,
// gbm1 = gb_factor - 1 evaluated once per run (same value as the reference's).
NICR_HD double mobility(double conc, double hh, double active_gb, double bm, double bo, double gbm1) {
    return conc * ((1. - hh) * bm * (1. + gbm1 * active_gb) + hh * bo);
}
// std::min / std::max / std::clamp tie and NaN semantics
NICR_HD double smin(double a, double b) { return (b < a) ? b : a; }
NICR_HD double smax(double a, double b) { return (a < b) ? b : a; }
NICR_HD double sclamp(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

// Evolving-grain energy terms (3S:104-113); W = eta_W, A = eta_A
NICR_HD double grain_deta(double e, double S, double phi, double W, double A) {
    return e * (W * (S - (1. - h(phi)) + 2. * (S - e * e)) + A * h(phi));
}
NICR_HD double grain_dphi(double S, double phi, double W, double A) {
    return 0.5 * hp(phi) * (W * (S - (1. - h(phi))) + A * S);
}
NICR_HD double grain_energy_density(double S, double P, double phi, double W, double A) {
    const double H = h(phi), d = S - (1. - H);
    return 0.25 * W * d * d + W * P + 0.5 * A * H * S;
}

// Derived eta coefficients (3S:88-103). Evaluated on the host only.
struct EtaCoef {
    double K, ell, A, scale;
};
inline double reference_gb_width(double fwhm, double dx) {
    return fwhm * dx * std::sqrt(PI) / (2. * std::sqrt(std::log(2.)));
}
inline EtaCoef eta_coef(double fwhm, double dx, double W, double kappa, double penalty) {
    EtaCoef e;
    if (kappa > 0.) e.K = kappa;
    else {
        const double ell = 3. * reference_gb_width(fwhm, dx) / 8.;
        e.K = 2. * W * ell * ell;
    }
    e.ell = std::sqrt(e.K / (2. * W));
    e.A = penalty < 0. ? W : penalty;
    e.scale = reference_gb_width(fwhm, dx) / (8. * e.ell / 3.);
    return e;
}

// Division by a run constant b, correctly rounded (bit-identical to a / b).
// q1 = a*RN(1/b) refined by one FMA residual step is accepted only when an
// exact FMA residual proves it is the nearest double: |a - q1*b| < |b|*ulp(q1)/2
// (strict, so ties are excluded; q1 a power of two is excluded because its
// lower neighbour is closer). The residual is exact whenever q1 is within an
// ulp of a/b, and when it is not, its rounded value cannot pass the test, so
// an accepted q1 is always RN(a/b). Zeros return a * RN(1/b), the exactly
// signed zero. Outside the guarded exponent range (subnormals, infinities,
// NaNs) the IEEE division is used. The scale factor
// 2^(53-E) (E = exponent of q1) keeps the comparison free of underflow.
struct DivC {
    double b, rb;   // divisor and RN(1/b)
    int fast;       // b normal with 2^-60 <= |b| <= 2^60
    int pad;
};
inline DivC make_divc(double b) {
    DivC d;
    d.b = b;
    d.rb = 1.0 / b;
    const double ab = std::fabs(b);
    d.fast = (std::isnormal(b) && ab >= std::ldexp(1.0, -60) && ab <= std::ldexp(1.0, 60)) ? 1 : 0;
    d.pad = 0;
    return d;
}
#ifdef __CUDACC__
// IEEE division kept out of line: it is only the rare fallback, and inlining
// it at every call site would multiply the kernels' instruction footprint.
__device__ __noinline__ double ieee_div(double a, double b);
__device__ __forceinline__ double xdiv(double a, const DivC& d) {
#if defined(NICR_DIV_RECIP)
    return __dmul_rn(a, d.rb);
#elif defined(NICR_DIV_IEEE)
    return __ddiv_rn(a, d.b);
#else
    // Zeros (common: the Laplacian of a uniform region) return at once; the
    // rest is computed without branches, and one rarely taken branch picks
    // the IEEE division when the certificate fails.
    const long long ab = __double_as_longlong(a);
    const int ea = (int)((ab >> 52) & 0x7FF);
    const double q0 = __dmul_rn(a, d.rb);
    // +-0 / b is an exactly signed zero, which a * RN(1/b) reproduces
    if (d.fast && (ab << 1) == 0) return q0;
    const double r0 = __fma_rn(-q0, d.b, a);
    const double q1 = __fma_rn(r0, d.rb, q0);
    const double r1 = __fma_rn(-q1, d.b, a);
    const long long qb = __double_as_longlong(q1);
    const int eq = (int)((qb >> 52) & 0x7FF);
    // 2^(1076 - eq) = 1 / (ulp(q1) / 2); meaningful when a is in range, which
    // the certificate requires (the quotient's exponent then lies in [63, 1983])
    const double scale = __longlong_as_double((long long)((unsigned long long)(2099 - eq) << 52));
    const bool cert = ea >= 123 && ea <= 1923 && (qb & 0x000FFFFFFFFFFFFFLL) != 0 &&
                      __dmul_rn(fabs(r1), scale) < fabs(d.b);
    if (d.fast && cert) return q1;
#if defined(NICR_DIV_INLINE_FALLBACK)
    return __ddiv_rn(a, d.b);
#else
    return ieee_div(a, d.b);
#endif
#endif
}
#endif

// Double-double accumulation (Knuth two-sum). Budget sums that the reference
// keeps in 80-bit long double are kept as hi+lo pairs with ~106-bit precision.
struct DD {
    double hi, lo;
};
NICR_HD DD dd_add(DD a, double b) {
    const double s = a.hi + b;
    const double bb = s - a.hi;
    const double err = (a.hi - (s - bb)) + (b - bb);
    const double lo = a.lo + err;
    const double hi = s + lo;
    return DD{hi, lo - (hi - s)};
}
NICR_HD DD dd_add(DD a, DD b) {
    DD r = dd_add(a, b.hi);
    return dd_add(r, b.lo);
}

}  // namespace nicr
