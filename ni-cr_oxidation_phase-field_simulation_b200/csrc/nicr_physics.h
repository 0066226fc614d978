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
// The host stores y = RN(1/b) and the double-word reciprocal zh = RD(1/b),
// zl = RN(1/b - zh) >= 0 (Brisebarre, Muller, Raina, "Accelerating correctly
// rounded floating-point division when the divisor is known in advance",
// IEEE Trans. Comput. 53(8), 2004), the latter two scaled by 2^128. For b > 0
// with 2^-60 <= b <= 2^60 and a numerator a:
//   as = a * 2^128                  exact for |a| < 2^895, subnormals included,
//   q0 = RN(a*zh' + RN(a*zl'))      within (1/2 + 2^-51) ulp of as/b,
//   e  = q0*b - as                  exact: q0 is within one ulp of as/b, and
//                                   as/b >= 2^-1006 keeps its bits normal,
//   qs = RN(q0 - e*y)               = RN(as/b), Markstein's correction theorem
//                                   (IBM J. Res. Dev. 34(1), 1990: q0 within one
//                                   ulp, y within half an ulp of 1/b, exact
//                                   remainder => the correctly rounded quotient),
//   q  = qs * 2^-128                exact whenever a/b is normal or zero.
// The scaling keeps tiny numerators (the tails of diffusing fields) exact.
// Zeros come out with the IEEE sign because zl >= 0 and e is formed as
// q0*b - as. A quotient that is subnormal (qs nonzero below 2^-894, which the
// final scaling would round a second time), infinite or NaN (infinite, NaN or
// huge numerators), or any quotient of a divisor outside the range, is
// flagged. tests/division_check.c restates this on the host and checks it
// against IEEE division, near-midpoint quotients included.
struct DivC {
    double b, rb;      // divisor and y = RN(1/b) (the reciprocal form multiplies by it)
    double zh, zl;     // 2^128 RD(1/b) and 2^128 RN(1/b - RD(1/b))
    unsigned gate;     // 0 when b is in range, else 1 (every quotient flagged)
    unsigned pad;
};
inline DivC make_divc(double b) {
    DivC d;
    d.b = b;
    d.rb = 1.0 / b;
    double zh = d.rb;
    double rem = std::fma(-zh, b, 1.0);   // exact: zh is within one ulp of 1/b
    if (rem < 0.) {
        zh = std::nextafter(zh, 0.0);
        rem = std::fma(-zh, b, 1.0);
    }
    d.zh = std::ldexp(zh, 128);
    d.zl = std::ldexp(rem / b, 128);
    const bool in_range = std::isnormal(b) && b > 0. && b >= std::ldexp(1.0, -60) && b <= std::ldexp(1.0, 60);
    d.gate = in_range ? 0u : 1u;
    d.pad = 0;
    return d;
}
#ifdef __CUDACC__
// IEEE division kept out of line: it is only the rare fallback, and inlining
// it at every call site would multiply the kernels' instruction footprint.
__device__ __noinline__ double ieee_div(double a, double b);
// The exact quotient; a flagged one (see DivC) sets `bad` (the value returned
// for it is then not the IEEE quotient), so a caller can test once for a
// whole group of divisions and recompute the group with IEEE division.
__device__ __forceinline__ double xdiv_flag(double a, const DivC& d, unsigned& bad) {
    const double as = __dmul_rn(a, 0x1p128);
    const double q0 = __fma_rn(a, d.zh, __dmul_rn(a, d.zl));
    const double e = __fma_rn(q0, d.b, -as);
    const double qs = __fma_rn(-e, d.rb, q0);
    // |qs| in (0, 2^-894): a subnormal quotient; >= 2^1024: infinite or NaN
    const unsigned u = (unsigned)__double2hiint(qs) & 0x7FFFFFFFu;
    bad |= ((u - 1u) < 0x080FFFFFu || u >= 0x7FF00000u || d.gate) ? 1u : 0u;
    return __dmul_rn(qs, 0x1p-128);
}
__device__ __forceinline__ double xdiv(double a, const DivC& d) {
    unsigned bad = 0;
    const double q = xdiv_flag(a, d, bad);
    return bad ? ieee_div(a, d.b) : q;
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
